// Shared-memory mixed-radix FFT over pencils, used by the fused
// Fourier-acceleration passes (the GPU form of GLU's FOURIER_ACCELERATE3/2,
// src/Gfix/FACG.c:77-95 and src/Gfix/CFACG.c:69-88, where FFTW transforms
// each packed field, multiplies by psq and transforms back).
//
// Algorithm: Stockham auto-sort, one radix-R butterfly per thread and stage,
// ping-pong between two shared-memory tiles.  Radices 8, 4, 2, 3, 5 have
// register kernels; any other prime factor uses a direct DFT.  Twiddles come
// from a table tw[k] = exp(-2 pi i k / N) computed on the host in FP64;
// the backward (+i) direction conjugates them.  Like FFTW, neither direction
// normalises.
#pragma once

#include "su3.cuh"

namespace gfix {

constexpr int kMaxStages = 12;
constexpr int kMaxRadix = 16;

struct FftAxis {
  int n;
  int nstages;
  int radix[kMaxStages];
  int tw_off;  // offset of this length's table inside the twiddle pool
};

// pencil p, element j -> tile offset (p / pin) * ps_hi + (p % pin) * ps_lo
// + j * js
struct PencilMap {
  int npencil, pin, ps_lo, ps_hi, js;
};

__device__ __forceinline__ int pencil_off(const PencilMap &m, int p) {
  return (p / m.pin) * m.ps_hi + (p % m.pin) * m.ps_lo;
}

template <typename R>
__device__ __forceinline__ cx<R> twiddle(const cx<R> *tw, int k, bool bwd) {
  cx<R> w = tw[k];
  if (bwd) w.y = -w.y;
  return w;
}

// in-register DFT of size r: v[q] <- sum_s v[s] W_r^{sq}, W_r = tw[N/r]
template <typename R>
__device__ __forceinline__ void dft_reg(cx<R> *v, int r, const cx<R> *tw,
                                        int N, bool bwd) {
  if (r == 2) {
    cx<R> a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (r == 4) {
    const cx<R> w = twiddle(tw, N / 4, bwd);
    cx<R> a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    cx<R> b0 = cadd(v[1], v[3]), b1 = cmul(csub(v[1], v[3]), w);
    v[0] = cadd(a0, b0);
    v[1] = cadd(a1, b1);
    v[2] = csub(a0, b0);
    v[3] = csub(a1, b1);
  } else if (r == 8) {
    const cx<R> w4 = twiddle(tw, N / 4, bwd);
    cx<R> e[4], o[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      e[k] = v[2 * k];
      o[k] = v[2 * k + 1];
    }
    {
      cx<R> a0 = cadd(e[0], e[2]), a1 = csub(e[0], e[2]);
      cx<R> b0 = cadd(e[1], e[3]), b1 = cmul(csub(e[1], e[3]), w4);
      e[0] = cadd(a0, b0); e[1] = cadd(a1, b1);
      e[2] = csub(a0, b0); e[3] = csub(a1, b1);
    }
    {
      cx<R> a0 = cadd(o[0], o[2]), a1 = csub(o[0], o[2]);
      cx<R> b0 = cadd(o[1], o[3]), b1 = cmul(csub(o[1], o[3]), w4);
      o[0] = cadd(a0, b0); o[1] = cadd(a1, b1);
      o[2] = csub(a0, b0); o[3] = csub(a1, b1);
    }
    const int s8 = N / 8;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const cx<R> t = cmul(o[q], twiddle(tw, q * s8, bwd));
      v[q] = cadd(e[q], t);
      v[q + 4] = csub(e[q], t);
    }
  } else {
    // direct DFT for 3, 5 and any other prime
    cx<R> out[kMaxRadix];
    const int sr = N / r;
    for (int q = 0; q < r; q++) {
      cx<R> acc = v[0];
      for (int s = 1; s < r; s++)
        acc = cadd(acc, cmul(v[s], twiddle(tw, ((s * q) % r) * sr, bwd)));
      out[q] = acc;
    }
    for (int q = 0; q < r; q++) v[q] = out[q];
  }
}

// One Stockham stage of compile-time radix RDX (0 = runtime radix r with
// the generic direct DFT) over every pencil of the tile.
template <typename R, int RDX>
__device__ __forceinline__ void stockham_stage(const cx<R> *src, cx<R> *dst,
                                               const PencilMap &m, int N,
                                               int r_rt, int Ns,
                                               const cx<R> *tw, bool bwd) {
  constexpr int RMAX = RDX ? RDX : kMaxRadix;
  const int r = RDX ? RDX : r_rt;
  const int nb = N / r;
  const int total = m.npencil * nb;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int p = idx / nb, j = idx - p * nb;
    const int po = pencil_off(m, p);
    const int jm = j % Ns;
    const int step = jm * (N / (Ns * r));
    cx<R> v[RMAX];
#pragma unroll
    for (int s = 0; s < RMAX; s++) {
      if (RDX == 0 && s >= r) break;
      v[s] = src[po + (j + s * nb) * m.js];
      if (s > 0 && step) v[s] = cmul(v[s], twiddle(tw, s * step, bwd));
    }
    dft_reg(v, r, tw, N, bwd);
    const int base = (j / Ns) * Ns * r + jm;
#pragma unroll
    for (int s = 0; s < RMAX; s++) {
      if (RDX == 0 && s >= r) break;
      dst[po + (base + s * Ns) * m.js] = v[s];
    }
  }
}

// Full transform of every pencil of a tile; returns the buffer that holds
// the result (a or b).  All threads of the block must call it.
template <typename R>
__device__ cx<R> *smem_fft(cx<R> *a, cx<R> *b, const PencilMap &m,
                           const FftAxis &ax, const cx<R> *tw, bool bwd) {
  const int N = ax.n;
  int Ns = 1;
  cx<R> *src = a, *dst = b;
  for (int st = 0; st < ax.nstages; st++) {
    const int r = ax.radix[st];
    switch (r) {
      case 8: stockham_stage<R, 8>(src, dst, m, N, r, Ns, tw, bwd); break;
      case 4: stockham_stage<R, 4>(src, dst, m, N, r, Ns, tw, bwd); break;
      case 2: stockham_stage<R, 2>(src, dst, m, N, r, Ns, tw, bwd); break;
      case 3: stockham_stage<R, 3>(src, dst, m, N, r, Ns, tw, bwd); break;
      default: stockham_stage<R, 0>(src, dst, m, N, r, Ns, tw, bwd); break;
    }
    __syncthreads();
    cx<R> *t = src;
    src = dst;
    dst = t;
    Ns *= r;
  }
  return src;
}

}  // namespace gfix
