// Shared-memory mixed-radix FFT over pencils, used by the fused
// Fourier-acceleration passes (the GPU form of GLU's FOURIER_ACCELERATE3/2,
// src/Gfix/FACG.c:77-95 and src/Gfix/CFACG.c:69-88, where FFTW transforms
// each packed field, multiplies by psq and transforms back).
//
// Algorithm: Stockham auto-sort in place: per stage each thread loads its
// radix-R butterflies into registers, the block synchronises, and the
// outputs overwrite the tile.  Radices 8, 4 and 2 have dedicated register
// kernels; 3, 5 and 7 use a direct DFT.  Twiddles come
// from a table tw[k] = exp(-2 pi i k / N) computed on the host in FP64;
// the backward (+i) direction conjugates them.  Like FFTW, neither direction
// normalises.
#pragma once

#include "su3.cuh"

namespace gfix {

constexpr int kMaxStages = 12;
constexpr int kMaxRadix = 7;   // largest prime factor of an extent

// one Stockham stage: radix r, nb = N / r butterflies per pencil, Ns the
// product of the earlier radices, step0 = N / (Ns r); *_sh = log2 of nb or
// Ns when it is a power of two (else -1), so that the index arithmetic of
// the common power-of-two sizes needs no integer division
struct FftStage {
  int r, nb, Ns, step0, nb_sh, ns_sh;
};

struct FftAxis {
  int n;
  int nstages;
  int tw_off;  // offset of this length's table inside the twiddle pool
  FftStage st[kMaxStages];
};

// pencil p, element j -> tile offset (p / pin) * ps_hi + (p % pin) * ps_lo
// + j * js
struct PencilMap {
  int npencil, pin, pin_sh, ps_lo, ps_hi, js;
};

__host__ __device__ __forceinline__ int log2_if_pow2(int v) {
  if (v <= 0 || (v & (v - 1))) return -1;
  int k = 0;
  while ((1 << k) < v) k++;
  return k;
}

__device__ __forceinline__ int fdiv(int x, int d, int sh) {
  return sh >= 0 ? (x >> sh) : x / d;
}

__device__ __forceinline__ PencilMap pmap(int npencil, int pin, int ps_lo,
                                          int ps_hi, int js) {
  PencilMap m;
  m.npencil = npencil;
  m.pin = pin;
  m.pin_sh = log2_if_pow2(pin);
  m.ps_lo = ps_lo;
  m.ps_hi = ps_hi;
  m.js = js;
  return m;
}

__device__ __forceinline__ int pencil_off(const PencilMap &m, int p) {
  const int q = fdiv(p, m.pin, m.pin_sh);
  return q * m.ps_hi + (p - q * m.pin) * m.ps_lo;
}

template <typename R>
__device__ __forceinline__ cx<R> twiddle(const cx<R> *tw, int k, bool bwd) {
  cx<R> w = tw[k];
  if (bwd) w.y = -w.y;
  return w;
}

// in-register DFT of size RDX: v[q] <- sum_s v[s] W^{sq}, W = tw[N/RDX]
template <typename R, int RDX>
__device__ __forceinline__ void dft_reg(cx<R> *v, const cx<R> *tw, int N,
                                        bool bwd) {
  if constexpr (RDX == 2) {
    cx<R> a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (RDX == 4) {
    const cx<R> w = twiddle(tw, N / 4, bwd);
    cx<R> a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    cx<R> b0 = cadd(v[1], v[3]), b1 = cmul(csub(v[1], v[3]), w);
    v[0] = cadd(a0, b0);
    v[1] = cadd(a1, b1);
    v[2] = csub(a0, b0);
    v[3] = csub(a1, b1);
  } else if constexpr (RDX == 8) {
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
    // direct DFT for 3, 5, 7
    cx<R> out[RDX];
    const int sr = N / RDX;
#pragma unroll
    for (int q = 0; q < RDX; q++) {
      cx<R> acc = v[0];
#pragma unroll
      for (int s = 1; s < RDX; s++)
        acc = cadd(acc, cmul(v[s], twiddle(tw, ((s * q) % RDX) * sr, bwd)));
      out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < RDX; q++) v[q] = out[q];
  }
}

// radices 8, 4, 2, 3, 5, 7 and the Stockham stage table of length n
// radix orders of the generic passes' stage tables (the autotuner tries
// them; 0, largest radices first, is the default)
constexpr int kRadixOrders = 3;
constexpr int kRadixPref[kRadixOrders][6] = {
    {8, 4, 2, 3, 5, 7}, {4, 8, 2, 3, 5, 7}, {2, 4, 8, 3, 5, 7}};

static inline int factorize(int n, FftAxis &ax, int order = 0) {
  ax.n = n;
  ax.nstages = 0;
  int m = n;
  int rad[kMaxStages];
  int ns = 0;
  const int *pref = kRadixPref[order];
  for (int i = 0; i < 6; i++)
    for (const int r = pref[i]; m % r == 0 && m > 1;) {
      if (ns == kMaxStages) return -1;
      rad[ns++] = r;
      m /= r;
    }
  if (m > 1) return -1;  // a prime factor above kMaxRadix
  if (ns == 0) rad[ns++] = 1;
  int Ns = 1;
  for (int k = 0; k < ns; k++) {
    FftStage &S = ax.st[k];
    S.r = rad[k];
    S.nb = n / rad[k];
    S.Ns = Ns;
    S.step0 = n / (Ns * rad[k]);
    S.nb_sh = log2_if_pow2(S.nb);
    S.ns_sh = log2_if_pow2(Ns);
    Ns *= rad[k];
  }
  ax.nstages = ns;
  return 0;
}

// Elements one thread holds per stage (PT): a tile of n elements is handled
// by at least n / PT threads.  8 in FP64 and 16 in FP32 keep the butterflies
// in registers; 16 in FP64 serves tiles too large for 512 threads.

// One in-place Stockham stage of radix RDX over every pencil of the tile:
// each thread reads its butterflies into registers, the block synchronises,
// and the results overwrite the same tile.
template <typename R, int PT, int RDX>
__device__ __forceinline__ void stockham_stage(cx<R> *buf, const PencilMap &m,
                                               const FftStage S, int N,
                                               const cx<R> *tw, bool bwd) {
  constexpr int K = (PT + RDX - 1) / RDX;
  const int nb = S.nb, Ns = S.Ns;
  const int total = m.npencil * nb;
  cx<R> v[K][RDX];
  int dst[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int idx = threadIdx.x + k * blockDim.x;
    dst[k] = -1;
    if (idx < total) {
      const int p = fdiv(idx, nb, S.nb_sh), j = idx - p * nb;
      const int po = pencil_off(m, p);
      const int jq = fdiv(j, Ns, S.ns_sh), jm = j - jq * Ns;
      const int step = jm * S.step0;
#pragma unroll
      for (int s = 0; s < RDX; s++) {
        v[k][s] = buf[po + (j + s * nb) * m.js];
        if (s > 0 && step) v[k][s] = cmul(v[k][s], twiddle(tw, s * step, bwd));
      }
      dft_reg<R, RDX>(v[k], tw, N, bwd);
      dst[k] = po + (jq * Ns * RDX + jm) * m.js;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) {
    if (dst[k] >= 0) {
#pragma unroll
      for (int s = 0; s < RDX; s++) buf[dst[k] + s * Ns * m.js] = v[k][s];
    }
  }
  __syncthreads();
}

// Full in-place transform of every pencil of a tile.  Radices 2, 3, 4, 5,
// 7, 8 (the host rejects extents with other prime factors).  All threads of
// the block must call it, with blockDim.x * PT >= tile elements.
// ODD adds the radix-5 and radix-7 stages (direct DFTs, more registers).
// `ax` should live in shared memory: its stage table is indexed at run time.
template <typename R, int PT, bool ODD>
__device__ void smem_fft(cx<R> *buf, const PencilMap &m, const FftAxis &ax,
                         const cx<R> *tw, bool bwd) {
  const int N = ax.n;
  for (int st = 0; st < ax.nstages; st++) {
    const FftStage S = ax.st[st];
    switch (S.r) {
      case 8: stockham_stage<R, PT, 8>(buf, m, S, N, tw, bwd); break;
      case 4: stockham_stage<R, PT, 4>(buf, m, S, N, tw, bwd); break;
      case 2: stockham_stage<R, PT, 2>(buf, m, S, N, tw, bwd); break;
      case 3: stockham_stage<R, PT, 3>(buf, m, S, N, tw, bwd); break;
      default:
        if constexpr (ODD) {
          if (S.r == 5) stockham_stage<R, PT, 5>(buf, m, S, N, tw, bwd);
          if (S.r == 7) stockham_stage<R, PT, 7>(buf, m, S, N, tw, bwd);
        }
        break;
    }
  }
}

// ---------------------------------------------------------------------
// compile-time Stockham stages (every extent, stride and pencil mapping a
// template constant), used by the compile-time passes

// radix of the next stage for a remaining length m
__host__ __device__ constexpr int ct_radix(int m) {
  return (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : 3;
}
// radix of the last stage of a length m (the first of the mirrored order)
__host__ __device__ constexpr int ct_radix_last(int m) {
  int r = ct_radix(m);
  while (m / r > 1) {
    m /= r;
    r = ct_radix(m);
  }
  return r;
}
// number of stages of a length n
__host__ __device__ constexpr int ct_nstages(int n) {
  int k = 0;
  while (n > 1) {
    n /= ct_radix(n);
    k++;
  }
  return k;
}
// the mirrored order (radix ct_radix_last of the remaining length at each
// stage) is the forward radix sequence reversed
__host__ __device__ constexpr bool ct_mirror_ok(int n) {
  int fwd[kMaxStages] = {}, k = 0;
  for (int m = n; m > 1 && k < kMaxStages; m /= fwd[k++]) fwd[k] = ct_radix(m);
  int ns = 1;
  for (int i = k - 1; i >= 0; i--) {
    if (ct_radix_last(n / ns) != fwd[i]) return false;
    ns *= fwd[i];
  }
  return ns == n;
}
// can the extent be transformed by the compile-time stages?
__host__ __device__ constexpr bool ct_ok(int n) {
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

// Stockham stages for pencils of length N; pencil p starts at
// (p / PIN) * PSHI + (p % PIN) * PSLO, elements are JS apart; BD threads.
// Consecutive threads take consecutive pencils at the same butterfly index:
// their elements are neighbours in shared memory (no bank conflicts for the
// tile layouts below) and they share one twiddle factor (a broadcast).
// The stages run from Ns up to (not including) END; MIR selects the
// mirrored radix order (any order of the radices is a valid Stockham
// sequence: the twiddle of a stage depends only on Ns and its radix).
template <typename R, int N, int Ns, int NP, int PIN, int PSLO, int PSHI,
          int JS, int BD, bool MIR = false, int END = N>
__device__ __forceinline__ void ct_stages(cx<R> *buf, const cx<R> *tw,
                                          bool bwd) {
  if constexpr (Ns < END) {
    constexpr int RDX = MIR ? ct_radix_last(N / Ns) : ct_radix(N / Ns);
    constexpr int NB = N / RDX;
    constexpr int TOTAL = NP * NB;
    constexpr int K = (TOTAL + BD - 1) / BD;
    constexpr int STEP0 = N / (Ns * RDX);
    cx<R> v[K][RDX];
    int dst[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int idx = threadIdx.x + k * BD;
      dst[k] = -1;
      if (TOTAL % BD == 0 || idx < TOTAL) {
        const int p = idx % NP, j = idx / NP;
        const int po = (p / PIN) * PSHI + (p % PIN) * PSLO;
        const int jq = j / Ns, jm = j % Ns;
#pragma unroll
        for (int s = 0; s < RDX; s++) {
          v[k][s] = buf[po + (j + s * NB) * JS];
          if constexpr (Ns > 1)
            if (s > 0) v[k][s] = cmul(v[k][s], twiddle(tw, s * jm * STEP0, bwd));
        }
        dft_reg<R, RDX>(v[k], tw, N, bwd);
        dst[k] = po + (jq * Ns * RDX + jm) * JS;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (dst[k] >= 0) {
#pragma unroll
        for (int s = 0; s < RDX; s++) buf[dst[k] + s * Ns * JS] = v[k][s];
      }
    }
    __syncthreads();
    ct_stages<R, N, Ns * RDX, NP, PIN, PSLO, PSHI, JS, BD, MIR, END>(buf, tw,
                                                                    bwd);
  }
}

// One Stockham stage (length N, product of the earlier radices Ns, radix
// RDX) over NP pencils whose element i is read by ld(p, i) and written by
// st(p, i, value): the first stage of a pass reading its pencils from
// global memory, or the last one writing them there.  No barrier between
// the loads and the stores (source and destination differ); AFTER puts one
// after the stores.
template <typename R, int N, int Ns, int RDX, int NP, int BD, bool AFTER,
          class Ld, class St>
__device__ __forceinline__ void ct_stage_io(const cx<R> *tw, bool bwd, Ld ld,
                                            St st) {
  constexpr int NB = N / RDX;
  constexpr int TOTAL = NP * NB;
  constexpr int K = (TOTAL + BD - 1) / BD;
  constexpr int STEP0 = N / (Ns * RDX);
  cx<R> v[K][RDX];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int idx = threadIdx.x + k * BD;
    if (TOTAL % BD == 0 || idx < TOTAL) {
      const int p = idx % NP, j = idx / NP;
      const int jq = j / Ns, jm = j % Ns;
#pragma unroll
      for (int s = 0; s < RDX; s++) v[k][s] = ld(p, j + s * NB);
#pragma unroll
      for (int s = 1; s < RDX; s++)
        if constexpr (Ns > 1) v[k][s] = cmul(v[k][s], twiddle(tw, s * jm * STEP0, bwd));
      dft_reg<R, RDX>(v[k], tw, N, bwd);
#pragma unroll
      for (int s = 0; s < RDX; s++) st(p, jq * Ns * RDX + jm + s * Ns, v[k][s]);
    }
  }
  if constexpr (AFTER) __syncthreads();
}

// The last forward stage of a length N, a scale sc(p, i) of every output
// element and the first backward stage of the mirrored radix order, in
// registers: the forward stage leaves element j + s * N / RL of each pencil
// with the thread that the mirrored backward stage (radix RL, Ns = 1) reads
// it from, so the pair costs one shared-memory round trip instead of three
// (two stages and the scaling pass).
// a product rounded on its own (never contracted into a following add), so
// that a scale applied in registers rounds as one applied in a separate pass
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <typename R, int N, int NP, int PIN, int PSLO, int PSHI, int JS,
          int BD, class Sc>
__device__ __forceinline__ void ct_mid(cx<R> *buf, const cx<R> *tw, Sc sc) {
  constexpr int RL = ct_radix_last(N);
  constexpr int NB = N / RL;  // the forward stage's Ns
  constexpr int TOTAL = NP * NB;
  constexpr int K = (TOTAL + BD - 1) / BD;
  cx<R> v[K][RL];
  int dst[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int idx = threadIdx.x + k * BD;
    dst[k] = -1;
    if (TOTAL % BD == 0 || idx < TOTAL) {
      const int p = idx % NP, j = idx / NP;
      const int po = (p / PIN) * PSHI + (p % PIN) * PSLO;
#pragma unroll
      for (int s = 0; s < RL; s++) v[k][s] = buf[po + (j + s * NB) * JS];
#pragma unroll
      for (int s = 1; s < RL; s++)
        if constexpr (NB > 1) v[k][s] = cmul(v[k][s], twiddle(tw, s * j, false));
      dft_reg<R, RL>(v[k], tw, N, false);
#pragma unroll
      for (int s = 0; s < RL; s++) {
        const R f = sc(p, j + s * NB);
        v[k][s] = mk<R>(mul_rn(v[k][s].x, f), mul_rn(v[k][s].y, f));
      }
      dft_reg<R, RL>(v[k], tw, N, true);
      dst[k] = po + j * RL * JS;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) {
    if (dst[k] >= 0) {
#pragma unroll
      for (int s = 0; s < RL; s++) buf[dst[k] + s * JS] = v[k][s];
    }
  }
  __syncthreads();
}

// threads of a tile of n elements: one radix-8 butterfly each (32..1024
// threads), two for tiles above 8192 elements
__host__ __device__ constexpr int ct_threads(int n) {
  return n / 8 < 32 ? 32 : (n / 8 <= 1024 ? n / 8 : n / 16);
}
// resident blocks asked of the compiler: 1024 threads per SM at least
__host__ __device__ constexpr int ct_minb(int n) {
  return 1024 / ct_threads(n) < 1 ? 1 : 1024 / ct_threads(n);
}
// z(,t) tiles of n elements of type R that take two blocks per SM: FP32
// tiles of 8192 elements and more whose shared memory fits twice (the
// 4x32x64 and 2x48x96 tiles, 66 and 74 KB) run n/16 threads, 16 elements
// each, so that each block's stages run while the other waits at a barrier:
// 0.094 against 0.105 ms per 32^3x64 pass with one 1024-thread block, 0.768
// against 0.864 ms per 48^3x96 pass with one 576-thread block.  FP64 tiles
// of those sizes fill an SM's shared memory alone.
template <typename R>
__host__ __device__ constexpr bool zt_two_blocks(int n) {
  return sizeof(R) == 4 && n >= 8192 && 2 * n * 8 <= 200 * 1024;
}
template <typename R>
__host__ __device__ constexpr int zt_threads(int n) {
  return zt_two_blocks<R>(n) ? n / 16 : ct_threads(n);
}
template <typename R>
__host__ __device__ constexpr int zt_minb(int n) {
  return zt_two_blocks<R>(n) ? 2
                             : (1024 / zt_threads<R>(n) < 1 ? 1 : 1024 / zt_threads<R>(n));
}
// padding of the t-stride of a zt tile of B x columns: t-planes start B
// elements apart modulo 8, so the z-stage pencils of 8 (FP64) or 16 (FP32)
// consecutive threads fall in distinct banks
__host__ __device__ constexpr int zt_pad(int b) { return b < 16 ? b : 0; }

}  // namespace gfix
