// The two FFT passes of the Fourier acceleration (the GPU form of GLU's
// FOURIER_ACCELERATE3, src/Gfix/FACG.c:77-95, and FOURIER_ACCELERATE2,
// src/Gfix/CFACG.c:69-88).  Included by kernels.cuh inside namespace gfix.
//
//   k_fft_xy  one xy-plane of one field per block: x then y transform,
//             forward, or inverse fused with GLU's PR sums
//   k_fft_zt  a tile of zt_b x-columns at fixed y (Landau: all z and t;
//             Coulomb: all z of one slice): forward z (t), * psq, inverse
//
// Tiles live in shared memory with padded strides (xy row pitch Lx+1, zt
// t-stride Lz*zt_b+1) so that the column/t pencils spread over the banks.
// Twiddle tables are staged in shared memory next to the tile.

template <typename R>
__device__ __forceinline__ void stage_twiddles(cx<R> *dst, const cx<R> *src,
                                               int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
}

template <typename R, int PT, bool ODD>
__global__ void __launch_bounds__(512, 2) k_fft_xy(Ctx<R> c, int bwd, int prsum) {
  if (c.st->done) return;
  if (c.skip && c.skip[blockIdx.x / c.L[2]]) return;  // finished slice
  extern __shared__ unsigned char smem_raw[];
  __shared__ FftAxis s_ax[2];
  const int Lx = c.L[0], Ly = c.L[1], P = c.xy_pitch;
  cx<R> *A = reinterpret_cast<cx<R> *>(smem_raw);
  cx<R> *twx = A + P * Ly;
  cx<R> *twy = twx + Lx;
  if (threadIdx.x == 0) {
    s_ax[0] = c.ax[0];
    s_ax[1] = c.ax[1];
  }
  stage_twiddles(twx, c.tw + c.ax[0].tw_off, Lx);
  stage_twiddles(twy, c.tw + c.ax[1].tw_off, Ly);
  const int plane = blockIdx.x, field = blockIdx.y;
  const int par = c.st->parity;
  const size_t base = (size_t)field * c.V + (size_t)plane * Lx * Ly;
  cx<R> *data = c.fb[par] + base;
  const int n = Lx * Ly;
  const int lx_sh = log2_if_pow2(Lx);
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < n) {
      const int y = fdiv(e, Lx, lx_sh);
      A[y * P + (e - y * Lx)] = data[e];
    }
  }
  __syncthreads();
  const PencilMap mx = pmap(Ly, 1, 0, P, 1);   // rows
  const PencilMap my = pmap(Lx, Lx, 1, 0, P);  // columns
  smem_fft<R, PT, ODD>(A, mx, s_ax[0], twx, bwd != 0);
  smem_fft<R, PT, ODD>(A, my, s_ax[1], twy, bwd != 0);
  double v[2] = {0.0, 0.0};
  const cx<R> *old = c.fb[par ^ 1] + base;
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e >= n) continue;
    const int y = fdiv(e, Lx, lx_sh);
    const cx<R> w = A[y * P + (e - y * Lx)];
    data[e] = w;
    if (prsum) {
      const cx<R> od = old[e];
      const double a = w.x, b = w.y;
      const double tr = a - (double)od.x, ti = b - (double)od.y;
      if (field == 0) {
        v[0] += 2.0 * (a * a + b * b + a * b);
        v[1] += 2.0 * (a * tr + b * ti) + (a * ti + b * tr);
      } else {
        v[0] += 2.0 * (a * a + b * b);
        v[1] += 2.0 * (a * tr + b * ti);
      }
    }
  }
  if (prsum) {
    block_sum_store<2>(v, c.part + 2 * (blockIdx.y * gridDim.x + blockIdx.x));
    if (threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0)
      c.st->nblocks = gridDim.x * gridDim.y;
  }
}

template <typename R, int PT, bool ODD>
__global__ void __launch_bounds__(512, 2) k_fft_zt(Ctx<R> c) {
  if (c.st->done) return;
  if (c.skip && c.skip[blockIdx.x / ((c.L[0] / c.zt_b) * c.L[1])]) return;
  extern __shared__ unsigned char smem_raw[];
  __shared__ FftAxis s_ax[2];
  const int Lx = c.L[0], Ly = c.L[1], Lz = c.L[2], Lt = c.L[3];
  const int Bw = c.zt_b;
  const bool four = (c.ndim == 4);
  const int nt = four ? Lt : 1;
  const int TS = four ? Lz * Bw + 1 : Lz * Bw;  // padded t-stride
  cx<R> *A = reinterpret_cast<cx<R> *>(smem_raw);
  cx<R> *twz = A + TS * nt;
  cx<R> *twt = twz + Lz;
  if (threadIdx.x == 0) {
    s_ax[0] = c.ax[2];
    s_ax[1] = c.ax[3];
  }
  stage_twiddles(twz, c.tw + c.ax[2].tw_off, Lz);
  if (four) stage_twiddles(twt, c.tw + c.ax[3].tw_off, Lt);
  const int nxb = Lx / Bw;
  int tile = blockIdx.x;
  const int xb = tile % nxb;
  tile /= nxb;
  const int y = tile % Ly;
  const int tslice = four ? 0 : tile / Ly;
  const int field = blockIdx.y;
  cx<R> *data = c.fb[c.st->parity] + (size_t)field * c.V;
  const int x0 = xb * Bw;
  const int n = Bw * Lz * nt;
  const size_t sz = (size_t)Lx * Ly;  // site stride of z
  const size_t base = (size_t)x0 + (size_t)Lx * y + sz * Lz * tslice;
  const int b_sh = log2_if_pow2(Bw), z_sh = log2_if_pow2(Lz);
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < n) {
      const int q = fdiv(e, Bw, b_sh), b = e - q * Bw;
      const int t = fdiv(q, Lz, z_sh), z = q - t * Lz;
      A[b + Bw * z + TS * t] = data[base + b + sz * q];
    }
  }
  __syncthreads();
  const PencilMap mz = pmap(nt * Bw, Bw, 1, TS, Bw);
  const PencilMap mt = pmap(Lz * Bw, Lz * Bw, 1, 0, TS);
  smem_fft<R, PT, ODD>(A, mz, s_ax[0], twz, false);
  if (four) smem_fft<R, PT, ODD>(A, mt, s_ax[1], twt, false);
  const double D = four ? 4.0 : 3.0;
  const double cxy = c.cs[1 * c.cs_ld + y];
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e >= n) continue;
    const int q = fdiv(e, Bw, b_sh), b = e - q * Bw;
    const int t = fdiv(q, Lz, z_sh), z = q - t * Lz;
    double kcos = 0.0;
    kcos += c.cs[x0 + b];
    kcos += cxy;
    kcos += c.cs[2 * c.cs_ld + z];
    if (four) kcos += c.cs[3 * c.cs_ld + t];
    const double p2 = (kcos == D) ? 1.0 : 2.0 * (D - kcos);
    const R ps = (R)(c.maxp * __drcp_rn(p2));
    const int o = b + Bw * z + TS * t;
    A[o] = mk<R>(A[o].x * ps, A[o].y * ps);
  }
  __syncthreads();
  if (four) smem_fft<R, PT, ODD>(A, mt, s_ax[1], twt, true);
  smem_fft<R, PT, ODD>(A, mz, s_ax[0], twz, true);
#pragma unroll
  for (int k = 0; k < PT; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < n) {
      const int q = fdiv(e, Bw, b_sh), b = e - q * Bw;
      const int t = fdiv(q, Lz, z_sh), z = q - t * Lz;
      data[base + b + sz * q] = A[b + Bw * z + TS * t];
    }
  }
}
