// Compile-time specialised FFT passes for the common lattice extents
// (products of 2 and 3 up to 64).  Same algorithm, tiles and results as the
// generic passes in fft_pass.cuh (in-place Stockham stages in shared memory,
// radix 8/4/2/3, twiddles staged in shared memory), but every extent, stride
// and pencil mapping is a template constant, so the per-butterfly index
// arithmetic folds to shifts and multiply-adds and every loop unrolls.
// Included by kernels.cuh inside namespace gfix, after fft_pass.cuh; the
// stage template ct_stages is in fft.cuh.

// xy-plane pass with compile-time extents (see k_fft_xy)
template <typename R, int LX, int LY>
__global__ void __launch_bounds__(ct_threads(LX *LY), ct_minb(LX *LY))
    k_fft_xy_ct(Ctx<R> c, int bwd, int prsum) {
  if (c.st->done) return;
  if (c.skip && c.skip[blockIdx.x / c.L[2]]) return;  // finished slice
  constexpr int P = LX + 1, N = LX * LY, BD = ct_threads(N);
  constexpr int EPT = (N + BD - 1) / BD;
  extern __shared__ unsigned char smem_raw[];
  cx<R> *A = reinterpret_cast<cx<R> *>(smem_raw);
  cx<R> *twx = A + P * LY;
  cx<R> *twy = twx + LX;
  stage_twiddles(twx, c.tw + c.ax[0].tw_off, LX);
  stage_twiddles(twy, c.tw + c.ax[1].tw_off, LY);
  const int plane = blockIdx.x, field = blockIdx.y;
  const int par = c.st->parity;
  const size_t base = (size_t)field * c.V + (size_t)plane * N;
  cx<R> *data = c.fb[par] + base;
#pragma unroll
  for (int k = 0; k < EPT; k++) {
    const int e = threadIdx.x + k * BD;
    if (N % BD == 0 || e < N) A[(e / LX) * P + e % LX] = data[e];
  }
  __syncthreads();
  ct_stages<R, LX, 1, LY, 1, 0, P, 1, BD>(A, twx, bwd != 0);   // rows
  ct_stages<R, LY, 1, LX, LX, 1, 0, P, BD>(A, twy, bwd != 0);  // columns
  double v[2] = {0.0, 0.0};
  const cx<R> *old = c.fb[par ^ 1] + base;
#pragma unroll
  for (int k = 0; k < EPT; k++) {
    const int e = threadIdx.x + k * BD;
    if (N % BD != 0 && e >= N) continue;
    const cx<R> w = A[(e / LX) * P + e % LX];
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

// z(,t) pass with compile-time extents (see k_fft_zt).  NT = Lt for Landau
// (z and t transformed); NT = 1 for Coulomb (z only, one slice per tile).
template <typename R, int LZ, int NT, int B>
__global__ void __launch_bounds__(zt_threads<R>(B *LZ *NT), zt_minb<R>(B *LZ *NT))
    k_fft_zt_ct(Ctx<R> c) {
  if (c.st->done) return;
  if constexpr (NT == 1)
    if (c.skip && c.skip[blockIdx.x / ((c.L[0] / B) * c.L[1])]) return;
  constexpr bool FOUR = NT > 1;
  constexpr int TS = FOUR ? LZ * B + zt_pad(B) : LZ * B;  // padded t-stride
  constexpr int N = B * LZ * NT, BD = zt_threads<R>(N);
  constexpr int EPT = (N + BD - 1) / BD;
  extern __shared__ unsigned char smem_raw[];
  cx<R> *A = reinterpret_cast<cx<R> *>(smem_raw);
  cx<R> *twz = A + TS * NT;
  cx<R> *twt = twz + LZ;
  stage_twiddles(twz, c.tw + c.ax[2].tw_off, LZ);
  if constexpr (FOUR) stage_twiddles(twt, c.tw + c.ax[3].tw_off, NT);
  const int Lx = c.L[0], Ly = c.L[1];
  const int nxb = Lx / B;
  int tile = blockIdx.x;
  const int xb = tile % nxb;
  tile /= nxb;
  const int y = tile % Ly;
  const int tslice = FOUR ? 0 : tile / Ly;
  const int field = blockIdx.y;
  cx<R> *data = c.fb[c.st->parity] + (size_t)field * c.V;
  const int x0 = xb * B;
  const size_t sz = (size_t)Lx * Ly;
  const size_t base = (size_t)x0 + (size_t)Lx * y + sz * LZ * tslice;
  const double D = FOUR ? 4.0 : 3.0;
  const double cxy = c.cs[1 * c.cs_ld + y];
  if constexpr (FOUR || ct_nstages(LZ) >= 2) {
    // Fused form: the first forward z stage reads the columns from global
    // memory, the last forward stage of the innermost transform (t, or z
    // for Coulomb), psq and the first backward stage share registers (the
    // backward stages of that transform run in the mirrored radix order),
    // and the last backward z stage writes global memory.  z pencil p:
    // column b = p % B of t-plane p / B; t pencil p: column b = p % B at
    // z = p / B.
    static_assert(ct_mirror_ok(LZ) && ct_mirror_ok(NT), "radix order");
    constexpr int NPZ = NT * B, R1 = ct_radix(LZ), RLZ = ct_radix_last(LZ);
    auto gidx = [&](int p, int z) {
      return base + (p % B) + sz * (z + LZ * (p / B));
    };
    auto sidx = [&](int p, int z) { return (p / B) * TS + (p % B) + z * B; };
    auto psq = [&](int b, int z, int t) -> R {
      double kcos = 0.0;
      kcos += c.cs[x0 + b];
      kcos += cxy;
      kcos += c.cs[2 * c.cs_ld + z];
      if constexpr (FOUR) kcos += c.cs[3 * c.cs_ld + t];
      const double p2 = (kcos == D) ? 1.0 : 2.0 * (D - kcos);
      return (R)(c.maxp * __drcp_rn(p2));
    };
    __syncthreads();  // twiddles staged
    ct_stage_io<R, LZ, 1, R1, NPZ, BD, true>(
        twz, false, [&](int p, int z) { return data[gidx(p, z)]; },
        [&](int p, int z, cx<R> v) { A[sidx(p, z)] = v; });
    if constexpr (FOUR) {
      constexpr int RLT = ct_radix_last(NT);
      ct_stages<R, LZ, R1, NPZ, B, 1, TS, B, BD>(A, twz, false);
      ct_stages<R, NT, 1, LZ * B, LZ * B, 1, 0, TS, BD, false, NT / RLT>(A, twt, false);
      ct_mid<R, NT, LZ * B, LZ * B, 1, 0, TS, BD>(
          A, twt, [&](int p, int t) { return psq(p % B, p / B, t); });
      ct_stages<R, NT, RLT, LZ * B, LZ * B, 1, 0, TS, BD, true>(A, twt, true);
      ct_stages<R, LZ, 1, NPZ, B, 1, TS, B, BD, false, LZ / RLZ>(A, twz, true);
      ct_stage_io<R, LZ, LZ / RLZ, RLZ, NPZ, BD, false>(
          twz, true, [&](int p, int z) { return A[sidx(p, z)]; },
          [&](int p, int z, cx<R> v) { data[gidx(p, z)] = v; });
    } else {
      ct_stages<R, LZ, R1, NPZ, B, 1, TS, B, BD, false, LZ / RLZ>(A, twz, false);
      ct_mid<R, LZ, NPZ, B, 1, TS, B, BD>(
          A, twz, [&](int p, int z) { return psq(p % B, z, 0); });
      ct_stages<R, LZ, RLZ, NPZ, B, 1, TS, B, BD, true, LZ / R1>(A, twz, true);
      ct_stage_io<R, LZ, LZ / R1, R1, NPZ, BD, false>(
          twz, true, [&](int p, int z) { return A[sidx(p, z)]; },
          [&](int p, int z, cx<R> v) { data[gidx(p, z)] = v; });
    }
  } else {  // generic form: z (and t) stages in shared memory
#pragma unroll
    for (int k = 0; k < EPT; k++) {
      const int e = threadIdx.x + k * BD;
      if (N % BD == 0 || e < N) {
        const int q = e / B, b = e % B, t = q / LZ, z = q % LZ;
        A[b + B * z + TS * t] = data[base + b + sz * q];
      }
    }
    __syncthreads();
    ct_stages<R, LZ, 1, NT * B, B, 1, TS, B, BD>(A, twz, false);
    if constexpr (FOUR) ct_stages<R, NT, 1, LZ * B, LZ * B, 1, 0, TS, BD>(A, twt, false);
#pragma unroll
    for (int k = 0; k < EPT; k++) {
      const int e = threadIdx.x + k * BD;
      if (N % BD != 0 && e >= N) continue;
      const int q = e / B, b = e % B, t = q / LZ, z = q % LZ;
      double kcos = 0.0;
      kcos += c.cs[x0 + b];
      kcos += cxy;
      kcos += c.cs[2 * c.cs_ld + z];
      if constexpr (FOUR) kcos += c.cs[3 * c.cs_ld + t];
      const double p2 = (kcos == D) ? 1.0 : 2.0 * (D - kcos);
      const R ps = (R)(c.maxp * __drcp_rn(p2));
      const int o = b + B * z + TS * t;
      A[o] = mk<R>(A[o].x * ps, A[o].y * ps);
    }
    __syncthreads();
    if constexpr (FOUR) ct_stages<R, NT, 1, LZ * B, LZ * B, 1, 0, TS, BD>(A, twt, true);
    ct_stages<R, LZ, 1, NT * B, B, 1, TS, B, BD>(A, twz, true);
#pragma unroll
    for (int k = 0; k < EPT; k++) {
      const int e = threadIdx.x + k * BD;
      if (N % BD == 0 || e < N) {
        const int q = e / B, b = e % B, t = q / LZ, z = q % LZ;
        data[base + b + sz * q] = A[b + B * z + TS * t];
      }
    }
  }
}
