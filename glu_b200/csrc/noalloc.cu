// gfix_theta_functional_noalloc: GLU's theta_test_lin and gauge functional
// of device-resident links, computed without allocating any memory.
//
// Some callers cannot allocate device memory at the moment they call in:
// lattice codes that hand all of HBM to their own arena allocator at start-up
// (a cudaMalloc then fails, or takes memory the arena counts on), and
// stream-ordered pipelines that must not call cudaMalloc/cudaFree because
// those calls synchronise the whole device.  For them this entry point keeps
// its only scratch -- one pair of partial sums per thread block -- in a fixed
// file-scope device array of kScratchBlocks x 2 doubles (1 MiB).  Every GPU
// that loads this library holds that array until the process exits; lattices
// needing more blocks than the array has (more than 16,777,216 sites) are
// rejected with an error.
//
// The array is shared by every call: calls that overlap on the GPU race on
// it.  The first call on a device looks up the array's device address with
// cudaGetSymbolAddress; make that first call before any stream capture.
// Both kernels run on the stream the caller passes, in its order, and the
// call returns without waiting for them.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/glu_gfix.h"

namespace {

constexpr int kNaThreads = 256;
constexpr int kScratchBlocks = 65536;  // 65536 blocks x 256 sites
constexpr int kMaxDevices = 64;
constexpr double kLocalTr49 = 0.4444444444444444;  // lin_derivs.c:72

// per-block partial sums {sum of local tr(dA dA), sum of Re tr U}
static __device__ __align__(256) double g_scratch[kScratchBlocks * 2];

// device address of g_scratch on each device (host code cannot use the
// symbol's own name as a device pointer)
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_mu;
thread_local char g_msg[256] = "";

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// fixed-order block sum of two values; thread 0 stores them at out[0..1]
__device__ __forceinline__ void na_block_sum2(double a, double b,
                                              double *out) {
  __shared__ double sh[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  a = na_warp_sum(a);
  b = na_warp_sum(b);
  if (lane == 0) {
    sh[0][warp] = a;
    sh[1][warp] = b;
  }
  __syncthreads();
  if (warp == 0) {
    a = na_warp_sum(lane < nw ? sh[0][lane] : 0.0);
    b = na_warp_sum(lane < nw ? sh[1][lane] : 0.0);
    if (lane == 0) {
      out[0] = a;
      out[1] = b;
    }
  }
}

// one site: the local tr(dA dA) of GLU's fast derivative
// (src/Gfix/lin_derivs.c:74-193) and sum_mu Re tr U_mu(x), from links in the
// flat layout double[V][4][9][2]
__global__ void __launch_bounds__(kNaThreads)
    k_na_partials(const double2 *__restrict__ U, int L0, int L1, int L2,
                  int L3, double *scratch) {
  const int V = L0 * L1 * L2 * L3;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  double tr = 0.0, re = 0.0;
  if (s < V) {
    const int L[4] = {L0, L1, L2, L3};
    const int st[4] = {1, L0, L0 * L1, L0 * L1 * L2};
    int x[4], r = s;
    for (int mu = 0; mu < 4; mu++) {
      x[mu] = r % L[mu];
      r /= L[mu];
    }
    double R0 = 0, R1 = 0, I1 = 0, R2 = 0, I2 = 0, R3 = 0, R4 = 0, I4 = 0;
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      const int sb = x[mu] == 0 ? s + (L[mu] - 1) * st[mu] : s - st[mu];
      const double2 *q = U + ((size_t)s * 4 + mu) * 9;
      const double2 *b = U + ((size_t)sb * 4 + mu) * 9;
      R0 += 2.0 * b[0].y - b[4].y - b[8].y;
      R0 += -2.0 * q[0].y + q[4].y + q[8].y;
      R1 += b[1].x - b[3].x - q[1].x + q[3].x;
      I1 += b[1].y + b[3].y - q[1].y - q[3].y;
      R2 += b[2].x - b[6].x - q[2].x + q[6].x;
      I2 += b[2].y + b[6].y - q[2].y - q[6].y;
      R3 += 2.0 * b[4].y - b[0].y - b[8].y;
      R3 += -2.0 * q[4].y + q[0].y + q[8].y;
      R4 += b[5].x - b[7].x - q[5].x + q[7].x;
      I4 += b[5].y + b[7].y - q[5].y - q[7].y;
      re += q[0].x + q[4].x + q[8].x;
    }
    tr = kLocalTr49 * (R0 * R0 + R3 * (R3 + R0)) +
         (R1 * R1 + I1 * I1 + R2 * R2 + I2 * I2 + R4 * R4 + I4 * I4);
  }
  na_block_sum2(tr, re, scratch + 2 * blockIdx.x);
}

// one block: fixed-order sum of the partials; out[0] = theta_test_lin
// = 2 sum / (NC V) (src/Gfix/gftests.c:249), out[1] = the functional
// 1 - sum Re tr U / (ND NC V) (src/Gfix/gftests.c:146)
__global__ void __launch_bounds__(1024)
    k_na_finish(const double *scratch, int nblocks, double V, double *out) {
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
    a += scratch[2 * i];
    b += scratch[2 * i + 1];
  }
  __shared__ double tot[2];
  na_block_sum2(a, b, tot);
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = 2.0 * tot[0] / (3.0 * V);
    out[1] = 1.0 - tot[1] / (12.0 * V);
  }
}

int na_fail(const char *m) {
  snprintf(g_msg, sizeof g_msg, "%s", m);
  return -1;
}

}  // namespace

extern "C" {

const char *gfix_noalloc_error(void) { return g_msg; }

int gfix_theta_functional_noalloc(const double *d_links, const size_t dims[4],
                                  double *d_out, void *stream) {
  if (!d_links || !dims || !d_out) return na_fail("null argument");
  // the volume is checked after every factor, before any extent is
  // narrowed to int, so no product can wrap below the limit
  constexpr size_t kMaxSites = (size_t)kScratchBlocks * kNaThreads;
  size_t V = 1;
  for (int i = 0; i < 4; i++) {
    if (dims[i] < 2) return na_fail("every extent must be at least 2");
    if (dims[i] > kMaxSites || V * dims[i] > kMaxSites)
      return na_fail("lattice too large for the fixed scratch: at most "
                     "16777216 sites");
    V *= dims[i];
  }
  const size_t nblocks = (V + kNaThreads - 1) / kNaThreads;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return na_fail("no usable CUDA device");
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
      // set-up on the first call on this device (device is current)
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess) {
        snprintf(g_msg, sizeof g_msg, "cudaGetSymbolAddress: %s",
                 cudaGetErrorString(e));
        return -1;
      }
      g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  // every slot k_na_finish reads is written first by this call's
  // k_na_partials, so no clearing is needed
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_na_partials<<<(unsigned)nblocks, kNaThreads, 0, s>>>(
      reinterpret_cast<const double2 *>(d_links), (int)dims[0], (int)dims[1],
      (int)dims[2], (int)dims[3], scratch);
  k_na_finish<<<1, 1024, 0, s>>>(scratch, (int)nblocks, (double)V, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(g_msg, sizeof g_msg, "launch: %s", cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

}  // extern "C"
