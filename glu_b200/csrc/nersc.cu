// NERSC configuration payloads <-> links on the GPU (GLU's I/O layer,
// src/IO/readers.c:169-310 and src/IO/writers.c, formats 4D_SU3_GAUGE (the
// top two rows of each link, 12 reals) and 4D_SU3_GAUGE_3x3 (18 reals)).
//
// The payload is the binary part of a NERSC file: for every site (x
// fastest), for every direction, the link's reals in row-major (re, im)
// order, as IEEE 64- or 32-bit numbers of either byte order.  The NERSC
// checksum is the 32-bit wrapping sum, over every stored number in host
// byte order, of its 32-bit words (readers.c:279-293), so blocks add their
// partial sums in any order and the result is exact.  The third row of a
// 12-real link is conj(row0 x row1) (readers.c:50-58), formed here with
// unfused products so that it rounds like the plain C expression.
//
// Links on the host side are GLU's double[V][4][9][2].  Self-contained: no
// engine, no workspace cache; each call stages through device buffers of
// its own.

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/glu_gfix.h"

namespace {

thread_local std::string t_err;

int nfail(const char *msg, cudaError_t e = cudaSuccess) {
  t_err = msg;
  if (e != cudaSuccess) {
    t_err += ": ";
    t_err += cudaGetErrorString(e);
  }
  return -1;
}

#define NCK(call)                                        \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return nfail(#call, e_);      \
  } while (0)

__device__ __forceinline__ uint32_t bswap32(uint32_t v) {
  return __byte_perm(v, 0, 0x0123);
}

// the j-th stored real of a link, in host order, plus its checksum words
__device__ __forceinline__ double load_real(const unsigned char *p, int bytes,
                                            bool swap, uint32_t *ck) {
  if (bytes == 8) {
    const uint2 w = *reinterpret_cast<const uint2 *>(p);
    const uint32_t lo = swap ? bswap32(w.y) : w.x;
    const uint32_t hi = swap ? bswap32(w.x) : w.y;
    *ck += lo + hi;
    return __hiloint2double((int)hi, (int)lo);
  }
  uint32_t w = *reinterpret_cast<const uint32_t *>(p);
  if (swap) w = bswap32(w);
  *ck += w;
  return (double)__uint_as_float(w);
}

__device__ __forceinline__ void store_real(unsigned char *p, int bytes, bool swap,
                                           double v, uint32_t *ck) {
  if (bytes == 8) {
    const uint32_t lo = (uint32_t)__double2loint(v), hi = (uint32_t)__double2hiint(v);
    *ck += lo + hi;
    uint2 w;
    w.x = swap ? bswap32(hi) : lo;
    w.y = swap ? bswap32(lo) : hi;
    *reinterpret_cast<uint2 *>(p) = w;
    return;
  }
  uint32_t w = __float_as_uint((float)v);
  *ck += w;
  *reinterpret_cast<uint32_t *>(p) = swap ? bswap32(w) : w;
}

// a * b - c * d for complex numbers (re, im), unfused
__device__ __forceinline__ double2 cmul_sub(double2 a, double2 b, double2 c,
                                            double2 d) {
  const double abr = __dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
  const double abi = __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x));
  const double cdr = __dsub_rn(__dmul_rn(c.x, d.x), __dmul_rn(c.y, d.y));
  const double cdi = __dadd_rn(__dmul_rn(c.x, d.y), __dmul_rn(c.y, d.x));
  return make_double2(__dsub_rn(abr, cdr), __dsub_rn(abi, cdi));
}

__device__ __forceinline__ void block_add(uint32_t v, uint32_t *total) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(total, v);
}

// one thread per link
__global__ void k_nersc_decode(const unsigned char *pay, size_t nlinks, int nreal,
                               int bytes, int swap, double2 *links,
                               uint32_t *cksum) {
  const size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  uint32_t ck = 0;
  if (l < nlinks) {
    const unsigned char *p = pay + l * (size_t)nreal * bytes;
    double2 o[9];
#pragma unroll
    for (int e = 0; e < 9; e++) {
      if (2 * e < nreal) {
        const double re = load_real(p + (size_t)(2 * e) * bytes, bytes, swap, &ck);
        const double im = load_real(p + (size_t)(2 * e + 1) * bytes, bytes, swap, &ck);
        o[e] = make_double2(re, im);
      }
    }
    if (nreal == 12) {
      // row 2 = conj(row0 x row1)
      double2 c;
      c = cmul_sub(o[1], o[5], o[2], o[4]);
      o[6] = make_double2(c.x, -c.y);
      c = cmul_sub(o[2], o[3], o[0], o[5]);
      o[7] = make_double2(c.x, -c.y);
      c = cmul_sub(o[0], o[4], o[1], o[3]);
      o[8] = make_double2(c.x, -c.y);
    }
    double2 *out = links + l * 9;
#pragma unroll
    for (int e = 0; e < 9; e++) out[e] = o[e];
  }
  block_add(ck, cksum);
}

__global__ void k_nersc_encode(const double2 *links, size_t nlinks, int nreal,
                               int bytes, int swap, unsigned char *pay,
                               uint32_t *cksum) {
  const size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  uint32_t ck = 0;
  if (l < nlinks) {
    unsigned char *p = pay + l * (size_t)nreal * bytes;
    const double2 *in = links + l * 9;
    for (int e = 0; 2 * e < nreal; e++) {
      const double2 v = in[e];
      store_real(p + (size_t)(2 * e) * bytes, bytes, swap, v.x, &ck);
      store_real(p + (size_t)(2 * e + 1) * bytes, bytes, swap, v.y, &ck);
    }
  }
  block_add(ck, cksum);
}

// SCIDAC / ILDG checksums (src/IO/writers.c:210-224, readers.c:256-263):
// per site the CRC-32 (the zlib / IEEE 802.3 polynomial, reflected) of the
// site's stored bytes, rotated left by (site % 29) and by (site % 31), all
// XORed -- exact in any order.  One thread per site, a 256-entry table.
__constant__ uint32_t c_crc_table[256];

__global__ void k_scidac_crc(const unsigned char *pay, size_t site_bytes,
                             size_t nsites, uint32_t *sums) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  uint32_t a = 0, b = 0;
  if (i < nsites) {
    const unsigned char *p = pay + i * site_bytes;
    uint32_t crc = 0xFFFFFFFFu;
    for (size_t k = 0; k < site_bytes; k++)
      crc = c_crc_table[(crc ^ p[k]) & 0xFFu] ^ (crc >> 8);
    crc ^= 0xFFFFFFFFu;
    const uint32_t r29 = (uint32_t)(i % 29), r31 = (uint32_t)(i % 31);
    a = r29 ? (crc << r29) | (crc >> (32 - r29)) : crc;
    b = r31 ? (crc << r31) | (crc >> (32 - r31)) : crc;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a ^= __shfl_down_sync(0xffffffffu, a, o);
    b ^= __shfl_down_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicXor(sums, a);
    atomicXor(sums + 1, b);
  }
}

int upload_crc_table() {
  static bool done = false;
  if (done) return 0;
  uint32_t t[256];
  for (uint32_t n = 0; n < 256; n++) {
    uint32_t c = n;
    for (int k = 0; k < 8; k++) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
    t[n] = c;
  }
  NCK(cudaMemcpyToSymbol(c_crc_table, t, sizeof t));
  done = true;
  return 0;
}

int check_args(const size_t dims[4], int nreal, int bytes, size_t *nlinks) {
  if (!dims) return nfail("null dims");
  if (nreal != 12 && nreal != 18) return nfail("reals per link must be 12 or 18");
  if (bytes != 8 && bytes != 4) return nfail("bytes per real must be 8 or 4");
  size_t v = 1;
  for (int i = 0; i < 4; i++) {
    if (dims[i] < 1) return nfail("zero extent");
    v *= dims[i];
  }
  *nlinks = v * 4;
  return 0;
}

// little-endian hosts: a big-endian payload is byte-swapped
bool need_swap(int big_endian) {
  const uint16_t probe = 1;
  unsigned char b;
  memcpy(&b, &probe, 1);
  const bool host_little = b == 1;
  return host_little == (big_endian != 0);
}

}  // namespace

extern "C" {

const char *gfix_nersc_error(void) { return t_err.c_str(); }

int gfix_nersc_decode(const void *payload, const size_t dims[4], int nreal,
                      int bytes_per_real, int big_endian, double *links,
                      uint32_t *checksum) {
  size_t nl = 0;
  if (check_args(dims, nreal, bytes_per_real, &nl)) return -1;
  if (!payload || !links) return nfail("null payload or links");
  const size_t pbytes = nl * nreal * bytes_per_real, lbytes = nl * 9 * sizeof(double2);
  unsigned char *d_p = nullptr;
  double2 *d_l = nullptr;
  uint32_t *d_c = nullptr;
  int rc = 0;
  cudaStream_t s = nullptr;
  do {
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) ||
        (e = cudaMalloc(&d_p, pbytes)) || (e = cudaMalloc(&d_l, lbytes)) ||
        (e = cudaMalloc(&d_c, sizeof(uint32_t)))) {
      rc = nfail("device buffers", e);
      break;
    }
    if ((e = cudaMemsetAsync(d_c, 0, sizeof(uint32_t), s)) ||
        (e = cudaMemcpyAsync(d_p, payload, pbytes, cudaMemcpyHostToDevice, s))) {
      rc = nfail("copy in", e);
      break;
    }
    const unsigned nb = (unsigned)((nl + 255) / 256);
    k_nersc_decode<<<nb, 256, 0, s>>>(d_p, nl, nreal, bytes_per_real,
                                      need_swap(big_endian), d_l, d_c);
    uint32_t ck = 0;
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(links, d_l, lbytes, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&ck, d_c, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s))) {
      rc = nfail("decode", e);
      break;
    }
    if (checksum) *checksum = ck;
  } while (0);
  cudaFree(d_p);
  cudaFree(d_l);
  cudaFree(d_c);
  if (s) cudaStreamDestroy(s);
  return rc;
}

int gfix_nersc_encode(const double *links, const size_t dims[4], int nreal,
                      int bytes_per_real, int big_endian, void *payload,
                      uint32_t *checksum) {
  size_t nl = 0;
  if (check_args(dims, nreal, bytes_per_real, &nl)) return -1;
  if (!payload || !links) return nfail("null payload or links");
  const size_t pbytes = nl * nreal * bytes_per_real, lbytes = nl * 9 * sizeof(double2);
  unsigned char *d_p = nullptr;
  double2 *d_l = nullptr;
  uint32_t *d_c = nullptr;
  int rc = 0;
  cudaStream_t s = nullptr;
  do {
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) ||
        (e = cudaMalloc(&d_p, pbytes)) || (e = cudaMalloc(&d_l, lbytes)) ||
        (e = cudaMalloc(&d_c, sizeof(uint32_t)))) {
      rc = nfail("device buffers", e);
      break;
    }
    if ((e = cudaMemsetAsync(d_c, 0, sizeof(uint32_t), s)) ||
        (e = cudaMemcpyAsync(d_l, links, lbytes, cudaMemcpyHostToDevice, s))) {
      rc = nfail("copy in", e);
      break;
    }
    const unsigned nb = (unsigned)((nl + 255) / 256);
    k_nersc_encode<<<nb, 256, 0, s>>>(d_l, nl, nreal, bytes_per_real,
                                      need_swap(big_endian), d_p, d_c);
    uint32_t ck = 0;
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(payload, d_p, pbytes, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&ck, d_c, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s))) {
      rc = nfail("encode", e);
      break;
    }
    if (checksum) *checksum = ck;
  } while (0);
  cudaFree(d_p);
  cudaFree(d_l);
  cudaFree(d_c);
  if (s) cudaStreamDestroy(s);
  return rc;
}

int gfix_scidac_checksum(const void *payload, size_t site_bytes, size_t nsites,
                         uint32_t *suma, uint32_t *sumb) {
  if (!payload || !site_bytes || !suma || !sumb) return nfail("null argument");
  if (upload_crc_table()) return -1;
  const size_t bytes = site_bytes * nsites;
  unsigned char *d_p = nullptr;
  uint32_t *d_s = nullptr;
  int rc = 0;
  cudaStream_t s = nullptr;
  do {
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) ||
        (e = cudaMalloc(&d_p, bytes ? bytes : 1)) ||
        (e = cudaMalloc(&d_s, 2 * sizeof(uint32_t)))) {
      rc = nfail("device buffers", e);
      break;
    }
    if ((e = cudaMemsetAsync(d_s, 0, 2 * sizeof(uint32_t), s)) ||
        (e = cudaMemcpyAsync(d_p, payload, bytes, cudaMemcpyHostToDevice, s))) {
      rc = nfail("copy in", e);
      break;
    }
    if (nsites) {
      const unsigned nb = (unsigned)((nsites + 127) / 128);
      k_scidac_crc<<<nb, 128, 0, s>>>(d_p, site_bytes, nsites, d_s);
    }
    uint32_t h[2] = {0, 0};
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(h, d_s, sizeof h, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s))) {
      rc = nfail("checksum", e);
      break;
    }
    *suma = h[0];
    *sumb = h[1];
  } while (0);
  cudaFree(d_p);
  cudaFree(d_s);
  if (s) cudaStreamDestroy(s);
  return rc;
}

}  // extern "C"
