// Shared device helpers for libdqz: complex arithmetic on interleaved
// (re, im) pairs, CTA-wide reductions, and decoding of node-tensor shapes
// from the packed graph tables.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/dqz.h"

namespace dqz {

// ---------------------------------------------------------------- complex
typedef double2 cd;  // complex128 as (re, im)

__host__ __device__ __forceinline__ cd mk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cd czero() { return make_double2(0.0, 0.0); }
__host__ __device__ __forceinline__ cd cadd(cd a, cd b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cd csub(cd a, cd b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cd cmul(cd a, cd b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// conj(a) * b
__host__ __device__ __forceinline__ cd cmulc(cd a, cd b) { return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
__host__ __device__ __forceinline__ cd cconj(cd a) { return mk(a.x, -a.y); }
__host__ __device__ __forceinline__ cd cscale(cd a, double s) { return mk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double cabs2(cd a) { return a.x * a.x + a.y * a.y; }
// acc += a * b
__device__ __forceinline__ void cfma(cd &acc, cd a, cd b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfmac(cd &acc, cd a, cd b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
__device__ __forceinline__ cd cdiv(cd a, cd b) {
  double den = b.x * b.x + b.y * b.y;
  return mk((a.x * b.x + a.y * b.y) / den, (a.y * b.x - a.x * b.y) / den);
}

// ------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Sum over each 16-lane half of the warp (every lane takes part).
__device__ __forceinline__ double half_sum(double v) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ cd warp_csum(cd v) {
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  return v;
}

// Warp copy of n16 16-byte chunks between non-overlapping buffers: each lane
// issues up to four loads before their stores, so a message costs one memory
// round trip per 2 KB instead of one per element.
__device__ __forceinline__ void warp_copy16(uint4 *__restrict__ dst, const uint4 *__restrict__ src, int n16) {
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < n16; base += 128) {
    uint4 buf[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int i = base + lane + 32 * j;
      if (i < n16) buf[j] = src[i];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int i = base + lane + 32 * j;
      if (i < n16) dst[i] = buf[j];
    }
  }
}

// Sum over the CTA; every thread gets the result. `red` needs 33 doubles of
// shared memory. Contains __syncthreads, so all threads must call it.
__device__ __forceinline__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < nw ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

// --------------------------------------------------------------- shapes
struct NodeShape {
  int k;            // degree
  int d;            // physical dimension
  int half0;        // first half-edge
  int dims[DQZ_MAX_DEGREE];
  long long stride[DQZ_MAX_DEGREE];  // element strides of the bonds
  long long size;   // d * prod dims
};

__device__ __forceinline__ void load_shape(const dqz_graph_t &g, int v, NodeShape &s) {
  s.k = g.node_degree[v];
  s.d = g.node_phys[v];
  s.half0 = g.node_half[v];
  long long st = s.d;
  for (int j = s.k - 1; j >= 0; --j) {
    int e = g.half_edge[s.half0 + j];
    s.dims[j] = g.edge_chi[e];
    s.stride[j] = st;
    st *= s.dims[j];
  }
  s.size = st;
}

// Division by a loop-invariant 32-bit divisor d >= 1 through a multiply-high,
// the round-up method of Granlund and Montgomery ("Division by invariant
// integers using multiplication", PLDI 1994): s = ceil(log2 d),
// m = floor(2^32 (2^s - d) / d) + 1 (< 2^32), x / d = (umulhi(x, m) + x) >> s
// for every 32-bit x. A hardware-free integer division costs a long
// instruction sequence; this one a multiply-high, an add and a shift.
// For d < 2^21 the multiplier comes from one correctly rounded double
// division: the numerator 2^32 (2^s - d) is exact in a double, and the exact
// quotient is never within the division's rounding error of an integer
// (checked exhaustively for every such d), so its floor is exact.
struct FastDiv {
  unsigned d, m, s;
  __device__ __forceinline__ explicit FastDiv(unsigned dv) : d(dv) {
    s = dv > 1 ? 32u - (unsigned)__clz(dv - 1u) : 0u;
    const unsigned long long num = (1ull << 32) * ((1ull << s) - dv);
    if (dv < (1u << 21))
      m = (unsigned)((unsigned long long)floor((double)num / (double)dv) + 1ull);
    else
      m = (unsigned)(num / dv + 1ull);
  }
  __device__ __forceinline__ unsigned div(unsigned x) const {
    return (unsigned)(((unsigned long long)__umulhi(x, m) + x) >> s);
  }
};

// Generic CTA-cooperative mode product on a row-major tensor:
//   Y[l, i, r] = sum_b M(i, b) X[l, b, r],  M(i, b) = m[i * rs + b * cs] (optionally conj)
// X has shape (L, qin, R); Y has shape (L, qout, R). X and Y must not alias.
// Index arithmetic is 32-bit when both tensors have fewer than 2^31 entries
// (always so for shared-memory operands); 64-bit division is a long
// instruction sequence and otherwise dominates these small contractions.
template <bool CONJ, typename I>
__device__ __forceinline__ void mode_product_idx(const cd *__restrict__ X, cd *__restrict__ Y, I L, int qin,
                                                 int qout, I R, const cd *__restrict__ m, int rs, int cs) {
  const I total = L * (I)qout * R;
  for (I o = threadIdx.x; o < total; o += blockDim.x) {
    I r = o % R;
    I t = o / R;
    int i = (int)(t % (I)qout);
    I l = t / (I)qout;
    const cd *x = X + (long long)(l * (I)qin) * R + r;
    const cd *mm = m + (long long)i * rs;
    cd acc = czero();
    for (int b = 0; b < qin; ++b) {
      cd mv = mm[(long long)b * cs];
      if (CONJ) mv = cconj(mv);
      cfma(acc, mv, x[(long long)b * R]);
    }
    Y[o] = acc;
  }
}

// The same with 32-bit indices and the divisions by R and qout through FastDiv
// (total < 2^31).
template <bool CONJ>
__device__ __forceinline__ void mode_product_fast(const cd *__restrict__ X, cd *__restrict__ Y, unsigned L, int qin,
                                                  int qout, unsigned R, const cd *__restrict__ m, int rs, int cs) {
  const unsigned total = L * (unsigned)qout * R;
  const FastDiv fR(R), fq((unsigned)qout);
  for (unsigned o = threadIdx.x; o < total; o += blockDim.x) {
    const unsigned t = fR.div(o);
    const unsigned r = o - t * R;
    const unsigned l = fq.div(t);
    const int i = (int)(t - l * (unsigned)qout);
    const cd *x = X + (l * (unsigned)qin) * R + r;
    const cd *mm = m + (long long)i * rs;
    cd acc = czero();
    for (int b = 0; b < qin; ++b) {
      cd mv = mm[(long long)b * cs];
      if (CONJ) mv = cconj(mv);
      cfma(acc, mv, x[(long long)b * R]);
    }
    Y[o] = acc;
  }
}

// The same products register-tiled: a thread owns MT outputs i x RT outputs r
// of one l, so each loaded entry of X serves MT products and each entry of m
// serves RT (one load per complex FMA instead of two). Each output is
// still one chain over b in increasing order, so the results are
// bit-identical to mode_product_fast.
template <bool CONJ>
__device__ __forceinline__ void mode_product_tiled(const cd *__restrict__ X, cd *__restrict__ Y, unsigned L,
                                                   int qin, int qout, unsigned R, const cd *__restrict__ m, int rs,
                                                   int cs) {
  constexpr int MT = 2, RT = 2;
  const unsigned ni = ((unsigned)qout + MT - 1) / MT, nr = (R + RT - 1) / RT;
  const unsigned tiles = L * ni * nr;
  const FastDiv fnr(nr), fni(ni);
  for (unsigned t = threadIdx.x; t < tiles; t += blockDim.x) {
    const unsigned u = fnr.div(t);
    const unsigned rb = t - u * nr;
    const unsigned l = fni.div(u);
    const unsigned ib = u - l * ni;
    const int i0 = (int)ib * MT;
    const unsigned r0 = rb * RT;
    const cd *x = X + (l * (unsigned)qin) * R + r0;
    cd acc[MT][RT];
#pragma unroll
    for (int a = 0; a < MT; ++a)
#pragma unroll
      for (int c = 0; c < RT; ++c) acc[a][c] = czero();
    for (int b = 0; b < qin; ++b) {
      cd xv[RT], mv[MT];
#pragma unroll
      for (int c = 0; c < RT; ++c) xv[c] = r0 + c < R ? x[(long long)b * R + c] : czero();
#pragma unroll
      for (int a = 0; a < MT; ++a) {
        cd v = i0 + a < qout ? m[(long long)(i0 + a) * rs + (long long)b * cs] : czero();
        if (CONJ) v = cconj(v);
        mv[a] = v;
      }
#pragma unroll
      for (int a = 0; a < MT; ++a)
#pragma unroll
        for (int c = 0; c < RT; ++c) cfma(acc[a][c], mv[a], xv[c]);
    }
#pragma unroll
    for (int a = 0; a < MT; ++a)
#pragma unroll
      for (int c = 0; c < RT; ++c)
        if (i0 + a < qout && r0 + c < R) Y[(l * (unsigned)qout + (unsigned)(i0 + a)) * R + r0 + c] = acc[a][c];
  }
}

template <bool CONJ>
__device__ __forceinline__ void mode_product(const cd *__restrict__ X, cd *__restrict__ Y, long long L, int qin,
                                             int qout, long long R, const cd *__restrict__ m, int rs, int cs) {
  const long long big = (qin > qout ? qin : qout);
  // tiles when there is at least one 2 x 2 tile per thread
  if (L * big * R < (1ll << 31) && qout >= 8 && R >= 2 && L * qout * R >= 4 * (long long)blockDim.x)
    mode_product_tiled<CONJ>(X, Y, (unsigned)L, qin, qout, (unsigned)R, m, rs, cs);
  else if (L * big * R < (1ll << 31))
    mode_product_fast<CONJ>(X, Y, (unsigned)L, qin, qout, (unsigned)R, m, rs, cs);
  else
    mode_product_idx<CONJ, long long>(X, Y, L, qin, qout, R, m, rs, cs);
}

}  // namespace dqz

#define DQZ_CHECK_LAUNCH()                                    \
  do {                                                        \
    cudaError_t _e = cudaGetLastError();                      \
    if (_e != cudaSuccess) return DQZ_ERR_CUDA;               \
  } while (0)

// Raises a kernel's dynamic shared-memory limit once per device (the
// attribute persists in the context), so that later launches -- including
// launches recorded into a CUDA graph -- make no further attribute calls.
#define DQZ_SMEM_ATTR_ONCE(kernel, bytes)                                                          \
  do {                                                                                             \
    static bool _dqz_attr_done[64] = {false};                                                      \
    int _dqz_dev = 0;                                                                              \
    if (cudaGetDevice(&_dqz_dev) != cudaSuccess || _dqz_dev < 0 || _dqz_dev >= 64) return DQZ_ERR_CUDA; \
    if (!_dqz_attr_done[_dqz_dev]) {                                                               \
      if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(bytes)) != \
          cudaSuccess)                                                                             \
        return DQZ_ERR_CUDA;                                                                       \
      _dqz_attr_done[_dqz_dev] = true;                                                             \
    }                                                                                              \
  } while (0)
