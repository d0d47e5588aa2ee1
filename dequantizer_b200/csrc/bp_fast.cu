// Shape-specialised BP node update for degree-3 nodes with all bonds of
// dimension CHI (8 or 16) and physical dimension 2, in complex128 (FP64) or
// complex64 (FP32) -- the workload of random 3-regular graphs.
//
// Same arithmetic as tensor_ops.py:36-60 (pass_through_node), organised as
// small GEMMs on shared memory. One CTA owns one half-edge h = (v, e); for each
// physical index s it stages the slice T_s[a][b][c] = T[a, b, c, s] in shared
// memory and computes, with f < g the two other bonds,
//     W1 = T_s  x_f m_f,   W2 = W1 x_g m_g      (mode products)
//     P_w = partial of out_e over batch index w (one warp each)
//     out_e += sum_w P_w                          (fixed order)
// where x_f contracts bond f with a message's second index. Each warp
// computes whole CHI x CHI complex tiles with a register block of
// (CHI/8) x (CHI/4) outputs per lane; all strides are compile-time.
// After both s, out_e is divided by its trace and written as n2e[h].
#include "common.cuh"

using namespace dqz;

namespace {

template <typename C>
struct RealOf;
template <>
struct RealOf<double2> {
  typedef double R;
};
template <>
struct RealOf<float2> {
  typedef float R;
};

// Out(i, j) = sum_k A(i, k) * B(k, j) over k < KLEN, A(i,k) = A[i*SAI + k*SAK]
// (conjugated when CONJA), B(k,j) = B[k*SBK + j*SBJ]. Lane owns rows
// (lane>>2) + 8r and columns (lane&3) + 4c.
template <int CHI, int KLEN, int SAI, int SAK, int SBK, int SBJ, bool CONJA, typename C>
__device__ __forceinline__ void warp_tile(const C *__restrict__ A, const C *__restrict__ B,
                                          typename RealOf<C>::R (&re)[CHI / 8][CHI / 4],
                                          typename RealOf<C>::R (&im)[CHI / 8][CHI / 4]) {
  typedef typename RealOf<C>::R R;
  constexpr int RI = CHI / 8, RJ = CHI / 4;
  const int lane = threadIdx.x & 31;
  const int i0 = lane >> 2, j0 = lane & 3;
#pragma unroll
  for (int r = 0; r < RI; ++r)
#pragma unroll
    for (int c = 0; c < RJ; ++c) re[r][c] = im[r][c] = R(0);
#pragma unroll 4
  for (int k = 0; k < KLEN; ++k) {
    C a[RI], b[RJ];
#pragma unroll
    for (int r = 0; r < RI; ++r) a[r] = A[(i0 + 8 * r) * SAI + k * SAK];
#pragma unroll
    for (int c = 0; c < RJ; ++c) b[c] = B[k * SBK + (j0 + 4 * c) * SBJ];
#pragma unroll
    for (int r = 0; r < RI; ++r)
#pragma unroll
      for (int c = 0; c < RJ; ++c) {
        if (CONJA) {
          re[r][c] = fma(a[r].x, b[c].x, re[r][c]);
          re[r][c] = fma(a[r].y, b[c].y, re[r][c]);
          im[r][c] = fma(a[r].x, b[c].y, im[r][c]);
          im[r][c] = fma(-a[r].y, b[c].x, im[r][c]);
        } else {
          re[r][c] = fma(a[r].x, b[c].x, re[r][c]);
          re[r][c] = fma(-a[r].y, b[c].y, re[r][c]);
          im[r][c] = fma(a[r].x, b[c].y, im[r][c]);
          im[r][c] = fma(a[r].y, b[c].x, im[r][c]);
        }
      }
  }
}

template <int CHI, int SOI, int SOJ, typename C>
__device__ __forceinline__ void store_tile(C *O, const typename RealOf<C>::R (&re)[CHI / 8][CHI / 4],
                                           const typename RealOf<C>::R (&im)[CHI / 8][CHI / 4]) {
  const int lane = threadIdx.x & 31;
  const int i0 = lane >> 2, j0 = lane & 3;
#pragma unroll
  for (int r = 0; r < CHI / 8; ++r)
#pragma unroll
    for (int c = 0; c < CHI / 4; ++c) {
      C v;
      v.x = re[r][c];
      v.y = im[r][c];
      O[(i0 + 8 * r) * SOI + (j0 + 4 * c) * SOJ] = v;
    }
}

// Shared-memory strides of a CHI^3 slab [a][b][c] (c fastest) and of a CHI x CHI
// message: rows are padded by one element and slabs by one more, so that the
// distinct addresses a quarter-warp (16-byte elements) or half-warp (8-byte
// elements) touches in one load land in distinct banks.
template <int CHI>
struct Pad {
  static constexpr int RS = CHI + 1;       // b stride
  static constexpr int SS = CHI * RS + 1;  // a stride
  static constexpr int MS = CHI + 1;       // message row stride
  static constexpr int SLAB = CHI * SS;    // elements per slab buffer
};

// Y = X x_bond m (m[i][k] row-major, leading dimension MS), warp w owns
// batch index w.
template <int CHI, int BOND, typename C>
__device__ __forceinline__ void mode_product(const C *__restrict__ X, const C *__restrict__ m, C *__restrict__ Y) {
  typedef typename RealOf<C>::R R;
  constexpr int RS = Pad<CHI>::RS, SS = Pad<CHI>::SS, MS = Pad<CHI>::MS;
  const int w = threadIdx.x >> 5;
  R re[CHI / 8][CHI / 4], im[CHI / 8][CHI / 4];
  if (BOND == 0) {  // Y[a'][w][c] = sum_a m[a'][a] X[a][w][c]
    warp_tile<CHI, CHI, MS, 1, SS, 1, false>(m, X + w * RS, re, im);
    store_tile<CHI, SS, 1>(Y + w * RS, re, im);
  } else if (BOND == 1) {  // Y[w][b'][c] = sum_b m[b'][b] X[w][b][c]
    warp_tile<CHI, CHI, MS, 1, RS, 1, false>(m, X + w * SS, re, im);
    store_tile<CHI, RS, 1>(Y + w * SS, re, im);
  } else {  // Y[w][b][c'] = sum_c X[w][b][c] m[c'][c]
    warp_tile<CHI, CHI, RS, 1, 1, MS, false>(X + w * SS, m, re, im);
    store_tile<CHI, RS, 1>(Y + w * SS, re, im);
  }
}

// Partial tile of out_e for batch index w: P[w][i][j] at w*SS + i*RS + j.
template <int CHI, int E, typename C>
__device__ __forceinline__ void final_partial(const C *__restrict__ T, const C *__restrict__ Y, C *__restrict__ P) {
  typedef typename RealOf<C>::R R;
  constexpr int RS = Pad<CHI>::RS, SS = Pad<CHI>::SS;
  const int w = threadIdx.x >> 5;
  R re[CHI / 8][CHI / 4], im[CHI / 8][CHI / 4];
  if (E == 0) {  // sum_c conj(T[i][w][c]) Y[j][w][c]
    warp_tile<CHI, CHI, SS, 1, 1, SS, true>(T + w * RS, Y + w * RS, re, im);
  } else if (E == 1) {  // sum_c conj(T[w][i][c]) Y[w][j][c]
    warp_tile<CHI, CHI, RS, 1, 1, RS, true>(T + w * SS, Y + w * SS, re, im);
  } else {  // sum_b conj(T[w][b][i]) Y[w][b][j]
    warp_tile<CHI, CHI, 1, RS, RS, 1, true>(T + w * SS, Y + w * SS, re, im);
  }
  store_tile<CHI, RS, 1>(P + w * SS, re, im);
}

template <int CHI, int E, typename C>
__device__ __forceinline__ void products_and_partial(const C *sT, const C *m_lo, const C *m_hi, C *sW1, C *sW2) {
  // the two other bonds in ascending order
  constexpr int F = E == 0 ? 1 : 0;
  constexpr int G = E == 2 ? 1 : 2;
  mode_product<CHI, F>(sT, m_lo, sW1);
  __syncthreads();
  mode_product<CHI, G>(sW1, m_hi, sW2);
  __syncthreads();
  final_partial<CHI, E>(sT, sW2, sW1);
  __syncthreads();
}

__device__ __forceinline__ const void *msg_ptr(const dqz_graph_t &g, int hf, const void *n2e_old,
                                               const void *e2n_old, const void *n2e_new, const uint8_t *src_sel,
                                               size_t esize) {
  const int sel = src_sel[hf];
  const int64_t off = sel == DQZ_SRC_E2N_OLD ? g.half_msg_off[hf] : g.half_msg_off[g.half_twin[hf]];
  const void *base = sel == DQZ_SRC_E2N_OLD ? e2n_old : (sel == DQZ_SRC_N2E_NEW ? n2e_new : n2e_old);
  return (const unsigned char *)base + off * esize;
}

template <int CHI, typename C>
__global__ void __launch_bounds__(32 * CHI) bp_node_k3(dqz_graph_t g, const C *__restrict__ T, const C *n2e_old,
                                                       const C *e2n_old, C *n2e_new,
                                                       const uint8_t *__restrict__ src_sel,
                                                       const int32_t *__restrict__ halves, int n_halves,
                                                       int *error_flag) {
  typedef typename RealOf<C>::R R;
  constexpr int S2 = CHI * CHI;
  constexpr int RS = Pad<CHI>::RS, SS = Pad<CHI>::SS, MS = Pad<CHI>::MS, SLAB = Pad<CHI>::SLAB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *sT = reinterpret_cast<C *>(smem_raw);
  C *sW1 = sT + SLAB;
  C *sW2 = sW1 + SLAB;
  C *sM = sW2 + SLAB;  // two messages, CHI * MS each
  __shared__ R trace_re, trace_im;

  for (int item = blockIdx.x; item < n_halves; item += gridDim.x) {
    const int h = halves[item];
    const int v = g.half_node[h];
    const int h0 = g.node_half[v];
    const int e = h - h0;
    bool ok = g.node_degree[v] == 3 && g.node_phys[v] == 2;
    for (int f = 0; f < 3 && ok; ++f) ok = g.edge_chi[g.half_edge[h0 + f]] == CHI;
    if (!ok) {
      if (threadIdx.x == 0) atomicExch(error_flag, 1);
      continue;
    }
    const int f_lo = e == 0 ? 1 : 0, f_hi = e == 2 ? 1 : 2;
    const C *m_lo = (const C *)msg_ptr(g, h0 + f_lo, n2e_old, e2n_old, n2e_new, src_sel, sizeof(C));
    const C *m_hi = (const C *)msg_ptr(g, h0 + f_hi, n2e_old, e2n_old, n2e_new, src_sel, sizeof(C));
    for (int i = threadIdx.x; i < S2; i += blockDim.x) {
      const int r = i / CHI, c = i % CHI;
      sM[r * MS + c] = m_lo[i];
      sM[CHI * MS + r * MS + c] = m_hi[i];
    }
    const C *Tv = T + g.node_off[v];
    R acc_re = R(0), acc_im = R(0);  // out_e[t] for t = threadIdx.x < S2
    for (int s = 0; s < 2; ++s) {
      for (int i = threadIdx.x; i < CHI * S2; i += blockDim.x) {
        const int a = i / S2, b = (i / CHI) % CHI, c = i % CHI;
        sT[a * SS + b * RS + c] = Tv[2 * i + s];
      }
      __syncthreads();
      if (e == 0)
        products_and_partial<CHI, 0>(sT, sM, sM + CHI * MS, sW1, sW2);
      else if (e == 1)
        products_and_partial<CHI, 1>(sT, sM, sM + CHI * MS, sW1, sW2);
      else
        products_and_partial<CHI, 2>(sT, sM, sM + CHI * MS, sW1, sW2);
      for (int t = threadIdx.x; t < S2; t += blockDim.x) {
        const int off = (t / CHI) * RS + t % CHI;
        R sr = R(0), si = R(0);
#pragma unroll 4
        for (int w = 0; w < CHI; ++w) {
          const C p = sW1[w * SS + off];
          sr += p.x;
          si += p.y;
        }
        acc_re += sr;
        acc_im += si;
      }
      __syncthreads();
    }
    // trace, then the normalised message
    const int t = threadIdx.x;
    if (t < S2) {
      sW2[t].x = acc_re;
      sW2[t].y = acc_im;
    }
    __syncthreads();
    if (t == 0) {
      R tr = 0, ti = 0;
      for (int i = 0; i < CHI; ++i) {
        tr += sW2[i * CHI + i].x;
        ti += sW2[i * CHI + i].y;
      }
      trace_re = tr;
      trace_im = ti;
    }
    __syncthreads();
    if (t < S2) {
      const R tr = trace_re, ti = trace_im;
      const R den = tr * tr + ti * ti;
      C o;
      o.x = (acc_re * tr + acc_im * ti) / den;
      o.y = (acc_im * tr - acc_re * ti) / den;
      n2e_new[g.half_msg_off[h] + t] = o;
    }
    __syncthreads();
  }
}

template <int CHI, typename C>
size_t k3_smem() {
  return (3 * (size_t)Pad<CHI>::SLAB + 2 * (size_t)CHI * Pad<CHI>::MS) * sizeof(C);
}

template <int CHI, typename C>
int launch_k3(const dqz_graph_t *g, const void *T, const void *n2e_old, const void *e2n_old, void *n2e_new,
              const uint8_t *src_sel, const int32_t *halves, int n_halves, int *error_flag, cudaStream_t stream) {
  const size_t smem = k3_smem<CHI, C>();
  if (smem > 227 * 1024) return DQZ_ERR_UNSUPPORTED;
  DQZ_SMEM_ATTR_ONCE((bp_node_k3<CHI, C>), smem);
  bp_node_k3<CHI, C><<<n_halves, 32 * CHI, smem, stream>>>(*g, (const C *)T, (const C *)n2e_old,
                                                           (const C *)e2n_old, (C *)n2e_new, src_sel, halves,
                                                           n_halves, error_flag);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

// X <- X x_bond m in place for batch index w (the warp's slice of X is both
// read and written; every lane finishes its reads before any lane stores).
template <int CHI, int BOND, typename C>
__device__ __forceinline__ void mode_product_inplace(C *X, const C *__restrict__ m, int w) {
  typedef typename RealOf<C>::R R;
  constexpr int RS = Pad<CHI>::RS, SS = Pad<CHI>::SS, MS = Pad<CHI>::MS;
  R re[CHI / 8][CHI / 4], im[CHI / 8][CHI / 4];
  if (BOND == 0) {
    warp_tile<CHI, CHI, MS, 1, SS, 1, false>(m, X + w * RS, re, im);
    __syncwarp();
    store_tile<CHI, SS, 1>(X + w * RS, re, im);
  } else if (BOND == 1) {
    warp_tile<CHI, CHI, MS, 1, RS, 1, false>(m, X + w * SS, re, im);
    __syncwarp();
    store_tile<CHI, RS, 1>(X + w * SS, re, im);
  } else {
    warp_tile<CHI, CHI, RS, 1, 1, MS, false>(X + w * SS, m, re, im);
    __syncwarp();
    store_tile<CHI, RS, 1>(X + w * SS, re, im);
  }
}

// Vidal-gauge absorption (tensor_ops.py:88-93, absorb_by_node) for degree-3
// nodes with bonds of dimension CHI and physical dimension 2, complex128:
//     T'[a'][b'][c'][s] = sum_{a,b,c} G0[a][a'] G1[b][b'] G2[c][c'] T[a][b][c][s]
// (G_f = the orthogonaliser of the node's f-th half-edge, row-major), then
// T' / ||T'||_F. One CTA of 2 * CHI warps per node: both physical slabs stay
// in padded shared memory, warp (s, w) owns batch index w of slab s in each
// of the three in-place mode products, and the norm is reduced from shared
// memory before the single write.
template <int CHI>
__global__ void __launch_bounds__(64 * CHI) absorb_k3(dqz_graph_t g, const double2 *__restrict__ Tin,
                                                      const double2 *__restrict__ orth, double2 *Tout,
                                                      const int32_t *__restrict__ sel, int total, int *error_flag) {
  typedef double2 C;
  constexpr int S2 = CHI * CHI, S3 = CHI * S2;
  constexpr int RS = Pad<CHI>::RS, SS = Pad<CHI>::SS, MS = Pad<CHI>::MS, SLAB = Pad<CHI>::SLAB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *sX = reinterpret_cast<C *>(smem_raw);  // two slabs
  C *sM = sX + 2 * SLAB;                    // three transposed orthogonalisers, CHI * MS each
  __shared__ double red[48];
  const int warp = threadIdx.x >> 5;
  C *mine = sX + (warp / CHI) * SLAB;
  const int w = warp % CHI;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    const int v = sel ? sel[item] : item;
    const int h0 = g.node_half[v];
    bool ok = g.node_degree[v] == 3 && g.node_phys[v] == 2;
    for (int f = 0; f < 3 && ok; ++f) ok = g.edge_chi[g.half_edge[h0 + f]] == CHI;
    if (!ok) {
      if (threadIdx.x == 0) atomicExch(error_flag, 1);
      continue;
    }
    for (int i = threadIdx.x; i < 3 * S2; i += blockDim.x) {
      const int f = i / S2, a = (i / CHI) % CHI, j = i % CHI;
      sM[f * CHI * MS + j * MS + a] = orth[g.half_msg_off[h0 + f] + a * CHI + j];
    }
    const C *T = Tin + g.node_off[v];
    for (int i = threadIdx.x; i < 2 * S3; i += blockDim.x) {
      const int t = i >> 1;
      sX[(i & 1) * SLAB + (t / S2) * SS + ((t / CHI) % CHI) * RS + t % CHI] = T[i];
    }
    __syncthreads();
    mode_product_inplace<CHI, 0>(mine, sM, w);
    __syncthreads();
    mode_product_inplace<CHI, 1>(mine, sM + CHI * MS, w);
    __syncthreads();
    mode_product_inplace<CHI, 2>(mine, sM + 2 * CHI * MS, w);
    __syncthreads();
    double n2 = 0.0;
    for (int i = threadIdx.x; i < 2 * S3; i += blockDim.x) {
      const int t = i >> 1;
      const C x = sX[(i & 1) * SLAB + (t / S2) * SS + ((t / CHI) % CHI) * RS + t % CHI];
      n2 += x.x * x.x + x.y * x.y;
    }
    const double inv = 1.0 / sqrt(block_sum(n2, red));
    C *O = Tout + g.node_off[v];
    for (int i = threadIdx.x; i < 2 * S3; i += blockDim.x) {
      const int t = i >> 1;
      const C x = sX[(i & 1) * SLAB + (t / S2) * SS + ((t / CHI) % CHI) * RS + t % CHI];
      O[i] = make_double2(x.x * inv, x.y * inv);
    }
    __syncthreads();
  }
}

template <int CHI>
int launch_absorb_k3(const dqz_graph_t *g, const void *tin, const void *orth, void *tout, const int32_t *sel,
                     int total, int *error_flag, cudaStream_t stream) {
  const size_t smem = (2 * (size_t)Pad<CHI>::SLAB + 3 * (size_t)CHI * Pad<CHI>::MS) * sizeof(double2);
  if (smem > 227 * 1024) return DQZ_ERR_UNSUPPORTED;
  DQZ_SMEM_ATTR_ONCE(absorb_k3<CHI>, smem);
  absorb_k3<CHI><<<total, 64 * CHI, smem, stream>>>(*g, (const double2 *)tin, (const double2 *)orth,
                                                     (double2 *)tout, sel, total, error_flag);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

template <typename W>
__global__ void edge_pass_words(dqz_graph_t g, const W *n2e_old, const W *n2e_new, const uint8_t *edge_new,
                                W *e2n_new) {
  const int wpb = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int h = blockIdx.x * wpb + (threadIdx.x >> 5); h < g.n_halves; h += gridDim.x * wpb) {
    const int e = g.half_edge[h], tw = g.half_twin[h];
    if (e < 0 || tw < 0) continue;
    const int c = g.edge_chi[e];
    const W *src = (edge_new[h] ? n2e_new : n2e_old) + g.half_msg_off[tw];
    W *dst = e2n_new + g.half_msg_off[h];
    const int bytes = c * c * (int)sizeof(W);
    if (bytes % 16 == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0)
      warp_copy16(reinterpret_cast<uint4 *>(dst), reinterpret_cast<const uint4 *>(src), bytes / 16);
    else
      for (int i = lane; i < c * c; i += 32) dst[i] = src[i];
  }
}

}  // namespace

extern "C" int dqz_bp_node_update_k3(const dqz_graph_t *g, int32_t chi, int32_t precision, const void *tensors,
                                     const void *n2e_old, const void *e2n_old, void *n2e_new, const uint8_t *src_sel,
                                     const int32_t *halves, int32_t n_halves, int32_t *error_flag,
                                     cudaStream_t stream) {
  if (!g || !tensors || !n2e_old || !e2n_old || !n2e_new || !src_sel || !halves || !error_flag || n_halves < 0)
    return DQZ_ERR_ARG;
  if (n_halves == 0) return DQZ_OK;
  if (precision == 64) {
    if (chi == 16) return launch_k3<16, double2>(g, tensors, n2e_old, e2n_old, n2e_new, src_sel, halves, n_halves,
                                                 error_flag, stream);
    if (chi == 8) return launch_k3<8, double2>(g, tensors, n2e_old, e2n_old, n2e_new, src_sel, halves, n_halves,
                                               error_flag, stream);
  } else if (precision == 32) {
    if (chi == 16) return launch_k3<16, float2>(g, tensors, n2e_old, e2n_old, n2e_new, src_sel, halves, n_halves,
                                                error_flag, stream);
    if (chi == 8) return launch_k3<8, float2>(g, tensors, n2e_old, e2n_old, n2e_new, src_sel, halves, n_halves,
                                              error_flag, stream);
  }
  return DQZ_ERR_UNSUPPORTED;
}

extern "C" int dqz_absorb_k3(const dqz_graph_t *g, int32_t chi, const void *tensors_in, const void *orth,
                             void *tensors_out, const int32_t *nodes, int32_t n_sel, int32_t *error_flag,
                             cudaStream_t stream) {
  if (!g || !tensors_in || !orth || !tensors_out || !error_flag) return DQZ_ERR_ARG;
  if (nodes && (n_sel < 0 || n_sel > g->n_nodes)) return DQZ_ERR_ARG;
  const int total = nodes ? n_sel : g->n_nodes;
  if (total == 0) return DQZ_OK;
  if (chi == 16) return launch_absorb_k3<16>(g, tensors_in, orth, tensors_out, nodes, total, error_flag, stream);
  if (chi == 8) return launch_absorb_k3<8>(g, tensors_in, orth, tensors_out, nodes, total, error_flag, stream);
  return DQZ_ERR_UNSUPPORTED;
}

extern "C" int dqz_bp_edge_pass_c64(const dqz_graph_t *g, const void *n2e_old, const void *n2e_new,
                                    const uint8_t *edge_new, void *e2n_new, cudaStream_t stream) {
  if (!g || !n2e_old || !n2e_new || !edge_new || !e2n_new) return DQZ_ERR_ARG;
  if (g->n_halves == 0) return DQZ_OK;
  const int wpb = 8;
  edge_pass_words<float2><<<(g->n_halves + wpb - 1) / wpb, 32 * wpb, 0, stream>>>(
      *g, (const float2 *)n2e_old, (const float2 *)n2e_new, edge_new, (float2 *)e2n_new);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
