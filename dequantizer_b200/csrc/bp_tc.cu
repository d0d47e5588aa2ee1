// BP node update on tensor cores: BF16 operands, FP32 accumulation, for
// degree-3 nodes with bonds of dimension 16 and physical dimension 2 (the
// mixed-precision form of tensor_ops.py:36-60 for random 3-regular graphs).
//
// One CTA (8 warps) owns one node and produces its three outgoing messages.
// The node tensor is kept in HBM as BF16 planes (converted once by
// dqz_pack_bf16_planes; it does not change between sweeps): per node,
// [s][re|im][a][b][c]. For each physical index s the two planes are copied
// (cp.async, 16 B) into a padded natural layout Tn[a*SS + b*RS + c], and every
// GEMM operand is a view of it, read with ldmatrix (.trans where the
// contracted index is not the contiguous one):
//   X    = T x_0 m_0                 rows (b,c), k = a      (shared prefix)
//   Y2_1 = X x_2 m_2 -> out_1        rows (b,a'), k = c
//   Y2_2 = X x_1 m_1 -> out_2        rows (c,a'), k = b
//   X    = T x_1 m_1, Y2_0 = X x_2 m_2 -> out_0
//   out_e[m][n] += sum_x Y2_e[m][x] conj(T[.., n_e, ..][x])   (final)
// where x_f contracts bond f with a message's second index. A complex product
// is four real BF16 products (re*re - im*im, re*im + im*re) with the minus
// sign applied by flipping BF16 sign bits in the operand registers. The final
// contraction splits K = 256 over the warps; partials are summed in a fixed
// order. The message n2e[v, e][n][m] = out_e[m][n] / trace, complex64.
#include <cuda_bf16.h>

#include "common.cuh"
#include "mma_bf16.cuh"

namespace {

constexpr int CH = 16;
constexpr int RS = 24;              // b stride of the natural layout (bf16)
constexpr int SS = CH * RS + 8;     // a stride (392)
constexpr int NAT = CH * SS;        // elements per natural-layout plane (6272)
constexpr int LDM = 24;             // row stride of message operands
constexpr int LD4 = 264;            // row stride of Y2 (K = 256 rows)
constexpr int TC_THREADS = 256;
constexpr int NODE_BF16 = 2 * 2 * CH * CH * CH;  // bf16 elements per node in HBM

struct __align__(16) TcSmem {
  __nv_bfloat16 Tn[2][NAT];           // [re,im] natural layout of T_s
  __nv_bfloat16 X[2][NAT];            // natural layout of a mode product; final partials reuse it
  __nv_bfloat16 Y2[2][2][CH * LD4];   // two Y2 buffers x [re,im], rows e, k = x
  __nv_bfloat16 M[3][2][CH * LDM];    // messages of bonds 0,1,2 x [re,im], rows n, k
  float redw[8][2];
  float red[2];
};
static_assert(sizeof(float) * 8 * 2 * 2 * 32 * 4 <= sizeof(__nv_bfloat16) * 2 * NAT, "partials fit in X");

// --- fragment loaders. For an A tile (16 m x 16 k) the four 8x8 matrices are
// (m 0-7,k 0-7), (m 8-15,k 0-7), (m 0-7,k 8-15), (m 8-15,k 8-15); lane i
// addresses row i%8 of matrix i/8. `row(mm, kk)` gives the element address
// of A(m = mm, k = kk) for the non-transposed form (rows m, k contiguous);
// for the transposed form the address of A(m, k) with m contiguous.

// A from rows m with k contiguous: p(m) + k.
__device__ __forceinline__ void load_a_rows(const __nv_bfloat16 *base, int mstride, int k0, uint32_t (&a)[4]) {
  const int lane = threadIdx.x & 31, j = lane >> 3;
  const __nv_bfloat16 *p = base + ((j & 1) * 8 + (lane & 7)) * mstride + k0 + (j >> 1) * 8;
  ldsm_x4(saddr(p), a[0], a[1], a[2], a[3]);
}
// A with m contiguous, memory rows indexed by k: element (m, k) at base + k*kstride + m.
__device__ __forceinline__ void load_a_trans(const __nv_bfloat16 *base, int kstride, uint32_t (&a)[4]) {
  const int lane = threadIdx.x & 31, j = lane >> 3;
  const __nv_bfloat16 *p = base + ((j >> 1) * 8 + (lane & 7)) * kstride + (j & 1) * 8;
  ldsm_x4_t(saddr(p), a[0], a[1], a[2], a[3]);
}
// B fragments of two n-tiles from rows n with k contiguous: element (k, n) at base + n*nstride + k.
__device__ __forceinline__ void load_b_rows(const __nv_bfloat16 *base, int nstride, uint32_t (&b)[2][2]) {
  const int lane = threadIdx.x & 31, j = lane >> 3;
  const __nv_bfloat16 *p = base + ((j >> 1) * 8 + (lane & 7)) * nstride + (j & 1) * 8;
  ldsm_x4(saddr(p), b[0][0], b[0][1], b[1][0], b[1][1]);
}
// B fragments of two n-tiles with n contiguous, memory rows indexed by k:
// element (k, n) at base + k*kstride + n.
__device__ __forceinline__ void load_b_trans(const __nv_bfloat16 *base, int kstride, uint32_t (&b)[2][2]) {
  const int lane = threadIdx.x & 31, j = lane >> 3;
  const __nv_bfloat16 *p = base + ((j & 1) * 8 + (lane & 7)) * kstride + (j >> 1) * 8;
  ldsm_x4_t(saddr(p), b[0][0], b[0][1], b[1][0], b[1][1]);
}

// D fragment element (row r, col c) of an m16n8 tile: held by lane
// (r%8)*4 + c/2 in register (r/8)*2 + c%2.
struct Frag {
  int g, t;  // lane / 4, lane % 4
};

// Final of one output: partials of D[m][n] = sum_x Y2[m][x] conj(B(x, n)) over the
// warp's two k-steps, written to `part`; B given by a loader functor.
template <typename LoadB>
__device__ __forceinline__ void final_partial(const __nv_bfloat16 *Y2r, const __nv_bfloat16 *Y2i, LoadB load_b,
                                              float *part) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float dr[2][4] = {}, di[2][4] = {};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int k0 = (2 * w + q) * 16;
    uint32_t yr[4], yi[4], br[2][2], bi[2][2];
    load_a_rows(Y2r, LD4, k0, yr);
    load_a_rows(Y2i, LD4, k0, yi);
    load_b(k0, br, bi);
    cmma_conjb(yr, yi, br, bi, dr, di);
  }
  // part[w][nt][re,im][lane][reg]
#pragma unroll
  for (int nt = 0; nt < 2; ++nt)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      part[(((w * 2 + nt) * 2 + 0) * 32 + lane) * 4 + r] = dr[nt][r];
      part[(((w * 2 + nt) * 2 + 1) * 32 + lane) * 4 + r] = di[nt][r];
    }
}

__device__ __forceinline__ void reduce_partials(const float *part, float &acc_re, float &acc_im) {
  const int tid = threadIdx.x;
  const int m = tid >> 4, n = tid & 15;
  const int nt = n >> 3, col = n & 7;
  const int src_lane = ((m & 7) << 2) | (col >> 1);
  const int reg = ((m >> 3) << 1) | (col & 1);
  float sr = 0.f, si = 0.f;
#pragma unroll
  for (int ww = 0; ww < 8; ++ww) {
    sr += part[(((ww * 2 + nt) * 2 + 0) * 32 + src_lane) * 4 + reg];
    si += part[(((ww * 2 + nt) * 2 + 1) * 32 + src_lane) * 4 + reg];
  }
  acc_re += sr;
  acc_im += si;
}

__global__ void __launch_bounds__(TC_THREADS, 2) bp_node_k3_tc(dqz_graph_t g, const __nv_bfloat16 *__restrict__ Tb,
                                                                const float2 *n2e_old, const float2 *e2n_old,
                                                                float2 *n2e_new, const uint8_t *__restrict__ src_sel,
                                                                const int32_t *__restrict__ nodes, int n_nodes,
                                                                int *error_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TcSmem &S = *reinterpret_cast<TcSmem *>(smem_raw);
  float *part = reinterpret_cast<float *>(&S.X[0][0]);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;

  for (int item = blockIdx.x; item < n_nodes; item += gridDim.x) {
    const int v = nodes[item];
    const int h0 = g.node_half[v];
    bool ok = g.node_degree[v] == 3 && g.node_phys[v] == 2;
    for (int q = 0; q < 3 && ok; ++q) ok = g.edge_chi[g.half_edge[h0 + q]] == CH;
    if (!ok) {
      if (tid == 0) atomicExch(error_flag, 1);
      continue;
    }
    {  // messages of the three bonds, rows n, k (tid <-> (n, k))
      const int n = tid >> 4, k = tid & 15;
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        const float2 x = msg_c64(g, h0 + f, n2e_old, e2n_old, n2e_new, src_sel)[n * CH + k];
        S.M[f][0][n * LDM + k] = __float2bfloat16_rn(x.x);
        S.M[f][1][n * LDM + k] = __float2bfloat16_rn(x.y);
      }
    }
    const __nv_bfloat16 *Tv = Tb + (size_t)v * NODE_BF16;
    float acc[3][2] = {};  // out_e[m][n], m = tid >> 4, n = tid & 15

    for (int s = 0; s < 2; ++s) {
      // ---- stage T_s: 2 planes x 256 rows (a,b) x 2 chunks of 8 c, 16 B each
      for (int q = tid; q < 1024; q += TC_THREADS) {
        const int p = q >> 9, rem = q & 511, row = rem >> 1, half = rem & 1;
        const int a = row >> 4, b = row & 15;
        const __nv_bfloat16 *src = Tv + ((s * 2 + p) * CH * CH + row) * CH + half * 8;
        const uint32_t dst = saddr(&S.Tn[p][a * SS + b * RS + half * 8]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
      }
      asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
      __syncthreads();

      // ---- PRE: X[a'][b][c] = sum_a m0[a'][a] T[a][b][c]; m-tile = b (rows c), k = a
      {
        uint32_t br[2][2], bi[2][2];
        load_b_rows(S.M[0][0], LDM, br);
        load_b_rows(S.M[0][1], LDM, bi);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int b = 2 * w + q;
          uint32_t ar[4], ai[4];
          load_a_trans(&S.Tn[0][b * RS], SS, ar);
          load_a_trans(&S.Tn[1][b * RS], SS, ai);
          float dr[2][4] = {}, di[2][4] = {};
          cmma(ar, ai, br, bi, dr, di);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              const int c = gq + 8 * (r >> 1), ap = nt * 8 + 2 * tq + (r & 1);
              S.X[0][ap * SS + b * RS + c] = __float2bfloat16_rn(dr[nt][r]);
              S.X[1][ap * SS + b * RS + c] = __float2bfloat16_rn(di[nt][r]);
            }
        }
      }
      __syncthreads();

      // ---- MP2 for e = 1: Y2_1[b][a'*16 + c'] = sum_c X[a'][b][c] m2[c'][c]; m-tile = b (rows a')
      // ---- MP2 for e = 2: Y2_2[c][a'*16 + b'] = sum_b X[a'][b][c] m1[b'][b]; m-tile = a' (rows c)
      {
        uint32_t br[2][2], bi[2][2], cr[2][2], ci[2][2];
        load_b_rows(S.M[2][0], LDM, br);
        load_b_rows(S.M[2][1], LDM, bi);
        load_b_rows(S.M[1][0], LDM, cr);
        load_b_rows(S.M[1][1], LDM, ci);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int t = 2 * w + q;
          {  // e = 1, m-tile b = t
            uint32_t ar[4], ai[4];
            load_a_rows(&S.X[0][t * RS], SS, 0, ar);
            load_a_rows(&S.X[1][t * RS], SS, 0, ai);
            float dr[2][4] = {}, di[2][4] = {};
            cmma(ar, ai, br, bi, dr, di);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
              for (int hh = 0; hh < 2; ++hh) {
                const int ap = gq + 8 * hh, cp = nt * 8 + 2 * tq;
                *reinterpret_cast<__nv_bfloat162 *>(&S.Y2[0][0][t * LD4 + ap * CH + cp]) =
                    __floats2bfloat162_rn(dr[nt][2 * hh], dr[nt][2 * hh + 1]);
                *reinterpret_cast<__nv_bfloat162 *>(&S.Y2[0][1][t * LD4 + ap * CH + cp]) =
                    __floats2bfloat162_rn(di[nt][2 * hh], di[nt][2 * hh + 1]);
              }
          }
          {  // e = 2, m-tile a' = t, rows c, k = b
            uint32_t ar[4], ai[4];
            load_a_trans(&S.X[0][t * SS], RS, ar);
            load_a_trans(&S.X[1][t * SS], RS, ai);
            float dr[2][4] = {}, di[2][4] = {};
            cmma(ar, ai, cr, ci, dr, di);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
              for (int hh = 0; hh < 2; ++hh) {
                const int c = gq + 8 * hh, bp = nt * 8 + 2 * tq;
                *reinterpret_cast<__nv_bfloat162 *>(&S.Y2[1][0][c * LD4 + t * CH + bp]) =
                    __floats2bfloat162_rn(dr[nt][2 * hh], dr[nt][2 * hh + 1]);
                *reinterpret_cast<__nv_bfloat162 *>(&S.Y2[1][1][c * LD4 + t * CH + bp]) =
                    __floats2bfloat162_rn(di[nt][2 * hh], di[nt][2 * hh + 1]);
              }
          }
        }
      }
      __syncthreads();

      // ---- FIN e = 1: out1[b][b''] = sum_{a,c} Y2_1[b][a*16+c] conj(T[a][b''][c])
      final_partial(S.Y2[0][0], S.Y2[0][1],
                    [&](int k0, uint32_t (&br)[2][2], uint32_t (&bi)[2][2]) {
                      const int a = k0 >> 4;  // k0 = a*16 (+0): the k-step covers c = 0..15
                      load_b_rows(&S.Tn[0][a * SS], RS, br);
                      load_b_rows(&S.Tn[1][a * SS], RS, bi);
                    },
                    part);
      __syncthreads();
      reduce_partials(part, acc[1][0], acc[1][1]);
      __syncthreads();
      // ---- FIN e = 2: out2[c][c''] = sum_{a,b} Y2_2[c][a*16+b] conj(T[a][b][c''])
      final_partial(S.Y2[1][0], S.Y2[1][1],
                    [&](int k0, uint32_t (&br)[2][2], uint32_t (&bi)[2][2]) {
                      const int a = k0 >> 4;  // k = (a, b), b = 0..15 within the step
                      load_b_trans(&S.Tn[0][a * SS], RS, br);
                      load_b_trans(&S.Tn[1][a * SS], RS, bi);
                    },
                    part);
      __syncthreads();
      reduce_partials(part, acc[2][0], acc[2][1]);
      __syncthreads();

      // ---- e = 0: X[a][b'][c] = sum_b m1[b'][b] T[a][b][c]; m-tile = a (rows c), k = b
      {
        uint32_t br[2][2], bi[2][2];
        load_b_rows(S.M[1][0], LDM, br);
        load_b_rows(S.M[1][1], LDM, bi);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int a = 2 * w + q;
          uint32_t ar[4], ai[4];
          load_a_trans(&S.Tn[0][a * SS], RS, ar);
          load_a_trans(&S.Tn[1][a * SS], RS, ai);
          float dr[2][4] = {}, di[2][4] = {};
          cmma(ar, ai, br, bi, dr, di);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              const int c = gq + 8 * (r >> 1), bp = nt * 8 + 2 * tq + (r & 1);
              S.X[0][a * SS + bp * RS + c] = __float2bfloat16_rn(dr[nt][r]);
              S.X[1][a * SS + bp * RS + c] = __float2bfloat16_rn(di[nt][r]);
            }
        }
      }
      __syncthreads();
      // ---- MP2 e = 0: Y2_0[a][b'*16 + c'] = sum_c X[a][b'][c] m2[c'][c]; m-tile = a (rows b')
      {
        uint32_t br[2][2], bi[2][2];
        load_b_rows(S.M[2][0], LDM, br);
        load_b_rows(S.M[2][1], LDM, bi);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int a = 2 * w + q;
          uint32_t ar[4], ai[4];
          load_a_rows(&S.X[0][a * SS], RS, 0, ar);
          load_a_rows(&S.X[1][a * SS], RS, 0, ai);
          float dr[2][4] = {}, di[2][4] = {};
          cmma(ar, ai, br, bi, dr, di);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
              const int bp = gq + 8 * hh, cp = nt * 8 + 2 * tq;
              *reinterpret_cast<__nv_bfloat162 *>(&S.Y2[0][0][a * LD4 + bp * CH + cp]) =
                  __floats2bfloat162_rn(dr[nt][2 * hh], dr[nt][2 * hh + 1]);
              *reinterpret_cast<__nv_bfloat162 *>(&S.Y2[0][1][a * LD4 + bp * CH + cp]) =
                  __floats2bfloat162_rn(di[nt][2 * hh], di[nt][2 * hh + 1]);
            }
        }
      }
      __syncthreads();
      // ---- FIN e = 0: out0[a][a''] = sum_{b,c} Y2_0[a][b*16+c] conj(T[a''][b][c])
      final_partial(S.Y2[0][0], S.Y2[0][1],
                    [&](int k0, uint32_t (&br)[2][2], uint32_t (&bi)[2][2]) {
                      const int b = k0 >> 4;  // k = (b, c), c = 0..15 within the step
                      load_b_rows(&S.Tn[0][b * RS], SS, br);
                      load_b_rows(&S.Tn[1][b * RS], SS, bi);
                    },
                    part);
      __syncthreads();
      reduce_partials(part, acc[0][0], acc[0][1]);
      __syncthreads();
    }

    // ---- normalise by the trace and store message[n][m] = out_e[m][n] / tr
    const int m = tid >> 4, n = tid & 15;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      float tre = (m == n) ? acc[e][0] : 0.f, tim = (m == n) ? acc[e][1] : 0.f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        tre += __shfl_xor_sync(0xffffffffu, tre, o);
        tim += __shfl_xor_sync(0xffffffffu, tim, o);
      }
      if (lane == 0) {
        S.redw[w][0] = tre;
        S.redw[w][1] = tim;
      }
      __syncthreads();
      if (tid == 0) {
        float sr = 0.f, si = 0.f;
        for (int ww = 0; ww < 8; ++ww) {
          sr += S.redw[ww][0];
          si += S.redw[ww][1];
        }
        S.red[0] = sr;
        S.red[1] = si;
      }
      __syncthreads();
      const float tr = S.red[0], ti = S.red[1];
      const float den = tr * tr + ti * ti;
      float2 o;
      o.x = (acc[e][0] * tr + acc[e][1] * ti) / den;
      o.y = (acc[e][1] * tr - acc[e][0] * ti) / den;
      n2e_new[g.half_msg_off[h0 + e] + n * CH + m] = o;
      __syncthreads();
    }
  }
}

// T (complex64, node v at node_off[v], [a][b][c][s]) -> Tb (bf16, node v at
// v * NODE_BF16, [s][re|im][a][b][c]).
__global__ void pack_bf16_planes_kernel(dqz_graph_t g, const float2 *__restrict__ T, __nv_bfloat16 *Tb) {
  const int per = CH * CH * CH;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)g.n_nodes * per;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(i / per), x = (int)(i % per);
    const float2 *t = T + g.node_off[v] + 2 * x;
    __nv_bfloat16 *o = Tb + (size_t)v * NODE_BF16 + x;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const float2 val = t[s];
      o[(s * 2 + 0) * per] = __float2bfloat16_rn(val.x);
      o[(s * 2 + 1) * per] = __float2bfloat16_rn(val.y);
    }
  }
}

}  // namespace

extern "C" int dqz_pack_bf16_planes(const dqz_graph_t *g, const void *tensors_c64, void *tensors_bf16,
                                    cudaStream_t stream) {
  if (!g || !tensors_c64 || !tensors_bf16) return DQZ_ERR_ARG;
  if (g->n_nodes == 0) return DQZ_OK;
  pack_bf16_planes_kernel<<<148 * 8, 256, 0, stream>>>(*g, (const float2 *)tensors_c64,
                                                       (__nv_bfloat16 *)tensors_bf16);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_bp_node_update_k3_tc(const dqz_graph_t *g, const void *tensors_bf16, const void *n2e_old,
                                        const void *e2n_old, void *n2e_new, const uint8_t *src_sel,
                                        const int32_t *nodes, int32_t n_nodes, int32_t *error_flag,
                                        cudaStream_t stream) {
  if (!g || !tensors_bf16 || !n2e_old || !e2n_old || !n2e_new || !src_sel || !nodes || !error_flag || n_nodes < 0)
    return DQZ_ERR_ARG;
  if (n_nodes == 0) return DQZ_OK;
  const size_t smem = sizeof(TcSmem);
  DQZ_SMEM_ATTR_ONCE(bp_node_k3_tc, smem);
  bp_node_k3_tc<<<n_nodes, TC_THREADS, smem, stream>>>(*g, (const __nv_bfloat16 *)tensors_bf16,
                                                       (const float2 *)n2e_old, (const float2 *)e2n_old,
                                                       (float2 *)n2e_new, src_sel, nodes, n_nodes, error_flag);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
