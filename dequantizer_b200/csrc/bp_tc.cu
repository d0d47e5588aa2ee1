// BP node update on tensor cores: BF16 operands, FP32 accumulation, for
// degree-3 nodes with bonds of dimension 16 and physical dimension 2, on
// complex64 node tensors and messages (the mixed-precision form of
// tensor_ops.py:36-60; selected by dqz_bp_node_update_k3 with precision 16).
//
// One CTA (8 warps) owns one half-edge h = (v, e); f < g are the other two
// bonds. For each physical index s the slice T_s is staged in shared memory
// as BF16 real / imaginary planes in two layouts, and
//   MP1: Y1[(e,g)][f'] = sum_f T[(e,g)][f] m_f[f'][f]      (256 x 16 x 16)
//   MP2: Y2[(e,f')][g'] = sum_g Y1[(e,f')][g] m_g[g'][g]   (256 x 16 x 16)
//   FIN: out[a][a'] += sum_x Y2[a][x] conj(T[a'][x])        (16 x 16 x 256)
// run as mma.sync.m16n8k16 BF16 tiles; a complex product is four real ones
// (re*re - im*im, re*im + im*re) on the planes, the minus sign applied by
// flipping BF16 sign bits in the operand registers. Fragments are loaded
// with ldmatrix from K-contiguous rows padded to avoid bank conflicts.
// The final contraction splits K over the warps; partials are summed in a
// fixed order. The message is divided by its trace and stored as complex64.
#include <cuda_bf16.h>

#include "common.cuh"

namespace {

constexpr int CH = 16;
constexpr int LD1 = 24;   // bf16 row stride of K = 16 rows (48 B)
constexpr int LD4 = 264;  // bf16 row stride of K = 256 rows (528 B)
constexpr int TC_THREADS = 256;

struct __align__(16) TcSmem {
  __nv_bfloat16 T1r[256 * LD1], T1i[256 * LD1];  // rows (e,g), k = f
  __nv_bfloat16 Y1r[256 * LD1], Y1i[256 * LD1];  // rows (e,f'), k = g
  __nv_bfloat16 T4r[16 * LD4], T4i[16 * LD4];    // rows e, k = f*16 + g
  __nv_bfloat16 Y2r[16 * LD4], Y2i[16 * LD4];    // rows e, k = f'*16 + g'
  __nv_bfloat16 Mfr[16 * LD1], Mfi[16 * LD1], Mgr[16 * LD1], Mgi[16 * LD1];  // rows n, k
  float part[8][2][2][32][4];  // [warp][n-tile][re,im][lane][reg]
  float redw[8][2];
  float red[2];
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragment of the 16 x 16 tile at (row0, k0) of a K-contiguous matrix.
__device__ __forceinline__ void load_a(const __nv_bfloat16 *M, int ld, int row0, int k0, uint32_t (&a)[4]) {
  const int lane = threadIdx.x & 31, j = lane >> 3;
  const __nv_bfloat16 *p = M + (row0 + (j & 1) * 8 + (lane & 7)) * ld + k0 + (j >> 1) * 8;
  ldsm_x4(smem_addr(p), a[0], a[1], a[2], a[3]);
}

// B fragments of two n-tiles (rows n0..n0+15) at k0 of a K-contiguous
// matrix stored by rows n: b[nt][0..1].
__device__ __forceinline__ void load_b2(const __nv_bfloat16 *M, int ld, int n0, int k0, uint32_t (&b)[2][2]) {
  const int lane = threadIdx.x & 31, j = lane >> 3;
  const __nv_bfloat16 *p = M + (n0 + (j >> 1) * 8 + (lane & 7)) * ld + k0 + (j & 1) * 8;
  ldsm_x4(smem_addr(p), b[0][0], b[0][1], b[1][0], b[1][1]);
}

__device__ __forceinline__ void neg4(const uint32_t (&a)[4], uint32_t (&o)[4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = a[i] ^ 0x80008000u;
}

// D (16 x 16 complex, two n-tiles, re/im) = A (16 x 16, planes ar/ai) * B
// where B(k, n) = M[n][k] (planes mr/mi):
//   Dr += Ar Br - Ai Bi,  Di += Ar Bi + Ai Br.
__device__ __forceinline__ void cmma_tile(const uint32_t (&ar)[4], const uint32_t (&ai)[4], const uint32_t (&br)[2][2],
                                          const uint32_t (&bi)[2][2], float (&dr)[2][4], float (&di)[2][4]) {
  uint32_t nai[4];
  neg4(ai, nai);
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    mma_bf16(dr[nt], ar, br[nt][0], br[nt][1]);
    mma_bf16(dr[nt], nai, bi[nt][0], bi[nt][1]);
    mma_bf16(di[nt], ar, bi[nt][0], bi[nt][1]);
    mma_bf16(di[nt], ai, br[nt][0], br[nt][1]);
  }
}

__device__ __forceinline__ const float2 *msg_c64(const dqz_graph_t &g, int hf, const float2 *n2e_old,
                                                 const float2 *e2n_old, const float2 *n2e_new,
                                                 const uint8_t *src_sel) {
  const int sel = src_sel[hf];
  if (sel == DQZ_SRC_E2N_OLD) return e2n_old + g.half_msg_off[hf];
  return (sel == DQZ_SRC_N2E_NEW ? n2e_new : n2e_old) + g.half_msg_off[g.half_twin[hf]];
}

__global__ void __launch_bounds__(TC_THREADS) bp_node_k3_bf16(dqz_graph_t g, const float2 *__restrict__ T,
                                                               const float2 *n2e_old, const float2 *e2n_old,
                                                               float2 *n2e_new, const uint8_t *__restrict__ src_sel,
                                                               const int32_t *__restrict__ halves, int n_halves,
                                                               int *error_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TcSmem &S = *reinterpret_cast<TcSmem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;

  for (int item = blockIdx.x; item < n_halves; item += gridDim.x) {
    const int h = halves[item];
    const int v = g.half_node[h];
    const int h0 = g.node_half[v];
    const int e = h - h0;
    bool ok = g.node_degree[v] == 3 && g.node_phys[v] == 2;
    for (int q = 0; q < 3 && ok; ++q) ok = g.edge_chi[g.half_edge[h0 + q]] == CH;
    if (!ok) {
      if (tid == 0) atomicExch(error_flag, 1);
      continue;
    }
    const int f = e == 0 ? 1 : 0, gb = e == 2 ? 1 : 2;
    const float2 *mf = msg_c64(g, h0 + f, n2e_old, e2n_old, n2e_new, src_sel);
    const float2 *mg = msg_c64(g, h0 + gb, n2e_old, e2n_old, n2e_new, src_sel);
    {
      const int n = tid >> 4, k = tid & 15;  // 256 threads <-> 16 x 16 entries
      const float2 a = mf[n * CH + k], b = mg[n * CH + k];
      S.Mfr[n * LD1 + k] = __float2bfloat16_rn(a.x);
      S.Mfi[n * LD1 + k] = __float2bfloat16_rn(a.y);
      S.Mgr[n * LD1 + k] = __float2bfloat16_rn(b.x);
      S.Mgi[n * LD1 + k] = __float2bfloat16_rn(b.y);
    }
    const float2 *Tv = T + g.node_off[v];
    float acc_re = 0.f, acc_im = 0.f;  // out[a][a'] with a = tid >> 4, a' = tid & 15

    for (int s = 0; s < 2; ++s) {
      // ---- stage T_s in both layouts
      for (int x = tid; x < CH * CH * CH; x += TC_THREADS) {
        const int idx[3] = {x >> 8, (x >> 4) & 15, x & 15};
        const float2 t = Tv[2 * x + s];
        const int ie = idx[e], jf = idx[f], jg = idx[gb];
        const __nv_bfloat16 tr = __float2bfloat16_rn(t.x), ti = __float2bfloat16_rn(t.y);
        S.T1r[(ie * CH + jg) * LD1 + jf] = tr;
        S.T1i[(ie * CH + jg) * LD1 + jf] = ti;
        S.T4r[ie * LD4 + jf * CH + jg] = tr;
        S.T4i[ie * LD4 + jf * CH + jg] = ti;
      }
      __syncthreads();

      // ---- MP1: warp w owns m-tiles (= values of e) 2w, 2w+1
      {
        uint32_t br[2][2], bi[2][2];
        load_b2(S.Mfr, LD1, 0, 0, br);
        load_b2(S.Mfi, LD1, 0, 0, bi);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int mt = 2 * w + q;
          uint32_t ar[4], ai[4];
          load_a(S.T1r, LD1, mt * 16, 0, ar);
          load_a(S.T1i, LD1, mt * 16, 0, ai);
          float dr[2][4] = {}, di[2][4] = {};
          cmma_tile(ar, ai, br, bi, dr, di);
          // D1 element (row g-index r, col f') -> Y1[(mt*16 + f')][r]
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            const int fp = nt * 8 + 2 * tq;
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
              const int r = gq + 8 * hh;
              S.Y1r[(mt * CH + fp) * LD1 + r] = __float2bfloat16_rn(dr[nt][2 * hh]);
              S.Y1r[(mt * CH + fp + 1) * LD1 + r] = __float2bfloat16_rn(dr[nt][2 * hh + 1]);
              S.Y1i[(mt * CH + fp) * LD1 + r] = __float2bfloat16_rn(di[nt][2 * hh]);
              S.Y1i[(mt * CH + fp + 1) * LD1 + r] = __float2bfloat16_rn(di[nt][2 * hh + 1]);
            }
          }
        }
      }
      __syncthreads();

      // ---- MP2: rows (e, f'), k = g; output to Y2[e][f'*16 + g']
      {
        uint32_t br[2][2], bi[2][2];
        load_b2(S.Mgr, LD1, 0, 0, br);
        load_b2(S.Mgi, LD1, 0, 0, bi);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int mt = 2 * w + q;
          uint32_t ar[4], ai[4];
          load_a(S.Y1r, LD1, mt * 16, 0, ar);
          load_a(S.Y1i, LD1, mt * 16, 0, ai);
          float dr[2][4] = {}, di[2][4] = {};
          cmma_tile(ar, ai, br, bi, dr, di);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            const int gp = nt * 8 + 2 * tq;
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
              const int fp = gq + 8 * hh;
              __nv_bfloat162 vr = __floats2bfloat162_rn(dr[nt][2 * hh], dr[nt][2 * hh + 1]);
              __nv_bfloat162 vi = __floats2bfloat162_rn(di[nt][2 * hh], di[nt][2 * hh + 1]);
              *reinterpret_cast<__nv_bfloat162 *>(&S.Y2r[mt * LD4 + fp * CH + gp]) = vr;
              *reinterpret_cast<__nv_bfloat162 *>(&S.Y2i[mt * LD4 + fp * CH + gp]) = vi;
            }
          }
        }
      }
      __syncthreads();

      // ---- FIN: D[a][a'] = sum_x Y2[a][x] conj(T4[a'][x]); warp w owns k-steps 2w, 2w+1
      {
        float dr[2][4] = {}, di[2][4] = {};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int k0 = (2 * w + q) * 16;
          uint32_t yr[4], yi[4], nyr[4], br[2][2], bi[2][2];
          load_a(S.Y2r, LD4, 0, k0, yr);
          load_a(S.Y2i, LD4, 0, k0, yi);
          load_b2(S.T4r, LD4, 0, k0, br);
          load_b2(S.T4i, LD4, 0, k0, bi);
          neg4(yr, nyr);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            mma_bf16(dr[nt], yr, br[nt][0], br[nt][1]);   // Yr Tr
            mma_bf16(dr[nt], yi, bi[nt][0], bi[nt][1]);   // + Yi Ti
            mma_bf16(di[nt], yi, br[nt][0], br[nt][1]);   // Yi Tr
            mma_bf16(di[nt], nyr, bi[nt][0], bi[nt][1]);  // - Yr Ti
          }
        }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            S.part[w][nt][0][lane][r] = dr[nt][r];
            S.part[w][nt][1][lane][r] = di[nt][r];
          }
      }
      __syncthreads();
      {
        // thread <-> (a, a'): fragment position of D[a][a']
        const int a = tid >> 4, ap = tid & 15;
        const int nt = ap >> 3, col = ap & 7;
        const int src_lane = ((a & 7) << 2) | (col >> 1);
        const int reg = ((a >> 3) << 1) | (col & 1);
        float sr = 0.f, si = 0.f;
#pragma unroll
        for (int ww = 0; ww < 8; ++ww) {
          sr += S.part[ww][nt][0][src_lane][reg];
          si += S.part[ww][nt][1][src_lane][reg];
        }
        acc_re += sr;
        acc_im += si;
      }
      __syncthreads();
    }

    // ---- trace and store: message[a'][a] = out[a][a'] / trace
    const int a = tid >> 4, ap = tid & 15;
    float tre = (a == ap) ? acc_re : 0.f, tim = (a == ap) ? acc_im : 0.f;
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
    o.x = (acc_re * tr + acc_im * ti) / den;
    o.y = (acc_im * tr - acc_re * ti) / den;
    n2e_new[g.half_msg_off[h] + ap * CH + a] = o;
    __syncthreads();
  }
}

}  // namespace

// Launched from dqz_bp_node_update_k3 (bp_fast.cu) for precision 16.
int dqz_launch_k3_bf16(const dqz_graph_t *g, const void *T, const void *n2e_old, const void *e2n_old, void *n2e_new,
                       const uint8_t *src_sel, const int32_t *halves, int n_halves, int *error_flag,
                       cudaStream_t stream) {
  const size_t smem = sizeof(TcSmem);
  if (cudaFuncSetAttribute(bp_node_k3_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return DQZ_ERR_CUDA;
  bp_node_k3_bf16<<<n_halves, TC_THREADS, smem, stream>>>(*g, (const float2 *)T, (const float2 *)n2e_old,
                                                           (const float2 *)e2n_old, (float2 *)n2e_new, src_sel,
                                                           halves, n_halves, error_flag);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
