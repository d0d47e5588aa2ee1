// BP node update on the 5th-generation tensor cores (tcgen05, accumulators in
// tensor memory) for degree-3 nodes with bonds of dimension 16 and physical
// dimension 2: BF16 operands, FP32 accumulation, complex64 messages (the mixed
// form of tensor_ops.py:36-60, pass_through_node, on random 3-regular graphs).
//
// One CTA (8 warps) owns one node at a time and produces its three outgoing
// messages. With x_f contracting bond f of T with a message's second index and
// a, b, c the three bonds, each physical slice T_s goes through
//   stage 1 (tcgen05):  X  = T x_0 m0          rows (c, b), k = a
//                       X" = T x_2 m2          rows (a, b), k = c
//   stage 2 (tcgen05):  Y1 = X  x_2 m2         rows (b, a'), k = c
//                       Y2 = X  x_1 m1         rows (c, a'), k = b
//                       Y0 = X" x_1 m1         rows (a, c'), k = b
//   final (mma.sync):   out_1[b][b"] += sum_{a',c'} Y1[b][a'][c'] conj(T[a'][b"][c'])
//                       out_2[c][c"] += sum_{a',b'} Y2[c][a'][b'] conj(T[a'][b'][c"])
//                       out_0[a][a"] += sum_{c',b'} Y0[a][c'][b'] conj(T[a"][b'][c'])
// and the message n2e[v, e][n][m] = out_e[m][n] / trace(out_e).
//
// Every mode product is an M = 256 GEMM with N = 16 complex, issued as two
// 128-row tiles of two `tcgen05.mma.kind::f16` each (M128 N32 K16): the real
// plane of the operand against [Re m^T | Im m^T] and the imaginary plane
// against [-Im m^T | Re m^T], so the 32 accumulator columns hold Re | Im of
// the product. Operands sit in shared memory as 8 x 8 "core matrices" (eight
// 16-byte rows) without swizzle, addressed by UMMA shared-memory descriptors;
// the node tensor is kept in HBM in the two core layouts the descriptors and
// the final ldmatrix loads need. Each layout of a slice is one 16 KB
// `cp.async.bulk` completing on an mbarrier, issued a slice or a node ahead
// into three buffers (L1 of the slice in use, L2 of slices 0 and 1), so the
// copies land while the tensor cores work. The next node's metadata chain
// (node -> half-edges -> message offsets) is walked one dependent load per
// tensor-core wait by one thread, and its messages are loaded during the
// final products into a second operand buffer. Accumulators are read back with
// `tcgen05.ld`, rounded to BF16 and stored straight into the next stage's
// operand layout (paddings keep those stores free of bank conflicts). The
// final contractions have M = 16 (a 16 x 16 result over K = 256), too narrow
// for a tcgen05 tile, and run as warp-level m16n8k16 products on the same
// shared-memory cores.
//
// Every wait is bounded: on a timeout the kernel sets *error_flag to 2, waits
// (bounded) for the copies it issued, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "mma_bf16.cuh"

namespace {

constexpr int UM_THREADS = 256;
constexpr int PLANE = 4096;                 // BF16 elements of one 16^3 plane
constexpr int S_ELEMS = 4 * PLANE;          // one slice: L1 re, L1 im, L2 re, L2 im
constexpr int NODE_ELEMS = 2 * S_ELEMS;     // one node in HBM
constexpr uint32_t S_BYTES = S_ELEMS * 2;   // 32 KB per bulk copy
constexpr uint32_t TMEM_COLS = 256;

// Node-tensor core layouts (element offsets within a plane):
//   L1: core (c, a_hi, b_hi) = [a_lo rows][b_lo contiguous]
//   L2: core (a, b_hi, c_hi) = [b_lo rows][c_lo contiguous]
__host__ __device__ __forceinline__ int off_l1(int a, int b, int c) {
  return ((c * 2 + (a >> 3)) * 2 + (b >> 3)) * 64 + (a & 7) * 8 + (b & 7);
}
__host__ __device__ __forceinline__ int off_l2(int a, int b, int c) {
  return ((a * 2 + (b >> 3)) * 2 + (c >> 3)) * 64 + (b & 7) * 8 + (c & 7);
}

// Stage-1 outputs (operands of stage 2), per plane:
//   XS  (X for Y1, k = c): core rows c_lo, a'_lo contiguous; group (b_hi, a'_hi, b_lo)
//       every 72 elements (144 B), c_hi every XS_L elements
//   XS2 (X for Y2, k = b): core rows b_lo, a'_lo contiguous; group (c, a'_hi) every 64, b_hi every 2048
//   XP  (X" for Y0, k = b): core rows b_lo, c'_lo contiguous; group (a, c'_hi) every 64, b_hi every 2048
constexpr int XS_SBO = 72;
constexpr int XS_L = 32 * XS_SBO;
constexpr int XS_PLANE = 2 * XS_L;
constexpr int XS2_PLANE = PLANE;
constexpr int XP_PLANE = PLANE;
constexpr int X_ELEMS = 2 * (XS_PLANE + XS2_PLANE + XP_PLANE);
// Stage-2 outputs (A operands of the final products): per K-step (a' or c')
// a block of four cores [m_lo rows][k_lo contiguous], blocks every Y_AS
// elements (528 B: rows of consecutive K-steps fall in different banks).
constexpr int Y_AS = 264;
constexpr int Y_PLANE = 16 * Y_AS;
constexpr int Y_ELEMS = 6 * Y_PLANE;
constexpr int PART_FLOATS = 3 * 2 * 8 * 256;  // final partials: (output, re|im, warp, fragment position)
constexpr int XY_BYTES = X_ELEMS * 2;
static_assert(Y_ELEMS * 2 <= XY_BYTES && PART_FLOATS * 4 <= XY_BYTES, "aliases fit the X region");

// Metadata of a node, filled for the next node one dependent level at a time
// while the current node waits on the tensor cores, then read by all threads.
struct NodeMeta {
  int v, ok;
  int off[3];   // half_msg_off of the node's half-edges (where its messages go)
  int src[3];   // source arena of each incoming message: 0 e2n_old, 1 n2e_old, 2 n2e_new
  int moff[3];  // element offset of each incoming message in that arena
};
struct MetaChain {  // intermediate levels of the next node's metadata
  int v, vn, h0, deg, phys;  // vn: the node after it
  int he[3], sel[3], hoff[3], tw[3];
};

struct __align__(128) UmSmem {
  __nv_bfloat16 L1[2 * PLANE];     // L1 re | im of the slice in use (bulk-copy destination)
  __nv_bfloat16 L2[2][2 * PLANE];  // L2 re | im of slice 0 and of slice 1
  __nv_bfloat16 XY[X_ELEMS];       // stage-1 outputs, then stage-2 outputs, then partials
  __nv_bfloat16 B[2][3][2][512];   // [node parity][bond]: [Re m^T | Im m^T], [-Im m^T | Re m^T], K-major
  unsigned long long bar_a, bar_b[2], bar_m;
  uint32_t tmem;
  NodeMeta meta[2];
  MetaChain chain;
  float redw[8][6];
};

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint64_t sdesc(const void *p, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  // UMMA shared-memory descriptor, no swizzle: start >> 4 in [0,14), leading
  // byte offset >> 4 in [16,30), stride byte offset >> 4 in [32,46), version 1 at 46.
  const uint32_t a = saddr(p);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, B K-major,
// A K-major or MN-major, N = 32, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(bool a_mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((32u >> 3) << 17) |
         ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred P1;\nmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n"
        "selp.b32 %0, 1, 0, P1;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (the ld and its wait
// in one statement, so no use of the registers can move above the wait).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Eight FP32 values -> eight BF16 in one 16-byte shared store.
__device__ __forceinline__ void st_bf16x8(__nv_bfloat16 *dst, const float *v) {
  uint4 u;
  __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]);
  __nv_bfloat162 h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
  u.x = *reinterpret_cast<uint32_t *>(&h0);
  u.y = *reinterpret_cast<uint32_t *>(&h1);
  u.z = *reinterpret_cast<uint32_t *>(&h2);
  u.w = *reinterpret_cast<uint32_t *>(&h3);
  *reinterpret_cast<uint4 *>(dst) = u;
}

// Writes the Re (v[0..15]) and Im (v[16..31]) halves of one accumulator row as
// two 8-element chunks per plane at re + off_k(k_hi), im + off_k(k_hi).
template <typename Off>
__device__ __forceinline__ void store_row(__nv_bfloat16 *re, __nv_bfloat16 *im, const float (&v)[32], Off off) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    st_bf16x8(re + off(h), v + 8 * h);
    st_bf16x8(im + off(h), v + 16 + 8 * h);
  }
}

// ldmatrix address of lane `lane` for a 16 x 16 fragment made of four cores:
// core(i) = base of the 8 x 8 core for matrix index i = lane / 8.
template <typename Core>
__device__ __forceinline__ uint32_t frag_addr(const __nv_bfloat16 *base, Core core) {
  const int lane = threadIdx.x & 31;
  return saddr(base + core(lane >> 3) + (lane & 7) * 8);
}

__global__ void __launch_bounds__(UM_THREADS, 2)
    bp_node_k3_umma(dqz_graph_t g, const __nv_bfloat16 *__restrict__ Tu, const float2 *n2e_old, const float2 *e2n_old,
                    float2 *n2e_new, const uint8_t *__restrict__ src_sel, const int32_t *__restrict__ nodes,
                    int n_nodes, int *error_flag) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  UmSmem &S = *reinterpret_cast<UmSmem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, wq = w & 3;
  const uint32_t bar_a = saddr(&S.bar_a), bar_m = saddr(&S.bar_m);
  const uint32_t bar_b0 = saddr(&S.bar_b[0]), bar_b1 = saddr(&S.bar_b[1]);

  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_b0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_b1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_m) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&S.tmem)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t tl = tmem + ((uint32_t)(32 * wq) << 16);  // this warp's TMEM lanes
  // mbarrier phases and copies in flight (identical in every thread)
  uint32_t ph_a = 0, ph_b0 = 0, ph_b1 = 0, ph_m = 0;
  int pend_a = 0, pend_b0 = 0, pend_b1 = 0;

  __nv_bfloat16 *L1r = S.L1, *L1i = S.L1 + PLANE;
  __nv_bfloat16 *XSr = S.XY, *XSi = XSr + XS_PLANE;
  __nv_bfloat16 *XS2r = XSi + XS_PLANE, *XS2i = XS2r + XS2_PLANE;
  __nv_bfloat16 *XPr = XS2i + XS2_PLANE, *XPi = XPr + XP_PLANE;
  __nv_bfloat16 *Y1r = S.XY, *Y1i = Y1r + Y_PLANE, *Y2r = Y1i + Y_PLANE, *Y2i = Y2r + Y_PLANE;
  __nv_bfloat16 *Y0r = Y2i + Y_PLANE, *Y0i = Y0r + Y_PLANE;
  float *part = reinterpret_cast<float *>(S.XY);
  constexpr uint32_t ID_MN = idesc_bf16(true), ID_K = idesc_bf16(false);

  // ---- helpers (block-uniform control flow)
  auto copy_l1 = [&](int v, int s) {  // L1 part of slice s of node v -> S.L1
    if (tid == 0) {
      fence_async_smem();
      bulk_load(saddr(S.L1), Tu + (size_t)v * NODE_ELEMS + s * S_ELEMS, S_BYTES / 2, bar_a);
    }
    pend_a = 1;
  };
  auto copy_l2 = [&](int v, int s) {  // L2 part of slice s of node v -> S.L2[s]
    if (tid == 0) {
      fence_async_smem();
      bulk_load(saddr(S.L2[s]), Tu + (size_t)v * NODE_ELEMS + s * S_ELEMS + 2 * PLANE, S_BYTES / 2,
                s ? bar_b1 : bar_b0);
    }
    if (s) pend_b1 = 1;
    else pend_b0 = 1;
  };
  // chain levels of the next node's metadata, one thread
  auto level_v = [&](int it) { S.chain.v = nodes[it]; };
  auto level_node = [&]() {
    const int v = S.chain.v;
    S.chain.h0 = g.node_half[v];
    S.chain.deg = g.node_degree[v];
    S.chain.phys = g.node_phys[v];
  };
  auto level_halves = [&]() {
    if (S.chain.deg < 3) return;
    const int h0 = S.chain.h0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      S.chain.he[q] = g.half_edge[h0 + q];
      S.chain.sel[q] = src_sel[h0 + q];
      S.chain.hoff[q] = (int)g.half_msg_off[h0 + q];
      S.chain.tw[q] = g.half_twin[h0 + q];
    }
  };
  auto level_finish = [&](int buf) {
    NodeMeta &M = S.meta[buf];
    bool ok = S.chain.deg == 3 && S.chain.phys == 2;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int sel = S.chain.sel[q], tw = S.chain.tw[q];
      ok = ok && tw >= 0 && S.chain.he[q] >= 0 && g.edge_chi[S.chain.he[q]] == 16;
      M.off[q] = S.chain.hoff[q];
      M.src[q] = sel == DQZ_SRC_E2N_OLD ? 0 : (sel == DQZ_SRC_N2E_NEW ? 2 : 1);
      M.moff[q] = sel == DQZ_SRC_E2N_OLD ? S.chain.hoff[q] : (ok ? (int)g.half_msg_off[tw] : 0);
    }
    M.v = S.chain.v;
    M.ok = ok;
  };
  // this thread's element (n, k) = (tid >> 4, tid & 15) of the three incoming messages
  auto load_msgs = [&](int buf, float2 (&x)[3]) {
    const NodeMeta &M = S.meta[buf];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float2 *base = M.src[q] == 0 ? e2n_old : (M.src[q] == 2 ? n2e_new : n2e_old);
      x[q] = M.ok ? base[M.moff[q] + tid] : make_float2(0.f, 0.f);
    }
  };
  auto store_msgs = [&](int buf, const float2 (&x)[3]) {
    const int n = tid >> 4, k = tid & 15;
    const int o_lo = ((n >> 3) * 2 + (k >> 3)) * 64 + (n & 7) * 8 + (k & 7);
    const int o_hi = (((n + 16) >> 3) * 2 + (k >> 3)) * 64 + (n & 7) * 8 + (k & 7);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      S.B[buf][q][0][o_lo] = __float2bfloat16_rn(x[q].x);
      S.B[buf][q][0][o_hi] = __float2bfloat16_rn(x[q].y);
      S.B[buf][q][1][o_lo] = __float2bfloat16_rn(-x[q].y);
      S.B[buf][q][1][o_hi] = __float2bfloat16_rn(x[q].x);
    }
    fence_async_smem();
  };
  // everything for node index `it` at once (first node of the CTA, and after a skipped node)
  auto prepare_blocking = [&](int it, int buf) {
    if (tid == 32) {
      level_v(it);
      level_node();
      level_halves();
      level_finish(buf);
      S.chain.vn = it + (int)gridDim.x < n_nodes ? nodes[it + gridDim.x] : 0;
    }
    __syncthreads();
    float2 x[3];
    load_msgs(buf, x);
    store_msgs(buf, x);
    const int v = S.meta[buf].v;
    copy_l1(v, 0);
    copy_l2(v, 0);
    copy_l2(v, 1);
  };
  auto wait_bar = [&](uint32_t bar, uint32_t &ph) -> bool {
    const bool good = mbar_wait(bar, ph);
    ph ^= 1;
    return good;
  };

  int cur = 0;
  if (blockIdx.x < n_nodes) prepare_blocking(blockIdx.x, 0);

  for (int item = blockIdx.x; item < n_nodes; item += gridDim.x) {
    const int next = item + gridDim.x;
    const bool has_next = next < n_nodes;
    if (tid == 32) S.chain.v = S.chain.vn;
    __syncthreads();
    const int v = S.meta[cur].v;
    if (!S.meta[cur].ok) {  // unsupported shape: drop its copies, prepare the next node
      if (tid == 0) atomicExch(error_flag, 1);
      bool good = wait_bar(bar_a, ph_a) & wait_bar(bar_b0, ph_b0) & wait_bar(bar_b1, ph_b1);
      if (__syncthreads_or(!good)) goto fail;
      pend_a = pend_b0 = pend_b1 = 0;
      if (has_next) prepare_blocking(next, cur ^ 1);
      cur ^= 1;
      continue;
    }
    float fr[3][2][4] = {}, fi[3][2][4] = {};  // this warp's partial final products
    float2 xn[3];                               // next node's message elements

    for (int s = 0; s < 2; ++s) {
      {
        bool good = wait_bar(bar_a, ph_a);
        good &= s ? wait_bar(bar_b1, ph_b1) : wait_bar(bar_b0, ph_b0);
        if (__syncthreads_or(!good)) goto fail;
        pend_a = 0;
        if (s) pend_b1 = 0;
        else pend_b0 = 0;
      }
      __nv_bfloat16 *L2r = S.L2[s], *L2i = S.L2[s] + PLANE;
      const __nv_bfloat16(*Bm)[2][512] = S.B[cur];

      // ---- stage 1: X = T x_0 m0 (TMEM cols 0..63), X" = T x_2 m2 (cols 64..127)
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          // A = L1 MN-major: rows (c, b_lo) for b_hi = t, k = a; SBO 512 B (c), LBO 256 B (a_hi)
          umma(tmem + 32 * t, sdesc(L1r + 64 * t, 256, 512), sdesc(Bm[0][0], 128, 256), ID_MN, 0);
          umma(tmem + 32 * t, sdesc(L1i + 64 * t, 256, 512), sdesc(Bm[0][1], 128, 256), ID_MN, 1);
          // A = L2 K-major: rows (a, b) for a_hi = t, k = c; SBO 256 B (a, b_hi), LBO 128 B (c_hi)
          umma(tmem + 64 + 32 * t, sdesc(L2r + 2048 * t, 128, 256), sdesc(Bm[2][0], 128, 256), ID_K, 0);
          umma(tmem + 64 + 32 * t, sdesc(L2i + 2048 * t, 128, 256), sdesc(Bm[2][1], 128, 256), ID_K, 1);
        }
        umma_commit(bar_m);
      }
      if (tid == 32 && has_next) {  // next node's metadata while the tensor cores run
        if (s == 0) level_node();
        else level_finish(cur ^ 1);
      }
      {
        const bool good = wait_bar(bar_m, ph_m);
        if (__syncthreads_or(!good)) goto fail;
      }
      tc_fence_after();
      {
        const int m = 32 * wq + lane;
        float val[32];
        if (w < 4) {
#pragma unroll
          for (int t = 0; t < 2; ++t) {  // X tile t: row m = c*8 + b_lo, b = 8t + b_lo
            tmem_ld32(tl + 32 * t, val);
            const int c = m >> 3, bl = m & 7;
            store_row(XSr, XSi, val, [&](int ah) {
              return (c >> 3) * XS_L + ((t * 2 + ah) * 8 + bl) * XS_SBO + (c & 7) * 8;
            });
            store_row(XS2r, XS2i, val, [&](int ah) { return t * 2048 + (c * 2 + ah) * 64 + bl * 8; });
          }
        } else {
#pragma unroll
          for (int t = 0; t < 2; ++t) {  // X" tile t: row m = (a - 8t)*16 + b
            tmem_ld32(tl + 64 + 32 * t, val);
            const int a = 8 * t + (m >> 4), b = m & 15;
            store_row(XPr, XPi, val, [&](int ch) { return (b >> 3) * 2048 + (a * 2 + ch) * 64 + (b & 7) * 8; });
          }
        }
      }
      fence_async_smem();
      tc_fence_before();
      __syncthreads();

      // ---- stage 2: Y1 = X x_2 m2 (cols 128..191), Y2 = X x_1 m1 (192..255), Y0 = X" x_1 m1 (0..63)
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          // XS MN-major: tile b_hi = t, groups (a'_hi, b_lo) every 144 B, k = c (c_hi every XS_L)
          umma(tmem + 128 + 32 * t, sdesc(XSr + t * 16 * XS_SBO, XS_L * 2, XS_SBO * 2), sdesc(Bm[2][0], 128, 256),
               ID_MN, 0);
          umma(tmem + 128 + 32 * t, sdesc(XSi + t * 16 * XS_SBO, XS_L * 2, XS_SBO * 2), sdesc(Bm[2][1], 128, 256),
               ID_MN, 1);
          // XS2 MN-major: tile c_hi = t, groups (c_lo, a'_hi) every 128 B, k = b (b_hi every 4096 B)
          umma(tmem + 192 + 32 * t, sdesc(XS2r + 1024 * t, 4096, 128), sdesc(Bm[1][0], 128, 256), ID_MN, 0);
          umma(tmem + 192 + 32 * t, sdesc(XS2i + 1024 * t, 4096, 128), sdesc(Bm[1][1], 128, 256), ID_MN, 1);
          // XP MN-major: tile a_hi = t, groups (a_lo, c'_hi) every 128 B, k = b (b_hi every 4096 B)
          umma(tmem + 32 * t, sdesc(XPr + 1024 * t, 4096, 128), sdesc(Bm[1][0], 128, 256), ID_MN, 0);
          umma(tmem + 32 * t, sdesc(XPi + 1024 * t, 4096, 128), sdesc(Bm[1][1], 128, 256), ID_MN, 1);
        }
        umma_commit(bar_m);
      }
      if (tid == 32 && has_next) {
        if (s == 0) level_halves();
        else if (next + (int)gridDim.x < n_nodes) S.chain.vn = nodes[next + gridDim.x];
      }
      {
        const bool good = wait_bar(bar_m, ph_m);
        if (__syncthreads_or(!good)) goto fail;
      }
      tc_fence_after();
      {
        const int m = 32 * wq + lane;
        float val[32];
        const int t0 = w < 4 ? 0 : 1;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          tmem_ld32(tl + (w < 4 ? 128 : 192) + 32 * t, val);
          if (w < 4) {  // Y1 tile b_hi = t: row m = (a'_hi*8 + b_lo)*8 + a'_lo
            const int ap = (m >> 6) * 8 + (m & 7), bl = (m >> 3) & 7;
            store_row(Y1r, Y1i, val, [&](int ch) { return ap * Y_AS + (t * 2 + ch) * 64 + bl * 8; });
          } else {  // Y2 tile c_hi = t: row m = c_lo*16 + a'
            const int ap = m & 15, cl = m >> 4;
            store_row(Y2r, Y2i, val, [&](int bh) { return ap * Y_AS + (t * 2 + bh) * 64 + cl * 8; });
          }
        }
        tmem_ld32(tl + 32 * t0, val);  // Y0 tile a_hi = t0: row m = a_lo*16 + c'
        const int cp = m & 15, al = m >> 4;
        store_row(Y0r, Y0i, val, [&](int bh) { return cp * Y_AS + (t0 * 2 + bh) * 64 + al * 8; });
      }
      tc_fence_before();
      __syncthreads();
      if (s == 1 && has_next) load_msgs(cur ^ 1, xn);  // lands while the final products run

      // ---- final products (mma.sync): warp w takes K-steps 2w, 2w+1 of each; out_0 first, as it is
      // the only reader of L1, which then takes the next slice
      auto ya = [&](int j, int i) { return j * Y_AS + ((i & 1) * 2 + (i >> 1)) * 64; };
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int j = 2 * w + q;
        uint32_t ar[4], ai[4], br[2][2], bi[2][2];
        // out_0: A = Y0 at K-step c' = j; B = T[a"][b'][c'] from L1 (rows a", b' contiguous)
        auto l1_rows = [&](int i) { return ((j * 2 + (i >> 1)) * 2 + (i & 1)) * 64; };
        auto yj = [&](int i) { return ya(j, i); };
        ldsm_x4(frag_addr(Y0r, yj), ar[0], ar[1], ar[2], ar[3]);
        ldsm_x4(frag_addr(Y0i, yj), ai[0], ai[1], ai[2], ai[3]);
        ldsm_x4(frag_addr(L1r, l1_rows), br[0][0], br[0][1], br[1][0], br[1][1]);
        ldsm_x4(frag_addr(L1i, l1_rows), bi[0][0], bi[0][1], bi[1][0], bi[1][1]);
        cmma_conjb(ar, ai, br, bi, fr[0], fi[0]);
      }
      __syncthreads();
      if (s == 0) copy_l1(v, 1);
      else if (has_next) copy_l1(S.chain.v, 0);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int j = 2 * w + q;
        uint32_t ar[4], ai[4], br[2][2], bi[2][2];
        auto yj = [&](int i) { return ya(j, i); };
        auto l2_rows = [&](int i) { return ((j * 2 + (i >> 1)) * 2 + (i & 1)) * 64; };
        auto l2_trans = [&](int i) { return ((j * 2 + (i & 1)) * 2 + (i >> 1)) * 64; };
        // out_1: A = Y1 at K-step a' = j; B = T[a'][b"][c'] from L2 (rows b", c' contiguous)
        ldsm_x4(frag_addr(Y1r, yj), ar[0], ar[1], ar[2], ar[3]);
        ldsm_x4(frag_addr(Y1i, yj), ai[0], ai[1], ai[2], ai[3]);
        ldsm_x4(frag_addr(L2r, l2_rows), br[0][0], br[0][1], br[1][0], br[1][1]);
        ldsm_x4(frag_addr(L2i, l2_rows), bi[0][0], bi[0][1], bi[1][0], bi[1][1]);
        cmma_conjb(ar, ai, br, bi, fr[1], fi[1]);
        // out_2: A = Y2 at K-step a' = j; B = T[a'][b'][c"] from L2 (rows b', c" contiguous: transposed load)
        ldsm_x4(frag_addr(Y2r, yj), ar[0], ar[1], ar[2], ar[3]);
        ldsm_x4(frag_addr(Y2i, yj), ai[0], ai[1], ai[2], ai[3]);
        ldsm_x4_t(frag_addr(L2r, l2_trans), br[0][0], br[0][1], br[1][0], br[1][1]);
        ldsm_x4_t(frag_addr(L2i, l2_trans), bi[0][0], bi[0][1], bi[1][0], bi[1][1]);
        cmma_conjb(ar, ai, br, bi, fr[2], fi[2]);
      }
      __syncthreads();
      if (has_next) copy_l2(S.chain.v, s);  // this slice's L2 buffer now takes the next node's
    }
    if (has_next) store_msgs(cur ^ 1, xn);

    // ---- reduce the warps' partials in a fixed order, normalise by the trace, store.
    // Partials are written and read in MMA-fragment order (position p = (nt, lane, r),
    // thread t sums position t over the 8 warps): both sides free of bank conflicts.
    // The normalised messages go through the (now idle) operand buffer of this node
    // so that each thread writes one consecutive element of each message.
#pragma unroll
    for (int e = 0; e < 3; ++e)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        *reinterpret_cast<float4 *>(&part[(((e * 2 + 0) * 8 + w) * 2 + nt) * 128 + lane * 4]) =
            make_float4(fr[e][nt][0], fr[e][nt][1], fr[e][nt][2], fr[e][nt][3]);
        *reinterpret_cast<float4 *>(&part[(((e * 2 + 1) * 8 + w) * 2 + nt) * 128 + lane * 4]) =
            make_float4(fi[e][nt][0], fi[e][nt][1], fi[e][nt][2], fi[e][nt][3]);
      }
    __syncthreads();
    {
      const int nt = tid >> 7, fl = (tid >> 2) & 31, r = tid & 3;  // fragment position of this thread
      const int m = (fl >> 2) + 8 * (r >> 1), n = nt * 8 + 2 * (fl & 3) + (r & 1);
      float are[3], aim[3], tq[6];
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        are[e] = aim[e] = 0.f;
#pragma unroll
        for (int ww = 0; ww < 8; ++ww) {
          are[e] += part[(((e * 2 + 0) * 8 + ww) * 2 + nt) * 128 + (tid & 127)];
          aim[e] += part[(((e * 2 + 1) * 8 + ww) * 2 + nt) * 128 + (tid & 127)];
        }
        tq[2 * e] = (m == n) ? are[e] : 0.f;
        tq[2 * e + 1] = (m == n) ? aim[e] : 0.f;
      }
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tq[i] += __shfl_xor_sync(0xffffffffu, tq[i], o);
      if (lane == 0)
#pragma unroll
        for (int i = 0; i < 6; ++i) S.redw[w][i] = tq[i];
      __syncthreads();
      float2 *out_s = reinterpret_cast<float2 *>(&S.B[cur][0][0][0]);  // 3 x 256 complex64
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        float tr = 0.f, ti = 0.f;
#pragma unroll
        for (int ww = 0; ww < 8; ++ww) {
          tr += S.redw[ww][2 * e];
          ti += S.redw[ww][2 * e + 1];
        }
        const float den = tr * tr + ti * ti;
        float2 o;
        o.x = (are[e] * tr + aim[e] * ti) / den;
        o.y = (aim[e] * tr - are[e] * ti) / den;
        out_s[e * 256 + n * 16 + (m ^ n)] = o;  // message[n][m] = out_e[m][n] / trace (columns XOR-swizzled)
      }
      __syncthreads();
#pragma unroll
      for (int e = 0; e < 3; ++e) n2e_new[S.meta[cur].off[e] + tid] = out_s[e * 256 + (tid ^ (tid >> 4))];
    }
    cur ^= 1;
  }
  goto done;

fail:
  if (tid == 0) {
    atomicExch(error_flag, 2);
    // let issued copies land before the CTA exits
    if (pend_a) mbar_wait(bar_a, ph_a);
    if (pend_b0) mbar_wait(bar_b0, ph_b0);
    if (pend_b1) mbar_wait(bar_b1, ph_b1);
  }

done:
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (w == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// T (complex64, node v at node_off[v], [a][b][c][s]) -> Tu (BF16, node v at
// v * NODE_ELEMS, [s][L1 re, L1 im, L2 re, L2 im][4096]).
__global__ void pack_bf16_umma_kernel(dqz_graph_t g, const float2 *__restrict__ T, __nv_bfloat16 *Tu, int first,
                                      int count) {
  const int per = 4096;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)count * per;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = first + (int)(i / per), x = (int)(i % per);
    const int a = x >> 8, b = (x >> 4) & 15, c = x & 15;
    const float2 *t = T + g.node_off[v] + 2 * x;
    const int o1 = off_l1(a, b, c), o2 = off_l2(a, b, c);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const float2 val = t[s];
      __nv_bfloat16 *o = Tu + (size_t)v * NODE_ELEMS + s * S_ELEMS;
      o[o1] = __float2bfloat16_rn(val.x);
      o[PLANE + o1] = __float2bfloat16_rn(val.y);
      o[2 * PLANE + o2] = __float2bfloat16_rn(val.x);
      o[3 * PLANE + o2] = __float2bfloat16_rn(val.y);
    }
  }
}

}  // namespace

extern "C" size_t dqz_bf16_umma_elems_per_node(void) { return NODE_ELEMS; }

extern "C" int dqz_pack_bf16_umma(const dqz_graph_t *g, const void *tensors_c64, void *tensors_bf16,
                                  cudaStream_t stream) {
  if (!g || !tensors_c64 || !tensors_bf16) return DQZ_ERR_ARG;
  if (((uintptr_t)tensors_bf16 & 15) != 0) return DQZ_ERR_ARG;
  if (g->n_nodes == 0) return DQZ_OK;
  pack_bf16_umma_kernel<<<148 * 8, 256, 0, stream>>>(*g, (const float2 *)tensors_c64, (__nv_bfloat16 *)tensors_bf16,
                                                     0, g->n_nodes);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_pack_bf16_umma_nodes(const dqz_graph_t *g, const void *tensors_c64, void *tensors_bf16,
                                        int32_t first, int32_t count, cudaStream_t stream) {
  if (!g || !tensors_c64 || !tensors_bf16 || first < 0 || count < 0 || first + count > g->n_nodes) return DQZ_ERR_ARG;
  if (((uintptr_t)tensors_bf16 & 15) != 0) return DQZ_ERR_ARG;
  if (count == 0) return DQZ_OK;
  const long long blocks = ((long long)count * 4096 + 255) / 256;
  const int grid = (int)(blocks < 148 * 8 ? blocks : 148 * 8);
  pack_bf16_umma_kernel<<<grid, 256, 0, stream>>>(*g, (const float2 *)tensors_c64, (__nv_bfloat16 *)tensors_bf16,
                                                  first, count);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_bp_node_update_k3_umma(const dqz_graph_t *g, const void *tensors_bf16, const void *n2e_old,
                                          const void *e2n_old, void *n2e_new, const uint8_t *src_sel,
                                          const int32_t *nodes, int32_t n_nodes, int32_t *error_flag,
                                          cudaStream_t stream) {
  if (!g || !tensors_bf16 || !n2e_old || !e2n_old || !n2e_new || !src_sel || !nodes || !error_flag || n_nodes < 0)
    return DQZ_ERR_ARG;
  if (((uintptr_t)tensors_bf16 & 15) != 0) return DQZ_ERR_ARG;  // bulk copies start on 16-byte boundaries
  if (n_nodes == 0) return DQZ_OK;
  const size_t smem = sizeof(UmSmem);
  DQZ_SMEM_ATTR_ONCE(bp_node_k3_umma, smem);
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DQZ_ERR_CUDA;
  static bool carveout_done[64] = {false};
  if (!carveout_done[dev]) {  // two CTAs of ~113 KB per SM need the whole shared-memory carveout
    if (cudaFuncSetAttribute(bp_node_k3_umma, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
      return DQZ_ERR_CUDA;
    carveout_done[dev] = true;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = n_nodes < 2 * sms ? n_nodes : 2 * sms;
  bp_node_k3_umma<<<grid, UM_THREADS, smem, stream>>>(*g, (const __nv_bfloat16 *)tensors_bf16,
                                                      (const float2 *)n2e_old, (const float2 *)e2n_old,
                                                      (float2 *)n2e_new, src_sel, nodes, n_nodes, error_flag);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
