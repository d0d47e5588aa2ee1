// Belief-propagation kernels (FP64 / complex128, generic shapes).
//
// Node update, replacing dequantizer/src/tensor_ops.py:36-60
// (pass_through_node) inside the sweep of mappings/belief_propagation.py:24-64.
// One CTA owns one half-edge h = (node v, bond e). It walks the bond-e slices
// T[.., a_e = a, ..] of the node tensor, contracts each slice with the k-1
// incoming messages (mode products in shared memory or CTA scratch), and
// accumulates column a of the outgoing message,
//     m_out[a', a] = sum_x conj(T_slice(a')[x]) Y_a[x],
// then divides by the trace.
//
// The incoming message of every bond is chosen per half-edge (src_sel), which
// reproduces the reference's synchronous sweep (all DQZ_SRC_E2N_OLD), its
// asynchronous sweep in traversal order (a mix, with nodes launched level by
// level) and a flooding schedule (all DQZ_SRC_N2E_OLD).
#include "common.cuh"

using namespace dqz;

namespace {

constexpr int BP_THREADS = 256;

__device__ __forceinline__ const cd *incoming_msg(const dqz_graph_t &g, int hf, const cd *n2e_old, const cd *e2n_old,
                                                  const cd *n2e_new, const uint8_t *src_sel) {
  int sel = src_sel[hf];
  if (sel == DQZ_SRC_E2N_OLD) return e2n_old + g.half_msg_off[hf];
  int tw = g.half_twin[hf];
  return (sel == DQZ_SRC_N2E_NEW ? n2e_new : n2e_old) + g.half_msg_off[tw];
}

// Column a of the unnormalised outgoing message of bond e of a node (tensor
// Tv, shape s): out[ap][a] = sum_x conj(T_slice(ap)[x]) Y_a[x], with Y_a the
// bond-e slice a contracted with the k-1 incoming messages; `put(ap, value)`
// stores each entry. bufA / bufB hold two slices. Whole CTA; ends with a barrier.
template <typename Put>
__device__ __forceinline__ void node_slice_column(const dqz_graph_t &g, const cd *__restrict__ Tv, const NodeShape &s,
                                                  int e, const cd *n2e_old, const cd *e2n_old, const cd *n2e_new,
                                                  const uint8_t *__restrict__ src_sel, int a, cd *bufA, cd *bufB,
                                                  Put put) {
  const int ce = s.dims[e];
  const long long Re = s.stride[e];
  const long long P = s.size / ce;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // P < 2^31 for every slice held on chip: the division by Re via FastDiv
  const bool small = P * ce < (1ll << 31);
  const FastDiv fRe((unsigned)(small ? Re : 1));
  if (small) {
    for (unsigned x = threadIdx.x; x < (unsigned)P; x += blockDim.x) {
      const unsigned l = fRe.div(x), r = x - l * (unsigned)Re;
      bufA[x] = Tv[(l * (unsigned)ce + (unsigned)a) * (unsigned)Re + r];
    }
  } else {
    for (long long x = threadIdx.x; x < P; x += blockDim.x) {
      long long l = x / Re, r = x - l * Re;
      bufA[x] = Tv[(l * ce + a) * Re + r];
    }
  }
  __syncthreads();
  cd *cur = bufA, *nxt = bufB;
  long long Lj = 1;
  for (int f = 0; f < s.k; ++f) {
    if (f == e) continue;
    const int q = s.dims[f];
    const long long R = P / Lj / q;
    const cd *m = incoming_msg(g, s.half0 + f, n2e_old, e2n_old, n2e_new, src_sel);
    mode_product<false>(cur, nxt, Lj, q, q, R, m, q, 1);
    __syncthreads();
    cd *t = cur;
    cur = nxt;
    nxt = t;
    Lj *= q;
  }
  for (int ap = warp; ap < ce; ap += nw) {
    cd acc = czero();
    if (small) {
      for (unsigned x = lane; x < (unsigned)P; x += 32) {
        const unsigned l = fRe.div(x), r = x - l * (unsigned)Re;
        cfmac(acc, Tv[(l * (unsigned)ce + (unsigned)ap) * (unsigned)Re + r], cur[x]);
      }
    } else {
      for (long long x = lane; x < P; x += 32) {
        long long l = x / Re, r = x - l * Re;
        cfmac(acc, Tv[(l * ce + ap) * Re + r], cur[x]);
      }
    }
    acc = warp_csum(acc);
    if (lane == 0) put(ap, acc);
  }
  __syncthreads();
}

// dst (ce x ce) /= its trace, the trace summed by one thread in index order.
// Whole CTA; src may equal dst.
__device__ __forceinline__ void normalise_by_trace(const cd *src, cd *dst, int ce, cd &trace_sh) {
  if (threadIdx.x == 0) {
    cd tr = czero();
    for (int i = 0; i < ce; ++i) tr = cadd(tr, src[i * ce + i]);
    trace_sh = tr;
  }
  __syncthreads();
  const cd tr = trace_sh;
  for (int i = threadIdx.x; i < ce * ce; i += blockDim.x) dst[i] = cdiv(src[i], tr);
  __syncthreads();
}

// n2e_new[h] for one half-edge h by the whole CTA (out: ce x ce, bufA / bufB:
// two slices, trace_sh: one shared complex). Ends with a barrier.
__device__ __forceinline__ void node_update_half(const dqz_graph_t &g, const cd *__restrict__ T, const cd *n2e_old,
                                                 const cd *e2n_old, cd *n2e_new, const uint8_t *__restrict__ src_sel,
                                                 int h, cd *out, cd *bufA, cd *bufB, cd &trace_sh) {
  const int v = g.half_node[h];
  NodeShape s;
  load_shape(g, v, s);
  const int e = h - s.half0;
  const int ce = s.dims[e];
  const cd *Tv = T + g.node_off[v];
  for (int a = 0; a < ce; ++a)
    node_slice_column(g, Tv, s, e, n2e_old, e2n_old, n2e_new, src_sel, a, bufA, bufB,
                      [&](int ap, cd val) { out[ap * ce + a] = val; });
  normalise_by_trace(out, n2e_new + g.half_msg_off[h], ce, trace_sh);
}

__global__ void __launch_bounds__(BP_THREADS) bp_node_generic(dqz_graph_t g, const cd *__restrict__ T,
                                                              const cd *n2e_old, const cd *e2n_old, cd *n2e_new,
                                                              const uint8_t *__restrict__ src_sel,
                                                              const int32_t *__restrict__ halves, int n_halves,
                                                              int max_slice, int max_chi, cd *scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd *out = reinterpret_cast<cd *>(smem_raw + 48 * sizeof(double));  // max_chi^2
  cd *bufA, *bufB;
  if (scratch) {
    bufA = scratch + (long long)blockIdx.x * 2 * max_slice;
  } else {
    bufA = out + (long long)max_chi * max_chi;
  }
  bufB = bufA + max_slice;
  __shared__ cd trace_sh;
  for (int item = blockIdx.x; item < n_halves; item += gridDim.x)
    node_update_half(g, T, n2e_old, e2n_old, n2e_new, src_sel, halves[item], out, bufA, bufB, trace_sh);
}

// ---- one warp per half-edge, for small nodes. The same elements in the same
// order as node_update_half (each mode-product output by one lane, the final
// column by the lanes' partial sums and warp_csum, the trace by one lane), so
// the messages are bit-identical; phases are separated by __syncwarp only.
__device__ __forceinline__ void warp_mode_product(const cd *__restrict__ X, cd *__restrict__ Y, unsigned L, int q,
                                                  unsigned R, const cd *__restrict__ m) {
  // plain 32-bit divisions: a lane runs a handful of outputs here (small
  // nodes), fewer than it takes to amortise a FastDiv set-up
  const unsigned total = L * (unsigned)q * R;
  for (unsigned o = threadIdx.x & 31; o < total; o += 32) {
    const unsigned t = o / R;
    const unsigned r = o - t * R;
    const unsigned l = t / (unsigned)q;
    const int i = (int)(t - l * (unsigned)q);
    const cd *x = X + (l * (unsigned)q) * R + r;
    cd acc = czero();
    for (int b = 0; b < q; ++b) cfma(acc, m[(long long)i * q + b], x[(long long)b * R]);
    Y[o] = acc;
  }
}

__device__ __forceinline__ void warp_node_update_half(const dqz_graph_t &g, const cd *__restrict__ T, const cd *n2e_old,
                                                      const cd *e2n_old, cd *n2e_new,
                                                      const uint8_t *__restrict__ src_sel, int h, cd *out, cd *bufA,
                                                      cd *bufB, cd *Ts, cd *Ms) {
  const int lane = threadIdx.x & 31;
  const int v = g.half_node[h];
  NodeShape s;
  load_shape(g, v, s);
  const int e = h - s.half0;
  const int ce = s.dims[e];
  const unsigned Re = (unsigned)s.stride[e];
  const unsigned P = (unsigned)(s.size / ce);
  const FastDiv fRe(Re);
  // the node tensor and the k-1 incoming messages staged once (their global
  // loads all in flight together), then everything runs from shared memory
  {
    const cd *Tv = T + g.node_off[v];
    for (unsigned x = lane; x < (unsigned)s.size; x += 32) Ts[x] = Tv[x];
    int off = 0;
    for (int f = 0; f < s.k; ++f) {
      if (f == e) continue;
      const int q2 = s.dims[f] * s.dims[f];
      const cd *m = incoming_msg(g, s.half0 + f, n2e_old, e2n_old, n2e_new, src_sel);
      for (int x = lane; x < q2; x += 32) Ms[off + x] = m[x];
      off += q2;
    }
    __syncwarp();
  }
  for (int a = 0; a < ce; ++a) {
    for (unsigned x = lane; x < P; x += 32) {
      const unsigned l = fRe.div(x), r = x - l * Re;
      bufA[x] = Ts[(l * (unsigned)ce + (unsigned)a) * Re + r];
    }
    __syncwarp();
    cd *cur = bufA, *nxt = bufB;
    unsigned Lj = 1;
    int off = 0;
    for (int f = 0; f < s.k; ++f) {
      if (f == e) continue;
      const int q = s.dims[f];
      const unsigned R = P / Lj / (unsigned)q;
      warp_mode_product(cur, nxt, Lj, q, R, Ms + off);
      __syncwarp();
      cd *t = cur;
      cur = nxt;
      nxt = t;
      Lj *= (unsigned)q;
      off += q * q;
    }
    for (int ap = 0; ap < ce; ++ap) {
      cd acc = czero();
      for (unsigned x = lane; x < P; x += 32) {
        const unsigned l = fRe.div(x), r = x - l * Re;
        cfmac(acc, Ts[(l * (unsigned)ce + (unsigned)ap) * Re + r], cur[x]);
      }
      acc = warp_csum(acc);
      if (lane == 0) out[ap * ce + a] = acc;
    }
    __syncwarp();
  }
  cd tr = czero();
  if (lane == 0)
    for (int i = 0; i < ce; ++i) tr = cadd(tr, out[i * ce + i]);
  tr.x = __shfl_sync(0xffffffffu, tr.x, 0);
  tr.y = __shfl_sync(0xffffffffu, tr.y, 0);
  cd *dst = n2e_new + g.half_msg_off[h];
  for (int i = lane; i < ce * ce; i += 32) dst[i] = cdiv(out[i], tr);
  __syncwarp();
}

// A whole asynchronous sweep in one CTA, for graphs of small nodes: the
// warps take the half-edges of a level (one each), a __syncthreads closes the
// level, then the edge pass. No grid barrier; bit-identical to the per-level
// launches. Per warp: out (max_chi^2) and two slices in shared memory.
constexpr int ONECTA_THREADS = 1024;
// per warp: out (max_chi^2), two slices, the node tensor (max_slice x max_chi),
// the incoming messages ((DQZ_MAX_DEGREE - 1) x max_chi^2)
__host__ __device__ inline size_t round_up16(size_t x) { return (x + 15) & ~(size_t)15; }
__host__ __device__ inline size_t onecta_warp_elems(int max_slice, int max_chi) {
  return (size_t)max_chi * max_chi + 2 * (size_t)max_slice + (size_t)max_slice * max_chi +
         (size_t)(DQZ_MAX_DEGREE - 1) * max_chi * max_chi;
}

__global__ void __launch_bounds__(ONECTA_THREADS) bp_sweep_onecta_kernel(
    dqz_graph_t g, const cd *__restrict__ T, const cd *n2e_old, const cd *e2n_old, cd *n2e_new, cd *e2n_new,
    const uint8_t *__restrict__ src_sel, const uint8_t *__restrict__ edge_new, const int32_t *__restrict__ halves,
    const int32_t *__restrict__ level_off, int n_levels, int max_slice, int max_chi) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  cd *out = reinterpret_cast<cd *>(smem_raw) + (size_t)warp * onecta_warp_elems(max_slice, max_chi);
  cd *bufA = out + (size_t)max_chi * max_chi;
  cd *bufB = bufA + max_slice;
  cd *Ts = bufB + max_slice;
  cd *Ms = Ts + (size_t)max_slice * max_chi;
  for (int lv = 0; lv < n_levels; ++lv) {
    for (int item = level_off[lv] + warp; item < level_off[lv + 1]; item += nw)
      warp_node_update_half(g, T, n2e_old, e2n_old, n2e_new, src_sel, halves[item], out, bufA, bufB, Ts, Ms);
    __syncthreads();
  }
  for (int h = warp; h < g.n_halves; h += nw) {
    const int e = g.half_edge[h];
    const int tw = g.half_twin[h];
    if (e < 0 || tw < 0) continue;
    const int c = g.edge_chi[e];
    const cd *src = (edge_new[h] ? n2e_new : n2e_old) + g.half_msg_off[tw];
    cd *dst = e2n_new + g.half_msg_off[h];
    warp_copy16(reinterpret_cast<uint4 *>(dst), reinterpret_cast<const uint4 *>(src), c * c);
  }
}

// ---- the one-CTA sweep with a host-built plan: per item (the order of the
// level table) DQZ_PLAN_WORDS words: node offset, degree k, physical
// dimension d, slot e of the outgoing bond, outgoing message offset, the k
// bond dimensions (DQZ_MAX_DEGREE words), then per other bond in bond order
// its incoming message as offset * 4 + source (DQZ_SRC_*). A warp reads its
// item's words in one coalesced load instead of walking node -> half-edges
// -> edges -> twins (six dependent loads), then stages the tensor and the
// messages at once. Same arithmetic as warp_node_update_half.
__device__ __forceinline__ void warp_plan_item(const long long *pw, const cd *__restrict__ T, const cd *n2e_old,
                                               const cd *e2n_old, cd *n2e_new, cd *out, cd *bufA, cd *bufB, cd *Ts,
                                               cd *Ms) {
  const int lane = threadIdx.x & 31;
  const int k = (int)pw[1], d = (int)pw[2], e = (int)pw[3];
  const long long *dims = pw + 5;
  unsigned size = (unsigned)d, Re = (unsigned)d;
  for (int f = k - 1; f >= 0; --f) {
    if (f == e) Re = size;
    size *= (unsigned)dims[f];
  }
  const int ce = (int)dims[e];
  const unsigned P = size / (unsigned)ce;
  {
    const cd *Tv = T + pw[0];
    for (unsigned x = lane; x < size; x += 32) Ts[x] = Tv[x];
    int off = 0, slot = 0;
    for (int f = 0; f < k; ++f) {
      if (f == e) continue;
      const int q2 = (int)(dims[f] * dims[f]);
      const long long code = pw[5 + DQZ_MAX_DEGREE + slot];
      const int src = (int)(code & 3);
      const cd *m = (src == DQZ_SRC_E2N_OLD ? e2n_old : (src == DQZ_SRC_N2E_NEW ? n2e_new : n2e_old)) + (code >> 2);
      for (int x = lane; x < q2; x += 32) Ms[off + x] = m[x];
      off += q2;
      ++slot;
    }
    __syncwarp();
  }
  for (int a = 0; a < ce; ++a) {
    for (unsigned x = lane; x < P; x += 32) {
      const unsigned l = x / Re, r = x - l * Re;
      bufA[x] = Ts[(l * (unsigned)ce + (unsigned)a) * Re + r];
    }
    __syncwarp();
    cd *cur = bufA, *nxt = bufB;
    unsigned Lj = 1;
    int off = 0;
    for (int f = 0; f < k; ++f) {
      if (f == e) continue;
      const int q = (int)dims[f];
      const unsigned R = P / Lj / (unsigned)q;
      warp_mode_product(cur, nxt, Lj, q, R, Ms + off);
      __syncwarp();
      cd *t = cur;
      cur = nxt;
      nxt = t;
      Lj *= (unsigned)q;
      off += q * q;
    }
    for (int ap = 0; ap < ce; ++ap) {
      cd acc = czero();
      for (unsigned x = lane; x < P; x += 32) {
        const unsigned l = x / Re, r = x - l * Re;
        cfmac(acc, Ts[(l * (unsigned)ce + (unsigned)ap) * Re + r], cur[x]);
      }
      acc = warp_csum(acc);
      if (lane == 0) out[ap * ce + a] = acc;
    }
    __syncwarp();
  }
  cd tr = czero();
  if (lane == 0)
    for (int i = 0; i < ce; ++i) tr = cadd(tr, out[i * ce + i]);
  tr.x = __shfl_sync(0xffffffffu, tr.x, 0);
  tr.y = __shfl_sync(0xffffffffu, tr.y, 0);
  cd *dst = n2e_new + pw[4];
  for (int i = lane; i < ce * ce; i += 32) dst[i] = cdiv(out[i], tr);
  __syncwarp();
}

__global__ void __launch_bounds__(ONECTA_THREADS) bp_sweep_planned_kernel(
    dqz_graph_t g, const cd *__restrict__ T, const cd *n2e_old, const cd *e2n_old, cd *n2e_new, cd *e2n_new,
    const uint8_t *__restrict__ edge_new, const long long *__restrict__ plan, const int32_t *__restrict__ level_off,
    int n_levels, int max_slice, int max_chi) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  long long *pw = reinterpret_cast<long long *>(smem_raw) + (size_t)warp * DQZ_PLAN_WORDS;
  cd *out = reinterpret_cast<cd *>(smem_raw + round_up16((size_t)nw * DQZ_PLAN_WORDS * sizeof(long long))) +
            (size_t)warp * onecta_warp_elems(max_slice, max_chi);
  cd *bufA = out + (size_t)max_chi * max_chi;
  cd *bufB = bufA + max_slice;
  cd *Ts = bufB + max_slice;
  cd *Ms = Ts + (size_t)max_slice * max_chi;
  for (int lv = 0; lv < n_levels; ++lv) {
    for (int item = level_off[lv] + warp; item < level_off[lv + 1]; item += nw) {
      if (lane < DQZ_PLAN_WORDS) pw[lane] = plan[(long long)item * DQZ_PLAN_WORDS + lane];
      __syncwarp();
      warp_plan_item(pw, T, n2e_old, e2n_old, n2e_new, out, bufA, bufB, Ts, Ms);
    }
    __syncthreads();
  }
  for (int h = warp; h < g.n_halves; h += nw) {
    const int e = g.half_edge[h];
    const int tw = g.half_twin[h];
    if (e < 0 || tw < 0) continue;
    const int c = g.edge_chi[e];
    const cd *src = (edge_new[h] ? n2e_new : n2e_old) + g.half_msg_off[tw];
    cd *dst = e2n_new + g.half_msg_off[h];
    warp_copy16(reinterpret_cast<uint4 *>(dst), reinterpret_cast<const uint4 *>(src), c * c);
  }
}

// Grid-wide barrier for a cooperative launch: one arrival counter and one
// generation word (sync[0], sync[1], zero at launch). The last block to arrive
// resets the counter and advances the generation; the others poll it, at
// most `limit` times. Returns false in every thread of a block that gave up
// (it has set *error_flag to 3).
__device__ __forceinline__ bool grid_barrier(unsigned *sync, unsigned &gen, int *error_flag) {
  __shared__ int ok_sh;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    const unsigned target = gen + 1;
    if (atomicAdd(&sync[0], 1u) == gridDim.x - 1) {
      atomicExch(&sync[0], 0u);
      __threadfence();
      atomicExch(&sync[1], target);
    } else {
      ok = 0;
      for (int it = 0; it < (1 << 24); ++it) {
        if (atomicAdd(&sync[1], 0u) == target) {
          ok = 1;
          break;
        }
        __nanosleep(32);
      }
      if (!ok) atomicExch(error_flag, 3);
    }
    __threadfence();
    ok_sh = ok;
  }
  __syncthreads();
  ++gen;
  return ok_sh != 0;
}

// A whole sweep in one cooperative launch: node levels in order (the
// asynchronous schedule's dependency levels), a grid barrier after each, then
// the edge pass. Every half-edge is computed exactly as bp_node_generic does.
__global__ void __launch_bounds__(BP_THREADS) bp_sweep_levels_kernel(
    dqz_graph_t g, const cd *__restrict__ T, const cd *n2e_old, const cd *e2n_old, cd *n2e_new, cd *e2n_new,
    const uint8_t *__restrict__ src_sel, const uint8_t *__restrict__ edge_new, const int32_t *__restrict__ halves,
    const int32_t *__restrict__ level_off, int n_levels, int max_slice, int max_chi, unsigned *sync,
    int *error_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd *out = reinterpret_cast<cd *>(smem_raw + 48 * sizeof(double));
  cd *bufA = out + (long long)max_chi * max_chi;
  cd *bufB = bufA + max_slice;
  __shared__ cd trace_sh;
  unsigned gen = 0;
  for (int lv = 0; lv < n_levels; ++lv) {
    for (int item = level_off[lv] + blockIdx.x; item < level_off[lv + 1]; item += gridDim.x)
      node_update_half(g, T, n2e_old, e2n_old, n2e_new, src_sel, halves[item], out, bufA, bufB, trace_sh);
    if (!grid_barrier(sync, gen, error_flag)) return;
  }
  // edge pass: e2n_new[h] = (edge_new[h] ? n2e_new : n2e_old)[twin(h)], one warp per half-edge
  const int wpb = blockDim.x >> 5;
  for (int h = blockIdx.x * wpb + (threadIdx.x >> 5); h < g.n_halves; h += gridDim.x * wpb) {
    const int e = g.half_edge[h];
    const int tw = g.half_twin[h];
    if (e < 0 || tw < 0) continue;
    const int c = g.edge_chi[e];
    const cd *src = (edge_new[h] ? n2e_new : n2e_old) + g.half_msg_off[tw];
    cd *dst = e2n_new + g.half_msg_off[h];
    warp_copy16(reinterpret_cast<uint4 *>(dst), reinterpret_cast<const uint4 *>(src), c * c);
  }
}

// The same sweep with each half-edge's slices spread over the grid (for
// large bonds, where a level has few half-edges but each carries much work):
// per level, every (half-edge, slice) item writes its unnormalised column of
// the outgoing message; after a grid barrier each half-edge of the level is
// divided by its trace; a second barrier closes the level. Same arithmetic and
// order as bp_node_generic, so the messages are bit-identical.
// Twice the threads of the per-level kernels: a level's items all run at
// once, so the level lasts as long as one item, and more threads per item
// shorten it (two CTAs of 512 threads still fit per SM).
constexpr int SLICED_THREADS = 512;
__global__ void __launch_bounds__(SLICED_THREADS, 2) bp_sweep_sliced_kernel(
    dqz_graph_t g, const cd *__restrict__ T, const cd *n2e_old, const cd *e2n_old, cd *n2e_new, cd *e2n_new,
    const uint8_t *__restrict__ src_sel, const uint8_t *__restrict__ edge_new, const int32_t *__restrict__ halves,
    const int32_t *__restrict__ level_off, const int32_t *__restrict__ item_half,
    const int32_t *__restrict__ item_slice, const int32_t *__restrict__ item_off, int n_levels, int max_slice,
    int max_chi, unsigned *sync, int *error_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd *bufA = reinterpret_cast<cd *>(smem_raw + 48 * sizeof(double)) + (long long)max_chi * max_chi;
  cd *bufB = bufA + max_slice;
  __shared__ cd trace_sh;
  unsigned gen = 0;
  for (int lv = 0; lv < n_levels; ++lv) {
    for (int item = item_off[lv] + blockIdx.x; item < item_off[lv + 1]; item += gridDim.x) {
      const int h = item_half[item], a = item_slice[item];
      const int v = g.half_node[h];
      NodeShape s;
      load_shape(g, v, s);
      const int e = h - s.half0;
      const int ce = s.dims[e];
      cd *dst = n2e_new + g.half_msg_off[h];
      node_slice_column(g, T + g.node_off[v], s, e, n2e_old, e2n_old, n2e_new, src_sel, a, bufA, bufB,
                        [&](int ap, cd val) { dst[ap * ce + a] = val; });
    }
    if (!grid_barrier(sync, gen, error_flag)) return;
    for (int i = level_off[lv] + blockIdx.x; i < level_off[lv + 1]; i += gridDim.x) {
      const int h = halves[i];
      const int ce = g.edge_chi[g.half_edge[h]];
      cd *m = n2e_new + g.half_msg_off[h];
      normalise_by_trace(m, m, ce, trace_sh);
    }
    if (!grid_barrier(sync, gen, error_flag)) return;
  }
  const int wpb = blockDim.x >> 5;
  for (int h = blockIdx.x * wpb + (threadIdx.x >> 5); h < g.n_halves; h += gridDim.x * wpb) {
    const int e = g.half_edge[h];
    const int tw = g.half_twin[h];
    if (e < 0 || tw < 0) continue;
    const int c = g.edge_chi[e];
    const cd *src = (edge_new[h] ? n2e_new : n2e_old) + g.half_msg_off[tw];
    cd *dst = e2n_new + g.half_msg_off[h];
    warp_copy16(reinterpret_cast<uint4 *>(dst), reinterpret_cast<const uint4 *>(src), c * c);
  }
}

__global__ void bp_edge_pass_kernel(dqz_graph_t g, const cd *n2e_old, const cd *n2e_new,
                                    const uint8_t *__restrict__ edge_new, cd *e2n_new) {
  const int nh = g.n_halves;
  // one warp per half-edge
  const int warps_per_block = blockDim.x >> 5;
  for (int h = blockIdx.x * warps_per_block + (threadIdx.x >> 5); h < nh; h += gridDim.x * warps_per_block) {
    const int e = g.half_edge[h];
    const int tw = g.half_twin[h];
    if (e < 0 || tw < 0) continue;
    const int c = g.edge_chi[e];
    const cd *src = (edge_new[h] ? n2e_new : n2e_old) + g.half_msg_off[tw];
    cd *dst = e2n_new + g.half_msg_off[h];
    warp_copy16(reinterpret_cast<uint4 *>(dst), reinterpret_cast<const uint4 *>(src), c * c);
  }
}

// partial[h] = |n2e_a[h] - n2e_b[h]|_F, partial[2E + h] = |e2n_a[h] - e2n_b[h]|_F
__global__ void msg_dist_kernel(dqz_graph_t g, const cd *n2e_a, const cd *n2e_b, const cd *e2n_a, const cd *e2n_b,
                                double *partial) {
  const int nh = g.n_halves;
  const int wpb = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < 2 * nh; w += gridDim.x * wpb) {
    const int h = w < nh ? w : w - nh;
    const cd *A = (w < nh ? n2e_a : e2n_a) + g.half_msg_off[h];
    const cd *B = (w < nh ? n2e_b : e2n_b) + g.half_msg_off[h];
    const int e = g.half_edge[h];
    if (e < 0) {
      if (lane == 0) partial[w] = 0.0;
      continue;
    }
    const int c = g.edge_chi[e];
    double acc = 0.0;
    for (int i = lane; i < c * c; i += 32) acc += cabs2(csub(A[i], B[i]));
    acc = warp_sum(acc);
    if (lane == 0) partial[w] = sqrt(acc);
  }
}

// partial[h] = |a[h] - b[h]|_F over the node->edge messages of complex64 arenas.
__global__ void msg_dist_c64_kernel(dqz_graph_t g, const float2 *a, const float2 *b, double *partial) {
  const int nh = g.n_halves;
  const int wpb = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int h = blockIdx.x * wpb + (threadIdx.x >> 5); h < nh; h += gridDim.x * wpb) {
    const int e = g.half_edge[h];
    if (e < 0) {
      if (lane == 0) partial[h] = 0.0;
      continue;
    }
    const int c = g.edge_chi[e];
    const float2 *A = a + g.half_msg_off[h], *B = b + g.half_msg_off[h];
    double acc = 0.0;
    for (int i = lane; i < c * c; i += 32) {
      const double dx = (double)A[i].x - (double)B[i].x, dy = (double)A[i].y - (double)B[i].y;
      acc += dx * dx + dy * dy;
    }
    acc = warp_sum(acc);
    if (lane == 0) partial[h] = sqrt(acc);
  }
}

// out[0] = sum(partial[0..n)) * scale, deterministic single-CTA reduction.
__global__ void reduce_sum_kernel(const double *partial, int n, double scale, double *out) {
  __shared__ double red[48];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) out[0] = acc * scale;
}

size_t bp_smem_bytes(int max_slice, int max_chi, bool use_scratch) {
  size_t b = 48 * sizeof(double) + (size_t)max_chi * max_chi * sizeof(cd);
  if (!use_scratch) b += 2 * (size_t)max_slice * sizeof(cd);
  return b;
}

constexpr size_t BP_SMEM_LIMIT = 200 * 1024;
constexpr int BP_SCRATCH_GRID = 148 * 4;

}  // namespace

extern "C" size_t dqz_bp_node_scratch_bytes(int32_t n_halves, int32_t max_slice, int32_t max_chi) {
  if (bp_smem_bytes(max_slice, max_chi, false) <= BP_SMEM_LIMIT) return 0;
  int grid = n_halves < BP_SCRATCH_GRID ? n_halves : BP_SCRATCH_GRID;
  return (size_t)grid * 2 * (size_t)max_slice * sizeof(cd);
}

extern "C" int dqz_bp_node_update(const dqz_graph_t *g, const void *tensors, const void *n2e_old,
                                  const void *e2n_old, void *n2e_new, const uint8_t *src_sel,
                                  const int32_t *halves, int32_t n_halves, int32_t max_slice, int32_t max_chi,
                                  void *scratch, cudaStream_t stream) {
  if (!g || !tensors || !n2e_new || !src_sel || !halves || n_halves < 0 || max_slice <= 0) return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  if (n_halves == 0) return DQZ_OK;
  const bool use_scratch = bp_smem_bytes(max_slice, max_chi, false) > BP_SMEM_LIMIT;
  if (use_scratch && !scratch) return DQZ_ERR_ARG;
  const size_t smem = bp_smem_bytes(max_slice, max_chi, use_scratch);
  if (smem > BP_SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;
  DQZ_SMEM_ATTR_ONCE(bp_node_generic, BP_SMEM_LIMIT);
  int grid = use_scratch ? (n_halves < BP_SCRATCH_GRID ? n_halves : BP_SCRATCH_GRID) : n_halves;
  bp_node_generic<<<grid, BP_THREADS, smem, stream>>>(
      *g, (const cd *)tensors, (const cd *)n2e_old, (const cd *)e2n_old, (cd *)n2e_new, src_sel, halves, n_halves,
      max_slice, max_chi, use_scratch ? (cd *)scratch : nullptr);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_bp_edge_pass(const dqz_graph_t *g, const void *n2e_old, const void *n2e_new,
                                const uint8_t *edge_new, void *e2n_new, int32_t max_chi, cudaStream_t stream) {
  if (!g || !n2e_old || !n2e_new || !edge_new || !e2n_new) return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  const int nh = g->n_halves;
  if (nh == 0) return DQZ_OK;
  const int wpb = 8;
  int grid = (nh + wpb - 1) / wpb;
  bp_edge_pass_kernel<<<grid, wpb * 32, 0, stream>>>(*g, (const cd *)n2e_old, (const cd *)n2e_new, edge_new,
                                                    (cd *)e2n_new);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_messages_distance(const dqz_graph_t *g, const void *n2e_a, const void *n2e_b, const void *e2n_a,
                                     const void *e2n_b, double *partial, double *out, int32_t max_chi,
                                     cudaStream_t stream) {
  if (!g || !n2e_a || !n2e_b || !e2n_a || !e2n_b || !partial || !out) return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  const int nh = g->n_halves;
  if (nh == 0) return DQZ_ERR_ARG;
  const int wpb = 8;
  int grid = (2 * nh + wpb - 1) / wpb;
  msg_dist_kernel<<<grid, wpb * 32, 0, stream>>>(*g, (const cd *)n2e_a, (const cd *)n2e_b, (const cd *)e2n_a,
                                                (const cd *)e2n_b, partial);
  DQZ_CHECK_LAUNCH();
  reduce_sum_kernel<<<1, 256, 0, stream>>>(partial, 2 * nh, 1.0 / (2.0 * nh), out);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_reduce_sum(const double *partial, int32_t n, double scale, double *out, cudaStream_t stream) {
  if (!partial || !out || n <= 0) return DQZ_ERR_ARG;
  reduce_sum_kernel<<<1, 256, 0, stream>>>(partial, n, scale, out);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_bp_sweep_levels(const dqz_graph_t *g, const void *tensors, const void *n2e_old,
                                   const void *e2n_old, void *n2e_new, void *e2n_new, const uint8_t *src_sel,
                                   const uint8_t *edge_new, const int32_t *halves, const int32_t *level_off,
                                   int32_t n_levels, int32_t max_level, int32_t max_slice, int32_t max_chi,
                                   uint32_t *sync, int32_t *error_flag, cudaStream_t stream) {
  if (!g || !tensors || !n2e_old || !e2n_old || !n2e_new || !e2n_new || !src_sel || !edge_new || !halves ||
      !level_off || !sync || !error_flag || n_levels <= 0 || max_level <= 0 || max_slice <= 0)
    return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  // Small nodes (bond slices up to 256 elements) and narrow levels (at most
  // two half-edges per warp): the whole sweep in one CTA, a warp per
  // half-edge and __syncthreads between levels (no grid barrier). Knob
  // DQZ_TUNE_SWEEP_ONECTA: 1 = never, 2 = wherever the warps' buffers fit.
  {
    const int knob = dqz_get_tuning(DQZ_TUNE_SWEEP_ONECTA);
    const size_t per_warp = onecta_warp_elems(max_slice, max_chi) * sizeof(cd);
    int warps = (int)(BP_SMEM_LIMIT / per_warp);
    if (warps > ONECTA_THREADS / 32) warps = ONECTA_THREADS / 32;
    const bool rule = max_slice <= 256 && warps >= 8 && max_level <= 2 * warps;
    if (knob != 1 && warps >= 1 && (rule || knob == 2)) {
      DQZ_SMEM_ATTR_ONCE(bp_sweep_onecta_kernel, BP_SMEM_LIMIT);
      bp_sweep_onecta_kernel<<<1, 32 * warps, (size_t)warps * per_warp, stream>>>(
          *g, (const cd *)tensors, (const cd *)n2e_old, (const cd *)e2n_old, (cd *)n2e_new, (cd *)e2n_new, src_sel,
          edge_new, halves, level_off, (int)n_levels, (int)max_slice, (int)max_chi);
      DQZ_CHECK_LAUNCH();
      return DQZ_OK;
    }
  }
  const size_t smem = bp_smem_bytes(max_slice, max_chi, false);
  if (smem > BP_SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;  // the per-level launches use global scratch then
  DQZ_SMEM_ATTR_ONCE(bp_sweep_levels_kernel, BP_SMEM_LIMIT);
  int dev = 0, sms = 148, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DQZ_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_sweep_levels_kernel, BP_THREADS, smem) !=
          cudaSuccess ||
      per_sm < 1)
    return DQZ_ERR_UNSUPPORTED;
  int grid = max_level;  // one CTA per half-edge of the widest level, all co-resident
  if (grid > sms * per_sm) grid = sms * per_sm;
  if (cudaMemsetAsync(sync, 0, 2 * sizeof(uint32_t), stream) != cudaSuccess) return DQZ_ERR_CUDA;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(BP_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, bp_sweep_levels_kernel, *g, (const cd *)tensors, (const cd *)n2e_old,
                         (const cd *)e2n_old, (cd *)n2e_new, (cd *)e2n_new, src_sel, edge_new, halves, level_off,
                         (int)n_levels, (int)max_slice, (int)max_chi, (unsigned *)sync, (int *)error_flag) !=
      cudaSuccess)
    return DQZ_ERR_CUDA;
  return DQZ_OK;
}

extern "C" int dqz_bp_sweep_planned(const dqz_graph_t *g, const void *tensors, const void *n2e_old,
                                    const void *e2n_old, void *n2e_new, void *e2n_new, const uint8_t *edge_new,
                                    const int64_t *plan, const int32_t *level_off, int32_t n_levels,
                                    int32_t max_level, int32_t max_slice, int32_t max_chi, cudaStream_t stream) {
  if (!g || !tensors || !n2e_old || !e2n_old || !n2e_new || !e2n_new || !edge_new || !plan || !level_off ||
      n_levels <= 0 || max_level <= 0 || max_slice <= 0)
    return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  const size_t per_warp = onecta_warp_elems(max_slice, max_chi) * sizeof(cd);
  int warps = ONECTA_THREADS / 32;
  while (warps > 8 && round_up16((size_t)warps * DQZ_PLAN_WORDS * sizeof(long long)) + warps * per_warp >
                          BP_SMEM_LIMIT)
    --warps;
  const size_t smem = round_up16((size_t)warps * DQZ_PLAN_WORDS * sizeof(long long)) + warps * per_warp;
  if (smem > BP_SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;
  DQZ_SMEM_ATTR_ONCE(bp_sweep_planned_kernel, BP_SMEM_LIMIT);
  bp_sweep_planned_kernel<<<1, 32 * warps, smem, stream>>>(
      *g, (const cd *)tensors, (const cd *)n2e_old, (const cd *)e2n_old, (cd *)n2e_new, (cd *)e2n_new, edge_new,
      (const long long *)plan, level_off, (int)n_levels, (int)max_slice, (int)max_chi);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_message_changes_c64(const dqz_graph_t *g, const void *n2e_a, const void *n2e_b, double *partial,
                                       cudaStream_t stream) {
  if (!g || !n2e_a || !n2e_b || !partial) return DQZ_ERR_ARG;
  const int nh = g->n_halves;
  if (nh == 0) return DQZ_OK;
  const int wpb = 8;
  msg_dist_c64_kernel<<<(nh + wpb - 1) / wpb, wpb * 32, 0, stream>>>(*g, (const float2 *)n2e_a, (const float2 *)n2e_b,
                                                                   partial);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_bp_sweep_sliced(const dqz_graph_t *g, const void *tensors, const void *n2e_old,
                                   const void *e2n_old, void *n2e_new, void *e2n_new, const uint8_t *src_sel,
                                   const uint8_t *edge_new, const int32_t *halves, const int32_t *level_off,
                                   const int32_t *item_half, const int32_t *item_slice, const int32_t *item_off,
                                   int32_t n_levels, int32_t max_items, int32_t max_slice, int32_t max_chi,
                                   uint32_t *sync, int32_t *error_flag, cudaStream_t stream) {
  if (!g || !tensors || !n2e_old || !e2n_old || !n2e_new || !e2n_new || !src_sel || !edge_new || !halves ||
      !level_off || !item_half || !item_slice || !item_off || !sync || !error_flag || n_levels <= 0 ||
      max_items <= 0 || max_slice <= 0)
    return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  const size_t smem = bp_smem_bytes(max_slice, max_chi, false);
  if (smem > BP_SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;
  DQZ_SMEM_ATTR_ONCE(bp_sweep_sliced_kernel, BP_SMEM_LIMIT);
  int dev = 0, sms = 148, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DQZ_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_sweep_sliced_kernel, SLICED_THREADS, smem) !=
          cudaSuccess ||
      per_sm < 1)
    return DQZ_ERR_UNSUPPORTED;
  int grid = max_items;  // all co-resident
  if (grid > sms * per_sm) grid = sms * per_sm;
  if (cudaMemsetAsync(sync, 0, 2 * sizeof(uint32_t), stream) != cudaSuccess) return DQZ_ERR_CUDA;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(SLICED_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, bp_sweep_sliced_kernel, *g, (const cd *)tensors, (const cd *)n2e_old,
                         (const cd *)e2n_old, (cd *)n2e_new, (cd *)e2n_new, src_sel, edge_new, halves, level_off,
                         item_half, item_slice, item_off, (int)n_levels, (int)max_slice, (int)max_chi,
                         (unsigned *)sync, (int *)error_flag) != cudaSuccess)
    return DQZ_ERR_CUDA;
  return DQZ_OK;
}
