// Adjoint of the BP node update (FP64 / complex128): the transposed message
// sweep used to solve the implicit adjoint system at a BP fixed point.
//
// Forward (tensor_ops.py:36-60, pass_through_node) for node v, bond e:
//   Y_e  = T x_{f != e} m_f          (m_f contracted over its second index)
//   M_e  = sum_{rest} conj(T)[.., a'@e, ..] Y_e[.., a@e, ..]
//   out  = M_e / tr(M_e)
// Reverse, with cotangents in the convention grad z = dL/dRe z + i dL/dIm z:
//   gM        = gout / conj(t) - conj(sum(conj(gout) M) / t^2) I
//   gY        = T x_e gM          (gY[.., a, ..] = sum_a' gM[a', a] T[.., a', ..])
//   gT       += Y x_e conj(gM)    (gT[.., a', ..] += sum_a conj(gM[a', a]) Y[.., a, ..])
//   g m_f    += gram(Z_f, gY) ^T   with Z_f = T x_{g != e, f} m_g
//   gT       += gY x_{f != e} m_f^H
// One CTA per node; every tensor-sized buffer lives in a per-CTA slice of a
// global scratch area, the small matrices in shared memory.
#include "common.cuh"

using namespace dqz;

namespace {

constexpr int VJP_THREADS = 256;
constexpr int VJP_BUFS = 6;  // Y, gY, W1, W2, TC, spare
constexpr int VJP_GRID_MAX = 148 * 4;

struct Dims {
  long long L, R;  // products before the bond and after it (phys included)
  int q;
};

__device__ __forceinline__ Dims bond_dims(const NodeShape &s, int f) {
  Dims d;
  d.q = s.dims[f];
  d.R = s.stride[f];
  d.L = s.size / (d.R * d.q);
  return d;
}

// dst = src x_{f in mask} (m_f as M(i = b, j = a) = m_f[b q + a]); the result
// ends in dst (tmp is the other ping-pong buffer). src may be global T.
__device__ void chain_into(const NodeShape &s, const cd *src, unsigned mask, const cd *const *msgs, cd *dst,
                           cd *tmp) {
  int n = 0;
  for (int f = 0; f < s.k; ++f) n += (mask >> f) & 1u;
  if (n == 0) {
    for (long long i = threadIdx.x; i < s.size; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    return;
  }
  // parity: the last product must write dst
  cd *nxt = (n & 1) ? dst : tmp;
  cd *oth = (n & 1) ? tmp : dst;
  const cd *cur = src;
  for (int f = 0; f < s.k; ++f) {
    if (!((mask >> f) & 1u)) continue;
    const Dims d = bond_dims(s, f);
    mode_product<false>(cur, nxt, d.L, d.q, d.q, d.R, msgs[f], d.q, 1);
    __syncthreads();
    cur = nxt;
    cd *t = nxt;
    nxt = oth;
    oth = t;
  }
}

// out[a1][a2] = sum_{l, r} conj(X[l, a1, r]) Y[l, a2, r] over bond f.
__device__ void gram(const cd *X, const cd *Y, const Dims &d, cd *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long LR = d.L * d.R;
  for (int p = warp; p < d.q * d.q; p += nw) {
    const int a1 = p / d.q, a2 = p % d.q;
    cd acc = czero();
    for (long long x = lane; x < LR; x += 32) {
      const long long l = x / d.R, r = x - l * d.R;
      cfmac(acc, X[(l * d.q + a1) * d.R + r], Y[(l * d.q + a2) * d.R + r]);
    }
    acc = warp_csum(acc);
    if (lane == 0) out[p] = acc;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(VJP_THREADS) bp_vjp_kernel(dqz_graph_t g, const cd *__restrict__ Tall,
                                                             const cd *__restrict__ e2n,
                                                             const cd *__restrict__ n2e_cot, cd *e2n_cot, cd *t_cot,
                                                             const int32_t *__restrict__ nodes, int n_nodes,
                                                             int max_size, int max_chi, cd *scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd *gM = reinterpret_cast<cd *>(smem_raw);  // max_chi^2
  cd *Mm = gM + max_chi * max_chi;             // max_chi^2
  __shared__ cd tr_sh, s_sh;
  cd *Yb = scratch + (long long)blockIdx.x * VJP_BUFS * max_size;
  cd *GY = Yb + max_size, *W1 = GY + max_size, *W2 = W1 + max_size, *TC = W2 + max_size;
  for (int item = blockIdx.x; item < n_nodes; item += gridDim.x) {
    const int v = nodes[item];
    NodeShape s;
    load_shape(g, v, s);
    bool fits = s.size <= max_size;
    for (int f = 0; f < s.k; ++f) fits = fits && s.dims[f] <= max_chi;
    if (!fits) {  // outside the caller's bounds: mark the node's cotangents
      for (int f = 0; f < s.k; ++f)
        if (threadIdx.x == 0) e2n_cot[g.half_msg_off[s.half0 + f]] = mk(__longlong_as_double(0x7ff8000000000000ll), 0.0);
      continue;
    }
    const cd *T = Tall + g.node_off[v];
    const cd *msgs[DQZ_MAX_DEGREE];
    for (int f = 0; f < s.k; ++f) msgs[f] = e2n + g.half_msg_off[s.half0 + f];
    const unsigned all = (1u << s.k) - 1u;
    for (int f = 0; f < s.k; ++f) {
      cd *gm = e2n_cot + g.half_msg_off[s.half0 + f];
      for (int i = threadIdx.x; i < s.dims[f] * s.dims[f]; i += blockDim.x) gm[i] = czero();
    }
    if (t_cot)
      for (long long i = threadIdx.x; i < s.size; i += blockDim.x) TC[i] = czero();
    __syncthreads();
    for (int e = 0; e < s.k; ++e) {
      const Dims de = bond_dims(s, e);
      const int q = de.q;
      const cd *Ge = n2e_cot + g.half_msg_off[s.half0 + e];
      chain_into(s, T, all & ~(1u << e), msgs, Yb, W1);
      gram(T, Yb, de, Mm);
      if (threadIdx.x == 0) {
        cd t = czero();
        for (int i = 0; i < q; ++i) t = cadd(t, Mm[i * q + i]);
        cd acc = czero();
        for (int i = 0; i < q * q; ++i) cfmac(acc, Ge[i], Mm[i]);  // sum conj(G) M
        tr_sh = t;
        s_sh = cdiv(acc, cmul(t, t));
      }
      __syncthreads();
      const cd ct = cconj(tr_sh), cs = cconj(s_sh);
      for (int i = threadIdx.x; i < q * q; i += blockDim.x) {
        cd gmv = cdiv(Ge[i], ct);
        if (i / q == i % q) gmv = csub(gmv, cs);
        gM[i] = gmv;
      }
      __syncthreads();
      // gY[l, a, r] = sum_a' gM[a', a] T[l, a', r]
      mode_product<false>(T, GY, de.L, q, q, de.R, gM, 1, q);
      __syncthreads();
      if (t_cot) {
        // TC[l, a', r] += sum_a conj(gM[a', a]) Y[l, a, r]
        mode_product<true>(Yb, W1, de.L, q, q, de.R, gM, q, 1);
        __syncthreads();
        for (long long i = threadIdx.x; i < s.size; i += blockDim.x) TC[i] = cadd(TC[i], W1[i]);
        __syncthreads();
      }
      for (int f = 0; f < s.k; ++f) {
        if (f == e) continue;
        const Dims df = bond_dims(s, f);
        chain_into(s, T, all & ~(1u << e) & ~(1u << f), msgs, W1, W2);
        gram(W1, GY, df, Mm);  // Mm[a][b] = sum conj(Z[a]) gY[b]
        cd *gm = e2n_cot + g.half_msg_off[s.half0 + f];
        for (int i = threadIdx.x; i < df.q * df.q; i += blockDim.x) {
          const int b = i / df.q, a = i % df.q;
          gm[i] = cadd(gm[i], Mm[a * df.q + b]);
        }
        __syncthreads();
      }
      if (t_cot) {
        // TC += gY x_{f != e} m_f^H  (gT[.., a, ..] = sum_b conj(m_f[b, a]) W[.., b, ..])
        const cd *cur = GY;
        cd *nxt = W1, *oth = W2;
        for (int f = 0; f < s.k; ++f) {
          if (f == e) continue;
          const Dims df = bond_dims(s, f);
          mode_product<true>(cur, nxt, df.L, df.q, df.q, df.R, msgs[f], 1, df.q);
          __syncthreads();
          cur = nxt;
          cd *t = nxt;
          nxt = oth;
          oth = t;
        }
        for (long long i = threadIdx.x; i < s.size; i += blockDim.x) TC[i] = cadd(TC[i], cur[i]);
        __syncthreads();
      }
    }
    if (t_cot) {
      cd *out = t_cot + g.node_off[v];
      for (long long i = threadIdx.x; i < s.size; i += blockDim.x) out[i] = cadd(out[i], TC[i]);
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" size_t dqz_bp_node_vjp_scratch_bytes(int32_t n_nodes, int32_t max_size) {
  if (n_nodes <= 0 || max_size <= 0) return 0;
  const int grid = n_nodes < VJP_GRID_MAX ? n_nodes : VJP_GRID_MAX;
  return (size_t)grid * VJP_BUFS * (size_t)max_size * sizeof(cd);
}

extern "C" int dqz_bp_node_vjp(const dqz_graph_t *g, const void *tensors, const void *e2n, const void *n2e_cot,
                               void *e2n_cot, void *t_cot, const int32_t *nodes, int32_t n_nodes, int32_t max_size,
                               int32_t max_chi, void *scratch, cudaStream_t stream) {
  if (!g || !tensors || !e2n || !n2e_cot || !e2n_cot || !nodes || !scratch || n_nodes < 0 || max_size <= 0)
    return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  if (n_nodes == 0) return DQZ_OK;
  const size_t smem = 2 * (size_t)max_chi * max_chi * sizeof(cd);
  DQZ_SMEM_ATTR_ONCE(bp_vjp_kernel, 200 * 1024);
  const int grid = n_nodes < VJP_GRID_MAX ? n_nodes : VJP_GRID_MAX;
  bp_vjp_kernel<<<grid, VJP_THREADS, smem, stream>>>(*g, (const cd *)tensors, (const cd *)e2n, (const cd *)n2e_cot,
                                                     (cd *)e2n_cot, (cd *)t_cot, nodes, n_nodes, max_size, max_chi,
                                                     (cd *)scratch);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
