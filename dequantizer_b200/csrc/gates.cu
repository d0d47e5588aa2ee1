// Gate kernels (FP64 / complex128):
//  * apply1            -- graph/tensor_graph.py:268-275
//  * apply_half_gates  -- tensor_ops.py:221-262 (untruncated apply2)
//  * simple_update     -- tensor_ops.py:265-389 (+ tensor_graph.py:294-375),
//                         one CTA per edge of a node-disjoint batch.
#include <cooperative_groups.h>

#include "linalg.cuh"

using namespace dqz;

namespace {

constexpr int GATE_THREADS = 256;
constexpr size_t SMEM_LIMIT = 200 * 1024;
const double F32_MAX = 3.4028234663852886e38;
constexpr int HALF_STRIDE = 4 * DQZ_MAX_PHYS * DQZ_MAX_PHYS;  // complex entries per gate half
constexpr int SHAPE_ROW = DQZ_MAX_DEGREE + 4;                 // k, d, slot, r, dims...

__device__ __forceinline__ double safe_inverse(double l, double eps) { return 1.0 / ((l < eps ? F32_MAX : 0.0) + l); }
__device__ __forceinline__ double safe_truncate(double l, double eps) { return l > eps ? l : 0.0; }

// ------------------------------------------------------------------ apply1
__global__ void __launch_bounds__(GATE_THREADS) apply1_kernel(dqz_graph_t g, cd *Tall, const int32_t *nodes,
                                                               const cd *gates, int n) {
  __shared__ double red[48];
  __shared__ cd G[DQZ_MAX_PHYS * DQZ_MAX_PHYS];
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    const int v = nodes[j];
    NodeShape s;
    load_shape(g, v, s);
    const int d = s.d;
    for (int i = threadIdx.x; i < d * d; i += blockDim.x) G[i] = gates[(long long)j * DQZ_MAX_PHYS * DQZ_MAX_PHYS + i];
    __syncthreads();
    cd *T = Tall + g.node_off[v];
    const long long B = s.size / d;
    double n2 = 0.0;
    for (long long b = threadIdx.x; b < B; b += blockDim.x) {
      for (int o = 0; o < d; ++o) {
        cd acc = czero();
        for (int i = 0; i < d; ++i) cfma(acc, T[b * d + i], G[o * d + i]);
        n2 += cabs2(acc);
      }
    }
    n2 = block_sum(n2, red);
    const double inv = 1.0 / sqrt(n2);
    for (long long b = threadIdx.x; b < B; b += blockDim.x) {
      cd row[DQZ_MAX_PHYS];
      for (int i = 0; i < d; ++i) row[i] = T[b * d + i];
      for (int o = 0; o < d; ++o) {
        cd acc = czero();
        for (int i = 0; i < d; ++i) cfma(acc, row[i], G[o * d + i]);
        T[b * d + o] = cscale(acc, inv);
      }
    }
    __syncthreads();
  }
}

// -------------------------------------------------------- apply half gates
__global__ void __launch_bounds__(GATE_THREADS) half_gates_kernel(const cd *Tin, cd *Tout, const int64_t *in_off,
                                                                   const int64_t *out_off, const int32_t *shape,
                                                                   const cd *halves, int n) {
  __shared__ double red[48];
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    const int32_t *sh = shape + (long long)j * SHAPE_ROW;
    const int k = sh[0], d = sh[1], slot = sh[2], r = sh[3];
    long long in_stride[DQZ_MAX_DEGREE], out_dims[DQZ_MAX_DEGREE];
    long long st = d;
    for (int f = k - 1; f >= 0; --f) {
      in_stride[f] = st;
      st *= sh[4 + f];
      out_dims[f] = sh[4 + f] * (f == slot ? r : 1);
    }
    long long out_size = d;
    for (int f = 0; f < k; ++f) out_size *= out_dims[f];
    const cd *T = Tin + in_off[j];
    const cd *H = halves + (long long)j * HALF_STRIDE;
    cd *O = Tout + out_off[j];
    double n2 = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
      double inv = 1.0;
      if (pass == 1) inv = 1.0 / sqrt(block_sum(n2, red));
      for (long long idx = threadIdx.x; idx < out_size; idx += blockDim.x) {
        long long rem = idx;
        const int o = (int)(rem % d);
        rem /= d;
        long long base = 0;
        int rho = 0;
        for (int f = k - 1; f >= 0; --f) {
          long long a = rem % out_dims[f];
          rem /= out_dims[f];
          if (f == slot) {
            rho = (int)(a % r);
            a /= r;
          }
          base += a * in_stride[f];
        }
        cd acc = czero();
        for (int i = 0; i < d; ++i) cfma(acc, T[base + i], H[(rho * d + o) * d + i]);
        if (pass == 0)
          n2 += cabs2(acc);
        else
          O[idx] = cscale(acc, inv);
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------- simple update
struct SUSide {
  int node, slot, k, d, half0;
  int dims[DQZ_MAX_DEGREE];
  long long stride[DQZ_MAX_DEGREE];
  const double *lam[DQZ_MAX_DEGREE];
  int M;  // rows: d * prod_{f != slot} dims
};

__device__ void su_load_side(const dqz_graph_t &g, const double *lambdas, int h, SUSide &S) {
  S.node = g.half_node[h];
  NodeShape s;
  load_shape(g, S.node, s);
  S.k = s.k;
  S.d = s.d;
  S.half0 = s.half0;
  S.slot = h - s.half0;
  for (int f = 0; f < s.k; ++f) {
    S.dims[f] = s.dims[f];
    S.stride[f] = s.stride[f];
    S.lam[f] = lambdas + g.edge_lam_off[g.half_edge[s.half0 + f]];
  }
  S.M = (int)(s.size / s.dims[S.slot]);
}

// Decompose row R = (other bonds in order, o): returns the tensor offset
// without the slot bond and the physical index, and the product of
// lambda weights (or of their safe inverses).
// (32-bit index arithmetic: the entry points refuse rows x columns >= 2^31)
__device__ __forceinline__ long long su_row(const SUSide &S, unsigned R, int &o, double &wt, bool inverse,
                                            double eps) {
  const unsigned rd = R / (unsigned)S.d;
  o = (int)(R - rd * (unsigned)S.d);
  unsigned rem = rd;
  long long off = 0;
  wt = 1.0;
  for (int f = S.k - 1; f >= 0; --f) {
    if (f == S.slot) continue;
    const unsigned df = (unsigned)S.dims[f];
    const unsigned rq = rem / df;
    const int a = (int)(rem - rq * df);
    rem = rq;
    off += a * S.stride[f];
    const double l = S.lam[f][a];
    wt *= inverse ? safe_inverse(l, eps) : l;
  }
  return off;
}

// A (M x K col-major): A[R, (a_e, rho)] = sum_i T[.., a_e, .., i] h[rho][o][i] prod lambda, normalised.
__device__ void su_build(const SUSide &S, const cd *T, const cd *H, int r, cd *A, double *red) {
  const int ce = S.dims[S.slot];
  const int K = ce * r;
  const unsigned MK = (unsigned)S.M * (unsigned)K;
  const int d = S.d;
  double n2 = 0.0;
  for (unsigned idx = threadIdx.x; idx < MK; idx += blockDim.x) {
    const unsigned C = idx / (unsigned)S.M;
    const unsigned R = idx - C * (unsigned)S.M;
    const int ae = C / r, rho = C % r;
    int o;
    double wt;
    const long long off = su_row(S, R, o, wt, false, 0.0) + ae * S.stride[S.slot];
    cd acc = czero();
    for (int i = 0; i < d; ++i) cfma(acc, T[off + i], H[(rho * d + o) * d + i]);
    acc = cscale(acc, wt);
    A[idx] = acc;
    n2 += cabs2(acc);
  }
  n2 = block_sum(n2, red);
  const double inv = 1.0 / sqrt(n2);
  for (unsigned idx = threadIdx.x; idx < MK; idx += blockDim.x) A[idx] = cscale(A[idx], inv);
  __syncthreads();
}

// Gamma[.., c, .., o] = X[R, c] * prod safe_inv(lambda), new bond dimension `rank`.
__device__ void su_write(const SUSide &S, const cd *X, int rank, cd *T, double eps) {
  // strides with the new slot dimension
  long long nst[DQZ_MAX_DEGREE];
  long long st = S.d;
  for (int f = S.k - 1; f >= 0; --f) {
    nst[f] = st;
    st *= (f == S.slot) ? rank : S.dims[f];
  }
  const unsigned total = (unsigned)S.M * (unsigned)rank;
  for (unsigned idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const unsigned c = idx / (unsigned)S.M;
    const unsigned R = idx - c * (unsigned)S.M;
    const unsigned rd = R / (unsigned)S.d;
    const int o = (int)(R - rd * (unsigned)S.d);
    unsigned rem = rd;
    long long off = o + (long long)c * nst[S.slot];
    double wt = 1.0;
    for (int f = S.k - 1; f >= 0; --f) {
      if (f == S.slot) continue;
      const unsigned df = (unsigned)S.dims[f];
      const unsigned rq = rem / df;
      const int a = (int)(rem - rq * df);
      rem = rq;
      off += a * nst[f];
      wt *= safe_inverse(S.lam[f][a], eps);
    }
    T[off] = cscale(X[idx], wt);
  }
}

// Jobs whose A matrix has fewer rows on both sides (bonds below 16 between
// degree-3 nodes) stay on the global-scratch kernel, which runs several jobs
// per SM; the on-chip form takes the larger ones that fit.
constexpr int SUF_MIN_ROWS = 256;

// Dimensions of one side of a job in the shared-memory form (below):
//   B = lambda-weighted node tensor, rows b (the other bonds), columns (a, i)
//       (updated bond, physical index): MB x KB;
//   S = R_B with the half gate applied, rows (c, o), columns (a, rho): MS x KS;
//   muB / muS = min(rows, columns): reflector counts, rows of R.
struct SufDims {
  int MB, KB, muB, MS, KS, muS;
};

__device__ __forceinline__ void suf_dims(const SUSide &S, int r, SufDims &D) {
  const int ce = S.dims[S.slot];
  D.MB = S.M / S.d;
  D.KB = ce * S.d;
  D.muB = D.MB < D.KB ? D.MB : D.KB;
  D.MS = D.muB * S.d;
  D.KS = ce * r;
  D.muS = D.MS < D.KS ? D.MS : D.KS;
}

__host__ __device__ __forceinline__ long long suf_even(long long x) { return (x + 1) & ~1ll; }

// Largest kept rank of a job: max_rank when it cuts below K = KS, else K.
__host__ __device__ __forceinline__ int suf_rank_bound(int K, int max_rank) {
  return (max_rank > 0 && max_rank < K) ? max_rank : K;
}

// Size of the combined core | W region: the core SVD needs 2 K^2; later the
// same space holds V^H V (muB^2) and then V^H Z (muB x d*rank).
__device__ __forceinline__ long long suf_cw(const SufDims &D, int d, int rk) {
  const long long K = D.KS;
  long long cw = 2 * K * K;
  const long long g = (long long)D.muB * (D.muB > d * rk ? D.muB : d * rk);
  return suf_even(cw > g ? cw : g);
}

// X region: the kept columns (MS x rk), and before them the R^H work matrix
// of the core SVD (K x K at most).
__device__ __forceinline__ long long suf_x(const SufDims &D, int rk) {
  const long long a = (long long)D.MS * rk, b = (long long)D.KS * D.KS;
  return suf_even(a > b ? a : b);
}

// Complex entries of one side's shared-memory layout, in this order:
//   S [MS*KS] | tauS [muS] | B [MB*KB] | tauB [muB] | core, W [cw] | X [suf_x]
__device__ __forceinline__ long long suf_need(const SufDims &D, int d, int rk) {
  return suf_even((long long)D.MS * D.KS) + suf_even(D.muS) + suf_even((long long)D.MB * D.KB) + suf_even(D.muB) +
         suf_cw(D, d, rk) + suf_x(D, rk);
}

// Whether a job runs in the shared-memory form with `cap` complex entries
// per CTA. Both CTAs of a cluster, and the fallback kernel, decide alike.
__device__ __forceinline__ bool suf_fits(const SUSide &U, const SUSide &V, int r, int max_rank, long long cap) {
  if (cap <= 0 || (U.M < SUF_MIN_ROWS && V.M < SUF_MIN_ROWS)) return false;
  SufDims du, dv;
  suf_dims(U, r, du);
  suf_dims(V, r, dv);
  if (du.KS > DQZ_MAX_CHI) return false;
  const int rk = suf_rank_bound(du.KS, max_rank);
  return suf_need(du, U.d, rk) <= cap && suf_need(dv, V.d, rk) <= cap;
}

__host__ __device__ inline size_t su_scratch_per_job(int max_rows, int max_cols) {
  return 4 * (size_t)max_rows * max_cols * sizeof(cd);
}

__global__ void __launch_bounds__(GATE_THREADS) simple_update_kernel(
    dqz_graph_t g, cd *Tall, double *lambdas, const int32_t *edges, const uint8_t *ctrl_first, const cd *halves,
    const int32_t *ranks, int n, double eps, int max_rank, int max_rows, int max_cols, double *err_out,
    double *ent_out, cd *scratch, const uint8_t *done) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *red = reinterpret_cast<double *>(smem_raw);
  int *flag = reinterpret_cast<int *>(red + 48);
  cd *tau_u = reinterpret_cast<cd *>(flag + 4);
  cd *tau_v = tau_u + max_cols;
  cd *core = tau_v + max_cols;
  cd *W = core + max_cols * max_cols;
  cd *Xq = W + max_cols * max_cols;  // R^H of the QR-preconditioned core SVD
  cd *tau_c = Xq + max_cols * max_cols;
  double *sv = reinterpret_cast<double *>(tau_c + max_cols);
  int *perm = reinterpret_cast<int *>(sv + max_cols);
  int *acc = perm + max_cols;
  __shared__ double lam_sh[2 * DQZ_MAX_CHI];

  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    const int e = edges[j];
    const bool first = ctrl_first[j] != 0;
    const int hu = g.edge_half[2 * e + (first ? 0 : 1)];
    const int hv = g.edge_half[2 * e + (first ? 1 : 0)];
    SUSide U, V;
    su_load_side(g, lambdas, hu, U);
    su_load_side(g, lambdas, hv, V);
    const int r = ranks[j];
    if (done && done[j]) continue;  // done by the on-chip form (its marks, taken on the original shapes)
    const int ce = U.dims[U.slot];
    const int K = ce * r;
    cd *Au = scratch + (size_t)blockIdx.x * (su_scratch_per_job(max_rows, max_cols) / sizeof(cd));
    cd *Xu = Au + (size_t)max_rows * max_cols;
    cd *Av = Xu + (size_t)max_rows * max_cols;
    cd *Xv = Av + (size_t)max_rows * max_cols;
    const cd *Hu = halves + (long long)j * 2 * HALF_STRIDE;
    const cd *Hv = Hu + HALF_STRIDE;
    cd *Tu = Tall + g.node_off[U.node];
    cd *Tv = Tall + g.node_off[V.node];
    const double *lam_e = lambdas + g.edge_lam_off[e];

    su_build(U, Tu, Hu, r, Au, red);
    su_build(V, Tv, Hv, r, Av, red);
    householder_qr_owned(Au, U.M, K, tau_u);
    householder_qr_owned(Av, V.M, K, tau_v);
    const int mu = U.M < K ? U.M : K;
    const int mv = V.M < K ? V.M : K;
    const int kk = mu < mv ? mu : mv;
    const bool tall = mu >= mv;
    // Z = core (mu x mv) if tall else core^H (mv x mu); column-major, ld = zr.
    const int zr = tall ? mu : mv;
    for (int idx = threadIdx.x; idx < mu * mv; idx += blockDim.x) {
      const int i = idx % mu, jj = idx / mu;
      cd a = czero();
      for (int c = (i > jj ? i : jj); c < K; ++c)
        cfma(a, cscale(Au[(long long)c * U.M + i], lam_e[c / r]), Av[(long long)c * V.M + jj]);
      if (tall)
        core[jj * mu + i] = a;
      else
        core[i * mv + jj] = cconj(a);
    }
    __syncthreads();
    hestenes_qr(core, zr, kk, W, Xq, tau_c, sv, flag, acc, red);
    sort_desc(sv, kk, perm);
    const int rank = (max_rank > 0 && max_rank < kk) ? max_rank : kk;
    // unit columns of Z; null ones among the `rank` kept are completed below
    // (the others are never read: they stay zero and count as accepted)
    for (int idx = threadIdx.x; idx < zr * kk; idx += blockDim.x) {
      const int c = idx / zr;
      const double sc = sv[c];
      core[idx] = sc > 1e-300 ? cscale(core[idx], 1.0 / sc) : czero();
    }
    for (int p = threadIdx.x; p < kk; p += blockDim.x) {
      const int c = perm[p];
      acc[c] = (sv[c] > 1e-300 || p >= rank) ? 1 : 0;
    }
    __syncthreads();
    complete_orthonormal(core, zr, zr, kk, acc);
    // U columns: tall -> core (mu rows); else W (mu rows).
    // V^T columns (= conj of right singular vectors): tall -> conj(W) (mv rows); else conj(core) (mv rows).
    const cd *Ub = tall ? core : W;
    const cd *Vb = tall ? W : core;
    const int ldu = tall ? mu : kk, ldv = tall ? kk : mv;
    double n2 = 0.0;
    for (int c = threadIdx.x; c < kk; c += blockDim.x) {
      const double l = safe_truncate(sv[perm[c]], eps);
      lam_sh[c] = l;
      n2 += l * l;
    }
    n2 = block_sum(n2, red);
    if (threadIdx.x == 0) {
      double ent = 0.0, er = 0.0;
      for (int c = 0; c < kk; ++c) {
        const double p = lam_sh[c] * lam_sh[c] / n2;
        if (p > 0.0) ent -= p * log(p);
        if (c >= rank) er += p;
      }
      err_out[j] = sqrt(er);
      ent_out[j] = ent;
    }
    // X_u = [U[:, perm[:rank]]; 0], X_v = [conj(V)[:, perm[:rank]]; 0]
    for (long long idx = threadIdx.x; idx < (long long)U.M * rank; idx += blockDim.x) {
      const int i = (int)(idx % U.M), c = (int)(idx / U.M);
      Xu[idx] = i < mu ? Ub[(long long)perm[c] * ldu + i] : czero();
    }
    for (long long idx = threadIdx.x; idx < (long long)V.M * rank; idx += blockDim.x) {
      const int i = (int)(idx % V.M), c = (int)(idx / V.M);
      Xv[idx] = i < mv ? cconj(Vb[(long long)perm[c] * ldv + i]) : czero();
    }
    __syncthreads();
    apply_q(Au, U.M, mu, tau_u, Xu, U.M, rank);
    apply_q(Av, V.M, mv, tau_v, Xv, V.M, rank);
    su_write(U, Xu, rank, Tu, eps);
    su_write(V, Xv, rank, Tv, eps);
    double *lam_out = lambdas + g.edge_lam_off[e];
    __syncthreads();
    for (int c = threadIdx.x; c < rank; c += blockDim.x) lam_out[c] = lam_sh[c];
    if (threadIdx.x == 0) g.edge_chi[e] = rank;
    __syncthreads();
  }
}

size_t su_smem_bytes(int max_cols) {
  return 48 * sizeof(double) + 4 * sizeof(int) + 3 * (size_t)max_cols * sizeof(cd) +
         3 * (size_t)max_cols * max_cols * sizeof(cd) + (size_t)max_cols * sizeof(double) +
         2 * (size_t)max_cols * sizeof(int);
}

// ------------------------------------------------ simple update, on chip
// The same job (tensor_ops.py:265-389) with every matrix in shared memory, for
// jobs that fit (bonds up to 16 between degree-3 nodes, rank-2 gates). One
// cluster of two CTAs per job: CTA 0 works on the controlling side, CTA 1 on
// the controlled side, each on its own SM.
//  * The side's matrix A[(b, o), (a, rho)] = sum_i B[b, (a, i)] h[rho][o][i]
//    (b: the other bonds, o / i: physical out / in, a: the updated bond,
//    rho: gate rank, B = lambda-weighted node tensor) factors in two steps:
//    B = Q_B R_B (Householder, MB x KB), then S = R_B h = Q_S R_S (Householder,
//    MS x KS with MS = min(MB, KB) d), so A = (Q_B x I_o) Q_S R_S: R_A = R_S,
//    the factor the core needs (LAPACK's R up to the signs of its rows, a
//    gauge). B is half the size of A, and S is small.
//  * The two CTAs swap R_S through distributed shared memory, build the same
//    core R_u diag(lambda) R_v^T and run the same SVD (bit-identical in both).
//  * Gamma = (Q_B x I_o) Q_S [U; 0] / lambda: Q_S by its reflectors, Q_B in
//    compact-WY form I - V T V^H (LAPACK zlarft), the output rows computed
//    straight into the node tensor in HBM. No global scratch.
constexpr int SUF_THREADS = 512;
constexpr size_t SUF_SMEM_MAX = 220 * 1024;  // dynamic shared memory per CTA (plus ~2.3 KB static)

template <int THREADS, int MIN_BLOCKS>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, MIN_BLOCKS)
    simple_update_onchip_kernel(dqz_graph_t g, cd *Tall, double *lambdas, const int32_t *edges,
                                const uint8_t *ctrl_first, const cd *halves, const int32_t *ranks, int n, double eps,
                                int max_rank, double *err_out, double *ent_out, long long cap, uint8_t *done,
                                cd *gws, int chained) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the side's matrices: in shared memory, or (gws) in this CTA's slice of a
  // global workspace of `cap` entries per CTA, for jobs above shared memory
  cd *sm = gws ? gws + (long long)blockIdx.x * cap : reinterpret_cast<cd *>(smem_raw);
  __shared__ double red[48];
  __shared__ int flag[4];
  __shared__ double sv[DQZ_MAX_CHI], lam_sh[DQZ_MAX_CHI], lam_in[DQZ_MAX_CHI];
  __shared__ int perm[DQZ_MAX_CHI], acc[DQZ_MAX_CHI];
  __shared__ cd tau_c[DQZ_MAX_CHI];
  const int side = (int)cluster.block_rank();  // 0: controlling node, 1: controlled node
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;

  for (int j = (int)(blockIdx.x >> 1); j < n; j += (int)(gridDim.x >> 1)) {
    const int e = edges[j];
    const bool first = ctrl_first[j] != 0;
    const int hu = g.edge_half[2 * e + (first ? 0 : 1)];
    const int hv = g.edge_half[2 * e + (first ? 1 : 0)];
    SUSide U, V;
    su_load_side(g, lambdas, hu, U);
    su_load_side(g, lambdas, hv, V);
    const int r = ranks[j];
    // decided on the job's shapes before any update; the mark tells the
    // global-scratch kernel (launched next) which jobs are done, since this
    // launch changes the bond dimensions the decision reads
    // chained: a launch before this one marked the jobs it did (their shapes
    // have changed since); the others are decided here and marked when done
    if (chained && done[j]) continue;
    const bool fits = suf_fits(U, V, r, max_rank, cap);
    if (side == 0 && threadIdx.x == 0 && (fits || !chained)) done[j] = fits ? 1 : 0;
    if (!fits) continue;  // left to the global-scratch kernel; same decision in both CTAs
    const SUSide &X = side ? V : U;
    SufDims D, Du, Dv;
    suf_dims(U, r, Du);
    suf_dims(V, r, Dv);
    D = side ? Dv : Du;
    const int d = X.d, K = D.KS;
    cd *Sm = sm;
    cd *tauS = Sm + suf_even((long long)D.MS * D.KS);
    cd *Bm = tauS + suf_even(D.muS);
    cd *tauB = Bm + suf_even((long long)D.MB * D.KB);
    cd *core = tauB + suf_even(D.muB);
    cd *W = core + (long long)K * K;
    cd *Xm = core + suf_cw(D, d, suf_rank_bound(K, max_rank));
    const cd *H = halves + (long long)j * 2 * HALF_STRIDE + side * HALF_STRIDE;
    cd *T = Tall + g.node_off[X.node];

    // ---- B[b, (a, i)] = wt(b) T[.., a, .., i], column-major (ld MB)
    {
      const int ce = X.dims[X.slot];
      const int total = D.MB * D.KB;
      for (int idx = tid; idx < total; idx += nt) {
        const int i = idx % d;
        const int t = idx / d;
        const int a = t % ce;
        const int b = t / ce;
        unsigned rem = (unsigned)b;
        long long off = 0;
        double wt = 1.0;
        for (int f = X.k - 1; f >= 0; --f) {
          if (f == X.slot) continue;
          const unsigned df = (unsigned)X.dims[f];
          const unsigned rq = rem / df;
          const int af = (int)(rem - rq * df);
          rem = rq;
          off += af * X.stride[f];
          wt *= X.lam[f][af];
        }
        Bm[b + (long long)(a * d + i) * D.MB] = cscale(T[off + a * X.stride[X.slot] + i], wt);
      }
      __syncthreads();
    }
    householder_qr_owned(Bm, D.MB, D.KB, tauB);

    // ---- S[(c, o), (a, rho)] = sum_i R_B[c, (a, i)] h[rho][o][i], normalised (|A|_F = |S|_F)
    {
      double n2 = 0.0;
      const long long total = (long long)D.MS * D.KS;
      for (long long idx = tid; idx < total; idx += nt) {
        const int row = (int)(idx % D.MS), col = (int)(idx / D.MS);
        const int c = row / d, o = row % d, a = col / r, rho = col % r;
        cd v = czero();
        for (int i = 0; i < d; ++i) {
          const int cb = a * d + i;
          if (cb >= c) cfma(v, Bm[c + (long long)cb * D.MB], H[(rho * d + o) * d + i]);
        }
        Sm[idx] = v;
        n2 += cabs2(v);
      }
      n2 = block_sum(n2, red);
      const double inv = 1.0 / sqrt(n2);
      for (long long idx = tid; idx < total; idx += nt) Sm[idx] = cscale(Sm[idx], inv);
      __syncthreads();
    }
    householder_qr_owned(Sm, D.MS, D.KS, tauS);

    // ---- swap R_S: the partner's R (muS x K, upper trapezoidal) into W, then the core
    if (gws) __threadfence();
    cluster.sync();
    const SufDims &Dp = side ? Du : Dv;
    if (gws) {  // the partner's workspace slice, read past L1
      const cd *Sp = gws + (long long)(blockIdx.x ^ 1u) * cap;
      for (int idx = tid; idx < Dp.muS * K; idx += nt) {
        const int i = idx % Dp.muS, c = idx / Dp.muS;
        W[idx] = c >= i ? __ldcg(Sp + i + (long long)c * Dp.MS) : czero();
      }
    } else {
      const cd *Sp = cluster.map_shared_rank(Sm, side ^ 1);
      for (int idx = tid; idx < Dp.muS * K; idx += nt) {
        const int i = idx % Dp.muS, c = idx / Dp.muS;
        W[idx] = c >= i ? Sp[i + (long long)c * Dp.MS] : czero();
      }
    }
    // lambda of the updated bond, read before CTA 0 can overwrite it at the end of the job
    for (int c = tid; c < X.dims[X.slot]; c += nt) lam_in[c] = lambdas[g.edge_lam_off[e] + c];
    cluster.sync();  // both copies done: S may be overwritten from here on
    const int mu = Du.muS, mv = Dv.muS;
    const cd *Ru = side ? W : Sm;
    const cd *Rv = side ? Sm : W;
    const int ldu_r = side ? mu : Du.MS, ldv_r = side ? Dv.MS : mv;
    const int kk = mu < mv ? mu : mv;
    const bool tall = mu >= mv;
    const int zr = tall ? mu : mv;
    for (int idx = tid; idx < mu * mv; idx += nt) {  // core = R_u diag(lambda_e x 1_r) R_v^T (Z of the old form)
      const int i = idx % mu, jj = idx / mu;
      cd v = czero();
      for (int c = (i > jj ? i : jj); c < K; ++c)
        cfma(v, cscale(Ru[i + (long long)c * ldu_r], lam_in[c / r]), Rv[jj + (long long)c * ldv_r]);
      if (tall)
        core[jj * mu + i] = v;
      else
        core[i * mv + jj] = cconj(v);
    }
    __syncthreads();
    hestenes_qr(core, zr, kk, W, Xm, tau_c, sv, flag, acc, red);  // Xm is free until X is formed below
    sort_desc(sv, kk, perm);
    const int rank = (max_rank > 0 && max_rank < kk) ? max_rank : kk;
    for (int idx = tid; idx < zr * kk; idx += nt) {
      const int c = idx / zr;
      const double sc = sv[c];
      core[idx] = sc > 1e-300 ? cscale(core[idx], 1.0 / sc) : czero();
    }
    for (int p = tid; p < kk; p += nt) {
      const int c = perm[p];
      acc[c] = (sv[c] > 1e-300 || p >= rank) ? 1 : 0;
    }
    __syncthreads();
    complete_orthonormal(core, zr, zr, kk, acc);
    const cd *Ub = tall ? core : W;
    const cd *Vb = tall ? W : core;
    const int ldu = tall ? mu : kk, ldv = tall ? kk : mv;
    {
      double n2 = 0.0;
      for (int c = tid; c < kk; c += nt) {
        const double l = safe_truncate(sv[perm[c]], eps);
        lam_sh[c] = l;
        n2 += l * l;
      }
      n2 = block_sum(n2, red);
      if (side == 0 && tid == 0) {
        double ent = 0.0, er = 0.0;
        for (int c = 0; c < kk; ++c) {
          const double p = lam_sh[c] * lam_sh[c] / n2;
          if (p > 0.0) ent -= p * log(p);
          if (c >= rank) er += p;
        }
        err_out[j] = sqrt(er);
        ent_out[j] = ent;
      }
    }
    // X = [U[:, perm[:rank]]; 0] (controlling side) or [conj(V)[:, perm[:rank]]; 0], MS x rank
    {
      const int myu = side ? mv : mu;
      for (int idx = tid; idx < D.MS * rank; idx += nt) {
        const int i = idx % D.MS, c = idx / D.MS;
        cd v = czero();
        if (i < myu) v = side ? cconj(Vb[(long long)perm[c] * ldv + i]) : Ub[(long long)perm[c] * ldu + i];
        Xm[idx] = v;
      }
      __syncthreads();
    }
    apply_q(Sm, D.MS, D.muS, tauS, Xm, D.MS, rank);  // X <- Q_S X (its trailing barrier orders the reads below)

    // ---- compact WY of Q_B = H_0 .. H_{k-1} = I - V T V^H, k = muB
    const int k = D.muB, p = d * rank;
    cd *G = core;  // V^H V, then V^H Z, then T V^H Z (k x max(k, p)), column-major ld k
    cd *Tw = Sm;   // T, k x k upper triangular, ld k (S is no longer needed)
    auto vb = [&](int row, int c) -> cd {  // V[row, c], row >= c
      return row == c ? mk(1.0, 0.0) : Bm[row + (long long)c * D.MB];
    };
    for (int pr = warp; pr < k * k; pr += nw) {  // G[i, jj] for i < jj, one warp each
      const int i = pr % k, jj = pr / k;
      if (i >= jj) continue;
      cd v = czero();
      for (int row = jj + lane; row < D.MB; row += 32) cfmac(v, Bm[row + (long long)i * D.MB], vb(row, jj));
      v = warp_csum(v);
      if (lane == 0) G[i + (long long)jj * k] = v;
    }
    __syncthreads();
    if (warp == 0) {  // T[:j, j] = T[:j, :j] (-tau_j G[:j, j]), T[j, j] = tau_j (zlarft, forward, columnwise)
      for (int jj = 0; jj < k; ++jj) {
        const cd tj = tauB[jj];
        for (int i0 = 0; i0 < jj; i0 += 32) {
          const int i = i0 + lane;
          cd v = czero();
          if (i < jj)
            for (int l = i; l < jj; ++l) cfma(v, Tw[i + (long long)l * k], G[l + (long long)jj * k]);
          __syncwarp();
          if (i < jj) Tw[i + (long long)jj * k] = cmul(mk(-tj.x, -tj.y), v);
          __syncwarp();
        }
        if (lane == 0) Tw[jj + (long long)jj * k] = tj;
        for (int i = jj + 1 + lane; i < k; i += 32) Tw[i + (long long)jj * k] = czero();
        __syncwarp();
      }
    }
    __syncthreads();
    // V^H Z (k x p): Z[row, q = col * d + o] = X[row * d + o, col] for row < k
    for (int idx = tid; idx < k * p; idx += nt) {
      const int c = idx % k, q = idx / k;
      const int col = q / d, o = q % d;
      cd v = czero();
      for (int row = c; row < k; ++row) cfmac(v, vb(row, c), Xm[(row * d + o) + (long long)col * D.MS]);
      G[idx] = v;
    }
    __syncthreads();
    // G <- T G: one thread per entry (rows i consecutive: T's column reads
    // contiguous, G's a broadcast), held in registers across a barrier and
    // written in place, a chunk of entries at a time in increasing index: an
    // entry reads rows >= its own of its column, which earlier chunks never write
    for (int base = 0; base < k * p; base += 8 * nt) {
      cd vals[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int idx = base + tid + u * nt;
        vals[u] = czero();
        if (idx < k * p) {
          const int i = idx % k, q = idx / k;
          const cd *gq = G + (long long)q * k;
          cd v = czero();
          for (int l = i; l < k; ++l) cfma(v, Tw[i + (long long)l * k], gq[l]);
          vals[u] = v;
        }
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int idx = base + tid + u * nt;
        if (idx < k * p) G[idx] = vals[u];
      }
      __syncthreads();
    }
    // ---- Gamma[b, .., col, .., o] = ((Q_B Z)[b, q]) * prod safe_inv(lambda), bond `rank`
    {
      long long nst[DQZ_MAX_DEGREE];
      long long st = d;
      for (int f = X.k - 1; f >= 0; --f) {
        nst[f] = st;
        st *= (f == X.slot) ? rank : X.dims[f];
      }
      // consecutive threads take consecutive rows b: V's columns are read
      // contiguously and G[:, q] is one broadcast (q-major threads had every
      // lane of a warp on its own row of G, one shared-memory bank)
      const int total = D.MB * p;
      for (int idx = tid; idx < total; idx += nt) {
        const int b = idx % D.MB;
        const int q = idx / D.MB;
        const int col = q / d, o = q % d;
        cd v = b < k ? Xm[(b * d + o) + (long long)col * D.MS] : czero();
        const cd *gq = G + (long long)q * k;
        const int cmax = b < k ? b : k - 1;
        for (int c = 0; c <= cmax; ++c) v = csub(v, cmul(vb(b, c), gq[c]));
        unsigned rem = (unsigned)b;
        long long off = o + (long long)col * nst[X.slot];
        double wt = 1.0;
        for (int f = X.k - 1; f >= 0; --f) {
          if (f == X.slot) continue;
          const unsigned df = (unsigned)X.dims[f];
          const unsigned rq = rem / df;
          const int af = (int)(rem - rq * df);
          rem = rq;
          off += af * nst[f];
          wt *= safe_inverse(X.lam[f][af], eps);
        }
        T[off] = cscale(v, wt);
      }
    }
    if (side == 0) {
      double *lam_out = lambdas + g.edge_lam_off[e];
      for (int c = tid; c < rank; c += nt) lam_out[c] = lam_sh[c];
      if (tid == 0) g.edge_chi[e] = rank;
    }
    // the next job reads lambdas (this edge's, written by CTA 0) and edge_chi
    cluster.sync();
  }
}

constexpr int SU_GRID_MAX = 148 * 4;

}  // namespace

extern "C" int dqz_apply1(const dqz_graph_t *g, void *tensors, const int32_t *nodes, const void *gates, int32_t n,
                          cudaStream_t stream) {
  if (!g || !tensors || !nodes || !gates || n < 0) return DQZ_ERR_ARG;
  if (n == 0) return DQZ_OK;
  apply1_kernel<<<n, GATE_THREADS, 0, stream>>>(*g, (cd *)tensors, nodes, (const cd *)gates, n);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_apply_half_gates(const void *tensors_in, void *tensors_out, const int64_t *in_off,
                                    const int64_t *out_off, const int32_t *shape, const void *halves, int32_t n,
                                    cudaStream_t stream) {
  if (!tensors_in || !tensors_out || !in_off || !out_off || !shape || !halves || n < 0) return DQZ_ERR_ARG;
  if (n == 0) return DQZ_OK;
  half_gates_kernel<<<n, GATE_THREADS, 0, stream>>>((const cd *)tensors_in, (cd *)tensors_out, in_off, out_off,
                                                    shape, (const cd *)halves, n);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

// Scratch of dqz_simple_update: one byte per job (which jobs the on-chip form
// did), rounded up to 256 bytes, then one slice per CTA of the global-scratch
// kernel.
__host__ __device__ inline size_t su_marks_bytes(int32_t n) { return ((size_t)n + 255) & ~(size_t)255; }

// The cluster form with a global workspace (jobs above shared memory): at most
// SU_CLUSTER_PAIRS jobs in flight (one CTA per SM), each CTA's slice bounded
// by the side's need for matrices of max_rows x max_cols (B and S at most
// max_rows x max_cols each, core / W / X at most 3 max_cols^2 beyond that).
constexpr int SU_CLUSTER_PAIRS = 148;
__host__ __device__ inline long long su_cluster_cap(int max_rows, int max_cols) {
  return suf_even(2ll * max_rows * max_cols + 3ll * max_cols * max_cols + 8ll * max_cols + 64);
}
inline int su_cluster_pairs(int n) { return n < SU_CLUSTER_PAIRS ? n : SU_CLUSTER_PAIRS; }

extern "C" size_t dqz_simple_update_scratch_bytes(int32_t n, int32_t max_rows, int32_t max_cols) {
  int grid = n < SU_GRID_MAX ? n : SU_GRID_MAX;
  const size_t one_cta = (size_t)grid * su_scratch_per_job(max_rows, max_cols);
  const size_t cluster = (max_rows >= SUF_MIN_ROWS && n > 0)
                             ? (size_t)2 * su_cluster_pairs(n) * su_cluster_cap(max_rows, max_cols) * sizeof(cd)
                             : 0;
  return su_marks_bytes(n) + (one_cta > cluster ? one_cta : cluster);
}

extern "C" int dqz_simple_update(const dqz_graph_t *g, void *tensors, double *lambdas, const int32_t *edges,
                                 const uint8_t *ctrl_is_first, const void *halves, const int32_t *ranks, int32_t n,
                                 double eps, int32_t max_rank, int32_t max_rows, int32_t max_cols, double *err,
                                 double *entropy, void *scratch, cudaStream_t stream) {
  if (!g || !tensors || !lambdas || !edges || !ctrl_is_first || !halves || !ranks || !err || !entropy || !scratch)
    return DQZ_ERR_ARG;
  if (n < 0 || max_rows <= 0 || max_cols <= 0) return DQZ_ERR_ARG;
  if (max_cols > DQZ_MAX_CHI || (long long)max_rows * max_cols >= (1ll << 31)) return DQZ_ERR_UNSUPPORTED;
  if (n == 0) return DQZ_OK;
  const size_t smem = su_smem_bytes(max_cols);
  if (smem > SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;
  // jobs of A matrices with 256 rows or more (bond 16 and up between degree-3
  // nodes) go to the on-chip form where they fit; the global-scratch kernel
  // below then takes only the others
  uint8_t *marks = nullptr;
  cd *job_scratch = reinterpret_cast<cd *>(static_cast<char *>(scratch) + su_marks_bytes(n));
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess) return DQZ_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // The on-chip form finishes a job sooner; the one-CTA kernel, several jobs
  // per SM, has more throughput on large batches (measured at bond 16: 440
  // jobs in 5.2 ms on chip, 4.4 ms on the one-CTA kernel; 112 jobs in 2.0 vs
  // 3.3 ms). Batches of up to one job per SM take the on-chip form; the jobs
  // of such a batch above shared memory (bond 32 between degree-3 nodes: a
  // 1024 x 64 B per side) then take the same cluster form with its matrices
  // in a global workspace (both sides at once, the two-step QR), the rest the
  // one-CTA kernel. Knob DQZ_TUNE_SU_ONCHIP: 1 = the one-CTA kernel only,
  // 2 = the cluster forms at any batch size, 3 = no global-workspace form.
  const int knob = dqz_get_tuning(DQZ_TUNE_SU_ONCHIP);
  const int pairs = n < sms / 2 ? n : sms / 2;  // one CTA per SM, two per cluster
  if (max_rows >= SUF_MIN_ROWS && (knob == 4 || (knob == 0 && n > sms))) {
    // large batches (and knob 4): every 256-row job on the global-workspace
    // cluster form, 256 threads a CTA, two clusters per SM pair (measured at
    // bond 16: 3,924 jobs in 35.4 ms against 40.2 ms on the one-CTA kernel;
    // 440 jobs 4.05 against 4.69 ms)
    auto *gws = simple_update_onchip_kernel<256, 2>;
    marks = static_cast<uint8_t *>(scratch);
    const int cp = su_cluster_pairs(n) < sms ? su_cluster_pairs(n) : sms;
    gws<<<2 * cp, 256, 0, stream>>>(*g, (cd *)tensors, lambdas, edges, ctrl_is_first, (const cd *)halves, ranks, n,
                                    eps, max_rank, err, entropy, su_cluster_cap(max_rows, max_cols), marks,
                                    job_scratch, 0);
    DQZ_CHECK_LAUNCH();
  } else if (max_rows >= SUF_MIN_ROWS && (n <= sms || knob == 2) && knob != 1) {
    auto *onchip = simple_update_onchip_kernel<SUF_THREADS, 1>;
    DQZ_SMEM_ATTR_ONCE(onchip, SUF_SMEM_MAX);
    const long long cap = (long long)(SUF_SMEM_MAX / sizeof(cd));
    marks = static_cast<uint8_t *>(scratch);
    onchip<<<2 * pairs, SUF_THREADS, SUF_SMEM_MAX, stream>>>(
        *g, (cd *)tensors, lambdas, edges, ctrl_is_first, (const cd *)halves, ranks, n, eps, max_rank, err, entropy,
        cap, marks, nullptr, 0);
    DQZ_CHECK_LAUNCH();
    if (knob != 3) {
      const int cp = su_cluster_pairs(n) < pairs ? su_cluster_pairs(n) : pairs;
      onchip<<<2 * cp, SUF_THREADS, 0, stream>>>(
          *g, (cd *)tensors, lambdas, edges, ctrl_is_first, (const cd *)halves, ranks, n, eps, max_rank, err,
          entropy, su_cluster_cap(max_rows, max_cols), marks, job_scratch, 1);
      DQZ_CHECK_LAUNCH();
    }
  }
  DQZ_SMEM_ATTR_ONCE(simple_update_kernel, SMEM_LIMIT);
  // three CTAs per SM by default: with four the jobs' global scratch spills
  // from L2 (measured at bond 16: 3,924 jobs in 40.1 ms with 444 CTAs, 53.5 ms
  // with 592, 51.4 ms with 296; 440 jobs: 4.7 ms with 444 or 592)
  int grid = n < 3 * sms ? n : 3 * sms;
  if (grid > SU_GRID_MAX) grid = SU_GRID_MAX;
  const int tuned = dqz_get_tuning(DQZ_TUNE_SU_GRID);  // never above the scratch sizing (SU_GRID_MAX)
  if (tuned > 0) grid = tuned < (n < SU_GRID_MAX ? n : SU_GRID_MAX) ? tuned : (n < SU_GRID_MAX ? n : SU_GRID_MAX);
  simple_update_kernel<<<grid, GATE_THREADS, smem, stream>>>(*g, (cd *)tensors, lambdas, edges, ctrl_is_first,
                                                             (const cd *)halves, ranks, n, eps, max_rank, max_rows,
                                                             max_cols, err, entropy, job_scratch, marks);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

// ------------------------------------------- simple update, no allocation
// Scratch for dqz_simple_update_noalloc. It is part of the library image, so
// every GPU that loads libdqz keeps these bytes until the process exits. In
// host code `noalloc_scratch` only names a host-side stand-in: device code
// receives the address that cudaGetSymbolAddress returns for the current
// device.
static __device__ __align__(256) unsigned char noalloc_scratch[DQZ_NOALLOC_SCRATCH_BYTES];

#include <mutex>

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex noalloc_mutex;
void *noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};

// Device address of noalloc_scratch on the current device, looked up once
// per device (the first call on a device does this).
int noalloc_address(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DQZ_ERR_CUDA;
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return DQZ_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(noalloc_mutex);
  if (!noalloc_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, noalloc_scratch) != cudaSuccess || !p) return DQZ_ERR_CUDA;
    noalloc_ptr[dev] = p;
  }
  *out = noalloc_ptr[dev];
  return DQZ_OK;
}

}  // namespace

extern "C" int dqz_simple_update_noalloc(const dqz_graph_t *g, void *tensors, double *lambdas, const int32_t *edges,
                                         const uint8_t *ctrl_is_first, const void *halves, const int32_t *ranks,
                                         int32_t n, double eps, int32_t max_rank, int32_t max_rows, int32_t max_cols,
                                         double *err, double *entropy, cudaStream_t stream) {
  if (!g || !tensors || !lambdas || !edges || !ctrl_is_first || !halves || !ranks || !err || !entropy)
    return DQZ_ERR_ARG;
  if (n < 0 || max_rows <= 0 || max_cols <= 0) return DQZ_ERR_ARG;
  if (max_cols > DQZ_MAX_CHI || (long long)max_rows * max_cols >= (1ll << 31)) return DQZ_ERR_UNSUPPORTED;
  const size_t per_job = su_scratch_per_job(max_rows, max_cols);
  if (per_job > (size_t)DQZ_NOALLOC_SCRATCH_BYTES) return DQZ_ERR_UNSUPPORTED;
  if (n == 0) return DQZ_OK;
  const size_t smem = su_smem_bytes(max_cols);
  if (smem > SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;
  void *scratch = nullptr;
  const int st = noalloc_address(&scratch);
  if (st != DQZ_OK) return st;
  // as many CTAs as job scratch slices fit in the array; each CTA loops over jobs
  size_t slots = (size_t)DQZ_NOALLOC_SCRATCH_BYTES / per_job;
  int grid = n < SU_GRID_MAX ? n : SU_GRID_MAX;
  if ((size_t)grid > slots) grid = (int)slots;
  const int tuned = dqz_get_tuning(DQZ_TUNE_SU_GRID);  // the tuned grid, never above the slices
  if (tuned > 0 && tuned < grid) grid = tuned;
  DQZ_SMEM_ATTR_ONCE(simple_update_kernel, SMEM_LIMIT);
  simple_update_kernel<<<grid, GATE_THREADS, smem, stream>>>(*g, (cd *)tensors, lambdas, edges, ctrl_is_first,
                                                             (const cd *)halves, ranks, n, eps, max_rank, max_rows,
                                                             max_cols, err, entropy, (cd *)scratch, nullptr);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
