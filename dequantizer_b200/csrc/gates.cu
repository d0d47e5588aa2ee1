// Gate kernels (FP64 / complex128):
//  * apply1            -- graph/tensor_graph.py:268-275
//  * apply_half_gates  -- tensor_ops.py:221-262 (untruncated apply2)
//  * simple_update     -- tensor_ops.py:265-389 (+ tensor_graph.py:294-375),
//                         one CTA per edge of a node-disjoint batch.
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
__device__ __forceinline__ long long su_row(const SUSide &S, long long R, int &o, double &wt, bool inverse,
                                            double eps) {
  o = (int)(R % S.d);
  long long rem = R / S.d;
  long long off = 0;
  wt = 1.0;
  for (int f = S.k - 1; f >= 0; --f) {
    if (f == S.slot) continue;
    const int a = (int)(rem % S.dims[f]);
    rem /= S.dims[f];
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
  const long long MK = (long long)S.M * K;
  const int d = S.d;
  double n2 = 0.0;
  for (long long idx = threadIdx.x; idx < MK; idx += blockDim.x) {
    const long long R = idx % S.M;
    const int C = (int)(idx / S.M);
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
  for (long long idx = threadIdx.x; idx < MK; idx += blockDim.x) A[idx] = cscale(A[idx], inv);
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
  const long long total = (long long)S.M * rank;
  for (long long idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const long long R = idx % S.M;
    const int c = (int)(idx / S.M);
    const int o = (int)(R % S.d);
    long long rem = R / S.d;
    long long off = o + (long long)c * nst[S.slot];
    double wt = 1.0;
    for (int f = S.k - 1; f >= 0; --f) {
      if (f == S.slot) continue;
      const int a = (int)(rem % S.dims[f]);
      rem /= S.dims[f];
      off += a * nst[f];
      wt *= safe_inverse(S.lam[f][a], eps);
    }
    T[off] = cscale(X[idx], wt);
  }
}

__host__ __device__ inline size_t su_scratch_per_job(int max_rows, int max_cols) {
  return 4 * (size_t)max_rows * max_cols * sizeof(cd);
}

__global__ void __launch_bounds__(GATE_THREADS) simple_update_kernel(
    dqz_graph_t g, cd *Tall, double *lambdas, const int32_t *edges, const uint8_t *ctrl_first, const cd *halves,
    const int32_t *ranks, int n, double eps, int max_rank, int max_rows, int max_cols, double *err_out,
    double *ent_out, cd *scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *red = reinterpret_cast<double *>(smem_raw);
  int *flag = reinterpret_cast<int *>(red + 48);
  cd *tau_u = reinterpret_cast<cd *>(flag + 4);
  cd *tau_v = tau_u + max_cols;
  cd *core = tau_v + max_cols;
  cd *W = core + max_cols * max_cols;
  double *sv = reinterpret_cast<double *>(W + max_cols * max_cols);
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
    householder_qr(Au, U.M, K, tau_u, red);
    householder_qr(Av, V.M, K, tau_v, red);
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
    hestenes(core, zr, zr, kk, W, kk, sv, flag, red);
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
  return 48 * sizeof(double) + 4 * sizeof(int) + 2 * (size_t)max_cols * sizeof(cd) +
         2 * (size_t)max_cols * max_cols * sizeof(cd) + (size_t)max_cols * sizeof(double) +
         2 * (size_t)max_cols * sizeof(int);
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

extern "C" size_t dqz_simple_update_scratch_bytes(int32_t n, int32_t max_rows, int32_t max_cols) {
  int grid = n < SU_GRID_MAX ? n : SU_GRID_MAX;
  return (size_t)grid * su_scratch_per_job(max_rows, max_cols);
}

extern "C" int dqz_simple_update(const dqz_graph_t *g, void *tensors, double *lambdas, const int32_t *edges,
                                 const uint8_t *ctrl_is_first, const void *halves, const int32_t *ranks, int32_t n,
                                 double eps, int32_t max_rank, int32_t max_rows, int32_t max_cols, double *err,
                                 double *entropy, void *scratch, cudaStream_t stream) {
  if (!g || !tensors || !lambdas || !edges || !ctrl_is_first || !halves || !ranks || !err || !entropy || !scratch)
    return DQZ_ERR_ARG;
  if (n < 0 || max_rows <= 0 || max_cols <= 0) return DQZ_ERR_ARG;
  if (max_cols > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  if (n == 0) return DQZ_OK;
  const size_t smem = su_smem_bytes(max_cols);
  if (smem > SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;
  DQZ_SMEM_ATTR_ONCE(simple_update_kernel, SMEM_LIMIT);
  int grid = n < SU_GRID_MAX ? n : SU_GRID_MAX;
  const int tuned = dqz_get_tuning(DQZ_TUNE_SU_GRID);  // never above the scratch sizing (SU_GRID_MAX)
  if (tuned > 0 && tuned < grid) grid = tuned;
  simple_update_kernel<<<grid, GATE_THREADS, smem, stream>>>(*g, (cd *)tensors, lambdas, edges, ctrl_is_first,
                                                             (const cd *)halves, ranks, n, eps, max_rank, max_rows,
                                                             max_cols, err, entropy, (cd *)scratch);
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
  if (max_cols > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
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
                                                             max_cols, err, entropy, (cd *)scratch);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
