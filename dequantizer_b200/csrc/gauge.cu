// Gauge kernels (FP64 / complex128):
//  * vidal_edges    -- tensor_ops.py:108-130 (edge_svd): one warp per edge for
//                      chi <= 16, one CTA per edge above
//  * absorb         -- tensor_ops.py:88-93 (absorb_by_node), one CTA per node
//  * vidal_distance -- tensor_ops.py:143-175 + mappings/vidal_distance.py:17-42:
//                      one warp per half-edge for chi <= 16, one CTA per
//                      half-edge above
// vidal_edges, absorb and vidal_distance take an optional list of the
// edges / nodes / half-edges to process (null = all).
//  * symmetric      -- tensor_ops.py:189-199 (canonicalize)
//  * lambdas->msgs  -- mappings/symmetric_gauge.py:50-61
//  * density        -- mappings/density_matrix.py:16-37
#include "linalg.cuh"

using namespace dqz;

namespace {

constexpr int GAUGE_THREADS = 256;
constexpr size_t SMEM_LIMIT = 200 * 1024;
constexpr int WARP_MAX_CHI = 16;     // largest bond of the one-warp kernels
constexpr int WARP_ROTS = 17;        // rotation slots per warp (n / 2 + 1 for n <= 32)
constexpr size_t WARP_BLOCK_SMEM = 96 * 1024;
constexpr int SCRATCH_GRID = 148 * 4;
const double F32_MAX = 3.4028234663852886e38;

__device__ __forceinline__ double safe_inverse(double l, double eps) { return 1.0 / ((l < eps ? F32_MAX : 0.0) + l); }
__device__ __forceinline__ double safe_truncate(double l, double eps) { return l > eps ? l : 0.0; }

// ----------------------------------------------------------- vidal edges
// Work buffers per edge (each chi^2 complex): Af Vf Ab Vb Qf Qb C W, plus
// wf wb s wif wib (chi doubles each), perm/acc ints.
__host__ __device__ inline size_t vidal_edge_bytes(int c) {
  return 8 * (size_t)c * c * sizeof(cd) + 5 * (size_t)c * sizeof(double) + 2 * (size_t)c * sizeof(int) + 64;
}

// The eigenvalue weights of sqrt(m) and its safe inverse, once per eigenvalue
// (not per matrix element): w <- sqrt(safe_truncate(w)), wi <- sqrt(safe_inverse(w)).
__device__ __forceinline__ void sqrt_weights(double *w, double *wi, int c, double eps, int i0, int step) {
  for (int k = i0; k < c; k += step) {
    const double l = w[k];
    wi[k] = sqrt(safe_inverse(l, eps));
    w[k] = sqrt(safe_truncate(l, eps));
  }
}

__host__ __device__ inline size_t round16(size_t x) { return (x + 15) & ~(size_t)15; }

__global__ void __launch_bounds__(GAUGE_THREADS) vidal_edges_kernel(dqz_graph_t g, const cd *__restrict__ n2e,
                                                                     double eps, cd *orth, double *lambdas,
                                                                     int max_chi, unsigned char *scratch,
                                                                     const int32_t *__restrict__ sel, int n_sel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *red = reinterpret_cast<double *>(smem_raw);
  Rot *rots = reinterpret_cast<Rot *>(smem_raw + 48 * sizeof(double));
  int *flag = reinterpret_cast<int *>(rots + (DQZ_MAX_CHI / 2 + 1));
  unsigned char *base = reinterpret_cast<unsigned char *>(flag + 4);
  if (scratch) base = scratch + (size_t)blockIdx.x * vidal_edge_bytes(max_chi);
  const int M2 = max_chi * max_chi;
  cd *Af = reinterpret_cast<cd *>(base);
  cd *Vf = Af + M2, *Ab = Vf + M2, *Vb = Ab + M2, *Qf = Vb + M2, *Qb = Qf + M2, *C = Qb + M2, *W = C + M2;
  double *wf = reinterpret_cast<double *>(W + M2);
  double *wb = wf + max_chi, *sv = wb + max_chi, *wif = sv + max_chi, *wib = wif + max_chi;
  int *perm = reinterpret_cast<int *>(wib + max_chi);
  const int tid = threadIdx.x, nt = blockDim.x;

  const int total = sel ? n_sel : g.n_edges;
  for (int it = blockIdx.x; it < total; it += gridDim.x) {
    const int e = sel ? sel[it] : it;
    const int h0 = g.edge_half[2 * e], h1 = g.edge_half[2 * e + 1];
    const int c = g.edge_chi[e];
    const cd *mf = n2e + g.half_msg_off[h0];
    const cd *mb = n2e + g.half_msg_off[h1];
    for (int i = tid; i < c * c; i += nt) {
      Af[i] = mf[i];
      Ab[i] = mb[i];
    }
    __syncthreads();
    herm_eigh(Af, c, Vf, c, c, wf, rots, red);
    herm_eigh(Ab, c, Vb, c, c, wb, rots, red);
    sqrt_weights(wf, wif, c, eps, tid, nt);
    sqrt_weights(wb, wib, c, eps, tid, nt);
    __syncthreads();
    // Af <- sqrt(m_f), Qf <- sqrt(m_f)^+ (safe), same for b.
    for (int idx = tid; idx < c * c; idx += nt) {
      const int i = idx / c, j = idx % c;
      cd sf = czero(), sif = czero(), sb = czero(), sib = czero();
      for (int k = 0; k < c; ++k) {
        cd pf = cmul(Vf[i * c + k], cconj(Vf[j * c + k]));
        cd pb = cmul(Vb[i * c + k], cconj(Vb[j * c + k]));
        sf = cadd(sf, cscale(pf, wf[k]));
        sif = cadd(sif, cscale(pf, wif[k]));
        sb = cadd(sb, cscale(pb, wb[k]));
        sib = cadd(sib, cscale(pb, wib[k]));
      }
      Af[idx] = sf;
      Qf[idx] = sif;
      Ab[idx] = sb;
      Qb[idx] = sib;
    }
    __syncthreads();
    // C = sqrt(m_f) sqrt(m_b)^T, column-major for the one-sided Jacobi.
    for (int idx = tid; idx < c * c; idx += nt) {
      const int i = idx / c, j = idx % c;
      cd acc = czero();
      for (int k = 0; k < c; ++k) cfma(acc, Af[i * c + k], Ab[j * c + k]);
      C[j * c + i] = acc;
    }
    __syncthreads();
    hestenes(C, c, c, c, W, c, sv, flag, red);
    sort_desc(sv, c, perm);
    // lambda = sigma / |sigma|, truncated; U (into Af) and V^* (into Ab)
    // masked and Frobenius-normalised.
    double nrm2 = 0.0;
    for (int j = tid; j < c; j += nt) nrm2 += sv[j] * sv[j];
    nrm2 = block_sum(nrm2, red);
    const double inv_n = 1.0 / sqrt(nrm2);
    double *lam = lambdas + g.edge_lam_off[e];
    for (int j = tid; j < c; j += nt) lam[j] = safe_truncate(sv[perm[j]] * inv_n, eps);
    __syncthreads();
    double un = 0.0, vn = 0.0;
    for (int idx = tid; idx < c * c; idx += nt) {
      const int i = idx / c, j = idx % c;  // row i, column j
      const int pj = perm[j];
      const bool keep = lam[j] > eps && sv[pj] > 0.0;
      cd u = keep ? cscale(C[pj * c + i], 1.0 / sv[pj]) : czero();
      cd w = keep ? cconj(W[pj * c + i]) : czero();
      Af[i * c + j] = u;
      Ab[i * c + j] = w;
      un += cabs2(u);
      vn += cabs2(w);
    }
    un = block_sum(un, red);
    vn = block_sum(vn, red);
    const double iu = 1.0 / sqrt(un), iv = 1.0 / sqrt(vn);
    cd *Gf = orth + g.half_msg_off[h0];
    cd *Gb = orth + g.half_msg_off[h1];
    for (int idx = tid; idx < c * c; idx += nt) {
      const int i = idx / c, j = idx % c;
      cd af = czero(), ab = czero();
      for (int k = 0; k < c; ++k) {
        cfma(af, Qf[i * c + k], Af[k * c + j]);
        cfma(ab, Qb[i * c + k], Ab[k * c + j]);
      }
      Gf[idx] = cscale(af, iu);
      Gb[idx] = cscale(ab, iv);
    }
    __syncthreads();
  }
}

// One warp per edge (chi <= WARP_MAX_CHI): the same steps as
// vidal_edges_kernel on the warp's own slice of shared memory.
__host__ __device__ inline size_t warp_edge_bytes(int c) {
  return round16(WARP_ROTS * sizeof(Rot)) + round16(vidal_edge_bytes(c));
}

__global__ void __launch_bounds__(GAUGE_THREADS) vidal_edges_warp_kernel(dqz_graph_t g, const cd *__restrict__ n2e,
                                                                          double eps, cd *orth, double *lambdas,
                                                                          int max_chi,
                                                                          const int32_t *__restrict__ sel, int n_sel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  unsigned char *wbase = smem_raw + (size_t)wid * warp_edge_bytes(max_chi);
  Rot *rots = reinterpret_cast<Rot *>(wbase);
  unsigned char *base = wbase + round16(WARP_ROTS * sizeof(Rot));
  const int M2 = max_chi * max_chi;
  cd *Af = reinterpret_cast<cd *>(base);
  cd *Vf = Af + M2, *Ab = Vf + M2, *Vb = Ab + M2, *Qf = Vb + M2, *Qb = Qf + M2, *C = Qb + M2, *W = C + M2;
  double *wf = reinterpret_cast<double *>(W + M2);
  double *wb = wf + max_chi, *sv = wb + max_chi, *wif = sv + max_chi, *wib = wif + max_chi;
  int *perm = reinterpret_cast<int *>(wib + max_chi);
  const int total = sel ? n_sel : g.n_edges;
  for (int it = blockIdx.x * wpb + wid; it < total; it += gridDim.x * wpb) {
    const int e = sel ? sel[it] : it;
    const int h0 = g.edge_half[2 * e], h1 = g.edge_half[2 * e + 1];
    const int c = g.edge_chi[e];
    double *lam = lambdas + g.edge_lam_off[e];
    if (c > max_chi) {  // the caller's max_chi is below this bond: flag it
      if (lane == 0) lam[0] = __longlong_as_double(0x7ff8000000000000ll);
      continue;
    }
    const cd *mf = n2e + g.half_msg_off[h0];
    const cd *mb = n2e + g.half_msg_off[h1];
    for (int i = lane; i < c * c; i += 32) {
      Af[i] = mf[i];
      Ab[i] = mb[i];
    }
    __syncwarp();
    warp_herm_eigh(Af, c, Vf, c, c, wf, rots);
    warp_herm_eigh(Ab, c, Vb, c, c, wb, rots);
    sqrt_weights(wf, wif, c, eps, lane, 32);
    sqrt_weights(wb, wib, c, eps, lane, 32);
    __syncwarp();
    for (int idx = lane; idx < c * c; idx += 32) {
      const int i = idx / c, j = idx % c;
      cd sf = czero(), sif = czero(), sb = czero(), sib = czero();
      for (int k = 0; k < c; ++k) {
        cd pf = cmul(Vf[i * c + k], cconj(Vf[j * c + k]));
        cd pb = cmul(Vb[i * c + k], cconj(Vb[j * c + k]));
        sf = cadd(sf, cscale(pf, wf[k]));
        sif = cadd(sif, cscale(pf, wif[k]));
        sb = cadd(sb, cscale(pb, wb[k]));
        sib = cadd(sib, cscale(pb, wib[k]));
      }
      Af[idx] = sf;
      Qf[idx] = sif;
      Ab[idx] = sb;
      Qb[idx] = sib;
    }
    __syncwarp();
    // C = sqrt(m_f) sqrt(m_b)^T, column-major for the one-sided Jacobi.
    for (int idx = lane; idx < c * c; idx += 32) {
      const int i = idx / c, j = idx % c;
      cd acc = czero();
      for (int k = 0; k < c; ++k) cfma(acc, Af[i * c + k], Ab[j * c + k]);
      C[j * c + i] = acc;
    }
    __syncwarp();
    warp_hestenes(C, c, c, c, W, c, sv);
    warp_sort_desc(sv, c, perm);
    double nrm2 = 0.0;
    for (int j = lane; j < c; j += 32) nrm2 += sv[j] * sv[j];
    nrm2 = warp_sum(nrm2);
    const double inv_n = 1.0 / sqrt(nrm2);
    for (int j = lane; j < c; j += 32) lam[j] = safe_truncate(sv[perm[j]] * inv_n, eps);
    __syncwarp();
    double un = 0.0, vn = 0.0;
    for (int idx = lane; idx < c * c; idx += 32) {
      const int i = idx / c, j = idx % c;
      const int pj = perm[j];
      const bool keep = lam[j] > eps && sv[pj] > 0.0;
      cd u = keep ? cscale(C[pj * c + i], 1.0 / sv[pj]) : czero();
      cd w = keep ? cconj(W[pj * c + i]) : czero();
      Af[i * c + j] = u;
      Ab[i * c + j] = w;
      un += cabs2(u);
      vn += cabs2(w);
    }
    un = warp_sum(un);
    vn = warp_sum(vn);
    __syncwarp();
    const double iu = 1.0 / sqrt(un), iv = 1.0 / sqrt(vn);
    cd *Gf = orth + g.half_msg_off[h0];
    cd *Gb = orth + g.half_msg_off[h1];
    for (int idx = lane; idx < c * c; idx += 32) {
      const int i = idx / c, j = idx % c;
      cd af = czero(), ab = czero();
      for (int k = 0; k < c; ++k) {
        cfma(af, Qf[i * c + k], Af[k * c + j]);
        cfma(ab, Qb[i * c + k], Ab[k * c + j]);
      }
      Gf[idx] = cscale(af, iu);
      Gb[idx] = cscale(ab, iv);
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------------- absorb
__global__ void __launch_bounds__(GAUGE_THREADS) absorb_kernel(dqz_graph_t g, const cd *__restrict__ Tin,
                                                                const cd *__restrict__ orth, cd *Tout, int max_size,
                                                                cd *scratch, const int32_t *__restrict__ sel,
                                                                int n_sel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *red = reinterpret_cast<double *>(smem_raw);
  cd *bufA = scratch ? scratch + (long long)blockIdx.x * 2 * max_size
                     : reinterpret_cast<cd *>(smem_raw + 48 * sizeof(double));
  cd *bufB = bufA + max_size;
  const int total = sel ? n_sel : g.n_nodes;
  for (int it = blockIdx.x; it < total; it += gridDim.x) {
    const int v = sel ? sel[it] : it;
    NodeShape s;
    load_shape(g, v, s);
    const cd *T = Tin + g.node_off[v];
    for (long long i = threadIdx.x; i < s.size; i += blockDim.x) bufA[i] = T[i];
    __syncthreads();
    cd *cur = bufA, *nxt = bufB;
    long long L = 1;
    for (int f = 0; f < s.k; ++f) {
      const int q = s.dims[f];
      const long long R = s.size / L / q;
      const cd *G = orth + g.half_msg_off[s.half0 + f];
      // new[.., j, ..] = sum_a G[a][j] T[.., a, ..]
      mode_product<false>(cur, nxt, L, q, q, R, G, 1, q);
      __syncthreads();
      cd *t = cur;
      cur = nxt;
      nxt = t;
      L *= q;
    }
    double n2 = 0.0;
    for (long long i = threadIdx.x; i < s.size; i += blockDim.x) n2 += cabs2(cur[i]);
    n2 = block_sum(n2, red);
    const double inv = 1.0 / sqrt(n2);
    cd *O = Tout + g.node_off[v];
    for (long long i = threadIdx.x; i < s.size; i += blockDim.x) O[i] = cscale(cur[i], inv);
    __syncthreads();
  }
}

// Nodes too large for shared memory: one CTA per (node, j), j the output
// index of the node's first bond. X = sum_a orth_0[a][j] T[a, ..] (the first
// mode product restricted to j, T read through L2), then the other bonds'
// mode products on X in shared memory, each element computed as the
// whole-tensor mode products compute it; X is written unnormalised and its
// squared norm to partial[it * DQZ_MAX_CHI + j]. absorb_scale_kernel then
// divides each node by the square root of its partials' sum (j order).
__global__ void __launch_bounds__(GAUGE_THREADS) absorb_split_kernel(dqz_graph_t g, const cd *__restrict__ Tin,
                                                                      const cd *__restrict__ orth,
                                                                      cd *__restrict__ Tout, long long max_slice,
                                                                      double *partial,
                                                                      const int32_t *__restrict__ sel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *red = reinterpret_cast<double *>(smem_raw);
  cd *bufA = reinterpret_cast<cd *>(smem_raw + 48 * sizeof(double));
  cd *bufB = bufA + max_slice;
  const int it = blockIdx.x, j = blockIdx.y;
  const int v = sel ? sel[it] : it;
  NodeShape s;
  load_shape(g, v, s);
  const int c0 = s.k > 0 ? s.dims[0] : 1;
  if (j >= c0) return;
  const long long P0 = s.size / c0;
  const cd *T = Tin + g.node_off[v];
  if (s.k > 0) {
    const cd *G0 = orth + g.half_msg_off[s.half0];
    for (long long r = threadIdx.x; r < P0; r += blockDim.x) {
      cd acc = czero();
      for (int b = 0; b < c0; ++b) cfma(acc, G0[b * c0 + j], T[b * P0 + r]);
      bufA[r] = acc;
    }
  } else {
    for (long long r = threadIdx.x; r < P0; r += blockDim.x) bufA[r] = T[r];
  }
  __syncthreads();
  cd *cur = bufA, *nxt = bufB;
  long long L = 1;
  for (int f = 1; f < s.k; ++f) {
    const int q = s.dims[f];
    const long long R = P0 / L / q;
    mode_product<false>(cur, nxt, L, q, q, R, orth + g.half_msg_off[s.half0 + f], 1, q);
    __syncthreads();
    cd *t = cur;
    cur = nxt;
    nxt = t;
    L *= q;
  }
  double n2 = 0.0;
  cd *O = Tout + g.node_off[v] + (long long)j * P0;
  for (long long r = threadIdx.x; r < P0; r += blockDim.x) {
    n2 += cabs2(cur[r]);
    O[r] = cur[r];
  }
  n2 = block_sum(n2, red);
  if (threadIdx.x == 0) partial[(long long)it * DQZ_MAX_CHI + j] = n2;
}

__global__ void __launch_bounds__(GAUGE_THREADS) absorb_scale_kernel(dqz_graph_t g, cd *Tout,
                                                                      const double *__restrict__ partial,
                                                                      const int32_t *__restrict__ sel) {
  __shared__ double inv_sh;
  const int it = blockIdx.x;
  const int v = sel ? sel[it] : it;
  NodeShape s;
  load_shape(g, v, s);
  if (threadIdx.x == 0) {
    const int c0 = s.k > 0 ? s.dims[0] : 1;
    double n2 = 0.0;
    for (int j = 0; j < c0; ++j) n2 += partial[(long long)it * DQZ_MAX_CHI + j];
    inv_sh = 1.0 / sqrt(n2);
  }
  __syncthreads();
  const double inv = inv_sh;
  cd *O = Tout + g.node_off[v];
  for (long long i = threadIdx.x; i < s.size; i += blockDim.x) O[i] = cscale(O[i], inv);
}

// ---------------------------------------------------------- vidal distance
// partial[h] = trace norm of (R/tr R - ideal) for bond e of node v (h = (v,e)),
// one CTA per half-edge. R = Y^H Y with Y[x][a] = T[.., a@e, ..](x) *
// prod_{f != e} lambda_f[idx_f(x)] (the lambda^2-weighted reduced matrix). The
// bond slice is staged through shared memory VDT_CHUNK elements at a time
// (rows x padded columns, row stride cp + 1: conflict-free column reads); R
// is register-tiled: each thread accumulates a 4 x 4 tile of the upper
// triangle of R (tiles ti <= tj) over every `splits`-th row of the chunk, 16
// complex FMAs per 8 shared loads, and the splits' tiles are summed in index
// order at the end. The trace norm comes from the eigenvalues of the
// Hermitian matrix (herm_eigh without vectors).
constexpr int VDT_CHUNK = 2048;            // staged elements per chunk
constexpr int VDT_PART = GAUGE_THREADS * 16;  // split partial tiles (cd)

__host__ __device__ inline int vdt_cp(int c) { return (c + 3) & ~3; }
__host__ __device__ inline int vdt_rows(int c) {
  const int r = VDT_CHUNK / vdt_cp(c);
  return r < 1 ? 1 : r;
}
__host__ __device__ inline size_t vdt_union_elems(int c) {
  const size_t y = (size_t)vdt_rows(c) * (vdt_cp(c) + 1);
  return y > (size_t)VDT_PART ? y : (size_t)VDT_PART;
}
// eigh header | union(Y chunk, split partials) | row weights | R | w
__host__ __device__ inline size_t vdt_smem(int max_chi) {
  int rmax = 0;
  for (int c = 1; c <= max_chi; ++c) rmax = vdt_rows(c) > rmax ? vdt_rows(c) : rmax;
  size_t u = 0;
  for (int c = 1; c <= max_chi; ++c) u = vdt_union_elems(c) > u ? vdt_union_elems(c) : u;
  return round16(48 * sizeof(double) + (DQZ_MAX_CHI / 2 + 1) * sizeof(Rot)) + u * sizeof(cd) +
         round16((size_t)rmax * sizeof(double)) + (size_t)max_chi * max_chi * sizeof(cd) +
         (size_t)max_chi * sizeof(double);
}

__global__ void __launch_bounds__(GAUGE_THREADS) vidal_distance_kernel(dqz_graph_t g, const cd *__restrict__ Tall,
                                                                        const double *__restrict__ lambdas,
                                                                        double eps, double *partial, int max_chi,
                                                                        const int32_t *__restrict__ sel, int n_sel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *red = reinterpret_cast<double *>(smem_raw);
  cd *U = reinterpret_cast<cd *>(smem_raw + round16(48 * sizeof(double) + (DQZ_MAX_CHI / 2 + 1) * sizeof(Rot)));
  size_t umax = 0;
  int rmax = 0;
  for (int c = 1; c <= max_chi; ++c) {
    umax = vdt_union_elems(c) > umax ? vdt_union_elems(c) : umax;
    rmax = vdt_rows(c) > rmax ? vdt_rows(c) : rmax;
  }
  double *wrow = reinterpret_cast<double *>(U + umax);
  cd *Rm = reinterpret_cast<cd *>(reinterpret_cast<unsigned char *>(wrow) + round16((size_t)rmax * sizeof(double)));
  __shared__ cd trace_sh;
  __shared__ int count_sh;
  const int total = sel ? n_sel : g.n_halves;
  const int tid = threadIdx.x;
  for (int it = blockIdx.x; it < total; it += gridDim.x) {
    const int h = sel ? sel[it] : it;
    const int v = g.half_node[h];
    NodeShape s;
    load_shape(g, v, s);
    const int e = h - s.half0;
    const int ce = s.dims[e];
    const cd *T = Tall + g.node_off[v];
    const long long Re = s.stride[e];
    const long long P = s.size / ce;
    const double *lam[DQZ_MAX_DEGREE];
    for (int f = 0; f < s.k; ++f) lam[f] = lambdas + g.edge_lam_off[g.half_edge[s.half0 + f]];
    const int cp = vdt_cp(ce), ld = cp + 1, rows = vdt_rows(ce);
    const int nt = cp / 4, ntl = nt * (nt + 1) / 2;
    const int splits = GAUGE_THREADS / ntl;  // >= 1: ntl <= 136
    const int tile = tid % ntl, split = tid / ntl;
    const bool active = split < splits;
    int ti = 0, rem = tile;
    while (rem >= nt - ti) {
      rem -= nt - ti;
      ++ti;
    }
    const int tj = ti + rem;
    cd acc[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int m = 0; m < 4; ++m) acc[k][m] = czero();
    // 32-bit index arithmetic below 2^31 entries (64-bit division is a long
    // instruction sequence, and the staging runs it per entry)
    const bool small = s.size < (1ll << 31);
    const FastDiv fRe((unsigned)(small ? Re : 1));
    for (long long x0 = 0; x0 < P; x0 += rows) {
      const int nr = (int)((P - x0) < rows ? (P - x0) : rows);
      for (int xl = tid; xl < nr; xl += GAUGE_THREADS) {
        double wt = 1.0;
        if (small) {
          const unsigned x = (unsigned)(x0 + xl);
          const unsigned l = fRe.div(x), r = x - l * (unsigned)Re;
          const unsigned o0 = (l * (unsigned)ce) * (unsigned)Re + r;
          for (int f = 0; f < s.k; ++f) {
            if (f == e) continue;
            wt *= lam[f][(o0 / (unsigned)s.stride[f]) % (unsigned)s.dims[f]];
          }
        } else {
          const long long x = x0 + xl;
          const long long l = x / Re, r = x - l * Re;
          const long long o0 = (l * ce) * Re + r;
          for (int f = 0; f < s.k; ++f) {
            if (f == e) continue;
            wt *= lam[f][(int)((o0 / s.stride[f]) % s.dims[f])];
          }
        }
        wrow[xl] = wt;
      }
      __syncthreads();
      for (int q = tid; q < nr * cp; q += GAUGE_THREADS) {
        const int xl = q % nr, a = q / nr;
        cd y = czero();
        if (a < ce) {
          if (small) {
            const unsigned x = (unsigned)(x0 + xl);
            const unsigned l = fRe.div(x), r = x - l * (unsigned)Re;
            y = cscale(T[(l * (unsigned)ce + (unsigned)a) * (unsigned)Re + r], wrow[xl]);
          } else {
            const long long x = x0 + xl;
            const long long l = x / Re, r = x - l * Re;
            y = cscale(T[(l * ce + a) * Re + r], wrow[xl]);
          }
        }
        U[xl * ld + a] = y;
      }
      __syncthreads();
      if (active) {
        for (int xl = split; xl < nr; xl += splits) {
          const cd *row = U + xl * ld;
          cd yi[4], yj[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            yi[k] = row[4 * ti + k];
            yj[k] = row[4 * tj + k];
          }
#pragma unroll
          for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int m = 0; m < 4; ++m) cfmac(acc[k][m], yi[k], yj[m]);
        }
      }
      __syncthreads();
    }
    // the splits' tiles, summed in split order
    if (active) {
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int m = 0; m < 4; ++m) U[(split * ntl + tile) * 16 + k * 4 + m] = acc[k][m];
    }
    __syncthreads();
    for (int q = tid; q < ntl * 16; q += GAUGE_THREADS) {
      const int tl = q / 16, km = q % 16;
      cd sum = U[tl * 16 + km];
      for (int sp = 1; sp < splits; ++sp) sum = cadd(sum, U[(sp * ntl + tl) * 16 + km]);
      int a = 0, rr = tl;
      while (rr >= nt - a) {
        rr -= nt - a;
        ++a;
      }
      const int i = 4 * a + km / 4, j = 4 * (a + rr) + km % 4;
      if (i < ce && j < ce && i <= j) {
        Rm[i * ce + j] = sum;
        if (i < j) Rm[j * ce + i] = cconj(sum);
      }
    }
    __syncthreads();
    if (tid == 0) {
      cd tr = czero();
      for (int i = 0; i < ce; ++i) tr = cadd(tr, Rm[i * ce + i]);
      trace_sh = tr;
    }
    __syncthreads();
    const cd tr = trace_sh;
    for (int i = tid; i < ce * ce; i += blockDim.x) Rm[i] = cdiv(Rm[i], tr);
    __syncthreads();
    if (tid == 0) {
      int cnt = 0;
      for (int i = 0; i < ce; ++i) cnt += Rm[i * ce + i].x > eps ? 1 : 0;
      count_sh = cnt;
    }
    __syncthreads();
    const double idv = 1.0 / (double)count_sh;
    for (int i = tid; i < ce; i += blockDim.x)
      if (Rm[i * ce + i].x > eps) Rm[i * ce + i].x -= idv;
    __syncthreads();
    // the trace norm from the eigenvalues (tridiagonal reduction + implicit
    // QL; the staging area is free again for its vectors)
    const double t = herm_trace_norm(Rm, ce, ce, U, U + DQZ_MAX_CHI, reinterpret_cast<double *>(U + 2 * DQZ_MAX_CHI),
                                     reinterpret_cast<double *>(U + 3 * DQZ_MAX_CHI), red);
    if (tid == 0) partial[h] = t;
    __syncthreads();
  }
}

// One warp per half-edge (chi <= WARP_MAX_CHI). The bond slice is streamed
// through the warp's shared memory in chunks of VD_CHUNK rows as
// Y[x][a] = T[.., a@e, ..](x) * prod_{f != e} lambda_f[idx_f(x)], so that
// R = Y^H Y (the lambda^2-weighted reduced matrix) reads every tensor entry
// from L2 once; each lane accumulates up to VD_PAIRS entries (a' <= a) of R
// from the staged rows, and the trace norm comes from warp_herm_eigh.
constexpr int VD_CHUNK = 32;
constexpr int VD_PAIRS = (WARP_MAX_CHI * (WARP_MAX_CHI + 1) / 2 + 31) / 32;

__host__ __device__ inline size_t warp_vd_bytes(int c) {
  return round16(WARP_ROTS * sizeof(Rot)) + round16((size_t)c * c * sizeof(cd)) + round16((size_t)c * sizeof(double)) +
         round16(VD_CHUNK * sizeof(double)) + round16((size_t)VD_CHUNK * c * sizeof(cd));
}

__global__ void __launch_bounds__(GAUGE_THREADS, 3) vidal_distance_warp_kernel(
    dqz_graph_t g, const cd *__restrict__ Tall, const double *__restrict__ lambdas, double eps, double *partial,
    int max_chi, const int32_t *__restrict__ sel, int n_sel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  unsigned char *wbase = smem_raw + (size_t)wid * warp_vd_bytes(max_chi);
  Rot *rots = reinterpret_cast<Rot *>(wbase);
  unsigned char *q = wbase + round16(WARP_ROTS * sizeof(Rot));
  cd *Rm = reinterpret_cast<cd *>(q);
  q += round16((size_t)max_chi * max_chi * sizeof(cd));
  double *wv = reinterpret_cast<double *>(q);
  q += round16((size_t)max_chi * sizeof(double));
  double *wl = reinterpret_cast<double *>(q);
  q += round16(VD_CHUNK * sizeof(double));
  cd *Ys = reinterpret_cast<cd *>(q);
  const int total = sel ? n_sel : g.n_halves;
  for (int it = blockIdx.x * wpb + wid; it < total; it += gridDim.x * wpb) {
    const int h = sel ? sel[it] : it;
    const int v = g.half_node[h];
    NodeShape s;
    load_shape(g, v, s);
    const int e = h - s.half0;
    const int ce = s.dims[e];
    if (ce > max_chi || s.size >= (1ll << 31)) {  // outside the caller's bounds: flag it
      if (lane == 0) partial[h] = __longlong_as_double(0x7ff8000000000000ll);
      continue;
    }
    const int P = (int)(s.size / ce), Re = (int)s.stride[e];
    const cd *T = Tall + g.node_off[v];
    const int npair = ce * (ce + 1) / 2;
    int pa[VD_PAIRS], pb[VD_PAIRS];
    cd acc[VD_PAIRS];
#pragma unroll
    for (int j = 0; j < VD_PAIRS; ++j) {
      const int pi = lane + 32 * j;
      pa[j] = -1;
      pb[j] = 0;
      acc[j] = czero();
      if (pi < npair) {
        int ap = 0, rem = pi;
        while (rem >= ce - ap) {
          rem -= ce - ap;
          ++ap;
        }
        pa[j] = ap;
        pb[j] = ap + rem;
      }
    }
    for (int x0 = 0; x0 < P; x0 += VD_CHUNK) {
      const int nx = P - x0 < VD_CHUNK ? P - x0 : VD_CHUNK;
      if (lane < nx) {  // lambda weight (not squared) of row x0 + lane
        const int x = x0 + lane, l = x / Re, r = x - l * Re;
        const int o0 = l * ce * Re + r;  // offset with a_e = 0
        double wt = 1.0;
        for (int f = 0; f < s.k; ++f) {
          if (f == e) continue;
          const int idx = (o0 / (int)s.stride[f]) % s.dims[f];
          wt *= lambdas[g.edge_lam_off[g.half_edge[s.half0 + f]] + idx];
        }
        wl[lane] = wt;
      }
      __syncwarp();
      for (int t = lane; t < nx * ce; t += 32) {  // rows x fastest across lanes
        const int a = t / nx, jx = t - a * nx;
        const int x = x0 + jx, l = x / Re, r = x - l * Re;
        Ys[jx * ce + a] = cscale(T[(long long)(l * ce + a) * Re + r], wl[jx]);
      }
      __syncwarp();
      for (int jx = 0; jx < nx; ++jx) {
        const cd *row = Ys + jx * ce;
#pragma unroll
        for (int j = 0; j < VD_PAIRS; ++j)
          if (pa[j] >= 0) cfmac(acc[j], row[pa[j]], row[pb[j]]);
      }
      __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < VD_PAIRS; ++j)
      if (pa[j] >= 0) {
        Rm[pa[j] * ce + pb[j]] = acc[j];
        Rm[pb[j] * ce + pa[j]] = cconj(acc[j]);
      }
    __syncwarp();
    cd tr = czero();
    for (int i = 0; i < ce; ++i) tr = cadd(tr, Rm[i * ce + i]);
    int cnt = 0;
    for (int i = 0; i < ce; ++i) cnt += cdiv(Rm[i * ce + i], tr).x > eps ? 1 : 0;
    __syncwarp();
    for (int i = lane; i < ce * ce; i += 32) Rm[i] = cdiv(Rm[i], tr);
    __syncwarp();
    const double idv = 1.0 / (double)cnt;
    for (int i = lane; i < ce; i += 32)
      if (Rm[i * ce + i].x > eps) Rm[i * ce + i].x -= idv;
    __syncwarp();
    warp_herm_eigh(Rm, ce, nullptr, 0, ce, wv, rots);
    double t = 0.0;
    for (int i = lane; i < ce; i += 32) t += fabs(wv[i]);
    t = warp_sum(t);
    if (lane == 0) partial[h] = t;
    __syncwarp();
  }
}

// ---------------------------------------------------------- symmetric gauge
__global__ void __launch_bounds__(GAUGE_THREADS) symmetric_kernel(dqz_graph_t g, const cd *__restrict__ Tin,
                                                                   const double *__restrict__ lambdas, double eps,
                                                                   cd *Tout) {
  __shared__ double red[48];
  for (int v = blockIdx.x; v < g.n_nodes; v += gridDim.x) {
    NodeShape s;
    load_shape(g, v, s);
    const double *lam[DQZ_MAX_DEGREE];
    for (int f = 0; f < s.k; ++f) lam[f] = lambdas + g.edge_lam_off[g.half_edge[s.half0 + f]];
    const cd *T = Tin + g.node_off[v];
    cd *O = Tout + g.node_off[v];
    double n2 = 0.0;
    for (long long i = threadIdx.x; i < s.size; i += blockDim.x) {
      double wt = 1.0;
      for (int f = 0; f < s.k; ++f) wt *= sqrt(safe_truncate(lam[f][(i / s.stride[f]) % s.dims[f]], eps));
      n2 += cabs2(T[i]) * wt * wt;
    }
    n2 = block_sum(n2, red);
    const double inv = 1.0 / sqrt(n2);
    for (long long i = threadIdx.x; i < s.size; i += blockDim.x) {
      double wt = 1.0;
      for (int f = 0; f < s.k; ++f) wt *= sqrt(safe_truncate(lam[f][(i / s.stride[f]) % s.dims[f]], eps));
      O[i] = cscale(T[i], wt * inv);
    }
    __syncthreads();
  }
}

__global__ void lambdas_to_messages_kernel(dqz_graph_t g, const double *__restrict__ lambdas, cd *n2e, cd *e2n) {
  const int nh = g.n_halves;
  const int wpb = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int h = blockIdx.x * wpb + (threadIdx.x >> 5); h < nh; h += gridDim.x * wpb) {
    const int e = g.half_edge[h];
    if (e < 0) continue;
    const int c = g.edge_chi[e];
    const double *lam = lambdas + g.edge_lam_off[e];
    cd *a = n2e + g.half_msg_off[h];
    cd *b = e2n + g.half_msg_off[h];
    for (int i = lane; i < c * c; i += 32) {
      cd val = (i / c == i % c) ? mk(lam[i / c], 0.0) : czero();
      a[i] = val;
      b[i] = val;
    }
  }
}

// -------------------------------------------------------- density matrices
__global__ void __launch_bounds__(GAUGE_THREADS) density_kernel(dqz_graph_t g, const cd *__restrict__ Tall,
                                                                 const cd *__restrict__ e2n,
                                                                 const int32_t *__restrict__ nodes, int n_nodes,
                                                                 cd *rho, int max_size, cd *scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd *bufA = scratch ? scratch + (long long)blockIdx.x * 2 * max_size : reinterpret_cast<cd *>(smem_raw);
  cd *bufB = bufA + max_size;
  __shared__ cd rho_sh[DQZ_MAX_PHYS * DQZ_MAX_PHYS];
  __shared__ cd trace_sh;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int item = blockIdx.x; item < n_nodes; item += gridDim.x) {
    const int v = nodes[item];
    NodeShape s;
    load_shape(g, v, s);
    const cd *T = Tall + g.node_off[v];
    for (long long i = threadIdx.x; i < s.size; i += blockDim.x) bufA[i] = T[i];
    __syncthreads();
    cd *cur = bufA, *nxt = bufB;
    long long L = 1;
    for (int f = 0; f < s.k; ++f) {
      const int q = s.dims[f];
      const long long R = s.size / L / q;
      const cd *m = e2n + g.half_msg_off[s.half0 + f];
      mode_product<false>(cur, nxt, L, q, q, R, m, q, 1);
      __syncthreads();
      cd *t = cur;
      cur = nxt;
      nxt = t;
      L *= q;
    }
    const int d = s.d;
    const long long B = s.size / d;
    for (int p = warp; p < d * d; p += nw) {
      const int si = p / d, sj = p % d;
      cd acc = czero();
      for (long long b = lane; b < B; b += 32) cfmac(acc, T[b * d + sj], cur[b * d + si]);
      acc = warp_csum(acc);
      if (lane == 0) rho_sh[si * d + sj] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      cd tr = czero();
      for (int i = 0; i < d; ++i) tr = cadd(tr, rho_sh[i * d + i]);
      trace_sh = tr;
    }
    __syncthreads();
    cd *out = rho + (long long)item * DQZ_MAX_PHYS * DQZ_MAX_PHYS;
    for (int i = threadIdx.x; i < d * d; i += blockDim.x) out[i] = cdiv(rho_sh[i], trace_sh);
    __syncthreads();
  }
}

size_t eigh_smem(int max_chi) {
  return 48 * sizeof(double) + (DQZ_MAX_CHI / 2 + 1) * sizeof(Rot) + 4 * sizeof(int);
}

}  // namespace

extern "C" size_t dqz_vidal_edges_scratch_bytes(int32_t n_edges, int32_t max_chi) {
  size_t need = eigh_smem(max_chi) + vidal_edge_bytes(max_chi);
  if (need <= SMEM_LIMIT) return 0;
  int grid = n_edges < SCRATCH_GRID ? n_edges : SCRATCH_GRID;
  return (size_t)grid * vidal_edge_bytes(max_chi);
}

extern "C" int dqz_vidal_edges(const dqz_graph_t *g, const void *n2e, double eps, void *orth, double *lambdas,
                               int32_t max_chi, const int32_t *edges, int32_t n_sel, void *scratch,
                               cudaStream_t stream) {
  if (!g || !n2e || !orth || !lambdas) return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  if (edges && (n_sel < 0 || n_sel > g->n_edges)) return DQZ_ERR_ARG;
  const int total = edges ? n_sel : g->n_edges;
  if (total == 0) return DQZ_OK;
  if (max_chi <= WARP_MAX_CHI && dqz_get_tuning(DQZ_TUNE_GAUGE_PATH) != 2) {
    const size_t per = warp_edge_bytes(max_chi);
    int wpb = (int)(WARP_BLOCK_SMEM / per);
    wpb = wpb < 1 ? 1 : (wpb > GAUGE_THREADS / 32 ? GAUGE_THREADS / 32 : wpb);
    const int tuned = dqz_get_tuning(DQZ_TUNE_GAUGE_EDGE_WARPS);
    if (tuned > 0 && (size_t)tuned * per <= SMEM_LIMIT) wpb = tuned;
    DQZ_SMEM_ATTR_ONCE(vidal_edges_warp_kernel, SMEM_LIMIT);
    vidal_edges_warp_kernel<<<(total + wpb - 1) / wpb, 32 * wpb, wpb * per, stream>>>(
        *g, (const cd *)n2e, eps, (cd *)orth, lambdas, max_chi, edges, total);
    DQZ_CHECK_LAUNCH();
    return DQZ_OK;
  }
  size_t need = eigh_smem(max_chi) + vidal_edge_bytes(max_chi);
  const bool use_scratch = need > SMEM_LIMIT;
  if (use_scratch && !scratch) return DQZ_ERR_ARG;
  size_t smem = use_scratch ? eigh_smem(max_chi) : need;
  DQZ_SMEM_ATTR_ONCE(vidal_edges_kernel, SMEM_LIMIT);
  int grid = use_scratch ? (total < SCRATCH_GRID ? total : SCRATCH_GRID) : total;
  vidal_edges_kernel<<<grid, GAUGE_THREADS, smem, stream>>>(*g, (const cd *)n2e, eps, (cd *)orth, lambdas, max_chi,
                                                           use_scratch ? (unsigned char *)scratch : nullptr, edges,
                                                           total);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" size_t dqz_absorb_scratch_bytes(int32_t n_nodes, int32_t max_size) {
  size_t need = 48 * sizeof(double) + 2 * (size_t)max_size * sizeof(cd);
  if (need <= SMEM_LIMIT) return 0;
  int grid = n_nodes < SCRATCH_GRID ? n_nodes : SCRATCH_GRID;
  return (size_t)grid * 2 * (size_t)max_size * sizeof(cd);
}

extern "C" int dqz_absorb(const dqz_graph_t *g, const void *tensors_in, const void *orth, void *tensors_out,
                          int32_t max_size, const int32_t *nodes, int32_t n_sel, void *scratch,
                          cudaStream_t stream) {
  if (!g || !tensors_in || !orth || !tensors_out || max_size <= 0) return DQZ_ERR_ARG;
  if (nodes && (n_sel < 0 || n_sel > g->n_nodes)) return DQZ_ERR_ARG;
  const int total = nodes ? n_sel : g->n_nodes;
  if (total == 0) return DQZ_OK;
  size_t need = 48 * sizeof(double) + 2 * (size_t)max_size * sizeof(cd);
  const bool use_scratch = need > SMEM_LIMIT;
  if (use_scratch && !scratch) return DQZ_ERR_ARG;
  DQZ_SMEM_ATTR_ONCE(absorb_kernel, SMEM_LIMIT);
  int grid = use_scratch ? (total < SCRATCH_GRID ? total : SCRATCH_GRID) : total;
  absorb_kernel<<<grid, GAUGE_THREADS, use_scratch ? 48 * sizeof(double) : need, stream>>>(
      *g, (const cd *)tensors_in, (const cd *)orth, (cd *)tensors_out, max_size,
      use_scratch ? (cd *)scratch : nullptr, nodes, total);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" size_t dqz_absorb_split_scratch_bytes(int32_t n_nodes) {
  return (size_t)(n_nodes > 0 ? n_nodes : 0) * DQZ_MAX_CHI * sizeof(double);
}

extern "C" int dqz_absorb_split(const dqz_graph_t *g, const void *tensors_in, const void *orth, void *tensors_out,
                                int64_t max_slice, const int32_t *nodes, int32_t n_sel, void *scratch,
                                cudaStream_t stream) {
  if (!g || !tensors_in || !orth || !tensors_out || !scratch || max_slice <= 0) return DQZ_ERR_ARG;
  if (tensors_in == tensors_out) return DQZ_ERR_ARG;
  if (nodes && (n_sel < 0 || n_sel > g->n_nodes)) return DQZ_ERR_ARG;
  const int total = nodes ? n_sel : g->n_nodes;
  if (total == 0) return DQZ_OK;
  if (max_slice < DQZ_MAX_PHYS) max_slice = DQZ_MAX_PHYS;  // a node without bonds is its own slice
  const size_t smem = 48 * sizeof(double) + 2 * (size_t)max_slice * sizeof(cd);
  if (smem > SMEM_LIMIT) return DQZ_ERR_UNSUPPORTED;
  DQZ_SMEM_ATTR_ONCE(absorb_split_kernel, SMEM_LIMIT);
  absorb_split_kernel<<<dim3(total, DQZ_MAX_CHI), GAUGE_THREADS, smem, stream>>>(
      *g, (const cd *)tensors_in, (const cd *)orth, (cd *)tensors_out, (long long)max_slice, (double *)scratch, nodes);
  DQZ_CHECK_LAUNCH();
  absorb_scale_kernel<<<total, GAUGE_THREADS, 0, stream>>>(*g, (cd *)tensors_out, (const double *)scratch, nodes);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_vidal_distance(const dqz_graph_t *g, const void *tensors, const double *lambdas, double eps,
                                  double *partial, double *out, int32_t max_chi, int32_t max_slice,
                                  const int32_t *halves, int32_t n_sel, cudaStream_t stream) {
  if (!g || !tensors || !lambdas || !partial) return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  const int nh = g->n_halves;
  if (nh == 0 || g->n_edges == 0) return DQZ_ERR_ARG;
  if (halves && (n_sel < 0 || n_sel > nh)) return DQZ_ERR_ARG;
  const int total = halves ? n_sel : nh;
  if (total > 0) {
    if (max_chi <= WARP_MAX_CHI && dqz_get_tuning(DQZ_TUNE_GAUGE_PATH) != 2) {
      const size_t per = warp_vd_bytes(max_chi);
      int wpb = (int)(WARP_BLOCK_SMEM / per);
      wpb = wpb < 1 ? 1 : (wpb > GAUGE_THREADS / 32 ? GAUGE_THREADS / 32 : wpb);
      const int tuned = dqz_get_tuning(DQZ_TUNE_GAUGE_DIST_WARPS);
      if (tuned > 0 && (size_t)tuned * per <= SMEM_LIMIT) wpb = tuned;
      DQZ_SMEM_ATTR_ONCE(vidal_distance_warp_kernel, SMEM_LIMIT);
      vidal_distance_warp_kernel<<<(total + wpb - 1) / wpb, 32 * wpb, wpb * per, stream>>>(
          *g, (const cd *)tensors, lambdas, eps, partial, max_chi, halves, total);
    } else {
      const size_t smem = vdt_smem(max_chi);
      DQZ_SMEM_ATTR_ONCE(vidal_distance_kernel, SMEM_LIMIT);
      vidal_distance_kernel<<<total, GAUGE_THREADS, smem, stream>>>(*g, (const cd *)tensors, lambdas, eps, partial,
                                                                    max_chi, halves, total);
    }
    DQZ_CHECK_LAUNCH();
  }
  if (!out) return DQZ_OK;
  return dqz_reduce_sum(partial, nh, 1.0 / (2.0 * g->n_edges), out, stream);
}

extern "C" int dqz_symmetric_gauge(const dqz_graph_t *g, const void *tensors_in, const double *lambdas, double eps,
                                   void *tensors_out, cudaStream_t stream) {
  if (!g || !tensors_in || !lambdas || !tensors_out) return DQZ_ERR_ARG;
  if (g->n_nodes == 0) return DQZ_OK;
  symmetric_kernel<<<g->n_nodes, GAUGE_THREADS, 0, stream>>>(*g, (const cd *)tensors_in, lambdas, eps,
                                                              (cd *)tensors_out);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_lambdas_to_messages(const dqz_graph_t *g, const double *lambdas, void *n2e, void *e2n,
                                       int32_t max_chi, cudaStream_t stream) {
  if (!g || !lambdas || !n2e || !e2n) return DQZ_ERR_ARG;
  if (max_chi <= 0 || max_chi > DQZ_MAX_CHI) return DQZ_ERR_UNSUPPORTED;
  const int nh = g->n_halves;
  if (nh == 0) return DQZ_OK;
  lambdas_to_messages_kernel<<<(nh + 7) / 8, 256, 0, stream>>>(*g, lambdas, (cd *)n2e, (cd *)e2n);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" size_t dqz_density_scratch_bytes(int32_t n_nodes, int32_t max_size) {
  size_t need = 2 * (size_t)max_size * sizeof(cd);
  if (need <= SMEM_LIMIT) return 0;
  int grid = n_nodes < SCRATCH_GRID ? n_nodes : SCRATCH_GRID;
  return (size_t)grid * 2 * (size_t)max_size * sizeof(cd);
}

extern "C" int dqz_density_matrices(const dqz_graph_t *g, const void *tensors, const void *e2n,
                                    const int32_t *nodes, int32_t n_nodes, void *rho, int32_t max_size,
                                    void *scratch, cudaStream_t stream) {
  if (!g || !tensors || !e2n || !nodes || !rho || n_nodes < 0 || max_size <= 0) return DQZ_ERR_ARG;
  if (n_nodes == 0) return DQZ_OK;
  size_t need = 2 * (size_t)max_size * sizeof(cd);
  const bool use_scratch = need > SMEM_LIMIT;
  if (use_scratch && !scratch) return DQZ_ERR_ARG;
  DQZ_SMEM_ATTR_ONCE(density_kernel, SMEM_LIMIT);
  int grid = use_scratch ? (n_nodes < SCRATCH_GRID ? n_nodes : SCRATCH_GRID) : n_nodes;
  density_kernel<<<grid, GAUGE_THREADS, use_scratch ? 0 : need, stream>>>(
      *g, (const cd *)tensors, (const cd *)e2n, nodes, n_nodes, (cd *)rho, max_size,
      use_scratch ? (cd *)scratch : nullptr);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
