// CTA-cooperative small dense linear algebra in FP64 for libdqz:
//  * herm_eigh  -- parallel cyclic Jacobi for Hermitian n x n (n <= 128), the
//                  message eigendecompositions of tensor_ops.py:115-120 and the
//                  trace norm of tensor_ops.py:173 (Hermitian operand).
//  * hestenes   -- one-sided Jacobi SVD on the columns of an m x n matrix, the
//                  SVDs of tensor_ops.py:121 and :360.
//  * householder_qr / apply_q -- LAPACK-convention (zgeqr2 / zung2r) QR, the
//                  QR of tensor_ops.py:288.
//  * warp_herm_eigh / warp_hestenes / warp_sort_desc -- one-warp forms of the
//                  above for matrices up to 32 x 32.
// Pairs are scheduled with the round-robin (circle) ordering, so each step
// rotates n/2 disjoint index pairs at once.
#pragma once

#include "common.cuh"

namespace dqz {

struct Rot {
  int p, q;
  cd j00, j01, j10, j11;
};

// Pair i of round-robin step `step` for an even count np: (0, step+1) for
// i == 0, otherwise (step+i, step-i) modulo np-1, shifted by one.
// (step < np - 1 and i < np / 2, so each modulo is one conditional step.)
__device__ __forceinline__ void rr_pair(int step, int i, int np, int &p, int &q) {
  const int m = np - 1;
  if (i == 0) {
    p = 0;
    q = step + 1;
  } else {
    int a = step + i, b = step - i;
    if (a >= m) a -= m;
    if (b < 0) b += m;
    p = a + 1;
    q = b + 1;
  }
  if (p > q) {
    int t = p;
    p = q;
    q = t;
  }
}

// Unitary J = D R that diagonalises the Hermitian 2x2 [[a, c], [conj(c), b]]
// (a, b real): D = diag(c/|c|, 1), R the real Jacobi rotation of
// [[a, |c|], [|c|, b]]. Returns false when c is negligible.
// One reciprocal square root gives both 1/|c| (phase and tau) and no
// divisions by |c|; cos = 1/sqrt(1 + t^2) is another (FP64 division and
// square root are long instruction sequences, and this runs per pair and step).
__device__ __forceinline__ bool jacobi_rot(double a, double b, cd c, Rot &r) {
  const double ac2 = cabs2(c);
  if (!(ac2 > 1e-300)) return false;
  const double inv_ac = rsqrt(ac2);
  const double tau = (b - a) * 0.5 * inv_ac;
  const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
  const double cs = rsqrt(1.0 + t * t);
  const double sn = t * cs;
  const cd ph = mk(c.x * inv_ac, c.y * inv_ac);
  r.j00 = cscale(ph, cs);
  r.j01 = cscale(ph, sn);
  r.j10 = mk(-sn, 0.0);
  r.j11 = mk(cs, 0.0);
  return true;
}

// One Jacobi step's update A <- J^H A J on the 2 x 2 blocks of the step's
// index pairs (rows of pair P, columns of pair Q): each entry gets the column
// rotation of its column pair and then the row rotation of its row pair,
// exactly as a column pass followed by a row pass would apply them, but in one
// pass over A (one barrier less a step). Pairs are those of rr_pair; a pair's
// second index may be the padding index n (never rotated).
__device__ __forceinline__ void jacobi_block_update(cd *A, int lda, int n, int np, int step, const Rot *rots, int P,
                                                    int Q) {
  int p1, q1, p2, q2;
  rr_pair(step, P, np, p1, q1);
  rr_pair(step, Q, np, p2, q2);
  const Rot &r1 = rots[P], &r2 = rots[Q];
  const bool rot1 = r1.p >= 0, rot2 = r2.p >= 0;
  if (!rot1 && !rot2) return;
  const bool v1 = q1 < n, v2 = q2 < n;
  cd b00 = A[p1 * lda + p2];
  cd b01 = v2 ? A[p1 * lda + q2] : czero();
  cd b10 = v1 ? A[q1 * lda + p2] : czero();
  cd b11 = (v1 && v2) ? A[q1 * lda + q2] : czero();
  if (rot2) {  // columns (p2, q2): A J
    const cd n00 = cadd(cmul(b00, r2.j00), cmul(b01, r2.j10)), n01 = cadd(cmul(b00, r2.j01), cmul(b01, r2.j11));
    const cd n10 = cadd(cmul(b10, r2.j00), cmul(b11, r2.j10)), n11 = cadd(cmul(b10, r2.j01), cmul(b11, r2.j11));
    b00 = n00;
    b01 = n01;
    b10 = n10;
    b11 = n11;
  }
  if (rot1) {  // rows (p1, q1): J^H A
    const cd n00 = cadd(cmulc(r1.j00, b00), cmulc(r1.j10, b10)), n10 = cadd(cmulc(r1.j01, b00), cmulc(r1.j11, b10));
    const cd n01 = cadd(cmulc(r1.j00, b01), cmulc(r1.j10, b11)), n11 = cadd(cmulc(r1.j01, b01), cmulc(r1.j11, b11));
    b00 = n00;
    b01 = n01;
    b10 = n10;
    b11 = n11;
  }
  A[p1 * lda + p2] = b00;
  if (v2) A[p1 * lda + q2] = b01;
  if (v1) A[q1 * lda + p2] = b10;
  if (v1 && v2) A[q1 * lda + q2] = b11;
}

// Hermitian eigendecomposition. A (n x n, row-major, lda) is destroyed; on
// return w[i] holds eigenvalue i and column i of V (row-major, ldv) the
// matching eigenvector (unsorted); V may be null (eigenvalues only, the same
// values). rots: >= n/2+1 entries, red: 33 doubles, all in shared memory.
// The input is first made exactly Hermitian ((A + A^H) / 2, real diagonal):
// an anti-Hermitian rounding residual is invisible to the rotations, which
// read the upper triangle only, and would otherwise keep the off-diagonal
// norm above any relative stopping threshold. Convergence is measured on the
// upper triangle; a sweep that rotates nothing also ends the iteration.
static __device__ void herm_eigh(cd *A, int lda, cd *V, int ldv, int n, double *w, Rot *rots, double *red,
                          int max_sweeps = 40) {
  const int tid = threadIdx.x, nt = blockDim.x;
  __shared__ int rotated_sh;
  if (V)
    for (int i = tid; i < n * n; i += nt) V[(i / n) * ldv + (i % n)] = (i / n == i % n) ? mk(1.0, 0.0) : czero();
  for (int i = tid; i < n * n; i += nt) {
    const int r = i / n, c = i % n;
    if (r < c) {
      const cd u = A[r * lda + c], l = A[c * lda + r];
      const cd h = mk(0.5 * (u.x + l.x), 0.5 * (u.y - l.y));
      A[r * lda + c] = h;
      A[c * lda + r] = cconj(h);
    } else if (r == c) {
      A[r * lda + c].y = 0.0;
    }
  }
  __syncthreads();
  const int np = n + (n & 1);
  const int npairs = np / 2;
  if (n > 1) {
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
      // reset before the barriers inside block_sum; read after the last step
      if (tid == 0) rotated_sh = 0;
      double off = 0.0, dia = 0.0;
      for (int i = tid; i < n * n; i += nt) {
        int r = i / n, c = i % n;
        double v = cabs2(A[r * lda + c]);
        if (r == c)
          dia += v;
        else if (r < c)
          off += 2.0 * v;
      }
      off = block_sum(off, red);
      dia = block_sum(dia, red);
      if (off == 0.0 || off <= 1e-30 * dia) break;
      for (int step = 0; step < np - 1; ++step) {
        for (int i = tid; i < npairs; i += nt) {
          int p, q;
          rr_pair(step, i, np, p, q);
          Rot r;
          r.p = -1;
          r.q = q;
          if (q < n) {
            double a = A[p * lda + p].x, b = A[q * lda + q].x;
            cd c = A[p * lda + q];
            double ac2 = cabs2(c);
            if (ac2 > 0.0 && ac2 >= 1e-36 * (a * a + b * b) && jacobi_rot(a, b, c, r)) {
              r.p = p;
              rotated_sh = 1;
            }
          }
          rots[i] = r;
        }
        __syncthreads();
        // A <- J^H A J by 2 x 2 blocks, V <- V J on columns (p, q)
        for (int blk = tid; blk < npairs * npairs; blk += nt)
          jacobi_block_update(A, lda, n, np, step, rots, blk / npairs, blk % npairs);
        if (V)
          for (int idx = tid; idx < npairs * n; idx += nt) {
            const Rot &r = rots[idx / n];
            if (r.p < 0) continue;
            const int row = idx % n;
            const cd x = V[row * ldv + r.p], y = V[row * ldv + r.q];
            V[row * ldv + r.p] = cadd(cmul(x, r.j00), cmul(y, r.j10));
            V[row * ldv + r.q] = cadd(cmul(x, r.j01), cmul(y, r.j11));
          }
        __syncthreads();
      }
      if (!rotated_sh) break;
      __syncthreads();
    }
  }
  for (int i = tid; i < n; i += nt) w[i] = A[i * lda + i].x;
  __syncthreads();
}

// Sum of |eigenvalues| (the trace norm) of a Hermitian n x n matrix A
// (row-major, lda; destroyed), n <= 64. The eigenvalues without vectors, in
// far fewer CTA barriers than the Jacobi forms: Householder reduction to a
// real tridiagonal matrix (the lower-triangle steps of LAPACK's zhetd2: per
// column k, H = I - tau v v^H from x = A[k+1:, k], x' = tau A22 v,
// w = x' - tau^* (v^H x') v / 2, A22 -= w v^H + v w^H; five barriers a
// column), then every eigenvalue of the tridiagonal at once by bisection
// with Sturm counts, one thread each (Barth, Martin and Wilkinson, Numer.
// Math. 9 (1967) 386-393; implicit QL on one thread was ten times slower
// here). Scratch in shared memory: v, x (n complex
// each), d, e (n doubles each), red (33 doubles). The input must be Hermitian
// up to rounding (the imaginary parts of its diagonal are ignored).
static __device__ double herm_trace_norm(cd *A, int lda, int n, cd *v, cd *x, double *d, double *e, double *red) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  __shared__ cd tau_sh, scale_sh, s_sh;
  __shared__ int skip_sh;
  __shared__ double norm_sh;
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;  // length of the column below the diagonal
    double xn2 = 0.0;
    for (int i = 2 + tid; i <= m; i += nt) xn2 += cabs2(A[(long long)(k + i) * lda + k]);
    xn2 = block_sum(xn2, red);
    if (tid == 0) {
      const cd alpha = A[(long long)(k + 1) * lda + k];
      int skip = xn2 == 0.0 && alpha.y == 0.0;
      if (!skip) {
        const double beta = -copysign(sqrt(cabs2(alpha) + xn2), alpha.x);
        tau_sh = mk((beta - alpha.x) / beta, -alpha.y / beta);
        scale_sh = cdiv(mk(1.0, 0.0), mk(alpha.x - beta, alpha.y));
        A[(long long)(k + 1) * lda + k] = mk(beta, 0.0);
      }
      skip_sh = skip;
    }
    __syncthreads();
    if (skip_sh) continue;
    const cd tau = tau_sh, sc = scale_sh;
    for (int i = tid; i < m; i += nt) v[i] = i == 0 ? mk(1.0, 0.0) : cmul(A[(long long)(k + 1 + i) * lda + k], sc);
    __syncthreads();
    // x = tau A22 v, a warp per row
    for (int i = warp; i < m; i += nw) {
      const cd *row = A + (long long)(k + 1 + i) * lda + (k + 1);
      cd acc = czero();
      for (int j = lane; j < m; j += 32) cfma(acc, row[j], v[j]);
      acc = warp_csum(acc);
      if (lane == 0) x[i] = cmul(tau, acc);
    }
    __syncthreads();
    if (warp == 0) {  // s = v^H x
      cd acc = czero();
      for (int j = lane; j < m; j += 32) cfmac(acc, v[j], x[j]);
      acc = warp_csum(acc);
      if (lane == 0) s_sh = acc;
    }
    __syncthreads();
    const cd hs = cmul(mk(0.5 * tau.x, -0.5 * tau.y), s_sh);  // tau^* s / 2
    for (int i = tid; i < m; i += nt) x[i] = csub(x[i], cmul(hs, v[i]));
    __syncthreads();
    for (int idx = tid; idx < m * m; idx += nt) {
      const int i = idx / m, j = idx - i * m;
      cd *a = A + (long long)(k + 1 + i) * lda + (k + 1 + j);
      *a = csub(*a, cadd(cmul(x[i], cconj(v[j])), cmul(v[i], cconj(x[j]))));
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) {
    d[i] = A[(long long)i * lda + i].x;
    e[i] = i + 1 < n ? sqrt(cabs2(A[(long long)(i + 1) * lda + i])) : 0.0;
  }
  __syncthreads();
  // eigenvalue j by bisection on thread j: Sturm counts (negative pivots of
  // T - x I = L D L^T) against the Gershgorin interval, halved until it is a
  // few ulps wide (at most 80 halvings)
  if (tid < n) {
    double lo = 0.0, hi = 0.0;
    for (int i = 0; i < n; ++i) {
      const double r = (i > 0 ? e[i - 1] : 0.0) + (i + 1 < n ? e[i] : 0.0);
      lo = i == 0 ? d[i] - r : fmin(lo, d[i] - r);
      hi = i == 0 ? d[i] + r : fmax(hi, d[i] + r);
    }
    const double span = fmax(fabs(lo), fabs(hi));
    const double pivmin = 1e-300 + 2.220446049250313e-16 * 2.220446049250313e-16 * span * span;
    for (int it = 0; it < 80 && hi - lo > 4.0 * 2.220446049250313e-16 * span; ++it) {
      const double mid = 0.5 * (lo + hi);
      int count = 0;
      double q = 1.0;
      for (int i = 0; i < n; ++i) {
        q = d[i] - mid - (i > 0 ? e[i - 1] * e[i - 1] / q : 0.0);
        if (fabs(q) < pivmin) q = -pivmin;
        count += q < 0.0;
      }
      if (count <= tid)
        lo = mid;
      else
        hi = mid;
    }
    x[tid].x = 0.5 * (lo + hi);
  }
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int i = 0; i < n; ++i) t += fabs(x[i].x);
    norm_sh = t;
  }
  __syncthreads();
  return norm_sh;
}

// One-sided Jacobi SVD on the columns of A (m x n, column-major, lda), m >= n
// is not required but only min(m, n) columns come out non-zero when m < n.
// On return column j of A is s_j u_j, V (n x n, column-major, ldv) holds the
// right singular vectors, s[j] = |A_j| (unsorted). One warp rotates a pair.
// Columns whose squared norm falls to (m eps)^2 ||A||_F^2 are numerically
// null: they take part in no rotation (their mutual orthogonality is rounding
// noise and never settles) and are returned with s[j] = 0.
__host__ __device__ inline double hestenes_null_scale(int m) {
  const double t = (double)(m > 1 ? m : 1) * 2.220446049250313e-16;
  return t * t;
}

static __device__ void hestenes(cd *A, int lda, int m, int n, cd *V, int ldv, double *s, int *flag, double *red,
                         int max_sweeps = 60) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  for (int i = tid; i < n * n; i += nt) V[(i / n) * ldv + (i % n)] = (i / n == i % n) ? mk(1.0, 0.0) : czero();
  const double tol = 1.1e-16 * sqrt((double)(m > 1 ? m : 1)) * 2.0;
  const int np = n + (n & 1);
  const int npairs = np / 2;
  double fro = 0.0;
  for (int i = tid; i < m * n; i += nt) fro += cabs2(A[(long long)(i / m) * lda + (i % m)]);
  const double null_thr = hestenes_null_scale(m) * block_sum(fro, red);
  // With more pairs per round than warps, each 16-lane half of a warp takes a
  // pair, so a warp's two pairs run side by side instead of one after the other.
  const bool half = npairs > nw;
  const int hw = half ? lane >> 4 : 0, hl = half ? lane & 15 : lane, ls = half ? 16 : 32, per = half ? 2 : 1;
  if (n > 1) {
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
      if (tid == 0) *flag = 0;
      __syncthreads();
      for (int step = 0; step < np - 1; ++step) {
        for (int ib = warp * per; ib < npairs; ib += nw * per) {  // warp-uniform trip count
          const int i = ib + hw;
          int p = 0, q = n;
          if (i < npairs) rr_pair(step, i, np, p, q);
          const bool live = q < n;
          cd *ap = A + (long long)p * lda, *aq = A + (long long)(live ? q : p) * lda;
          double al = 0.0, be = 0.0;
          cd ga = czero();
          if (live)
            for (int r = hl; r < m; r += ls) {
              cd x = ap[r], y = aq[r];
              al += cabs2(x);
              be += cabs2(y);
              cfmac(ga, x, y);
            }
          if (half) {
            al = half_sum(al);
            be = half_sum(be);
            ga = mk(half_sum(ga.x), half_sum(ga.y));
          } else {
            al = warp_sum(al);
            be = warp_sum(be);
            ga = warp_csum(ga);
          }
          if (!live || !(al > null_thr) || !(be > null_thr) || !(cabs2(ga) > tol * tol * al * be)) continue;
          Rot r;
          if (!jacobi_rot(al, be, ga, r)) continue;
          if (hl == 0) *flag = 1;
          for (int k = hl; k < m; k += ls) {
            cd x = ap[k], y = aq[k];
            ap[k] = cadd(cmul(x, r.j00), cmul(y, r.j10));
            aq[k] = cadd(cmul(x, r.j01), cmul(y, r.j11));
          }
          cd *vp = V + (long long)p * ldv, *vq = V + (long long)q * ldv;
          for (int k = hl; k < n; k += ls) {
            cd x = vp[k], y = vq[k];
            vp[k] = cadd(cmul(x, r.j00), cmul(y, r.j10));
            vq[k] = cadd(cmul(x, r.j01), cmul(y, r.j11));
          }
        }
        __syncthreads();
      }
      if (*flag == 0) break;
      __syncthreads();
    }
  }
  for (int j = warp; j < n; j += nw) {
    double t = 0.0;
    for (int r = lane; r < m; r += 32) t += cabs2(A[(long long)j * lda + r]);
    t = warp_sum(t);
    if (lane == 0) s[j] = t > null_thr ? sqrt(t) : 0.0;
  }
  __syncthreads();
}

// perm[j] = index of the j-th largest s (stable). n <= blockDim.
static __device__ void sort_desc(const double *s, int n, int *perm) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    int rank = 0;
    double sj = s[j];
    for (int i = 0; i < n; ++i) {
      double si = s[i];
      if (si > sj || (si == sj && i < j)) ++rank;
    }
    perm[rank] = j;
  }
  __syncthreads();
}

// Completes the columns of U (m x ncol, column-major, ldu) flagged in
// `null_col` to an orthonormal set: each flagged column becomes the first unit
// vector e_c, orthogonalised (twice) against all accepted columns, that keeps
// norm > 0.5. Run by warp 0; `acc` must hold the non-null flags on entry.
static __device__ void complete_orthonormal(cd *U, int ldu, int m, int ncol, int *acc) {
  const int lane = threadIdx.x & 31;
  if ((threadIdx.x >> 5) == 0) {
    int cand = 0;
    for (int j = 0; j < ncol; ++j) {
      if (acc[j]) continue;
      cd *uj = U + (long long)j * ldu;
      bool done = false;
      while (!done && cand < m) {
        for (int r = lane; r < m; r += 32) uj[r] = (r == cand) ? mk(1.0, 0.0) : czero();
        __syncwarp();
        for (int pass = 0; pass < 2; ++pass) {
          for (int i = 0; i < ncol; ++i) {
            if (!acc[i]) continue;
            const cd *ui = U + (long long)i * ldu;
            cd dot = czero();
            for (int r = lane; r < m; r += 32) cfmac(dot, ui[r], uj[r]);
            dot = warp_csum(dot);
            for (int r = lane; r < m; r += 32) uj[r] = csub(uj[r], cmul(ui[r], dot));
            __syncwarp();
          }
        }
        double nn = 0.0;
        for (int r = lane; r < m; r += 32) nn += cabs2(uj[r]);
        nn = warp_sum(nn);
        ++cand;
        if (nn > 0.25) {
          double inv = 1.0 / sqrt(nn);
          for (int r = lane; r < m; r += 32) uj[r] = cscale(uj[r], inv);
          __syncwarp();
          if (lane == 0) acc[j] = 1;
          __syncwarp();
          done = true;
        }
      }
    }
  }
  __syncthreads();
}

// LAPACK-convention Householder QR of A (M x K, column-major, ld = M):
// H_j = I - tau_j v_j v_j^H, v_j[j] = 1, v_j below the diagonal of column j,
// R on and above the diagonal, beta real (zlarfg). H_j^H is applied to the
// trailing columns (zgeqr2).
static __device__ void householder_qr(cd *A, int M, int K, cd *tau, double *red) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int kk = M < K ? M : K;
  for (int j = 0; j < kk; ++j) {
    cd *col = A + (long long)j * M;
    double s = 0.0;
    for (int r = j + 1 + tid; r < M; r += nt) s += cabs2(col[r]);
    s = block_sum(s, red);
    cd alpha = col[j];
    cd t;
    if (s == 0.0 && alpha.y == 0.0) {
      t = czero();
    } else {
      double beta = -copysign(sqrt(cabs2(alpha) + s), alpha.x);
      t = mk((beta - alpha.x) / beta, -alpha.y / beta);
      cd sc = cdiv(mk(1.0, 0.0), mk(alpha.x - beta, alpha.y));
      for (int r = j + 1 + tid; r < M; r += nt) col[r] = cmul(col[r], sc);
      __syncthreads();
      if (tid == 0) col[j] = mk(beta, 0.0);
    }
    if (tid == 0) tau[j] = t;
    __syncthreads();
    if (t.x != 0.0 || t.y != 0.0) {
      for (int c = j + 1 + warp; c < K; c += nw) {
        cd *ac = A + (long long)c * M;
        cd w = czero();
        if (lane == 0) w = ac[j];
        for (int r = j + 1 + lane; r < M; r += 32) cfmac(w, col[r], ac[r]);
        w = warp_csum(w);
        cd f = cmulc(t, w);  // conj(tau) * w
        if (lane == 0) ac[j] = csub(ac[j], f);
        for (int r = j + 1 + lane; r < M; r += 32) ac[r] = csub(ac[r], cmul(col[r], f));
      }
    }
    __syncthreads();
  }
}

// The same factorisation (same reflector convention) with one barrier per
// column: warp w owns the columns c with c % (warps) == w. After applying
// reflector j to its columns, the owner of column j + 1 builds reflector j + 1
// from that column at once (norm by a warp reduction, zlarfg's beta and tau),
// so the next barrier publishes both. For matrices in shared memory.
__device__ __forceinline__ void qr_make_reflector(cd *A, int M, int j, cd *tau) {
  const int lane = threadIdx.x & 31;
  cd *col = A + (long long)j * M;
  double s = 0.0;
  for (int r = j + 1 + lane; r < M; r += 32) s += cabs2(col[r]);
  s = warp_sum(s);
  const cd alpha = col[j];
  cd t = czero();
  if (!(s == 0.0 && alpha.y == 0.0)) {
    const double beta = -copysign(sqrt(cabs2(alpha) + s), alpha.x);
    t = mk((beta - alpha.x) / beta, -alpha.y / beta);
    const cd sc = cdiv(mk(1.0, 0.0), mk(alpha.x - beta, alpha.y));
    for (int r = j + 1 + lane; r < M; r += 32) col[r] = cmul(col[r], sc);
    __syncwarp();
    if (lane == 0) col[j] = mk(beta, 0.0);
  }
  if (lane == 0) tau[j] = t;
  __syncwarp();
}

static __device__ void householder_qr_owned(cd *A, int M, int K, cd *tau) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int kk = M < K ? M : K;
  if (kk > 0 && warp == 0) qr_make_reflector(A, M, 0, tau);
  __syncthreads();
  for (int j = 0; j < kk; ++j) {
    const cd t = tau[j];
    const cd *v = A + (long long)j * M;
    for (int c = j + 1 + ((warp - (j + 1) % nw + nw) % nw); c < K; c += nw) {  // this warp's columns > j
      if (t.x != 0.0 || t.y != 0.0) {
        cd *ac = A + (long long)c * M;
        cd w = czero();
        if (lane == 0) w = ac[j];
        for (int r = j + 1 + lane; r < M; r += 32) cfmac(w, v[r], ac[r]);
        w = warp_csum(w);
        const cd f = cmulc(t, w);  // conj(tau) * w
        if (lane == 0) ac[j] = csub(ac[j], f);
        for (int r = j + 1 + lane; r < M; r += 32) ac[r] = csub(ac[r], cmul(v[r], f));
        __syncwarp();
      }
      if (c == j + 1 && j + 1 < kk) qr_make_reflector(A, M, j + 1, tau);
    }
    __syncthreads();
  }
}

// X <- Q X with Q = H_0 ... H_{kk-1} from householder_qr; X is M x p,
// column-major (ldx).
static __device__ void apply_q(const cd *A, int M, int kk, const cd *tau, cd *X, int ldx, int p) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = kk - 1; j >= 0; --j) {
    cd t = tau[j];
    if (t.x != 0.0 || t.y != 0.0) {
      const cd *v = A + (long long)j * M;
      for (int c = warp; c < p; c += nw) {
        cd *xc = X + (long long)c * ldx;
        cd w = czero();
        if (lane == 0) w = xc[j];
        for (int r = j + 1 + lane; r < M; r += 32) cfmac(w, v[r], xc[r]);
        w = warp_csum(w);
        cd f = cmul(t, w);
        if (lane == 0) xc[j] = csub(xc[j], f);
        for (int r = j + 1 + lane; r < M; r += 32) xc[r] = csub(xc[r], cmul(v[r], f));
      }
    }
    __syncthreads();
  }
}

// hestenes on Z (zr x kk, column-major, ld zr, zr >= kk) with QR
// preconditioning: Z = Q R (Householder), one-sided Jacobi on X = R^H
// (R^H = U_x S V_x^H, so Z = (Q V_x) S U_x^H). The columns of R^H start
// closer to orthogonal than Z's, and the Jacobi iteration needs about half
// the sweeps on the graded cores of the simple update. Same contract as
// hestenes(Z, zr, zr, kk, V, kk, ...): on return column j of Z is s_j u_j (zero
// for a numerically null s_j), V (kk x kk, ld kk) holds orthonormal right
// singular vectors (null columns completed), s unsorted. V must have room for
// zr x kk entries; X (kk x kk) and tau (kk) are scratch; acc (kk ints) is
// overwritten. All in shared memory.
static __device__ void hestenes_qr(cd *Z, int zr, int kk, cd *V, cd *X, cd *tau, double *s, int *flag, int *acc,
                                   double *red) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  householder_qr_owned(Z, zr, kk, tau);
  for (int idx = tid; idx < kk * kk; idx += nt) {  // X = R^H
    const int i = idx % kk, j = idx / kk;
    X[idx] = j <= i ? cconj(Z[j + (long long)i * zr]) : czero();
  }
  __syncthreads();
  hestenes(X, kk, kk, kk, V, kk, s, flag, red);  // X = U_x S, V = V_x
  // V_x (ld kk) spread to ld zr with zero rows kk..zr-1, last column first (new
  // positions lie at or after the old ones); one warp, kk <= 64 (two rows a lane)
  if (warp == 0 && zr != kk) {
    for (int j = kk - 1; j >= 0; --j) {
      const cd v0 = lane < kk ? V[lane + (long long)j * kk] : czero();
      const cd v1 = lane + 32 < kk ? V[lane + 32 + (long long)j * kk] : czero();
      __syncwarp();
      for (int i = lane; i < zr; i += 32) V[i + (long long)j * zr] = i < kk ? (i < 32 ? v0 : v1) : czero();
      __syncwarp();
    }
  }
  __syncthreads();
  apply_q(Z, zr, kk, tau, V, zr, kk);  // V = Q [V_x; 0] = U_Z
  for (int idx = tid; idx < zr * kk; idx += nt) Z[idx] = cscale(V[idx], s[idx / zr]);
  __syncthreads();
  for (int idx = tid; idx < kk * kk; idx += nt) {  // V = U_x (normalised columns of X)
    const double sj = s[idx / kk];
    V[idx] = sj > 0.0 ? cscale(X[idx], 1.0 / sj) : czero();
  }
  for (int j = tid; j < kk; j += nt) acc[j] = s[j] > 0.0 ? 1 : 0;
  __syncthreads();
  complete_orthonormal(V, kk, kk, kk, acc);
}

// ------------------------------------------------------------------ warp
// Warp-synchronous forms for small matrices (n <= 32): one warp owns a
// matrix in its own shared memory, so phases are separated by __syncwarp
// only and many matrices proceed per SM at once. Same Hermitisation,
// rotations, pair schedule and stopping rules as the CTA forms above.

// Hermitian eigendecomposition (herm_eigh). V may be null (eigenvalues only).
// rots: >= n/2+1 entries of the warp's shared memory.
static __device__ void warp_herm_eigh(cd *A, int lda, cd *V, int ldv, int n, double *w, Rot *rots,
                                      int max_sweeps = 40) {
  const int lane = threadIdx.x & 31;
  if (V)
    for (int i = lane; i < n * n; i += 32) V[(i / n) * ldv + (i % n)] = (i / n == i % n) ? mk(1.0, 0.0) : czero();
  for (int i = lane; i < n * n; i += 32) {
    const int r = i / n, c = i % n;
    if (r < c) {
      const cd u = A[r * lda + c], l = A[c * lda + r];
      const cd h = mk(0.5 * (u.x + l.x), 0.5 * (u.y - l.y));
      A[r * lda + c] = h;
      A[c * lda + r] = cconj(h);
    } else if (r == c) {
      A[r * lda + c].y = 0.0;
    }
  }
  __syncwarp();
  const int np = n + (n & 1);
  const int npairs = np / 2;
  if (n > 1) {
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
      double off = 0.0, dia = 0.0;
      for (int i = lane; i < n * n; i += 32) {
        int r = i / n, c = i % n;
        double v = cabs2(A[r * lda + c]);
        if (r == c)
          dia += v;
        else if (r < c)
          off += 2.0 * v;
      }
      off = warp_sum(off);
      dia = warp_sum(dia);
      if (off == 0.0 || off <= 1e-30 * dia) break;
      bool rotated = false;
      for (int step = 0; step < np - 1; ++step) {
        if (lane < npairs) {
          int p, q;
          rr_pair(step, lane, np, p, q);
          Rot r;
          r.p = -1;
          r.q = q;
          if (q < n) {
            double a = A[p * lda + p].x, b = A[q * lda + q].x;
            cd c = A[p * lda + q];
            double ac2 = cabs2(c);
            if (ac2 > 0.0 && ac2 >= 1e-36 * (a * a + b * b) && jacobi_rot(a, b, c, r)) {
              r.p = p;
              rotated = true;
            }
          }
          rots[lane] = r;
        }
        __syncwarp();
        for (int blk = lane; blk < npairs * npairs; blk += 32)
          jacobi_block_update(A, lda, n, np, step, rots, blk / npairs, blk % npairs);
        if (V)
          for (int idx = lane; idx < npairs * n; idx += 32) {
            const Rot &r = rots[idx / n];
            if (r.p < 0) continue;
            const int row = idx % n;
            const cd x = V[row * ldv + r.p], y = V[row * ldv + r.q];
            V[row * ldv + r.p] = cadd(cmul(x, r.j00), cmul(y, r.j10));
            V[row * ldv + r.q] = cadd(cmul(x, r.j01), cmul(y, r.j11));
          }
        __syncwarp();
      }
      if (!__any_sync(0xffffffffu, rotated)) break;
    }
  }
  for (int i = lane; i < n; i += 32) w[i] = A[i * lda + i].x;
  __syncwarp();
}

// One-sided Jacobi SVD (hestenes) of A (m x n, column-major, lda); lane i
// rotates pair i of each round-robin step, looping over the rows itself.
// Same null-column rule as hestenes.
static __device__ void warp_hestenes(cd *A, int lda, int m, int n, cd *V, int ldv, double *s, int max_sweeps = 60) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < n * n; i += 32) V[(i / n) * ldv + (i % n)] = (i / n == i % n) ? mk(1.0, 0.0) : czero();
  const double tol = 1.1e-16 * sqrt((double)(m > 1 ? m : 1)) * 2.0;
  const int np = n + (n & 1);
  const int npairs = np / 2;
  double fro = 0.0;
  for (int i = lane; i < m * n; i += 32) fro += cabs2(A[(long long)(i / m) * lda + (i % m)]);
  const double null_thr = hestenes_null_scale(m) * warp_sum(fro);
  __syncwarp();
  // lpp consecutive lanes share a column pair (rows strided by lpp, sums over
  // the group by xor shuffles): all 32 lanes work when a round has few pairs.
  int lpp = 32;
  while (lpp > 1 && lpp * npairs > 32) lpp >>= 1;
  const int grp = lane / lpp, sub = lane % lpp, ppass = 32 / lpp;
  if (n > 1) {
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
      bool rotated = false;
      for (int step = 0; step < np - 1; ++step) {
        for (int i0 = 0; i0 < npairs; i0 += ppass) {  // warp-uniform trip count
          const int i = i0 + grp;
          int p = 0, q = n;
          if (i < npairs) rr_pair(step, i, np, p, q);
          const bool live = q < n;
          cd *ap = A + (long long)p * lda, *aq = A + (long long)(live ? q : p) * lda;
          double al = 0.0, be = 0.0;
          cd ga = czero();
          if (live)
            for (int r = sub; r < m; r += lpp) {
              cd x = ap[r], y = aq[r];
              al += cabs2(x);
              be += cabs2(y);
              cfmac(ga, x, y);
            }
          for (int o = lpp >> 1; o > 0; o >>= 1) {
            al += __shfl_xor_sync(0xffffffffu, al, o);
            be += __shfl_xor_sync(0xffffffffu, be, o);
            ga.x += __shfl_xor_sync(0xffffffffu, ga.x, o);
            ga.y += __shfl_xor_sync(0xffffffffu, ga.y, o);
          }
          Rot rt;
          if (live && al > null_thr && be > null_thr && cabs2(ga) > tol * tol * al * be && jacobi_rot(al, be, ga, rt)) {
            rotated = true;
            for (int k = sub; k < m; k += lpp) {
              cd x = ap[k], y = aq[k];
              ap[k] = cadd(cmul(x, rt.j00), cmul(y, rt.j10));
              aq[k] = cadd(cmul(x, rt.j01), cmul(y, rt.j11));
            }
            cd *vp = V + (long long)p * ldv, *vq = V + (long long)q * ldv;
            for (int k = sub; k < n; k += lpp) {
              cd x = vp[k], y = vq[k];
              vp[k] = cadd(cmul(x, rt.j00), cmul(y, rt.j10));
              vq[k] = cadd(cmul(x, rt.j01), cmul(y, rt.j11));
            }
          }
        }
        __syncwarp();
      }
      if (!__any_sync(0xffffffffu, rotated)) break;
    }
  }
  for (int j = lane; j < n; j += 32) {
    double t = 0.0;
    for (int r = 0; r < m; ++r) t += cabs2(A[(long long)j * lda + r]);
    s[j] = t > null_thr ? sqrt(t) : 0.0;
  }
  __syncwarp();
}

// perm[j] = index of the j-th largest s (stable), n <= 32, by one warp.
static __device__ void warp_sort_desc(const double *s, int n, int *perm) {
  const int lane = threadIdx.x & 31;
  if (lane < n) {
    int rank = 0;
    double sj = s[lane];
    for (int i = 0; i < n; ++i) {
      double si = s[i];
      if (si > sj || (si == sj && i < lane)) ++rank;
    }
    perm[rank] = lane;
  }
  __syncwarp();
}

}  // namespace dqz
