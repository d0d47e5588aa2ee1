// Batched reduced QR (FP64 / complex128) with the LAPACK conventions of the
// simple update's QR (tensor_ops.py:288): Householder reflectors as in
// zgeqr2, Q formed from them as in zung2r. One CTA per matrix; the matrix
// and the columns of Q being formed live in a per-CTA slice of a global
// scratch area (a 512 x 32 complex matrix is 256 KB, above shared memory).
#include "linalg.cuh"

using namespace dqz;

namespace {

constexpr int QR_THREADS = 256;
constexpr int QR_GRID_MAX = 148 * 4;

__host__ __device__ inline size_t qr_scratch_per_matrix(int m, int k) {
  const int kk = m < k ? m : k;
  return ((size_t)m * k + (size_t)m * kk) * sizeof(cd);
}

__global__ void __launch_bounds__(QR_THREADS) qr_batched_kernel(const cd *__restrict__ A, long long batch, int m,
                                                                int k, cd *Q, cd *R, cd *scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd *tau = reinterpret_cast<cd *>(smem_raw);
  const int kk = m < k ? m : k;
  const int tid = threadIdx.x, nt = blockDim.x;
  cd *W = scratch + (long long)blockIdx.x * (qr_scratch_per_matrix(m, k) / sizeof(cd));
  cd *X = W + (long long)m * k;
  for (long long b = blockIdx.x; b < batch; b += gridDim.x) {
    const cd *Ab = A + b * (long long)m * k;
    for (int idx = tid; idx < m * k; idx += nt) {  // row-major in, column-major work
      const int i = idx / k, j = idx - (idx / k) * k;
      W[(long long)j * m + i] = Ab[idx];
    }
    __syncthreads();
    householder_qr_owned(W, m, k, tau);
    cd *Rb = R + b * (long long)kk * k;
    for (int idx = tid; idx < kk * k; idx += nt) {
      const int i = idx / k, j = idx - (idx / k) * k;
      Rb[idx] = j >= i ? W[(long long)j * m + i] : czero();
    }
    for (int idx = tid; idx < m * kk; idx += nt) X[idx] = (idx % m == idx / m) ? mk(1.0, 0.0) : czero();
    __syncthreads();
    apply_q(W, m, kk, tau, X, m, kk);
    cd *Qb = Q + b * (long long)m * kk;
    for (int idx = tid; idx < m * kk; idx += nt) {
      const int i = idx / kk, c = idx - (idx / kk) * kk;
      Qb[idx] = X[(long long)c * m + i];
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" size_t dqz_qr_batched_scratch_bytes(int64_t batch, int32_t m, int32_t k) {
  if (batch <= 0 || m <= 0 || k <= 0) return 0;
  const long long grid = batch < QR_GRID_MAX ? batch : QR_GRID_MAX;
  return (size_t)grid * qr_scratch_per_matrix(m, k);
}

extern "C" int dqz_qr_batched(const void *a, int64_t batch, int32_t m, int32_t k, void *q, void *r, void *scratch,
                              cudaStream_t stream) {
  if (!a || !q || !r || !scratch || batch < 0 || m <= 0 || k <= 0) return DQZ_ERR_ARG;
  if ((long long)m * k >= (1ll << 31)) return DQZ_ERR_UNSUPPORTED;
  if (batch == 0) return DQZ_OK;
  const int kk = m < k ? m : k;
  const size_t smem = (size_t)kk * sizeof(cd);
  if (smem > 48 * 1024) return DQZ_ERR_UNSUPPORTED;
  const int grid = batch < QR_GRID_MAX ? (int)batch : QR_GRID_MAX;
  qr_batched_kernel<<<grid, QR_THREADS, smem, stream>>>((const cd *)a, (long long)batch, m, k, (cd *)q, (cd *)r,
                                                         (cd *)scratch);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
