// Dense state-vector kernels (complex128) for the exact emulator used to
// validate the BP emulator (quantum_emulator/exact_quantum_emulator.py:11-147).
// The state has 2^n amplitudes; the qubit at position p (traversal order of
// the nodes) is bit n-1-p of the amplitude index, so position 0 is the most
// significant bit, as in the reference's reshape(n * (2,)).
// Every kernel is a grid-stride loop over independent amplitude groups (HBM
// bound: one read and one write of the state per gate).
#include "common.cuh"

using namespace dqz;

namespace {

constexpr int SV_THREADS = 256;
constexpr int SV_GRID = 148 * 8;

// Index with a zero bit inserted at position b: the t-th index whose bit b is 0.
__device__ __forceinline__ unsigned long long insert_zero(unsigned long long t, int b) {
  const unsigned long long low = t & ((1ull << b) - 1ull);
  return ((t >> b) << (b + 1)) | low;
}

__global__ void sv_basis_kernel(cd *psi, unsigned long long size, unsigned long long index) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < size;
       i += (unsigned long long)gridDim.x * blockDim.x)
    psi[i] = (i == index) ? mk(1.0, 0.0) : czero();
}

// new[o] = sum_i g[o][i] old[i] on bit b.
__global__ void sv_apply1_kernel(cd *psi, unsigned long long pairs, int b, cd g00, cd g01, cd g10, cd g11) {
  const unsigned long long mask = 1ull << b;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < pairs;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long i0 = insert_zero(t, b), i1 = i0 | mask;
    const cd a0 = psi[i0], a1 = psi[i1];
    psi[i0] = cadd(cmul(g00, a0), cmul(g01, a1));
    psi[i1] = cadd(cmul(g10, a0), cmul(g11, a1));
  }
}

struct Gate4 {
  cd g[16];  // g[o1][o2][i1][i2]
};

// new[o1 o2] = sum g[o1][o2][i1][i2] old[i1 i2] on bits b1 (first qubit), b2.
__global__ void sv_apply2_kernel(cd *psi, unsigned long long quads, int b1, int b2, const Gate4 G) {
  const cd *g = G.g;
  const int lo = b1 < b2 ? b1 : b2, hi = b1 < b2 ? b2 : b1;
  const unsigned long long m1 = 1ull << b1, m2 = 1ull << b2;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < quads;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long base = insert_zero(insert_zero(t, lo), hi);
    unsigned long long idx[4];
    cd a[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) {  // x = i1 * 2 + i2
      idx[x] = base | ((x >> 1) ? m1 : 0ull) | ((x & 1) ? m2 : 0ull);
      a[x] = psi[idx[x]];
    }
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      cd acc = czero();
#pragma unroll
      for (int x = 0; x < 4; ++x) acc = cadd(acc, cmul(g[o * 4 + x], a[x]));
      psi[idx[o]] = acc;
    }
  }
}

// partial[block] = (rho00, rho01, rho10, rho11) over the block's pairs on bit b.
__global__ void __launch_bounds__(SV_THREADS) sv_density_kernel(const cd *__restrict__ psi, unsigned long long pairs,
                                                                int b, cd *partial) {
  __shared__ double red[48];
  const unsigned long long mask = 1ull << b;
  cd r00 = czero(), r01 = czero(), r10 = czero(), r11 = czero();
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < pairs;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long i0 = insert_zero(t, b);
    const cd a0 = psi[i0], a1 = psi[i0 | mask];
    // rho[s][s'] = psi[s] conj(psi[s'])
    r00 = cadd(r00, cmul(a0, cconj(a0)));
    r01 = cadd(r01, cmul(a0, cconj(a1)));
    r10 = cadd(r10, cmul(a1, cconj(a0)));
    r11 = cadd(r11, cmul(a1, cconj(a1)));
  }
  double v[8] = {r00.x, r00.y, r01.x, r01.y, r10.x, r10.y, r11.x, r11.y};
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = block_sum(v[j], red);
  if (threadIdx.x == 0)
    for (int j = 0; j < 4; ++j) partial[(long long)blockIdx.x * 4 + j] = mk(v[2 * j], v[2 * j + 1]);
}

// rho = sum of the partials in block order (deterministic).
__global__ void sv_density_reduce_kernel(const cd *partial, int n_part, cd *rho) {
  __shared__ double red[48];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int p = threadIdx.x; p < n_part; p += blockDim.x)
    for (int j = 0; j < 4; ++j) {
      v[2 * j] += partial[(long long)p * 4 + j].x;
      v[2 * j + 1] += partial[(long long)p * 4 + j].y;
    }
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = block_sum(v[j], red);
  if (threadIdx.x == 0)
    for (int j = 0; j < 4; ++j) rho[j] = mk(v[2 * j], v[2 * j + 1]);
}

// Keep the branch bit b == result scaled by `scale`, zero the other.
__global__ void sv_project_kernel(cd *psi, unsigned long long pairs, int b, int result, double scale) {
  const unsigned long long mask = 1ull << b;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < pairs;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long i0 = insert_zero(t, b), i1 = i0 | mask;
    if (result == 0) {
      psi[i0] = cscale(psi[i0], scale);
      psi[i1] = czero();
    } else {
      psi[i0] = czero();
      psi[i1] = cscale(psi[i1], scale);
    }
  }
}

inline int sv_grid(unsigned long long work) {
  const unsigned long long g = (work + SV_THREADS - 1) / SV_THREADS;
  return (int)(g < SV_GRID ? (g > 0 ? g : 1) : SV_GRID);
}

bool bad_n(int32_t n) { return n < 1 || n > DQZ_SV_MAX_QUBITS; }

}  // namespace

extern "C" int dqz_sv_set_basis(void *state, int32_t n, int64_t index, cudaStream_t stream) {
  if (!state || bad_n(n) || index < 0 || (unsigned long long)index >= (1ull << n)) return DQZ_ERR_ARG;
  const unsigned long long size = 1ull << n;
  sv_basis_kernel<<<sv_grid(size), SV_THREADS, 0, stream>>>((cd *)state, size, (unsigned long long)index);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_sv_apply1(void *state, int32_t n, int32_t pos, const double *gate, cudaStream_t stream) {
  if (!state || !gate || bad_n(n) || pos < 0 || pos >= n) return DQZ_ERR_ARG;
  const unsigned long long pairs = 1ull << (n - 1);
  sv_apply1_kernel<<<sv_grid(pairs), SV_THREADS, 0, stream>>>((cd *)state, pairs, n - 1 - pos, mk(gate[0], gate[1]),
                                                              mk(gate[2], gate[3]), mk(gate[4], gate[5]),
                                                              mk(gate[6], gate[7]));
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_sv_apply2(void *state, int32_t n, int32_t pos1, int32_t pos2, const double *gate,
                             cudaStream_t stream) {
  if (!state || !gate || bad_n(n) || n < 2 || pos1 < 0 || pos1 >= n || pos2 < 0 || pos2 >= n || pos1 == pos2)
    return DQZ_ERR_ARG;
  Gate4 G;
  for (int i = 0; i < 16; ++i) G.g[i] = mk(gate[2 * i], gate[2 * i + 1]);
  const unsigned long long quads = 1ull << (n - 2);
  sv_apply2_kernel<<<sv_grid(quads), SV_THREADS, 0, stream>>>((cd *)state, quads, n - 1 - pos1, n - 1 - pos2, G);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" size_t dqz_sv_density_scratch_bytes(int32_t n) {
  if (bad_n(n)) return 0;
  return (size_t)sv_grid(1ull << (n - 1)) * 4 * sizeof(cd);
}

extern "C" int dqz_sv_density1(const void *state, int32_t n, int32_t pos, void *rho, void *scratch,
                               cudaStream_t stream) {
  if (!state || !rho || !scratch || bad_n(n) || pos < 0 || pos >= n) return DQZ_ERR_ARG;
  const unsigned long long pairs = 1ull << (n - 1);
  const int grid = sv_grid(pairs);
  sv_density_kernel<<<grid, SV_THREADS, 0, stream>>>((const cd *)state, pairs, n - 1 - pos, (cd *)scratch);
  DQZ_CHECK_LAUNCH();
  sv_density_reduce_kernel<<<1, SV_THREADS, 0, stream>>>((const cd *)scratch, grid, (cd *)rho);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

extern "C" int dqz_sv_project(void *state, int32_t n, int32_t pos, int32_t result, double scale,
                              cudaStream_t stream) {
  if (!state || bad_n(n) || pos < 0 || pos >= n || (result != 0 && result != 1)) return DQZ_ERR_ARG;
  const unsigned long long pairs = 1ull << (n - 1);
  sv_project_kernel<<<sv_grid(pairs), SV_THREADS, 0, stream>>>((cd *)state, pairs, n - 1 - pos, result, scale);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
