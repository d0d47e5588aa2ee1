// Library-level entry points of libdqz.
#include "common.cuh"

extern "C" int dqz_version(void) { return 1; }

extern "C" int dqz_device_supported(int device) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 0;
  return prop.major == 10 ? 1 : 0;
}

namespace {
int32_t g_tuning[DQZ_TUNE_COUNT] = {0, 0, 0, 0, 0, 0};
}

extern "C" int dqz_set_tuning(int32_t knob, int32_t value) {
  if (knob < 0 || knob >= DQZ_TUNE_COUNT || value < 0) return DQZ_ERR_ARG;
  if ((knob == DQZ_TUNE_GAUGE_EDGE_WARPS || knob == DQZ_TUNE_GAUGE_DIST_WARPS) && value > 8) return DQZ_ERR_ARG;
  if (knob == DQZ_TUNE_GAUGE_PATH && value > 2) return DQZ_ERR_ARG;
  if (knob == DQZ_TUNE_SU_ONCHIP && value > 4) return DQZ_ERR_ARG;
  if (knob == DQZ_TUNE_SWEEP_ONECTA && value > 2) return DQZ_ERR_ARG;
  g_tuning[knob] = value;
  return DQZ_OK;
}

extern "C" int32_t dqz_get_tuning(int32_t knob) {
  if (knob < 0 || knob >= DQZ_TUNE_COUNT) return -1;
  return g_tuning[knob];
}

namespace {

using dqz::cd;

// One warp per segment: partial[i] = |a[seg_i] - b[seg_i]|_F
__global__ void segment_distance_kernel(const cd *a, const cd *b, const int64_t *off, int n, double *partial) {
  const int wpb = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < n; i += gridDim.x * wpb) {
    double acc = 0.0;
    for (int64_t j = off[i] + lane; j < off[i + 1]; j += 32) acc += dqz::cabs2(dqz::csub(a[j], b[j]));
    acc = dqz::warp_sum(acc);
    if (lane == 0) partial[i] = sqrt(acc);
  }
}

// One CTA per segment, 16-byte or 8-byte words.
template <typename W>
__global__ void repack_kernel(const W *src, W *dst, const int64_t *src_off, const int64_t *dst_off,
                              const int64_t *count, int n) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const W *s = src + src_off[i];
    W *d = dst + dst_off[i];
    for (int64_t j = threadIdx.x; j < count[i]; j += blockDim.x) d[j] = s[j];
  }
}

}  // namespace

extern "C" int dqz_segment_distance(const void *a, const void *b, const int64_t *seg_off, int32_t n,
                                    double *partial, double *out, cudaStream_t stream) {
  if (!a || !b || !seg_off || !partial || !out || n <= 0) return DQZ_ERR_ARG;
  const int wpb = 8;
  segment_distance_kernel<<<(n + wpb - 1) / wpb, wpb * 32, 0, stream>>>((const cd *)a, (const cd *)b, seg_off, n,
                                                                        partial);
  DQZ_CHECK_LAUNCH();
  return dqz_reduce_sum(partial, n, 1.0 / (double)n, out, stream);
}

extern "C" int dqz_repack(const void *src, void *dst, const int64_t *src_off, const int64_t *dst_off,
                          const int64_t *count, int32_t n, int32_t elem_bytes, cudaStream_t stream) {
  if (!src || !dst || !src_off || !dst_off || !count || n < 0) return DQZ_ERR_ARG;
  if (n == 0) return DQZ_OK;
  const int grid = n < 65535 ? n : 65535;
  if (elem_bytes == 16)
    repack_kernel<double2><<<grid, 256, 0, stream>>>((const double2 *)src, (double2 *)dst, src_off, dst_off, count,
                                                     n);
  else if (elem_bytes == 8)
    repack_kernel<double><<<grid, 256, 0, stream>>>((const double *)src, (double *)dst, src_off, dst_off, count, n);
  else
    return DQZ_ERR_ARG;
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}

namespace {

// Grid-stride count of non-finite words (NaN or +-Inf); one atomic per warp.
template <typename F>
__global__ void count_nonfinite_kernel(const F *x, int64_t n, int32_t *count) {
  int local = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    local += isfinite(x[i]) ? 0 : 1;
  local = __reduce_add_sync(0xffffffffu, local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

}  // namespace

extern "C" int dqz_count_nonfinite(const void *data, int64_t n, int32_t elem_bytes, int32_t *count,
                                   cudaStream_t stream) {
  if (!data || !count || n < 0 || (elem_bytes != 4 && elem_bytes != 8)) return DQZ_ERR_ARG;
  if (n == 0) return DQZ_OK;
  const int64_t blocks = (n + 255) / 256;
  const int grid = (int)(blocks < 148 * 8 ? blocks : 148 * 8);
  if (elem_bytes == 8)
    count_nonfinite_kernel<double><<<grid, 256, 0, stream>>>((const double *)data, n, count);
  else
    count_nonfinite_kernel<float><<<grid, 256, 0, stream>>>((const float *)data, n, count);
  DQZ_CHECK_LAUNCH();
  return DQZ_OK;
}
