// BF16 warp-level tensor-core helpers shared by the degree-3 BP kernels:
// ldmatrix fragment loads, the m16n8k16 BF16 MMA with FP32 accumulation, and
// complex 16 x 16 tiles built from four real products (the minus sign of
// re*re - im*im applied by flipping BF16 sign bits in operand registers).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"

namespace {

__device__ __forceinline__ uint32_t saddr(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void neg4(const uint32_t (&a)[4], uint32_t (&o)[4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = a[i] ^ 0x80008000u;
}

// Complex tile: D(16 x 16) += A * B, Dr += Ar Br - Ai Bi, Di += Ar Bi + Ai Br.
__device__ __forceinline__ void cmma(const uint32_t (&ar)[4], const uint32_t (&ai)[4], const uint32_t (&br)[2][2],
                                     const uint32_t (&bi)[2][2], float (&dr)[2][4], float (&di)[2][4]) {
  uint32_t nai[4];
  neg4(ai, nai);
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    mma_bf16(dr[nt], ar, br[nt][0], br[nt][1]);
    mma_bf16(dr[nt], nai, bi[nt][0], bi[nt][1]);
    mma_bf16(di[nt], ar, bi[nt][0], bi[nt][1]);
    mma_bf16(di[nt], ai, br[nt][0], br[nt][1]);
  }
}
// Conjugated B: D += A * conj(B): Dr += Ar Br + Ai Bi, Di += Ai Br - Ar Bi.
__device__ __forceinline__ void cmma_conjb(const uint32_t (&ar)[4], const uint32_t (&ai)[4],
                                           const uint32_t (&br)[2][2], const uint32_t (&bi)[2][2],
                                           float (&dr)[2][4], float (&di)[2][4]) {
  uint32_t nar[4];
  neg4(ar, nar);
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    mma_bf16(dr[nt], ar, br[nt][0], br[nt][1]);
    mma_bf16(dr[nt], ai, bi[nt][0], bi[nt][1]);
    mma_bf16(di[nt], ai, br[nt][0], br[nt][1]);
    mma_bf16(di[nt], nar, bi[nt][0], bi[nt][1]);
  }
}

// Complex64 message of half-edge hf as selected by the sweep schedule.
__device__ __forceinline__ const float2 *msg_c64(const dqz_graph_t &g, int hf, const float2 *n2e_old,
                                                 const float2 *e2n_old, const float2 *n2e_new,
                                                 const uint8_t *src_sel) {
  const int sel = src_sel[hf];
  if (sel == DQZ_SRC_E2N_OLD) return e2n_old + g.half_msg_off[hf];
  return (sel == DQZ_SRC_N2E_NEW ? n2e_new : n2e_old) + g.half_msg_off[g.half_twin[hf]];
}

}  // namespace
