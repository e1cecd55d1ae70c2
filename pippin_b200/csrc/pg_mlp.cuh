// Device side of the learned warm start's network: 24 -> 128 -> 128 -> 128
// -> 3 (ReLU) on the 5th-generation tensor cores. A block takes 128 samples
// at a time, one thread each; each layer is one accumulation chain of
// tcgen05.mma (kind::f16, BF16 operands from shared memory, FP32 accumulator
// D[128][N] in tensor memory) issued by one thread, completed through an
// mbarrier; the epilogue reads each thread's row of D with tcgen05.ld (warp
// w owns tensor-memory lanes 32w..32w+31, lane = sample), adds the bias,
// applies ReLU and writes the BF16 row into shared memory as the next
// layer's A operand. The weights are staged in shared memory once per block
// (76 KB, already in the operands' canonical layout, pg_mlp.h).
//
// Every wait on the tensor cores is bounded: when one runs out, the block
// sets *err, writes 0 for its rows, waits (bounded) for what it issued,
// frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "pg_mlp.h"

namespace pg {

constexpr int MLP_TC_ROWS = 128;     // samples per block: the MMA's M
constexpr int MLP_TC_THREADS = 128;  // one thread per sample (four warps: the four lane quarters)
constexpr int MLP_TC_COLS = 128;     // tensor-memory columns of the accumulator (FP32, N <= 128)

// shared memory of a block (bytes): weights, layer-1 inputs, activations,
// FP32 side data; offsets multiples of 128
constexpr size_t MLP_SM_W = sizeof(uint16_t) * MLP_BF16_ELEMS;
constexpr size_t MLP_SM_X = sizeof(uint16_t) * MLP_TC_ROWS * MLP_K1;
constexpr size_t MLP_SM_H = sizeof(uint16_t) * MLP_TC_ROWS * MLP_H;
constexpr size_t MLP_SM_F = (sizeof(float) * MLP_F32_ELEMS + 127) / 128 * 128;
constexpr size_t MLP_SMEM = MLP_SM_W + MLP_SM_X + MLP_SM_H + MLP_SM_F;
static_assert(MLP_SM_W % 128 == 0 && MLP_SM_X % 128 == 0 && MLP_SM_H % 128 == 0, "operand alignment");

__device__ inline uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ inline uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory descriptor of a K-major operand without swizzle: start
// address, leading-dimension byte offset 128 (the next 8 k-columns' core
// matrix follows the current one), stride-dimension byte offset sbo (the
// next 8 rows), descriptor version 1; addresses in 16-byte units.
__device__ inline uint64_t umma_desc(uint32_t saddr, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
         (1ull << 46);
}

// Instruction descriptor: BF16 x BF16 -> FP32, A and B K-major, M = 128, N.
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(MLP_TC_ROWS >> 4) << 24);
}

// D (+)= A B' for one k16 step; accumulate = 0 starts the chain
__device__ inline void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

__device__ inline void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// waits for phase `parity` of the mbarrier to complete; false when the
// bound runs out first
__device__ inline bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 20); it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// this thread's 32 FP32 accumulator columns [col, col + 32) of its lane
__device__ inline void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}

// The block's copy of the weights and side data: every thread issues all of
// its asynchronous copies before waiting on any.
__device__ inline void mlp_stage(const MlpDevice& d, uint16_t* W, float* F) {
  static_assert(MLP_SM_W % 16 == 0, "whole 16-byte chunks");
  const char* src = reinterpret_cast<const char*>(d.w);
  char* dst = reinterpret_cast<char*>(W);
  for (int i = threadIdx.x; i < (int)(MLP_SM_W / 16); i += blockDim.x) {
    size_t sg = __cvta_generic_to_global(src + 16 * i);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst + 16 * i)), "l"(sg) : "memory");
  }
  for (int i = threadIdx.x; i < MLP_F32_ELEMS; i += blockDim.x) {
    size_t sg = __cvta_generic_to_global(d.f + i);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(F + i)), "l"(sg) : "memory");
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Y[r][3] = net(X[r][24]) for r in [0, n), 128 rows a block at a time. Every
// thread of the block (MLP_TC_THREADS) calls it; smem holds MLP_SMEM bytes.
__device__ inline void mlp_tc_rows(const MlpDevice& d, const float* X, int64_t n, float* Y, unsigned char* smem) {
  __shared__ __align__(8) unsigned long long bar;
  __shared__ uint32_t tmem_slot;
  if ((int64_t)blockIdx.x * MLP_TC_ROWS >= n) return;
  uint16_t* W = reinterpret_cast<uint16_t*>(smem);
  uint16_t* Xs = reinterpret_cast<uint16_t*>(smem + MLP_SM_W);
  uint16_t* H = reinterpret_cast<uint16_t*>(smem + MLP_SM_W + MLP_SM_X);
  float* F = reinterpret_cast<float*>(smem + MLP_SM_W + MLP_SM_X + MLP_SM_H);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t barp = smem_addr(&bar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barp) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(MLP_TC_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  mlp_stage(d, W, F);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's quarter of the lanes
  const float* mean = F;
  const float* scale = F + MLP_IN;
  const float* oscale = F + 2 * MLP_IN;
  const float* bias = F + 2 * MLP_IN + MLP_OUT;  // b1 | b2 | b3 | b4
  const uint32_t sW = smem_addr(W), sX = smem_addr(Xs), sH = smem_addr(H);
  uint32_t parity = 0;
  bool ok = true;
  for (int64_t base = (int64_t)blockIdx.x * MLP_TC_ROWS; base < n && ok; base += (int64_t)gridDim.x * MLP_TC_ROWS) {
    const int64_t row = base + tid;
    // layer-1 operand: this thread's normalised features as one BF16 row (24 -> 32)
    {
      float x[MLP_K1];
#pragma unroll
      for (int k = 0; k < MLP_K1; k++) x[k] = (k < MLP_IN && row < n) ? (X[row * MLP_IN + k] - mean[k]) * scale[k] : 0.f;
#pragma unroll
      for (int c = 0; c < MLP_K1 / 8; c++) {
        uint4 v = make_uint4(pack_bf16(x[8 * c], x[8 * c + 1]), pack_bf16(x[8 * c + 2], x[8 * c + 3]),
                             pack_bf16(x[8 * c + 4], x[8 * c + 5]), pack_bf16(x[8 * c + 6], x[8 * c + 7]));
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(Xs) + umma_offset(tid, 8 * c, MLP_K1)) = v;
      }
    }
    float out[MLP_N4];
#pragma unroll
    for (int layer = 0; layer < 4 && ok; layer++) {
      const int K = layer == 0 ? MLP_K1 : MLP_H, N = layer == 3 ? MLP_N4 : MLP_H;
      const uint32_t a = layer == 0 ? sX : sH;
      const uint32_t b = sW + 2u * (uint32_t)(layer == 0 ? MLP_WU1 : layer == 1 ? MLP_WU2 : layer == 2 ? MLP_WU3 : MLP_WU4);
      // the operand rows written by every thread reach the tensor cores' view
      proxy_fence();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t sbo = (uint32_t)(K / 8) * 128u;
        for (int k = 0; k < K / 16; k++)
          umma_f16(tmem, umma_desc(a + 256u * k, sbo), umma_desc(b + 256u * k, sbo), umma_idesc(N), k > 0 ? 1u : 0u);
        umma_commit(barp);
      }
      // every thread waits; the block gives up together when any thread's wait ran out
      if (!__syncthreads_and(mbar_wait(barp, parity) ? 1 : 0)) {
        ok = false;
        break;
      }
      parity ^= 1u;
      tc_fence_after();
      if (layer < 3) {
        const float* bl = bias + layer * MLP_H;
#pragma unroll
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
          float v[32];
          tmem_ld32(lane_base + (uint32_t)c0, v);
#pragma unroll
          for (int c = 0; c < 4; c++) {
            float h[8];
#pragma unroll
            for (int j = 0; j < 8; j++) h[j] = fmaxf(v[8 * c + j] + bl[c0 + 8 * c + j], 0.f);
            uint4 u = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]),
                                 pack_bf16(h[6], h[7]));
            *reinterpret_cast<uint4*>(reinterpret_cast<char*>(H) + umma_offset(tid, c0 + 8 * c, MLP_H)) = u;
          }
        }
      } else {
        float v[32];
        tmem_ld32(lane_base, v);
#pragma unroll
        for (int j = 0; j < MLP_N4; j++) out[j] = v[j];
      }
    }
    __syncthreads();  // the last layer's reads of H and the next group's writes of Xs, H
    if (row < n)
      for (int j = 0; j < MLP_OUT; j++) Y[row * MLP_OUT + j] = ok ? (out[j] + bias[3 * MLP_H + j]) * oscale[j] : 0.f;
  }
  if (!ok) {
    if (tid == 0) {
      atomicExch(d.err, 1);
      mbar_wait(barp, parity);  // what was issued completes (bounded) before the memory goes
    }
    for (int64_t r = (int64_t)blockIdx.x * MLP_TC_ROWS + tid; r < n; r += (int64_t)gridDim.x * MLP_TC_ROWS)
      for (int j = 0; j < MLP_OUT; j++) Y[r * MLP_OUT + j] = 0.f;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(MLP_TC_COLS) : "memory");
  }
}

}  // namespace pg
