// Device side of the learned warm start's network: BF16 tensor-core
// inference of 24 -> 128 -> 128 -> 128 -> 3 (ReLU) for groups of 16 samples
// on a block of MLP_WARPS warps (mma.sync m16n8k16, FP32 accumulation). The
// weights are staged in shared memory once per block; each warp computes its
// own 32 of a hidden layer's 128 outputs, so that a layer's chain of
// dependent MMAs is 4x shorter than one warp doing all of them; the layer's
// BF16 activations go through shared memory (one block barrier per layer) to
// become every warp's A fragments of the next layer. Layer 4 (3 outputs, one
// n-tile) runs on warp 0.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "pg_mlp.h"

namespace pg {

__device__ inline uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ inline void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B fragment of W (row n = output, k = input; row stride ld) for the n8 tile
// at n0 and the k16 tile at k0
__device__ inline void bfrag(const uint16_t* W, int ld, int n0, int k0, int g, int tq, uint32_t* b0, uint32_t* b1) {
  const uint16_t* r = W + (n0 + g) * ld + k0 + 2 * tq;
  *b0 = *reinterpret_cast<const uint32_t*>(r);
  *b1 = *reinterpret_cast<const uint32_t*>(r + 8);
}

constexpr int MLP_WARPS = 4;
constexpr int MLP_NW = MLP_H / MLP_WARPS;  // outputs of a hidden layer per warp
constexpr int MLP_LDA = MLP_H + 8;         // row stride (bf16) of the activation tile

// this warp's 32 outputs of a hidden layer for the 16 samples whose A
// fragments are a (KT k-tiles), plus bias and ReLU, stored as BF16 rows of
// the activation tile `out` [16][MLP_LDA]
template <int KT>
__device__ inline void hidden_slice(const uint32_t (&a)[KT][4], const uint16_t* W, int ld, const float* bias, int n0,
                                    int g, int tq, uint16_t* out) {
  float c[MLP_NW / 8][4];
#pragma unroll
  for (int t = 0; t < MLP_NW / 8; t++) c[t][0] = c[t][1] = c[t][2] = c[t][3] = 0.f;
#pragma unroll
  for (int kt = 0; kt < KT; kt++)
#pragma unroll
    for (int t = 0; t < MLP_NW / 8; t++) {
      uint32_t b0, b1;
      bfrag(W, ld, n0 + 8 * t, 16 * kt, g, tq, &b0, &b1);
      mma_bf16(c[t], a[kt], b0, b1);
    }
#pragma unroll
  for (int t = 0; t < MLP_NW / 8; t++) {
    int col = n0 + 8 * t + 2 * tq;
    *reinterpret_cast<uint32_t*>(out + g * MLP_LDA + col) =
        pack_bf16(fmaxf(c[t][0] + bias[col], 0.f), fmaxf(c[t][1] + bias[col + 1], 0.f));
    *reinterpret_cast<uint32_t*>(out + (g + 8) * MLP_LDA + col) =
        pack_bf16(fmaxf(c[t][2] + bias[col], 0.f), fmaxf(c[t][3] + bias[col + 1], 0.f));
  }
}

// A fragments (8 k-tiles) of the 16 x 128 activation tile
__device__ inline void afrags(const uint16_t* act, int g, int tq, uint32_t (&a)[8][4]) {
#pragma unroll
  for (int kt = 0; kt < 8; kt++) {
    int c = 16 * kt + 2 * tq;
    a[kt][0] = *reinterpret_cast<const uint32_t*>(act + g * MLP_LDA + c);
    a[kt][1] = *reinterpret_cast<const uint32_t*>(act + (g + 8) * MLP_LDA + c);
    a[kt][2] = *reinterpret_cast<const uint32_t*>(act + g * MLP_LDA + c + 8);
    a[kt][3] = *reinterpret_cast<const uint32_t*>(act + (g + 8) * MLP_LDA + c + 8);
  }
}

// The block's copy of the weights: every thread issues all of its 16-byte
// asynchronous copies (cp.async) before waiting on any, so the 84 KB arrive
// in about one round trip instead of one per loop pass. stage_weights_begin
// only issues them (the block may work meanwhile); stage_weights_end waits
// for this thread's copies and then for the block.
__device__ inline void stage_weights_begin(const MlpDevice& d, uint16_t* W, float* F) {
  static_assert((sizeof(uint16_t) * MLP_BF16_ELEMS) % 16 == 0, "whole 16-byte chunks");
  const char* src = reinterpret_cast<const char*>(d.w);
  char* dst = reinterpret_cast<char*>(W);
  for (int i = threadIdx.x; i < (int)(sizeof(uint16_t) * MLP_BF16_ELEMS / 16); i += blockDim.x) {
    unsigned sd = (unsigned)__cvta_generic_to_shared(dst + 16 * i);
    size_t sg = __cvta_generic_to_global(src + 16 * i);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sd), "l"(sg) : "memory");
  }
  for (int i = threadIdx.x; i < MLP_F32_ELEMS; i += blockDim.x) {
    unsigned sd = (unsigned)__cvta_generic_to_shared(F + i);
    size_t sg = __cvta_generic_to_global(d.f + i);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sd), "l"(sg) : "memory");
  }
}
__device__ inline void stage_weights_end() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}
__device__ inline void stage_weights(const MlpDevice& d, uint16_t* W, float* F) {
  stage_weights_begin(d, W, F);
  stage_weights_end();
}

// shared memory of a block: weights, FP32 side data, two activation tiles
// and the group's 16 x 24 input features (FP32)
constexpr size_t MLP_SMEM_W = sizeof(uint16_t) * MLP_BF16_ELEMS;
constexpr size_t MLP_SMEM_F = sizeof(float) * MLP_F32_ELEMS;
constexpr size_t MLP_SMEM_ACT = sizeof(uint16_t) * 16 * MLP_LDA;
constexpr size_t MLP_SMEM_X = sizeof(float) * 16 * MLP_IN;
constexpr size_t MLP_SMEM = MLP_SMEM_W + MLP_SMEM_F + 2 * MLP_SMEM_ACT + MLP_SMEM_X;

struct MlpSmem {
  uint16_t* W;
  float* F;
  uint16_t *act0, *act1;
  float* X;  // [16][24] the group's features (raw, normalised on use)
};
__device__ inline MlpSmem mlp_smem_layout(unsigned char* smem) {
  MlpSmem s;
  s.W = reinterpret_cast<uint16_t*>(smem);
  s.F = reinterpret_cast<float*>(smem + MLP_SMEM_W);
  s.act0 = reinterpret_cast<uint16_t*>(smem + MLP_SMEM_W + MLP_SMEM_F);
  s.act1 = s.act0 + 16 * MLP_LDA;
  s.X = reinterpret_cast<float*>(smem + MLP_SMEM_W + MLP_SMEM_F + 2 * MLP_SMEM_ACT);
  return s;
}

// The network on the group of 16 samples in S.X (rows r with base + r >= n
// are padding): Y[base + r] = the 3 frame forces. Every thread of the block
// calls it (it holds block barriers); S.X must be complete on entry.
__device__ inline void mlp_group(const MlpSmem& S, int64_t base, int64_t n, float* Y) {
  const uint16_t* W1 = S.W;
  const uint16_t* W2 = W1 + MLP_H * MLP_LD1;
  const uint16_t* W3 = W2 + MLP_H * MLP_LDH;
  const uint16_t* W4 = W3 + MLP_H * MLP_LDH;
  const float* mean = S.F;
  const float* scale = S.F + MLP_IN;
  const float* oscale = S.F + 2 * MLP_IN;
  const float* b1 = S.F + 2 * MLP_IN + MLP_OUT;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int g = lane >> 2, tq = lane & 3;
  int n0 = warp * MLP_NW;
  int64_t r0 = base + g, r1 = base + g + 8;
  auto x = [&](int row, int c) -> float {
    return (base + row < n && c < MLP_IN) ? (S.X[row * MLP_IN + c] - mean[c]) * scale[c] : 0.f;
  };
  uint32_t a1[2][4];
#pragma unroll
  for (int kt = 0; kt < 2; kt++) {
    int c = 16 * kt + 2 * tq;
    a1[kt][0] = pack_bf16(x(g, c), x(g, c + 1));
    a1[kt][1] = pack_bf16(x(g + 8, c), x(g + 8, c + 1));
    a1[kt][2] = pack_bf16(x(g, c + 8), x(g, c + 9));
    a1[kt][3] = pack_bf16(x(g + 8, c + 8), x(g + 8, c + 9));
  }
  hidden_slice<2>(a1, W1, MLP_LD1, b1, n0, g, tq, S.act0);
  __syncthreads();
  uint32_t a[8][4];
  afrags(S.act0, g, tq, a);
  hidden_slice<8>(a, W2, MLP_LDH, b1 + MLP_H, n0, g, tq, S.act1);
  __syncthreads();
  afrags(S.act1, g, tq, a);
  hidden_slice<8>(a, W3, MLP_LDH, b1 + 2 * MLP_H, n0, g, tq, S.act0);
  __syncthreads();
  if (warp == 0) {
    afrags(S.act0, g, tq, a);
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < 8; kt++) {
      uint32_t b0, bb;
      bfrag(W4, MLP_LDH, 0, 16 * kt, g, tq, &b0, &bb);
      mma_bf16(c, a[kt], b0, bb);
    }
    const float* b4 = b1 + 3 * MLP_H;
    for (int j = 0; j < 4; j++) {
      int col = 2 * tq + (j & 1);
      int64_t r = j < 2 ? r0 : r1;
      if (col < MLP_OUT && r < n) Y[r * MLP_OUT + col] = (c[j] + b4[col]) * oscale[col];
    }
  }
  __syncthreads();  // act0 and X are rewritten by the next group
}

}  // namespace pg
