// Layout of the learned warm start's network (24 -> 128 -> 128 -> 128 -> 3,
// ReLU between layers) as one FP32 array: input normalisation, output scale,
// then each layer's weights [out][in] and bias.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pg {

constexpr int MLP_IN = 24, MLP_H = 128, MLP_OUT = 3;
constexpr int MLP_IN_MEAN = 0;                              // [24] feature mean
constexpr int MLP_IN_SCALE = MLP_IN_MEAN + MLP_IN;          // [24] 1 / feature std
constexpr int MLP_OUT_SCALE = MLP_IN_SCALE + MLP_IN;        // [3] target std
constexpr int MLP_W1 = MLP_OUT_SCALE + MLP_OUT;             // [128][24]
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;             // [128]
constexpr int MLP_W2 = MLP_B1 + MLP_H;                      // [128][128]
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;                      // [128][128]
constexpr int MLP_B3 = MLP_W3 + MLP_H * MLP_H;
constexpr int MLP_W4 = MLP_B3 + MLP_H;                      // [3][128]
constexpr int MLP_B4 = MLP_W4 + MLP_OUT * MLP_H;            // [3]
constexpr int MLP_SIZE = MLP_B4 + MLP_OUT;                  // 36662 floats
constexpr int MLP_PARAMS = MLP_SIZE - MLP_W1;               // 36611 trained parameters

// BF16 copy of the weights for the tensor-core forward pass (tcgen05.mma,
// operands in shared memory): each layer's W [out][in] in the canonical
// K-major layout without swizzle that the MMA's shared-memory descriptor
// reads, 8 x 8 core matrices of 128 contiguous bytes: element (r, k) of an
// R x K operand at byte umma_offset(r, k, K). Layer 1's inputs are padded to
// 32, layer 4's 3 outputs to 16 (the smallest N of an M = 128 MMA).
constexpr int MLP_K1 = 32;   // layer-1 inputs padded to two k16 steps
constexpr int MLP_N4 = 16;   // layer-4 outputs padded to the smallest N
constexpr int MLP_WU1 = 0;                              // [128][32]  (bf16 elements)
constexpr int MLP_WU2 = MLP_WU1 + MLP_H * MLP_K1;       // [128][128]
constexpr int MLP_WU3 = MLP_WU2 + MLP_H * MLP_H;        // [128][128]
constexpr int MLP_WU4 = MLP_WU3 + MLP_H * MLP_H;        // [16][128]
constexpr int MLP_BF16_ELEMS = MLP_WU4 + MLP_N4 * MLP_H;
// FP32 side data of the forward pass: in mean, in scale, out scale, biases
constexpr int MLP_F32_ELEMS = 2 * MLP_IN + MLP_OUT + 3 * MLP_H + MLP_N4;

// byte offset of element (r, k) in an R x K canonical operand (K a multiple of 8)
__host__ __device__ constexpr size_t umma_offset(int r, int k, int K) {
  return (size_t)(r / 8) * (K / 8) * 128 + (size_t)(k / 8) * 128 + (size_t)(r % 8) * 16 + (size_t)(k % 8) * 2;
}

struct MlpDevice {
  const uint16_t* w;  // MLP_BF16_ELEMS bf16 (W1 | W2 | W3 | W4, canonical operand layout)
  const float* f;     // MLP_F32_ELEMS (in_mean | in_scale | out_scale | b1 | b2 | b3 | b4 padded)
  int* err;           // set when a wait on the tensor cores ran out (the rows then predict 0)
};

// packs the FP32 array into the forward pass's device layout (host side)
void mlp_pack(const float* weights, uint16_t* w_bf16, float* f32);
// allows the forward kernels their shared memory (once, before launches or captures)
cudaError_t mlp_prepare();
// Y[n][3] = net(X[n][24]) on the tensor cores (tcgen05), on stream s
cudaError_t mlp_forward(const MlpDevice& d, const float* X, int64_t n, float* Y, cudaStream_t s);
// the same over min(*count, cap) rows, count read on the device (for launches
// whose row count the host does not know)
cudaError_t mlp_forward_counted(const MlpDevice& d, const float* X, const int* count, int64_t cap, float* Y,
                                cudaStream_t s);

}  // namespace pg
