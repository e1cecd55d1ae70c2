// The learned warm start's network: inference on the tensor cores and
// training kernels.
//
// Inference (mlp_forward_kernel, mlp_count_kernel; device side in
// pg_mlp.cuh): tcgen05.mma with BF16 operands in shared memory and FP32
// accumulators in tensor memory, 128 samples a block, the 76 KB of BF16
// weights staged once per block in the operands' canonical layout.
//
// Training (mlp_train_*): FP32 throughout (master weights, activations,
// gradients, Adam moments), simple tiled kernels: the network is small
// (36,611 parameters) and a batch of a few thousand samples is a few GFLOP.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pg_mlp.cuh"

namespace pg {

static uint16_t to_bf16(float x) {
  __nv_bfloat16 b = __float2bfloat16_rn(x);
  uint16_t u;
  std::memcpy(&u, &b, 2);
  return u;
}

void mlp_pack(const float* wt, uint16_t* w, float* f) {
  std::fill(w, w + MLP_BF16_ELEMS, to_bf16(0.0f));
  std::fill(f, f + MLP_F32_ELEMS, 0.0f);
  // W[out][in] of each layer into its canonical operand layout (pg_mlp.h)
  auto put = [&](int base, int rows, int K, int src, int in) {
    for (int n = 0; n < rows; n++)
      for (int k = 0; k < in; k++) w[base + umma_offset(n, k, K) / 2] = to_bf16(wt[src + n * in + k]);
  };
  put(MLP_WU1, MLP_H, MLP_K1, MLP_W1, MLP_IN);
  put(MLP_WU2, MLP_H, MLP_H, MLP_W2, MLP_H);
  put(MLP_WU3, MLP_H, MLP_H, MLP_W3, MLP_H);
  put(MLP_WU4, MLP_OUT, MLP_H, MLP_W4, MLP_H);
  std::memcpy(f, wt + MLP_IN_MEAN, sizeof(float) * (2 * MLP_IN + MLP_OUT));
  float* b = f + 2 * MLP_IN + MLP_OUT;
  std::memcpy(b, wt + MLP_B1, sizeof(float) * MLP_H);
  std::memcpy(b + MLP_H, wt + MLP_B2, sizeof(float) * MLP_H);
  std::memcpy(b + 2 * MLP_H, wt + MLP_B3, sizeof(float) * MLP_H);
  std::memcpy(b + 3 * MLP_H, wt + MLP_B4, sizeof(float) * MLP_OUT);
}

// ---------------------------------------------------------------- inference
// the standalone forward pass (pg_mlp_forward): features from global memory
__global__ void __launch_bounds__(MLP_TC_THREADS) mlp_forward_kernel(MlpDevice d, const float* X, int64_t n, float* Y) {
  extern __shared__ __align__(128) unsigned char smem[];
  mlp_tc_rows(d, X, n, Y, smem);
}

// the learned start's forward pass: min(*count, cap) rows, counted on the
// device by the collision phase
__global__ void __launch_bounds__(MLP_TC_THREADS) mlp_count_kernel(MlpDevice d, const float* X, const int* count,
                                                                   int64_t cap, float* Y) {
  extern __shared__ __align__(128) unsigned char smem[];
  int64_t n = *count;
  mlp_tc_rows(d, X, n < cap ? n : cap, Y, smem);
}

cudaError_t mlp_prepare() {
  cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(mlp_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_SMEM);
  return e;
}

// blocks of 128 rows: one resident an SM (its shared memory), at most two
// waves of a 148-SM GPU; each block stages the weights once and loops
static unsigned mlp_blocks(int64_t rows) {
  int64_t b = (rows + MLP_TC_ROWS - 1) / MLP_TC_ROWS;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 296));
}

cudaError_t mlp_forward_counted(const MlpDevice& d, const float* X, const int* count, int64_t cap, float* Y,
                                cudaStream_t s) {
  // the grid covers the capacity; blocks past the device-side count return at once
  if (cap <= 0) return cudaSuccess;
  mlp_count_kernel<<<mlp_blocks(cap), MLP_TC_THREADS, MLP_SMEM, s>>>(d, X, count, cap, Y);
  return cudaGetLastError();
}

cudaError_t mlp_forward(const MlpDevice& d, const float* X, int64_t n, float* Y, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  mlp_forward_kernel<<<mlp_blocks(n), MLP_TC_THREADS, MLP_SMEM, s>>>(d, X, n, Y);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- training
// C[i][j] = act(sum_k A(i, k) B(k, j) + bias[j]), A(i, k) = A[i*sai + k*sak],
// B(k, j) = B[k*sbk + j*sbj]; act = ReLU when relu != 0; rows of C are
// multiplied by (mask[i][j] > 0) when a mask is given (the ReLU derivative)
constexpr int GT = 32;
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const float* A, long sai, long sak,
                                                   const float* B, long sbk, long sbj, float* C, const float* bias,
                                                   int relu, const float* mask) {
  __shared__ float As[GT][GT + 1], Bs[GT][GT + 1];
  int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT;
  float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
  for (int k0 = 0; k0 < K; k0 += GT) {
    for (int t = threadIdx.x; t < GT * GT; t += 256) {
      int r = t / GT, c = t % GT;
      int i = i0 + r, k = k0 + c;
      As[r][c] = (i < M && k < K) ? A[i * sai + k * sak] : 0.f;
      int kk = k0 + r, j = j0 + c;
      Bs[r][c] = (kk < K && j < N) ? B[kk * sbk + j * sbj] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < GT; k++) {
      float a0 = As[2 * ty][k], a1 = As[2 * ty + 1][k];
      float b0 = Bs[k][2 * tx], b1 = Bs[k][2 * tx + 1];
      acc[0][0] += a0 * b0;
      acc[0][1] += a0 * b1;
      acc[1][0] += a1 * b0;
      acc[1][1] += a1 * b1;
    }
    __syncthreads();
  }
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      int i = i0 + 2 * ty + u, j = j0 + 2 * tx + v;
      if (i >= M || j >= N) continue;
      float x = acc[u][v] + (bias ? bias[j] : 0.f);
      if (relu) x = fmaxf(x, 0.f);
      if (mask && !(mask[(long)i * N + j] > 0.f)) x = 0.f;
      C[(long)i * N + j] = x;
    }
}

static cudaError_t gemm(int M, int N, int K, const float* A, long sai, long sak, const float* B, long sbk, long sbj,
                        float* C, const float* bias, int relu, const float* mask, cudaStream_t s) {
  dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
  gemm_kernel<<<grid, 256, 0, s>>>(M, N, K, A, sai, sak, B, sbk, sbj, C, bias, relu, mask);
  return cudaGetLastError();
}

// Weight gradients C = A' B over a batch (A: K x M, B: K x N, both row-major
// with row strides lda, ldb; K the batch) split along K: block (x, y, z)
// sums rows [z kc, (z + 1) kc) of its 32 x 32 tile of C into part[z], and
// sum_splits adds the splits in order (deterministic). Both operands are
// read along their rows, so the loads coalesce.
constexpr int SPLITS = 32;
__global__ void __launch_bounds__(256) gemm_atb_kernel(int M, int N, int K, int kc, const float* A, int lda,
                                                       const float* B, int ldb, float* part) {
  __shared__ float As[GT][GT + 1], Bs[GT][GT + 1];
  int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT;
  int k_begin = blockIdx.z * kc, k_end = min(K, k_begin + kc);
  float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
  for (int k0 = k_begin; k0 < k_end; k0 += GT) {
    for (int t = threadIdx.x; t < GT * GT; t += 256) {
      int kk = t / GT, c = t % GT;
      int k = k0 + kk;
      As[kk][c] = (k < k_end && i0 + c < M) ? A[(long)k * lda + i0 + c] : 0.f;
      Bs[kk][c] = (k < k_end && j0 + c < N) ? B[(long)k * ldb + j0 + c] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < GT; k++) {
      float a0 = As[k][2 * ty], a1 = As[k][2 * ty + 1];
      float b0 = Bs[k][2 * tx], b1 = Bs[k][2 * tx + 1];
      acc[0][0] += a0 * b0;
      acc[0][1] += a0 * b1;
      acc[1][0] += a1 * b0;
      acc[1][1] += a1 * b1;
    }
    __syncthreads();
  }
  float* P = part + (size_t)blockIdx.z * M * N;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      int i = i0 + 2 * ty + u, j = j0 + 2 * tx + v;
      if (i < M && j < N) P[(long)i * N + j] = acc[u][v];
    }
}

// out[t] = sum over z of part[z][t], z in order
__global__ void sum_splits_kernel(const float* part, int splits, int n, float* out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float s = 0.f;
  for (int z = 0; z < splits; z++) s += part[(size_t)z * n + t];
  out[t] = s;
}

// column sums of dY (M x N) split along M: part[z][j] = sum of rows [z rc, (z + 1) rc)
__global__ void colsum_split_kernel(const float* dY, int M, int N, int rc, float* part) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int r0 = blockIdx.y * rc, r1 = min(M, r0 + rc);
  float s = 0.f;
  for (int i = r0; i < r1; i++) s += dY[(long)i * N + j];
  part[(size_t)blockIdx.y * N + j] = s;
}

static cudaError_t gemm_atb(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C,
                            float* part, cudaStream_t s) {
  int kc = (K + SPLITS - 1) / SPLITS;
  dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT, SPLITS);
  gemm_atb_kernel<<<grid, 256, 0, s>>>(M, N, K, kc, A, lda, B, ldb, part);
  sum_splits_kernel<<<(M * N + 255) / 256, 256, 0, s>>>(part, SPLITS, M * N, C);
  return cudaGetLastError();
}

// the bias gradients' row splits: short column runs per thread (32 rows of a
// batch of 8192), so that the first pass has a block per split
constexpr int COLSUM_SPLITS = 256;
static_assert(COLSUM_SPLITS * MLP_H <= SPLITS * MLP_H * MLP_H, "colsum partial sums fit the split-K buffer");

static cudaError_t colsum(const float* dY, int M, int N, float* db, float* part, cudaStream_t s) {
  int rc = (M + COLSUM_SPLITS - 1) / COLSUM_SPLITS;
  colsum_split_kernel<<<dim3((N + 127) / 128, COLSUM_SPLITS), 128, 0, s>>>(dY, M, N, rc, part);
  sum_splits_kernel<<<(N + 255) / 256, 256, 0, s>>>(part, COLSUM_SPLITS, N, db);
  return cudaGetLastError();
}

// dO = 2 (O - Y) / (M * 3); each block's share of sum (O - Y)^2 / (M * 3) into lpart[block]
__global__ void __launch_bounds__(256) mse_kernel(const float* O, const float* Y, int M, float* dO, double* lpart) {
  __shared__ double red[256];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  float inv = 1.0f / (float)(M * MLP_OUT);
  double v = 0.0;
  if (t < M * MLP_OUT) {
    float d = O[t] - Y[t];
    dO[t] = 2.0f * d * inv;
    v = (double)(d * d) * inv;
  }
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) lpart[blockIdx.x] = red[0];
}

// loss += the blocks' shares, in block order (one thread)
__global__ void loss_add_kernel(const double* lpart, int nblocks, double* loss) {
  double s = 0.0;
  for (int b = 0; b < nblocks; b++) s += lpart[b];
  *loss += s;
}

// Adam (Kingma & Ba 2015) on every parameter
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float gt = g[t];
  float mt = b1 * m[t] + (1.f - b1) * gt, vt = b2 * v[t] + (1.f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

// rows of src picked by idx into dst (width w)
__global__ void gather_kernel(const float* src, const int* idx, int n, int w, float* dst) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * w) return;
  dst[t] = src[(long)idx[t / w] * w + t % w];
}

// Forward and backward of the normalised network on one batch: activations
// in H (3 x M x 128) and O (M x 3), gradients of the mean squared error into
// grad (same layout as the parameters). P and grad start at W1.
struct TrainBufs {
  float *H, *O, *dO, *dA, *dB;
  float* part;     // SPLITS x 128 x 128 split-K partial sums
  double* lpart;   // per-block loss shares
  double* loss;
};
// the partial-sum buffers' sizes for batches of M samples
inline size_t train_part_floats() { return (size_t)SPLITS * MLP_H * MLP_H; }
inline size_t train_lpart_doubles(int M) { return (size_t)(M * MLP_OUT + 255) / 256; }
static cudaError_t mlp_batch_grad(const float* P, const float* Xn, const float* Yn, int M, float* grad,
                                  const TrainBufs& t, cudaStream_t s) {
  auto w = [&](int off) { return P + (off - MLP_W1); };
  auto gw = [&](int off) { return grad + (off - MLP_W1); };
  float* H1 = t.H;
  float* H2 = t.H + (long)M * MLP_H;
  float* H3 = t.H + 2L * M * MLP_H;
  cudaError_t e;
#define G_(call) \
  if ((e = (call)) != cudaSuccess) return e
  G_(gemm(M, MLP_H, MLP_IN, Xn, MLP_IN, 1, w(MLP_W1), 1, MLP_IN, H1, w(MLP_B1), 1, nullptr, s));
  G_(gemm(M, MLP_H, MLP_H, H1, MLP_H, 1, w(MLP_W2), 1, MLP_H, H2, w(MLP_B2), 1, nullptr, s));
  G_(gemm(M, MLP_H, MLP_H, H2, MLP_H, 1, w(MLP_W3), 1, MLP_H, H3, w(MLP_B3), 1, nullptr, s));
  G_(gemm(M, MLP_OUT, MLP_H, H3, MLP_H, 1, w(MLP_W4), 1, MLP_H, t.O, w(MLP_B4), 0, nullptr, s));
  {
    int nb = (M * MLP_OUT + 255) / 256;
    mse_kernel<<<nb, 256, 0, s>>>(t.O, Yn, M, t.dO, t.lpart);
    loss_add_kernel<<<1, 1, 0, s>>>(t.lpart, nb, t.loss);
  }
  // layer 4: dW4 = dO' H3, db4, dH3 = dO W4 * (H3 > 0)
  G_(gemm_atb(MLP_OUT, MLP_H, M, t.dO, MLP_OUT, H3, MLP_H, gw(MLP_W4), t.part, s));
  G_(colsum(t.dO, M, MLP_OUT, gw(MLP_B4), t.part, s));
  G_(gemm(M, MLP_H, MLP_OUT, t.dO, MLP_OUT, 1, w(MLP_W4), MLP_H, 1, t.dA, nullptr, 0, H3, s));
  // layer 3
  G_(gemm_atb(MLP_H, MLP_H, M, t.dA, MLP_H, H2, MLP_H, gw(MLP_W3), t.part, s));
  G_(colsum(t.dA, M, MLP_H, gw(MLP_B3), t.part, s));
  G_(gemm(M, MLP_H, MLP_H, t.dA, MLP_H, 1, w(MLP_W3), MLP_H, 1, t.dB, nullptr, 0, H2, s));
  // layer 2
  G_(gemm_atb(MLP_H, MLP_H, M, t.dB, MLP_H, H1, MLP_H, gw(MLP_W2), t.part, s));
  G_(colsum(t.dB, M, MLP_H, gw(MLP_B2), t.part, s));
  G_(gemm(M, MLP_H, MLP_H, t.dB, MLP_H, 1, w(MLP_W2), MLP_H, 1, t.dA, nullptr, 0, H1, s));
  // layer 1
  G_(gemm_atb(MLP_H, MLP_IN, M, t.dA, MLP_H, Xn, MLP_IN, gw(MLP_W1), t.part, s));
  G_(colsum(t.dA, M, MLP_H, gw(MLP_B1), t.part, s));
#undef G_
  return cudaGetLastError();
}

}  // namespace pg

// ---------------------------------------------------------------- C-ABI
#include "../../include/pippin_b200.h"
#include "../../include/pippin_b200_mlp.h"

namespace pg {
void internal_set_error(const std::string& msg);
}

namespace {

using namespace pg;

int mlp_fail(int code, const std::string& msg) {
  internal_set_error(msg);
  return code;
}
#define MCK(x)                                                                                  \
  do {                                                                                          \
    cudaError_t _e = (x);                                                                       \
    if (_e != cudaSuccess) return mlp_fail(PG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); \
  } while (0)

// device buffers freed on scope exit
struct DevBufs {
  std::vector<void*> ptrs;
  ~DevBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  cudaError_t alloc(T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<size_t>(n, 1));
    if (e == cudaSuccess) ptrs.push_back(q);
    *p = static_cast<T*>(q);
    return e;
  }
};

// normalised copies of X (with the blob's mean and scale) and Y (/ out scale)
void normalise(const float* wt, const float* X, const float* Y, int64_t n, std::vector<float>& Xn,
               std::vector<float>& Yn) {
  Xn.resize((size_t)n * MLP_IN);
  Yn.resize((size_t)n * MLP_OUT);
  for (int64_t i = 0; i < n; i++) {
    for (int k = 0; k < MLP_IN; k++)
      Xn[i * MLP_IN + k] = (X[i * MLP_IN + k] - wt[MLP_IN_MEAN + k]) * wt[MLP_IN_SCALE + k];
    for (int k = 0; k < MLP_OUT; k++) Yn[i * MLP_OUT + k] = Y[i * MLP_OUT + k] / wt[MLP_OUT_SCALE + k];
  }
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

extern "C" {

int pg_mlp_forward(const float* weights, size_t wlen, const float* X, int64_t n, float* Y) {
  if (!weights || wlen != (size_t)MLP_SIZE) return mlp_fail(PG_ERR_LENGTH, "mlp weights must hold 36662 floats");
  if (n < 0 || (n > 0 && (!X || !Y))) return mlp_fail(PG_ERR_INVALID, "NULL argument");
  if (n == 0) return PG_OK;
  std::vector<uint16_t> wb(MLP_BF16_ELEMS);
  std::vector<float> fb(MLP_F32_ELEMS);
  mlp_pack(weights, wb.data(), fb.data());
  DevBufs d;
  uint16_t* dw;
  float *df, *dx, *dy;
  int* derr;
  MCK(d.alloc(&dw, MLP_BF16_ELEMS));
  MCK(d.alloc(&df, MLP_F32_ELEMS));
  MCK(d.alloc(&dx, (size_t)n * MLP_IN));
  MCK(d.alloc(&dy, (size_t)n * MLP_OUT));
  MCK(d.alloc(&derr, 1));
  MCK(cudaMemset(derr, 0, sizeof(int)));
  MCK(cudaMemcpy(dw, wb.data(), sizeof(uint16_t) * MLP_BF16_ELEMS, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(df, fb.data(), sizeof(float) * MLP_F32_ELEMS, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dx, X, sizeof(float) * n * MLP_IN, cudaMemcpyHostToDevice));
  MCK(mlp_prepare());
  MCK(mlp_forward(MlpDevice{dw, df, derr}, dx, n, dy, 0));
  MCK(cudaMemcpy(Y, dy, sizeof(float) * n * MLP_OUT, cudaMemcpyDeviceToHost));
  int err = 0;
  MCK(cudaMemcpy(&err, derr, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return mlp_fail(PG_ERR_CUDA, "mlp_forward: a wait on the tensor cores ran out");
  return PG_OK;
}

int pg_mlp_loss_grad(const float* weights, size_t wlen, const float* X, const float* Y, int64_t n, float* grad,
                     size_t glen, double* loss) {
  if (!weights || wlen != (size_t)MLP_SIZE) return mlp_fail(PG_ERR_LENGTH, "mlp weights must hold 36662 floats");
  if (!grad || glen != (size_t)MLP_PARAMS) return mlp_fail(PG_ERR_LENGTH, "gradient must hold 36611 floats");
  if (n <= 0 || n > (1 << 24) || !X || !Y) return mlp_fail(PG_ERR_INVALID, "need 1 to 2^24 samples");
  std::vector<float> Xn, Yn;
  normalise(weights, X, Y, n, Xn, Yn);
  int M = (int)n;
  DevBufs d;
  float *P, *G, *dX, *dY;
  TrainBufs t;
  MCK(d.alloc(&P, MLP_PARAMS));
  MCK(d.alloc(&G, MLP_PARAMS));
  MCK(d.alloc(&dX, (size_t)M * MLP_IN));
  MCK(d.alloc(&dY, (size_t)M * MLP_OUT));
  MCK(d.alloc(&t.H, 3 * (size_t)M * MLP_H));
  MCK(d.alloc(&t.O, (size_t)M * MLP_OUT));
  MCK(d.alloc(&t.dO, (size_t)M * MLP_OUT));
  MCK(d.alloc(&t.dA, (size_t)M * MLP_H));
  MCK(d.alloc(&t.dB, (size_t)M * MLP_H));
  MCK(d.alloc(&t.part, train_part_floats()));
  MCK(d.alloc(&t.lpart, train_lpart_doubles(M)));
  MCK(d.alloc(&t.loss, 1));
  MCK(cudaMemcpy(P, weights + MLP_W1, sizeof(float) * MLP_PARAMS, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dX, Xn.data(), sizeof(float) * Xn.size(), cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dY, Yn.data(), sizeof(float) * Yn.size(), cudaMemcpyHostToDevice));
  MCK(cudaMemset(t.loss, 0, sizeof(double)));
  MCK(mlp_batch_grad(P, dX, dY, M, G, t, 0));
  MCK(cudaMemcpy(grad, G, sizeof(float) * MLP_PARAMS, cudaMemcpyDeviceToHost));
  double l = 0.0;
  MCK(cudaMemcpy(&l, t.loss, sizeof(double), cudaMemcpyDeviceToHost));
  if (loss) *loss = l;
  return PG_OK;
}

int pg_mlp_train(const float* X, const float* Y, int64_t n, int epochs, int batch, float lr, uint64_t seed,
                 float* weights, size_t wlen, double* epoch_loss) {
  if (!weights || wlen != (size_t)MLP_SIZE) return mlp_fail(PG_ERR_LENGTH, "mlp weights must hold 36662 floats");
  if (n <= 0 || n > (1 << 26) || !X || !Y) return mlp_fail(PG_ERR_INVALID, "need 1 to 2^26 samples");
  if (epochs < 0 || batch < 1 || batch > 65536 || !(lr > 0.0f)) return mlp_fail(PG_ERR_INVALID, "bad training options");
  // normalisation: feature mean / std, target std (features of zero spread keep scale 1)
  std::vector<float> wt(MLP_SIZE, 0.0f);
  for (int k = 0; k < MLP_IN; k++) {
    double s = 0.0, s2 = 0.0;
    for (int64_t i = 0; i < n; i++) {
      double x = X[i * MLP_IN + k];
      s += x;
      s2 += x * x;
    }
    double mean = s / n, var = std::max(s2 / n - mean * mean, 0.0);
    wt[MLP_IN_MEAN + k] = (float)mean;
    wt[MLP_IN_SCALE + k] = var > 1e-20 ? (float)(1.0 / std::sqrt(var)) : 1.0f;
  }
  for (int k = 0; k < MLP_OUT; k++) {
    double s2 = 0.0;
    for (int64_t i = 0; i < n; i++) s2 += (double)Y[i * MLP_OUT + k] * Y[i * MLP_OUT + k];
    double rms = std::sqrt(s2 / n);
    wt[MLP_OUT_SCALE + k] = rms > 1e-20 ? (float)rms : 1.0f;
  }
  // He-uniform initialisation, zero biases
  uint64_t st = seed;
  auto init = [&](int off, int rows, int cols) {
    double a = std::sqrt(6.0 / cols);
    for (int i = 0; i < rows * cols; i++) wt[off + i] = (float)((2.0 * uniform01(st) - 1.0) * a);
  };
  init(MLP_W1, MLP_H, MLP_IN);
  init(MLP_W2, MLP_H, MLP_H);
  init(MLP_W3, MLP_H, MLP_H);
  init(MLP_W4, MLP_OUT, MLP_H);
  std::vector<float> Xn, Yn;
  normalise(wt.data(), X, Y, n, Xn, Yn);
  int M = (int)std::min<int64_t>(batch, n);
  DevBufs d;
  float *P, *G, *Mo, *Vo, *dX, *dY, *bX, *bY;
  int* idx;
  TrainBufs t;
  MCK(d.alloc(&P, MLP_PARAMS));
  MCK(d.alloc(&G, MLP_PARAMS));
  MCK(d.alloc(&Mo, MLP_PARAMS));
  MCK(d.alloc(&Vo, MLP_PARAMS));
  MCK(d.alloc(&dX, (size_t)n * MLP_IN));
  MCK(d.alloc(&dY, (size_t)n * MLP_OUT));
  MCK(d.alloc(&bX, (size_t)M * MLP_IN));
  MCK(d.alloc(&bY, (size_t)M * MLP_OUT));
  MCK(d.alloc(&idx, (size_t)n));
  MCK(d.alloc(&t.H, 3 * (size_t)M * MLP_H));
  MCK(d.alloc(&t.O, (size_t)M * MLP_OUT));
  MCK(d.alloc(&t.dO, (size_t)M * MLP_OUT));
  MCK(d.alloc(&t.dA, (size_t)M * MLP_H));
  MCK(d.alloc(&t.dB, (size_t)M * MLP_H));
  MCK(d.alloc(&t.part, train_part_floats()));
  MCK(d.alloc(&t.lpart, train_lpart_doubles(M)));
  MCK(d.alloc(&t.loss, 1));
  MCK(cudaMemcpy(P, wt.data() + MLP_W1, sizeof(float) * MLP_PARAMS, cudaMemcpyHostToDevice));
  MCK(cudaMemset(Mo, 0, sizeof(float) * MLP_PARAMS));
  MCK(cudaMemset(Vo, 0, sizeof(float) * MLP_PARAMS));
  MCK(cudaMemcpy(dX, Xn.data(), sizeof(float) * Xn.size(), cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dY, Yn.data(), sizeof(float) * Yn.size(), cudaMemcpyHostToDevice));
  std::vector<int> perm((size_t)n);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  int64_t step = 0;
  for (int ep = 0; ep < epochs; ep++) {
    for (int64_t i = 0; i < n; i++) perm[i] = (int)i;
    for (int64_t i = n - 1; i > 0; i--) std::swap(perm[i], perm[(size_t)(uniform01(st) * (i + 1))]);
    MCK(cudaMemcpy(idx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    MCK(cudaMemset(t.loss, 0, sizeof(double)));
    int nb = 0;
    for (int64_t s0 = 0; s0 + M <= n; s0 += M, nb++) {
      gather_kernel<<<(M * MLP_IN + 255) / 256, 256>>>(dX, idx + s0, M, MLP_IN, bX);
      gather_kernel<<<(M * MLP_OUT + 255) / 256, 256>>>(dY, idx + s0, M, MLP_OUT, bY);
      MCK(mlp_batch_grad(P, bX, bY, M, G, t, 0));
      step++;
      float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
      adam_kernel<<<(MLP_PARAMS + 255) / 256, 256>>>(P, G, Mo, Vo, MLP_PARAMS, lr, b1, b2, eps, c1, c2);
      MCK(cudaGetLastError());
    }
    double l = 0.0;
    MCK(cudaMemcpy(&l, t.loss, sizeof(double), cudaMemcpyDeviceToHost));
    if (epoch_loss) epoch_loss[ep] = nb ? l / nb : 0.0;
  }
  MCK(cudaMemcpy(wt.data() + MLP_W1, P, sizeof(float) * MLP_PARAMS, cudaMemcpyDeviceToHost));
  std::memcpy(weights, wt.data(), sizeof(float) * MLP_SIZE);
  return PG_OK;
}

}  // extern "C"
