// Register-resident Cholesky factorisation and solves for the small dense
// matrices of models with at most 16 dofs (crates/pippin/src/math.rs:425-463),
// used by tiles of 16 or 32 lanes in place of the shared-memory versions in
// pg_linalg.cuh.
//
// Lane i keeps row i of the matrix in registers. The factorisation is
// right-looking: at column j every lane forms 1/L_jj = rsqrt(d) and
// L_jj = d / sqrt(d) itself from the diagonal shuffled out of lane j (so no
// lane waits on a shared write for it), scales its own entry below the pivot,
// publishes it, and after one tile sync applies the rank-1 update to its row,
// reading the finished column as broadcast loads. A block-diagonal matrix
// (several dof trees) factors to the same block-diagonal L: entries across
// blocks start at zero and stay exactly zero.
//
// The solves keep the unknown of row i in lane i's register; each step of
// the forward and backward sweep is one shuffle of the finished unknown and
// one FMA per lane, with the L entry the lane needs read from shared memory.
#pragma once
#include "pg_linalg.cuh"

namespace pg {

constexpr int SMALL_N = 16;  // largest matrix the register path factors

// dot_ref's summation order (four interleaved partial sums for n >= 8, then
// the tail) for a row held in registers against a vector in shared memory.
__device__ inline double dot_ref_reg(const double (&a)[SMALL_N], const double* x, int n) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  int n4 = n >= 8 ? (n & ~3) : 0;
#pragma unroll
  for (int k = 0; k < SMALL_N; k++)
    if (k < n4) s[k & 3] += a[k] * x[k];
  double t = (s[0] + s[1]) + (s[2] + s[3]);
#pragma unroll
  for (int k = 0; k < SMALL_N; k++)
    if (k >= n4 && k < n) t += a[k] * x[k];
  return t;
}

// The same for a row in shared memory, as a loop (small code).
__device__ inline double dot_ref_sm(const double* a, const double* x, int n) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int n4 = n >= 8 ? (n & ~3) : 0;
#pragma unroll 1
  for (int k = 0; k < n4; k += 4) {
    s0 += a[k] * x[k];
    s1 += a[k + 1] * x[k + 1];
    s2 += a[k + 2] * x[k + 2];
    s3 += a[k + 3] * x[k + 3];
  }
  double t = (s0 + s1) + (s2 + s3);
#pragma unroll 1
  for (int k = n4; k < n; k++) t += a[k] * x[k];
  return t;
}

// Factor the rows held in registers (lane i: a[k] = A_ik, k <= i) into L,
// written to L (shared, stride lda: lower triangle and diagonal) as each
// column finishes and left in a[]; *rv = 1 / L_ii on lane i. Returns false
// (uniformly over the tile) if a pivot is not positive. The pivot's
// reciprocal comes from one reciprocal square root, not a square root and a
// division.
template <int G>
__device__ inline bool chol_reg(const Tile<G>& T, double (&a)[SMALL_N], int n, double* L, int lda, double* rv) {
  const int i = T.lane();
  const bool row = i < n;
#pragma unroll
  for (int j = 0; j < SMALL_N; j++) {
    if (j >= n) break;
    double d = T.bcast(a[j], j);
    if (!(d > 0.0)) return false;  // d is the same on every lane
    double inv = rsqrt(d);  // 1 / L_jj; L_jj = d / sqrt(d) as d * inv
    double l = 0.0;
    if (i == j) {
      a[j] = d * inv;
      *rv = inv;
    } else if (i > j) {
      l = a[j] * inv;
      a[j] = l;
    }
    if (row && i >= j) L[i * lda + j] = a[j];
    T.sync();
#pragma unroll
    for (int k = j + 1; k < SMALL_N; k++)
      if (k < n) a[k] -= l * L[k * lda + j];
  }
  return true;
}

// chol_reg with the rows of L left in registers (lane i: a[k] = L_ik, k <= i)
// and the entries below the diagonal also written to the packed store Lr
// (row k's entries L_k0 .. L_k,k-1 at k(k-1)/2, so that every offset the
// unrolled loops use is a constant), which is how the lanes exchange them:
// every entry has its own slot, so one tile sync per column suffices.
// *rv = 1 / L_ii. Same arithmetic as chol_reg.
template <int G>
__device__ inline bool chol_regx(const Tile<G>& T, double (&a)[SMALL_N], int n, double* Lr, double* rv) {
  const int i = T.lane();
  double* row = Lr + (i < n ? i * (i - 1) / 2 : 0);  // this lane's row of the store
#pragma unroll
  for (int j = 0; j < SMALL_N; j++) {
    if (j >= n) break;
    double d = T.bcast(a[j], j);
    if (!(d > 0.0)) return false;  // d is the same on every lane
    double inv = rsqrt(d);  // 1 / L_jj; L_jj = d / sqrt(d) as d * inv
    double l = 0.0;
    if (i == j) {
      a[j] = d * inv;
      *rv = inv;
    } else if (i > j) {
      l = a[j] * inv;
      a[j] = l;
      if (i < n) row[j] = l;
    }
    T.sync();
#pragma unroll
    for (int k = j + 1; k < SMALL_N; k++)
      if (k < n) a[k] -= l * Lr[k * (k - 1) / 2 + j];
  }
  return true;
}

// solve_reg for a factor from chol_regx: the forward sweep uses the row in
// registers, the backward sweep reads L_ji from the packed store; each step
// is one shuffle of the finished unknown and one FMA per lane, with no syncs.
template <int G>
__device__ inline double solve_regx(const Tile<G>& T, const double (&a)[SMALL_N], int n, const double* Lr, double ri,
                                    double xi) {
  const int i = T.lane();
#pragma unroll
  for (int j = 0; j < SMALL_N; j++) {
    if (j >= n) break;
    double y = T.bcast(xi * ri, j);
    if (i > j) xi -= a[j] * y;
  }
  xi *= ri;
  const double* col = Lr + (i < SMALL_N ? i : 0);  // col[j(j-1)/2] = L_ji
#pragma unroll
  for (int j = SMALL_N - 1; j >= 0; j--) {
    if (j >= n) continue;
    double y = T.bcast(xi * ri, j);
    if (i < j) xi -= col[j * (j - 1) / 2] * y;
    asm volatile("" ::: "memory");  // one load a step, not all of them up front
  }
  return xi * ri;
}

// In-place L L^T = A for the n x n matrix at A (row-major, stride lda; the
// lower triangle is read, the lower triangle and diagonal are overwritten
// with L, the strict upper triangle is left alone); rinv[i] = 1 / L_ii.
// Returns false (uniformly over the tile) if a pivot is not positive.
template <int G>
__device__ __noinline__ bool chol_small(const Tile<G>& T, double* A, int lda, int n, double* rinv) {
  static_assert(G >= SMALL_N, "one lane per row");
  const int i = T.lane();
  const bool row = i < n;
  double a[SMALL_N];
#pragma unroll
  for (int k = 0; k < SMALL_N; k++) a[k] = (row && k <= i) ? A[i * lda + k] : 0.0;
  double rv = 0.0;
  if (!chol_reg(T, a, n, A, lda, &rv)) return false;
  if (row) rinv[i] = rv;
  T.sync();
  return true;
}

// The solution component of lane i of L L^T x = b, given b_i (xi), 1/L_ii
// (ri) and L in shared memory (stride lda). Same arithmetic as solve_blocks.
template <int G>
__device__ inline double solve_reg(const Tile<G>& T, const double* L, int lda, int n, double ri, double xi) {
  const int i = T.lane();
  const bool row = i < n;
  // forward: x_i -= L_ij (x_j / L_jj) for i > j, then x_i /= L_ii
#pragma unroll
  for (int j = 0; j < SMALL_N; j++) {
    if (j >= n) break;
    double y = T.bcast(xi * ri, j);
    if (row && i > j) xi -= L[i * lda + j] * y;
  }
  xi *= ri;
  // backward: x_i -= L_ji (x_j / L_jj) for i < j, then x_i /= L_ii
#pragma unroll
  for (int j = SMALL_N - 1; j >= 0; j--) {
    if (j >= n) continue;
    double y = T.bcast(xi * ri, j);
    if (i < j) xi -= L[j * lda + i] * y;
  }
  return xi * ri;
}

// Solve L L^T x = b in place (x holds b on entry), with L and rinv from
// chol_small (or chol_blocks on one block). Same arithmetic as solve_blocks.
template <int G>
__device__ __noinline__ void solve_small(const Tile<G>& T, const double* L, int lda, int n, const double* rinv,
                                         double* x) {
  static_assert(G >= SMALL_N, "one lane per row");
  const int i = T.lane();
  const bool row = i < n;
  double xi = solve_reg(T, L, lda, n, row ? rinv[i] : 0.0, row ? x[i] : 0.0);
  T.sync();
  if (row) x[i] = xi;
  T.sync();
}

// Factor / solve on the register path when the tile and the matrix allow it,
// else on the shared-memory block path. Block arguments as chol_blocks.
template <int G>
__device__ inline bool chol_auto(const Tile<G>& T, double* A, int lda, int n, int nblk, const int* blk,
                                 const int* dof_block, int maxbs, double* rinv) {
  if constexpr (G >= SMALL_N) {
    if (n <= SMALL_N) return chol_small(T, A, lda, n, rinv);
  }
  return chol_blocks(T, A, lda, n, nblk, blk, dof_block, maxbs, rinv);
}

template <int G>
__device__ inline void solve_auto(const Tile<G>& T, const double* L, int lda, int n, int nblk, const int* blk,
                                  const int* dof_block, int maxbs, const double* rinv, double* x) {
  if constexpr (G >= SMALL_N) {
    if (n <= SMALL_N) {
      solve_small(T, L, lda, n, rinv, x);
      return;
    }
  }
  solve_blocks(T, L, lda, n, nblk, blk, dof_block, maxbs, rinv, x);
}

}  // namespace pg
