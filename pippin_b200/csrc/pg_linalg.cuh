// Tile-parallel dense FP64 factorisation and solves for the small per-env
// matrices: block-diagonal Cholesky LL^T (crates/pippin/src/math.rs:425-463),
// factored column by column with one lane per row below the diagonal and all
// diagonal blocks advancing together; triangular solves with one lane per
// block. Each entry is computed with the reference's dot-product order.
#pragma once
#include "pg_math.cuh"
#include "pg_tile.cuh"

namespace pg {

// Blocks are [blk[2b], blk[2b+1]); dof_block maps an index to its block
// (null: one block covering [0, n)). Returns false (on every lane) when a
// pivot is not positive.
template <int G>
__device__ bool chol_blocks(const Tile<G>& T, double* A, int stride, int n, int nblk, const int* blk,
                            const int* dof_block, int maxbs) {
  int lane = T.lane();
  bool ok = true;
  for (int jl = 0; jl < maxbs; jl++) {
    // diagonal entries of column jl of every block
    for (int b = lane; b < nblk; b += G) {
      int s0 = blk ? blk[2 * b] : 0, s1 = blk ? blk[2 * b + 1] : n;
      int j = s0 + jl;
      if (j >= s1) continue;
      double* rj = A + j * stride + s0;
      double d = A[j * stride + j] - dot_ref(rj, 1, rj, 1, jl);
      if (d <= 0.0) ok = false;
      A[j * stride + j] = sqrt(d);
    }
    if (!T.all(ok)) return false;
    T.sync();
    // rows below the diagonal
    for (int i = lane; i < n; i += G) {
      int b = dof_block ? dof_block[i] : 0;
      int s0 = blk ? blk[2 * b] : 0, s1 = blk ? blk[2 * b + 1] : n;
      int j = s0 + jl;
      if (j >= s1 || i <= j) continue;
      double inv = 1.0 / A[j * stride + j];
      double* ri = A + i * stride + s0;
      ri[jl] = (ri[jl] - dot_ref(ri, 1, A + j * stride + s0, 1, jl)) * inv;
    }
    T.sync();
  }
  return true;
}

// Solve L L^T x = b in place on each block (math.rs:451-463).
template <int G>
__device__ void solve_blocks(const Tile<G>& T, const double* L, int stride, int n, int nblk, const int* blk,
                             double* x) {
  for (int b = T.lane(); b < nblk; b += G) {
    int s0 = blk ? blk[2 * b] : 0, s1 = blk ? blk[2 * b + 1] : n;
    for (int i = s0; i < s1; i++) x[i] = (x[i] - dot_ref(L + i * stride + s0, 1, x + s0, 1, i - s0)) / L[i * stride + i];
    for (int i = s1 - 1; i >= s0; i--) {
      x[i] /= L[i * stride + i];
      double xi = -x[i];
      const double* li = L + i * stride + s0;
      for (int k = 0; k < i - s0; k++) x[s0 + k] += xi * li[k];
    }
  }
  T.sync();
}

}  // namespace pg
