// Tile-parallel dense FP64 factorisation and solves for the small per-env
// matrices (crates/pippin/src/math.rs:425-463).
//
// Cholesky LL^T is left-looking, column by column: the block's lane for the
// column forms the pivot with the reference's dot-product order, then one
// lane per row below it forms L[i][j] (again the reference's order). All
// diagonal blocks advance together. The reciprocal pivots are kept for the
// solves, which are column-oriented: at step j every row below (forward) or
// above (backward) subtracts its multiple of the finished unknown in
// parallel, one tile sync per step.
#pragma once
#include "pg_math.cuh"
#include "pg_tile.cuh"

namespace pg {

// Blocks: nblk of them, [blk[2b], blk[2b+1]); with blk == nullptr a single
// block [0, n). dof_block maps a row to its block. rinv[i] = 1 / L[i][i].
// Returns false (uniformly) if a pivot is not positive.
template <int G>
__device__ __noinline__ bool chol_blocks(const Tile<G>& T, double* A, int stride, int n, int nblk, const int* blk,
                            const int* dof_block, int maxbs, double* rinv) {
  int lane = T.lane();
  bool ok = true;
  for (int jl = 0; jl < maxbs; jl++) {
    for (int b = lane; b < nblk; b += G) {
      int s0 = blk ? blk[2 * b] : 0, s1 = blk ? blk[2 * b + 1] : n;
      int j = s0 + jl;
      if (j >= s1) continue;
      const double* rj = A + j * stride + s0;
      double d = A[j * stride + j] - dot_ref(rj, 1, rj, 1, jl);
      if (!(d > 0.0)) ok = false;
      double r = sqrt(d);
      A[j * stride + j] = r;
      rinv[j] = 1.0 / r;
    }
    if (!T.all(ok)) return false;
    T.sync();
    for (int i = lane; i < n; i += G) {
      int s0 = 0, s1 = n;
      if (blk) {
        int b = dof_block[i];
        s0 = blk[2 * b];
        s1 = blk[2 * b + 1];
      }
      int j = s0 + jl;
      if (j >= s1 || i <= j) continue;
      double* ri = A + i * stride + s0;
      ri[jl] = (ri[jl] - dot_ref(ri, 1, A + j * stride + s0, 1, jl)) * rinv[j];
    }
    T.sync();
  }
  return true;
}

// Solve L L^T x = b in place on every block, given chol_blocks' factor and
// reciprocal pivots.
template <int G>
__device__ __noinline__ void solve_blocks(const Tile<G>& T, const double* L, int stride, int n, int nblk, const int* blk,
                             const int* dof_block, int maxbs, const double* rinv, double* x) {
  int lane = T.lane();
  // forward: x[i] -= L[i][j] y_j for i > j in j's block, y_j = x[j] / L[j][j]
  for (int jl = 0; jl < maxbs; jl++) {
    for (int i = lane; i < n; i += G) {
      int s0 = 0, s1 = n;
      if (blk) {
        int b = dof_block[i];
        s0 = blk[2 * b];
        s1 = blk[2 * b + 1];
      }
      int j = s0 + jl;
      if (j >= s1 || i <= j) continue;
      x[i] -= L[i * stride + j] * (x[j] * rinv[j]);
    }
    T.sync();
  }
  for (int i = lane; i < n; i += G) x[i] *= rinv[i];
  T.sync();
  // backward: x[i] -= L[j][i] x_j for i < j in j's block
  for (int jl = maxbs - 1; jl >= 0; jl--) {
    for (int i = lane; i < n; i += G) {
      int s0 = 0, s1 = n;
      if (blk) {
        int b = dof_block[i];
        s0 = blk[2 * b];
        s1 = blk[2 * b + 1];
      }
      int j = s0 + jl;
      if (j >= s1 || i >= j) continue;
      x[i] -= L[j * stride + i] * (x[j] * rinv[j]);
    }
    T.sync();
  }
  for (int i = lane; i < n; i += G) x[i] *= rinv[i];
  T.sync();
}

}  // namespace pg
