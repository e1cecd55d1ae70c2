// Cholesky factorisation and solves for the small dense matrices of models
// with at most 16 dofs (crates/pippin/src/math.rs:425-463), for tiles of 16
// or 32 lanes with one lane per row, in place of the block versions in
// pg_linalg.cuh. Two forms, chosen by measurement:
//
// chol_left / solve_left (the smooth phase's factors, the damped solve,
// set_const): the reference's left-looking column order in shared memory,
// one column per pass of a loop. The code is a few dozen instructions, which
// matters more in a kernel that runs a long stretch of straight-line code
// per env than the extra dot-product latency does.
//
// chol_regx / solve_regx (the register Newton, factoring every iteration):
// right-looking with the lane's row in registers and the column loop
// unrolled, so each column's rank-1 update is independent FMAs; the
// finished entries go to a packed store that the lanes exchange them
// through. Every lane forms 1/L_jj = rsqrt(d) from the diagonal shuffled
// out of lane j, so no lane waits on a shared write for the pivot.
//
// In both, the solves keep the unknown of row i in lane i's register; each
// step of the forward and backward sweep is one shuffle of the finished
// unknown, one load and one FMA per lane. A block-diagonal matrix (several
// dof trees) factors to the same block-diagonal L: entries across blocks
// start at zero and stay exactly zero.
#pragma once
#include "pg_linalg.cuh"

namespace pg {

constexpr int SMALL_N = 16;  // largest matrix the one-lane-per-row path factors

// dot_ref's summation order (four interleaved partial sums for n >= 8, then
// the tail) for a row and a vector in shared memory, as a loop (small code).
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

// Store of a factor's entries: row k's entries L_k0 .. at row(k), a matrix
// with row stride ld (lower triangle and diagonal).
struct LStrided {
  double* p;
  int ld;
  __device__ double* row(int k) const { return p + k * ld; }
};

// L L^T = A in place in the store (math.rs:425-447's column order: pivot
// L_jj = sqrt(A_jj - row_j . row_j), then L_ij = (A_ij - row_i . row_j) / L_jj
// below it, each dot over the first j entries in dot_ref's order), one column
// per pass of a loop with one lane per row. On entry row i of the store holds
// A_i0 .. A_i,i-1 and dg = A_ii on lane i. In pass j every lane i >= j forms
// its dot with row j (lane j's is the pivot's), the pivot comes to every
// lane by one shuffle, and 1/L_jj from one reciprocal square root
// (L_jj = d * rsqrt(d)); lane i > j overwrites A_ij with L_ij, lane j writes
// L_jj when `diag`. One tile sync per column. *rv = 1 / L_ii on lane i.
// Returns false (uniformly over the tile) if a pivot is not positive.
template <int G, class S>
__device__ inline bool chol_left(const Tile<G>& T, const S& st, int n, double dg, bool diag, double* rv) {
  const int i = T.lane();
  const bool row = i < n;
  double* mine = st.row(row ? i : 0);
  T.sync();  // every row in place
#pragma unroll 1
  for (int j = 0; j < n; j++) {
    const double* rj = st.row(j);
    double s = (row && i >= j) ? dot_ref_sm(mine, rj, j) : 0.0;
    double d = T.bcast(dg - s, j);
    if (!(d > 0.0)) return false;  // d is the same on every lane
    double inv = rsqrt(d);
    if (i == j) {
      *rv = inv;
      if (diag) mine[j] = d * inv;
    } else if (row && i > j) {
      mine[j] = (mine[j] - s) * inv;
    }
    T.sync();
  }
  return true;
}

// chol_left on two matrices of the same size at once (the smooth phase's M
// and M + hD): each pass does both columns' dots and pivots, so the two
// chains of dependent steps overlap. Same arithmetic as two chol_left calls;
// false if either has a pivot that is not positive.
template <int G, class S>
__device__ inline bool chol_left2(const Tile<G>& T, const S& s1, const S& s2, int n, double dg1, double dg2,
                                  double* rv1, double* rv2) {
  const int i = T.lane();
  const bool row = i < n;
  double* m1 = s1.row(row ? i : 0);
  double* m2 = s2.row(row ? i : 0);
  T.sync();  // every row in place
#pragma unroll 1
  for (int j = 0; j < n; j++) {
    const double* r1 = s1.row(j);
    const double* r2 = s2.row(j);
    double a1 = 0.0, a2 = 0.0;
    if (row && i >= j) {
      a1 = dot_ref_sm(m1, r1, j);
      a2 = dot_ref_sm(m2, r2, j);
    }
    double d1 = T.bcast(dg1 - a1, j);
    double d2 = T.bcast(dg2 - a2, j);
    if (!(d1 > 0.0) || !(d2 > 0.0)) return false;  // the same on every lane
    double inv1 = rsqrt(d1), inv2 = rsqrt(d2);
    if (i == j) {
      *rv1 = inv1;
      *rv2 = inv2;
      m1[j] = d1 * inv1;
      m2[j] = d2 * inv2;
    } else if (row && i > j) {
      m1[j] = (m1[j] - a1) * inv1;
      m2[j] = (m2[j] - a2) * inv2;
    }
    T.sync();
  }
  return true;
}

// The solution component of lane i of L L^T x = b, given b_i (xi), 1/L_ii
// (ri) and the factor's store: forward x_i -= L_ij (x_j / L_jj) for i > j,
// then x_i /= L_ii; backward x_i -= L_ji (x_j / L_jj) for i < j, then
// x_i /= L_ii. Each step is one shuffle of the finished unknown, one load
// and one FMA per lane.
template <int G, class S>
__device__ inline double solve_left(const Tile<G>& T, const S& st, int n, double ri, double xi) {
  const int i = T.lane();
  const bool row = i < n;
  const double* mine = st.row(row ? i : 0);
#pragma unroll 1
  for (int j = 0; j < n; j++) {
    double lij = (row && i > j) ? mine[j] : 0.0;
    double y = T.bcast(xi * ri, j);
    if (row && i > j) xi -= lij * y;
  }
  xi *= ri;
#pragma unroll 1
  for (int j = n - 1; j >= 0; j--) {
    double lji = i < j ? st.row(j)[i] : 0.0;
    double y = T.bcast(xi * ri, j);
    if (i < j) xi -= lji * y;
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
  double rv = 0.0;
  if (!chol_left(T, LStrided{A, lda}, n, row ? A[i * lda + i] : 0.0, true, &rv)) return false;
  if (row) rinv[i] = rv;
  T.sync();
  return true;
}

// chol_small on A and A2 (both n x n, stride lda) side by side.
template <int G>
__device__ __noinline__ bool chol_small2(const Tile<G>& T, double* A, double* A2, int lda, int n, double* rinv,
                                         double* rinv2) {
  static_assert(G >= SMALL_N, "one lane per row");
  const int i = T.lane();
  const bool row = i < n;
  double rv1 = 0.0, rv2 = 0.0;
  if (!chol_left2(T, LStrided{A, lda}, LStrided{A2, lda}, n, row ? A[i * lda + i] : 0.0,
                  row ? A2[i * lda + i] : 0.0, &rv1, &rv2))
    return false;
  if (row) {
    rinv[i] = rv1;
    rinv2[i] = rv2;
  }
  T.sync();
  return true;
}

// Solve L L^T x = b in place (x holds b on entry), with L and rinv from
// chol_small (or chol_blocks on one block).
template <int G>
__device__ __noinline__ void solve_small(const Tile<G>& T, const double* L, int lda, int n, const double* rinv,
                                         double* x) {
  static_assert(G >= SMALL_N, "one lane per row");
  const int i = T.lane();
  const bool row = i < n;
  double xi = solve_left(T, LStrided{const_cast<double*>(L), lda}, n, row ? rinv[i] : 0.0, row ? x[i] : 0.0);
  T.sync();
  if (row) x[i] = xi;
  T.sync();
}

// Right-looking L L^T = A with the rows of L left in registers (lane i:
// a[k] = A_ik, k <= i, on entry, a[k] = L_ik on return)
// and the entries below the diagonal also written to the packed store Lr
// (row k's entries L_k0 .. L_k,k-1 at k(k-1)/2, so that every offset the
// unrolled loops use is a constant), which is how the lanes exchange them:
// every entry has its own slot, so one tile sync per column suffices.
// *rv = 1 / L_ii. The pivot's reciprocal comes from one reciprocal square
// root (L_jj = d / sqrt(d) as d * rsqrt(d)).
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

// The solve for a factor from chol_regx: the forward sweep uses the row in
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

// Factor / solve one lane per row when the tile and the matrix allow it,
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
