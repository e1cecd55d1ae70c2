// A tile of G lanes (G = 8, 16 or 32) that cooperates on one environment.
// Reductions are butterfly (xor) all-reduces, so every lane ends with the
// bit-identical value and control flow that depends on it stays uniform.
#pragma once
#include <cooperative_groups.h>

namespace pg {
namespace cg = cooperative_groups;

template <int G>
struct Tile {
  cg::thread_block_tile<G> t;
  __device__ explicit Tile(cg::thread_block_tile<G> tt) : t(tt) {}
  __device__ int lane() const { return (int)t.thread_rank(); }
  __device__ void sync() const { t.sync(); }
  template <class T>
  __device__ T bcast(T v, int src) const {
    return t.shfl(v, src);
  }
  __device__ double sum(double v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += t.shfl_xor(v, o);
    return v;
  }
  __device__ int isum(int v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += t.shfl_xor(v, o);
    return v;
  }
  __device__ int ior(int v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v |= t.shfl_xor(v, o);
    return v;
  }
  __device__ double fmax(double v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = ::fmax(v, t.shfl_xor(v, o));
    return v;
  }
  __device__ int imin(int v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = ::min(v, t.shfl_xor(v, o));
    return v;
  }
  // the largest *v over the tile, ties to the smallest *idx; on every lane
  __device__ void argmax(double* v, int* idx) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      double ov = t.shfl_xor(*v, o);
      int oi = t.shfl_xor(*idx, o);
      if (ov > *v || (ov == *v && oi < *idx)) {
        *v = ov;
        *idx = oi;
      }
    }
  }
  // bit k set when lane k's b is true
  __device__ unsigned ballot(bool b) const { return t.ballot(b ? 1 : 0); }
  __device__ bool all(bool b) const { return t.all(b ? 1 : 0) != 0; }
  __device__ bool any(bool b) const { return t.any(b ? 1 : 0) != 0; }
  // exclusive prefix sum over lanes; *total gets the sum over the tile
  __device__ int excl_scan(int v, int* total) const {
    int x = v;
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
      int y = t.shfl_up(x, o);
      if (lane() >= o) x += y;
    }
    *total = t.shfl(x, G - 1);
    return x - v;
  }
};

// Global -> shared copies issued back to back without waiting (cp.async);
// load_wait() completes this lane's copies, a tile sync then publishes them.
__device__ inline void cp_async8(double* dst_shared, const double* src_global) {
  unsigned d = (unsigned)__cvta_generic_to_shared(dst_shared);
  size_t s = __cvta_generic_to_global(src_global);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(s) : "memory");
}
template <int G>
__device__ inline void load_async(const Tile<G>& T, double* dst_shared, const double* src_global, int n) {
  for (int k = T.lane(); k < n; k += G) cp_async8(dst_shared + k, src_global + k);
}
__device__ inline void load_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Pull `bytes` of global memory into L1 (one 128-byte line per request,
// spread over the tile's lanes), so that the dependent loads that follow hit
// L1 instead of waiting on L2 one after another.
template <int G>
__device__ inline void prefetch_l1(const Tile<G>& T, const void* p, size_t bytes) {
  const char* c = static_cast<const char*>(p);
  for (size_t off = (size_t)T.lane() * 128; off < bytes; off += (size_t)G * 128)
    asm volatile("prefetch.global.L1 [%0];\n" ::"l"(c + off));
}

}  // namespace pg
