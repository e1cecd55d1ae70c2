/* pippin_b200 measurement helpers (no counterpart in the reference). */
#ifndef PIPPIN_B200_TOOLS_H
#define PIPPIN_B200_TOOLS_H

#include "pippin_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* FP64 FMA throughput of `device` in TFLOP/s (2 FLOPs per FMA), timed with
 * CUDA events over one launch of `iters` rounds of 8 x 16 dependent FMAs per
 * thread; the denominator of the FP64-pipe roofline. ms_out may be NULL.
 * Returns 0 on success. */
int pg_fp64_peak(int device, int iters, double* tflops, double* ms_out);

/* Runs `nstep` substeps of envs [start, end) phase kernel by phase kernel,
 * with a CUDA event on the handle's stream between the phases, and adds up
 * the device time of each phase in ms_out[0..3] (smooth dynamics, collision,
 * Newton, and the learned start's inference, which runs between collision
 * and Newton in PG_WARM_LEARNED mode and is 0 otherwise). ctrl_dev, when not
 * NULL, holds (end - start) x nu controls in device memory, copied in before
 * the first substep as pg_step_device does. Steps the simulation like
 * pg_step; synchronises once per substep. Returns PG_OK or a PG_ERR_* code. */
int pg_time_phases(pg_handle* h, int64_t start, int64_t end, int64_t nstep, const double* ctrl_dev,
                   float* ms_out);

/* The launch shape of one phase kernel (0 smooth dynamics, 1 collision,
 * 2 Newton): lanes per env, envs per block, blocks. Any pointer may be NULL.
 * Returns PG_OK or PG_ERR_INVALID. */
int pg_phase_launch(const pg_handle* h, int phase, int* lanes_per_env, int* envs_per_block, int* blocks);

/* How many Newton-phase tiles pg_step_static runs at once out of its fixed
 * scratch array, for tiles of `tile_bytes` and blocks of `tiles_per_block`
 * tiles (a whole number of blocks; the envs beyond them follow in turn).
 * PG_ERR_UNSUPPORTED, with *tiles = 0 and the message pg_step_static gives,
 * when one block does not fit. Pure arithmetic: needs no GPU. */
int pg_static_tiles(size_t tile_bytes, int tiles_per_block, int64_t* tiles);

/* Support vertices of mesh `mesh`'s convex hull as the collision kernel
 * finds them: for each of n directions (host memory, [n][3], in the mesh's
 * own frame) the index of the hull vertex with the largest projection on it
 * (vertex[n], host memory). Hulls of 64 vertices or more walk their vertex
 * graph from vertex 0 and 26 seed vertices, smaller ones scan: the support
 * query of crates/pippin/src/fasthull.rs:76-120. Synchronises the handle's
 * stream. Returns PG_OK or a PG_ERR_* code. */
int pg_hull_support(pg_handle* h, int mesh, const double* dirs, int64_t n, int32_t* vertex);

#ifdef __cplusplus
}
#endif

#endif
