// cell_sort.cuh -- particles ordered by their deposit cell, and the deposits that exploit it.
//
// The reference deposits and gathers particle by particle in the caller's order
// (deposit_particles, code/open_spacecharge_mod.f90:257-283; interpolate_field, :311-390).
// On the GPU the order decides the cost: in random order every particle's CIC stencil is a
// separate set of L2 transactions, while particles sorted by cell share them.  This module
// sorts by the deposit cell (a counting sort keyed by the cell's lowest corner) and
// provides deposits whose work is per run of equal cells instead of per particle.
#pragma once

#include "particle_kernels.cuh"

namespace osc {

// Counting sort by deposit cell.  key(m) = i + nx*(j + ny*k) of the lowest corner of the
// particle's cell, computed with the deposit's formula (mode 0 of DepositArgs), or N =
// nx*ny*nz for a particle whose stencil leaves the mesh or whose coordinate is not finite
// (those go last).  Within a cell the order is unspecified.
//   keys/ranks: per particle (np); counts: N + 1 zeroed words on entry, per-cell starts
//   (exclusive prefix sums) on exit, with counts[N + 1] = np; partials: scan scratch of
//   cell_scan_partials(N + 2) words.  counters[0] += outside, counters[1] += non-finite.
int launch_cell_keys(const DepositArgs &a, uint32_t *keys, uint32_t *ranks, uint32_t *counts,
                     unsigned long long *counters, cudaStream_t st);
int64_t cell_scan_partials(int64_t n);
int launch_cell_scan(uint32_t *counts, int64_t n, uint32_t *partials, cudaStream_t st);
// Sorted copies: pos = start[key[m]] + rank[m]; xs[pos] = x[m] (y, z, q alike; q and qs
// may be null), perm64/perm32 (either may be null) [pos] = m, inv (nullable) [m] = pos.
int launch_cell_scatter(int64_t np, const uint32_t *keys, const uint32_t *ranks, const uint32_t *start,
                        const double *x, const double *y, const double *z, const double *q, double *xs,
                        double *ys, double *zs, double *qs, int64_t *perm64, uint32_t *inv, cudaStream_t st);

// FP32 quad-grid deposit (the layout of launch_deposit_quad) for particles in cell order:
// each lane walks a run of consecutive particles, sums the quad contributions of equal
// cells in FP32 with compensated two-sum accumulation, and adds each run's sum to the grid
// with two float4 reductions.  Correct for any order; in cell order most particles add
// nothing to L2.
int launch_deposit_quad_runs(const DepositArgs &a, float *quad, unsigned long long *counters, cudaStream_t st);

// Fixed-point deposit (the contributions of launch_deposit<unsigned long long>, rounded
// identically) with each run of equal cells summed exactly in 64-bit integers before its
// eight integer reductions: the same bits as the per-particle fixed-point deposit for any
// particle order, with few reductions when the particles are in cell order.
int launch_deposit_fixed_runs(const DepositArgs &a, unsigned long long *acc, unsigned long long *counters,
                              cudaStream_t st);

// E[m][c] = Es[inv[m]][c]: fields gathered in sorted order back to the caller's order.
int launch_unpermute_rows3(int64_t np, const uint32_t *inv, const double *Es, double *E, cudaStream_t st);

}  // namespace osc
