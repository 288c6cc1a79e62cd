// particle_kernels.cuh -- charge deposition, field interpolation and particle reductions.
#pragma once

#include "osc_common.cuh"

namespace osc {

// CIC deposition.  mode 0 follows deposit_particles (code/open_spacecharge_mod.f90:257-283):
// ip = floor((x-xmin)*dxi + 1) with the product rounded before the add (no fused multiply-
// add, as the reference evaluates it, so a particle on a cell plane gets the reference's
// cell), low-node weight ab = ((xmin-x) + ip*dx)*dxi, charge per
// particle.  mode 1 follows depose_rho_scalar (code/test_mod.f90:442-470): ip uses the
// global lower index nlogbl, lost particles are skipped, weights carry no charge (the grid
// is scaled afterwards).  Particles whose stencil leaves the array are counted, not written.
struct DepositArgs {
    int64_t np;
    const double *x, *y, *z, *q, *lost;
    double xmin, ymin, zmin, dx, dy, dz, dxi, dyi, dzi;
    int nlo[3], nhi[3], nlogbl[3];
    int nx, ny, nz;
    int mode;
    double charge1;  // charge per particle when q == nullptr (mode 0)
    int check_finite;
    double fx_scale;  // fixed-point accumulation: units per unit charge
    // launch shape chosen by the autotuner (0 = built-in default): particles per lane of the
    // run-aggregated deposits (4 or 8) and CTAs per SM of the per-particle deposit
    int tile = 0;
    int ctas = 0;
};
// Cell and low-node weights of deposit_particles (mode 0; code/open_spacecharge_mod.f90:
// 259-269): ip = floor((x-xmin)*dxi + 1) with the product rounded before the add, and
// ab = ((xmin-x) + ip*dx)*dxi with every product and sum rounded separately (no fused
// multiply-add), as the reference and the oracle evaluate them.  Returns 0 with the cell's
// array indices (i, j, k) and weights when the 2x2x2 stencil lies inside the array, 1 when
// it leaves it, 2 for a non-finite coordinate (only when a.check_finite is set; otherwise
// such a particle lands outside).
struct CicCell {
    int i, j, k;
    double ab, de, gh;
};
__device__ __forceinline__ int cic_cell_mode0(const DepositArgs &a, double xm, double ym, double zm, CicCell &c) {
    if (a.check_finite && !(isfinite(xm) && isfinite(ym) && isfinite(zm))) return 2;
    const double fx = floor(__dadd_rn(__dmul_rn(xm - a.xmin, a.dxi), 1.0));
    const double fy = floor(__dadd_rn(__dmul_rn(ym - a.ymin, a.dyi), 1.0));
    const double fz = floor(__dadd_rn(__dmul_rn(zm - a.zmin, a.dzi), 1.0));
    if (!(fx >= a.nlo[0] && fx + 1 <= a.nhi[0] && fy >= a.nlo[1] && fy + 1 <= a.nhi[1] && fz >= a.nlo[2] &&
          fz + 1 <= a.nhi[2]))
        return 1;
    c.ab = __dmul_rn(__dadd_rn(a.xmin - xm, __dmul_rn(fx, a.dx)), a.dxi);
    c.de = __dmul_rn(__dadd_rn(a.ymin - ym, __dmul_rn(fy, a.dy)), a.dyi);
    c.gh = __dmul_rn(__dadd_rn(a.zmin - zm, __dmul_rn(fz, a.dz)), a.dzi);
    c.i = (int)fx - a.nlo[0];
    c.j = (int)fy - a.nlo[1];
    c.k = (int)fz - a.nlo[2];
    return 0;
}

// counters[0] += outside particles, counters[1] += non-finite particles.  TA = float or
// double: floating-point atomics; TA = unsigned long long: each contribution rounded to
// a 64-bit fixed-point integer (value * fx_scale), so the sum is exact and independent of
// the order of the atomics (deterministic deposition).
template <typename TA>
int launch_deposit(const DepositArgs &a, TA *rho, unsigned long long *counters, cudaStream_t st);
// out[n] = mult * (signed) acc[n] / fx_scale
template <typename TO>
int launch_fixed_to_real(const unsigned long long *acc, TO *out, double fx_scale, double mult, int64_t n,
                         cudaStream_t st);

// FP32 step deposit: two float4 atomics per particle into a quad grid (N float4; node
// (i,j,k) holds the plane-k contributions to nodes (i,j), (i+1,j), (i,j+1), (i+1,j+1)),
// then launch_quad_to_nodes sums every node's four slots in a fixed order.
int launch_deposit_quad(const DepositArgs &a, float *quad, unsigned long long *counters, cudaStream_t st);
int launch_quad_to_nodes(const float *quad, float *rho, int nx, int ny, int nz, cudaStream_t st);

// CIC gather (interpolate_field, code/open_spacecharge_mod.f90:311-390): clamp cells to
// [1, nhi-1] (and the array), weights computed after clamping, 8-node sum in the
// reference's order.  Source: a vec4<T> interleaved grid or three double planes.
struct InterpArgs {
    int64_t np;
    const double *x, *y, *z;
    double min[3], delta[3], hinv[3];
    int nlo[3], nhi[3];
    int nx, ny, nz;
    // launch shape chosen by the autotuner (0 = built-in default): particles per lane of the
    // cell-ordered gather (4 or 8) and CTAs per SM of the per-particle gather
    int tile = 0;
    int ctas = 0;
};
template <typename T>
int launch_interp_vec4(const InterpArgs &a, const void *E4, double *E, unsigned long long *nclamp,
                       cudaStream_t st);
// out_f32 != 0: E is float [np][3]
template <typename T>
int launch_interp_vec4_any(const InterpArgs &a, const void *E4, void *E, int out_f32,
                           unsigned long long *nclamp, cudaStream_t st);
int launch_interp_planes(const InterpArgs &a, const double *F, double *out,
                         unsigned long long *nclamp, cudaStream_t st);
// Gather from an x-pair grid: node n holds (E(n), E(n+1)) as two float4 in one 32-byte
// sector, so the 8 nodes of a particle come from 4 sectors.
int launch_interp_pairs(const InterpArgs &a, const float4 *E8, double *E, unsigned long long *nclamp,
                        cudaStream_t st);
// The same gather for particles in cell order: runs of consecutive particles in one cell
// share their stencil's loads; coordinates and E move as 256-bit vectors.  Bit-identical
// to launch_interp_pairs for any order.
int launch_interp_pairs_runs(const InterpArgs &a, const float4 *E8, double *E, unsigned long long *nclamp,
                             cudaStream_t st);

// Bounding box {xmin,xmax,ymin,ymax,zmin,zmax} of the particles, written to bb (device)
// through order-preserving 64-bit keys; also counts non-finite coordinates.
int launch_bbox(int64_t np, const double *x, const double *y, const double *z,
                unsigned long long *keys /*6*/, double *bb /*6*/, unsigned long long *nonfinite,
                cudaStream_t st);
// Deterministic sum of q (two passes, fixed order) into *out.
// Sum of q (or, with max_abs, the largest |q|), reduced in a fixed order.
int launch_sum(int64_t n, const double *q, double *partials /*>= 1024*/, double *out, cudaStream_t st,
               bool max_abs = false);

// ---- batches of bunches ---------------------------------------------------------------
// One CTA's share of a batched particle pass: particles [beg, end) of bunch `bunch`.
struct BatchJob {
    int bunch;
    int64_t beg, end;
};
// Per-bunch arguments of the batched passes: particle pointers already offset to the
// bunch, its mesh, the first node of its grid in the batch arrays and its E output.
struct BunchArgs {
    DepositArgs d;
    InterpArgs in;
    int64_t node_off;
    double *E;
};
// cnt[4b + 0] += outside, cnt[4b + 1] += non-finite (deposit); cnt[4b + 2] += clamped (interp)
int launch_batch_deposit_quad(const BunchArgs *bunches, const BatchJob *jobs, int njobs, float *quad,
                              unsigned long long *cnt, cudaStream_t st);
int launch_batch_interp_pairs(const BunchArgs *bunches, const BatchJob *jobs, int njobs, const float *e8,
                              unsigned long long *cnt, cudaStream_t st);
// Per-bunch min/max of x, y, z, non-finite count and sum of q (out: [nbunch][8] doubles);
// job0[b] .. job0[b+1] are the jobs of bunch b; keys [njobs][7], qsum [njobs] scratch.
int launch_batch_stats(const BunchArgs *bunches, const BatchJob *jobs, int njobs, const int *job0, int nbunch,
                       unsigned long long *keys, double *qsum, double *out, cudaStream_t st);

// ---- adjoint of the step ---------------------------------------------------------------
// acc[c][n] += g[m][c] * (deposit weight of particle m at node n); acc is [3][N] doubles.
int launch_deposit_vec3(const DepositArgs &a, const double *g, double *acc, cudaStream_t st);
// Particle gradients of sum_m gE[m] . E(x_m): the gather term through the E planes [3][N]
// and the deposit term through the adjoint potential lam [N]; gq (nullable) = lam(x_m).
int launch_vjp_particles(const InterpArgs &ia, const DepositArgs &da, const double *E, const double *lam,
                         const double *gE, double *gx, double *gy, double *gz, double *gq, cudaStream_t st);

// FP32 adjoint: the three gradient components deposited into three quad grids (quad3 =
// [3][N] float4, the layout of launch_deposit_quad; weights times g[m][c] instead of q).
int launch_deposit_quad3(const DepositArgs &a, const double *g, float *quad3, cudaStream_t st);
// Slot 3 of every x-pair node of e8 (the grid launch_interp_pairs reads) set to lam:
// node n holds lam(n) and lam(n+1) (0 past the row end).
int launch_pack_lambda(float *e8, const double *lam, int nx, int64_t n, cudaStream_t st);
// launch_vjp_particles with E and lam read from one x-pair grid (Ex, Ey, Ez, lam per node).
int launch_vjp_pairs(const InterpArgs &ia, const DepositArgs &da, const float *e8, const double *gE, double *gx,
                     double *gy, double *gz, double *gq, cudaStream_t st);

// E planes [3][N] (f64) to the x-pair grid read by launch_interp_pairs (e8 32-byte aligned).
int launch_planes_to_pairs(const double *E, float *e8, int nx, int64_t n, cudaStream_t st);

}  // namespace osc
