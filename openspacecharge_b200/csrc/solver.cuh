// solver.cuh -- field-solve pipelines on one context.
#pragma once

#include "../../include/opensc_gpu.h"
#include "context.cuh"
#include "grid_kernels.cuh"
#include "particle_kernels.cuh"

namespace osc {

// 1/(4 pi eps0) of osc_freespace_solver2: `299792458.0**2*1.00000000055d-7` squares a
// single-precision literal (code/open_spacecharge_mod.f90:547).
inline double fpei_solver2() {
    const float c = 299792458.0f;
    return (double)(c * c) * 1.00000000055e-7;
}
// c_light of space_charge_3d, also a single-precision literal (code/open_spacecharge_mod.f90:436).
inline double c_light_sc3d() { return (double)299792458.0f; }
// Legacy core module constants (code/open_spacecharge_core_mod.f90:51, :515).
inline double fpei_legacy() { return 299792458.0 * 299792458.0 * 1.0e-7; }
const double CLIGHT_CORE = 299792458.0;
// fftconvcorr3d's single-precision `299792458.**2*1.e-7` (core:783).
inline double fpei_pipe() {
    const float c = 299792458.0f;
    float v = c * c;
    v = v * 1.0e-7f;
    return (double)v;
}

struct FreeSpaceJob {
    int nx = 0, ny = 0, nz = 0;
    double delta[3] = {0, 0, 0}, gamma = 1, offset[3] = {0, 0, 0};
    int at_cathode = 0;
    double img_zoff = 0;  // 2*min(3) + (max(3)-min(3))
    int want_phi = 0, want_e = 1;
    int calc_b = 0;
    double bcoef = 0;     // beta/c_light
    double *phi = nullptr;  // device f64 [N]
    double *E = nullptr;    // device f64 [3][N]
    double *B = nullptr;    // device f64 [3][N]
    void *E4 = nullptr;     // device vec4<T> [N], or the x-pair grid vec4<T> [N][2]
    int e4_pairs = 0;       // 1: E4 is the x-pair grid read by launch_interp_pairs
    // FP32 only: the deposit's quad grid (float4 [N]); when set, the x transform sums each
    // node from it and the rho argument is not read
    const float4 *quad = nullptr;
    // FP32, warp-engine z lengths only: sum3 = 1 makes the three quad grids stacked in quad
    // ([3][N]) the inputs of one output, sum_c K_c a_c (K_c the E_c kernel), written times
    // acc_coef into slot 3 of the x-pair grid E4 (the adjoint potential of the step)
    int sum3 = 0;
    // E components computed (bit c: E_c); each one is also added, times acc_coef, into
    // the single plane Eacc when that is set (adjoint solves accumulate a potential)
    int comp_mask = 7;
    double *Eacc = nullptr;
    double acc_coef = 0;
    // batch of nbatch equal grids stacked in rho and E4 (E4 output only); the spectra come
    // from gbatch (member b at data + b*g_bstride elements) instead of the Green cache
    int nbatch = 1;
    const GSpecDev *gbatch = nullptr;
    int ngbatch = 0;
    int64_t g_bstride = 0;
};

// Corner block arguments of the IGF primitive of component icomp (0 phi, 1..3 E).
CornerArgs green_corner_args(const int n[3], const double delta[3], double gamma, const double off[3], int icomp);
// Stored spectra of all-symmetric kernels of nb members with equal grids from their corner
// blocks F ((n+1)^3 each, corner index n-1 first): member b written at out + b*out_bstride.
// Along axis d the members in [odd[d][0], odd[d][1]) are odd, the others even.
template <typename T>
int green_sym_lines3(osc_ctx *c, const double *F, int nb, int nx, int ny, int nz, const int odd[3][2], int zinner,
                     int zpitch, T *out, int64_t out_bstride);

// Optimised IGF convolution (cached half-spectra, pruned transforms) in precision T.
template <typename T, typename TIn>
int freespace_opt(osc_ctx *c, const FreeSpaceJob &job, const TIn *rho);
// The reference algorithm in FP64 (full zero-padded complex FFTs, G rebuilt per call).
int freespace_plain(osc_ctx *c, const FreeSpaceJob &job, const double *rho);

// ---- one grid over z slabs (FP32) ----------------------------------------------------
// A rank holding the planes [z0, z0 + nzl) of the nx x ny x nz grid and the half-spectrum
// columns [col0, col0 + ncols) (column ky*(nx+1) + kx) runs the free-space solve in three
// stages around two transposes that the caller makes:
// forward x and y transforms of its planes: quad grid of nzl planes (float4 per node, as
// the deposit leaves it) -> spectrum planes X2 [nzl][2ny][nx+1];
int slab_forward(osc_ctx *c, int nx, int ny, int nzl, const float4 *quad, cplx<float> *X2);
// the z pass of its columns: in [nz][ncols] -> out [3][ncols][nz] (E components, window
// z < nz), with the cached Green spectra of the whole grid (geometry of j);
int slab_zpass(osc_ctx *c, const FreeSpaceJob &j, int col0, int ncols, const cplx<float> *in, cplx<float> *out);
// inverse y and x transforms of its planes: X3 [3][2ny][nx+1][nzl] (kz innermost) -> the
// x-pair E grid of its planes (float4 [nzl*ny*nx][2], as launch_interp_pairs reads it).
int slab_inverse(osc_ctx *c, int nx, int ny, int nzl, const cplx<float> *X3, float4 *e8);

// Full in-place C2C transform of an (Nx,Ny,Nz) array with per-axis signs.
template <typename T>
int fft3d_full(osc_ctx *c, cplx<T> *a, int Nx, int Ny, int Nz, int sx, int sy, int sz);

// Legacy solvers (FP64, reference algorithms).
int legacy_freespace(osc_ctx *c, const int nlo[3], const int nhi[3], const int npad[3],
                     const double delta[3], double gam0, const double *rho, int direct, int igf,
                     double *phi, double *E, double *B);
int legacy_cathode(osc_ctx *c, const int nlo[3], const int nhi[3], const int npad[3],
                   const double umin[3], const double delta[3], double gam0, double *rho,
                   int direct, int igf, int imethod, double *phi, double *E, double *B);
int pipe_green_build(osc_ctx *c, const int nlo[3], const int nhi[3], const int npad[3],
                     const double delta[3], const double umin[3], double gam, double a, double b);
// Pipe potential phi from rho (or, FP32 with npad 1, from the deposit's quad grid), then
// E = -grad phi as FP64 planes E and/or the FP32 x-pair grid e8 (E null: e8 only, written
// straight from phi), and B from the planes when B is given.
int pipe_solve(osc_ctx *c, int precision, const double delta[3], double gam0, const double *rho,
               double *phi, double *E, double *B, const float4 *quad = nullptr, float *e8 = nullptr);
// pipe_solve after checking that the pipe Green set was built for this mesh.
int pipe_solve_checked(osc_ctx *ctx, const osc_mesh3d *mesh, int precision, const double *rho, double *phi,
                       double *E, double *B, const float4 *quad, float *e8);

}  // namespace osc
