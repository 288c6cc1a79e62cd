// grid_kernels.cuh -- Green-function construction and grid elementwise kernels.
#pragma once

#include "fft_kernels.cuh"

namespace osc {

// Corner primitives F(ca,cb,cc) of osc_get_cgrn_freespace on the half-cell-offset grid
// u = ca*dx + umin (code/open_spacecharge_mod.f90:659-692), for ca in [c0.x, c0.x+cd.x) etc.
struct CornerArgs {
    int cdx, cdy, cdz;     // extents of the evaluated corner block
    int c0x, c0y, c0z;     // first corner index
    double dx, dy, dz;     // dz already multiplied by gamma
    double umin, vmin, wmin;
    double factor;
    int icomp;
};
int launch_igf_corners(double *F, const CornerArgs &a, cudaStream_t st);
// Corner blocks of up to four components of one geometry in one launch (arguments by
// value): component i writes F + i * fstride, a[i] cdx*cdy*cdz points each.
struct CornerSet {
    CornerArgs a[4];
    int n;
};
int launch_igf_corners_set(double *F, const CornerSet &s, int64_t fstride, cudaStream_t st);

// Reference layout: cgrn(i,j,k) = 8-corner difference for i<N-1.., raw corner value on the
// last faces, as complex128 over the full (Nx,Ny,Nz) grid (code/open_spacecharge_mod.f90:697-705).
int launch_igf_diff_ref(const double *F, double2 *cg, int Nx, int Ny, int Nz, cudaStream_t st);

// Centred kernel on the doubled grid for the optimised path: g at displacement a in
// [-(n-1), n-1] stored at index a mod N, zero at index n; axes with sym mirror a<0 from
// a>0 with the given parity.  F holds corners [c0, c0+cd) per axis.
struct CenterArgs {
    int nx, ny, nz;
    int symx, symy, symz;
    int parx, pary, parz;
    int c0x, c0y, c0z, cdx, cdy;
};
int launch_green_center(const double *F, double2 *cg, const CenterArgs &a, cudaStream_t st);

// All-symmetric geometries: the non-negative octant h[c][b][a] (a < nx, b < ny, c < nz) of
// the centred kernel from corners F of extent (n+1) per axis starting at index n-1.
// nbatch members: corner blocks (n+1)^3 apart in F, octants n^3 apart in h.
// h = the 8-corner differences of F (FP64), rounded once to TH.
template <typename TH>
int launch_green_octant(const double *F, TH *h, int nx, int ny, int nz, int nbatch, cudaStream_t st);
// Corner blocks of nbatch geometries (args_dev: device array), fstride apart, npts each.
int launch_igf_corners_batch(double *F, const CornerArgs *args_dev, int nbatch, int64_t fstride, int64_t npts,
                             cudaStream_t st);

// Stored half-spectrum extraction: kx in [0,nx], ky in [0,dimy), kz in [0,dimz), times scale;
// layout [kz][ky][kx], or [ky][kx][kz] with columns zpitch elements apart when zpitch > 0
// (padding zeroed).  fold_mul >= 0 multiplies the value at kz by -exp(2 pi i fold_mul kz / Nz)
// (the image z-flip phase); -1 leaves it.
template <typename T>
int launch_green_extract(const double2 *ghat, void *out, int nx, int Nx, int Ny, int dimy, int dimz,
                         int real_valued, int imag_unit, double scale, int zpitch, int fold_mul, int Nz,
                         cudaStream_t st);
// Column pitch (elements) of the kz-innermost layout: dimz rounded up to 16 bytes.
inline int green_zpitch(int dimz, size_t elem_bytes) {
    const int q = (int)(16 / elem_bytes) > 0 ? (int)(16 / elem_bytes) : 1;
    return (dimz + q - 1) / q * q;
}

// ---- plain (reference-algorithm) path helpers ---------------------------------------
// crho = 0 everywhere, rho (sign * flipped-in-z if flipz) in the low octant.
int launch_pad_rho(const double *rho, double2 *crho, int nx, int ny, int nz, int Nx, int Ny, int Nz,
                   double sign, int flipz, cudaStream_t st);
int launch_cmul(double2 *a, const double2 *b, int64_t M, cudaStream_t st);
// out[c-plane] = factr * Re(c(i+si, j+sj, k+sk)); accumulate=1 adds into out.
int launch_extract_re(const double2 *c, int Nx, int Ny, int si, int sj, int sk, int nx, int ny, int nz,
                      double factr, double *out, int accumulate, cudaStream_t st);

// ---- field epilogues --------------------------------------------------------------
// B = coef*(-Ey, Ex, 0) (+= when accumulate) over N nodes, planes [3][N].
int launch_bfield(const double *E, double *B, int64_t N, double coef, int accumulate, cudaStream_t st);
int launch_axpy(double *y, const double *x, double a, int64_t n, cudaStream_t st);
int launch_scale(double *y, double a, int64_t n, cudaStream_t st);
// Centred differences with first-order one-sided edges (core:87-104).
int launch_fd_efield(const double *phi, double *E, int nx, int ny, int nz, double dx, double dy,
                     double dz, double gam0, cudaStream_t st);
// As launch_fd_efield, written as the x-pair grid (float4 [N][2]) of launch_interp_pairs.
int launch_fd_efield_pairs(const double *phi, float *e8, int nx, int ny, int nz, double dx, double dy, double dz,
                           double gam0, cudaStream_t st);
// In-place flip of a [nz][ny][nx] grid along z.
int launch_flip_z(double *a, int nx, int ny, int nz, cudaStream_t st);
// vec4<T> interleaved grid -> three double planes [3][N] (and optional B from E).
template <typename T>
int launch_vec4_to_planes(const void *E4, double *E, int64_t N, cudaStream_t st);
int launch_f32_to_f64(const float *a, double *b, int64_t n, cudaStream_t st);
int launch_f64_to_f32(const double *a, float *b, int64_t n, cudaStream_t st);

// ---- legacy point-evaluated Green functions (core:454-497, :1135-1230) ---------------
struct LegacyGrnArgs {
    int px, py, pz;            // period (array extent) per axis
    int glox, gloy, gloz;      // Fortran lower bounds of the array
    int shx, shy, shz;         // ishift etc.
    int wrapx, wrapy, wrapz;   // 1: index = glo + mod(i-glo+shift, period); 0: see below
    double dx, dy, dz, gam;
    double w_off;              // added to w (zshft) when wrapz; for wrapz=0, w = k*dz + w_off
    int icomp, igfflag;
};
int launch_legacy_green(double2 *cg, const LegacyGrnArgs &a, cudaStream_t st);

// Rectangular-pipe Green array t (osc_getgrnpipe, core:632-715) via separable tables.
struct PipeGrnArgs {
    int px, py, pz;
    int glox, gloy, gloz;
    int shx, shy, shz;
    int wrapx, wrapy;
    double hx, hy, hz, xmin, ymin, gam, a, b;
    int isg, jsg;
};
int pipe_green_scratch_doubles(const PipeGrnArgs &a);
int launch_pipe_green(double2 *cg, double *scratch, const PipeGrnArgs &a, cudaStream_t st);

}  // namespace osc
