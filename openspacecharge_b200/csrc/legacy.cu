// legacy.cu -- the reference's older solvers on the GPU: the legacy free-space solver, the
// cathode-image methods 1 (convolution/correlation) and 2 (shifted Green function), and the
// rectangular conducting pipe (code/open_spacecharge_core_mod.f90).
//
// The legacy solvers and the pipe's reference path restate the Fortran in FP64 with the
// same padded period 2(nhi-nlo)+1+npad, point-evaluated Green functions, full complex
// transforms with the reference's per-axis signs and low-corner extraction.  The pipe also
// has an optimised path (FP32 or FP64 half-spectrum convolution, FP64 mode sums): the four
// convolution/correlation terms of fftconvcorr3d become four outputs of the z-pass kernel,
// with each correlation sign turned into an index flip of that output along x or y, and
// the terms summed in the x epilogue.
#include <cstdio>
#include <cstring>
#include <vector>

#include <type_traits>

#include "../../include/opensc_gpu.h"
#include "solver.cuh"

namespace osc {

#define TRY(...)                  \
    do {                          \
        int rc_ = (__VA_ARGS__);  \
        if (rc_) return rc_;      \
    } while (0)

static int kchk(osc_ctx *c, int rc, const char *what) {
    if (rc == OSC_OK) return OSC_OK;
    cudaError_t e = cudaGetLastError();
    return set_err(c, rc == OSC_E_FFT_SIZE ? rc : OSC_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

namespace {

struct LGeom {
    int n[3], period[3], glo[3], shift[3];
    int64_t N, M;
};

// osc_alloc_freespace_array (core:151-182): bounds nlo-nhi .. nhi-nlo+npad.
int lgeom(osc_ctx *c, const int nlo[3], const int nhi[3], const int npad[3], LGeom &g) {
    g.N = 1;
    g.M = 1;
    for (int d = 0; d < 3; ++d) {
        g.n[d] = nhi[d] - nlo[d] + 1;
        if (g.n[d] < 2) return set_err(c, OSC_E_INVALID, "mesh axis %d has fewer than 2 nodes", d);
        if (npad[d] < 0) return set_err(c, OSC_E_INVALID, "npad must be >= 0");
        g.glo[d] = nlo[d] - nhi[d];
        g.period[d] = 2 * (nhi[d] - nlo[d]) + 1 + npad[d];
        g.shift[d] = g.period[d] / 2 - (npad[d] + 1) / 2;
        FFTPlan p;
        if (!make_fft_plan(g.period[d], p))
            return set_err(c, OSC_E_FFT_SIZE,
                           "transform length %d: Error return from FFT package due to transform length. "
                           "Try increasing the padding by 1 in each dimension and re-run",
                           g.period[d]);
        g.N *= g.n[d];
        g.M *= g.period[d];
    }
    return OSC_OK;
}

// getrhotilde (core:435-449): crho = 0, rho in the low corner, FFT (1,1,1).
int rhotilde(osc_ctx *c, const LGeom &g, const double *rho, double2 *crho) {
    {
        Launch L_(c, "plain_pad");
        TRY(kchk(c, launch_pad_rho(rho, crho, g.n[0], g.n[1], g.n[2], g.period[0], g.period[1], g.period[2], 1.0, 0,
                                   c->stream),
                 "pad rho"));
    }
    return fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(crho), g.period[0], g.period[1], g.period[2], 1, 1, 1);
}

LegacyGrnArgs grn_args(const LGeom &g, const double delta[3], double gam, int icomp, int igfflag) {
    LegacyGrnArgs a;
    a.px = g.period[0]; a.py = g.period[1]; a.pz = g.period[2];
    a.glox = g.glo[0]; a.gloy = g.glo[1]; a.gloz = g.glo[2];
    a.shx = g.shift[0]; a.shy = g.shift[1]; a.shz = g.shift[2];
    a.wrapx = a.wrapy = a.wrapz = 1;
    a.dx = delta[0]; a.dy = delta[1]; a.dz = delta[2];
    a.gam = gam;
    a.w_off = 0.0;
    a.icomp = icomp;
    a.igfflag = igfflag;
    return a;
}

// Green values then FFT with the given signs.
int grn_transform(osc_ctx *c, const LGeom &g, const LegacyGrnArgs &a, double2 *cg, const int sg[3]) {
    {
        Launch L_(c, "legacy_green");
        TRY(kchk(c, launch_legacy_green(cg, a, c->stream), "legacy green"));
    }
    return fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(cg), g.period[0], g.period[1], g.period[2], sg[0],
                              sg[1], sg[2]);
}

// conv3d / imageconvcorr3d (core:503-529, :1237-1264): cg = crho*cg, inverse FFT with
// signs isg, out = coef * Re(low-corner window).
int conv_extract(osc_ctx *c, const LGeom &g, const double2 *crho, double2 *cg, const int isg[3], double coef,
                 double *out, int accumulate) {
    {
        Launch L_(c, "plain_cmul");
        TRY(kchk(c, launch_cmul(cg, crho, g.M, c->stream), "cmul"));
    }
    TRY(fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(cg), g.period[0], g.period[1], g.period[2], isg[0],
                           isg[1], isg[2]));
    Launch L_(c, "plain_extract");
    return kchk(c, launch_extract_re(cg, g.period[0], g.period[1], 0, 0, 0, g.n[0], g.n[1], g.n[2], coef, out,
                                     accumulate, c->stream),
                "extract");
}

double legacy_factr(const LGeom &g) {
    return 1.0 / ((1.0 * g.period[0]) * (1.0 * g.period[1]) * (1.0 * g.period[2])) * fpei_legacy() * 1.0;
}

}  // namespace

// osc_freespace_solver (core:30-138) on device arrays.
int legacy_freespace(osc_ctx *c, const int nlo[3], const int nhi[3], const int npad[3], const double delta[3],
                     double gam0, const double *rho, int direct, int igf, double *phi, double *E, double *B) {
    if (!igf && direct)
        return set_err(c, OSC_E_UNSUPPORTED, "Error: Direct field calc must use integrated Green function");
    LGeom g;
    TRY(lgeom(c, nlo, nhi, npad, g));
    double2 *crho, *cg;
    TRY(ws_get(c, "plain_crho", sizeof(double2) * g.M, (void **)&crho));
    TRY(ws_get(c, "plain_cgrn", sizeof(double2) * g.M, (void **)&cg));
    const int fwd[3] = {1, 1, 1}, inv[3] = {-1, -1, -1};
    const double factr = legacy_factr(g);
    TRY(rhotilde(c, g, rho, crho));
    if (!direct) {
        TRY(grn_transform(c, g, grn_args(g, delta, gam0, 0, igf), cg, fwd));
        TRY(conv_extract(c, g, crho, cg, inv, factr, phi, 0));
        Launch L_(c, "fd_efield");
        TRY(kchk(c, launch_fd_efield(phi, E, g.n[0], g.n[1], g.n[2], delta[0], delta[1], delta[2], gam0, c->stream),
                 "fd"));
    } else {
        for (int icomp = 1; icomp <= 3; ++icomp) {
            TRY(grn_transform(c, g, grn_args(g, delta, gam0, icomp, igf), cg, fwd));
            TRY(conv_extract(c, g, crho, cg, inv, factr, E + (icomp - 1) * g.N, 0));
        }
    }
    const double beta0 = std::sqrt(1 - 1 / (gam0 * gam0));
    Launch L_(c, "plain_bfield");
    return kchk(c, launch_bfield(E, B, g.N, beta0 / CLIGHT_CORE, 0, c->stream), "bfield");
}

// osc_cathodeimages_solver (core:905-1083) on device arrays; rho is flipped in place by
// method 2, as in the reference.
int legacy_cathode(osc_ctx *c, const int nlo[3], const int nhi[3], const int npad[3], const double umin[3],
                   const double delta[3], double gam0, double *rho, int direct, int igf, int imethod, double *phi,
                   double *E, double *B) {
    if (!igf && direct)
        return set_err(c, OSC_E_UNSUPPORTED, "Error: Direct field calc must use integrated Green function");
    LGeom g;
    TRY(lgeom(c, nlo, nhi, npad, g));
    double2 *crho, *cg;
    double *img, *phimg;
    TRY(ws_get(c, "plain_crho", sizeof(double2) * g.M, (void **)&crho));
    TRY(ws_get(c, "plain_cgrn", sizeof(double2) * g.M, (void **)&cg));
    TRY(ws_get(c, "legacy_img", sizeof(double) * 3 * g.N, (void **)&img));
    TRY(ws_get(c, "legacy_phimg", sizeof(double) * g.N, (void **)&phimg));
    const int fwd[3] = {1, 1, 1}, inv[3] = {-1, -1, -1};
    const int fwd_corr[3] = {1, 1, -1}, inv_corr[3] = {-1, -1, 1};
    const double factr = legacy_factr(g);
    // osc_getgrnimageconvcorr (core:1185-1230): z runs over the array index k of bounds
    // 2*nlo(3).. with w = k*dz + 2*umin(3) - 2*nlo(3)*delta(3)
    auto corr_args = [&](int icomp) {
        LegacyGrnArgs a = grn_args(g, delta, gam0, icomp, igf);
        a.wrapz = 0;
        a.gloz = 2 * nlo[2];
        a.w_off = 2.0 * umin[2] - 2.0 * nlo[2] * delta[2];
        return a;
    };
    // osc_getgrnimageshift (core:1135-1178): w = kp*dz + zshft
    const double umax3 = umin[2] + (nhi[2] - nlo[2]) * delta[2];
    const double zshft = umin[2] + umax3;
    auto shift_args = [&](int icomp) {
        LegacyGrnArgs a = grn_args(g, delta, gam0, icomp, igf);
        a.w_off = zshft;
        return a;
    };
    auto flip = [&]() -> int {
        Launch L_(c, "flip_z");
        return kchk(c, launch_flip_z(rho, g.n[0], g.n[1], g.n[2], c->stream), "flip");
    };
    TRY(rhotilde(c, g, rho, crho));
    if (!direct) {
        TRY(grn_transform(c, g, grn_args(g, delta, gam0, 0, igf), cg, fwd));
        TRY(conv_extract(c, g, crho, cg, inv, factr, phi, 0));
        if (imethod == 1) {
            TRY(grn_transform(c, g, corr_args(0), cg, fwd_corr));
            TRY(conv_extract(c, g, crho, cg, inv_corr, factr, phimg, 0));
        } else {
            TRY(flip());
            TRY(rhotilde(c, g, rho, crho));
            TRY(grn_transform(c, g, shift_args(0), cg, fwd));
            TRY(conv_extract(c, g, crho, cg, inv, factr, phimg, 0));
        }
        {
            Launch L_(c, "plain_axpy");
            TRY(kchk(c, launch_axpy(phi, phimg, -1.0, g.N, c->stream), "axpy"));
        }
        Launch L_(c, "fd_efield", 2);
        TRY(kchk(c, launch_fd_efield(phi, E, g.n[0], g.n[1], g.n[2], delta[0], delta[1], delta[2], gam0, c->stream),
                 "fd"));
        TRY(kchk(c, launch_fd_efield(phimg, img, g.n[0], g.n[1], g.n[2], delta[0], delta[1], delta[2], gam0,
                                     c->stream),
                 "fd image"));
    } else {
        for (int icomp = 1; icomp <= 3; ++icomp) {
            TRY(grn_transform(c, g, grn_args(g, delta, gam0, icomp, igf), cg, fwd));
            TRY(conv_extract(c, g, crho, cg, inv, factr, E + (icomp - 1) * g.N, 0));
        }
        if (imethod != 1) {
            TRY(flip());
            TRY(rhotilde(c, g, rho, crho));
        }
        for (int icomp = 1; icomp <= 3; ++icomp) {
            if (imethod == 1) {
                TRY(grn_transform(c, g, corr_args(icomp), cg, fwd_corr));
                TRY(conv_extract(c, g, crho, cg, inv_corr, factr, img + (icomp - 1) * g.N, 0));
            } else {
                TRY(grn_transform(c, g, shift_args(icomp), cg, fwd));
                TRY(conv_extract(c, g, crho, cg, inv, factr, img + (icomp - 1) * g.N, 0));
            }
            Launch L_(c, "plain_axpy");
            TRY(kchk(c, launch_axpy(E + (icomp - 1) * g.N, img + (icomp - 1) * g.N, -1.0, g.N, c->stream), "axpy"));
        }
    }
    // B from the direct plus image fields: E was reduced by img, add it back twice (core:1076-1077)
    const double coef = std::sqrt(1 - 1 / (gam0 * gam0)) / CLIGHT_CORE;
    Launch L_(c, "plain_bfield", 2);
    TRY(kchk(c, launch_bfield(E, B, g.N, coef, 0, c->stream), "bfield"));
    return kchk(c, launch_bfield(img, B, g.N, 2.0 * coef, 1, c->stream), "bfield image");
}

// ---------------------------------------------------------------------------------------
// Rectangular pipe.  The four transformed Green arrays (the reference's module-global
// cgrn1..4) live on the context.
static const int PIPE_FWD[4][3] = {{1, 1, 1}, {1, -1, 1}, {-1, 1, 1}, {-1, -1, 1}};
static const int PIPE_INV[4][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, -1, -1}, {1, 1, -1}};
static const double PIPE_SIGN[4] = {1.0, -1.0, -1.0, 1.0};

static int pipe_alloc(osc_ctx *c, const LGeom &g) {
    PipeGreen &p = c->pipe;
    for (int t = 0; t < 4; ++t) {
        if (p.g[t].p && p.g[t].bytes >= sizeof(double2) * (size_t)g.M) continue;
        if (p.g[t].p) {
            cudaStreamSynchronize(c->stream);
            cudaFree(p.g[t].p);
        }
        p.g[t].p = nullptr;
        p.g[t].bytes = 0;
        if (cudaMalloc(&p.g[t].p, sizeof(double2) * (size_t)g.M) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, OSC_E_ALLOC, "pipe Green array: cudaMalloc failed");
        }
        p.g[t].bytes = sizeof(double2) * (size_t)g.M;
    }
    p.comb_prec = -1;  // optimised copies are rebuilt from the new arrays on demand
    return OSC_OK;
}

int pipe_green_build(osc_ctx *c, const int nlo[3], const int nhi[3], const int npad[3], const double delta[3],
                     const double umin[3], double gam, double a, double b) {
    LGeom g;
    TRY(lgeom(c, nlo, nhi, npad, g));
    if (!(a > 0 && b > 0)) return set_err(c, OSC_E_INVALID, "pipe aperture must be positive");
    TRY(pipe_alloc(c, g));
    PipeGreen &p = c->pipe;
    double *scratch;
    PipeGrnArgs pa;
    pa.px = g.period[0]; pa.py = g.period[1]; pa.pz = g.period[2];
    pa.glox = g.glo[0]; pa.gloy = g.glo[1]; pa.gloz = g.glo[2];
    pa.shx = g.shift[0]; pa.shy = g.shift[1]; pa.shz = g.shift[2];
    pa.hx = delta[0]; pa.hy = delta[1]; pa.hz = delta[2];
    pa.xmin = umin[0]; pa.ymin = umin[1];
    pa.gam = gam; pa.a = a; pa.b = b;
    TRY(ws_get(c, "pipe_tables", sizeof(double) * pipe_green_scratch_doubles(pa), (void **)&scratch));
    // osc_getgrnpipe (core:632-715): arrays 2 and 4 take v = 2*ymin + j*hy, arrays 3 and 4
    // take u = 2*xmin + i*hx; rfun signs (i,j) = (1,1), (1,-1), (-1,1), (-1,-1)
    const int ij[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    for (int t = 0; t < 4; ++t) {
        pa.wrapx = (t == 0 || t == 1);
        pa.wrapy = (t == 0 || t == 2);
        pa.isg = ij[t][0];
        pa.jsg = ij[t][1];
        double2 *gt = reinterpret_cast<double2 *>(p.g[t].p);
        {
            Launch L_(c, "pipe_green", 2);
            TRY(kchk(c, launch_pipe_green(gt, scratch, pa, c->stream), "pipe green"));
        }
        TRY(fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(gt), g.period[0], g.period[1], g.period[2],
                               PIPE_FWD[t][0], PIPE_FWD[t][1], PIPE_FWD[t][2]));
    }
    for (int d = 0; d < 3; ++d) {
        p.nlo[d] = nlo[d];
        p.nhi[d] = nhi[d];
        p.npad[d] = npad[d];
        p.period[d] = g.period[d];
        p.delta[d] = delta[d];
        p.umin[d] = umin[d];
        p.umax[d] = umin[d] + (nhi[d] - nlo[d]) * delta[d];
    }
    p.apipe = a;
    p.bpipe = b;
    p.gamma = gam;
    p.valid = true;
    return OSC_OK;
}

// Half-spectrum copies of the four arrays, scaled by the term sign and fpei/M, for the
// optimised pipeline (FP32 or FP64 storage).
template <typename T> static int pipe_comb(osc_ctx *c, const LGeom &g) {
    PipeGreen &p = c->pipe;
    const int prec = sizeof(T) == 4 ? 0 : 1;
    if (p.comb_prec == prec) return OSC_OK;
    const int nx = g.n[0];
    const size_t each = (size_t)(nx + 1) * g.period[1] * g.period[2] * sizeof(cplx<T>);
    if (p.comb.bytes < 4 * each) {
        if (p.comb.p) {
            cudaStreamSynchronize(c->stream);
            cudaFree(p.comb.p);
        }
        p.comb.p = nullptr;
        p.comb.bytes = 0;
        if (cudaMalloc(&p.comb.p, 4 * each) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, OSC_E_ALLOC, "pipe spectra: cudaMalloc failed");
        }
        p.comb.bytes = 4 * each;
    }
    const double factr = 1.0 / ((1.0 * g.period[0]) * (1.0 * g.period[1]) * (1.0 * g.period[2])) * fpei_pipe() * 1.0;
    for (int t = 0; t < 4; ++t) {
        Launch L_(c, "green_extract");
        TRY(kchk(c, launch_green_extract<T>(reinterpret_cast<const double2 *>(p.g[t].p),
                                            reinterpret_cast<char *>(p.comb.p) + t * each, nx, g.period[0],
                                            g.period[1], g.period[1], g.period[2], 0, 0, PIPE_SIGN[t] * factr,
                                            zconv_warp_ok(g.period[2], g.n[2], (int)sizeof(T))
                                                ? green_zpitch(g.period[2], sizeof(cplx<T>))
                                                : 0,
                                            -1, 0, c->stream),
                 "pipe extract"));
    }
    p.comb_prec = prec;
    return OSC_OK;
}

// Optimised pipe potential: phi = sum_t sign_t * fpei/M * IFFT_{inv_t}(rho_hat * G_t).
template <typename T>
static int pipe_phi_opt(osc_ctx *c, const LGeom &g, const double *rho, double *phi, const float4 *quad = nullptr) {
    typedef cplx<T> V;
    TRY(pipe_comb<T>(c, g));
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int Nx = g.period[0], Ny = g.period[1], Nz = g.period[2], nxh = nx + 1;
    FFTPlan px, py, pz;
    make_fft_plan(Nx, px);
    make_fft_plan(Ny, py);
    make_fft_plan(Nz, pz);
    const int nout = 4;
    V *X1, *X2, *X3, *X4;
    TRY(ws_get(c, "fs_x1", sizeof(V) * (size_t)nxh * ny * nz, (void **)&X1));
    TRY(ws_get(c, "fs_x2", sizeof(V) * (size_t)nxh * Ny * nz, (void **)&X2));
    TRY(ws_get(c, "fs_x3", sizeof(V) * (size_t)nout * nxh * Ny * nz, (void **)&X3));
    TRY(ws_get(c, "fs_x4", sizeof(V) * (size_t)nout * nxh * ny * nz, (void **)&X4));
    TwPair<V> twx, twy, twz;
    TRY(twiddles<T>(c, Nx, &twx));
    TRY(twiddles<T>(c, Ny, &twy));
    TRY(twiddles<T>(c, Nz, &twz));
    R2CArgs ra;
    ra.p = px;
    ra.nin = nx;
    ra.nrows = (int64_t)ny * nz;
    ra.in_rstride = nx;
    ra.out_rstride = nxh;
    {
        Launch L_(c, "fft_x_r2c");
        if constexpr (std::is_same<T, float>::value) {
            if (quad) {  // the deposit's quad grid, summed to nodes as it is loaded
                ra.qny = ny;
                TRY(kchk(c, launch_r2c_rows<float, float4>(quad, X1, ra, twx, c->stream), "x r2c"));
            } else {
                TRY(kchk(c, launch_r2c_rows<T, double>(rho, X1, ra, twx, c->stream), "x r2c"));
            }
        } else {
            TRY(kchk(c, launch_r2c_rows<T, double>(rho, X1, ra, twx, c->stream), "x r2c"));
        }
    }
    LineArgs ly;
    std::memset(&ly, 0, sizeof(ly));
    ly.p = py;
    ly.sign = +1;
    ly.ncols = nxh;
    ly.in_len = ny;
    ly.out_len = Ny;
    ly.in_pstride = (int64_t)nxh * ny;
    ly.in_cstride = 1;
    ly.in_estride = nxh;
    ly.out_pstride = (int64_t)nxh * Ny;
    ly.out_cstride = 1;
    ly.out_estride = nxh;
    ly.scale = 1.0;
    ly.flat_lines = 1;  // tiles over the (z, kx) line sequence, in both y passes
    {
        Launch L_(c, "fft_y_fwd");
        TRY(kchk(c, launch_lines<T>(X1, X2, ly, nz, 1, false, twy, c->stream), "y forward"));
    }
    ZConvArgs za;
    std::memset(&za, 0, sizeof(za));
    za.p = pz;
    za.nz = nz;
    za.ncols = nxh * Ny;
    za.nxh = nxh;
    za.Ny = Ny;
    za.ny = ny;
    za.in_estride = (int64_t)nxh * Ny;
    za.out_estride = (int64_t)nxh * Ny;
    za.out_colstride = 1;
    za.out_cstride = (int64_t)nxh * Ny * nz;
    za.nout = nout;
    za.ng = 4;
    za.fault = c->d_fault;
    if (c->test_wait_timeout) {  // test only: waits that must run out quickly
        za.poll_limit = 64;
        za.skip_copies = 1;
    }
    const size_t each = (size_t)nxh * Ny * Nz;
    for (int t = 0; t < 4; ++t) {
        za.gdir[t] = t;
        za.gimg[t] = -1;
        GSpecDev &s = za.g[t];
        s.data = reinterpret_cast<const V *>(c->pipe.comb.p) + t * each;
        s.real_valued = 0;
        s.imag_unit = 0;
        s.sym_y = s.sym_z = 0;
        s.par_y = s.par_z = 1;
        s.dimy = Ny;
        s.dimz = Nz;
        s.zinner = zconv_warp_ok(Nz, nz, (int)sizeof(T)) ? 1 : 0;
        s.zpitch = s.zinner ? green_zpitch(Nz, sizeof(V)) : Nz;
    }
    {
        Launch L_(c, "fft_z_conv");
        TRY(kchk(c, launch_zconv<T>(X2, X3, za, twz, 0, c->stream), "z conv"));
    }
    // inverse sign +1 along an axis = standard inverse read at the mirrored index
    LineArgs li = ly;
    li.sign = -1;
    li.in_len = Ny;
    li.out_len = ny;
    li.in_pstride = (int64_t)nxh * Ny;
    li.in_zstride = (int64_t)nxh * Ny * nz;
    li.out_pstride = (int64_t)nxh * ny;
    li.out_zstride = (int64_t)nxh * ny * nz;
    li.flip_mask = 0;
    for (int t = 0; t < 4; ++t)
        if (PIPE_INV[t][1] > 0) li.flip_mask |= 1u << t;
    {
        Launch L_(c, "fft_y_inv");
        TRY(kchk(c, launch_lines<T>(X3, X4, li, nz, nout, false, twy, c->stream), "y inverse"));
    }
    C2RArgs cr;
    std::memset(&cr, 0, sizeof(cr));
    cr.p = px;
    cr.nout = nx;
    cr.nrows = (int64_t)ny * nz;
    cr.in_rstride = nxh;
    cr.in_cstride = (int64_t)nxh * ny * nz;
    cr.ncomp = nout;
    for (int t = 0; t < 4; ++t) {
        if (PIPE_INV[t][0] > 0) cr.flip_mask |= 1u << t;
        cr.ndest[t] = 1;
        cr.dest[t][0].ptr = phi;
        cr.dest[t][0].kind = t == 0 ? 1 : 3;
        cr.dest[t][0].slot = 0;
        cr.dest[t][0].coef = 1.0;
    }
    Launch L_(c, "fft_x_c2r");
    return kchk(c, launch_c2r_rows<T>(X4, cr, twx, c->stream), "x c2r");
}

int pipe_solve(osc_ctx *c, int precision, const double delta[3], double gam0, const double *rho, double *phi,
               double *E, double *B, const float4 *quad, float *e8) {
    PipeGreen &p = c->pipe;
    LGeom g;
    TRY(lgeom(c, p.nlo, p.nhi, p.npad, g));
    const bool opt = precision != OSC_PREC_FP64_PLAIN && p.npad[0] == 1 && p.npad[1] == 1 && p.npad[2] == 1;
    if (quad && !(opt && precision == OSC_PREC_FP32))
        return set_err(c, OSC_E_INVALID, "pipe solve: quad-grid input needs the FP32 path and npad = 1");
    if (opt) {
        if (precision == OSC_PREC_FP32) TRY(pipe_phi_opt<float>(c, g, rho, phi, quad));
        else TRY(pipe_phi_opt<double>(c, g, rho, phi));
    } else {
        // fftconvcorr3d (core:763-818), term by term into phi
        double2 *crho, *ct;
        TRY(ws_get(c, "plain_crho", sizeof(double2) * g.M, (void **)&crho));
        TRY(ws_get(c, "plain_cgrn", sizeof(double2) * g.M, (void **)&ct));
        TRY(rhotilde(c, g, rho, crho));
        const double factr = 1.0 / ((1.0 * g.period[0]) * (1.0 * g.period[1]) * (1.0 * g.period[2])) * fpei_pipe() * 1.0;
        for (int t = 0; t < 4; ++t) {
            if (cudaMemcpyAsync(ct, p.g[t].p, sizeof(double2) * g.M, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
                return set_err(c, OSC_E_CUDA, "copy pipe Green array");
            TRY(conv_extract(c, g, crho, ct, PIPE_INV[t], PIPE_SIGN[t] * factr, phi, t > 0));
        }
    }
    if (e8 && !E && !B) {  // E only as the x-pair grid of the FP32 gather
        Launch L_(c, "fd_efield");
        return kchk(c, launch_fd_efield_pairs(phi, e8, g.n[0], g.n[1], g.n[2], delta[0], delta[1], delta[2], gam0,
                                              c->stream),
                    "fd pairs");
    }
    if (!E) return set_err(c, OSC_E_INVALID, "pipe solve: E planes needed");
    {
        Launch L_(c, "fd_efield");
        TRY(kchk(c, launch_fd_efield(phi, E, g.n[0], g.n[1], g.n[2], delta[0], delta[1], delta[2], gam0, c->stream),
                 "fd"));
    }
    if (e8) {
        Launch L_(c, "planes_to_pairs");
        TRY(kchk(c, launch_planes_to_pairs(E, e8, g.n[0], g.N, c->stream), "E pairs"));
    }
    if (!B) return OSC_OK;
    const double beta0 = std::sqrt(1 - 1 / (gam0 * gam0));
    Launch L_(c, "plain_bfield");
    return kchk(c, launch_bfield(E, B, g.N, beta0 / CLIGHT_CORE, 0, c->stream), "bfield");
}

// The checks of osc_space_charge_rectpipe_dev (Green set computed for this mesh), then the
// solve; the fused pipe step's entry to pipe_solve.
int pipe_solve_checked(osc_ctx *ctx, const osc_mesh3d *mesh, int precision, const double *rho, double *phi,
                       double *E, double *B, const float4 *quad, float *e8) {
    PipeGreen &p = ctx->pipe;
    bool same = p.valid;
    for (int d = 0; d < 3 && same; ++d)
        same = p.nlo[d] == mesh->nlo[d] && p.nhi[d] == mesh->nhi[d] && p.npad[d] == mesh->npad[d];
    if (!same)
        return set_err(ctx, OSC_E_STATE,
                       "something wrong. rectpipe green functions should have been computed during initialization "
                       "(call osc_rectpipe_green or osc_read_rectpipe_grn for this mesh first)");
    return pipe_solve(ctx, precision, mesh->delta, mesh->gamma, rho, phi, E, B, quad, e8);
}

}  // namespace osc

// ---------------------------------------------------------------------------------------
using namespace osc;

namespace {
int mesh_n(osc_ctx *c, const osc_mesh3d *m, int64_t *N) {
    if (!m) return set_err(c, OSC_E_INVALID, "mesh is NULL");
    *N = 1;
    for (int d = 0; d < 3; ++d) {
        const int n = m->nhi[d] - m->nlo[d] + 1;
        if (n < 2) return set_err(c, OSC_E_INVALID, "mesh axis %d has fewer than 2 nodes", d);
        *N *= n;
    }
    return OSC_OK;
}
int cp(osc_ctx *c, void *dst, const void *src, size_t bytes, cudaMemcpyKind k) {
    return cuda_check(c, cudaMemcpyAsync(dst, src, bytes, k, c->stream), "copy");
}
int syncc(osc_ctx *c) { return ctx_sync(c); }
}  // namespace

extern "C" {

int osc_space_charge_freespace(osc_ctx *ctx, const osc_mesh3d *mesh, const double *rho, int direct_field_calc,
                               int integrated_green_function, int precision, double *phi, double *efield,
                               double *bfield) {
    if (!ctx) return OSC_E_INVALID;
    (void)precision;  // the legacy solver runs the reference algorithm in FP64
    int64_t N;
    TRY(mesh_n(ctx, mesh, &N));
    if (!rho || !efield || !bfield || (!direct_field_calc && !phi))
        return set_err(ctx, OSC_E_INVALID, "space_charge_freespace arrays");
    double *d_rho, *d_phi, *d_E, *d_B;
    TRY(ws_get(ctx, "h_rho", sizeof(double) * N, (void **)&d_rho));
    TRY(ws_get(ctx, "h_phi", sizeof(double) * N, (void **)&d_phi));
    TRY(ws_get(ctx, "h_E", sizeof(double) * 3 * N, (void **)&d_E));
    TRY(ws_get(ctx, "h_B", sizeof(double) * 3 * N, (void **)&d_B));
    TRY(cp(ctx, d_rho, rho, sizeof(double) * N, cudaMemcpyHostToDevice));
    const int nlo[3] = {mesh->nlo[0], mesh->nlo[1], mesh->nlo[2]}, nhi[3] = {mesh->nhi[0], mesh->nhi[1], mesh->nhi[2]};
    const int npad[3] = {mesh->npad[0], mesh->npad[1], mesh->npad[2]};
    TRY(legacy_freespace(ctx, nlo, nhi, npad, mesh->delta, mesh->gamma, d_rho, direct_field_calc ? 1 : 0,
                         integrated_green_function ? 1 : 0, d_phi, d_E, d_B));
    if (!direct_field_calc) TRY(cp(ctx, phi, d_phi, sizeof(double) * N, cudaMemcpyDeviceToHost));
    TRY(cp(ctx, efield, d_E, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    TRY(cp(ctx, bfield, d_B, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    return syncc(ctx);
}

int osc_space_charge_cathodeimages(osc_ctx *ctx, const osc_mesh3d *mesh, double *rho, int direct_field_calc,
                                   int integrated_green_function, int image_method, int precision, double *phi,
                                   double *efield, double *bfield) {
    if (!ctx) return OSC_E_INVALID;
    (void)precision;
    int64_t N;
    TRY(mesh_n(ctx, mesh, &N));
    if (!rho || !efield || !bfield || (!direct_field_calc && !phi))
        return set_err(ctx, OSC_E_INVALID, "space_charge_cathodeimages arrays");
    const int imethod = image_method == 2 ? 2 : 1;  // code/open_spacecharge_mod.f90:97-98
    double *d_rho, *d_phi, *d_E, *d_B;
    TRY(ws_get(ctx, "h_rho", sizeof(double) * N, (void **)&d_rho));
    TRY(ws_get(ctx, "h_phi", sizeof(double) * N, (void **)&d_phi));
    TRY(ws_get(ctx, "h_E", sizeof(double) * 3 * N, (void **)&d_E));
    TRY(ws_get(ctx, "h_B", sizeof(double) * 3 * N, (void **)&d_B));
    TRY(cp(ctx, d_rho, rho, sizeof(double) * N, cudaMemcpyHostToDevice));
    const int nlo[3] = {mesh->nlo[0], mesh->nlo[1], mesh->nlo[2]}, nhi[3] = {mesh->nhi[0], mesh->nhi[1], mesh->nhi[2]};
    const int npad[3] = {mesh->npad[0], mesh->npad[1], mesh->npad[2]};
    TRY(legacy_cathode(ctx, nlo, nhi, npad, mesh->min, mesh->delta, mesh->gamma, d_rho, direct_field_calc ? 1 : 0,
                       integrated_green_function ? 1 : 0, imethod, d_phi, d_E, d_B));
    if (imethod == 2) TRY(cp(ctx, rho, d_rho, sizeof(double) * N, cudaMemcpyDeviceToHost));
    if (!direct_field_calc) TRY(cp(ctx, phi, d_phi, sizeof(double) * N, cudaMemcpyDeviceToHost));
    TRY(cp(ctx, efield, d_E, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    TRY(cp(ctx, bfield, d_B, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    return syncc(ctx);
}

int osc_rectpipe_green(osc_ctx *ctx, const osc_mesh3d *mesh, double apipe, double bpipe, int precision) {
    if (!ctx) return OSC_E_INVALID;
    int64_t N;
    TRY(mesh_n(ctx, mesh, &N));
    if (precision < 0 || precision > 2) return set_err(ctx, OSC_E_INVALID, "precision");
    const int nlo[3] = {mesh->nlo[0], mesh->nlo[1], mesh->nlo[2]}, nhi[3] = {mesh->nhi[0], mesh->nhi[1], mesh->nhi[2]};
    const int npad[3] = {mesh->npad[0], mesh->npad[1], mesh->npad[2]};
    TRY(pipe_green_build(ctx, nlo, nhi, npad, mesh->delta, mesh->min, mesh->gamma, apipe, bpipe));
    return syncc(ctx);
}

int osc_space_charge_rectpipe(osc_ctx *ctx, const osc_mesh3d *mesh, const double *rho, double apipe, double bpipe,
                              int direct_field_calc, int integrated_green_function, int precision, double *phi,
                              double *efield, double *bfield) {
    if (!ctx) return OSC_E_INVALID;
    (void)apipe;
    (void)bpipe;
    (void)integrated_green_function;
    int64_t N;
    TRY(mesh_n(ctx, mesh, &N));
    if (precision < 0 || precision > 2) return set_err(ctx, OSC_E_INVALID, "precision");
    if (!rho || !phi || !efield || !bfield) return set_err(ctx, OSC_E_INVALID, "space_charge_rectpipe arrays");
    if (direct_field_calc)
        return set_err(ctx, OSC_E_UNSUPPORTED,
                       "**********ERROR********* rectpipe implementation presently requires directfieldcalc=0");
    PipeGreen &p = ctx->pipe;
    bool same = p.valid;
    for (int d = 0; d < 3 && same; ++d)
        same = p.nlo[d] == mesh->nlo[d] && p.nhi[d] == mesh->nhi[d] && p.npad[d] == mesh->npad[d];
    if (!same)
        return set_err(ctx, OSC_E_STATE,
                       "something wrong. rectpipe green functions should have been computed during initialization "
                       "(call osc_rectpipe_green or osc_read_rectpipe_grn for this mesh first)");
    double *d_rho, *d_phi, *d_E, *d_B;
    TRY(ws_get(ctx, "h_rho", sizeof(double) * N, (void **)&d_rho));
    TRY(ws_get(ctx, "h_phi", sizeof(double) * N, (void **)&d_phi));
    TRY(ws_get(ctx, "h_E", sizeof(double) * 3 * N, (void **)&d_E));
    TRY(ws_get(ctx, "h_B", sizeof(double) * 3 * N, (void **)&d_B));
    TRY(cp(ctx, d_rho, rho, sizeof(double) * N, cudaMemcpyHostToDevice));
    TRY(pipe_solve(ctx, precision, mesh->delta, mesh->gamma, d_rho, d_phi, d_E, d_B));
    TRY(cp(ctx, phi, d_phi, sizeof(double) * N, cudaMemcpyDeviceToHost));
    TRY(cp(ctx, efield, d_E, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    TRY(cp(ctx, bfield, d_B, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    return syncc(ctx);
}

int osc_space_charge_rectpipe_dev(osc_ctx *ctx, const osc_mesh3d *mesh, const double *d_rho, double apipe,
                                  double bpipe, int direct_field_calc, int integrated_green_function, int precision,
                                  double *d_phi, double *d_efield, double *d_bfield) {
    if (!ctx) return OSC_E_INVALID;
    (void)apipe;
    (void)bpipe;
    (void)integrated_green_function;
    int64_t N;
    TRY(mesh_n(ctx, mesh, &N));
    if (precision < 0 || precision > 2) return set_err(ctx, OSC_E_INVALID, "precision");
    if (!d_rho || !d_phi || !d_efield || !d_bfield) return set_err(ctx, OSC_E_INVALID, "space_charge_rectpipe arrays");
    if (direct_field_calc)
        return set_err(ctx, OSC_E_UNSUPPORTED,
                       "**********ERROR********* rectpipe implementation presently requires directfieldcalc=0");
    PipeGreen &p = ctx->pipe;
    bool same = p.valid;
    for (int d = 0; d < 3 && same; ++d)
        same = p.nlo[d] == mesh->nlo[d] && p.nhi[d] == mesh->nhi[d] && p.npad[d] == mesh->npad[d];
    if (!same)
        return set_err(ctx, OSC_E_STATE,
                       "something wrong. rectpipe green functions should have been computed during initialization "
                       "(call osc_rectpipe_green or osc_read_rectpipe_grn for this mesh first)");
    return pipe_solve(ctx, precision, mesh->delta, mesh->gamma, d_rho, d_phi, d_efield, d_bfield);
}

// ---- rectpipegrn.dat (core:825-870): gfortran unformatted sequential records --------------
namespace {
const int64_t kMaxSub = 2147483639;  // largest gfortran subrecord payload (2^31 - 9)

bool write_record(FILE *f, const void *data, int64_t bytes) {
    const char *p = static_cast<const char *>(data);
    int64_t left = bytes;
    bool first = true;
    do {
        const int64_t chunk = left > kMaxSub ? kMaxSub : left;
        const bool last = (left - chunk) == 0;
        int32_t head = (int32_t)(last ? chunk : -chunk);
        int32_t tail = (int32_t)(first ? chunk : -chunk);
        if (fwrite(&head, 4, 1, f) != 1) return false;
        if (chunk && fwrite(p, 1, (size_t)chunk, f) != (size_t)chunk) return false;
        if (fwrite(&tail, 4, 1, f) != 1) return false;
        p += chunk;
        left -= chunk;
        first = false;
    } while (left > 0);
    return true;
}

bool read_record(FILE *f, std::vector<char> &out) {
    out.clear();
    for (;;) {
        int32_t head, tail;
        if (fread(&head, 4, 1, f) != 1) return false;
        const int64_t len = head < 0 ? -(int64_t)head : head;
        const size_t at = out.size();
        out.resize(at + (size_t)len);
        if (len && fread(out.data() + at, 1, (size_t)len, f) != (size_t)len) return false;
        if (fread(&tail, 4, 1, f) != 1) return false;
        if (head >= 0) return true;
    }
}
}  // namespace

int osc_write_rectpipe_grn(osc_ctx *ctx, const char *path, double apipe, double bpipe, const osc_mesh3d *mesh) {
    if (!ctx || !path || !mesh) return OSC_E_INVALID;
    PipeGreen &p = ctx->pipe;
    if (!p.valid) return set_err(ctx, OSC_E_STATE, "no pipe Green functions on this context");
    const int64_t M = (int64_t)p.period[0] * p.period[1] * p.period[2];
    std::vector<char> hdr;
    auto put = [&](const void *v, size_t n) {
        const char *c = static_cast<const char *>(v);
        hdr.insert(hdr.end(), c, c + n);
    };
    const double d[11] = {apipe, bpipe, mesh->delta[0], mesh->delta[1], mesh->delta[2], mesh->min[0], mesh->min[1],
                          mesh->min[2], mesh->max[0], mesh->max[1], mesh->max[2]};
    put(d, sizeof(d));
    const int32_t iv[9] = {mesh->nlo[0], mesh->nlo[1], mesh->nlo[2], mesh->nhi[0], mesh->nhi[1], mesh->nhi[2],
                           p.period[0], p.period[1], p.period[2]};
    put(iv, sizeof(iv));
    put(&mesh->gamma, sizeof(double));
    std::vector<char> body((size_t)(4 * M * sizeof(double2)));
    for (int t = 0; t < 4; ++t)
        TRY(cp(ctx, body.data() + t * M * sizeof(double2), p.g[t].p, M * sizeof(double2), cudaMemcpyDeviceToHost));
    TRY(syncc(ctx));
    FILE *f = fopen(path, "wb");
    if (!f) return set_err(ctx, OSC_E_INVALID, "cannot open %s for writing", path);
    const bool ok = write_record(f, hdr.data(), (int64_t)hdr.size()) && write_record(f, body.data(), (int64_t)body.size());
    fclose(f);
    if (!ok) return set_err(ctx, OSC_E_INVALID, "write to %s failed", path);
    return OSC_OK;
}

int osc_read_rectpipe_grn(osc_ctx *ctx, const char *path, const osc_mesh3d *mesh, double *apipe, double *bpipe) {
    if (!ctx || !path || !mesh) return OSC_E_INVALID;
    const int nlo[3] = {mesh->nlo[0], mesh->nlo[1], mesh->nlo[2]}, nhi[3] = {mesh->nhi[0], mesh->nhi[1], mesh->nhi[2]};
    const int npad[3] = {mesh->npad[0], mesh->npad[1], mesh->npad[2]};
    LGeom g;
    TRY(lgeom(ctx, nlo, nhi, npad, g));
    FILE *f = fopen(path, "rb");
    if (!f) return set_err(ctx, OSC_E_INVALID, "cannot open %s", path);
    std::vector<char> hdr, body;
    const bool ok = read_record(f, hdr) && read_record(f, body);
    fclose(f);
    if (!ok || hdr.size() != 11 * 8 + 9 * 4 + 8) return set_err(ctx, OSC_E_INVALID, "%s: bad record structure", path);
    double d[11], gam;
    int32_t iv[9];
    std::memcpy(d, hdr.data(), sizeof(d));
    std::memcpy(iv, hdr.data() + sizeof(d), sizeof(iv));
    std::memcpy(&gam, hdr.data() + sizeof(d) + sizeof(iv), sizeof(double));
    if (iv[6] != g.period[0] || iv[7] != g.period[1] || iv[8] != g.period[2] ||
        body.size() != (size_t)(4 * g.M * sizeof(double2)))
        return set_err(ctx, OSC_E_INVALID, "%s: array sizes differ from this mesh", path);
    TRY(pipe_alloc(ctx, g));
    PipeGreen &p = ctx->pipe;
    for (int t = 0; t < 4; ++t)
        TRY(cp(ctx, p.g[t].p, body.data() + t * g.M * sizeof(double2), g.M * sizeof(double2), cudaMemcpyHostToDevice));
    TRY(syncc(ctx));
    for (int q = 0; q < 3; ++q) {
        p.nlo[q] = nlo[q];
        p.nhi[q] = nhi[q];
        p.npad[q] = npad[q];
        p.period[q] = g.period[q];
        p.delta[q] = d[2 + q];
        p.umin[q] = d[5 + q];
        p.umax[q] = d[8 + q];
    }
    p.apipe = d[0];
    p.bpipe = d[1];
    p.gamma = gam;
    p.valid = true;
    if (apipe) *apipe = d[0];
    if (bpipe) *bpipe = d[1];
    return OSC_OK;
}

}  // extern "C"
