// solver.cu -- free-space IGF field solves: the optimised pipeline and the plain FP64 path.
//
// Optimised pipeline (osc_freespace_solver2 semantics, code/open_spacecharge_mod.f90:535):
// the kernel g is stored "centred" (displacement a at index a mod 2n), which makes the
// physical output window [0,n) in every axis -- the same linear map as the reference's
// shifted extraction at n-1.  Its spectrum is computed once in FP64 and cached, stored as
// a half spectrum (real input along x), and where the offset along an axis is zero the
// kernel's parity halves the stored extent along y and z and makes the spectrum purely
// real or imaginary.  The cathode image (-rho flipped in z) is folded into the same
// spectral product, so the image costs one more spectrum read, not one more solve.
#include <cstring>
#include <sstream>
#include <type_traits>

#include "solver.cuh"

namespace osc {

#define TRY(...)                   \
    do {                           \
        int rc_ = (__VA_ARGS__);   \
        if (rc_) return rc_;       \
    } while (0)

static int kerr(osc_ctx *c, int rc, const char *what) {
    if (rc == OSC_OK) return OSC_OK;
    if (rc == OSC_E_FFT_SIZE) return set_err(c, rc, "%s: unsupported transform length", what);
    cudaError_t e = cudaGetLastError();
    return set_err(c, rc, "%s: %s", what, cudaGetErrorString(e));
}

template <typename T>
int fft3d_full(osc_ctx *c, cplx<T> *a, int Nx, int Ny, int Nz, int sx, int sy, int sz) {
    const int Ls[3] = {Nx, Ny, Nz};
    const int sg[3] = {sx, sy, sz};
    for (int ax = 0; ax < 3; ++ax) {
        if (sg[ax] == 0) continue;
        LineArgs la;
        if (!make_fft_plan(Ls[ax], la.p)) return set_err(c, OSC_E_FFT_SIZE, "FFT length %d unsupported", Ls[ax]);
        TwPair<cplx<T>> tw;
        TRY(twiddles<T>(c, Ls[ax], &tw));
        la.sign = sg[ax];
        la.in_len = la.out_len = Ls[ax];
        la.out_lo = 0;
        la.scale = 1.0;
        la.in_zstride = la.out_zstride = 0;
        la.flip_mask = 0;
        int nplanes = 1;
        bool row = false;
        if (ax == 0) {
            la.ncols = Ny * Nz;
            la.in_pstride = la.out_pstride = 0;
            la.in_cstride = la.out_cstride = Nx;
            la.in_estride = la.out_estride = 1;
            row = true;
        } else if (ax == 1) {
            la.ncols = Nx;
            nplanes = Nz;
            la.in_pstride = la.out_pstride = (int64_t)Nx * Ny;
            la.in_cstride = la.out_cstride = 1;
            la.in_estride = la.out_estride = Nx;
        } else {
            la.ncols = Nx * Ny;
            la.in_pstride = la.out_pstride = 0;
            la.in_cstride = la.out_cstride = 1;
            la.in_estride = la.out_estride = (int64_t)Nx * Ny;
        }
        Launch L_(c, ax == 0 ? "fft_x_c2c" : (ax == 1 ? "fft_y_c2c" : "fft_z_c2c"));
        TRY(kerr(c, launch_lines<T>(a, a, la, nplanes, 1, row, tw, c->stream), "fft3d_full"));
    }
    return OSC_OK;
}
template int fft3d_full<float>(osc_ctx *, cplx<float> *, int, int, int, int, int, int);
template int fft3d_full<double>(osc_ctx *, cplx<double> *, int, int, int, int, int, int);

// Corner block of the IGF primitive of one component (osc_get_cgrn_freespace,
// code/open_spacecharge_mod.f90:648-668): on symmetric axes (offset 0) only the corners
// n-1 .. 2n-1 of the doubled grid, which the mirrored kernel needs, else all 2n.
CornerArgs green_corner_args(const int n[3], const double delta[3], double gamma, const double off[3], int icomp) {
    int sym[3], c0[3], cd[3], N[3];
    for (int d = 0; d < 3; ++d) {
        sym[d] = off[d] == 0.0 ? 1 : 0;
        N[d] = 2 * n[d];
        c0[d] = sym[d] ? n[d] - 1 : 0;
        cd[d] = sym[d] ? n[d] + 1 : 2 * n[d];
    }
    CornerArgs ca;
    ca.cdx = cd[0]; ca.cdy = cd[1]; ca.cdz = cd[2];
    ca.c0x = c0[0]; ca.c0y = c0[1]; ca.c0z = c0[2];
    ca.dx = delta[0];
    ca.dy = delta[1];
    ca.dz = delta[2] * gamma;
    ca.factor = (icomp == 1 || icomp == 2) ? gamma / (ca.dx * ca.dy * ca.dz) : 1.0 / (ca.dx * ca.dy * ca.dz);
    ca.umin = (double)(0.5f - (float)(N[0] / 2)) * ca.dx + off[0];
    ca.vmin = (double)(0.5f - (float)(N[1] / 2)) * ca.dy + off[1];
    ca.wmin = (double)(0.5f - (float)(N[2] / 2)) * ca.dz + off[2] * gamma;
    ca.icomp = icomp;
    return ca;
}

// ------------------------------------------------------------------------------------
// Stored spectra of all-symmetric kernels (offset 0 on every axis) of nb geometries with
// equal grids, from their corner blocks F ((n+1)^3 apart): octant differences, then even/
// odd transforms along x, y and z; the last pass applies fpei/M and writes the stored
// layout (zinner: [ky][kx][kz] with columns zpitch apart, else [kz][ky][kx]) of member b at
// out + b * out_bstride.  Equals the extraction of the FP64 doubled-grid FFT
// (osc_get_cgrn_freespace + ccfft3d, code/open_spacecharge_mod.f90:633-705,
// code/fft_interface_mod.f90:96-143) up to rounding.  The corner primitives and their
// 8-corner differences, whose log/atan terms cancel catastrophically at large offsets,
// are always FP64; the line transforms run in T: FP64 for FP64 spectra, FP32 (from the
// octant values rounded once) for the FP32 path, whose stored spectrum is FP32 anyway.
template <typename T>
int green_sym_lines3(osc_ctx *c, const double *F, int nb, int nx, int ny, int nz, const int odd[3][2], int zinner,
                     int zpitch, T *out, int64_t out_bstride) {
    const int nxh = nx + 1, nyh = ny + 1;
    T *h, *hx, *hy;
    TRY(ws_get(c, "green_h", sizeof(T) * (size_t)nb * nx * ny * nz, (void **)&h));
    TRY(ws_get(c, "green_hx", sizeof(T) * (size_t)nb * nxh * ny * nz, (void **)&hx));
    TRY(ws_get(c, "green_hy", sizeof(T) * (size_t)nb * nxh * nyh * nz, (void **)&hy));
    {
        Launch L_(c, "green_octant");
        TRY(kerr(c, launch_green_octant<T>(F, h, nx, ny, nz, nb, c->stream), "green octant"));
    }
    FFTPlan px, py, pz;
    if (!make_fft_plan(2 * nx, px) || !make_fft_plan(2 * ny, py) || !make_fft_plan(2 * nz, pz))
        return set_err(c, OSC_E_FFT_SIZE, "doubled grid lengths must be 2^a 3^b 5^c");
    TwPair<cplx<T>> twx, twy, twz;
    TRY(twiddles<T>(c, 2 * nx, &twx));
    TRY(twiddles<T>(c, 2 * ny, &twy));
    TRY(twiddles<T>(c, 2 * nz, &twz));
    Launch L_(c, "green_sym_lines", 3);
    SymArgs a;
    const std::string tp = sizeof(T) == 4 ? "f32" : "f64";
    // x: rows h[c][b][0..nx) -> hx[c][b][0..nx]
    a.p = px; a.n = nx; a.odd_lo = odd[0][0]; a.odd_hi = odd[0][1]; a.nq = ny;
    a.npq = (int64_t)ny * nz; a.nlines = nb * a.npq;
    a.in_ps = (int64_t)ny * nx; a.in_qs = nx; a.in_es = 1; a.in_bs = (int64_t)nx * ny * nz;
    a.out_ps = (int64_t)ny * nxh; a.out_qs = nxh; a.out_es = 1; a.out_bs = (int64_t)nxh * ny * nz;
    a.scale = 1.0;
    a.nl_div = tune_get(c, "sym_nl_div:" + tp + ":L" + std::to_string(2 * nx));
    TRY(kerr(c, launch_sym_lines<T, T, T>(h, hx, a, twx, true, true, c->stream), "green x"));
    // y: lines (c, kx) of hx -> hy[c][ky][kx]
    a.p = py; a.n = ny; a.odd_lo = odd[1][0]; a.odd_hi = odd[1][1]; a.nq = nxh;
    a.npq = (int64_t)nz * nxh; a.nlines = nb * a.npq;
    a.in_ps = (int64_t)ny * nxh; a.in_qs = 1; a.in_es = nxh; a.in_bs = (int64_t)nxh * ny * nz;
    a.out_ps = (int64_t)nyh * nxh; a.out_qs = 1; a.out_es = nxh; a.out_bs = (int64_t)nxh * nyh * nz;
    a.nl_div = tune_get(c, "sym_nl_div:" + tp + ":L" + std::to_string(2 * ny));
    TRY(kerr(c, launch_sym_lines<T, T, T>(hx, hy, a, twy, false, false, c->stream), "green y"));
    // z: lines (ky, kx) of hy -> stored spectrum, scaled by fpei/M
    a.p = pz; a.n = nz; a.odd_lo = odd[2][0]; a.odd_hi = odd[2][1]; a.nq = nxh;
    a.npq = (int64_t)nyh * nxh; a.nlines = nb * a.npq;
    a.in_ps = nxh; a.in_qs = 1; a.in_es = (int64_t)nyh * nxh; a.in_bs = (int64_t)nxh * nyh * nz;
    if (zinner) {
        a.out_ps = (int64_t)nxh * zpitch; a.out_qs = zpitch; a.out_es = 1;
    } else {
        a.out_ps = nxh; a.out_qs = 1; a.out_es = (int64_t)nyh * nxh;
    }
    a.out_bs = out_bstride;
    a.scale = fpei_solver2() / (8.0 * nx * ny * nz);
    a.nl_div = tune_get(c, "sym_nl_div:" + tp + ":L" + std::to_string(2 * nz));
    TRY(kerr(c, launch_sym_lines<T, T, T>(hy, out, a, twz, false, zinner != 0, c->stream), "green z"));
    return OSC_OK;
}
template int green_sym_lines3<float>(osc_ctx *, const double *, int, int, int, int, const int (*)[2], int, int,
                                     float *, int64_t);
template int green_sym_lines3<double>(osc_ctx *, const double *, int, int, int, int, const int (*)[2], int, int,
                                      double *, int64_t);

// All components of a geometry with zero offset (even or odd along every axis) at once:
// the corner blocks of every component in one launch, then the octant differences and the
// three even/odd line passes with the components as batch members (per axis, the member of
// that axis' E component is the odd one); one buffer holds the stored spectra of all
// components, in gs.buf[0], and gs.spec[i] points at component comps[i].
template <typename T>
static int green_sym_set(osc_ctx *c, int nx, int ny, int nz, const double delta[3], double gamma, const int *comps,
                         int ncomp, GreenSet &gs) {
    const int n[3] = {nx, ny, nz};
    const double off0[3] = {0.0, 0.0, 0.0};
    const int64_t fstride = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    double *F;
    TRY(ws_get(c, "green_F", sizeof(double) * (size_t)ncomp * fstride, (void **)&F));
    CornerSet cs;
    cs.n = ncomp;
    for (int i = 0; i < ncomp; ++i) cs.a[i] = green_corner_args(n, delta, gamma, off0, comps[i]);
    {
        Launch L_(c, "green_corners");
        TRY(kerr(c, launch_igf_corners_set(F, cs, fstride, c->stream), "green corners"));
    }
    const int zinner = zconv_warp_ok(2 * nz, nz, (int)sizeof(T)) ? 1 : 0;
    const int zp = zinner ? green_zpitch(nz + 1, sizeof(T)) : nz + 1;
    const int64_t per = (int64_t)(nx + 1) * (ny + 1) * zp;
    DevBuf store;
    TRY(green_alloc(c, sizeof(T) * (size_t)per * ncomp, store));
    int odd[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    for (int i = 0; i < ncomp; ++i)
        if (comps[i] >= 1) {
            odd[comps[i] - 1][0] = i;
            odd[comps[i] - 1][1] = i + 1;
        }
    int rc = zinner ? cuda_check(c, cudaMemsetAsync(store.p, 0, store.bytes, c->stream), "memset spectra") : OSC_OK;
    if (!rc) rc = green_sym_lines3<T>(c, F, ncomp, nx, ny, nz, odd, zinner, zp, reinterpret_cast<T *>(store.p), per);
    if (rc) {
        green_release(c, store);
        return rc;
    }
    const int base = gs.nspec;
    gs.buf[base] = store;
    gs.bytes += store.bytes;
    for (int i = 0; i < ncomp; ++i) {
        GSpecDev &s = gs.spec[base + i];
        s = GSpecDev{};
        s.data = reinterpret_cast<T *>(store.p) + i * per;
        s.real_valued = 1;
        s.imag_unit = comps[i] != 0 ? 1 : 0;
        s.sym_y = s.sym_z = 1;
        s.par_y = comps[i] == 2 ? -1 : 1;
        s.par_z = comps[i] == 3 ? -1 : 1;
        s.dimy = ny + 1;
        s.dimz = nz + 1;
        s.zinner = zinner;
        s.zpitch = zp;
    }
    gs.nspec += ncomp;
    return OSC_OK;
}

// ------------------------------------------------------------------------------------
// Green spectrum of one component (icomp 0 phi, 1..3 E) of a kernel with a non-zero offset
// on some axis (all-symmetric kernels go through green_sym_set): corners, the centred
// complex doubled grid, an FP64 3D FFT and the extraction into the stored layout.
template <typename T>
static int build_green_component(osc_ctx *c, int nx, int ny, int nz, const double delta[3], double gamma,
                                 const double off[3], int icomp, bool image, DevBuf &store, GSpecDev &spec) {
    const int n[3] = {nx, ny, nz};
    const int N[3] = {2 * nx, 2 * ny, 2 * nz};
    const int64_t M = (int64_t)N[0] * N[1] * N[2];
    int sym[3], par[3] = {1, 1, 1}, c0[3], cd[3];
    for (int d = 0; d < 3; ++d) sym[d] = off[d] == 0.0 ? 1 : 0;
    if (icomp >= 1) par[icomp - 1] = -1;
    for (int d = 0; d < 3; ++d) {
        c0[d] = sym[d] ? n[d] - 1 : 0;
        cd[d] = sym[d] ? n[d] + 1 : 2 * n[d];
    }
    double *F;
    double2 *cg;
    TRY(ws_get(c, "green_F", sizeof(double) * (size_t)cd[0] * cd[1] * cd[2], (void **)&F));
    const CornerArgs ca = green_corner_args(n, delta, gamma, off, icomp);
    {
        Launch L_(c, "green_corners");
        TRY(kerr(c, launch_igf_corners(F, ca, c->stream), "green corners"));
    }
    TRY(ws_get(c, "green_cg", sizeof(double2) * (size_t)M, (void **)&cg));
    CenterArgs ce;
    ce.nx = nx; ce.ny = ny; ce.nz = nz;
    ce.symx = sym[0]; ce.symy = sym[1]; ce.symz = sym[2];
    ce.parx = par[0]; ce.pary = par[1]; ce.parz = par[2];
    ce.c0x = c0[0]; ce.c0y = c0[1]; ce.c0z = c0[2];
    ce.cdx = cd[0]; ce.cdy = cd[1];
    {
        Launch L_(c, "green_center");
        TRY(kerr(c, launch_green_center(F, cg, ce, c->stream), "green center"));
    }
    TRY(fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(cg), N[0], N[1], N[2], 1, 1, 1));
    spec.real_valued = (sym[0] && sym[1] && sym[2]) ? 1 : 0;
    spec.imag_unit = (spec.real_valued && icomp != 0) ? 1 : 0;
    spec.sym_y = sym[1];
    spec.sym_z = sym[2];
    spec.par_y = par[1];
    spec.par_z = par[2];
    spec.dimy = sym[1] ? ny + 1 : N[1];
    spec.dimz = sym[2] ? nz + 1 : N[2];
    spec.zinner = zconv_warp_ok(N[2], nz, (int)sizeof(T)) ? 1 : 0;
    spec.zpitch = spec.zinner ? green_zpitch(spec.dimz, spec.real_valued ? sizeof(T) : sizeof(cplx<T>)) : spec.dimz;
    // an image spectrum even/odd in x and y: half of z stored, flip phase applied, for the
    // image z pass (its value at Nz - kz is par_x par_y times the conjugate of that at kz)
    const bool herm = image && sym[0] && sym[1] && !sym[2] && zconv_img_ok(N[2], nz, (int)sizeof(T));
    if (herm) {
        spec.dimz = nz + 1;
        spec.zpitch = green_zpitch(spec.dimz, sizeof(cplx<T>));
        spec.herm_img = 1;
        spec.par_h = par[0] * par[1];
    }
    const size_t elems = (size_t)(nx + 1) * spec.dimy * spec.zpitch;
    const size_t bytes = elems * (spec.real_valued ? sizeof(T) : sizeof(cplx<T>));
    TRY(green_alloc(c, bytes, store));
    const double scale = fpei_solver2() / (double)M;
    {
        Launch L_(c, "green_extract");
        TRY(kerr(c, launch_green_extract<T>(cg, store.p, nx, N[0], N[1], spec.dimy, spec.dimz, spec.real_valued,
                                            spec.imag_unit, scale, spec.zinner ? spec.zpitch : 0, herm ? nz - 1 : -1,
                                            N[2], c->stream),
                 "green extract"));
    }
    spec.data = store.p;
    return OSC_OK;
}

static std::string fs_key(const FreeSpaceJob &j, int tbytes, const int *comps, int ncomp) {
    std::ostringstream s;
    s.precision(17);
    s << "fs|" << tbytes << "|" << j.nx << "," << j.ny << "," << j.nz << "|" << j.delta[0] << "," << j.delta[1]
      << "," << j.delta[2] << "|" << j.gamma << "|" << j.offset[0] << "," << j.offset[1] << "," << j.offset[2]
      << "|" << (j.at_cathode ? j.img_zoff : 0.0) << "|" << j.at_cathode << "|";
    for (int i = 0; i < ncomp; ++i) s << comps[i];
    return s.str();
}

// Cached Green set for a job: spectra [direct comps..., image comps...].
template <typename T>
static int green_set(osc_ctx *c, const FreeSpaceJob &j, const int *comps, int ncomp, GreenSet **out) {
    const std::string key = fs_key(j, (int)sizeof(T), comps, ncomp);
    if (GreenSet *g = gcache_find(c, key)) {
        *out = g;
        return OSC_OK;
    }
    GreenSet gs;
    gs.key = key;
    const int nsets = j.at_cathode ? 2 : 1;
    for (int s = 0; s < nsets; ++s) {
        double off[3] = {j.offset[0], j.offset[1], j.offset[2]};
        if (s == 1) off[2] = off[2] + j.img_zoff;
        if (off[0] == 0.0 && off[1] == 0.0 && off[2] == 0.0) {
            const int rc = green_sym_set<T>(c, j.nx, j.ny, j.nz, j.delta, j.gamma, comps, ncomp, gs);
            if (rc) {
                for (int q = 0; q < gs.nspec; ++q) green_release(c, gs.buf[q]);
                return rc;
            }
            continue;
        }
        for (int i = 0; i < ncomp; ++i) {
            const int k = gs.nspec;
            int rc = build_green_component<T>(c, j.nx, j.ny, j.nz, j.delta, j.gamma, off, comps[i], s == 1,
                                                       gs.buf[k], gs.spec[k]);
            if (rc) {
                for (int q = 0; q <= k; ++q) green_release(c, gs.buf[q]);
                return rc;
            }
            gs.bytes += gs.buf[k].bytes;
            gs.nspec++;
        }
    }
    *out = gcache_insert(c, std::move(gs));
    return OSC_OK;
}

template <typename T, typename TIn>
int freespace_opt(osc_ctx *c, const FreeSpaceJob &j, const TIn *rho) {
    typedef cplx<T> V;
    const int nx = j.nx, ny = j.ny, nz = j.nz;
    const int Nx = 2 * nx, Ny = 2 * ny, Nz = 2 * nz, nxh = nx + 1;
    const int64_t N = (int64_t)nx * ny * nz;
    FFTPlan px, py, pz;
    if (!make_fft_plan(Nx, px) || !make_fft_plan(Ny, py) || !make_fft_plan(Nz, pz))
        return set_err(c, OSC_E_FFT_SIZE, "doubled grid %dx%dx%d: lengths must be 2^a 3^b 5^c <= %d", Nx, Ny, Nz,
                       FFT_MAX_LEN);
    int comps[4], ncomp = 0;
    if (j.want_phi) comps[ncomp++] = 0;
    if (j.want_e || j.calc_b)
        for (int q = 1; q <= 3; ++q) comps[ncomp++] = q;
    if (ncomp == 0) return OSC_OK;
    const int B = j.nbatch > 0 ? j.nbatch : 1;
    if (B > 1 && (j.phi || j.E || j.B || !j.E4 || !j.gbatch || j.at_cathode))
        return set_err(c, OSC_E_INVALID, "batched solves produce the E grid only");
    if (j.sum3 && (B > 1 || !j.quad || !j.E4 || !j.e4_pairs || j.phi || j.E || j.B || j.at_cathode || j.want_phi ||
                   j.calc_b || !std::is_same<T, float>::value))
        return set_err(c, OSC_E_INVALID, "summed solve: FP32 quad inputs to the x-pair grid only");
    // input and output members: the summed solve reads three grids and writes one
    const int Bin = j.sum3 ? 3 : B, Bout = j.sum3 ? 1 : B;
    GreenSet local;
    GreenSet *gs = &local;
    if (j.gbatch) {
        if (j.ngbatch != ncomp) return set_err(c, OSC_E_INVALID, "batched spectra: %d components given", j.ngbatch);
        for (int i = 0; i < ncomp; ++i) local.spec[i] = j.gbatch[i];
        local.nspec = ncomp;
    } else {
        TRY(green_set<T>(c, j, comps, ncomp, &gs));
    }
    auto spec_index = [&](int icomp, bool img) {
        for (int i = 0; i < ncomp; ++i)
            if (comps[i] == icomp) return img ? ncomp + i : i;
        return -1;
    };
    // outputs of the z-convolution and their destinations
    ZConvArgs za;
    C2RArgs cr;
    std::memset(&za, 0, sizeof(za));
    std::memset(&cr, 0, sizeof(cr));
    int nout = 0;
    auto add_out = [&](int icomp, double icoef) {
        za.gdir[nout] = spec_index(icomp, false);
        za.gimg[nout] = j.at_cathode ? spec_index(icomp, true) : -1;
        za.img_coef[nout] = icoef;
        cr.ndest[nout] = 0;
        return nout++;
    };
    auto add_dest = [&](int o, void *ptr, int kind, int slot, double coef) {
        OutDest &d = cr.dest[o][cr.ndest[o]++];
        d.ptr = ptr;
        d.kind = kind;
        d.slot = slot;
        d.coef = coef;
        d.last_x = nx - 1;
    };
    if (j.sum3) {
        za.nsum = 3;
        for (int q = 0; q < 3; ++q) {
            za.gdir[q] = spec_index(q + 1, false);
            za.gimg[q] = -1;
        }
        cr.ndest[0] = 0;
        nout = 1;
        add_dest(0, j.E4, 4, 3, j.acc_coef);
    } else {
    if (j.want_phi && j.phi) add_dest(add_out(0, 1.0), j.phi, 1, 0, 1.0);
    if (j.want_e || j.calc_b) {
        for (int q = 0; q < 3; ++q) {
            if (!((j.comp_mask >> q) & 1) && !j.calc_b) continue;
            const int o = add_out(q + 1, 1.0);
            if (j.Eacc) add_dest(o, j.Eacc, 3, 0, j.acc_coef);
            if (j.E) add_dest(o, j.E + q * N, 1, 0, 1.0);
            if (j.E4) {  // staged in the x epilogue and written as whole nodes or pairs
                cr.e8 = j.E4;
                cr.e8_comp[q] = o;
                cr.e8_node = j.e4_pairs ? 0 : 1;
            }
            if (j.calc_b && j.B && !j.at_cathode) {
                if (q == 1) add_dest(o, j.B, 1, 0, -j.bcoef);
                if (q == 0) add_dest(o, j.B + N, 1, 0, j.bcoef);
            }
        }
        if (j.calc_b && j.B && j.at_cathode) {
            // image charges move the other way: B from (direct - image) fields
            add_dest(add_out(1, -1.0), j.B + N, 1, 0, j.bcoef);
            add_dest(add_out(2, -1.0), j.B, 1, 0, -j.bcoef);
        }
    }
    }  // summed solve or per-output destinations
    if (j.calc_b && j.B) TRY(cuda_check(c, cudaMemsetAsync(j.B + 2 * N, 0, sizeof(double) * N, c->stream), "memset B"));

    V *X1, *X2, *X3, *X4;
    TRY(ws_get(c, "fs_x1", sizeof(V) * (size_t)Bin * nxh * ny * nz, (void **)&X1));
    TRY(ws_get(c, "fs_x2", sizeof(V) * (size_t)Bin * nxh * Ny * nz, (void **)&X2));
    TRY(ws_get(c, "fs_x3", sizeof(V) * (size_t)nout * Bout * nxh * Ny * nz, (void **)&X3));
    TRY(ws_get(c, "fs_x4", sizeof(V) * (size_t)nout * Bout * nxh * ny * nz, (void **)&X4));
    TwPair<V> twx, twy, twz;
    TRY(twiddles<T>(c, Nx, &twx));
    TRY(twiddles<T>(c, Ny, &twy));
    TRY(twiddles<T>(c, Nz, &twz));

    // x: real rows -> half spectra, [z][y][kx] (batch members stacked along z)
    R2CArgs ra;
    ra.p = px;
    ra.nin = nx;
    ra.nrows = (int64_t)Bin * ny * nz;
    ra.in_rstride = nx;
    ra.out_rstride = nxh;
    const std::string tprec = sizeof(T) == 4 ? "f32" : "f64";
    ra.nl_div = tune_get(c, "r2c_nl_div:" + tprec + ":L" + std::to_string(Nx));
    {
        Launch L_(c, "fft_x_r2c");
        if constexpr (std::is_same<T, float>::value) {
            if (j.quad) {
                ra.qny = ny;
                TRY(kerr(c, launch_r2c_rows<float, float4>(j.quad, X1, ra, twx, c->stream), "x r2c"));
            } else {
                TRY(kerr(c, launch_r2c_rows<T, TIn>(rho, X1, ra, twx, c->stream), "x r2c"));
            }
        } else {
            TRY(kerr(c, launch_r2c_rows<T, TIn>(rho, X1, ra, twx, c->stream), "x r2c"));
        }
    }
    // y forward: [z][y][kx] -> [z][ky][kx]
    LineArgs ly;
    ly.p = py;
    ly.sign = +1;
    ly.ncols = nxh;
    ly.in_len = ny;
    ly.out_lo = 0;
    ly.out_len = Ny;
    ly.in_pstride = (int64_t)nxh * ny;
    ly.in_cstride = 1;
    ly.in_estride = nxh;
    ly.in_zstride = 0;
    ly.out_pstride = (int64_t)nxh * Ny;
    ly.out_cstride = 1;
    ly.out_estride = nxh;
    ly.out_zstride = 0;
    ly.scale = 1.0;
    ly.flip_mask = 0;
    ly.nl_div = tune_get(c, std::string("lines_nl_div:") + (sizeof(T) == 4 ? "f32" : "f64") + ":L" + std::to_string(Ny));
    ly.flat_lines = 1;  // tiles over the (z, kx) line sequence: no part-empty tile per plane
    {
        Launch L_(c, "fft_y_fwd");
        TRY(kerr(c, launch_lines<T>(X1, X2, ly, Bin * nz, 1, false, twy, c->stream), "y forward"));
    }
    // z: forward, spectral product, inverse
    za.p = pz;
    za.nz = nz;
    za.ncols = nxh * Ny;
    za.nxh = nxh;
    za.Ny = Ny;
    za.ny = ny;
    za.in_estride = (int64_t)nxh * Ny;
    // the warp-per-column z pass writes its spectra kz-innermost ([o][b][ky][kx][z]); the
    // inverse y and x passes then read them with adjacent z in adjacent lines
    const bool zin = zconv_warp_ok(Nz, nz, (int)sizeof(T));
    za.out_estride = zin ? 1 : (int64_t)nxh * Ny;
    za.out_colstride = zin ? nz : 1;
    za.out_cstride = (int64_t)Bout * nxh * Ny * nz;
    za.nout = nout;
    za.img_phase_mul = nz - 1;
    za.ng = gs->nspec;
    za.fault = c->d_fault;
    za.engine = tune_get(c, "zconv_engine:" + std::string(sizeof(T) == 4 ? "f32" : "f64") + ":L" + std::to_string(Nz));
    if (c->test_wait_timeout) {  // test only: waits that must run out quickly
        za.poll_limit = 64;
        za.skip_copies = 1;
    }
    za.nbatch = j.sum3 ? 1 : B;
    za.in_bstride = za.out_bstride = (int64_t)nxh * Ny * nz;
    za.g_bstride = j.gbatch ? j.g_bstride : 0;
    for (int i = 0; i < gs->nspec; ++i) za.g[i] = gs->spec[i];
    {
        Launch L_(c, "fft_z_conv");
        TRY(kerr(c, launch_zconv<T>(X2, X3, za, twz, 0, c->stream), "z convolution"));
    }
    // y inverse, window [0,ny)
    LineArgs li = ly;
    li.sign = -1;
    li.in_len = Ny;
    li.out_len = ny;
    li.in_zstride = (int64_t)Bout * nxh * Ny * nz;
    li.out_zstride = (int64_t)Bout * nxh * ny * nz;
    if (zin) {  // lines (kx, z) with z fastest, members as planes
        li.ncols = nxh * nz;
        li.in_cstride = li.out_cstride = 1;
        li.in_estride = li.out_estride = (int64_t)nxh * nz;
        li.in_pstride = (int64_t)nxh * Ny * nz;
        li.out_pstride = (int64_t)nxh * ny * nz;
    } else {
        li.in_pstride = (int64_t)nxh * Ny;
        li.out_pstride = (int64_t)nxh * ny;
    }
    // lines (kx, z) fill whole tiles already; lines kx per plane z tile the flat sequence
    li.flat_lines = zin ? 0 : 1;
    {
        Launch L_(c, "fft_y_inv");
        TRY(kerr(c, launch_lines<T>(X3, X4, li, zin ? Bout : Bout * nz, nout, false, twy, c->stream), "y inverse"));
    }
    // x: half spectra -> real rows [0,nx), scattered to the outputs
    cr.p = px;
    cr.nout = nx;
    cr.nrows = (int64_t)Bout * ny * nz;
    cr.in_rstride = zin ? (int64_t)nxh * nz : nxh;
    cr.in_cstride = (int64_t)Bout * nxh * ny * nz;
    cr.zin = zin ? 1 : 0;
    cr.zin_nz = nz;
    cr.zin_ny = ny;
    cr.ncomp = nout;
    cr.nl_div = tune_get(c, "c2r_nl_div:" + tprec + ":L" + std::to_string(Nx));
    {
        Launch L_(c, "fft_x_c2r");
        TRY(kerr(c, launch_c2r_rows<T>(X4, cr, twx, c->stream), "x c2r"));
    }
    return OSC_OK;
}
// ------------------------------------------------------------------------------------
// z slabs: the passes of freespace_opt<float> with the planes or columns of one rank.
int slab_forward(osc_ctx *c, int nx, int ny, int nzl, const float4 *quad, cplx<float> *X2) {
    typedef cplx<float> V;
    const int Nx = 2 * nx, Ny = 2 * ny, nxh = nx + 1;
    FFTPlan px, py;
    if (!make_fft_plan(Nx, px) || !make_fft_plan(Ny, py))
        return set_err(c, OSC_E_FFT_SIZE, "doubled grid %dx%d: lengths must be 2^a 3^b 5^c", Nx, Ny);
    if (nzl < 1) return OSC_OK;
    V *X1;
    TRY(ws_get(c, "slab_x1", sizeof(V) * (size_t)nxh * ny * nzl, (void **)&X1));
    TwPair<V> twx, twy;
    TRY(twiddles<float>(c, Nx, &twx));
    TRY(twiddles<float>(c, Ny, &twy));
    R2CArgs ra;
    ra.p = px;
    ra.nin = nx;
    ra.nrows = (int64_t)ny * nzl;
    ra.in_rstride = nx;
    ra.out_rstride = nxh;
    ra.qny = ny;
    ra.nl_div = tune_get(c, "r2c_nl_div:f32:L" + std::to_string(Nx));
    {
        Launch L_(c, "fft_x_r2c");
        TRY(kerr(c, launch_r2c_rows<float, float4>(quad, X1, ra, twx, c->stream), "x r2c"));
    }
    LineArgs ly;
    ly.p = py;
    ly.sign = +1;
    ly.ncols = nxh;
    ly.in_len = ny;
    ly.out_lo = 0;
    ly.out_len = Ny;
    ly.in_pstride = (int64_t)nxh * ny;
    ly.in_cstride = 1;
    ly.in_estride = nxh;
    ly.in_zstride = 0;
    ly.out_pstride = (int64_t)nxh * Ny;
    ly.out_cstride = 1;
    ly.out_estride = nxh;
    ly.out_zstride = 0;
    ly.scale = 1.0;
    ly.flip_mask = 0;
    ly.nl_div = tune_get(c, "lines_nl_div:f32:L" + std::to_string(Ny));
    ly.flat_lines = 1;
    Launch L_(c, "fft_y_fwd");
    return kerr(c, launch_lines<float>(X1, X2, ly, nzl, 1, false, twy, c->stream), "y forward");
}

int slab_zpass(osc_ctx *c, const FreeSpaceJob &j, int col0, int ncols, const cplx<float> *in, cplx<float> *out) {
    const int nx = j.nx, ny = j.ny, nz = j.nz, nxh = nx + 1, Ny = 2 * ny, Nz = 2 * nz;
    if (!zconv_warp_ok(Nz, nz, 4))
        return set_err(c, OSC_E_UNSUPPORTED, "z slabs: doubled z length %d has no warp-per-column z pass", Nz);
    if (col0 < 0 || ncols < 0 || (int64_t)col0 + ncols > (int64_t)nxh * Ny)
        return set_err(c, OSC_E_INVALID, "z slabs: columns [%d, %d) outside the %d columns", col0, col0 + ncols,
                       nxh * Ny);
    if (ncols == 0) return OSC_OK;
    FFTPlan pz;
    if (!make_fft_plan(Nz, pz)) return set_err(c, OSC_E_FFT_SIZE, "doubled z length %d", Nz);
    const int comps[3] = {1, 2, 3};
    GreenSet *gs;
    TRY(green_set<float>(c, j, comps, 3, &gs));
    TwPair<cplx<float>> twz;
    TRY(twiddles<float>(c, Nz, &twz));
    ZConvArgs za;
    std::memset(&za, 0, sizeof(za));
    za.p = pz;
    za.nz = nz;
    za.ncols = ncols;
    za.col_base = col0;
    za.nxh = nxh;
    za.Ny = Ny;
    za.ny = ny;
    za.in_estride = ncols;
    za.out_estride = 1;
    za.out_colstride = nz;
    za.out_cstride = (int64_t)ncols * nz;
    za.nout = 3;
    for (int q = 0; q < 3; ++q) {
        za.gdir[q] = q;
        za.gimg[q] = -1;
        za.img_coef[q] = 1.0;
    }
    za.ng = gs->nspec;
    for (int i = 0; i < gs->nspec; ++i) za.g[i] = gs->spec[i];
    za.fault = c->d_fault;
    za.nbatch = 1;
    Launch L_(c, "fft_z_conv");
    return kerr(c, launch_zconv<float>(in, out, za, twz, 0, c->stream), "z convolution");
}

int slab_inverse(osc_ctx *c, int nx, int ny, int nzl, const cplx<float> *X3, float4 *e8) {
    typedef cplx<float> V;
    const int Nx = 2 * nx, Ny = 2 * ny, nxh = nx + 1;
    FFTPlan px, py;
    if (!make_fft_plan(Nx, px) || !make_fft_plan(Ny, py))
        return set_err(c, OSC_E_FFT_SIZE, "doubled grid %dx%d: lengths must be 2^a 3^b 5^c", Nx, Ny);
    if (nzl < 1) return OSC_OK;
    V *X4;
    TRY(ws_get(c, "slab_x4", sizeof(V) * 3 * (size_t)nxh * ny * nzl, (void **)&X4));
    TwPair<V> twx, twy;
    TRY(twiddles<float>(c, Nx, &twx));
    TRY(twiddles<float>(c, Ny, &twy));
    // y inverse over the lines (kx, z) with z fastest, window [0, ny)
    LineArgs li;
    li.p = py;
    li.sign = -1;
    li.ncols = nxh * nzl;
    li.in_len = Ny;
    li.out_lo = 0;
    li.out_len = ny;
    li.in_cstride = li.out_cstride = 1;
    li.in_estride = li.out_estride = (int64_t)nxh * nzl;
    li.in_pstride = li.in_zstride = (int64_t)nxh * Ny * nzl;
    li.out_pstride = li.out_zstride = (int64_t)nxh * ny * nzl;
    li.scale = 1.0;
    li.flip_mask = 0;
    li.nl_div = tune_get(c, "lines_nl_div:f32:L" + std::to_string(Ny));
    {
        Launch L_(c, "fft_y_inv");
        TRY(kerr(c, launch_lines<float>(X3, X4, li, 1, 3, false, twy, c->stream), "y inverse"));
    }
    C2RArgs cr;
    std::memset(&cr, 0, sizeof(cr));
    cr.p = px;
    cr.nout = nx;
    cr.nrows = (int64_t)ny * nzl;
    cr.in_rstride = (int64_t)nxh * nzl;
    cr.in_cstride = (int64_t)nxh * ny * nzl;
    cr.zin = 1;
    cr.zin_nz = nzl;
    cr.zin_ny = ny;
    cr.ncomp = 3;
    cr.e8 = e8;
    for (int q = 0; q < 3; ++q) cr.e8_comp[q] = q;
    cr.e8_node = 0;
    cr.nl_div = tune_get(c, "c2r_nl_div:f32:L" + std::to_string(Nx));
    Launch L_(c, "fft_x_c2r");
    return kerr(c, launch_c2r_rows<float>(X4, cr, twx, c->stream), "x c2r");
}

template int freespace_opt<float, float>(osc_ctx *, const FreeSpaceJob &, const float *);
template int freespace_opt<float, double>(osc_ctx *, const FreeSpaceJob &, const double *);
template int freespace_opt<double, double>(osc_ctx *, const FreeSpaceJob &, const double *);

// ------------------------------------------------------------------------------------
// osc_freespace_solver2 restated on the GPU in FP64, one call = one solve: zero-padded
// complex rho, full 3D transforms, G built and transformed for every component.
static int solver2_plain(osc_ctx *c, int nx, int ny, int nz, const double delta[3], double gamma, const double off[3],
                         const double *rho, double rho_sign, int flipz, double *phi, double *E, int accumulate) {
    const int Nx = 2 * nx, Ny = 2 * ny, Nz = 2 * nz;
    const int64_t M = (int64_t)Nx * Ny * Nz, N = (int64_t)nx * ny * nz;
    double2 *crho, *cgrn;
    double *F;
    TRY(ws_get(c, "plain_crho", sizeof(double2) * (size_t)M, (void **)&crho));
    TRY(ws_get(c, "plain_cgrn", sizeof(double2) * (size_t)M, (void **)&cgrn));
    TRY(ws_get(c, "plain_F", sizeof(double) * (size_t)M, (void **)&F));
    {
        Launch L_(c, "plain_pad");
        TRY(kerr(c, launch_pad_rho(rho, crho, nx, ny, nz, Nx, Ny, Nz, rho_sign, flipz, c->stream), "pad"));
    }
    TRY(fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(crho), Nx, Ny, Nz, 1, 1, 1));
    const double factr = fpei_solver2() / ((double)Nx * Ny * Nz);
    for (int icomp = 0; icomp <= 3; ++icomp) {
        if (icomp == 0 && !phi) continue;
        if (icomp == 1 && !E) break;
        CornerArgs ca;
        ca.cdx = Nx; ca.cdy = Ny; ca.cdz = Nz;
        ca.c0x = ca.c0y = ca.c0z = 0;
        ca.dx = delta[0];
        ca.dy = delta[1];
        ca.dz = delta[2] * gamma;
        ca.factor = (icomp == 1 || icomp == 2) ? gamma / (ca.dx * ca.dy * ca.dz) : 1.0 / (ca.dx * ca.dy * ca.dz);
        ca.umin = (double)(0.5f - (float)(Nx / 2)) * ca.dx + off[0];
        ca.vmin = (double)(0.5f - (float)(Ny / 2)) * ca.dy + off[1];
        ca.wmin = (double)(0.5f - (float)(Nz / 2)) * ca.dz + off[2] * gamma;
        ca.icomp = icomp;
        {
            Launch L_(c, "plain_green_corners");
            TRY(kerr(c, launch_igf_corners(F, ca, c->stream), "plain corners"));
        }
        {
            Launch L_(c, "plain_green_diff");
            TRY(kerr(c, launch_igf_diff_ref(F, cgrn, Nx, Ny, Nz, c->stream), "plain diff"));
        }
        TRY(fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(cgrn), Nx, Ny, Nz, 1, 1, 1));
        {
            Launch L_(c, "plain_cmul");
            TRY(kerr(c, launch_cmul(cgrn, crho, M, c->stream), "plain cmul"));
        }
        TRY(fft3d_full<double>(c, reinterpret_cast<cplx<double> *>(cgrn), Nx, Ny, Nz, -1, -1, -1));
        double *out = icomp == 0 ? phi : E + (int64_t)(icomp - 1) * N;
        {
            Launch L_(c, "plain_extract");
            TRY(kerr(c, launch_extract_re(cgrn, Nx, Ny, nx - 1, ny - 1, nz - 1, nx, ny, nz, factr, out, accumulate,
                                          c->stream),
                     "plain extract"));
        }
    }
    return OSC_OK;
}

// space_charge_3d (code/open_spacecharge_mod.f90:431-489) in the plain FP64 path.
int freespace_plain(osc_ctx *c, const FreeSpaceJob &j, const double *rho) {
    const int64_t N = (int64_t)j.nx * j.ny * j.nz;
    double *Eout = j.E;
    if (!Eout && (j.want_e || j.calc_b)) TRY(ws_get(c, "plain_E", sizeof(double) * 3 * N, (void **)&Eout));
    TRY(solver2_plain(c, j.nx, j.ny, j.nz, j.delta, j.gamma, j.offset, rho, 1.0, 0, j.want_phi ? j.phi : nullptr,
                      (j.want_e || j.calc_b) ? Eout : nullptr, 0));
    if (j.calc_b && j.B) {
        Launch L_(c, "plain_bfield");
        TRY(kerr(c, launch_bfield(Eout, j.B, N, j.bcoef, 0, c->stream), "bfield"));
    }
    if (j.at_cathode) {
        double off[3] = {j.offset[0], j.offset[1], j.offset[2] + j.img_zoff};
        double *img, *phimg = nullptr;
        TRY(ws_get(c, "plain_img", sizeof(double) * 3 * N, (void **)&img));
        if (j.want_phi && j.phi) TRY(ws_get(c, "plain_phimg", sizeof(double) * N, (void **)&phimg));
        TRY(solver2_plain(c, j.nx, j.ny, j.nz, j.delta, j.gamma, off, rho, -1.0, 1, phimg,
                          (j.want_e || j.calc_b) ? img : nullptr, 0));
        if (j.calc_b && j.B) {
            Launch L_(c, "plain_bfield");
            TRY(kerr(c, launch_bfield(img, j.B, N, -j.bcoef, 1, c->stream), "bfield image"));
        }
        if (Eout) {
            Launch L_(c, "plain_axpy");
            TRY(kerr(c, launch_axpy(Eout, img, 1.0, 3 * N, c->stream), "image add"));
        }
        if (phimg) {
            Launch L_(c, "plain_axpy");
            TRY(kerr(c, launch_axpy(j.phi, phimg, 1.0, N, c->stream), "image phi add"));
        }
    }
    if (j.E4) {
        // the plain path hands interpolation the field as three planes; callers use E
        return set_err(c, OSC_E_INVALID, "plain path writes E planes only");
    }
    return OSC_OK;
}

}  // namespace osc
