/*
 * opensc_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see opensc_oracle.h).
 *
 * An FP64 CPU restatement of the reference's space-charge path, loop for loop, in the
 * reference's order of floating-point operations where that order is observable.  Each
 * function cites the reference routine it follows (paths relative to the reference repo).
 * Built with -ffp-contract=off so that no multiply-add is fused, as in the reference's
 * default gfortran build for x86-64.
 *
 * Deliberate deviations (all on inputs where the reference indexes out of bounds):
 *   - deposit routines skip and count particles whose 2x2x2 stencil leaves the mesh;
 *   - interpolate_field clamps to the array bounds as well as to [1, nhi-1].
 *
 * Parity unpinned for the field solve: the reference has no golden vectors and cannot be
 * built here; see the header for what does pin this file.
 */
#include "opensc_oracle.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

namespace {

/* ------------------------------------------------------------------------------------ */
/* 1D mixed-radix Stockham FFT (stands in for Singleton's sfft,                          */
/* code/fast_fourier_am.f90:90, which supports prime factors up to 23).                  */
/* ------------------------------------------------------------------------------------ */
struct Plan {
    int n = 0, sign = 1;
    std::vector<int> radix;
    std::vector<cd> tw; /* tw[m] = exp(sign*2*pi*i*m/n) */
};

bool factorize(int n, std::vector<int> &r) {
    r.clear();
    if (n < 1) return false;
    int m = n;
    while (m % 4 == 0) { r.push_back(4); m /= 4; }
    while (m % 2 == 0) { r.push_back(2); m /= 2; }
    for (int p = 3; p <= 23; p += 2)
        while (m % p == 0) { r.push_back(p); m /= p; }
    return m == 1;
}

bool make_plan(int n, int sign, Plan &P) {
    P.n = n;
    P.sign = sign >= 0 ? 1 : -1;
    if (!factorize(n, P.radix)) return false;
    P.tw.resize(n);
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < n; ++m) {
        /* reduce to the first octant's worth of accuracy: angle = 2*pi*m/n */
        double ang = two_pi * (double)m / (double)n;
        P.tw[m] = cd(std::cos(ang), P.sign * std::sin(ang));
    }
    return true;
}

inline void dft_small(int R, cd *v, const Plan &P) {
    const double s = (double)P.sign;
    if (R == 2) {
        cd a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    } else if (R == 4) {
        cd a = v[0], b = v[1], c = v[2], d = v[3];
        cd apc = a + c, amc = a - c, bpd = b + d, bmd = b - d;
        cd jbmd(-s * bmd.imag(), s * bmd.real()); /* s*i*(b-d) */
        v[0] = apc + bpd;
        v[1] = amc + jbmd;
        v[2] = apc - bpd;
        v[3] = amc - jbmd;
    } else if (R == 3) {
        const double h = 0.86602540378443864676372317075294;
        cd a = v[0], b = v[1], c = v[2];
        cd t = b + c, d = b - c;
        cd m = a - 0.5 * t;
        cd jd(-s * h * d.imag(), s * h * d.real());
        v[0] = a + t;
        v[1] = m + jd;
        v[2] = m - jd;
    } else {
        cd out[23];
        const int step = P.n / R;
        for (int q = 0; q < R; ++q) {
            cd acc = 0.0;
            for (int r = 0; r < R; ++r) acc += v[r] * P.tw[(size_t)((r * q) % R) * step];
            out[q] = acc;
        }
        for (int q = 0; q < R; ++q) v[q] = out[q];
    }
}

void fft_line(const Plan &P, cd *x, cd *work) {
    const int n = P.n;
    if (n <= 1) return;
    cd *src = x, *dst = work;
    int Ns = 1;
    for (int R : P.radix) {
        const int nr = n / R;
        const int tstep = n / (Ns * R);
        for (int j = 0; j < nr; ++j) {
            const int k = j % Ns;
            cd v[23];
            for (int r = 0; r < R; ++r) {
                cd val = src[j + r * nr];
                if (r && k) val *= P.tw[(size_t)r * k * tstep];
                v[r] = val;
            }
            dft_small(R, v, P);
            const int idxD = (j / Ns) * Ns * R + k;
            for (int q = 0; q < R; ++q) dst[idxD + q * Ns] = v[q];
        }
        std::swap(src, dst);
        Ns *= R;
    }
    if (src != x) std::memcpy(x, src, sizeof(cd) * n);
}

/* Batched 1D transform along one axis of an (n1,n2,n3) column-major complex array. */
void fft_axis(cd *a, int n1, int n2, int n3, int axis, int sign) {
    const int len = axis == 0 ? n1 : (axis == 1 ? n2 : n3);
    if (len <= 1) return;
    Plan P;
    make_plan(len, sign, P);
    const int64_t stride = axis == 0 ? 1 : (axis == 1 ? n1 : (int64_t)n1 * n2);
    /* lines: enumerate the two other indices; group 8 adjacent lines for strided axes */
    const int B = axis == 0 ? 1 : 8;
    int64_t nlines_a, nlines_b; /* inner (contiguous-ish) and outer */
    if (axis == 0) { nlines_a = 1; nlines_b = (int64_t)n2 * n3; }
    else if (axis == 1) { nlines_a = n1; nlines_b = n3; }
    else { nlines_a = n1; nlines_b = n2; }
    const int64_t nblk_a = (nlines_a + B - 1) / B;
    const int64_t nwork = nblk_a * nlines_b;
#pragma omp parallel
    {
        std::vector<cd> buf((size_t)B * len), work(len);
#pragma omp for schedule(static)
        for (int64_t w = 0; w < nwork; ++w) {
            const int64_t ib = w % nblk_a, ob = w / nblk_a;
            if (axis == 0) {
                cd *line = a + ob * (int64_t)n1;
                fft_line(P, line, work.data());
                continue;
            }
            const int64_t i0 = ib * B;
            const int cnt = (int)std::min<int64_t>(B, nlines_a - i0);
            int64_t base;
            if (axis == 1) base = i0 + (int64_t)n1 * n2 * ob;
            else base = i0 + (int64_t)n1 * ob;
            for (int e = 0; e < len; ++e)
                for (int c = 0; c < cnt; ++c) buf[(size_t)c * len + e] = a[base + c + e * stride];
            for (int c = 0; c < cnt; ++c) fft_line(P, buf.data() + (size_t)c * len, work.data());
            for (int e = 0; e < len; ++e)
                for (int c = 0; c < cnt; ++c) a[base + c + e * stride] = buf[(size_t)c * len + e];
        }
    }
}

/* ccfft3d (code/fft_interface_mod.f90:96-143): x pass, y pass, z pass, sign idir(axis). */
int ccfft3d(cd *a, const int idir[3], int n1, int n2, int n3) {
    if (!orc_fft_supported(n1) || !orc_fft_supported(n2) || !orc_fft_supported(n3)) return 1;
    if (idir[0] == 0 && idir[1] == 0 && idir[2] == 0) return 0;
    fft_axis(a, n1, n2, n3, 0, idir[0]);
    fft_axis(a, n1, n2, n3, 1, idir[1]);
    fft_axis(a, n1, n2, n3, 2, idir[2]);
    return 0;
}

inline int64_t idx3(int i, int j, int k, int n1, int n2) {
    return (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)n2 * k);
}

/* 1/(4 pi eps0) as the reference spells it.  `299792458.0` is a default-kind (single
 * precision) literal in Fortran, so the squared speed of light is a float32 product. */
inline double fpei_solver2() { /* code/open_spacecharge_mod.f90:547 */
    const float c = 299792458.0f;
    return (double)(c * c) * 1.00000000055e-7;
}
inline double fpei_legacy() { /* code/open_spacecharge_core_mod.f90:515, :1250 */
    return 299792458.0 * 299792458.0 * 1.0e-7;
}
inline double fpei_pipe() { /* code/open_spacecharge_core_mod.f90:783 (all single precision) */
    const float c = 299792458.0f;
    float v = c * c;
    v = v * 1.0e-7f;
    return (double)v;
}
/* code/open_spacecharge_mod.f90:436: `real(dp), parameter :: c_light = 299792458.0` */
inline double c_light_sc3d() { return (double)299792458.0f; }
const double clight_core = 299792458.0; /* core module: 299792458.d0 */

/* Fortran MOD for a non-negative dividend. */
inline int fmod_pos(int a, int p) { return a % p; }

} // namespace

extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_fft_supported(int n) {
    std::vector<int> r;
    return factorize(n, r) ? 1 : 0;
}

int orc_ccfft3d(double *a, const int idir[3], int n1, int n2, int n3) {
    return ccfft3d(reinterpret_cast<cd *>(a), idir, n1, n2, n3);
}

/* code/open_spacecharge_mod.f90:741-747 */
double orc_lafun2(double x, double y, double z) {
    double r = std::sqrt(x * x + y * y + z * z);
    double t = -((z * z) * std::atan(x * y / (z * r))) / 2;
    t = t - ((y * y) * std::atan(x * z / (y * r))) / 2;
    t = t - ((x * x) * std::atan(y * z / (x * r))) / 2;
    t = t + y * z * std::log(x + r);
    t = t + x * z * std::log(y + r);
    t = t + x * y * std::log(z + r);
    return t;
}

/* code/open_spacecharge_mod.f90:721-726 */
double orc_xlafun2(double x, double y, double z) {
    double r = std::sqrt(x * x + y * y + z * z);
    return x * std::atan((y * z) / (r * x)) - z * std::log(r + y) +
           y * std::log((r - z) / (r + z)) / 2;
}

/* osc_get_cgrn_freespace, code/open_spacecharge_mod.f90:633-707.  cgrn is complex. */
void orc_get_cgrn_freespace(double *cgrn_, int isize, int jsize, int ksize, const double delta[3],
                            double gamma, int icomp, const double *offset) {
    cd *cgrn = reinterpret_cast<cd *>(cgrn_);
    const double dx = delta[0], dy = delta[1], dz = delta[2] * gamma;
    double factor;
    if (icomp == 1 || icomp == 2) factor = gamma / (dx * dy * dz);
    else factor = 1.0 / (dx * dy * dz);
    /* (0.5-isize/2) is single precision in the reference; exact for these sizes */
    double umin = (double)(0.5f - (float)(isize / 2)) * dx;
    double vmin = (double)(0.5f - (float)(jsize / 2)) * dy;
    double wmin = (double)(0.5f - (float)(ksize / 2)) * dz;
    if (offset) {
        umin = umin + offset[0];
        vmin = vmin + offset[1];
        wmin = wmin + offset[2] * gamma;
    }
    const int64_t M = (int64_t)isize * jsize * ksize;
    std::vector<double> f(M);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < ksize; ++k) {
        const double w = k * dz + wmin;
        for (int j = 0; j < jsize; ++j) {
            const double v = j * dy + vmin;
            for (int i = 0; i < isize; ++i) {
                const double u = i * dx + umin;
                double g = 0;
                if (icomp == 0) g = orc_lafun2(u, v, w) * factor;
                if (icomp == 1) g = orc_xlafun2(u, v, w) * factor;
                if (icomp == 2) g = orc_xlafun2(v, w, u) * factor;
                if (icomp == 3) g = orc_xlafun2(w, u, v) * factor;
                f[idx3(i, j, k, isize, jsize)] = g;
            }
        }
    }
    /* 8-corner difference over 1:n-1 (array semantics: the right side uses old values);
       the last plane in each dimension keeps the raw corner value. */
#pragma omp parallel for schedule(static)
    for (int k = 0; k < ksize; ++k)
        for (int j = 0; j < jsize; ++j)
            for (int i = 0; i < isize; ++i) {
                double g;
                if (i < isize - 1 && j < jsize - 1 && k < ksize - 1) {
                    auto F = [&](int a, int b, int c) { return f[idx3(a, b, c, isize, jsize)]; };
                    g = +F(i + 1, j + 1, k + 1);
                    g = g - F(i, j + 1, k + 1);
                    g = g - F(i + 1, j, k + 1);
                    g = g - F(i + 1, j + 1, k);
                    g = g - F(i, j, k);
                    g = g + F(i, j, k + 1);
                    g = g + F(i, j + 1, k);
                    g = g + F(i + 1, j, k);
                } else {
                    g = f[idx3(i, j, k, isize, jsize)];
                }
                cgrn[idx3(i, j, k, isize, jsize)] = cd(g, 0.0);
            }
}

/* osc_freespace_solver2, code/open_spacecharge_mod.f90:535-597 */
int orc_freespace_solver2(const double *rho, const int n[3], double gamma, const double delta[3],
                          const double *offset, double *efield, double *phi) {
    const int nx = n[0], ny = n[1], nz = n[2];
    const int nx2 = 2 * nx, ny2 = 2 * ny, nz2 = 2 * nz;
    const int64_t M = (int64_t)nx2 * ny2 * nz2, N = (int64_t)nx * ny * nz;
    std::vector<cd> crho(M, cd(0, 0)), cgrn(M);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                crho[idx3(i, j, k, nx2, ny2)] = cd(rho[idx3(i, j, k, nx, ny)], 0.0);
    const int fwd[3] = {1, 1, 1}, inv[3] = {-1, -1, -1};
    if (ccfft3d(crho.data(), fwd, nx2, ny2, nz2)) return 3;
    const double fpei = fpei_solver2();
    for (int icomp = 0; icomp <= 3; ++icomp) {
        if (icomp == 0 && !phi) continue;
        if (icomp == 1 && !efield) break;
        orc_get_cgrn_freespace(reinterpret_cast<double *>(cgrn.data()), nx2, ny2, nz2, delta,
                               gamma, icomp, offset);
        ccfft3d(cgrn.data(), fwd, nx2, ny2, nz2);
#pragma omp parallel for schedule(static)
        for (int64_t m = 0; m < M; ++m) cgrn[m] = crho[m] * cgrn[m];
        ccfft3d(cgrn.data(), inv, nx2, ny2, nz2);
        const int ishift = nx - 1, jshift = ny - 1, kshift = nz - 1;
        const double factr = fpei / ((double)nx2 * ny2 * nz2);
        double *out = icomp == 0 ? phi : efield + (int64_t)(icomp - 1) * N;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    out[idx3(i, j, k, nx, ny)] =
                        factr * cgrn[idx3(i + ishift, j + jshift, k + kshift, nx2, ny2)].real();
    }
    return 0;
}

/* space_charge_3d, code/open_spacecharge_mod.f90:431-489 */
int orc_space_charge_3d(const orc_mesh *mesh, const double *rho, const double *offset,
                        int at_cathode, int calc_bfield, double *efield, double *bfield) {
    const int n[3] = {mesh->nhi[0] - mesh->nlo[0] + 1, mesh->nhi[1] - mesh->nlo[1] + 1,
                      mesh->nhi[2] - mesh->nlo[2] + 1};
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    double offset0[3] = {0, 0, 0};
    if (offset) for (int d = 0; d < 3; ++d) offset0[d] = offset[d];
    int rc = orc_freespace_solver2(rho, n, mesh->gamma, mesh->delta, offset0, efield, nullptr);
    if (rc) return rc;
    const double c_light = c_light_sc3d();
    double beta = 0;
    if (calc_bfield) {
        beta = std::sqrt(1 - 1 / (mesh->gamma * mesh->gamma));
        for (int64_t m = 0; m < 3 * N; ++m) bfield[m] = 0;
        for (int64_t m = 0; m < N; ++m) {
            bfield[m] = -(beta / c_light) * efield[N + m];
            bfield[N + m] = (beta / c_light) * efield[m];
        }
    }
    if (!at_cathode) return 0;
    offset0[2] = offset0[2] + 2 * mesh->min[2] + (mesh->max[2] - mesh->min[2]);
    std::vector<double> rimg(N), img(3 * N);
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i)
                rimg[idx3(i, j, k, n[0], n[1])] = -rho[idx3(i, j, n[2] - 1 - k, n[0], n[1])];
    rc = orc_freespace_solver2(rimg.data(), n, mesh->gamma, mesh->delta, offset0, img.data(),
                               nullptr);
    if (rc) return rc;
    if (calc_bfield) {
        for (int64_t m = 0; m < N; ++m) {
            bfield[m] = bfield[m] + (beta / c_light) * img[N + m];
            bfield[N + m] = bfield[N + m] - (beta / c_light) * img[m];
        }
    }
    for (int64_t m = 0; m < 3 * N; ++m) efield[m] = efield[m] + img[m];
    return 0;
}

/* deposit_particles, code/open_spacecharge_mod.f90:156-288.
 * Returns 0, or 8 when neither qa nor total_charge is given (the reference prints and
 * returns before touching rho). */
int orc_deposit_particles(int64_t np, const double *xa, const double *ya, const double *za,
                          const double *qa, const double *total_charge, int resize_mesh,
                          orc_mesh *mesh, double *rho, int64_t *n_outside) {
    if (resize_mesh) {
        double mn[3], mx[3], delta[3];
        const double *p[3] = {xa, ya, za};
        for (int d = 0; d < 3; ++d) {
            double lo = p[d][0], hi = p[d][0];
            for (int64_t m = 1; m < np; ++m) {
                if (p[d][m] < lo) lo = p[d][m];
                if (p[d][m] > hi) hi = p[d][m];
            }
            mn[d] = lo;
            mx[d] = hi;
        }
        for (int d = 0; d < 3; ++d)
            delta[d] = (mx[d] - mn[d]) / (double)(mesh->nhi[d] - mesh->nlo[d]);
        for (int d = 0; d < 3; ++d) {
            mn[d] = mn[d] - 1.0e-6 * delta[d];
            mx[d] = mx[d] + 1.0e-6 * delta[d];
        }
        for (int d = 0; d < 3; ++d)
            delta[d] = (mx[d] - mn[d]) / (double)(mesh->nhi[d] - mesh->nlo[d]);
        for (int d = 0; d < 3; ++d) {
            mesh->min[d] = mn[d];
            mesh->max[d] = mx[d];
            mesh->delta[d] = delta[d];
        }
    }
    const double dx = mesh->delta[0], dy = mesh->delta[1], dz = mesh->delta[2];
    const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
    const int ilo = mesh->nlo[0], jlo = mesh->nlo[1], klo = mesh->nlo[2];
    const int ihi = mesh->nhi[0], jhi = mesh->nhi[1], khi = mesh->nhi[2];
    const int nx = ihi - ilo + 1, ny = jhi - jlo + 1, nz = khi - klo + 1;
    const double xmin = mesh->min[0], ymin = mesh->min[1], zmin = mesh->min[2];
    double charge1 = 0;
    if (qa) {
        double s = 0;
        for (int64_t m = 0; m < np; ++m) s += qa[m];
        mesh->charge = s;
    } else if (total_charge) {
        mesh->charge = *total_charge;
        charge1 = *total_charge / (double)np;
    } else {
        return 8;
    }
    for (int64_t m = 0; m < (int64_t)nx * ny * nz; ++m) rho[m] = 0;
    int64_t nout = 0;
    for (int64_t m = 0; m < np; ++m) {
        const int ip = (int)std::floor((xa[m] - xmin) * dxi + 1);
        const int jp = (int)std::floor((ya[m] - ymin) * dyi + 1);
        const int kp = (int)std::floor((za[m] - zmin) * dzi + 1);
        const double ab = ((xmin - xa[m]) + ip * dx) * dxi;
        const double de = ((ymin - ya[m]) + jp * dy) * dyi;
        const double gh = ((zmin - za[m]) + kp * dz) * dzi;
        if (qa) charge1 = qa[m];
        if (ip < ilo || jp < jlo || kp < klo || ip + 1 > ihi || jp + 1 > jhi || kp + 1 > khi) {
            ++nout; /* the reference writes out of bounds here */
            continue;
        }
        const int i = ip - ilo, j = jp - jlo, k = kp - klo;
        auto R = [&](int a, int b, int c) -> double & { return rho[idx3(a, b, c, nx, ny)]; };
        R(i, j, k) = R(i, j, k) + ab * de * gh * charge1;
        R(i, j + 1, k) = R(i, j + 1, k) + ab * (1. - de) * gh * charge1;
        R(i, j + 1, k + 1) = R(i, j + 1, k + 1) + ab * (1. - de) * (1. - gh) * charge1;
        R(i, j, k + 1) = R(i, j, k + 1) + ab * de * (1. - gh) * charge1;
        R(i + 1, j, k + 1) = R(i + 1, j, k + 1) + (1. - ab) * de * (1. - gh) * charge1;
        R(i + 1, j + 1, k + 1) = R(i + 1, j + 1, k + 1) + (1. - ab) * (1. - de) * (1. - gh) * charge1;
        R(i + 1, j + 1, k) = R(i + 1, j + 1, k) + (1. - ab) * (1. - de) * gh * charge1;
        R(i + 1, j, k) = R(i + 1, j, k) + (1. - ab) * de * gh * charge1;
    }
    if (n_outside) *n_outside = nout;
    return 0;
}

/* interpolate_field, code/open_spacecharge_mod.f90:311-390, one call per point.
 * E and B are [np][3]; either may be null.  Returns the number of clamped points. */
int64_t orc_interpolate_field(const orc_mesh *mesh, const double *efield, const double *bfield,
                              int64_t np, const double *x, const double *y, const double *z,
                              double *E, double *B) {
    const int nx = mesh->nhi[0] - mesh->nlo[0] + 1, ny = mesh->nhi[1] - mesh->nlo[1] + 1,
              nz = mesh->nhi[2] - mesh->nlo[2] + 1;
    const int64_t N = (int64_t)nx * ny * nz;
    const double hxi = 1.0 / mesh->delta[0], hyi = 1.0 / mesh->delta[1], hzi = 1.0 / mesh->delta[2];
    int64_t nclamp = 0;
    for (int64_t m = 0; m < np; ++m) {
        int ip = (int)std::floor((x[m] - mesh->min[0]) * hxi + 1);
        int jp = (int)std::floor((y[m] - mesh->min[1]) * hyi + 1);
        int kp = (int)std::floor((z[m] - mesh->min[2]) * hzi + 1);
        int flag = 0;
        const int p[3] = {ip, jp, kp};
        int q[3];
        for (int d = 0; d < 3; ++d) {
            int v = p[d];
            const int lo = std::max(1, mesh->nlo[d]);
            const int hi = mesh->nhi[d] - 1;
            if (v < 1 || v > mesh->nhi[d] - 1) { flag = 1; v = v < 1 ? 1 : mesh->nhi[d] - 1; }
            if (v < lo) { flag = 1; v = lo; }
            if (v > hi) { flag = 1; v = hi; }
            q[d] = v;
        }
        ip = q[0]; jp = q[1]; kp = q[2];
        nclamp += flag;
        const double ab = ((mesh->min[0] - x[m]) + ip * mesh->delta[0]) * hxi;
        const double de = ((mesh->min[1] - y[m]) + jp * mesh->delta[1]) * hyi;
        const double gh = ((mesh->min[2] - z[m]) + kp * mesh->delta[2]) * hzi;
        const int i = ip - mesh->nlo[0], j = jp - mesh->nlo[1], k = kp - mesh->nlo[2];
        const double *fields[2] = {efield, bfield};
        double *outs[2] = {E, B};
        for (int f = 0; f < 2; ++f) {
            if (!fields[f] || !outs[f]) continue;
            for (int c = 0; c < 3; ++c) {
                const double *F = fields[f] + (int64_t)c * N;
                auto A = [&](int a, int b, int cc) { return F[idx3(a, b, cc, nx, ny)]; };
                double v = A(i, j, k) * ab * de * gh;
                v = v + A(i, j + 1, k) * ab * (1. - de) * gh;
                v = v + A(i, j + 1, k + 1) * ab * (1. - de) * (1. - gh);
                v = v + A(i, j, k + 1) * ab * de * (1. - gh);
                v = v + A(i + 1, j, k + 1) * (1. - ab) * de * (1. - gh);
                v = v + A(i + 1, j + 1, k + 1) * (1. - ab) * (1. - de) * (1. - gh);
                v = v + A(i + 1, j + 1, k) * (1. - ab) * (1. - de) * gh;
                v = v + A(i + 1, j, k) * (1. - ab) * de * gh;
                outs[f][3 * m + c] = v;
            }
        }
    }
    return nclamp;
}

/* getbeamboundingbox, code/test_mod.f90:366-407 -> bb = {xmin,xmax,ymin,ymax,zmin,zmax} */
void orc_getbeamboundingbox(int64_t np, const double *x, const double *y, const double *z,
                            double bb[6]) {
    double v[6];
    for (int d = 0; d < 6; ++d) v[d] = -9999999.;
    if (np > 0) {
        const double *p[3] = {x, y, z};
        for (int d = 0; d < 3; ++d) {
            double lo = p[d][0], hi = p[d][0];
            for (int64_t m = 1; m < np; ++m) {
                if (p[d][m] < lo) lo = p[d][m];
                if (p[d][m] > hi) hi = p[d][m];
            }
            v[d] = -lo;
            v[3 + d] = hi;
        }
    }
    bb[0] = -v[0]; bb[1] = v[3];
    bb[2] = -v[1]; bb[3] = v[4];
    bb[4] = -v[2]; bb[5] = v[5];
}

/* get_mesh_quantities, code/test_mod.f90:288-358 */
void orc_get_mesh_quantities(int64_t np, const double *xa, const double *ya, const double *za,
                             const int nlo[3], const int nhi[3], int isetzmin, double delta[3],
                             double umin[3]) {
    const double eps = 1.e-13;
    double bb[6];
    orc_getbeamboundingbox(np, xa, ya, za, bb);
    double sml[3] = {bb[0], bb[2], bb[4]}, big[3] = {bb[1], bb[3], bb[5]};
    for (int d = 0; d < 3; ++d) {
        big[d] = big[d] * (1.0 + std::copysign(1.0, big[d]) * eps);
        sml[d] = sml[d] * (1.0 - std::copysign(1.0, sml[d]) * eps);
    }
    for (int d = 0; d < 3; ++d) {
        const int n = nhi[d] - nlo[d] + 1;
        delta[d] = (big[d] - sml[d]) / (double)(n - 3);
        umin[d] = sml[d] - delta[d];
    }
    if (isetzmin == 1) {
        const int nz = nhi[2] - nlo[2] + 1;
        const double zsml = 1.e-9;
        delta[2] = (big[2] - zsml) / (double)(nz - 1);
        umin[2] = zsml;
    }
}

/* depose_rho_scalar, code/test_mod.f90:410-474.  Returns ifail (skipped particles). */
int64_t orc_depose_rho_scalar(int64_t np, const double *xa, const double *ya, const double *za,
                              const double *lostflag, double *rho, double chrgpermacro,
                              const int nlo[3], const int nhi[3], const double delta[3],
                              const double umin[3], const int nlogbl[3]) {
    const int nx = nhi[0] - nlo[0] + 1, ny = nhi[1] - nlo[1] + 1, nz = nhi[2] - nlo[2] + 1;
    const int ilo = nlo[0], jlo = nlo[1], klo = nlo[2];
    const int ihi = nx, jhi = ny, khi = nz; /* size(rho,d), as the reference writes it */
    const double dx = delta[0], dy = delta[1], dz = delta[2];
    const double xmin = umin[0], ymin = umin[1], zmin = umin[2];
    const int ilogbl = nlogbl[0], jlogbl = nlogbl[1], klogbl = nlogbl[2];
    const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
    const int64_t N = (int64_t)nx * ny * nz;
    for (int64_t m = 0; m < N; ++m) rho[m] = 0.0;
    int64_t ifail = 0;
    for (int64_t m = 0; m < np; ++m) {
        if (lostflag && lostflag[m] != 0.0) continue;
        const int ip = (int)std::floor((xa[m] - xmin) * dxi + ilogbl);
        const int jp = (int)std::floor((ya[m] - ymin) * dyi + jlogbl);
        const int kp = (int)std::floor((za[m] - zmin) * dzi + klogbl);
        const double ab = ((xmin - xa[m]) + (ip - ilogbl + 1) * dx) * dxi;
        const double de = ((ymin - ya[m]) + (jp - jlogbl + 1) * dy) * dyi;
        const double gh = ((zmin - za[m]) + (kp - klogbl + 1) * dz) * dzi;
        if (ip < ilo || jp < jlo || kp < klo || ip > ihi || jp > jhi || kp > khi) {
            ++ifail;
            continue;
        }
        /* array offsets; the upper stencil node must also lie in the array */
        const int i = ip - ilo, j = jp - jlo, k = kp - klo;
        if (i + 1 >= nx || j + 1 >= ny || k + 1 >= nz) {
            ++ifail; /* the reference writes out of bounds here */
            continue;
        }
        auto R = [&](int a, int b, int c) -> double & { return rho[idx3(a, b, c, nx, ny)]; };
        R(i, j, k) = R(i, j, k) + ab * de * gh;
        R(i, j + 1, k) = R(i, j + 1, k) + ab * (1. - de) * gh;
        R(i, j + 1, k + 1) = R(i, j + 1, k + 1) + ab * (1. - de) * (1. - gh);
        R(i, j, k + 1) = R(i, j, k + 1) + ab * de * (1. - gh);
        R(i + 1, j, k + 1) = R(i + 1, j, k + 1) + (1. - ab) * de * (1. - gh);
        R(i + 1, j + 1, k + 1) = R(i + 1, j + 1, k + 1) + (1. - ab) * (1. - de) * (1. - gh);
        R(i + 1, j + 1, k) = R(i + 1, j + 1, k) + (1. - ab) * (1. - de) * gh;
        R(i + 1, j, k) = R(i + 1, j, k) + (1. - ab) * de * gh;
    }
    for (int64_t m = 0; m < N; ++m) rho[m] = rho[m] * chrgpermacro;
    return ifail;
}

/* ------------------------------------------------------------------------------------ */
/* Legacy point-evaluated IGFs, code/open_spacecharge_core_mod.f90:189-428               */
/* ------------------------------------------------------------------------------------ */
static double coulombfun(double u, double v, double w, double gam) { /* core:189-200 */
    if (u == 0.0 && v == 0.0 && w == 0.0) return 0.0;
    return 1.0 / std::sqrt(u * u + v * v + (gam * w) * (gam * w));
}
static double lafun(double x, double y, double z) { /* core:229-238 */
    double r = std::sqrt(x * x + y * y + z * z);
    double res = -0.5 * (z * z) * std::atan(x * y / (z * r));
    res = res - 0.5 * (y * y) * std::atan(x * z / (y * r));
    res = res - 0.5 * (x * x) * std::atan(y * z / (x * r));
    res = res + y * z * std::log(x + r);
    res = res + x * z * std::log(y + r);
    res = res + x * y * std::log(z + r);
    return res;
}
static double xlafun(double x, double y, double z) { /* core:377-392 */
    double r = std::sqrt(x * x + y * y + z * z);
    double res = z - x * std::atan(z / x) + x * std::atan(y * z / (x * r));
    if (y + r != 0) res = res - z * std::log(y + r);
    if (z + r != 0) res = res - y * std::log(z + r);
    return res;
}
static double ylafun(double x, double y, double z) { /* core:397-407 */
    double r = std::sqrt(x * x + y * y + z * z);
    double res = x - y * std::atan(x / y) + y * std::atan(z * x / (y * r));
    if (z + r != 0) res = res - x * std::log(z + r);
    if (x + r != 0) res = res - z * std::log(x + r);
    return res;
}
static double zlafun(double x, double y, double z) { /* core:412-428 */
    double r = std::sqrt(x * x + y * y + z * z);
    double res = y - z * std::atan(y / z) + z * std::atan(x * y / (z * r));
    if (x + r != 0) res = res - y * std::log(x + r);
    if (y + r != 0) res = res - x * std::log(y + r);
    return res;
}
typedef double (*lfun_t)(double, double, double);
static double igf_corner_sum(lfun_t f, double x1, double x2, double y1, double y2, double z1,
                             double z2) {
    double res = f(x2, y2, z2);
    res = res - f(x1, y2, z2);
    res = res - f(x2, y1, z2);
    res = res - f(x2, y2, z1);
    res = res - f(x1, y1, z1);
    res = res + f(x1, y1, z2);
    res = res + f(x1, y2, z1);
    res = res + f(x2, y1, z1);
    return res;
}

/* igfcoulombfun / igfexfun / igfeyfun / igfezfun / coulombfun, core:205-372 */
double orc_igf_point(int icomp, int igfflag, double u, double v, double w, double gam, double dx,
                     double dy, double dz) {
    if (igfflag == 0) return icomp == 0 ? coulombfun(u, v, w, gam) : 0.0;
    const double x1 = u - 0.5 * dx, x2 = u + 0.5 * dx;
    const double y1 = v - 0.5 * dy, y2 = v + 0.5 * dy;
    const double z1 = (w - 0.5 * dz) * gam, z2 = (w + 0.5 * dz) * gam;
    if (icomp == 0) {
        double res = igf_corner_sum(lafun, x1, x2, y1, y2, z1, z2);
        return res / (dx * dy * dz * gam);
    }
    const bool inside = x1 < 0.0 && x2 > 0.0 && y1 < 0.0 && y2 > 0.0 && z1 < 0.0 && z2 > 0.0;
    double res = 0.0;
    if (!inside) {
        lfun_t f = icomp == 1 ? xlafun : (icomp == 2 ? ylafun : zlafun);
        res = igf_corner_sum(f, x1, x2, y1, y2, z1, z2);
    }
    if (icomp == 3) return res / (dx * dy * dz * gam);
    return res / (dx * dy * dz);
}

} /* extern "C" */

namespace {

/* osc_getgrnfree (core:454-497) without the FFT: cgrn over [glo, glo+period). */
void getgrnfree_values(cd *cgrn, const double delta[3], double gam, const int glo[3],
                       const int period[3], const int npad[3], int icomp, int igfflag,
                       double zshft, bool use_zshft) {
    const double dx = delta[0], dy = delta[1], dz = delta[2];
    int shift[3];
    for (int d = 0; d < 3; ++d) shift[d] = period[d] / 2 - (npad[d] + 1) / 2;
#pragma omp parallel for schedule(static)
    for (int kk = 0; kk < period[2]; ++kk) {
        const int kp = glo[2] + fmod_pos(kk + shift[2], period[2]);
        const double w = use_zshft ? kp * dz + zshft : kp * dz;
        for (int jj = 0; jj < period[1]; ++jj) {
            const int jp = glo[1] + fmod_pos(jj + shift[1], period[1]);
            const double v = jp * dy;
            for (int ii = 0; ii < period[0]; ++ii) {
                const int ip = glo[0] + fmod_pos(ii + shift[0], period[0]);
                const double u = ip * dx;
                double g = orc_igf_point(icomp, igfflag, u, v, w, gam, dx, dy, dz);
                cgrn[idx3(ii, jj, kk, period[0], period[1])] = cd(g, 0.0);
            }
        }
    }
}

/* getrhotilde (core:435-449): crho = 0, rho in the low octant, FFT (1,1,1). */
void getrhotilde(const double *rho, cd *crho, const int n[3], const int period[3]) {
    const int64_t M = (int64_t)period[0] * period[1] * period[2];
    for (int64_t m = 0; m < M; ++m) crho[m] = cd(0, 0);
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i)
                crho[idx3(i, j, k, period[0], period[1])] = cd(rho[idx3(i, j, k, n[0], n[1])], 0);
    const int fwd[3] = {1, 1, 1};
    ccfft3d(crho, fwd, period[0], period[1], period[2]);
}

/* conv3d (core:503-529) and imageconvcorr3d (core:1237-1264): product, inverse FFT with
 * the given signs, store the low-corner window times fpei/period^3. */
void conv_extract(const cd *crho, const cd *qgrn, double *con, const int n[3],
                  const int period[3], const int isgn[3], double fpei) {
    const int64_t M = (int64_t)period[0] * period[1] * period[2];
    std::vector<cd> ccon(M);
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < M; ++m) ccon[m] = crho[m] * qgrn[m];
    ccfft3d(ccon.data(), isgn, period[0], period[1], period[2]);
    const double factr = 1.0 / ((1.0 * period[0]) * (1.0 * period[1]) * (1.0 * period[2])) * fpei * 1.0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i)
                con[idx3(i, j, k, n[0], n[1])] = factr * ccon[idx3(i, j, k, period[0], period[1])].real();
}

/* Centred differences with first-order one-sided edges (core:87-104, :588-605, :994-1014). */
void fd_efield(const double *phi, double *efield, const int n[3], const double delta[3],
               double gam0) {
    const int nx = n[0], ny = n[1], nz = n[2];
    const int64_t N = (int64_t)nx * ny * nz;
    const double dx = delta[0], dy = delta[1], dz = delta[2];
    for (int k = 0; k < nz; ++k) {
        int km1 = k - 1; if (km1 < 0) km1 = k;
        int kp1 = k + 1; if (kp1 > nz - 1) kp1 = k;
        const double zfac = (km1 == k || kp1 == k) ? 2.0 : 1.0;
        for (int j = 0; j < ny; ++j) {
            int jm1 = j - 1; if (jm1 < 0) jm1 = j;
            int jp1 = j + 1; if (jp1 > ny - 1) jp1 = j;
            const double yfac = (jm1 == j || jp1 == j) ? 2.0 : 1.0;
            for (int i = 0; i < nx; ++i) {
                int im1 = i - 1; if (im1 < 0) im1 = i;
                int ip1 = i + 1; if (ip1 > nx - 1) ip1 = i;
                const double xfac = (im1 == i || ip1 == i) ? 2.0 : 1.0;
                auto P = [&](int a, int b, int c) { return phi[idx3(a, b, c, nx, ny)]; };
                const int64_t m = idx3(i, j, k, nx, ny);
                efield[m] = -(P(ip1, j, k) - P(im1, j, k)) / (2.0 * dx) * gam0 * xfac;
                efield[N + m] = -(P(i, jp1, k) - P(i, jm1, k)) / (2.0 * dy) * gam0 * yfac;
                efield[2 * N + m] = -(P(i, j, kp1) - P(i, j, km1)) / (2.0 * dz) / gam0 * zfac;
            }
        }
    }
}

void legacy_bfield(const double *efield, double *bfield, int64_t N, double gam0) {
    const double beta0 = std::sqrt(1 - 1 / (gam0 * gam0));
    for (int64_t m = 0; m < N; ++m) {
        bfield[m] = -efield[N + m] * beta0 / clight_core;
        bfield[N + m] = efield[m] * beta0 / clight_core;
        bfield[2 * N + m] = 0.0;
    }
}

} // namespace

extern "C" {

/* osc_freespace_solver, code/open_spacecharge_core_mod.f90:30-138 */
int orc_freespace_solver(const double *rho, double gam0, const double delta[3], double *phi,
                         double *efield, double *bfield, const int nlo[3], const int nhi[3],
                         const int npad[3], int idirectfieldcalc, int igfflag) {
    if (igfflag == 0 && idirectfieldcalc == 1) return 9; /* prints an error and returns */
    int n[3], glo[3], period[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = nhi[d] - nlo[d] + 1;
        glo[d] = nlo[d] - nhi[d];
        period[d] = (nhi[d] - nlo[d] + npad[d]) - glo[d] + 1;
        if (!orc_fft_supported(period[d])) return 3;
    }
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    const int64_t M = (int64_t)period[0] * period[1] * period[2];
    std::vector<cd> crho(M), cgrn(M);
    const int fwd[3] = {1, 1, 1}, inv[3] = {-1, -1, -1};
    const double fpei = fpei_legacy();
    if (idirectfieldcalc == 0) {
        getrhotilde(rho, crho.data(), n, period);
        getgrnfree_values(cgrn.data(), delta, gam0, glo, period, npad, 0, igfflag, 0, false);
        ccfft3d(cgrn.data(), fwd, period[0], period[1], period[2]);
        conv_extract(crho.data(), cgrn.data(), phi, n, period, inv, fpei);
        fd_efield(phi, efield, n, delta, gam0);
    }
    if (idirectfieldcalc == 1) {
        getrhotilde(rho, crho.data(), n, period);
        for (int icomp = 1; icomp <= 3; ++icomp) {
            getgrnfree_values(cgrn.data(), delta, gam0, glo, period, npad, icomp, igfflag, 0, false);
            ccfft3d(cgrn.data(), fwd, period[0], period[1], period[2]);
            conv_extract(crho.data(), cgrn.data(), efield + (icomp - 1) * N, n, period, inv, fpei);
        }
    }
    legacy_bfield(efield, bfield, N, gam0);
    return 0;
}

/* osc_cathodeimages_solver, code/open_spacecharge_core_mod.f90:905-1083.
 * Method 2 flips rho in z in place, as the reference does. */
int orc_cathodeimages_solver(double *rho, double gam0, const double umin[3], const double delta[3],
                             double *phi, double *efield, double *bfield, const int nlo[3],
                             const int nhi[3], const int npad[3], int idirectfieldcalc,
                             int igfflag, int imethod) {
    if (igfflag == 0 && idirectfieldcalc == 1) return 9;
    int n[3], glo[3], period[3], g2lo[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = nhi[d] - nlo[d] + 1;
        glo[d] = nlo[d] - nhi[d];
        period[d] = (nhi[d] - nlo[d] + npad[d]) - glo[d] + 1;
        if (!orc_fft_supported(period[d])) return 3;
    }
    /* osc_alloc_image_array (core:1095-1128) */
    g2lo[0] = glo[0];
    g2lo[1] = glo[1];
    g2lo[2] = 2 * nlo[2];
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    const int64_t M = (int64_t)period[0] * period[1] * period[2];
    std::vector<cd> crho(M), cgrn(M);
    std::vector<double> img(3 * N), phiimg;
    const int fwd[3] = {1, 1, 1}, inv[3] = {-1, -1, -1};
    const int fwd_corr[3] = {1, 1, -1}, inv_corr[3] = {-1, -1, 1};
    const double fpei = fpei_legacy();
    const double dx = delta[0], dy = delta[1], dz = delta[2];

    /* osc_getgrnimageconvcorr (core:1185-1230): z index is the actual Fortran index k */
    auto grn_convcorr = [&](int icomp) {
        int shift[3];
        for (int d = 0; d < 3; ++d) shift[d] = period[d] / 2 - (npad[d] + 1) / 2;
#pragma omp parallel for schedule(static)
        for (int kk = 0; kk < period[2]; ++kk) {
            const int kp = g2lo[2] + kk;
            const double w = kp * dz + 2.0 * umin[2] - 2.0 * nlo[2] * delta[2];
            for (int jj = 0; jj < period[1]; ++jj) {
                const int jp = g2lo[1] + fmod_pos(jj + shift[1], period[1]);
                const double v = jp * dy;
                for (int ii = 0; ii < period[0]; ++ii) {
                    const int ip = g2lo[0] + fmod_pos(ii + shift[0], period[0]);
                    const double u = ip * dx;
                    cgrn[idx3(ii, jj, kk, period[0], period[1])] =
                        cd(orc_igf_point(icomp, igfflag, u, v, w, gam0, dx, dy, dz), 0.0);
                }
            }
        }
        ccfft3d(cgrn.data(), fwd_corr, period[0], period[1], period[2]);
    };
    auto flip_rho = [&]() {
        const int khalflen = (nhi[2] - nlo[2] + 1) / 2;
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
                for (int k = 0; k < khalflen; ++k) {
                    double &a = rho[idx3(i, j, k, n[0], n[1])];
                    double &b = rho[idx3(i, j, n[2] - 1 - k, n[0], n[1])];
                    double r1 = a, r2 = b;
                    a = r2;
                    b = r1;
                }
    };
    const double umax3 = umin[2] + (nhi[2] - nlo[2]) * delta[2];
    const double zshft = umin[2] + umax3;

    if (idirectfieldcalc == 0) {
        getrhotilde(rho, crho.data(), n, period);
        getgrnfree_values(cgrn.data(), delta, gam0, glo, period, npad, 0, igfflag, 0, false);
        ccfft3d(cgrn.data(), fwd, period[0], period[1], period[2]);
        conv_extract(crho.data(), cgrn.data(), phi, n, period, inv, fpei);
        phiimg.assign(N, 0.0);
        if (imethod == 1) {
            grn_convcorr(0);
            conv_extract(crho.data(), cgrn.data(), phiimg.data(), n, period, inv_corr, fpei);
        } else {
            flip_rho();
            getrhotilde(rho, crho.data(), n, period);
            getgrnfree_values(cgrn.data(), delta, gam0, glo, period, npad, 0, igfflag, zshft, true);
            ccfft3d(cgrn.data(), fwd, period[0], period[1], period[2]);
            conv_extract(crho.data(), cgrn.data(), phiimg.data(), n, period, inv, fpei);
        }
        for (int64_t m = 0; m < N; ++m) phi[m] = phi[m] - phiimg[m];
        fd_efield(phi, efield, n, delta, gam0);
        fd_efield(phiimg.data(), img.data(), n, delta, gam0);
    }
    if (idirectfieldcalc == 1) {
        getrhotilde(rho, crho.data(), n, period);
        for (int icomp = 1; icomp <= 3; ++icomp) {
            getgrnfree_values(cgrn.data(), delta, gam0, glo, period, npad, icomp, igfflag, 0, false);
            ccfft3d(cgrn.data(), fwd, period[0], period[1], period[2]);
            conv_extract(crho.data(), cgrn.data(), efield + (icomp - 1) * N, n, period, inv, fpei);
        }
        if (imethod == 1) {
            for (int icomp = 1; icomp <= 3; ++icomp) {
                grn_convcorr(icomp);
                conv_extract(crho.data(), cgrn.data(), img.data() + (icomp - 1) * N, n, period,
                             inv_corr, fpei);
                for (int64_t m = 0; m < N; ++m)
                    efield[(icomp - 1) * N + m] = efield[(icomp - 1) * N + m] - img[(icomp - 1) * N + m];
            }
        } else {
            flip_rho();
            getrhotilde(rho, crho.data(), n, period);
            for (int icomp = 1; icomp <= 3; ++icomp) {
                getgrnfree_values(cgrn.data(), delta, gam0, glo, period, npad, icomp, igfflag,
                                  zshft, true);
                ccfft3d(cgrn.data(), fwd, period[0], period[1], period[2]);
                conv_extract(crho.data(), cgrn.data(), img.data() + (icomp - 1) * N, n, period,
                             inv, fpei);
                for (int64_t m = 0; m < N; ++m)
                    efield[(icomp - 1) * N + m] = efield[(icomp - 1) * N + m] - img[(icomp - 1) * N + m];
            }
        }
    }
    const double beta0 = std::sqrt(1 - 1 / (gam0 * gam0));
    for (int64_t m = 0; m < N; ++m) {
        bfield[m] = -(efield[N + m] + 2.0 * img[N + m]) * beta0 / clight_core;
        bfield[N + m] = (efield[m] + 2.0 * img[m]) * beta0 / clight_core;
        bfield[2 * N + m] = 0.0;
    }
    return 0;
}

/* rfun, code/open_spacecharge_core_mod.f90:723-755 */
double orc_rfun(double u, double v, double w, double gam, double a, double b, double hz, int i,
                int j) {
    const double pi = std::acos(-1.0);
    const double ainv = 1.0 / a, binv = 1.0 / b;
    const double piainv = pi * ainv, pibinv = pi * binv;
    double res = 0.0;
    for (int m = 1; m <= 5; ++m) {
        for (int n = 1; n <= 5; ++n) {
            const double kapmn = std::sqrt((m * pi * ainv) * (m * pi * ainv) + (n * pi * binv) * (n * pi * binv));
            double zfun = (std::exp(-kapmn * std::fabs(gam * w - hz)) -
                           2.0 * std::exp(-kapmn * std::fabs(gam * w)) +
                           std::exp(-kapmn * std::fabs(gam * w + hz))) /
                          (hz * hz * (kapmn * kapmn));
            if (w == 0) zfun = zfun + 2.0 / (hz * kapmn);
            int im = 1, jn = 1;
            for (int q = 0; q < m; ++q) im *= i;
            for (int q = 0; q < n; ++q) jn *= j;
            const double term = (double)(im * jn) * std::cos(m * u * piainv) *
                                std::cos(n * v * pibinv) * zfun / kapmn;
            res = res + term;
        }
    }
    res = res * 2.0 * pi * ainv * binv;
    return res;
}

/* osc_alloc_rectpipe_arrays (core:876-898) + osc_getgrnpipe (core:632-715). */
int orc_getgrnpipe(double gam, double a, double b, const double delta[3], const double umin[3],
                   const int nlo[3], const int nhi[3], const int npad[3], double *cgrn1_,
                   double *cgrn2_, double *cgrn3_, double *cgrn4_) {
    int period[3], glo[3], shift[3];
    for (int d = 0; d < 3; ++d) {
        glo[d] = nlo[d] - nhi[d];
        period[d] = 2 * (nhi[d] - nlo[d]) + 1 + npad[d];
        shift[d] = period[d] / 2 - (npad[d] + 1) / 2;
        if (!orc_fft_supported(period[d])) return 3;
    }
    const double hx = delta[0], hy = delta[1], hz = delta[2];
    const double xmin = umin[0], ymin = umin[1];
    cd *g[4] = {reinterpret_cast<cd *>(cgrn1_), reinterpret_cast<cd *>(cgrn2_),
                reinterpret_cast<cd *>(cgrn3_), reinterpret_cast<cd *>(cgrn4_)};
    const int signs[4][3] = {{1, 1, 1}, {1, -1, 1}, {-1, 1, 1}, {-1, -1, 1}};
    const int ij[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    for (int t = 0; t < 4; ++t) {
        const bool wrapx = (t == 0 || t == 1), wrapy = (t == 0 || t == 2);
#pragma omp parallel for schedule(static)
        for (int kk = 0; kk < period[2]; ++kk) {
            const int kp = glo[2] + fmod_pos(kk + shift[2], period[2]);
            const double w = kp * hz;
            for (int jj = 0; jj < period[1]; ++jj) {
                double v;
                if (wrapy) v = (glo[1] + fmod_pos(jj + shift[1], period[1])) * hy;
                else v = 2.0 * ymin + jj * hy;
                for (int ii = 0; ii < period[0]; ++ii) {
                    double u;
                    if (wrapx) u = (glo[0] + fmod_pos(ii + shift[0], period[0])) * hx;
                    else u = 2.0 * xmin + ii * hx;
                    g[t][idx3(ii, jj, kk, period[0], period[1])] =
                        cd(orc_rfun(u, v, w, gam, a, b, hz, ij[t][0], ij[t][1]), 0.0);
                }
            }
        }
        ccfft3d(g[t], signs[t], period[0], period[1], period[2]);
    }
    return 0;
}

/* osc_rectpipe_solver (core:536-624) with fftconvcorr3d (core:763-818). */
int orc_rectpipe_solver(const double *rho, const double *cgrn1, const double *cgrn2,
                        const double *cgrn3, const double *cgrn4, double gam0,
                        const double delta[3], double *phi, double *efield, double *bfield,
                        const int nlo[3], const int nhi[3], const int npad[3],
                        int idirectfieldcalc) {
    int n[3], period[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = nhi[d] - nlo[d] + 1;
        period[d] = 2 * (nhi[d] - nlo[d]) + 1 + npad[d];
    }
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    const int64_t M = (int64_t)period[0] * period[1] * period[2];
    if (idirectfieldcalc == 0) {
        std::vector<cd> crho(M), ccon(M), ctmp(M);
        getrhotilde(rho, crho.data(), n, period);
        const cd *q[4] = {reinterpret_cast<const cd *>(cgrn1), reinterpret_cast<const cd *>(cgrn2),
                          reinterpret_cast<const cd *>(cgrn3), reinterpret_cast<const cd *>(cgrn4)};
        const int isg[4][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, -1, -1}, {1, 1, -1}};
        for (int64_t m = 0; m < M; ++m) ccon[m] = crho[m] * q[0][m];
        ccfft3d(ccon.data(), isg[0], period[0], period[1], period[2]);
        for (int t = 1; t < 4; ++t) {
            for (int64_t m = 0; m < M; ++m) ctmp[m] = crho[m] * q[t][m];
            ccfft3d(ctmp.data(), isg[t], period[0], period[1], period[2]);
            if (t < 3)
                for (int64_t m = 0; m < M; ++m) ccon[m] = ccon[m] - ctmp[m];
            else
                for (int64_t m = 0; m < M; ++m) ccon[m] = ccon[m] + ctmp[m];
        }
        const double fpei = fpei_pipe();
        const double factr = 1.0 / ((1.0 * period[0]) * (1.0 * period[1]) * (1.0 * period[2])) * fpei * 1.0;
        for (int k = 0; k < n[2]; ++k)
            for (int j = 0; j < n[1]; ++j)
                for (int i = 0; i < n[0]; ++i)
                    phi[idx3(i, j, k, n[0], n[1])] = factr * ccon[idx3(i, j, k, period[0], period[1])].real();
        fd_efield(phi, efield, n, delta, gam0);
    } else {
        return 9; /* "rectpipe implementation presently requires directfieldcalc=0" */
    }
    legacy_bfield(efield, bfield, N, gam0);
    return 0;
}

} /* extern "C" */
