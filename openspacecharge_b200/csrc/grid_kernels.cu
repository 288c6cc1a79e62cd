// grid_kernels.cu -- Green-function construction (FP64) and grid elementwise kernels.
#include <algorithm>
#include "grid_kernels.cuh"
#include "osc_igf.cuh"

namespace osc {

static inline int ok() { return cudaGetLastError() == cudaSuccess ? OSC_OK : OSC_E_CUDA; }
static inline unsigned nblocks(int64_t n, int bs) {
    int64_t b = (n + bs - 1) / bs;
    return (unsigned)(b < 1 ? 1 : (b > (1 << 30) ? (1 << 30) : b));
}
#define GRID_STRIDE(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// ------------------------------------------------------------------------------------
__global__ void k_igf_corners(double *__restrict__ F, CornerArgs a) {
    const int64_t n = (int64_t)a.cdx * a.cdy * a.cdz;
    GRID_STRIDE(idx, n) {
        const int cx = (int)(idx % a.cdx);
        const int64_t r = idx / a.cdx;
        const int cy = (int)(r % a.cdy);
        const int cz = (int)(r / a.cdy);
        const double u = (a.c0x + cx) * a.dx + a.umin;
        const double v = (a.c0y + cy) * a.dy + a.vmin;
        const double w = (a.c0z + cz) * a.dz + a.wmin;
        F[idx] = igf_primitive(a.icomp, u, v, w) * a.factor;
    }
}
int launch_igf_corners(double *F, const CornerArgs &a, cudaStream_t st) {
    const int64_t n = (int64_t)a.cdx * a.cdy * a.cdz;
    k_igf_corners<<<nblocks(n, 256), 256, 0, st>>>(F, a);
    return ok();
}

__global__ void k_igf_diff_ref(const double *__restrict__ F, double2 *__restrict__ cg, int Nx, int Ny, int Nz) {
    const int64_t n = (int64_t)Nx * Ny * Nz;
    GRID_STRIDE(idx, n) {
        const int i = (int)(idx % Nx);
        const int64_t r = idx / Nx;
        const int j = (int)(r % Ny);
        const int k = (int)(r / Ny);
        double g;
        if (i < Nx - 1 && j < Ny - 1 && k < Nz - 1) {
            auto f = [&](int a, int b, int c) { return F[a + (int64_t)Nx * (b + (int64_t)Ny * c)]; };
            g = +f(i + 1, j + 1, k + 1);
            g = g - f(i, j + 1, k + 1);
            g = g - f(i + 1, j, k + 1);
            g = g - f(i + 1, j + 1, k);
            g = g - f(i, j, k);
            g = g + f(i, j, k + 1);
            g = g + f(i, j + 1, k);
            g = g + f(i + 1, j, k);
        } else {
            g = F[idx];
        }
        cg[idx] = make_double2(g, 0.0);
    }
}
int launch_igf_diff_ref(const double *F, double2 *cg, int Nx, int Ny, int Nz, cudaStream_t st) {
    k_igf_diff_ref<<<nblocks((int64_t)Nx * Ny * Nz, 256), 256, 0, st>>>(F, cg, Nx, Ny, Nz);
    return ok();
}

// displacement of doubled-grid index p (0..2n-1) in the centred layout; flag p == n
__device__ __forceinline__ int disp_of(int p, int n, bool &zero) {
    zero = (p == n);
    return p < n ? p : p - 2 * n;
}

__global__ void k_green_center(const double *__restrict__ F, double2 *__restrict__ cg, CenterArgs a) {
    const int Nx = 2 * a.nx, Ny = 2 * a.ny, Nz = 2 * a.nz;
    const int64_t n = (int64_t)Nx * Ny * Nz;
    GRID_STRIDE(idx, n) {
        const int px = (int)(idx % Nx);
        const int64_t r = idx / Nx;
        const int py = (int)(r % Ny);
        const int pz = (int)(r / Ny);
        bool zx, zy, zz;
        int ax = disp_of(px, a.nx, zx), ay = disp_of(py, a.ny, zy), az = disp_of(pz, a.nz, zz);
        double g = 0.0;
        if (!(zx || zy || zz)) {
            bool neg = false;
            if (a.symx && ax < 0) { ax = -ax; neg ^= (a.parx < 0); }
            if (a.symy && ay < 0) { ay = -ay; neg ^= (a.pary < 0); }
            if (a.symz && az < 0) { az = -az; neg ^= (a.parz < 0); }
            // corner indices of cell a: a+n-1 and a+n, relative to the evaluated block
            const int i = ax + a.nx - 1 - a.c0x, j = ay + a.ny - 1 - a.c0y, k = az + a.nz - 1 - a.c0z;
            auto f = [&](int p, int q, int s) { return F[p + (int64_t)a.cdx * (q + (int64_t)a.cdy * s)]; };
            g = +f(i + 1, j + 1, k + 1);
            g = g - f(i, j + 1, k + 1);
            g = g - f(i + 1, j, k + 1);
            g = g - f(i + 1, j + 1, k);
            g = g - f(i, j, k);
            g = g + f(i, j, k + 1);
            g = g + f(i, j + 1, k);
            g = g + f(i + 1, j, k);
            if (neg) g = -g;
        }
        cg[idx] = make_double2(g, 0.0);
    }
}
int launch_green_center(const double *F, double2 *cg, const CenterArgs &a, cudaStream_t st) {
    const int64_t n = (int64_t)8 * a.nx * a.ny * a.nz;
    k_green_center<<<nblocks(n, 256), 256, 0, st>>>(F, cg, a);
    return ok();
}

// Octant of the centred kernel for all-symmetric geometries: h[c][b][a] = g at displacement
// (a, b, c) >= 0, the 8-corner difference of the cell whose corners are a, a+1 (the corner
// block starts at index n-1 of the doubled grid, so cell a uses corners a and a+1).
template <typename TH>
__global__ void k_green_octant(const double *__restrict__ F, TH *__restrict__ h, int nx, int ny, int nz) {
    const int cdx = nx + 1, cdy = ny + 1;
    const int n = nx * ny * nz;  // one member's octant (< 2^31 nodes)
    F += blockIdx.y * ((int64_t)cdx * cdy * (nz + 1));  // batch member
    h += blockIdx.y * (int64_t)n;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        const int i = idx % nx, r = idx / nx;
        const int j = r % ny, k = r / ny;
        const double *f0 = F + i + cdx * (j + cdy * k);
        const int sy = cdx, sz = cdx * cdy;
        double g = +f0[1 + sy + sz];
        g = g - f0[sy + sz];
        g = g - f0[1 + sz];
        g = g - f0[1 + sy];
        g = g - f0[0];
        g = g + f0[sz];
        g = g + f0[sy];
        g = g + f0[1];
        h[idx] = (TH)g;
    }
}
template <typename TH>
int launch_green_octant(const double *F, TH *h, int nx, int ny, int nz, int nbatch, cudaStream_t st) {
    const dim3 grid(nblocks((int64_t)nx * ny * nz, 256), (unsigned)nbatch);
    k_green_octant<TH><<<grid, 256, 0, st>>>(F, h, nx, ny, nz);
    return ok();
}
template int launch_green_octant<double>(const double *, double *, int, int, int, int, cudaStream_t);
template int launch_green_octant<float>(const double *, float *, int, int, int, int, cudaStream_t);

// Corner blocks of several geometries: member blockIdx.y uses args[blockIdx.y] and writes
// F + blockIdx.y * fstride.
__global__ void k_igf_corners_batch(double *__restrict__ F, const CornerArgs *__restrict__ args, int64_t fstride) {
    const CornerArgs a = args[blockIdx.y];
    F += blockIdx.y * fstride;
    const int64_t n = (int64_t)a.cdx * a.cdy * a.cdz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    auto at = [&](int64_t idx) {
        const int cx = (int)(idx % a.cdx);
        const int64_t r = idx / a.cdx;
        const int cy = (int)(r % a.cdy);
        const int cz = (int)(r / a.cdy);
        const double u = (a.c0x + cx) * a.dx + a.umin;
        const double v = (a.c0y + cy) * a.dy + a.vmin;
        const double w = (a.c0z + cz) * a.dz + a.wmin;
        return igf_primitive(a.icomp, u, v, w) * a.factor;
    };
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 2 * stride) {
        const int64_t i1 = i0 + stride;  // two points per thread and trip, as k_igf_corners_set
        const double f0 = at(i0);
        const double f1 = i1 < n ? at(i1) : 0.0;
        F[i0] = f0;
        if (i1 < n) F[i1] = f1;
    }
}
__global__ void k_igf_corners_set(double *__restrict__ F, CornerSet s, int64_t fstride) {
    const CornerArgs a = s.a[blockIdx.y];
    F += blockIdx.y * fstride;
    const int64_t n = (int64_t)a.cdx * a.cdy * a.cdz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    auto at = [&](int64_t idx) {
        const int cx = (int)(idx % a.cdx);
        const int64_t r = idx / a.cdx;
        const int cy = (int)(r % a.cdy);
        const int cz = (int)(r / a.cdy);
        const double u = (a.c0x + cx) * a.dx + a.umin;
        const double v = (a.c0y + cy) * a.dy + a.vmin;
        const double w = (a.c0z + cz) * a.dz + a.wmin;
        return igf_primitive(a.icomp, u, v, w) * a.factor;
    };
    // two points per thread and trip: the two dependency chains of log/atan evaluations
    // interleave
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 2 * stride) {
        const int64_t i1 = i0 + stride;
        const double f0 = at(i0);
        const double f1 = i1 < n ? at(i1) : 0.0;
        F[i0] = f0;
        if (i1 < n) F[i1] = f1;
    }
}
int launch_igf_corners_set(double *F, const CornerSet &s, int64_t fstride, cudaStream_t st) {
    if (s.n < 1 || s.n > 4) return 1;
    int64_t npts = 0;
    for (int i = 0; i < s.n; ++i) npts = std::max(npts, (int64_t)s.a[i].cdx * s.a[i].cdy * s.a[i].cdz);
    const dim3 grid(nblocks((npts + 1) / 2, 256), (unsigned)s.n);  // two points per thread
    k_igf_corners_set<<<grid, 256, 0, st>>>(F, s, fstride);
    return ok();
}

int launch_igf_corners_batch(double *F, const CornerArgs *args_dev, int nbatch, int64_t fstride, int64_t npts,
                             cudaStream_t st) {
    const dim3 grid(nblocks((npts + 1) / 2, 256), (unsigned)nbatch);  // two points per thread
    k_igf_corners_batch<<<grid, 256, 0, st>>>(F, args_dev, fstride);
    return ok();
}

template <typename T>
__global__ void k_green_extract(const double2 *__restrict__ ghat, void *out, int nx, int Nx, int Ny,
                                int dimy, int dimz, int real_valued, int imag_unit, double scale, int zpitch,
                                int fold_mul, int Nz) {
    const int nxh = nx + 1;
    const int64_t n = (int64_t)nxh * dimy * (zpitch > 0 ? zpitch : dimz);
    GRID_STRIDE(idx, n) {
        int kx, ky, kz;
        if (zpitch > 0) {  // [ky][kx][kz], columns zpitch apart
            kz = (int)(idx % zpitch);
            const int64_t r = idx / zpitch;
            kx = (int)(r % nxh);
            ky = (int)(r / nxh);
        } else {  // [kz][ky][kx]
            kx = (int)(idx % nxh);
            const int64_t r = idx / nxh;
            ky = (int)(r % dimy);
            kz = (int)(r / dimy);
        }
        double2 v = make_double2(0.0, 0.0);
        if (kz < dimz) v = ghat[kx + (int64_t)Nx * (ky + (int64_t)Ny * kz)];
        if (fold_mul >= 0 && kz < dimz) {
            // times -exp(2 pi i m kz / Nz), the phase of the image charge's z flip
            const int64_t ph = ((int64_t)fold_mul * kz) % Nz;
            double sn, cs;
            sincospi(2.0 * (double)ph / (double)Nz, &sn, &cs);
            v = make_double2(-(v.x * cs - v.y * sn), -(v.x * sn + v.y * cs));
        }
        if (real_valued) reinterpret_cast<T *>(out)[idx] = (T)((imag_unit ? v.y : v.x) * scale);
        else reinterpret_cast<cplx<T> *>(out)[idx] = mk<T>((T)(v.x * scale), (T)(v.y * scale));
    }
}
template <typename T>
int launch_green_extract(const double2 *ghat, void *out, int nx, int Nx, int Ny, int dimy, int dimz,
                         int real_valued, int imag_unit, double scale, int zpitch, int fold_mul, int Nz,
                         cudaStream_t st) {
    const int64_t n = (int64_t)(nx + 1) * dimy * (zpitch > 0 ? zpitch : dimz);
    k_green_extract<T><<<nblocks(n, 256), 256, 0, st>>>(ghat, out, nx, Nx, Ny, dimy, dimz, real_valued,
                                                        imag_unit, scale, zpitch, fold_mul, Nz);
    return ok();
}
template int launch_green_extract<float>(const double2 *, void *, int, int, int, int, int, int, int, double, int,
                                         int, int, cudaStream_t);
template int launch_green_extract<double>(const double2 *, void *, int, int, int, int, int, int, int, double, int,
                                          int, int, cudaStream_t);

// ------------------------------------------------------------------------------------
__global__ void k_pad_rho(const double *__restrict__ rho, double2 *__restrict__ crho, int nx, int ny, int nz,
                          int Nx, int Ny, int Nz, double sign, int flipz) {
    const int64_t n = (int64_t)Nx * Ny * Nz;
    GRID_STRIDE(idx, n) {
        const int i = (int)(idx % Nx);
        const int64_t r = idx / Nx;
        const int j = (int)(r % Ny);
        const int k = (int)(r / Ny);
        double v = 0.0;
        if (i < nx && j < ny && k < nz) {
            const int ks = flipz ? nz - 1 - k : k;
            v = sign * rho[i + (int64_t)nx * (j + (int64_t)ny * ks)];
        }
        crho[idx] = make_double2(v, 0.0);
    }
}
int launch_pad_rho(const double *rho, double2 *crho, int nx, int ny, int nz, int Nx, int Ny, int Nz,
                   double sign, int flipz, cudaStream_t st) {
    k_pad_rho<<<nblocks((int64_t)Nx * Ny * Nz, 256), 256, 0, st>>>(rho, crho, nx, ny, nz, Nx, Ny, Nz, sign, flipz);
    return ok();
}

__global__ void k_cmul(double2 *__restrict__ a, const double2 *__restrict__ b, int64_t M) {
    GRID_STRIDE(i, M) {
        const double2 x = b[i], y = a[i];  // a = b*a (cgrn = crho*cgrn)
        a[i] = make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
    }
}
int launch_cmul(double2 *a, const double2 *b, int64_t M, cudaStream_t st) {
    k_cmul<<<nblocks(M, 256), 256, 0, st>>>(a, b, M);
    return ok();
}

__global__ void k_extract_re(const double2 *__restrict__ c, int Nx, int Ny, int si, int sj, int sk, int nx,
                             int ny, int nz, double factr, double *__restrict__ out, int accumulate) {
    const int64_t n = (int64_t)nx * ny * nz;
    GRID_STRIDE(idx, n) {
        const int i = (int)(idx % nx);
        const int64_t r = idx / nx;
        const int j = (int)(r % ny);
        const int k = (int)(r / ny);
        const double v = factr * c[(i + si) + (int64_t)Nx * ((j + sj) + (int64_t)Ny * (k + sk))].x;
        out[idx] = accumulate ? out[idx] + v : v;
    }
}
int launch_extract_re(const double2 *c, int Nx, int Ny, int si, int sj, int sk, int nx, int ny, int nz,
                      double factr, double *out, int accumulate, cudaStream_t st) {
    k_extract_re<<<nblocks((int64_t)nx * ny * nz, 256), 256, 0, st>>>(c, Nx, Ny, si, sj, sk, nx, ny, nz, factr,
                                                                      out, accumulate);
    return ok();
}

__global__ void k_bfield(const double *__restrict__ E, double *__restrict__ B, int64_t N, double coef,
                         int accumulate) {
    GRID_STRIDE(m, N) {
        const double bx = -coef * E[N + m], by = coef * E[m];
        if (accumulate) {
            B[m] = B[m] + bx;
            B[N + m] = B[N + m] + by;
        } else {
            B[m] = bx;
            B[N + m] = by;
            B[2 * N + m] = 0.0;
        }
    }
}
int launch_bfield(const double *E, double *B, int64_t N, double coef, int accumulate, cudaStream_t st) {
    k_bfield<<<nblocks(N, 256), 256, 0, st>>>(E, B, N, coef, accumulate);
    return ok();
}

__global__ void k_axpy(double *y, const double *x, double a, int64_t n) {
    GRID_STRIDE(i, n) y[i] = y[i] + a * x[i];
}
int launch_axpy(double *y, const double *x, double a, int64_t n, cudaStream_t st) {
    k_axpy<<<nblocks(n, 256), 256, 0, st>>>(y, x, a, n);
    return ok();
}
__global__ void k_scale(double *y, double a, int64_t n) {
    GRID_STRIDE(i, n) y[i] = y[i] * a;
}
int launch_scale(double *y, double a, int64_t n, cudaStream_t st) {
    k_scale<<<nblocks(n, 256), 256, 0, st>>>(y, a, n);
    return ok();
}

__global__ void k_fd_efield(const double *__restrict__ phi, double *__restrict__ E, int nx, int ny, int nz,
                            double dx, double dy, double dz, double gam0) {
    const int64_t N = (int64_t)nx * ny * nz;
    GRID_STRIDE(m, N) {
        const int i = (int)(m % nx);
        const int64_t r = m / nx;
        const int j = (int)(r % ny);
        const int k = (int)(r / ny);
        int km1 = k - 1; if (km1 < 0) km1 = k;
        int kp1 = k + 1; if (kp1 > nz - 1) kp1 = k;
        const double zfac = (km1 == k || kp1 == k) ? 2.0 : 1.0;
        int jm1 = j - 1; if (jm1 < 0) jm1 = j;
        int jp1 = j + 1; if (jp1 > ny - 1) jp1 = j;
        const double yfac = (jm1 == j || jp1 == j) ? 2.0 : 1.0;
        int im1 = i - 1; if (im1 < 0) im1 = i;
        int ip1 = i + 1; if (ip1 > nx - 1) ip1 = i;
        const double xfac = (im1 == i || ip1 == i) ? 2.0 : 1.0;
        auto P = [&](int a, int b, int c) { return phi[a + (int64_t)nx * (b + (int64_t)ny * c)]; };
        E[m] = -(P(ip1, j, k) - P(im1, j, k)) / (2.0 * dx) * gam0 * xfac;
        E[N + m] = -(P(i, jp1, k) - P(i, jm1, k)) / (2.0 * dy) * gam0 * yfac;
        E[2 * N + m] = -(P(i, j, kp1) - P(i, j, km1)) / (2.0 * dz) / gam0 * zfac;
    }
}
int launch_fd_efield(const double *phi, double *E, int nx, int ny, int nz, double dx, double dy, double dz,
                     double gam0, cudaStream_t st) {
    k_fd_efield<<<nblocks((int64_t)nx * ny * nz, 256), 256, 0, st>>>(phi, E, nx, ny, nz, dx, dy, dz, gam0);
    return ok();
}

// The same finite differences written as the x-pair grid read by the FP32 gather: node m
// holds (Ex,Ey,Ez,0) of m and of m+1 (0 past the row end), each value the FP32 rounding of
// the FP64 difference, as the planes and their repacking into pairs give.
__global__ void k_fd_efield_pairs(const double *__restrict__ phi, float4 *__restrict__ e8, int nx, int ny, int nz,
                                  double dx, double dy, double dz, double gam0) {
    const int64_t N = (int64_t)nx * ny * nz;
    GRID_STRIDE(m, N) {
        const int i = (int)(m % nx);
        const int64_t r = m / nx;
        const int j = (int)(r % ny);
        const int k = (int)(r / ny);
        int km1 = k - 1; if (km1 < 0) km1 = k;
        int kp1 = k + 1; if (kp1 > nz - 1) kp1 = k;
        const double zfac = (km1 == k || kp1 == k) ? 2.0 : 1.0;
        int jm1 = j - 1; if (jm1 < 0) jm1 = j;
        int jp1 = j + 1; if (jp1 > ny - 1) jp1 = j;
        const double yfac = (jm1 == j || jp1 == j) ? 2.0 : 1.0;
        int im1 = i - 1; if (im1 < 0) im1 = i;
        int ip1 = i + 1; if (ip1 > nx - 1) ip1 = i;
        const double xfac = (im1 == i || ip1 == i) ? 2.0 : 1.0;
        auto P = [&](int a, int b, int c) { return phi[a + (int64_t)nx * (b + (int64_t)ny * c)]; };
        const double ex = -(P(ip1, j, k) - P(im1, j, k)) / (2.0 * dx) * gam0 * xfac;
        const double ey = -(P(i, jp1, k) - P(i, jm1, k)) / (2.0 * dy) * gam0 * yfac;
        const double ez = -(P(i, j, kp1) - P(i, j, km1)) / (2.0 * dz) / gam0 * zfac;
        const float4 v = make_float4((float)ex, (float)ey, (float)ez, 0.f);
        e8[2 * m] = v;
        if (i > 0) e8[2 * (m - 1) + 1] = v;
        if (i == nx - 1) e8[2 * m + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}
int launch_fd_efield_pairs(const double *phi, float *e8, int nx, int ny, int nz, double dx, double dy, double dz,
                           double gam0, cudaStream_t st) {
    k_fd_efield_pairs<<<nblocks((int64_t)nx * ny * nz, 256), 256, 0, st>>>(phi, reinterpret_cast<float4 *>(e8), nx, ny,
                                                                           nz, dx, dy, dz, gam0);
    return ok();
}

__global__ void k_flip_z(double *a, int nx, int ny, int nz) {
    const int64_t plane = (int64_t)nx * ny;
    const int64_t n = plane * (nz / 2);
    GRID_STRIDE(m, n) {
        const int64_t xy = m % plane;
        const int k = (int)(m / plane);
        double *p = a + xy + plane * k, *q = a + xy + plane * (nz - 1 - k);
        const double t = *p;
        *p = *q;
        *q = t;
    }
}
int launch_flip_z(double *a, int nx, int ny, int nz, cudaStream_t st) {
    k_flip_z<<<nblocks((int64_t)nx * ny * (nz / 2), 256), 256, 0, st>>>(a, nx, ny, nz);
    return ok();
}

template <typename T>
__global__ void k_vec4_to_planes(const vec4<T> *__restrict__ E4, double *__restrict__ E, int64_t N) {
    GRID_STRIDE(m, N) {
        const vec4<T> v = E4[m];
        E[m] = (double)v.x;
        E[N + m] = (double)v.y;
        E[2 * N + m] = (double)v.z;
    }
}
template <typename T> int launch_vec4_to_planes(const void *E4, double *E, int64_t N, cudaStream_t st) {
    k_vec4_to_planes<T><<<nblocks(N, 256), 256, 0, st>>>(reinterpret_cast<const vec4<T> *>(E4), E, N);
    return ok();
}
template int launch_vec4_to_planes<float>(const void *, double *, int64_t, cudaStream_t);
template int launch_vec4_to_planes<double>(const void *, double *, int64_t, cudaStream_t);

__global__ void k_f32_to_f64(const float *a, double *b, int64_t n) { GRID_STRIDE(i, n) b[i] = (double)a[i]; }
__global__ void k_f64_to_f32(const double *a, float *b, int64_t n) { GRID_STRIDE(i, n) b[i] = (float)a[i]; }
int launch_f32_to_f64(const float *a, double *b, int64_t n, cudaStream_t st) {
    k_f32_to_f64<<<nblocks(n, 256), 256, 0, st>>>(a, b, n);
    return ok();
}
int launch_f64_to_f32(const double *a, float *b, int64_t n, cudaStream_t st) {
    k_f64_to_f32<<<nblocks(n, 256), 256, 0, st>>>(a, b, n);
    return ok();
}

// ------------------------------------------------------------------------------------
__global__ void k_legacy_green(double2 *__restrict__ cg, LegacyGrnArgs a) {
    const int64_t n = (int64_t)a.px * a.py * a.pz;
    GRID_STRIDE(idx, n) {
        const int ii = (int)(idx % a.px);
        const int64_t r = idx / a.px;
        const int jj = (int)(r % a.py);
        const int kk = (int)(r / a.py);
        const int ip = a.glox + (ii + a.shx) % a.px;
        const int jp = a.gloy + (jj + a.shy) % a.py;
        double w;
        if (a.wrapz) w = (a.gloz + (kk + a.shz) % a.pz) * a.dz + a.w_off;
        else w = (a.gloz + kk) * a.dz + a.w_off;
        const double u = ip * a.dx, v = jp * a.dy;
        cg[idx] = make_double2(igf_point(a.icomp, a.igfflag, u, v, w, a.gam, a.dx, a.dy, a.dz), 0.0);
    }
}
int launch_legacy_green(double2 *cg, const LegacyGrnArgs &a, cudaStream_t st) {
    k_legacy_green<<<nblocks((int64_t)a.px * a.py * a.pz, 256), 256, 0, st>>>(cg, a);
    return ok();
}

// rfun (core:723-755) as sum over 5x5 modes of ij*cos_u*cos_v*zfun/kappa, with the per-axis
// factors tabulated first (they depend on one coordinate each).
__global__ void k_pipe_tables(double *cu, double *cv, double *zf, double *kap, PipeGrnArgs a) {
    const double pi = 3.14159265358979323846264338327950288;
    const double ainv = 1.0 / a.a, binv = 1.0 / a.b;
    const double piainv = pi * ainv, pibinv = pi * binv;
    const int ntot = 5 * a.px + 5 * a.py + 25 * a.pz + 25;
    GRID_STRIDE(t, ntot) {
        int q = (int)t;
        if (q < 5 * a.px) {
            const int m = q / a.px + 1, ii = q % a.px;
            const double u = a.wrapx ? (a.glox + (ii + a.shx) % a.px) * a.hx : 2.0 * a.xmin + ii * a.hx;
            cu[q] = cos(m * u * piainv);
            continue;
        }
        q -= 5 * a.px;
        if (q < 5 * a.py) {
            const int n = q / a.py + 1, jj = q % a.py;
            const double v = a.wrapy ? (a.gloy + (jj + a.shy) % a.py) * a.hy : 2.0 * a.ymin + jj * a.hy;
            cv[q] = cos(n * v * pibinv);
            continue;
        }
        q -= 5 * a.py;
        if (q < 25 * a.pz) {
            const int mn = q / a.pz, kk = q % a.pz;
            const int m = mn / 5 + 1, n = mn % 5 + 1;
            const double kapmn = sqrt((m * pi * ainv) * (m * pi * ainv) + (n * pi * binv) * (n * pi * binv));
            const double w = (a.gloz + (kk + a.shz) % a.pz) * a.hz;
            const double gam = a.gam, hz = a.hz;
            double zfun = (exp(-kapmn * fabs(gam * w - hz)) - 2.0 * exp(-kapmn * fabs(gam * w)) +
                           exp(-kapmn * fabs(gam * w + hz))) /
                          (hz * hz * (kapmn * kapmn));
            if (w == 0) zfun = zfun + 2.0 / (hz * kapmn);
            zf[q] = zfun;
            continue;
        }
        q -= 25 * a.pz;
        const int m = q / 5 + 1, n = q % 5 + 1;
        kap[q] = sqrt((m * pi * ainv) * (m * pi * ainv) + (n * pi * binv) * (n * pi * binv));
    }
}

__global__ void k_pipe_green(double2 *__restrict__ cg, const double *__restrict__ cu, const double *__restrict__ cv,
                             const double *__restrict__ zf, const double *__restrict__ kap, PipeGrnArgs a) {
    const double pi = 3.14159265358979323846264338327950288;
    const double norm_a = 1.0 / a.a, norm_b = 1.0 / a.b;
    const int64_t n = (int64_t)a.px * a.py * a.pz;
    GRID_STRIDE(idx, n) {
        const int ii = (int)(idx % a.px);
        const int64_t r = idx / a.px;
        const int jj = (int)(r % a.py);
        const int kk = (int)(r / a.py);
        double res = 0.0;
#pragma unroll
        for (int m = 1; m <= 5; ++m) {
            const int im = (a.isg < 0 && (m & 1)) ? -1 : 1;
#pragma unroll
            for (int nn = 1; nn <= 5; ++nn) {
                const int jn = (a.jsg < 0 && (nn & 1)) ? -1 : 1;
                const int mn = (m - 1) * 5 + (nn - 1);
                const double term = (double)(im * jn) * cu[(m - 1) * a.px + ii] * cv[(nn - 1) * a.py + jj] *
                                    zf[mn * a.pz + kk] / kap[mn];
                res = res + term;
            }
        }
        res = res * 2.0 * pi * norm_a * norm_b;
        cg[idx] = make_double2(res, 0.0);
    }
}
int pipe_green_scratch_doubles(const PipeGrnArgs &a) { return 5 * a.px + 5 * a.py + 25 * a.pz + 25; }
int launch_pipe_green(double2 *cg, double *scratch, const PipeGrnArgs &a, cudaStream_t st) {
    double *cu = scratch, *cv = cu + 5 * a.px, *zf = cv + 5 * a.py, *kap = zf + 25 * a.pz;
    k_pipe_tables<<<nblocks(pipe_green_scratch_doubles(a), 256), 256, 0, st>>>(cu, cv, zf, kap, a);
    int rc = ok();
    if (rc) return rc;
    k_pipe_green<<<nblocks((int64_t)a.px * a.py * a.pz, 256), 256, 0, st>>>(cg, cu, cv, zf, kap, a);
    return ok();
}

}  // namespace osc
