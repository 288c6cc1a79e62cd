// particle_kernels.cu -- CIC deposition, CIC interpolation, bounding box and charge sum.
#include "particle_kernels.cuh"

namespace osc {

static inline int ok() { return cudaGetLastError() == cudaSuccess ? OSC_OK : OSC_E_CUDA; }
static inline unsigned nblocks(int64_t n, int bs, int64_t cap = (1 << 20)) {
    int64_t b = (n + bs - 1) / bs;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}
#define GRID_STRIDE(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// Deposits add without reading the old value back: reductions (red), not atomics that
// return a value, so a thread never waits for the L2's answer.
__device__ __forceinline__ void red_add(float *p, float v) {
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void red_add(double *p, double v) {
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void red_add(unsigned long long *p, unsigned long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_add(float4 *p, float4 v) {
    asm volatile("red.global.add.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}
__device__ __forceinline__ void atomic_add_t(float *p, double v, double) { red_add(p, (float)v); }
__device__ __forceinline__ void atomic_add_t(double *p, double v, double) { red_add(p, v); }
// Fixed point: two's-complement addition of the rounded contribution (exact, associative).
__device__ __forceinline__ void atomic_add_t(unsigned long long *p, double v, double scale) {
    red_add(p, (unsigned long long)__double2ll_rn(v * scale));
}

// Warp-aggregated counter increment.
__device__ __forceinline__ void count_one(unsigned long long *c, bool pred) {
    const unsigned mask = __ballot_sync(__activemask(), pred);
    if (pred && (threadIdx.x & 31) == __ffs(mask) - 1) atomicAdd(c, (unsigned long long)__popc(mask));
}

template <typename TA>
__global__ void __launch_bounds__(256) k_deposit(DepositArgs a, TA *__restrict__ rho,
                                                 unsigned long long *__restrict__ counters) {
    const int64_t plane = (int64_t)a.nx * a.ny;
    GRID_STRIDE(m, a.np) {
        bool skip = false, outside = false, nonfinite = false;
        if (a.lost && a.lost[m] != 0.0) skip = true;
        const double xm = a.x[m], ym = a.y[m], zm = a.z[m];
        if (!skip && a.check_finite && !(isfinite(xm) && isfinite(ym) && isfinite(zm))) {
            nonfinite = true;
            skip = true;
        }
        double fx, fy, fz, ab, de, gh;
        int i = 0, j = 0, k = 0;
        if (!skip) {
            if (a.mode == 0) {
                // the 2x2x2 stencil must lie inside the array
                CicCell cc = {0, 0, 0, 0.0, 0.0, 0.0};
                outside = cic_cell_mode0(a, xm, ym, zm, cc) != 0;
                ab = cc.ab;
                de = cc.de;
                gh = cc.gh;
                fx = cc.i + a.nlo[0];
                fy = cc.j + a.nlo[1];
                fz = cc.k + a.nlo[2];
            } else {
                fx = floor(__dmul_rn(xm - a.xmin, a.dxi) + a.nlogbl[0]);
                fy = floor(__dmul_rn(ym - a.ymin, a.dyi) + a.nlogbl[1]);
                fz = floor(__dmul_rn(zm - a.zmin, a.dzi) + a.nlogbl[2]);
                ab = ((a.xmin - xm) + (fx - a.nlogbl[0] + 1) * a.dx) * a.dxi;
                de = ((a.ymin - ym) + (fy - a.nlogbl[1] + 1) * a.dy) * a.dyi;
                gh = ((a.zmin - zm) + (fz - a.nlogbl[2] + 1) * a.dz) * a.dzi;
                // reference check (ip < ilo or ip > size) and the array bound of ip+1
                outside = !(fx >= a.nlo[0] && fx <= a.nx && fy >= a.nlo[1] && fy <= a.ny && fz >= a.nlo[2] &&
                            fz <= a.nz) ||
                          !(fx - a.nlo[0] + 1 < a.nx && fy - a.nlo[1] + 1 < a.ny && fz - a.nlo[2] + 1 < a.nz);
            }
            if (!outside) {
                i = (int)fx - a.nlo[0];
                j = (int)fy - a.nlo[1];
                k = (int)fz - a.nlo[2];
            }
        }
        count_one(&counters[0], !skip && outside);
        count_one(&counters[1], nonfinite);
        if (skip || outside) continue;
        const double c = a.mode == 0 ? (a.q ? a.q[m] : a.charge1) : 1.0;
        const double omab = 1. - ab, omde = 1. - de, omgh = 1. - gh;
        TA *r0 = rho + i + (int64_t)a.nx * j + plane * k;
        atomic_add_t(r0, ab * de * gh * c, a.fx_scale);
        atomic_add_t(r0 + a.nx, ab * omde * gh * c, a.fx_scale);
        atomic_add_t(r0 + a.nx + plane, ab * omde * omgh * c, a.fx_scale);
        atomic_add_t(r0 + plane, ab * de * omgh * c, a.fx_scale);
        atomic_add_t(r0 + 1 + plane, omab * de * omgh * c, a.fx_scale);
        atomic_add_t(r0 + 1 + a.nx + plane, omab * omde * omgh * c, a.fx_scale);
        atomic_add_t(r0 + 1 + a.nx, omab * omde * gh * c, a.fx_scale);
        atomic_add_t(r0 + 1, omab * de * gh * c, a.fx_scale);
    }
}

template <typename TA>
int launch_deposit(const DepositArgs &a, TA *rho, unsigned long long *counters, cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    k_deposit<TA><<<nblocks(a.np, 256, 148 * 64), 256, 0, st>>>(a, rho, counters);
    return ok();
}
template int launch_deposit<float>(const DepositArgs &, float *, unsigned long long *, cudaStream_t);
template int launch_deposit<double>(const DepositArgs &, double *, unsigned long long *, cudaStream_t);
template int launch_deposit<unsigned long long>(const DepositArgs &, unsigned long long *, unsigned long long *,
                                                cudaStream_t);

template <typename TO>
__global__ void k_fixed_to_real(const unsigned long long *__restrict__ acc, TO *__restrict__ out, double f, int64_t n) {
    GRID_STRIDE(i, n) out[i] = (TO)((double)(long long)acc[i] * f);
}
template <typename TO>
int launch_fixed_to_real(const unsigned long long *acc, TO *out, double fx_scale, double mult, int64_t n,
                         cudaStream_t st) {
    k_fixed_to_real<TO><<<nblocks(n, 256), 256, 0, st>>>(acc, out, mult / fx_scale, n);
    return ok();
}
template int launch_fixed_to_real<float>(const unsigned long long *, float *, double, double, int64_t, cudaStream_t);
template int launch_fixed_to_real<double>(const unsigned long long *, double *, double, double, int64_t, cudaStream_t);

// ------------------------------------------------------------------------------------
// FP32 deposit in two passes.  Pass 1 adds each particle to a quad grid: node (i,j,k) holds
// the contributions to the four nodes (i,j), (i+1,j), (i,j+1), (i+1,j+1) of plane k that
// come from the cells whose lowest corner is (i,j,k) or (i,j,k-1), so a particle costs two
// float4 atomics (planes k and k+1) on a 16-byte-per-node grid that stays in L2.  The
// weights are the factors of deposit_particles (code/open_spacecharge_mod.f90:274-281).
// Pass 2 sums every node's four quad slots in a fixed order.
// One particle of the quad deposit: 0 deposited, 1 outside the mesh, 2 non-finite.
__device__ __forceinline__ int quad_one(const DepositArgs &a, float4 *__restrict__ quad, int64_t plane, double xm,
                                        double ym, double zm, double c) {
    CicCell cc = {0, 0, 0, 0.0, 0.0, 0.0};
    const int st = cic_cell_mode0(a, xm, ym, zm, cc);
    if (st) return st;
    const double ab = cc.ab, de = cc.de, gh = cc.gh;
    const double omab = 1. - ab, omde = 1. - de, omgh = 1. - gh;
    const double lo = gh * c, hi = omgh * c;
    const int i = cc.i, j = cc.j, k = cc.k;
    float4 *q0 = quad + ((int64_t)i + (int64_t)a.nx * j + plane * k);
    red_add(q0, make_float4((float)(ab * de * lo), (float)(omab * de * lo), (float)(ab * omde * lo),
                              (float)(omab * omde * lo)));
    red_add(q0 + plane, make_float4((float)(ab * de * hi), (float)(omab * de * hi), (float)(ab * omde * hi),
                                      (float)(omab * omde * hi)));
    return 0;
}

__global__ void __launch_bounds__(256) k_deposit_quad(DepositArgs a, float4 *__restrict__ quad,
                                                      unsigned long long *__restrict__ counters) {
    const int64_t plane = (int64_t)a.nx * a.ny;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // the next particle's coordinates and charge are loaded before this one's atomics
    double xn = 0, yn = 0, zn = 0, qn = a.charge1;
    if (m < a.np) {
        xn = __ldg(a.x + m);
        yn = __ldg(a.y + m);
        zn = __ldg(a.z + m);
        if (a.q) qn = __ldg(a.q + m);
    }
    for (; m < a.np; m += stride) {
        const double xm = xn, ym = yn, zm = zn, c = qn;
        const int64_t mn = m + stride;
        if (mn < a.np) {
            xn = __ldg(a.x + mn);
            yn = __ldg(a.y + mn);
            zn = __ldg(a.z + mn);
            if (a.q) qn = __ldg(a.q + mn);
        }
        const int st = quad_one(a, quad, plane, xm, ym, zm, c);
        count_one(&counters[0], st == 1);
        count_one(&counters[1], st == 2);
    }
}

int launch_deposit_quad(const DepositArgs &a, float *quad, unsigned long long *counters, cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    // default: one particle per thread; the autotuner may cap the grid at a.ctas CTAs per SM
    const int64_t cap = a.ctas > 0 ? 148 * (int64_t)a.ctas : (1 << 20);
    k_deposit_quad<<<nblocks(a.np, 256, cap), 256, 0, st>>>(a, reinterpret_cast<float4 *>(quad), counters);
    return ok();
}

// rho(i,j,k) = Q(i,j).x + Q(i-1,j).y + Q(i,j-1).z + Q(i-1,j-1).w of plane k, in that order.
__global__ void __launch_bounds__(256) k_quad_to_nodes(const float4 *__restrict__ quad, float *__restrict__ rho,
                                                       int nx, int ny, int64_t n) {
    GRID_STRIDE(idx, n) {
        const int i = (int)(idx % nx), j = (int)((idx / nx) % ny);
        float s = __ldg(&quad[idx].x);
        if (i > 0) s += __ldg(&quad[idx - 1].y);
        if (j > 0) s += __ldg(&quad[idx - nx].z);
        if (i > 0 && j > 0) s += __ldg(&quad[idx - nx - 1].w);
        rho[idx] = s;
    }
}

int launch_quad_to_nodes(const float *quad, float *rho, int nx, int ny, int nz, cudaStream_t st) {
    const int64_t n = (int64_t)nx * ny * nz;
    k_quad_to_nodes<<<nblocks(n, 256, 148 * 16), 256, 0, st>>>(reinterpret_cast<const float4 *>(quad), rho, nx, ny,
                                                               n);
    return ok();
}

// ------------------------------------------------------------------------------------
struct Cell {
    int i, j, k;
    double ab, de, gh;
};

__device__ __forceinline__ bool locate(const InterpArgs &a, double x, double y, double z, Cell &c) {
    const double pos[3] = {x, y, z};
    int idx[3];
    double w[3];
    bool flag = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double f = floor(__dmul_rn(pos[d] - a.min[d], a.hinv[d]) + 1);
        const double hi = (double)(a.nhi[d] - 1);
        if (!(f >= 1.0 && f <= hi)) {  // NaN lands here too
            flag = true;
            f = (f < 1.0 || f != f) ? 1.0 : hi;
        }
        const double lo_arr = (double)a.nlo[d];
        if (f < lo_arr) { flag = true; f = lo_arr; }
        w[d] = ((a.min[d] - pos[d]) + f * a.delta[d]) * a.hinv[d];
        idx[d] = (int)f - a.nlo[d];
    }
    c.i = idx[0]; c.j = idx[1]; c.k = idx[2];
    c.ab = w[0]; c.de = w[1]; c.gh = w[2];
    return flag;
}

template <typename T>
__device__ __forceinline__ void load_node(const vec4<T> *g, int64_t n, double &a, double &b, double &c) {
    if constexpr (sizeof(T) == 8) {  // one 256-bit read-only load per node
        double w;
        asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(w) : "l"(g + n));
    } else {
        const vec4<T> v = __ldg(g + n);
        a = (double)v.x;
        b = (double)v.y;
        c = (double)v.z;
    }
}

template <typename T, typename TO>
__global__ void __launch_bounds__(256) k_interp_vec4(InterpArgs a, const vec4<T> *__restrict__ g, TO *__restrict__ E,
                                                     unsigned long long *__restrict__ nclamp) {
    // E goes through a per-warp shared-memory stage and is stored as contiguous rows (as in
    // k_interp_pairs); the loop runs while the warp's first particle exists
    __shared__ TO stage[256 * 3];
    const int lane = threadIdx.x & 31;
    TO *ws = stage + (threadIdx.x - lane) * 3;
    const int64_t plane = (int64_t)a.nx * a.ny;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m - lane < a.np; m += stride) {
        bool fl = false;
        if (m < a.np) {
            Cell c;
            fl = locate(a, a.x[m], a.y[m], a.z[m], c);
            const int64_t n0 = c.i + (int64_t)a.nx * c.j + plane * c.k;
            const double ab = c.ab, de = c.de, gh = c.gh;
            const double omab = 1. - ab, omde = 1. - de, omgh = 1. - gh;
            const int64_t nodes[8] = {n0, n0 + a.nx, n0 + a.nx + plane, n0 + plane,
                                      n0 + 1 + plane, n0 + 1 + a.nx + plane, n0 + 1 + a.nx, n0 + 1};
            const double wts[8] = {ab * de * gh, ab * omde * gh, ab * omde * omgh, ab * de * omgh,
                                   omab * de * omgh, omab * omde * omgh, omab * omde * gh, omab * de * gh};
            double ex = 0, ey = 0, ez = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                double vx, vy, vz;
                load_node<T>(g, nodes[q], vx, vy, vz);
                ex = ex + vx * wts[q];
                ey = ey + vy * wts[q];
                ez = ez + vz * wts[q];
            }
            ws[3 * lane] = (TO)ex;
            ws[3 * lane + 1] = (TO)ey;
            ws[3 * lane + 2] = (TO)ez;
        }
        count_one(nclamp, fl);
        __syncwarp();
        const int64_t o0 = 3 * (m - lane), n3 = 3 * a.np;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const int e = 32 * t + lane;
            if (o0 + e < n3) E[o0 + e] = ws[e];
        }
        __syncwarp();
    }
}

template <typename T>
int launch_interp_vec4(const InterpArgs &a, const void *E4, double *E, unsigned long long *nclamp, cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    k_interp_vec4<T, double><<<nblocks(a.np, 256, 148 * 64), 256, 0, st>>>(a, reinterpret_cast<const vec4<T> *>(E4),
                                                                            E, nclamp);
    return ok();
}
template <typename T>
int launch_interp_vec4_any(const InterpArgs &a, const void *E4, void *E, int out_f32, unsigned long long *nclamp,
                           cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    if (out_f32)
        k_interp_vec4<T, float><<<nblocks(a.np, 256, 148 * 64), 256, 0, st>>>(
            a, reinterpret_cast<const vec4<T> *>(E4), reinterpret_cast<float *>(E), nclamp);
    else
        k_interp_vec4<T, double><<<nblocks(a.np, 256, 148 * 64), 256, 0, st>>>(
            a, reinterpret_cast<const vec4<T> *>(E4), reinterpret_cast<double *>(E), nclamp);
    return ok();
}
template int launch_interp_vec4<float>(const InterpArgs &, const void *, double *, unsigned long long *, cudaStream_t);
template int launch_interp_vec4<double>(const InterpArgs &, const void *, double *, unsigned long long *, cudaStream_t);
template int launch_interp_vec4_any<float>(const InterpArgs &, const void *, void *, int, unsigned long long *, cudaStream_t);
template int launch_interp_vec4_any<double>(const InterpArgs &, const void *, void *, int, unsigned long long *, cudaStream_t);

// Three double planes [3][N], reference order of the 8-term sum per component.
__global__ void __launch_bounds__(256) k_interp_planes(InterpArgs a, const double *__restrict__ F,
                                                       double *__restrict__ out,
                                                       unsigned long long *__restrict__ nclamp) {
    const int64_t plane = (int64_t)a.nx * a.ny;
    const int64_t N = plane * a.nz;
    GRID_STRIDE(m, a.np) {
        Cell c;
        const bool fl = locate(a, a.x[m], a.y[m], a.z[m], c);
        count_one(nclamp, fl);
        const int64_t n0 = c.i + (int64_t)a.nx * c.j + plane * c.k;
        const double ab = c.ab, de = c.de, gh = c.gh;
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
            const double *A = F + comp * N;
            double v = A[n0] * ab * de * gh;
            v = v + A[n0 + a.nx] * ab * (1. - de) * gh;
            v = v + A[n0 + a.nx + plane] * ab * (1. - de) * (1. - gh);
            v = v + A[n0 + plane] * ab * de * (1. - gh);
            v = v + A[n0 + 1 + plane] * (1. - ab) * de * (1. - gh);
            v = v + A[n0 + 1 + a.nx + plane] * (1. - ab) * (1. - de) * (1. - gh);
            v = v + A[n0 + 1 + a.nx] * (1. - ab) * (1. - de) * gh;
            v = v + A[n0 + 1] * (1. - ab) * de * gh;
            out[3 * m + comp] = v;
        }
    }
}
// One x-pair (two float4, 32 bytes, 32-byte aligned) with a single 256-bit read-only load:
// half the L1 tag lookups of two 128-bit loads for the same bytes.
__device__ __forceinline__ void ldg_pair(const float4 *p, float4 &lo, float4 &hi) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(lo.x), "=f"(lo.y), "=f"(lo.z), "=f"(lo.w), "=f"(hi.x), "=f"(hi.y), "=f"(hi.z), "=f"(hi.w)
        : "l"(p));
}

// E at a particle from the four x-pairs of its stencil (rows (j,k), (j+1,k), (j+1,k+1),
// (j,k+1), each holding nodes i and i+1), with explicit fused multiply-adds so that every
// gather kernel rounds alike.
__device__ __forceinline__ void pair_sum(const float4 (&lo)[4], const float4 (&hi)[4], double ab, double de,
                                         double gh, double &ex, double &ey, double &ez) {
    const double omab = 1. - ab, omde = 1. - de, omgh = 1. - gh;
    const double wy[4] = {de * gh, omde * gh, omde * omgh, de * omgh};
    ex = ey = ez = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double w0 = ab * wy[q], w1 = omab * wy[q];
        ex = __fma_rn((double)lo[q].x, w0, __fma_rn((double)hi[q].x, w1, ex));
        ey = __fma_rn((double)lo[q].y, w0, __fma_rn((double)hi[q].y, w1, ey));
        ez = __fma_rn((double)lo[q].z, w0, __fma_rn((double)hi[q].z, w1, ez));
    }
}

// One particle of the x-pair gather; returns true when its cell was clamped.
__device__ __forceinline__ bool interp_pair_one(const InterpArgs &a, const float4 *__restrict__ g8, int64_t plane,
                                                double xm, double ym, double zm, double *__restrict__ Eo) {
    Cell c;
    const bool fl = locate(a, xm, ym, zm, c);
    const int64_t n0 = c.i + (int64_t)a.nx * c.j + plane * c.k;
    // (j,k), (j+1,k), (j+1,k+1), (j,k+1) rows; each pair = nodes i and i+1
    const int64_t rows[4] = {n0, n0 + a.nx, n0 + a.nx + plane, n0 + plane};
    float4 lo[4], hi[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) ldg_pair(g8 + 2 * rows[q], lo[q], hi[q]);
    double ex, ey, ez;
    pair_sum(lo, hi, c.ab, c.de, c.gh, ex, ey, ez);
    Eo[0] = ex;
    Eo[1] = ey;
    Eo[2] = ez;
    return fl;
}

// A warp handles 32 consecutive particles per iteration.  Their 96 output doubles are staged
// in shared memory and written as three contiguous 256-byte rows: 6 L2 write requests per
// warp instead of 18 for three strided 8-byte stores per lane, on a kernel whose limit is the
// L1's request port to L2.
__global__ void __launch_bounds__(256) k_interp_pairs(InterpArgs a, const float4 *__restrict__ g8,
                                                      double *__restrict__ E, unsigned long long *__restrict__ nclamp) {
    __shared__ double stage[256 * 3];
    const int lane = threadIdx.x & 31;
    double *ws = stage + (threadIdx.x - lane) * 3;
    const int64_t plane = (int64_t)a.nx * a.ny;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // the next particle's coordinates are loaded while this particle's field is gathered
    double xn = 0, yn = 0, zn = 0;
    if (m < a.np) {
        xn = __ldg(a.x + m);
        yn = __ldg(a.y + m);
        zn = __ldg(a.z + m);
    }
    // the loop runs while the warp's first particle exists, so all lanes take the same trips
    for (; m - lane < a.np; m += stride) {
        const double xm = xn, ym = yn, zm = zn;
        const int64_t mn = m + stride;
        if (mn < a.np) {
            xn = __ldg(a.x + mn);
            yn = __ldg(a.y + mn);
            zn = __ldg(a.z + mn);
        }
        const bool live = m < a.np;
        bool fl = false;
        if (live) fl = interp_pair_one(a, g8, plane, xm, ym, zm, ws + 3 * lane);
        count_one(nclamp, fl);
        __syncwarp();
        const int64_t o0 = 3 * (m - lane), n3 = 3 * a.np;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const int e = 32 * t + lane;
            if (o0 + e < n3) E[o0 + e] = ws[e];
        }
        __syncwarp();
    }
}

// Gather for particles in cell order.  Lane l of warp chunk w owns the RUN consecutive
// particles from (32 w + l) RUN (RUN = 4 or 8, chosen by the autotuner): their coordinates
// come in as 256-bit loads (32-byte aligned arrays), consecutive particles in the same cell
// reuse the four x-pairs loaded for the first of them, and the lane's 3 RUN consecutive
// output doubles leave as 256-bit stores.  Per particle the arithmetic is pair_sum's, as in
// k_interp_pairs, so E is bit-identical to it for any order.
__device__ __forceinline__ void ldg_v4(const double *p, double *v) {
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}
template <int RUN>
__global__ void __launch_bounds__(256, RUN == 4 ? 3 : 2) k_interp_pairs_runs(InterpArgs a, const float4 *__restrict__ g8, bool vec,
                                                           double *__restrict__ E,
                                                           unsigned long long *__restrict__ nclamp) {
    static_assert(RUN % 4 == 0, "runs of whole 256-bit vectors");
    const int64_t plane = (int64_t)a.nx * a.ny;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 * RUN < a.np; w += nwarps) {
        const int64_t m0 = (w * 32 + lane) * RUN;
        const bool full = vec && m0 + RUN <= a.np;
        double xs[RUN], ys[RUN], zs[RUN];
        if (full) {
#pragma unroll
            for (int v = 0; v < RUN / 4; ++v) {
                ldg_v4(a.x + m0 + 4 * v, xs + 4 * v);
                ldg_v4(a.y + m0 + 4 * v, ys + 4 * v);
                ldg_v4(a.z + m0 + 4 * v, zs + 4 * v);
            }
        } else {
#pragma unroll
            for (int t = 0; t < RUN; ++t) {
                const bool ok = m0 + t < a.np;
                xs[t] = ok ? __ldg(a.x + m0 + t) : 0.0;
                ys[t] = ok ? __ldg(a.y + m0 + t) : 0.0;
                zs[t] = ok ? __ldg(a.z + m0 + t) : 0.0;
            }
        }
        double out[3 * RUN];
        int64_t cur = -1;
        float4 lo[4], hi[4];
        unsigned ncl = 0;
#pragma unroll
        for (int t = 0; t < RUN; ++t) {
            out[3 * t] = out[3 * t + 1] = out[3 * t + 2] = 0.0;
            if (m0 + t >= a.np) continue;
            Cell c;
            ncl += locate(a, xs[t], ys[t], zs[t], c) ? 1u : 0u;
            const int64_t n0 = c.i + (int64_t)a.nx * c.j + plane * c.k;
            if (n0 != cur) {
                const int64_t rows[4] = {n0, n0 + a.nx, n0 + a.nx + plane, n0 + plane};
#pragma unroll
                for (int q = 0; q < 4; ++q) ldg_pair(g8 + 2 * rows[q], lo[q], hi[q]);
                cur = n0;
            }
            double ex, ey, ez;
            pair_sum(lo, hi, c.ab, c.de, c.gh, ex, ey, ez);
            out[3 * t] = ex;
            out[3 * t + 1] = ey;
            out[3 * t + 2] = ez;
        }
        double *dst = E + 3 * m0;
        if (full) {
#pragma unroll
            for (int v = 0; v < 3 * RUN / 4; ++v)
                asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(dst + 4 * v), "d"(out[4 * v]),
                             "d"(out[4 * v + 1]), "d"(out[4 * v + 2]), "d"(out[4 * v + 3])
                             : "memory");
        } else {
#pragma unroll
            for (int e = 0; e < 3 * RUN; ++e)
                if (m0 + e / 3 < a.np) dst[e] = out[e];
        }
        ncl = __reduce_add_sync(0xffffffffu, ncl);
        if (lane == 0 && ncl) atomicAdd(nclamp, (unsigned long long)ncl);
    }
}

int launch_interp_pairs_runs(const InterpArgs &a, const float4 *E8, double *E, unsigned long long *nclamp,
                             cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    if (reinterpret_cast<uintptr_t>(E8) % 32) return OSC_E_INVALID;
    auto al = [](const void *p) { return reinterpret_cast<uintptr_t>(p) % 32 == 0; };
    const bool vec = al(a.x) && al(a.y) && al(a.z) && al(E);
    const int run = a.tile == 8 ? 8 : 4;
    const int64_t chunks = (a.np + 32 * run - 1) / (32 * run);
    const unsigned nb = nblocks(chunks * 32, 256, 148 * (int64_t)(a.ctas > 0 ? a.ctas : 16));
    if (run == 8)
        k_interp_pairs_runs<8><<<nb, 256, 0, st>>>(a, E8, vec, E, nclamp);
    else
        k_interp_pairs_runs<4><<<nb, 256, 0, st>>>(a, E8, vec, E, nclamp);
    return ok();
}

int launch_interp_pairs(const InterpArgs &a, const float4 *E8, double *E, unsigned long long *nclamp,
                        cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    if (reinterpret_cast<uintptr_t>(E8) % 32) return OSC_E_INVALID;
    const int64_t cap = 148 * (int64_t)(a.ctas > 0 ? a.ctas : 64);
    k_interp_pairs<<<nblocks(a.np, 256, cap), 256, 0, st>>>(a, E8, E, nclamp);
    return ok();
}

int launch_interp_planes(const InterpArgs &a, const double *F, double *out, unsigned long long *nclamp,
                         cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    k_interp_planes<<<nblocks(a.np, 256, 148 * 64), 256, 0, st>>>(a, F, out, nclamp);
    return ok();
}

// ------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ord_key(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_val(unsigned long long u) {
    const unsigned long long b = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
    return __longlong_as_double((long long)b);
}

__global__ void k_bbox_init(unsigned long long *keys, unsigned long long *nonfinite) {
    if (threadIdx.x < 6) keys[threadIdx.x] = (threadIdx.x & 1) ? 0ull : ~0ull;
    if (threadIdx.x == 0) *nonfinite = 0;
}
__global__ void __launch_bounds__(256) k_bbox(int64_t np, const double *__restrict__ x, const double *__restrict__ y,
                                              const double *__restrict__ z, unsigned long long *keys,
                                              unsigned long long *nonfinite) {
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0};
    unsigned long long bad = 0;
    const double *p[3] = {x, y, z};
    // four particles per thread and trip, their twelve loads issued before any is used
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m0 < np; m0 += 4 * stride) {
        double v[4][3];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t m = m0 + u * stride;
#pragma unroll
            for (int d = 0; d < 3; ++d) v[u][d] = m < np ? __ldg(p[d] + m) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (m0 + u * stride >= np) break;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (!isfinite(v[u][d])) {
                    ++bad;
                    continue;
                }
                const unsigned long long k = ord_key(v[u][d]);
                lo[d] = k < lo[d] ? k : lo[d];
                hi[d] = k > hi[d] ? k : hi[d];
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        for (int off = 16; off; off >>= 1) {
            const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[d], off);
            const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi[d], off);
            lo[d] = a < lo[d] ? a : lo[d];
            hi[d] = b > hi[d] ? b : hi[d];
        }
    }
    for (int off = 16; off; off >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, off);
    // the block's warps combine in shared memory, then one thread adds the block's extremes:
    // seven atomics per block instead of per warp on the same seven words
    __shared__ unsigned long long sk[8][7];
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sk[w][2 * d] = lo[d];
            sk[w][2 * d + 1] = hi[d];
        }
        sk[w][6] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int v = 1; v < nw; ++v)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                lo[d] = sk[v][2 * d] < lo[d] ? sk[v][2 * d] : lo[d];
                hi[d] = sk[v][2 * d + 1] > hi[d] ? sk[v][2 * d + 1] : hi[d];
            }
        for (int v = 1; v < nw; ++v) bad += sk[v][6];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            atomicMin(&keys[2 * d], lo[d]);
            atomicMax(&keys[2 * d + 1], hi[d]);
        }
        if (bad) atomicAdd(nonfinite, bad);
    }
}
__global__ void k_bbox_final(const unsigned long long *keys, double *bb) {
    if (threadIdx.x < 6) bb[threadIdx.x] = ord_val(keys[threadIdx.x]);
}
int launch_bbox(int64_t np, const double *x, const double *y, const double *z, unsigned long long *keys, double *bb,
                unsigned long long *nonfinite, cudaStream_t st) {
    k_bbox_init<<<1, 32, 0, st>>>(keys, nonfinite);
    if (np > 0) k_bbox<<<nblocks(np, 256, 148 * 16), 256, 0, st>>>(np, x, y, z, keys, nonfinite);
    k_bbox_final<<<1, 32, 0, st>>>(keys, bb);
    return ok();
}

// Deterministic two-pass reductions of a particle array: op 0 sum, 1 maximum of |q|.
__device__ __forceinline__ double red_op(double a, double b, int op) { return op ? fmax(a, b) : a + b; }
__global__ void __launch_bounds__(256) k_sum_partial(int64_t n, const double *__restrict__ q, double *partials, int op) {
    __shared__ double sh[256];
    double s = 0;
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t beg = blockIdx.x * chunk, end = min(n, beg + chunk);
    for (int64_t m = beg + threadIdx.x; m < end; m += blockDim.x) s = red_op(s, op ? fabs(q[m]) : q[m], op);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = red_op(sh[threadIdx.x], sh[threadIdx.x + w], op);
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}
__global__ void k_sum_final(const double *partials, int np, double *out, int op) {
    __shared__ double sh[1024];
    sh[threadIdx.x] = threadIdx.x < np ? partials[threadIdx.x] : 0.0;
    __syncthreads();
    for (int w = 512; w; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = red_op(sh[threadIdx.x], sh[threadIdx.x + w], op);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}
int launch_sum(int64_t n, const double *q, double *partials, double *out, cudaStream_t st, bool max_abs) {
    k_sum_partial<<<1024, 256, 0, st>>>(n, q, partials, max_abs ? 1 : 0);
    k_sum_final<<<1, 1024, 0, st>>>(partials, 1024, out, max_abs ? 1 : 0);
    return ok();
}

// ------------------------------------------------------------------------------------
// Batched particle passes: CTA j handles particles [jobs[j].beg, jobs[j].end) of bunch
// jobs[j].bunch with that bunch's arguments; per-bunch counters cnt[4b + 0] outside,
// +1 non-finite, +2 clamped.
__global__ void __launch_bounds__(256) k_batch_deposit_quad(const BunchArgs *__restrict__ bunches,
                                                            const BatchJob *__restrict__ jobs, float4 *quad,
                                                            unsigned long long *cnt) {
    const BatchJob jb = jobs[blockIdx.x];
    const DepositArgs &a = bunches[jb.bunch].d;
    float4 *qb = quad + bunches[jb.bunch].node_off;
    const int64_t plane = (int64_t)a.nx * a.ny;
    for (int64_t m = jb.beg + threadIdx.x; m < jb.end; m += blockDim.x) {
        const double c = a.q ? a.q[m] : a.charge1;
        const int st = quad_one(a, qb, plane, a.x[m], a.y[m], a.z[m], c);
        count_one(&cnt[4 * jb.bunch + 0], st == 1);
        count_one(&cnt[4 * jb.bunch + 1], st == 2);
    }
}
int launch_batch_deposit_quad(const BunchArgs *bunches, const BatchJob *jobs, int njobs, float *quad,
                              unsigned long long *cnt, cudaStream_t st) {
    if (njobs <= 0) return OSC_OK;
    k_batch_deposit_quad<<<njobs, 256, 0, st>>>(bunches, jobs, reinterpret_cast<float4 *>(quad), cnt);
    return ok();
}

__global__ void __launch_bounds__(256) k_batch_interp_pairs(const BunchArgs *__restrict__ bunches,
                                                            const BatchJob *__restrict__ jobs,
                                                            const float4 *__restrict__ e8, unsigned long long *cnt) {
    const BatchJob jb = jobs[blockIdx.x];
    const InterpArgs &a = bunches[jb.bunch].in;
    const float4 *g8 = e8 + 2 * bunches[jb.bunch].node_off;
    double *E = bunches[jb.bunch].E;
    const int64_t plane = (int64_t)a.nx * a.ny;
    // E staged per warp and stored as contiguous rows, as in k_interp_pairs
    __shared__ double stage[256 * 3];
    const int lane = threadIdx.x & 31;
    double *ws = stage + (threadIdx.x - lane) * 3;
    for (int64_t m = jb.beg + threadIdx.x; m - lane < jb.end; m += blockDim.x) {
        bool fl = false;
        if (m < jb.end) fl = interp_pair_one(a, g8, plane, a.x[m], a.y[m], a.z[m], ws + 3 * lane);
        count_one(&cnt[4 * jb.bunch + 2], fl);
        __syncwarp();
        const int64_t o0 = 3 * (m - lane), n3 = 3 * jb.end;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const int e = 32 * t + lane;
            if (o0 + e < n3) E[o0 + e] = ws[e];
        }
        __syncwarp();
    }
}
int launch_batch_interp_pairs(const BunchArgs *bunches, const BatchJob *jobs, int njobs, const float *e8,
                              unsigned long long *cnt, cudaStream_t st) {
    if (njobs <= 0) return OSC_OK;
    k_batch_interp_pairs<<<njobs, 256, 0, st>>>(bunches, jobs, reinterpret_cast<const float4 *>(e8), cnt);
    return ok();
}

// Per job: ordered min/max keys of x, y, z (6), non-finite count, and the sum of q in
// index order within the CTA; then per bunch, its jobs combined in job order.
__global__ void __launch_bounds__(256) k_batch_stats(const BunchArgs *__restrict__ bunches,
                                                     const BatchJob *__restrict__ jobs, unsigned long long *keys,
                                                     double *qsum) {
    const BatchJob jb = jobs[blockIdx.x];
    const DepositArgs &a = bunches[jb.bunch].d;
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0}, bad = 0;
    double qs = 0;
    const double *p[3] = {a.x, a.y, a.z};
    for (int64_t m = jb.beg + threadIdx.x; m < jb.end; m += blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double v = p[d][m];
            if (!isfinite(v)) { ++bad; continue; }
            const unsigned long long k = ord_key(v);
            lo[d] = k < lo[d] ? k : lo[d];
            hi[d] = k > hi[d] ? k : hi[d];
        }
        if (a.q) qs += a.q[m];
    }
    __shared__ unsigned long long sk[7][256];
    __shared__ double sq[256];
    for (int d = 0; d < 3; ++d) {
        sk[2 * d][threadIdx.x] = lo[d];
        sk[2 * d + 1][threadIdx.x] = hi[d];
    }
    sk[6][threadIdx.x] = bad;
    sq[threadIdx.x] = qs;
    __syncthreads();
    for (int w = 128; w; w >>= 1) {
        if (threadIdx.x < w) {
            const int t = threadIdx.x;
            for (int d = 0; d < 3; ++d) {
                sk[2 * d][t] = min(sk[2 * d][t], sk[2 * d][t + w]);
                sk[2 * d + 1][t] = max(sk[2 * d + 1][t], sk[2 * d + 1][t + w]);
            }
            sk[6][t] += sk[6][t + w];
            sq[t] += sq[t + w];
        }
        __syncthreads();
    }
    if (threadIdx.x < 7) keys[7 * (int64_t)blockIdx.x + threadIdx.x] = sk[threadIdx.x][0];
    if (threadIdx.x == 0) qsum[blockIdx.x] = sq[0];
}
// out[8b .. 8b+5] = min/max of x, y, z as doubles, out[8b+6] = non-finite count,
// out[8b+7] = sum of q
__global__ void k_batch_stats_final(const int *__restrict__ job0, int nbunch, const unsigned long long *keys,
                                    const double *qsum, double *out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbunch) return;
    unsigned long long k[7] = {~0ull, 0, ~0ull, 0, ~0ull, 0, 0};
    double qs = 0;
    for (int j = job0[b]; j < job0[b + 1]; ++j) {
        for (int d = 0; d < 3; ++d) {
            k[2 * d] = min(k[2 * d], keys[7 * (int64_t)j + 2 * d]);
            k[2 * d + 1] = max(k[2 * d + 1], keys[7 * (int64_t)j + 2 * d + 1]);
        }
        k[6] += keys[7 * (int64_t)j + 6];
        qs += qsum[j];
    }
    for (int d = 0; d < 6; ++d) out[8 * b + d] = ord_val(k[d]);
    out[8 * b + 6] = (double)k[6];
    out[8 * b + 7] = qs;
}
int launch_batch_stats(const BunchArgs *bunches, const BatchJob *jobs, int njobs, const int *job0, int nbunch,
                       unsigned long long *keys, double *qsum, double *out, cudaStream_t st) {
    if (njobs > 0) k_batch_stats<<<njobs, 256, 0, st>>>(bunches, jobs, keys, qsum);
    k_batch_stats_final<<<(nbunch + 127) / 128, 128, 0, st>>>(job0, nbunch, keys, qsum, out);
    return ok();
}

// ------------------------------------------------------------------------------------
// Adjoint of the step.  Both the deposit (deposit_particles) and the gather
// (interpolate_field) are trilinear in the particle position within a cell, with the low
// node weighted ab = ((min - x) + f*delta)/delta, so d ab/dx = -1/delta.

// a[c][n] += sum over particles of g[m][c] times the particle's deposit weight of node n.
__global__ void __launch_bounds__(256) k_deposit_vec3(DepositArgs a, const double *__restrict__ g,
                                                      double *__restrict__ acc) {
    const int64_t plane = (int64_t)a.nx * a.ny, N = plane * a.nz;
    GRID_STRIDE(m, a.np) {
        const double xm = a.x[m], ym = a.y[m], zm = a.z[m];
        const double fx = floor(__dmul_rn(xm - a.xmin, a.dxi) + 1);
        const double fy = floor(__dmul_rn(ym - a.ymin, a.dyi) + 1);
        const double fz = floor(__dmul_rn(zm - a.zmin, a.dzi) + 1);
        if (!(fx >= a.nlo[0] && fx + 1 <= a.nhi[0] && fy >= a.nlo[1] && fy + 1 <= a.nhi[1] && fz >= a.nlo[2] &&
              fz + 1 <= a.nhi[2]))
            continue;
        const double ab = ((a.xmin - xm) + fx * a.dx) * a.dxi;
        const double de = ((a.ymin - ym) + fy * a.dy) * a.dyi;
        const double gh = ((a.zmin - zm) + fz * a.dz) * a.dzi;
        const int i = (int)fx - a.nlo[0], j = (int)fy - a.nlo[1], k = (int)fz - a.nlo[2];
        const int64_t n0 = i + (int64_t)a.nx * j + plane * k;
        double w[8];
        int64_t off[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int dx = t & 1, dy = (t >> 1) & 1, dz = t >> 2;
            w[t] = (dx ? 1. - ab : ab) * (dy ? 1. - de : de) * (dz ? 1. - gh : gh);
            off[t] = n0 + dx + (int64_t)a.nx * dy + plane * dz;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double gc = g[3 * m + c];
            if (gc == 0.0) continue;
#pragma unroll
            for (int t = 0; t < 8; ++t) red_add(acc + c * N + off[t], w[t] * gc);
        }
    }
}
int launch_deposit_vec3(const DepositArgs &a, const double *g, double *acc, cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    k_deposit_vec3<<<nblocks(a.np, 256, 148 * 64), 256, 0, st>>>(a, g, acc);
    return ok();
}

// Three quad grids at once: the CIC weights of a particle are computed once and each of
// the three gradient components adds two float4 reductions (planes k and k+1), the slots
// of quad_one in the same order.
__global__ void __launch_bounds__(256) k_deposit_quad3(DepositArgs a, const double *__restrict__ g,
                                                       float4 *__restrict__ quad3) {
    const int64_t plane = (int64_t)a.nx * a.ny, N = plane * a.nz;
    GRID_STRIDE(m, a.np) {
        const double xm = a.x[m], ym = a.y[m], zm = a.z[m];
        const double fx = floor(__dmul_rn(xm - a.xmin, a.dxi) + 1);
        const double fy = floor(__dmul_rn(ym - a.ymin, a.dyi) + 1);
        const double fz = floor(__dmul_rn(zm - a.zmin, a.dzi) + 1);
        if (!(fx >= a.nlo[0] && fx + 1 <= a.nhi[0] && fy >= a.nlo[1] && fy + 1 <= a.nhi[1] && fz >= a.nlo[2] &&
              fz + 1 <= a.nhi[2]))
            continue;
        const double ab = ((a.xmin - xm) + fx * a.dx) * a.dxi;
        const double de = ((a.ymin - ym) + fy * a.dy) * a.dyi;
        const double gh = ((a.zmin - zm) + fz * a.dz) * a.dzi;
        const double omab = 1. - ab, omde = 1. - de, omgh = 1. - gh;
        const int i = (int)fx - a.nlo[0], j = (int)fy - a.nlo[1], k = (int)fz - a.nlo[2];
        float4 *q0 = quad3 + ((int64_t)i + (int64_t)a.nx * j + plane * k);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double gc = g[3 * m + c];
            if (gc == 0.0) continue;
            const double lo = gh * gc, hi = omgh * gc;
            red_add(q0 + c * N, make_float4((float)(ab * de * lo), (float)(omab * de * lo), (float)(ab * omde * lo),
                                            (float)(omab * omde * lo)));
            red_add(q0 + c * N + plane, make_float4((float)(ab * de * hi), (float)(omab * de * hi),
                                                    (float)(ab * omde * hi), (float)(omab * omde * hi)));
        }
    }
}
int launch_deposit_quad3(const DepositArgs &a, const double *g, float *quad3, cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    k_deposit_quad3<<<nblocks(a.np, 256, 148 * 64), 256, 0, st>>>(a, g, reinterpret_cast<float4 *>(quad3));
    return ok();
}

__global__ void k_pack_lambda(float *__restrict__ e8, const double *__restrict__ lam, int nx, int64_t n) {
    GRID_STRIDE(idx, n) {
        const bool last = (idx % nx) == nx - 1;
        e8[8 * idx + 3] = (float)lam[idx];
        e8[8 * idx + 7] = last ? 0.f : (float)lam[idx + 1];
    }
}
int launch_pack_lambda(float *e8, const double *lam, int nx, int64_t n, cudaStream_t st) {
    k_pack_lambda<<<nblocks(n, 256), 256, 0, st>>>(e8, lam, nx, n);
    return ok();
}

// Value and gradient of the trilinear interpolant of F on the cell (i,j,k) with low-node
// weights (ab, de, gh): returns F(x) and d/dx, d/dy, d/dz.
__device__ __forceinline__ void trilinear_grad(const double *__restrict__ F, int64_t n0, int nx, int64_t plane,
                                               double ab, double de, double gh, const double hinv[3],
                                               double &val, double grad[3]) {
    double f[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) f[t] = F[n0 + (t & 1) + (int64_t)nx * ((t >> 1) & 1) + plane * (t >> 2)];
    const double wx[2] = {ab, 1. - ab}, wy[2] = {de, 1. - de}, wz[2] = {gh, 1. - gh};
    double v = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int a = t & 1, b = (t >> 1) & 1, c = t >> 2;
        v += wx[a] * wy[b] * wz[c] * f[t];
        gx += (a ? 1. : -1.) * wy[b] * wz[c] * f[t];
        gy += wx[a] * (b ? 1. : -1.) * wz[c] * f[t];
        gz += wx[a] * wy[b] * (c ? 1. : -1.) * f[t];
    }
    val = v;
    grad[0] = gx * hinv[0];
    grad[1] = gy * hinv[1];
    grad[2] = gz * hinv[2];
}

// Per particle: g_x = sum_c gE[c] grad E_c(x) (gather at the clamped interpolation cell)
// + q grad lambda(x) (deposit cell; particles outside the mesh deposit nothing), and
// g_q = lambda(x), where lambda is the adjoint potential.
__global__ void __launch_bounds__(256) k_vjp_particles(InterpArgs ia, DepositArgs da, const double *__restrict__ E,
                                                       const double *__restrict__ lam, const double *__restrict__ gE,
                                                       double *gx, double *gy, double *gz, double *gq) {
    const int64_t plane = (int64_t)ia.nx * ia.ny, N = plane * ia.nz;
    GRID_STRIDE(m, ia.np) {
        const double xm = ia.x[m], ym = ia.y[m], zm = ia.z[m];
        double g[3] = {0, 0, 0};
        Cell c;
        locate(ia, xm, ym, zm, c);
        const int64_t n0 = c.i + (int64_t)ia.nx * c.j + plane * c.k;
        for (int comp = 0; comp < 3; ++comp) {
            const double w = gE[3 * m + comp];
            if (w == 0.0) continue;
            double v, gr[3];
            trilinear_grad(E + comp * N, n0, ia.nx, plane, c.ab, c.de, c.gh, ia.hinv, v, gr);
            g[0] += w * gr[0];
            g[1] += w * gr[1];
            g[2] += w * gr[2];
        }
        double lv = 0;
        const double fx = floor(__dmul_rn(xm - da.xmin, da.dxi) + 1);
        const double fy = floor(__dmul_rn(ym - da.ymin, da.dyi) + 1);
        const double fz = floor(__dmul_rn(zm - da.zmin, da.dzi) + 1);
        if (fx >= da.nlo[0] && fx + 1 <= da.nhi[0] && fy >= da.nlo[1] && fy + 1 <= da.nhi[1] && fz >= da.nlo[2] &&
            fz + 1 <= da.nhi[2]) {
            const double ab = ((da.xmin - xm) + fx * da.dx) * da.dxi;
            const double de = ((da.ymin - ym) + fy * da.dy) * da.dyi;
            const double gh = ((da.zmin - zm) + fz * da.dz) * da.dzi;
            const int i = (int)fx - da.nlo[0], j = (int)fy - da.nlo[1], k = (int)fz - da.nlo[2];
            const double hinv[3] = {da.dxi, da.dyi, da.dzi};
            double gr[3];
            trilinear_grad(lam, i + (int64_t)da.nx * j + plane * k, da.nx, plane, ab, de, gh, hinv, lv, gr);
            const double q = da.q ? da.q[m] : da.charge1;
            g[0] += q * gr[0];
            g[1] += q * gr[1];
            g[2] += q * gr[2];
        }
        gx[m] = g[0];
        gy[m] = g[1];
        gz[m] = g[2];
        if (gq) gq[m] = lv;
    }
}
// k_vjp_particles on the x-pair grid: one cell, four 256-bit loads give the 8 nodes' (Ex,
// Ey, Ez, lam).  A particle whose deposit cell is valid has that cell as its interpolation
// cell (same formula, same range), so the lam term uses the same nodes; other particles
// deposit nothing and get no lam term.
__global__ void __launch_bounds__(256) k_vjp_pairs(InterpArgs ia, DepositArgs da, const float4 *__restrict__ g8,
                                                   const double *__restrict__ gE, double *gx, double *gy, double *gz,
                                                   double *gq) {
    const int64_t plane = (int64_t)ia.nx * ia.ny;
    // the warp's 32 particles' dL/dE (96 doubles) are read as three contiguous 256-byte rows
    // into shared memory; the loop runs while the warp's first particle exists
    __shared__ double stage[256 * 3];
    const int lane = threadIdx.x & 31;
    double *ws = stage + (threadIdx.x - lane) * 3;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m - lane < ia.np; m += stride) {
        // coordinates first, so that their loads are in flight with the dL/dE rows
        double xm = 0, ym = 0, zm = 0;
        if (m < ia.np) {
            xm = ia.x[m];
            ym = ia.y[m];
            zm = ia.z[m];
        }
        {
            const int64_t o0 = 3 * (m - lane), n3 = 3 * ia.np;
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const int e = 32 * t + lane;
                if (o0 + e < n3) ws[e] = gE[o0 + e];
            }
        }
        __syncwarp();
        const double gEm[3] = {ws[3 * lane], ws[3 * lane + 1], ws[3 * lane + 2]};
        __syncwarp();
        if (m >= ia.np) continue;
        Cell c;
        locate(ia, xm, ym, zm, c);
        const int64_t n0 = c.i + (int64_t)ia.nx * c.j + plane * c.k;
        // t = dx + 2 dy + 4 dz: rows (dy, dz) hold nodes i (lo) and i+1 (hi)
        const int64_t rows[4] = {n0, n0 + ia.nx, n0 + plane, n0 + ia.nx + plane};
        float4 lo[4], hi[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) ldg_pair(g8 + 2 * rows[r], lo[r], hi[r]);
        const double wx[2] = {c.ab, 1. - c.ab}, wy[2] = {c.de, 1. - c.de}, wz[2] = {c.gh, 1. - c.gh};
        double val[4] = {0, 0, 0, 0}, d[4][3] = {};
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int a = t & 1, b = (t >> 1) & 1, cz = t >> 2;
            const float4 f = a ? hi[b + 2 * cz] : lo[b + 2 * cz];
            const double fv[4] = {f.x, f.y, f.z, f.w};
            const double w = wx[a] * wy[b] * wz[cz];
            const double sx = (a ? 1. : -1.) * wy[b] * wz[cz], sy = wx[a] * (b ? 1. : -1.) * wz[cz],
                         sz = wx[a] * wy[b] * (cz ? 1. : -1.);
#pragma unroll
            for (int f4 = 0; f4 < 4; ++f4) {
                val[f4] += w * fv[f4];
                d[f4][0] += sx * fv[f4];
                d[f4][1] += sy * fv[f4];
                d[f4][2] += sz * fv[f4];
            }
        }
        double g[3] = {0, 0, 0};
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
            const double w = gEm[comp];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) g[ax] += w * d[comp][ax] * ia.hinv[ax];
        }
        double lv = 0;
        const double fx = floor(__dmul_rn(xm - da.xmin, da.dxi) + 1);
        const double fy = floor(__dmul_rn(ym - da.ymin, da.dyi) + 1);
        const double fz = floor(__dmul_rn(zm - da.zmin, da.dzi) + 1);
        if (fx >= da.nlo[0] && fx + 1 <= da.nhi[0] && fy >= da.nlo[1] && fy + 1 <= da.nhi[1] && fz >= da.nlo[2] &&
            fz + 1 <= da.nhi[2]) {
            const double q = da.q ? da.q[m] : da.charge1;
            lv = val[3];
            g[0] += q * d[3][0] * ia.hinv[0];
            g[1] += q * d[3][1] * ia.hinv[1];
            g[2] += q * d[3][2] * ia.hinv[2];
        }
        gx[m] = g[0];
        gy[m] = g[1];
        gz[m] = g[2];
        if (gq) gq[m] = lv;
    }
}
int launch_vjp_pairs(const InterpArgs &ia, const DepositArgs &da, const float *e8, const double *gE, double *gx,
                     double *gy, double *gz, double *gq, cudaStream_t st) {
    if (ia.np <= 0) return OSC_OK;
    if (reinterpret_cast<uintptr_t>(e8) % 32) return OSC_E_INVALID;
    k_vjp_pairs<<<nblocks(ia.np, 256, 148 * 64), 256, 0, st>>>(ia, da, reinterpret_cast<const float4 *>(e8), gE, gx,
                                                               gy, gz, gq);
    return ok();
}

int launch_vjp_particles(const InterpArgs &ia, const DepositArgs &da, const double *E, const double *lam,
                         const double *gE, double *gx, double *gy, double *gz, double *gq, cudaStream_t st) {
    if (ia.np <= 0) return OSC_OK;
    k_vjp_particles<<<nblocks(ia.np, 256, 148 * 64), 256, 0, st>>>(ia, da, E, lam, gE, gx, gy, gz, gq);
    return ok();
}

// ------------------------------------------------------------------------------------
// E planes [3][N] (f64) -> x-pair grid (f32): node n holds (Ex,Ey,Ez,0) at n and at n+1, the
// last node of a row (E(n), 0); one 256-bit store per node.
__global__ void __launch_bounds__(256) k_planes_to_pairs(const double *__restrict__ E, float4 *__restrict__ e8,
                                                         int nx, int64_t n) {
    GRID_STRIDE(i, n) {
        const int x = (int)(i % nx);
        const bool last = x == nx - 1;
        const float4 lo = make_float4((float)E[i], (float)E[i + n], (float)E[i + 2 * n], 0.f);
        const float4 hi = last ? make_float4(0.f, 0.f, 0.f, 0.f)
                               : make_float4((float)E[i + 1], (float)E[i + 1 + n], (float)E[i + 1 + 2 * n], 0.f);
        asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(e8 + 2 * i), "f"(lo.x), "f"(lo.y),
                     "f"(lo.z), "f"(lo.w), "f"(hi.x), "f"(hi.y), "f"(hi.z), "f"(hi.w)
                     : "memory");
    }
}
int launch_planes_to_pairs(const double *E, float *e8, int nx, int64_t n, cudaStream_t st) {
    if (reinterpret_cast<uintptr_t>(e8) % 32) return OSC_E_INVALID;
    k_planes_to_pairs<<<nblocks(n, 256), 256, 0, st>>>(E, reinterpret_cast<float4 *>(e8), nx, n);
    return ok();
}

}  // namespace osc
