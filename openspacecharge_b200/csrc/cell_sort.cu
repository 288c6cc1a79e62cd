// cell_sort.cu -- counting sort of particles by deposit cell, run-aggregated deposits, and
// the permutation of gathered fields back to the caller's order.
#include "cell_sort.cuh"

namespace osc {

static inline int ok() { return cudaGetLastError() == cudaSuccess ? OSC_OK : OSC_E_CUDA; }
static inline unsigned nblocks(int64_t n, int bs, int64_t cap) {
    int64_t b = (n + bs - 1) / bs;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

__device__ __forceinline__ void red_add4(float4 *p, float4 v) {
    asm volatile("red.global.add.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}
__device__ __forceinline__ void red_add_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Linear index of a cell's lowest corner (< N <= 2^30: every axis is at most 1024 nodes,
// the largest doubled FFT length being 2048).
__device__ __forceinline__ uint32_t cell_key(const DepositArgs &a, const CicCell &c) {
    return (uint32_t)c.i + (uint32_t)a.nx * ((uint32_t)c.j + (uint32_t)a.ny * (uint32_t)c.k);
}

// ------------------------------------------------------------------------------------
// Keys and ranks.  Lanes of a warp whose particles share a cell take consecutive ranks
// from one atomic (most of a warp in cell order, rarely in random order).  The trip count
// is uniform per warp (m - lane is the warp's first particle), so the warp votes are full.
__global__ void __launch_bounds__(256) k_cell_keys(DepositArgs a, uint32_t *__restrict__ keys,
                                                   uint32_t *__restrict__ ranks, uint32_t *__restrict__ counts,
                                                   unsigned long long *__restrict__ counters) {
    const uint32_t N = (uint32_t)a.nx * (uint32_t)a.ny * (uint32_t)a.nz;
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m - lane < a.np; m += stride) {
        const bool live = m < a.np;
        uint32_t key = 0xffffffffu;  // lanes past the end: a key no particle has
        int st = 0;
        if (live) {
            CicCell c = {0, 0, 0, 0.0, 0.0, 0.0};
            st = cic_cell_mode0(a, __ldg(a.x + m), __ldg(a.y + m), __ldg(a.z + m), c);
            key = st ? N : cell_key(a, c);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (live && lane == leader) base = atomicAdd(counts + key, (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (live) {
            keys[m] = key;
            ranks[m] = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
        }
        const unsigned out = __ballot_sync(0xffffffffu, live && st == 1);
        const unsigned bad = __ballot_sync(0xffffffffu, live && st == 2);
        if (lane == 0) {
            if (out) atomicAdd(counters, (unsigned long long)__popc(out));
            if (bad) atomicAdd(counters + 1, (unsigned long long)__popc(bad));
        }
    }
}

int launch_cell_keys(const DepositArgs &a, uint32_t *keys, uint32_t *ranks, uint32_t *counts,
                     unsigned long long *counters, cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    k_cell_keys<<<nblocks(a.np, 256, 148 * 16), 256, 0, st>>>(a, keys, ranks, counts, counters);
    return ok();
}

// ------------------------------------------------------------------------------------
// Exclusive prefix sums of n 32-bit counts in place: blocks of kScanItems, then the block
// totals (one CTA, in chunks with a running carry), then the block offsets added.
constexpr int kScanThreads = 256, kScanPer = 8, kScanItems = kScanThreads * kScanPer;

int64_t cell_scan_partials(int64_t n) { return (n + kScanItems - 1) / kScanItems; }

// Exclusive scan of one value per thread across the CTA; *total receives the CTA sum.
__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t v, uint32_t *warp_sums, uint32_t *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += t;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? warp_sums[lane] : 0u, wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += t;
        }
        if (lane < nw) warp_sums[lane] = wi - w;  // exclusive offset of each warp
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const uint32_t r = warp_sums[warp] + inc - v;
    __syncthreads();  // warp_sums is reused by the caller's next scan
    return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(uint32_t *__restrict__ c, int64_t n,
                                                              uint32_t *__restrict__ partials) {
    __shared__ uint32_t ws[32];
    __shared__ uint32_t tot;
    const int64_t base = (int64_t)blockIdx.x * kScanItems + (int64_t)threadIdx.x * kScanPer;
    uint32_t v[kScanPer], s = 0;
#pragma unroll
    for (int t = 0; t < kScanPer; ++t) {
        v[t] = base + t < n ? c[base + t] : 0u;
        s += v[t];
    }
    uint32_t run = cta_exclusive_scan(s, ws, &tot);
#pragma unroll
    for (int t = 0; t < kScanPer; ++t) {
        if (base + t < n) c[base + t] = run;
        run += v[t];
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_partials(uint32_t *__restrict__ p, int64_t np_) {
    __shared__ uint32_t ws[32];
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (int64_t b0 = 0; b0 < np_; b0 += blockDim.x) {
        const int64_t i = b0 + threadIdx.x;
        const uint32_t v = i < np_ ? p[i] : 0u;
        const uint32_t e = cta_exclusive_scan(v, ws, &tot);
        if (i < np_) p[i] = carry + e;
        carry += tot;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_scan_add(uint32_t *__restrict__ c, int64_t n,
                                                  const uint32_t *__restrict__ partials) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        c[i] += partials[i / kScanItems];
}

int launch_cell_scan(uint32_t *counts, int64_t n, uint32_t *partials, cudaStream_t st) {
    if (n <= 0) return OSC_OK;
    const int64_t nb = cell_scan_partials(n);
    if (nb > 0x7fffffff) return OSC_E_INVALID;
    k_scan_blocks<<<(unsigned)nb, kScanThreads, 0, st>>>(counts, n, partials);
    k_scan_partials<<<1, 1024, 0, st>>>(partials, nb);
    k_scan_add<<<nblocks(n, 256, 148 * 16), 256, 0, st>>>(counts, n, partials);
    return ok();
}

// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_cell_scatter(int64_t np, const uint32_t *__restrict__ keys,
                                                      const uint32_t *__restrict__ ranks,
                                                      const uint32_t *__restrict__ start, const double *__restrict__ x,
                                                      const double *__restrict__ y, const double *__restrict__ z,
                                                      const double *__restrict__ q, double *__restrict__ xs,
                                                      double *__restrict__ ys, double *__restrict__ zs,
                                                      double *__restrict__ qs, int64_t *__restrict__ perm64,
                                                      uint32_t *__restrict__ inv) {
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < np; m += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t pos = __ldg(start + __ldg(keys + m)) + __ldg(ranks + m);
        xs[pos] = __ldg(x + m);
        ys[pos] = __ldg(y + m);
        zs[pos] = __ldg(z + m);
        if (q) qs[pos] = __ldg(q + m);
        if (perm64) perm64[pos] = m;
        if (inv) inv[m] = pos;
    }
}

int launch_cell_scatter(int64_t np, const uint32_t *keys, const uint32_t *ranks, const uint32_t *start,
                        const double *x, const double *y, const double *z, const double *q, double *xs,
                        double *ys, double *zs, double *qs, int64_t *perm64, uint32_t *inv, cudaStream_t st) {
    if (np <= 0) return OSC_OK;
    if ((q == nullptr) != (qs == nullptr)) return OSC_E_INVALID;
    k_cell_scatter<<<nblocks(np, 256, 148 * 16), 256, 0, st>>>(np, keys, ranks, start, x, y, z, q, xs, ys, zs, qs,
                                                               perm64, inv);
    return ok();
}

// ------------------------------------------------------------------------------------
// Run-aggregated deposits.  Lane l of warp chunk w owns the RUN consecutive particles
// starting at (32 w + l) RUN (RUN = 4 or 8, the deposit tile the autotuner picks): it loads
// them (256-bit loads when the arrays are 32-byte aligned), walks them in order, sums the
// contributions of consecutive particles in the same cell, and adds a run's sum to the grid
// when the cell changes and at the end.  Particles outside the mesh are counted and skipped
// without ending a run.
template <int RUN>
__device__ __forceinline__ void load_run(const double *__restrict__ p, int64_t m0, int64_t np, bool vec,
                                         double (&v)[RUN]) {
    if (vec && m0 + RUN <= np) {
#pragma unroll
        for (int u = 0; u < RUN / 4; ++u)
            asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                : "=d"(v[4 * u]), "=d"(v[4 * u + 1]), "=d"(v[4 * u + 2]), "=d"(v[4 * u + 3])
                : "l"(p + m0 + 4 * u));
    } else {
#pragma unroll
        for (int t = 0; t < RUN; ++t) v[t] = m0 + t < np ? __ldg(p + m0 + t) : 0.0;
    }
}

// s + c += v with the rounding error of the sum kept in c (Knuth's two-sum).
__device__ __forceinline__ void two_sum_add(float &s, float &c, float v) {
    const float t = s + v;
    const float bp = t - s;
    const float e = (s - (t - bp)) + (v - bp);
    s = t;
    c += e;
}

template <int kRun, bool HQ>
__global__ void __launch_bounds__(256, kRun == 4 ? 3 : 2) k_deposit_quad_runs(DepositArgs a, float4 *__restrict__ quad, bool vec,
                                                           unsigned long long *__restrict__ counters) {
    const int64_t plane = (int64_t)a.nx * a.ny;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 * kRun < a.np; w += nwarps) {
        const int64_t m0 = (w * 32 + lane) * kRun;
        // HQ: charges per particle; otherwise every particle carries a.charge1
        double xs[kRun], ys[kRun], zs[kRun], qs[HQ ? kRun : 1];
        load_run<kRun>(a.x, m0, a.np, vec, xs);
        load_run<kRun>(a.y, m0, a.np, vec, ys);
        load_run<kRun>(a.z, m0, a.np, vec, zs);
        if constexpr (HQ) load_run<kRun>(a.q, m0, a.np, vec, qs);
        int64_t cur = -1;
        float s[8], c[8];
        int nout = 0, nbad = 0;
#pragma unroll
        for (int t = 0; t < kRun; ++t) {
            if (m0 + t >= a.np) break;
            CicCell cc = {0, 0, 0, 0.0, 0.0, 0.0};
            const int st = cic_cell_mode0(a, xs[t], ys[t], zs[t], cc);
            if (st) {
                nout += st == 1;
                nbad += st == 2;
                continue;
            }
            // the quad contributions of deposit_particles' weights (code/open_spacecharge_mod.f90:274-281)
            const double omab = 1. - cc.ab, omde = 1. - cc.de, omgh = 1. - cc.gh;
            const double qm = HQ ? qs[HQ ? t : 0] : a.charge1;
            const double lo = cc.gh * qm, hi = omgh * qm;
            const float v[8] = {(float)(cc.ab * cc.de * lo), (float)(omab * cc.de * lo), (float)(cc.ab * omde * lo),
                                (float)(omab * omde * lo),   (float)(cc.ab * cc.de * hi), (float)(omab * cc.de * hi),
                                (float)(cc.ab * omde * hi),  (float)(omab * omde * hi)};
            const int64_t key = cc.i + (int64_t)a.nx * cc.j + plane * cc.k;
            if (key != cur) {
                if (cur >= 0) {
                    red_add4(quad + cur, make_float4(s[0] + c[0], s[1] + c[1], s[2] + c[2], s[3] + c[3]));
                    red_add4(quad + cur + plane, make_float4(s[4] + c[4], s[5] + c[5], s[6] + c[6], s[7] + c[7]));
                }
                cur = key;
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    s[e] = v[e];
                    c[e] = 0.f;
                }
            } else {
#pragma unroll
                for (int e = 0; e < 8; ++e) two_sum_add(s[e], c[e], v[e]);
            }
        }
        if (cur >= 0) {
            red_add4(quad + cur, make_float4(s[0] + c[0], s[1] + c[1], s[2] + c[2], s[3] + c[3]));
            red_add4(quad + cur + plane, make_float4(s[4] + c[4], s[5] + c[5], s[6] + c[6], s[7] + c[7]));
        }
        nout = __reduce_add_sync(0xffffffffu, (unsigned)nout);
        nbad = __reduce_add_sync(0xffffffffu, (unsigned)nbad);
        if (lane == 0) {
            if (nout) atomicAdd(counters, (unsigned long long)nout);
            if (nbad) atomicAdd(counters + 1, (unsigned long long)nbad);
        }
    }
}

static bool aligned32(const void *p) { return p == nullptr || reinterpret_cast<uintptr_t>(p) % 32 == 0; }

int launch_deposit_quad_runs(const DepositArgs &a, float *quad, unsigned long long *counters, cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    if (a.mode != 0 || a.lost) return OSC_E_INVALID;
    const bool vec = aligned32(a.x) && aligned32(a.y) && aligned32(a.z) && aligned32(a.q);
    const int run = a.tile == 8 ? 8 : 4;
    const int64_t chunks = (a.np + 32 * run - 1) / (32 * run);
    const unsigned nb = nblocks(chunks * 32, 256, 148 * (int64_t)(a.ctas > 0 ? a.ctas : 16));
    float4 *q4 = reinterpret_cast<float4 *>(quad);
    if (run == 8) {
        if (a.q) k_deposit_quad_runs<8, true><<<nb, 256, 0, st>>>(a, q4, vec, counters);
        else k_deposit_quad_runs<8, false><<<nb, 256, 0, st>>>(a, q4, vec, counters);
    } else {
        if (a.q) k_deposit_quad_runs<4, true><<<nb, 256, 0, st>>>(a, q4, vec, counters);
        else k_deposit_quad_runs<4, false><<<nb, 256, 0, st>>>(a, q4, vec, counters);
    }
    return ok();
}

// Fixed point: the eight contributions of k_deposit<unsigned long long> (the same double
// products in the same order, rounded to integers with the same scale), summed per run in
// 64-bit integers, which is exact, so the node sums are those of the per-particle kernel.
template <int kRun>
__global__ void __launch_bounds__(256) k_deposit_fixed_runs(DepositArgs a, unsigned long long *__restrict__ acc,
                                                            bool vec, unsigned long long *__restrict__ counters) {
    const int64_t plane = (int64_t)a.nx * a.ny;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 * kRun < a.np; w += nwarps) {
        const int64_t m0 = (w * 32 + lane) * kRun;
        double xs[kRun], ys[kRun], zs[kRun], qs[kRun];
        load_run<kRun>(a.x, m0, a.np, vec, xs);
        load_run<kRun>(a.y, m0, a.np, vec, ys);
        load_run<kRun>(a.z, m0, a.np, vec, zs);
        if (a.q) {
            load_run<kRun>(a.q, m0, a.np, vec, qs);
        } else {
#pragma unroll
            for (int t = 0; t < kRun; ++t) qs[t] = a.charge1;
        }
        int64_t cur = -1;
        long long s[8];
        int nout = 0, nbad = 0;
        auto flush = [&]() {
            // node order of k_deposit: (i,j,k) (i,j+1,k) (i,j+1,k+1) (i,j,k+1) (i+1,j,k+1)
            // (i+1,j+1,k+1) (i+1,j+1,k) (i+1,j,k)
            unsigned long long *r0 = acc + cur;
            red_add_u64(r0, (unsigned long long)s[0]);
            red_add_u64(r0 + a.nx, (unsigned long long)s[1]);
            red_add_u64(r0 + a.nx + plane, (unsigned long long)s[2]);
            red_add_u64(r0 + plane, (unsigned long long)s[3]);
            red_add_u64(r0 + 1 + plane, (unsigned long long)s[4]);
            red_add_u64(r0 + 1 + a.nx + plane, (unsigned long long)s[5]);
            red_add_u64(r0 + 1 + a.nx, (unsigned long long)s[6]);
            red_add_u64(r0 + 1, (unsigned long long)s[7]);
        };
#pragma unroll
        for (int t = 0; t < kRun; ++t) {
            if (m0 + t >= a.np) break;
            CicCell cc = {0, 0, 0, 0.0, 0.0, 0.0};
            const int st = cic_cell_mode0(a, xs[t], ys[t], zs[t], cc);
            if (st) {
                nout += st == 1;
                nbad += st == 2;
                continue;
            }
            const double ab = cc.ab, de = cc.de, gh = cc.gh, q = qs[t];
            const double omab = 1. - ab, omde = 1. - de, omgh = 1. - gh;
            const double sc = a.fx_scale;
            const long long v[8] = {__double2ll_rn(ab * de * gh * q * sc),     __double2ll_rn(ab * omde * gh * q * sc),
                                    __double2ll_rn(ab * omde * omgh * q * sc), __double2ll_rn(ab * de * omgh * q * sc),
                                    __double2ll_rn(omab * de * omgh * q * sc), __double2ll_rn(omab * omde * omgh * q * sc),
                                    __double2ll_rn(omab * omde * gh * q * sc), __double2ll_rn(omab * de * gh * q * sc)};
            const int64_t key = cc.i + (int64_t)a.nx * cc.j + plane * cc.k;
            if (key != cur) {
                if (cur >= 0) flush();
                cur = key;
#pragma unroll
                for (int e = 0; e < 8; ++e) s[e] = v[e];
            } else {
#pragma unroll
                for (int e = 0; e < 8; ++e) s[e] += v[e];
            }
        }
        if (cur >= 0) flush();
        nout = __reduce_add_sync(0xffffffffu, (unsigned)nout);
        nbad = __reduce_add_sync(0xffffffffu, (unsigned)nbad);
        if (lane == 0) {
            if (nout) atomicAdd(counters, (unsigned long long)nout);
            if (nbad) atomicAdd(counters + 1, (unsigned long long)nbad);
        }
    }
}

int launch_deposit_fixed_runs(const DepositArgs &a, unsigned long long *acc, unsigned long long *counters,
                              cudaStream_t st) {
    if (a.np <= 0) return OSC_OK;
    if (a.mode != 0 || a.lost) return OSC_E_INVALID;
    const bool vec = aligned32(a.x) && aligned32(a.y) && aligned32(a.z) && aligned32(a.q);
    const int run = a.tile == 8 ? 8 : 4;
    const int64_t chunks = (a.np + 32 * run - 1) / (32 * run);
    const unsigned nb = nblocks(chunks * 32, 256, 148 * (int64_t)(a.ctas > 0 ? a.ctas : 16));
    if (run == 8)
        k_deposit_fixed_runs<8><<<nb, 256, 0, st>>>(a, acc, vec, counters);
    else
        k_deposit_fixed_runs<4><<<nb, 256, 0, st>>>(a, acc, vec, counters);
    return ok();
}

// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_unpermute_rows3(int64_t np, const uint32_t *__restrict__ inv,
                                                         const double *__restrict__ Es, double *__restrict__ E) {
    // a warp's 32 rows are staged and stored as three contiguous 256-byte rows
    __shared__ double stage[256 * 3];
    const int lane = threadIdx.x & 31;
    double *ws = stage + (threadIdx.x - lane) * 3;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m - lane < np; m += stride) {
        if (m < np) {
            const double *src = Es + 3 * (int64_t)__ldg(inv + m);
            ws[3 * lane] = __ldg(src);
            ws[3 * lane + 1] = __ldg(src + 1);
            ws[3 * lane + 2] = __ldg(src + 2);
        }
        __syncwarp();
        const int64_t o0 = 3 * (m - lane), n3 = 3 * np;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const int e = 32 * t + lane;
            if (o0 + e < n3) E[o0 + e] = ws[e];
        }
        __syncwarp();
    }
}

int launch_unpermute_rows3(int64_t np, const uint32_t *inv, const double *Es, double *E, cudaStream_t st) {
    if (np <= 0) return OSC_OK;
    k_unpermute_rows3<<<nblocks(np, 256, 148 * 16), 256, 0, st>>>(np, inv, Es, E);
    return ok();
}

}  // namespace osc
