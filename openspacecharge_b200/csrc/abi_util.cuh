// abi_util.cuh -- host helpers shared by the extern "C" entry points (abi.cu, batch.cu).
#pragma once
#include <cmath>
#include <cstring>

#include "../../include/opensc_gpu.h"
#include "cell_sort.cuh"
#include "solver.cuh"

#define TRY(...)                 \
    do {                         \
        int rc_ = (__VA_ARGS__); \
        if (rc_) return rc_;     \
    } while (0)
#define CK(call, what) TRY(cuda_check(ctx, (call), what))

namespace osc_abi {
using namespace osc;

inline int bad(osc_ctx *ctx, const char *what) { return set_err(ctx, OSC_E_INVALID, "invalid argument: %s", what); }

inline int mesh_dims(osc_ctx *ctx, const osc_mesh3d *m, int n[3]) {
    if (!m) return bad(ctx, "mesh is NULL");
    for (int d = 0; d < 3; ++d) {
        n[d] = m->nhi[d] - m->nlo[d] + 1;
        if (n[d] < 2) return set_err(ctx, OSC_E_INVALID, "mesh axis %d has %d nodes (need >= 2)", d, n[d]);
    }
    return OSC_OK;
}

inline int check_prec(osc_ctx *ctx, int p) {
    if (p < 0 || p > 2) return bad(ctx, "precision must be OSC_PREC_FP32, OSC_PREC_FP64 or OSC_PREC_FP64_PLAIN");
    return OSC_OK;
}

inline int h2d(osc_ctx *ctx, void *d, const void *h, size_t bytes) {
    return cuda_check(ctx, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ctx->stream), "H2D copy");
}
inline int d2h(osc_ctx *ctx, void *h, const void *d, size_t bytes) {
    return cuda_check(ctx, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, ctx->stream), "D2H copy");
}
inline int sync(osc_ctx *ctx) { return ctx_sync(ctx); }

// Auxiliary streams of a context: kAuxSlots streams and kAuxSlots + 1 events, created once
// (the last event belongs to the main stream).
constexpr int kAuxSlots = 4;
inline int ensure_aux(osc_ctx *ctx) {
    if (ctx->capturing &&
        ((int)ctx->aux.size() < kAuxSlots || (int)ctx->aux_ev.size() < kAuxSlots + 1 || !ctx->cap_stream))
        return set_err(ctx, OSC_E_UNSUPPORTED, "auxiliary streams would be created during graph capture");
    if (!ctx->cap_stream) CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking), "capture stream");
    while ((int)ctx->aux.size() < kAuxSlots) {
        cudaStream_t s;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "aux stream");
        ctx->aux.push_back(s);
    }
    while ((int)ctx->aux_ev.size() < kAuxSlots + 1) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "aux event");
        ctx->aux_ev.push_back(e);
    }
    return OSC_OK;
}

// Stage a host array on the device under a workspace name.
template <typename T> inline int stage_in(osc_ctx *ctx, const char *name, const T *h, size_t n, T **d) {
    if (!h) {
        *d = nullptr;
        return OSC_OK;
    }
    TRY(ws_get(ctx, name, sizeof(T) * n, (void **)d));
    return h2d(ctx, *d, h, sizeof(T) * n);
}

// Mesh refit of deposit_particles (code/open_spacecharge_mod.f90:176-189) from the
// particle bounding box: the box widened by 1e-6 cells on each side.
inline void apply_refit(osc_mesh3d *mesh, const double bmin[3], const double bmax[3]) {
    double mn[3] = {bmin[0], bmin[1], bmin[2]}, mx[3] = {bmax[0], bmax[1], bmax[2]}, delta[3];
    for (int d = 0; d < 3; ++d) delta[d] = (mx[d] - mn[d]) / (double)(mesh->nhi[d] - mesh->nlo[d]);
    for (int d = 0; d < 3; ++d) {
        mn[d] = mn[d] - 1.0e-6 * delta[d];
        mx[d] = mx[d] + 1.0e-6 * delta[d];
    }
    for (int d = 0; d < 3; ++d) delta[d] = (mx[d] - mn[d]) / (double)(mesh->nhi[d] - mesh->nlo[d]);
    for (int d = 0; d < 3; ++d) {
        mesh->min[d] = mn[d];
        mesh->max[d] = mx[d];
        mesh->delta[d] = delta[d];
    }
}

// Reference mesh refit of deposit_particles (code/open_spacecharge_mod.f90:176-189) from
// the particle bounding box computed on the device.
inline int refit_mesh(osc_ctx *ctx, int64_t np, const double *x, const double *y, const double *z, osc_mesh3d *mesh) {
    if (np <= 0) return set_err(ctx, OSC_E_INVALID, "resize_mesh needs at least one particle");
    double *bb;
    TRY(ws_get(ctx, "bbox", sizeof(double) * 8, (void **)&bb));
    {
        Launch L_(ctx, "bbox", 3);
        TRY(launch_bbox(np, x, y, z, ctx->d_small + 8, bb, ctx->d_small + 16, ctx->stream) ? set_err(ctx, OSC_E_CUDA, "bbox") : 0);
    }
    double hb[6];
    TRY(d2h(ctx, hb, bb, sizeof(hb)));
    TRY(d2h(ctx, ctx->h_small + 16, ctx->d_small + 16, sizeof(unsigned long long)));
    TRY(sync(ctx));
    if (ctx->h_small[16]) return set_err(ctx, OSC_E_NAN, "%llu non-finite particle coordinates", ctx->h_small[16]);
    const double mn[3] = {hb[0], hb[2], hb[4]}, mx[3] = {hb[1], hb[3], hb[5]};
    apply_refit(mesh, mn, mx);
    return OSC_OK;
}

inline int set_charge(osc_ctx *ctx, int64_t np, const double *q, const double *total_charge, osc_mesh3d *mesh,
               double *charge1) {
    if (q) {
        double *out;
        TRY(ws_get(ctx, "qsum", sizeof(double), (void **)&out));
        {
            Launch L_(ctx, "charge_sum", 2);
            if (launch_sum(np, q, ctx->d_partials, out, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "charge sum");
        }
        double s = 0;
        TRY(d2h(ctx, &s, out, sizeof(double)));
        TRY(sync(ctx));
        mesh->charge = s;
        *charge1 = 0;
    } else if (total_charge) {
        mesh->charge = *total_charge;
        *charge1 = *total_charge / (double)np;
    } else {
        return set_err(ctx, OSC_E_NOCHARGE, "Error, must specify qa or total_charge");
    }
    return OSC_OK;
}

inline DepositArgs deposit_args(const osc_mesh3d *m, const int n[3], int64_t np, const double *x, const double *y,
                         const double *z, const double *q, double charge1, int check_finite) {
    DepositArgs a;
    std::memset(&a, 0, sizeof(a));
    a.np = np;
    a.x = x; a.y = y; a.z = z; a.q = q; a.lost = nullptr;
    a.xmin = m->min[0]; a.ymin = m->min[1]; a.zmin = m->min[2];
    a.dx = m->delta[0]; a.dy = m->delta[1]; a.dz = m->delta[2];
    a.dxi = 1.0 / a.dx; a.dyi = 1.0 / a.dy; a.dzi = 1.0 / a.dz;
    for (int d = 0; d < 3; ++d) {
        a.nlo[d] = m->nlo[d];
        a.nhi[d] = m->nhi[d];
        a.nlogbl[d] = m->nlo[d];
    }
    a.nx = n[0]; a.ny = n[1]; a.nz = n[2];
    a.mode = 0;
    a.charge1 = charge1;
    a.check_finite = check_finite;
    return a;
}

// Counting sort of a's particles by deposit cell (cell_sort.cuh) into xs, ys, zs, qs (qs
// when a.q is set); perm64[pos] = original index and inv[m] = sorted position, each when
// non-null.  Five kernels: keys, three scan passes, scatter.
inline int cell_sort(osc_ctx *ctx, const DepositArgs &a, double *xs, double *ys, double *zs, double *qs,
                     int64_t *perm64, uint32_t *inv) {
    if (a.np >= (int64_t)0xffffffff) return set_err(ctx, OSC_E_UNSUPPORTED, "cell sort: at most 2^32 - 2 particles");
    if (a.mode != 0 || a.lost) return set_err(ctx, OSC_E_INVALID, "cell sort: deposit_particles cells only");
    const int64_t N = (int64_t)a.nx * a.ny * a.nz;
    uint32_t *keys, *ranks, *counts, *parts;
    TRY(ws_get(ctx, "cs_keys", sizeof(uint32_t) * (size_t)a.np, (void **)&keys));
    TRY(ws_get(ctx, "cs_ranks", sizeof(uint32_t) * (size_t)a.np, (void **)&ranks));
    TRY(ws_get(ctx, "cs_counts", sizeof(uint32_t) * (size_t)(N + 2), (void **)&counts));
    TRY(ws_get(ctx, "cs_parts", sizeof(uint32_t) * (size_t)cell_scan_partials(N + 2), (void **)&parts));
    CK(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)(N + 2), ctx->stream), "memset cell counts");
    // the sort's own outside/non-finite counts go to scratch words 24-25 (the deposit counts)
    CK(cudaMemsetAsync(ctx->d_small + 24, 0, 2 * sizeof(unsigned long long), ctx->stream), "memset sort counters");
    {
        Launch L_(ctx, "cell_keys");
        if (launch_cell_keys(a, keys, ranks, counts, ctx->d_small + 24, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "cell keys");
    }
    {
        Launch L_(ctx, "cell_scan", 3);
        if (launch_cell_scan(counts, N + 2, parts, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "cell scan");
    }
    Launch L_(ctx, "cell_scatter");
    if (launch_cell_scatter(a.np, keys, ranks, counts, a.x, a.y, a.z, a.q, xs, ys, zs, qs, perm64, inv, ctx->stream))
        return set_err(ctx, OSC_E_CUDA, "cell scatter");
    return OSC_OK;
}

// a's particles sorted by cell into the named workspaces "<prefix>x" ...; a then points at
// the copies.  inv (nullable) receives the original-to-sorted map.
inline int cell_sort_ws(osc_ctx *ctx, DepositArgs &a, const char *prefix, uint32_t **inv) {
    double *xs, *ys, *zs, *qs = nullptr;
    const std::string p(prefix);
    const size_t b = sizeof(double) * (size_t)a.np;
    TRY(ws_get(ctx, (p + "x").c_str(), b, (void **)&xs));
    TRY(ws_get(ctx, (p + "y").c_str(), b, (void **)&ys));
    TRY(ws_get(ctx, (p + "z").c_str(), b, (void **)&zs));
    if (a.q) TRY(ws_get(ctx, (p + "q").c_str(), b, (void **)&qs));
    uint32_t *iv = nullptr;
    if (inv) TRY(ws_get(ctx, (p + "inv").c_str(), sizeof(uint32_t) * (size_t)a.np, (void **)&iv));
    TRY(cell_sort(ctx, a, xs, ys, zs, qs, nullptr, iv));
    a.x = xs;
    a.y = ys;
    a.z = zs;
    a.q = qs;
    if (inv) *inv = iv;
    return OSC_OK;
}

// Deposition of a.np particles into rho (zeroed here).  OSC_DEPOSIT_ATOMIC uses
// floating-point atomics of the type of rho; OSC_DEPOSIT_DETERMINISTIC accumulates 64-bit
// fixed-point integers and converts once, so rho is bit-identical for any particle order;
// OSC_DEPOSIT_SORTED_SEGMENT gives the same bits from particles in cell order (sorted here
// unless cell_ordered says the caller's order already is), each run of equal cells summed
// exactly in registers before its reductions.  The fixed-point unit is a power of two
// chosen from np * max|q| (order-independent), so that no node sum can exceed 2^62 units.
// rho = mult * sum.
template <typename TR>
inline int deposit_rho(osc_ctx *ctx, DepositArgs a, TR *rho, int64_t N, double mult, bool cell_ordered = false) {
    if (ctx->deposit_mode == OSC_DEPOSIT_ATOMIC) {
        CK(cudaMemsetAsync(rho, 0, sizeof(TR) * N, ctx->stream), "memset rho");
        {
            Launch L_(ctx, sizeof(TR) == 8 ? "deposit_f64" : "deposit_f32");
            if (launch_deposit<TR>(a, rho, ctx->d_small, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "deposit");
        }
        if (mult != 1.0) {
            if constexpr (sizeof(TR) == 8) {
                Launch L_(ctx, "scale");
                if (launch_scale(rho, mult, N, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "scale");
            } else {
                return set_err(ctx, OSC_E_INVALID, "scaled FP32 deposit");
            }
        }
        return OSC_OK;
    }
    double qmax;
    if (a.mode == 0 && a.q) {
        double *out;
        TRY(ws_get(ctx, "qmax", sizeof(double), (void **)&out));
        {
            Launch L_(ctx, "charge_max", 2);
            if (launch_sum(a.np, a.q, ctx->d_partials, out, ctx->stream, true))
                return set_err(ctx, OSC_E_CUDA, "charge max");
        }
        TRY(d2h(ctx, &qmax, out, sizeof(double)));
        TRY(sync(ctx));
    } else {
        qmax = a.mode == 0 ? std::fabs(a.charge1) : 1.0;
    }
    const double bound = (double)a.np * qmax;  // >= sum of |contributions| at any node
    a.fx_scale = 1.0;
    if (bound > 0 && std::isfinite(bound)) {
        int e;
        std::frexp(bound, &e);  // bound < 2^e
        a.fx_scale = std::ldexp(1.0, 62 - e);
    }
    unsigned long long *acc;
    TRY(ws_get(ctx, "rho_fixed", sizeof(unsigned long long) * N, (void **)&acc));
    CK(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * N, ctx->stream), "memset fixed");
    if (ctx->deposit_mode == OSC_DEPOSIT_SORTED_SEGMENT && a.mode == 0 && !a.lost) {
        if (!cell_ordered) TRY(cell_sort_ws(ctx, a, "dsort_", nullptr));
        Launch L_(ctx, "deposit_fixed_runs");
        if (launch_deposit_fixed_runs(a, acc, ctx->d_small, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "deposit");
    } else {
        Launch L_(ctx, "deposit_fixed");
        if (launch_deposit<unsigned long long>(a, acc, ctx->d_small, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "deposit");
    }
    {
        Launch L_(ctx, "fixed_to_real");
        if (launch_fixed_to_real<TR>(acc, rho, a.fx_scale, mult, N, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "fixed to real");
    }
    return OSC_OK;
}

inline InterpArgs interp_args(const osc_mesh3d *m, const int n[3], int64_t np, const double *x, const double *y,
                       const double *z) {
    InterpArgs a;
    a.np = np;
    a.x = x; a.y = y; a.z = z;
    for (int d = 0; d < 3; ++d) {
        a.min[d] = m->min[d];
        a.delta[d] = m->delta[d];
        a.hinv[d] = 1.0 / m->delta[d];
        a.nlo[d] = m->nlo[d];
        a.nhi[d] = m->nhi[d];
    }
    a.nx = n[0]; a.ny = n[1]; a.nz = n[2];
    return a;
}

inline int counters_reset(osc_ctx *ctx) {
    return cuda_check(ctx, cudaMemsetAsync(ctx->d_small, 0, sizeof(unsigned long long) * 8, ctx->stream), "memset counters");
}
// counters: [0] outside, [1] non-finite, [2] clamped
inline int counters_read(osc_ctx *ctx, unsigned long long out[3]) {
    TRY(d2h(ctx, ctx->h_small, ctx->d_small, sizeof(unsigned long long) * 3));
    TRY(sync(ctx));
    for (int i = 0; i < 3; ++i) out[i] = ctx->h_small[i];
    return OSC_OK;
}

inline FreeSpaceJob fs_job(const osc_mesh3d *mesh, const int n[3], const double *offset, int at_cathode, int calc_b) {
    FreeSpaceJob j;
    j.nx = n[0]; j.ny = n[1]; j.nz = n[2];
    for (int d = 0; d < 3; ++d) {
        j.delta[d] = mesh->delta[d];
        j.offset[d] = offset ? offset[d] : 0.0;
    }
    j.gamma = mesh->gamma;
    j.at_cathode = at_cathode ? 1 : 0;
    // offset0(3) + 2*min(3) + (max(3)-min(3)) (code/open_spacecharge_mod.f90:472)
    j.img_zoff = 2 * mesh->min[2] + (mesh->max[2] - mesh->min[2]);
    j.calc_b = calc_b ? 1 : 0;
    if (calc_b) {
        const double beta = std::sqrt(1 - 1 / (mesh->gamma * mesh->gamma));
        j.bcoef = beta / c_light_sc3d();
    }
    return j;
}

inline int run_freespace(osc_ctx *ctx, const FreeSpaceJob &j, const double *d_rho, int precision) {
    switch (precision) {
    case OSC_PREC_FP32: return freespace_opt<float, double>(ctx, j, d_rho);
    case OSC_PREC_FP64: return freespace_opt<double, double>(ctx, j, d_rho);
    default: return freespace_plain(ctx, j, d_rho);
    }
}

}  // namespace osc_abi
