// abi.cu -- extern "C" entry points of libopensc_b200.so (declared in include/opensc_gpu.h).
#include <cmath>
#include <cstring>
#include <new>

#include "abi_util.cuh"

using namespace osc;
using namespace osc_abi;


extern "C" {

const char *osc_version(void) { return "opensc_b200 0.1.0 (sm_100a)"; }

int osc_ctx_create(int device, osc_ctx **out) {
    if (!out) return OSC_E_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return OSC_E_CUDA;
    }
    if (device < 0 || device >= ndev) return OSC_E_INVALID;
    osc_ctx *ctx = new (std::nothrow) osc_ctx();
    if (!ctx) return OSC_E_ALLOC;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_small, sizeof(unsigned long long) * 64) != cudaSuccess ||
        cudaMallocHost(&ctx->h_small, sizeof(unsigned long long) * 64) != cudaSuccess ||
        cudaMalloc(&ctx->d_partials, sizeof(double) * 1024) != cudaSuccess ||
        cudaHostAlloc((void **)&ctx->h_fault, sizeof(unsigned), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&ctx->d_fault, ctx->h_fault, 0) != cudaSuccess) {
        cudaGetLastError();
        osc_ctx_destroy(ctx);
        return OSC_E_CUDA;
    }
    *ctx->h_fault = 0;
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return OSC_OK;
}

int osc_ctx_destroy(osc_ctx *ctx) {
    if (!ctx) return OSC_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->batch_plans.clear();  // graph executables and their buffers
    for (auto &kv : ctx->ws) cudaFree(kv.second.p);
    for (auto &kv : ctx->tw32) cudaFree(kv.second.p);
    for (auto &kv : ctx->tw64) cudaFree(kv.second.p);
    gcache_free_all(ctx);
    for (int t = 0; t < 4; ++t) cudaFree(ctx->pipe.g[t].p);
    cudaFree(ctx->pipe.comb.p);
    for (auto &r : ctx->prof_pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->d_small) cudaFree(ctx->d_small);
    if (ctx->h_small) cudaFreeHost(ctx->h_small);
    if (ctx->d_partials) cudaFree(ctx->d_partials);
    if (ctx->h_fault) cudaFreeHost(ctx->h_fault);
    for (auto s : ctx->aux) cudaStreamDestroy(s);
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
    if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
    for (auto e : ctx->copy_ev) cudaEventDestroy(e);
    for (auto e : ctx->aux_ev) cudaEventDestroy(e);
    if (ctx->switch_ev) cudaEventDestroy(ctx->switch_ev);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return OSC_OK;
}

const char *osc_last_error(const osc_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int osc_ctx_set_stream(osc_ctx *ctx, void *s) {
    if (!ctx) return OSC_E_INVALID;
    cudaStream_t ns = s == OSC_OWN_STREAM ? ctx->own_stream : (cudaStream_t)s;
    if (ns != ctx->stream) {
        // work on the new stream starts after everything issued on the old one: the context's
        // workspaces and Green buffers are reused without further synchronisation
        if (!ctx->switch_ev && cudaEventCreateWithFlags(&ctx->switch_ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            ctx->switch_ev = nullptr;
            return set_err(ctx, OSC_E_CUDA, "set_stream: event creation failed");
        }
        if (cudaEventRecord(ctx->switch_ev, ctx->stream) != cudaSuccess ||
            cudaStreamWaitEvent(ns, ctx->switch_ev, 0) != cudaSuccess) {
            cudaGetLastError();
            return set_err(ctx, OSC_E_CUDA, "set_stream: ordering the new stream after the old one failed");
        }
    }
    ctx->stream = ns;
    return OSC_OK;
}

int osc_ctx_set_option(osc_ctx *ctx, int option, int64_t v) {
    if (!ctx) return OSC_E_INVALID;
    switch (option) {
    case OSC_OPT_PRECISION: TRY(check_prec(ctx, (int)v)); ctx->precision = (int)v; return OSC_OK;
    case OSC_OPT_DEPOSIT_MODE:
        if (v != OSC_DEPOSIT_ATOMIC && v != OSC_DEPOSIT_DETERMINISTIC && v != OSC_DEPOSIT_SORTED_SEGMENT)
            return bad(ctx, "deposit mode");
        ctx->deposit_mode = (int)v;
        return OSC_OK;
    case OSC_OPT_PARTICLE_ORDER:
        if (v != OSC_ORDER_ANY && v != OSC_ORDER_CELL_SORTED && v != OSC_ORDER_SORT) return bad(ctx, "particle order");
        ctx->particle_order = (int)v;
        return OSC_OK;
    case OSC_OPT_STRICT_BOUNDS: ctx->strict_bounds = v ? 1 : 0; return OSC_OK;
    case OSC_OPT_GREEN_CACHE_MB: ctx->gcache_budget = (size_t)(v < 0 ? 0 : v) << 20; return OSC_OK;
    case OSC_OPT_PROFILE: ctx->profile = v ? 1 : 0; return OSC_OK;
    case OSC_OPT_CHECK_FINITE: ctx->check_finite = v ? 1 : 0; return OSC_OK;
    case OSC_OPT_TEST_WAIT_TIMEOUT: ctx->test_wait_timeout = v ? 1 : 0; return OSC_OK;
    case OSC_OPT_BATCH_GRAPH: ctx->batch_graph = v ? 1 : 0; return OSC_OK;
    case OSC_OPT_VJP_REUSE_FORWARD: ctx->vjp_reuse = v ? 1 : 0; return OSC_OK;
    default: return bad(ctx, "unknown option");
    }
}

int osc_ctx_get_option(osc_ctx *ctx, int option, int64_t *v) {
    if (!ctx || !v) return OSC_E_INVALID;
    switch (option) {
    case OSC_OPT_PRECISION: *v = ctx->precision; return OSC_OK;
    case OSC_OPT_DEPOSIT_MODE: *v = ctx->deposit_mode; return OSC_OK;
    case OSC_OPT_PARTICLE_ORDER: *v = ctx->particle_order; return OSC_OK;
    case OSC_OPT_STRICT_BOUNDS: *v = ctx->strict_bounds; return OSC_OK;
    case OSC_OPT_GREEN_CACHE_MB: *v = (int64_t)(ctx->gcache_budget >> 20); return OSC_OK;
    case OSC_OPT_PROFILE: *v = ctx->profile; return OSC_OK;
    case OSC_OPT_CHECK_FINITE: *v = ctx->check_finite; return OSC_OK;
    case OSC_OPT_TEST_WAIT_TIMEOUT: *v = ctx->test_wait_timeout; return OSC_OK;
    case OSC_OPT_BATCH_GRAPH: *v = ctx->batch_graph; return OSC_OK;
    case OSC_OPT_VJP_REUSE_FORWARD: *v = ctx->vjp_reuse; return OSC_OK;
    default: return bad(ctx, "unknown option");
    }
}

// Tuning keys and their allowed values: the launch shapes the kernels accept.
static bool tuning_value_ok(const std::string &key, int v) {
    if (key == "deposit_run" || key == "gather_run") return v == 0 || v == 4 || v == 8;
    if (key == "deposit_ctas_per_sm" || key == "gather_ctas_per_sm" || key == "deposit_runs_ctas_per_sm" ||
        key == "gather_runs_ctas_per_sm")
        return v == 0 || v == 4 || v == 8 || v == 16 || v == 32 || v == 64 || v == 128;
    if (key.rfind("lines_nl_div:", 0) == 0 || key.rfind("r2c_nl_div:", 0) == 0 || key.rfind("c2r_nl_div:", 0) == 0)
        return v == 0 || v == 1 || v == 2;
    if (key.rfind("zconv_engine:", 0) == 0) return v == 0 || v == 1 || v == 2;
    if (key.rfind("sym_nl_div:", 0) == 0) return v == 0 || v == 1 || v == 2 || v == 4;
    if (key == "batch_copy_chunks") return v >= 0 && v <= 16;
    return false;
}

int osc_ctx_set_tuning(osc_ctx *ctx, const char *key, int value) {
    if (!ctx || !key) return OSC_E_INVALID;
    const std::string k(key);
    if (!tuning_value_ok(k, value)) return set_err(ctx, OSC_E_INVALID, "tuning %s = %d is not a valid choice", key, value);
    if (value == 0) ctx->tuning.erase(k);  // the built-in default
    else ctx->tuning[k] = value;
    ++ctx->tune_gen;
    return OSC_OK;
}

int osc_ctx_get_tuning(osc_ctx *ctx, const char *key, int *value) {
    if (!ctx || !key || !value) return OSC_E_INVALID;
    *value = tune_get(ctx, key, 0);
    return OSC_OK;
}

int osc_ctx_synchronize(osc_ctx *ctx) {
    if (!ctx) return OSC_E_INVALID;
    return sync(ctx);
}

int osc_clear_green_cache(osc_ctx *ctx) {
    if (!ctx) return OSC_E_INVALID;
    TRY(sync(ctx));
    gcache_free_all(ctx);
    return OSC_OK;
}

int osc_profile_reset(osc_ctx *ctx) {
    if (!ctx) return OSC_E_INVALID;
    prof_flush(ctx);
    ctx->prof.clear();
    return OSC_OK;
}
int osc_profile_count(osc_ctx *ctx, int *n) {
    if (!ctx || !n) return OSC_E_INVALID;
    prof_flush(ctx);
    *n = (int)ctx->prof.size();
    return OSC_OK;
}
int osc_profile_entry(osc_ctx *ctx, int i, const char **name, int64_t *launches, double *ms) {
    if (!ctx) return OSC_E_INVALID;
    prof_flush(ctx);
    if (i < 0 || i >= (int)ctx->prof.size()) return OSC_E_INVALID;
    auto it = ctx->prof.begin();
    std::advance(it, i);
    if (name) *name = it->first.c_str();
    if (launches) *launches = it->second.launches;
    if (ms) *ms = it->second.ms;
    return OSC_OK;
}
int osc_launch_count(osc_ctx *ctx, int64_t *n) {
    if (!ctx || !n) return OSC_E_INVALID;
    *n = ctx->launches;
    return OSC_OK;
}
int osc_graph_launch_count(osc_ctx *ctx, int64_t *n) {
    if (!ctx || !n) return OSC_E_INVALID;
    *n = ctx->graph_launches;
    return OSC_OK;
}

// ---------------------------------------------------------------------------------------
int osc_sort_particles_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int64_t np, const double *x, const double *y,
                           const double *z, const double *q, double *xs, double *ys, double *zs, double *qs,
                           int64_t *perm, int64_t *n_outside) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (np < 0 || (np > 0 && (!x || !y || !z || !xs || !ys || !zs))) return bad(ctx, "sort arrays");
    if ((q == nullptr) != (qs == nullptr)) return bad(ctx, "q and qs must both be given or both be NULL");
    if (np > 0 && (xs == x || ys == y || zs == z || (q && qs == q)))
        return bad(ctx, "sorted copies must not alias the input arrays");
    if (!(mesh->delta[0] > 0 && mesh->delta[1] > 0 && mesh->delta[2] > 0)) return bad(ctx, "mesh delta must be positive");
    if (n_outside) *n_outside = 0;
    if (np == 0) return OSC_OK;
    DepositArgs a = deposit_args(mesh, n, np, x, y, z, q, 0.0, 1);
    TRY(cell_sort(ctx, a, xs, ys, zs, qs, perm, nullptr));
    if (n_outside) {
        unsigned long long h[2];
        TRY(d2h(ctx, h, ctx->d_small + 24, sizeof(h)));
        TRY(sync(ctx));
        *n_outside = (int64_t)(h[0] + h[1]);
    }
    return OSC_OK;
}

// ---------------------------------------------------------------------------------------
int osc_deposit_particles_dev(osc_ctx *ctx, int64_t np, const double *x, const double *y, const double *z,
                              const double *q, const double *total_charge, int resize_mesh, osc_mesh3d *mesh,
                              double *rho, int64_t *n_outside) {
    if (!ctx) return OSC_E_INVALID;
    if (np < 0 || (np > 0 && (!x || !y || !z)) || !rho) return bad(ctx, "deposit arrays");
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (resize_mesh) TRY(refit_mesh(ctx, np, x, y, z, mesh));
    double charge1 = 0;
    if (np == 0 && !q && total_charge) {
        mesh->charge = *total_charge;
    } else {
        TRY(set_charge(ctx, np, q, total_charge, mesh, &charge1));
    }
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    TRY(counters_reset(ctx));
    DepositArgs a = deposit_args(mesh, n, np, x, y, z, q, charge1, ctx->check_finite);
    TRY(deposit_rho<double>(ctx, a, rho, N, 1.0, ctx->particle_order == OSC_ORDER_CELL_SORTED));
    if (n_outside || ctx->strict_bounds || ctx->check_finite) {
        unsigned long long cnt[3];
        TRY(counters_read(ctx, cnt));
        if (n_outside) *n_outside = (int64_t)cnt[0];
        if (ctx->check_finite && cnt[1]) return set_err(ctx, OSC_E_NAN, "%llu non-finite particles", cnt[1]);
        if (ctx->strict_bounds && cnt[0]) return set_err(ctx, OSC_E_BOUNDS, "%llu particles outside the mesh", cnt[0]);
    }
    return OSC_OK;
}

int osc_deposit_particles(osc_ctx *ctx, int64_t np, const double *xa, const double *ya, const double *za,
                          const double *qa, const double *total_charge, int resize_mesh, osc_mesh3d *mesh,
                          double *rho, int64_t *n_outside) {
    if (!ctx) return OSC_E_INVALID;
    if (np < 0 || (np > 0 && (!xa || !ya || !za)) || !rho) return bad(ctx, "deposit arrays");
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (!qa && !total_charge) return set_err(ctx, OSC_E_NOCHARGE, "Error, must specify qa or total_charge");
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    double *dx, *dy, *dz, *dq, *drho;
    TRY(stage_in(ctx, "h_x", xa, np, &dx));
    TRY(stage_in(ctx, "h_y", ya, np, &dy));
    TRY(stage_in(ctx, "h_z", za, np, &dz));
    TRY(stage_in(ctx, "h_q", qa, np, &dq));
    TRY(ws_get(ctx, "h_rho", sizeof(double) * N, (void **)&drho));
    int64_t nout = 0;
    TRY(osc_deposit_particles_dev(ctx, np, dx, dy, dz, dq, total_charge, resize_mesh, mesh, drho, &nout));
    TRY(d2h(ctx, rho, drho, sizeof(double) * N));
    TRY(sync(ctx));
    if (n_outside) *n_outside = nout;
    return OSC_OK;
}

int osc_get_mesh_quantities(osc_ctx *ctx, int64_t np, const double *xa, const double *ya, const double *za,
                            const int32_t nlo[3], const int32_t nhi[3], int isetzmin, double delta[3],
                            double umin[3]) {
    if (!ctx) return OSC_E_INVALID;
    if (np < 0 || (np > 0 && (!xa || !ya || !za)) || !nlo || !nhi || !delta || !umin) return bad(ctx, "mesh quantities");
    // getbeamboundingbox (code/test_mod.f90:366): host min/max, as the arrays are host arrays
    double sml[3], big[3];
    const double *p[3] = {xa, ya, za};
    for (int d = 0; d < 3; ++d) {
        if (np > 0) {
            double lo = p[d][0], hi = p[d][0];
            for (int64_t m = 1; m < np; ++m) {
                if (p[d][m] < lo) lo = p[d][m];
                if (p[d][m] > hi) hi = p[d][m];
            }
            sml[d] = lo;
            big[d] = hi;
        } else {
            sml[d] = 9999999.;
            big[d] = -9999999.;
        }
    }
    const double eps = 1.e-13;
    for (int d = 0; d < 3; ++d) {
        big[d] = big[d] * (1.0 + std::copysign(1.0, big[d]) * eps);
        sml[d] = sml[d] * (1.0 - std::copysign(1.0, sml[d]) * eps);
        const int nn = nhi[d] - nlo[d] + 1;
        if (nn <= 3) return set_err(ctx, OSC_E_INVALID, "get_mesh_quantities needs more than 3 nodes per axis");
        delta[d] = (big[d] - sml[d]) / (double)(nn - 3);
        umin[d] = sml[d] - delta[d];
    }
    if (isetzmin == 1) {
        const int nz = nhi[2] - nlo[2] + 1;
        const double zsml = 1.e-9;
        delta[2] = (big[2] - zsml) / (double)(nz - 1);
        umin[2] = zsml;
    }
    return OSC_OK;
}

int osc_depose_rho_scalar(osc_ctx *ctx, int64_t np, const double *xa, const double *ya, const double *za,
                          const double *lostflag, double chrgpermacro, const int32_t nlo[3], const int32_t nhi[3],
                          const double delta[3], const double umin[3], double *rho, int64_t *ifail) {
    if (!ctx) return OSC_E_INVALID;
    if (np < 0 || (np > 0 && (!xa || !ya || !za)) || !rho || !nlo || !nhi || !delta || !umin) return bad(ctx, "depose");
    osc_mesh3d m;
    std::memset(&m, 0, sizeof(m));
    for (int d = 0; d < 3; ++d) {
        m.nlo[d] = nlo[d];
        m.nhi[d] = nhi[d];
        m.min[d] = umin[d];
        m.delta[d] = delta[d];
    }
    int n[3];
    TRY(mesh_dims(ctx, &m, n));
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    double *dx, *dy, *dz, *dl, *drho;
    TRY(stage_in(ctx, "h_x", xa, np, &dx));
    TRY(stage_in(ctx, "h_y", ya, np, &dy));
    TRY(stage_in(ctx, "h_z", za, np, &dz));
    TRY(stage_in(ctx, "h_q", lostflag, np, &dl));
    TRY(ws_get(ctx, "h_rho", sizeof(double) * N, (void **)&drho));
    TRY(counters_reset(ctx));
    DepositArgs a = deposit_args(&m, n, np, dx, dy, dz, nullptr, 1.0, 0);
    a.lost = dl;
    a.mode = 1;
    TRY(deposit_rho<double>(ctx, a, drho, N, chrgpermacro));
    TRY(d2h(ctx, rho, drho, sizeof(double) * N));
    unsigned long long cnt[3];
    TRY(counters_read(ctx, cnt));
    if (ifail) *ifail = (int64_t)cnt[0];
    return OSC_OK;
}

// ---------------------------------------------------------------------------------------
int osc_space_charge_3d_dev(osc_ctx *ctx, const osc_mesh3d *mesh, const double *d_rho, const double *offset,
                            int at_cathode, int calc_bfield, int precision, double *d_efield, double *d_bfield) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    TRY(check_prec(ctx, precision));
    if (!d_rho || !d_efield || (calc_bfield && !d_bfield)) return bad(ctx, "space_charge_3d arrays");
    if (!(mesh->gamma >= 1.0)) return set_err(ctx, OSC_E_INVALID, "gamma must be >= 1");
    FreeSpaceJob j = fs_job(mesh, n, offset, at_cathode, calc_bfield);
    j.E = d_efield;
    j.B = calc_bfield ? d_bfield : nullptr;
    return run_freespace(ctx, j, d_rho, precision);
}

int osc_space_charge_3d(osc_ctx *ctx, const osc_mesh3d *mesh, const double *rho, const double *offset,
                        int at_cathode, int calc_bfield, int precision, double *efield, double *bfield) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (!rho || !efield || (calc_bfield && !bfield)) return bad(ctx, "space_charge_3d arrays");
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    double *drho, *dE, *dB = nullptr;
    TRY(stage_in(ctx, "h_rho", rho, N, &drho));
    TRY(ws_get(ctx, "h_E", sizeof(double) * 3 * N, (void **)&dE));
    if (calc_bfield) TRY(ws_get(ctx, "h_B", sizeof(double) * 3 * N, (void **)&dB));
    TRY(osc_space_charge_3d_dev(ctx, mesh, drho, offset, at_cathode, calc_bfield, precision, dE, dB));
    TRY(d2h(ctx, efield, dE, sizeof(double) * 3 * N));
    if (calc_bfield) TRY(d2h(ctx, bfield, dB, sizeof(double) * 3 * N));
    return sync(ctx);
}

int osc_freespace_solver2(osc_ctx *ctx, const int32_t n3[3], const double *rho, double gamma, const double delta[3],
                          const double *offset, int precision, double *efield, double *phi) {
    if (!ctx) return OSC_E_INVALID;
    if (!n3 || !rho || !delta || (!efield && !phi)) return bad(ctx, "freespace_solver2 arguments");
    TRY(check_prec(ctx, precision));
    osc_mesh3d m;
    std::memset(&m, 0, sizeof(m));
    for (int d = 0; d < 3; ++d) {
        m.nlo[d] = 1;
        m.nhi[d] = n3[d];
        m.delta[d] = delta[d];
    }
    m.gamma = gamma;
    int n[3];
    TRY(mesh_dims(ctx, &m, n));
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    double *drho, *dE = nullptr, *dP = nullptr;
    TRY(stage_in(ctx, "h_rho", rho, N, &drho));
    if (efield) TRY(ws_get(ctx, "h_E", sizeof(double) * 3 * N, (void **)&dE));
    if (phi) TRY(ws_get(ctx, "h_phi", sizeof(double) * N, (void **)&dP));
    FreeSpaceJob j = fs_job(&m, n, offset, 0, 0);
    j.want_phi = phi ? 1 : 0;
    j.want_e = efield ? 1 : 0;
    j.E = dE;
    j.phi = dP;
    TRY(run_freespace(ctx, j, drho, precision));
    if (efield) TRY(d2h(ctx, efield, dE, sizeof(double) * 3 * N));
    if (phi) TRY(d2h(ctx, phi, dP, sizeof(double) * N));
    return sync(ctx);
}

// ---------------------------------------------------------------------------------------
int osc_interpolate_field_dev(osc_ctx *ctx, const osc_mesh3d *mesh, const double *d_efield, const double *d_bfield,
                              int64_t np, const double *x, const double *y, const double *z, double *E, double *B,
                              int64_t *n_clamped) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (np < 0 || (np > 0 && (!x || !y || !z))) return bad(ctx, "interpolate arrays");
    if ((d_efield && !E) || (d_bfield && !B)) return bad(ctx, "interpolate outputs");
    TRY(counters_reset(ctx));
    InterpArgs a = interp_args(mesh, n, np, x, y, z);
    if (d_efield && E) {
        Launch L_(ctx, "interp_f64");
        if (launch_interp_planes(a, d_efield, E, ctx->d_small + 2, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
    }
    if (d_bfield && B) {
        Launch L_(ctx, "interp_f64");
        if (launch_interp_planes(a, d_bfield, B, ctx->d_small + 3, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
    }
    if (n_clamped) {
        unsigned long long cnt[3];
        TRY(counters_read(ctx, cnt));
        *n_clamped = (int64_t)cnt[2];
    }
    return OSC_OK;
}

int osc_interpolate_field(osc_ctx *ctx, const osc_mesh3d *mesh, const double *efield, const double *bfield,
                          int64_t np, const double *x, const double *y, const double *z, double *E, double *B,
                          int64_t *n_clamped) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (np < 0 || (np > 0 && (!x || !y || !z))) return bad(ctx, "interpolate arrays");
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    double *dx, *dy, *dz, *dE = nullptr, *dB = nullptr, *oE = nullptr, *oB = nullptr;
    TRY(stage_in(ctx, "h_x", x, np, &dx));
    TRY(stage_in(ctx, "h_y", y, np, &dy));
    TRY(stage_in(ctx, "h_z", z, np, &dz));
    if (efield && E) {
        TRY(stage_in(ctx, "h_E", efield, 3 * N, &dE));
        TRY(ws_get(ctx, "h_pE", sizeof(double) * 3 * (size_t)np, (void **)&oE));
    }
    if (bfield && B) {
        TRY(stage_in(ctx, "h_B", bfield, 3 * N, &dB));
        TRY(ws_get(ctx, "h_pB", sizeof(double) * 3 * (size_t)np, (void **)&oB));
    }
    int64_t ncl = 0;
    TRY(osc_interpolate_field_dev(ctx, mesh, dE, dB, np, dx, dy, dz, oE, oB, &ncl));
    if (oE) TRY(d2h(ctx, E, oE, sizeof(double) * 3 * np));
    if (oB) TRY(d2h(ctx, B, oB, sizeof(double) * 3 * np));
    TRY(sync(ctx));
    if (n_clamped) *n_clamped = ncl;
    return OSC_OK;
}

// ---------------------------------------------------------------------------------------
int osc_space_charge_step_dev(osc_ctx *ctx, osc_mesh3d *mesh, int64_t np, const double *x, const double *y,
                              const double *z, const double *q, const double *total_charge, int resize_mesh,
                              int at_cathode, int precision, double *E, double *B) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    TRY(check_prec(ctx, precision));
    if (np <= 0 || !x || !y || !z || !E) return bad(ctx, "step arrays");
    if (!q && !total_charge) return set_err(ctx, OSC_E_NOCHARGE, "Error, must specify qa or total_charge");
    if (!(mesh->gamma >= 1.0)) return set_err(ctx, OSC_E_INVALID, "gamma must be >= 1");
    ++ctx->step_calls;  // any earlier step's kept E grid is out of date from here on
    if (resize_mesh) TRY(refit_mesh(ctx, np, x, y, z, mesh));
    double charge1 = 0;
    if (q) TRY(set_charge(ctx, np, q, total_charge, mesh, &charge1));
    else {
        mesh->charge = *total_charge;
        charge1 = *total_charge / (double)np;
    }
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    TRY(counters_reset(ctx));
    DepositArgs da = deposit_args(mesh, n, np, x, y, z, q, charge1, ctx->check_finite);
    InterpArgs ia = interp_args(mesh, n, np, x, y, z);
    FreeSpaceJob j = fs_job(mesh, n, nullptr, at_cathode, B != nullptr);
    // launch shapes from the autotuner (per-particle kernels in any order, run kernels in
    // cell order)
    const bool runs = ctx->particle_order != OSC_ORDER_ANY;
    da.tile = tune_get(ctx, "deposit_run");
    ia.tile = tune_get(ctx, "gather_run");
    da.ctas = tune_get(ctx, runs ? "deposit_runs_ctas_per_sm" : "deposit_ctas_per_sm");
    ia.ctas = tune_get(ctx, runs ? "gather_runs_ctas_per_sm" : "gather_ctas_per_sm");
    if (precision == OSC_PREC_FP64_PLAIN) {
        double *rho, *Eg, *Bg = nullptr;
        TRY(ws_get(ctx, "st_rho64", sizeof(double) * N, (void **)&rho));
        TRY(ws_get(ctx, "st_Eg", sizeof(double) * 3 * N, (void **)&Eg));
        if (B) TRY(ws_get(ctx, "st_Bg", sizeof(double) * 3 * N, (void **)&Bg));
        TRY(deposit_rho<double>(ctx, da, rho, N, 1.0, ctx->particle_order == OSC_ORDER_CELL_SORTED));
        j.E = Eg;
        j.B = Bg;
        TRY(freespace_plain(ctx, j, rho));
        {
            Launch L_(ctx, "interp_f64");
            if (launch_interp_planes(ia, Eg, E, ctx->d_small + 2, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
        }
        if (B) {
            Launch L_(ctx, "interp_f64");
            if (launch_interp_planes(ia, Bg, B, ctx->d_small + 3, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
        }
        return OSC_OK;
    }
    if (precision == OSC_PREC_FP32) {
        // deposit: two float4 atomics per particle into a quad grid, summed to nodes in a
        // fixed order by the x transform's loads; field: E written as an x-pair grid;
        // interpolation: 4 sectors/particle.  Particles in cell order (the caller's, or
        // sorted here) deposit per run of equal cells and gather from shared sectors.
        const int order = ctx->particle_order;
        uint32_t *inv = nullptr;
        if (order == OSC_ORDER_SORT) {
            TRY(cell_sort_ws(ctx, da, "st_s", &inv));
            ia.x = da.x;
            ia.y = da.y;
            ia.z = da.z;
        }
        float *rho = nullptr, *quad;
        void *E8;
        TRY(ws_get(ctx, "st_E8", sizeof(float4) * 2 * N, &E8));
        if (ctx->deposit_mode != OSC_DEPOSIT_ATOMIC) {
            TRY(ws_get(ctx, "st_rho32", sizeof(float) * N, (void **)&rho));
            TRY(deposit_rho<float>(ctx, da, rho, N, 1.0, order != OSC_ORDER_ANY));
        } else {
            TRY(ws_get(ctx, "st_quad", sizeof(float) * 4 * N, (void **)&quad));
            CK(cudaMemsetAsync(quad, 0, sizeof(float) * 4 * N, ctx->stream), "memset quad");
            {
                Launch L_(ctx, order == OSC_ORDER_ANY ? "deposit_f32" : "deposit_f32_runs");
                if ((order == OSC_ORDER_ANY ? launch_deposit_quad(da, quad, ctx->d_small, ctx->stream)
                                            : launch_deposit_quad_runs(da, quad, ctx->d_small, ctx->stream)))
                    return set_err(ctx, OSC_E_CUDA, "deposit");
            }
            j.quad = reinterpret_cast<const float4 *>(quad);
        }
        j.E4 = E8;
        j.e4_pairs = 1;
        j.B = nullptr;
        if (B) {
            double *Bg;
            TRY(ws_get(ctx, "st_Bg", sizeof(double) * 3 * N, (void **)&Bg));
            j.B = Bg;
        }
        TRY(freespace_opt<float, float>(ctx, j, rho));
        if (!at_cathode) {  // the E grid of this free-space step, for the adjoint
            osc_ctx::FwdRecord &f = ctx->fwd;
            f.call = ctx->step_calls;
            f.np = np;
            for (int d = 0; d < 3; ++d) {
                f.nlo[d] = mesh->nlo[d];
                f.nhi[d] = mesh->nhi[d];
                f.min[d] = mesh->min[d];
                f.delta[d] = mesh->delta[d];
            }
            f.gamma = mesh->gamma;
            f.charge1 = charge1;
            f.x = x;
            f.y = y;
            f.z = z;
            f.q = q;
            f.e8 = E8;
        }
        // with the particles sorted here, E and B are gathered in sorted order and then
        // permuted back to the caller's order
        double *Eo = E, *Bo = B;
        if (inv) {
            TRY(ws_get(ctx, "st_sE", sizeof(double) * 3 * (size_t)np, (void **)&Eo));
            if (B) TRY(ws_get(ctx, "st_sB", sizeof(double) * 3 * (size_t)np, (void **)&Bo));
        }
        {
            Launch L_(ctx, order == OSC_ORDER_ANY ? "interp_f32" : "interp_f32_runs");
            if ((order == OSC_ORDER_ANY
                     ? launch_interp_pairs(ia, reinterpret_cast<const float4 *>(E8), Eo, ctx->d_small + 2, ctx->stream)
                     : launch_interp_pairs_runs(ia, reinterpret_cast<const float4 *>(E8), Eo, ctx->d_small + 2,
                                                ctx->stream)))
                return set_err(ctx, OSC_E_CUDA, "interp");
        }
        if (B) {
            Launch L_(ctx, "interp_f64");
            if (launch_interp_planes(ia, j.B, Bo, ctx->d_small + 3, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
        }
        if (inv) {
            Launch L_(ctx, "unpermute", B ? 2 : 1);
            if (launch_unpermute_rows3(np, inv, Eo, E, ctx->stream) ||
                (B && launch_unpermute_rows3(np, inv, Bo, B, ctx->stream)))
                return set_err(ctx, OSC_E_CUDA, "unpermute");
        }
        return OSC_OK;
    }
    // OSC_PREC_FP64: optimised pipeline in double
    double *rho;
    void *E4;
    TRY(ws_get(ctx, "st_rho64", sizeof(double) * N, (void **)&rho));
    TRY(ws_get(ctx, "st_E4d", sizeof(double4) * N, &E4));
    TRY(deposit_rho<double>(ctx, da, rho, N, 1.0, ctx->particle_order == OSC_ORDER_CELL_SORTED));
    j.E4 = E4;
    if (B) {
        double *Bg;
        TRY(ws_get(ctx, "st_Bg", sizeof(double) * 3 * N, (void **)&Bg));
        j.B = Bg;
    }
    TRY(freespace_opt<double, double>(ctx, j, rho));
    {
        Launch L_(ctx, "interp_f64");
        if (launch_interp_vec4<double>(ia, E4, E, ctx->d_small + 2, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
    }
    if (B) {
        Launch L_(ctx, "interp_f64");
        if (launch_interp_planes(ia, j.B, B, ctx->d_small + 3, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
    }
    return OSC_OK;
}

int osc_space_charge_step(osc_ctx *ctx, osc_mesh3d *mesh, int64_t np, const double *x, const double *y,
                          const double *z, const double *q, const double *total_charge, int resize_mesh,
                          int at_cathode, int precision, double *E, double *B) {
    if (!ctx) return OSC_E_INVALID;
    if (np <= 0 || !x || !y || !z || !E) return bad(ctx, "step arrays");
    double *dx, *dy, *dz, *dq, *dE, *dB = nullptr;
    TRY(stage_in(ctx, "h_x", x, np, &dx));
    TRY(stage_in(ctx, "h_y", y, np, &dy));
    TRY(stage_in(ctx, "h_z", z, np, &dz));
    TRY(stage_in(ctx, "h_q", q, np, &dq));
    TRY(ws_get(ctx, "h_pE", sizeof(double) * 3 * (size_t)np, (void **)&dE));
    if (B) TRY(ws_get(ctx, "h_pB", sizeof(double) * 3 * (size_t)np, (void **)&dB));
    TRY(osc_space_charge_step_dev(ctx, mesh, np, dx, dy, dz, dq, total_charge, resize_mesh, at_cathode, precision, dE,
                                  dB));
    TRY(d2h(ctx, E, dE, sizeof(double) * 3 * np));
    if (B) TRY(d2h(ctx, B, dB, sizeof(double) * 3 * np));
    return sync(ctx);
}

}  // extern "C"
