// slab.cu -- one grid solved over several GPUs by z slabs (osc_slab_*, declared in
// include/opensc_gpu.h): the stages a rank runs between the exchanges that the caller
// makes (openspacecharge_b200/slab.py does them with torch.distributed).
//
// The reference's multi-rank prototype distributes the doubled grid over MPI ranks and
// moves it between layouts with all-to-alls (mpi_devel/code/open_spacecharge_mod.f90:
// 722-990, movetodoublesizer2c / movetosinglesizec2r); here a rank keeps the planes
// [z0, z0 + nzl) of the physical grid for the deposit, the x and y transforms, the inverse
// and the gather, and the half-spectrum columns [col0, col0 + ncols) for the z pass.  FP32.
#include "abi_util.cuh"

using namespace osc;
using namespace osc_abi;

namespace {

// The global mesh restricted to planes [p0, p1] of its z nodes (0-based, inclusive).
osc_mesh3d planes_of(const osc_mesh3d &m, int p0, int p1) {
    osc_mesh3d s = m;
    s.nlo[2] = m.nlo[2] + p0;
    s.nhi[2] = m.nlo[2] + p1;
    return s;
}

int check_slab(osc_ctx *ctx, const osc_mesh3d *mesh, int z0, int nzl, int n[3]) {
    TRY(mesh_dims(ctx, mesh, n));
    if (z0 < 0 || nzl < 1 || z0 + nzl > n[2])
        return set_err(ctx, OSC_E_INVALID, "z slab [%d, %d) outside the %d planes", z0, z0 + nzl, n[2]);
    return OSC_OK;
}

}  // namespace

extern "C" {

int osc_slab_deposit_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int z0, int nzl, int64_t np, const double *x,
                         const double *y, const double *z, const double *q, double charge1, float *quad,
                         int64_t *n_outside) {
    if (!ctx || !mesh || !quad) return OSC_E_INVALID;
    int n[3];
    TRY(check_slab(ctx, mesh, z0, nzl, n));
    if (np < 0 || (np > 0 && (!x || !y || !z))) return bad(ctx, "slab deposit arrays");
    // planes z0 .. z0 + nzl, the last one the next slab's first (a ghost plane the caller
    // adds into the next rank's quad grid); the top slab has no next plane
    const int top = z0 + nzl < n[2] ? z0 + nzl : n[2] - 1;
    const osc_mesh3d m = planes_of(*mesh, z0, top);
    const int nl[3] = {n[0], n[1], top - z0 + 1};
    const int64_t nodes = (int64_t)n[0] * n[1] * (nzl + 1);
    CK(cudaMemsetAsync(quad, 0, sizeof(float4) * nodes, ctx->stream), "memset slab quad");
    TRY(counters_reset(ctx));
    if (np > 0) {
        DepositArgs da = deposit_args(&m, nl, np, x, y, z, q, q ? 0.0 : charge1, ctx->check_finite);
        da.ctas = tune_get(ctx, "deposit_ctas_per_sm");
        Launch L_(ctx, "deposit_f32");
        if (launch_deposit_quad(da, quad, ctx->d_small, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "slab deposit");
    }
    if (n_outside) {
        unsigned long long cnt[3];
        TRY(counters_read(ctx, cnt));
        *n_outside = (int64_t)(cnt[0] + cnt[1]);
    }
    return OSC_OK;
}

int osc_slab_forward_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int z0, int nzl, const float *quad, void *X2) {
    if (!ctx || !mesh || !quad || !X2) return OSC_E_INVALID;
    int n[3];
    TRY(check_slab(ctx, mesh, z0, nzl, n));
    return slab_forward(ctx, n[0], n[1], nzl, reinterpret_cast<const float4 *>(quad),
                        reinterpret_cast<cplx<float> *>(X2));
}

int osc_slab_zpass_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int col0, int ncols, const void *in, void *out) {
    if (!ctx || !mesh || (ncols > 0 && (!in || !out))) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    if (!(mesh->gamma >= 1.0)) return set_err(ctx, OSC_E_INVALID, "gamma must be >= 1");
    const FreeSpaceJob j = fs_job(mesh, n, nullptr, 0, 0);
    return slab_zpass(ctx, j, col0, ncols, reinterpret_cast<const cplx<float> *>(in),
                      reinterpret_cast<cplx<float> *>(out));
}

int osc_slab_inverse_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int z0, int nzl, const void *X3, float *e8) {
    if (!ctx || !mesh || !X3 || !e8) return OSC_E_INVALID;
    int n[3];
    TRY(check_slab(ctx, mesh, z0, nzl, n));
    return slab_inverse(ctx, n[0], n[1], nzl, reinterpret_cast<const cplx<float> *>(X3),
                        reinterpret_cast<float4 *>(e8));
}

int osc_slab_interp_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int p0, int np_planes, int64_t np, const double *x,
                        const double *y, const double *z, const float *e8, double *E) {
    if (!ctx || !mesh || !e8 || (np > 0 && (!x || !y || !z || !E))) return OSC_E_INVALID;
    int n[3];
    TRY(check_slab(ctx, mesh, p0, np_planes, n));
    if (np_planes < 2) return set_err(ctx, OSC_E_INVALID, "slab gather needs at least 2 planes");
    if (np == 0) return OSC_OK;
    const osc_mesh3d m = planes_of(*mesh, p0, p0 + np_planes - 1);
    const int nl[3] = {n[0], n[1], np_planes};
    InterpArgs ia = interp_args(&m, nl, np, x, y, z);
    ia.ctas = tune_get(ctx, "gather_ctas_per_sm");
    Launch L_(ctx, "interp_f32");
    if (launch_interp_pairs(ia, reinterpret_cast<const float4 *>(e8), E, ctx->d_small + 2, ctx->stream))
        return set_err(ctx, OSC_E_CUDA, "slab interp");
    return OSC_OK;
}

}  // extern "C"
