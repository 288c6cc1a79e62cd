// adjoint.cu -- vector-Jacobian product of the fused step (osc_space_charge_step_vjp_dev).
//
// The step maps particle positions x_m and charges q_m to E(x_m): a CIC deposit rho =
// sum_m q_m W(x_m), the free-space solve E_c = K_c rho (space_charge_3d,
// code/open_spacecharge_mod.f90:431-489) and the CIC gather E_c(x_m) (interpolate_field,
// :311-390).  Given gE[m] = dL/dE(x_m), the chain rule gives
//   dL/dx_m = sum_c gE_c[m] grad E_c(x_m) + q_m grad lambda(x_m),   dL/dq_m = lambda(x_m),
// with the adjoint potential lambda = sum_c K_c^T a_c and a_c = sum_m gE_c[m] W(x_m).
// Each K_c is a convolution with a kernel that is odd along axis c on the same centred
// window, so K_c^T = -K_c: lambda is three forward solves of the deposited gradients,
// one component each, accumulated with coefficient -1.  The mesh is held fixed.  The FP32
// path deposits into quad grids and gathers E and lambda from one x-pair grid, as the FP32
// step does; the FP64 path (and the deterministic deposit mode) uses FP64 planes.
#include "abi_util.cuh"

using namespace osc;
using namespace osc_abi;

extern "C" {

int osc_space_charge_step_vjp_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int64_t np, const double *x, const double *y,
                                  const double *z, const double *q, double total_charge, int precision,
                                  const double *gE, double *gx, double *gy, double *gz, double *gq) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    TRY(check_prec(ctx, precision));
    if (np <= 0 || !x || !y || !z || !gE || !gx || !gy || !gz) return bad(ctx, "vjp arrays");
    if (!(mesh->gamma >= 1.0)) return set_err(ctx, OSC_E_INVALID, "gamma must be >= 1");
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    const double charge1 = q ? 0.0 : total_charge / (double)np;
    DepositArgs da = deposit_args(mesh, n, np, x, y, z, q, charge1, 0);
    InterpArgs ia = interp_args(mesh, n, np, x, y, z);
    if (precision == OSC_PREC_FP32 && ctx->deposit_mode == OSC_DEPOSIT_ATOMIC) {
        // FP32: quad-grid deposits (the x transform sums the nodes as it loads them), E and
        // lambda in one x-pair grid, one gather of four 256-bit loads per particle
        float *quad3, *e8;
        double *lam;
        // E on the grid: the last FP32 step's, when allowed and it matches this call (its
        // slot 3 then takes lambda), else deposited and solved here
        const osc_ctx::FwdRecord &f = ctx->fwd;
        bool reuse = ctx->vjp_reuse && f.call == ctx->step_calls && f.e8 && f.np == np && f.x == x &&
                     f.y == y && f.z == z && f.q == q && f.gamma == mesh->gamma && f.charge1 == charge1;
        for (int d = 0; d < 3 && reuse; ++d)
            reuse = f.nlo[d] == mesh->nlo[d] && f.nhi[d] == mesh->nhi[d] && f.min[d] == mesh->min[d] &&
                    f.delta[d] == mesh->delta[d];
        TRY(ws_get(ctx, "vjp_quad3", sizeof(float4) * 3 * N, (void **)&quad3));
        TRY(ws_get(ctx, "vjp_lambda", sizeof(double) * N, (void **)&lam));
        TRY(counters_reset(ctx));
        CK(cudaMemsetAsync(quad3, 0, sizeof(float4) * 3 * N, ctx->stream), "memset quad3");
        CK(cudaMemsetAsync(lam, 0, sizeof(double) * N, ctx->stream), "memset lambda");  // three-solve path
        if (reuse) {
            e8 = reinterpret_cast<float *>(f.e8);
        } else {
            float *quad;
            TRY(ws_get(ctx, "vjp_quad", sizeof(float4) * N, (void **)&quad));
            TRY(ws_get(ctx, "vjp_e8", sizeof(float4) * 2 * N, (void **)&e8));
            CK(cudaMemsetAsync(quad, 0, sizeof(float4) * N, ctx->stream), "memset quad");
            {
                Launch L_(ctx, "deposit_f32");
                if (launch_deposit_quad(da, quad, ctx->d_small, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "deposit");
            }
            FreeSpaceJob j = fs_job(mesh, n, nullptr, 0, 0);
            j.quad = reinterpret_cast<const float4 *>(quad);
            j.E4 = e8;
            j.e4_pairs = 1;
            TRY(freespace_opt<float, float>(ctx, j, nullptr));
        }
        {
            Launch L_(ctx, "vjp_deposit");
            if (launch_deposit_quad3(da, gE, quad3, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "vjp deposit");
        }
        if (zconv_warp_ok(2 * n[2], n[2], (int)sizeof(float))) {
            // one solve: the three gradient grids are transformed, multiplied by their
            // kernels' spectra and summed before a single inverse, which writes lambda
            // straight into slot 3 of the x-pair grid
            FreeSpaceJob js = fs_job(mesh, n, nullptr, 0, 0);
            js.quad = reinterpret_cast<const float4 *>(quad3);
            js.sum3 = 1;
            js.E4 = e8;
            js.e4_pairs = 1;
            js.acc_coef = -1.0;
            TRY(freespace_opt<float, float>(ctx, js, nullptr));
        } else {
            for (int c = 0; c < 3; ++c) {
                FreeSpaceJob jc = fs_job(mesh, n, nullptr, 0, 0);
                jc.quad = reinterpret_cast<const float4 *>(quad3) + c * N;
                jc.comp_mask = 1 << c;
                jc.Eacc = lam;
                jc.acc_coef = -1.0;
                TRY(freespace_opt<float, float>(ctx, jc, nullptr));
            }
            Launch L_(ctx, "vjp_pack");
            if (launch_pack_lambda(e8, lam, n[0], N, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "pack lambda");
        }
        Launch L_(ctx, "vjp_particles");
        if (launch_vjp_pairs(ia, da, e8, gE, gx, gy, gz, gq, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "vjp gather");
        return OSC_OK;
    }
    double *rho, *Eg, *acc, *lam;
    TRY(ws_get(ctx, "vjp_rho", sizeof(double) * N, (void **)&rho));
    TRY(ws_get(ctx, "vjp_E", sizeof(double) * 3 * N, (void **)&Eg));
    TRY(ws_get(ctx, "vjp_a", sizeof(double) * 3 * N, (void **)&acc));
    TRY(ws_get(ctx, "vjp_lambda", sizeof(double) * N, (void **)&lam));
    const int prec = precision == OSC_PREC_FP32 ? OSC_PREC_FP32 : OSC_PREC_FP64;
    TRY(counters_reset(ctx));
    // forward field on the grid (the gather term needs it)
    TRY(deposit_rho<double>(ctx, da, rho, N, 1.0));
    FreeSpaceJob j = fs_job(mesh, n, nullptr, 0, 0);
    j.E = Eg;
    TRY(run_freespace(ctx, j, rho, prec));
    // deposited gradients a_c and the adjoint potential
    CK(cudaMemsetAsync(acc, 0, sizeof(double) * 3 * N, ctx->stream), "memset a");
    CK(cudaMemsetAsync(lam, 0, sizeof(double) * N, ctx->stream), "memset lambda");
    {
        Launch L_(ctx, "vjp_deposit");
        if (launch_deposit_vec3(da, gE, acc, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "vjp deposit");
    }
    for (int c = 0; c < 3; ++c) {
        FreeSpaceJob jc = fs_job(mesh, n, nullptr, 0, 0);
        jc.comp_mask = 1 << c;
        jc.Eacc = lam;
        jc.acc_coef = -1.0;
        TRY(run_freespace(ctx, jc, acc + c * N, prec));
    }
    {
        Launch L_(ctx, "vjp_particles");
        if (launch_vjp_particles(ia, da, Eg, lam, gE, gx, gy, gz, gq, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "vjp gather");
    }
    return OSC_OK;
}

}  // extern "C"
