// pipe_step.cu -- the fused space-charge step in a rectangular pipe
// (osc_space_charge_step_rectpipe_dev, declared in include/opensc_gpu.h).
//
// The reference's test program does deposit (depose_rho_scalar), space_charge_rectpipe and
// interpolate_field per particle (code/test_opensc.f90:156, :203-216, :247); this runs the
// three on the device in one call.  The pipe Green spectra must have been built or read for
// the mesh first (osc_rectpipe_green / osc_read_rectpipe_grn), as in the reference.  FP32:
// the quad-grid deposit and the x-pair gather of the free-space step around the FP32 pipe
// convolution; FP64 precisions: FP64 deposit and the reference-order gather.
#include "abi_util.cuh"

using namespace osc;
using namespace osc_abi;

extern "C" {

int osc_space_charge_step_rectpipe_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int64_t np, const double *x,
                                       const double *y, const double *z, const double *q, const double *total_charge,
                                       double apipe, double bpipe, int precision, double *E, double *B) {
    if (!ctx) return OSC_E_INVALID;
    int n[3];
    TRY(mesh_dims(ctx, mesh, n));
    TRY(check_prec(ctx, precision));
    if (np <= 0 || !x || !y || !z || !E) return bad(ctx, "pipe step arrays");
    if (!q && !total_charge) return set_err(ctx, OSC_E_NOCHARGE, "Error, must specify qa or total_charge");
    const int64_t N = (int64_t)n[0] * n[1] * n[2];
    osc_mesh3d m = *mesh;
    double charge1 = 0;
    if (q) TRY(set_charge(ctx, np, q, total_charge, &m, &charge1));
    else charge1 = *total_charge / (double)np;
    double *rho, *phi, *Eg, *Bg;
    TRY(ws_get(ctx, "ps_rho64", sizeof(double) * N, (void **)&rho));
    TRY(ws_get(ctx, "ps_phi", sizeof(double) * N, (void **)&phi));
    TRY(ws_get(ctx, "ps_E", sizeof(double) * 3 * N, (void **)&Eg));
    TRY(ws_get(ctx, "ps_B", sizeof(double) * 3 * N, (void **)&Bg));
    TRY(counters_reset(ctx));
    DepositArgs da = deposit_args(&m, n, np, x, y, z, q, charge1, ctx->check_finite);
    InterpArgs ia = interp_args(&m, n, np, x, y, z);
    const bool fp32 = precision == OSC_PREC_FP32 && ctx->deposit_mode == OSC_DEPOSIT_ATOMIC;
    if (fp32 && m.npad[0] == 1 && m.npad[1] == 1 && m.npad[2] == 1) {
        // the x transform reads the quad grid; E goes straight from phi to the x-pair grid
        // (and to FP64 planes only when B is wanted)
        float *quad, *e8;
        TRY(ws_get(ctx, "ps_quad", sizeof(float) * 4 * N, (void **)&quad));
        TRY(ws_get(ctx, "ps_E8", sizeof(float) * 8 * N, (void **)&e8));
        CK(cudaMemsetAsync(quad, 0, sizeof(float) * 4 * N, ctx->stream), "memset quad");
        {
            Launch L_(ctx, "deposit_f32");
            if (launch_deposit_quad(da, quad, ctx->d_small, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "deposit");
        }
        TRY(pipe_solve_checked(ctx, &m, precision, nullptr, phi, B ? Eg : nullptr, B ? Bg : nullptr,
                               reinterpret_cast<const float4 *>(quad), e8));
        {
            Launch L_(ctx, "interp_f32");
            if (launch_interp_pairs(ia, reinterpret_cast<const float4 *>(e8), E, ctx->d_small + 2, ctx->stream))
                return set_err(ctx, OSC_E_CUDA, "interp");
        }
        if (B) {
            Launch L_(ctx, "interp_f64");
            if (launch_interp_planes(ia, Bg, B, ctx->d_small + 3, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
        }
        return OSC_OK;
    }
    if (fp32) {
        float *quad, *rho32;
        TRY(ws_get(ctx, "ps_quad", sizeof(float) * 4 * N, (void **)&quad));
        TRY(ws_get(ctx, "ps_rho32", sizeof(float) * N, (void **)&rho32));
        CK(cudaMemsetAsync(quad, 0, sizeof(float) * 4 * N, ctx->stream), "memset quad");
        {
            Launch L_(ctx, "deposit_f32");
            if (launch_deposit_quad(da, quad, ctx->d_small, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "deposit");
        }
        {
            Launch L_(ctx, "quad_to_nodes");
            if (launch_quad_to_nodes(quad, rho32, n[0], n[1], n[2], ctx->stream))
                return set_err(ctx, OSC_E_CUDA, "quad to nodes");
        }
        {
            Launch L_(ctx, "f32_to_f64");
            if (launch_f32_to_f64(rho32, rho, N, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "rho to f64");
        }
    } else {
        TRY(deposit_rho<double>(ctx, da, rho, N, 1.0));
    }
    TRY(osc_space_charge_rectpipe_dev(ctx, &m, rho, apipe, bpipe, 0, 1, precision, phi, Eg, Bg));
    if (fp32) {
        float *e8;
        TRY(ws_get(ctx, "ps_E8", sizeof(float) * 8 * N, (void **)&e8));
        {
            Launch L_(ctx, "planes_to_pairs");
            if (launch_planes_to_pairs(Eg, e8, n[0], N, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "E pairs");
        }
        Launch L_(ctx, "interp_f32");
        if (launch_interp_pairs(ia, reinterpret_cast<const float4 *>(e8), E, ctx->d_small + 2, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "interp");
    } else {
        Launch L_(ctx, "interp_f64");
        if (launch_interp_planes(ia, Eg, E, ctx->d_small + 2, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
    }
    if (B) {
        Launch L_(ctx, "interp_f64");
        if (launch_interp_planes(ia, Bg, B, ctx->d_small + 3, ctx->stream)) return set_err(ctx, OSC_E_CUDA, "interp");
    }
    return OSC_OK;
}

}  // extern "C"
