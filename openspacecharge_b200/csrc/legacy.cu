// legacy.cu -- placeholder, replaced below
#include "../../include/opensc_gpu.h"
#include "solver.cuh"
extern "C" {
int osc_space_charge_freespace(osc_ctx *ctx, const osc_mesh3d *, const double *, int, int, int, double *, double *, double *) { return OSC_E_UNSUPPORTED; }
int osc_space_charge_cathodeimages(osc_ctx *, const osc_mesh3d *, double *, int, int, int, int, double *, double *, double *) { return OSC_E_UNSUPPORTED; }
int osc_rectpipe_green(osc_ctx *, const osc_mesh3d *, double, double, int) { return OSC_E_UNSUPPORTED; }
int osc_space_charge_rectpipe(osc_ctx *, const osc_mesh3d *, const double *, double, double, int, int, int, double *, double *, double *) { return OSC_E_UNSUPPORTED; }
int osc_write_rectpipe_grn(osc_ctx *, const char *, double, double, const osc_mesh3d *) { return OSC_E_UNSUPPORTED; }
int osc_read_rectpipe_grn(osc_ctx *, const char *, const osc_mesh3d *, double *, double *) { return OSC_E_UNSUPPORTED; }
}
