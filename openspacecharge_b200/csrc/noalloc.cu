// noalloc.cu -- charge deposition that allocates no memory.
//
// Who needs this: code that may not call cudaMalloc at the point where it deposits
// charge -- e.g. a tracking loop that runs inside a memory pool owned by another framework
// (which forbids allocations behind its back), a real-time loop that cannot afford the
// implicit device synchronisation of cudaMalloc/cudaFree, or a host program that must not
// create a library context (the context allocates its workspaces when it is created).
// This entry point needs no context: the caller passes a stream and device buffers, and
// the FP32 accumulation grid the deposit works in lives in a fixed array compiled into the
// library.
//
// Cost of that array: OSC_NOALLOC_MAX_NODES floats (16 MiB) plus a few counters, held on
// every GPU that loads this library until the process exits.
#include <cuda.h>

#include <cmath>
#include <mutex>

#include "../../include/opensc_gpu.h"
#include "grid_kernels.cuh"
#include "particle_kernels.cuh"

namespace {

constexpr int64_t kMaxNodes = OSC_NOALLOC_MAX_NODES;
constexpr int kCounterWords = 32;  // 256 bytes of counters after the grid

// FP32 accumulation grid (kMaxNodes floats) followed by the outside/non-finite counters.
// On the host this name is only a handle for cudaGetSymbolAddress, never a device address.
__device__ __align__(256) unsigned char g_noalloc_scratch[kMaxNodes * sizeof(float) + kCounterWords * 8];

// The array's device address belongs to one CUDA context.  It is looked up once per
// context (normally once per device: the primary context) and cached under the context
// handle, so a caller that makes another driver context current gets that context's
// address.  cudaDeviceReset destroys the primary context and with it this address: a
// process that resets a device must not call the entry point on that device afterwards.
constexpr int kMaxContexts = 64;
struct ScratchSlot {
    void *cuctx;
    void *addr;
};
ScratchSlot g_slots[kMaxContexts] = {};
int g_nslots = 0;
std::mutex g_scratch_mu;

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);

int fail(char *errbuf, size_t errlen, int code, const char *msg) {
    if (errbuf && errlen > 0) {
        size_t n = 0;
        while (msg[n] && n + 1 < errlen) {
            errbuf[n] = msg[n];
            ++n;
        }
        errbuf[n] = 0;
    }
    return code;
}

// Device address of the scratch array in the current context (set-up on first use).
int scratch_address(void **out, char *errbuf, size_t errlen) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return fail(errbuf, errlen, OSC_E_CUDA, "no current CUDA device");
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    static CtxGetCurrentFn get_current = nullptr;
    if (!get_current) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &qr) != cudaSuccess ||
            qr != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return fail(errbuf, errlen, OSC_E_CUDA, "cuCtxGetCurrent is not available");
        }
        get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    CUcontext cur = nullptr;
    if (get_current(&cur) != CUDA_SUCCESS) return fail(errbuf, errlen, OSC_E_CUDA, "cuCtxGetCurrent failed");
    if (!cur) {
        // nothing current yet: cudaSetDevice initialises the device's primary context
        if (cudaSetDevice(dev) != cudaSuccess || get_current(&cur) != CUDA_SUCCESS || !cur) {
            cudaGetLastError();
            return fail(errbuf, errlen, OSC_E_CUDA, "no current CUDA context");
        }
    }
    for (int i = 0; i < g_nslots; ++i)
        if (g_slots[i].cuctx == (void *)cur) {
            *out = g_slots[i].addr;
            return OSC_OK;
        }
    if (g_nslots == kMaxContexts) return fail(errbuf, errlen, OSC_E_CUDA, "too many CUDA contexts");
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail(errbuf, errlen, OSC_E_CUDA, "cudaGetSymbolAddress of the deposit scratch array failed");
    }
    g_slots[g_nslots++] = ScratchSlot{(void *)cur, p};
    *out = p;
    return OSC_OK;
}

}  // namespace

extern "C" {

int osc_deposit_particles_dev_noalloc(void *cuda_stream, const osc_mesh3d *mesh, int64_t np, const double *d_x,
                                      const double *d_y, const double *d_z, const double *d_q,
                                      double total_charge, double *d_rho, int64_t *n_outside, char *errbuf,
                                      size_t errlen) {
    if (!mesh || np < 0 || (np > 0 && (!d_x || !d_y || !d_z)) || !d_rho)
        return fail(errbuf, errlen, OSC_E_INVALID, "invalid argument: mesh, particle arrays or rho is NULL");
    // node count in 64-bit arithmetic, checked after every factor: no product can wrap
    int n[3];
    int64_t nodes = 1;
    for (int d = 0; d < 3; ++d) {
        const int64_t nd = (int64_t)mesh->nhi[d] - (int64_t)mesh->nlo[d] + 1;
        if (nd < 2) return fail(errbuf, errlen, OSC_E_INVALID, "mesh axis with fewer than 2 nodes");
        if (nd > kMaxNodes || nodes * nd > kMaxNodes)
            return fail(errbuf, errlen, OSC_E_INVALID,
                        "mesh has more nodes than the no-allocation deposit holds (OSC_NOALLOC_MAX_NODES = 4194304)");
        n[d] = (int)nd;
        nodes *= nd;
    }
    if (!std::isfinite(total_charge))
        return fail(errbuf, errlen, OSC_E_INVALID, "total_charge must be finite");
    // the reference's "must specify qa or total_charge" branch (rho untouched)
    if (!d_q && total_charge == 0.0)
        return fail(errbuf, errlen, OSC_E_NOCHARGE, "Error, must specify qa or total_charge");
    if (!(mesh->delta[0] > 0 && mesh->delta[1] > 0 && mesh->delta[2] > 0))
        return fail(errbuf, errlen, OSC_E_INVALID, "mesh delta must be positive");
    void *base = nullptr;
    int rc = scratch_address(&base, errbuf, errlen);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    float *grid = reinterpret_cast<float *>(base);
    unsigned long long *counters = reinterpret_cast<unsigned long long *>(
        reinterpret_cast<unsigned char *>(base) + kMaxNodes * sizeof(float));
    // the array keeps the previous call's sums: clear the part this call uses
    if (cudaMemsetAsync(grid, 0, sizeof(float) * nodes, st) != cudaSuccess ||
        cudaMemsetAsync(counters, 0, 8 * kCounterWords, st) != cudaSuccess) {
        cudaGetLastError();
        return fail(errbuf, errlen, OSC_E_CUDA, "clearing the deposit scratch array failed");
    }
    osc::DepositArgs a;
    a.fx_scale = 1.0;
    a.np = np;
    a.x = d_x;
    a.y = d_y;
    a.z = d_z;
    a.q = d_q;
    a.lost = nullptr;
    a.xmin = mesh->min[0];
    a.ymin = mesh->min[1];
    a.zmin = mesh->min[2];
    a.dx = mesh->delta[0];
    a.dy = mesh->delta[1];
    a.dz = mesh->delta[2];
    a.dxi = 1.0 / a.dx;
    a.dyi = 1.0 / a.dy;
    a.dzi = 1.0 / a.dz;
    for (int d = 0; d < 3; ++d) {
        a.nlo[d] = mesh->nlo[d];
        a.nhi[d] = mesh->nhi[d];
        a.nlogbl[d] = mesh->nlo[d];
    }
    a.nx = n[0];
    a.ny = n[1];
    a.nz = n[2];
    a.mode = 0;
    a.charge1 = np > 0 ? total_charge / (double)np : 0.0;
    a.check_finite = 1;
    if (osc::launch_deposit<float>(a, grid, counters, st) || osc::launch_f32_to_f64(grid, d_rho, nodes, st))
        return fail(errbuf, errlen, OSC_E_CUDA, "deposit kernel launch failed");
    if (n_outside) {
        // out-of-mesh and non-finite particles, the count the context entry point reports
        unsigned long long h[2] = {0, 0};
        if (cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return fail(errbuf, errlen, OSC_E_CUDA, "reading the out-of-mesh count failed");
        }
        *n_outside = (int64_t)(h[0] + h[1]);
    }
    return fail(errbuf, errlen, OSC_OK, "");
}

}  // extern "C"
