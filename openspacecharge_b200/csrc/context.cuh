// context.cuh -- per-context state: stream, workspaces, Green-spectrum cache, profiling.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <list>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "fft_kernels.cuh"

struct osc_ctx;

namespace osc {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// One cached Green spectrum set: the stored spectra of all components of one geometry.
struct GreenSet {
    std::string key;
    int nspec = 0;
    DevBuf buf[8];
    GSpecDev spec[8];
    size_t bytes = 0;
    uint64_t stamp = 0;
};

struct ProfRec {
    std::string name;
    cudaEvent_t a, b;
};
struct ProfSum {
    int64_t launches = 0;
    double ms = 0;
};

// Transformed pipe Green arrays (the reference's module-global cgrn1..4, core:22-23).
struct PipeGreen {
    bool valid = false;
    int nlo[3], nhi[3], npad[3], period[3];
    double apipe = 0, bpipe = 0, gamma = 0, delta[3], umin[3], umax[3];
    DevBuf g[4];          // complex128 full spectra in the reference layout (FP64 plain path)
    DevBuf comb;          // combined single-kernel spectrum for the optimised path
    int comb_prec = -1;
    GSpecDev comb_spec;
};

}  // namespace osc

struct osc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    // auxiliary streams for independent work inside one call (batched bunches of different
    // grid shapes); ws_slot != 0 while work is issued on aux[ws_slot - 1]
    std::vector<cudaStream_t> aux;
    std::vector<cudaEvent_t> aux_ev;
    cudaEvent_t switch_ev = nullptr;  // orders a newly set stream after the previous one
    // private stream that graph captures run on (the caller's stream may be the legacy
    // default stream, which cannot be captured); the graphs launch on the caller's stream
    cudaStream_t cap_stream = nullptr;
    // copy streams of the batched step from host arrays (chunks of bunches copied in and out
    // while others compute) and their events
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    std::vector<cudaEvent_t> copy_ev;
    int ws_slot = 0;
    std::string err;
    // options
    int precision = 0;
    int deposit_mode = 0;
    int particle_order = 0;  // OSC_ORDER_*
    // launch shapes picked by the autotuner (osc_ctx_set_tuning), by key; absent = default
    std::map<std::string, int> tuning;
    int strict_bounds = 0;
    int profile = 0;
    int check_finite = 0;
    int test_wait_timeout = 0;  // OSC_OPT_TEST_WAIT_TIMEOUT
    int batch_graph = 1;        // OSC_OPT_BATCH_GRAPH
    size_t gcache_budget = (size_t)4096 << 20;
    // CUDA-graph capture of a batched step: while capturing, nothing may allocate (ws_get,
    // twiddles and the auxiliary streams refuse instead); ws_gen counts workspace
    // (re)allocations and tune_gen tuning changes, so a captured graph whose buffers or
    // launch shapes went stale is captured again
    int capturing = 0;
    uint64_t ws_gen = 0, tune_gen = 0;
    int64_t graph_launches = 0;  // batched steps run as one graph launch
    // the FP32 step's x-pair E grid, kept for the adjoint (OSC_OPT_VJP_REUSE_FORWARD):
    // every step call counts in step_calls; fwd records the last FP32 step's inputs
    int vjp_reuse = 0;
    int64_t step_calls = 0;
    struct FwdRecord {
        int64_t call = -1, np = 0;
        int nlo[3], nhi[3];
        double min[3], delta[3], gamma, charge1;
        const double *x, *y, *z, *q;
        void *e8 = nullptr;
    } fwd;
    // captured batched steps by call signature (batch.cu), most recently used first
    std::list<std::shared_ptr<void>> batch_plans;
    // workspaces by name
    std::map<std::string, osc::DevBuf> ws;
    std::map<int, osc::DevBuf> tw32, tw64;
    std::list<osc::GreenSet> gcache;
    // spectrum buffers of evicted sets, reused (same byte size) by the next builds; all
    // cache users run on the context stream, so reuse is stream-ordered
    std::vector<osc::DevBuf> gpool;
    uint64_t stamp = 0;
    // small device/pinned scratch for counters and reductions
    unsigned long long *d_small = nullptr;  // 64 words
    unsigned long long *h_small = nullptr;  // pinned 64 words
    double *d_partials = nullptr;           // 1024 doubles
    // host-mapped word where kernels report bounded waits that gave up (0 = none)
    unsigned *h_fault = nullptr;
    unsigned *d_fault = nullptr;
    // profiling
    std::vector<osc::ProfRec> prof_pending;
    std::map<std::string, osc::ProfSum> prof;
    std::vector<cudaEvent_t> ev_pool;
    int64_t launches = 0;
    osc::PipeGreen pipe;
};

namespace osc {

int set_err(osc_ctx *c, int code, const char *fmt, ...);
int cuda_check(osc_ctx *c, cudaError_t e, const char *what);
// Synchronises the context stream, then reports (and clears) a fault word set by a kernel.
int ctx_sync(osc_ctx *c);
// Named device workspace of at least `bytes` (grown by reallocation; contents not kept).
int ws_get(osc_ctx *c, const char *name, size_t bytes, void **out);
// Twiddle tables of length L (runtime table and, when L has a static engine, its
// per-stage table), built once per context in FP64.
template <typename T> int twiddles(osc_ctx *c, int L, TwPair<cplx<T>> *out);

// Kernel-launch bookkeeping and optional per-kernel CUDA-event timing.
struct Launch {
    osc_ctx *c;
    const char *name;
    int nk;
    cudaEvent_t a = nullptr;
    Launch(osc_ctx *c_, const char *name_, int nk_ = 1);
    ~Launch();
};
int prof_flush(osc_ctx *c);
// Tuned value of `key` (autotuner), or def when none was set.
int tune_get(const osc_ctx *c, const std::string &key, int def = 0);

// Green-spectrum cache.  A budget of 0 disables it: every solve rebuilds its spectra (the
// reference's behaviour, code/open_spacecharge_mod.f90:570-573) into reused buffers.
GreenSet *gcache_find(osc_ctx *c, const std::string &key);
GreenSet *gcache_insert(osc_ctx *c, GreenSet &&g);
// Device buffer of exactly `bytes` for a new spectrum: a pooled buffer of that size, else
// least recently used sets are evicted into the pool while the cache is over budget, else
// cudaMalloc.
int green_alloc(osc_ctx *c, size_t bytes, DevBuf &out);
// Returns an unused spectrum buffer to the pool.
void green_release(osc_ctx *c, DevBuf &b);
// Frees every cached set and pooled buffer (after synchronising the stream).
void gcache_free_all(osc_ctx *c);

}  // namespace osc
