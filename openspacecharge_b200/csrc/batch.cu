// batch.cu -- batched space-charge steps over many independent bunches
// (osc_batch_space_charge_step*, declared in include/opensc_gpu.h).
//
// FP32: one pass over all particles computes every bunch's bounding box and charge, one
// thread per bunch refits its mesh and writes its arguments on the device, one pass
// deposits every bunch into its own quad grid, then each group of bunches with the same
// grid shape is solved by the batched pipeline (Green spectra of all members from batched
// corner blocks and even/odd line transforms; the stacked FFT passes with the members as
// extra rows, planes and columns) on one of four streams, and one pass interpolates E for
// every particle.  Nothing in the step waits for the host, so a call whose signature
// (grids, particle counts and offsets, pointers, options) repeats replays the step as one
// captured CUDA graph.  The reference solves one bunch per call (space_charge_3d,
// code/open_spacecharge_mod.f90:431-489).
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "abi_util.cuh"

using namespace osc;
using namespace osc_abi;

namespace {

constexpr int64_t kJobParticles = 4096;  // particles per CTA of the batched particle passes

struct Group {
    int n[3];
    std::vector<int> members;
    int64_t node0 = 0;  // first node of the group's stacked grids in the batch arrays
};

constexpr int kSlots = kAuxSlots;  // grid-shape groups solved concurrently on auxiliary streams

// Issues work on auxiliary slot `slot` (1-based) for its lifetime; restores the main stream.
struct SlotGuard {
    osc_ctx *c;
    cudaStream_t main;
    SlotGuard(osc_ctx *ctx, int slot) : c(ctx), main(ctx->stream) {
        c->stream = c->aux[slot - 1];
        c->ws_slot = slot;
    }
    ~SlotGuard() {
        c->stream = main;
        c->ws_slot = 0;
    }
};

int check_bunches(osc_ctx *ctx, int nb, const osc_bunch *bs, const double *x, const double *y, const double *z,
                  const double *E) {
    if (nb <= 0 || !bs) return bad(ctx, "batch needs at least one bunch");
    if (!x || !y || !z || !E) return bad(ctx, "batch arrays");
    for (int b = 0; b < nb; ++b) {
        int n[3];
        TRY(mesh_dims(ctx, &bs[b].mesh, n));
        if (bs[b].np <= 0 || bs[b].offset < 0) return set_err(ctx, OSC_E_INVALID, "bunch %d: np must be >= 1", b);
        if (!(bs[b].mesh.gamma >= 1.0)) return set_err(ctx, OSC_E_INVALID, "bunch %d: gamma must be >= 1", b);
    }
    return OSC_OK;
}

// ---- one FP32 batched step, issued without host synchronisation -----------------------
// The host fills each bunch's mesh and charge into pinned staging (BunchIn); the step copies
// it to the device, computes the bounding boxes and charges, and k_batch_setup refits the
// meshes and writes every bunch's deposit, gather and Green-corner arguments on the device,
// so nothing in the step waits for the host: the whole step can be captured in one CUDA
// graph.  The results come back through pinned staging (BunchOut, counters).

struct BunchIn {
    double min[3], max[3], delta[3], gamma, total_charge;
};
struct BunchOut {
    double stats[8];  // bounding box (xmin, xmax, ymin, ymax, zmin, zmax), non-finite, sum q
    double min[3], max[3], delta[3], charge;
};
// Static placement of a bunch: its first corner block (component 1) in the batch's corner
// array, the members of its group (blocks of one component), its grid.
struct BunchMap {
    int ca0, cstride;
    int n[3], nlo[3], nhi[3];
    int64_t np;
};

// Mesh refit (apply_refit), deposit / gather arguments (deposit_args, interp_args) and Green
// corner arguments (green_corner_args with zero offset) of every bunch, with every product,
// sum and quotient rounded separately as the host evaluates them, so the meshes and
// arguments are bit-identical to those of a single step.
__global__ void k_batch_setup(int nb, const BunchMap *__restrict__ map, const BunchIn *__restrict__ in,
                              const double *__restrict__ stats, int resize, int has_q, BunchArgs *ba,
                              CornerArgs *ca, BunchOut *out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const BunchMap m = map[b];
    const BunchIn bi = in[b];
    const double *st = stats + 8 * (int64_t)b;
    double mn[3], mx[3], dl[3];
    for (int d = 0; d < 3; ++d) {
        mn[d] = bi.min[d];
        mx[d] = bi.max[d];
        dl[d] = bi.delta[d];
    }
    if (resize && !(st[6] > 0)) {  // with non-finite coordinates the call fails; keep the mesh
        for (int d = 0; d < 3; ++d) {
            const double cells = (double)(m.nhi[d] - m.nlo[d]);
            double lo = st[2 * d], hi = st[2 * d + 1];
            const double d0 = __ddiv_rn(__dsub_rn(hi, lo), cells);
            lo = __dsub_rn(lo, __dmul_rn(1.0e-6, d0));
            hi = __dadd_rn(hi, __dmul_rn(1.0e-6, d0));
            mn[d] = lo;
            mx[d] = hi;
            dl[d] = __ddiv_rn(__dsub_rn(hi, lo), cells);
        }
    }
    const double charge = has_q ? st[7] : bi.total_charge;
    const double charge1 = has_q ? 0.0 : __ddiv_rn(bi.total_charge, (double)m.np);
    DepositArgs &da = ba[b].d;
    da.xmin = mn[0];
    da.ymin = mn[1];
    da.zmin = mn[2];
    da.dx = dl[0];
    da.dy = dl[1];
    da.dz = dl[2];
    da.dxi = __ddiv_rn(1.0, dl[0]);
    da.dyi = __ddiv_rn(1.0, dl[1]);
    da.dzi = __ddiv_rn(1.0, dl[2]);
    da.charge1 = charge1;
    InterpArgs &ia = ba[b].in;
    for (int d = 0; d < 3; ++d) {
        ia.min[d] = mn[d];
        ia.delta[d] = dl[d];
        ia.hinv[d] = __ddiv_rn(1.0, dl[d]);
    }
    const double dz = __dmul_rn(dl[2], bi.gamma);
    const double vol = __dmul_rn(__dmul_rn(dl[0], dl[1]), dz);
    for (int comp = 1; comp <= 3; ++comp) {
        CornerArgs &c = ca[m.ca0 + (comp - 1) * m.cstride];
        c.cdx = m.n[0] + 1;
        c.cdy = m.n[1] + 1;
        c.cdz = m.n[2] + 1;
        c.c0x = m.n[0] - 1;
        c.c0y = m.n[1] - 1;
        c.c0z = m.n[2] - 1;
        c.dx = dl[0];
        c.dy = dl[1];
        c.dz = dz;
        c.factor = (comp == 1 || comp == 2) ? __ddiv_rn(bi.gamma, vol) : __ddiv_rn(1.0, vol);
        c.umin = __dadd_rn(__dmul_rn((double)__fsub_rn(0.5f, (float)m.n[0]), dl[0]), 0.0);
        c.vmin = __dadd_rn(__dmul_rn((double)__fsub_rn(0.5f, (float)m.n[1]), dl[1]), 0.0);
        c.wmin = __dadd_rn(__dmul_rn((double)__fsub_rn(0.5f, (float)m.n[2]), dz), __dmul_rn(0.0, bi.gamma));
        c.icomp = comp;
    }
    BunchOut &o = out[b];
    for (int i = 0; i < 8; ++i) o.stats[i] = st[i];
    for (int d = 0; d < 3; ++d) {
        o.min[d] = mn[d];
        o.max[d] = mx[d];
        o.delta[d] = dl[d];
    }
    o.charge = charge;
}

// Everything of one call signature that does not change from step to step: the CTA jobs of
// the particle passes, the groups of equal grids and their stream slots, the static halves
// of the bunch arguments, and (after the second call) the captured graph.
struct BatchPlan {
    std::string key;
    int nb = 0, njobs = 0, resize = 0, has_q = 0;
    int64_t nodes = 0;
    size_t max_f = 0, max_g = 0;
    std::vector<Group> groups;
    std::vector<int> slot_of;      // auxiliary stream slot of each group
    std::vector<size_t> ca_off;    // first corner block of each group
    std::vector<int> issue_order;  // groups, largest first
    DevBuf d_ba, d_jobs, d_job0, d_ca, d_map, d_in, d_out;
    BunchIn *h_in = nullptr;
    BunchOut *h_out = nullptr;
    unsigned long long *h_cnt = nullptr;
    int calls = 0;
    cudaGraphExec_t exec = nullptr;
    uint64_t ws_gen = 0;
    int64_t step_launches = 0;  // kernels of one step, counted while capturing
    ~BatchPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        for (DevBuf *b : {&d_ba, &d_jobs, &d_job0, &d_ca, &d_map, &d_in, &d_out})
            if (b->p) cudaFree(b->p);
        if (h_in) cudaFreeHost(h_in);
        if (h_out) cudaFreeHost(h_out);
        if (h_cnt) cudaFreeHost(h_cnt);
    }
};

int dev_alloc(osc_ctx *ctx, DevBuf &b, size_t bytes) {
    bytes = bytes ? bytes : 16;
    if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return set_err(ctx, OSC_E_ALLOC, "batch plan: cudaMalloc(%zu) failed", bytes);
    }
    b.bytes = bytes;
    return OSC_OK;
}

std::string plan_key(const osc_ctx *ctx, int nb, const osc_bunch *bs, const double *x, const double *y,
                     const double *z, const double *q, int resize, const double *E) {
    std::vector<int64_t> k;
    k.reserve(8 + 8 * (size_t)nb);
    for (const void *p : {(const void *)x, (const void *)y, (const void *)z, (const void *)q, (const void *)E})
        k.push_back((int64_t)(uintptr_t)p);
    k.push_back(resize);
    k.push_back(ctx->check_finite);
    k.push_back((int64_t)ctx->tune_gen);
    for (int b = 0; b < nb; ++b) {
        for (int d = 0; d < 3; ++d) {
            k.push_back(bs[b].mesh.nlo[d]);
            k.push_back(bs[b].mesh.nhi[d]);
        }
        k.push_back(bs[b].np);
        k.push_back(bs[b].offset);
    }
    return std::string(reinterpret_cast<const char *>(k.data()), k.size() * sizeof(int64_t));
}

int make_plan(osc_ctx *ctx, BatchPlan &P, int nb, const osc_bunch *bs, const double *x, const double *y,
              const double *z, const double *q, int resize, double *E) {
    P.nb = nb;
    P.resize = resize;
    P.has_q = q ? 1 : 0;
    // CTA jobs of the particle passes, bunch by bunch
    std::vector<BatchJob> jobs;
    std::vector<int> job0(nb + 1);
    for (int b = 0; b < nb; ++b) {
        job0[b] = (int)jobs.size();
        for (int64_t beg = 0; beg < bs[b].np; beg += kJobParticles)
            jobs.push_back(BatchJob{b, beg, std::min(beg + kJobParticles, bs[b].np)});
    }
    job0[nb] = (int)jobs.size();
    P.njobs = (int)jobs.size();
    // groups of equal grids (map order), members stacked along z in the batch arrays
    std::map<std::tuple<int, int, int>, Group> gm;
    for (int b = 0; b < nb; ++b) {
        int n[3];
        TRY(mesh_dims(ctx, &bs[b].mesh, n));
        Group &g = gm[std::make_tuple(n[0], n[1], n[2])];
        for (int d = 0; d < 3; ++d) g.n[d] = n[d];
        g.members.push_back(b);
    }
    for (auto &kv : gm) P.groups.push_back(kv.second);
    std::vector<BunchArgs> ba(nb);
    std::memset(ba.data(), 0, sizeof(BunchArgs) * nb);
    std::vector<BunchMap> map(nb);
    size_t nca = 0;
    for (Group &g : P.groups) {
        const int64_t N = (int64_t)g.n[0] * g.n[1] * g.n[2];
        const int B = (int)g.members.size();
        g.node0 = P.nodes;
        P.ca_off.push_back(nca);
        for (int i = 0; i < B; ++i) {
            const int b = g.members[i];
            const int64_t o = bs[b].offset;
            // static fields; the mesh-dependent ones are written by k_batch_setup
            ba[b].d = deposit_args(&bs[b].mesh, g.n, bs[b].np, x + o, y + o, z + o, q ? q + o : nullptr, 0.0,
                                   ctx->check_finite);
            ba[b].in = interp_args(&bs[b].mesh, g.n, bs[b].np, x + o, y + o, z + o);
            ba[b].node_off = P.nodes + (int64_t)i * N;
            ba[b].E = E + 3 * o;
            BunchMap &m = map[b];
            m.ca0 = (int)(nca + i);
            m.cstride = B;
            for (int d = 0; d < 3; ++d) {
                m.n[d] = g.n[d];
                m.nlo[d] = bs[b].mesh.nlo[d];
                m.nhi[d] = bs[b].mesh.nhi[d];
            }
            m.np = bs[b].np;
        }
        nca += 3 * (size_t)B;
        P.nodes += N * B;
        P.max_f = std::max(P.max_f, 3 * (size_t)B * (g.n[0] + 1) * (g.n[1] + 1) * (g.n[2] + 1));
        const int zp = green_zpitch(g.n[2] + 1, sizeof(float));
        P.max_g = std::max(P.max_g, 3 * (size_t)B * (g.n[0] + 1) * (g.n[1] + 1) * zp);
    }
    // largest groups first, each on the stream with the least work queued so far, so the
    // streams finish together (cost ~ members x corner-block nodes)
    auto gcost = [](const Group &g) {
        return (double)g.members.size() * (g.n[0] + 1) * (double)(g.n[1] + 1) * (double)(g.n[2] + 1);
    };
    for (int i = 0; i < (int)P.groups.size(); ++i) P.issue_order.push_back(i);
    std::stable_sort(P.issue_order.begin(), P.issue_order.end(),
                     [&](int u, int v) { return gcost(P.groups[u]) > gcost(P.groups[v]); });
    P.slot_of.assign(P.groups.size(), 0);
    double queued[kSlots] = {};
    for (int gi : P.issue_order) {
        int slot = 0;
        for (int s2 = 1; s2 < kSlots; ++s2)
            if (queued[s2] < queued[slot]) slot = s2;
        queued[slot] += gcost(P.groups[gi]);
        P.slot_of[gi] = slot + 1;
    }
    TRY(dev_alloc(ctx, P.d_ba, sizeof(BunchArgs) * nb));
    TRY(dev_alloc(ctx, P.d_jobs, sizeof(BatchJob) * jobs.size()));
    TRY(dev_alloc(ctx, P.d_job0, sizeof(int) * job0.size()));
    TRY(dev_alloc(ctx, P.d_ca, sizeof(CornerArgs) * nca));
    TRY(dev_alloc(ctx, P.d_map, sizeof(BunchMap) * nb));
    TRY(dev_alloc(ctx, P.d_in, sizeof(BunchIn) * nb));
    TRY(dev_alloc(ctx, P.d_out, sizeof(BunchOut) * nb));
    if (cudaMallocHost(&P.h_in, sizeof(BunchIn) * nb) != cudaSuccess ||
        cudaMallocHost(&P.h_out, sizeof(BunchOut) * nb) != cudaSuccess ||
        cudaMallocHost(&P.h_cnt, sizeof(unsigned long long) * 4 * nb) != cudaSuccess) {
        cudaGetLastError();
        return set_err(ctx, OSC_E_ALLOC, "batch plan: pinned staging");
    }
    TRY(h2d(ctx, P.d_ba.p, ba.data(), sizeof(BunchArgs) * nb));
    TRY(h2d(ctx, P.d_jobs.p, jobs.data(), sizeof(BatchJob) * jobs.size()));
    TRY(h2d(ctx, P.d_job0.p, job0.data(), sizeof(int) * job0.size()));
    TRY(h2d(ctx, P.d_map.p, map.data(), sizeof(BunchMap) * nb));
    return sync(ctx);  // the pageable sources above go out of scope
}

// Every workspace the step uses, grown before the step is issued (growing synchronises).
int batch_workspaces(osc_ctx *ctx, const BatchPlan &P) {
    size_t x1 = 0, x2 = 0, x3 = 0, x4 = 0, h = 0, hx = 0, hy = 0;
    for (const Group &g : P.groups) {
        const size_t B = g.members.size(), nx = g.n[0], ny = g.n[1], nz = g.n[2];
        x1 = std::max(x1, B * (nx + 1) * ny * nz);
        x2 = std::max(x2, B * (nx + 1) * 2 * ny * nz);
        x3 = std::max(x3, 3 * B * (nx + 1) * 2 * ny * nz);
        x4 = std::max(x4, 3 * B * (nx + 1) * ny * nz);
        h = std::max(h, 3 * B * nx * ny * nz);
        hx = std::max(hx, 3 * B * (nx + 1) * ny * nz);
        hy = std::max(hy, 3 * B * (nx + 1) * (ny + 1) * nz);
    }
    TRY(ensure_aux(ctx));
    void *p;
    for (int slot = 1; slot <= kSlots; ++slot) {
        SlotGuard sg(ctx, slot);
        TRY(ws_get(ctx, "fs_x1", sizeof(float2) * x1, &p));
        TRY(ws_get(ctx, "fs_x2", sizeof(float2) * x2, &p));
        TRY(ws_get(ctx, "fs_x3", sizeof(float2) * x3, &p));
        TRY(ws_get(ctx, "fs_x4", sizeof(float2) * x4, &p));
        TRY(ws_get(ctx, "green_h", sizeof(double) * h, &p));
        TRY(ws_get(ctx, "green_hx", sizeof(double) * hx, &p));
        TRY(ws_get(ctx, "green_hy", sizeof(double) * hy, &p));
        TRY(ws_get(ctx, "batch_F", sizeof(double) * P.max_f, &p));
        TRY(ws_get(ctx, "batch_green", sizeof(float) * P.max_g, &p));
    }
    TRY(ws_get(ctx, "batch_keys", sizeof(unsigned long long) * 7 * (size_t)std::max(P.njobs, 1), &p));
    TRY(ws_get(ctx, "batch_qsum", sizeof(double) * (size_t)std::max(P.njobs, 1), &p));
    TRY(ws_get(ctx, "batch_stats", sizeof(double) * 8 * (size_t)P.nb, &p));
    TRY(ws_get(ctx, "batch_quad", sizeof(float) * 4 * (size_t)P.nodes, &p));
    TRY(ws_get(ctx, "batch_e8", sizeof(float) * 8 * (size_t)P.nodes, &p));
    TRY(ws_get(ctx, "batch_cnt", sizeof(unsigned long long) * 4 * (size_t)P.nb, &p));
    return OSC_OK;
}

// The step's device work on the context stream (and the auxiliary streams it forks and
// joins): no host synchronisation, no allocation.
int batch_issue(osc_ctx *ctx, BatchPlan &P) {
    const int nb = P.nb;
    BunchArgs *d_ba = reinterpret_cast<BunchArgs *>(P.d_ba.p);
    const BatchJob *d_jobs = reinterpret_cast<const BatchJob *>(P.d_jobs.p);
    CornerArgs *d_ca = reinterpret_cast<CornerArgs *>(P.d_ca.p);
    unsigned long long *keys, *cnt;
    double *qsum, *stats;
    float *quad, *e8;
    TRY(ws_get(ctx, "batch_keys", sizeof(unsigned long long) * 7 * (size_t)std::max(P.njobs, 1), (void **)&keys));
    TRY(ws_get(ctx, "batch_qsum", sizeof(double) * (size_t)std::max(P.njobs, 1), (void **)&qsum));
    TRY(ws_get(ctx, "batch_stats", sizeof(double) * 8 * (size_t)nb, (void **)&stats));
    TRY(ws_get(ctx, "batch_quad", sizeof(float) * 4 * (size_t)P.nodes, (void **)&quad));
    TRY(ws_get(ctx, "batch_e8", sizeof(float) * 8 * (size_t)P.nodes, (void **)&e8));
    TRY(ws_get(ctx, "batch_cnt", sizeof(unsigned long long) * 4 * (size_t)nb, (void **)&cnt));
    CK(cudaMemcpyAsync(P.d_in.p, P.h_in, sizeof(BunchIn) * nb, cudaMemcpyHostToDevice, ctx->stream), "meshes in");
    // bounding boxes, non-finite counts and charges of all bunches, then the meshes and
    // arguments on the device
    {
        Launch L_(ctx, "batch_stats", 2);
        if (launch_batch_stats(d_ba, d_jobs, P.njobs, reinterpret_cast<const int *>(P.d_job0.p), nb, keys, qsum,
                               stats, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "batch stats");
    }
    {
        Launch L_(ctx, "batch_setup");
        k_batch_setup<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(
            nb, reinterpret_cast<const BunchMap *>(P.d_map.p), reinterpret_cast<const BunchIn *>(P.d_in.p), stats,
            P.resize, P.has_q, d_ba, d_ca, reinterpret_cast<BunchOut *>(P.d_out.p));
        CK(cudaGetLastError(), "batch setup");
    }
    // deposit every bunch into its quad grid
    CK(cudaMemsetAsync(quad, 0, sizeof(float) * 4 * (size_t)P.nodes, ctx->stream), "memset quad");
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 4 * (size_t)nb, ctx->stream), "memset counters");
    {
        Launch L_(ctx, "batch_deposit");
        if (launch_batch_deposit_quad(d_ba, d_jobs, P.njobs, quad, cnt, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "batch deposit");
    }
    // field of every group: groups of different shapes are independent, so they run on
    // kSlots auxiliary streams (each with its own workspaces) after the deposit
    CK(cudaEventRecord(ctx->aux_ev[kSlots], ctx->stream), "record deposit");
    for (int s2 = 0; s2 < kSlots; ++s2) CK(cudaStreamWaitEvent(ctx->aux[s2], ctx->aux_ev[kSlots], 0), "wait deposit");
    for (int gi : P.issue_order) {
        const Group &g = P.groups[gi];
        SlotGuard sg(ctx, P.slot_of[gi]);
        float *gbuf;
        double *F;
        TRY(ws_get(ctx, "batch_F", sizeof(double) * P.max_f, (void **)&F));
        TRY(ws_get(ctx, "batch_green", sizeof(float) * P.max_g, (void **)&gbuf));
        const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
        const int B = (int)g.members.size();
        const int zinner = zconv_warp_ok(2 * nz, nz, 4) ? 1 : 0;
        const int zp = zinner ? green_zpitch(nz + 1, sizeof(float)) : nz + 1;
        const int64_t per = (int64_t)(nx + 1) * (ny + 1) * zp;
        const int64_t fstride = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
        if (zinner) CK(cudaMemsetAsync(gbuf, 0, sizeof(float) * 3 * B * per, ctx->stream), "memset spectra");
        // Green spectra of the three E components of every member: members m = comp*B + i
        {
            Launch L_(ctx, "green_corners");
            if (launch_igf_corners_batch(F, d_ca + P.ca_off[gi], 3 * B, fstride, fstride, ctx->stream))
                return set_err(ctx, OSC_E_CUDA, "batch corners");
        }
        const int odd[3][2] = {{0, B}, {B, 2 * B}, {2 * B, 3 * B}};
        TRY(green_sym_lines3<float>(ctx, F, 3 * B, nx, ny, nz, odd, zinner, zp, gbuf, per));
        GSpecDev spec[3];
        for (int comp = 1; comp <= 3; ++comp) {
            GSpecDev &s = spec[comp - 1];
            s.data = gbuf + (int64_t)(comp - 1) * B * per;
            s.real_valued = 1;
            s.imag_unit = 1;
            s.sym_y = s.sym_z = 1;
            s.par_y = comp == 2 ? -1 : 1;
            s.par_z = comp == 3 ? -1 : 1;
            s.dimy = ny + 1;
            s.dimz = nz + 1;
            s.zinner = zinner;
            s.zpitch = zp;
        }
        FreeSpaceJob j;
        j.nx = nx;
        j.ny = ny;
        j.nz = nz;
        j.want_e = 1;
        j.E4 = e8 + 8 * g.node0;
        j.e4_pairs = 1;
        j.nbatch = B;
        j.gbatch = spec;
        j.ngbatch = 3;
        j.g_bstride = per;
        j.quad = reinterpret_cast<const float4 *>(quad) + g.node0;  // the x transform sums the nodes
        TRY(freespace_opt<float, float>(ctx, j, nullptr));
    }
    for (int s2 = 0; s2 < kSlots; ++s2) {
        CK(cudaEventRecord(ctx->aux_ev[s2], ctx->aux[s2]), "record group");
        CK(cudaStreamWaitEvent(ctx->stream, ctx->aux_ev[s2], 0), "wait groups");
    }
    {
        Launch L_(ctx, "batch_interp");
        if (launch_batch_interp_pairs(d_ba, d_jobs, P.njobs, e8, cnt, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "batch interp");
    }
    CK(cudaMemcpyAsync(P.h_out, P.d_out.p, sizeof(BunchOut) * nb, cudaMemcpyDeviceToHost, ctx->stream), "meshes out");
    CK(cudaMemcpyAsync(P.h_cnt, cnt, sizeof(unsigned long long) * 4 * nb, cudaMemcpyDeviceToHost, ctx->stream),
       "counters out");
    return OSC_OK;
}

// Captures batch_issue into a graph executable (the call's workspaces, twiddle tables and
// streams exist already: the first call of a signature ran the step directly).  A capture
// that fails leaves the plan without a graph and the step runs directly.
int batch_capture(osc_ctx *ctx, BatchPlan &P) {
    cudaGraph_t graph = nullptr;
    // captured on the private stream (nothing runs while capturing); launched on the caller's
    const cudaError_t eb = cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (eb != cudaSuccess) {
        cudaGetLastError();
        return set_err(ctx, OSC_E_CUDA, "batch graph capture: %s", cudaGetErrorString(eb));
    }
    cudaStream_t user = ctx->stream;
    ctx->stream = ctx->cap_stream;
    ctx->capturing = 1;
    const int64_t l0 = ctx->launches;
    const int rc = batch_issue(ctx, P);
    const int64_t step_launches = ctx->launches - l0;  // counted when the graph runs
    ctx->launches = l0;
    ctx->capturing = 0;
    ctx->stream = user;
    const cudaError_t e = cudaStreamEndCapture(ctx->cap_stream, &graph);
    if (rc || e != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc ? rc : set_err(ctx, OSC_E_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&P.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        P.exec = nullptr;
        cudaGetLastError();
        return set_err(ctx, OSC_E_CUDA, "batch graph instantiate: %s", cudaGetErrorString(ei));
    }
    P.step_launches = step_launches;
    P.ws_gen = ctx->ws_gen;
    return OSC_OK;
}

int batch_fp32(osc_ctx *ctx, int nb, osc_bunch *bs, const double *x, const double *y, const double *z,
               const double *q, int resize, double *E) {
    const std::string key = plan_key(ctx, nb, bs, x, y, z, q, resize, E);
    std::shared_ptr<BatchPlan> P;
    for (auto it = ctx->batch_plans.begin(); it != ctx->batch_plans.end(); ++it) {
        auto p = std::static_pointer_cast<BatchPlan>(*it);
        if (p->key == key) {
            P = p;
            ctx->batch_plans.splice(ctx->batch_plans.begin(), ctx->batch_plans, it);
            break;
        }
    }
    if (!P) {
        P = std::make_shared<BatchPlan>();
        P->key = key;
        TRY(make_plan(ctx, *P, nb, bs, x, y, z, q, resize, E));
        ctx->batch_plans.push_front(P);
        constexpr size_t kMaxPlans = 12;  // a host-array call plans each of its chunks
        while (ctx->batch_plans.size() > kMaxPlans) {
            TRY(sync(ctx));
            ctx->batch_plans.pop_back();
        }
    }
    TRY(batch_workspaces(ctx, *P));
    if (P->exec && P->ws_gen != ctx->ws_gen) {  // a workspace moved since the capture
        cudaGraphExecDestroy(P->exec);
        P->exec = nullptr;
    }
    for (int b = 0; b < nb; ++b) {
        BunchIn &bi = P->h_in[b];
        for (int d = 0; d < 3; ++d) {
            bi.min[d] = bs[b].mesh.min[d];
            bi.max[d] = bs[b].mesh.max[d];
            bi.delta[d] = bs[b].mesh.delta[d];
        }
        bi.gamma = bs[b].mesh.gamma;
        bi.total_charge = bs[b].total_charge;
    }
    // the first call of a signature runs directly; the second captures the step, and that
    // and every later call run it as one graph launch (profiling times launches one by one)
    const bool graph = ctx->batch_graph && !ctx->profile && P->calls >= 1;
    if (graph && !P->exec && batch_capture(ctx, *P) != OSC_OK) {
        ctx->err.clear();
        cudaGetLastError();
    }
    if (graph && P->exec) {
        CK(cudaGraphLaunch(P->exec, ctx->stream), "batch graph launch");
        ctx->launches += P->step_launches;
        ctx->graph_launches++;
    } else {
        TRY(batch_issue(ctx, *P));
    }
    P->calls++;
    TRY(sync(ctx));
    for (int b = 0; b < nb; ++b) {
        const double *st = P->h_out[b].stats;
        if ((resize || ctx->check_finite) && st[6] > 0)
            return set_err(ctx, OSC_E_NAN, "bunch %d: %.0f non-finite particle coordinates", b, st[6]);
    }
    for (int b = 0; b < nb; ++b) {
        const BunchOut &o = P->h_out[b];
        if (resize)
            for (int d = 0; d < 3; ++d) {
                bs[b].mesh.min[d] = o.min[d];
                bs[b].mesh.max[d] = o.max[d];
                bs[b].mesh.delta[d] = o.delta[d];
            }
        bs[b].mesh.charge = o.charge;
        bs[b].n_outside = (int64_t)P->h_cnt[4 * (size_t)b];
    }
    for (int b = 0; b < nb; ++b) {
        const unsigned long long *hc = P->h_cnt + 4 * (size_t)b;
        if (ctx->check_finite && hc[1])
            return set_err(ctx, OSC_E_NAN, "bunch %d: %llu non-finite particles", b, hc[1]);
        if (ctx->strict_bounds && hc[0])
            return set_err(ctx, OSC_E_BOUNDS, "bunch %d: %llu particles outside the mesh", b, hc[0]);
    }
    return OSC_OK;
}

// The FP32 batch from host arrays, pipelined over chunks of bunches: every chunk's
// particles are copied in on one stream as soon as the call starts, each chunk is solved
// (one batched step) once its copy has landed, and its E rows go back on another stream
// while the next chunk is solved and later chunks are still coming in, so the two copy
// directions and the solves overlap.  Chunks are consecutive bunches in offset order with
// about equal particle counts; a chunk copies the particle range its bunches span.
constexpr int kCopyChunks = 8;  // default; tuning key batch_copy_chunks (1 to 16)

int batch_host_pipelined(osc_ctx *ctx, int nb, osc_bunch *bs, const double *x, const double *y, const double *z,
                         const double *q, int resize, int64_t total, double *E) {
    double *dx, *dy, *dz, *dq = nullptr, *dE;
    TRY(ws_get(ctx, "h_x", sizeof(double) * (size_t)total, (void **)&dx));
    TRY(ws_get(ctx, "h_y", sizeof(double) * (size_t)total, (void **)&dy));
    TRY(ws_get(ctx, "h_z", sizeof(double) * (size_t)total, (void **)&dz));
    if (q) TRY(ws_get(ctx, "h_q", sizeof(double) * (size_t)total, (void **)&dq));
    TRY(ws_get(ctx, "h_pE", sizeof(double) * 3 * (size_t)total, (void **)&dE));
    const int K = std::min(tune_get(ctx, "batch_copy_chunks", kCopyChunks), nb);
    if (!ctx->copy_in) CK(cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking), "copy-in stream");
    if (!ctx->copy_out) CK(cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking), "copy-out stream");
    while ((int)ctx->copy_ev.size() < K + 1) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "copy event");
        ctx->copy_ev.push_back(e);
    }
    // chunks of consecutive bunches (offset order), about total/K particles each
    std::vector<int> order(nb);
    for (int b = 0; b < nb; ++b) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int u, int v) { return bs[u].offset < bs[v].offset; });
    int64_t nall = 0;
    for (int b = 0; b < nb; ++b) nall += bs[b].np;
    std::vector<int> first(K + 1, nb);
    first[0] = 0;
    {
        int c = 1;
        int64_t acc = 0;
        for (int i = 0; i < nb - 1 && c < K; ++i) {
            acc += bs[order[i]].np;
            const int left = nb - (i + 1);  // bunches after this one; every chunk keeps one
            if ((acc * K >= nall * (int64_t)c && left >= K - c) || left == K - c) first[c++] = i + 1;
        }
    }
    std::vector<int64_t> lo(K), hi(K);
    for (int c = 0; c < K; ++c) {
        lo[c] = INT64_MAX;
        hi[c] = 0;
        for (int i = first[c]; i < first[c + 1]; ++i) {
            lo[c] = std::min(lo[c], bs[order[i]].offset);
            hi[c] = std::max(hi[c], bs[order[i]].offset + bs[order[i]].np);
        }
    }
    // the copy-in stream starts after the work already queued on the context's stream
    CK(cudaEventRecord(ctx->copy_ev[K], ctx->stream), "record queued work");
    CK(cudaStreamWaitEvent(ctx->copy_in, ctx->copy_ev[K], 0), "order copies");
    for (int c = 0; c < K; ++c) {
        const size_t n = (size_t)(hi[c] - lo[c]), o = (size_t)lo[c];
        for (const auto &pr : {std::make_pair(dx, x), std::make_pair(dy, y), std::make_pair(dz, z),
                               std::make_pair(dq, q)})
            if (pr.second)
                CK(cudaMemcpyAsync(pr.first + o, pr.second + o, sizeof(double) * n, cudaMemcpyHostToDevice,
                                   ctx->copy_in),
                   "H2D copy");
        CK(cudaEventRecord(ctx->copy_ev[c], ctx->copy_in), "record copy");
    }
    auto drain = [&]() {
        cudaStreamSynchronize(ctx->copy_in);
        cudaStreamSynchronize(ctx->copy_out);
    };
    std::vector<osc_bunch> sub;
    for (int c = 0; c < K; ++c) {
        cudaError_t e = cudaStreamWaitEvent(ctx->stream, ctx->copy_ev[c], 0);
        if (e != cudaSuccess) {
            drain();
            return cuda_check(ctx, e, "wait for copy");
        }
        sub.clear();
        for (int i = first[c]; i < first[c + 1]; ++i) sub.push_back(bs[order[i]]);
        const int rc = batch_fp32(ctx, (int)sub.size(), sub.data(), dx, dy, dz, dq, resize, dE);
        for (int i = first[c]; i < first[c + 1]; ++i) bs[order[i]] = sub[i - first[c]];
        if (rc) {
            drain();
            return rc;
        }
        // batch_fp32 returned after synchronising: the chunk's E rows are final
        const size_t n = (size_t)(hi[c] - lo[c]), o = (size_t)lo[c];
        e = cudaMemcpyAsync(E + 3 * o, dE + 3 * o, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ctx->copy_out);
        if (e != cudaSuccess) {
            drain();
            return cuda_check(ctx, e, "D2H copy");
        }
    }
    return cuda_check(ctx, cudaStreamSynchronize(ctx->copy_out), "copy-out synchronize");
}

}  // namespace

extern "C" {

int osc_batch_space_charge_step_dev(osc_ctx *ctx, int nbunch, osc_bunch *bunches, const double *x, const double *y,
                                    const double *z, const double *q, int resize_mesh, int precision, double *E) {
    if (!ctx) return OSC_E_INVALID;
    TRY(check_prec(ctx, precision));
    TRY(check_bunches(ctx, nbunch, bunches, x, y, z, E));
    if (precision == OSC_PREC_FP32) return batch_fp32(ctx, nbunch, bunches, x, y, z, q, resize_mesh, E);
    for (int b = 0; b < nbunch; ++b) {
        osc_bunch &B = bunches[b];
        const int64_t o = B.offset;
        int64_t nout = 0;
        TRY(osc_space_charge_step_dev(ctx, &B.mesh, B.np, x + o, y + o, z + o, q ? q + o : nullptr,
                                      q ? nullptr : &B.total_charge, resize_mesh, 0, precision, E + 3 * o, nullptr));
        unsigned long long cnt[3];
        TRY(counters_read(ctx, cnt));
        nout = (int64_t)cnt[0];
        B.n_outside = nout;
    }
    return OSC_OK;
}

int osc_batch_space_charge_step(osc_ctx *ctx, int nbunch, osc_bunch *bunches, const double *x, const double *y,
                                const double *z, const double *q, int resize_mesh, int precision, double *E) {
    if (!ctx) return OSC_E_INVALID;
    TRY(check_bunches(ctx, nbunch, bunches, x, y, z, E));
    int64_t total = 0;
    for (int b = 0; b < nbunch; ++b) total = std::max(total, bunches[b].offset + bunches[b].np);
    if (precision == OSC_PREC_FP32 && nbunch >= 2) return batch_host_pipelined(ctx, nbunch, bunches, x, y, z, q,
                                                                               resize_mesh, total, E);
    double *dx, *dy, *dz, *dq, *dE;
    TRY(stage_in(ctx, "h_x", x, (size_t)total, &dx));
    TRY(stage_in(ctx, "h_y", y, (size_t)total, &dy));
    TRY(stage_in(ctx, "h_z", z, (size_t)total, &dz));
    TRY(stage_in(ctx, "h_q", q, (size_t)total, &dq));
    TRY(ws_get(ctx, "h_pE", sizeof(double) * 3 * (size_t)total, (void **)&dE));
    TRY(osc_batch_space_charge_step_dev(ctx, nbunch, bunches, dx, dy, dz, dq, resize_mesh, precision, dE));
    TRY(d2h(ctx, E, dE, sizeof(double) * 3 * (size_t)total));
    return sync(ctx);
}

}  // extern "C"
