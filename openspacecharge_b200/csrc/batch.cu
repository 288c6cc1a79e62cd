// batch.cu -- batched space-charge steps over many independent bunches
// (osc_batch_space_charge_step*, declared in include/opensc_gpu.h).
//
// FP32: one pass over all particles computes every bunch's bounding box and charge, the
// host refits the meshes (one synchronisation), one pass deposits every bunch into its
// own quad grid, then each group of bunches with the same grid shape is solved by the
// batched pipeline (Green spectra of all members from batched corner blocks and even/odd
// line transforms; the stacked FFT passes with the members as extra rows, planes and
// columns), and one pass interpolates E for every particle.  The reference solves one
// bunch per call (space_charge_3d, code/open_spacecharge_mod.f90:431-489).
#include <algorithm>
#include <map>
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

int upload(osc_ctx *ctx, const char *name, const void *h, size_t bytes, void **d) {
    TRY(ws_get(ctx, name, bytes > 0 ? bytes : 16, d));
    if (bytes == 0) return OSC_OK;
    return h2d(ctx, *d, h, bytes);
}

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

int batch_fp32(osc_ctx *ctx, int nb, osc_bunch *bs, const double *x, const double *y, const double *z,
               const double *q, int resize, double *E) {
    // CTA jobs of the particle passes, bunch by bunch
    std::vector<BatchJob> jobs;
    std::vector<int> job0(nb + 1);
    for (int b = 0; b < nb; ++b) {
        job0[b] = (int)jobs.size();
        for (int64_t beg = 0; beg < bs[b].np; beg += kJobParticles)
            jobs.push_back(BatchJob{b, beg, std::min(beg + kJobParticles, bs[b].np)});
    }
    job0[nb] = (int)jobs.size();
    const int njobs = (int)jobs.size();
    std::vector<BunchArgs> ba(nb);
    std::memset(ba.data(), 0, sizeof(BunchArgs) * nb);
    for (int b = 0; b < nb; ++b) {
        const int64_t o = bs[b].offset;
        ba[b].d.x = x + o;
        ba[b].d.y = y + o;
        ba[b].d.z = z + o;
        ba[b].d.q = q ? q + o : nullptr;
        ba[b].d.np = bs[b].np;
    }
    BunchArgs *d_ba;
    BatchJob *d_jobs;
    int *d_job0;
    TRY(upload(ctx, "batch_args", ba.data(), sizeof(BunchArgs) * nb, (void **)&d_ba));
    TRY(upload(ctx, "batch_jobs", jobs.data(), sizeof(BatchJob) * njobs, (void **)&d_jobs));
    TRY(upload(ctx, "batch_job0", job0.data(), sizeof(int) * (nb + 1), (void **)&d_job0));
    // bounding boxes, non-finite counts and charges of all bunches, one synchronisation
    unsigned long long *keys;
    double *qsum, *stats;
    TRY(ws_get(ctx, "batch_keys", sizeof(unsigned long long) * 7 * (size_t)std::max(njobs, 1), (void **)&keys));
    TRY(ws_get(ctx, "batch_qsum", sizeof(double) * (size_t)std::max(njobs, 1), (void **)&qsum));
    TRY(ws_get(ctx, "batch_stats", sizeof(double) * 8 * (size_t)nb, (void **)&stats));
    {
        Launch L_(ctx, "batch_stats", 2);
        if (launch_batch_stats(d_ba, d_jobs, njobs, d_job0, nb, keys, qsum, stats, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "batch stats");
    }
    std::vector<double> hst(8 * (size_t)nb);
    TRY(d2h(ctx, hst.data(), stats, sizeof(double) * hst.size()));
    TRY(sync(ctx));
    std::vector<double> charge1(nb);
    for (int b = 0; b < nb; ++b) {
        const double *st = &hst[8 * (size_t)b];
        if ((resize || ctx->check_finite) && st[6] > 0)
            return set_err(ctx, OSC_E_NAN, "bunch %d: %.0f non-finite particle coordinates", b, st[6]);
        if (resize) {
            const double mn[3] = {st[0], st[2], st[4]}, mx[3] = {st[1], st[3], st[5]};
            apply_refit(&bs[b].mesh, mn, mx);
        }
        if (q) {
            bs[b].mesh.charge = st[7];
            charge1[b] = 0;
        } else {
            bs[b].mesh.charge = bs[b].total_charge;
            charge1[b] = bs[b].total_charge / (double)bs[b].np;
        }
    }
    // groups of equal grids; members stacked along z in the batch arrays
    std::map<std::tuple<int, int, int>, Group> groups;
    for (int b = 0; b < nb; ++b) {
        int n[3];
        TRY(mesh_dims(ctx, &bs[b].mesh, n));
        Group &g = groups[std::make_tuple(n[0], n[1], n[2])];
        for (int d = 0; d < 3; ++d) g.n[d] = n[d];
        g.members.push_back(b);
    }
    int64_t nodes = 0;
    size_t max_f = 0, max_g = 0;
    for (auto &kv : groups) {
        Group &g = kv.second;
        const int64_t N = (int64_t)g.n[0] * g.n[1] * g.n[2];
        g.node0 = nodes;
        for (size_t i = 0; i < g.members.size(); ++i) {
            const int b = g.members[i];
            BunchArgs &a = ba[b];
            const int64_t o = bs[b].offset;
            a.d = deposit_args(&bs[b].mesh, g.n, bs[b].np, x + o, y + o, z + o, q ? q + o : nullptr, charge1[b],
                               ctx->check_finite);
            a.in = interp_args(&bs[b].mesh, g.n, bs[b].np, x + o, y + o, z + o);
            a.node_off = nodes + (int64_t)i * N;
            a.E = E + 3 * o;
        }
        nodes += N * (int64_t)g.members.size();
        const size_t B = g.members.size();
        max_f = std::max(max_f, 3 * B * (size_t)(g.n[0] + 1) * (g.n[1] + 1) * (g.n[2] + 1));
        const int zp = green_zpitch(g.n[2] + 1, sizeof(float));
        max_g = std::max(max_g, 3 * B * (size_t)(g.n[0] + 1) * (g.n[1] + 1) * zp);
    }
    TRY(upload(ctx, "batch_args", ba.data(), sizeof(BunchArgs) * nb, (void **)&d_ba));
    // corner-block arguments of every group's members and components, one upload
    std::vector<CornerArgs> ca_all;
    std::vector<size_t> ca_off;
    for (auto &kv : groups) {
        Group &g = kv.second;
        const int B = (int)g.members.size();
        const double off0[3] = {0, 0, 0};
        ca_off.push_back(ca_all.size());
        for (int comp = 1; comp <= 3; ++comp)
            for (int i = 0; i < B; ++i) {
                const osc_mesh3d &m = bs[g.members[i]].mesh;
                ca_all.push_back(green_corner_args(g.n, m.delta, m.gamma, off0, comp));
            }
    }
    CornerArgs *d_ca_all;
    TRY(upload(ctx, "batch_corners", ca_all.data(), sizeof(CornerArgs) * ca_all.size(), (void **)&d_ca_all));
    // grow the per-group workspaces to the largest group once (growing one synchronises)
    {
        size_t x1 = 0, x2 = 0, x3 = 0, x4 = 0, h = 0, hx = 0, hy = 0;
        for (auto &kv : groups) {
            const Group &g = kv.second;
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
        for (int slot = 1; slot <= kSlots; ++slot) {
            SlotGuard sg(ctx, slot);
            void *p;
            TRY(ws_get(ctx, "fs_x1", sizeof(float2) * x1, &p));
            TRY(ws_get(ctx, "fs_x2", sizeof(float2) * x2, &p));
            TRY(ws_get(ctx, "fs_x3", sizeof(float2) * x3, &p));
            TRY(ws_get(ctx, "fs_x4", sizeof(float2) * x4, &p));
            TRY(ws_get(ctx, "green_h", sizeof(double) * h, &p));
            TRY(ws_get(ctx, "green_hx", sizeof(double) * hx, &p));
            TRY(ws_get(ctx, "green_hy", sizeof(double) * hy, &p));
            TRY(ws_get(ctx, "batch_F", sizeof(double) * max_f, &p));
            TRY(ws_get(ctx, "batch_green", sizeof(float) * max_g, &p));
        }
    }
    // deposit every bunch into its quad grid
    float *quad, *e8;
    unsigned long long *cnt;
    TRY(ws_get(ctx, "batch_quad", sizeof(float) * 4 * (size_t)nodes, (void **)&quad));
    TRY(ws_get(ctx, "batch_e8", sizeof(float) * 8 * (size_t)nodes, (void **)&e8));
    TRY(ws_get(ctx, "batch_cnt", sizeof(unsigned long long) * 4 * (size_t)nb, (void **)&cnt));
    CK(cudaMemsetAsync(quad, 0, sizeof(float) * 4 * (size_t)nodes, ctx->stream), "memset quad");
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 4 * (size_t)nb, ctx->stream), "memset counters");
    {
        Launch L_(ctx, "batch_deposit");
        if (launch_batch_deposit_quad(d_ba, d_jobs, njobs, quad, cnt, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "batch deposit");
    }
    // field of every group: groups of different shapes are independent, so they run on
    // kSlots auxiliary streams (each with its own workspaces) after the deposit
    CK(cudaEventRecord(ctx->aux_ev[kSlots], ctx->stream), "record deposit");
    for (int s2 = 0; s2 < kSlots; ++s2) CK(cudaStreamWaitEvent(ctx->aux[s2], ctx->aux_ev[kSlots], 0), "wait deposit");
    // largest groups first, each on the stream with the least work queued so far, so the
    // streams finish together (cost ~ members x corner-block nodes)
    std::vector<std::pair<Group *, size_t>> order;  // (group, index in map order)
    for (auto &kv : groups) order.push_back({&kv.second, order.size()});
    auto gcost = [](const Group *g) {
        return (double)g->members.size() * (g->n[0] + 1) * (double)(g->n[1] + 1) * (double)(g->n[2] + 1);
    };
    std::stable_sort(order.begin(), order.end(),
                     [&](const std::pair<Group *, size_t> &u, const std::pair<Group *, size_t> &v) {
                         return gcost(u.first) > gcost(v.first);
                     });
    double queued[kSlots] = {};
    for (auto &og : order) {
        Group &g = *og.first;
        int slot = 0;
        for (int s2 = 1; s2 < kSlots; ++s2)
            if (queued[s2] < queued[slot]) slot = s2;
        queued[slot] += gcost(&g);
        SlotGuard sg(ctx, slot + 1);
        float *gbuf;
        double *F;
        TRY(ws_get(ctx, "batch_F", sizeof(double) * max_f, (void **)&F));
        TRY(ws_get(ctx, "batch_green", sizeof(float) * max_g, (void **)&gbuf));
        const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
        const int B = (int)g.members.size();
        const int64_t N = (int64_t)nx * ny * nz;
        const int zinner = zconv_warp_ok(2 * nz, nz, 4) ? 1 : 0;
        const int zp = zinner ? green_zpitch(nz + 1, sizeof(float)) : nz + 1;
        const int64_t per = (int64_t)(nx + 1) * (ny + 1) * zp;
        const int64_t fstride = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
        if (zinner) CK(cudaMemsetAsync(gbuf, 0, sizeof(float) * 3 * B * per, ctx->stream), "memset spectra");
        // Green spectra of the three E components of every member: members m = comp*B + i
        const CornerArgs *d_ca = d_ca_all + ca_off[og.second];
        {
            Launch L_(ctx, "green_corners");
            if (launch_igf_corners_batch(F, d_ca, 3 * B, fstride, fstride, ctx->stream))
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
        (void)N;
    }
    for (int s2 = 0; s2 < kSlots; ++s2) {
        CK(cudaEventRecord(ctx->aux_ev[s2], ctx->aux[s2]), "record group");
        CK(cudaStreamWaitEvent(ctx->stream, ctx->aux_ev[s2], 0), "wait groups");
    }
    {
        Launch L_(ctx, "batch_interp");
        if (launch_batch_interp_pairs(d_ba, d_jobs, njobs, e8, cnt, ctx->stream))
            return set_err(ctx, OSC_E_CUDA, "batch interp");
    }
    std::vector<unsigned long long> hc(4 * (size_t)nb);
    TRY(d2h(ctx, hc.data(), cnt, sizeof(unsigned long long) * hc.size()));
    TRY(sync(ctx));
    for (int b = 0; b < nb; ++b) {
        bs[b].n_outside = (int64_t)hc[4 * (size_t)b];
        if (ctx->check_finite && hc[4 * (size_t)b + 1])
            return set_err(ctx, OSC_E_NAN, "bunch %d: %llu non-finite particles", b, hc[4 * (size_t)b + 1]);
        if (ctx->strict_bounds && hc[4 * (size_t)b])
            return set_err(ctx, OSC_E_BOUNDS, "bunch %d: %llu particles outside the mesh", b, hc[4 * (size_t)b]);
    }
    return OSC_OK;
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
