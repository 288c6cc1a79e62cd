// context.cu -- context lifetime, workspaces, twiddle tables, Green cache and profiling.
#include <cmath>

#include "context.cuh"

namespace osc {

int set_err(osc_ctx *c, int code, const char *fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

int cuda_check(osc_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return OSC_OK;
    const int code = (e == cudaErrorMemoryAllocation) ? OSC_E_ALLOC : OSC_E_CUDA;
    return set_err(c, code, "%s: %s", what, cudaGetErrorString(e));
}

int ws_get(osc_ctx *c, const char *name, size_t bytes, void **out) {
    // work running on an auxiliary stream slot gets its own copy of every workspace
    DevBuf &b = c->ws_slot ? c->ws[std::string(name) + "#" + std::to_string(c->ws_slot)] : c->ws[name];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
        if (c->capturing) return set_err(c, OSC_E_UNSUPPORTED, "workspace '%s' would grow during graph capture", name);
        ++c->ws_gen;
        if (b.p) {
            cudaStreamSynchronize(c->stream);
            cudaFree(b.p);
            b.p = nullptr;
            b.bytes = 0;
        }
        // round up to 2 MB so small growth does not reallocate every call
        const size_t rb = (bytes + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
        cudaError_t e = cudaMalloc(&b.p, rb);
        if (e != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return set_err(c, OSC_E_ALLOC, "workspace '%s': cudaMalloc(%zu) failed", name, rb);
        }
        b.bytes = rb;
    }
    *out = b.p;
    return OSC_OK;
}

int ctx_sync(osc_ctx *c) {
    const int rc = cuda_check(c, cudaStreamSynchronize(c->stream), "stream synchronize");
    if (rc) return rc;
    if (c->h_fault && *reinterpret_cast<volatile unsigned *>(c->h_fault)) {
        const unsigned f = *c->h_fault;
        *reinterpret_cast<volatile unsigned *>(c->h_fault) = 0;
        return set_err(c, OSC_E_TIMEOUT, "device wait gave up (fault code %u): a bulk copy did not complete", f);
    }
    return OSC_OK;
}

// exp(+2 pi i m/n) in FP64, reducing the angle to one octant so every entry is as exact as
// the FP64 sin/cos of an angle in [0, pi/4].
static void cis_exact(int64_t m, int64_t n, double &cs, double &sn) {
    m %= n;
    if (m < 0) m += n;
    const int64_t num = 8 * m;  // angle = 2*pi*num/(8n)
    const int oct = (int)(num / n);
    const double rem = (double)(num - (int64_t)oct * n) / (double)n;
    const double qpi = 0.78539816339744830961566084581988;  // pi/4
    const double a = rem * qpi;
    const double ca = std::cos(a), sa = std::sin(a);
    const double h2 = 0.70710678118654752440084436210485;
    switch (oct) {  // rotate by oct*pi/4
    case 0: cs = ca; sn = sa; break;
    case 1: cs = h2 * (ca - sa); sn = h2 * (ca + sa); break;
    case 2: cs = -sa; sn = ca; break;
    case 3: cs = -h2 * (ca + sa); sn = h2 * (ca - sa); break;
    case 4: cs = -ca; sn = -sa; break;
    case 5: cs = -h2 * (ca - sa); sn = -h2 * (ca + sa); break;
    case 6: cs = sa; sn = -ca; break;
    default: cs = h2 * (ca + sa); sn = -h2 * (ca - sa); break;
    }
}

template <typename T> static int upload(osc_ctx *c, const std::vector<cplx<T>> &h, DevBuf &b) {
    cudaError_t e = cudaMalloc(&b.p, sizeof(cplx<T>) * h.size());
    if (e != cudaSuccess) return cuda_check(c, e, "twiddle table");
    b.bytes = sizeof(cplx<T>) * h.size();
    e = cudaMemcpy(b.p, h.data(), b.bytes, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? OSC_OK : cuda_check(c, e, "twiddle upload");
}

// Per-stage table of a radix sequence: stage s (Ns = product of earlier radices, radix R)
// has entry (Ns-1) + k*(R-1) + (r-1) = exp(2 pi i r k/(Ns R)) for k < Ns, 1 <= r < R;
// L-1 entries in all.
template <typename T> static std::vector<cplx<T>> stage_table(int L, const int *rad, int nst) {
    std::vector<cplx<T>> h(L, mk<T>((T)1, (T)0));
    int Ns = 1;
    for (int s = 0; s < nst; ++s) {
        const int R = rad[s];
        for (int k = 0; k < Ns; ++k)
            for (int r = 1; r < R; ++r) {
                double cs, sn;
                cis_exact((int64_t)r * k, (int64_t)Ns * R, cs, sn);
                h[(Ns - 1) + k * (R - 1) + (r - 1)] = mk<T>((T)cs, (T)sn);
            }
        Ns *= R;
    }
    return h;
}

// Keys of the table map: L runtime table, -L static-engine stages, L + kWarpKey warp-engine
// stages (a null entry when the length has no such engine).
static constexpr int kWarpKey = 1 << 20;

template <typename T> int twiddles(osc_ctx *c, int L, TwPair<cplx<T>> *out) {
    auto &tab = sizeof(T) == 4 ? c->tw32 : c->tw64;
    if (c->capturing && (tab.find(L) == tab.end() || tab.find(-L) == tab.end() || tab.find(L + kWarpKey) == tab.end()))
        return set_err(c, OSC_E_UNSUPPORTED, "twiddle tables of length %d would be built during graph capture", L);
    if (tab.find(L) == tab.end()) {
        std::vector<cplx<T>> h(L);
        for (int m = 0; m < L; ++m) {
            double cs, sn;
            cis_exact(m, L, cs, sn);
            h[m] = mk<T>((T)cs, (T)sn);
        }
        DevBuf b;
        int rc = upload<T>(c, h, b);
        if (rc) return rc;
        tab[L] = b;
    }
    for (int which = 0; which < 2; ++which) {
        const int key = which == 0 ? -L : L + kWarpKey;
        if (tab.find(key) != tab.end()) continue;
        std::vector<cplx<T>> h;
        auto make = [&](auto eng) -> int {
            using E = decltype(eng);
            if constexpr (E::kLen > 0) h = stage_table<T>(L, E::kRad, E::kNst);
            return 0;
        };
        if (which == 0) dispatch_fft_len<T>(L, make);
        else dispatch_warp_len(L, make);
        DevBuf b{nullptr, 0};
        if (!h.empty()) {
            int rc = upload<T>(c, h, b);
            if (rc) return rc;
        }
        tab[key] = b;
    }
    out->rt = reinterpret_cast<const cplx<T> *>(tab[L].p);
    const DevBuf &s = tab[-L];
    out->st = s.p ? reinterpret_cast<const cplx<T> *>(s.p) : out->rt;
    const DevBuf &w = tab[L + kWarpKey];
    out->wt = w.p ? reinterpret_cast<const cplx<T> *>(w.p) : out->rt;
    return OSC_OK;
}
template int twiddles<float>(osc_ctx *, int, TwPair<cplx<float>> *);
template int twiddles<double>(osc_ctx *, int, TwPair<cplx<double>> *);

static cudaEvent_t ev_get(osc_ctx *c) {
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

Launch::Launch(osc_ctx *c_, const char *name_, int nk_) : c(c_), name(name_), nk(nk_) {
    c->launches += nk;
    if (c->profile) {
        a = ev_get(c);
        cudaEventRecord(a, c->stream);
    }
}
Launch::~Launch() {
    if (c->profile && a) {
        cudaEvent_t b = ev_get(c);
        cudaEventRecord(b, c->stream);
        c->prof_pending.push_back(ProfRec{name, a, b});
    }
}

int tune_get(const osc_ctx *c, const std::string &key, int def) {
    auto it = c->tuning.find(key);
    return it == c->tuning.end() ? def : it->second;
}

int prof_flush(osc_ctx *c) {
    if (c->prof_pending.empty()) return OSC_OK;
    cudaStreamSynchronize(c->stream);
    for (auto &r : c->prof_pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, r.a, r.b);
        ProfSum &s = c->prof[r.name];
        s.launches += 1;
        s.ms += ms;
        c->ev_pool.push_back(r.a);
        c->ev_pool.push_back(r.b);
    }
    c->prof_pending.clear();
    return OSC_OK;
}

GreenSet *gcache_find(osc_ctx *c, const std::string &key) {
    if (c->gcache_budget == 0) return nullptr;  // cache disabled: rebuild on every solve
    for (auto it = c->gcache.begin(); it != c->gcache.end(); ++it) {
        if (it->key == key) {
            it->stamp = ++c->stamp;
            return &*it;
        }
    }
    return nullptr;
}

static size_t gcache_bytes(const osc_ctx *c) {
    size_t t = 0;
    for (auto &s : c->gcache) t += s.bytes;
    return t;
}

// Moves the least recently used set's buffers into the pool; false when the cache is empty.
static bool gcache_evict_one(osc_ctx *c) {
    if (c->gcache.empty()) return false;
    auto victim = c->gcache.begin();
    for (auto it = c->gcache.begin(); it != c->gcache.end(); ++it)
        if (it->stamp < victim->stamp) victim = it;
    for (int i = 0; i < victim->nspec; ++i)
        if (victim->buf[i].p) c->gpool.push_back(victim->buf[i]);
    c->gcache.erase(victim);
    return true;
}

// Frees pooled buffers beyond the most recent 16.
static void gpool_trim(osc_ctx *c) {
    if (c->gpool.size() <= 16) return;
    cudaStreamSynchronize(c->stream);
    while (c->gpool.size() > 16) {
        cudaFree(c->gpool.front().p);
        c->gpool.erase(c->gpool.begin());
    }
}

int green_alloc(osc_ctx *c, size_t bytes, DevBuf &out) {
    for (;;) {
        for (size_t i = 0; i < c->gpool.size(); ++i)
            if (c->gpool[i].bytes == bytes) {
                out = c->gpool[i];
                c->gpool.erase(c->gpool.begin() + i);
                return OSC_OK;
            }
        if (gcache_bytes(c) + bytes <= c->gcache_budget || !gcache_evict_one(c)) break;
    }
    gpool_trim(c);
    out.p = nullptr;
    out.bytes = 0;
    cudaError_t e = cudaMalloc(&out.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        out.p = nullptr;
        return set_err(c, OSC_E_ALLOC, "Green spectrum: cudaMalloc(%zu) failed", bytes);
    }
    out.bytes = bytes;
    return OSC_OK;
}

void green_release(osc_ctx *c, DevBuf &b) {
    if (b.p) c->gpool.push_back(b);
    b.p = nullptr;
    b.bytes = 0;
}

GreenSet *gcache_insert(osc_ctx *c, GreenSet &&g) {
    // evict least recently used sets (into the pool) until the new one fits the budget; with
    // the cache disabled the new set is still kept, as the one the current solve uses
    while (gcache_bytes(c) + g.bytes > c->gcache_budget && gcache_evict_one(c)) {
    }
    gpool_trim(c);
    g.stamp = ++c->stamp;
    c->gcache.push_back(std::move(g));
    return &c->gcache.back();
}

void gcache_free_all(osc_ctx *c) {
    cudaStreamSynchronize(c->stream);
    for (auto &g : c->gcache)
        for (int i = 0; i < g.nspec; ++i) cudaFree(g.buf[i].p);
    c->gcache.clear();
    for (auto &b : c->gpool) cudaFree(b.p);
    c->gpool.clear();
}

}  // namespace osc
