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
    DevBuf &b = c->ws[name];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
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

template <typename T> int twiddles(osc_ctx *c, int L, const cplx<T> **out) {
    auto &tab = sizeof(T) == 4 ? c->tw32 : c->tw64;
    auto it = tab.find(L);
    if (it != tab.end()) {
        *out = reinterpret_cast<const cplx<T> *>(it->second.p);
        return OSC_OK;
    }
    std::vector<cplx<T>> h(L);
    // exp(+2 pi i m/L) in FP64, using the octant symmetry so every entry is as exact as
    // the FP64 sin/cos of an angle in [0, pi/4]
    for (int m = 0; m < L; ++m) {
        // reduce m/L to [0,1/8] turns
        const int64_t num = (int64_t)8 * m;  // angle = 2*pi*num/(8L)
        const int oct = (int)(num / L);      // octant 0..7
        const double rem = (double)(num - (int64_t)oct * L) / (double)L;  // fraction of an octant
        double cs, sn;
        const double qpi = 0.78539816339744830961566084581988;  // pi/4
        const double a = rem * qpi;
        const double ca = std::cos(a), sa = std::sin(a);
        const double h2 = 0.70710678118654752440084436210485;
        // rotate by oct*pi/4
        switch (oct) {
        case 0: cs = ca; sn = sa; break;
        case 1: cs = h2 * (ca - sa); sn = h2 * (ca + sa); break;
        case 2: cs = -sa; sn = ca; break;
        case 3: cs = -h2 * (ca + sa); sn = h2 * (ca - sa); break;
        case 4: cs = -ca; sn = -sa; break;
        case 5: cs = -h2 * (ca - sa); sn = -h2 * (ca + sa); break;
        case 6: cs = sa; sn = -ca; break;
        default: cs = h2 * (ca + sa); sn = -h2 * (ca - sa); break;
        }
        h[m] = mk<T>((T)cs, (T)sn);
    }
    DevBuf b;
    cudaError_t e = cudaMalloc(&b.p, sizeof(cplx<T>) * L);
    if (e != cudaSuccess) return cuda_check(c, e, "twiddle table");
    b.bytes = sizeof(cplx<T>) * L;
    e = cudaMemcpy(b.p, h.data(), b.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_check(c, e, "twiddle upload");
    tab[L] = b;
    *out = reinterpret_cast<const cplx<T> *>(b.p);
    return OSC_OK;
}
template int twiddles<float>(osc_ctx *, int, const cplx<float> **);
template int twiddles<double>(osc_ctx *, int, const cplx<double> **);

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
    for (auto it = c->gcache.begin(); it != c->gcache.end(); ++it) {
        if (it->key == key) {
            it->stamp = ++c->stamp;
            return &*it;
        }
    }
    return nullptr;
}

GreenSet *gcache_insert(osc_ctx *c, GreenSet &&g) {
    // evict least recently used sets until the new one fits the budget
    size_t total = g.bytes;
    for (auto &s : c->gcache) total += s.bytes;
    while (total > c->gcache_budget && !c->gcache.empty()) {
        auto victim = c->gcache.begin();
        for (auto it = c->gcache.begin(); it != c->gcache.end(); ++it)
            if (it->stamp < victim->stamp) victim = it;
        cudaStreamSynchronize(c->stream);
        for (int i = 0; i < victim->nspec; ++i) cudaFree(victim->buf[i].p);
        total -= victim->bytes;
        c->gcache.erase(victim);
    }
    g.stamp = ++c->stamp;
    c->gcache.push_back(std::move(g));
    return &c->gcache.back();
}

}  // namespace osc
