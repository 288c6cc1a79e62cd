// osc_fft.cuh -- shared-memory Stockham FFT building blocks for sm_100a.
//
// A CTA transforms NL independent lines of length L that sit interleaved in shared memory:
// element e of line l is buf[e*lstr + l] with lstr = NL+1 (odd, so the 8/16-byte complex
// accesses of a warp spread over all banks).  Threads are mapped line-fastest, so the NL
// lanes that share a butterfly index touch consecutive words.  Each stage is an in-place
// mixed-radix Stockham step: every thread loads the R inputs of its butterflies (with the
// stage twiddle), the CTA synchronises, then every thread writes its R outputs to their
// autosorted positions.  The CTA has L*NL/FFT_EPT threads, so each thread owns FFT_EPT
// complex values per stage and all butterflies of a stage fit in registers.
//
// Twiddles come from a table tw[m] = exp(+2*pi*i*m/L) computed on the host in FP64 (and
// rounded once for FP32) and staged in shared memory; sign -1 uses the conjugate.
// Convention: X[k] = sum_j x[j] exp(sign*2*pi*i*j*k/L), unnormalised -- the sign
// convention of the reference's ccfft3d / Singleton sfft (code/fft_interface_mod.f90:96).
#pragma once

#include "osc_common.cuh"

namespace osc {

constexpr int FFT_MAX_STAGES = 12;
constexpr int FFT_EPT = 16;
constexpr int FFT_MAX_LEN = 2048;

struct FFTPlan {
    int L;
    int nst;
    int radix[FFT_MAX_STAGES];
};

// Host: radix plan for L = 2^a 3^b 5^c (radix 8 first, then 4, 2, 3, 5).  Returns false
// for other lengths or L > FFT_MAX_LEN.
bool make_fft_plan(int L, FFTPlan &p);
// Threads of a CTA that transforms NL lines of length L.
inline int fft_threads(int L, int NL) { return (L * NL) / FFT_EPT; }
int pick_nl(int L, int nl_max, size_t elem_bytes, int nbuf, size_t budget);

template <typename V> __device__ __forceinline__ V tw_get(const V *tw, int m, int sign) {
    V w = tw[m];
    if (sign < 0) w.y = -w.y;
    return w;
}

template <int R> struct Dft;

template <> struct Dft<2> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int, const V *, int) {
        V a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <> struct Dft<4> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int s, const V *, int) {
        V apc = cadd(v[0], v[2]), amc = csub(v[0], v[2]);
        V bpd = cadd(v[1], v[3]), bmd = csub(v[1], v[3]);
        V jb = cmul_si(bmd, s);
        v[0] = cadd(apc, bpd);
        v[1] = cadd(amc, jb);
        v[2] = csub(apc, bpd);
        v[3] = csub(amc, jb);
    }
};

template <> struct Dft<8> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int s, const V *, int) {
        typedef decltype(v[0].x) T;
        const T h = (T)0.70710678118654752440084436210485;
        V a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            a[r] = cadd(v[r], v[r + 4]);
            b[r] = csub(v[r], v[r + 4]);
        }
        // b_r *= w8^r, w8 = exp(s*i*pi/4)
        {
            V t = b[1];  // * h(1 + s i)
            V u;
            u.x = h * (t.x - (T)s * t.y);
            u.y = h * (t.y + (T)s * t.x);
            b[1] = u;
            b[2] = cmul_si(b[2], s);
            t = b[3];  // * h(-1 + s i)
            u.x = h * (-t.x - (T)s * t.y);
            u.y = h * (-t.y + (T)s * t.x);
            b[3] = u;
        }
        Dft<4>::run(a, s, (const V *)nullptr, 0);
        Dft<4>::run(b, s, (const V *)nullptr, 0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            v[2 * q] = a[q];
            v[2 * q + 1] = b[q];
        }
    }
};

template <> struct Dft<3> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int s, const V *tw, int L) {
        typedef decltype(v[0].x) T;
        const T h = tw[L / 3].y;  // sin(2*pi/3)
        V a = v[0], t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        V m;
        m.x = a.x - (T)0.5 * t.x;
        m.y = a.y - (T)0.5 * t.y;
        V jd;
        jd.x = -(T)s * h * d.y;
        jd.y = (T)s * h * d.x;
        v[0] = cadd(a, t);
        v[1] = cadd(m, jd);
        v[2] = csub(m, jd);
    }
};

template <> struct Dft<5> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int s, const V *tw, int L) {
        V out[5];
        const int step = L / 5;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            V acc = v[0];
#pragma unroll
            for (int r = 1; r < 5; ++r) acc = cadd(acc, cmul(v[r], tw_get(tw, ((r * q) % 5) * step, s)));
            out[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) v[q] = out[q];
    }
};

// One Stockham stage over NL interleaved lines; all threads of the CTA must call it.
template <typename V, int R, int NL>
__device__ __forceinline__ void stockham_stage(V *buf, int lstr, int L, int Ns, const V *tw, int sign) {
    constexpr int MAXB = (FFT_EPT + R - 1) / R;
    const int nthreads = blockDim.x * blockDim.y;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nb = L / R;
    const int total = nb * NL;
    const int tstep = L / (Ns * R);
    V v[MAXB][R];
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        const int b = tid + q * nthreads;
        if (b < total) {
            const int line = b % NL;
            const int j = b / NL;
            const int k = j % Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                V x = buf[(j + r * nb) * lstr + line];
                if (r) x = cmul(x, tw_get(tw, r * k * tstep, sign));
                v[q][r] = x;
            }
            Dft<R>::run(v[q], sign, tw, L);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        const int b = tid + q * nthreads;
        if (b < total) {
            const int line = b % NL;
            const int j = b / NL;
            const int k = j % Ns;
            const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[(idxD + r * Ns) * lstr + line] = v[q][r];
        }
    }
    __syncthreads();
}

// Full transform of the NL interleaved lines in buf.  Caller synchronises before.
template <typename V, int NL>
__device__ __forceinline__ void fft_smem(V *buf, int lstr, const FFTPlan &p, const V *tw, int sign) {
    int Ns = 1;
    for (int s = 0; s < p.nst; ++s) {
        const int R = p.radix[s];
        switch (R) {
        case 8: stockham_stage<V, 8, NL>(buf, lstr, p.L, Ns, tw, sign); break;
        case 4: stockham_stage<V, 4, NL>(buf, lstr, p.L, Ns, tw, sign); break;
        case 2: stockham_stage<V, 2, NL>(buf, lstr, p.L, Ns, tw, sign); break;
        case 3: stockham_stage<V, 3, NL>(buf, lstr, p.L, Ns, tw, sign); break;
        default: stockham_stage<V, 5, NL>(buf, lstr, p.L, Ns, tw, sign); break;
        }
        Ns *= R;
    }
}

// Compile-time version of one stage: L, Ns, R and NL are constants, so every index is a
// shift or a multiply by a constant and all butterflies stay in registers.
template <typename V, int R, int NL, int L, int Ns>
__device__ __forceinline__ void stage_ct(V *buf, const V *tw, int sign) {
    constexpr int lstr = NL + 1;
    constexpr int MAXB = (FFT_EPT + R - 1) / R;
    constexpr int nb = L / R;
    constexpr int total = nb * NL;
    constexpr int tstep = L / (Ns * R);
    constexpr int nthreads = L * NL / FFT_EPT;
    const int tid = threadIdx.x;
    V v[MAXB][R];
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        const int b = tid + q * nthreads;
        if (total % nthreads == 0 || b < total) {
            const int line = b % NL, j = b / NL, k = j % Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                V x = buf[(j + r * nb) * lstr + line];
                if (r && Ns > 1) x = cmul(x, tw_get(tw, r * k * tstep, sign));
                v[q][r] = x;
            }
            Dft<R>::run(v[q], sign, tw, L);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        const int b = tid + q * nthreads;
        if (total % nthreads == 0 || b < total) {
            const int line = b % NL, j = b / NL, k = j % Ns;
            const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[(idxD + r * Ns) * lstr + line] = v[q][r];
        }
    }
    __syncthreads();
}

template <typename V, int NL, int L, int Ns, int R, int... Rest>
__device__ __forceinline__ void fft_ct(V *buf, const V *tw, int sign) {
    stage_ct<V, R, NL, L, Ns>(buf, tw, sign);
    if constexpr (sizeof...(Rest) > 0) fft_ct<V, NL, L, Ns * R, Rest...>(buf, tw, sign);
}

// FFT engines.  FftRuntime follows a runtime radix plan (any supported length); its
// CTAs are capped at 256 threads so the generic stage code keeps its registers.
// FftStatic<L, R...> is the compile-time radix sequence for one length.
struct FftRuntime {
    static constexpr int kLen = 0;
    static constexpr int kMaxThreads = 256;
    template <typename V, int NL>
    __device__ __forceinline__ static void run(V *buf, const FFTPlan &p, const V *tw, int sign) {
        fft_smem<V, NL>(buf, NL + 1, p, tw, sign);
    }
};
template <int L_, int... Rs> struct FftStatic {
    static constexpr int kLen = L_;
    static constexpr int kMaxThreads = 512;
    template <typename V, int NL>
    __device__ __forceinline__ static void run(V *buf, const FFTPlan &, const V *tw, int sign) {
        fft_ct<V, NL, L_, 1, Rs...>(buf, tw, sign);
    }
};

// Lines per CTA for a static engine: the largest NL <= nl_max with a whole number of
// threads, at most 512 threads, and nbuf line buffers within ~100 KB of shared memory.
constexpr int nl_static(int L, int nl_max, int elem_bytes, int nbuf) {
    int nl = nl_max;
    while (nl > 2 && ((L * nl) % FFT_EPT != 0 || (L * nl) / FFT_EPT > 512 ||
                      nbuf * L * (nl + 1) * elem_bytes + L * elem_bytes > 100 * 1024))
        nl /= 2;
    return nl;
}

// Calls f(engine) with the static engine for L when there is one, else FftRuntime.
template <class F> inline int dispatch_fft_len(int L, F &&f) {
    switch (L) {
    case 32: return f(FftStatic<32, 8, 4>{});
    case 64: return f(FftStatic<64, 8, 8>{});
    case 96: return f(FftStatic<96, 8, 4, 3>{});
    case 128: return f(FftStatic<128, 8, 4, 4>{});
    case 192: return f(FftStatic<192, 8, 8, 3>{});
    case 256: return f(FftStatic<256, 8, 8, 4>{});
    case 384: return f(FftStatic<384, 8, 8, 2, 3>{});
    case 512: return f(FftStatic<512, 8, 8, 8>{});
    default: return f(FftRuntime{});
    }
}

// Stage the twiddle table of length L into shared memory.
template <typename V> __device__ __forceinline__ void load_twiddles(V *tw_s, const V *tw_g, int L) {
    const int nthreads = blockDim.x * blockDim.y;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    for (int m = tid; m < L; m += nthreads) tw_s[m] = tw_g[m];
}

}  // namespace osc
