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
// Two engines share these stages.  FftStatic<L, R...> fixes the radix sequence at compile
// time (every index is a shift or a constant multiply) and reads its twiddles from a
// per-stage table laid out [stage][k][r-1], so the lanes of a warp read consecutive words.
// Its first stage can skip the zero upper half of the input (forward transforms of the
// zero-padded doubled grid) and its last stage can skip the upper half of the output
// (inverse transforms whose physical window is the lower half).  FftRuntime follows a
// runtime radix plan for any other 2^a 3^b 5^c length with the table tw[m]=exp(2 pi i m/L).
//
// Twiddles are computed on the host in FP64 and rounded once for FP32; sign -1 uses the
// conjugate.  Convention: X[k] = sum_j x[j] exp(sign*2*pi*i*j*k/L), unnormalised -- the sign
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
// for other lengths, odd lengths or L > FFT_MAX_LEN.
bool make_fft_plan(int L, FFTPlan &p);
// Threads of a CTA that transforms NL lines of length L.
inline int fft_threads(int L, int NL, int ept = FFT_EPT) { return (L * NL) / ept; }

template <typename V> __device__ __forceinline__ V tw_get(const V *tw, int m, int sign) {
    V w = tw[m];
    if (sign < 0) w.y = -w.y;
    return w;
}

// Small DFTs in registers: y[q] = sum_r v[r] exp(s*2*pi*i*r*q/R).
template <int R> struct Dft;

template <> struct Dft<2> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int) {
        V a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <> struct Dft<4> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int s) {
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
    template <typename V> __device__ __forceinline__ static void run(V *v, int s) {
        typedef decltype(v[0].x) T;
        const T h = (T)0.70710678118654752440084436210485;  // cos(pi/4)
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
        Dft<4>::run(a, s);
        Dft<4>::run(b, s);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            v[2 * q] = a[q];
            v[2 * q + 1] = b[q];
        }
    }
};

// Radix 16 by decimation in frequency: X[2q] is the 8-point DFT of a_r = v_r + v_{r+8},
// X[2q+1] the 8-point DFT of b_r = (v_r - v_{r+8}) w16^r, w16 = exp(s i pi/8).
template <> struct Dft<16> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int s) {
        typedef decltype(v[0].x) T;
        const T c1 = (T)0.92387953251128675612818318939679;  // cos(pi/8)
        const T s1 = (T)0.38268343236508977172845998403040;  // sin(pi/8)
        const T h = (T)0.70710678118654752440084436210485;   // cos(pi/4)
        const T sg = (T)s;
        V a[8], b[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            a[r] = cadd(v[r], v[r + 8]);
            b[r] = csub(v[r], v[r + 8]);
        }
        // b_r *= cos(r pi/8) + s i sin(r pi/8)
        auto rot = [&](V &t, T cr, T sr) {
            const V u = t;
            t.x = cr * u.x - sg * sr * u.y;
            t.y = cr * u.y + sg * sr * u.x;
        };
        rot(b[1], c1, s1);
        rot(b[2], h, h);
        rot(b[3], s1, c1);
        b[4] = cmul_si(b[4], s);
        rot(b[5], -s1, c1);
        rot(b[6], -h, h);
        rot(b[7], -c1, s1);
        Dft<8>::run(a, s);
        Dft<8>::run(b, s);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            v[2 * q] = a[q];
            v[2 * q + 1] = b[q];
        }
    }
};

template <> struct Dft<3> {
    template <typename V> __device__ __forceinline__ static void run(V *v, int s) {
        typedef decltype(v[0].x) T;
        const T h = (T)0.86602540378443864676372317075294;  // sin(2 pi/3)
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
    template <typename V> __device__ __forceinline__ static void run(V *v, int s) {
        typedef decltype(v[0].x) T;
        const T c1 = (T)0.30901699437494742410229341718282;   // cos(2 pi/5)
        const T c2 = (T)-0.80901699437494742410229341718282;  // cos(4 pi/5)
        const T s1 = (T)0.95105651629515357211643933337938;   // sin(2 pi/5)
        const T s2 = (T)0.58778525229247312916870595463907;   // sin(4 pi/5)
        const V x0 = v[0];
        const V a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        const V a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        V p1, p2, q1, q2;
        p1.x = x0.x + c1 * a1.x + c2 * a2.x;
        p1.y = x0.y + c1 * a1.y + c2 * a2.y;
        p2.x = x0.x + c2 * a1.x + c1 * a2.x;
        p2.y = x0.y + c2 * a1.y + c1 * a2.y;
        q1.x = s1 * b1.x + s2 * b2.x;
        q1.y = s1 * b1.y + s2 * b2.y;
        q2.x = s2 * b1.x - s1 * b2.x;
        q2.y = s2 * b1.y - s1 * b2.y;
        const V j1 = cmul_si(q1, s), j2 = cmul_si(q2, s);
        v[0] = cadd(x0, cadd(a1, a2));
        v[1] = cadd(p1, j1);
        v[4] = csub(p1, j1);
        v[2] = cadd(p2, j2);
        v[3] = csub(p2, j2);
    }
};

// ---- runtime-plan engine ----------------------------------------------------------------
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
            Dft<R>::run(v[q], sign);
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

// ---- compile-time engine ------------------------------------------------------------------
// MODE 0: full stage; 1: first stage whose upper input half is zero (not read);
// 2: last stage whose upper output half is not needed (not written).
template <typename V, int R, int NL, int L, int Ns, int MODE, int EPT>
__device__ __forceinline__ void stage_ct(V *buf, const V *tw, int sign) {
    constexpr int lstr = NL + 1;
    constexpr int MAXB = (EPT + R - 1) / R;
    constexpr int nb = L / R;
    constexpr int total = nb * NL;
    constexpr int nthreads = L * NL / EPT;
    constexpr int toff = Ns - 1;  // this stage's block of the per-stage twiddle table
    constexpr bool half_in = MODE == 1 && (R % 2 == 0);
    constexpr bool half_out = MODE == 2 && (R % 2 == 0);
    const int tid = threadIdx.x;
    V v[MAXB][R];
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        const int b = tid + q * nthreads;
        if (total % nthreads == 0 || b < total) {
            const int line = b % NL, j = b / NL, k = j % Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                V x;
                if (half_in && r >= R / 2) {
                    x.x = 0;
                    x.y = 0;
                } else {
                    x = buf[(j + r * nb) * lstr + line];
                    if (r && Ns > 1) x = cmul(x, tw_get(tw, toff + k * (R - 1) + (r - 1), sign));
                }
                v[q][r] = x;
            }
            Dft<R>::run(v[q], sign);
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
            for (int r = 0; r < R; ++r)
                if (!half_out || r < R / 2) buf[(idxD + r * Ns) * lstr + line] = v[q][r];
        }
    }
    __syncthreads();
}

template <typename V, int NL, int L, int Ns, bool HIN, bool HOUT, int EPT, int R, int... Rest>
__device__ __forceinline__ void fft_ct(V *buf, const V *tw, int sign) {
    constexpr bool last = sizeof...(Rest) == 0;
    constexpr int mode = (Ns == 1 && HIN) ? 1 : ((last && HOUT) ? 2 : 0);
    stage_ct<V, R, NL, L, Ns, mode, EPT>(buf, tw, sign);
    if constexpr (!last) fft_ct<V, NL, L, Ns * R, false, HOUT, EPT, Rest...>(buf, tw, sign);
}

// Stage with explicit input and output functors: ld(e, line) -> V and st(e, line, V).
// The first stage of a transform can read straight from global memory (or compute its
// input, e.g. a spectral product) and the last stage can write straight to global memory,
// which saves two shared-memory passes per transform.
template <typename V, int R, int NL, int L, int Ns, bool HALF_IN, bool HALF_OUT, int EPT, class LD, class ST>
__device__ __forceinline__ void stage_io(const LD &ld, const ST &st, const V *tw, int sign) {
    constexpr int MAXB = (EPT + R - 1) / R;
    constexpr int nb = L / R;
    constexpr int total = nb * NL;
    constexpr int nthreads = L * NL / EPT;
    constexpr int toff = Ns - 1;
    constexpr bool half_in = HALF_IN && (R % 2 == 0);
    constexpr bool half_out = HALF_OUT && (R % 2 == 0);
    const int tid = threadIdx.x;
    V v[MAXB][R];
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        const int b = tid + q * nthreads;
        if (total % nthreads == 0 || b < total) {
            const int line = b % NL, j = b / NL, k = j % Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                V x;
                if (half_in && r >= R / 2) {
                    x.x = 0;
                    x.y = 0;
                } else {
                    x = ld(j + r * nb, line);
                    if (r && Ns > 1) x = cmul(x, tw_get(tw, toff + k * (R - 1) + (r - 1), sign));
                }
                v[q][r] = x;
            }
            Dft<R>::run(v[q], sign);
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
            for (int r = 0; r < R; ++r)
                if (!half_out || r < R / 2) st(idxD + r * Ns, line, v[q][r]);
        }
    }
    __syncthreads();
}

template <int... Rs> struct Radices {};

template <typename V, int NL, int L, int Ns, bool HIN, bool HOUT, int EPT, int R, int... Rest, class LD, class ST>
__device__ __forceinline__ void fft_io_rec(Radices<R, Rest...>, V *buf, const V *tw, int sign, const LD &ld,
                                           const ST &st) {
    constexpr bool first = Ns == 1, last = sizeof...(Rest) == 0;
    constexpr int lstr = NL + 1;
    auto sld = [buf](int e, int l) -> V { return buf[e * lstr + l]; };
    auto sst = [buf](int e, int l, const V &x) { buf[e * lstr + l] = x; };
    if constexpr (first && last) stage_io<V, R, NL, L, Ns, HIN, HOUT, EPT>(ld, st, tw, sign);
    else if constexpr (first) stage_io<V, R, NL, L, Ns, HIN, false, EPT>(ld, sst, tw, sign);
    else if constexpr (last) stage_io<V, R, NL, L, Ns, false, HOUT, EPT>(sld, st, tw, sign);
    else stage_io<V, R, NL, L, Ns, false, false, EPT>(sld, sst, tw, sign);
    if constexpr (!last) fft_io_rec<V, NL, L, Ns * R, HIN, HOUT, EPT>(Radices<Rest...>{}, buf, tw, sign, ld, st);
}

// FFT engines.  FftRuntime CTAs are capped at 256 threads so the generic stage code keeps
// its registers; FftStatic CTAs at 512.  HIN/HOUT only change the static engine.
//
// run_io(buf, plan, tw, sign, ld, st): transform with input ld(e, line) (asked only for
// e < L/2 when HIN) and output st(e, line, v) (called only for e < L/2 when HOUT; storers
// must themselves ignore indices outside their window).  buf is the working buffer; ld may
// read another shared buffer.
struct FftRuntime {
    static constexpr int kLen = 0;
    static constexpr int kEPT = FFT_EPT;
    static constexpr int kMaxThreads = 256;
    static constexpr int kNst = 0;
    static constexpr int kRad[1] = {0};
    template <typename V, int NL, bool HIN, bool HOUT>
    __device__ __forceinline__ static void run(V *buf, const FFTPlan &p, const V *tw, int sign) {
        fft_smem<V, NL>(buf, NL + 1, p, tw, sign);
    }
    template <typename V, int NL, bool HIN, bool HOUT, class LD, class ST>
    __device__ __forceinline__ static void run_io(V *buf, const FFTPlan &p, const V *tw, int sign, const LD &ld,
                                                  const ST &st) {
        const int L = p.L, nthreads = blockDim.x, tid = threadIdx.x;
        constexpr int lstr = NL + 1;
        for (int idx = tid; idx < NL * L; idx += nthreads) {
            const int e = idx / NL, l = idx - e * NL;
            buf[e * lstr + l] = ld(e, l);
        }
        __syncthreads();
        fft_smem<V, NL>(buf, lstr, p, tw, sign);
        for (int idx = tid; idx < NL * L; idx += nthreads) {
            const int e = idx / NL, l = idx - e * NL;
            st(e, l, buf[e * lstr + l]);
        }
        __syncthreads();
    }
};
// Static engine with EPT_ complex values per thread and stage (L*NL/EPT_ threads per CTA).
template <int EPT_, int L_, int... Rs> struct FftStaticT {
    static constexpr int kLen = L_;
    static constexpr int kEPT = EPT_;
    static constexpr int kMaxThreads = 512;
    static constexpr int kNst = sizeof...(Rs);
    static constexpr int kRad[sizeof...(Rs)] = {Rs...};
    template <typename V, int NL, bool HIN, bool HOUT>
    __device__ __forceinline__ static void run(V *buf, const FFTPlan &, const V *tw, int sign) {
        fft_ct<V, NL, L_, 1, HIN, HOUT, EPT_, Rs...>(buf, tw, sign);
    }
    template <typename V, int NL, bool HIN, bool HOUT, class LD, class ST>
    __device__ __forceinline__ static void run_io(V *buf, const FFTPlan &, const V *tw, int sign, const LD &ld,
                                                  const ST &st) {
        fft_io_rec<V, NL, L_, 1, HIN, HOUT, EPT_>(Radices<Rs...>{}, buf, tw, sign, ld, st);
    }
};
// FP32 transforms: 16 values per thread.  FP64: 8 (half the registers of the same bytes),
// with radices of at most 8 so that every thread owns a butterfly in every stage.
template <int L_, int... Rs> using FftStatic = FftStaticT<FFT_EPT, L_, Rs...>;
template <int L_, int... Rs> using FftStatic8 = FftStaticT<8, L_, Rs...>;

// Lines per CTA for a static engine: the largest NL <= nl_max with a whole number of
// threads, at most 512 threads, and nbuf line buffers within budget bytes of shared memory.
constexpr int nl_static(int L, int nl_max, int elem_bytes, int nbuf, int budget = 100 * 1024, int ept = FFT_EPT) {
    int nl = nl_max;
    while (nl > 2 && ((L * nl) % ept != 0 || (L * nl) / ept > 512 ||
                      nbuf * L * (nl + 1) * elem_bytes + L * elem_bytes > budget))
        nl /= 2;
    return nl;
}

// Calls f(engine) with the static engine for L when there is one, else FftRuntime.  T is
// the real type of the transform: FP64 transforms use 8 values per thread and radices up to
// 8; FP32 transforms 8 values per thread up to L = 192 (the many short lines of batched
// small grids) and 16 from L = 256 (where the 8-value engines measured slower).
template <typename T, class F> inline int dispatch_fft_len(int L, F &&f) {
    if constexpr (sizeof(T) == 8) {
        switch (L) {
        case 32: return f(FftStatic8<32, 8, 4>{});
        case 64: return f(FftStatic8<64, 8, 8>{});
        case 96: return f(FftStatic8<96, 8, 4, 3>{});
        case 128: return f(FftStatic8<128, 8, 4, 4>{});
        case 192: return f(FftStatic8<192, 8, 8, 3>{});
        case 256: return f(FftStatic8<256, 8, 8, 4>{});
        case 384: return f(FftStatic8<384, 8, 8, 2, 3>{});
        case 512: return f(FftStatic8<512, 8, 8, 8>{});
        default: return f(FftRuntime{});
        }
    } else {
        switch (L) {
        case 32: return f(FftStatic8<32, 8, 4>{});
        case 64: return f(FftStatic8<64, 8, 8>{});
        case 96: return f(FftStatic8<96, 8, 4, 3>{});
        case 128: return f(FftStatic8<128, 8, 4, 4>{});
        case 192: return f(FftStatic8<192, 8, 8, 3>{});
        case 256: return f(FftStatic<256, 8, 8, 4>{});
        case 384: return f(FftStatic<384, 8, 8, 2, 3>{});
        case 512: return f(FftStatic<512, 8, 8, 8>{});
        default: return f(FftRuntime{});
        }
    }
}

// Radix sequences of the warp-per-column engine of the z pass (first radix == last radix,
// even); WarpNone for lengths without one.
template <int L_, int... Rs> struct WarpFft {
    static constexpr int kLen = L_;
    static constexpr int kNst = sizeof...(Rs);
    static constexpr int kRad[sizeof...(Rs)] = {Rs...};
};
struct WarpNone {
    static constexpr int kLen = 0;
    static constexpr int kNst = 0;
    static constexpr int kRad[1] = {0};
};
template <class F> inline int dispatch_warp_len(int L, F &&f) {
    switch (L) {
    case 96: return f(WarpFft<96, 4, 2, 3, 4>{});
    case 128: return f(WarpFft<128, 4, 8, 4>{});
    case 192: return f(WarpFft<192, 4, 4, 3, 4>{});
    case 256: return f(WarpFft<256, 8, 4, 8>{});
    case 384: return f(WarpFft<384, 4, 8, 3, 4>{});
    case 512: return f(WarpFft<512, 8, 8, 8>{});
    default: return f(WarpNone{});
    }
}

// Twiddle tables of one length: rt[m] = exp(2 pi i m/L) for the runtime engine; st is the
// per-stage table of the static engine ([stage][k][r-1], L-1 entries), or rt when the
// length has no static engine; wt the same for the warp engine of the z pass (or rt).
template <typename V> struct TwPair {
    const V *rt;
    const V *st;
    const V *wt;
};

// Stage the twiddle table of length n into shared memory.
template <typename V> __device__ __forceinline__ void load_twiddles(V *tw_s, const V *tw_g, int n) {
    const int nthreads = blockDim.x * blockDim.y;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    for (int m = tid; m < n; m += nthreads) tw_s[m] = tw_g[m];
}

}  // namespace osc
