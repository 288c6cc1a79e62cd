// zconv_warp.cuh -- the z pass of the free-space convolution with one warp per column.
//
// A CTA of W warps owns W adjacent (kx,ky) columns.  It loads the non-zero half of the
// columns (z in [0,nz), coalesced across the W columns) into one shared buffer per warp;
// every warp then transforms its own column with warp-synchronous Stockham stages.  The
// radix sequence starts and ends with the same radix, so the butterflies a lane owns in the
// forward transform's last stage are exactly the inputs it owns in an inverse transform's
// first stage: the forward spectrum stays in registers, the product with the cached Green
// spectrum is formed in registers and fed straight into the inverse's first butterflies.
// The inverse's last stage (window z < nz only) is stored by the warp itself when the
// output is kz-innermost (one contiguous column per warp), else it goes back to the warp
// buffer and the CTA stores its W columns with coalesced writes.
//
// Warp buffers are padded by one element per sixteen (p = e + e/16) for 8-byte complex
// values and one per eight (p = e + e/8) for 16-byte ones, and are 4 mod 16 (8-byte) or
// 2 mod 8 (16-byte) elements apart.  A shared-memory access of 8-byte values is served a
// half warp at a time, of 16-byte values a quarter warp at a time; under these paddings the
// stride-R writes of the first stage, the unit-stride reads of the others and the
// column-interleaved CTA loads of 4 warps fall on distinct banks.  For 16-byte values the
// writes of the middle stages are conflict-free too.  For 8-byte values a radix-8 middle
// stage with Ns = 8 writes two output groups 64 elements apart per half warp, which the
// one-in-sixteen padding puts on overlapping banks; the buffer between that stage and the
// next takes layout 1 (wpadl), under which those writes and the next stage's reads are both
// conflict-free.  The Green spectra of this kernel are stored with kz
// innermost (GSpecDev::zinner), so the 32 lanes of a warp read 32 consecutive kz.  When
// all spectra are real and even/odd in z (free space without images), each CTA fetches the
// Green columns of its W columns into shared memory with bulk copies at launch, which
// complete while the forward transforms run.
#pragma once

#include "async_copy.cuh"
#include "fft_kernels.cuh"

namespace osc {

// Warps per CTA and resident CTAs per SM the register allocation of k_zconv_warp is sized
// for: FP32 4 warps x 6 CTAs (<= 85 registers; 8 warps x 3 CTAs measured 171 us against 153
// for the 128x128x256 step, the CTA-wide waits for the loads and Green copies being shorter
// with fewer warps); FP64 holds twice the bytes per value, 4 warps x 2 CTAs.
template <typename T> constexpr int zw_warps() { return 4; }
template <typename T> constexpr int zw_minb() { return sizeof(T) == 4 ? 6 : 2; }


// padding shift of a complex type: 4 (one element in 16) for 8-byte, 3 (one in 8) for 16-byte
template <typename V> constexpr int wpad_shift() { return sizeof(V) >= 16 ? 3 : 4; }
template <typename V> __device__ __forceinline__ int wpad(int e) { return e + (e >> wpad_shift<V>()); }
// Layout 1, for 8-byte values between a radix-8 stage with Ns = 8 and the next stage: one
// pad element in 16 plus four in 64.  That stage writes, per half warp, two output groups 64
// elements apart (x = 64g + k + 8r, k < 8); the extra four per 64 puts them 8 banks pairs
// apart, while 16 consecutive elements (the next stage's reads) keep distinct banks.
template <typename V, int LAY> __device__ __forceinline__ int wpadl(int e) {
    return LAY ? e + (e >> 4) + 4 * (e >> 6) : wpad<V>(e);
}
constexpr int zw_lay_of(int vbytes, int Ns, int R) { return vbytes == 8 && Ns == 8 && R == 8 ? 1 : 0; }
// elements per warp buffer of real type T: the largest padded index of either layout plus
// one, rounded up to 4 mod 16 (FP32) or 2 mod 8 (FP64) so that the 4 warp buffers start on
// different banks
template <typename T> constexpr int wbuf_len(int L) {
    return sizeof(T) == 4
               ? (L + (L - 1) / 16 + 4 * ((L - 1) / 64) + 1) + ((4 - (L + (L - 1) / 16 + 4 * ((L - 1) / 64) + 1)) % 16 + 16) % 16
               : (L + L / 8) + ((2 - (L + L / 8)) % 8 + 8) % 8;
}

// One stage of one warp's transform: butterflies j = lane + 32q (j < L/R), input elements
// j + (L/R) r, outputs (j/Ns) Ns R + j%Ns + Ns r; per-stage twiddles at (Ns-1) + k(R-1) + r-1.
// Padded positions of a butterfly's R elements are a per-lane base plus compile-time
// offsets wherever the padding allows it.
// LDL / STL: layouts (0 = wpad, 1 = wpadl<V, 1>) of the buffer this stage reads and writes.
template <typename V, int R, int L, int Ns, int LDL = 0, int STL = 0> struct WStage {
    static constexpr int nb = L / R;
    static constexpr int Q = (nb + 31) / 32;
    static constexpr bool full = nb % 32 == 0;
    static constexpr int PS = wpad_shift<V>(), PB = 1 << PS;  // one pad element per PB
    // wpadl(j + r nb) = wpadl(j) + r ld_step: layout 0 when PB | nb; layout 1 when 64 | nb
    static constexpr bool ld_lin = LDL ? nb % 64 == 0 : nb % PB == 0;
    static constexpr int ld_step = LDL ? nb + nb / 16 + nb / 16 : nb + nb / PB;
    // store: 1 = Ns multiple of PB, 2 = Ns | PB and PB | Ns R, 3 = Ns R | PB, 0 = per element;
    // layout 1 takes form 2 when Ns | 16, 16 | Ns R and Ns R | 64 (one 64-block per butterfly)
    static constexpr int st_kind =
        STL ? ((16 % Ns == 0 && (Ns * R) % 16 == 0 && 64 % (Ns * R) == 0) ? 2 : 0)
            : Ns % PB == 0 ? 1 : (PB % Ns == 0 && (Ns * R) % PB == 0) ? 2 : (PB % (Ns * R) == 0) ? 3 : 0;
    __device__ __forceinline__ static constexpr int st_off(int r) {
        return STL ? r * Ns + ((r * Ns) >> 4)
                   : st_kind == 1 ? r * (Ns + Ns / PB) : st_kind == 2 ? r * Ns + ((r * Ns) >> PS) : r * Ns;
    }

    __device__ __forceinline__ static void load(const V *wb, const V *tw, int sign, int lane, V (&v)[Q][R],
                                                bool half_in) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q, k = j % Ns;
            const int pb = wpadl<V, LDL>(j);
            if (full || j < nb) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    V x;
                    if (half_in && r >= R / 2) {
                        x.x = 0;
                        x.y = 0;
                    } else {
                        x = wb[ld_lin ? pb + r * ld_step : wpadl<V, LDL>(j + r * nb)];
                        if (r && Ns > 1) x = cmul(x, tw_get(tw, (Ns - 1) + k * (R - 1) + (r - 1), sign));
                    }
                    v[q][r] = x;
                }
            }
        }
    }
    __device__ __forceinline__ static void dft(V (&v)[Q][R], int sign) {
#pragma unroll
        for (int q = 0; q < Q; ++q) Dft<R>::run(v[q], sign);
    }
    __device__ __forceinline__ static void store(V *wb, int lane, const V (&v)[Q][R]) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q, k = j % Ns;
            if (full || j < nb) {
                const int idxD = (j / Ns) * Ns * R + k;
                const int pb = wpadl<V, STL>(idxD);
#pragma unroll
                for (int r = 0; r < R; ++r) wb[st_kind ? pb + st_off(r) : wpadl<V, STL>(idxD + r * Ns)] = v[q][r];
            }
        }
    }
};

// Stages strictly between the first and the last, in place in the warp buffer; LIN is the
// layout of the buffer the stage reads (the first stage writes layout 0).
template <typename V, int L, int LIN, int Ns, int R, int... Rest>
__device__ __forceinline__ void wfft_mid(V *wb, const V *tw, int sign, int lane) {
    if constexpr (sizeof...(Rest) > 0) {
        constexpr int LOUT = zw_lay_of((int)sizeof(V), Ns, R);
        typedef WStage<V, R, L, Ns, LIN, LOUT> S;
        V v[S::Q][R];
        S::load(wb, tw, sign, lane, v, false);
        S::dft(v, sign);
        __syncwarp();
        S::store(wb, lane, v);
        __syncwarp();
        wfft_mid<V, L, LOUT, Ns * R, Rest...>(wb, tw, sign, lane);
    }
}
template <typename V, int L, int R0, int... Rest>
__device__ __forceinline__ void wfft_mid_of(Radices<R0, Rest...>, V *wb, const V *tw, int sign, int lane) {
    wfft_mid<V, L, 0, R0, Rest...>(wb, tw, sign, lane);
}
// layout of the buffer the last stage reads: written by the second-to-last stage
template <typename V, int... Rs> constexpr int zw_last_lay() {
    constexpr int n = sizeof...(Rs);
    constexpr int r[n] = {Rs...};
    int ns = 1;
    for (int i = 0; i + 2 < n; ++i) ns *= r[i];
    return n >= 3 ? zw_lay_of((int)sizeof(V), ns, r[n - 2]) : 0;
}

// Green term modes of the kernel.
constexpr int ZW_DIRECT = 0;  // spectra read from global memory
constexpr int ZW_IMAGE = 1;   // as 0, plus the mirrored-image term
constexpr int ZW_STAGED = 2;  // real, z-symmetric spectra staged in shared memory by bulk copies
constexpr int ZW_SUM = 3;     // as 2, for a.nsum inputs (members) and one output: the sum over
                              // members s of (spectrum gdir[s]) x (transform of input s)

template <typename T, int W, int MODE, int L, int... Rs>
__global__ void __launch_bounds__(W * 32, zw_minb<T>()) k_zconv_warp(const cplx<T> *__restrict__ in, cplx<T> *__restrict__ out,
                                                       ZConvArgs a, const cplx<T> *__restrict__ twg,
                                                       const cplx<T> *__restrict__ tw_rt) {
    typedef cplx<T> V;
    constexpr bool IMG = MODE == ZW_IMAGE, SUM = MODE == ZW_SUM, GS = MODE == ZW_STAGED || SUM;
    constexpr int RF = WarpFft<L, Rs...>::kRad[0];
    static_assert(RF == WarpFft<L, Rs...>::kRad[sizeof...(Rs) - 1], "first and last radix must match");
    static_assert(RF % 2 == 0, "first radix must be even");
    typedef WStage<V, RF, L, 1> S0;       // first stage
    typedef WStage<V, RF, L, L / RF, zw_last_lay<V, Rs...>()> SL;  // last stage
    constexpr int NB = L / RF, Q = S0::Q, WB = wbuf_len<T>(L);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t gbar;
    __shared__ int gfail;
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *wbufs = tw + L;
    V *rbufs = wbufs + W * WB;                          // IMG: forward spectra, read at mirrored kz
    T *gst = reinterpret_cast<T *>(wbufs + W * WB);     // GS: Green columns [W][nst][zpitch]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = blockIdx.x * W;
    const int zp = a.g[0].zpitch;
    const int nst = SUM ? a.nsum : a.nout;  // staged Green columns per (kx,ky) column
    in += blockIdx.y * a.in_bstride;
    out += blockIdx.y * a.out_bstride;
    const int64_t goff = blockIdx.y * a.g_bstride;
    V *wb = wbufs + warp * WB;
    if (GS) {
        if (threadIdx.x == 0) {
            mbar_init(&gbar, 1);
            const int ncv = min(W, a.ncols - col0);
            mbar_arrive_expect_tx(&gbar, (unsigned)(ncv * nst * zp * (int)sizeof(T)));
            for (int c = 0; c < ncv; ++c) {
                const int col = a.col_base + col0 + c, ky = col / a.nxh, kx = col - ky * a.nxh;
                for (int o = 0; o < nst; ++o) {
                    const GSpecDev &g = a.g[a.gdir[o]];
                    const int yy = (g.sym_y && ky > a.ny) ? a.Ny - ky : ky;
                    const T *src = reinterpret_cast<const T *>(g.data) + goff + ((int64_t)yy * a.nxh + kx) * zp;
                    if (!a.skip_copies) bulk_g2s(gst + (c * nst + o) * zp, src, (unsigned)(zp * sizeof(T)), &gbar);
                }
            }
        }
    }
    load_twiddles(tw, twg, L);
    // the non-zero half (z < nz) of this CTA's W columns of input `src`, into the warp buffers
    auto load_columns = [&](const cplx<T> *__restrict__ src) {
        for (int idx = threadIdx.x; idx < W * a.nz; idx += W * 32) {
            const int e = idx / W, c = idx - e * W;
            const int col = col0 + c;
            V v = mk<T>(0, 0);
            if (col < a.ncols) v = src[(int64_t)e * a.in_estride + col];
            wbufs[c * WB + wpad<V>(e)] = v;
        }
    };
    // forward transform (sign +1) of this warp's column; the upper half of its input is zero.
    // rh[q][r] is the spectrum at kz = lane + 32q + NB r
    auto forward = [&](V (&rh)[Q][RF]) {
        V v[Q][RF];
        S0::load(wb, tw, +1, lane, v, true);
        S0::dft(v, +1);
        __syncwarp();
        S0::store(wb, lane, v);
        __syncwarp();
        wfft_mid_of<V, L>(Radices<Rs...>{}, wb, tw, +1, lane);
        SL::load(wb, tw, +1, lane, rh, false);
        SL::dft(rh, +1);
    };
    // CTA-wide wait for the staged Green columns; false when the copies did not complete
    auto wait_green = [&]() -> bool {
        if (threadIdx.x == 0) {
            const bool ok = mbar_wait_bounded(&gbar, 0, a.poll_limit);
            if (!ok) {
                report_fault(a.fault, FAULT_BULK_WAIT);
                // let copies in flight land before leaving.  If this wait runs out too, the
                // CTA leaves with copies that may still be in flight into its shared memory;
                // the CTA reads none of it, and the host reports the call as timed out
                mbar_wait_bounded(&gbar, 0, a.poll_limit);
            }
            gfail = ok ? 0 : 1;
        }
        __syncthreads();
        return !gfail;  // CTA-uniform
    };
    const int colc = a.col_base + min(col0 + warp, a.ncols - 1);
    const int ky = colc / a.nxh, kx = colc - ky * a.nxh;
    // v = rh times the staged Green column `slot` of spectrum g (real, even/odd in z)
    auto staged_product = [&](const V (&rh)[Q][RF], int gd, int slot, V (&v)[Q][RF]) {
        const GSpecDev &g = a.g[gd];
        const T *gc = gst + (warp * nst + slot) * zp;
        const bool yneg = g.sym_y && ky > a.ny && g.par_y < 0;
        const bool zodd = g.par_z < 0, iu = g.imag_unit;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            if (S0::full || j < NB) {
#pragma unroll
                for (int r = 0; r < RF; ++r) {
                    const int e = j + NB * r;
                    T sv;
                    if (r < RF / 2) {
                        sv = gc[e];
                    } else {  // kz >= nz: the value at Nz - kz, odd spectra change sign
                        sv = gc[L - e];
                        if (zodd && e != a.nz) sv = -sv;
                    }
                    if (yneg) sv = -sv;
                    const V x = rh[q][r];
                    v[q][r] = iu ? mk<T>(-x.y * sv, x.x * sv) : mk<T>(x.x * sv, x.y * sv);
                }
            }
        }
    };
    // inverse transform of v (first stage from registers) and the store of output o's
    // window z < nz; false when the store went through the CTA (all warps must follow)
    auto inverse_store = [&](V (&v)[Q][RF], int o) {
        S0::dft(v, -1);
        S0::store(wb, lane, v);
        __syncwarp();
        wfft_mid_of<V, L>(Radices<Rs...>{}, wb, tw, -1, lane);
        SL::load(wb, tw, -1, lane, v, false);
        SL::dft(v, -1);
        __syncwarp();
        if (a.out_estride == 1) {  // kz-innermost output: this warp's column is contiguous
            if (col0 + warp < a.ncols) {
                V *dst = out + (int64_t)o * a.out_cstride + (int64_t)(col0 + warp) * a.out_colstride;
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int j = lane + 32 * q;
                    if (S0::full || j < NB)
#pragma unroll
                        for (int r = 0; r < RF / 2; ++r) dst[j + NB * r] = v[q][r];  // z = j + NB r < L/2
                }
            }
            return;  // wb is this warp's alone: the next output's first stage writes it
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            if (S0::full || j < NB)
#pragma unroll
                for (int r = 0; r < RF / 2; ++r) wb[wpad<V>(j + NB * r)] = v[q][r];  // z = j + NB r < L/2
        }
        __syncthreads();
        V *dst = out + (int64_t)o * a.out_cstride;
        for (int idx = threadIdx.x; idx < W * a.nz; idx += W * 32) {
            const int e = idx / W, c = idx - e * W;
            const int col = col0 + c;
            if (col < a.ncols) dst[(int64_t)e * a.out_estride + (int64_t)col * a.out_colstride] = wbufs[c * WB + wpad<V>(e)];
        }
        __syncthreads();
    };

    if constexpr (SUM) {
        // one output: sum over the inputs of (Green spectrum s) x (transform of input s)
        V acc[Q][RF];
        for (int sidx = 0; sidx < a.nsum; ++sidx) {
            if (sidx) __syncthreads();  // every warp is done with the previous input's columns
            load_columns(in + sidx * a.in_bstride);
            __syncthreads();
            V rh[Q][RF];
            forward(rh);
            if (sidx == 0 && !wait_green()) return;
            __syncwarp();
            V v[Q][RF];
            staged_product(rh, a.gdir[sidx], sidx, v);
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < RF; ++r) acc[q][r] = sidx ? cadd(acc[q][r], v[q][r]) : v[q][r];
        }
        inverse_store(acc, 0);
        return;
    }

    load_columns(in);
    __syncthreads();
    V rh[Q][RF];
    forward(rh);
    V *rb = rbufs + warp * WB;
    if (IMG) {
        // the image spectrum -w^((nz-1) kz) rho_hat(-kz) of this lane's kz, formed once for all
        // outputs: rho_hat(-kz) is held by another lane, so the spectrum goes through rb, and
        // rb then keeps each lane's image values at its own positions
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            if (S0::full || j < NB)
#pragma unroll
                for (int r = 0; r < RF; ++r) rb[wpad<V>(j + NB * r)] = rh[q][r];
        }
        __syncwarp();
        V im[Q][RF];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            if (S0::full || j < NB) {
#pragma unroll
                for (int r = 0; r < RF; ++r) {
                    const int e = j + NB * r;
                    const V rm = rb[wpad<V>(e == 0 ? 0 : L - e)];
                    // (nz-1)*kz < 2^21: 32-bit index arithmetic
                    const V ph = __ldg(tw_rt + (int)(((unsigned)a.img_phase_mul * (unsigned)e) % (unsigned)L));
                    const V ri = cmul(ph, rm);
                    im[q][r] = mk<T>(-ri.x, -ri.y);
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
            if (S0::full || j < NB)
#pragma unroll
                for (int r = 0; r < RF; ++r) rb[wpad<V>(j + NB * r)] = im[q][r];
        }
    }
    if (GS && !wait_green()) return;
    __syncwarp();
    for (int o = 0; o < a.nout; ++o) {
        const int gd = a.gdir[o], gi = a.gimg[o];
        V v[Q][RF];
        if (GS) {
            staged_product(rh, gd, o, v);
        } else {
            const T icoef = (T)a.img_coef[o];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int j = lane + 32 * q;
                if (S0::full || j < NB) {
#pragma unroll
                    for (int r = 0; r < RF; ++r) {
                        const int e = j + NB * r;
                        V S = mk<T>(0, 0);
                        if (gd >= 0)
                            S = cmul(rh[q][r], g_lookup<T>(a.g[gd], kx, ky, e, a.nxh, a.Ny, a.ny, L, a.nz, goff));
                        if (IMG && gi >= 0) {
                            // spectrum of -rho flipped in z, formed above: -w^((nz-1) kz) * rho_hat(-kz)
                            const V ri = cscale(rb[wpad<V>(e)], icoef);
                            S = cadd(S, cmul(ri, g_lookup<T>(a.g[gi], kx, ky, e, a.nxh, a.Ny, a.ny, L, a.nz, goff)));
                        }
                        v[q][r] = S;
                    }
                }
            }
        }
        inverse_store(v, o);
    }
}

// Shared memory bytes of k_zconv_warp for length L, W warps; zp = Green column pitch
// (elements) of the staged mode.
template <typename T> inline size_t zconv_warp_smem(int L, int W, int mode, int nout, int zp) {
    size_t b = sizeof(cplx<T>) * ((size_t)L + (size_t)W * wbuf_len<T>(L));
    if (mode == ZW_IMAGE) b += sizeof(cplx<T>) * (size_t)W * wbuf_len<T>(L);
    if (mode == ZW_STAGED || mode == ZW_SUM) b += sizeof(T) * (size_t)W * nout * zp;
    return b;
}

}  // namespace osc
