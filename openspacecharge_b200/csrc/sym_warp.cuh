// sym_warp.cuh -- the even/odd line transforms of the Green build (SymArgs) on the warp
// engine: one warp per pair of real lines, one complex transform of length L = 2n.
//
// A line x[0..n) (x[n] = 0) is extended to the period L as x[L - e] = par x[e]; two lines
// a, b are packed as z = a + i b and Z = FFT(z) gives, at k in [0, n],
//   sum_e a[e] w^(ek) = (Z(k) + conj Z(L-k)) / 2,  sum_e b[e] w^(ek) = (Z(k) - conj Z(L-k)) / 2i,
// which is real for an even line and i times real for an odd one (the stored s[k]).  The CTA
// engine (k_sym_lines) runs NL interleaved lines through shared memory at every radix stage;
// here the CTA loads 2W lines into its W warp buffers (coalesced across the lines, or along
// them for contiguous rows), each warp transforms its pair with the register-resident
// Stockham stages of the z pass (two exchanges through its buffer at L = 512), and Z(L-k) is
// a shuffle from the lane holding the mirror butterfly (as in the image z pass).  Outputs
// contiguous along k are stored by the warps; strided ones go back through the buffers and
// are stored by the CTA with consecutive lines in consecutive threads.
#pragma once

#include "zconv_img.cuh"

namespace osc {

constexpr int SW_WARPS = 8;  // 16 lines per CTA: 64-byte rows of FP32 lines, the twiddle table per 8 pairs
template <typename T> constexpr int sw_minb() { return sizeof(T) == 4 ? 4 : 1; }

template <typename TC, typename TI, typename TO, bool ROW, bool KF, int L, int... Rs>
__global__ void __launch_bounds__(SW_WARPS * 32, sw_minb<TC>())
    k_sym_warp(const TI *__restrict__ in, TO *__restrict__ out, SymArgs a, const cplx<TC> *__restrict__ twg) {
    typedef cplx<TC> V;
    constexpr int W = SW_WARPS, n = L / 2;
    constexpr int RF = WarpFft<L, Rs...>::kRad[0];
    static_assert(RF == WarpFft<L, Rs...>::kRad[sizeof...(Rs) - 1], "first and last radix must match");
    static_assert(RF % 2 == 0, "first radix must be even");
    typedef WStage<V, RF, L, 1> S0;
    typedef WStage<V, RF, L, L / RF, zw_last_lay<V, Rs...>()> SL;
    constexpr int NB = L / RF, Q = S0::Q, WB = wbuf_len<TC>(L);
    static_assert(NB % 32 == 0 || NB < 32, "the mirror of a butterfly must sit in register Q-1-q");
    static_assert(2 * WB >= 2 * (n + 1), "a warp buffer holds the two output lines");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int64_t bin[2 * W], bout[2 * W];
    __shared__ int podd[2 * W];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *wbufs = tw + L;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t r0 = (int64_t)blockIdx.x * (2 * W);
    if (tid < 2 * W) {  // line start offsets
        const int64_t r = r0 + tid;
        int64_t oi = -1, oo = -1;
        int odd = 0;
        if (r < a.nlines) {
            const int64_t bi = r / a.npq, rl = r - bi * a.npq;
            const int64_t pi = rl / a.nq, qi = rl - pi * a.nq;
            oi = bi * a.in_bs + pi * a.in_ps + qi * a.in_qs;
            oo = bi * a.out_bs + pi * a.out_ps + qi * a.out_qs;
            odd = bi >= a.odd_lo && bi < a.odd_hi;
        }
        bin[tid] = oi;
        bout[tid] = oo;
        podd[tid] = odd;
    }
    load_twiddles(tw, twg, L);
    __syncthreads();
    // the 2W lines, x[e] and its parity image at L - e, component (line & 1) of warp
    // buffer line >> 1; x[n] = 0
    for (int idx = tid; idx < 2 * W * n; idx += W * 32) {
        int rr, e;
        if (ROW) { rr = idx / n; e = idx - rr * n; }
        else { e = idx / (2 * W); rr = idx - e * (2 * W); }
        const int64_t o = bin[rr];
        TC v = (TC)0;
        if (o >= 0) v = (TC)in[o + (int64_t)e * a.in_es];
        TC *wl = reinterpret_cast<TC *>(wbufs + (rr >> 1) * WB);
        wl[2 * wpad<V>(e) + (rr & 1)] = v;
        if (e > 0) wl[2 * wpad<V>(L - e) + (rr & 1)] = podd[rr] ? -v : v;
    }
    if (tid < 2 * W) reinterpret_cast<TC *>(wbufs + (tid >> 1) * WB)[2 * wpad<V>(n) + (tid & 1)] = (TC)0;
    __syncthreads();
    V *wb = wbufs + warp * WB;
    V rh[Q][RF];  // Z at k = lane + 32q + NB r
    {
        V v[Q][RF];
        S0::load(wb, tw, +1, lane, v, false);
        S0::dft(v, +1);
        __syncwarp();
        S0::store(wb, lane, v);
        __syncwarp();
        wfft_mid_of<V, L>(Radices<Rs...>{}, wb, tw, +1, lane);
        SL::load(wb, tw, +1, lane, rh, false);
        SL::dft(rh, +1);
    }
    __syncwarp();  // every lane has read its buffer: KF = false reuses it for the outputs
    const int partner = S0::full ? ((32 - lane) & 31) : ((NB - lane) & 31);
    const int64_t o0 = bout[2 * warp], o1 = bout[2 * warp + 1];
    const bool odd0 = podd[2 * warp] != 0, odd1 = podd[2 * warp + 1] != 0;
    const TC hf = (TC)0.5, sc = (TC)a.scale;
    TC *wl = reinterpret_cast<TC *>(wb);  // KF = false: the two lines [2][n + 1]
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = lane + 32 * q;
#pragma unroll
        for (int r = 0; r < RF; ++r) {
            // Z(L - k): butterfly NB - j, register RF - 1 - r (j > 0); lane 0 holds j = 0
            // (register (RF - r) mod RF) and j = 32q (register Q - q) itself
            V m = shfl_c<TC>(rh[Q - 1 - q][RF - 1 - r], partner);
            if (lane == 0) m = q == 0 ? rh[0][(RF - r) % RF] : rh[(Q - q) % Q][RF - 1 - r];
            const bool has = (S0::full || j < NB) && (r < RF / 2 || (r == RF / 2 && j == 0));
            if (has) {
                const int k = j + NB * r;  // k <= n
                const V Z = rh[q][r];
                const TC s0 = (!odd0 ? hf * (Z.x + m.x) : hf * (Z.y - m.y)) * sc;
                const TC s1 = (!odd1 ? hf * (Z.y + m.y) : hf * (m.x - Z.x)) * sc;
                if (KF) {
                    if (o0 >= 0) out[o0 + (int64_t)k * a.out_es] = (TO)s0;
                    if (o1 >= 0) out[o1 + (int64_t)k * a.out_es] = (TO)s1;
                } else {
                    wl[k] = s0;
                    wl[(n + 1) + k] = s1;
                }
            }
        }
    }
    if (!KF) {
        __syncthreads();
        for (int idx = tid; idx < 2 * W * (n + 1); idx += W * 32) {
            const int k = idx / (2 * W), rr = idx - k * (2 * W);
            const int64_t o = bout[rr];
            if (o >= 0)
                out[o + (int64_t)k * a.out_es] =
                    (TO) reinterpret_cast<const TC *>(wbufs + (rr >> 1) * WB)[(rr & 1) * (n + 1) + k];
        }
    }
}

template <typename TC> inline size_t sym_warp_smem(int L) {
    return sizeof(cplx<TC>) * ((size_t)L + (size_t)SW_WARPS * wbuf_len<TC>(L));
}

}  // namespace osc
