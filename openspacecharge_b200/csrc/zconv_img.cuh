// zconv_img.cuh -- the z pass of the cathode-image convolution, one warp per column, with
// both Green columns staged in shared memory.
//
// With images the spectral product of output o at (kx, ky, kz) is
//   S(kz) = rho_hat(kz) G_o(kz) + c_o rho_hat(Nz - kz) G'_o(kz),
// G_o the direct spectrum (real, even/odd in z, as in the staged free-space pass) and G'_o
// the image spectrum with the flip phase -exp(2 pi i (nz-1) kz / Nz) already applied when it
// was built (GSpecDev::herm_img).  The image kernel is even/odd in x and y, so after the x
// and y transforms each of its columns is real up to a constant factor and its z spectrum
// obeys G'(Nz - kz) = par_h conj(G'(kz)) -- the factor keeps that relation, par_h = +-1 the
// product of the x and y parities; only kz in [0, nz] is stored.
//
// A CTA of 4 warps owns the columns (kx0, yy), (kx0+1, yy), (kx0, Ny-yy), (kx0+1, Ny-yy):
// the two rows that read the same stored Green row yy (rows 0 and ny have no partner, and
// their second pair of warps idles), so each CTA fetches 2 x nout direct and 2 x nout image
// Green columns with bulk copies at launch, once for both rows.  rho_hat(Nz - kz) lives in
// another lane of the same warp (the mirror of butterfly j is Nb - j, Nb = L / R), so it is
// a shuffle from lane -l mod 32; lane 0 holds its own mirrors.
#pragma once

#include "zconv_warp.cuh"

namespace osc {

constexpr int ZI_WARPS = 4;
// resident CTAs per SM the register allocation is sized for: with images FP32 holds 41 KB of
// shared memory per CTA at L = 512 (5 CTAs), FP64 80 KB (2 CTAs); without, FP32 29 KB (6
// CTAs, the occupancy of the unpaired warp engine)
template <typename T, bool IMG> constexpr int zi_minb() { return sizeof(T) == 4 ? (IMG ? 5 : 6) : 2; }

template <typename T> __device__ __forceinline__ cplx<T> shfl_c(cplx<T> v, int src) {
    v.x = __shfl_sync(0xffffffffu, v.x, src);
    v.y = __shfl_sync(0xffffffffu, v.y, src);
    return v;
}

// IMG false: the free-space product alone (no image spectra staged or read), the same
// column pairing halving the Green columns each CTA fetches.
template <typename T, bool IMG, int L, int... Rs>
__global__ void __launch_bounds__(ZI_WARPS * 32, zi_minb<T, IMG>())
    k_zconv_img(const cplx<T> *__restrict__ in, cplx<T> *__restrict__ out, ZConvArgs a,
                const cplx<T> *__restrict__ twg) {
    typedef cplx<T> V;
    constexpr int W = ZI_WARPS;
    constexpr int RF = WarpFft<L, Rs...>::kRad[0];
    static_assert(RF == WarpFft<L, Rs...>::kRad[sizeof...(Rs) - 1], "first and last radix must match");
    static_assert(RF % 2 == 0, "first radix must be even");
    typedef WStage<V, RF, L, 1> S0;
    typedef WStage<V, RF, L, L / RF, zw_last_lay<V, Rs...>()> SL;
    constexpr int NB = L / RF, Q = S0::Q, WB = wbuf_len<T>(L);
    static_assert(NB % 32 == 0 || NB < 32, "the mirror of a butterfly must sit in register Q-1-q");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t gbar;
    __shared__ int gfail;
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *wbufs = tw + L;
    const int nout = a.nout;
    const int zp = a.g[a.gdir[0]].zpitch, zpi = IMG ? a.g[a.gimg[0]].zpitch : 0;
    T *gdst = reinterpret_cast<T *>(wbufs + W * WB);          // direct columns [2][nout][zp]
    V *gist = reinterpret_cast<V *>(gdst + 2 * nout * zp);    // image columns [2][nout][zpi] (IMG)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nkp = (a.nxh + 1) >> 1;
    const int yy = blockIdx.x / nkp, kx0 = 2 * (blockIdx.x - yy * nkp);
    // column of slot c (kx0 + (c & 1), row yy or Ny - yy), or -1
    auto col_of = [&](int c) -> int {
        const int kx = kx0 + (c & 1);
        if (kx >= a.nxh) return -1;
        if (c >> 1) return (yy == 0 || yy == a.ny) ? -1 : (a.Ny - yy) * a.nxh + kx;
        return yy * a.nxh + kx;
    };
    in += blockIdx.y * a.in_bstride;
    out += blockIdx.y * a.out_bstride;
    V *wb = wbufs + warp * WB;
    if (threadIdx.x == 0) {
        mbar_init(&gbar, 1);
        const int nk = min(2, a.nxh - kx0);
        mbar_arrive_expect_tx(&gbar, (unsigned)(nk * nout * (zp * (int)sizeof(T) + (IMG ? zpi * (int)sizeof(V) : 0))));
        for (int kk = 0; kk < nk; ++kk) {
            const int64_t row = (int64_t)yy * a.nxh + kx0 + kk;
            for (int o = 0; o < nout; ++o) {
                const T *sd = reinterpret_cast<const T *>(a.g[a.gdir[o]].data) + blockIdx.y * a.g_bstride + row * zp;
                if (!a.skip_copies) {
                    bulk_g2s(gdst + (kk * nout + o) * zp, sd, (unsigned)(zp * sizeof(T)), &gbar);
                    if (IMG) {
                        const V *si = reinterpret_cast<const V *>(a.g[a.gimg[o]].data) + row * zpi;
                        bulk_g2s(gist + (kk * nout + o) * zpi, si, (unsigned)(zpi * sizeof(V)), &gbar);
                    }
                }
            }
        }
    }
    load_twiddles(tw, twg, L);
    for (int idx = threadIdx.x; idx < W * a.nz; idx += W * 32) {
        const int e = idx / W, c = idx - e * W;
        const int col = col_of(c);
        V v = mk<T>(0, 0);
        if (col >= 0) v = in[(int64_t)e * a.in_estride + col];
        wbufs[c * WB + wpad<V>(e)] = v;
    }
    __syncthreads();
    // forward transform (sign +1); rh[q][r] is the spectrum at kz = lane + 32q + NB r
    V rh[Q][RF];
    {
        V v[Q][RF];
        S0::load(wb, tw, +1, lane, v, true);
        S0::dft(v, +1);
        __syncwarp();
        S0::store(wb, lane, v);
        __syncwarp();
        wfft_mid_of<V, L>(Radices<Rs...>{}, wb, tw, +1, lane);
        SL::load(wb, tw, +1, lane, rh, false);
        SL::dft(rh, +1);
    }
    if (threadIdx.x == 0) {
        const bool ok = mbar_wait_bounded(&gbar, 0, a.poll_limit);
        if (!ok) {
            report_fault(a.fault, FAULT_BULK_WAIT);
            // let copies in flight land before leaving (bounded as well)
            mbar_wait_bounded(&gbar, 0, a.poll_limit);
        }
        gfail = ok ? 0 : 1;
    }
    __syncthreads();
    if (gfail) return;
    const int mycol = col_of(warp);
    const int kk = warp & 1;
    const bool mrow = (warp >> 1) != 0;  // ky = Ny - yy > ny
    // lane holding the mirror butterfly NB - j (lanes >= NB of a short transform hold none)
    const int partner = S0::full ? ((32 - lane) & 31) : ((NB - lane) & 31);
    for (int o = 0; o < nout; ++o) {
        const GSpecDev &gd = a.g[a.gdir[o]];
        const bool dneg = mrow && gd.par_y < 0, zodd = gd.par_z < 0, iu = gd.imag_unit;
        T icoef = 0, ph = 0;
        if (IMG) {
            const GSpecDev &gi = a.g[a.gimg[o]];
            icoef = (T)a.img_coef[o];
            if (mrow && gi.par_y < 0) icoef = -icoef;
            ph = (T)gi.par_h;
        }
        const T *gc = gdst + (kk * nout + o) * zp;
        const V *gic = gist + (kk * nout + o) * zpi;
        V v[Q][RF];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = lane + 32 * q;
#pragma unroll
            for (int r = 0; r < RF; ++r) {
                // rho_hat(L - e): butterfly NB - j, register RF - 1 - r (j > 0); lane 0 keeps
                // j = 0 (register (RF - r) mod RF) and j = 32q (register Q - q) itself
                V m = mk<T>(0, 0);
                if (IMG) {
                    m = shfl_c<T>(rh[Q - 1 - q][RF - 1 - r], partner);
                    if (lane == 0) m = q == 0 ? rh[0][(RF - r) % RF] : rh[(Q - q) % Q][RF - 1 - r];
                }
                if (S0::full || j < NB) {
                    const int e = j + NB * r;
                    T sv;
                    V gv = mk<T>(0, 0);
                    if (r < RF / 2) {
                        sv = gc[e];
                        if (IMG) gv = gic[e];
                    } else {  // kz >= nz: the stored values at L - kz
                        sv = gc[L - e];
                        if (zodd && e != a.nz) sv = -sv;
                        if (IMG) {
                            const V h = gic[L - e];
                            gv = mk<T>(ph * h.x, -ph * h.y);
                        }
                    }
                    if (dneg) sv = -sv;
                    const V x = rh[q][r];
                    V s = iu ? mk<T>(-x.y * sv, x.x * sv) : mk<T>(x.x * sv, x.y * sv);
                    if (IMG) {
                        const V t = cmul(m, gv);
                        s.x += icoef * t.x;
                        s.y += icoef * t.y;
                    }
                    v[q][r] = s;
                }
            }
        }
        // inverse transform, first stage from registers; the warp stores z < nz of its column
        S0::dft(v, -1);
        S0::store(wb, lane, v);
        __syncwarp();
        wfft_mid_of<V, L>(Radices<Rs...>{}, wb, tw, -1, lane);
        SL::load(wb, tw, -1, lane, v, false);
        SL::dft(v, -1);
        __syncwarp();
        if (mycol >= 0) {
            V *dst = out + (int64_t)o * a.out_cstride + (int64_t)mycol * a.out_colstride;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int j = lane + 32 * q;
                if (S0::full || j < NB)
#pragma unroll
                    for (int r = 0; r < RF / 2; ++r) dst[j + NB * r] = v[q][r];
            }
        }
    }
}

// Shared memory bytes of k_zconv_img: zp, zpi = pitches (elements) of the direct (real) and
// image (complex) Green columns, zpi = 0 without images.
template <typename T> inline size_t zconv_img_smem(int L, int nout, int zp, int zpi) {
    return sizeof(cplx<T>) * ((size_t)L + (size_t)ZI_WARPS * wbuf_len<T>(L)) +
           2 * (size_t)nout * (sizeof(T) * (size_t)zp + sizeof(cplx<T>) * (size_t)zpi);
}

}  // namespace osc
