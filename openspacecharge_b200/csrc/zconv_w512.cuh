// zconv_w512.cuh -- the z pass at length 512 (FP32, staged real Green spectra) with one
// shared-memory exchange per transform: an alternative engine the autotuner may pick
// (tuning key zconv_engine:f32:L512 = 1).
//
// The radix-8 warp engine (zconv_warp.cuh) moves every value of a 512-point column through
// shared memory twice per transform.  Here a transform is 512 = 16 x 32:
//   forward (sign +1), lane l holding x[l + 32 m] (m = 0..15, the upper half zero):
//     a 16-point DFT over m in registers, the twiddles w512^(l k1), one exchange through a
//     16 x 33 warp buffer, so that lane t holds the values of k1 = t mod 16 for the lanes
//     l = 2a + t/16, a 16-point DFT over a in registers, and a radix-2 combination of the
//     partner lanes t and t^16 (a shuffle) with the twiddles w32^k;
//   lane t then holds the spectrum at kz = k1 + 16 k + 256 c (k = 0..15, c = t/16), which is
//   multiplied by the staged Green column in registers;
//   inverse (sign -1), the mirror image: the radix-2 combination of the partner lanes, a
//   16-point DFT, the twiddles w512^(-(2a+c) k1), one exchange, a 16-point DFT, after which
//   lane l holds z = l + 32 n1 and stores n1 < 8 (the window z < 256) of its column.
// Per column that is one exchange per transform instead of two.  The w32 factors are
// constants; the lane twiddles of both transforms come from one table per CTA,
// tf[k1][l] = w512^(l k1) with rows 33 entries apart: the forward reads a row (32
// consecutive entries), the inverse reads w512^((2a + c) k1) = tf[k1][2a + c] across the rows,
// which the odd pitch spreads over distinct banks -- read from the plain 512-entry table, the
// strides l*k1 would fall on few banks.
#pragma once

#include "zconv_warp.cuh"

namespace osc {

// cos(pi k/16), sin(pi k/16), k = 0..15: w32^k = C[k] + s i S[k]
__device__ __forceinline__ float w32c(int k) {
    constexpr float C[16] = {1.0f, 0.9807852804032304f, 0.9238795325112867f, 0.8314696123025452f,
                             0.7071067811865476f, 0.5555702330196023f, 0.38268343236508984f, 0.19509032201612833f,
                             0.0f, -0.1950903220161282f, -0.3826834323650897f, -0.555570233019602f,
                             -0.7071067811865475f, -0.8314696123025453f, -0.9238795325112867f, -0.9807852804032304f};
    return C[k];
}
__device__ __forceinline__ float w32s(int k) {
    constexpr float S[16] = {0.0f, 0.19509032201612825f, 0.3826834323650898f, 0.5555702330196022f,
                             0.7071067811865475f, 0.8314696123025452f, 0.9238795325112867f, 0.9807852804032304f,
                             1.0f, 0.9807852804032304f, 0.9238795325112867f, 0.8314696123025455f,
                             0.7071067811865476f, 0.5555702330196022f, 0.3826834323650899f, 0.1950903220161286f};
    return S[k];
}

constexpr int W5_PITCH = 33;             // row pitch (complex) of the 16-row exchange layout
constexpr int W5_BUF = 16 * W5_PITCH + 4;  // per-warp buffer, 4 mod 16 apart between warps

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
    v.x = __shfl_xor_sync(0xffffffffu, v.x, m);
    v.y = __shfl_xor_sync(0xffffffffu, v.y, m);
    return v;
}

// Forward transform of this warp's column (buffer wb holds x[z], z < 256, linearly);
// returns in s[k] the spectrum at kz = (lane & 15) + 16 k + 256 (lane >> 4).  tf: the
// forward lane twiddles, [k1][lane].
__device__ __forceinline__ void w512_forward(float2 *wb, const float2 *__restrict__ tf, int lane, float2 (&s)[16]) {
    constexpr int P = W5_PITCH;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = wb[lane + 32 * m];
#pragma unroll
    for (int m = 8; m < 16; ++m) v[m] = make_float2(0.f, 0.f);
    Dft<16>::run(v, +1);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) v[k1] = cmul(v[k1], tf[k1 * P + lane]);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) wb[k1 * W5_PITCH + lane] = v[k1];
    __syncwarp();
    const int k1 = lane & 15, c = lane >> 4;
#pragma unroll
    for (int a = 0; a < 16; ++a) v[a] = wb[k1 * W5_PITCH + 2 * a + c];
    Dft<16>::run(v, +1);
    // X[k1 + 16 k] = Y0[k] + w32^k Y1[k], X[k1 + 16 k + 256] = Y0[k] - w32^k Y1[k]
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const float2 p = shfl_xor2(v[k], 16);
        const float2 y0 = c ? p : v[k], y1 = c ? v[k] : p;
        const float2 t = cmul(y1, make_float2(w32c(k), w32s(k)));
        s[k] = c ? csub(y0, t) : cadd(y0, t);
    }
}

// Inverse transform of a spectrum in the layout w512_forward returns; stores the window
// z < 256 of the result at dst[z] (when store is set).  tf: the twiddle table of
// w512_forward, read conjugated.
__device__ __forceinline__ void w512_inverse(float2 *wb, const float2 *__restrict__ tf, int lane, float2 (&s)[16],
                                             float2 *__restrict__ dst, bool store) {
    const int k1 = lane & 15, c = lane >> 4;
    float2 v[16];
    // U[k] = X[k] + X[k+16] (c = 0), (X[k] - X[k+16]) w32^-k (c = 1)
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        // branch-free: the two half warps take different sides of the butterfly
        const float2 p = shfl_xor2(s[k], 16);
        const float2 d = c ? csub(p, s[k]) : cadd(s[k], p);
        const float2 w = c ? make_float2(w32c(k), -w32s(k)) : make_float2(1.f, 0.f);
        v[k] = cmul(d, w);
    }
    Dft<16>::run(v, -1);
    // V[a] at n2 = 2a + c, times w512^(-n2 k1)
#pragma unroll
    for (int a = 0; a < 16; ++a) v[a] = cmulc(v[a], tf[k1 * W5_PITCH + 2 * a + c]);
    __syncwarp();
#pragma unroll
    for (int a = 0; a < 16; ++a) wb[k1 * W5_PITCH + 2 * a + c] = v[a];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = wb[q * W5_PITCH + lane];
    Dft<16>::run(v, -1);
    if (store) {
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) dst[lane + 32 * n1] = v[n1];
    }
}

// The z pass with staged real Green spectra (free space, no image), one warp per (kx,ky)
// column, W warps per CTA; the arguments and outputs are those of
// k_zconv_warp<float, W, ZW_STAGED, 512, ...> with a kz-innermost output.
template <int W>
__global__ void __launch_bounds__(W * 32, 6) k_zconv_w512(const float2 *__restrict__ in, float2 *__restrict__ out,
                                                          ZConvArgs a, const float2 *__restrict__ tw_rt) {
    constexpr int L = 512;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t gbar;
    __shared__ int gfail;
    float2 *tf = reinterpret_cast<float2 *>(smem_raw);  // [16][W5_PITCH]: w512^(l k1)
    float2 *wbufs = tf + 16 * W5_PITCH;
    float *gst = reinterpret_cast<float *>(wbufs + W * W5_BUF);  // Green columns [W][nout][zpitch]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = blockIdx.x * W;
    const int zp = a.g[0].zpitch;
    const int nst = a.nout;
    in += blockIdx.y * a.in_bstride;
    out += blockIdx.y * a.out_bstride;
    const int64_t goff = blockIdx.y * a.g_bstride;
    float2 *wb = wbufs + warp * W5_BUF;
    if (threadIdx.x == 0) {
        mbar_init(&gbar, 1);
        const int ncv = min(W, a.ncols - col0);
        mbar_arrive_expect_tx(&gbar, (unsigned)(ncv * nst * zp * (int)sizeof(float)));
        for (int cc = 0; cc < ncv; ++cc) {
            const int col = col0 + cc, ky = col / a.nxh, kx = col - ky * a.nxh;
            for (int o = 0; o < nst; ++o) {
                const GSpecDev &g = a.g[a.gdir[o]];
                const int yy = (g.sym_y && ky > a.ny) ? a.Ny - ky : ky;
                const float *src = reinterpret_cast<const float *>(g.data) + goff + ((int64_t)yy * a.nxh + kx) * zp;
                if (!a.skip_copies) bulk_g2s(gst + (cc * nst + o) * zp, src, (unsigned)(zp * sizeof(float)), &gbar);
            }
        }
    }
    for (int m = threadIdx.x; m < 16 * 32; m += W * 32) {
        const int r = m >> 5, t = m & 31;
        tf[r * W5_PITCH + t] = tw_rt[(t * r) & (L - 1)];
    }
    // the non-zero half (z < nz) of the W columns, coalesced across the columns
    for (int idx = threadIdx.x; idx < W * a.nz; idx += W * 32) {
        const int e = idx / W, cc = idx - e * W;
        const int col = col0 + cc;
        float2 v = make_float2(0.f, 0.f);
        if (col < a.ncols) v = in[(int64_t)e * a.in_estride + col];
        wbufs[cc * W5_BUF + e] = v;
    }
    __syncthreads();
    float2 s[16];
    w512_forward(wb, tf, lane, s);
    // CTA-wide wait for the staged Green columns (bounded; a give-up is reported)
    if (threadIdx.x == 0) {
        const bool ok = mbar_wait_bounded(&gbar, 0, a.poll_limit);
        if (!ok) {
            report_fault(a.fault, FAULT_BULK_WAIT);
            mbar_wait_bounded(&gbar, 0, a.poll_limit);
        }
        gfail = ok ? 0 : 1;
    }
    __syncthreads();
    if (gfail) return;
    const int colc = min(col0 + warp, a.ncols - 1);
    const int ky = colc / a.nxh;
    const bool live = col0 + warp < a.ncols;
    const int k1 = lane & 15, c = lane >> 4;
    for (int o = 0; o < a.nout; ++o) {
        const GSpecDev &g = a.g[a.gdir[o]];
        const float *gc = gst + (warp * nst + o) * zp;
        const bool yneg = g.sym_y && ky > a.ny && g.par_y < 0;
        const bool zodd = g.par_z < 0, iu = g.imag_unit;
        float2 v[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int kz = k1 + 16 * k + 256 * c;
            // kz >= nz (c = 1): the value at L - kz, odd spectra change sign (kz = nz excepted)
            float sv = gc[c ? L - kz : kz];
            const bool neg = (c && zodd && kz != a.nz) != yneg;
            sv = neg ? -sv : sv;
            const float2 x = s[k];
            v[k] = iu ? make_float2(-x.y * sv, x.x * sv) : make_float2(x.x * sv, x.y * sv);
        }
        float2 *dst = out + (int64_t)o * a.out_cstride + (int64_t)(col0 + warp) * a.out_colstride;
        w512_inverse(wb, tf, lane, v, dst, live);
    }
}

template <int W> inline size_t zconv_w512_smem(int nout, int zp) {
    return sizeof(float2) * (16 * W5_PITCH + (size_t)W * W5_BUF) + sizeof(float) * (size_t)W * nout * zp;
}

}  // namespace osc
