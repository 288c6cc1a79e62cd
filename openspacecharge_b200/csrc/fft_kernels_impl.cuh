// fft_kernels_impl.cuh -- batched shared-memory FFT kernels for the IGF convolution (sm_100a).
// Included by fft_kernels_f32.cu and fft_kernels_f64.cu, which instantiate one precision each.
//
// The free-space solve runs as five kernels over HBM (FP32 path, G spectra cached):
//   k_r2c_rows  x: real rho rows -> half spectra (two rows packed per complex line)
//   k_lines     y: forward C2C along y (input window [0,ny))
//   k_zconv     z: forward along z, multiply by the stored Green spectra, inverse along z
//   k_lines     y: inverse C2C along y (output window [0,ny))
//   k_c2r_rows  x: inverse to real rows, epilogue scatters E (and B) to their layouts
// Zero padding of the doubled grid is never stored: loads past the physical window are
// zeros (or, for the static engines, not read at all) and stores cover only the window.
#pragma once
#include <cstdio>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include "fft_kernels.cuh"
#include "zconv_warp.cuh"
#include "zconv_w512.cuh"
#include "zconv_img.cuh"

namespace osc {

#ifdef OSC_FFT_DEFINE_PLAN
bool make_fft_plan(int L, FFTPlan &p) {
    if (L < 2 || L > FFT_MAX_LEN || (L % 2) != 0) return false;
    p.L = L;
    p.nst = 0;
    int m = L;
    while (m % 8 == 0) { p.radix[p.nst++] = 8; m /= 8; }
    while (m % 4 == 0) { p.radix[p.nst++] = 4; m /= 4; }
    while (m % 2 == 0) { p.radix[p.nst++] = 2; m /= 2; }
    while (m % 3 == 0) { p.radix[p.nst++] = 3; m /= 3; }
    while (m % 5 == 0) { p.radix[p.nst++] = 5; m /= 5; }
    return m == 1 && p.nst <= FFT_MAX_STAGES;
}
// The warp-per-column z pass (FP32 and FP64) for the lengths of the warp registry.
bool zconv_warp_ok(int L, int nz, int elem_bytes) {
    if ((elem_bytes != 4 && elem_bytes != 8) || 2 * nz != L) return false;
    return dispatch_warp_len(L, [](auto eng) -> int { return decltype(eng)::kLen > 0 ? 1 : 0; }) != 0;
}
bool zconv_img_ok(int L, int nz, int elem_bytes) {
    if (!zconv_warp_ok(L, nz, elem_bytes)) return false;
    return dispatch_warp_len(L, [](auto eng) -> int {
               using E = decltype(eng);
               if constexpr (E::kLen > 0) {
                   constexpr int nb = E::kLen / E::kRad[0];
                   return nb % 32 == 0 || nb < 32 ? 1 : 0;
               }
               return 0;
           }) != 0;
}
#endif

// Engine-specific twiddle table in global memory.
template <class E, typename V> __host__ __device__ inline const V *eng_tw(const TwPair<V> &t) {
    return E::kLen > 0 ? t.st : t.rt;
}

// ------------------------------------------------------------------------------------
// MODE 0: full transform; 1: input window is the lower half (static engines skip it);
// 2: output window is the lower half and is not flipped (static engines skip the rest).
template <typename T, int NL, bool ROW, class E, int MODE>
__global__ void __launch_bounds__(E::kMaxThreads) k_lines(const cplx<T> *in, cplx<T> *out, LineArgs a,
                                                          const cplx<T> *__restrict__ twg) {
    typedef cplx<T> V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    const int L = E::kLen ? E::kLen : a.p.L;
    V *buf = tw + L;
    constexpr int lstr = NL + 1;
    const int nthreads = blockDim.x, tid = threadIdx.x;
    const int col0 = blockIdx.x * NL;
    const V *src = in + (int64_t)blockIdx.z * a.in_zstride + (int64_t)blockIdx.y * a.in_pstride;
    V *dst = out + (int64_t)blockIdx.z * a.out_zstride + (int64_t)blockIdx.y * a.out_pstride;
    load_twiddles(tw, twg, L);
    if (!ROW) {
        // columns: the first stage reads global memory, the last stage writes it
        __syncthreads();
        const bool flip = (a.flip_mask >> blockIdx.z) & 1u;
        const T sc = (T)a.scale;
        if (a.flat_lines > 0) {
            // tile over the flat line sequence: line col0 + l is column (c0 + l) of plane pl0,
            // or column (c0 + l - ncols) of plane pl0 + 1 (NL <= ncols, so at most one wrap)
            const int pl0 = col0 / a.ncols, c0 = col0 - pl0 * a.ncols;
            const V *src0 = in + (int64_t)blockIdx.z * a.in_zstride + (int64_t)pl0 * a.in_pstride;
            V *dst0 = out + (int64_t)blockIdx.z * a.out_zstride + (int64_t)pl0 * a.out_pstride;
            const int64_t in_wrap = a.in_pstride - (int64_t)a.ncols * a.in_cstride;
            const int64_t out_wrap = a.out_pstride - (int64_t)a.ncols * a.out_cstride;
            auto ld = [&](int e, int l) -> V {
                const int c = c0 + l;
                V v = mk<T>(0, 0);
                if (e < a.in_len && col0 + l < a.flat_lines)
                    v = src0[(int64_t)c * a.in_cstride + (c >= a.ncols ? in_wrap : 0) + (int64_t)e * a.in_estride];
                return v;
            };
            auto st = [&](int p, int l, const V &v) {
                const int c = c0 + l;
                const int e = (flip ? (L - p) % L : p) - a.out_lo;
                if (col0 + l < a.flat_lines && e >= 0 && e < a.out_len)
                    dst0[(int64_t)c * a.out_cstride + (c >= a.ncols ? out_wrap : 0) + (int64_t)e * a.out_estride] =
                        cscale(v, sc);
            };
            E::template run_io<V, NL, MODE == 1, MODE == 2>(buf, a.p, tw, a.sign, ld, st);
            return;
        }
        auto ld = [&](int e, int l) -> V {
            const int col = col0 + l;
            V v = mk<T>(0, 0);
            if (e < a.in_len && col < a.ncols) v = src[(int64_t)col * a.in_cstride + (int64_t)e * a.in_estride];
            return v;
        };
        auto st = [&](int p, int l, const V &v) {
            const int col = col0 + l;
            const int e = (flip ? (L - p) % L : p) - a.out_lo;
            if (col < a.ncols && e >= 0 && e < a.out_len)
                dst[(int64_t)col * a.out_cstride + (int64_t)e * a.out_estride] = cscale(v, sc);
        };
        E::template run_io<V, NL, MODE == 1, MODE == 2>(buf, a.p, tw, a.sign, ld, st);
        return;
    }
    // the static first stage skips the zero half (MODE 1 launches only with in_len == L/2)
    const int ld_len = (E::kLen > 0 && MODE == 1) ? E::kLen / 2 : L;
    const int nld = NL * ld_len;
    for (int idx = tid; idx < nld; idx += nthreads) {
        int e, c;
        if (ROW) { c = idx / ld_len; e = idx - c * ld_len; }
        else { e = idx / NL; c = idx - e * NL; }
        V v = mk<T>(0, 0);
        const int col = col0 + c;
        if (e < a.in_len && col < a.ncols) v = src[(int64_t)col * a.in_cstride + (int64_t)e * a.in_estride];
        buf[e * lstr + c] = v;
    }
    __syncthreads();
    E::template run<V, NL, MODE == 1, MODE == 2>(buf, a.p, tw, a.sign);
    const int nst = NL * a.out_len;
    const T sc = (T)a.scale;
    for (int idx = tid; idx < nst; idx += nthreads) {
        int e, c;
        if (ROW) { c = idx / a.out_len; e = idx - c * a.out_len; }
        else { e = idx / NL; c = idx - e * NL; }
        const int col = col0 + c;
        const int src_e = ((a.flip_mask >> blockIdx.z) & 1u) ? (L - (e + a.out_lo)) % L : e + a.out_lo;
        if (col < a.ncols)
            dst[(int64_t)col * a.out_cstride + (int64_t)e * a.out_estride] = cscale(buf[src_e * lstr + c], sc);
    }
}

// ------------------------------------------------------------------------------------
// Element e of real input row `row` (row < nrows, e < nin).
template <typename TIn>
__device__ __forceinline__ TIn r2c_in(const TIn *__restrict__ in, const R2CArgs &a, int64_t row, int e) {
    return in[row * a.in_rstride + e];
}
// Quad-grid input of the FP32 deposit: node (i,j) of a plane is the sum of the four
// contributions held at (i,j).x, (i-1,j).y, (i,j-1).z and (i-1,j-1).w, added in that
// fixed order (the order of k_quad_to_nodes, so rho is the same to the bit).
__device__ __forceinline__ float r2c_in(const float4 *__restrict__ in, const R2CArgs &a, int64_t row, int e) {
    const float4 *q = in + row * a.in_rstride + e;
    const bool jn = (row % a.qny) > 0;
    float s = __ldg(&q->x);
    if (e > 0) s += __ldg(&q[-1].y);
    if (jn) s += __ldg(&q[-a.in_rstride].z);
    if (e > 0 && jn) s += __ldg(&q[-a.in_rstride - 1].w);
    return s;
}

// resident CTAs the register allocation of k_r2c_rows is bounded for: 4 (32 registers, no
// spills) for the FP32 step's quad-grid input on the 8-values-per-thread engine at L = 256,
// whose loads wait on L2 (35.4 against 40.8 us at 40 registers and 3 CTAs); 1 otherwise
template <typename T, typename TIn, class E> constexpr int r2c_minb() {
    return (std::is_same<TIn, float4>::value && E::kLen == 256 && E::kEPT == 8) ? 4 : 1;
}
template <typename T, typename TIn, int NL, class E, bool HIN>
__global__ void __launch_bounds__(E::kMaxThreads, r2c_minb<T, TIn, E>()) k_r2c_rows(const TIn *__restrict__ in, cplx<T> *__restrict__ out,
                                                             R2CArgs a, const cplx<T> *__restrict__ twg) {
    typedef cplx<T> V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    const int L = E::kLen ? E::kLen : a.p.L;
    V *buf = tw + L;
    constexpr int lstr = NL + 1;
    // static engines launch with L*NL/E::kEPT threads: compile-time trip counts below
    const int nthreads = E::kLen ? E::kLen * NL / E::kEPT : (int)blockDim.x, tid = threadIdx.x;
    const int64_t row0 = (int64_t)blockIdx.x * (2 * NL);
    load_twiddles(tw, twg, L);
    const int ld_len = (E::kLen > 0 && HIN) ? E::kLen / 2 : L;  // HIN launches only with nin == L/2
    if constexpr (E::kLen > 0) {
        // all of a thread's loads are issued before any is stored to shared memory
        constexpr int LDL = HIN ? E::kLen / 2 : E::kLen, NT = E::kLen * NL / E::kEPT;
        constexpr int IT = (2 * NL * LDL + NT - 1) / NT;
        T v[IT];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int idx = tid + it * NT, rr = idx / LDL, e = idx - rr * LDL;
            const int64_t row = row0 + rr;
            v[it] = 0;
            if (idx < 2 * NL * LDL && row < a.nrows && e < a.nin) v[it] = (T)r2c_in(in, a, row, e);
        }
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int idx = tid + it * NT, rr = idx / LDL, e = idx - rr * LDL;
            if (idx < 2 * NL * LDL) reinterpret_cast<T *>(&buf[e * lstr + (rr >> 1)])[rr & 1] = v[it];
        }
    } else {
        for (int idx = tid; idx < 2 * NL * ld_len; idx += nthreads) {
            const int rr = idx / ld_len, e = idx - rr * ld_len;
            const int64_t row = row0 + rr;
            T v = 0;
            if (row < a.nrows && e < a.nin) v = (T)r2c_in(in, a, row, e);
            T *slot = reinterpret_cast<T *>(&buf[e * lstr + (rr >> 1)]);
            slot[rr & 1] = v;
        }
    }
    __syncthreads();
    E::template run<V, NL, HIN, false>(buf, a.p, tw, +1);
    const int nh = L / 2 + 1;
    for (int idx = tid; idx < 2 * NL * nh; idx += nthreads) {
        const int rr = idx / nh, k = idx - rr * nh;
        const int64_t row = row0 + rr;
        if (row >= a.nrows) continue;
        const int line = rr >> 1;
        const V Z = buf[k * lstr + line];
        const V Zm = buf[((L - k) % L) * lstr + line];
        V r;
        if ((rr & 1) == 0) {  // (Z + conj Zm)/2
            r.x = (T)0.5 * (Z.x + Zm.x);
            r.y = (T)0.5 * (Z.y - Zm.y);
        } else {  // (Z - conj Zm)/(2i)
            r.x = (T)0.5 * (Z.y + Zm.y);
            r.y = (T)0.5 * (Zm.x - Z.x);
        }
        out[row * a.out_rstride + k] = r;
    }
}

// ------------------------------------------------------------------------------------
// Input offset and output grid row of real row r of an x inverse (see C2RArgs::zin).
__device__ __forceinline__ void row_bases(const C2RArgs &a, int64_t r, int64_t &in_off, int64_t &out_row) {
    if (!a.zin) {
        in_off = r * a.in_rstride;
        out_row = r;
        return;
    }
    const int64_t t = r / a.zin_nz, z = r - t * a.zin_nz;  // t = b*ny + y
    const int64_t b = t / a.zin_ny, y = t - b * a.zin_ny;
    in_off = t * a.in_rstride + z;
    out_row = (b * a.zin_nz + z) * a.zin_ny + y;
}

template <typename T>
__device__ __forceinline__ void write_dest(const OutDest &d, int64_t gidx, int x, T val) {
    // vec4 grids also write their unused 4th slot, so every 32-byte sector is written whole
    switch (d.kind) {
    case 0: {
        T *p = reinterpret_cast<T *>(d.ptr) + gidx * 4;
        p[d.slot] = (T)(d.coef * val);
        if (d.slot == 2) p[3] = (T)0;
        break;
    }
    case 1: reinterpret_cast<double *>(d.ptr)[gidx] = d.coef * (double)val; break;
    case 3: reinterpret_cast<double *>(d.ptr)[gidx] += d.coef * (double)val; break;
    case 4: {  // x-pair grid: node n holds (E(n), E(n+1)) as two vec4; the last node's
               // second half is never read and is zeroed
        T *p = reinterpret_cast<T *>(d.ptr);
        const T v = (T)(d.coef * val);
        p[gidx * 8 + d.slot] = v;
        if (d.slot == 2) p[gidx * 8 + 3] = (T)0;
        if (x > 0) {
            p[(gidx - 1) * 8 + 4 + d.slot] = v;
            if (d.slot == 2) p[(gidx - 1) * 8 + 7] = (T)0;
        }
        if (x == d.last_x) {
            p[gidx * 8 + 4 + d.slot] = (T)0;
            if (d.slot == 2) p[gidx * 8 + 7] = (T)0;
        }
        break;
    }
    default: reinterpret_cast<T *>(d.ptr)[gidx] = (T)(d.coef * val); break;
    }
}

template <typename T, int NL, class E, bool HOUT>
__global__ void __launch_bounds__(E::kMaxThreads) k_c2r_rows(const cplx<T> *__restrict__ in, C2RArgs a,
                                                             const cplx<T> *__restrict__ twg) {
    typedef cplx<T> V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    const int L = E::kLen ? E::kLen : a.p.L;
    V *buf = tw + L;
    constexpr int lstr = NL + 1;
    const int nthreads = blockDim.x, tid = threadIdx.x;
    const int64_t row0 = (int64_t)blockIdx.x * (2 * NL);
    const int half = L / 2;
    T *res = reinterpret_cast<T *>(buf + L * lstr);  // [3][2*NL][nout] when a.e8 is set
    __shared__ int64_t rin[2 * NL], rout[2 * NL];
    for (int t = tid; t < 2 * NL; t += nthreads) row_bases(a, row0 + t, rin[t], rout[t]);
    const int64_t ies = a.zin ? a.zin_nz : 1;
    load_twiddles(tw, twg, L);
    __syncthreads();
    for (int c = 0; c < a.ncomp; ++c) {
        const V *src = in + (int64_t)c * a.in_cstride;
        for (int idx = tid; idx < NL * L; idx += nthreads) {
            int line, k;
            if (a.zin) {  // adjacent lines (adjacent z) fastest for the kz-innermost spectra
                k = idx / NL;
                line = idx - k * NL;
            } else {
                line = idx / L;
                k = idx - line * L;
            }
            const int64_t ra = row0 + 2 * line, rb = ra + 1;
            const int kk = k <= half ? k : L - k;
            V A = mk<T>(0, 0), B = mk<T>(0, 0);
            if (ra < a.nrows) A = src[rin[2 * line] + kk * ies];
            if (rb < a.nrows) B = src[rin[2 * line + 1] + kk * ies];
            if (k == 0 || k == half) { A.y = 0; B.y = 0; }
            if (k > half) { A.y = -A.y; B.y = -B.y; }
            buf[k * lstr + line] = mk<T>(A.x - B.y, A.y + B.x);
        }
        __syncthreads();
        E::template run<V, NL, false, HOUT>(buf, a.p, tw, -1);
        for (int idx = tid; idx < 2 * NL * a.nout; idx += nthreads) {
            const int rr = idx / a.nout, x = idx - rr * a.nout;
            const int64_t row = row0 + rr;
            if (row >= a.nrows) continue;
            const int xs = ((a.flip_mask >> c) & 1u) ? (L - x) % L : x;
            const V z = buf[xs * lstr + (rr >> 1)];
            const T val = (rr & 1) ? z.y : z.x;
            const int64_t gidx = rout[rr] * a.nout + x;
            for (int d = 0; d < a.ndest[c]; ++d) write_dest<T>(a.dest[c][d], gidx, x, val);
            if (a.e8) {
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    if (a.e8_comp[q] == c) res[(q * 2 * NL + rr) * a.nout + x] = val;
            }
        }
        __syncthreads();
    }
    if (a.e8) {
        // x-pair grid rows: node n gets (E(n), E(n+1)), the row's last node (E(n), 0)
        typedef vec4<T> V4;
        V4 *g = reinterpret_cast<V4 *>(a.e8);
        for (int idx = tid; idx < 2 * NL * a.nout; idx += nthreads) {
            const int rr = idx / a.nout, x = idx - rr * a.nout;
            const int64_t row = row0 + rr;
            if (row >= a.nrows) continue;
            const int64_t gidx = rout[rr] * a.nout + x;
            const T *r0 = res + rr * a.nout + x;
            const int64_t cs = (int64_t)2 * NL * a.nout;
            V4 lo, hi;
            lo.x = r0[0];
            lo.y = r0[cs];
            lo.z = r0[2 * cs];
            lo.w = (T)0;
            if (x + 1 < a.nout) {
                hi.x = r0[1];
                hi.y = r0[cs + 1];
                hi.z = r0[2 * cs + 1];
            } else {
                hi.x = hi.y = hi.z = (T)0;
            }
            hi.w = (T)0;
            if (a.e8_node) {
                g[gidx] = lo;
            } else {
                g[2 * gidx] = lo;
                g[2 * gidx + 1] = hi;
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// HALF: nz == L/2, so the static engine's forward first stage skips the zero half and
// its inverse last stage skips the upper half, which is never stored.  The forward
// transform reads the column straight from global memory into its first stage; each
// inverse transform computes its input (spectrum times Green spectrum, plus the image term)
// inside its first stage and writes its last stage straight to global memory.
template <typename T, int NL, class E, bool HALF>
__global__ void __launch_bounds__(E::kMaxThreads) k_zconv(const cplx<T> *__restrict__ in, cplx<T> *__restrict__ out,
                                                          ZConvArgs a, const cplx<T> *__restrict__ twg,
                                                          const cplx<T> *__restrict__ tw_rt) {
    typedef cplx<T> V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    const int L = E::kLen ? E::kLen : a.p.L;
    V *rhat = tw + L;
    constexpr int lstr = NL + 1;
    V *buf = rhat + L * lstr;
    const int col0 = blockIdx.x * NL;
    in += blockIdx.y * a.in_bstride;
    out += blockIdx.y * a.out_bstride;
    const int64_t goff = blockIdx.y * a.g_bstride;
    load_twiddles(tw, twg, L);
    __syncthreads();
    auto ld_in = [&](int e, int l) -> V {
        const int col = col0 + l;
        V v = mk<T>(0, 0);
        if (e < a.nz && col < a.ncols) v = in[(int64_t)e * a.in_estride + col];
        return v;
    };
    auto st_rhat = [&](int e, int l, const V &v) { rhat[e * lstr + l] = v; };
    E::template run_io<V, NL, HALF, false>(rhat, a.p, tw, +1, ld_in, st_rhat);
    for (int o = 0; o < a.nout; ++o) {
        const int gd = a.gdir[o], gi = a.gimg[o];
        const T icoef = (T)a.img_coef[o];
        auto ld_mul = [&](int e, int l) -> V {
            const int col = min(col0 + l, a.ncols - 1);
            const int ky = col / a.nxh, kx = col - ky * a.nxh;
            V S = mk<T>(0, 0);
            if (gd >= 0)
                S = cmul(rhat[e * lstr + l], g_lookup<T>(a.g[gd], kx, ky, e, a.nxh, a.Ny, a.ny, L, a.nz, goff));
            if (gi >= 0) {
                // spectrum of -rho flipped in z: -w^((nz-1) kz) * rho_hat(-kz)
                const V rm = rhat[((L - e) % L) * lstr + l];
                const V ph = __ldg(tw_rt + (int)(((int64_t)a.img_phase_mul * e) % L));
                V ri = cmul(ph, rm);
                ri.x = -ri.x * icoef;
                ri.y = -ri.y * icoef;
                S = cadd(S, cmul(ri, g_lookup<T>(a.g[gi], kx, ky, e, a.nxh, a.Ny, a.ny, L, a.nz, goff)));
            }
            return S;
        };
        V *dst = out + (int64_t)o * a.out_cstride;
        auto st_out = [&](int e, int l, const V &v) {
            const int col = col0 + l;
            if (e < a.nz && col < a.ncols) dst[(int64_t)e * a.out_estride + (int64_t)col * a.out_colstride] = v;
        };
        E::template run_io<V, NL, false, HALF>(buf, a.p, tw, -1, ld_mul, st_out);
    }
}

// x inverse of the FP32 step: three E components of 2*NLC real rows each go through one
// transform batch of 3*NLC complex lines, and every output node of the window x < L/2 is
// written as one 32-byte x-pair (E(x), E(x+1)) with a single 256-bit store.  Requires the
// static engine for L, nout = L/2, no index flips and no other destinations.
__device__ __forceinline__ void st_pair(float4 *p, const float4 &lo, const float4 &hi) {
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(lo.x), "f"(lo.y), "f"(lo.z),
                 "f"(lo.w), "f"(hi.x), "f"(hi.y), "f"(hi.z), "f"(hi.w)
                 : "memory");
}
__device__ __forceinline__ void st_node(double4 *p, double x, double y, double z) {
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(x), "d"(y), "d"(z), "d"(0.0) : "memory");
}
template <typename T, class E> constexpr int c2r_e8_nlc() {
    return (E::kLen <= 128 ? 16 : (E::kLen <= 256 ? 8 : 4)) / (sizeof(T) == 8 ? 2 : 1);
}

// FP32: x-pair nodes (E(x), E(x+1)) with one 256-bit store; FP64: nodes (Ex, Ey, Ez, 0)
// with one 256-bit store.
template <typename T, int NLC, class E>
__global__ void __launch_bounds__(E::kLen * 3 * NLC / E::kEPT, sizeof(T) == 4 ? 3 : 1) k_c2r_e8(const cplx<T> *__restrict__ in, C2RArgs a,
                                                                      const cplx<T> *__restrict__ twg) {
    typedef cplx<T> V;
    constexpr int L = E::kLen, NLT = 3 * NLC, lstr = NLT + 1, half = L / 2, nout = L / 2;
    constexpr int nthreads = L * NLT / E::kEPT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *buf = tw + L;
    const int tid = threadIdx.x;
    const int64_t row0 = (int64_t)blockIdx.x * (2 * NLC);
    __shared__ int64_t rin[2 * NLC], rout[2 * NLC];
    for (int t = tid; t < 2 * NLC; t += nthreads) row_bases(a, row0 + t, rin[t], rout[t]);
    const int64_t ies = a.zin ? a.zin_nz : 1;
    load_twiddles(tw, twg, L);
    __syncthreads();
    // line = two real rows A + iB; each stored value k <= L/2 is read once and also gives
    // the line's value at L-k (from the conjugates)
    constexpr int nk = half + 1, IT = (NLT * nk + nthreads - 1) / nthreads;
    auto slot_of = [&](int idx, int &c, int &line, int &k) {
        if (a.zin) {  // rows (adjacent z) fastest: coalesced reads of the kz-innermost spectra
            k = idx / NLT;
            const int rem = idx - k * NLT;
            c = rem / NLC;
            line = rem - c * NLC;
        } else {
            c = idx / (NLC * nk);
            const int rem = idx - c * (NLC * nk);
            line = rem / nk;
            k = rem - line * nk;
        }
    };
    // all of a thread's loads are issued before any is stored to shared memory
    V A[IT], B[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int idx = tid + it * nthreads;
        A[it] = mk<T>(0, 0);
        B[it] = mk<T>(0, 0);
        if (idx < NLT * nk) {
            int c, line, k;
            slot_of(idx, c, line, k);
            const V *src = in + (int64_t)a.e8_comp[c] * a.in_cstride;
            const int64_t ra = row0 + 2 * line, rb = ra + 1;
            if (ra < a.nrows) A[it] = src[rin[2 * line] + k * ies];
            if (rb < a.nrows) B[it] = src[rin[2 * line + 1] + k * ies];
        }
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int idx = tid + it * nthreads;
        if (idx < NLT * nk) {
            int c, line, k;
            slot_of(idx, c, line, k);
            V a0 = A[it], b0 = B[it];
            if (k == 0 || k == half) { a0.y = 0; b0.y = 0; }
            buf[k * lstr + c * NLC + line] = mk<T>(a0.x - b0.y, a0.y + b0.x);
            if (k > 0 && k < half) buf[(L - k) * lstr + c * NLC + line] = mk<T>(a0.x + b0.y, b0.x - a0.y);
        }
    }
    __syncthreads();
    E::template run<V, NLT, false, true>(buf, a.p, tw, -1);
    for (int idx = tid; idx < 2 * NLC * nout; idx += nthreads) {
        const int rr = idx / nout, x = idx - rr * nout;
        const int64_t row = row0 + rr;
        if (row >= a.nrows) continue;
        const int ln = rr >> 1;
        const bool odd = rr & 1;
        T e0[3], e1[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const V z0 = buf[x * lstr + c * NLC + ln];
            e0[c] = odd ? z0.y : z0.x;
            if constexpr (sizeof(T) == 4) {
                if (x + 1 < nout) {
                    const V z1 = buf[(x + 1) * lstr + c * NLC + ln];
                    e1[c] = odd ? z1.y : z1.x;
                } else {
                    e1[c] = 0;
                }
            }
        }
        if constexpr (sizeof(T) == 4) {
            st_pair(reinterpret_cast<float4 *>(a.e8) + 2 * (rout[rr] * nout + x),
                    make_float4(e0[0], e0[1], e0[2], 0.f), make_float4(e1[0], e1[1], e1[2], 0.f));
        } else {
            st_node(reinterpret_cast<double4 *>(a.e8) + rout[rr] * nout + x, e0[0], e0[1], e0[2]);
        }
    }
}

// Even/odd real line transforms (Green spectra): two real lines per complex line, the
// parity extension formed in the load, the halves separated after the transform.  TC is
// the arithmetic type (and that of the twiddles), TI the input's, TO the output's.
template <typename TC, typename TI, typename TO, int NL, class E, bool LDE, bool STK>
__global__ void __launch_bounds__(E::kMaxThreads) k_sym_lines(const TI *__restrict__ in, TO *__restrict__ out,
                                                              SymArgs a, const cplx<TC> *__restrict__ twg) {
    typedef cplx<TC> V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int64_t bin[2 * NL], bout[2 * NL];
    __shared__ int podd[2 * NL];
    V *tw = reinterpret_cast<V *>(smem_raw);
    const int L = E::kLen ? E::kLen : a.p.L;
    V *buf = tw + L;
    constexpr int lstr = NL + 1;
    const int nthreads = blockDim.x, tid = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * (2 * NL);
    const int n = a.n;
    for (int t = tid; t < 2 * NL; t += nthreads) {  // line start offsets, once per line
        const int64_t r = r0 + t;
        int64_t oi = -1, oo = -1;
        int odd = 0;
        if (r < a.nlines) {
            const int64_t bi = r / a.npq, rl = r - bi * a.npq;
            const int64_t pi = rl / a.nq, qi = rl - pi * a.nq;
            oi = bi * a.in_bs + pi * a.in_ps + qi * a.in_qs;
            oo = bi * a.out_bs + pi * a.out_ps + qi * a.out_qs;
            odd = bi >= a.odd_lo && bi < a.odd_hi;
        }
        bin[t] = oi;
        bout[t] = oo;
        podd[t] = odd;
    }
    load_twiddles(tw, twg, L);
    __syncthreads();
    if constexpr (E::kLen > 0) {
        // static engine (L = 2n known, L*NL/E::kEPT threads): each thread first loads its
        // share of the n+1 distinct values of every line into registers (all loads in
        // flight), then writes each value at e and its parity image at L-e
        constexpr int nh = E::kLen / 2, NK = nh + 1, TOT = 2 * NL * NK;
        constexpr int NT = E::kLen * NL / E::kEPT, IT = (TOT + NT - 1) / NT;
        TC v[IT];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int idx = tid + it * NT;
            v[it] = (TC)0;
            if (idx < TOT) {
                int rr, e;
                if (LDE) { rr = idx / NK; e = idx - rr * NK; }
                else { e = idx / (2 * NL); rr = idx - e * (2 * NL); }
                const int64_t o = bin[rr];
                if (o >= 0 && e != nh) v[it] = (TC)in[o + (int64_t)e * a.in_es];
            }
        }
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int idx = tid + it * NT;
            if (idx < TOT) {
                int rr, e;
                if (LDE) { rr = idx / NK; e = idx - rr * NK; }
                else { e = idx / (2 * NL); rr = idx - e * (2 * NL); }
                reinterpret_cast<TC *>(&buf[e * lstr + (rr >> 1)])[rr & 1] = v[it];
                if (e > 0 && e < nh)
                    reinterpret_cast<TC *>(&buf[(E::kLen - e) * lstr + (rr >> 1)])[rr & 1] =
                        podd[rr] ? -v[it] : v[it];
            }
        }
    } else {
        for (int idx = tid; idx < 2 * NL * L; idx += nthreads) {
            int rr, e;
            if (LDE) { rr = idx / L; e = idx - rr * L; }
            else { e = idx / (2 * NL); rr = idx - e * (2 * NL); }
            const int64_t o = bin[rr];
            TC v = (TC)0;
            if (o >= 0 && e != n) {
                const int src = e < n ? e : L - e;
                v = (TC)in[o + (int64_t)src * a.in_es];
                if (e > n && podd[rr]) v = -v;
            }
            TC *slot = reinterpret_cast<TC *>(&buf[e * lstr + (rr >> 1)]);
            slot[rr & 1] = v;
        }
    }
    __syncthreads();
    E::template run<V, NL, false, false>(buf, a.p, tw, +1);
    const int nk = n + 1;
    for (int idx = tid; idx < 2 * NL * nk; idx += nthreads) {
        int rr, k;
        if (STK) { rr = idx / nk; k = idx - rr * nk; }
        else { k = idx / (2 * NL); rr = idx - k * (2 * NL); }
        const int64_t o = bout[rr];
        if (o < 0) continue;
        const V Z = buf[k * lstr + (rr >> 1)];
        const V Zm = buf[((L - k) % L) * lstr + (rr >> 1)];
        const bool odd = podd[rr];
        TC sv;
        const TC hf = (TC)0.5;
        if ((rr & 1) == 0) sv = !odd ? hf * (Z.x + Zm.x) : hf * (Z.y - Zm.y);
        else sv = !odd ? hf * (Z.y + Zm.y) : hf * (Zm.x - Z.x);
        out[o + (int64_t)k * a.out_es] = (TO)(sv * (TC)a.scale);
    }
}

// ------------------------------------------------------------------------------------
// Launchers.  Shared memory above 48 KB needs the opt-in attribute, set per kernel.
// The attribute is set once per kernel, device and size (a lookup instead of a driver call
// on every launch of the many small launches of a batch).
template <typename K> inline int set_smem(K kern, size_t bytes) {
    if (bytes > 227 * 1024) return OSC_E_INVALID;
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return OSC_E_CUDA;
    const auto key = std::make_pair(reinterpret_cast<const void *>(kern), dev);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = done.find(key);
        if (it != done.end() && it->second >= bytes) return OSC_OK;
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return OSC_E_CUDA;
    std::lock_guard<std::mutex> lk(mu);
    size_t &v = done[key];
    if (bytes > v) v = bytes;
    return OSC_OK;
}
inline int launch_ok() { return cudaGetLastError() == cudaSuccess ? OSC_OK : OSC_E_CUDA; }

// Runtime-engine NL: a whole number of threads, <= 256 threads, buffers within budget.
inline int pick_nl_rt(int L, int nl_max, size_t elem, int nbuf) {
    for (int nl = nl_max; nl >= 2; nl /= 2) {
        if ((L * nl) % FFT_EPT != 0 || fft_threads(L, nl) > FftRuntime::kMaxThreads) continue;
        if ((size_t)nbuf * L * (nl + 1) * elem + L * elem > 110 * 1024 && nl > 2) continue;
        return nl;
    }
    return 0;
}

// Calls f(std::integral_constant<int, NL>) for the engine's lines-per-CTA.  Static engines
// use a compile-time NL: the widest that fits (one line buffer) or, for the two-buffer
// z-pass, at most 4 lines in ~48 KB so several CTAs share an SM.
template <typename T, class E, class F>
inline int with_nl(int L, int nbuf, int nl_max, int nl_req, F &&f, int nl_div = 0) {
    if constexpr (E::kLen > 0) {
        (void)L;
        (void)nl_req;
        (void)nl_max;
        constexpr int NL1 = nl_static(E::kLen, sizeof(T) == 4 ? 16 : 8, (int)sizeof(cplx<T>), 1, 100 * 1024, E::kEPT);
        constexpr int NL2 = nl_static(E::kLen, 4, (int)sizeof(cplx<T>), 2, 64 * 1024, E::kEPT);
        if (nbuf >= 2) return f(std::integral_constant<int, NL2>{});
        // the autotuner's alternative tile: half the lines per CTA (more, smaller CTAs)
        constexpr int NLH = NL1 >= 4 && ((E::kLen * (NL1 / 2)) % E::kEPT) == 0 ? NL1 / 2 : NL1;
        if (nl_div == 2 && NLH != NL1) return f(std::integral_constant<int, NLH>{});
        return f(std::integral_constant<int, NL1>{});
    } else {
        int nl = nl_req > 0 ? nl_req : pick_nl_rt(L, nl_max, sizeof(cplx<T>), nbuf);
        switch (nl) {
        case 16: return f(std::integral_constant<int, 16>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 4: return f(std::integral_constant<int, 4>{});
        case 2: return f(std::integral_constant<int, 2>{});
        default: return OSC_E_FFT_SIZE;
        }
    }
}

template <typename T, int NL, bool ROW, class E, int MODE>
inline int launch_lines_k(const cplx<T> *in, cplx<T> *out, const LineArgs &a, int nplanes, int ncomp, const cplx<T> *tw,
                          cudaStream_t st) {
    const int L = a.p.L;
    const int nt = fft_threads(L, NL, E::kEPT);
    if (nt < 1 || nt > E::kMaxThreads || (L * NL) % E::kEPT) return OSC_E_FFT_SIZE;
    const size_t sm = sizeof(cplx<T>) * ((size_t)L + (size_t)L * (NL + 1));
    auto kern = k_lines<T, NL, ROW, E, MODE>;
    int rc = set_smem(kern, sm);
    if (rc) return rc;
    // the flat tiling needs a column layout, at most one plane wrap per tile and int line indices
    const bool flat = !ROW && a.flat_lines > 0 && a.ncols >= NL && (int64_t)a.ncols * nplanes < (1ll << 30);
    LineArgs af = a;
    af.flat_lines = flat ? a.ncols * nplanes : 0;
    dim3 grid(flat ? (unsigned)ceil_div(af.flat_lines, NL) : (unsigned)ceil_div(a.ncols, NL),
              flat ? 1u : (unsigned)nplanes, (unsigned)ncomp);
    kern<<<grid, nt, sm, st>>>(in, out, af, tw);
    return launch_ok();
}

template <typename T>
int launch_lines(const cplx<T> *in, cplx<T> *out, const LineArgs &a, int nplanes, int ncomp, bool row_mode,
                 const TwPair<cplx<T>> &tw, cudaStream_t st) {
    const int L = a.p.L;
    return dispatch_fft_len<T>(L, [&](auto eng) -> int {
        using E = decltype(eng);
        const cplx<T> *twe = eng_tw<E>(tw);
        return with_nl<T, E>(L, 1, sizeof(T) == 4 ? 16 : 8, 0, [&](auto nlc) -> int {
            constexpr int NL = decltype(nlc)::value;
            if (row_mode) return launch_lines_k<T, NL, true, E, 0>(in, out, a, nplanes, ncomp, twe, st);
            if constexpr (E::kLen > 0) {
                if (2 * a.in_len == L && a.out_len == L && a.out_lo == 0)
                    return launch_lines_k<T, NL, false, E, 1>(in, out, a, nplanes, ncomp, twe, st);
                if (a.in_len == L && 2 * a.out_len == L && a.out_lo == 0 && a.flip_mask == 0)
                    return launch_lines_k<T, NL, false, E, 2>(in, out, a, nplanes, ncomp, twe, st);
            }
            return launch_lines_k<T, NL, false, E, 0>(in, out, a, nplanes, ncomp, twe, st);
        }, row_mode ? 0 : a.nl_div);
    });
}

template <typename T, typename TIn>
int launch_r2c_rows(const TIn *in, cplx<T> *out, const R2CArgs &a, const TwPair<cplx<T>> &tw, cudaStream_t st) {
    const int L = a.p.L;
    // the FP32 x transform at L = 256 runs faster with 8 values per thread (the other FP32
    // passes at 256 do not); same radices as the 16-value engine, so the same twiddle table
    auto dispatch = [&](auto &&f) -> int {
        if constexpr (sizeof(T) == 4)
            if (L == 256) return f(FftStatic8<256, 8, 8, 4>{});
        return dispatch_fft_len<T>(L, f);
    };
    return dispatch([&](auto eng) -> int {
        using E = decltype(eng);
        const cplx<T> *twe = eng_tw<E>(tw);
        return with_nl<T, E>(L, 1, sizeof(T) == 4 ? 16 : 8, 0, [&](auto nlc) -> int {
            constexpr int NL = decltype(nlc)::value;
            const int nt = fft_threads(L, NL, E::kEPT);
            if (nt < 1 || nt > E::kMaxThreads || (L * NL) % E::kEPT) return OSC_E_FFT_SIZE;
            const size_t sm = sizeof(cplx<T>) * ((size_t)L + (size_t)L * (NL + 1));
            const unsigned nblk = (unsigned)ceil_div(a.nrows, 2 * NL);
            if (E::kLen > 0 && 2 * a.nin == L) {
                auto kern = k_r2c_rows<T, TIn, NL, E, true>;
                int rc = set_smem(kern, sm);
                if (rc) return rc;
                kern<<<nblk, nt, sm, st>>>(in, out, a, twe);
            } else {
                auto kern = k_r2c_rows<T, TIn, NL, E, false>;
                int rc = set_smem(kern, sm);
                if (rc) return rc;
                kern<<<nblk, nt, sm, st>>>(in, out, a, twe);
            }
            return launch_ok();
        }, a.nl_div);
    });
}

template <typename T>
int launch_c2r_rows(const cplx<T> *in, const C2RArgs &a, const TwPair<cplx<T>> &tw, cudaStream_t st) {
    const int L = a.p.L;
    // FP32 x-pairs or FP64 nodes: the specialised kernel; other combinations: generic
    if (a.e8 && (a.e8_node != 0) == (sizeof(T) == 8)) {
        bool e8_only = a.e8 && a.ncomp == 3 && a.flip_mask == 0 && 2 * a.nout == L &&
                       reinterpret_cast<uintptr_t>(a.e8) % 32 == 0;
        for (int c = 0; c < a.ncomp && e8_only; ++c) e8_only = a.ndest[c] == 0;
        if (e8_only) {
            const int rc = dispatch_fft_len<T>(L, [&](auto eng) -> int {
                using E = decltype(eng);
                if constexpr (E::kLen > 0) {
                    auto go = [&](auto nlcc) -> int {
                        constexpr int NLC = decltype(nlcc)::value;
                        constexpr int nt = E::kLen * 3 * NLC / E::kEPT;
                        const size_t sm = sizeof(cplx<T>) * ((size_t)E::kLen + (size_t)E::kLen * (3 * NLC + 1));
                        auto kern = k_c2r_e8<T, NLC, E>;
                        int r = set_smem(kern, sm);
                        if (r) return r;
                        kern<<<(unsigned)ceil_div(a.nrows, 2 * NLC), nt, sm, st>>>(in, a, tw.st);
                        return launch_ok();
                    };
                    constexpr int NLC = c2r_e8_nlc<T, E>();
                    // the autotuner's alternative tile: half the rows per CTA
                    constexpr int NLH = NLC >= 2 && (E::kLen * 3 * (NLC / 2)) % E::kEPT == 0 ? NLC / 2 : NLC;
                    if (a.nl_div == 2 && NLH != NLC) return go(std::integral_constant<int, NLH>{});
                    return go(std::integral_constant<int, NLC>{});
                }
                return -1;  // no static engine: generic kernel
            });
            if (rc != -1) return rc;
        }
    }
    return dispatch_fft_len<T>(L, [&](auto eng) -> int {
        using E = decltype(eng);
        const cplx<T> *twe = eng_tw<E>(tw);
        return with_nl<T, E>(L, 1, sizeof(T) == 4 ? 16 : 8, 0, [&](auto nlc) -> int {
            constexpr int NL = decltype(nlc)::value;
            const int nt = fft_threads(L, NL, E::kEPT);
            if (nt < 1 || nt > E::kMaxThreads || (L * NL) % E::kEPT) return OSC_E_FFT_SIZE;
            const size_t sm = sizeof(cplx<T>) * ((size_t)L + (size_t)L * (NL + 1)) +
                              (a.e8 ? sizeof(T) * 3 * 2 * NL * (size_t)a.nout : 0);
            const unsigned nblk = (unsigned)ceil_div(a.nrows, 2 * NL);
            if (E::kLen > 0 && 2 * a.nout == L && a.flip_mask == 0) {
                auto kern = k_c2r_rows<T, NL, E, true>;
                int rc = set_smem(kern, sm);
                if (rc) return rc;
                kern<<<nblk, nt, sm, st>>>(in, a, twe);
            } else {
                auto kern = k_c2r_rows<T, NL, E, false>;
                int rc = set_smem(kern, sm);
                if (rc) return rc;
                kern<<<nblk, nt, sm, st>>>(in, a, twe);
            }
            return launch_ok();
        });
    });
}

template <typename T, int W, int MODE, int L, int... Rs>
inline int launch_zconv_warp_k(const cplx<T> *in, cplx<T> *out, const ZConvArgs &a, const TwPair<cplx<T>> &tw,
                               cudaStream_t st) {
    const size_t sm = zconv_warp_smem<T>(L, W, MODE, MODE == ZW_SUM ? a.nsum : a.nout, a.g[0].zpitch);
    auto kern = k_zconv_warp<T, W, MODE, L, Rs...>;
    int rc = set_smem(kern, sm);
    if (rc) return rc;
    // summed inputs: the members are the inputs of one output, read by every CTA
    const unsigned gy = MODE == ZW_SUM ? 1u : (unsigned)(a.nbatch > 0 ? a.nbatch : 1);
    const dim3 grid((unsigned)ceil_div(a.ncols, W), gy);
    kern<<<grid, W * 32, sm, st>>>(in, out, a, tw.wt, tw.rt);
    return launch_ok();
}
template <typename T, int MODE, int L, int... Rs>
inline int launch_zconv_warp(WarpFft<L, Rs...>, const cplx<T> *in, cplx<T> *out, const ZConvArgs &a,
                             const TwPair<cplx<T>> &tw, cudaStream_t st) {
    return launch_zconv_warp_k<T, zw_warps<T>(), MODE, L, Rs...>(in, out, a, tw, st);
}

// Staged Green columns need real spectra, even/odd in z, one common 16-byte column pitch
// (one column per output, or per input when the inputs are summed).
template <typename T> inline bool zconv_can_stage(const ZConvArgs &a) {
    const int zp = a.g[0].zpitch;
    if (zp <= 0 || (zp * sizeof(T)) % 16) return false;
    const int ns = a.nsum > 0 ? a.nsum : a.nout;
    for (int o = 0; o < ns; ++o) {
        const int gd = a.gdir[o];
        if (gd < 0 || a.gimg[o] >= 0) return false;
        const GSpecDev &g = a.g[gd];
        if (!g.real_valued || !g.sym_z || !g.zinner || g.zpitch != zp || g.dimz > zp) return false;
        if (reinterpret_cast<uintptr_t>(g.data) % 16) return false;
    }
    return zconv_warp_smem<T>(a.p.L, zw_warps<T>(), ZW_STAGED, ns, zp) <= 100 * 1024;
}

// The image z pass: every output has a staged-compatible direct spectrum and a herm_img
// image spectrum, each kind with one 16-byte column pitch; kz-innermost output.
template <typename T> inline bool zconv_img_can(const ZConvArgs &a) {
    if (a.nout < 1 || a.nsum > 0 || a.out_estride != 1 || a.g_bstride != 0) return false;
    const int zp = a.g[a.gdir[0] >= 0 ? a.gdir[0] : 0].zpitch, zpi = a.g[a.gimg[0] >= 0 ? a.gimg[0] : 0].zpitch;
    if ((zp * sizeof(T)) % 16 || (zpi * sizeof(cplx<T>)) % 16) return false;
    for (int o = 0; o < a.nout; ++o) {
        const int gd = a.gdir[o], gi = a.gimg[o];
        if (gd < 0 || gi < 0) return false;
        const GSpecDev &d = a.g[gd], &m = a.g[gi];
        if (!d.real_valued || !d.sym_z || !d.sym_y || !d.zinner || d.zpitch != zp || d.dimz > zp) return false;
        if (!m.herm_img || !m.sym_y || !m.zinner || m.zpitch != zpi || m.dimz != a.nz + 1 || m.dimz > zpi) return false;
        if (reinterpret_cast<uintptr_t>(d.data) % 16 || reinterpret_cast<uintptr_t>(m.data) % 16) return false;
    }
    return zconv_img_smem<T>(a.p.L, a.nout, zp, zpi) <= 200 * 1024;
}
// The same kernel without images (the staged free-space product, Green columns shared by
// the rows ky and Ny - ky): staged spectra, all even/odd in y, kz-innermost output; batched
// members (blockIdx.y) may carry their own spectra g_bstride elements apart.
template <typename T> inline bool zconv_pair_can(const ZConvArgs &a) {
    if (a.nout < 1 || a.nsum > 0 || a.out_estride != 1) return false;
    for (int o = 0; o < a.nout; ++o)
        if (a.gdir[o] < 0 || !a.g[a.gdir[o]].sym_y) return false;
    return zconv_img_smem<T>(a.p.L, a.nout, a.g[a.gdir[0]].zpitch, 0) <= 200 * 1024;
}
template <typename T, bool IMG, int L, int... Rs>
inline int launch_zconv_img(WarpFft<L, Rs...>, const cplx<T> *in, cplx<T> *out, const ZConvArgs &a,
                            const TwPair<cplx<T>> &tw, cudaStream_t st) {
    const size_t sm = zconv_img_smem<T>(L, a.nout, a.g[a.gdir[0]].zpitch, IMG ? a.g[a.gimg[0]].zpitch : 0);
    auto kern = k_zconv_img<T, IMG, L, Rs...>;
    int rc = set_smem(kern, sm);
    if (rc) return rc;
    const int nkp = (a.nxh + 1) / 2;
    const dim3 grid((unsigned)(nkp * (a.ny + 1)), (unsigned)(a.nbatch > 0 ? a.nbatch : 1));
    kern<<<grid, ZI_WARPS * 32, sm, st>>>(in, out, a, tw.wt);
    return launch_ok();
}

inline int launch_zconv_w512(const float2 *in, float2 *out, const ZConvArgs &a, const float2 *rt, cudaStream_t st) {
    constexpr int W = 4;
    const size_t sm = zconv_w512_smem<W>(a.nout, a.g[0].zpitch);
    auto kern = k_zconv_w512<W>;
    int rc = set_smem(kern, sm);
    if (rc) return rc;
    const dim3 grid((unsigned)ceil_div(a.ncols, W), (unsigned)(a.nbatch > 0 ? a.nbatch : 1));
    kern<<<grid, W * 32, sm, st>>>(in, out, a, rt);
    return launch_ok();
}

template <typename T>
int launch_zconv(const cplx<T> *in, cplx<T> *out, const ZConvArgs &a, const TwPair<cplx<T>> &tw, int nl,
                 cudaStream_t st) {
    const int L = a.p.L;
    // a column range of a z slab (col_base > 0) runs on the radix warp engine only
    if (a.col_base != 0 && (!zconv_warp_ok(L, a.nz, (int)sizeof(T)) || a.nsum > 0)) return OSC_E_UNSUPPORTED;
    if (zconv_warp_ok(L, a.nz, (int)sizeof(T))) {
        for (int i = 0; i < a.ng; ++i)
            if (!a.g[i].zinner) return OSC_E_INVALID;  // spectra stored for the other z pass
        bool img = false, herm = false;
        for (int o = 0; o < a.nout; ++o) {
            img |= a.gimg[o] >= 0;
            herm |= a.gimg[o] >= 0 && a.g[a.gimg[o]].herm_img;
        }
        if (tw.wt == tw.rt) return OSC_E_INVALID;
        if (herm) {  // image spectra stored for the image z pass: no other kernel reads them
            if (a.col_base != 0 || !zconv_img_ok(L, a.nz, (int)sizeof(T)) || !zconv_img_can<T>(a))
                return OSC_E_INVALID;
            return dispatch_warp_len(L, [&](auto eng) -> int {
                using E = decltype(eng);
                if constexpr (E::kLen > 0) {
                    constexpr int nb = E::kLen / E::kRad[0];
                    if constexpr (nb % 32 == 0 || nb < 32) return launch_zconv_img<T, true>(eng, in, out, a, tw, st);
                }
                return OSC_E_INVALID;
            });
        }
        const bool staged = !img && zconv_can_stage<T>(a);
        if (a.nsum > 0 && (img || !staged || a.nout != 1)) return OSC_E_UNSUPPORTED;
        if constexpr (sizeof(T) == 4) {
            if (L == 512 && staged && a.nsum == 0 && a.out_estride == 1 && a.engine == 1 && a.col_base == 0 &&
                zconv_w512_smem<4>(a.nout, a.g[0].zpitch) <= 100 * 1024)
                return launch_zconv_w512(in, out, a, tw.rt, st);
        }
        // engine 2: the staged product with Green columns shared by the rows ky and Ny - ky
        const bool pair = staged && a.engine == 2 && a.col_base == 0 && zconv_img_ok(L, a.nz, (int)sizeof(T)) &&
                          zconv_pair_can<T>(a);
        return dispatch_warp_len(L, [&](auto eng) -> int {
            using E = decltype(eng);
            if constexpr (E::kLen > 0) {
                constexpr int nb = E::kLen / E::kRad[0];
                if constexpr (nb % 32 == 0 || nb < 32)
                    if (pair) return launch_zconv_img<T, false>(eng, in, out, a, tw, st);
                if (a.nsum > 0) return launch_zconv_warp<T, ZW_SUM>(eng, in, out, a, tw, st);
                if (img) return launch_zconv_warp<T, ZW_IMAGE>(eng, in, out, a, tw, st);
                if (staged) return launch_zconv_warp<T, ZW_STAGED>(eng, in, out, a, tw, st);
                return launch_zconv_warp<T, ZW_DIRECT>(eng, in, out, a, tw, st);
            }
            return OSC_E_INVALID;
        });
    }
    if (a.nsum > 0) return OSC_E_UNSUPPORTED;  // summed inputs: warp engine lengths only
    for (int i = 0; i < a.ng; ++i)
        if (a.g[i].zinner) return OSC_E_INVALID;
    return dispatch_fft_len<T>(L, [&](auto eng) -> int {
        using E = decltype(eng);
        const cplx<T> *twe = eng_tw<E>(tw);
        return with_nl<T, E>(L, 2, sizeof(T) == 4 ? 8 : 4, nl, [&](auto nlc) -> int {
            constexpr int NL = decltype(nlc)::value;
            const int nt = fft_threads(L, NL, E::kEPT);
            if (nt < 1 || nt > E::kMaxThreads || (L * NL) % E::kEPT) return OSC_E_FFT_SIZE;
            const size_t sm = sizeof(cplx<T>) * ((size_t)L + 2 * (size_t)L * (NL + 1));
            const dim3 nblk((unsigned)ceil_div(a.ncols, NL), (unsigned)(a.nbatch > 0 ? a.nbatch : 1));
            if (E::kLen > 0 && 2 * a.nz == L) {
                auto kern = k_zconv<T, NL, E, true>;
                int rc = set_smem(kern, sm);
                if (rc) return rc;
                kern<<<nblk, nt, sm, st>>>(in, out, a, twe, tw.rt);
            } else {
                auto kern = k_zconv<T, NL, E, false>;
                int rc = set_smem(kern, sm);
                if (rc) return rc;
                kern<<<nblk, nt, sm, st>>>(in, out, a, twe, tw.rt);
            }
            return launch_ok();
        });
    });
}

template <typename TC, typename TI, typename TO>
int launch_sym_lines(const TI *in, TO *out, const SymArgs &a, const TwPair<cplx<TC>> &tw, bool row_load,
                     bool k_fast_store, cudaStream_t st) {
    const int L = a.p.L;
    if (L != 2 * a.n) return OSC_E_INVALID;
    return dispatch_fft_len<TC>(L, [&](auto eng) -> int {
        using E = decltype(eng);
        const cplx<TC> *twe = eng_tw<E>(tw);
        // static engines: up to 16 line pairs per CTA, so the short lines of small batch
        // groups still give CTAs of several warps
        auto with_sym_nl = [&](auto &&f) -> int {
            if constexpr (E::kLen > 0) {
                constexpr int NL1 = nl_static(E::kLen, 16, (int)sizeof(cplx<TC>), 1, 100 * 1024, E::kEPT);
                // the autotuner's alternative tiles: a half or a quarter of the line pairs per
                // CTA (more CTAs for grids whose line count fills barely more than one wave)
                constexpr int NL2 = NL1 >= 4 && (E::kLen * (NL1 / 2)) % E::kEPT == 0 ? NL1 / 2 : NL1;
                constexpr int NL4 = NL2 >= 4 && (E::kLen * (NL2 / 2)) % E::kEPT == 0 ? NL2 / 2 : NL2;
                if (a.nl_div == 4 && NL4 != NL1) return f(std::integral_constant<int, NL4>{});
                if (a.nl_div >= 2 && NL2 != NL1) return f(std::integral_constant<int, NL2>{});
                return f(std::integral_constant<int, NL1>{});
            } else {
                return with_nl<TC, E>(L, 1, 8, 0, f);
            }
        };
        return with_sym_nl([&](auto nlc) -> int {
            constexpr int NL = decltype(nlc)::value;
            const int nt = fft_threads(L, NL, E::kEPT);
            if (nt < 1 || nt > E::kMaxThreads || (L * NL) % E::kEPT) return OSC_E_FFT_SIZE;
            const size_t sm = sizeof(cplx<TC>) * ((size_t)L + (size_t)L * (NL + 1));
            const unsigned nblk = (unsigned)ceil_div(a.nlines, 2 * NL);
            auto go = [&](auto kern) -> int {
                int rc = set_smem(kern, sm);
                if (rc) return rc;
                kern<<<nblk, nt, sm, st>>>(in, out, a, twe);
                return launch_ok();
            };
            if (row_load) return k_fast_store ? go(k_sym_lines<TC, TI, TO, NL, E, true, true>)
                                              : go(k_sym_lines<TC, TI, TO, NL, E, true, false>);
            return k_fast_store ? go(k_sym_lines<TC, TI, TO, NL, E, false, true>)
                                : go(k_sym_lines<TC, TI, TO, NL, E, false, false>);
        });
    });
}

}  // namespace osc
