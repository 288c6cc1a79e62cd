// fft_kernels.cuh -- argument blocks and launchers of the FFT-based convolution kernels.
#pragma once

#include "osc_fft.cuh"

namespace osc {

// Generic batched C2C transform of lines along one axis, with zero-padded input window
// [0, in_len) and output window [out_lo, out_lo + out_len).  Element (plane, col, e) sits at
// plane*pstride + col*cstride + e*estride; blockIdx.z selects one of several component
// arrays (zstride apart).  ROW=true: lines are contiguous rows (global accesses walk e);
// ROW=false: lines are adjacent columns (global accesses walk col).
struct LineArgs {
    FFTPlan p;
    int sign;
    int ncols;
    int in_len, out_lo, out_len;
    int64_t in_pstride, in_cstride, in_estride, in_zstride;
    int64_t out_pstride, out_cstride, out_estride, out_zstride;
    double scale;
    unsigned flip_mask;  // bit z: component z stores element (L-e) mod L at e (index flip)
    int nl_div = 0;      // autotuner: 2 halves the lines per CTA of a static engine (0/1: default)
    // > 0: the column tiles run over the flat sequence of flat_lines = ncols * nplanes lines
    // (plane-major), so a tile may end in one plane and continue in the next (column
    // layouts only, needs ncols >= the lines per CTA); 0: one row of tiles per plane
    int flat_lines = 0;
};

// Forward transform of real rows (length nin, zero-padded to L) packed two per complex
// line; writes the L/2+1 non-negative frequencies of every row.
struct R2CArgs {
    FFTPlan p;
    int nin;
    int64_t nrows;
    int64_t in_rstride;   // elements between rows of the real input
    int64_t out_rstride;  // complex elements between output rows
    int qny = 0;          // quad-grid input (float4): rows per plane, for the node sum's y neighbour
    int nl_div = 0;       // autotuner: 2 halves the rows per CTA (0/1: default)
};

// Where the real result of one inverse component goes.
struct OutDest {
    void *ptr;        // nullptr = unused
    int kind;         // 0: slot of a vec4<T> grid, 1: double plane, 2: T plane, 3: add to a double
                      // plane, 4: slot of an x-pair grid (node n holds vec4 E(n), E(n+1))
    int slot;         // vec4 component (kinds 0 and 4)
    int last_x;       // kind 4: the last x index of a row
    double coef;      // multiplier
};
constexpr int MAX_OUT = 6;
constexpr int MAX_DEST = 4;

// Inverse transform of Hermitian rows (L/2+1 stored frequencies) to real rows, keeping
// x in [0, nout), for ncomp component arrays; each component's result goes to up to
// MAX_DEST destinations (grid index = row*nout + x, i.e. [z][y][x]).
struct C2RArgs {
    FFTPlan p;
    int nout;
    int64_t nrows;
    int64_t in_rstride, in_cstride;
    int ncomp;
    unsigned flip_mask;   // bit c: component c is read at x -> (L-x) mod L (index flip)
    void *e8;             // optional x-pair grid vec4<T>[N][2] filled from components e8_comp
    int e8_comp[3];       // components giving (Ex, Ey, Ez) of the x-pair grid
    int e8_node;          // 1: e8 is a plain node grid vec4<T>[N] (Ex, Ey, Ez, 0) instead
    int ndest[MAX_OUT];
    OutDest dest[MAX_OUT][MAX_DEST];
    // zin != 0: the input spectra are kz-innermost, [c][b][y][kx][z] with zin_nz planes per
    // member and zin_ny rows y; row r = (b*ny + y)*nz + z starts at (b*ny + y)*(nx+1)*nz + z
    // with elements nz apart and goes to grid row (b*nz + z)*ny + y ([z][y][x] per member).
    int zin, zin_nz, zin_ny;
    int nl_div;           // autotuner: 2 halves the rows per CTA (0/1: default)
};

// Stored Green spectrum of one kernel component on the half-spectrum grid
// kx in [0, nx], ky in [0, Ny), kz in [0, Nz).  Axes with sym_* hold only k <= n and the
// value at N-k is par_* times the value at k.  real_valued spectra store one T per point
// meaning s (imag_unit=0) or i*s (imag_unit=1); others store cplx<T>.  Layout [kz][ky][kx],
// or [ky][kx][kz] when zinner is set (the layout of the warp-per-column z pass), with
// columns zpitch >= dimz elements apart (a multiple of 16 bytes).
// herm_img marks a cathode-image spectrum in the layout of the image z pass (zconv_img.cuh):
// complex, kz-innermost, kz in [0, Nz/2] only (the value at Nz - kz is par_h times the
// conjugate of the value at kz), the image flip phase -exp(2 pi i (Nz/2 - 1) kz / Nz) applied.
struct GSpecDev {
    const void *data;
    int real_valued, imag_unit;
    int sym_y, sym_z, par_y, par_z;
    int dimy, dimz;
    int zinner, zpitch;
    int herm_img = 0, par_h = 1;
};

// Value of a stored Green spectrum at (kx, ky, kz) of the Nx/2+1 x Ny x Nz half spectrum.
template <typename T>
__device__ __forceinline__ cplx<T> g_lookup(const GSpecDev &g, int kx, int ky, int kz, int nxh,
                                            int Ny, int ny, int Nz, int nz, int64_t goff = 0) {
    int yy = ky, zz = kz;
    bool neg = false;
    if (g.sym_y && ky > ny) { yy = Ny - ky; neg ^= (g.par_y < 0); }
    if (g.sym_z && kz > nz) { zz = Nz - kz; neg ^= (g.par_z < 0); }
    const int64_t idx =
        goff + (g.zinner ? ((int64_t)yy * nxh + kx) * g.zpitch + zz : ((int64_t)zz * g.dimy + yy) * nxh + kx);
    if (g.real_valued) {
        T s = __ldg(reinterpret_cast<const T *>(g.data) + idx);
        if (neg) s = -s;
        return g.imag_unit ? mk<T>(0, s) : mk<T>(s, 0);
    }
    cplx<T> v = __ldg(reinterpret_cast<const cplx<T> *>(g.data) + idx);
    if (neg) { v.x = -v.x; v.y = -v.y; }
    return v;
}

// Fused z pass of the free-space convolution: forward transform of each (kx,ky) column
// (nz non-zero planes, length Nz), multiply by stored Green spectra (optionally adding the
// mirrored-image term), inverse transform, keep z in [0, nz) of every output.
struct ZConvArgs {
    FFTPlan p;       // length Nz
    int nz;
    int ncols;       // (nx+1)*Ny
    int nxh, Ny, ny;
    int64_t in_estride;   // complex elements between z planes of the input (= ncols)
    int64_t out_estride;  // between z planes of the output (1: z-innermost output)
    int64_t out_colstride;  // between (kx,ky) columns of the output (nz when z-innermost)
    int64_t out_cstride;  // between output components
    int nout;
    int gdir[MAX_OUT];    // index into g[] of the direct term (-1 none)
    int gimg[MAX_OUT];    // index into g[] of the image term (-1 none)
    double img_coef[MAX_OUT];
    int img_phase_mul;    // image spectrum = -w^(img_phase_mul*kz) * rho_hat(-kz)
    int ng;
    GSpecDev g[8];
    unsigned *fault;      // host-mapped fault word (bounded waits that gave up), or null
    unsigned poll_limit;  // polls of a bounded mbarrier wait (0: MBAR_POLL_LIMIT)
    int skip_copies;      // test only: arm the Green-column barrier but issue no bulk copy,
                          // so the bounded wait runs out and the fault path is exercised
    int engine;           // FP32 length 512, staged spectra: 0 the radix-8 warp engine, 1 the
                          // one-exchange 16 x 32 engine (autotuner key zconv_engine)
    // batches of equal grids (blockIdx.y = member): input, output and spectrum offsets of
    // member b are b*in_bstride, b*out_bstride and b*g_bstride (elements of the spectrum)
    int nbatch;
    int64_t in_bstride, out_bstride, g_bstride;
    // > 0: the nsum members are the inputs of the single output (warp engine, staged real
    // spectra): out = inverse of sum_s spectrum[gdir[s]] x forward(input s)
    int nsum;
    // global index of local column 0 (a z slab's share of the columns, warp engine 0): the
    // Green spectra are read at column col_base + col, input and output at col
    int col_base;
};

// Transform of real lines that are even (par = +1) or odd (par = -1) about index 0 on the
// period L = 2n, of which only x[0..n) is stored (x[L-a] = par x[a], x[n] = 0): returns the
// real s[k], k in [0, n], with sum_a x[a] exp(+2 pi i a k/L) = s[k] (even) or i s[k] (odd),
// times scale.  Real lines are enumerated as (b, p, q), q fastest (q < nq, p*nq + q < npq);
// line (b, p, q) starts at b*bs + p*ps + q*qs and its elements are es apart, for input and
// output separately.
struct SymArgs {
    FFTPlan p;  // length L = 2n
    int n;
    int odd_lo, odd_hi;  // members b in [odd_lo, odd_hi) are odd (par -1), the others even
    int64_t nlines;
    int nq;
    int64_t in_ps, in_qs, in_es;
    int64_t out_ps, out_qs, out_es;
    double scale;
    // batches: lines of member b are the lines [b*npq, (b+1)*npq), offset by b*in_bs, b*out_bs
    int64_t npq, in_bs, out_bs;
    int nl_div = 0;  // autotuner: 2 or 4 divides the line pairs per CTA of a static engine
};
// row_load: elements of a line are contiguous in the input (load along the line);
// k_fast_store: outputs of a line are contiguous (store along the line).
// TC: arithmetic type of the transform (double, or float from octant values rounded once).
template <typename TC, typename TI, typename TO>
int launch_sym_lines(const TI *in, TO *out, const SymArgs &a, const TwPair<cplx<TC>> &tw, bool row_load,
                     bool k_fast_store, cudaStream_t st);

template <typename T>
int launch_lines(const cplx<T> *in, cplx<T> *out, const LineArgs &a, int nplanes, int ncomp,
                 bool row_mode, const TwPair<cplx<T>> &tw, cudaStream_t st);
template <typename T, typename TIn>
int launch_r2c_rows(const TIn *in, cplx<T> *out, const R2CArgs &a, const TwPair<cplx<T>> &tw, cudaStream_t st);
template <typename T>
int launch_c2r_rows(const cplx<T> *in, const C2RArgs &a, const TwPair<cplx<T>> &tw, cudaStream_t st);
// True when the z pass of length L with nz = L/2 non-zero planes runs the warp-per-column
// kernel, whose Green spectra must be stored with zinner set.
bool zconv_warp_ok(int L, int nz, int elem_bytes);
// True when the cathode-image z pass (zconv_img.cuh) covers length L: the warp-per-column
// lengths whose first-stage butterfly count L/R is a multiple of 32 or below 32.
bool zconv_img_ok(int L, int nz, int elem_bytes);
template <typename T>
int launch_zconv(const cplx<T> *in, cplx<T> *out, const ZConvArgs &a, const TwPair<cplx<T>> &tw,
                 int nl, cudaStream_t st);

}  // namespace osc
