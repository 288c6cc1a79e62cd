/*
 * opensc_gpu.h -- C ABI of the B200 space-charge library (libopensc_b200.so).
 *
 * Each entry point replaces one routine of OpenSpaceCharge's Fortran module API
 * (RobertRyne/OpenSpaceCharge, code/open_spacecharge_mod.f90 and
 * code/open_spacecharge_core_mod.f90); the routine it replaces is cited above it.  The
 * Fortran host binds these with iso_c_binding (fortran/open_spacecharge_mod.f90).
 *
 * Conventions
 *   - Every function returns an int status: OSC_OK (0) or an OSC_E_* code.  Nothing exits,
 *     aborts or traps; osc_last_error() gives a message for the last failure on a context.
 *   - Grids are Fortran column-major, x fastest: a(i,j,k) at i + nx*(j + ny*k).  Field
 *     grids are [3][nz][ny][nx] (efield(:,:,:,1:3), component slowest).  Particle fields
 *     are [np][3] (a Fortran E(3,np) array).
 *   - Host-pointer entry points take REAL64 host arrays, like the Fortran module; *_dev
 *     entry points take device pointers and do no host<->device copies.
 *   - A context owns one CUDA stream, its workspaces and the Green-spectrum cache.  One
 *     context per host thread; calls on one context are serialised by the caller.
 */
#ifndef OPENSC_GPU_H
#define OPENSC_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OSC_API __attribute__((visibility("default")))
#else
#define OSC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define OSC_OK 0
#define OSC_E_INVALID 1     /* bad argument: null pointer, non-positive size, bad enum */
#define OSC_E_BOUNDS 2      /* particles outside the mesh while strict bounds are on */
#define OSC_E_FFT_SIZE 3    /* a doubled grid length is not 2^a 3^b 5^c or exceeds 2048 */
#define OSC_E_ALLOC 4       /* device or pinned-host allocation failed */
#define OSC_E_CUDA 5        /* a CUDA runtime call failed */
#define OSC_E_TIMEOUT 6     /* a bounded device wait gave up */
#define OSC_E_NAN 7         /* non-finite particle coordinate or charge */
#define OSC_E_NOCHARGE 8    /* neither qa nor total_charge given (reference prints, returns) */
#define OSC_E_UNSUPPORTED 9 /* combination the reference rejects (e.g. direct E in a pipe) */
#define OSC_E_STATE 10      /* call order violated (e.g. pipe solve before its Green set) */

/* ---- precision / path ------------------------------------------------------------ */
#define OSC_PREC_FP32 0       /* complex64 convolution, FP64 Green build, cached spectra */
#define OSC_PREC_FP64 1       /* same pipeline in FP64 / complex128 */
#define OSC_PREC_FP64_PLAIN 2 /* the reference algorithm on the GPU in FP64: full complex
                                 zero-padded FFTs, Green function rebuilt on every call */

/* ---- deposition modes ------------------------------------------------------------ */
#define OSC_DEPOSIT_ATOMIC 0        /* floating-point atomics (order-dependent last bits) */
#define OSC_DEPOSIT_DETERMINISTIC 1 /* 64-bit fixed-point atomics: rho bit-identical for any
                                       particle order and run to run */
#define OSC_DEPOSIT_SORTED_SEGMENT 2 /* the same bits as OSC_DEPOSIT_DETERMINISTIC from particles
                                        in cell order (sorted by the call unless
                                        OSC_OPT_PARTICLE_ORDER says they already are): each
                                        run of particles in one cell is summed exactly in
                                        64-bit integers before its eight reductions */

/* ---- particle order (OSC_OPT_PARTICLE_ORDER) ------------------------------------------
 * The reference deposits and gathers in the caller's particle order.  On the GPU, particles
 * in cell order (sorted by the cell osc_sort_particles_dev uses) share their CIC stencils'
 * memory transactions.  Results are the same for every setting up to FP32 rounding (and
 * bit-identical in the fixed-point deposit modes). */
#define OSC_ORDER_ANY 0         /* any order: one set of reductions and gathers per particle */
#define OSC_ORDER_CELL_SORTED 1 /* the caller's particles are in cell order (e.g. kept sorted
                                   by osc_sort_particles_dev between tracking steps): deposits
                                   sum runs of equal cells before reducing; still correct if
                                   the order is not sorted, only slower */
#define OSC_ORDER_SORT 2        /* the FP32 step sorts a copy of the particles by cell,
                                   deposits and gathers in that order, and returns E (and B)
                                   in the caller's order */

/* ---- context options (osc_ctx_set_option) ---------------------------------------- */
#define OSC_OPT_PRECISION 1      /* default precision for host entry points */
#define OSC_OPT_DEPOSIT_MODE 2   /* OSC_DEPOSIT_* */
#define OSC_OPT_STRICT_BOUNDS 3  /* 1: out-of-mesh particles make deposit return OSC_E_BOUNDS */
#define OSC_OPT_GREEN_CACHE_MB 4 /* byte budget of the Green-spectrum cache (default 4096); 0
                                    rebuilds the spectra on every solve, as the reference does */
#define OSC_OPT_PROFILE 5        /* 1: time every kernel with CUDA events (osc_profile_*) */
#define OSC_OPT_CHECK_FINITE 6   /* 1: deposit rejects non-finite coordinates (OSC_E_NAN) */
#define OSC_OPT_PARTICLE_ORDER 8 /* OSC_ORDER_* (default OSC_ORDER_ANY) */
#define OSC_OPT_TEST_WAIT_TIMEOUT 7 /* test only, 1: the z pass arms its Green-column barrier
                                       but issues no bulk copy and polls 64 times, so its
                                       bounded wait gives up; the call returns OSC_E_TIMEOUT
                                       and the context stays usable */
#define OSC_OPT_BATCH_GRAPH 9    /* 1 (default): an FP32 batched step whose call signature
                                    repeats runs as one CUDA graph launch (0: direct launches) */
#define OSC_OPT_VJP_REUSE_FORWARD 10 /* 1: osc_space_charge_step_vjp_dev (FP32) takes E on the
                                        grid from the last osc_space_charge_step_dev (FP32) of
                                        this context instead of depositing and solving again,
                                        when that step had the same mesh, particle and charge
                                        arrays and particle count and no other step ran since;
                                        the caller guarantees the arrays' contents did not
                                        change in between (0, the default: always recompute) */

typedef struct osc_ctx osc_ctx;

/* Scalar members of mesh3d_struct (code/open_spacecharge_mod.f90:14-27), laid out so a
 * Fortran bind(C) derived type with the same members maps onto it. */
typedef struct osc_mesh3d {
    int32_t nlo[3];    /* lowest grid index per axis (Fortran lbound) */
    int32_t nhi[3];    /* highest grid index per axis */
    int32_t npad[3];   /* padding of the legacy cyclic convolution */
    double min[3];     /* grid origin (m) */
    double max[3];     /* grid end (m) */
    double delta[3];   /* grid spacing (m) */
    double gamma;      /* relativistic gamma */
    double charge;     /* total charge on the mesh (C) */
} osc_mesh3d;

/* ---- context ------------------------------------------------------------------------
 * No reference counterpart: the reference keeps module-global Green arrays
 * (code/open_spacecharge_core_mod.f90:22-23) and is not re-entrant. */
OSC_API int osc_ctx_create(int device, osc_ctx **out);
OSC_API int osc_ctx_destroy(osc_ctx *ctx);
OSC_API const char *osc_last_error(const osc_ctx *ctx);
/* cuda_stream is a cudaStream_t; NULL is CUDA's default stream, as everywhere in CUDA, and
   OSC_OWN_STREAM selects the context's own (non-blocking) stream, the initial one.  Work
   issued on the new stream waits (on the device) for all work issued on the previous one. */
#define OSC_OWN_STREAM ((void *)-1)
OSC_API int osc_ctx_set_stream(osc_ctx *ctx, void *cuda_stream);
OSC_API int osc_ctx_set_option(osc_ctx *ctx, int option, int64_t value);
OSC_API int osc_ctx_get_option(osc_ctx *ctx, int option, int64_t *value);
OSC_API int osc_ctx_synchronize(osc_ctx *ctx);
/* Launch shapes chosen by an autotuner (openspacecharge_b200.autotune times the candidates
 * on the GPU and keeps the winners in a JSON cache keyed by GPU, kernel and length); no
 * reference counterpart.  Keys and values (0 restores the built-in default):
 *   "deposit_run", "gather_run": particles per lane of the cell-ordered deposit and gather
 *     (4 or 8);
 *   "deposit_ctas_per_sm", "gather_ctas_per_sm", "deposit_runs_ctas_per_sm",
 *   "gather_runs_ctas_per_sm": grid size of the per-particle and run kernels, CTAs per SM
 *     (4, 8, 16, 32, 64 or 128);
 *   "lines_nl_div:<f32|f64>:L<length>": 2 halves the lines per CTA of the y transforms of
 *     that doubled length; "r2c_nl_div:..." and "c2r_nl_div:..." the rows per CTA of the
 *     forward and inverse x transforms;
 *   "zconv_engine:<f32|f64>:L<length>": the free-space z pass of that doubled z length on
 *     the radix warp engine (0), the one-exchange 16 x 32 engine (1, FP32 length 512 only),
 *     or the warp engine with CTAs that pair the rows ky and Ny - ky and fetch their common
 *     Green columns once (2);
 *   "batch_copy_chunks": chunks of bunches the FP32 osc_batch_space_charge_step (host
 *     arrays) copies in, solves and copies out in a pipeline (1 to 16; 1: one copy in, one
 *     batched step, one copy out);
 *   "sym_nl_div:<f32|f64>:L<length>": 2 or 4 divides the line pairs per CTA of the Green
 *     build's even/odd line transforms of that doubled length.
 * Results are identical for every choice; only the time changes. */
OSC_API int osc_ctx_set_tuning(osc_ctx *ctx, const char *key, int value);
OSC_API int osc_ctx_get_tuning(osc_ctx *ctx, const char *key, int *value);
OSC_API int osc_clear_green_cache(osc_ctx *ctx);
OSC_API const char *osc_version(void);
/* Kernel profile (OSC_OPT_PROFILE=1): per kernel name, launches and summed ms. */
OSC_API int osc_profile_reset(osc_ctx *ctx);
OSC_API int osc_profile_count(osc_ctx *ctx, int *n);
OSC_API int osc_profile_entry(osc_ctx *ctx, int i, const char **name, int64_t *launches, double *ms);
/* Number of kernels this library launched on the context since creation. */
OSC_API int osc_launch_count(osc_ctx *ctx, int64_t *n);
/* Batched steps of this context that ran as one CUDA graph launch (OSC_OPT_BATCH_GRAPH). */
OSC_API int osc_graph_launch_count(osc_ctx *ctx, int64_t *n);

/* ---- deposition -------------------------------------------------------------------
 * Replaces deposit_particles (code/open_spacecharge_mod.f90:156-288).  qa may be NULL, then
 * total_charge must be non-NULL (else OSC_E_NOCHARGE, rho untouched, like the reference's
 * print-and-return).  resize_mesh != 0 refits min/max/delta to the bunch with the
 * reference's 1e-6*delta padding.  mesh->charge is set.  rho is [nz][ny][nx] REAL64.
 * Particles whose 2x2x2 stencil leaves the mesh are skipped and counted in *n_outside
 * (the reference writes out of bounds there). */
OSC_API int osc_deposit_particles(osc_ctx *ctx, int64_t np, const double *xa, const double *ya,
                          const double *za, const double *qa, const double *total_charge,
                          int resize_mesh, osc_mesh3d *mesh, double *rho, int64_t *n_outside);
OSC_API int osc_deposit_particles_dev(osc_ctx *ctx, int64_t np, const double *d_x, const double *d_y,
                              const double *d_z, const double *d_q, const double *total_charge,
                              int resize_mesh, osc_mesh3d *mesh, double *d_rho,
                              int64_t *n_outside);

/* No counterpart in the reference.  Charge deposition for callers that may not allocate
 * device memory (inside another framework's memory pool, in loops that cannot absorb the
 * synchronisation of cudaMalloc/cudaFree, or without a library context, whose creation
 * allocates).  It needs no context and allocates nothing: the caller passes a stream, the
 * mesh and device buffers; the deposit accumulates in FP32 in a fixed array compiled into
 * the library (OSC_NOALLOC_MAX_NODES floats, 16 MiB, held on every GPU that loads the
 * library until the process exits) and writes REAL64 rho.  Meshes with more nodes are
 * rejected with OSC_E_INVALID (the node count is formed in 64-bit arithmetic and checked
 * after every factor, so no mesh can wrap it).  Charges are d_q per particle, or
 * total_charge/np when d_q is NULL.  With d_q NULL a zero total_charge stands for the
 * reference's missing charge ("must specify qa or total_charge"): OSC_E_NOCHARGE, rho
 * untouched; a non-finite total_charge is OSC_E_INVALID.  The mesh is not refitted and mesh->charge is not
 * touched.  *n_outside counts particles outside the mesh plus particles with a non-finite
 * coordinate, the count osc_deposit_particles_dev reports with its default options.  The
 * first call in a CUDA context (normally once per device) looks up the array's device
 * address (make that first call before any stream capture); cudaDeviceReset invalidates
 * it.  All calls share the one array, so calls whose work overlaps on the GPU race.
 * errbuf (optional, errlen bytes) receives a message. */
#define OSC_NOALLOC_MAX_NODES 4194304
OSC_API int osc_deposit_particles_dev_noalloc(void *cuda_stream, const osc_mesh3d *mesh, int64_t np,
                                              const double *d_x, const double *d_y, const double *d_z,
                                              const double *d_q, double total_charge, double *d_rho,
                                              int64_t *n_outside, char *errbuf, size_t errlen);

/* No counterpart in the reference (it deposits in the caller's order,
 * code/open_spacecharge_mod.f90:257-283).  Counting sort of the particles by deposit cell:
 * the key of a particle is the linear index i + nx*(j + ny*k) of its cell's lowest corner
 * under deposit_particles' formula (the cell osc_deposit_particles uses); particles whose
 * stencil leaves the mesh or with a non-finite coordinate go last.  Within a cell the order
 * is unspecified.  Writes the sorted copies xs, ys, zs (and qs when q is given; q and qs
 * are both NULL or both set; no output may alias an input) and, when perm is non-NULL,
 * perm[s] = the original index of sorted particle s, so a tracking code can apply the same
 * permutation to its other particle arrays.  *n_outside (optional) counts the particles
 * sorted last.  Device pointers; np < 2^32 - 1. */
OSC_API int osc_sort_particles_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int64_t np, const double *d_x,
                                   const double *d_y, const double *d_z, const double *d_q, double *d_xs,
                                   double *d_ys, double *d_zs, double *d_qs, int64_t *d_perm, int64_t *n_outside);

/* Replaces get_mesh_quantities (code/test_mod.f90:288-358), the test-path mesh rule:
 * delta=(max-min)/(n-3), min=bunch_min-delta; isetzmin=1 pins zmin=1e-9 for cathodes. */
OSC_API int osc_get_mesh_quantities(osc_ctx *ctx, int64_t np, const double *xa, const double *ya,
                            const double *za, const int32_t nlo[3], const int32_t nhi[3],
                            int isetzmin, double delta[3], double umin[3]);
/* Replaces depose_rho_scalar (code/test_mod.f90:410-474).  lostflag may be NULL; rho is
 * scaled by chrgpermacro; *ifail counts skipped (out-of-mesh) particles. */
OSC_API int osc_depose_rho_scalar(osc_ctx *ctx, int64_t np, const double *xa, const double *ya,
                          const double *za, const double *lostflag, double chrgpermacro,
                          const int32_t nlo[3], const int32_t nhi[3], const double delta[3],
                          const double umin[3], double *rho, int64_t *ifail);

/* ---- field solves ------------------------------------------------------------------
 * Replaces space_charge_3d (code/open_spacecharge_mod.f90:431-489): IGF free-space field
 * (and the cathode image when at_cathode != 0), optional B.  offset may be NULL. */
OSC_API int osc_space_charge_3d(osc_ctx *ctx, const osc_mesh3d *mesh, const double *rho,
                        const double *offset, int at_cathode, int calc_bfield, int precision,
                        double *efield, double *bfield);
OSC_API int osc_space_charge_3d_dev(osc_ctx *ctx, const osc_mesh3d *mesh, const double *d_rho,
                            const double *offset, int at_cathode, int calc_bfield,
                            int precision, double *d_efield, double *d_bfield);
/* Replaces osc_freespace_solver2 (code/open_spacecharge_mod.f90:535-597); phi (the
 * icomp=0 branch) and efield are each optional (NULL). */
OSC_API int osc_freespace_solver2(osc_ctx *ctx, const int32_t n[3], const double *rho, double gamma,
                          const double delta[3], const double *offset, int precision,
                          double *efield, double *phi);
/* Replaces space_charge_freespace (code/open_spacecharge_mod.f90:60-75), which runs the
 * legacy osc_freespace_solver (code/open_spacecharge_core_mod.f90:30-138). */
OSC_API int osc_space_charge_freespace(osc_ctx *ctx, const osc_mesh3d *mesh, const double *rho,
                               int direct_field_calc, int integrated_green_function,
                               int precision, double *phi, double *efield, double *bfield);
/* Replaces space_charge_cathodeimages (code/open_spacecharge_mod.f90:83-103) ->
 * osc_cathodeimages_solver (code/open_spacecharge_core_mod.f90:905-1083).  image_method 1
 * (convolution/correlation) or 2 (shifted Green function).  Method 2 leaves rho flipped in
 * z on return, as the reference does. */
OSC_API int osc_space_charge_cathodeimages(osc_ctx *ctx, const osc_mesh3d *mesh, double *rho,
                                   int direct_field_calc, int integrated_green_function,
                                   int image_method, int precision, double *phi,
                                   double *efield, double *bfield);

/* ---- rectangular pipe ----------------------------------------------------------------
 * Replaces osc_alloc_rectpipe_arrays + osc_getgrnpipe (code/open_spacecharge_core_mod.f90:
 * 876-898, 632-715): builds and caches the four transformed pipe Green arrays on the
 * context (the reference's module-global cgrn1..4).  umin is the mesh origin. */
OSC_API int osc_rectpipe_green(osc_ctx *ctx, const osc_mesh3d *mesh, double apipe, double bpipe,
                       int precision);
/* Replaces space_charge_rectpipe (code/open_spacecharge_mod.f90:110-127) ->
 * osc_rectpipe_solver (core:536-624).  direct_field_calc must be 0 (the reference prints
 * an error otherwise: OSC_E_UNSUPPORTED).  Needs osc_rectpipe_green first (OSC_E_STATE). */
OSC_API int osc_space_charge_rectpipe(osc_ctx *ctx, const osc_mesh3d *mesh, const double *rho,
                              double apipe, double bpipe, int direct_field_calc,
                              int integrated_green_function, int precision, double *phi,
                              double *efield, double *bfield);
/* Device pointers, asynchronous on the context stream; otherwise as above. */
OSC_API int osc_space_charge_rectpipe_dev(osc_ctx *ctx, const osc_mesh3d *mesh, const double *d_rho,
                                          double apipe, double bpipe, int direct_field_calc,
                                          int integrated_green_function, int precision, double *d_phi,
                                          double *d_efield, double *d_bfield);
/* Fused step in the pipe (device pointers): deposit of the np particles (charges q, or
 * total_charge/np each), pipe potential and its finite-difference E and B
 * (space_charge_rectpipe with direct_field_calc = 0) and the gather of E (and B when B is
 * non-NULL) at every particle, as the reference's test program does with
 * depose_rho_scalar, space_charge_rectpipe and interpolate_field (code/test_opensc.f90:156,
 * :203-216, :247).  The mesh is used as given (the pipe mesh spans the walls) and needs its
 * Green spectra first (osc_rectpipe_green or osc_read_rectpipe_grn).  E, B are [np][3]. */
OSC_API int osc_space_charge_step_rectpipe_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int64_t np, const double *d_x,
                                               const double *d_y, const double *d_z, const double *d_q,
                                               const double *total_charge, double apipe, double bpipe,
                                               int precision, double *d_E, double *d_B);
/* Replace osc_write_rectpipe_grn / osc_read_rectpipe_grn (core:825-870): a header record
 * and cgrn1..4 as complex128, Fortran unformatted sequential layout. */
OSC_API int osc_write_rectpipe_grn(osc_ctx *ctx, const char *path, double apipe, double bpipe,
                           const osc_mesh3d *mesh);
OSC_API int osc_read_rectpipe_grn(osc_ctx *ctx, const char *path, const osc_mesh3d *mesh,
                          double *apipe, double *bpipe);

/* ---- interpolation -------------------------------------------------------------------
 * Replaces interpolate_field (code/open_spacecharge_mod.f90:311-390), batched over np
 * points.  efield/bfield are grids ([3][nz][ny][nx]); either may be NULL together with
 * its output.  E and B are [np][3].  Out-of-range points are clamped to cells [1,nhi-1]
 * as in the reference and counted in *n_clamped (the reference prints them). */
OSC_API int osc_interpolate_field(osc_ctx *ctx, const osc_mesh3d *mesh, const double *efield,
                          const double *bfield, int64_t np, const double *x, const double *y,
                          const double *z, double *E, double *B, int64_t *n_clamped);
OSC_API int osc_interpolate_field_dev(osc_ctx *ctx, const osc_mesh3d *mesh, const double *d_efield,
                              const double *d_bfield, int64_t np, const double *d_x,
                              const double *d_y, const double *d_z, double *d_E, double *d_B,
                              int64_t *n_clamped);

/* ---- fused step ------------------------------------------------------------------------
 * deposit_particles + space_charge_3d + interpolate_field at every particle in one call
 * (code/test_opensc.f90:156-228 does the same three steps).  Host buffers; *_dev takes
 * device pointers.  If resize_mesh is 0 the mesh geometry is used as given and the Green
 * spectrum is reused from the cache.  E is [np][3]; B may be NULL. */
OSC_API int osc_space_charge_step(osc_ctx *ctx, osc_mesh3d *mesh, int64_t np, const double *x,
                          const double *y, const double *z, const double *q,
                          const double *total_charge, int resize_mesh, int at_cathode,
                          int precision, double *E, double *B);
OSC_API int osc_space_charge_step_dev(osc_ctx *ctx, osc_mesh3d *mesh, int64_t np, const double *d_x,
                              const double *d_y, const double *d_z, const double *d_q,
                              const double *total_charge, int resize_mesh, int at_cathode,
                              int precision, double *d_E, double *d_B);

/* ---- line-out and plane files ---------------------------------------------------------
 * Replace write_lines / write_plane of the reference's test program
 * (code/test_opensc.f90:237-295): x_lineout.dat, y_lineout.dat, z_lineout.dat (x y z Ex Ey
 * Ez, Fortran '(6(1pe14.7,1x))', points (i-1)*delta+min for i = nlo..nhi-1 along one axis
 * through (xcent, ycent, zcent)) and x_z_Ex_Ez_By.dat (x z Ex Ez By, list-directed, plane
 * y = 0), written into dir (NULL or "": the working directory).  efield/bfield are host
 * grids [3][nz][ny][nx].  osc_format_1pe14_7 writes one value as Fortran 1PE14.7 (14
 * characters and a terminating NUL into out15). */
OSC_API int osc_write_lines(osc_ctx *ctx, const osc_mesh3d *mesh, const double *efield, double xcent,
                            double ycent, double zcent, const char *dir);
OSC_API int osc_write_plane(osc_ctx *ctx, const osc_mesh3d *mesh, const double *efield, const double *bfield,
                            const char *dir);
OSC_API int osc_format_1pe14_7(double v, char *out15);

/* ---- adjoint of the step ---------------------------------------------------------------
 * Vector-Jacobian product of the fused step with the mesh held fixed: given gE = dL/dE at
 * every particle ([np][3]), returns dL/dx, dL/dy, dL/dz and (gq non-NULL) dL/dq per
 * particle.  Charges are q, or total_charge/np each when q is NULL.  Device pointers.
 * OSC_PREC_FP32 runs the field solves in FP32, the other precisions in FP64; the
 * deposits and gathers are FP64.  The reference has no adjoint: this is the backward pass
 * behind a differentiable (torch.autograd) step. */
OSC_API int osc_space_charge_step_vjp_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int64_t np, const double *d_x,
                                          const double *d_y, const double *d_z, const double *d_q,
                                          double total_charge, int precision, const double *d_gE, double *d_gx,
                                          double *d_gy, double *d_gz, double *d_gq);

/* ---- batched steps ---------------------------------------------------------------------
 * Many independent bunches, each with its own mesh, in one call: the fused step above for
 * every bunch (free space, no cathode image, E only).  The reference solves one bunch per
 * call (space_charge_3d, code/open_spacecharge_mod.f90:431-489, called from
 * code/test_opensc.f90:184); a tracking code with many bunches calls it in a loop, which
 * this replaces.  Particles of all bunches are concatenated: bunch b owns entries
 * [offset, offset + np) of x, y, z, q and of the rows of E ([total][3]).  With resize_mesh
 * each bunch's mesh is refit to its particles as deposit_particles does; the Green
 * spectra are rebuilt for every bunch on every call (meshes change between steps).
 * OSC_PREC_FP32 runs all bunches through batched kernels, grouped by grid shape; the
 * FP64 precisions solve the bunches one after another. */
typedef struct osc_bunch {
    osc_mesh3d mesh;      /* in: nlo, nhi, gamma (+ min, max, delta without resize);
                             out: fitted geometry and charge */
    int64_t offset;       /* first particle of this bunch in the concatenated arrays */
    int64_t np;           /* particles of this bunch (>= 1) */
    double total_charge;  /* charge of the bunch when q is NULL */
    int64_t n_outside;    /* out: particles outside the mesh (not deposited) */
} osc_bunch;

OSC_API int osc_batch_space_charge_step(osc_ctx *ctx, int nbunch, osc_bunch *bunches, const double *x,
                                        const double *y, const double *z, const double *q, int resize_mesh,
                                        int precision, double *E);
OSC_API int osc_batch_space_charge_step_dev(osc_ctx *ctx, int nbunch, osc_bunch *bunches, const double *d_x,
                                            const double *d_y, const double *d_z, const double *d_q,
                                            int resize_mesh, int precision, double *d_E);

/* ---- one grid over several GPUs by z slabs (FP32) -------------------------------------
 * Replaces, for grids that outgrow one GPU, the reference's multi-rank prototype, which
 * moves the doubled grid between rank layouts with MPI all-to-alls
 * (mpi_devel/code/open_spacecharge_mod.f90:722-990).  Rank r of P keeps the z planes
 * [z0, z0 + nzl) of the nx x ny x nz grid (0-based, the mesh's planes nlo[2] + z0 ...) and
 * the half-spectrum columns [col0, col0 + ncols) (column ky*(nx+1) + kx, ky < 2ny,
 * kx <= nx); the caller makes the exchanges between the stages (openspacecharge_b200/
 * slab.py does them with torch.distributed over NCCL):
 *  1. osc_slab_deposit_dev: the rank's particles (each with its deposit cell in
 *     [z0, z0 + nzl), see below) into a quad grid of nzl + 1 planes (float4 per node, 16
 *     bytes; zeroed first).  Its last plane belongs to the next rank: add it into that
 *     rank's plane 0 (the halo sum; the top slab leaves it zero).  q NULL: charge1 per
 *     particle (the total charge over the particles of all ranks).  *n_outside (optional,
 *     synchronises) counts this rank's particles outside the mesh or non-finite.
 *  2. osc_slab_forward_dev: x and y transforms of the nzl planes of the quad grid into X2,
 *     complex64 [nzl][2ny][nx+1].
 *  3. all-to-all: rank s gets, from every rank, the columns [col0_s, col0_s + ncols_s) of
 *     its planes, assembled as in[nz][ncols_s] (planes in global order).
 *  4. osc_slab_zpass_dev: the z pass of the rank's columns: out[3][ncols][nz] (complex64,
 *     the E components, kz innermost), with the Green spectra of the whole grid (built
 *     once per geometry on every rank, cached); doubled z lengths of the warp engine only
 *     (96, 128, 192, 256, 384, 512).
 *  5. all-to-all back: rank s gets out[c][col][z0_s .. z0_s + nzl_s) of every rank's
 *     columns, assembled as X3[3][2ny][nx+1][nzl_s].
 *  6. osc_slab_inverse_dev: inverse y and x transforms into the rank's x-pair E grid,
 *     float4 [nzl][ny][nx][2] (32 bytes per node).
 *  7. halo: the gather reads planes z0 - 1 (from the previous rank) to z0 + nzl (from the
 *     next); osc_slab_interp_dev gathers E at the rank's particles from an x-pair grid of
 *     the planes [p0, p0 + np_planes).
 * Particle ownership: rank r holds the particles whose deposit cell k = floor((z - zmin) *
 * (1/dz) + 1) - nlo[2] (the deposit's formula) lies in [z0, z0 + nzl), clamped into
 * [0, nz - 2] for particles beyond the mesh (as openspacecharge_b200.slab.owner_of does).
 * The gather's cell can be one lower than the deposit's, hence the plane below the slab.
 * Results equal osc_space_charge_step_dev's FP32 E to FP32 round-off. */
OSC_API int osc_slab_deposit_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int z0, int nzl, int64_t np,
                                 const double *d_x, const double *d_y, const double *d_z, const double *d_q,
                                 double charge1, float *d_quad, int64_t *n_outside);
OSC_API int osc_slab_forward_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int z0, int nzl, const float *d_quad,
                                 void *d_X2);
OSC_API int osc_slab_zpass_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int col0, int ncols, const void *d_in,
                               void *d_out);
OSC_API int osc_slab_inverse_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int z0, int nzl, const void *d_X3,
                                 float *d_e8);
OSC_API int osc_slab_interp_dev(osc_ctx *ctx, const osc_mesh3d *mesh, int p0, int np_planes, int64_t np,
                                const double *d_x, const double *d_y, const double *d_z, const float *d_e8,
                                double *d_E);

#ifdef __cplusplus
}
#endif
#endif /* OPENSC_GPU_H */
