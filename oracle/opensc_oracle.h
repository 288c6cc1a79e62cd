/*
 * opensc_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of OpenSpaceCharge's space-charge path (RobertRyne/OpenSpaceCharge,
 * code/open_spacecharge_mod.f90, code/open_spacecharge_core_mod.f90, code/test_mod.f90,
 * code/fft_interface_mod.f90).  It is the checker for the CUDA product and the timed CPU
 * baseline ("port").  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference leg may load it.  The product library never links it.
 *
 * Parity status: the reference ships no golden vectors and cannot be compiled in this
 * environment (it is Fortran 2008; no Fortran compiler is installed).  The restatement is
 * pinned bit-exactly on get_mesh_quantities against the reference's own printed run output
 * (examples/benchmark.ipynb), and on the field solve only by the notebook's published
 * cathode cross-method differences and by analytic known-answer tests.  The field solve
 * itself is therefore "parity unpinned" by reference data.
 *
 * Conventions (same as the reference):
 *   - 3D arrays are column-major, x fastest: a(i,j,k) at i + n1*(j + n2*k) (0-based here).
 *   - efield/bfield are [3][nz][ny][nx] (component slowest), like efield(:,:,:,3).
 *   - complex arrays are interleaved (re, im) doubles.
 *   - FFT sign s: X[k] = sum_j x[j] exp(s*2*pi*i*j*k/n), unnormalised (Singleton's isn).
 */
#ifndef OPENSC_ORACLE_H
#define OPENSC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scalar members of mesh3d_struct (code/open_spacecharge_mod.f90:14-27). */
typedef struct orc_mesh {
    int nlo[3], nhi[3], npad[3];
    double min[3], max[3], delta[3];
    double gamma, charge;
} orc_mesh;

/* ---- L1: FFT (code/fft_interface_mod.f90:96-143) ---- */
int orc_ccfft3d(double *a, const int idir[3], int n1, int n2, int n3);
int orc_fft_supported(int n);

/* ---- free-space IGF and solver2 (code/open_spacecharge_mod.f90:535-747) ---- */
double orc_lafun2(double x, double y, double z);
double orc_xlafun2(double x, double y, double z);
void orc_get_cgrn_freespace(double *cgrn, int isize, int jsize, int ksize, const double delta[3],
                            double gamma, int icomp, const double *offset);
int orc_freespace_solver2(const double *rho, const int n[3], double gamma, const double delta[3],
                          const double *offset, double *efield, double *phi);
int orc_space_charge_3d(const orc_mesh *mesh, const double *rho, const double *offset,
                        int at_cathode, int calc_bfield, double *efield, double *bfield);

/* ---- deposition / interpolation (code/open_spacecharge_mod.f90:156-390) ---- */
int orc_deposit_particles(int64_t np, const double *xa, const double *ya, const double *za,
                          const double *qa, const double *total_charge, int resize_mesh,
                          orc_mesh *mesh, double *rho, int64_t *n_outside);
int64_t orc_interpolate_field(const orc_mesh *mesh, const double *efield, const double *bfield,
                              int64_t np, const double *x, const double *y, const double *z,
                              double *E, double *B);

/* ---- test-path mesh and deposit (code/test_mod.f90:288-474) ---- */
void orc_getbeamboundingbox(int64_t np, const double *x, const double *y, const double *z,
                            double bb[6]);
void orc_get_mesh_quantities(int64_t np, const double *xa, const double *ya, const double *za,
                             const int nlo[3], const int nhi[3], int isetzmin, double delta[3],
                             double umin[3]);
int64_t orc_depose_rho_scalar(int64_t np, const double *xa, const double *ya, const double *za,
                              const double *lostflag, double *rho, double chrgpermacro,
                              const int nlo[3], const int nhi[3], const double delta[3],
                              const double umin[3], const int nlogbl[3]);

/* ---- legacy free-space solver (code/open_spacecharge_core_mod.f90:30-529) ---- */
int orc_freespace_solver(const double *rho, double gam0, const double delta[3], double *phi,
                         double *efield, double *bfield, const int nlo[3], const int nhi[3],
                         const int npad[3], int idirectfieldcalc, int igfflag);
double orc_igf_point(int icomp, int igfflag, double u, double v, double w, double gam, double dx,
                     double dy, double dz);

/* ---- legacy cathode images, methods 1 and 2 (core:905-1264) ---- */
int orc_cathodeimages_solver(double *rho, double gam0, const double umin[3], const double delta[3],
                             double *phi, double *efield, double *bfield, const int nlo[3],
                             const int nhi[3], const int npad[3], int idirectfieldcalc,
                             int igfflag, int imethod);

/* ---- rectangular pipe (core:536-898) ---- */
double orc_rfun(double u, double v, double w, double gam, double a, double b, double hz, int i,
                int j);
/* Builds the four transformed Green arrays (complex, each prod(2(nhi-nlo)+1+npad)). */
int orc_getgrnpipe(double gam, double a, double b, const double delta[3], const double umin[3],
                   const int nlo[3], const int nhi[3], const int npad[3], double *cgrn1,
                   double *cgrn2, double *cgrn3, double *cgrn4);
int orc_rectpipe_solver(const double *rho, const double *cgrn1, const double *cgrn2,
                        const double *cgrn3, const double *cgrn4, double gam0,
                        const double delta[3], double *phi, double *efield, double *bfield,
                        const int nlo[3], const int nhi[3], const int npad[3],
                        int idirectfieldcalc);

/* Wall-clock helpers for the CPU baseline. */
int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
