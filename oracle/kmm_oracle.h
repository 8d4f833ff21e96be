/*
 * kmm_oracle.h -- CPU restatement of the reference's KMM timestep (TEST INFRASTRUCTURE).
 *
 * This library is the parity checker for the GPU implementation and the timed
 * CPU baseline.  It is NOT part of the product: only tests/, the smoke check and
 * bench.py's cpu_baseline / reference legs load it.
 *
 * It restates, in plain C (FP64, OpenMP over y-planes / kx slabs like the
 * reference), the routines of ryankellybp11/Polymer_DNS FFTW_DNS/code/src/dns:
 * solvers.f90, derivatives.f90, helpers.f90 (norm, xyzfft, polymer coupling),
 * part_track.f90 (tracer path) and the time loop of main_dns.f90.  Each
 * function cites the reference lines it follows.  FFTW3 (not vendored in the
 * reference) is replaced by the oracle's own mixed-radix Stockham FFT that
 * reproduces FFTW's unnormalised REDFT00 / r2c / c2r / c2c conventions.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists on
 * this image or the GPU hosts, and the reference ships no tests or golden
 * vectors.  The oracle is therefore "parity unpinned" against the reference
 * binary; it is pinned instead by mathematical known answers (DCT-I identity,
 * exact Chebyshev derivatives of polynomials, manufactured Helmholtz / Robin
 * solutions, steady laminar Poiseuille, viscous decay of single modes,
 * uniform-flow tracer advection) in tests/test_oracle_known_answers.py.
 *
 * The API mirrors include/kmm.h (same kmm_params, same field ids, same routine
 * granularity) so tests drive both sides identically.
 */
#ifndef KMM_ORACLE_H
#define KMM_ORACLE_H
#include <stddef.h>
#include "../include/kmm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

int    orc_ctx_create(const kmm_params *p, orc_ctx **out);
void   orc_ctx_destroy(orc_ctx *c);
/* host pointer of a field (allocated and zeroed on first use), NULL if unknown */
void  *orc_field(orc_ctx *c, int field);
int    orc_field_size(orc_ctx *c, int field, size_t *nelem, int *elem_bytes);
int    orc_copy(orc_ctx *c, int dst, int src);
int    orc_zero(orc_ctx *c, int field);
int    orc_set_it(orc_ctx *c, int it);
int    orc_get_stats(orc_ctx *c, kmm_stats *s);
double orc_dpdx(orc_ctx *c);
/* OpenMP threads of the parallel loops (n <= 0: all host cores); returns the count in effect */
int    orc_set_threads(int n);

/* transforms (the FFTW conventions the reference relies on) */
int    orc_dct1(int n, const double *in, double *out);                 /* REDFT00, length n      */
int    orc_fft(int n, const double *in, double *out, int sign);        /* c2c, unnormalised      */
int    orc_rfft(int n, const double *in, double *out);                 /* r2c, n/2+1 outputs     */
int    orc_irfft(int n, const double *in, double *out);                /* c2r, n outputs         */

/* routines: same meaning as the kmm_* entry points of the same name */
int orc_cderiv(orc_ctx *c, int f, int df);
int orc_wallderiv(orc_ctx *c, int f, int order, int wall, int out, int iy);
int orc_gradv(orc_ctx *c);
int orc_gradscl(orc_ctx *c);
int orc_derivscji(orc_ctx *c);
int orc_gfcn(orc_ctx *c);
int orc_phirhs(orc_ctx *c, int v, int fn, int fnm1, double var);
int orc_solve(orc_ctx *c, int u, double g, int ib);
int orc_penta(orc_ctx *c, int u, double g, int ib, double at, double bt, double ab, double bb);
int orc_uzero(orc_ctx *c, int uflag);
int orc_phi_from_v(orc_ctx *c);
int orc_influence(orc_ctx *c);
int orc_veloc(orc_ctx *c);
int orc_vort(orc_ctx *c);
int orc_nonlin(orc_ctx *c);
int orc_vcw3dp(orc_ctx *c);
int orc_norm(orc_ctx *c, int f);
int orc_xyzfft(orc_ctx *c, int dst, int src);
int orc_polynl(orc_ctx *c);
int orc_polyforce(orc_ctx *c);
int orc_subforce(orc_ctx *c);
int orc_filter(orc_ctx *c);
int orc_initial(orc_ctx *c);
int orc_step(orc_ctx *c);
int orc_run(orc_ctx *c, int n);
int orc_tracer_update(orc_ctx *c);
int orc_inertial_update(orc_ctx *c);   /* particle_flag > 0: Maxey-Riley RK4, part_track.f90:617-1075 */
int orc_init_part(orc_ctx *c);
/* interpolation cells of the particles, as kmm_tracer_cells (part_track.f90:560-577) */
int orc_tracer_cells(orc_ctx *c, int *cells, size_t n);
/* swirl strength from the closed-form eigenvalues (helpers.f90:197-404) on the last 3/2-grid gradients */
int orc_calcswirl(orc_ctx *c);
/* scl_flag = 4: the targets (x, y, z grid indices, 1-based, 3 ints each) the last source was placed
 * at, in order; returns their number (n: ints available in ijk) */
int orc_target_list(orc_ctx *c, int *ijk, int n);
int orc_flowstats(orc_ctx *c, double *prof, double *scal);

#ifdef __cplusplus
}
#endif
#endif
