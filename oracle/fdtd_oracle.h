/*
 * fdtd_oracle.h -- CPU restatement of the FDTD hot path, for checking only.
 *
 * TEST INFRASTRUCTURE.  Only tests/, the smoke check and bench.py's CPU
 * baseline leg load this library, and only as the checker.  The product
 * (lib/libfdtd_b200.so) never links or calls it.
 *
 * What it restates (reference file:line):
 *   Yee E/H semi-implicit update      timefield3d.c:1679-1837
 *   step order (shell save, E, E-ABC, H, H-ABC)   timefield3d.c:2787-2849
 *   Mur first-order ABC + shell save  timefield3d.c:2275-2721, 246-346
 *   mode source / adjoint source      timefield3d.c:2977-3068
 *   mode overlap + running DFT        timefield3d.c:3176-3239, complex.c:169-193
 *   power normalisation               mode.c:1267-1379
 *   y-slice running DFT               timefield3d.c:2922-2975
 *   taper edge store / ep-gradient / vertex gradient   adjoint3d.c:259-418
 * What it defines (no reference counterpart): the convolutional PML (CPML)
 * boundary and the multi-wavelength overlap monitors.
 *
 * Arithmetic follows the reference exactly: fields in double, materials and
 * sources in float promoted to double, the same operation order, no FMA
 * (built without -march, so x86-64 SSE2 double mul/add).  Layout is SoA:
 * component m of cell (i,j,k) lives at f[m][i + nx*(j + ny*k)].
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_BOUNDARY_PEC = 0, ORC_BOUNDARY_MUR = 1, ORC_BOUNDARY_CPML = 2 };

typedef struct orc_grid orc_grid;

orc_grid *orc_new(int nx, int ny, int nz, double dx);
void orc_free(orc_grid *g);
void orc_zero(orc_grid *g);                 /* fields, shell copy, sources, psi */
double *orc_field(orc_grid *g, int m);      /* m = 0..5: Ex Ey Ez Hx Hy Hz */
float *orc_ep(orc_grid *g, int c);          /* c = 0..2 */
float *orc_mu(orc_grid *g, int c);
float *orc_sig(orc_grid *g, int m);         /* m = 0..2 electric, 3..5 magnetic */
float *orc_src(orc_grid *g, int m);         /* full-grid sources, like timefield3d.sources */
void orc_set_boundary(orc_grid *g, int boundary);
/* CPML: npml cells on every face, polynomial grading of order `order`.
 * sigma_max <= 0 selects 0.8*(order+1)/dx.  Profiles are built for time step dt. */
void orc_set_cpml(orc_grid *g, int npml, int order, double sigma_max,
                  double kappa_max, double alpha_max, double dt);
/* 1-D CPML coefficient tables, for the engine's parity tests.
 * which: 0 b_E, 1 a_E, 2 1/kappa_E, 3 b_H, 4 a_H, 5 1/kappa_H; axis 0..2. */
const double *orc_cpml_profile(orc_grid *g, int which, int axis);

void orc_step(orc_grid *g, double dt);      /* one full leapfrog step */
void orc_step_threads(int nthreads);        /* OpenMP threads for the stencil */

/* Modes: complex double interleaved (re, im); entry 6*(i + mi*j) + m. */
double orc_mode_power_norm(const double *mode, int mi, int mj, double mdisc);
void orc_mode_power_normalize(double *mode, int mi, int mj, double mdisc);
void orc_mode_source(orc_grid *g, int cx, int cy, int cz, double *mode, int mi, int mj,
                     double mdisc, double phase, double amplitude, int reverse);
void orc_mode_source_adjoint(orc_grid *g, int cx, int cy, int cz, double *mode, int mi,
                             int mj, double mdisc, double phase, int reverse);
/* returns the instantaneous overlap in inst[2]; adds e^{i phase} * inst to cum[2] */
void orc_mode_overlap(orc_grid *g, int cx, int cy, int cz, double *mode, int mi, int mj,
                      double mdisc, double phase, int reverse, double *cum, double *inst);
/* instantaneous overlap without normalising the mode (mode already normalised) */
void orc_overlap_instant(orc_grid *g, int cx, int cy, int cz, const double *mode, int mi,
                         int mj, double mdisc, int reverse, double *inst);
/* e^{i x} by the reference's power series (complex.c:169-193) */
void orc_cexp_series(double x, double *re, double *im);
/* phase reduction with the reference's 9-digit pi (timefield3d.c:3235) */
double orc_reduce_phase(double phase);
/* y-slice running DFT of all 6 components (timefield3d.c:2922-2943);
 * acc is complex interleaved, 6*nx*nz entries, index 2*(m + 6*(i + nx*k)). */
void orc_dft_y_slice(orc_grid *g, double phase, int slice, double *acc);

/* Taper edge store and gradients (adjoint3d.c:259-418).  Storage is E only,
 * layout [t][k - start][j - bottom][edge][3], edge 0 = right, 1 = left. */
void orc_taper_store(orc_grid *g, int seg_num, int start, int end, int bottom, int top,
                     const int *left, const int *right, int t, double *store);
void orc_taper_ep_gradient(int height, int length, int duration, const double *fwd,
                           const double *adj, double *ep_grad);
void orc_taper_vertex_gradient(int seg_num, int height, int length, const double *ep_grad,
                               double ep_diff, double *left_grad, double *right_grad);

#ifdef __cplusplus
}
#endif
#endif
