/*
 * modegen -- writes a waveguide eigenmode with the reference's own solver.
 *
 * Test infrastructure only.  The reference driver loads its launch/output modes
 * from mode_files/*.txt (3d_fdtd.c:47-61), which the reference repository does
 * not ship.  This harness builds the strip cross-section with the reference's
 * mode API and calls its Arnoldi beta^2 solver (mode.c:3461-3616), then writes
 * the result in the reference's text format with mode_file_print
 * (mode.c:843-894), so that mode_file_load (mode.c:949-1038) and the engine's
 * own loader read the same numbers.
 *
 * usage: modegen nx ny disc core_left core_right core_bottom core_top
 *                ep_clad ep_core lambda krylov tol out.txt
 *
 * The cladding fills the window; the core is the rectangle
 * [core_left, core_right) x [core_bottom, core_top) (mode.c:2308-2328).
 * Confinement 2 (zero field on the window edge, mode.c:1614-1632), no PML,
 * lateral symmetrisation off: with it on (mode.c:4494-4527) the solver's
 * rand() start vector settles on the TM-like mode of a Si strip; with it off it
 * returns the fundamental TE mode (n_eff 2.474 for 500 x 225 nm at 1.55 um).
 * Links oracle/_ref/libref.so.
 */
#include <stdio.h>
#include <stdlib.h>
#include "complex.h"
#include "matrix.h"
#include "mode.h"

int main(int argc, char **argv)
{
    if (argc != 14) {
        fprintf(stderr, "usage: %s nx ny disc l r b t ep_clad ep_core lambda krylov tol out.txt\n", argv[0]);
        return 2;
    }
    int nx = atoi(argv[1]), ny = atoi(argv[2]);
    double disc = atof(argv[3]);
    int l = atoi(argv[4]), r = atoi(argv[5]), b = atoi(argv[6]), t = atoi(argv[7]);
    double ep_clad = atof(argv[8]), ep_core = atof(argv[9]);
    double lambda = atof(argv[10]);
    int krylov = atoi(argv[11]);
    double tol = atof(argv[12]);
    const char *out = argv[13];

    /* same 9-digit pi the reference driver uses for omega (3d_fdtd.c:12,37) */
    double omega = 2 * 3.141592652 / lambda;

    mode m = mode_new(nx, ny, disc);
    mode_set_background(m, complex_from_doubles(ep_clad, 0), complex_from_doubles(1, 0));
    mode_make_rectangle(m, complex_from_doubles(ep_core, 0), complex_from_doubles(1, 0), l, r, b, t);

    complex beta = mode_solve_beta_squared(&m, omega, tol, NULL, 0, krylov, 2, 0);
    fprintf(stderr, "modegen: beta = %.9f%+.9fi  n_eff = %.9f\n", beta.re, beta.im, beta.re / omega);

    FILE *f = fopen(out, "w");
    if (!f) { perror(out); return 1; }
    mode_file_print(f, m, 2);
    fclose(f);
    mode_free(m);
    return 0;
}
