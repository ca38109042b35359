/* taper_driver.c -- the reference driver's call sequence (3d_fdtd.c:97-187)
 * on the small Si taper of the golden fixtures, written in C against the
 * reference's own headers.  It is compiled twice by oracle/Makefile (target
 * `dropin`):
 *
 *   taper_driver_ref   linked with the reference's complex.o matrix.o mode.o
 *                      timefield3d.o adjoint3d.o (its CPU implementation)
 *   taper_driver_b200  linked with complex.o matrix.o mode.o and
 *                      libfdtd_b200.so in place of timefield3d.o adjoint3d.o
 *
 * so the struct layouts and signatures of the drop-in are checked by a C
 * compiler and linker, not by a binding.  tests/test_c_dropin.py runs both and
 * compares what they write.
 *
 *   taper_driver_* <mode file (reference text format)> <output file>
 *
 * Output (binary, native endianness): 3 complex cumulative overlaps (launched,
 * reflected, transmitted), the 6 field components of the output plane after
 * the forward run (nx*ny*6 doubles, the reference's AoS order), the same after
 * the adjoint run, the ep gradient (2*H*L doubles), the left and right vertex
 * gradients (seg_num+1 doubles each), the updated left and right edges
 * (seg_num+1 ints each) and the update's return flag (int).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "matrix.h"
#include "complex.h"
#include "mode.h"
#include "timefield3d.h"
#include "adjoint3d.h"
#ifdef FDTD_B200
#include "fdtd_b200.h"
#endif

#define PI 3.141592652

static void put(FILE *f, const void *p, size_t n)
{
    if (fwrite(p, 1, n, f) != n) {
        fprintf(stderr, "short write\n");
        exit(2);
    }
}

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s <mode file> <output file>\n", argv[0]);
        return 2;
    }
    /* the small taper of tests/golden/make_golden.py (wg_setup) */
    const int nx = 40, ny = 28, nz = 72, T = 400, seg_num = 4;
    const int bottom = 11, top = 16, z0 = 24, z1 = 48, src_z = 12, launch_z = 16, out_z = 58;
    const double disc = 0.05, ep_core = 12.1, ep_clad = 2.085;
    int left[5] = {15, 14, 12, 12, 13}, right[5] = {25, 26, 27, 28, 27};
    const double omega = 2 * PI / 1.55, delta_t = 0.99 * disc / sqrt(3);
    const int cx = nx / 2, cy = (bottom + top) / 2;
    int i;

    FILE *md = fopen(argv[1], "r");
    if (!md) return 2;
    mode launch_mode = mode_file_load(md);
    fclose(md);
    md = fopen(argv[1], "r");
    mode output_mode = mode_file_load(md);
    fclose(md);

    timefield3d main_field = timefield3d_new(nx, ny, nz, disc);
    timefield3d_set_background(main_field, ep_clad, 1.0);
    timefield3d_set_waveguide(main_field, ep_core, 15, 25, 0, z0, bottom, top);
    timefield3d_set_waveguide(main_field, ep_core, 13, 27, z1, nz, bottom, top);
    adjoint3d_taper taper = adjoint3d_taper_new(ep_core, 1.0, seg_num, z0, z1, left, right, bottom, top, T);
    adjoint3d_taper_insert(main_field, taper);

    /* forward run */
    complex launched = complex_zero(), reflected = complex_zero(), transmitted = complex_zero();
    timefield3d_zero_fields(main_field);
    for (i = 0; i < T; i++) {
        double amplitude = i < 300 ? exp(-(i - 120) * (i - 120) / (2 * 40.0 * 40.0)) : 0;
        double phase = i * delta_t * omega;
        timefield3d_mode_source(main_field, cx, cy, src_z, launch_mode, phase, amplitude, 0);
        timefield3d_apply_timestep_omp_full(main_field, delta_t);
        timefield3d_update_fourier_fields_y_slice_omp(main_field, phase, cy);
        timefield3d_mode_overlap(main_field, cx, cy, launch_z, launch_mode, phase, 0, &launched);
        timefield3d_mode_overlap(main_field, cx, cy, launch_z, launch_mode, phase, 1, &reflected);
        timefield3d_mode_overlap(main_field, cx, cy, out_z, output_mode, phase, 0, &transmitted);
        adjoint3d_taper_store_forward_fields(taper, main_field, i);
    }
    FILE *out = fopen(argv[2], "wb");
    if (!out) return 2;
    put(out, &launched, sizeof(complex));
    put(out, &reflected, sizeof(complex));
    put(out, &transmitted, sizeof(complex));
    double *fields = timefield3d_get_fields(main_field);
    put(out, fields + (size_t)6 * nx * ny * out_z, sizeof(double) * 6 * nx * ny);

    /* adjoint run (3d_fdtd.c:143-165) */
    double transmission_phase = complex_angle(transmitted);
    mode_smul(complex_exp(complex_from_doubles(0, transmission_phase + PI / 2)), output_mode);
    timefield3d_zero_fields(main_field);
    for (i = T - 1; i >= 0; i--) {
        double phase = (i + 1) * delta_t * omega;
        timefield3d_mode_source_adjoint(main_field, cx, cy, out_z, output_mode, phase, 0);
        timefield3d_apply_timestep_omp_full(main_field, delta_t);
        adjoint3d_taper_store_adjoint_fields(taper, main_field, i);
    }
    fields = timefield3d_get_fields(main_field);
    put(out, fields + (size_t)6 * nx * ny * out_z, sizeof(double) * 6 * nx * ny);

    /* gradients and the edge update (3d_fdtd.c:167-175) */
    adjoint3d_taper_calculate_ep_gradient(taper);
    adjoint3d_taper_calculate_gradients_from_ep_gradient(taper, ep_core - ep_clad);
    double improvement = 0.2 * (complex_mag(launched) - complex_mag(transmitted));
    int flag = adjoint3d_taper_update_asymmetric(taper, improvement, main_field.disc, 4);
    put(out, taper.ep_gradient, sizeof(double) * 2 * (top - bottom) * (z1 - z0));
    put(out, taper.left_grad, sizeof(double) * (seg_num + 1));
    put(out, taper.right_grad, sizeof(double) * (seg_num + 1));
    put(out, taper.left, sizeof(int) * (seg_num + 1));
    put(out, taper.right, sizeof(int) * (seg_num + 1));
    put(out, &flag, sizeof(int));
    fclose(out);
#ifdef FDTD_B200
    if (fdtd_last_error()) {
        fprintf(stderr, "libfdtd_b200: %s\n", fdtd_last_error_message());
        return 1;
    }
#endif
    printf("launched %.12e %.12e transmitted %.12e %.12e flag %d\n", launched.re, launched.im, transmitted.re,
           transmitted.im, flag);
    return 0;
}
