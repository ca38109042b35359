// host_ref.h -- host-side parts of the reference call surface (internal header).
#pragma once

#include "../../include/fdtd_b200.h"

namespace fdtd {

void raster_background(timefield3d psi, float ep, float mu);
void raster_top_half_plane(timefield3d psi, float ep, float mu, int bottom);
void raster_background_permittivity(timefield3d psi, float ep);
void raster_background_permeability(timefield3d psi, float mu);
void raster_background_conductivity(timefield3d psi, float sig, int magnetic);
// what = 0: permittivity, 1: electric conductivity
void raster_prism(timefield3d psi, float v, int sx, int ex, int sy, int ey, int sz, int ez, int what);
void raster_taper(timefield3d psi, double ep, double mu, int start_left, int start_right, int end_left, int end_right,
                  int start_z, int end_z, int bottom, int top);
void taper_insert(timefield3d psi, const adjoint3d_taper &t);
void taper_vertex_gradients(const adjoint3d_taper &t, double ep_diff);
int taper_update_symmetric(const adjoint3d_taper &t, double goal, double disc, int min_width);
int taper_update_asymmetric(const adjoint3d_taper &t, double goal, double disc, int min_width);
int write_permittivity_y_slice(timefield3d psi, const char *filename, int left, int right, int start, int end,
                               int y_slice, double ep_min, double ep_max);
void cexp_series(double x, double *re, double *im);
double reduce_phase(double phase);

}  // namespace fdtd
