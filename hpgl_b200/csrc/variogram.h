// Experimental variograms and layer stacking on the GPU (variogram.cu).
#pragma once
#include "../../include/cvariogram.h"

namespace hpgl_b200 {

// fill_ellipsoid_directions (host: three rotations).
void cv_fill_ellipsoid(ellipsoid_t *ell, double azimuth, double dip, double rotation);

// Per-lag sums of squared differences and pair counts of calc_variograms
// (first min(num_lags, result_length) lags).
void cv_grid(const variogram_search_template_t &t, const hard_data_t &data, int result_length, int percent,
             double *sums, unsigned long long *counts);

// The same for calc_variograms_from_point_set.
void cv_points(const variogram_search_template_t &t, const cont_point_set_t &points, int result_length, double *sums,
               unsigned long long *counts);

// cvar_stack_layers into result->m_data.
void cv_stack_layers(const float_data_t *layers, const int *markers, int nlayers, int nz, float scalez, int blank,
                     float_data_t *result);

}  // namespace hpgl_b200
