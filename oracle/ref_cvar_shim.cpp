// ORACLE — test infrastructure only.  extern "C" wrappers, compiled against
// the reference's _cvariogram/api.h, around the reference's internal
// functions that its C ABI does not export (calc_search_template_window,
// calc_lag_areas, is_in_tunnel; variograms.cpp:26-225), so that tests can
// compare the restatement with them.
#include <stdlib.h>

#include "api.h"

extern "C" {
void ref_cvar_window(variogram_search_template_t *t, double *w) {
    search_template_window_t win;
    calc_search_template_window(t, &win);
    w[0] = win.m_min_i;
    w[1] = win.m_min_j;
    w[2] = win.m_min_k;
    w[3] = win.m_max_i;
    w[4] = win.m_max_j;
    w[5] = win.m_max_k;
}
long long ref_cvar_lag_areas(variogram_search_template_t *t) {
    int n = 0;
    lag_point_t *p = calc_lag_areas(t, &n);
    free(p);
    return n;
}
int ref_cvar_in_tunnel(variogram_search_template_t *t, double x, double y, double z) {
    vector_t v;
    v.m_data[0] = x;
    v.m_data[1] = y;
    v.m_data[2] = z;
    return is_in_tunnel(t, &v) ? 1 : 0;
}
}
