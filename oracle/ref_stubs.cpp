// ORACLE — test infrastructure only.  Link stubs for the reference's
// sequential-simulation entry points (hpgl_core.h:85-117), which api.cpp
// references but which are outside the kriging path and need boost::random
// plus a blob missing from the reference tree.  Calling one throws.
#include "stdafx.h"
#include "hpgl_core.h"
#include "hpgl_exception.h"
#include "sgs_params.h"
#include "ik_params.h"
#include "progress_reporter.h"

namespace hpgl {
static void not_built(const char *what) {
    throw hpgl_exception(what, "sequential simulation is not built into the oracle library");
}
void sequential_gaussian_simulation(const sugarbox_grid_t &, const sgs_params_t &, cont_property_array_t &,
                                    const hpgl_non_parametric_cdf_t *, const unsigned char *) {
    not_built("sequential_gaussian_simulation");
}
void sequential_gaussian_simulation_lvm(const sugarbox_grid_t &, const sgs_params_t &, const mean_t *,
                                        cont_property_array_t &, const hpgl_non_parametric_cdf_t *,
                                        const unsigned char *) {
    not_built("sequential_gaussian_simulation_lvm");
}
void sequential_indicator_simulation(indicator_property_array_t &, const sugarbox_grid_t &, const ik_params_t &,
                                     int, progress_reporter_t &, bool, const unsigned char *) {
    not_built("sequential_indicator_simulation");
}
void sequential_indicator_simulation_lvm(indicator_property_array_t &, const sugarbox_grid_t &,
                                         const ik_params_t &, int, const mean_t **, progress_reporter_t &, bool,
                                         const unsigned char *) {
    not_built("sequential_indicator_simulation_lvm");
}
}  // namespace hpgl
