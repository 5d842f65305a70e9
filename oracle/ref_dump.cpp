// ORACLE — test infrastructure only.
//
// Dump driver compiled against the reference's own headers.  The reference's
// C ABI returns only the float estimate and the mask; this driver runs the
// same per-node steps as kriging_interpolation (kriging_interpolation.h:275-313)
// with the same covariance objects the drivers build (ordinary_kriging.cpp:27-34,
// simple_kriging.cpp:60-67, lvm_kriging.cpp:23-30, indicator_kriging.h:71-81,
// median_ik.cpp:49-59) and exports, per node: the neighbour index list in
// search order (indexed_neighbour_lookup_t::find), the kriging weights, the
// variance (sk/ok_kriging_weights_3 with calc_variance), the status and the
// estimate.  It pins the oracle restatement's neighbour lists, weights and
// variances to the reference code itself.
#include "stdafx.h"
#include <omp.h>
#include "api.h"
#include "typedefs.h"
#include "property_array.h"
#include "sugarbox_grid.h"
#include "ok_params.h"
#include "cov_model.h"
#include "precalculated_covariance.h"
#include "covariance_field.h"
#include "mean_provider.h"
#include "my_kriging_weights.h"
#include "kriging_interpolation.h"
#include "sugarbox_indexed_neighbour_lookup.h"
#include "is_informed_predicate.h"

using namespace hpgl;

namespace {
void fill_ok_params(const hpgl_ok_params_t *p, ok_params_t &o) {
    o.m_covariance_type = (covariance_type_t)p->m_covariance_type;
    o.set_ranges(p->m_ranges[0], p->m_ranges[1], p->m_ranges[2]);
    o.set_angles(p->m_angles[0], p->m_angles[1], p->m_angles[2]);
    o.m_sill = p->m_sill;
    o.m_nugget = p->m_nugget;
    o.set_radiuses(p->m_radiuses[0], p->m_radiuses[1], p->m_radiuses[2]);
    o.m_max_neighbours = p->m_max_neighbours;
}

struct dump_out {
    int max_out;
    int *nb_count;
    int *nb_index;
    double *weights;
    double *variance;
    int *status;
    double *estimate;
};

template <typename values_t, typename means_t, typename cov_t, typename wc_t, typename result_t, typename pred_t>
void dump_node(const values_t &values, const pred_t &pred, node_index_t node, const cov_t &cov, const means_t &mp,
               const indexed_neighbour_lookup_t<sugarbox_grid_t, cov_t> &nl, const wc_t &wc, long slot,
               const dump_out &o) {
    typedef sugarbox_location_t coord_t;
    std::vector<node_index_t> indices;
    std::vector<kriging_weight_t> weights;
    std::vector<mean_t> means;
    std::vector<typename values_t::value_type> vals;
    std::vector<coord_t> coords;
    coord_t node_coord;
    nl.find(node, pred, node_coord, indices, coords);
    int n = (int)indices.size();
    if (o.nb_count) o.nb_count[slot] = n;
    for (int i = 0; i < n && i < o.max_out; ++i) {
        if (o.nb_index) o.nb_index[slot * o.max_out + i] = indices[i];
    }
    double variance = -1;
    if (n <= 0) {
        if (o.status) o.status[slot] = KI_NO_NEIGHBOURS;
        return;
    }
    select(mp, indices, means);
    bool ok = wc(node_coord, mp[node], coords, means, cov, weights, variance);
    if (o.variance) o.variance[slot] = variance;
    if (o.weights)
        for (int i = 0; i < n && i < o.max_out; ++i) o.weights[slot * o.max_out + i] = weights[i];
    if (!ok) {
        if (o.status) o.status[slot] = KI_SINGULARITY;
        return;
    }
    if (o.status) o.status[slot] = KI_SUCCESS;
    select(values, indices, vals);
    result_t r = combine<typename values_t::value_type, result_t>(vals, weights, means, mp[node]);
    if (o.estimate) o.estimate[slot] = (double)r;
}
}  // namespace

extern "C" {

// kind: 0 = ordinary, 1 = simple (mean given), 2 = locally varying mean.
// Kriges every uninformed node, like cont_kriging (cont_kriging.h:78-105).
int ref_dump_cont(int kind, int nx, int ny, int nz, float *values, unsigned char *mask, const float *mean_cube,
                  const hpgl_ok_params_t *p, double sk_mean, int max_out, int *nb_count, int *nb_index,
                  double *weights, double *variance, int *status, double *estimate, int threads) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        sugarbox_grid_t grid;
        grid.init(nx, ny, nz);
        int size = nx * ny * nz;
        cont_property_array_t prop(values, mask, size);
        ok_params_t params;
        fill_ok_params(p, params);
        dump_out o = {max_out, nb_count, nb_index, weights, variance, status, estimate};
        is_informed_predicate_t<cont_property_array_t> pred(prop);
        if (kind == 0) {
            cov_model_t cov(params);
            indexed_neighbour_lookup_t<sugarbox_grid_t, cov_model_t> nl(&grid, &cov, params);
            for (node_index_t n = 0; n < size; ++n)
                if (prop.is_informed(n)) nl.add_node(n);
            no_mean_t mp;
            ok_weight_calculator_t wc;
#pragma omp parallel for schedule(dynamic, 256)
            for (node_index_t n = 0; n < size; ++n)
                if (!prop.is_informed(n)) dump_node<cont_property_array_t, no_mean_t, cov_model_t, ok_weight_calculator_t, cont_value_t>(prop, pred, n, cov, mp, nl, wc, n, o);
        } else {
            precalculated_covariances_t cov(cov_model_t(params), params.m_radiuses);
            indexed_neighbour_lookup_t<sugarbox_grid_t, precalculated_covariances_t> nl(&grid, &cov, params);
            for (node_index_t n = 0; n < size; ++n)
                if (prop.is_informed(n)) nl.add_node(n);
            sk_weight_calculator_t wc;
            if (kind == 1) {
                single_mean_t mp(sk_mean);
#pragma omp parallel for schedule(dynamic, 256)
                for (node_index_t n = 0; n < size; ++n)
                    if (!prop.is_informed(n)) dump_node<cont_property_array_t, single_mean_t, precalculated_covariances_t, sk_weight_calculator_t, cont_value_t>(prop, pred, n, cov, mp, nl, wc, n, o);
            } else {
                const mean_t *mp = mean_cube;
#pragma omp parallel for schedule(dynamic, 256)
                for (node_index_t n = 0; n < size; ++n)
                    if (!prop.is_informed(n)) dump_node<cont_property_array_t, const mean_t *, precalculated_covariances_t, sk_weight_calculator_t, cont_value_t>(prop, pred, n, cov, mp, nl, wc, n, o);
            }
        }
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "ref_dump_cont: %s\n", e.what());
        return 1;
    }
}

// kind: 3 = indicator kriging for one category `category` with marginal
// probability `marginal` (indicator_kriging.h:98-112: every node is kriged);
// 4 = median IK (median_ik.cpp:49-81), `marginal` = marginal_probs[1].
int ref_dump_ind(int kind, int nx, int ny, int nz, unsigned char *codes, unsigned char *mask, int category,
                 const hpgl_ok_params_t *p, double marginal, int max_out, int *nb_count, int *nb_index,
                 double *weights, double *variance, int *status, double *estimate, int threads) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        sugarbox_grid_t grid;
        grid.init(nx, ny, nz);
        int size = nx * ny * nz;
        indicator_property_array_t prop(codes, mask, size, kind == 4 ? 2 : category + 1);
        ok_params_t params;
        fill_ok_params(p, params);
        dump_out o = {max_out, nb_count, nb_index, weights, variance, status, estimate};
        is_informed_predicate_t<indicator_property_array_t> pred(prop);
        sk_weight_calculator_t wc;
        if (kind == 3) {
            precalculated_covariances_t cov(cov_model_t(params), params.m_radiuses);
            indexed_neighbour_lookup_t<sugarbox_grid_t, precalculated_covariances_t> nl(&grid, &cov, params);
            for (node_index_t n = 0; n < size; ++n)
                if (prop.is_informed(n)) nl.add_node(n);
            indicator_array_adapter_t adapter(&prop, (indicator_value_t)category);
            std::vector<indicator_probability_t> mps(1, (indicator_probability_t)marginal);
            std::vector<single_mean_t> means;
            create_means(mps, means);
#pragma omp parallel for schedule(dynamic, 256)
            for (node_index_t n = 0; n < size; ++n)
                dump_node<indicator_array_adapter_t, single_mean_t, precalculated_covariances_t, sk_weight_calculator_t, indicator_probability_t>(adapter, pred, n, cov, means[0], nl, wc, n, o);
        } else {
            covariance_field_t cov(params.m_radiuses, cov_model_t(params));
            indexed_neighbour_lookup_t<sugarbox_grid_t, covariance_field_t> nl(&grid, &cov, params);
            for (node_index_t n = 0; n < size; ++n)
                if (prop.is_informed(n)) nl.add_node(n);
            indicator_array_adapter_t adapter(&prop, 1);
            single_mean_t mp(marginal);
#pragma omp parallel for schedule(dynamic, 256)
            for (node_index_t n = 0; n < size; ++n)
                dump_node<indicator_array_adapter_t, single_mean_t, covariance_field_t, sk_weight_calculator_t, double>(adapter, pred, n, cov, mp, nl, wc, n, o);
        }
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "ref_dump_ind: %s\n", e.what());
        return 1;
    }
}

// Template of the search (calc_cov_field, covariance_field.h:62-106), sorted,
// as (dx, dy, dz) triples; returns its length, or -1 when `cap` is too small.
int ref_template(const hpgl_ok_params_t *p, int *out_xyz, int cap) {
    ok_params_t params;
    fill_ok_params(p, params);
    cov_model_t cov(params);
    std::vector<sugarbox_vector_t> v;
    calc_cov_field<cov_model_t, sugarbox_location_t>(params.m_radiuses, cov, v);
    if ((int)v.size() > cap) return -1;
    for (size_t i = 0; i < v.size(); ++i) {
        out_xyz[3 * i] = v[i][0];
        out_xyz[3 * i + 1] = v[i][1];
        out_xyz[3 * i + 2] = v[i][2];
    }
    return (int)v.size();
}
}

extern "C" {
// Times nothing itself: runs the reference's per-node kriging
// (kriging_interpolation, kriging_interpolation.h:228-265, with the lookup
// and covariance objects its drivers build) on the nodes of `node_list`, in
// an OpenMP loop like cont_kriging's (cont_kriging.h:392-429).  The lookup
// construction (template sort, clusterizer fill) runs first and is included.
// kind: 0 OK, 1 SK.  Estimates go to out[i] (NaN on failure).  Returns 0.
int ref_sample_cont(int kind, int nx, int ny, int nz, float *values, unsigned char *mask, const hpgl_ok_params_t *p,
                    double sk_mean, const int *node_list, int n_nodes, int threads, float *out) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        sugarbox_grid_t grid;
        grid.init(nx, ny, nz);
        int size = nx * ny * nz;
        cont_property_array_t prop(values, mask, size);
        ok_params_t params;
        fill_ok_params(p, params);
        is_informed_predicate_t<cont_property_array_t> pred(prop);
        if (kind == 0) {
            cov_model_t cov(params);
            indexed_neighbour_lookup_t<sugarbox_grid_t, cov_model_t> nl(&grid, &cov, params);
            for (node_index_t n = 0; n < size; ++n)
                if (prop.is_informed(n)) nl.add_node(n);
            no_mean_t mp;
            ok_weight_calculator_t wc;
#pragma omp parallel for
            for (int i = 0; i < n_nodes; ++i) {
                cont_value_t v;
                ki_result_t r = kriging_interpolation(prop, pred, node_list[i], cov, mp, nl, wc, v);
                out[i] = r == KI_SUCCESS ? v : NAN;
            }
        } else {
            precalculated_covariances_t cov(cov_model_t(params), params.m_radiuses);
            indexed_neighbour_lookup_t<sugarbox_grid_t, precalculated_covariances_t> nl(&grid, &cov, params);
            for (node_index_t n = 0; n < size; ++n)
                if (prop.is_informed(n)) nl.add_node(n);
            single_mean_t mp(sk_mean);
            sk_weight_calculator_t wc;
#pragma omp parallel for
            for (int i = 0; i < n_nodes; ++i) {
                cont_value_t v;
                ki_result_t r = kriging_interpolation(prop, pred, node_list[i], cov, mp, nl, wc, v);
                out[i] = r == KI_SUCCESS ? v : NAN;
            }
        }
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "ref_sample_cont: %s\n", e.what());
        return 1;
    }
}
}
