// extern "C" entry points of hpgl.so: the reference's kriging ABI
// (src/geo_bsd/hpgl/api.h, api.cpp) plus this library's additions, all declared
// in include/hpgl.h.  Every entry point catches every error and records it
// for hpgl_get_last_exception_message / hpgl_get_last_error.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hpgl.h"
#include "engine.h"
#include "kernels.cuh"
#include "plan.h"
#include "sgs_host.h"
#include "textio.h"
#include "variogram.h"

using namespace hpgl_b200;

namespace {
std::mutex g_err_mutex;
std::string g_last_message;
int g_last_error = 0;
int (*g_output_handler)(char *, void *) = nullptr;
void *g_output_param = nullptr;
int (*g_progress_handler)(char *, int, void *) = nullptr;
void *g_progress_param = nullptr;

void set_error(int code, const std::string &msg) {
    std::lock_guard<std::mutex> l(g_err_mutex);
    g_last_error = code;
    g_last_message = msg;
}

void log_line(const std::string &s) {
    if (g_output_handler) g_output_handler((char *)s.c_str(), g_output_param);
}

template <typename F>
int guarded(const char *where, F f) {
    try {
        f();
        set_error(HPGL_OK, "");
        return HPGL_OK;
    } catch (const HpglError &e) {
        set_error(e.code, std::string(where) + ": " + e.message);
        return e.code;
    } catch (const std::bad_alloc &) {
        set_error(HPGL_E_CAPACITY, std::string(where) + ": out of host memory");
        return HPGL_E_CAPACITY;
    } catch (const std::exception &e) {
        set_error(HPGL_E_INTERNAL, std::string(where) + ": " + e.what());
        return HPGL_E_INTERNAL;
    } catch (...) {
        set_error(HPGL_E_INTERNAL, std::string(where) + ": unknown error");
        return HPGL_E_INTERNAL;
    }
}

long long volume(const hpgl_shape_t *s) {
    if (!s) throw HpglError{HPGL_E_INVALID, "shape is null"};
    return (long long)s->m_data[0] * s->m_data[1] * s->m_data[2];
}

hpgl_ik_params_t from_ok(const hpgl_ok_params_t *p) {
    if (!p) throw HpglError{HPGL_E_INVALID, "params are null"};
    hpgl_ik_params_t q;
    memset(&q, 0, sizeof(q));
    q.m_covariance_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i) {
        q.m_ranges[i] = p->m_ranges[i];
        q.m_angles[i] = p->m_angles[i];
        q.m_radiuses[i] = p->m_radiuses[i];
    }
    q.m_sill = p->m_sill;
    q.m_nugget = p->m_nugget;
    q.m_max_neighbours = p->m_max_neighbours;
    return q;
}

hpgl_b200_job_t base_job(int kind, const hpgl_shape_t *shape) {
    hpgl_b200_job_t j;
    memset(&j, 0, sizeof(j));
    j.kind = kind;
    j.nx = shape->m_data[0];
    j.ny = shape->m_data[1];
    j.nz = shape->m_data[2];
    j.precision = -1;
    return j;
}

void run(const char *name, hpgl_b200_job_t &job, hpgl_b200_result_t &res) {
    run_job(job, res);
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %lld systems in %.3f ms (plan %.3f, device %.3f)\n", name, res.systems,
             res.ms_total, res.ms_plan, res.ms_device);
    log_line(buf);
}

}  // namespace

namespace {
// The INC / GSLIB entry points' errors keep the reference's own messages, "where: what".
template <typename F>
void guarded_io(const char *where, F f) {
    try {
        f();
        set_error(HPGL_OK, "");
    } catch (const HpglError &e) {
        set_error(e.code, e.message);
    } catch (const std::bad_alloc &) {
        set_error(HPGL_E_CAPACITY, std::string(where) + ": out of host memory");
    } catch (const std::exception &e) {
        set_error(HPGL_E_INTERNAL, std::string(where) + ": " + e.what());
    } catch (...) {
        set_error(HPGL_E_INTERNAL, std::string(where) + ": unknown error");
    }
}

// init_remap_table (api.cpp:117-136 of the reference): the indicator values
// that the bytes 0..indicator_count-1 are written as.
std::vector<unsigned char> remap_table(const unsigned char *values, int values_count, int indicator_count) {
    std::vector<unsigned char> t;
    if (values_count > 0 && !values) throw HpglError{HPGL_E_INVALID, "values are null"};
    if (values_count == indicator_count) {
        t.assign(values, values + values_count);
    } else if (values_count > indicator_count) {
        log_line("Given " + std::to_string(values_count) + " values for " + std::to_string(indicator_count) +
                 " indicators. Ignoring extra values.\n");
        t.assign(values, values + indicator_count);
    } else {
        if (values_count > 0)
            log_line("Warning: Given " + std::to_string(values_count) + " values for " +
                     std::to_string(indicator_count) + " indicators. Ignoring values. Using [0, 1, 2 ..]\n");
        for (int i = 0; i < indicator_count; ++i) t.push_back((unsigned char)i);
    }
    return t;
}

// (unsigned char) of a double as the x86-64 compilers convert it: through a
// 32-bit integer, keeping the low byte.
unsigned char byte_of_double(double v) {
    if (!(v > -2147483649.0 && v < 2147483648.0)) return 0;
    return (unsigned char)(unsigned)(int)v;
}

}  // namespace

extern "C" {

char *hpgl_get_last_exception_message(void) {
    std::lock_guard<std::mutex> l(g_err_mutex);
    return (char *)g_last_message.c_str();
}

int hpgl_get_last_error(void) {
    std::lock_guard<std::mutex> l(g_err_mutex);
    return g_last_error;
}

void hpgl_set_output_handler(int (*handler)(char *, void *), void *param) {
    g_output_handler = handler;
    g_output_param = param;
}

void hpgl_set_progress_handler(int (*handler)(char *, int, void *), void *param) {
    g_progress_handler = handler;
    g_progress_param = param;
}

void hpgl_set_thread_num(int n_threads) { set_host_threads(n_threads); }
int hpgl_get_thread_num(void) { return host_threads(); }

void hpgl_b200_set_precision(int precision) {
    guarded("hpgl_b200_set_precision", [&] {
        if (precision != HPGL_PRECISION_FP64 && precision != HPGL_PRECISION_MIXED)
            throw HpglError{HPGL_E_INVALID, "unknown precision"};
        set_default_precision(precision);
    });
}
int hpgl_b200_get_precision(void) { return default_precision(); }

void hpgl_b200_set_sim_window(int window) {
    guarded("hpgl_b200_set_sim_window", [&] {
        if (window == 0) window = 1 << 18;
        if (window < 1 || window > (1 << 24)) throw HpglError{HPGL_E_INVALID, "window must be in [1, 2^24]"};
        set_sim_window(window);
    });
}

void hpgl_ordinary_kriging(hpgl_cont_masked_array_t *input_data, hpgl_ok_params_t *params,
                           hpgl_cont_masked_array_t *output_data) {
    guarded("hpgl_ordinary_kriging", [&] {
        if (!input_data || !output_data) throw HpglError{HPGL_E_INVALID, "null array"};
        if (volume(&input_data->m_shape) != volume(&output_data->m_shape))
            throw HpglError{HPGL_E_INVALID, "input and output sizes differ"};
        hpgl_ik_params_t p = from_ok(params);
        hpgl_b200_job_t job = base_job(HPGL_KIND_OK, &input_data->m_shape);
        job.values = input_data->m_data;
        job.mask = input_data->m_mask;
        job.params = &p;
        job.n_params = 1;
        hpgl_b200_result_t res;
        memset(&res, 0, sizeof(res));
        res.out_values = output_data->m_data;
        res.out_mask = output_data->m_mask;
        run("Ordinary Kriging", job, res);
    });
}

void hpgl_simple_kriging(float *input_data, unsigned char *input_mask, hpgl_shape_t *input_data_shape,
                         hpgl_sk_params_t *params, float *output_data, unsigned char *output_mask,
                         hpgl_shape_t *output_data_shape) {
    guarded("hpgl_simple_kriging", [&] {
        if (!params) throw HpglError{HPGL_E_INVALID, "params are null"};
        if (volume(input_data_shape) != volume(output_data_shape))
            throw HpglError{HPGL_E_INVALID, "input and output sizes differ"};
        hpgl_ok_params_t okp;
        okp.m_covariance_type = params->m_covariance_type;
        for (int i = 0; i < 3; ++i) {
            okp.m_ranges[i] = params->m_ranges[i];
            okp.m_angles[i] = params->m_angles[i];
            okp.m_radiuses[i] = params->m_radiuses[i];
        }
        okp.m_sill = params->m_sill;
        okp.m_nugget = params->m_nugget;
        okp.m_max_neighbours = params->m_max_neighbours;
        hpgl_ik_params_t p = from_ok(&okp);
        hpgl_b200_job_t job = base_job(HPGL_KIND_SK, input_data_shape);
        job.values = input_data;
        job.mask = input_mask;
        job.params = &p;
        job.n_params = 1;
        // api.cpp:255-258: the mean is used only when not automatic.
        job.sk_automatic_mean = params->m_automatic_mean ? 1 : 0;
        job.sk_mean = params->m_mean;
        hpgl_b200_result_t res;
        memset(&res, 0, sizeof(res));
        res.out_values = output_data;
        res.out_mask = output_mask;
        run("Simple Kriging", job, res);
    });
}

void hpgl_lvm_kriging(float *input_data, unsigned char *input_mask, hpgl_shape_t *input_data_shape, float *mean_data,
                      hpgl_shape_t *mean_data_shape, hpgl_ok_params_t *params, float *output_data,
                      unsigned char *output_mask, hpgl_shape_t *output_data_shape) {
    guarded("hpgl_lvm_kriging", [&] {
        long long n = volume(input_data_shape);
        if (mean_data_shape && volume(mean_data_shape) != n)
            throw HpglError{HPGL_E_INVALID, "mean cube size differs from the input size"};
        if (output_data_shape && volume(output_data_shape) != n)
            throw HpglError{HPGL_E_INVALID, "input and output sizes differ"};
        hpgl_ik_params_t p = from_ok(params);
        hpgl_b200_job_t job = base_job(HPGL_KIND_LVM, input_data_shape);
        job.values = input_data;
        job.mask = input_mask;
        job.mean = mean_data;
        job.params = &p;
        job.n_params = 1;
        hpgl_b200_result_t res;
        memset(&res, 0, sizeof(res));
        res.out_values = output_data;
        res.out_mask = output_mask;
        run("LVM Kriging", job, res);
    });
}

void hpgl_indicator_kriging(hpgl_ind_masked_array_t *in_data, hpgl_ind_masked_array_t *out_data,
                            hpgl_ik_params_t *params, int indicator_count) {
    guarded("hpgl_indicator_kriging", [&] {
        if (!in_data || !out_data || !params) throw HpglError{HPGL_E_INVALID, "null argument"};
        if (indicator_count < 1) throw HpglError{HPGL_E_INVALID, "indicator_count must be >= 1"};
        if (volume(&in_data->m_shape) != volume(&out_data->m_shape))
            throw HpglError{HPGL_E_INVALID, "input and output sizes differ"};
        hpgl_b200_job_t job = base_job(HPGL_KIND_IK, &in_data->m_shape);
        job.codes = in_data->m_data;
        job.mask = in_data->m_mask;
        job.params = params;
        job.n_params = indicator_count;
        hpgl_b200_result_t res;
        memset(&res, 0, sizeof(res));
        res.out_codes = out_data->m_data;
        res.out_mask = out_data->m_mask;
        run("Indicator Kriging", job, res);
    });
}

void hpgl_median_ik(hpgl_ind_masked_array_t *in_data, hpgl_median_ik_params_t *params,
                    hpgl_ind_masked_array_t *out_data) {
    guarded("hpgl_median_ik", [&] {
        if (!in_data || !out_data || !params) throw HpglError{HPGL_E_INVALID, "null argument"};
        // median_ik.cpp:35-43
        if (volume(&in_data->m_shape) != volume(&out_data->m_shape))
            throw HpglError{HPGL_E_INVALID, "Input property size is not equal output property size"};
        hpgl_ok_params_t okp;
        okp.m_covariance_type = params->m_covariance_type;
        for (int i = 0; i < 3; ++i) {
            okp.m_ranges[i] = params->m_ranges[i];
            okp.m_angles[i] = params->m_angles[i];
            okp.m_radiuses[i] = params->m_radiuses[i];
        }
        okp.m_sill = params->m_sill;
        okp.m_nugget = params->m_nugget;
        okp.m_max_neighbours = params->m_max_neighbours;
        hpgl_ik_params_t p = from_ok(&okp);
        hpgl_b200_job_t job = base_job(HPGL_KIND_MEDIAN_IK, &in_data->m_shape);
        job.codes = in_data->m_data;
        job.mask = in_data->m_mask;
        job.params = &p;
        job.n_params = 1;
        job.median_marginal1 = params->m_marginal_probs[1];
        hpgl_b200_result_t res;
        memset(&res, 0, sizeof(res));
        res.out_codes = out_data->m_data;
        res.out_mask = out_data->m_mask;
        run("Median IK", job, res);
    });
}

int hpgl_b200_krige(const hpgl_b200_job_t *job, hpgl_b200_result_t *result) {
    return guarded("hpgl_b200_krige", [&] {
        if (!job || !result) throw HpglError{HPGL_E_INVALID, "null argument"};
        run_job(*job, *result);
    });
}

int hpgl_b200_bench(const hpgl_b200_job_t *job, hpgl_b200_result_t *result, hpgl_b200_bench_t *bench) {
    return guarded("hpgl_b200_bench", [&] {
        if (!job || !result || !bench) throw HpglError{HPGL_E_INVALID, "null argument"};
        if (bench->iters < 1 || bench->warmup < 0) throw HpglError{HPGL_E_INVALID, "iters must be >= 1"};
        bench_job(*job, *result, *bench);
    });
}

int hpgl_b200_set_launch(int family, int precision, int schedule, int blocks_per_sm) {
    return guarded("hpgl_b200_set_launch", [&] {
        if (family < 0 || family > 1 || precision < 0 || precision > 1 || schedule < 0 || schedule > 1 ||
            blocks_per_sm < 0)
            throw HpglError{HPGL_E_INVALID, "invalid launch setting"};
        LaunchTuning t;
        t.schedule = schedule;
        t.blocks_per_sm = blocks_per_sm;
        tuning_set(family, precision, t);
    });
}

int hpgl_b200_fma_peak(int precision, double *tflops) {
    return guarded("hpgl_b200_fma_peak", [&] {
        if (precision < 0 || precision > 1 || !tflops) throw HpglError{HPGL_E_INVALID, "invalid arguments"};
        *tflops = fma_peak_tflops(precision, 5);
    });
}

int hpgl_b200_autotune(const hpgl_b200_job_t *job, hpgl_b200_tune_t *report) {
    return guarded("hpgl_b200_autotune", [&] {
        if (!job || !report) throw HpglError{HPGL_E_INVALID, "null argument"};
        autotune_job(*job, *report);
    });
}

hpgl_b200_server_t *hpgl_b200_server_create(const hpgl_b200_server_config_t *config) {
    void *h = nullptr;
    guarded("hpgl_b200_server_create", [&] {
        if (!config) throw HpglError{HPGL_E_INVALID, "config is null"};
        h = server_create(*config);
    });
    return (hpgl_b200_server_t *)h;
}

long long hpgl_b200_server_submit(hpgl_b200_server_t *server, const hpgl_b200_job_t *job,
                                  hpgl_b200_result_t *result) {
    long long t = -1;
    int rc = guarded("hpgl_b200_server_submit", [&] {
        if (!server || !job) throw HpglError{HPGL_E_INVALID, "null argument"};
        t = server_submit(server, *job, result);
    });
    return rc == HPGL_OK ? t : -(long long)rc;
}

int hpgl_b200_server_wait(hpgl_b200_server_t *server, long long ticket, int timeout_ms) {
    int code = -1;
    std::string msg;
    int rc = guarded("hpgl_b200_server_wait", [&] {
        if (!server) throw HpglError{HPGL_E_INVALID, "null server"};
        code = server_wait(server, ticket, timeout_ms, msg);
    });
    if (rc != HPGL_OK) return rc;
    if (code > 0) set_error(code, "hpgl_b200_server job " + std::to_string(ticket) + ": " + msg);
    return code;
}

int hpgl_b200_server_stats(hpgl_b200_server_t *server, hpgl_b200_server_stats_t *stats) {
    return guarded("hpgl_b200_server_stats", [&] {
        if (!server || !stats) throw HpglError{HPGL_E_INVALID, "null argument"};
        server_stats(server, *stats);
    });
}

void hpgl_b200_server_destroy(hpgl_b200_server_t *server) {
    guarded("hpgl_b200_server_destroy", [&] {
        if (server) server_destroy(server);
    });
}

long long hpgl_b200_search_template(const hpgl_ik_params_t *params, int *out_xyz, long long cap) {
    long long n = -1;
    guarded("hpgl_b200_search_template", [&] {
        if (!params || (cap > 0 && !out_xyz)) throw HpglError{HPGL_E_INVALID, "null argument"};
        KrigingParams kp;
        kp.cov_type = params->m_covariance_type;
        for (int i = 0; i < 3; ++i) {
            kp.ranges[i] = params->m_ranges[i];
            kp.angles[i] = params->m_angles[i];
            kp.radii[i] = params->m_radiuses[i];
        }
        kp.sill = params->m_sill;
        kp.nugget = params->m_nugget;
        kp.max_neighbours = params->m_max_neighbours;
        kp.marginal_prob = params->m_marginal_prob;
        const unsigned char informed = 1;
        Plan P;
        try {
            build_plan(P, KIND_SK, 1, 1, 1, kp, &informed, host_threads());
        } catch (const std::domain_error &e) {
            throw HpglError{HPGL_E_UNSUPPORTED, e.what()};
        } catch (const std::invalid_argument &e) {
            throw HpglError{HPGL_E_INVALID, e.what()};
        }
        n = (long long)P.tmpl.size();
        for (long long i = 0; i < n && i < cap; ++i) {
            out_xyz[3 * i] = P.tmpl[i].dx;
            out_xyz[3 * i + 1] = P.tmpl[i].dy;
            out_xyz[3 * i + 2] = P.tmpl[i].dz;
        }
    });
    return n;
}

const char *hpgl_b200_version(void) { return "hpgl_b200 0.1 (sm_100a kriging path)"; }

int hpgl_simple_kriging_weights(float *center_coords, float *neighbours_x, float *neighbours_y, float *neighbours_z,
                                int neighbours_count, hpgl_cov_params_t *params, float *weights) {
    int rc = guarded("hpgl_simple_kriging_weights", [&] {
        sk_weights_alloc(center_coords, neighbours_x, neighbours_y, neighbours_z, neighbours_count, params, weights);
    });
    return rc == HPGL_OK ? 0 : -1;
}

int hpgl_b200_simple_kriging_weights_static(float *center_coords, float *neighbours_x, float *neighbours_y,
                                            float *neighbours_z, int neighbours_count, hpgl_cov_params_t *params,
                                            float *weights) {
    int rc = guarded("hpgl_b200_simple_kriging_weights_static", [&] {
        sk_weights_static(center_coords, neighbours_x, neighbours_y, neighbours_z, neighbours_count, params, weights);
    });
    return rc == HPGL_OK ? 0 : -1;
}

// INC / GSLIB property files (api.cpp:54-193 of the reference; textio.cu).
void hpgl_read_inc_file_float(char *filename, float undefined_value, int size, float *data, unsigned char *mask) {
    guarded_io("hpgl_read_inc_file_float", [&] {
        inc_read(filename, false, undefined_value, 0, size, data, nullptr, mask, nullptr, 0, nullptr);
    });
}
void hpgl_read_inc_file_byte(char *filename, int undefined_value, int size, unsigned char *data, unsigned char *mask,
                             unsigned char *values, int values_count) {
    guarded_io("hpgl_read_inc_file_byte", [&] {
        inc_read(filename, true, 0.f, undefined_value, size, nullptr, data, mask, values, values_count, nullptr);
    });
}
void hpgl_write_inc_file_float(char *filename, hpgl_cont_masked_array_t *arr, float undefined_value, char *name) {
    guarded_io("hpgl_write_inc_file_float", [&] {
        if (!arr) throw HpglError{HPGL_E_INVALID, "hpgl_write_inc_file_float: array is null"};
        prop_write(0, false, filename, name, arr->m_data, nullptr, arr->m_mask, volume(&arr->m_shape), undefined_value,
                   0, nullptr, 0, nullptr);
    });
}
void hpgl_write_inc_file_byte(char *filename, hpgl_ind_masked_array_t *arr, int undefined_value, char *name,
                              unsigned char *values, int values_count) {
    guarded_io("hpgl_write_inc_file_byte", [&] {
        if (!arr) throw HpglError{HPGL_E_INVALID, "hpgl_write_inc_file_byte: array is null"};
        const std::vector<unsigned char> t = remap_table(values, values_count, arr->m_indicator_count);
        prop_write(0, true, filename, name, nullptr, arr->m_data, arr->m_mask, volume(&arr->m_shape), 0.f,
                   (unsigned char)undefined_value, t.data(), (int)t.size(), nullptr);
    });
}
void hpgl_write_gslib_cont_property(hpgl_cont_masked_array_t *data, const char *filename, const char *name,
                                    double undefined_value) {
    guarded_io("hpgl_write_gslib_cont_property", [&] {
        if (!data) throw HpglError{HPGL_E_INVALID, "hpgl_write_gslib_cont_property: array is null"};
        prop_write(1, false, filename, name, data->m_data, nullptr, data->m_mask, volume(&data->m_shape),
                   (float)undefined_value, 0, nullptr, 0, nullptr);
    });
}
void hpgl_write_gslib_byte_property(hpgl_ind_masked_array_t *data, const char *filename, const char *name,
                                    double undefined_value, unsigned char *values, int values_count) {
    guarded_io("hpgl_write_gslib_byte_property", [&] {
        if (!data) throw HpglError{HPGL_E_INVALID, "hpgl_write_gslib_byte_property: array is null"};
        const std::vector<unsigned char> t = remap_table(values, values_count, data->m_indicator_count);
        prop_write(1, true, filename, name, nullptr, data->m_data, data->m_mask, volume(&data->m_shape), 0.f,
                   byte_of_double(undefined_value), t.data(), (int)t.size(), nullptr);
    });
}
long long hpgl_b200_inc_count_values(const char *filename) {
    long long n = -1;
    guarded_io("hpgl_b200_inc_count_values", [&] { n = inc_count(filename, false, nullptr); });
    return n;
}

void hpgl_b200_io_last_timing(hpgl_b200_io_timing_t *out) {
    if (!out) return;
    const TextIoTiming t = last_io_timing();
    out->ms_file = t.ms_file;
    out->ms_h2d = t.ms_h2d;
    out->ms_device = t.ms_device;
    out->ms_d2h = t.ms_d2h;
    out->ms_total = t.ms_total;
    out->bytes = t.bytes;
    out->tokens = t.tokens;
}

// Experimental variograms and layer stacking (the reference's _cvariogram
// library, api.h:91-141 there; variogram.cu).
void fill_ellipsoid_directions(ellipsoid_t *ell, double azimuth, double dip, double rotation) {
    guarded("fill_ellipsoid_directions", [&] {
        if (!ell) throw HpglError{HPGL_E_INVALID, "ellipsoid is null"};
        cv_fill_ellipsoid(ell, azimuth, dip, rotation);
    });
}

void calc_variograms(variogram_search_template_t *templ, hard_data_t *data, float *result_covariations,
                     int result_length, int percentToUse) {
    guarded("calc_variograms", [&] {
        if (!templ || !data || (!result_covariations && result_length > 0))
            throw HpglError{HPGL_E_INVALID, "null argument"};
        const int lags = std::min(templ->m_num_lags, result_length);
        if (lags <= 0) return;
        std::vector<double> sums(lags);
        std::vector<unsigned long long> counts(lags);
        cv_grid(*templ, *data, result_length, percentToUse, sums.data(), counts.data());
        // variograms.cpp:411-414: sum / count / 2, NaN for a lag without pairs
        for (int l = 0; l < lags; ++l) result_covariations[l] = (float)(sums[l] / (double)counts[l] / 2);
    });
}

void calc_variograms_from_point_set(variogram_search_template_t *templ, cont_point_set_t *point_set,
                                    float *result_covariations, int result_length) {
    guarded("calc_variograms_from_point_set", [&] {
        if (!templ || !point_set || (!result_covariations && result_length > 0))
            throw HpglError{HPGL_E_INVALID, "null argument"};
        const int lags = std::min(templ->m_num_lags, result_length);
        if (lags <= 0) return;
        std::vector<double> sums(lags);
        std::vector<unsigned long long> counts(lags);
        cv_points(*templ, *point_set, result_length, sums.data(), counts.data());
        // variograms.cpp:495-500: 0 for a lag without pairs
        for (int l = 0; l < lags; ++l)
            result_covariations[l] = counts[l] == 0 ? 0.f : (float)(sums[l] / (double)counts[l] / 2);
    });
}

void cvar_stack_layers(float_data_t *thick_layers, int *layer_markers, int layers_count, int nz, float scalez,
                       int blank_value, float_data_t *result) {
    guarded("cvar_stack_layers",
            [&] { cv_stack_layers(thick_layers, layer_markers, layers_count, nz, scalez, blank_value, result); });
}

int hpgl_b200_variogram_stats(variogram_search_template_t *templ, hard_data_t *data, cont_point_set_t *points,
                              int result_length, int percentToUse, double *sums, long long *counts) {
    return guarded("hpgl_b200_variogram_stats", [&] {
        if (!templ || !sums || !counts) throw HpglError{HPGL_E_INVALID, "null argument"};
        const int lags = std::min(templ->m_num_lags, result_length);
        if (lags <= 0) return;
        std::vector<unsigned long long> c(lags);
        if (points) cv_points(*templ, *points, result_length, sums, c.data());
        else if (data) cv_grid(*templ, *data, result_length, percentToUse, sums, c.data());
        else throw HpglError{HPGL_E_INVALID, "no data"};
        for (int l = 0; l < lags; ++l) counts[l] = (long long)c[l];
    });
}

// Sequential Gaussian simulation (api.cpp:409-469 of the reference), in
// place on the property.  With a CDF the informed values (and the LVM mean
// cube) are normal-score transformed first and every informed value is
// transformed back at the end (sequential_gaussian_simulation.cpp:32-35,
// 72-73, 97-103, 119-123).
static hpgl_ik_params_t sgs_ik_params(const hpgl_sgs_params_t *p) {
    hpgl_ik_params_t q;
    memset(&q, 0, sizeof(q));
    q.m_covariance_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i) {
        q.m_ranges[i] = p->m_ranges[i];
        q.m_angles[i] = p->m_angles[i];
        q.m_radiuses[i] = p->m_radiuses[i];
    }
    q.m_sill = p->m_sill;
    q.m_nugget = p->m_nugget;
    q.m_max_neighbours = p->m_max_neighbours;
    return q;
}

static void sgs_call(hpgl_cont_masked_array_t *data, hpgl_sgs_params_t *params, hpgl_non_parametric_cdf_t *cdf,
                     const float *lvm_mean, hpgl_ubyte_array_t *simulation_mask) {
    if (!data || !params) throw HpglError{HPGL_E_INVALID, "data or params are null"};
    if (!data->m_data || !data->m_mask) throw HpglError{HPGL_E_INVALID, "property arrays are null"};
    const long long n = volume(&data->m_shape);
    // refuse what the path cannot do before the CDF transform touches the data
    try {
        check_sim_path(n, params->m_seed);
    } catch (const std::domain_error &e) {
        throw HpglError{HPGL_E_UNSUPPORTED, e.what()};
    } catch (const std::invalid_argument &e) {
        throw HpglError{HPGL_E_INVALID, e.what()};
    }
    NonParametricCdf c{nullptr, nullptr, 0};
    std::vector<float> gaussian_mean;
    if (cdf) {
        if (!cdf->m_values || !cdf->m_probs || cdf->m_size <= 0)
            throw HpglError{HPGL_E_INVALID, "the CDF has no values"};
        c = NonParametricCdf{cdf->m_values, cdf->m_probs, cdf->m_size};
        cdf_to_gaussian(c, data->m_data, data->m_data, data->m_mask, n, host_threads());
        if (lvm_mean) {
            gaussian_mean.resize((size_t)n);
            cdf_to_gaussian(c, lvm_mean, gaussian_mean.data(), nullptr, n, host_threads());
            lvm_mean = gaussian_mean.data();
        }
    }
    const hpgl_ik_params_t q = sgs_ik_params(params);
    hpgl_b200_job_t j = base_job(lvm_mean ? HPGL_KIND_LVM
                                          : (params->m_kriging_kind == 1 ? HPGL_KIND_SK : HPGL_KIND_OK),
                                 &data->m_shape);
    j.values = data->m_data;
    j.mask = data->m_mask;
    j.mean = lvm_mean;
    j.params = &q;
    j.n_params = 1;
    j.sequential = 1;
    j.seed = params->m_seed;
    j.simulation_mask = simulation_mask ? simulation_mask->m_data : nullptr;
    hpgl_b200_result_t r;
    memset(&r, 0, sizeof(r));
    r.out_values = data->m_data;
    r.out_mask = data->m_mask;
    run("sequential Gaussian simulation", j, r);
    if (cdf) gaussian_to_cdf(c, data->m_data, data->m_mask, n, host_threads());
}

void hpgl_sgs_simulation(hpgl_cont_masked_array_t *data, hpgl_sgs_params_t *params, hpgl_non_parametric_cdf_t *cdf,
                         double *, hpgl_ubyte_array_t *simulation_mask) {
    // the stationary mean argument is unused: simple kriging runs with mean 0
    // (sequential_gaussian_simulation.cpp:39-41)
    guarded("hpgl_sgs_simulation", [&] { sgs_call(data, params, cdf, nullptr, simulation_mask); });
}

void hpgl_sgs_lvm_simulation(hpgl_cont_masked_array_t *data, hpgl_sgs_params_t *params,
                             hpgl_non_parametric_cdf_t *cdf, hpgl_float_array_t *means,
                             hpgl_ubyte_array_t *simulation_mask) {
    guarded("hpgl_sgs_lvm_simulation", [&] {
        if (!means || !means->m_data) throw HpglError{HPGL_E_INVALID, "mean array is null"};
        sgs_call(data, params, cdf, means->m_data, simulation_mask);
    });
}
// Sequential indicator simulation (api.cpp:517-580 of the reference), in
// place on the codes: one params entry per category; the LVM form takes a
// mean cube per category and, with use_correlograms, the correlogram
// weights (sequential_indicator_simulation.cpp:150-181).
static void sis_call(hpgl_ind_masked_array_t *data, hpgl_ik_params_t *params, int indicator_count, int seed,
                     const hpgl_float_array_t *means, hpgl_ubyte_array_t *simulation_mask, int use_correlograms) {
    if (!data || !params) throw HpglError{HPGL_E_INVALID, "data or params are null"};
    if (!data->m_data || !data->m_mask) throw HpglError{HPGL_E_INVALID, "property arrays are null"};
    if (indicator_count < 1 || indicator_count > 255) throw HpglError{HPGL_E_INVALID, "invalid indicator count"};
    hpgl_b200_job_t j = base_job(HPGL_KIND_IK, &data->m_shape);
    j.codes = data->m_data;
    j.mask = data->m_mask;
    j.params = params;
    j.n_params = indicator_count;
    j.sequential = 1;
    j.seed = seed;
    j.simulation_mask = simulation_mask ? simulation_mask->m_data : nullptr;
    std::vector<const float *> cubes;
    if (means) {
        const long long n = volume(&data->m_shape);
        for (int k = 0; k < indicator_count; ++k) {
            if (!means[k].m_data) throw HpglError{HPGL_E_INVALID, "mean array is null"};
            if (volume(&means[k].m_shape) != n) throw HpglError{HPGL_E_INVALID, "mean array size differs"};
            cubes.push_back(means[k].m_data);
        }
        j.category_means = cubes.data();
        j.correlogram = use_correlograms != 0;
    }
    hpgl_b200_result_t r;
    memset(&r, 0, sizeof(r));
    r.out_codes = data->m_data;
    r.out_mask = data->m_mask;
    run("sequential indicator simulation", j, r);
}

void hpgl_sis_simulation(hpgl_ind_masked_array_t *data, hpgl_ik_params_t *params, int indicator_count, int seed,
                         hpgl_ubyte_array_t *simulation_mask) {
    guarded("hpgl_sis_simulation",
            [&] { sis_call(data, params, indicator_count, seed, nullptr, simulation_mask, 0); });
}
void hpgl_sis_simulation_lvm(hpgl_ind_masked_array_t *data, hpgl_ik_params_t *params, hpgl_float_array_t *mean_data,
                             int indicator_count, int seed, hpgl_ubyte_array_t *simulation_mask,
                             int use_correlograms) {
    guarded("hpgl_sis_simulation_lvm", [&] {
        if (!mean_data) throw HpglError{HPGL_E_INVALID, "mean arrays are null"};
        sis_call(data, params, indicator_count, seed, mean_data, simulation_mask, use_correlograms);
    });
}
// hpgl_simple_cokriging_mark1/2 (api.cpp:587-713 of the reference): the
// three arrays must have the same size (the reference raises otherwise).
static void cokriging_sizes(const hpgl_cont_masked_array_t *a, const hpgl_cont_masked_array_t *b,
                            const hpgl_cont_masked_array_t *c) {
    if (!a || !b || !c) throw HpglError{HPGL_E_INVALID, "null array"};
    if (volume(&a->m_shape) != volume(&b->m_shape))
        throw HpglError{HPGL_E_INVALID, "size of secondary data is different from size of primary data"};
    if (volume(&a->m_shape) != volume(&c->m_shape))
        throw HpglError{HPGL_E_INVALID, "size of output data is different from size of primary data"};
}

void hpgl_simple_cokriging_mark1(hpgl_cont_masked_array_t *input_data, hpgl_cont_masked_array_t *secondary_data,
                                 hpgl_cokriging_m1_params_t *params, hpgl_cont_masked_array_t *output_data) {
    guarded("hpgl_simple_cokriging_mark1", [&] {
        cokriging_sizes(input_data, secondary_data, output_data);
        if (!params) throw HpglError{HPGL_E_INVALID, "params are null"};
        hpgl_ik_params_t p;
        memset(&p, 0, sizeof(p));
        p.m_covariance_type = params->m_covariance_type;
        for (int i = 0; i < 3; ++i) {
            p.m_ranges[i] = params->m_ranges[i];
            p.m_angles[i] = params->m_angles[i];
            p.m_radiuses[i] = params->m_radiuses[i];
        }
        p.m_sill = params->m_sill;
        p.m_nugget = params->m_nugget;
        p.m_max_neighbours = params->m_max_neighbours;
        hpgl_b200_job_t job = base_job(HPGL_KIND_COKRIGING_M1, &input_data->m_shape);
        job.values = input_data->m_data;
        job.mask = input_data->m_mask;
        job.secondary_values = secondary_data->m_data;
        job.secondary_mask = secondary_data->m_mask;
        job.params = &p;
        job.n_params = 1;
        job.primary_mean = params->m_primary_mean;
        job.secondary_mean = params->m_secondary_mean;
        job.secondary_variance = params->m_secondary_variance;
        job.correlation = params->m_correlation_coef;
        hpgl_b200_result_t res;
        memset(&res, 0, sizeof(res));
        res.out_values = output_data->m_data;
        res.out_mask = output_data->m_mask;
        run("Simple Colocated Cokriging Markov Model I", job, res);
    });
}

void hpgl_simple_cokriging_mark2(hpgl_cont_masked_array_t *primary_data, hpgl_cont_masked_array_t *secondary_data,
                                 hpgl_cokriging_m2_params_t *params, hpgl_cont_masked_array_t *output_data) {
    guarded("hpgl_simple_cokriging_mark2", [&] {
        cokriging_sizes(primary_data, secondary_data, output_data);
        if (!params) throw HpglError{HPGL_E_INVALID, "params are null"};
        const hpgl_cov_params_t &pc = params->m_primary_cov_params;
        hpgl_ik_params_t p;
        memset(&p, 0, sizeof(p));
        p.m_covariance_type = pc.m_covariance_type;
        for (int i = 0; i < 3; ++i) {
            p.m_ranges[i] = pc.m_ranges[i];
            p.m_angles[i] = pc.m_angles[i];
            p.m_radiuses[i] = params->m_radiuses[i];
        }
        p.m_sill = pc.m_sill;
        p.m_nugget = pc.m_nugget;
        p.m_max_neighbours = params->m_max_neighbours;
        hpgl_b200_job_t job = base_job(HPGL_KIND_COKRIGING_M2, &primary_data->m_shape);
        job.values = primary_data->m_data;
        job.mask = primary_data->m_mask;
        job.secondary_values = secondary_data->m_data;
        job.secondary_mask = secondary_data->m_mask;
        job.params = &p;
        job.n_params = 1;
        job.primary_mean = params->m_primary_mean;
        job.secondary_mean = params->m_secondary_mean;
        job.correlation = params->m_correlation_coef;
        job.secondary_cov = &params->m_secondary_cov_params;
        hpgl_b200_result_t res;
        memset(&res, 0, sizeof(res));
        res.out_values = output_data->m_data;
        res.out_mask = output_data->m_mask;
        run("Simple Colocated Cokriging Markov Model II", job, res);
    });
}

}  // extern "C"
