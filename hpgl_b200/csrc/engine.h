// Job execution on the GPU: uploads, device pipeline, downloads.
#pragma once
#include <string>
#include <vector>

#include "../../include/hpgl.h"
#include "plan.h"

namespace hpgl_b200 {

struct HpglError {
    int code;
    std::string message;
};

// Runs a job end to end (host buffers in, host buffers out).
void run_job(const hpgl_b200_job_t &job, hpgl_b200_result_t &res);

// Device-resident timing (see hpgl_b200_bench in include/hpgl.h).
void bench_job(const hpgl_b200_job_t &job, hpgl_b200_result_t &res, hpgl_b200_bench_t &bench);

// Autotuner of the per-node kernels' launch setting (see hpgl_b200_autotune).
void autotune_job(const hpgl_b200_job_t &job, hpgl_b200_tune_t &report);

// Simple-kriging weights of one point (sk_weights.cu).
void sk_weights_alloc(const float *center, const float *xs, const float *ys, const float *zs, int n,
                      const hpgl_cov_params_t *p, float *weights);

// The same without any device allocation (static scratch, sk_weights.cu).
void sk_weights_static(const float *center, const float *xs, const float *ys, const float *zs, int n,
                       const hpgl_cov_params_t *p, float *weights);

// Server (engine.cu); handles are Server* behind void*.
void *server_create(const hpgl_b200_server_config_t &cfg);
long long server_submit(void *h, const hpgl_b200_job_t &job, hpgl_b200_result_t *result);
int server_wait(void *h, long long ticket, int timeout_ms, std::string &message);
void server_stats(void *h, hpgl_b200_server_stats_t &st);
void server_destroy(void *h);

// Measured FMA-loop rate of the FP32 (precision 1) or FP64 (0) CUDA-core
// pipe, TFLOP/s (peak.cu).
double fma_peak_tflops(int precision, int repeats);

int default_precision();
void set_default_precision(int p);
// Window of the speculative simulation rounds (pending nodes per round).
void set_sim_window(int window);

}  // namespace hpgl_b200
