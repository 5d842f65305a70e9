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

// Simple-kriging weights of one point (sk_weights.cu).
void sk_weights_alloc(const float *center, const float *xs, const float *ys, const float *zs, int n,
                      const hpgl_cov_params_t *p, float *weights);

// The same without any device allocation (static scratch, sk_weights.cu).
void sk_weights_static(const float *center, const float *xs, const float *ys, const float *zs, int n,
                       const hpgl_cov_params_t *p, float *weights);

int default_precision();
void set_default_precision(int p);

}  // namespace hpgl_b200
