/*
 * hpgl.h — C ABI of the B200 kriging library (hpgl_b200/hpgl.so).
 *
 * The first part re-declares, with identical layouts and signatures, the
 * reference library's kriging interface (HPGL 0.9.9, src/geo_bsd/hpgl/api.h)
 * so that the reference's ctypes layer (src/geo_bsd/hpgl_wrap.py:141-311)
 * can load this library in place of `hpgl.so`.  Each declaration cites the
 * reference line it replaces.  The second part adds entry points with no
 * reference counterpart: an extended kriging call that exposes precision
 * control and per-node side outputs (variance, status, neighbour lists,
 * weights), error codes, and a device-resident benchmark hook.
 *
 * All buffers are caller-owned host memory.  Grids are Fortran ordered:
 * index = x + nx*(y + ny*z).  Output buffers must be pre-filled by the caller
 * with a copy of the input (the reference's Python layer does this,
 * geo.py:232-240): nodes the algorithm leaves alone (ordinary kriging
 * failures) keep that content.  Every call is synchronous and returns only
 * after the results are in the caller's buffers.
 *
 * Errors: the reference functions return void.  Here every entry point
 * catches all errors, records a message for hpgl_get_last_exception_message()
 * and a code for hpgl_get_last_error() (0 = success), and returns.
 */
#ifndef HPGL_B200_HPGL_H
#define HPGL_B200_HPGL_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference structs, api.h:18-146 (same field order and types) ---- */

typedef struct hpgl_shape_t {          /* api.h:18-22 */
    int m_data[3];
    int m_strides[3];                  /* ignored, as in the reference */
} hpgl_shape_t;

typedef struct hpgl_cont_masked_array_t {   /* api.h:24-29 */
    float *m_data;
    unsigned char *m_mask;
    hpgl_shape_t m_shape;
} hpgl_cont_masked_array_t;

typedef struct hpgl_ind_masked_array_t {    /* api.h:31-37 */
    unsigned char *m_data;
    unsigned char *m_mask;
    hpgl_shape_t m_shape;
    int m_indicator_count;
} hpgl_ind_masked_array_t;

typedef struct hpgl_float_array_t {         /* api.h:39-43 */
    float *m_data;
    hpgl_shape_t m_shape;
} hpgl_float_array_t;

typedef struct hpgl_ubyte_array_t {         /* api.h:45-49 */
    unsigned char *m_data;
    hpgl_shape_t m_shape;
} hpgl_ubyte_array_t;

typedef struct hpgl_ok_params_t {           /* api.h:51-60 */
    int m_covariance_type;             /* 0 spherical, 1 exponential, 2 gaussian */
    double m_ranges[3];
    double m_angles[3];                /* degrees */
    double m_sill;
    double m_nugget;
    int m_radiuses[3];
    int m_max_neighbours;
} hpgl_ok_params_t;

typedef struct hpgl_sk_params_t {           /* api.h:62-73 */
    int m_covariance_type;
    double m_ranges[3];
    double m_angles[3];
    double m_sill;
    double m_nugget;
    int m_radiuses[3];
    int m_max_neighbours;
    unsigned char m_automatic_mean;
    double m_mean;
} hpgl_sk_params_t;

typedef struct hpgl_cov_params_t {          /* api.h:75-82 */
    int m_covariance_type;
    double m_ranges[3];
    double m_angles[3];
    double m_sill;
    double m_nugget;
} hpgl_cov_params_t;

typedef struct hpgl_sgs_params_t {          /* api.h:84-96 */
    int m_covariance_type;
    double m_ranges[3];
    double m_angles[3];
    double m_sill;
    double m_nugget;
    int m_radiuses[3];
    int m_max_neighbours;
    int m_kriging_kind;
    long int m_seed;
    int m_min_neighbours;
} hpgl_sgs_params_t;

typedef struct hpgl_median_ik_params_t {    /* api.h:98-108 */
    int m_covariance_type;
    double m_ranges[3];
    double m_angles[3];
    double m_sill;
    double m_nugget;
    int m_radiuses[3];
    int m_max_neighbours;
    double m_marginal_probs[2];
} hpgl_median_ik_params_t;

typedef struct hpgl_ik_params_t {           /* api.h:110-120 */
    int m_covariance_type;
    double m_ranges[3];
    double m_angles[3];
    double m_sill;
    double m_nugget;
    int m_radiuses[3];
    int m_max_neighbours;
    double m_marginal_prob;
} hpgl_ik_params_t;

typedef struct hpgl_cokriging_m1_params_t { /* api.h:122-135 */
    int m_covariance_type;
    double m_ranges[3];
    double m_angles[3];
    double m_sill;
    double m_nugget;
    int m_radiuses[3];
    int m_max_neighbours;
    double m_primary_mean;
    double m_secondary_mean;
    double m_secondary_variance;
    double m_correlation_coef;
} hpgl_cokriging_m1_params_t;

typedef struct hpgl_cokriging_m2_params_t { /* api.h:137-146 */
    hpgl_cov_params_t m_primary_cov_params;
    hpgl_cov_params_t m_secondary_cov_params;
    int m_radiuses[3];
    int m_max_neighbours;
    double m_primary_mean;
    double m_secondary_mean;
    double m_correlation_coef;
} hpgl_cokriging_m2_params_t;

typedef struct hpgl_non_parametric_cdf_t {  /* api.h:148-153 */
    float *m_values;
    float *m_probs;
    long long m_size;
} hpgl_non_parametric_cdf_t;

/* ---- reference entry points, api.h:159-309 ---- */

/* api.h:159-160.  Message of the last failed call ("" after a success). */
char *hpgl_get_last_exception_message(void);

/* api.h:162-166.  Handlers receive the library's log lines / progress. */
void hpgl_set_output_handler(int (*handler)(char *str, void *param), void *param);
void hpgl_set_progress_handler(int (*handler)(char *stage, int percentage, void *param), void *param);

/* api.h:168-169.  Host worker threads of the library (planning steps). */
void hpgl_set_thread_num(int n_threads);
int hpgl_get_thread_num(void);

/* api.h:218-221, implemented by api.cpp:195-231.  Ordinary kriging. */
void hpgl_ordinary_kriging(hpgl_cont_masked_array_t *input_data, hpgl_ok_params_t *params,
                           hpgl_cont_masked_array_t *output_data);

/* api.h:223-230, api.cpp:261-288.  Simple kriging (mean given or automatic). */
void hpgl_simple_kriging(float *input_data, unsigned char *input_mask, hpgl_shape_t *input_data_shape,
                         hpgl_sk_params_t *params, float *output_data, unsigned char *output_mask,
                         hpgl_shape_t *output_data_shape);

/* api.h:242-251, api.cpp:344-383.  Locally varying mean kriging. */
void hpgl_lvm_kriging(float *input_data, unsigned char *input_mask, hpgl_shape_t *input_data_shape,
                      float *mean_data, hpgl_shape_t *mean_data_shape, hpgl_ok_params_t *params,
                      float *output_data, unsigned char *output_mask, hpgl_shape_t *output_data_shape);

/* api.h:267-272, api.cpp:385-406.  Indicator kriging, one params entry per
   category. */
void hpgl_indicator_kriging(hpgl_ind_masked_array_t *in_data, hpgl_ind_masked_array_t *out_data,
                            hpgl_ik_params_t *params, int indicator_count);

/* api.h:274-277, api.cpp:469-515.  Median indicator kriging (2 categories). */
void hpgl_median_ik(hpgl_ind_masked_array_t *in_data, hpgl_median_ik_params_t *params,
                    hpgl_ind_masked_array_t *out_data);

/* api.h:232-240, api.cpp:292-342.  Simple-kriging weights of one point
   from explicit neighbour coordinates, computed on the GPU.  Returns 0, or
   -1 with the last-error state set (singular system, bad arguments, more
   than 1024 neighbours).  With neighbours_count == 0 nothing is written. */
int hpgl_simple_kriging_weights(float *center_coords, float *neighbours_x, float *neighbours_y,
                                float *neighbours_z, int neighbours_count, hpgl_cov_params_t *params,
                                float *weights);

/* Eclipse INC and GSLIB property files (api.h:171-215; api.cpp:54-193 of the
   reference), parsed and formatted on the GPU.  Same arguments, results and
   files as the reference's; on failure the last-error state holds the
   reference's exception text ("read_prop_name: Property name not found.",
   "load_floats_into_vector: Error parsing 'x' string.", ...), where the
   reference's exception would have crossed the C boundary.
   hpgl_read_inc_file_float: `size` values, mask = (value != undefined).
   hpgl_read_inc_file_byte: `size` integer values as bytes, mask = (value !=
   undefined), informed bytes replaced by their index in `values`.
   The writers write every cell of the array's shape in memory order:
   INC = name line, one "%E" / "%d" line per cell, "/" line; GSLIB = "HPGL
   saved GSLIB file", "1", name line, one line per cell.  Byte values are
   written through the table built from `values` (the reference's
   init_remap_table); an informed byte outside that table is an error here. */
void hpgl_read_inc_file_float(char *filename, float undefined_value, int size, float *data, unsigned char *mask);
void hpgl_read_inc_file_byte(char *filename, int undefined_value, int size, unsigned char *data,
                             unsigned char *mask, unsigned char *values, int values_count);
void hpgl_write_inc_file_float(char *filename, hpgl_cont_masked_array_t *arr, float undefined_value, char *name);
void hpgl_write_inc_file_byte(char *filename, hpgl_ind_masked_array_t *arr, int undefined_value, char *name,
                              unsigned char *values, int values_count);
void hpgl_write_gslib_cont_property(hpgl_cont_masked_array_t *data, const char *filename, const char *name,
                                    double undefined_value);
void hpgl_write_gslib_byte_property(hpgl_ind_masked_array_t *data, const char *filename, const char *name,
                                    double undefined_value, unsigned char *values, int values_count);

/* api.h:253-265, 279-309.  Sequential Gaussian simulation (in place on the
   property; `cdf` optional: the normal-score transform around it; `mean`
   unused, simple kriging runs with mean 0, as in the reference) and
   sequential indicator simulation (in place on the codes; one params entry
   per category; the LVM form takes a mean array per category and, with
   use_correlograms, the correlogram weights).  `simulation_mask` optional:
   1 in the cells to simulate.  Results identical to the reference's; grids
   above 10^7 nodes and seeds negative as an int are refused. */
void hpgl_sgs_simulation(hpgl_cont_masked_array_t *prop, hpgl_sgs_params_t *params, hpgl_non_parametric_cdf_t *cdf,
                         double *mean, hpgl_ubyte_array_t *simulation_mask);
void hpgl_sgs_lvm_simulation(hpgl_cont_masked_array_t *data, hpgl_sgs_params_t *params,
                             hpgl_non_parametric_cdf_t *cdf, hpgl_float_array_t *means,
                             hpgl_ubyte_array_t *simulation_mask);
void hpgl_sis_simulation(hpgl_ind_masked_array_t *data, hpgl_ik_params_t *params, int indicator_count, int seed,
                         hpgl_ubyte_array_t *simulation_mask);
void hpgl_sis_simulation_lvm(hpgl_ind_masked_array_t *data, hpgl_ik_params_t *params, hpgl_float_array_t *mean_data,
                             int indicator_count, int seed, hpgl_ubyte_array_t *simulation_mask,
                             int use_correlograms);
void hpgl_simple_cokriging_mark1(hpgl_cont_masked_array_t *input_data, hpgl_cont_masked_array_t *secondary_data,
                                 hpgl_cokriging_m1_params_t *params, hpgl_cont_masked_array_t *output_data);
void hpgl_simple_cokriging_mark2(hpgl_cont_masked_array_t *primary_data, hpgl_cont_masked_array_t *secondary_data,
                                 hpgl_cokriging_m2_params_t *params, hpgl_cont_masked_array_t *output_data);

/* ---- additions (no counterpart in the reference) ---- */

/* 0 after a successful call, else one of HPGL_E_*. */
int hpgl_get_last_error(void);
#define HPGL_OK 0
#define HPGL_E_INVALID 1      /* bad arguments (sizes, params, null pointers) */
#define HPGL_E_CUDA 2         /* CUDA runtime error, or no usable GPU */
#define HPGL_E_UNSUPPORTED 3  /* outside this build (e.g. max_neighbours > 64) */
#define HPGL_E_CAPACITY 4     /* a device capacity limit was exceeded */
#define HPGL_E_INTERNAL 5

/* Arithmetic of the per-node solve used by the reference entry points above
   and by hpgl_b200_krige when its own field is -1.
   HPGL_PRECISION_FP64: the reference's FP64 Cholesky in its exact operation
   order — results bit-identical to the reference's.
   HPGL_PRECISION_MIXED: FP32 factorisation with FP64 iterative refinement;
   systems whose FP32 pivots fail a threshold, or whose refinement does not
   converge, are re-solved with the FP64 path.  Masks are identical to the
   reference's; estimates and variances agree to <= 1e-6 relative.
   The default is HPGL_PRECISION_FP64, or the value of the environment
   variable HPGL_B200_PRECISION ("fp64" / "mixed") at library load. */
#define HPGL_PRECISION_FP64 0
#define HPGL_PRECISION_MIXED 1
void hpgl_b200_set_precision(int precision);
int hpgl_b200_get_precision(void);

/* Sequential simulation runs in speculative rounds: the pending nodes of a
   window of the random path are kriged at once, and a node commits when no
   pending node of lower path rank lies in the part of its search template
   that the search read, so the result is the sequential one.  `window` is
   the number of pending nodes (0: the default 2^18); results do not depend
   on it. */
void hpgl_b200_set_sim_window(int window);

/* Kriging kinds of hpgl_b200_job_t. */
#define HPGL_KIND_OK 0
#define HPGL_KIND_SK 1
#define HPGL_KIND_LVM 2
#define HPGL_KIND_IK 3
#define HPGL_KIND_MEDIAN_IK 4
#define HPGL_KIND_COKRIGING_M1 5  /* colocated simple cokriging, Markov model I */
#define HPGL_KIND_COKRIGING_M2 6  /* colocated simple cokriging, Markov model II */

/* One kriging job for hpgl_b200_krige.  `params` holds `n_params` entries
   (one per category for IK, else 1); hpgl_ik_params_t carries every field
   the kinds need (m_marginal_prob is used by IK only). */
typedef struct hpgl_b200_job_t {
    int kind;
    int nx, ny, nz;
    const float *values;          /* OK / SK / LVM input values */
    const unsigned char *codes;   /* IK / median IK category codes */
    const unsigned char *mask;    /* informed flags */
    const float *mean;            /* LVM mean cube */
    const hpgl_ik_params_t *params;
    int n_params;
    int sk_automatic_mean;        /* SK: compute the mean of informed values */
    double sk_mean;               /* SK: mean when not automatic */
    double median_marginal1;      /* median IK: marginal probability of code 1 */
    int precision;                /* HPGL_PRECISION_*, or -1 for the global one */
    /* colocated simple cokriging (HPGL_KIND_COKRIGING_M1 / _M2): `values` and
       `mask` are the primary property, params[0] its covariance and search;
       always solved in FP64 in the reference's operation order */
    const float *secondary_values;
    const unsigned char *secondary_mask;
    double primary_mean, secondary_mean;
    double secondary_variance;    /* Markov model I: variance of the secondary */
    double correlation;           /* correlation coefficient of the two */
    const hpgl_cov_params_t *secondary_cov;  /* Markov model II: secondary covariance */
    /* sequential simulation: Gaussian (kinds OK, SK with mean 0, LVM) or
       indicator (kind IK, one params entry per category): the uninformed
       nodes inside `simulation_mask` (all when NULL) are simulated along the
       reference's random path for `seed`; always FP64 */
    int sequential;
    long long seed;
    const unsigned char *simulation_mask;
    /* sequential indicator simulation: optional per-category mean cubes
       (n_params pointers) in place of the marginal probabilities, and the
       correlogram weights for them */
    const float *const *category_means;
    int correlogram;
} hpgl_b200_job_t;

/* Outputs of hpgl_b200_krige.  out_values (cont) or out_codes (IK) and
   out_mask are required and must be pre-filled with the input (see above).
   The rest may be NULL.  Per "system slot" = node, or node*K + k for IK with
   categories whose parameters differ (node for IK with identical ones):
   variance     double   kriging variance (-1 when the solve failed)
   status       int8     0 solved, 1 no neighbours, 2 singular, -1 not kriged
   nb_count     int32    neighbour count
   nb_index     int32    neighbour node indices, nb_stride per slot
   weights      double   kriging weights, nb_stride per slot (cokriging: the
                         neighbours' then the secondary's, so nb_stride must
                         be >= max_neighbours + 1)
   probs        float    IK: probability per node*K + k; median IK: per node
   nb_stride must be >= max_neighbours when nb_index or weights is given. */
typedef struct hpgl_b200_result_t {
    float *out_values;
    unsigned char *out_codes;
    unsigned char *out_mask;
    double *variance;
    signed char *status;
    int *nb_count;
    int *nb_index;
    double *weights;
    float *probs;
    int nb_stride;
    /* filled by the call */
    long long systems;            /* kriging systems attempted */
    long long systems_fp64;       /* of those, solved by the FP64 path */
    long long failures;           /* no neighbours + singular */
    double ms_plan;               /* host planning (template, tables, buckets) */
    double ms_h2d;
    double ms_device;             /* device work, CUDA events */
    double ms_d2h;
    double ms_total;              /* wall time of the call */
    long long rounds;             /* sequential simulation: speculative rounds */
} hpgl_b200_result_t;

/* Runs one job on the GPU.  Returns 0 or an HPGL_E_* code (message via
   hpgl_get_last_exception_message). */
int hpgl_b200_krige(const hpgl_b200_job_t *job, hpgl_b200_result_t *result);

/* Device-resident timing of one job: uploads it once, runs `warmup`
   untimed and `iters` timed passes of the device pipeline (search, build,
   solve, estimate) with a write of `flush_bytes` between passes to flush L2,
   and reports per-pass milliseconds in ms_per_iter[iters] (CUDA events on the
   launching stream), the dominant kernel's average launch milliseconds and
   the number of kernel launches per pass.  The job's outputs of the last
   pass are written like hpgl_b200_krige's. */
typedef struct hpgl_b200_bench_t {
    int iters;
    int warmup;
    long long flush_bytes;
    double *ms_per_iter;
    double ms_top_kernel;         /* average duration of the top kernel */
    char top_kernel[64];
    int launches_per_iter;
    long long systems;
    long long systems_fp64;
    double ms_plan;
    double ms_search;             /* average device time of the first group's searches */
    double ms_resolve;            /* ... and of its FP64 re-solve of routed systems */
} hpgl_b200_bench_t;
int hpgl_b200_bench(const hpgl_b200_job_t *job, hpgl_b200_result_t *result, hpgl_b200_bench_t *bench);

/* No counterpart in the reference.  Launch autotuner: runs the job's device
   pass (planned and uploaded once, results discarded) under each candidate
   setting of the per-node kernels -- the fused template-search+solve kernel
   or separate search and solve kernels, and the number of persistent blocks
   per SM -- times each (median of three passes after an L2 flush) and keeps
   the fastest for the job's family (max_neighbours <= 32, or above) and
   precision; every later call of that family and precision in the process
   uses it.  Without a tuning run the separate schedule at full occupancy
   is used.  Returns 0, or -1 with the error recorded. */
#define HPGL_B200_TUNE_MAX 16
typedef struct hpgl_b200_tune_t {
    int candidates;                        /* settings tried */
    int schedule[HPGL_B200_TUNE_MAX];      /* 0 separate search and solve, 1 fused */
    int blocks_per_sm[HPGL_B200_TUNE_MAX]; /* 0 = as many as fit */
    double ms[HPGL_B200_TUNE_MAX];         /* device time of one pass */
    int chosen;                            /* index of the setting now in force */
    int family;                            /* 0: max_neighbours <= 32, 1: above */
    int precision;                         /* HPGL_PRECISION_* tuned */
} hpgl_b200_tune_t;
int hpgl_b200_autotune(const hpgl_b200_job_t *job, hpgl_b200_tune_t *report);
/* No counterpart in the reference.  Sets the launch setting of a family
   (0: max_neighbours <= 32, 1: above) and precision directly (schedule 0
   separate, 1 fused; blocks_per_sm 0 = as many as fit).  Returns 0, or -1
   on invalid arguments. */
int hpgl_b200_set_launch(int family, int precision, int schedule, int blocks_per_sm);

/* No counterpart in the reference.  The measured rate of the CUDA-core pipe
   the solves run on: FP32 (precision 1, packed two-wide multiply-adds) or
   FP64 (precision 0), from a kernel of independent multiply-add chains
   timed alone (best of 5 launches after a warm-up), in TFLOP/s (2 flop per
   multiply-add).  The roofline denominator of the solve kernels.  Returns 0,
   or -1 (see hpgl_get_last_exception_message). */
int hpgl_b200_fma_peak(int precision, double *tflops);

/* No counterpart in the reference.  hpgl_simple_kriging_weights for callers
   that cannot allocate device memory: cudaMalloc and cudaFree synchronise
   the whole device, stalling the caller's other GPU work, and a host
   application that has reserved the GPU's memory for its own pool leaves
   nothing to allocate.  Same arguments, results and error convention as
   hpgl_simple_kriging_weights; it calls no cudaMalloc, cudaFree or other
   allocating routine.  Its scratch is a fixed device array inside the
   library, present on every GPU that loads it until the process exits, sized
   for at most HPGL_B200_STATIC_WEIGHTS_MAX neighbours: larger counts return
   -1 with HPGL_E_CAPACITY.  Each call looks up the array's device address
   on the current device; the first call on a device also loads the library
   there (make that first call before any stream capture).  The copies and
   the kernel run on the calling thread's per-thread default stream.  All
   calls share the array and it keeps the last call's contents; this entry
   point's calls are serialised with each other by a lock inside the library,
   and calls that overlapped on the GPU would race on it. */
#define HPGL_B200_STATIC_WEIGHTS_MAX 256
int hpgl_b200_simple_kriging_weights_static(float *center_coords, float *neighbours_x, float *neighbours_y,
                                            float *neighbours_z, int neighbours_count, hpgl_cov_params_t *params,
                                            float *weights);

/* Serving: continuous batching of kriging jobs (no counterpart in the
   reference).  Jobs are planned on host workers, admitted as soon as a
   stream slot is free and their device footprint fits in the HBM budget,
   and run concurrently on the GPU, each on its own stream; a job that
   arrives while others run starts as soon as one finishes.  Each result is
   exactly what hpgl_b200_krige returns for that job.  The caller keeps the
   job's input arrays and the result's buffers alive until the job completes
   (hpgl_b200_server_wait); the job struct and its params array are copied at
   submission. */
typedef struct hpgl_b200_server_t hpgl_b200_server_t;
typedef struct hpgl_b200_server_config_t {
    long long hbm_budget_bytes;   /* device memory the in-flight jobs may hold */
    int max_inflight;             /* concurrent jobs (streams), 1..64 */
    int worker_threads;           /* host planning/IO threads; 0 = 2 * max_inflight */
} hpgl_b200_server_config_t;
typedef struct hpgl_b200_server_stats_t {
    long long submitted, completed, failed;
    long long systems;            /* kriging systems of the completed jobs */
    double p50_ms, p99_ms, mean_ms; /* submit-to-completion latency */
    double wall_s;                /* first submission to last completion */
    double systems_per_s;
    int peak_inflight;
    long long peak_bytes;
    /* where the completed jobs' time went, means over the jobs: host
       planning, waiting for admission (a stream slot and HBM budget), and
       the run on the device with its copies (upload, kernels, download) */
    double mean_plan_ms, mean_wait_ms, mean_run_ms;
} hpgl_b200_server_stats_t;
/* Returns NULL on error (see hpgl_get_last_exception_message). */
hpgl_b200_server_t *hpgl_b200_server_create(const hpgl_b200_server_config_t *config);
/* Returns a ticket >= 0, or -HPGL_E_* on a rejected submission.  A job whose
   footprint exceeds the whole budget completes with HPGL_E_CAPACITY. */
long long hpgl_b200_server_submit(hpgl_b200_server_t *server, const hpgl_b200_job_t *job,
                                  hpgl_b200_result_t *result);
/* Waits up to timeout_ms (< 0: forever).  Returns the job's HPGL_* code once
   it completed, or -1 when it is still running. */
int hpgl_b200_server_wait(hpgl_b200_server_t *server, long long ticket, int timeout_ms);
int hpgl_b200_server_stats(hpgl_b200_server_t *server, hpgl_b200_server_stats_t *stats);
/* Waits for every submitted job, then releases the server. */
void hpgl_b200_server_destroy(hpgl_b200_server_t *server);

/* The sorted search template this build derives from `params` (host
   planning only, no GPU needed): offsets (dx, dy, dz) in the order the
   search walks them, i.e. the reference's calc_cov_field order
   (covariance_field.h:62-106).  Writes at most `cap` triples to out_xyz and
   returns the template's length (> cap: only the first cap written), or -1
   on error. */
long long hpgl_b200_search_template(const hpgl_ik_params_t *params, int *out_xyz, long long cap);

/* Number of values an INC file holds (value tokens before the first '/'
   outside a comment, or before the end of the file), or -1 on error.  Lets a
   caller size the buffers of hpgl_read_inc_file_float/_byte. */
long long hpgl_b200_inc_count_values(const char *filename);

/* Timings of the calling process's last INC/GSLIB call (or variogram call:
   ms_device = its kernels, tokens = candidate pairs), milliseconds. */
typedef struct {
    double ms_file;   /* reading or writing the file on the host */
    double ms_h2d;    /* host -> device copies */
    double ms_device; /* kernels (CUDA events) */
    double ms_d2h;    /* device -> host copies */
    double ms_total;
    long long bytes;  /* file size (read) or text size (written) */
    long long tokens; /* tokens read, or cells written */
} hpgl_b200_io_timing_t;
void hpgl_b200_io_last_timing(hpgl_b200_io_timing_t *out);

/* Library build and device description, e.g. for logs. */
const char *hpgl_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif /* HPGL_B200_HPGL_H */
