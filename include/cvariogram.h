/* C ABI of the experimental-variogram library, as the reference's
   src/geo_bsd/_cvariogram/api.h:1-144 declares it and its Python layer
   (geo_bsd/cvariogram.py:1-200) binds it.  hpgl.so exports these symbols
   beside the kriging ABI of hpgl.h; the variograms are computed on the GPU.
   Structs and signatures are the reference's. */
#ifndef HPGL_B200_CVARIOGRAM_H
#define HPGL_B200_CVARIOGRAM_H

#ifdef __cplusplus
extern "C" {
#endif

/* api.h:24-27 */
struct vector_t {
    double m_data[3];
};

/* api.h:29-37: direction i is column i of Rz(azimuth) Ry(dip) Rx(rotation) */
struct ellipsoid_t {
    struct vector_t m_direction1;
    struct vector_t m_direction2;
    struct vector_t m_direction3;
    double m_R1;
    double m_R2;
    double m_R3;
};

/* api.h:39-47: lags of width m_lag_width centred at m_first_lag_distance +
   k * m_lag_separation, k < m_num_lags; pairs whose separation lies in the
   ellipsoid's tunnel along direction 1 (radii R2, R3, opening m_tol_distance). */
struct variogram_search_template_t {
    double m_lag_width;
    double m_lag_separation;
    double m_tol_distance;
    int m_num_lags;
    double m_first_lag_distance;
    struct ellipsoid_t m_ellipsoid;
};

/* api.h:65-72 */
struct cont_point_set_t {
    float *xs;
    float *ys;
    float *zs;
    float *values;
    int size;
};

/* api.h:74-82: shapes and strides in elements */
struct hard_data_t {
    float *m_data;
    unsigned char *m_mask;
    int m_data_shape[3];
    int m_data_strides[3];
    int m_mask_shape[3];
    int m_mask_strides[3];
};

/* api.h:84-89 */
struct float_data_t {
    float *m_data;
    int m_data_shape[3];
    int m_data_strides[3];
};

/* ellipsoid.cpp:40-72 (host: three rotations, the reference's pi). */
void fill_ellipsoid_directions(struct ellipsoid_t *ell, double azimuth, double dip, double rotation);

/* variograms.cpp:335-417: the semivariance of every lag over all pairs of
   informed cells whose offset lies in the template's tunnel, counted into
   every lag whose window holds the offset's length; a lag without pairs is
   NaN (0/0), as in the reference.  percentToUse < 100 keeps that share of the
   pairs, chosen by a hash of (offset, cell) -- the reference draws rand().
   On the GPU; per-lag pair counts exact, sums exact to 2^-100 relative. */
void calc_variograms(struct variogram_search_template_t *templ, struct hard_data_t *data,
                     float *result_covariations, int result_length, int percentToUse);

/* variograms.cpp:419-503: the same over every ordered pair of points (a
   point with itself included); a lag without pairs is 0. */
void calc_variograms_from_point_set(struct variogram_search_template_t *templ, struct cont_point_set_t *point_set,
                                    float *result_covariations, int result_length);

/* stack_layers.cpp:7-21 / stack_layers.h:5-63: a cube of layer markers from
   thickness maps (negative thickness: blank from the eroded top up). */
void cvar_stack_layers(struct float_data_t *thick_layers, int *layer_markers, int layers_count, int nz, float scalez,
                       int blank_value, struct float_data_t *result);

/* Per-lag pair counts and sums of squared differences of calc_variograms /
   calc_variograms_from_point_set (points != 0: the point-set form, `data`
   unused), for callers that want them; 0 or an HPGL_E_* code (message via
   hpgl_get_last_exception_message). */
int hpgl_b200_variogram_stats(struct variogram_search_template_t *templ, struct hard_data_t *data,
                              struct cont_point_set_t *points, int result_length, int percentToUse,
                              double *sums, long long *counts);

#ifdef __cplusplus
}
#endif
#endif /* HPGL_B200_CVARIOGRAM_H */
