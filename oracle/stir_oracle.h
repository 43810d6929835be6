/*
 * stir_oracle.h -- CPU oracle for the ray-tracing projector pair and the
 * OSMAPOSL sub-iteration of STIR 6.5.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a restatement of STIR's algorithm on the
 * CPU (C++ with OpenMP), used as the parity checker by tests/, by smoke() and
 * as the timed CPU baseline of bench.py.  No product code path links to it.
 *
 * Two precisions are provided:
 *   - FP32 ("_f32"): every expression evaluated in float in the same order as
 *     STIR (the arithmetic STIR itself runs), used for parity;
 *   - FP64 ("_f64"): the same algorithm in double, used to state each
 *     result's error against an FP64 oracle.
 * Each function cites the STIR file:line it restates.
 */
#ifndef STIR_ORACLE_H
#define STIR_ORACLE_H

#include <stdint.h>
#include "../include/stir_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_handle or_handle;

/* precision: 32 or 64 */
or_handle* or_create(const b200rt_geometry* g, int precision, char* err, int errlen);
void or_destroy(or_handle* h);
int64_t or_projdata_size(const or_handle* h);
int64_t or_image_size(const or_handle* h);
int or_num_tof_bins(const or_handle* h);
int or_symmetries_used(const or_handle* h);
int or_num_basic_views(const or_handle* h);

/* row of one bin (basic row transformed by its symmetry operation); returns length or -1 */
int64_t or_get_row(or_handle* h, int seg, int view, int ax, int tang, int tof, int32_t* coords_zyx, double* values,
                   int64_t capacity);
/* sum over all bins of the row length */
int64_t or_total_nnz(or_handle* h, int nthreads);
/* number of distinct basic rows and their total length (fills the cache) */
int64_t or_basic_row_elements(or_handle* h, int nthreads, int64_t* num_basic_rows);

/* Projectors. Arrays in STIR order (image [z][y][x]; projdata ProjDataInMemory order).
   f32 arrays for precision 32 handles, f64 arrays for precision 64 handles. */
int or_forward_project_f32(or_handle* h, const float* image, float* projdata, int subset, int nsub, int nthreads);
int or_back_project_f32(or_handle* h, const float* projdata, float* image, int subset, int nsub, int nthreads);
int or_forward_project_f64(or_handle* h, const double* image, double* projdata, int subset, int nsub, int nthreads);
int or_back_project_f64(or_handle* h, const double* projdata, double* image, int subset, int nsub, int nthreads);

/* Sensitivity of one subset: back-projection of mult (or ones if mult is NULL),
   with the first and last axial position of segment 0 zeroed when
   zero_seg0_end_planes (distributable.cxx:146-158,161-225; ...AndProjData.cxx:1517-1539). */
int or_sensitivity_f32(or_handle* h, const float* mult, float* sens, int subset, int nsub, int zero_seg0_end_planes,
                       int nthreads);

/* One OSMAPOSL sub-iteration (OSMAPOSLReconstruction.cxx:371-516) on `estimate` (in/out).
   additive may be NULL.  sens is the sensitivity used for this subset. */
/* FP64 restatement of the sensitivity and of one OSMAPOSL sub-iteration (no kappa) on a precision-64 handle */
int or_sensitivity_f64(or_handle* h, const float* mult, double* sens, int subset, int nsub, int zero_seg0_end_planes,
                       int nthreads);
int or_osmaposl_update_f64(or_handle* h, double* estimate, const float* y, const float* additive, const double* sens,
                           int subset, int nsub, int subiteration_num, int zero_seg0_end_planes, const b200rt_prior* prior,
                           double min_rel, double max_rel, int nthreads);
int or_osmaposl_update_f32(or_handle* h, float* estimate, const float* y, const float* additive, const float* sens,
                           int subset, int nsub, int subiteration_num, int zero_seg0_end_planes,
                           const b200rt_prior* prior, const float* kappa, float min_rel, float max_rel, int nthreads,
                           int* num_cancelled);

/* The two halves of the update: the numerator A_S^T divide_and_truncate(y, A_S x + a), and the
   division / clamp / multiplication given it (u in/out). */
int or_osmaposl_numerator_f32(or_handle* h, const float* estimate, const float* y, const float* additive, int subset,
                              int nsub, int zero_seg0_end_planes, int nthreads, float* u, int* num_cancelled);
int or_osmaposl_apply_f32(or_handle* h, float* estimate, float* u, const float* sens, int nsub, int subiteration_num,
                          const b200rt_prior* prior, const float* kappa, float min_rel, float max_rel);

/* Poisson log-likelihood of one subset (accumulate_loglikelihood, recon_array_functions.cxx:335-377,
   RPC at ...AndProjData.cxx:1483-1515), FP64 accumulation.  additive / mult may be NULL. */
double or_log_likelihood_f32(or_handle* h, const float* image, const float* y, const float* additive, const float* mult,
                             int subset, int nsub, int zero_seg0_end_planes, int nthreads);

/* A^T [divide_and_truncate(y, A x + a) - m] over one subset (m = mult or ones) */
int or_loglik_gradient_f32(or_handle* h, const float* image, const float* y, const float* additive, const float* mult,
                           int subset, int nsub, int zero_seg0_end_planes, int nthreads, float* gradient);

/* prior Hessian times an image, accumulated into out (QuadraticPrior.cxx:603-688,
   RelativeDifferencePrior.cxx:535-621); image [z][y][x] */
int or_prior_hessian_times_input_f32(const b200rt_prior* prior, const float* image, const float* input,
                                     const float* kappa, int nz, int ny, int nx, float vz, float vy, float vx,
                                     float* out);

/* OSSPS (src/iterative/OSSPS/OSSPSReconstruction.cxx): the precomputed denominator
   A^T divide_and_truncate(A 1, (y n) n) (n: normalisation correction factors or NULL), the Quadratic prior's
   parabolic surrogate curvature, and one sub-iteration (x and denom in/out; sens = total sensitivity). */
int or_ossps_denominator_f32(or_handle* h, const float* y, const float* norm, int nthreads, float* denom);
int or_prior_curvature_f32(const b200rt_prior* prior, const float* kappa, int nz, int ny, int nx, float vz, float vy,
                           float vx, float* out);
int or_ossps_update_f32(or_handle* h, float* x, float* denom, const float* y, const float* additive, const float* mult,
                        const float* sens, int subset, int nsub, int subiteration_num, int start_subiteration_num,
                        int zero_seg0_end_planes, const b200rt_prior* prior, const float* kappa,
                        float relaxation_parameter, float relaxation_gamma, float upper_bound, int nthreads);

/* Prior gradient and value (QuadraticPrior.cxx:233-372, RelativeDifferencePrior.cxx:280-452);
   image [z][y][x]; voxel sizes z,y,x. */
int or_prior_gradient_f32(const b200rt_prior* prior, const float* image, const float* kappa, int nz, int ny, int nx,
                          float vz, float vy, float vx, float* gradient);
double or_prior_value_f32(const b200rt_prior* prior, const float* image, const float* kappa, int nz, int ny, int nx,
                          float vz, float vy, float vx);

/* list-mode objective over events (n x 5 ints: segment, view, axial, tangential, timing; values; additive terms or
   NULL): op 0 out += gradient terms, 1 returns the value, 2 out += Hessian times rhs; *invalid (may be NULL) gets
   the number of events outside the projection data */
double or_listmode_f32(or_handle* h, int op, const int32_t* bins, const float* values, const float* corr, int64_t n,
                       const float* x, const float* rhs, int subset, int nsub, int has_add, float* out,
                       int64_t* invalid);

/* GibbsPenalty<float, potential> (GibbsPenalty.inl): potential 1 Quadratic, 2 Relative Difference;
   op 0 value, 1 gradient, 2 gradient times input, 3 Hessian diagonal, 4 accumulate Hessian times input (out +=),
   5 Hessian of voxel (vz, vy, vx) into out.  Images [z][y][x]; weights [wz][wy][wx]; kappa may be NULL.
   Returns the value (op 0, 2), else 0. */
double or_gibbs_f32(int op, int potential, float beta, float gamma, float epsilon, const float* weights, int wz, int wy,
                    int wx, const float* kappa, const float* image, const float* input, int nz, int ny, int nx, int vz,
                    int vy, int vx, float* out);
/* default weights (x voxel size / distance), 27 or 9 (only_2D) floats; returns the z size */
int or_gibbs_default_weights(float vz, float vy, float vx, int only_2D, float* w);

/* Siddon tracer of one segment (RayTraceVoxelsOnCartesianGrid.cxx:51-269): appends to the
   arrays; returns the number of elements or -1 if capacity is exceeded. */
int64_t or_ray_trace(const float start_zyx[3], const float stop_zyx[3], const float voxel_size_zyx[3],
                     float normalisation_constant, int32_t* coords_zyx, float* values, int64_t capacity);

#ifdef __cplusplus
}
#endif
#endif
