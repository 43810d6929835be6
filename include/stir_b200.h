/*
 * stir_b200.h -- C ABI of the B200 ray-tracing projector pair and OSMAPOSL
 * sub-iteration for STIR.
 *
 * This is the drop-in boundary a STIR plug-in (a ProjectorByBinPair
 * registered under its own parsing keyword) binds to.  Every entry point uses
 * plain pointers, sizes and status codes; no C++ or torch type crosses it.
 *
 * Conventions
 *  - Every function returns B200RT_OK (0) or a negative status.  The message
 *    of the last failure on a handle is returned by b200rt_last_error().
 *  - Geometry follows STIR: projection data ProjDataInfoCylindrical{NoArcCorr,
 *    ArcCorr} built from Scanner parameters (src/buildblock/ProjDataInfo.cxx),
 *    images VoxelsOnCartesianGrid (src/buildblock/VoxelsOnCartesianGrid.cxx),
 *    matrix ProjMatrixByBinUsingRayTracing
 *    (src/recon_buildblock/ProjMatrixByBinUsingRayTracing.cxx).
 *  - Host arrays use STIR's own memory order:
 *      image       [z][y][x], x fastest (Array<3,float> of VoxelsOnCartesianGrid)
 *      projdata    ProjDataInMemory order: segment 0,+1,-1,+2,-2,... then
 *                  axial position, view, tangential position (tangential fastest)
 *                  (src/buildblock/ProjDataInMemory.cxx:190-235,
 *                   src/buildblock/ProjData.cxx:641-661)
 *  - Device arrays passed to the *_dev entry points use the device layout:
 *      image       [y][x][z], z fastest ("z-columns")
 *      projdata    [segment][view][tangential][axial], axial fastest
 *                  (segments in the order -S..+S)
 *    b200rt_image_to_device_layout() and friends convert between the two.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 */
#ifndef STIR_B200_H
#define STIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B200RT_ABI_VERSION 1
#define B200RT_MAX_SEGMENTS 255

/* status codes */
#define B200RT_OK 0
#define B200RT_ERR_INVALID_ARGUMENT (-1)
#define B200RT_ERR_UNSUPPORTED (-2)
#define B200RT_ERR_CUDA (-3)
#define B200RT_ERR_OUT_OF_MEMORY (-4)
#define B200RT_ERR_STATE (-5)
#define B200RT_ERR_TIMEOUT (-6)
#define B200RT_ERR_TOO_LARGE (-7)

/* back-projection accumulation modes */
#define B200RT_BACKPROJECT_ATOMIC 0        /* scatter with float atomics (fast; order-dependent rounding)  */
#define B200RT_BACKPROJECT_DETERMINISTIC 1 /* fixed-order float sums per work item, combined as 64-bit fixed
                                              point: order-independent, bit-identical from run to run */

/* attenuation modes (BinNormalisationFromAttenuationImage.cxx:138-170) */
#define B200RT_ATTENUATION_FACTORS 0 /* projdata = undo of ones: 1 / exp(A mu), the multiplicative factors */
#define B200RT_ATTENUATION_APPLY 1   /* projdata *= exp(A mu)   (apply: attenuation correction) */
#define B200RT_ATTENUATION_UNDO 2    /* projdata /= exp(A mu)   (undo: attenuate) */
/* normalisation chains (b200rt_normalisation_dev) */
#define B200RT_NORM_FACTORS 0 /* projdata = undo of ones: the multiplicative factors of the chain */
#define B200RT_NORM_APPLY 1   /* apply every term in order (correction)                        */
#define B200RT_NORM_UNDO 2    /* undo every term in order (the model's multiplicative effect)   */
#define B200RT_NORM_PROJDATA 1    /* BinNormalisationFromProjData: factors as projection data   */
#define B200RT_NORM_ATTENUATION 2 /* BinNormalisationFromAttenuationImage: a mu image (1/mm)    */

/* priors (src/recon_buildblock/QuadraticPrior.cxx, RelativeDifferencePrior.cxx) */
#define B200RT_PRIOR_NONE 0
#define B200RT_PRIOR_QUADRATIC 1
#define B200RT_PRIOR_RELATIVE_DIFFERENCE 2

/* OSMAPOSL MAP models (src/iterative/OSMAPOSL/OSMAPOSLReconstruction.cxx:415-456) */
#define B200RT_MAP_ADDITIVE 0
#define B200RT_MAP_MULTIPLICATIVE 1

/*
 * Geometry descriptor: the primary parameters from which STIR derives every
 * projector quantity.  Derived values (azimuthal sampling/offset, m offsets,
 * tan(theta), symmetry tables ...) are computed by the library with STIR's own
 * float arithmetic.
 */
typedef struct b200rt_geometry {
  /* Scanner (src/include/stir/Scanner.h) */
  int32_t num_rings;
  int32_t num_detectors_per_ring;
  float inner_ring_radius_mm;
  float average_depth_of_interaction_mm;
  float ring_spacing_mm;
  float default_bin_size_mm;
  float intrinsic_azimuthal_tilt_rad;
  float timing_resolution_ps;  /* TOF: coincidence timing FWHM, 0 for non-TOF */
  float size_of_timing_pos_ps; /* TOF: width of one unmashed timing position   */
  int32_t max_num_timing_poss; /* TOF: number of unmashed timing positions      */
  /* ProjDataInfoCylindrical (src/include/stir/ProjDataInfoCylindrical.h) */
  int32_t arc_corrected;      /* 0: NoArcCorr (s = R sin(t*pi/ndet)), 1: ArcCorr (s = t*bin) */
  float arccorr_bin_size_mm;  /* only for arc_corrected */
  int32_t num_views;
  int32_t num_tangential_poss;
  int32_t max_segment_num;    /* segments -max..+max */
  int32_t tof_mash_factor;    /* 0: non-TOF data; >0: TOF data with this mashing */
  int32_t min_ring_diff[B200RT_MAX_SEGMENTS]; /* index: segment + max_segment_num */
  int32_t max_ring_diff[B200RT_MAX_SEGMENTS];
  int32_t num_axial_poss[B200RT_MAX_SEGMENTS];
  /* VoxelsOnCartesianGrid (src/include/stir/VoxelsOnCartesianGrid.h) */
  int32_t nz, ny, nx;
  int32_t min_z, min_y, min_x; /* first index of each dimension */
  float voxel_size_z, voxel_size_y, voxel_size_x;
  float origin_z, origin_y, origin_x;
  /* ProjMatrixByBinUsingRayTracing keys (ProjMatrixByBinUsingRayTracing.cxx:75-104) */
  int32_t num_tangential_LORs;
  int32_t restrict_to_cylindrical_FOV;
  int32_t do_symmetry_90degrees_min_phi;
  int32_t do_symmetry_180degrees_min_phi;
  int32_t do_symmetry_swap_segment;
  int32_t do_symmetry_swap_s;
  int32_t do_symmetry_shift_z;
  /* TOF kernel cut-off.  0: STIR's (ProjMatrixByBin.inl:187-197: a timing bin gets 0 when both its ends lie at
   * least 4 sqrt(2) sigma = 5.66 sigma from the voxel on the same side, otherwise the whole Gaussian's integral over
   * the bin).  k > 0 (no STIR counterpart): the Gaussian truncated at +-k sigma, each timing bin getting the integral
   * of the kernel over its part of [-k sigma, k sigma], not renormalised. */
  float tof_kernel_truncation_sigmas;
} b200rt_geometry;

/* sizes and statistics of a set-up projector */
typedef struct b200rt_info {
  int64_t num_bins;          /* projection-data elements (all TOF bins)          */
  int64_t num_image_voxels;  /* nz*ny*nx                                         */
  int64_t num_basic_bins;    /* rows traced (STIR's basic bins)                  */
  int64_t num_row_elements;  /* stored elements of all basic rows                */
  int64_t total_nnz;         /* sum over all bins of their row length            */
  int32_t num_tof_bins;      /* 1 for non-TOF                                    */
  int32_t num_basic_views;
  int32_t symmetries_used;   /* bit 0: 90-phi, 1: 180-phi, 2: swap seg, 3: swap s, 4: shift z */
  int32_t reserved;
} b200rt_info;

typedef struct b200rt_prior {
  int32_t type;              /* B200RT_PRIOR_*                                   */
  float penalisation_factor; /* beta                                             */
  float gamma;               /* RDP gamma (STIR default 2)                       */
  float epsilon;             /* RDP epsilon (STIR default 0)                     */
  int32_t only_2D;           /* 1: 3x3 in-plane neighbourhood only               */
  int32_t map_model;         /* B200RT_MAP_*                                     */
  const float* kappa_dev;    /* optional kappa image (device layout) or NULL     */
} b200rt_prior;

typedef struct b200rt_projector b200rt_projector;

/* ---- life cycle --------------------------------------------------------- */

/* ProjectorByBinPair::set_up (src/include/stir/recon_buildblock/ProjectorByBinPair.h:60)
 * together with ProjMatrixByBinUsingRayTracing::set_up
 * (src/recon_buildblock/ProjMatrixByBinUsingRayTracing.cxx:238-407): validates the
 * geometry with STIR's rules, derives the symmetry tables and traces every
 * basic row on `device` (STIR's basic-bin cache, ProjMatrixByBin.inl:48-113). */
int b200rt_create(const b200rt_geometry* geometry, int device, b200rt_projector** out);
void b200rt_destroy(b200rt_projector* h);
/* message of the last failure on h (or of the last failed b200rt_create if h is NULL) */
const char* b200rt_last_error(const b200rt_projector* h);
int b200rt_get_info(const b200rt_projector* h, b200rt_info* out);
/* size in elements of projection data / image for this geometry */
int64_t b200rt_projdata_size(const b200rt_projector* h);
int64_t b200rt_image_size(const b200rt_projector* h);

/* One basic row (ProjMatrixByBin::get_proj_matrix_elems_for_one_bin,
 * src/include/stir/recon_buildblock/ProjMatrixByBin.inl:48-113) of bin
 * (segment, view, axial, tangential, timing): copies up to `capacity` elements
 * as (z,y,x) triples and values into host arrays; returns the row length
 * through *length.  Used by tests to compare rows with STIR's. */
int b200rt_get_row(b200rt_projector* h, int segment, int view, int axial, int tangential, int timing,
                   int32_t* coords_zyx, float* values, int64_t capacity, int64_t* length);

/* ---- layout conversion (device to device) ------------------------------- */
int b200rt_image_to_device_layout(b200rt_projector* h, const float* stir_dev, float* dev, void* stream);
int b200rt_image_from_device_layout(b200rt_projector* h, const float* dev, float* stir_dev, void* stream);
int b200rt_projdata_to_device_layout(b200rt_projector* h, const float* stir_dev, float* dev, void* stream);
int b200rt_projdata_from_device_layout(b200rt_projector* h, const float* dev, float* stir_dev, void* stream);

/* Viewgrams of device-layout projection data: the viewgram API of ForwardProjectorByBin / BackProjectorByBin
 * served from device buffers, as ForwardProjectorByBinParallelproj::actual_forward_project serves the related
 * viewgrams from the projection that set_input made (ForwardProjectorByBinParallelproj.cxx:128-145) and
 * BackProjectorByBinParallelproj::actual_back_project stores them for get_output's back projection
 * (BackProjectorByBinParallelproj.cxx:313-328).  A viewgram is STIR's Viewgram<float> of (segment, view, timing
 * position): [axial_pos][tangential_pos] floats.  `viewgram` may be host or device memory; with host memory the
 * call synchronises `stream` before it returns.  set: accumulate = 0 overwrites the viewgram, 1 adds to it.
 * B200RT_ERR_INVALID_ARGUMENT for a segment, view or timing position outside the projector's data. */
int b200rt_get_viewgram(b200rt_projector* h, const float* projdata_dev, int segment_num, int view_num,
                        int timing_pos_num, float* viewgram, void* stream);
int b200rt_set_viewgram(b200rt_projector* h, float* projdata_dev, int segment_num, int view_num, int timing_pos_num,
                        const float* viewgram, int accumulate, void* stream);

/* ---- projectors on device-resident data (device layouts) ---------------- */

/* ForwardProjectorByBin::forward_project(ProjData&, image, subset_num, num_subsets, zero)
 * (src/include/stir/recon_buildblock/ForwardProjectorByBin.h:108): writes the
 * bins of the views in subset `subset_num` of `num_subsets`
 * (detail::find_basic_vs_nums_in_subset, find_basic_vs_nums_in_subset.cxx:32-70);
 * num_subsets=1 projects everything.  Bins of other subsets are left as they are. */
int b200rt_forward_project_dev(b200rt_projector* h, const float* image_dev, float* projdata_dev,
                               int subset_num, int num_subsets, void* stream);

/* BackProjectorByBin::back_project(image, const ProjData&, subset_num, num_subsets)
 * (src/include/stir/recon_buildblock/BackProjectorByBin.h:111): image_dev is
 * overwritten with A^T of the subset's bins. */
int b200rt_back_project_dev(b200rt_projector* h, const float* projdata_dev, float* image_dev,
                            int subset_num, int num_subsets, int mode, void* stream);

/* ---- objective function and OSMAPOSL on device-resident data ----------- */

/* Sensitivity of one subset: A^T m over the subset's bins, m = mult_dev (device layout) or ones
 * when mult_dev is NULL, with the first and last axial position of segment 0 set to zero when
 * zero_seg0_end_planes (PoissonLogLikelihoodWithLinearModelForMeanAndProjData::add_subset_sensitivity,
 * src/recon_buildblock/PoissonLogLikelihoodWithLinearModelForMeanAndProjData.cxx:826-910, via
 * RPC_process_related_viewgrams_sensitivity_computation :1517-1539).  sens_dev is overwritten.
 * back_projection_mode: B200RT_BACKPROJECT_ATOMIC or _DETERMINISTIC. */
int b200rt_sensitivity_dev(b200rt_projector* h, const float* mult_dev, float* sens_dev, int subset_num, int num_subsets,
                           int zero_seg0_end_planes, int back_projection_mode, void* stream);

/* One OSMAPOSL sub-iteration on estimate_dev (in/out):
 * OSMAPOSLReconstruction::update_estimate (src/iterative/OSMAPOSL/OSMAPOSLReconstruction.cxx:371-516)
 * with the gradient of compute_sub_gradient_without_penalty_plus_sensitivity
 * (RPC_process_related_viewgrams_gradient<true>, ...AndProjData.cxx:1421-1481):
 *   u = A_S^T divide_and_truncate(y, A_S x + a);  u /= sens (or the MAP-OSL denominator of `prior`);
 *   u clamped to [min_rel, max_rel] unless subiteration_num == 1;  x *= u.
 * additive_dev may be NULL; prior may be NULL (no penalty).  update_dev (may be NULL) receives u.
 * The forward projection, the ratio and the count of cancelled singularities are one kernel. */
int b200rt_osmaposl_subiteration_dev(b200rt_projector* h, float* estimate_dev, const float* y_dev, const float* additive_dev,
                                     const float* sens_dev, int subset_num, int num_subsets, int subiteration_num,
                                     int zero_seg0_end_planes, const b200rt_prior* prior, float min_relative_change,
                                     float max_relative_change, int back_projection_mode, float* update_dev, void* stream);
/* The two halves of b200rt_osmaposl_subiteration_dev, for callers that combine partial numerators
 * (e.g. several GPUs each projecting part of a subset, then summing u with an all-reduce):
 *   numerator:    u = A_S^T divide_and_truncate(y, A_S x + a)   (numerator_dev overwritten)
 *   apply_update: u /= sens (or the MAP-OSL denominator), clamp unless subiteration_num == 1, x *= u. */
int b200rt_osmaposl_numerator_dev(b200rt_projector* h, const float* estimate_dev, const float* y_dev,
                                  const float* additive_dev, int subset_num, int num_subsets, int zero_seg0_end_planes,
                                  int back_projection_mode, float* numerator_dev, void* stream);
int b200rt_osmaposl_apply_update_dev(b200rt_projector* h, float* estimate_dev, float* numerator_dev, const float* sens_dev,
                                     int num_subsets, int subiteration_num, const b200rt_prior* prior,
                                     float min_relative_change, float max_relative_change, void* stream);

/* singularities cancelled by divide_and_truncate in the last sub-iteration (distributable.cxx:590-594); synchronises */
int b200rt_get_num_cancelled(b200rt_projector* h, int64_t* out);

/* The projector's device status word since creation or the last clear (no STIR counterpart: STIR's projectors run
 * on the host).  B200RT_STATUS_STAGING_TIMEOUT: a forward projection's bulk copy of image columns into shared memory
 * was not seen to complete within the kernel's wait limit, so that launch abandoned some path items and its
 * results are incomplete.  Synchronises; clear != 0 resets the word after reading it. */
#define B200RT_STATUS_STAGING_TIMEOUT 1u
int b200rt_get_device_status(b200rt_projector* h, uint32_t* status, int clear);

/* Poisson log-likelihood of one subset (accumulate_loglikelihood, src/buildblock/recon_array_functions.cxx:335-377,
 * RPC_process_related_viewgrams_accumulate_loglikelihood, ...AndProjData.cxx:1483-1515):
 * sum over bins of y log(ybar') - ybar', ybar' = max((A x + a) m, y/1e4), in FP64 with a fixed
 * summation order.  additive_dev and mult_dev may be NULL.  Synchronises and writes *out. */
int b200rt_log_likelihood_dev(b200rt_projector* h, const float* image_dev, const float* y_dev, const float* additive_dev,
                              const float* mult_dev, int subset_num, int num_subsets, int zero_seg0_end_planes, double* out,
                              void* stream);

/* Gradient of the subset log-likelihood:
 *   A_S^T [ divide_and_truncate(y, A_S x + a) - m ],  m = mult_dev or ones
 * (compute_sub_gradient_without_penalty, RPC_process_related_viewgrams_gradient<false>,
 * src/recon_buildblock/PoissonLogLikelihoodWithLinearModelForMeanAndProjData.cxx:1421-1481).  The
 * projection A x is recomputed here, never stored by the caller.  gradient_dev is overwritten. */
int b200rt_log_likelihood_gradient_dev(b200rt_projector* h, const float* image_dev, const float* y_dev,
                                       const float* additive_dev, const float* mult_dev, int subset_num, int num_subsets,
                                       int zero_seg0_end_planes, int back_projection_mode, float* gradient_dev,
                                       void* stream);

/* Prior value (QuadraticPrior::compute_value, src/recon_buildblock/QuadraticPrior.cxx:233-298;
 * RelativeDifferencePrior::compute_value, src/recon_buildblock/RelativeDifferencePrior.cxx:302-370), FP64 with a
 * fixed summation order.  Synchronises and writes *out. */
int b200rt_prior_value_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev, double* out,
                           void* stream);

/* View shard: the projector holds the projection data of `views` only (slot i = views[i]), in the device layout
 * [segment][slot][tangential][axial]; every projection-data array passed afterwards (y, additive, multiplicative
 * factors, projections) has that shard's size (b200rt_projdata_size).  Projections, sensitivities, the OSMAPOSL
 * numerator and update, the log-likelihood and its gradient, attenuation and normalisation then cover the bins of
 * those views only (lines of other views are skipped, and path items without a line in the shard); summed over
 * shards that partition the views they give the whole data's result.  For the multi-GPU reconstruction that keeps
 * only its share of y, a and m on each GPU (the data partition of STIR's MPI build, distributed.cxx:161-225).
 * Needs the column-staged kernels (non-TOF data; B200RT_ERR_UNSUPPORTED otherwise).  Entry points that address the
 * whole data (host buffers, layout conversions, viewgrams, streams, list mode, OSSPS, batches, the allocation-free
 * log-likelihood) return B200RT_ERR_STATE on a shard.  views = NULL or num_views = 0 restores the whole data. */
int b200rt_set_view_shard(b200rt_projector* h, const int32_t* views, int num_views);

/* A batch of images through one projector (no STIR counterpart: STIR projects one image at a time; the batches of
 * torch.autograd and of noise realisations).  Image b is at images_dev + b*image_stride (device layout), its
 * projection data at projdata_dev + b*projdata_stride; strides in floats, at least an image / the projection data.
 * Where the column-staged kernels apply (non-TOF projectors) each call is one launch over (path item, image);
 * otherwise, and for the deterministic back projection, the images go one at a time.  Results equal the
 * single-image entry points' (the forward bit for bit; the atomic back projection to the order of float additions).
 * Replaces a loop over ForwardProjectorByBin::forward_project / BackProjectorByBin::back_project
 * (src/recon_buildblock/ForwardProjectorByBin.cxx:168-230, BackProjectorByBin.cxx:182-229). */
int b200rt_forward_project_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                     float* projdata_dev, int64_t projdata_stride, int batch, int subset_num,
                                     int num_subsets, void* stream);
int b200rt_back_project_batch_dev(b200rt_projector* h, const float* projdata_dev, int64_t projdata_stride,
                                  float* images_dev, int64_t image_stride, int batch, int subset_num, int num_subsets,
                                  int back_projection_mode, void* stream);
/* b200rt_log_likelihood_dev / b200rt_log_likelihood_gradient_dev of every image of a batch: the data of image b at
 * y_dev + b*y_stride (additive, mult likewise; a stride of 0 shares one array across the batch; additive and mult
 * may be NULL).  values[batch] are written on the host (synchronises); gradient b at gradients_dev +
 * b*gradient_stride. */
int b200rt_log_likelihood_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                    const float* y_dev, int64_t y_stride, const float* additive_dev,
                                    int64_t additive_stride, const float* mult_dev, int64_t mult_stride, int batch,
                                    int subset_num, int num_subsets, int zero_seg0_end_planes, double* values,
                                    void* stream);
/* The log-likelihood of every image of the batch (as b200rt_log_likelihood_batch_dev, the same sums in the same
 * order) and, from the same projection, each image's gradient ratio divide_and_truncate(y, A x + a) - m written to
 * ratio_dev + b * ratio_stride (device layout; bins outside the subset are not written), so that the gradient is then
 * one b200rt_back_project_batch_dev of the ratios, without projecting again.  No STIR counterpart: STIR computes
 * the value (accumulate_loglikelihood, ...AndProjData.cxx:1483-1515) and the sub-gradient (:1421-1481) in separate
 * passes.  Column-staged projectors only (B200RT_ERR_UNSUPPORTED otherwise).  Synchronises and writes values[b]. */
int b200rt_log_likelihood_and_ratio_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                               const float* y_dev, int64_t y_stride, const float* additive_dev,
                                               int64_t additive_stride, const float* mult_dev, int64_t mult_stride,
                                               int batch, int subset_num, int num_subsets, int zero_seg0_end_planes,
                                               double* values, float* ratio_dev, int64_t ratio_stride, void* stream);
int b200rt_log_likelihood_gradient_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                             const float* y_dev, int64_t y_stride, const float* additive_dev,
                                             int64_t additive_stride, const float* mult_dev, int64_t mult_stride,
                                             int batch, int subset_num, int num_subsets, int zero_seg0_end_planes,
                                             int back_projection_mode, float* gradients_dev, int64_t gradient_stride,
                                             void* stream);

/* Allocation-free variant of b200rt_log_likelihood_dev.  No counterpart in the reference.
 * For callers that must not allocate device memory once they are set up: for example a
 * reconstruction service that hands all device memory to a caching allocator at start-up, or
 * that cannot afford the device-wide synchronisation a cudaMalloc/cudaFree implies in the middle
 * of a frame.  This call allocates nothing and copies nothing from the host: the subset's work list
 * and view list are selected on the device from tables made by b200rt_create, and its scratch (those
 * lists, the viewgram thresholds and one FP64 partial sum per work item) lives in a fixed 2.02 MiB
 * array compiled into the library, which every GPU that loads the library holds until the process
 * exits.  It runs the same kernel on the same work items as b200rt_log_likelihood_dev (path items,
 * or basic bins with all their timing bins for a TOF projector), so the two agree to the last bit.
 *   - limits: at most 131072 work items in the subset (path items, or basic bins), 4096 views of the
 *     subset, and 131072 viewgrams in the data (num_tof_bins * (2*max_segment_num+1) * num_views);
 *     larger requests return B200RT_ERR_TOO_LARGE with the counts in b200rt_last_error;
 *   - the result is written to out_dev, a device double the caller provides; the call is
 *     asynchronous on `stream` and does not synchronise;
 *   - all calls share the one array: calls that overlap on the GPU (other streams, other threads)
 *     race and corrupt each other's results;
 *   - the first call on a device looks up the array's device address (cudaGetSymbolAddress) and
 *     keeps it for the life of the process; make that first call before any stream capture, and do
 *     not reset the device (cudaDeviceReset) between calls. */
int b200rt_log_likelihood_dev_noalloc(b200rt_projector* h, const float* image_dev, const float* y_dev,
                                      const float* additive_dev, const float* mult_dev, int subset_num, int num_subsets,
                                      int zero_seg0_end_planes, double* out_dev, void* stream);

/* Prior gradient (QuadraticPrior::compute_gradient, src/recon_buildblock/QuadraticPrior.cxx:303-372;
 * RelativeDifferencePrior::compute_gradient, src/recon_buildblock/RelativeDifferencePrior.cxx:376-452),
 * images in device layout. */
int b200rt_prior_gradient_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev, float* gradient_dev,
                              void* stream);

/* BinNormalisationFromAttenuationImage on device-resident projection data (all bins, device layout):
 * the line integrals A mu of the attenuation image mu_dev (device layout, 1/mm) by this projector, then
 * `mode` (B200RT_ATTENUATION_*) with exp as STIR's in_place_exp.  Replaces set_up + apply/undo
 * (src/recon_buildblock/BinNormalisationFromAttenuationImage.cxx:122-170); non-TOF only, as STIR. */
int b200rt_attenuation_dev(b200rt_projector* h, const float* mu_dev, float* projdata_dev, int mode, void* stream);

/* One term of a normalisation chain: B200RT_NORM_PROJDATA with factors in device layout (non_tof = 1: factors of
 * the non-TOF data serving every timing bin, as BinNormalisationFromProjData allows), or B200RT_NORM_ATTENUATION
 * with a device-layout mu image. */
typedef struct b200rt_norm_term {
  int32_t kind;          /* B200RT_NORM_PROJDATA or B200RT_NORM_ATTENUATION */
  int32_t non_tof;       /* projection-data factors without timing bins    */
  const float* data_dev; /* the factors or the mu image                    */
} b200rt_norm_term;

/* ChainedBinNormalisation (src/recon_buildblock/ChainedBinNormalisation.cxx:91-143) of num_terms terms
 * (BinNormalisationFromProjData.cxx:131-150, BinNormalisationFromAttenuationImage.cxx:138-170) on
 * device-resident projection data (all bins, device layout): mode B200RT_NORM_APPLY applies the terms in order,
 * B200RT_NORM_UNDO undoes them in order (as ChainedBinNormalisation::undo), B200RT_NORM_FACTORS writes the undo
 * of ones (the multiplicative factors m of the Poisson model).  Attenuation terms need non-TOF data, as STIR. */
int b200rt_normalisation_dev(b200rt_projector* h, const b200rt_norm_term* terms, int num_terms, int mode,
                             float* projdata_dev, void* stream);

/* accumulate_Hessian_times_input of the prior (QuadraticPrior.cxx:603-688, RelativeDifferencePrior.cxx:535-621):
 * output += beta sum_k w_jk (f20(x_j, x_k) in_j + f11(x_j, x_k) in_k) (kappa_j kappa_k) at x = image_dev;
 * device layout images. */
int b200rt_prior_hessian_times_input_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev,
                                         const float* input_dev, float* output_dev, void* stream);

/* ---- OSSPS (src/iterative/OSSPS/OSSPSReconstruction.cxx) on device-resident data ---- */
/* precompute_denominator_of_conditioner_without_penalty (OSSPSReconstruction.cxx:184-221): minus the
 * approximate Hessian of the log-likelihood times ones, A^T divide_and_truncate(A 1, (y n) n) over all bins
 * (...AndProjData.cxx:955-1064), n = the normalisation's correction factors (NULL: none). */
int b200rt_ossps_denominator_dev(b200rt_projector* h, const float* y_dev, const float* norm_dev, float* denominator_dev,
                                 int back_projection_mode, void* stream);
/* OSSPSReconstruction::update_estimate (OSSPSReconstruction.cxx:284-410) on estimate_dev: at the first
 * sub-iteration (subiteration_num == start_subiteration_num) voxels with zero sensitivity (sens_dev: the total
 * sensitivity) are zeroed and denominator_dev is completed with 2 x the Quadratic prior's parabolic surrogate
 * curvature and thresholded to positive values, in place; then
 *   x += relax * (num_subsets * (g - prior_gradient / num_subsets)) / denominator, clamped to [0, upper_bound],
 * g = A_S^T [divide_and_truncate(y, A_S x + a) - m], relax = relaxation_parameter /
 * (1 + relaxation_gamma * (subiteration_num / num_subsets)).  prior: NULL, none or Quadratic. */
int b200rt_ossps_subiteration_dev(b200rt_projector* h, float* estimate_dev, float* denominator_dev, const float* y_dev,
                                  const float* additive_dev, const float* mult_dev, const float* sens_dev,
                                  int subset_num, int num_subsets, int subiteration_num, int start_subiteration_num,
                                  int zero_seg0_end_planes, const b200rt_prior* prior, float relaxation_parameter,
                                  float relaxation_gamma, float upper_bound, int back_projection_mode, void* stream);

/* ---- projectors on host arrays in STIR order (copies included) ---------- */
int b200rt_forward_project(b200rt_projector* h, const float* image_host, float* projdata_host,
                           int subset_num, int num_subsets);
int b200rt_back_project(b200rt_projector* h, const float* projdata_host, float* image_host,
                        int subset_num, int num_subsets, int mode);

/* ---- batched OSMAPOSL: several reconstructions per launch ---------------
 * STIR reconstructs the frames of a dynamic study one at a time (one OSMAPOSLReconstruction,
 * OSMAPOSLReconstruction.cxx:371-516, per frame); there is no batch interface to replace.  A batch
 * holds any number of reconstructions ("frames"), each with its own projector (image size), data,
 * sensitivities, subset count and prior.  Batched sub-iteration k advances every frame with
 * num_subiterations >= k by its own sub-iteration k, subset (start_subset + k - 1) % num_subsets, with
 * the result of b200rt_osmaposl_subiteration_dev (atomic back projection) up to float rounding.  Per k:
 * one persistent forward launch (ratio epilogue) and one persistent back projection cover every
 * frame's subset, and the frames' updates run as three launches over all frames; the data thresholds of
 * divide_and_truncate are computed once per b200rt_batch_run call.  Projectors passed to
 * add_frame must outlive the batch and are not used concurrently by the caller while it runs. */
typedef struct b200rt_batch b200rt_batch;

typedef struct {
  int ctas_per_sm_forward; /* persistent CTAs per SM; 0 = as many as fit */
  int ctas_per_sm_back;
  int order;               /* work order: 0 = frame by frame in basic-bin order, 1 = frame by frame, longest rows
                            * first, 2 = item by item across the frames of one geometry and subset */
  int kernels;             /* kernel family, B200RT_BATCH_KERNELS_* */
} b200rt_batch_config;
/* Kernel families of the batched projectors (how the work of a frame is cut into work items):
 * AUTO: the first the frames allow of PATHS, TOF_GROUPED, PACKED, BASIC_BINS;
 * PATHS: one CTA per (frame, path item), the image columns of the path staged in shared memory, lanes on axial
 *   positions (every frame's projector has path tables; the only family for deterministic frames);
 * TOF_GROUPED: one warp per (frame, basic bin) with all its timing bins in registers, lanes on (line, axial
 *   position) (TOF frames with one timing-bin count);
 * PACKED: one warp per (frame, basic bin or TOF bin), lanes on (line, axial position) (at most 16 axial positions);
 * BASIC_BINS: one CTA per (frame, basic bin or TOF bin), one warp per related line, lanes on axial positions. */
#define B200RT_BATCH_KERNELS_AUTO 0
#define B200RT_BATCH_KERNELS_PATHS 1
#define B200RT_BATCH_KERNELS_TOF_GROUPED 2
#define B200RT_BATCH_KERNELS_PACKED 3
#define B200RT_BATCH_KERNELS_BASIC_BINS 4

int b200rt_batch_create(int device, b200rt_batch** out);
void b200rt_batch_destroy(b200rt_batch* b);
const char* b200rt_batch_last_error(const b200rt_batch* b);
/* sensitivity_devs[num_subsets]: one image per subset (device layout; entries may repeat).
 * additive_dev and prior may be NULL.  *frame receives the frame's index. */
int b200rt_batch_add_frame(b200rt_batch* b, b200rt_projector* h, float* estimate_dev, const float* y_dev,
                           const float* additive_dev, const float* const* sensitivity_devs, int num_subsets,
                           int start_subset, int num_subiterations, int zero_seg0_end_planes, const b200rt_prior* prior,
                           float min_relative_change, float max_relative_change, int* frame);
/* Back projection of a frame: B200RT_BACKPROJECT_ATOMIC (the default) or B200RT_BACKPROJECT_DETERMINISTIC, whose
 * numerator is the same 64-bit fixed-point sum as b200rt_osmaposl_subiteration_dev's in that mode (scale from the
 * ratio's bound 1e4), so the frame's reconstruction is bit-reproducible and equal to its own one-frame run.
 * Deterministic frames need the column-staged kernels (non-TOF projectors; B200RT_ERR_UNSUPPORTED otherwise). */
int b200rt_batch_set_frame_mode(b200rt_batch* b, int frame, int back_projection_mode);
int b200rt_batch_num_frames(const b200rt_batch* b);
/* Runs batched sub-iterations first..first+count-1 on `stream`.  use_graph != 0: the sequence is
 * captured once into a CUDA graph (kept per (first, count) until a frame is added or the
 * configuration changes) and launched as one graph. */
int b200rt_batch_run(b200rt_batch* b, int first_subiteration, int count, int use_graph, void* stream);
/* Times the batched projectors of sub-iteration `subiteration` for each configuration the frames allow (kernel
 * family, CTAs per SM, work order), keeps the fastest and writes it to *out (may be NULL).  Estimates are not
 * changed; synchronises. */
int b200rt_batch_autotune(b200rt_batch* b, int subiteration, b200rt_batch_config* out);
int b200rt_batch_set_config(b200rt_batch* b, const b200rt_batch_config* config);
int b200rt_batch_get_config(const b200rt_batch* b, b200rt_batch_config* out);
/* cancelled singularities of one frame in the last batched sub-iteration it took part in; synchronises */
int b200rt_batch_get_num_cancelled(b200rt_batch* b, int frame, int64_t* out);

/* ---- list-mode objective (PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin) ----
 * Events as STIR's cached BinAndCorr records (the bin with its value, the additive term), in a device array.
 * Each event's row is the cached basic row with the event's symmetry operation and axial shift; an event belongs
 * to subset s of n when its basic bin's view mod n is s (LM_distributable_computation,
 * src/include/stir/recon_buildblock/distributable.txx:36-140).  Events whose bin lies outside the projector's data
 * are skipped and counted (b200rt_listmode_num_invalid); events of value 0 are skipped as STIR does. */
typedef struct b200rt_lm_event {
  int32_t segment, view, axial_pos, tangential_pos, timing_pos; /* Bin (timing_pos 0 for non-TOF)      */
  float value;                                                  /* the bin value: counts (usually 1)   */
  float corr;                                                   /* the additive term (used if has_add)  */
} b200rt_lm_event;

/* actual_compute_subset_gradient_without_penalty (…ListModeDataWithProjMatrixByBin.cxx:900-955) with
 * LM_gradient_and_value<true,false> (:750-785): gradient (+)= sum_e A_e^T (y_e / (A_e x + c_e)) over the subset's
 * events; accumulate = 0 zeroes gradient_dev first; subset_sensitivity_dev != NULL subtracts it afterwards
 * (add_sensitivity = false), NULL leaves the sum (add_sensitivity = true). */
int b200rt_listmode_gradient_dev(b200rt_projector* h, const b200rt_lm_event* events_dev, int64_t num_events,
                                 const float* image_dev, int subset_num, int num_subsets, int has_add,
                                 const float* subset_sensitivity_dev, int accumulate, float* gradient_dev,
                                 void* stream);
/* actual_compute_objective_function_without_penalty (:866-898) with LM_gradient_and_value<false,true>:
 * -sum_e y_e log(A_e x + c_e), a cancelled event (y > 1e4 (A x + c)) giving -y log(y / 1e4); FP64, fixed order.
 * The reference's inner product with the sensitivity (:895-898) discards its result, so it is not part of the
 * value.  Synchronises and writes *value. */
int b200rt_listmode_value_dev(b200rt_projector* h, const b200rt_lm_event* events_dev, int64_t num_events,
                              const float* image_dev, int subset_num, int num_subsets, int has_add, double* value,
                              void* stream);
/* actual_accumulate_sub_Hessian_times_input_without_penalty (:957-1000) with LM_Hessian (:787-820):
 * output += sum_e A_e^T (-y_e / (A_e x + c_e)^2 A_e rhs), skipping cancelled events and A_e rhs = 0. */
int b200rt_listmode_hessian_times_input_dev(b200rt_projector* h, const b200rt_lm_event* events_dev,
                                            int64_t num_events, const float* image_dev, const float* rhs_dev,
                                            int subset_num, int num_subsets, int has_add, float* output_dev,
                                            void* stream);
/* events skipped as outside the projection data since the last call of this function; synchronises */
int b200rt_listmode_num_invalid(b200rt_projector* h, int64_t* count);
/* How the three list-mode sums above visit the events' rows.
 * PER_EVENT: one warp per event walks the event's row (a gather for A_e x, a scatter for the back projection).
 * BINNED: the rows of all events of one bin are that bin's row, so A_e x is read from the forward projection A x
 *   of the subset, each event's term is added to its bin of a projection-data buffer h, and A^T h is one back
 *   projection of the subset.  The terms of one bin's events are summed before the weights multiply them, a
 *   rounding difference only; the cancellation rules and the value's FP64 sum are those of PER_EVENT.  Costs two
 *   (three for the Hessian) subset projections plus a few bytes per event, and three projection-data buffers.
 * AUTO (the default): BINNED when the events number at least 1/16 of the projector's bins, else PER_EVENT. */
#define B200RT_LISTMODE_AUTO 0
#define B200RT_LISTMODE_PER_EVENT 1
#define B200RT_LISTMODE_BINNED 2
int b200rt_listmode_set_method(b200rt_projector* h, int method);

/* ---- projection data streams (ProjDataFromStream) ------------------------
 * The bytes of a projection data file (from its data offset on, e.g. an Interfile ".s"), copied to the device
 * as they are, converted to or from the device layout on the GPU: the element addressing of
 * ProjDataFromStream::get_offset (src/buildblock/ProjDataFromStream.cxx:415-500), with the stream's number type,
 * byte order and scale factor.  Views and tangential positions are the projector's; the stream holds
 * num_segments segments in the order segment_sequence gives (num_axial_poss each) and num_timing_poss timing
 * positions (timing position numbers in timing_poss_sequence, or min..max when NULL).  Segments of the stream
 * that the projector does not use are skipped (as STIR with "maximum absolute segment number to process"); a
 * segment of the projector missing from the stream, or with other axial sizes, is an error. */
#define B200RT_STORAGE_SEGMENT_VIEW_AXIAL_TANG 0 /* Segment_View_AxialPos_TangPos (Timing_ outermost with TOF) */
#define B200RT_STORAGE_SEGMENT_AXIAL_VIEW_TANG 1 /* Segment_AxialPos_View_TangPos (Timing_ outermost with TOF) */
#define B200RT_NUMBER_SCHAR 0  /* NumericType::SCHAR  */
#define B200RT_NUMBER_UCHAR 1  /* NumericType::UCHAR  */
#define B200RT_NUMBER_SHORT 2  /* NumericType::SHORT  */
#define B200RT_NUMBER_USHORT 3 /* NumericType::USHORT */
#define B200RT_NUMBER_INT 4    /* NumericType::INT    */
#define B200RT_NUMBER_UINT 5   /* NumericType::UINT   */
#define B200RT_NUMBER_FLOAT 6  /* NumericType::FLOAT  */
#define B200RT_NUMBER_DOUBLE 7 /* NumericType::DOUBLE */

typedef struct b200rt_stream_format {
  int32_t storage_order;               /* B200RT_STORAGE_*                                            */
  int32_t number_type;                 /* B200RT_NUMBER_*                                             */
  int32_t swap_bytes;                  /* 1: the stream is big-endian (the GPU's order is little)      */
  float scale_factor;                  /* read: value = stored * scale_factor; write: must be 1       */
  int32_t num_segments;                /* segments in the stream                                      */
  const int32_t* segment_sequence;     /* host: segment number of the stream's i-th segment           */
  const int32_t* num_axial_poss;       /* host: axial positions of the stream's i-th segment          */
  int32_t num_timing_poss;             /* timing positions in the stream (1: non-TOF)                 */
  const int32_t* timing_poss_sequence; /* host: timing position number of the i-th, or NULL (min..max) */
} b200rt_stream_format;

/* bytes a stream of this format holds for the projector's views and tangential positions */
int b200rt_stream_bytes(b200rt_projector* h, const b200rt_stream_format* fmt, int64_t* bytes);
/* read: stream_dev (stream_bytes long, any alignment) -> projdata_dev (device layout, every bin written) */
int b200rt_projdata_from_stream_dev(b200rt_projector* h, const void* stream_dev, int64_t stream_bytes,
                                    const b200rt_stream_format* fmt, float* projdata_dev, void* stream);
/* write (ProjDataFromStream::set_segment with a float or double stream): the projector's segments into their
 * places in stream_dev; other bytes are left as they are */
int b200rt_projdata_to_stream_dev(b200rt_projector* h, const float* projdata_dev, const b200rt_stream_format* fmt,
                                  void* stream_dev, int64_t stream_bytes, void* stream);

/* ---- Gibbs penalties on device-resident images ---------------------------
 * GibbsQuadraticPenalty and GibbsRelativeDifferencePenalty (src/include/stir/recon_buildblock/GibbsPenalty.h,
 * GibbsPenalty.inl, GibbsQuadraticPenalty.h, GibbsRelativeDifferencePenalty.h) and their CUDA versions
 * CudaGibbsQuadraticPenalty / CudaGibbsRelativeDifferencePenalty (CUDA/CudaGibbsPenalty.h, .cuh), which copy
 * every image to and from the GPU per call: here the penalty is set up once (b200rt_gibbs_create replaces
 * set_up: weights, kappa, image size) and every operation reads and writes device images.  Each voxel's sum is
 * taken in the reference's types and order (GibbsPenalty.inl); scalars are reduced in a fixed order. */
#define B200RT_GIBBS_QUADRATIC 1
#define B200RT_GIBBS_RELATIVE_DIFFERENCE 2
#define B200RT_LAYOUT_DEVICE 0 /* [y][x][z], z fastest: the layout of the *_dev projector entry points */
#define B200RT_LAYOUT_STIR 1   /* [z][y][x], x fastest: STIR's Array<3,float> order */

typedef struct b200rt_gibbs_params {
  int32_t potential;          /* B200RT_GIBBS_*                                                    */
  float penalisation_factor;  /* beta                                                               */
  float gamma;                /* Relative Difference "gamma value" (STIR default 2)                 */
  float epsilon;              /* Relative Difference "epsilon value" (STIR default 1e-7)            */
  int32_t nz, ny, nx;         /* image size                                                         */
  int32_t layout;             /* B200RT_LAYOUT_*                                                    */
  float voxel_size_z, voxel_size_y, voxel_size_x; /* mm, for the default weights                    */
  int32_t only_2D;            /* default weights in the plane only (1x3x3)                          */
  int32_t weights_z, weights_y, weights_x; /* sizes of `weights`, 1..7 each (0 with weights NULL)   */
  const float* weights;       /* host [z][y][x], indices -(size/2)..size-1-size/2; NULL: default    */
                              /* weights, x voxel size / distance (compute_default_weights)         */
  const float* kappa_dev;     /* kappa image on the device in `layout`, or NULL (kappa = 1)         */
} b200rt_gibbs_params;

typedef struct b200rt_gibbs b200rt_gibbs;

/* set_up: validates the parameters, copies the weights; on failure *out = NULL and b200rt_last_error(NULL)
 * says why. */
int b200rt_gibbs_create(const b200rt_gibbs_params* params, int device, b200rt_gibbs** out);
void b200rt_gibbs_destroy(b200rt_gibbs* g);
const char* b200rt_gibbs_last_error(const b200rt_gibbs* g);

/* Arithmetic of the gradient (b200rt_gibbs_gradient_dev).  B200RT_GIBBS_ARITH_HOST (the default): GibbsPenalty.inl's
 * host loop, a double sum per voxel (src/include/stir/recon_buildblock/GibbsPenalty.inl).  B200RT_GIBBS_ARITH_CUDA:
 * STIR's CUDA build, a float sum per voxel over the whole neighbourhood and the float product weight x derivative
 * per term (CudaGibbsPenalty_gradient_kernel, src/include/stir/recon_buildblock/CUDA/CudaGibbsPenalty.cuh:141-206),
 * the drop-in arithmetic for CudaGibbsQuadraticPenalty / CudaGibbsRelativeDifferencePenalty.  The other operations
 * keep the host arithmetic. */
#define B200RT_GIBBS_ARITH_HOST 0
#define B200RT_GIBBS_ARITH_CUDA 1
int b200rt_gibbs_set_arithmetic(b200rt_gibbs* g, int arithmetic);
/* get_weights: sizes[3] = (z, y, x); w receives sizes[0]*sizes[1]*sizes[2] floats (may be NULL) */
int b200rt_gibbs_get_weights(const b200rt_gibbs* g, float* w, int32_t sizes[3]);
/* set_kappa_sptr: a device image in the penalty's layout, or NULL */
int b200rt_gibbs_set_kappa(b200rt_gibbs* g, const float* kappa_dev);
/* compute_value (GibbsPenalty.inl compute_value): beta sum_r sum_dr w_dr phi(x_r, x_r+dr) kappa_r kappa_r+dr, FP64;
 * synchronises and writes *value (host). */
int b200rt_gibbs_value_dev(b200rt_gibbs* g, const float* image_dev, double* value, void* stream);
/* compute_gradient: 2 beta sum_dr w_dr phi_10(x_r, x_r+dr) kappa kappa */
int b200rt_gibbs_gradient_dev(b200rt_gibbs* g, const float* image_dev, float* gradient_dev, void* stream);
/* compute_gradient_times_input: <gradient at image_dev, input_dev>, FP64; synchronises and writes *value (host). */
int b200rt_gibbs_gradient_times_input_dev(b200rt_gibbs* g, const float* input_dev, const float* image_dev,
                                          double* value, void* stream);
/* compute_Hessian_diagonal: 2 beta sum_dr w_dr phi_20(x_r, x_r+dr) kappa kappa */
int b200rt_gibbs_hessian_diagonal_dev(b200rt_gibbs* g, const float* image_dev, float* out_dev, void* stream);
/* accumulate_Hessian_times_input: output += 2 beta sum_dr w_dr (phi_20 in_r + phi_11 in_r+dr) kappa kappa */
int b200rt_gibbs_accumulate_hessian_times_input_dev(b200rt_gibbs* g, const float* image_dev, const float* input_dev,
                                                    float* output_dev, void* stream);
/* compute_Hessian of the voxel (z, y, x) (0-based indices): out_dev is overwritten with the voxel's Hessian row */
int b200rt_gibbs_hessian_dev(b200rt_gibbs* g, const float* image_dev, int z, int y, int x, float* out_dev,
                             void* stream);

#ifdef __cplusplus
}
#endif
#endif /* STIR_B200_H */
