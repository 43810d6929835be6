// Device-side data structures shared by the kernels and the host driver.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/stir_b200.h"

namespace b200 {

// A stored row element: voxel (z,y,x) packed into 32 bits and its value.
//   bits  0..10 : x + 1024   bits 11..21 : y + 1024   bits 22..31 : (z - zmin_row) ... see pack_zyx
// z is stored relative to a per-geometry row z bias so that the 10 bits cover [-512, 511].
struct __align__(8) RowElem {
  uint32_t zyx;
  float v;
};

__host__ __device__ inline uint32_t pack_zyx(int z, int y, int x) {
  return static_cast<uint32_t>(x + 1024) | (static_cast<uint32_t>(y + 1024) << 11) |
         (static_cast<uint32_t>(z + 512) << 22);
}
__host__ __device__ inline void unpack_zyx(uint32_t p, int& z, int& y, int& x) {
  x = static_cast<int>(p & 2047u) - 1024;
  y = static_cast<int>((p >> 11) & 2047u) - 1024;
  z = static_cast<int>(p >> 22) - 512;
}

// One ray of a basic bin (geometry.hpp Ray) as uploaded to the device
struct RayDev {
  float start[3];
  float stop[3];
  float norm_const;
};

// Per basic bin, for the row builder
struct BuildBinDev {
  int first_ray, num_rays;
  int direct, nlz;
  float z_origin_in_planes, z_centre, left_edge, tor_width;
  int64_t scratch_offset;  // first element of this bin's scratch (2*capacity elements)
  int capacity;
  int pad;
};

// A related line of a basic view-segment: target viewgram and the symmetry operation
//   flags: bit0 swap x<->y, bit1 negate x', bit2 negate y', bit3 z -> q - z
struct LineDev {
  int16_t view, seg;
  int8_t tang_sign, flags;
  int16_t q;
};

// Per basic bin, for the projectors
struct ProjBinDev {
  int64_t row_offset;
  int32_t row_len;
  int16_t tang;    // basic tangential position (>= 0 with the s symmetry)
  int16_t tof;
  int32_t first_line, num_lines;  // into lines[]
};

struct SegDev {
  int64_t dev_offset;  // device-layout offset of the segment (TOF bin 0)
  int32_t nax;
  int32_t npa;
};

// Kernel parameters of the projectors
struct ProjParams {
  const RowElem* rows;
  const ProjBinDev* bins;
  const LineDev* lines;
  const SegDev* segs;  // index seg + S
  int S;
  int num_views, num_tang, min_tang, max_tang;
  int num_tof, min_tof;
  int64_t tof_stride;
  int nz, ny, nx;      // image (device layout [y][x][z])
  int min_z, min_y, min_x;
  int max_row_len;
  int uniform_npa;  // planes per axial position if equal for all segments, else 0
  // a projector holding part of the views (b200rt_set_view_shard): the slot of every view in the device layout of
  // the projection data (-1: not held), or null when every view is held (slot = view); segs[].dev_offset and
  // tof_stride then describe the shard's layout [timing bin][segment][slot][tangential][axial]
  const int* view_slot;
  int max_nax;      // most axial positions of any segment
  // TOF data by basic bin (the TOF-grouped packed kernels): the non-TOF basic rows, every element's weight for
  // each timing bin ([element][timing bin], 0 where the TOF row has no element) and one entry per basic bin
  // (row_offset into tof_basic_rows, tof = min timing bin); null without TOF
  const RowElem* tof_basic_rows;
  const float* tof_w;
  const ProjBinDev* tof_basic;
};
// with at most this many axial positions per line the per-basic-bin kernels pack (line, axial position) pairs
// into the lanes of a warp (project.cu)
constexpr int kPackedMaxNax = 16;

// What the forward projector does with each projected bin A x:
//   kEpiNone:   store it;
//   kEpiRatio:  store divide_and_truncate(y, A x + a) (the OSMAPOSL gradient numerator);
//   kEpiLoglik: accumulate the Poisson log-likelihood of y given (A x + a) m in FP64, per CTA.
//   kEpiGradient: store divide_and_truncate(y, A x + a) - m (m = mult or 1): back-projected, the gradient of
//                the log-likelihood (RPC_process_related_viewgrams_gradient<false>, ...AndProjData.cxx:1462-1477).
//   kEpiLoglikRatio: both kEpiLoglik (the partial sums) and kEpiGradient (the stored ratio) from one projection.
constexpr int kEpiNone = 0;
constexpr int kEpiRatio = 1;
constexpr int kEpiLoglik = 2;
constexpr int kEpiGradient = 3;
constexpr int kEpiLoglikRatio = 4;
struct FwdEpilogue {
  int mode;
  int zero_ends;               // zero the first/last axial position of segment 0
  const float* y;              // measured data (device layout)
  const float* add;            // additive term or nullptr
  const float* mult;           // multiplicative term or nullptr (log-likelihood only)
  const float* small_value;    // per ((tof-min)*(2S+1)+segment+S)*num_views+view: max(viewgram y)*SMALL_NUM, >= 0
  unsigned int* cancelled;     // number of ratios clipped at 1e4
  double* partials;            // one log-likelihood partial sum per CTA
  // a batch of images projected in one launch (grid.y = image): image b's y, add, mult and thresholds are at these
  // strides (0: shared by the batch), its partial sums at b x grid.x
  int64_t y_stride, add_stride, mult_stride, sv_stride;
};

// One reconstruction of a batch: its geometry (index into a ProjParams table), estimate, ratio
// scratch (projection data of its geometry), numerator image and forward epilogue.
struct BatchFrameDev {
  int geom;
  const float* x;
  float* ratio;
  float* u;
  FwdEpilogue ep;
  // deterministic back projection of this frame: 64-bit fixed-point sums and their scale (null: float atomics)
  unsigned long long* acc64;
  const double* fixed_scale;
};
struct BatchItem {
  int frame;
  int bin;
};

// ---- column-staged projection (paths.cu) --------------------------------------------------------
// The basic bins that share a basic view and tangential position (one per segment) trace the same
// transaxial path, so their rows cross the same voxel columns (x, y).  A "path item" is such a group
// together with one transaxial symmetry operation T (swap, -x, -y): its lines (every segment, both z
// orientations) read the columns T(x, y) of the path, which one CTA copies to shared memory in chunks
// of K columns (all z of a column, contiguous in the [y][x][z] layout).

// Row element of a path: the column's index in the path ("slot", bits 0..15) and z + 512 (bits 16..31).
struct __align__(8) PathElem {
  uint32_t sz;
  float v;
};
struct PathLineDev {
  int line;          // index into lines[]
  int bin;           // basic bin (projection data position, tangential position)
  int64_t elem_off;  // first element of the bin's row in path order (sorted by slot, then z)
  int chunk_off;     // the row's chunk table in chunks[]: chunk c covers elements [tab[c], tab[c+1])
  int member;        // the bin's position among the path's basic bins (its segment)
};
struct PathItemDev {
  int col_offset, ncols;        // path columns in cols[], packed (x + 1024) | (y + 1024) << 11
  int first_line, num_lines;    // into path lines[]; the lines of one member are consecutive
  int flags;                    // T: bit 0 swap x/y, bit 1 negate x, bit 2 negate y
  int col_starts;               // the path's column table in col_starts[] (ncols + 1 entries)
  int64_t cmaj_off;             // the path's elements in column order in cmaj[]
};
// A path element in column order: z + 512 (bits 0..10), the member (bits 11..15), the column slot (bits 16..31),
// the value.
struct __align__(8) PathCElem {
  uint32_t mz;
  float v;
};
struct PathParams {
  const PathElem* elems;
  const uint32_t* cols;
  const PathLineDev* lines;
  const PathItemDev* items;
  const int* chunks;
  int K;          // columns per chunk
  int max_lines;  // lines of the largest item
  int nax_max;    // axial positions of the longest segment
  int npa_max;    // largest planes per axial position
  int max_chunk_elems;  // most elements of one row in one chunk
  const PathCElem* cmaj;  // every path's elements ordered by column, then member, then z
  const int* col_starts;  // per path: first element of each column in cmaj (relative), ncols + 1 entries
  int max_members;        // basic bins per path (basic segments)
  int max_acc;            // forward accumulators of the largest item: path_parts(lines) x sum of the lines' nax
  int zpad;               // >= 0: zeros of at least zpad planes between the staged columns, enough for every
                          // forward pass to read all its planes without range tests; -1: tests per lane
  unsigned* status;       // device word of the projector: bit 0 set when a staging copy was not seen to complete
                          // within the forward kernel's wait limit (that item's sums are then incomplete)
};

// parts each line's elements are split into (forward): an item's lines are processed in pairs (the two
// z orientations of a basic bin), so (pairs x parts) units keep the 8 warps of a CTA busy
__host__ __device__ inline int path_parts(int num_lines) { return num_lines >= 8 ? 4 : 8; }

struct PathLineSmem {
  int64_t out_base;  // device-layout projection index of (line, axial 0)
  int64_t elem_off;
  int chunk_off;
  int nax, npa;
  int zsign, zadd;  // z index in the image = zsign * (sz >> 16) + zadd  (z reflection, -512 bias, -min_z)
  int seg, view, tofi;
  int active;       // tangential position inside the projection data
  int member;
};
// a row element of one or two lines and one pass, in shared memory (forward)
struct __align__(16) PathXElem {
  int base;  // staged index of axial position 0, line 1
  int zt;    // staged index of axial position 0, line 2
  float v;
  int full;  // column slot in the chunk (bits 0..15); bit 30: z stays inside the image for every lane
};
constexpr int kPathWarpsH = 8;

__host__ __device__ inline int path_align16(int x) { return (x + 15) & ~15; }
// the back projection's per-line data, padded with zeros: d(a) at index F + a npa, F = path_dl_front(nz),
// read at F + z - zt for planes z in [0, nz + 127) and windows [zt, zt + (nax - 1) npa] that meet the image;
// indices [0, F) are zero
__host__ __device__ inline int path_dl_front(int nz) { return nz + 128; }
__host__ __device__ inline int path_dl_len(int nz, int nax_max, int npa_max) {
  return (2 * nz + 256 + (nax_max - 1) * npa_max + 3) & ~3;
}

// dynamic shared memory of a forward path CTA: staged columns, their image offsets, line set-up, line
// pairs and accumulator offsets, per-warp element buffers, per (line, part) accumulators (max_acc floats:
// the most, over the items, of path_parts(lines) x the lines' axial positions)
struct PathSmemFwd {
  int colbase, lines, pairs, rowoff, xbuf, acc, total;
};
// staged column ci starts at ci * path_col_stride + path_col_offset (a 16-byte boundary with padded staging), plane
// z at that start + z, plus, with padded staging, the column's 16-byte phase in global memory (0..3 floats): the
// padded columns are copied as whole 16-byte blocks, so the stride leaves zpad zero planes between columns
// whatever the phases
__host__ __device__ inline int path_col_stride(int nz, int zpad) { return zpad >= 0 ? (nz + zpad + 6) & ~3 : nz; }
__host__ __device__ inline int path_col_offset(int zpad) { return zpad > 0 ? zpad : 0; }
__host__ __device__ inline PathSmemFwd path_smem_fwd(int K, int nz, int zpad, int max_lines, int max_acc, int npa_max) {
  PathSmemFwd s;
  // staged columns (with the padding below the first and above the last) and a pass's overshoot
  s.colbase = path_align16((K * path_col_stride(nz, zpad) + 2 * path_col_offset(zpad) + 128 * npa_max) * 4);
  s.lines = path_align16(s.colbase + K * 4);
  s.pairs = path_align16(s.lines + max_lines * static_cast<int>(sizeof(PathLineSmem)));
  s.rowoff = path_align16(s.pairs + max_lines * 8);
  s.xbuf = path_align16(s.rowoff + max_lines * 4);
  s.acc = s.xbuf + kPathWarpsH * 32 * static_cast<int>(sizeof(PathXElem));
  s.total = path_align16(s.acc + max_acc * 4);
  return s;
}
// back path CTA: line set-up, per line (z sign, z offset, window length, data offset), per member its
// first line and line count, padded line data
struct PathSmemBack {
  int lines, lz, members, dl, ebuf, total;
};
__host__ __device__ inline PathSmemBack path_smem_back(int nz, int max_lines, int max_members, int nax_max,
                                                       int npa_max) {
  PathSmemBack s;
  s.lines = 0;
  s.lz = path_align16(max_lines * static_cast<int>(sizeof(PathLineSmem)));
  s.members = path_align16(s.lz + max_lines * 16);
  s.dl = path_align16(s.members + max_members * 8);
  s.ebuf = path_align16(s.dl + max_lines * path_dl_len(nz, nax_max, npa_max) * 4);
  s.total = s.ebuf + kPathWarpsH * 32 * 16;  // per warp: 32 column-order elements with their member's lines
  return s;
}

// launchers (paths.cu); the item lists hold indices into PathParams::items
cudaError_t launch_forward_paths(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                 const float* image, float* projdata, cudaStream_t st, const FwdEpilogue* ep);
cudaError_t launch_back_paths_atomic(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                     const float* projdata, float* image, cudaStream_t st, int zero_ends);
cudaError_t launch_back_paths_fixed(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                    const float* projdata, unsigned long long* acc, const double* scale,
                                    cudaStream_t st, int zero_ends);
// the same over a batch of images in one launch (grid.y = image): image b at image + b img_stride, its projection
// data at projdata + b pd_stride (the forward's epilogue data at the strides of FwdEpilogue)
cudaError_t launch_forward_paths_batch(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                       const float* images, int64_t img_stride, float* projdata, int64_t pd_stride,
                                       int batch, cudaStream_t st, const FwdEpilogue* ep);
cudaError_t launch_back_paths_atomic_batch(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                           const float* projdata, int64_t pd_stride, float* images, int64_t img_stride,
                                           int batch, cudaStream_t st, int zero_ends);

// persistent batched projectors over (frame, path item) work items (BatchItem::bin holds the path item)
cudaError_t launch_forward_batch_paths(const ProjParams* geoms, const PathParams* pgeoms, int npa, int smem_bytes,
                                       const BatchFrameDev* frames, const BatchItem* items, int nitems, unsigned* counter,
                                       int grid, cudaStream_t st);
cudaError_t launch_back_batch_paths(const ProjParams* geoms, const PathParams* pgeoms, int smem_bytes,
                                    const BatchFrameDev* frames, const BatchItem* items, int nitems, unsigned* counter,
                                    int grid, cudaStream_t st);
int batch_paths_max_ctas_per_sm(int npa, int smem_bytes, bool forward);

// One frame's OSMAPOSL update in a batched update launch (the arguments of launch_update)
struct BatchUpdateDev {
  float* u;
  float* x;
  const float* sens;
  float* g;
  int prior_type;
  float beta, gamma, epsilon;
  int dzmin, dzmax;
  float w[27];
  const float* kappa;
  int ny, nx, nz;
  int nblocks;
  float* partial_max;
  float* umax;
  int prior, map_model;
  float num_subsets, small_num;
  int clamp;
  float min_rel, max_rel;
};
void fill_batch_update(BatchUpdateDev& d, float* u, float* x, const float* sens, float* g, const b200rt_prior* prior,
                       const float prior_weights[27], int num_subsets, int subiteration_num, float min_rel, float max_rel,
                       int ny, int nx, int nz, float* partial_max, float* umax);
// the updates of several frames: three launches (grid.y = frame), max_blocks = the largest nblocks
cudaError_t launch_batch_update(const BatchUpdateDev* frames_dev, int nframes, int max_blocks, bool any_prior,
                                cudaStream_t st);

// launchers (project.cu)
cudaError_t launch_forward(const ProjParams& p, const int* bin_list, int nbins, const float* image, float* projdata,
                           cudaStream_t st, const FwdEpilogue* ep = nullptr);
// persistent batched projectors: `grid` CTAs take (frame, basic bin) items from *counter (zeroed by the caller)
cudaError_t launch_forward_batch(const ProjParams* geoms, int npa, size_t smem_bytes, const BatchFrameDev* frames,
                                 const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st);
cudaError_t launch_back_batch(const ProjParams* geoms, int npa, size_t smem_bytes, const BatchFrameDev* frames,
                              const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st);
// resident CTAs per SM of the batched kernels (0 on error); also sets their shared-memory limit
// batched packed kernels (frames whose segments have at most kPackedMaxNax axial positions): one item per warp
cudaError_t launch_forward_batch_packed(const ProjParams* geoms, const BatchFrameDev* frames, const BatchItem* items,
                                        int nitems, unsigned* counter, int grid, cudaStream_t st);
cudaError_t launch_back_batch_packed(const ProjParams* geoms, const BatchFrameDev* frames, const BatchItem* items,
                                     int nitems, unsigned* counter, int grid, cudaStream_t st);
int batch_packed_max_ctas_per_sm(bool forward);
// batched TOF-grouped kernels (TOF frames of packed geometries): items are (frame, basic bin of the TOF table)
cudaError_t launch_forward_batch_tof(const ProjParams* geoms, int num_tof, const BatchFrameDev* frames,
                                     const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st);
cudaError_t launch_back_batch_tof(const ProjParams* geoms, int num_tof, const BatchFrameDev* frames,
                                  const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st);
int batch_tof_max_ctas_per_sm(int num_tof, bool forward);
int batch_max_ctas_per_sm(int npa, size_t smem_bytes, bool forward);
// dynamic shared memory of the projection kernels for a row length bound
size_t proj_smem_bytes(int max_row_len);
// projdata == nullptr back-projects ones
cudaError_t launch_back_atomic(const ProjParams& p, const int* bin_list, int nbins, const float* projdata, float* image,
                               cudaStream_t st, int zero_ends = 0);
cudaError_t launch_image_to_dev(const float* stir, float* dev, int nz, int ny, int nx, cudaStream_t st);
cudaError_t launch_image_from_dev(const float* dev, float* stir, int nz, int ny, int nx, cudaStream_t st);
// per segment: STIR [ax][view*tang] <-> device [view*tang][ax]
cudaError_t launch_projdata_to_dev(const float* stir, float* dev, int nax, int64_t nvt, cudaStream_t st);
cudaError_t launch_projdata_from_dev(const float* dev, float* stir, int nax, int64_t nvt, cudaStream_t st);
// List-mode events (listmode.cu), the layout of b200rt_lm_event; table[(tof, seg, view, tang)] = (basic bin, line
// of the bin, basic view, 0) or x = -1 for a bin no line covers
struct LmEventDev {
  int seg, view, axial, tang, tof;
  float value, corr;
};
int listmode_num_blocks(int64_t n);
cudaError_t launch_subtract(float* out, const float* s, int64_t n, cudaStream_t st);  // out -= s
// op 0: out += gradient terms, 1: per-block value partials (listmode_num_blocks of them), 2: out += Hessian times rhs
cudaError_t launch_listmode(const ProjParams& p, const int4* table, const LmEventDev* events, int64_t n, int op,
                            const float* x, const float* rhs, int subset, int nsub, int has_add, float* out,
                            double* partial, unsigned* invalid, cudaStream_t st);
// binned form: fwd (and fwd_rhs for op 2) = the subset's forward projections (device layout); op 0 and 2 add each
// event's term to hist[bin] (device layout) for a back projection afterwards, op 1 writes
// listmode_binned_num_blocks partials
int listmode_binned_num_blocks(int64_t n);
cudaError_t launch_listmode_binned(const ProjParams& p, const int4* table, const LmEventDev* events, int64_t n, int op,
                                   const float* fwd, const float* fwd_rhs, int subset, int nsub, int has_add,
                                   float* hist, double* partial, unsigned* invalid, cudaStream_t st);
cudaError_t launch_add(float* out, const float* s, int64_t n, cudaStream_t st);  // out += s

// Projection data streams (stream.cu): NumericType codes and storage orders as b200rt_stream_format
constexpr int kNumSChar = 0, kNumUChar = 1, kNumShort = 2, kNumUShort = 3, kNumInt = 4, kNumUInt = 5, kNumFloat = 6,
              kNumDouble = 7;
constexpr int kStorageSegmentViewAxialTang = 0, kStorageSegmentAxialViewTang = 1;
// one segment of one timing position: its first element in the stream, its first float in the device layout
struct StreamSegment {
  int order, type, swap;
  float scale;
  int nax, nv, nt;
  int64_t stream_elem, dev_off;
};
int numeric_type_size(int type);  // 0 for an unknown type
cudaError_t launch_stream_segment(const StreamSegment& s, bool to_dev, const void* in, void* out, cudaStream_t st);

// Gibbs penalty (gibbs.cu): image size and layout (0: [y][x][z], 1: [z][y][x]) with the strides of z, y, x;
// weights [wz][wy][wx] with index ranges [-(w/2), w - 1 - w/2]
constexpr int kGibbsMaxWeights = 343;
struct GibbsDev {
  int potential;  // 1 Quadratic, 2 Relative Difference
  float beta, gamma, epsilon;
  int nz, ny, nx, layout;
  int64_t sz, sy, sx;
  int wz, wy, wx;
  const float* kappa;
  float w[kGibbsMaxWeights];
  double wd[27];  // the first 27 weights as double (the unrolled 3x3x3 / 1x3x3 paths)
};
// op: 0 value (-> *result, device), 1 gradient, 2 gradient times input (-> *result), 3 Hessian diagonal,
// 4 out += Hessian times input; partial holds gibbs_num_partials() doubles
int64_t gibbs_num_partials(const GibbsDev& g);
cudaError_t launch_gibbs(const GibbsDev& g, int op, const float* x, const float* in, float* out, double* partial,
                         double* result, cudaStream_t st);
cudaError_t launch_gibbs_hessian_voxel(const GibbsDev& g, const float* x, int z, int y, int xx, float* out,
                                       cudaStream_t st);
// the gradient with the arithmetic of STIR's CUDA build (float sums), B200RT_GIBBS_ARITH_CUDA
cudaError_t launch_gibbs_gradient_cuda(const GibbsDev& g, const float* x, float* out, cudaStream_t st);

// out[c * ld_out + r] = in[r * ld_in + c], r < rows, c < cols
// STIR order <-> device layout of the columns [c0, c0 + nc) (views x tangential positions) of every (timing bin,
// segment) of projection data, in one launch; tab: per segment (STIR offset, device offset, axial positions)
cudaError_t launch_projdata_layout_views(const float* in, float* out, const int64_t* tab, int nsegs, int ntof,
                                         int max_nax, int64_t tof_stride, int64_t nvt, int64_t c0, int64_t nc,
                                         bool to_dev, cudaStream_t st);
cudaError_t launch_transpose(const float* in, float* out, int rows, int64_t cols, int64_t ld_in, int64_t ld_out,
                             cudaStream_t st);

// deterministic back projection: contributions accumulated as int64 multiples of 1/scale
cudaError_t launch_back_fixed(const ProjParams& p, const int* bin_list, int nbins, const float* projdata,
                              unsigned long long* acc, const double* scale, cudaStream_t st, int zero_ends = 0);
// max |projdata| (nullptr data = 1) and the fixed-point scale 2^floor(62 - log2(max|d| * colmax * 1.01)) (osem.cu)
cudaError_t launch_fixed_scale(const float* projdata, int64_t n, const float* colmax, float* partial, double* scale,
                               cudaStream_t st);
cudaError_t launch_fill(float* p, int64_t n, float v, cudaStream_t st);
cudaError_t launch_prior_hessian_times_input(float* out, const float* x, const float* in, const b200rt_prior* prior,
                                             const float prior_weights[27], int ny, int nx, int nz, cudaStream_t st);
cudaError_t launch_zero_unidentifiable(float* x, const float* sens, int64_t n, cudaStream_t st);
// OSSPS: divide_and_truncate(A 1, (y n) n) in place per viewgram; the update (with, at the first sub-iteration,
// the unidentifiable voxels zeroed and the denominator completed and thresholded in place)
cudaError_t launch_hessian_ratio(float* fp, const float* y, const float* norm, const SegDev* segs, int S, int num_views,
                                 int num_tang, const int* views, int nviews, int num_tof, int64_t tof_stride,
                                 const float* small_value, cudaStream_t st);
cudaError_t launch_ossps_update(float* x, float* den, const float* g, float* pg, const float* sens, const b200rt_prior* prior,
                                const float prior_weights[27], int ny, int nx, int nz, int num_subsets, int first,
                                float relax, float upper, float* partial, float* minpos, cudaStream_t st);
cudaError_t launch_norm_projdata(const float* factors, float* projdata, int64_t n, int64_t fstride, int mode,
                                 cudaStream_t st);
cudaError_t launch_attenuation(const float* line_integrals, float* projdata, int64_t n, int mode, cudaStream_t st);
cudaError_t launch_fixed_to_float(const unsigned long long* acc, const double* scale, float* image, int64_t n,
                                  cudaStream_t st);
cudaError_t launch_max(const float* data, int64_t n, float* partial, float* out, cudaStream_t st);

// OSMAPOSL pieces (osem.cu)
// out index: ((tof bin - min) * (2S+1) + segment + S) * num_views + view
cudaError_t launch_viewgram_small_values(const float* y, const SegDev* segs, int S, int num_views, int num_tang,
                                         const int* views, int nviews, int zero_ends, int num_tof, int64_t tof_stride,
                                         float* out, cudaStream_t st, const int* view_slot = nullptr);
int update_num_blocks(int64_t n);
cudaError_t launch_update(float* u, float* x, const float* sens, float* g, const b200rt_prior* prior,
                          const float prior_weights[27], int num_subsets, int subiteration_num, float min_rel, float max_rel,
                          int ny, int nx, int nz, float* partial_max, float* umax, cudaStream_t st);
cudaError_t launch_prior_gradient(const float* x, float* g, const b200rt_prior* prior, const float prior_weights[27], int ny,
                                  int nx, int nz, float* partial_max, cudaStream_t st);
cudaError_t launch_reduce_sum(const double* partial, int n, double* out, cudaStream_t st);
// prior value (QuadraticPrior::compute_value :233-298, RelativeDifferencePrior::compute_value :302-370), FP64
cudaError_t launch_prior_value(const float* x, const b200rt_prior* prior, const float prior_weights[27], int ny, int nx,
                               int nz, double* partial, int npartial, double* out, cudaStream_t st);

// row builder (rows.cu)
struct RowKV {
  uint64_t key;  // (z,y,x) sort key << 8 | tag
  float v;
  uint32_t pad;
};
cudaError_t launch_build_rows(const RayDev* rays, const BuildBinDev* bins, int nbins, const float voxel_zyx[3],
                              RowKV* scratch, int* counts, cudaStream_t st);
// TOF rows: the non-TOF row of a basic bin weighted by the TOF kernel of one timing bin
// (ProjMatrixByBin::apply_tof_kernel, ProjMatrixByBin.inl:115-185)
struct TofJobDev {
  int64_t src_offset;  // non-TOF row
  int src_len;
  int tof_index;       // timing bin - min
  float mid[3], unit[3];  // LOR middle and direction (scanner coordinates), z,y,x
};
struct TofParams {
  float vox[3], origin[3];  // z,y,x
  float scanner_z_offset;
  float r_sqrt2_sigma;
  float trunc_n;            // 0: STIR's kernel cut-off; > 0: kernel truncated at +-trunc_n (in units of sqrt(2) sigma)
  const float* low;         // per timing bin
  const float* high;
  const double* erf_table;  // FastErf samples
  int erf_n;
  double erf_max, erf_period;
};
cudaError_t launch_tof_weights(const RowElem* src, const TofJobDev* jobs, int njobs, const TofParams& tp, int ntof,
                               float* w, cudaStream_t st);
// TOF-grouped packed projections over basic bins (items index ProjParams::tof_basic); forward with every epilogue
// (kEpiLoglik: one partial per item); back atomic (float) or fixed point
cudaError_t launch_forward_tof_grouped(const ProjParams& p, const int* items, int nitems, const float* image,
                                       float* projdata, cudaStream_t st, const FwdEpilogue* ep);
cudaError_t launch_back_tof_grouped(const ProjParams& p, const int* items, int nitems, const float* projdata,
                                    float* image, unsigned long long* acc, const double* scale, cudaStream_t st,
                                    int zero_ends);
cudaError_t launch_tof_rows(const RowElem* src, const TofJobDev* jobs, int njobs, const TofParams& tp,
                            const int64_t* out_offsets, RowElem* out, int* counts, cudaStream_t st);

cudaError_t launch_compact_rows(const BuildBinDev* bins, int nbins, const RowKV* scratch, const int64_t* out_offsets,
                                RowElem* rows, cudaStream_t st);

}  // namespace b200
