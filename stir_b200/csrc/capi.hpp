// Shared state of the C ABI (include/stir_b200.h): the projector handle, device buffers, error handling and
// the helpers the subsystem files (capi_*.cu) share.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/stir_b200.h"
#include "geometry.hpp"
#include "internal.hpp"

namespace b200 {
size_t projector_smem_bytes(const ProjParams& p);
}

using namespace b200;

namespace capi {

extern std::mutex g_err_mu;
extern std::string g_create_error;

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string& where)
      : std::runtime_error(where + ": " + cudaGetErrorString(c)), code(c) {}
};
inline void ck(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw CudaError(e, where);
}

template <typename T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() {}
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    if (count == 0) return;
    ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
    n = count;
  }
  void upload(const std::vector<T>& v, cudaStream_t st) {
    alloc(v.size());
    if (!v.empty()) ck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
  }
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) ck(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace capi

using namespace capi;

struct b200rt_projector {
  std::unique_ptr<Geometry> geo;
  int device = 0;
  std::string err;
  // device tables
  DevBuf<RowElem> rows;
  DevBuf<ProjBinDev> bins;
  DevBuf<LineDev> lines;
  DevBuf<SegDev> segs;
  // per segment of the whole data: STIR-order offset, device-layout offset, axial positions (layout changes)
  DevBuf<int64_t> layout_tab;
  ProjParams params{};
  // host copies
  std::vector<ProjBinDev> h_bins;
  std::vector<int> h_bin_view;  // basic view of each bin
  std::vector<int> h_bin_seg;
  std::vector<int> h_view_basic;  // basic view of each view (-1: none)
  // view shard (b200rt_set_view_shard): the views held, in slot order (empty: every view), each view's slot (-1: not
  // held) on the host and the device, the full layout's segment table, and the shard's data size and timing-bin stride
  std::vector<int> shard_views, h_view_slot;
  DevBuf<int> view_slot_dev;
  std::vector<SegDev> h_segs_full;
  int64_t shard_pd_size = 0, shard_tof_stride = 0;
  // basic views of h_bin_view, h_tof_basic_view, h_item_view and h_view_basic on the device (set-up)
  DevBuf<int> bin_view_dev, tof_basic_view_dev, item_view_dev, view_basic_dev;
  std::map<long long, int> bin_index;  // (view, seg, tang, tof) -> bin
  int64_t total_nnz = 0;
  int num_basic_views = 0;
  // subset work lists
  std::map<std::pair<int, int>, std::unique_ptr<DevBuf<int>>> subset_lists;
  std::map<std::pair<int, int>, int> subset_counts;
  std::map<std::pair<int, int>, std::unique_ptr<DevBuf<int>>> subset_views;  // all views of the subset
  std::map<std::pair<int, int>, int> subset_view_counts;
  // OSMAPOSL scratch
  DevBuf<float> ratio, upd, grad, small_value, partial_max, umax;
  DevBuf<float> ratio_batch;  // gradient ratios of an image batch (b200rt_log_likelihood_gradient_batch_dev)
  DevBuf<unsigned int> cancelled;
  DevBuf<unsigned int> dev_status;  // kernels' status word (PathParams::status)
  DevBuf<double> ll_partials, ll_sum;
  // deterministic back projection
  DevBuf<unsigned long long> acc64;
  DevBuf<double> fixed_scale;
  DevBuf<float> colmax, det_partial, det_bound;
  float det_bound_value = 0.f;
  bool colmax_ready = false;
  float prior_w[27] = {0};
  // OSSPS scratch: sub-gradient, prior gradient, image of ones, block minima
  DevBuf<float> ossps_g, ossps_pg, ones, ossps_partial, ossps_minpos;
  // column-staged projection (paths.cu): path items, their lines, rows in path order
  bool use_paths = false;
  DevBuf<PathElem> path_elems;
  DevBuf<uint32_t> path_cols;
  DevBuf<PathLineDev> path_lines;
  DevBuf<PathItemDev> path_items;
  DevBuf<int> path_chunks;
  DevBuf<PathCElem> path_cmaj;
  DevBuf<int> path_col_starts;
  PathParams pparams{};
  std::vector<int> h_item_view;  // basic view of each path item
  std::vector<PathItemDev> h_path_items;
  std::map<std::pair<int, int>, std::unique_ptr<DevBuf<int>>> path_lists;
  std::map<std::pair<int, int>, int> path_counts;
  // staging for the host API
  DevBuf<float> st_img_a, st_img_b, st_pd_a, st_pd_b;
  cudaStream_t stream = nullptr;
  // host API pipelining: path items grouped by the views they write, so that the copies of one group of
  // views overlap the projection of the next; copies on a second stream
  std::vector<int> h_item_out_view;  // the view of every line of the item (-1: lines of several views)
  bool paths_view_split = false;
  struct ViewGroups {
    std::unique_ptr<DevBuf<int>> list;  // the subset's items, group by group
    std::vector<int> off, v0;           // group g: items [off[g], off[g+1]), views [v0[g], v0[g+1])
  };
  std::map<std::pair<int, int>, ViewGroups> view_groups;
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> copy_events;
  // TOF by basic bin (the TOF-grouped packed kernels): non-TOF basic rows, per-element weights of every timing
  // bin, one entry per basic bin, its view, and the subsets' lists of basic bins
  DevBuf<RowElem> tof_basic_rows;
  DevBuf<float> tof_w;
  DevBuf<ProjBinDev> tof_basic;
  std::vector<int> h_tof_basic_view;
  std::map<std::pair<int, int>, std::unique_ptr<DevBuf<int>>> tof_group_lists;
  std::map<std::pair<int, int>, int> tof_group_counts;
  // list mode: the related lines on the host, (tof, seg, view, tang) -> (basic bin, line, basic view)
  std::vector<LineDev> h_lines;
  DevBuf<int4> lm_table;
  DevBuf<double> lm_partial, lm_sum;
  DevBuf<unsigned> lm_invalid;
  // binned list mode: A x and A rhs of the subset, the events' terms per bin, a scratch image
  int lm_method = B200RT_LISTMODE_AUTO;
  DevBuf<float> lm_fwd, lm_fwd_rhs, lm_hist, lm_img;
  // viewgram access: a viewgram in STIR order and a transposed copy
  DevBuf<float> vg_scratch;

  long long bin_key(int view, int seg, int tang, int tof) const {
    const Geometry& g = *geo;
    return ((static_cast<long long>(view) * (2 * g.S() + 1) + (seg + g.S())) * 4096 + (tang + 2048)) * 1024 + (tof + 512);
  }
};

namespace capi {

int fail(b200rt_projector* h, int code, const std::string& msg);
int status_of(const std::exception& e);
void setup_projector(b200rt_projector& h);
const int* subset_list(b200rt_projector& h, int subset, int nsub, int& count);
const int* path_list(b200rt_projector& h, int subset, int nsub, int& count);
const int* tof_group_list(b200rt_projector& h, int subset, int nsub, int& count);
void forward_subset(b200rt_projector& h, const float* image, float* out, int subset, int nsub, cudaStream_t st,
                    const FwdEpilogue* ep = nullptr);
const int* subset_views(b200rt_projector& h, int subset, int nsub, int& count);
void prior_weights(const Geometry& g, int only_2D, float w[27]);
void back_project_into(b200rt_projector& h, const float* pd, float* image, int subset, int nsub, int mode, int zero_ends,
                       cudaStream_t st, float max_abs = 0.f);
int check_subset(b200rt_projector* h, int subset, int nsub);
void ensure_colmax(b200rt_projector& h, float* scratch, cudaStream_t st);
cudaError_t projdata_layout(const b200rt_projector& h, const float* in, float* out, bool to_dev, cudaStream_t st);
cudaError_t projdata_layout_views(const b200rt_projector& h, const float* in, float* out, bool to_dev, int v0, int v1,
                                  cudaStream_t st);
cudaError_t copy_views(const Geometry& g, float* dst, const float* src, int v0, int v1, cudaMemcpyKind kind,
                       cudaStream_t st);
const b200rt_projector::ViewGroups& view_groups(b200rt_projector& h, int subset, int nsub);
void ensure_copy_stream(b200rt_projector& h);
void osmaposl_numerator(b200rt_projector& h, const float* x, const float* y, const float* add, int subset, int nsub,
                        int zero_ends, int mode, float* u, cudaStream_t st);
void osmaposl_apply(b200rt_projector& h, float* x, float* u, const float* sens, int nsub, int subiter,
                    const b200rt_prior* prior, float min_rel, float max_rel, cudaStream_t st);
int check_mode_prior(b200rt_projector* h, int mode, const b200rt_prior* prior);

// the projection data's size and timing-bin stride in the projector's layout (a view shard's, or the full one)
inline bool sharded(const b200rt_projector& h) { return !h.shard_views.empty(); }
inline int64_t pd_size(const b200rt_projector& h) { return sharded(h) ? h.shard_pd_size : h.geo->projdata_size(); }
inline int64_t pd_tof_stride(const b200rt_projector& h) { return sharded(h) ? h.shard_tof_stride : h.geo->tof_stride(); }
// entry points that address the full projection data refuse a view shard
int refuse_shard(b200rt_projector* h, const char* what);

}  // namespace capi
