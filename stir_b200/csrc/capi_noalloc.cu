// C ABI: the allocation-free log-likelihood.
#include "capi.hpp"

using namespace b200;

// ---------------------------------------------------------------------------
// Allocation-free log-likelihood: scratch in a fixed array compiled into the library.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxItems = 131072;       // work items of the subset (path items or basic bins)
constexpr int kNoAllocMaxViews = 4096;
constexpr int kNoAllocMaxViewgrams = 131072;   // timing bins x segments x views
constexpr size_t kNoAllocItemsOff = 0;
constexpr size_t kNoAllocViewsOff = kNoAllocItemsOff + sizeof(int) * kNoAllocMaxItems;
constexpr size_t kNoAllocSmallOff = kNoAllocViewsOff + sizeof(int) * kNoAllocMaxViews;
constexpr size_t kNoAllocPartialsOff = kNoAllocSmallOff + sizeof(float) * kNoAllocMaxViewgrams;
constexpr size_t kNoAllocBytes = kNoAllocPartialsOff + sizeof(double) * kNoAllocMaxItems;

// Shared by every call on a device; held by every GPU that loads the library until exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {nullptr};

// Device address of the scratch array on `device` (which must be current): looked up once per device and kept
// for the life of the process.
unsigned char* noalloc_scratch(int device) {
  if (device < 0 || device >= 256) throw std::runtime_error("device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* ptr = nullptr;
    ck(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress");
    g_noalloc_addr[device] = ptr;
  }
  return static_cast<unsigned char*>(g_noalloc_addr[device]);
}

// Indices i in ascending order with basic_view[i] >= 0 and basic_view[i] mod nsub == subset (the rule of
// find_basic_vs_nums_in_subset.cxx:32-70 and of the cached subset lists), written to out.  One CTA of 1024
// threads; the host counts the same predicate and sizes `out` for it.
__global__ void __launch_bounds__(1024) select_subset_kernel(const int* __restrict__ basic_view, int n, int subset,
                                                             int nsub, int* __restrict__ out) {
  __shared__ int warp_count[32];
  __shared__ int base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int start = 0; start < n; start += 1024) {
    const int i = start + static_cast<int>(threadIdx.x);
    const int v = i < n ? basic_view[i] : -1;
    const bool sel = v >= 0 && v % nsub == subset;
    const unsigned m = __ballot_sync(0xffffffffu, sel);
    if (lane == 0) warp_count[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < 32; ++w) {
      const int c = warp_count[w];
      before += w < warp ? c : 0;
      total += c;
    }
    if (sel) out[base + before + __popc(m & ((1u << lane) - 1u))] = i;
    __syncthreads();
    if (threadIdx.x == 0) base += total;
    __syncthreads();
  }
}

int count_in_subset(const std::vector<int>& basic_view, int subset, int nsub) {
  int c = 0;
  for (int v : basic_view) c += v >= 0 && v % nsub == subset;
  return c;
}

}  // namespace

extern "C" int b200rt_log_likelihood_dev_noalloc(b200rt_projector* h, const float* image_dev, const float* y_dev,
                                                 const float* additive_dev, const float* mult_dev, int subset_num,
                                                 int num_subsets, int zero_seg0_end_planes, double* out_dev,
                                                 void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_log_likelihood_dev_noalloc");
  if (!h || !image_dev || !y_dev || !out_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the same work list and kernel as b200rt_log_likelihood_dev (path items, TOF-grouped basic bins or basic
    // bins), so the partial sums and their order are the same; the lists are selected on the device from
    // tables made at set-up, and only counted here
    const bool grouped = !h->use_paths && h->params.tof_w;
    const std::vector<int>& keys_h = h->use_paths ? h->h_item_view : grouped ? h->h_tof_basic_view : h->h_bin_view;
    const int* keys_d = h->use_paths ? h->item_view_dev.p : grouped ? h->tof_basic_view_dev.p : h->bin_view_dev.p;
    const int n = count_in_subset(keys_h, subset_num, num_subsets);
    const int nv = count_in_subset(h->h_view_basic, subset_num, num_subsets);
    const int64_t nvg = static_cast<int64_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views();
    if (n > kNoAllocMaxItems || nv > kNoAllocMaxViews || nvg > kNoAllocMaxViewgrams)
      return fail(h, B200RT_ERR_TOO_LARGE,
                  "b200rt_log_likelihood_dev_noalloc: the subset has " + std::to_string(n) + " work items (at most " +
                      std::to_string(kNoAllocMaxItems) + "), " + std::to_string(nv) + " views (at most " +
                      std::to_string(kNoAllocMaxViews) + "), and the data " + std::to_string(nvg) +
                      " viewgrams = " + std::to_string(g.num_tof()) + " timing bins x " +
                      std::to_string(2 * g.S() + 1) + " segments x " + std::to_string(g.num_views()) +
                      " views (at most " + std::to_string(kNoAllocMaxViewgrams) + ")");
    if (n == 0) {
      ck(cudaMemsetAsync(out_dev, 0, sizeof(double), st), "memset");
      return B200RT_OK;
    }
    unsigned char* base = noalloc_scratch(h->device);
    int* d_items = reinterpret_cast<int*>(base + kNoAllocItemsOff);
    int* d_views = reinterpret_cast<int*>(base + kNoAllocViewsOff);
    float* d_small = reinterpret_cast<float*>(base + kNoAllocSmallOff);
    double* d_partials = reinterpret_cast<double*>(base + kNoAllocPartialsOff);
    // every list entry, threshold and partial the kernels read is written by this call first
    select_subset_kernel<<<1, 1024, 0, st>>>(keys_d, static_cast<int>(keys_h.size()), subset_num, num_subsets,
                                             d_items);
    ck(cudaGetLastError(), "work list");
    select_subset_kernel<<<1, 1024, 0, st>>>(h->view_basic_dev.p, g.num_views(), subset_num, num_subsets, d_views);
    ck(cudaGetLastError(), "view list");
    ck(launch_viewgram_small_values(y_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), d_views, nv,
                                    zero_seg0_end_planes, g.num_tof(), g.tof_stride(), d_small, st),
       "viewgram thresholds");
    FwdEpilogue ep{};
    ep.mode = kEpiLoglik;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.add = additive_dev;
    ep.mult = mult_dev;
    ep.small_value = d_small;
    ep.partials = d_partials;
    if (h->use_paths)
      ck(launch_forward_paths(h->params, h->pparams, d_items, n, image_dev, nullptr, st, &ep), "log-likelihood");
    else if (grouped)
      ck(launch_forward_tof_grouped(h->params, d_items, n, image_dev, nullptr, st, &ep), "log-likelihood");
    else
      ck(launch_forward(h->params, d_items, n, image_dev, nullptr, st, &ep), "log-likelihood");
    ck(launch_reduce_sum(d_partials, n, out_dev, st), "reduce");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}
