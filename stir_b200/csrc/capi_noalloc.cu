// C ABI: the allocation-free log-likelihood.
#include "capi.hpp"

using namespace b200;

// ---------------------------------------------------------------------------
// Allocation-free log-likelihood: scratch in a fixed array compiled into the library.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxBins = 131072;
constexpr int kNoAllocMaxViews = 4096;
constexpr int kNoAllocMaxViewgrams = 65536;
constexpr size_t kNoAllocBinsOff = 0;
constexpr size_t kNoAllocViewsOff = kNoAllocBinsOff + sizeof(int) * kNoAllocMaxBins;
constexpr size_t kNoAllocSmallOff = kNoAllocViewsOff + sizeof(int) * kNoAllocMaxViews;
constexpr size_t kNoAllocPartialsOff = kNoAllocSmallOff + sizeof(float) * kNoAllocMaxViewgrams;
constexpr size_t kNoAllocBytes = kNoAllocPartialsOff + sizeof(double) * kNoAllocMaxBins;

// Shared by every call on a device; held by every GPU that loads the library until exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {nullptr};

// Device address of the scratch array on `device` (which must be current): looked up once per device.
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

}  // namespace

extern "C" int b200rt_log_likelihood_dev_noalloc(b200rt_projector* h, const float* image_dev, const float* y_dev,
                                                 const float* additive_dev, const float* mult_dev, int subset_num,
                                                 int num_subsets, int zero_seg0_end_planes, double* out_dev,
                                                 void* stream) {
  if (!h || !image_dev || !y_dev || !out_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    // work lists on the host (no device allocation)
    std::vector<int> bins;
    for (int b = 0; b < static_cast<int>(h->h_bins.size()); ++b)
      if (h->h_bin_view[b] % num_subsets == subset_num) bins.push_back(b);
    std::vector<char> in(g.num_views(), 0);
    for (int v : g.basic_views()) {
      if (v % num_subsets != subset_num) continue;
      for (int seg : g.basic_segments()) {
        std::vector<RelatedLine> rel;
        g.related_lines(v, seg, true, rel);
        for (const auto& r : rel) in[r.view] = 1;
      }
    }
    std::vector<int> views;
    for (int v = 0; v < g.num_views(); ++v)
      if (in[v]) views.push_back(v);
    if (bins.size() > static_cast<size_t>(kNoAllocMaxBins) || views.size() > static_cast<size_t>(kNoAllocMaxViews) ||
        static_cast<int64_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views() > kNoAllocMaxViewgrams)
      return fail(h, B200RT_ERR_TOO_LARGE,
                  "b200rt_log_likelihood_dev_noalloc: more than 131072 basic bins, 4096 views or 65536 viewgrams");
    if (bins.empty()) {
      ck(cudaMemsetAsync(out_dev, 0, sizeof(double), st), "memset");
      return B200RT_OK;
    }
    unsigned char* base = noalloc_scratch(h->device);
    int* d_bins = reinterpret_cast<int*>(base + kNoAllocBinsOff);
    int* d_views = reinterpret_cast<int*>(base + kNoAllocViewsOff);
    float* d_small = reinterpret_cast<float*>(base + kNoAllocSmallOff);
    double* d_partials = reinterpret_cast<double*>(base + kNoAllocPartialsOff);
    ck(cudaMemcpyAsync(d_bins, bins.data(), bins.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    ck(cudaMemcpyAsync(d_views, views.data(), views.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    // every threshold and partial the kernels read is written by this call first; nothing stale is used
    ck(launch_viewgram_small_values(y_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), d_views,
                                    static_cast<int>(views.size()), zero_seg0_end_planes, g.num_tof(), g.tof_stride(),
                                    d_small, st),
       "viewgram thresholds");
    FwdEpilogue ep{};
    ep.mode = kEpiLoglik;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.add = additive_dev;
    ep.mult = mult_dev;
    ep.small_value = d_small;
    ep.partials = d_partials;
    const int n = static_cast<int>(bins.size());
    ck(launch_forward(h->params, d_bins, n, image_dev, nullptr, st, &ep), "log-likelihood");
    ck(launch_reduce_sum(d_partials, n, out_dev, st), "reduce");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}
