// C ABI of the B200 ray-tracing projector pair (include/stir_b200.h).
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

namespace {

std::mutex g_err_mu;
std::string g_create_error;

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

}  // namespace

struct b200rt_projector {
  std::unique_ptr<Geometry> geo;
  int device = 0;
  std::string err;
  // device tables
  DevBuf<RowElem> rows;
  DevBuf<ProjBinDev> bins;
  DevBuf<LineDev> lines;
  DevBuf<SegDev> segs;
  ProjParams params{};
  // host copies
  std::vector<ProjBinDev> h_bins;
  std::vector<int> h_bin_view;  // basic view of each bin
  std::vector<int> h_bin_seg;
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
  DevBuf<unsigned int> cancelled;
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

namespace {

int fail(b200rt_projector* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int status_of(const std::exception& e) {
  if (auto* ce = dynamic_cast<const CudaError*>(&e)) {
    return ce->code == cudaErrorMemoryAllocation ? B200RT_ERR_OUT_OF_MEMORY : B200RT_ERR_CUDA;
  }
  return B200RT_ERR_INVALID_ARGUMENT;
}

// Builds all basic rows on the device (ProjMatrixByBin cache fill) and the projector tables.
// Path items of a non-TOF projector (paths.cu): for each basic view and tangential position, the union of
// the columns (x, y) of its basic rows (one per basic segment; all the same path), each row re-sorted by
// (column slot, z), and one item per transaxial symmetry operation used by the related lines.  Leaves
// use_paths false where the column-staged kernels do not apply.
void build_paths(b200rt_projector& h, const std::vector<RowElem>& hr, const std::vector<LineDev>& lines,
                 int nviews, int nsegs, int ntangs, const std::vector<int>& bviews) {
  const Geometry& g = *h.geo;
  const ProjParams& p = h.params;
  const int nz = p.nz;
  if (g.num_tof() != 1 || nz < 1) return;
  int nax_max = 1;
  for (int sg = -g.S(); sg <= g.S(); ++sg) nax_max = std::max(nax_max, g.nax(sg));
  const int ngroups = nviews * ntangs;

  struct Group {
    std::vector<uint32_t> cols;
    std::vector<PathElem> elems;
    std::vector<int64_t> member_off;  // per segment: first element (relative)
    std::vector<int> chunks;
    std::vector<int> member_chunk;    // per segment: first chunk-table entry (relative)
    std::vector<PathCElem> cmaj;      // the elements in column order: slot, member, z
    std::vector<int> col_starts;      // first element of each column in cmaj, ncols + 1 entries
    int over = 0;                     // how far (planes) a forward pass reads outside [0, nz): the staging's padding
    bool ok = true;
  };
  std::vector<Group> groups(ngroups);
  auto work = [&](int g0, int g1) {
    std::vector<std::pair<uint64_t, float>> tmp;
    for (int gi = g0; gi < g1; ++gi) {
      Group& G = groups[gi];
      try {
        const int vi = gi / ntangs, ti = gi % ntangs;
        std::vector<uint32_t> keys;
        for (int si = 0; si < nsegs; ++si) {
          const ProjBinDev& pb = h.h_bins[(static_cast<size_t>(vi) * nsegs + si) * ntangs + ti];
          for (int k = 0; k < pb.row_len; ++k) keys.push_back(hr[pb.row_offset + k].zyx & 0x3fffffu);  // x, y bits
        }
        std::sort(keys.begin(), keys.end());
        keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
        if (keys.size() > 65535) {
          G.ok = false;
          continue;
        }
        G.cols = keys;
        const int ncols = static_cast<int>(keys.size());
        for (int si = 0; si < nsegs; ++si) {
          const ProjBinDev& pb = h.h_bins[(static_cast<size_t>(vi) * nsegs + si) * ntangs + ti];
          tmp.clear();
          for (int k = 0; k < pb.row_len; ++k) {
            const RowElem e = hr[pb.row_offset + k];
            const uint32_t slot =
                static_cast<uint32_t>(std::lower_bound(keys.begin(), keys.end(), e.zyx & 0x3fffffu) - keys.begin());
            const uint32_t zb = e.zyx >> 22;  // z + 512
            tmp.push_back({(static_cast<uint64_t>(slot) << 32) | (static_cast<uint64_t>(zb) << 16) | 0u, e.v});
          }
          std::stable_sort(tmp.begin(), tmp.end(), [](const std::pair<uint64_t, float>& a,
                                                      const std::pair<uint64_t, float>& b) { return a.first < b.first; });
          G.member_off.push_back(static_cast<int64_t>(G.elems.size()));
          for (const auto& t : tmp) {
            const uint32_t slot = static_cast<uint32_t>(t.first >> 32);
            const uint32_t zb = static_cast<uint32_t>((t.first >> 16) & 0xffffu);
            G.elems.push_back(PathElem{slot | (zb << 16), t.second});
          }
          // the planes a forward pass of each of the bin's lines reads for these elements
          for (int l = 0; l < pb.num_lines; ++l) {
            const LineDev& L = lines[pb.first_line + l];
            const int nax = g.nax(L.seg), npa = g.npa(L.seg);
            for (const auto& t : tmp) {
              const int z = static_cast<int>((t.first >> 16) & 0xffffu) - 512;
              const int zt = ((L.flags & 8) ? L.q - z : z) - p.min_z;
              for (int a0 = 0; a0 < nax; a0 += 128) {
                const int lo = zt + a0 * npa, hi = zt + (std::min(nax - a0, 128) + a0 - 1) * npa;
                if (hi < 0 || lo > nz - 1)
                  G.over = std::numeric_limits<int>::max();  // a window outside the image: no padded staging
                else
                  G.over = std::max(G.over, std::max(-lo, hi - (nz - 1)));
              }
            }
          }
        }
        // the same elements in column order (slot, then member, then z) for the back projection
        std::vector<size_t> cur(nsegs);
        for (int si = 0; si < nsegs; ++si) cur[si] = static_cast<size_t>(G.member_off[si]);
        for (int slot = 0; slot < ncols; ++slot) {
          G.col_starts.push_back(static_cast<int>(G.cmaj.size()));
          for (int si = 0; si < nsegs; ++si) {
            const size_t end = si + 1 < nsegs ? static_cast<size_t>(G.member_off[si + 1]) : G.elems.size();
            while (cur[si] < end && static_cast<int>(G.elems[cur[si]].sz & 0xffffu) == slot) {
              const PathElem& e = G.elems[cur[si]];
              G.cmaj.push_back(PathCElem{(e.sz >> 16) | (static_cast<uint32_t>(si) << 16), e.v});
              ++cur[si];
            }
          }
        }
        G.col_starts.push_back(static_cast<int>(G.cmaj.size()));
      } catch (const std::exception&) {
        G.ok = false;  // the per-basic-bin kernels are used instead
      }
    }
  };
  const int nthreads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) {
    const int g0 = static_cast<int>(static_cast<int64_t>(ngroups) * t / nthreads);
    const int g1 = static_cast<int>(static_cast<int64_t>(ngroups) * (t + 1) / nthreads);
    pool.emplace_back(work, g0, g1);
  }
  for (auto& th : pool) th.join();
  int over = 0;
  for (const Group& G : groups) {
    if (!G.ok) return;
    over = std::max(over, G.over);
  }
  // padded staging: zero planes between the staged columns cover every pass's reads outside [0, nz), so
  // the forward needs no per-lane range tests (a cap keeps the staging buffer small, and at most 2048 planes
  // per staged column keep every staged index within the 16 bits the padded kernels store it in)
  const int zpad = over <= 64 && nz + ((over + 3) & ~3) <= 2048 ? (over + 3) & ~3 : -1;
  const int K = std::max(8, 32768 / (4 * (nz + std::max(zpad, 0))));  // 32 KB of staged float columns
  // chunk c of a row covers its elements with slot in [c K, (c + 1) K)
  for (Group& G : groups) {
    const int ncols = static_cast<int>(G.cols.size());
    const int nch = (ncols + K - 1) / K;
    for (size_t m = 0; m < G.member_off.size(); ++m) {
      const size_t b0 = static_cast<size_t>(G.member_off[m]);
      const size_t b1 = m + 1 < G.member_off.size() ? static_cast<size_t>(G.member_off[m + 1]) : G.elems.size();
      G.member_chunk.push_back(static_cast<int>(G.chunks.size()));
      size_t k = b0;
      for (int c = 0; c <= nch; ++c) {
        const uint32_t lim = static_cast<uint32_t>(std::min(c * K, ncols));
        while (k < b1 && (G.elems[k].sz & 0xffffu) < lim) ++k;
        G.chunks.push_back(static_cast<int>(k - b0));
      }
    }
  }

  std::vector<PathElem> elems;
  std::vector<PathCElem> cmaj;
  std::vector<int> col_starts;
  std::vector<uint32_t> cols;
  std::vector<int> chunks;
  std::vector<PathLineDev> plines;
  std::vector<PathItemDev> items;
  std::vector<int> item_view, item_out_view;
  int max_lines = 1, max_acc = 1;
  for (int gi = 0; gi < ngroups; ++gi) {
    const Group& G = groups[gi];
    const int vi = gi / ntangs, ti = gi % ntangs;
    const int64_t elem_base = static_cast<int64_t>(elems.size());
    const int chunk_base = static_cast<int>(chunks.size());
    const int col_base = static_cast<int>(cols.size());
    const int64_t cmaj_base = static_cast<int64_t>(cmaj.size());
    const int cs_base = static_cast<int>(col_starts.size());
    cmaj.insert(cmaj.end(), G.cmaj.begin(), G.cmaj.end());
    col_starts.insert(col_starts.end(), G.col_starts.begin(), G.col_starts.end());
    elems.insert(elems.end(), G.elems.begin(), G.elems.end());
    chunks.insert(chunks.end(), G.chunks.begin(), G.chunks.end());
    cols.insert(cols.end(), G.cols.begin(), G.cols.end());
    for (int T = 0; T < 8; ++T) {
      PathItemDev it{};
      it.col_offset = col_base;
      it.ncols = static_cast<int>(G.cols.size());
      it.first_line = static_cast<int>(plines.size());
      it.flags = T;
      it.col_starts = cs_base;
      it.cmaj_off = cmaj_base;
      for (int si = 0; si < nsegs; ++si) {
        const int b = (vi * nsegs + si) * ntangs + ti;
        const ProjBinDev& pb = h.h_bins[b];
        for (int l = 0; l < pb.num_lines; ++l) {
          if ((lines[pb.first_line + l].flags & 7) != T) continue;
          PathLineDev pl{};
          pl.line = pb.first_line + l;
          pl.bin = b;
          pl.elem_off = elem_base + G.member_off[si];
          pl.chunk_off = chunk_base + G.member_chunk[si];
          pl.member = si;
          plines.push_back(pl);
        }
      }
      it.num_lines = static_cast<int>(plines.size()) - it.first_line;
      if (it.num_lines == 0) continue;
      max_lines = std::max(max_lines, it.num_lines);
      int nax_sum = 0;
      for (int l = it.first_line; l < it.first_line + it.num_lines; ++l) nax_sum += g.nax(lines[plines[l].line].seg);
      max_acc = std::max(max_acc, path_parts(it.num_lines) * nax_sum);
      items.push_back(it);
      item_view.push_back(bviews[vi]);
      int ov = lines[plines[it.first_line].line].view;
      for (int l = it.first_line; l < it.first_line + it.num_lines; ++l)
        if (lines[plines[l].line].view != ov) ov = -1;
      item_out_view.push_back(ov);
    }
  }
  if (elems.size() >= (size_t(1) << 31) || chunks.size() >= (size_t(1) << 31) || col_starts.size() >= (size_t(1) << 31))
    return;
  int npa_max = 1;
  for (int sg = -g.S(); sg <= g.S(); ++sg) npa_max = std::max(npa_max, g.npa(sg));
  int max_chunk = 1;
  for (const Group& G : groups)
    for (size_t m = 0; m < G.member_chunk.size(); ++m) {
      const int c1 = m + 1 < G.member_chunk.size() ? G.member_chunk[m + 1] : static_cast<int>(G.chunks.size());
      for (int c = G.member_chunk[m]; c + 1 < c1; ++c) max_chunk = std::max(max_chunk, G.chunks[c + 1] - G.chunks[c]);
    }
  if (path_smem_fwd(K, nz, zpad, max_lines, max_acc, npa_max).total > 200 * 1024 ||
      path_smem_back(nz, max_lines, nsegs, nax_max, npa_max).total > 200 * 1024)
    return;

  h.path_elems.upload(elems, h.stream);
  h.path_cols.upload(cols, h.stream);
  h.path_lines.upload(plines, h.stream);
  h.path_items.upload(items, h.stream);
  h.path_chunks.upload(chunks, h.stream);
  h.path_cmaj.upload(cmaj, h.stream);
  h.path_col_starts.upload(col_starts, h.stream);
  ck(cudaStreamSynchronize(h.stream), "path tables");
  PathParams& pp = h.pparams;
  pp.elems = h.path_elems.p;
  pp.cols = h.path_cols.p;
  pp.lines = h.path_lines.p;
  pp.items = h.path_items.p;
  pp.chunks = h.path_chunks.p;
  pp.K = K;
  pp.max_lines = max_lines;
  pp.nax_max = nax_max;
  pp.npa_max = npa_max;
  pp.max_chunk_elems = max_chunk;
  pp.cmaj = h.path_cmaj.p;
  pp.col_starts = h.path_col_starts.p;
  pp.max_members = nsegs;
  pp.max_acc = max_acc;
  pp.zpad = zpad;
  h.h_item_view = item_view;
  h.h_item_out_view = item_out_view;
  h.paths_view_split = std::find(item_out_view.begin(), item_out_view.end(), -1) == item_out_view.end();
  h.h_path_items = items;
  h.use_paths = true;
}

void setup_projector(b200rt_projector& h) {
  Geometry& g = *h.geo;
  DeviceGuard dg(h.device);
  ck(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking), "cudaStreamCreate");

  const std::vector<int> bviews = g.basic_views();
  const std::vector<int> bsegs = g.basic_segments();
  const std::vector<int> btangs = g.basic_tangs();
  h.num_basic_views = static_cast<int>(bviews.size());

  // related lines, shared by all bins of a (view, seg, tang==0) group
  std::vector<LineDev> lines;
  std::map<long long, std::pair<int, int>> line_groups;
  auto group_lines = [&](int view, int seg, bool tz) {
    const long long key = (static_cast<long long>(view) * 1024 + (seg + 512)) * 2 + (tz ? 1 : 0);
    auto it = line_groups.find(key);
    if (it != line_groups.end()) return it->second;
    std::vector<RelatedLine> rel;
    g.related_lines(view, seg, tz, rel);
    const int first = static_cast<int>(lines.size());
    for (const auto& r : rel) {
      LineDev L;
      L.view = static_cast<int16_t>(r.view);
      L.seg = static_cast<int16_t>(r.seg);
      L.tang_sign = static_cast<int8_t>(r.tang_sign);
      L.flags = static_cast<int8_t>((r.op.swap ? 1 : 0) | (r.op.sx < 0 ? 2 : 0) | (r.op.sy < 0 ? 4 : 0) | (r.op.zq ? 8 : 0));
      if (r.op.q < -32768 || r.op.q > 32767) throw std::runtime_error("z transform out of range");
      L.q = static_cast<int16_t>(r.op.q);
      lines.push_back(L);
    }
    const std::pair<int, int> v(first, static_cast<int>(rel.size()));
    line_groups[key] = v;
    return v;
  };

  std::vector<Ray> rays;
  std::vector<BasicBin> bbs;
  for (int v : bviews)
    for (int s : bsegs)
      for (int t : btangs) {
        bbs.push_back(g.make_basic_bin(v, s, t, 0, rays));
      }
  const int nb = static_cast<int>(bbs.size());
  h.h_bins.resize(nb);
  h.h_bin_view.resize(nb);
  h.h_bin_seg.resize(nb);

  // device copies of the rays
  std::vector<RayDev> hrays(rays.size());
  for (size_t i = 0; i < rays.size(); ++i) {
    for (int k = 0; k < 3; ++k) {
      hrays[i].start[k] = rays[i].start[k];
      hrays[i].stop[k] = rays[i].stop[k];
    }
    hrays[i].norm_const = rays[i].norm_const;
  }
  DevBuf<RayDev> d_rays;
  d_rays.upload(hrays, h.stream);

  // build in batches with bounded scratch (2*capacity RowKV elements per bin)
  const size_t budget = size_t(1) << 27;  // RowKV elements of scratch per batch (2 GiB)
  std::vector<int64_t> row_len(nb, 0);
  std::vector<std::unique_ptr<DevBuf<RowElem>>> batch_rows;
  std::vector<std::pair<int, int>> batch_ranges;
  DevBuf<RowKV> scratch;
  DevBuf<BuildBinDev> d_bb;
  DevBuf<int> d_counts;
  DevBuf<int64_t> d_off;
  const float vox[3] = {g.desc().voxel_size_z, g.desc().voxel_size_y, g.desc().voxel_size_x};
  int b0 = 0;
  while (b0 < nb) {
    std::vector<BuildBinDev> hb;
    size_t need = 0;
    int b1 = b0;
    while (b1 < nb) {
      const size_t c = 2 * static_cast<size_t>(bbs[b1].capacity);
      if (b1 > b0 && need + c > budget) break;
      BuildBinDev d{};
      d.first_ray = bbs[b1].first_ray;
      d.num_rays = bbs[b1].num_rays;
      d.direct = bbs[b1].direct;
      d.nlz = bbs[b1].num_lors_per_axial_pos;
      d.z_origin_in_planes = bbs[b1].z_origin_in_planes;
      d.z_centre = bbs[b1].z_centre;
      d.left_edge = bbs[b1].left_edge;
      d.tor_width = bbs[b1].tor_width;
      d.scratch_offset = static_cast<int64_t>(need);
      d.capacity = bbs[b1].capacity;
      hb.push_back(d);
      need += c;
      ++b1;
    }
    const int n = b1 - b0;
    scratch.alloc(std::max(need, scratch.n));
    d_bb.upload(hb, h.stream);
    d_counts.alloc(n);
    ck(launch_build_rows(d_rays.p, d_bb.p, n, vox, scratch.p, d_counts.p, h.stream), "build rows");
    std::vector<int> counts(n);
    ck(cudaMemcpyAsync(counts.data(), d_counts.p, n * sizeof(int), cudaMemcpyDeviceToHost, h.stream), "counts");
    ck(cudaStreamSynchronize(h.stream), "build rows");
    std::vector<int64_t> off(n + 1, 0);
    for (int i = 0; i < n; ++i) {
      if (counts[i] < 0) {
        static const char* why[] = {"", "ray split too deep", "row capacity exceeded", "add_adjacent_z capacity exceeded",
                                    "z copies capacity exceeded", "row element outside the packed coordinate range"};
        const int c = -counts[i];
        throw std::runtime_error(std::string("row builder: ") + (c >= 1 && c <= 5 ? why[c] : "unknown error"));
      }
      row_len[b0 + i] = counts[i];
      off[i + 1] = off[i] + counts[i];
    }
    d_off.upload(off, h.stream);
    auto out = std::make_unique<DevBuf<RowElem>>();
    out->alloc(std::max<int64_t>(off[n], 1));
    ck(launch_compact_rows(d_bb.p, n, scratch.p, d_off.p, out->p, h.stream), "compact rows");
    ck(cudaStreamSynchronize(h.stream), "compact rows");
    batch_rows.push_back(std::move(out));
    batch_ranges.push_back({b0, b1});
    b0 = b1;
  }
  scratch.release();

  int64_t total = 0;
  int max_len = 0;
  for (int b = 0; b < nb; ++b) {
    total += row_len[b];
    max_len = std::max<int>(max_len, static_cast<int>(row_len[b]));
  }
  h.rows.alloc(std::max<int64_t>(total, 1));
  int64_t pos = 0;
  for (size_t i = 0; i < batch_rows.size(); ++i) {
    int64_t cnt = 0;
    for (int b = batch_ranges[i].first; b < batch_ranges[i].second; ++b) cnt += row_len[b];
    if (cnt > 0)
      ck(cudaMemcpyAsync(h.rows.p + pos, batch_rows[i]->p, cnt * sizeof(RowElem), cudaMemcpyDeviceToDevice, h.stream),
         "rows");
    pos += cnt;
  }
  ck(cudaStreamSynchronize(h.stream), "rows");
  batch_rows.clear();

  if (g.num_tof() == 1) {
    pos = 0;
    for (int b = 0; b < nb; ++b) {
      const BasicBin& bb = bbs[b];
      const auto lg = group_lines(bb.view, bb.seg, bb.tang == 0);
      ProjBinDev pb{};
      pb.row_offset = pos;
      pb.row_len = static_cast<int32_t>(row_len[b]);
      pb.tang = static_cast<int16_t>(bb.tang);
      pb.tof = static_cast<int16_t>(bb.tof);
      pb.first_line = lg.first;
      pb.num_lines = lg.second;
      h.h_bins[b] = pb;
      h.h_bin_view[b] = bb.view;
      h.h_bin_seg[b] = bb.seg;
      h.bin_index[h.bin_key(bb.view, bb.seg, bb.tang, bb.tof)] = b;
      pos += row_len[b];
    }
  } else {
    // TOF: every basic row weighted by the kernel of each timing bin (ProjMatrixByBin.inl:66-72,115-185)
    const int nt = g.num_tof();
    std::vector<TofJobDev> jobs(static_cast<size_t>(nb) * nt);
    int64_t src = 0;
    for (int b = 0; b < nb; ++b) {
      float mid[3], unit[3];
      g.lor_middle_and_direction(bbs[b].seg, bbs[b].view, bbs[b].tang, mid, unit);
      for (int k = 0; k < nt; ++k) {
        TofJobDev& j = jobs[static_cast<size_t>(b) * nt + k];
        j.src_offset = src;
        j.src_len = static_cast<int>(row_len[b]);
        j.tof_index = k;
        for (int c = 0; c < 3; ++c) {
          j.mid[c] = mid[c];
          j.unit[c] = unit[c];
        }
      }
      src += row_len[b];
    }
    // FastErf table (numerics/FastErf.inl:21-36) with ProjMatrixByBin's 200000 samples on [-5,5]
    const int ns = 200000;
    const double emax = 5.0, period = (2 * emax) / ns;
    std::vector<double> table(ns + 2);
    for (int i = 0; i < ns + 2; ++i) table[i] = std::erf(i * period - emax);
    std::vector<float> low(nt), high(nt);
    for (int k = 0; k < nt; ++k) {
      low[k] = g.tof_low(g.min_tof() + k);
      high[k] = g.tof_high(g.min_tof() + k);
    }
    DevBuf<double> d_table;
    DevBuf<float> d_low, d_high;
    DevBuf<TofJobDev> d_jobs;
    d_table.upload(table, h.stream);
    d_low.upload(low, h.stream);
    d_high.upload(high, h.stream);
    d_jobs.upload(jobs, h.stream);
    TofParams tp{};
    tp.vox[0] = g.desc().voxel_size_z;
    tp.vox[1] = g.desc().voxel_size_y;
    tp.vox[2] = g.desc().voxel_size_x;
    tp.origin[0] = g.desc().origin_z;
    tp.origin[1] = g.desc().origin_y;
    tp.origin[2] = g.desc().origin_x;
    tp.scanner_z_offset = g.scanner_z_offset();
    tp.r_sqrt2_sigma = g.r_sqrt2_gauss_sigma();
    tp.low = d_low.p;
    tp.high = d_high.p;
    tp.erf_table = d_table.p;
    tp.erf_n = ns + 2;
    tp.erf_max = emax;
    tp.erf_period = period;
    const int njobs = static_cast<int>(jobs.size());
    DevBuf<int> d_cnt;
    d_cnt.alloc(njobs);
    ck(launch_tof_rows(h.rows.p, d_jobs.p, njobs, tp, nullptr, nullptr, d_cnt.p, h.stream), "TOF rows");
    std::vector<int> cnt(njobs);
    ck(cudaMemcpyAsync(cnt.data(), d_cnt.p, njobs * sizeof(int), cudaMemcpyDeviceToHost, h.stream), "counts");
    ck(cudaStreamSynchronize(h.stream), "TOF rows");
    std::vector<int64_t> off(njobs + 1, 0);
    for (int j = 0; j < njobs; ++j) off[j + 1] = off[j] + cnt[j];
    DevBuf<int64_t> d_off2;
    d_off2.upload(off, h.stream);
    DevBuf<RowElem> tof_rows;
    tof_rows.alloc(std::max<int64_t>(off[njobs], 1));
    ck(launch_tof_rows(h.rows.p, d_jobs.p, njobs, tp, d_off2.p, tof_rows.p, d_cnt.p, h.stream), "TOF rows");
    ck(cudaStreamSynchronize(h.stream), "TOF rows");
    std::swap(h.rows.p, tof_rows.p);
    std::swap(h.rows.n, tof_rows.n);
    total = off[njobs];
    {
      // keep the non-TOF rows (now in tof_rows) and the weights of every timing bin for the TOF-grouped kernels
      std::swap(h.tof_basic_rows.p, tof_rows.p);
      std::swap(h.tof_basic_rows.n, tof_rows.n);
      h.tof_w.alloc(std::max<int64_t>(src, 1) * nt);
      ck(launch_tof_weights(h.tof_basic_rows.p, d_jobs.p, njobs, tp, nt, h.tof_w.p, h.stream), "TOF weights");
      std::vector<ProjBinDev> tb(nb);
      h.h_tof_basic_view.resize(nb);
      for (int b = 0; b < nb; ++b) {
        const auto lg = group_lines(bbs[b].view, bbs[b].seg, bbs[b].tang == 0);
        ProjBinDev pb{};
        pb.row_offset = jobs[static_cast<size_t>(b) * nt].src_offset;
        pb.row_len = static_cast<int32_t>(row_len[b]);
        pb.tang = static_cast<int16_t>(bbs[b].tang);
        pb.tof = static_cast<int16_t>(g.min_tof());
        pb.first_line = lg.first;
        pb.num_lines = lg.second;
        tb[b] = pb;
        h.h_tof_basic_view[b] = bbs[b].view;
      }
      h.tof_basic.upload(tb, h.stream);
      ck(cudaStreamSynchronize(h.stream), "TOF weights");
    }
    h.h_bins.resize(njobs);
    h.h_bin_view.resize(njobs);
    h.h_bin_seg.resize(njobs);
    for (int b = 0; b < nb; ++b) {
      const BasicBin& bb = bbs[b];
      const auto lg = group_lines(bb.view, bb.seg, bb.tang == 0);
      for (int k = 0; k < nt; ++k) {
        const int j = b * nt + k;
        ProjBinDev pb{};
        pb.row_offset = off[j];
        pb.row_len = cnt[j];
        pb.tang = static_cast<int16_t>(bb.tang);
        pb.tof = static_cast<int16_t>(g.min_tof() + k);
        pb.first_line = lg.first;
        pb.num_lines = lg.second;
        h.h_bins[j] = pb;
        h.h_bin_view[j] = bb.view;
        h.h_bin_seg[j] = bb.seg;
        h.bin_index[h.bin_key(bb.view, bb.seg, bb.tang, g.min_tof() + k)] = j;
      }
    }
  }
  h.bins.upload(h.h_bins, h.stream);
  h.lines.upload(lines, h.stream);
  h.h_lines = lines;
  std::vector<SegDev> sd(2 * g.S() + 1);
  for (int s = -g.S(); s <= g.S(); ++s) {
    sd[s + g.S()].dev_offset = g.dev_segment_offset(s);
    sd[s + g.S()].nax = g.nax(s);
    sd[s + g.S()].npa = g.npa(s);
  }
  h.segs.upload(sd, h.stream);

  ProjParams& p = h.params;
  p.rows = h.rows.p;
  p.bins = h.bins.p;
  p.lines = h.lines.p;
  p.segs = h.segs.p;
  p.S = g.S();
  p.num_views = g.num_views();
  p.num_tang = g.num_tang();
  p.min_tang = g.min_tang();
  p.max_tang = g.max_tang();
  p.num_tof = g.num_tof();
  p.min_tof = g.min_tof();
  p.tof_stride = g.tof_stride();
  p.nz = g.desc().nz;
  p.ny = g.desc().ny;
  p.nx = g.desc().nx;
  p.min_z = g.desc().min_z;
  p.min_y = g.desc().min_y;
  p.min_x = g.desc().min_x;
  p.max_row_len = max_len;
  p.tof_basic_rows = h.tof_basic_rows.p;
  p.tof_w = h.tof_w.p;
  p.tof_basic = h.tof_basic.p;
  p.uniform_npa = g.npa(0);
  p.max_nax = 0;
  for (int s = -g.S(); s <= g.S(); ++s) p.max_nax = std::max(p.max_nax, g.nax(s));
  for (int s = -g.S(); s <= g.S(); ++s)
    if (g.npa(s) != p.uniform_npa) p.uniform_npa = 0;
  if (static_cast<int64_t>(p.nz) * p.ny * p.nx >= (int64_t(1) << 31)) throw std::runtime_error("image too large");
  const size_t smem = projector_smem_bytes(p);
  if (smem > 220 * 1024) throw std::runtime_error("basic row too long for shared memory");

  // total number of (bin, element) pairs inside the image
  {
    int64_t t = 0;
    std::vector<RowElem> hr(static_cast<size_t>(total));
    if (total > 0) ck(cudaMemcpy(hr.data(), h.rows.p, total * sizeof(RowElem), cudaMemcpyDeviceToHost), "rows");
    for (size_t b = 0; b < h.h_bins.size(); ++b) {
      const ProjBinDev& pb = h.h_bins[b];
      for (int l = 0; l < pb.num_lines; ++l) {
        const LineDev& L = lines[pb.first_line + l];
        const int tang = L.tang_sign * pb.tang;
        if (tang < g.min_tang() || tang > g.max_tang()) continue;
        const int npa = g.npa(L.seg), nax = g.nax(L.seg);
        for (int k = 0; k < pb.row_len; ++k) {
          int z, y, x;
          unpack_zyx(hr[pb.row_offset + k].zyx, z, y, x);
          const int zt = ((L.flags & 8) ? L.q - z : z) - p.min_z;
          // number of a in [0,nax) with 0 <= zt + npa*a < nz
          int lo = zt >= 0 ? 0 : (-zt + npa - 1) / npa;
          int hi = (p.nz - 1 - zt) >= 0 ? (p.nz - 1 - zt) / npa : -1;
          hi = std::min(hi, nax - 1);
          if (hi >= lo) t += hi - lo + 1;
        }
      }
    }
    h.total_nnz = t;
    if (g.num_tof() == 1)
      build_paths(h, hr, lines, static_cast<int>(bviews.size()), static_cast<int>(bsegs.size()),
                  static_cast<int>(btangs.size()), bviews);
  }
}

// device list of the basic bins in subset `subset` of `nsub` (find_basic_vs_nums_in_subset.cxx:32-70)
const int* subset_list(b200rt_projector& h, int subset, int nsub, int& count) {
  const auto key = std::make_pair(subset, nsub);
  auto it = h.subset_lists.find(key);
  if (it != h.subset_lists.end()) {
    count = h.subset_counts[key];
    return it->second->p;
  }
  std::vector<int> list;
  for (int b = 0; b < static_cast<int>(h.h_bins.size()); ++b)
    if (h.h_bin_view[b] % nsub == subset) list.push_back(b);
  auto buf = std::make_unique<DevBuf<int>>();
  buf->upload(list, h.stream);
  ck(cudaStreamSynchronize(h.stream), "subset list");
  count = static_cast<int>(list.size());
  h.subset_counts[key] = count;
  const int* p = buf->p;
  h.subset_lists[key] = std::move(buf);
  return p;
}

// path items (column-staged kernels) of a subset: those whose basic view v has v mod nsub == subset
const int* path_list(b200rt_projector& h, int subset, int nsub, int& count) {
  const auto key = std::make_pair(subset, nsub);
  auto it = h.path_lists.find(key);
  if (it != h.path_lists.end()) {
    count = h.path_counts[key];
    return it->second->p;
  }
  std::vector<int> list;
  for (int i = 0; i < static_cast<int>(h.h_item_view.size()); ++i)
    if (h.h_item_view[i] % nsub == subset) list.push_back(i);
  auto buf = std::make_unique<DevBuf<int>>();
  buf->upload(list, h.stream);
  ck(cudaStreamSynchronize(h.stream), "path list");
  count = static_cast<int>(list.size());
  h.path_counts[key] = count;
  const int* p = buf->p;
  h.path_lists[key] = std::move(buf);
  return p;
}

// basic bins (TOF-grouped kernels) of a subset: those whose basic view v has v mod nsub == subset
const int* tof_group_list(b200rt_projector& h, int subset, int nsub, int& count) {
  const auto key = std::make_pair(subset, nsub);
  auto it = h.tof_group_lists.find(key);
  if (it != h.tof_group_lists.end()) {
    count = h.tof_group_counts[key];
    return it->second->p;
  }
  std::vector<int> list;
  for (int b = 0; b < static_cast<int>(h.h_tof_basic_view.size()); ++b)
    if (h.h_tof_basic_view[b] % nsub == subset) list.push_back(b);
  auto buf = std::make_unique<DevBuf<int>>();
  buf->upload(list, h.stream);
  ck(cudaStreamSynchronize(h.stream), "TOF group list");
  count = static_cast<int>(list.size());
  h.tof_group_counts[key] = count;
  const int* p = buf->p;
  h.tof_group_lists[key] = std::move(buf);
  return p;
}

// forward projection of one subset with the column-staged kernel where it applies (not for the
// log-likelihood, whose per-CTA partial sums follow the basic bins), else the per-basic-bin kernel
void forward_subset(b200rt_projector& h, const float* image, float* out, int subset, int nsub, cudaStream_t st,
                    const FwdEpilogue* ep = nullptr) {
  int n = 0;
  if (h.use_paths && (!ep || ep->mode != kEpiLoglik)) {
    const int* list = path_list(h, subset, nsub, n);
    ck(launch_forward_paths(h.params, h.pparams, list, n, image, out, st, ep), "forward projection");
  } else if (h.params.tof_w && (!ep || ep->mode != kEpiLoglik)) {  // log-likelihood partials: see its entry point
    const int* list = tof_group_list(h, subset, nsub, n);
    ck(launch_forward_tof_grouped(h.params, list, n, image, out, st, ep), "forward projection");
  } else {
    const int* list = subset_list(h, subset, nsub, n);
    ck(launch_forward(h.params, list, n, image, out, st, ep), "forward projection");
  }
}

// device list of every view of the subset: the basic views and their symmetry partners
const int* subset_views(b200rt_projector& h, int subset, int nsub, int& count) {
  const auto key = std::make_pair(subset, nsub);
  auto it = h.subset_views.find(key);
  if (it != h.subset_views.end()) {
    count = h.subset_view_counts[key];
    return it->second->p;
  }
  const Geometry& g = *h.geo;
  std::vector<char> in(g.num_views(), 0);
  for (int v : g.basic_views()) {
    if (v % nsub != subset) continue;
    for (int seg : g.basic_segments()) {
      std::vector<RelatedLine> rel;
      g.related_lines(v, seg, true, rel);
      for (const auto& r : rel) in[r.view] = 1;
    }
  }
  std::vector<int> views;
  for (int v = 0; v < g.num_views(); ++v)
    if (in[v]) views.push_back(v);
  auto buf = std::make_unique<DevBuf<int>>();
  buf->upload(views, h.stream);
  ck(cudaStreamSynchronize(h.stream), "subset views");
  count = static_cast<int>(views.size());
  h.subset_view_counts[key] = count;
  const int* p = buf->p;
  h.subset_views[key] = std::move(buf);
  return p;
}

// QuadraticPrior / RelativeDifferencePrior weights: voxel_x / distance (QuadraticPrior.cxx:203-230)
void prior_weights(const Geometry& g, int only_2D, float w[27]) {
  const float vz = g.desc().voxel_size_z, vy = g.desc().voxel_size_y, vx = g.desc().voxel_size_x;
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        float v = 0.f;
        if (!(z == 0 && y == 0 && x == 0) && !(only_2D && z != 0)) {
          const float a = static_cast<float>(x) * vx, b = static_cast<float>(y) * vy, c = static_cast<float>(z) * vz;
          v = vx / std::sqrt(a * a + b * b + c * c);
        }
        w[(z + 1) * 9 + (y + 1) * 3 + (x + 1)] = v;
      }
}

// Back projection of the subset into image_dev (overwritten), atomic or deterministic.
// max_abs > 0: a bound on |pd| known in advance (the OSMAPOSL ratio is at most 1e4), which keeps the
// fixed-point scale independent of bins outside the subset
void back_project_into(b200rt_projector& h, const float* pd, float* image, int subset, int nsub, int mode, int zero_ends,
                       cudaStream_t st, float max_abs = 0.f) {
  const Geometry& g = *h.geo;
  const int64_t ni = g.image_size();
  int n = 0;
  const bool grouped = !h.use_paths && h.params.tof_w;
  const int* list = h.use_paths ? path_list(h, subset, nsub, n)
                    : grouped   ? tof_group_list(h, subset, nsub, n)
                                : subset_list(h, subset, nsub, n);
  if (mode == B200RT_BACKPROJECT_ATOMIC) {
    ck(cudaMemsetAsync(image, 0, sizeof(float) * ni, st), "memset");
    if (h.use_paths)
      ck(launch_back_paths_atomic(h.params, h.pparams, list, n, pd, image, st, zero_ends), "back projection");
    else if (grouped)
      ck(launch_back_tof_grouped(h.params, list, n, pd, image, nullptr, nullptr, st, zero_ends), "back projection");
    else
      ck(launch_back_atomic(h.params, list, n, pd, image, st, zero_ends), "back projection");
    return;
  }
  h.det_partial.alloc(std::max<int>(update_num_blocks(std::max<int64_t>(g.projdata_size(), ni)), 1));
  if (!h.colmax_ready) {
    // largest column sum of A (A^T 1 over every bin): bounds every voxel's sum of |w d| / max|d|
    h.colmax.alloc(1);
    int nall = 0;
    const int* all = h.use_paths ? path_list(h, 0, 1, nall)
                     : grouped   ? tof_group_list(h, 0, 1, nall)
                                 : subset_list(h, 0, 1, nall);
    ck(cudaMemsetAsync(image, 0, sizeof(float) * ni, st), "memset");
    if (h.use_paths)
      ck(launch_back_paths_atomic(h.params, h.pparams, all, nall, nullptr, image, st, 0), "column sums");
    else if (grouped)
      ck(launch_back_tof_grouped(h.params, all, nall, nullptr, image, nullptr, nullptr, st, 0), "column sums");
    else
      ck(launch_back_atomic(h.params, all, nall, nullptr, image, st, 0), "column sums");
    ck(launch_max(image, ni, h.det_partial.p, h.colmax.p, st), "column sums");
    h.colmax_ready = true;
  }
  h.acc64.alloc(ni);
  h.fixed_scale.alloc(1);
  if (max_abs > 0) {
    if (h.det_bound_value != max_abs) {
      h.det_bound.alloc(1);
      ck(cudaMemcpy(h.det_bound.p, &max_abs, sizeof(float), cudaMemcpyHostToDevice), "H2D");
      h.det_bound_value = max_abs;
    }
    ck(launch_fixed_scale(h.det_bound.p, 1, h.colmax.p, h.det_partial.p, h.fixed_scale.p, st), "scale");
  } else {
    ck(launch_fixed_scale(pd, pd ? g.projdata_size() : 1, h.colmax.p, h.det_partial.p, h.fixed_scale.p, st), "scale");
  }
  ck(cudaMemsetAsync(h.acc64.p, 0, sizeof(unsigned long long) * ni, st), "memset");
  if (h.use_paths)
    ck(launch_back_paths_fixed(h.params, h.pparams, list, n, pd, h.acc64.p, h.fixed_scale.p, st, zero_ends),
       "back projection");
  else if (grouped)
    ck(launch_back_tof_grouped(h.params, list, n, pd, nullptr, h.acc64.p, h.fixed_scale.p, st, zero_ends),
       "back projection");
  else
    ck(launch_back_fixed(h.params, list, n, pd, h.acc64.p, h.fixed_scale.p, st, zero_ends), "back projection");
  ck(launch_fixed_to_float(h.acc64.p, h.fixed_scale.p, image, ni, st), "back projection");
}

int check_subset(b200rt_projector* h, int subset, int nsub) {
  if (nsub < 1 || subset < 0 || subset >= nsub) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "invalid subset number");
  return B200RT_OK;
}

cudaError_t projdata_layout(const Geometry& g, const float* in, float* out, bool to_dev, cudaStream_t st) {
  const int64_t nvt = static_cast<int64_t>(g.num_views()) * g.num_tang();
  for (int k = 0; k < g.num_tof(); ++k)
    for (int s = -g.S(); s <= g.S(); ++s) {
      const int64_t so = k * g.tof_stride() + g.stir_segment_offset(s);
      const int64_t dv = k * g.tof_stride() + g.dev_segment_offset(s);
      const cudaError_t e = to_dev ? launch_projdata_to_dev(in + so, out + dv, g.nax(s), nvt, st)
                                   : launch_projdata_from_dev(in + dv, out + so, g.nax(s), nvt, st);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

// projection data layout change of the views [v0, v1) only (STIR order <-> device layout)
cudaError_t projdata_layout_views(const Geometry& g, const float* in, float* out, bool to_dev, int v0, int v1,
                                  cudaStream_t st) {
  const int64_t nt = g.num_tang(), nvt = static_cast<int64_t>(g.num_views()) * nt;
  const int64_t c0 = v0 * nt, nc = (v1 - v0) * nt;
  for (int k = 0; k < g.num_tof(); ++k)
    for (int s = -g.S(); s <= g.S(); ++s) {
      const int64_t so = k * g.tof_stride() + g.stir_segment_offset(s) + c0;
      const int64_t dv = k * g.tof_stride() + g.dev_segment_offset(s) + c0 * g.nax(s);
      const int nax = g.nax(s);
      const cudaError_t e = to_dev ? launch_transpose(in + so, out + dv, nax, nc, nvt, nax, st)
                                   : launch_transpose(in + dv, out + so, static_cast<int>(nc), nax, nax, nvt, st);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

// copy of the views [v0, v1) of projection data in STIR order (rows of views x tangential positions for every
// timing bin, segment and axial position): one strided copy
cudaError_t copy_views(const Geometry& g, float* dst, const float* src, int v0, int v1, cudaMemcpyKind kind,
                       cudaStream_t st) {
  const size_t nt = static_cast<size_t>(g.num_tang()), nvt = nt * static_cast<size_t>(g.num_views());
  const size_t rows = static_cast<size_t>(g.projdata_size()) / nvt;
  return cudaMemcpy2DAsync(dst + nt * v0, sizeof(float) * nvt, src + nt * v0, sizeof(float) * nvt,
                           sizeof(float) * nt * (v1 - v0), rows, kind, st);
}

constexpr int kHostViewGroups = 8;

// the subset's path items ordered by the group of views they write (kHostViewGroups view ranges)
const b200rt_projector::ViewGroups& view_groups(b200rt_projector& h, int subset, int nsub) {
  const auto key = std::make_pair(subset, nsub);
  auto it = h.view_groups.find(key);
  if (it != h.view_groups.end()) return it->second;
  const int nv = h.geo->num_views();
  const int G = std::min(kHostViewGroups, nv);
  b200rt_projector::ViewGroups vg;
  if (G == kHostViewGroups && nv >= 120) {
    // tapered (with at least 4 views per unit of size): the copy that cannot overlap a projection (the forward's last group, the back projection's first)
    // is of a small group; relative sizes 1, 2, 4, 8, 8, 4, 2, 1
    static const int w[kHostViewGroups] = {1, 2, 4, 8, 8, 4, 2, 1};
    int acc = 0, total = 0;
    for (int gi = 0; gi < G; ++gi) total += w[gi];
    vg.v0.push_back(0);
    for (int gi = 0; gi < G; ++gi) {
      acc += w[gi];
      vg.v0.push_back(std::max(vg.v0.back() + 1, static_cast<int>(static_cast<int64_t>(nv) * acc / total)));
    }
    vg.v0.back() = nv;
  } else {
    for (int gi = 0; gi <= G; ++gi) vg.v0.push_back(static_cast<int>(static_cast<int64_t>(nv) * gi / G));
  }
  std::vector<std::vector<int>> per(G);
  for (int i = 0; i < static_cast<int>(h.h_item_view.size()); ++i) {
    if (h.h_item_view[i] % nsub != subset) continue;
    const int gi = static_cast<int>(std::upper_bound(vg.v0.begin(), vg.v0.end(), h.h_item_out_view[i]) - vg.v0.begin()) - 1;
    per[gi].push_back(i);
  }
  std::vector<int> list;
  for (int gi = 0; gi < G; ++gi) {
    vg.off.push_back(static_cast<int>(list.size()));
    list.insert(list.end(), per[gi].begin(), per[gi].end());
  }
  vg.off.push_back(static_cast<int>(list.size()));
  vg.list = std::make_unique<DevBuf<int>>();
  vg.list->upload(list, h.stream);
  ck(cudaStreamSynchronize(h.stream), "view groups");
  return h.view_groups.emplace(key, std::move(vg)).first->second;
}

void ensure_copy_stream(b200rt_projector& h) {
  if (!h.copy_stream) ck(cudaStreamCreateWithFlags(&h.copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  while (h.copy_events.size() < kHostViewGroups + 1) {
    cudaEvent_t e = nullptr;
    ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    h.copy_events.push_back(e);
  }
}

}  // namespace

extern "C" {

int b200rt_create(const b200rt_geometry* geometry, int device, b200rt_projector** out) {
  if (!out) return B200RT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!geometry) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_create_error = "null geometry";
    return B200RT_ERR_INVALID_ARGUMENT;
  }
  auto h = std::make_unique<b200rt_projector>();
  try {
    int ndev = 0;
    ck(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) throw std::runtime_error("invalid CUDA device");
    h->device = device;
    h->geo = std::make_unique<Geometry>(*geometry);
    setup_projector(*h);
  } catch (const std::exception& e) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_create_error = e.what();
    const int st = status_of(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    h->stream = nullptr;
    return st == B200RT_ERR_INVALID_ARGUMENT && dynamic_cast<const CudaError*>(&e) == nullptr ? B200RT_ERR_INVALID_ARGUMENT : st;
  }
  *out = h.release();
  return B200RT_OK;
}

void b200rt_destroy(b200rt_projector* h) {
  if (!h) return;
  {
    DeviceGuard dg(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->subset_lists.clear();
    h->subset_views.clear();
    h->path_lists.clear();
    h->ossps_g.release();
    h->ossps_pg.release();
    h->ones.release();
    h->ossps_partial.release();
    h->ossps_minpos.release();
    h->path_elems.release();
    h->path_cols.release();
    h->path_lines.release();
    h->path_items.release();
    h->path_chunks.release();
    h->path_cmaj.release();
    h->path_col_starts.release();
    h->ratio.release();
    h->upd.release();
    h->grad.release();
    h->small_value.release();
    h->partial_max.release();
    h->umax.release();
    h->cancelled.release();
    h->ll_partials.release();
    h->acc64.release();
    h->fixed_scale.release();
    h->colmax.release();
    h->det_partial.release();
    h->det_bound.release();
    h->ll_sum.release();
    h->rows.release();
    h->bins.release();
    h->lines.release();
    h->segs.release();
    h->st_img_a.release();
    h->st_img_b.release();
    h->st_pd_a.release();
    h->st_pd_b.release();
    h->view_groups.clear();
    h->tof_group_lists.clear();
    h->tof_basic_rows.release();
    h->tof_w.release();
    h->tof_basic.release();
    h->lm_table.release();
    h->lm_partial.release();
    h->lm_sum.release();
    h->lm_invalid.release();
    h->lm_fwd.release();
    h->lm_fwd_rhs.release();
    h->lm_hist.release();
    h->lm_img.release();
    h->vg_scratch.release();
    if (h->copy_stream) {
      cudaStreamSynchronize(h->copy_stream);
      cudaStreamDestroy(h->copy_stream);
    }
    for (cudaEvent_t e : h->copy_events) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
  }
  delete h;
}

const char* b200rt_last_error(const b200rt_projector* h) {
  if (!h) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_create_error.c_str();
  }
  return h->err.c_str();
}

int b200rt_get_info(const b200rt_projector* h, b200rt_info* out) {
  if (!h || !out) return B200RT_ERR_INVALID_ARGUMENT;
  const Geometry& g = *h->geo;
  std::memset(out, 0, sizeof(*out));
  out->num_bins = g.projdata_size();
  out->num_image_voxels = g.image_size();
  out->num_basic_bins = static_cast<int64_t>(h->h_bins.size());
  out->num_row_elements = static_cast<int64_t>(h->rows.n);
  out->total_nnz = h->total_nnz;
  out->num_tof_bins = g.num_tof();
  out->num_basic_views = h->num_basic_views;
  out->symmetries_used = g.symmetry_bits();
  return B200RT_OK;
}

int64_t b200rt_projdata_size(const b200rt_projector* h) { return h ? h->geo->projdata_size() : -1; }
int64_t b200rt_image_size(const b200rt_projector* h) { return h ? h->geo->image_size() : -1; }

int b200rt_get_row(b200rt_projector* h, int segment, int view, int axial, int tangential, int timing, int32_t* coords_zyx,
                   float* values, int64_t capacity, int64_t* length) {
  if (!h || !length) return B200RT_ERR_INVALID_ARGUMENT;
  try {
    const Geometry& g = *h->geo;
    if (segment < -g.S() || segment > g.S() || view < 0 || view >= g.num_views() || axial < 0 || axial >= g.nax(segment) ||
        tangential < g.min_tang() || tangential > g.max_tang() || timing < g.min_tof() || timing >= g.min_tof() + g.num_tof())
      return fail(h, B200RT_ERR_INVALID_ARGUMENT, "bin out of range");
    const SymOp op = g.find_op(segment, view, axial, tangential);
    int s = segment, v = view, a = axial, t = tangential, k = timing;
    g.find_basic_bin(s, v, a, t, k);
    auto it = h->bin_index.find(h->bin_key(v, s, t, k));
    if (it == h->bin_index.end()) return fail(h, B200RT_ERR_STATE, "basic bin not found");
    const ProjBinDev& pb = h->h_bins[it->second];
    *length = pb.row_len;
    const int64_t n = std::min<int64_t>(pb.row_len, capacity);
    if (n <= 0) return B200RT_OK;
    if (!coords_zyx || !values) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null output arrays");
    DeviceGuard dg(h->device);
    std::vector<RowElem> r(n);
    ck(cudaMemcpy(r.data(), h->rows.p + pb.row_offset, n * sizeof(RowElem), cudaMemcpyDeviceToHost), "row");
    const int zs = g.npa(segment) * axial;
    for (int64_t i = 0; i < n; ++i) {
      int z, y, x;
      unpack_zyx(r[i].zyx, z, y, x);
      coords_zyx[3 * i + 2] = (op.swap ? y : x) * op.sx;
      coords_zyx[3 * i + 1] = (op.swap ? x : y) * op.sy;
      coords_zyx[3 * i] = (op.zq ? op.q - z : z) + zs;
      values[i] = r[i].v;
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_image_to_device_layout(b200rt_projector* h, const float* stir_dev, float* dev, void* stream) {
  if (!h || !stir_dev || !dev) return B200RT_ERR_INVALID_ARGUMENT;
  const auto& d = h->geo->desc();
  DeviceGuard dg(h->device);
  const cudaError_t e = launch_image_to_dev(stir_dev, dev, d.nz, d.ny, d.nx, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? B200RT_OK : fail(h, B200RT_ERR_CUDA, cudaGetErrorString(e));
}
int b200rt_image_from_device_layout(b200rt_projector* h, const float* dev, float* stir_dev, void* stream) {
  if (!h || !stir_dev || !dev) return B200RT_ERR_INVALID_ARGUMENT;
  const auto& d = h->geo->desc();
  DeviceGuard dg(h->device);
  const cudaError_t e = launch_image_from_dev(dev, stir_dev, d.nz, d.ny, d.nx, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? B200RT_OK : fail(h, B200RT_ERR_CUDA, cudaGetErrorString(e));
}
int b200rt_projdata_to_device_layout(b200rt_projector* h, const float* stir_dev, float* dev, void* stream) {
  if (!h || !stir_dev || !dev) return B200RT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  const cudaError_t e = projdata_layout(*h->geo, stir_dev, dev, true, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? B200RT_OK : fail(h, B200RT_ERR_CUDA, cudaGetErrorString(e));
}
int b200rt_projdata_from_device_layout(b200rt_projector* h, const float* dev, float* stir_dev, void* stream) {
  if (!h || !stir_dev || !dev) return B200RT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  const cudaError_t e = projdata_layout(*h->geo, dev, stir_dev, false, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? B200RT_OK : fail(h, B200RT_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"

namespace {

// the device-layout block of viewgram (segment, view, timing position): [tangential][axial], contiguous
const char* viewgram_block(const b200rt_projector& h, int seg, int view, int tof, int64_t& off, int& nax) {
  const Geometry& g = *h.geo;
  if (seg < -g.S() || seg > g.S()) return "segment out of range";
  if (view < 0 || view >= g.num_views()) return "view out of range";
  if (tof < g.min_tof() || tof >= g.min_tof() + g.num_tof()) return "timing position out of range";
  nax = g.nax(seg);
  off = static_cast<int64_t>(tof - g.min_tof()) * g.tof_stride() + g.dev_segment_offset(seg) +
        static_cast<int64_t>(view) * g.num_tang() * nax;
  return nullptr;
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" {

int b200rt_get_viewgram(b200rt_projector* h, const float* projdata_dev, int segment_num, int view_num,
                        int timing_pos_num, float* viewgram, void* stream) {
  if (!h || !projdata_dev || !viewgram) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  int64_t off = 0;
  int nax = 0;
  if (const char* why = viewgram_block(*h, segment_num, view_num, timing_pos_num, off, nax))
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, why);
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nt = h->geo->num_tang();
    const size_t n = static_cast<size_t>(nt) * nax;
    const bool dev_out = is_device_pointer(viewgram);
    float* dst = viewgram;
    if (!dev_out) {
      h->vg_scratch.alloc(std::max(h->vg_scratch.n, 2 * n));
      dst = h->vg_scratch.p;
    }
    ck(launch_transpose(projdata_dev + off, dst, nt, nax, nax, nt, st), "viewgram");
    if (!dev_out) {
      ck(cudaMemcpyAsync(viewgram, dst, sizeof(float) * n, cudaMemcpyDeviceToHost, st), "D2H");
      ck(cudaStreamSynchronize(st), "viewgram");
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_set_viewgram(b200rt_projector* h, float* projdata_dev, int segment_num, int view_num, int timing_pos_num,
                        const float* viewgram, int accumulate, void* stream) {
  if (!h || !projdata_dev || !viewgram) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  int64_t off = 0;
  int nax = 0;
  if (const char* why = viewgram_block(*h, segment_num, view_num, timing_pos_num, off, nax))
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, why);
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nt = h->geo->num_tang();
    const size_t n = static_cast<size_t>(nt) * nax;
    h->vg_scratch.alloc(std::max(h->vg_scratch.n, 2 * n));
    const float* src = viewgram;
    if (!is_device_pointer(viewgram)) {
      ck(cudaMemcpyAsync(h->vg_scratch.p, viewgram, sizeof(float) * n, cudaMemcpyHostToDevice, st), "H2D");
      src = h->vg_scratch.p;
    }
    // [axial][tangential] -> [tangential][axial]
    if (accumulate) {
      ck(launch_transpose(src, h->vg_scratch.p + n, nax, nt, nt, nax, st), "viewgram");
      ck(launch_add(projdata_dev + off, h->vg_scratch.p + n, static_cast<int64_t>(n), st), "viewgram");
    } else {
      ck(launch_transpose(src, projdata_dev + off, nax, nt, nt, nax, st), "viewgram");
    }
    // the host source may be reused by the caller as soon as this returns
    if (src != viewgram) ck(cudaStreamSynchronize(st), "viewgram");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_forward_project_dev(b200rt_projector* h, const float* image_dev, float* projdata_dev, int subset_num,
                               int num_subsets, void* stream) {
  if (!h || !image_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    forward_subset(*h, image_dev, projdata_dev, subset_num, num_subsets, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_back_project_dev(b200rt_projector* h, const float* projdata_dev, float* image_dev, int subset_num,
                            int num_subsets, int mode, void* stream) {
  if (!h || !image_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (mode != B200RT_BACKPROJECT_ATOMIC && mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    back_project_into(*h, projdata_dev, image_dev, subset_num, num_subsets, mode, 0, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_forward_project(b200rt_projector* h, const float* image_host, float* projdata_host, int subset_num,
                           int num_subsets) {
  if (!h || !image_host || !projdata_host) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = h->stream;
    h->st_img_a.alloc(g.image_size());
    h->st_img_b.alloc(g.image_size());
    h->st_pd_a.alloc(g.projdata_size());
    h->st_pd_b.alloc(g.projdata_size());
    ck(cudaMemcpyAsync(h->st_img_a.p, image_host, sizeof(float) * g.image_size(), cudaMemcpyHostToDevice, st), "H2D");
    ck(launch_image_to_dev(h->st_img_a.p, h->st_img_b.p, g.desc().nz, g.desc().ny, g.desc().nx, st), "layout");
    ck(cudaMemsetAsync(h->st_pd_b.p, 0, sizeof(float) * g.projdata_size(), st), "memset");
    if (h->use_paths && h->paths_view_split) {
      // group by group of views: projection, layout change, then the group's copy to the host on the copy
      // stream while the next group is projected
      const b200rt_projector::ViewGroups& vg = view_groups(*h, subset_num, num_subsets);
      ensure_copy_stream(*h);
      for (size_t gi = 0; gi + 1 < vg.v0.size(); ++gi) {
        const int n = vg.off[gi + 1] - vg.off[gi];
        if (n > 0)
          ck(launch_forward_paths(h->params, h->pparams, vg.list->p + vg.off[gi], n, h->st_img_b.p, h->st_pd_b.p, st,
                                  nullptr),
             "forward projection");
        ck(projdata_layout_views(g, h->st_pd_b.p, h->st_pd_a.p, false, vg.v0[gi], vg.v0[gi + 1], st), "layout");
        ck(cudaEventRecord(h->copy_events[gi], st), "cudaEventRecord");
        ck(cudaStreamWaitEvent(h->copy_stream, h->copy_events[gi], 0), "cudaStreamWaitEvent");
        ck(copy_views(g, projdata_host, h->st_pd_a.p, vg.v0[gi], vg.v0[gi + 1], cudaMemcpyDeviceToHost, h->copy_stream),
           "D2H");
      }
      ck(cudaStreamSynchronize(h->copy_stream), "forward projection");
      ck(cudaStreamSynchronize(st), "forward projection");
      return B200RT_OK;
    }
    forward_subset(*h, h->st_img_b.p, h->st_pd_b.p, subset_num, num_subsets, st);
    ck(projdata_layout(g, h->st_pd_b.p, h->st_pd_a.p, false, st), "layout");
    ck(cudaMemcpyAsync(projdata_host, h->st_pd_a.p, sizeof(float) * g.projdata_size(), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "forward projection");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_back_project(b200rt_projector* h, const float* projdata_host, float* image_host, int subset_num,
                        int num_subsets, int mode) {
  if (!h || !image_host || !projdata_host) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (mode != B200RT_BACKPROJECT_ATOMIC && mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = h->stream;
    h->st_img_a.alloc(g.image_size());
    h->st_img_b.alloc(g.image_size());
    h->st_pd_a.alloc(g.projdata_size());
    h->st_pd_b.alloc(g.projdata_size());
    if (h->use_paths && h->paths_view_split && mode == B200RT_BACKPROJECT_ATOMIC) {
      // group by group of views: the copy stream brings the groups' data in order, the projection stream
      // changes each group's layout and back-projects its items as soon as its data are in
      const b200rt_projector::ViewGroups& vg = view_groups(*h, subset_num, num_subsets);
      ensure_copy_stream(*h);
      const size_t G = vg.v0.size() - 1;
      ck(cudaEventRecord(h->copy_events[G], st), "cudaEventRecord");  // staging buffers free
      ck(cudaStreamWaitEvent(h->copy_stream, h->copy_events[G], 0), "cudaStreamWaitEvent");
      for (size_t gi = 0; gi < G; ++gi) {
        ck(copy_views(g, h->st_pd_a.p, projdata_host, vg.v0[gi], vg.v0[gi + 1], cudaMemcpyHostToDevice, h->copy_stream),
           "H2D");
        ck(cudaEventRecord(h->copy_events[gi], h->copy_stream), "cudaEventRecord");
      }
      ck(cudaMemsetAsync(h->st_img_b.p, 0, sizeof(float) * g.image_size(), st), "memset");
      for (size_t gi = 0; gi < G; ++gi) {
        ck(cudaStreamWaitEvent(st, h->copy_events[gi], 0), "cudaStreamWaitEvent");
        ck(projdata_layout_views(g, h->st_pd_a.p, h->st_pd_b.p, true, vg.v0[gi], vg.v0[gi + 1], st), "layout");
        const int n = vg.off[gi + 1] - vg.off[gi];
        if (n > 0)
          ck(launch_back_paths_atomic(h->params, h->pparams, vg.list->p + vg.off[gi], n, h->st_pd_b.p, h->st_img_b.p,
                                      st, 0),
             "back projection");
      }
    } else {
      ck(cudaMemcpyAsync(h->st_pd_a.p, projdata_host, sizeof(float) * g.projdata_size(), cudaMemcpyHostToDevice, st),
         "H2D");
      ck(projdata_layout(g, h->st_pd_a.p, h->st_pd_b.p, true, st), "layout");
      back_project_into(*h, h->st_pd_b.p, h->st_img_b.p, subset_num, num_subsets, mode, 0, st);
    }
    ck(launch_image_from_dev(h->st_img_b.p, h->st_img_a.p, g.desc().nz, g.desc().ny, g.desc().nx, st), "layout");
    ck(cudaMemcpyAsync(image_host, h->st_img_a.p, sizeof(float) * g.image_size(), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "back projection");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_sensitivity_dev(b200rt_projector* h, const float* mult_dev, float* sens_dev, int subset_num, int num_subsets,
                           int zero_seg0_end_planes, int back_projection_mode, void* stream) {
  if (!h || !sens_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (back_projection_mode != B200RT_BACKPROJECT_ATOMIC && back_projection_mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    back_project_into(*h, mult_dev, sens_dev, subset_num, num_subsets, back_projection_mode, zero_seg0_end_planes,
                      static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"

namespace {

// u = A_S^T divide_and_truncate(y, A_S x + a): fused forward projection/ratio, then back projection
void osmaposl_numerator(b200rt_projector& h, const float* x, const float* y, const float* add, int subset, int nsub,
                        int zero_ends, int mode, float* u, cudaStream_t st) {
  const Geometry& g = *h.geo;
  if (!h.ratio.p) {
    h.ratio.alloc(g.projdata_size());
    ck(cudaMemsetAsync(h.ratio.p, 0, sizeof(float) * g.projdata_size(), st), "memset");  // bins outside the subset
  }
  h.small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
  h.cancelled.alloc(1);
  int nv = 0;
  const int* views = subset_views(h, subset, nsub, nv);
  ck(launch_viewgram_small_values(y, h.segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, zero_ends, g.num_tof(),
                                  g.tof_stride(), h.small_value.p, st),
     "viewgram thresholds");
  ck(cudaMemsetAsync(h.cancelled.p, 0, sizeof(unsigned int), st), "memset");
  FwdEpilogue ep{};
  ep.mode = kEpiRatio;
  ep.zero_ends = zero_ends;
  ep.y = y;
  ep.add = add;
  ep.small_value = h.small_value.p;
  ep.cancelled = h.cancelled.p;
  forward_subset(h, x, h.ratio.p, subset, nsub, st, &ep);
  back_project_into(h, h.ratio.p, u, subset, nsub, mode, 0, st, 10000.F);
}

// u /= denominator, clamp, x *= u (OSMAPOSLReconstruction.cxx:394-510)
void osmaposl_apply(b200rt_projector& h, float* x, float* u, const float* sens, int nsub, int subiter,
                    const b200rt_prior* prior, float min_rel, float max_rel, cudaStream_t st) {
  const Geometry& g = *h.geo;
  const int64_t ni = g.image_size();
  h.partial_max.alloc(update_num_blocks(ni));
  h.umax.alloc(1);
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  if (has_prior) {
    h.grad.alloc(ni);
    prior_weights(g, prior->only_2D, h.prior_w);
  }
  ck(launch_update(u, x, sens, has_prior ? h.grad.p : nullptr, has_prior ? prior : nullptr, h.prior_w, nsub, subiter,
                   min_rel, max_rel, g.desc().ny, g.desc().nx, g.desc().nz, h.partial_max.p, h.umax.p, st),
     "update");
}

int check_mode_prior(b200rt_projector* h, int mode, const b200rt_prior* prior) {
  if (mode != B200RT_BACKPROJECT_ATOMIC && mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  if (prior && (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE))
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  return B200RT_OK;
}

}  // namespace

extern "C" {

int b200rt_osmaposl_subiteration_dev(b200rt_projector* h, float* estimate_dev, const float* y_dev, const float* additive_dev,
                                     const float* sens_dev, int subset_num, int num_subsets, int subiteration_num,
                                     int zero_seg0_end_planes, const b200rt_prior* prior, float min_relative_change,
                                     float max_relative_change, int back_projection_mode, float* update_dev, void* stream) {
  if (!h || !estimate_dev || !y_dev || !sens_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_mode_prior(h, back_projection_mode, prior)) return st;
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!update_dev) h->upd.alloc(h->geo->image_size());
    float* u = update_dev ? update_dev : h->upd.p;
    osmaposl_numerator(*h, estimate_dev, y_dev, additive_dev, subset_num, num_subsets, zero_seg0_end_planes,
                       back_projection_mode, u, st);
    osmaposl_apply(*h, estimate_dev, u, sens_dev, num_subsets, subiteration_num, prior, min_relative_change,
                   max_relative_change, st);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_osmaposl_numerator_dev(b200rt_projector* h, const float* estimate_dev, const float* y_dev,
                                  const float* additive_dev, int subset_num, int num_subsets, int zero_seg0_end_planes,
                                  int back_projection_mode, float* numerator_dev, void* stream) {
  if (!h || !estimate_dev || !y_dev || !numerator_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_mode_prior(h, back_projection_mode, nullptr)) return st;
  try {
    DeviceGuard dg(h->device);
    osmaposl_numerator(*h, estimate_dev, y_dev, additive_dev, subset_num, num_subsets, zero_seg0_end_planes,
                       back_projection_mode, numerator_dev, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_osmaposl_apply_update_dev(b200rt_projector* h, float* estimate_dev, float* numerator_dev, const float* sens_dev,
                                     int num_subsets, int subiteration_num, const b200rt_prior* prior,
                                     float min_relative_change, float max_relative_change, void* stream) {
  if (!h || !estimate_dev || !numerator_dev || !sens_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (num_subsets < 1) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "invalid number of subsets");
  if (int st = check_mode_prior(h, B200RT_BACKPROJECT_ATOMIC, prior)) return st;
  try {
    DeviceGuard dg(h->device);
    osmaposl_apply(*h, estimate_dev, numerator_dev, sens_dev, num_subsets, subiteration_num, prior, min_relative_change,
                   max_relative_change, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_get_num_cancelled(b200rt_projector* h, int64_t* out) {
  if (!h || !out) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    unsigned int c = 0;
    if (h->cancelled.p) ck(cudaMemcpy(&c, h->cancelled.p, sizeof(c), cudaMemcpyDeviceToHost), "D2H");
    *out = c;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_log_likelihood_dev(b200rt_projector* h, const float* image_dev, const float* y_dev, const float* additive_dev,
                              const float* mult_dev, int subset_num, int num_subsets, int zero_seg0_end_planes, double* out,
                              void* stream) {
  if (!h || !image_dev || !y_dev || !out) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int n = 0, nv = 0;
    // one partial sum per CTA: per path item with the column-staged kernel, else per basic bin
    const bool grouped = !h->use_paths && h->params.tof_w;  // one partial per basic bin with all timing bins
    const int* list = h->use_paths ? path_list(*h, subset_num, num_subsets, n)
                      : grouped    ? tof_group_list(*h, subset_num, num_subsets, n)
                                   : subset_list(*h, subset_num, num_subsets, n);
    const int* views = subset_views(*h, subset_num, num_subsets, nv);
    h->small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    if (h->ll_partials.n < static_cast<size_t>(std::max(n, 1))) h->ll_partials.alloc(std::max(n, 1));
    h->ll_sum.alloc(1);
    ck(launch_viewgram_small_values(y_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, zero_seg0_end_planes,
                                    g.num_tof(), g.tof_stride(), h->small_value.p, st),
       "viewgram thresholds");
    FwdEpilogue ep{};
    ep.mode = kEpiLoglik;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.add = additive_dev;
    ep.mult = mult_dev;
    ep.small_value = h->small_value.p;
    ep.partials = h->ll_partials.p;
    if (h->use_paths)
      ck(launch_forward_paths(h->params, h->pparams, list, n, image_dev, nullptr, st, &ep), "log-likelihood");
    else if (grouped)
      ck(launch_forward_tof_grouped(h->params, list, n, image_dev, nullptr, st, &ep), "log-likelihood");
    else
      ck(launch_forward(h->params, list, n, image_dev, nullptr, st, &ep), "log-likelihood");
    ck(launch_reduce_sum(h->ll_partials.p, n, h->ll_sum.p, st), "reduce");
    ck(cudaMemcpyAsync(out, h->ll_sum.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "log-likelihood");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_prior_gradient_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev, float* gradient_dev,
                              void* stream) {
  if (!h || !prior || !image_dev || !gradient_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (prior->type == B200RT_PRIOR_NONE || prior->penalisation_factor == 0) {
      ck(cudaMemsetAsync(gradient_dev, 0, sizeof(float) * g.image_size(), st), "memset");
      return B200RT_OK;
    }
    float w[27];
    prior_weights(g, prior->only_2D, w);
    h->partial_max.alloc(update_num_blocks(g.image_size()));
    ck(launch_prior_gradient(image_dev, gradient_dev, prior, w, g.desc().ny, g.desc().nx, g.desc().nz, h->partial_max.p, st),
       "prior gradient");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_log_likelihood_gradient_dev(b200rt_projector* h, const float* image_dev, const float* y_dev,
                                       const float* additive_dev, const float* mult_dev, int subset_num, int num_subsets,
                                       int zero_seg0_end_planes, int back_projection_mode, float* gradient_dev,
                                       void* stream) {
  if (!h || !image_dev || !y_dev || !gradient_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (back_projection_mode != B200RT_BACKPROJECT_ATOMIC && back_projection_mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!h->ratio.p) {
      h->ratio.alloc(g.projdata_size());
      ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * g.projdata_size(), st), "memset");
    }
    h->small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    h->cancelled.alloc(1);
    int nv = 0;
    const int* views = subset_views(*h, subset_num, num_subsets, nv);
    ck(launch_viewgram_small_values(y_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, zero_seg0_end_planes,
                                    g.num_tof(), g.tof_stride(), h->small_value.p, st),
       "viewgram thresholds");
    ck(cudaMemsetAsync(h->cancelled.p, 0, sizeof(unsigned int), st), "memset");
    FwdEpilogue ep{};
    ep.mode = kEpiGradient;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.add = additive_dev;
    ep.mult = mult_dev;
    ep.small_value = h->small_value.p;
    ep.cancelled = h->cancelled.p;
    forward_subset(*h, image_dev, h->ratio.p, subset_num, num_subsets, st, &ep);
    back_project_into(*h, h->ratio.p, gradient_dev, subset_num, num_subsets, back_projection_mode, 0, st);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_attenuation_dev(b200rt_projector* h, const float* mu_dev, float* projdata_dev, int mode, void* stream) {
  if (!h || !mu_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (mode < B200RT_ATTENUATION_FACTORS || mode > B200RT_ATTENUATION_UNDO)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown attenuation mode");
  if (h->geo->num_tof() > 1)
    return fail(h, B200RT_ERR_UNSUPPORTED,
                "BinNormalisationFromAttenuationImage limitation: currently can only handle non_TOF data.");
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Geometry& g = *h->geo;
    if (!h->ratio.p) {
      h->ratio.alloc(g.projdata_size());
      ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * g.projdata_size(), st), "memset");
    }
    forward_subset(*h, mu_dev, h->ratio.p, 0, 1, st);
    ck(launch_attenuation(h->ratio.p, projdata_dev, g.projdata_size(), mode, st), "attenuation");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_normalisation_dev(b200rt_projector* h, const b200rt_norm_term* terms, int num_terms, int mode,
                             float* projdata_dev, void* stream) {
  if (!h || !projdata_dev || (num_terms > 0 && !terms) || num_terms < 0)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (mode < B200RT_NORM_FACTORS || mode > B200RT_NORM_UNDO)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown normalisation mode");
  const Geometry& g = *h->geo;
  for (int t = 0; t < num_terms; ++t) {
    if (!terms[t].data_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null normalisation data");
    if (terms[t].kind == B200RT_NORM_ATTENUATION) {
      if (g.num_tof() > 1)
        return fail(h, B200RT_ERR_UNSUPPORTED,
                    "BinNormalisationFromAttenuationImage limitation: currently can only handle non_TOF data.");
    } else if (terms[t].kind != B200RT_NORM_PROJDATA) {
      return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown normalisation kind");
    }
  }
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = g.projdata_size();
    int step = mode;
    if (mode == B200RT_NORM_FACTORS) {
      ck(launch_fill(projdata_dev, n, 1.f, st), "fill");
      step = B200RT_NORM_UNDO;
    }
    for (int t = 0; t < num_terms; ++t) {
      if (terms[t].kind == B200RT_NORM_PROJDATA) {
        const int64_t fstride = (terms[t].non_tof && g.num_tof() > 1) ? g.tof_stride() : 0;
        ck(launch_norm_projdata(terms[t].data_dev, projdata_dev, n, fstride, step, st), "normalisation");
      } else {
        if (!h->ratio.p) {
          h->ratio.alloc(n);
          ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * n, st), "memset");
        }
        forward_subset(*h, terms[t].data_dev, h->ratio.p, 0, 1, st);
        ck(launch_attenuation(h->ratio.p, projdata_dev, n,
                              step == B200RT_NORM_APPLY ? B200RT_ATTENUATION_APPLY : B200RT_ATTENUATION_UNDO, st),
           "attenuation");
      }
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_ossps_denominator_dev(b200rt_projector* h, const float* y_dev, const float* norm_dev, float* denominator_dev,
                                 int back_projection_mode, void* stream) {
  if (!h || !y_dev || !denominator_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_mode_prior(h, back_projection_mode, nullptr)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!h->ratio.p) {
      h->ratio.alloc(g.projdata_size());
      ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * g.projdata_size(), st), "memset");
    }
    if (!h->ones.p) {
      h->ones.alloc(g.image_size());
      ck(launch_fill(h->ones.p, g.image_size(), 1.F, st), "fill");
    }
    h->small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    forward_subset(*h, h->ones.p, h->ratio.p, 0, 1, st);
    int nv = 0;
    const int* views = subset_views(*h, 0, 1, nv);
    // divide_and_truncate's small value from the forward projection of ones
    ck(launch_viewgram_small_values(h->ratio.p, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, 0, g.num_tof(),
                                    g.tof_stride(), h->small_value.p, st),
       "viewgram thresholds");
    ck(launch_hessian_ratio(h->ratio.p, y_dev, norm_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv,
                            g.num_tof(), g.tof_stride(), h->small_value.p, st),
       "Hessian data term");
    back_project_into(*h, h->ratio.p, denominator_dev, 0, 1, back_projection_mode, 0, st);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_ossps_subiteration_dev(b200rt_projector* h, float* estimate_dev, float* denominator_dev, const float* y_dev,
                                  const float* additive_dev, const float* mult_dev, const float* sens_dev,
                                  int subset_num, int num_subsets, int subiteration_num, int start_subiteration_num,
                                  int zero_seg0_end_planes, const b200rt_prior* prior, float relaxation_parameter,
                                  float relaxation_gamma, float upper_bound, int back_projection_mode, void* stream) {
  if (!h || !estimate_dev || !denominator_dev || !y_dev || !sens_dev)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_mode_prior(h, back_projection_mode, prior)) return st;
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  if (has_prior && prior->type != B200RT_PRIOR_QUADRATIC)
    return fail(h, B200RT_ERR_UNSUPPORTED, "OSSPS needs a prior with a parabolic surrogate (QuadraticPrior)");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t ni = g.image_size();
    h->ossps_g.alloc(ni);
    if (has_prior) h->ossps_pg.alloc(ni);
    h->ossps_partial.alloc(update_num_blocks(ni));
    h->ossps_minpos.alloc(1);
    const bool first = subiteration_num == start_subiteration_num;
    // fill_nonidentifiable_target_parameters at the first sub-iteration (OSSPSReconstruction.cxx:287-291)
    if (first) ck(launch_zero_unidentifiable(estimate_dev, sens_dev, ni, st), "unidentifiable voxels");
    if (int rc = b200rt_log_likelihood_gradient_dev(h, estimate_dev, y_dev, additive_dev, mult_dev, subset_num,
                                                    num_subsets, zero_seg0_end_planes, back_projection_mode,
                                                    h->ossps_g.p, stream))
      return rc;
    // relaxation_parameter / (1 + relaxation_gamma * (subiteration_num / num_subsets)), integer division
    // (OSSPSReconstruction.cxx:370-372)
    const float relax = relaxation_parameter / (1 + relaxation_gamma * (subiteration_num / num_subsets));
    if (has_prior) prior_weights(g, prior->only_2D, h->prior_w);
    ck(launch_ossps_update(estimate_dev, denominator_dev, h->ossps_g.p, has_prior ? h->ossps_pg.p : nullptr, sens_dev,
                           has_prior ? prior : nullptr, h->prior_w, g.desc().ny, g.desc().nx, g.desc().nz, num_subsets,
                           first ? 1 : 0, relax, upper_bound, h->ossps_partial.p, h->ossps_minpos.p, st),
       "OSSPS update");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_prior_hessian_times_input_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev,
                                         const float* input_dev, float* output_dev, void* stream) {
  if (!h || !prior || !image_dev || !input_dev || !output_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_mode_prior(h, B200RT_BACKPROJECT_ATOMIC, prior)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    float w[27];
    prior_weights(g, prior->only_2D, w);
    ck(launch_prior_hessian_times_input(output_dev, image_dev, input_dev, prior, w, g.desc().ny, g.desc().nx,
                                        g.desc().nz, static_cast<cudaStream_t>(stream)),
       "prior Hessian");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_prior_value_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev, double* out,
                           void* stream) {
  if (!h || !prior || !image_dev || !out) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (prior->type == B200RT_PRIOR_NONE || prior->penalisation_factor == 0) {
      *out = 0.0;
      return B200RT_OK;
    }
    float w[27];
    prior_weights(g, prior->only_2D, w);
    const int np = update_num_blocks(g.image_size());
    h->ll_partials.alloc(std::max<size_t>(h->ll_partials.n, static_cast<size_t>(np)));
    h->ll_sum.alloc(1);
    ck(launch_prior_value(image_dev, prior, w, g.desc().ny, g.desc().nx, g.desc().nz, h->ll_partials.p, np, h->ll_sum.p, st),
       "prior value");
    double v = 0.0;
    ck(cudaMemcpyAsync(&v, h->ll_sum.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "prior value");
    *out = v * prior->penalisation_factor;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"

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

// ---- batched OSMAPOSL ---------------------------------------------------------------------------
// Frames of a batch advance together.  Each batched sub-iteration is, on one stream:
//   per frame: viewgram thresholds of its subset, zero the cancelled count and the numerator
//   one persistent forward launch over the (frame, basic bin) items of every frame's subset, writing
//     divide_and_truncate(y, A x + a) into the frame's ratio buffer
//   one persistent back projection of those ratios into the frames' numerators
//   per frame: the update (division by the sensitivity or the MAP-OSL denominator, clamp, x *= u).
// Items are frame-major, so the CTAs share one or two frames' images in L2 at a time.  Everything the
// sequence touches is allocated and uploaded before it runs, so that it can be captured in a CUDA graph.

struct b200rt_batch {
  struct Frame {
    b200rt_projector* h = nullptr;
    int geom = 0;
    float* x = nullptr;
    const float* y = nullptr;
    const float* add = nullptr;
    std::vector<const float*> sens;
    int nsub = 1, start_subset = 0, num_subiters = 0, zero_ends = 0;
    bool has_prior = false;
    b200rt_prior prior{};
    float prior_w[27] = {0};
    float min_rel = 0.f, max_rel = 0.f;
    DevBuf<float> ratio, u, grad, small_value, partial_max, umax;
    DevBuf<unsigned int> cancelled;
  };
  int device = 0;
  std::string err;
  std::vector<std::unique_ptr<Frame>> frames;
  std::vector<b200rt_projector*> geoms;
  DevBuf<b200::ProjParams> d_geoms;
  DevBuf<b200::PathParams> d_pgeoms;
  bool paths = false;  // every frame's projector has path items: the column-staged batched kernels
  bool tof_grouped = false;  // otherwise, TOF frames with the timing bins of a basic bin grouped: TOF kernels
  int num_tof = 1;
  bool packed = false;  // otherwise, every segment of every frame has few axial positions: the packed kernels
  int smem_f = 0, smem_b = 0;
  DevBuf<b200::BatchFrameDev> d_frames;
  DevBuf<unsigned int> counters;  // work-queue heads of the forward and back launches
  bool ready = false;
  int npa = 0;
  size_t smem = 0;
  int num_sms = 0, max_fwd = 0, max_back = 0;
  b200rt_batch_config cfg{0, 0, 0};
  // item lists by (order, subset of each frame or -1)
  std::map<std::vector<int>, std::unique_ptr<DevBuf<b200::BatchItem>>> items;
  std::map<std::vector<int>, int> item_counts;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  // per batched sub-iteration: the update arguments of its frames (device table), their count, the most blocks
  std::map<int, std::unique_ptr<DevBuf<b200::BatchUpdateDev>>> updates;
  std::map<int, std::pair<int, int>> update_counts;
  cudaStream_t capture_stream = nullptr;
};

namespace {


int bfail(b200rt_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

void drop_graphs(b200rt_batch& b) {
  for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
  b.graphs.clear();
}

int frame_subset(const b200rt_batch::Frame& f, int k) { return (f.start_subset + k - 1) % f.nsub; }

// device tables and per-frame scratch; done once after the last add_frame
void batch_finalize(b200rt_batch& b) {
  if (b.ready) return;
  std::vector<b200::ProjParams> gp;
  int npa = -1, max_row = 1;
  for (auto* h : b.geoms) {
    gp.push_back(h->params);
    npa = npa < 0 ? h->params.uniform_npa : (npa == h->params.uniform_npa ? npa : 0);
    max_row = std::max(max_row, h->params.max_row_len);
  }
  b.npa = npa < 0 ? 0 : npa;
  b.smem = b200::proj_smem_bytes(max_row);
  cudaStream_t st = b.capture_stream;
  b.d_geoms.upload(gp, st);
  b.paths = true;
  for (auto* h : b.geoms) b.paths = b.paths && h->use_paths;
  b.tof_grouped = !b.paths;
  b.num_tof = b.geoms.empty() ? 1 : b.geoms[0]->params.num_tof;
  for (auto* h : b.geoms)  // one timing-bin count for the whole batch (the kernels' group size)
    b.tof_grouped = b.tof_grouped && h->params.tof_w != nullptr && h->params.num_tof == b.num_tof;
  b.packed = !b.paths && !b.tof_grouped;
  for (auto* h : b.geoms) b.packed = b.packed && h->params.max_nax <= b200::kPackedMaxNax;
  if (b.paths) {
    std::vector<b200::PathParams> pg;
    b.smem_f = b.smem_b = 0;
    for (auto* h : b.geoms) {
      const b200::PathParams& pp = h->pparams;
      pg.push_back(pp);
      b.smem_f = std::max(b.smem_f, b200::path_smem_fwd(pp.K, h->params.nz, pp.zpad, pp.max_lines, pp.max_acc,
                                                          pp.npa_max).total);
      b.smem_b = std::max(b.smem_b, b200::path_smem_back(h->params.nz, pp.max_lines, pp.max_members, pp.nax_max,
                                                          pp.npa_max).total);
    }
    b.d_pgeoms.upload(pg, st);
  }
  std::vector<BatchFrameDev> fd;
  for (auto& fp : b.frames) {
    auto& f = *fp;
    const b200::Geometry& g = *f.h->geo;
    f.ratio.alloc(g.projdata_size());
    f.u.alloc(g.image_size());
    if (f.has_prior) f.grad.alloc(g.image_size());
    f.small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    f.partial_max.alloc(b200::update_num_blocks(g.image_size()));
    f.umax.alloc(1);
    f.cancelled.alloc(1);
    for (int s = 0; s < f.nsub; ++s) {
      int nv = 0;
      subset_views(*f.h, s, f.nsub, nv);  // cached device view lists, uploaded now
    }
    {
      int nv = 0;
      subset_views(*f.h, 0, 1, nv);  // all views, for the thresholds
    }
    BatchFrameDev d{};
    d.geom = f.geom;
    d.x = f.x;
    d.ratio = f.ratio.p;
    d.u = f.u.p;
    d.ep.mode = b200::kEpiRatio;
    d.ep.zero_ends = f.zero_ends;
    d.ep.y = f.y;
    d.ep.add = f.add;
    d.ep.small_value = f.small_value.p;
    d.ep.cancelled = f.cancelled.p;
    fd.push_back(d);
  }
  b.d_frames.upload(fd, st);
  b.counters.alloc(2);
  ck(cudaDeviceGetAttribute(&b.num_sms, cudaDevAttrMultiProcessorCount, b.device), "device attribute");
  if (b.paths) {
    b.max_fwd = b200::batch_paths_max_ctas_per_sm(b.npa, b.smem_f, true);
    b.max_back = b200::batch_paths_max_ctas_per_sm(b.npa, b.smem_b, false);
  } else if (b.tof_grouped) {
    b.max_fwd = b200::batch_tof_max_ctas_per_sm(b.num_tof, true);
    b.max_back = b200::batch_tof_max_ctas_per_sm(b.num_tof, false);
  } else if (b.packed) {
    b.max_fwd = b200::batch_packed_max_ctas_per_sm(true);
    b.max_back = b200::batch_packed_max_ctas_per_sm(false);
  } else {
    b.max_fwd = b200::batch_max_ctas_per_sm(b.npa, b.smem, true);
    b.max_back = b200::batch_max_ctas_per_sm(b.npa, b.smem, false);
  }
  if (b.max_fwd < 1 || b.max_back < 1) throw std::runtime_error("batched projector does not fit on an SM");
  ck(cudaStreamSynchronize(st), "batch set-up");
  b.ready = true;
}

// the (frame, basic bin) work of batched sub-iteration k, uploaded on first use
const BatchItem* batch_items(b200rt_batch& b, int k, int order, int& count) {
  std::vector<int> key{order};
  for (auto& f : b.frames) key.push_back(k <= f->num_subiters ? frame_subset(*f, k) : -1);
  auto it = b.items.find(key);
  if (it != b.items.end()) {
    count = b.item_counts[key];
    return it->second->p;
  }
  std::vector<BatchItem> list;
  for (size_t fi = 0; fi < b.frames.size(); ++fi) {
    if (key[fi + 1] < 0) continue;
    const auto& f = *b.frames[fi];
    const b200rt_projector& h = *f.h;
    std::vector<int> bins;  // basic bins, or path items with the column-staged kernels
    if (b.paths) {
      for (int i = 0; i < static_cast<int>(h.h_item_view.size()); ++i)
        if (h.h_item_view[i] % f.nsub == key[fi + 1]) bins.push_back(i);
      if (order == 1) {
        std::stable_sort(bins.begin(), bins.end(), [&](int a, int c) {
          const auto& pa = h.h_path_items[a];
          const auto& pc = h.h_path_items[c];
          return static_cast<int64_t>(pa.ncols) * pa.num_lines > static_cast<int64_t>(pc.ncols) * pc.num_lines;
        });
      }
    } else if (b.tof_grouped) {
      for (int bin = 0; bin < static_cast<int>(h.h_tof_basic_view.size()); ++bin)
        if (h.h_tof_basic_view[bin] % f.nsub == key[fi + 1]) bins.push_back(bin);
    } else {
      for (int bin = 0; bin < static_cast<int>(h.h_bins.size()); ++bin)
        if (h.h_bin_view[bin] % f.nsub == key[fi + 1]) bins.push_back(bin);
      if (order == 1) {
        std::stable_sort(bins.begin(), bins.end(), [&](int a, int c) {
          const auto& pa = h.h_bins[a];
          const auto& pc = h.h_bins[c];
          return static_cast<int64_t>(pa.row_len) * pa.num_lines > static_cast<int64_t>(pc.row_len) * pc.num_lines;
        });
      }
    }
    for (int bin : bins) list.push_back(BatchItem{static_cast<int>(fi), bin});
  }
  auto buf = std::make_unique<DevBuf<BatchItem>>();
  buf->upload(list, b.capture_stream);
  ck(cudaStreamSynchronize(b.capture_stream), "batch items");
  count = static_cast<int>(list.size());
  b.item_counts[key] = count;
  const BatchItem* p = buf->p;
  b.items[key] = std::move(buf);
  return p;
}

int grid_of(const b200rt_batch& b, int per_sm, int max_per_sm) {
  const int c = per_sm > 0 ? std::min(per_sm, max_per_sm) : max_per_sm;
  return c * b.num_sms;
}

// divide_and_truncate's threshold of every viewgram of every frame taking part in sub-iterations first.. (it
// depends on the data only, so once per run covers all the run's subsets)
void batch_thresholds(b200rt_batch& b, int first, cudaStream_t st) {
  for (auto& fp : b.frames) {
    auto& f = *fp;
    if (first > f.num_subiters) continue;
    const b200::Geometry& g = *f.h->geo;
    int nv = 0;
    const int* views = subset_views(*f.h, 0, 1, nv);
    ck(launch_viewgram_small_values(f.y, f.h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, f.zero_ends,
                                    g.num_tof(), g.tof_stride(), f.small_value.p, st),
       "viewgram thresholds");
  }
}

// zero the numerators and cancelled counts of the frames taking part in sub-iteration k
void batch_zero(b200rt_batch& b, int k, cudaStream_t st) {
  for (auto& fp : b.frames) {
    auto& f = *fp;
    if (k > f.num_subiters) continue;
    ck(cudaMemsetAsync(f.cancelled.p, 0, sizeof(unsigned int), st), "memset");
    ck(cudaMemsetAsync(f.u.p, 0, sizeof(float) * f.h->geo->image_size(), st), "memset");
  }
}

// one batched launch of one direction (0 forward with the ratio epilogue, 1 back projection of the ratios)
cudaError_t batch_launch(b200rt_batch& b, int dir, const BatchItem* items, int n, int grid, cudaStream_t st) {
  if (b.paths)
    return dir == 0 ? b200::launch_forward_batch_paths(b.d_geoms.p, b.d_pgeoms.p, b.npa, b.smem_f, b.d_frames.p, items,
                                                       n, b.counters.p, grid, st)
                    : b200::launch_back_batch_paths(b.d_geoms.p, b.d_pgeoms.p, b.smem_b, b.d_frames.p, items, n,
                                                    b.counters.p + 1, grid, st);
  if (b.tof_grouped)
    return dir == 0 ? b200::launch_forward_batch_tof(b.d_geoms.p, b.num_tof, b.d_frames.p, items, n, b.counters.p, grid,
                                                     st)
                    : b200::launch_back_batch_tof(b.d_geoms.p, b.num_tof, b.d_frames.p, items, n, b.counters.p + 1,
                                                  grid, st);
  if (b.packed)
    return dir == 0 ? b200::launch_forward_batch_packed(b.d_geoms.p, b.d_frames.p, items, n, b.counters.p, grid, st)
                    : b200::launch_back_batch_packed(b.d_geoms.p, b.d_frames.p, items, n, b.counters.p + 1, grid, st);
  return dir == 0 ? b200::launch_forward_batch(b.d_geoms.p, b.npa, b.smem, b.d_frames.p, items, n, b.counters.p, grid, st)
                  : b200::launch_back_batch(b.d_geoms.p, b.npa, b.smem, b.d_frames.p, items, n, b.counters.p + 1, grid,
                                            st);
}

void batch_projections(b200rt_batch& b, int k, cudaStream_t st) {
  int n = 0;
  const BatchItem* items = batch_items(b, k, b.cfg.order, n);
  ck(cudaMemsetAsync(b.counters.p, 0, 2 * sizeof(unsigned int), st), "memset");
  ck(batch_launch(b, 0, items, n, grid_of(b, b.cfg.ctas_per_sm_forward, b.max_fwd), st), "batched forward projection");
  ck(batch_launch(b, 1, items, n, grid_of(b, b.cfg.ctas_per_sm_back, b.max_back), st), "batched back projection");
}

// the update arguments of the frames taking part in sub-iteration k, uploaded on first use
const b200::BatchUpdateDev* batch_updates(b200rt_batch& b, int k, int& count, int& max_blocks) {
  auto it = b.updates.find(k);
  if (it != b.updates.end()) {
    count = b.update_counts[k].first;
    max_blocks = b.update_counts[k].second;
    return it->second->p;
  }
  std::vector<b200::BatchUpdateDev> v;
  max_blocks = 1;
  for (auto& fp : b.frames) {
    auto& f = *fp;
    if (k > f.num_subiters) continue;
    const b200::Geometry& g = *f.h->geo;
    b200::BatchUpdateDev d;
    b200::fill_batch_update(d, f.u.p, f.x, f.sens[frame_subset(f, k)], f.has_prior ? f.grad.p : nullptr,
                            f.has_prior ? &f.prior : nullptr, f.prior_w, f.nsub, k, f.min_rel, f.max_rel, g.desc().ny,
                            g.desc().nx, g.desc().nz, f.partial_max.p, f.umax.p);
    max_blocks = std::max(max_blocks, d.nblocks);
    v.push_back(d);
  }
  auto buf = std::make_unique<DevBuf<b200::BatchUpdateDev>>();
  buf->upload(v, b.capture_stream);
  ck(cudaStreamSynchronize(b.capture_stream), "batch updates");
  count = static_cast<int>(v.size());
  b.update_counts[k] = {count, max_blocks};
  const b200::BatchUpdateDev* p = buf->p;
  b.updates[k] = std::move(buf);
  return p;
}

void batch_subiteration(b200rt_batch& b, int k, cudaStream_t st) {
  batch_zero(b, k, st);
  batch_projections(b, k, st);
  // every frame's update (OSMAPOSLReconstruction.cxx:394-510) in three launches
  int n = 0, max_blocks = 1;
  const b200::BatchUpdateDev* upd = batch_updates(b, k, n, max_blocks);
  ck(b200::launch_batch_update(upd, n, max_blocks, st), "update");
}

}  // namespace

extern "C" {

int b200rt_batch_create(int device, b200rt_batch** out) {
  if (!out) return B200RT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return B200RT_ERR_INVALID_ARGUMENT;
  auto b = std::make_unique<b200rt_batch>();
  b->device = device;
  try {
    DeviceGuard dg(device);
    ck(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  } catch (const std::exception&) {
    return B200RT_ERR_CUDA;
  }
  *out = b.release();
  return B200RT_OK;
}

void b200rt_batch_destroy(b200rt_batch* b) {
  if (!b) return;
  {
    DeviceGuard dg(b->device);
    if (b->capture_stream) cudaStreamSynchronize(b->capture_stream);
    cudaDeviceSynchronize();  // graphs may still run on a caller's stream
    drop_graphs(*b);
    b->items.clear();
    b->updates.clear();
    b->update_counts.clear();
    b->frames.clear();
    b->d_geoms.release();
    b->d_pgeoms.release();
    b->d_frames.release();
    b->counters.release();
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  }
  delete b;
}

const char* b200rt_batch_last_error(const b200rt_batch* b) { return b ? b->err.c_str() : "null batch"; }

int b200rt_batch_num_frames(const b200rt_batch* b) { return b ? static_cast<int>(b->frames.size()) : 0; }

int b200rt_batch_add_frame(b200rt_batch* b, b200rt_projector* h, float* estimate_dev, const float* y_dev,
                           const float* additive_dev, const float* const* sensitivity_devs, int num_subsets,
                           int start_subset, int num_subiterations, int zero_seg0_end_planes, const b200rt_prior* prior,
                           float min_relative_change, float max_relative_change, int* frame) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (!h || !estimate_dev || !y_dev || !sensitivity_devs) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (h->device != b->device) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "projector is on another device");
  if (num_subsets < 1 || start_subset < 0 || start_subset >= num_subsets)
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid subset number");
  if (num_subiterations < 1) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid number of sub-iterations");
  for (int s = 0; s < num_subsets; ++s)
    if (!sensitivity_devs[s]) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "null sensitivity");
  if (prior && (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE))
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  try {
    DeviceGuard dg(b->device);
    auto f = std::make_unique<b200rt_batch::Frame>();
    f->h = h;
    auto git = std::find(b->geoms.begin(), b->geoms.end(), h);
    f->geom = static_cast<int>(git - b->geoms.begin());
    if (git == b->geoms.end()) b->geoms.push_back(h);
    f->x = estimate_dev;
    f->y = y_dev;
    f->add = additive_dev;
    f->sens.assign(sensitivity_devs, sensitivity_devs + num_subsets);
    f->nsub = num_subsets;
    f->start_subset = start_subset;
    f->num_subiters = num_subiterations;
    f->zero_ends = zero_seg0_end_planes;
    f->has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
    if (f->has_prior) {
      f->prior = *prior;
      prior_weights(*h->geo, prior->only_2D, f->prior_w);
    }
    f->min_rel = min_relative_change;
    f->max_rel = max_relative_change;
    drop_graphs(*b);
    b->items.clear();
    b->updates.clear();
    b->update_counts.clear();
    b->item_counts.clear();
    b->ready = false;
    b->frames.push_back(std::move(f));
    if (frame) *frame = static_cast<int>(b->frames.size()) - 1;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return bfail(b, status_of(e), e.what());
  }
}

int b200rt_batch_run(b200rt_batch* b, int first_subiteration, int count, int use_graph, void* stream) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (first_subiteration < 1 || count < 0) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid sub-iteration range");
  if (b->frames.empty() || count == 0) return B200RT_OK;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    DeviceGuard dg(b->device);
    batch_finalize(*b);
    for (int k = first_subiteration; k < first_subiteration + count; ++k) {
      int n = 0;
      batch_items(*b, k, b->cfg.order, n);  // uploads happen here, never inside a capture
      int nu = 0, mb = 0;
      batch_updates(*b, k, nu, mb);
    }
    if (!use_graph) {
      batch_thresholds(*b, first_subiteration, st);
      for (int k = first_subiteration; k < first_subiteration + count; ++k) batch_subiteration(*b, k, st);
      return B200RT_OK;
    }
    const auto key = std::make_pair(first_subiteration, count);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaStream_t cs = b->capture_stream;
      ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
      try {
        batch_thresholds(*b, first_subiteration, cs);
        for (int k = first_subiteration; k < first_subiteration + count; ++k) batch_subiteration(*b, k, cs);
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      cudaGraph_t graph = nullptr;
      ck(cudaStreamEndCapture(cs, &graph), "cudaStreamEndCapture");
      cudaGraphExec_t exec = nullptr;
      const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      ck(e, "cudaGraphInstantiate");
      it = b->graphs.emplace(key, exec).first;
    }
    ck(cudaGraphLaunch(it->second, st), "cudaGraphLaunch");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return bfail(b, status_of(e), e.what());
  }
}

int b200rt_batch_autotune(b200rt_batch* b, int subiteration, b200rt_batch_config* out) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (subiteration < 1) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid sub-iteration");
  if (b->frames.empty()) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "empty batch");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  try {
    DeviceGuard dg(b->device);
    batch_finalize(*b);
    const cudaStream_t st = b->capture_stream;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    batch_thresholds(*b, subiteration, st);  // the forward epilogue reads them
    batch_zero(*b, subiteration, st);        // numerators are scratch
    // time one launch of one direction: the best of two after a warm-up
    auto time_launch = [&](int dir, const BatchItem* items, int n, int grid) {
      float t = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        ck(cudaMemsetAsync(b->counters.p, 0, 2 * sizeof(unsigned int), st), "memset");
        ck(cudaEventRecord(e0, st), "cudaEventRecord");
        ck(batch_launch(*b, dir, items, n, grid, st), dir == 0 ? "batched forward projection" : "batched back projection");
        ck(cudaEventRecord(e1, st), "cudaEventRecord");
        ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        if (rep > 0) t = std::min(t, ms);
      }
      return t;
    };
    float best_total = 1e30f;
    b200rt_batch_config best = b->cfg;
    for (int order = 0; order <= 1; ++order) {
      int n = 0;
      const BatchItem* items = batch_items(*b, subiteration, order, n);
      float tdir[2] = {1e30f, 1e30f};
      int cdir[2] = {1, 1};
      for (int dir = 0; dir < 2; ++dir)
        for (int c = 1; c <= (dir == 0 ? b->max_fwd : b->max_back); ++c) {
          const float t = time_launch(dir, items, n, c * b->num_sms);
          if (t < tdir[dir]) {
            tdir[dir] = t;
            cdir[dir] = c;
          }
        }
      if (tdir[0] + tdir[1] < best_total) {
        best_total = tdir[0] + tdir[1];
        best = b200rt_batch_config{cdir[0], cdir[1], order};
      }
    }
    b->cfg = best;
    if (out) *out = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs(*b);
    return B200RT_OK;
  } catch (const std::exception& e) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return bfail(b, status_of(e), e.what());
  }
}

int b200rt_batch_set_config(b200rt_batch* b, const b200rt_batch_config* config) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (!config || config->ctas_per_sm_forward < 0 || config->ctas_per_sm_back < 0 || config->order < 0 ||
      config->order > 1)
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid batch configuration");
  b->cfg = *config;
  drop_graphs(*b);
  return B200RT_OK;
}

int b200rt_batch_get_config(const b200rt_batch* b, b200rt_batch_config* out) {
  if (!b || !out) return B200RT_ERR_INVALID_ARGUMENT;
  *out = b->cfg;
  return B200RT_OK;
}

int b200rt_batch_get_num_cancelled(b200rt_batch* b, int frame, int64_t* out) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (!out || frame < 0 || frame >= static_cast<int>(b->frames.size()))
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid frame");
  *out = 0;
  auto& f = *b->frames[frame];
  if (!f.cancelled.p) return B200RT_OK;
  try {
    DeviceGuard dg(b->device);
    unsigned int c = 0;
    ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    ck(cudaMemcpy(&c, f.cancelled.p, sizeof(c), cudaMemcpyDeviceToHost), "D2H");
    *out = c;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return bfail(b, status_of(e), e.what());
  }
}

}  // extern "C"

/* ---- list mode ---------------------------------------------------------- */
namespace {

void ensure_lm_table(b200rt_projector& h) {
  if (h.lm_table.p) return;
  const Geometry& g = *h.geo;
  const int nseg = 2 * g.S() + 1, nv = g.num_views(), nt = g.num_tang(), ntof = g.num_tof();
  std::vector<int4> table(static_cast<size_t>(ntof) * nseg * nv * nt, make_int4(-1, -1, -1, 0));
  for (int b = 0; b < static_cast<int>(h.h_bins.size()); ++b) {
    const ProjBinDev& pb = h.h_bins[b];
    for (int l = 0; l < pb.num_lines; ++l) {
      const LineDev& L = h.h_lines[pb.first_line + l];
      const int tang = L.tang_sign * pb.tang;
      if (tang < g.min_tang() || tang > g.max_tang()) continue;
      const size_t k = ((static_cast<size_t>(pb.tof - g.min_tof()) * nseg + (L.seg + g.S())) * nv + L.view) * nt +
                       (tang - g.min_tang());
      table[k] = make_int4(b, l, h.h_bin_view[b], 0);
    }
  }
  h.lm_table.upload(table, h.stream);
  h.lm_invalid.alloc(1);
  ck(cudaMemsetAsync(h.lm_invalid.p, 0, sizeof(unsigned), h.stream), "memset");
  ck(cudaStreamSynchronize(h.stream), "list-mode table");
}

int lm_check(b200rt_projector* h, const b200rt_lm_event* ev, int64_t n, const float* x, int subset, int nsub) {
  if (!h || (!ev && n > 0) || !x || n < 0) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  return check_subset(h, subset, nsub);
}

// binned (projection kernels over the subset) or per event (one row walk per event): automatically binned once
// the events number at least 1/16 of the bins, where two whole-subset projections cost less than the events'
// rows (on the clinical geometry a forward plus a back projection take ~0.4 ns per bin, a row walk ~5 ns per
// event)
bool lm_binned(const b200rt_projector& h, int64_t n) {
  if (h.lm_method == B200RT_LISTMODE_PER_EVENT) return false;
  if (h.lm_method == B200RT_LISTMODE_BINNED) return n > 0;
  return n > 0 && n * 16 >= h.geo->projdata_size();
}

// A x of the subset into buf (device layout).  The buffer is zeroed when allocated: a bin no line reaches is
// never written and reads as 0, as its empty row would give.
const float* lm_forward(b200rt_projector& h, DevBuf<float>& buf, const float* x, int subset, int nsub,
                        cudaStream_t st) {
  const size_t np = static_cast<size_t>(h.geo->projdata_size());
  if (buf.n != np) {
    buf.alloc(np);
    ck(cudaMemsetAsync(buf.p, 0, sizeof(float) * np, st), "memset");
  }
  forward_subset(h, x, buf.p, subset, nsub, st);
  return buf.p;
}

float* lm_zeroed_hist(b200rt_projector& h, cudaStream_t st) {
  const size_t np = static_cast<size_t>(h.geo->projdata_size());
  h.lm_hist.alloc(np);
  ck(cudaMemsetAsync(h.lm_hist.p, 0, sizeof(float) * np, st), "memset");
  return h.lm_hist.p;
}

// out = A^T hist over the subset, or out += it
void lm_back(b200rt_projector& h, int subset, int nsub, int accumulate, float* out, cudaStream_t st) {
  if (!accumulate) {
    back_project_into(h, h.lm_hist.p, out, subset, nsub, B200RT_BACKPROJECT_ATOMIC, 0, st);
    return;
  }
  const int64_t ni = h.geo->image_size();
  h.lm_img.alloc(ni);
  back_project_into(h, h.lm_hist.p, h.lm_img.p, subset, nsub, B200RT_BACKPROJECT_ATOMIC, 0, st);
  ck(launch_add(out, h.lm_img.p, ni, st), "add");
}

}  // namespace

static_assert(sizeof(b200rt_lm_event) == sizeof(LmEventDev), "list-mode event layouts agree");

extern "C" {

int b200rt_listmode_gradient_dev(b200rt_projector* h, const b200rt_lm_event* events_dev, int64_t num_events,
                                 const float* image_dev, int subset_num, int num_subsets, int has_add,
                                 const float* subset_sensitivity_dev, int accumulate, float* gradient_dev,
                                 void* stream) {
  if (int st = lm_check(h, events_dev, num_events, image_dev, subset_num, num_subsets)) return st;
  if (!gradient_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t ni = h->geo->image_size();
    const auto* ev = reinterpret_cast<const LmEventDev*>(events_dev);
    if (lm_binned(*h, num_events)) {
      const float* fwd = lm_forward(*h, h->lm_fwd, image_dev, subset_num, num_subsets, st);
      ck(launch_listmode_binned(h->params, h->lm_table.p, ev, num_events, 0, fwd, nullptr, subset_num, num_subsets,
                                has_add, lm_zeroed_hist(*h, st), nullptr, h->lm_invalid.p, st),
         "list-mode gradient");
      lm_back(*h, subset_num, num_subsets, accumulate, gradient_dev, st);
    } else {
      if (!accumulate) ck(cudaMemsetAsync(gradient_dev, 0, sizeof(float) * ni, st), "memset");
      if (num_events > 0)
        ck(launch_listmode(h->params, h->lm_table.p, ev, num_events, 0, image_dev, nullptr, subset_num, num_subsets,
                           has_add, gradient_dev, nullptr, h->lm_invalid.p, st),
           "list-mode gradient");
    }
    if (subset_sensitivity_dev) ck(launch_subtract(gradient_dev, subset_sensitivity_dev, ni, st), "subtract");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_listmode_value_dev(b200rt_projector* h, const b200rt_lm_event* events_dev, int64_t num_events,
                              const float* image_dev, int subset_num, int num_subsets, int has_add, double* value,
                              void* stream) {
  if (int st = lm_check(h, events_dev, num_events, image_dev, subset_num, num_subsets)) return st;
  if (!value) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const auto* ev = reinterpret_cast<const LmEventDev*>(events_dev);
    const bool binned = lm_binned(*h, num_events);
    const int nb = binned ? listmode_binned_num_blocks(num_events) : listmode_num_blocks(num_events);
    h->lm_partial.alloc(std::max<size_t>(h->lm_partial.n, static_cast<size_t>(nb)));
    h->lm_sum.alloc(1);
    if (binned) {
      const float* fwd = lm_forward(*h, h->lm_fwd, image_dev, subset_num, num_subsets, st);
      ck(launch_listmode_binned(h->params, h->lm_table.p, ev, num_events, 1, fwd, nullptr, subset_num, num_subsets,
                                has_add, nullptr, h->lm_partial.p, h->lm_invalid.p, st),
         "list-mode value");
    } else {
      ck(launch_listmode(h->params, h->lm_table.p, ev, num_events, 1, image_dev, nullptr, subset_num, num_subsets,
                         has_add, nullptr, h->lm_partial.p, h->lm_invalid.p, st),
         "list-mode value");
    }
    ck(launch_reduce_sum(h->lm_partial.p, nb, h->lm_sum.p, st), "list-mode value");
    ck(cudaMemcpyAsync(value, h->lm_sum.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "list-mode value");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_listmode_hessian_times_input_dev(b200rt_projector* h, const b200rt_lm_event* events_dev,
                                            int64_t num_events, const float* image_dev, const float* rhs_dev,
                                            int subset_num, int num_subsets, int has_add, float* output_dev,
                                            void* stream) {
  if (int st = lm_check(h, events_dev, num_events, image_dev, subset_num, num_subsets)) return st;
  if (!rhs_dev || !output_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const auto* ev = reinterpret_cast<const LmEventDev*>(events_dev);
    if (lm_binned(*h, num_events)) {
      const float* fwd = lm_forward(*h, h->lm_fwd, image_dev, subset_num, num_subsets, st);
      const float* fwd_rhs = lm_forward(*h, h->lm_fwd_rhs, rhs_dev, subset_num, num_subsets, st);
      ck(launch_listmode_binned(h->params, h->lm_table.p, ev, num_events, 2, fwd, fwd_rhs, subset_num, num_subsets,
                                has_add, lm_zeroed_hist(*h, st), nullptr, h->lm_invalid.p, st),
         "list-mode Hessian");
      lm_back(*h, subset_num, num_subsets, 1, output_dev, st);
    } else if (num_events > 0) {
      ck(launch_listmode(h->params, h->lm_table.p, ev, num_events, 2, image_dev, rhs_dev, subset_num, num_subsets,
                         has_add, output_dev, nullptr, h->lm_invalid.p, st),
         "list-mode Hessian");
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_listmode_set_method(b200rt_projector* h, int method) {
  if (!h) return B200RT_ERR_INVALID_ARGUMENT;
  if (method != B200RT_LISTMODE_AUTO && method != B200RT_LISTMODE_PER_EVENT && method != B200RT_LISTMODE_BINNED)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown list-mode method");
  h->lm_method = method;
  return B200RT_OK;
}

int b200rt_listmode_num_invalid(b200rt_projector* h, int64_t* count) {
  if (!h || !count) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    unsigned v = 0;
    ck(cudaMemcpy(&v, h->lm_invalid.p, sizeof(unsigned), cudaMemcpyDeviceToHost), "D2H");
    ck(cudaMemset(h->lm_invalid.p, 0, sizeof(unsigned)), "memset");
    *count = v;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"

/* ---- projection data streams ------------------------------------------- */
namespace {

// the stream's segment groups for the projector's segments and timing positions; throws on a mismatch
std::vector<StreamSegment> stream_plan(const Geometry& g, const b200rt_stream_format& f, int64_t& total_elems) {
  if (f.storage_order != B200RT_STORAGE_SEGMENT_VIEW_AXIAL_TANG && f.storage_order != B200RT_STORAGE_SEGMENT_AXIAL_VIEW_TANG)
    throw std::invalid_argument("unsupported storage order");
  if (numeric_type_size(f.number_type) == 0) throw std::invalid_argument("unknown number type");
  if (f.num_segments < 1 || !f.segment_sequence || !f.num_axial_poss)
    throw std::invalid_argument("the stream needs its segment sequence and axial sizes");
  if (f.num_timing_poss != g.num_tof())
    throw std::invalid_argument("the stream's number of timing positions differs from the projector's");
  const int64_t nvt = static_cast<int64_t>(g.num_views()) * g.num_tang();
  int64_t size3d = 0;
  for (int i = 0; i < f.num_segments; ++i) {
    if (f.num_axial_poss[i] < 0) throw std::invalid_argument("negative axial size");
    size3d += f.num_axial_poss[i] * nvt;
  }
  total_elems = size3d * f.num_timing_poss;
  std::vector<StreamSegment> plan;
  for (int k = 0; k < g.num_tof(); ++k) {
    int ti = k;  // the stream's index of timing position min_tof + k
    if (f.timing_poss_sequence) {
      ti = -1;
      for (int i = 0; i < f.num_timing_poss; ++i)
        if (f.timing_poss_sequence[i] == g.min_tof() + k) ti = i;
      if (ti < 0) throw std::invalid_argument("a timing position of the projector is missing from the stream");
    }
    for (int s = -g.S(); s <= g.S(); ++s) {
      int64_t off = 0;
      int idx = -1;
      for (int i = 0; i < f.num_segments && idx < 0; ++i) {
        if (f.segment_sequence[i] == s)
          idx = i;
        else
          off += f.num_axial_poss[i] * nvt;
      }
      if (idx < 0) throw std::invalid_argument("segment " + std::to_string(s) + " is missing from the stream");
      if (f.num_axial_poss[idx] != g.nax(s))
        throw std::invalid_argument("segment " + std::to_string(s) + " has another number of axial positions");
      StreamSegment ss{};
      ss.order = f.storage_order == B200RT_STORAGE_SEGMENT_AXIAL_VIEW_TANG ? kStorageSegmentAxialViewTang
                                                                           : kStorageSegmentViewAxialTang;
      ss.type = f.number_type;
      ss.swap = f.swap_bytes ? 1 : 0;
      ss.scale = f.scale_factor;
      ss.nax = g.nax(s);
      ss.nv = g.num_views();
      ss.nt = g.num_tang();
      ss.stream_elem = ti * size3d + off;
      ss.dev_off = k * g.tof_stride() + g.dev_segment_offset(s);
      plan.push_back(ss);
    }
  }
  return plan;
}

}  // namespace

extern "C" {

int b200rt_stream_bytes(b200rt_projector* h, const b200rt_stream_format* fmt, int64_t* bytes) {
  if (!h || !fmt || !bytes) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    int64_t n = 0;
    stream_plan(*h->geo, *fmt, n);
    *bytes = n * numeric_type_size(fmt->number_type);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_projdata_from_stream_dev(b200rt_projector* h, const void* stream_dev, int64_t stream_bytes,
                                    const b200rt_stream_format* fmt, float* projdata_dev, void* stream) {
  if (!h || !stream_dev || !fmt || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    int64_t n = 0;
    const std::vector<StreamSegment> plan = stream_plan(*h->geo, *fmt, n);
    if (stream_bytes < n * numeric_type_size(fmt->number_type))
      return fail(h, B200RT_ERR_INVALID_ARGUMENT, "the stream is shorter than its format says");
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (const StreamSegment& ss : plan) ck(launch_stream_segment(ss, true, stream_dev, projdata_dev, st), "stream read");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_projdata_to_stream_dev(b200rt_projector* h, const float* projdata_dev, const b200rt_stream_format* fmt,
                                  void* stream_dev, int64_t stream_bytes, void* stream) {
  if (!h || !stream_dev || !fmt || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (fmt->number_type != B200RT_NUMBER_FLOAT && fmt->number_type != B200RT_NUMBER_DOUBLE)
    return fail(h, B200RT_ERR_UNSUPPORTED, "streams are written as float or double");
  if (fmt->scale_factor != 1.f) return fail(h, B200RT_ERR_UNSUPPORTED, "streams are written with scale factor 1");
  try {
    int64_t n = 0;
    const std::vector<StreamSegment> plan = stream_plan(*h->geo, *fmt, n);
    if (stream_bytes < n * numeric_type_size(fmt->number_type))
      return fail(h, B200RT_ERR_INVALID_ARGUMENT, "the stream is shorter than its format says");
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (const StreamSegment& ss : plan) ck(launch_stream_segment(ss, false, projdata_dev, stream_dev, st), "stream write");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"

/* ---- Gibbs penalties ---------------------------------------------------- */
struct b200rt_gibbs {
  int device = 0;
  GibbsDev d{};
  std::vector<float> host_w;
  DevBuf<double> partial, result;
  std::string err;
};

namespace {

int gfail(b200rt_gibbs* g, int code, const std::string& msg) {
  if (g) g->err = msg;
  return code;
}

int create_fail(int code, const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_create_error = msg;
  return code;
}

// one penalty operation: validates the pointers, runs on `stream`; scalar results are copied to *value
int gibbs_op(b200rt_gibbs* g, int op, const float* x, const float* in, float* out, double* value, void* stream) {
  if (!g || !x) return gfail(g, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if ((op == 0 || op == 2) && !value) return gfail(g, B200RT_ERR_INVALID_ARGUMENT, "null value pointer");
  if ((op == 1 || op == 3 || op == 4) && !out) return gfail(g, B200RT_ERR_INVALID_ARGUMENT, "null output");
  if ((op == 2 || op == 4) && !in) return gfail(g, B200RT_ERR_INVALID_ARGUMENT, "null input image");
  try {
    DeviceGuard dg(g->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = static_cast<int64_t>(g->d.nz) * g->d.ny * g->d.nx;
    if (g->d.beta == 0) {  // GibbsPenalty.inl: a zero penalisation factor gives 0, a zero gradient / diagonal
      if (op == 1 || op == 3) ck(cudaMemsetAsync(out, 0, sizeof(float) * n, st), "memset");
      if (value) *value = 0.0;
      return B200RT_OK;
    }
    if (op == 0 || op == 2) {
      g->partial.alloc(static_cast<size_t>(gibbs_num_partials(g->d)));
      g->result.alloc(1);
    }
    ck(launch_gibbs(g->d, op, x, in, out, g->partial.p, g->result.p, st), "Gibbs penalty");
    if (op == 0 || op == 2) {
      ck(cudaMemcpyAsync(value, g->result.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
      ck(cudaStreamSynchronize(st), "Gibbs penalty");
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return gfail(g, status_of(e), e.what());
  }
}

}  // namespace

extern "C" {

int b200rt_gibbs_create(const b200rt_gibbs_params* p, int device, b200rt_gibbs** out) {
  if (!out) return B200RT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!p) return create_fail(B200RT_ERR_INVALID_ARGUMENT, "null parameters");
  if (p->potential != B200RT_GIBBS_QUADRATIC && p->potential != B200RT_GIBBS_RELATIVE_DIFFERENCE)
    return create_fail(B200RT_ERR_INVALID_ARGUMENT, "unknown Gibbs potential");
  if (p->nz < 1 || p->ny < 1 || p->nx < 1) return create_fail(B200RT_ERR_INVALID_ARGUMENT, "empty image");
  if (static_cast<int64_t>(p->nz) * p->ny * p->nx >= (int64_t(1) << 31))
    return create_fail(B200RT_ERR_TOO_LARGE, "image of 2^31 voxels or more");
  if (p->layout != B200RT_LAYOUT_DEVICE && p->layout != B200RT_LAYOUT_STIR)
    return create_fail(B200RT_ERR_INVALID_ARGUMENT, "unknown image layout");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return create_fail(B200RT_ERR_INVALID_ARGUMENT, "invalid CUDA device");
  auto g = std::make_unique<b200rt_gibbs>();
  g->device = device;
  GibbsDev& d = g->d;
  d.potential = p->potential;
  d.beta = p->penalisation_factor;
  d.gamma = p->gamma;
  d.epsilon = p->epsilon;
  d.nz = p->nz;
  d.ny = p->ny;
  d.nx = p->nx;
  d.layout = p->layout;
  if (p->layout == B200RT_LAYOUT_DEVICE) {
    d.sz = 1;
    d.sx = p->nz;
    d.sy = static_cast<int64_t>(p->nz) * p->nx;
  } else {
    d.sx = 1;
    d.sy = p->nx;
    d.sz = static_cast<int64_t>(p->nx) * p->ny;
  }
  d.kappa = p->kappa_dev;
  if (p->weights) {
    const int wz = p->weights_z, wy = p->weights_y, wx = p->weights_x;
    if (wz < 1 || wy < 1 || wx < 1 || wz > 7 || wy > 7 || wx > 7)
      return create_fail(B200RT_ERR_INVALID_ARGUMENT, "weights sizes must be 1..7");
    d.wz = wz;
    d.wy = wy;
    d.wx = wx;
    g->host_w.assign(p->weights, p->weights + wz * wy * wx);
  } else {
    // compute_default_weights (GibbsPenalty.inl): x voxel size / Euclidean distance, centre 0
    if (!(p->voxel_size_x > 0 && p->voxel_size_y > 0 && p->voxel_size_z > 0))
      return create_fail(B200RT_ERR_INVALID_ARGUMENT, "default weights need positive voxel sizes");
    d.wz = p->only_2D ? 1 : 3;
    d.wy = d.wx = 3;
    const float vz = p->voxel_size_z, vy = p->voxel_size_y, vx = p->voxel_size_x;
    for (int z = -(d.wz / 2); z <= d.wz / 2; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x) {
          float v = 0.f;
          if (!(z == 0 && y == 0 && x == 0)) {
            const float a = static_cast<float>(x) * vx, b = static_cast<float>(y) * vy, c = static_cast<float>(z) * vz;
            v = vx / std::sqrt(a * a + b * b + c * c);
          }
          g->host_w.push_back(v);
        }
  }
  std::copy(g->host_w.begin(), g->host_w.end(), d.w);
  for (size_t i = 0; i < 27 && i < g->host_w.size(); ++i) d.wd[i] = static_cast<double>(g->host_w[i]);
  *out = g.release();
  return B200RT_OK;
}

void b200rt_gibbs_destroy(b200rt_gibbs* g) {
  if (!g) return;
  {
    DeviceGuard dg(g->device);
    g->partial.release();
    g->result.release();
  }
  delete g;
}

const char* b200rt_gibbs_last_error(const b200rt_gibbs* g) { return g ? g->err.c_str() : "null penalty"; }

int b200rt_gibbs_get_weights(const b200rt_gibbs* g, float* w, int32_t sizes[3]) {
  if (!g || !sizes) return B200RT_ERR_INVALID_ARGUMENT;
  sizes[0] = g->d.wz;
  sizes[1] = g->d.wy;
  sizes[2] = g->d.wx;
  if (w) std::copy(g->host_w.begin(), g->host_w.end(), w);
  return B200RT_OK;
}

int b200rt_gibbs_set_kappa(b200rt_gibbs* g, const float* kappa_dev) {
  if (!g) return B200RT_ERR_INVALID_ARGUMENT;
  g->d.kappa = kappa_dev;
  return B200RT_OK;
}

int b200rt_gibbs_value_dev(b200rt_gibbs* g, const float* image_dev, double* value, void* stream) {
  return gibbs_op(g, 0, image_dev, nullptr, nullptr, value, stream);
}

int b200rt_gibbs_gradient_dev(b200rt_gibbs* g, const float* image_dev, float* gradient_dev, void* stream) {
  return gibbs_op(g, 1, image_dev, nullptr, gradient_dev, nullptr, stream);
}

int b200rt_gibbs_gradient_times_input_dev(b200rt_gibbs* g, const float* input_dev, const float* image_dev,
                                          double* value, void* stream) {
  return gibbs_op(g, 2, image_dev, input_dev, nullptr, value, stream);
}

int b200rt_gibbs_hessian_diagonal_dev(b200rt_gibbs* g, const float* image_dev, float* out_dev, void* stream) {
  return gibbs_op(g, 3, image_dev, nullptr, out_dev, nullptr, stream);
}

int b200rt_gibbs_accumulate_hessian_times_input_dev(b200rt_gibbs* g, const float* image_dev, const float* input_dev,
                                                    float* output_dev, void* stream) {
  return gibbs_op(g, 4, image_dev, input_dev, output_dev, nullptr, stream);
}

int b200rt_gibbs_hessian_dev(b200rt_gibbs* g, const float* image_dev, int z, int y, int x, float* out_dev,
                             void* stream) {
  if (!g || !image_dev || !out_dev) return gfail(g, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (z < 0 || z >= g->d.nz || y < 0 || y >= g->d.ny || x < 0 || x >= g->d.nx)
    return gfail(g, B200RT_ERR_INVALID_ARGUMENT, "voxel outside the image");
  try {
    DeviceGuard dg(g->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = static_cast<int64_t>(g->d.nz) * g->d.ny * g->d.nx;
    ck(cudaMemsetAsync(out_dev, 0, sizeof(float) * n, st), "memset");
    if (g->d.beta != 0) ck(launch_gibbs_hessian_voxel(g->d, image_dev, z, y, x, out_dev, st), "Gibbs Hessian");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return gfail(g, status_of(e), e.what());
  }
}

}  // extern "C"
