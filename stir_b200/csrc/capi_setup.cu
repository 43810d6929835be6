// C ABI: projector set-up (rows, path tables, subset lists), creation, layouts.
#include "capi.hpp"

using namespace b200;

namespace capi {

std::mutex g_err_mu;
std::string g_create_error;

int fail(b200rt_projector* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int refuse_shard(b200rt_projector* h, const char* what) {
  return fail(h, B200RT_ERR_STATE, std::string(what) + ": not available on a view shard (b200rt_set_view_shard)");
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
        // column slots and basic segments must fit the packed elements (16 and 5 bits)
        if (keys.size() > 65535 || nsegs > 32) {
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
              G.cmaj.push_back(PathCElem{(e.sz >> 16) | (static_cast<uint32_t>(si) << 11) |
                                             (static_cast<uint32_t>(slot) << 16), e.v});
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
  // 34.25 KB of staged float columns: on the clinical geometry (nz 127, padding 24 planes) K = 58, the largest chunk
  // with which 4 forward CTAs still fit on an SM.  Forward projection of all its bins, measured: K 40 11.17 ms, 47
  // 10.22, 54 9.55, 58 9.20 (4 CTAs per SM); 61 9.01, 66-74 10.41-9.87, 81 9.51 (3 CTAs per SM; the batched
  // persistent forward then loses a quarter of its CTAs: dynamic OSEM 26.8 -> 24.6 frames/s at K 61); 94-135
  // 11.4-12.2 (2 CTAs per SM); 162 19.5 (1 CTA per SM)
  const int K = std::max(8, 35072 / (4 * (nz + std::max(zpad, 0))));
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
  h.dev_status.alloc(1);
  ck(cudaMemsetAsync(h.dev_status.p, 0, sizeof(unsigned), h.stream), "memset");
  ck(cudaStreamSynchronize(h.stream), "status word");
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
  pp.status = h.dev_status.p;
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
    tp.trunc_n = g.tof_truncation_n();
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
  h.h_segs_full = sd;
  std::vector<int64_t> lt;
  for (int s = -g.S(); s <= g.S(); ++s) {
    lt.push_back(g.stir_segment_offset(s));
    lt.push_back(g.dev_segment_offset(s));
    lt.push_back(g.nax(s));
  }
  h.layout_tab.upload(lt, h.stream);

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
  // the basic view of every entry of each work list (bins, TOF basic bins, path items) and of every view (-1: a
  // view no basic view reaches), on the device: the allocation-free entry point selects a subset's work and views
  // from these without host copies
  std::vector<int> view_basic(g.num_views(), -1);
  for (int v : g.basic_views())
    for (int seg : g.basic_segments()) {
      std::vector<RelatedLine> rel;
      g.related_lines(v, seg, true, rel);
      for (const auto& r : rel) view_basic[r.view] = v;
    }
  h.bin_view_dev.upload(h.h_bin_view, h.stream);
  h.view_basic_dev.upload(view_basic, h.stream);
  if (h.use_paths) h.item_view_dev.upload(h.h_item_view, h.stream);
  if (!h.h_tof_basic_view.empty()) h.tof_basic_view_dev.upload(h.h_tof_basic_view, h.stream);
  h.h_view_basic = std::move(view_basic);
  ck(cudaStreamSynchronize(h.stream), "basic view tables");
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
  for (int i = 0; i < static_cast<int>(h.h_item_view.size()); ++i) {
    if (h.h_item_view[i] % nsub != subset) continue;
    // a view shard skips the items whose lines all write views it does not hold
    const int ov = h.h_item_out_view.empty() ? -1 : h.h_item_out_view[i];
    if (sharded(h) && ov >= 0 && h.h_view_slot[ov] < 0) continue;
    list.push_back(i);
  }
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
                    const FwdEpilogue* ep) {
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
    if (in[v] && (!sharded(h) || h.h_view_slot[v] >= 0)) views.push_back(v);  // a view shard: the views it holds
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
// the largest column sum of A (A^T 1 over every bin), which bounds every voxel's sum of |w d| / max|d| (the fixed-point
// scale of the deterministic back projection); `scratch` is an image-sized buffer
void ensure_colmax(b200rt_projector& h, float* scratch, cudaStream_t st) {
  const Geometry& g = *h.geo;
  const int64_t ni = g.image_size();
  h.det_partial.alloc(std::max<int>(update_num_blocks(std::max<int64_t>(pd_size(h), ni)), 1));
  if (h.colmax_ready) return;
  const bool grouped = !h.use_paths && h.params.tof_w;
  h.colmax.alloc(1);
  int nall = 0;
  const int* all = h.use_paths ? path_list(h, 0, 1, nall)
                   : grouped   ? tof_group_list(h, 0, 1, nall)
                               : subset_list(h, 0, 1, nall);
  ck(cudaMemsetAsync(scratch, 0, sizeof(float) * ni, st), "memset");
  if (h.use_paths)
    ck(launch_back_paths_atomic(h.params, h.pparams, all, nall, nullptr, scratch, st, 0), "column sums");
  else if (grouped)
    ck(launch_back_tof_grouped(h.params, all, nall, nullptr, scratch, nullptr, nullptr, st, 0), "column sums");
  else
    ck(launch_back_atomic(h.params, all, nall, nullptr, scratch, st, 0), "column sums");
  ck(launch_max(scratch, ni, h.det_partial.p, h.colmax.p, st), "column sums");
  h.colmax_ready = true;
}

void back_project_into(b200rt_projector& h, const float* pd, float* image, int subset, int nsub, int mode, int zero_ends,
                       cudaStream_t st, float max_abs) {
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
  ensure_colmax(h, image, st);
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
    ck(launch_fixed_scale(pd, pd ? pd_size(h) : 1, h.colmax.p, h.det_partial.p, h.fixed_scale.p, st), "scale");
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

int max_nax(const Geometry& g) {
  int m = 0;
  for (int s = -g.S(); s <= g.S(); ++s) m = std::max(m, g.nax(s));
  return m;
}

cudaError_t projdata_layout(const b200rt_projector& h, const float* in, float* out, bool to_dev, cudaStream_t st) {
  const Geometry& g = *h.geo;
  return launch_projdata_layout_views(in, out, h.layout_tab.p, 2 * g.S() + 1, g.num_tof(), max_nax(g), g.tof_stride(),
                                      static_cast<int64_t>(g.num_views()) * g.num_tang(), 0,
                                      static_cast<int64_t>(g.num_views()) * g.num_tang(), to_dev, st);
}

// projection data layout change of the views [v0, v1) only (STIR order <-> device layout): one launch over every
// (timing bin, segment)
cudaError_t projdata_layout_views(const b200rt_projector& h, const float* in, float* out, bool to_dev, int v0, int v1,
                                  cudaStream_t st) {
  const Geometry& g = *h.geo;
  const int64_t nt = g.num_tang();
  return launch_projdata_layout_views(in, out, h.layout_tab.p, 2 * g.S() + 1, g.num_tof(), max_nax(g), g.tof_stride(),
                                      static_cast<int64_t>(g.num_views()) * nt, v0 * nt, (v1 - v0) * nt, to_dev, st);
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

}  // namespace capi

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
    // STIR's geometry checks (projection data, image grid, symmetries) run on the host first, so that an invalid
    // geometry gets STIR's message before any device work
    h->geo = std::make_unique<Geometry>(*geometry);
    int ndev = 0;
    ck(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) throw std::runtime_error("invalid CUDA device");
    h->device = device;
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
    h->ratio_batch.release();
    h->bin_view_dev.release();
    h->tof_basic_view_dev.release();
    h->item_view_dev.release();
    h->view_basic_dev.release();
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

int b200rt_set_view_shard(b200rt_projector* h, const int32_t* views, int num_views) {
  if (!h) return B200RT_ERR_INVALID_ARGUMENT;
  if (num_views < 0 || (num_views > 0 && !views)) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null view list");
  const Geometry& g = *h->geo;
  if (num_views > 0 && (!h->use_paths || g.num_tof() != 1))
    return fail(h, B200RT_ERR_UNSUPPORTED, "a view shard needs the column-staged kernels (non-TOF data)");
  std::vector<int> slot(g.num_views(), -1);
  for (int i = 0; i < num_views; ++i) {
    if (views[i] < 0 || views[i] >= g.num_views()) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "view out of range");
    if (slot[views[i]] >= 0) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "a view listed twice");
    slot[views[i]] = i;
  }
  try {
    DeviceGuard dg(h->device);
    ck(cudaStreamSynchronize(h->stream), "view shard");
    std::vector<SegDev> sd = h->h_segs_full;
    if (num_views > 0) {
      int64_t off = 0;
      for (int s = -g.S(); s <= g.S(); ++s) {
        sd[s + g.S()].dev_offset = off;
        off += static_cast<int64_t>(g.nax(s)) * num_views * g.num_tang();
      }
      h->shard_tof_stride = off;
      h->shard_pd_size = off;  // non-TOF
      h->view_slot_dev.upload(slot, h->stream);
    } else {
      h->view_slot_dev.release();
    }
    h->segs.upload(sd, h->stream);
    ck(cudaStreamSynchronize(h->stream), "view shard");
    h->shard_views.assign(views, views + num_views);
    h->h_view_slot = slot;
    h->params.segs = h->segs.p;
    h->params.view_slot = num_views > 0 ? h->view_slot_dev.p : nullptr;
    h->params.tof_stride = num_views > 0 ? h->shard_tof_stride : g.tof_stride();
    // every cached list and scratch sized by the data's layout is rebuilt on first use
    h->subset_lists.clear();
    h->subset_counts.clear();
    h->path_lists.clear();
    h->path_counts.clear();
    h->subset_views.clear();
    h->subset_view_counts.clear();
    h->view_groups.clear();
    h->colmax_ready = false;
    h->ratio.release();
    h->ratio_batch.release();
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_get_info(const b200rt_projector* h, b200rt_info* out) {
  if (!h || !out) return B200RT_ERR_INVALID_ARGUMENT;
  const Geometry& g = *h->geo;
  std::memset(out, 0, sizeof(*out));
  out->num_bins = pd_size(*h);
  out->num_image_voxels = g.image_size();
  out->num_basic_bins = static_cast<int64_t>(h->h_bins.size());
  out->num_row_elements = static_cast<int64_t>(h->rows.n);
  out->total_nnz = h->total_nnz;
  out->num_tof_bins = g.num_tof();
  out->num_basic_views = h->num_basic_views;
  out->symmetries_used = g.symmetry_bits();
  return B200RT_OK;
}

int64_t b200rt_projdata_size(const b200rt_projector* h) { return h ? pd_size(*h) : -1; }
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
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_projdata_to_device_layout");
  if (!h || !stir_dev || !dev) return B200RT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  const cudaError_t e = projdata_layout(*h, stir_dev, dev, true, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? B200RT_OK : fail(h, B200RT_ERR_CUDA, cudaGetErrorString(e));
}
int b200rt_projdata_from_device_layout(b200rt_projector* h, const float* dev, float* stir_dev, void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_projdata_from_device_layout");
  if (!h || !stir_dev || !dev) return B200RT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  const cudaError_t e = projdata_layout(*h, dev, stir_dev, false, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? B200RT_OK : fail(h, B200RT_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"
