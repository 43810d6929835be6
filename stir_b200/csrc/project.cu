// Forward and back projection with the rows of STIR's ray-tracing matrix,
// unfolding its symmetries on the fly.
//
// Work decomposition (one CTA per basic bin):
//   * the basic row (STIR's cached row, ProjMatrixByBin.inl:48-113) is staged in shared memory;
//   * each warp takes one related line at a time: a viewgram related by a symmetry
//     (DataSymmetriesForBins_PET_CartesianGrid::get_related_view_segment_numbers) at the
//     basic tangential position or its mirror;
//   * the warp's lanes are the axial positions of that line (the z-shift symmetry): lane a
//     reads voxel z' = (zq ? q - z : z) + npa*a, so with the image stored z-fastest
//     ([y][x][z]) the 32 lanes of a warp read consecutive floats of one column;
//   * the transformed column offsets of the row are computed once per line by the warp's
//     lanes in parallel (into shared memory) and reused for all axial positions.
//
// Forward: projdata[line][a] = sum_k image[col_k][z_k + npa*a] * w_k, z range-checked as in
//          ProjMatrixElemsForOneBin::forward_project (ProjMatrixElemsForOneBin.cxx:354-370).
// Back:    image[col_k][z_k + npa*a] += w_k * projdata[line][a] for projdata != 0
//          (ProjMatrixElemsForOneBin::back_project, :333-351), with float atomics.
//
// Lines with at most 16 axial positions (small scanners, TOF data) use the packed kernels below instead (a warp
// per basic bin, lanes = (line, axial position)); with TOF, the TOF-grouped kernels project all timing bins of a
// basic bin from its non-TOF row in one warp.
#include <type_traits>

#include "internal.hpp"
#include "epilogue.cuh"

namespace b200 {

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kAxPerLane = 4;  // axial positions per lane per pass: 128 per warp
// resident CTAs per SM the projection kernels are compiled for (registers <= 65536 / (CTAs * kThreads)):
// on the clinical geometry a sixth CTA per SM gains more than the few registers it spills cost
constexpr int kMinCtasForward = 6;
constexpr int kMinCtasBack = 6;

struct LineSetup {
  int64_t out_base;  // device-layout index of (line, axial 0)
  int nax, npa;
  int tofi;          // timing bin - min
};

__device__ __forceinline__ bool setup_line(const ProjParams& p, const ProjBinDev& pb, const LineDev& L, LineSetup& s) {
  const int tang = static_cast<int>(L.tang_sign) * pb.tang;
  if (tang < p.min_tang || tang > p.max_tang) return false;
  const SegDev sd = p.segs[L.seg + p.S];
  s.nax = sd.nax;
  s.npa = sd.npa;
  s.tofi = pb.tof - p.min_tof;
  s.out_base = static_cast<int64_t>(pb.tof - p.min_tof) * p.tof_stride + sd.dev_offset +
               (static_cast<int64_t>(L.view) * p.num_tang + (tang - p.min_tang)) * sd.nax;
  return true;
}

// A row element after the line's symmetry operation:
//   base = col*nz + zt, the image index of the element for axial position 0,
//   zt   = z' - min_z for axial position 0,
//   full = 1 when z' stays inside [0,nz) for every axial position of the current pass, so the
//          per-lane range checks can be skipped (a warp-uniform branch: all lanes read the same element).
struct __align__(16) XElem {
  int base;
  int zt;
  float v;
  int full;
};

constexpr int kChunk = 256;  // row elements transformed per warp at a time

__device__ __forceinline__ void transform_chunk(const ProjParams& p, const RowElem* srow, int c0, int cn, const LineDev& L,
                                                int npa, int a_first, int a_last, XElem* xbuf, int lane) {
  const int swap = L.flags & 1;
  const int sx = (L.flags & 2) ? -1 : 1;
  const int sy = (L.flags & 4) ? -1 : 1;
  const int zq = (L.flags & 8) ? 1 : 0;
  for (int k = lane; k < cn; k += 32) {
    const RowElem e = srow[c0 + k];
    int z, y, x;
    unpack_zyx(e.zyx, z, y, x);
    const int xt = (swap ? y : x) * sx;
    const int yt = (swap ? x : y) * sy;
    XElem o;
    o.zt = (zq ? static_cast<int>(L.q) - z : z) - p.min_z;
    o.base = ((yt - p.min_y) * p.nx + (xt - p.min_x)) * p.nz + o.zt;
    o.v = e.v;
    o.full = (o.zt + a_first * npa >= 0) && (o.zt + a_last * npa < p.nz);
    xbuf[k] = o;
  }
}

__device__ __forceinline__ void stage_row(const ProjParams& p, const ProjBinDev& pb, RowElem* srow) {
  for (int i = threadIdx.x; i < pb.row_len; i += blockDim.x) srow[i] = p.rows[pb.row_offset + i];
}

// One pass of one line: NJ groups of 32 axial positions starting at a0 (lane j*32+lane is axial
// a0+j*32+lane).  NPA: planes per axial position known at compile time (1, 2), or 0 for run time.
template <int NPA, int NJ, int EPI>
__device__ __forceinline__ void forward_pass(const ProjParams& p, const RowElem* srow, int n, const LineDev& L,
                                             const LineSetup& s, int a0, int nact, XElem* xbuf, int lane,
                                             const float* __restrict__ img, float* __restrict__ out, const FwdEpilogue& ep,
                                             double& ll, unsigned& ncancel) {
  const int npa = NPA ? NPA : s.npa;
  const int step = 32 * npa;
  const unsigned nz = static_cast<unsigned>(p.nz);
  int zoff[NJ];
  bool act[NJ];
  float acc[NJ];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    act[j] = j * 32 + lane < nact;
    zoff[j] = (a0 + j * 32 + lane) * npa;
    acc[j] = 0.f;
  }
  for (int c0 = 0; c0 < n; c0 += kChunk) {
    const int cn = min(kChunk, n - c0);
    __syncwarp();
    transform_chunk(p, srow, c0, cn, L, npa, a0, a0 + nact - 1, xbuf, lane);
    __syncwarp();
    for (int k = 0; k < cn; ++k) {
      const XElem e = xbuf[k];
      if (e.full) {
        const float* q = img + (e.base + zoff[0]);
#pragma unroll
        for (int j = 0; j < NJ; ++j)
          if (act[j]) acc[j] += __ldg(q + j * step) * e.v;
      } else {
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const int zz = e.zt + zoff[j];
          if (act[j] && static_cast<unsigned>(zz) < nz) acc[j] += __ldg(img + (e.base + zoff[j])) * e.v;
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j)
    if (act[j]) {
      const int a = a0 + j * 32 + lane;
      forward_store<EPI>(p, L.seg, L.view, s.tofi, s.nax, s.out_base + a, a, acc[j], out, ep, ll, ncancel);
    }
}

// Accumulation of one back-projected contribution w*d:
//   float image: red.global.add.f32 (order-dependent rounding);
//   fixed point: the contribution rounded to an integer multiple of 1/scale (scale a power of two) and added
//   with 64-bit integer atomics, so the sum is the same whatever the order of the additions (deterministic mode).
struct FloatAcc {
  float* img;
  __device__ __forceinline__ void add(int64_t i, float v) const { atomicAdd(img + i, v); }
};
struct FixedAcc {
  unsigned long long* acc;
  const double* scale;
  __device__ __forceinline__ void add(int64_t i, float v) const {
    atomicAdd(acc + i, static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(v) * *scale)));
  }
};

template <int NPA, int NJ, typename Acc>
__device__ __forceinline__ void back_pass(const ProjParams& p, const RowElem* srow, int n, const LineDev& L,
                                          const LineSetup& s, int a0, int nact, XElem* xbuf, int lane,
                                          const float* __restrict__ pd, const Acc& out, int zero_ends) {
  const int npa = NPA ? NPA : s.npa;
  const int step = 32 * npa;
  const unsigned nz = static_cast<unsigned>(p.nz);
  int zoff[NJ];
  bool act[NJ];
  float d[NJ];
  bool any = false;
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int a = a0 + j * 32 + lane;
    const bool in = j * 32 + lane < nact && !(zero_ends && L.seg == 0 && (a == 0 || a == s.nax - 1));
    // pd == nullptr back-projects ones (the sensitivity of RPC_process_related_viewgrams_sensitivity_computation)
    d[j] = in ? (pd ? __ldg(pd + s.out_base + a) : 1.f) : 0.f;
    act[j] = d[j] != 0.f;  // zero bins are skipped (ProjMatrixElemsForOneBin.cxx:339-340)
    zoff[j] = (a0 + j * 32 + lane) * npa;
    any |= act[j];
  }
  if (!__any_sync(0xffffffffu, any)) return;
  for (int c0 = 0; c0 < n; c0 += kChunk) {
    const int cn = min(kChunk, n - c0);
    __syncwarp();
    transform_chunk(p, srow, c0, cn, L, npa, a0, a0 + nact - 1, xbuf, lane);
    __syncwarp();
    for (int k = 0; k < cn; ++k) {
      const XElem e = xbuf[k];
      if (e.full) {
        const int64_t q = e.base + zoff[0];
#pragma unroll
        for (int j = 0; j < NJ; ++j)
          if (act[j]) out.add(q + j * step, e.v * d[j]);
      } else {
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const int zz = e.zt + zoff[j];
          if (act[j] && static_cast<unsigned>(zz) < nz) out.add(e.base + zoff[j], e.v * d[j]);
        }
      }
    }
  }
}

// All related lines of one basic bin (one CTA).
template <int NPA, int EPI>
__device__ __forceinline__ void forward_bin(const ProjParams& p, const ProjBinDev& pb, unsigned char* smem,
                                            const float* __restrict__ img, float* __restrict__ out, const FwdEpilogue& ep,
                                            double& ll, unsigned& ncancel) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  XElem* xbuf = reinterpret_cast<XElem*>(smem) + warp * kChunk;
  RowElem* srow = reinterpret_cast<RowElem*>(smem + sizeof(XElem) * kWarps * kChunk);
  const int n = pb.row_len;
  stage_row(p, pb, srow);
  __syncthreads();
  for (int l = warp; l < pb.num_lines; l += kWarps) {
    const LineDev L = p.lines[pb.first_line + l];
    LineSetup s;
    if (!setup_line(p, pb, L, s)) continue;
    for (int a0 = 0; a0 < s.nax; a0 += 32 * kAxPerLane) {
      const int nact = min(s.nax - a0, 32 * kAxPerLane);
      switch ((nact + 31) >> 5) {
        case 1: forward_pass<NPA, 1, EPI>(p, srow, n, L, s, a0, nact, xbuf, lane, img, out, ep, ll, ncancel); break;
        case 2: forward_pass<NPA, 2, EPI>(p, srow, n, L, s, a0, nact, xbuf, lane, img, out, ep, ll, ncancel); break;
        case 3: forward_pass<NPA, 3, EPI>(p, srow, n, L, s, a0, nact, xbuf, lane, img, out, ep, ll, ncancel); break;
        default: forward_pass<NPA, 4, EPI>(p, srow, n, L, s, a0, nact, xbuf, lane, img, out, ep, ll, ncancel); break;
      }
    }
  }
}

template <int NPA, int EPI>
__global__ void __launch_bounds__(kThreads, kMinCtasForward) forward_kernel(ProjParams p, const int* __restrict__ bin_list,
                                                           const float* __restrict__ img, float* __restrict__ out,
                                                           FwdEpilogue ep) {
  extern __shared__ __align__(16) unsigned char smem[];
  const ProjBinDev pb = p.bins[bin_list[blockIdx.x]];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double ll = 0.0;
  unsigned ncancel = 0;
  forward_bin<NPA, EPI>(p, pb, smem, img, out, ep, ll, ncancel);
  if (EPI == kEpiRatio || EPI == kEpiGradient) {
    // cancelled singularities (distributable.cxx:590-594)
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if (lane == 0 && ncancel && ep.cancelled) atomicAdd(ep.cancelled, ncancel);
  }
  if (EPI == kEpiLoglik) {
    // per-CTA partial sums, reduced in a fixed order by the caller: deterministic
    __shared__ double red[kWarps];
    for (int o = 16; o > 0; o >>= 1) ll += __shfl_xor_sync(0xffffffffu, ll, o);
    if (lane == 0) red[warp] = ll;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kWarps; ++w) t += red[w];
      ep.partials[blockIdx.x] = t;
    }
  }
}

template <int NPA, typename Acc>
__device__ __forceinline__ void back_bin(const ProjParams& p, const ProjBinDev& pb, unsigned char* smem,
                                         const float* __restrict__ pd, const Acc& img, int zero_ends) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  XElem* xbuf = reinterpret_cast<XElem*>(smem) + warp * kChunk;
  RowElem* srow = reinterpret_cast<RowElem*>(smem + sizeof(XElem) * kWarps * kChunk);
  const int n = pb.row_len;
  stage_row(p, pb, srow);
  __syncthreads();
  for (int l = warp; l < pb.num_lines; l += kWarps) {
    const LineDev L = p.lines[pb.first_line + l];
    LineSetup s;
    if (!setup_line(p, pb, L, s)) continue;
    for (int a0 = 0; a0 < s.nax; a0 += 32 * kAxPerLane) {
      const int nact = min(s.nax - a0, 32 * kAxPerLane);
      switch ((nact + 31) >> 5) {
        case 1: back_pass<NPA, 1>(p, srow, n, L, s, a0, nact, xbuf, lane, pd, img, zero_ends); break;
        case 2: back_pass<NPA, 2>(p, srow, n, L, s, a0, nact, xbuf, lane, pd, img, zero_ends); break;
        case 3: back_pass<NPA, 3>(p, srow, n, L, s, a0, nact, xbuf, lane, pd, img, zero_ends); break;
        default: back_pass<NPA, 4>(p, srow, n, L, s, a0, nact, xbuf, lane, pd, img, zero_ends); break;
      }
    }
  }
}

template <int NPA, typename Acc>
__global__ void __launch_bounds__(kThreads, kMinCtasBack) back_atomic_kernel(ProjParams p, const int* __restrict__ bin_list,
                                                               const float* __restrict__ pd, Acc img, int zero_ends) {
  extern __shared__ __align__(16) unsigned char smem[];
  const ProjBinDev pb = p.bins[bin_list[blockIdx.x]];
  back_bin<NPA, Acc>(p, pb, smem, pd, img, zero_ends);
}

// ---- packed kernels: few axial positions per line ----------------------------
// With at most 16 axial positions per line (small scanners, and TOF data, where every timing bin of a basic bin
// has its own row) the kernels above leave most lanes idle.  Here a warp takes a whole basic bin and its lanes
// are (related line, axial position) pairs, 32 / nax lines at a time; the warp reads the row 32 elements at a
// time (coalesced) and shuffles each element to every lane, which applies its own line's symmetry operation.
// Each lane sums its bin's elements in row order, as the kernels above do, so the sums are the same.
constexpr int kPackedWarps = 8;

struct PackedLane {
  bool act;
  int swap, sx, sy, zq, q, zoff;  // zoff = npa * a - min_z
  int a;
  LineSetup s;
  LineDev L;
};

__device__ __forceinline__ PackedLane packed_lane(const ProjParams& p, const ProjBinDev& pb, int l0, int G, int nax,
                                                  int lane) {
  PackedLane t{};
  const int gi = lane / nax;
  const int l = l0 + gi;
  t.a = lane - gi * nax;
  t.act = gi < G && l < pb.num_lines;
  if (t.act) {
    t.L = p.lines[pb.first_line + l];
    t.act = setup_line(p, pb, t.L, t.s);
  }
  if (t.act) {
    t.swap = t.L.flags & 1;
    t.sx = (t.L.flags & 2) ? -1 : 1;
    t.sy = (t.L.flags & 4) ? -1 : 1;
    t.zq = (t.L.flags & 8) ? 1 : 0;
    t.q = t.L.q;
    t.zoff = t.a * t.s.npa - p.min_z;
  }
  return t;
}

// nax of the basic bin's lines (a basic bin's related lines all have segments +-s)
__device__ __forceinline__ int packed_nax(const ProjParams& p, const ProjBinDev& pb) {
  return p.segs[p.lines[pb.first_line].seg + p.S].nax;
}

// the lane's (line, axial position) in the TOF-grouped kernels: packed (line groups of nax lanes) with at most
// kPackedMaxNax axial positions, else one line at a time in blocks of 32 axial positions from a0
__device__ __forceinline__ PackedLane tof_lane(const ProjParams& p, const ProjBinDev& pb, int l0, int G, int nax, int a0,
                                               int lane) {
  if (nax <= kPackedMaxNax) return packed_lane(p, pb, l0, G, nax, lane);
  PackedLane t{};
  t.a = a0 + lane;
  t.act = t.a < nax && l0 < pb.num_lines;
  if (t.act) {
    t.L = p.lines[pb.first_line + l0];
    t.act = setup_line(p, pb, t.L, t.s);
  }
  return t;
}

// The transformed elements of a batch of 32, per line of the group being projected: xs[g][k] = (image index of
// element k under line g without its z, z after the line's z operation - min_z); lane k computes element k for
// every line, so each transform is done once instead of once per axial position.
constexpr int kPackedMaxLines = 16;  // lines per basic bin handled per pass (32 / nax, at most the bin's lines)
struct PackedStage {
  int2 xs[kPackedMaxLines][33];  // padded: the lanes of different lines read the same k without bank conflicts
  float w[32];
};

// one basic bin by one warp (the lanes are (line, axial position) pairs); S is the warp's staging table
template <int EPI>
__device__ __forceinline__ void forward_packed_bin(const ProjParams& p, const ProjBinDev& pb, PackedStage& S,
                                                   const float* __restrict__ img, float* __restrict__ out,
                                                   const FwdEpilogue& ep, double& ll, unsigned& ncancel, int lane) {
  const RowElem* row = p.rows + pb.row_offset;
  const int nax = packed_nax(p, pb);
  const int G = min(32 / nax, kPackedMaxLines);
  const int gi = lane / nax;
  for (int l0 = 0; l0 < pb.num_lines; l0 += G) {
    const PackedLane t = packed_lane(p, pb, l0, G, nax, lane);
    const int ng = min(G, pb.num_lines - l0);
    float acc = 0.f;
    for (int k0 = 0; k0 < pb.row_len; k0 += 32) {
      const int cnt = min(32, pb.row_len - k0);
      __syncwarp();
      if (lane < cnt) {
        const RowElem e = row[k0 + lane];
        int z, y, x;
        unpack_zyx(e.zyx, z, y, x);
        S.w[lane] = e.v;
        for (int g = 0; g < ng; ++g) {
          const LineDev L = p.lines[pb.first_line + l0 + g];
          const int swap = L.flags & 1;
          const int xt = (swap ? y : x) * ((L.flags & 2) ? -1 : 1);
          const int yt = (swap ? x : y) * ((L.flags & 4) ? -1 : 1);
          const int zt = ((L.flags & 8) ? static_cast<int>(L.q) - z : z) - p.min_z;
          S.xs[g][lane] = make_int2(((yt - p.min_y) * p.nx + (xt - p.min_x)) * p.nz, zt);
        }
      }
      __syncwarp();
      if (t.act) {
        const int zoff = t.a * t.s.npa;
        int k = 0;
        for (; k + 4 <= cnt; k += 4) {
          int v[4];
          float xv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int2 X = S.xs[gi][k + u];
            const int zz = X.y + zoff;
            v[u] = (zz >= 0 && zz < p.nz) ? X.x + zz : -1;
            xv[u] = v[u] >= 0 ? __ldg(img + v[u]) : 0.f;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (v[u] >= 0) acc += xv[u] * S.w[k + u];
        }
        for (; k < cnt; ++k) {
          const int2 X = S.xs[gi][k];
          const int zz = X.y + zoff;
          if (zz >= 0 && zz < p.nz) acc += __ldg(img + X.x + zz) * S.w[k];
        }
      }
    }
    if (t.act) forward_store<EPI>(p, t.L.seg, t.L.view, t.s.tofi, t.s.nax, t.s.out_base + t.a, t.a, acc, out, ep, ll, ncancel);
  }
  __syncwarp();  // the staging table is free for the warp's next bin
}

template <int EPI>
__global__ void __launch_bounds__(kPackedWarps * 32) forward_packed_kernel(ProjParams p, const int* __restrict__ bin_list,
                                                                          int nbins, const float* __restrict__ img,
                                                                          float* __restrict__ out, FwdEpilogue ep) {
  __shared__ PackedStage stage[kPackedWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bi = blockIdx.x * kPackedWarps + warp;
  if (bi >= nbins) return;  // whole warps only: no block-wide synchronisation below
  double ll = 0.0;
  unsigned ncancel = 0;
  forward_packed_bin<EPI>(p, p.bins[bin_list[bi]], stage[warp], img, out, ep, ll, ncancel, lane);
  if (EPI == kEpiRatio || EPI == kEpiGradient) {
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if (lane == 0 && ncancel && ep.cancelled) atomicAdd(ep.cancelled, ncancel);
  }
  if (EPI == kEpiLoglik) {
    // one partial per basic bin (as the one-CTA-per-bin kernel), reduced in a fixed order by the caller
    for (int o = 16; o > 0; o >>= 1) ll += __shfl_xor_sync(0xffffffffu, ll, o);
    if (lane == 0) ep.partials[bi] = ll;
  }
}

template <typename Acc>
__device__ __forceinline__ void back_packed_bin(const ProjParams& p, const ProjBinDev& pb, PackedStage& S,
                                                const float* __restrict__ pd, const Acc& img, int zero_ends, int lane) {
  const RowElem* row = p.rows + pb.row_offset;
  const int nax = packed_nax(p, pb);
  const int G = min(32 / nax, kPackedMaxLines);
  const int gi = lane / nax;
  for (int l0 = 0; l0 < pb.num_lines; l0 += G) {
    PackedLane t = packed_lane(p, pb, l0, G, nax, lane);
    const int ng = min(G, pb.num_lines - l0);
    float d = 0.f;
    if (t.act && !(zero_ends && t.L.seg == 0 && (t.a == 0 || t.a == t.s.nax - 1)))
      d = pd ? __ldg(pd + t.s.out_base + t.a) : 1.f;  // pd == nullptr back-projects ones
    t.act = t.act && d != 0.f;  // zero bins are skipped (ProjMatrixElemsForOneBin.cxx:339-340)
    if (!__any_sync(0xffffffffu, t.act)) continue;
    const int zoff = t.a * t.s.npa;
    for (int k0 = 0; k0 < pb.row_len; k0 += 32) {
      const int cnt = min(32, pb.row_len - k0);
      __syncwarp();
      if (lane < cnt) {
        const RowElem e = row[k0 + lane];
        int z, y, x;
        unpack_zyx(e.zyx, z, y, x);
        S.w[lane] = e.v;
        for (int g = 0; g < ng; ++g) {
          const LineDev L = p.lines[pb.first_line + l0 + g];
          const int swap = L.flags & 1;
          const int xt = (swap ? y : x) * ((L.flags & 2) ? -1 : 1);
          const int yt = (swap ? x : y) * ((L.flags & 4) ? -1 : 1);
          const int zt = ((L.flags & 8) ? static_cast<int>(L.q) - z : z) - p.min_z;
          S.xs[g][lane] = make_int2(((yt - p.min_y) * p.nx + (xt - p.min_x)) * p.nz, zt);
        }
      }
      __syncwarp();
      if (t.act)
        for (int k = 0; k < cnt; ++k) {
          const int2 X = S.xs[gi][k];
          const int zz = X.y + zoff;
          if (zz >= 0 && zz < p.nz) img.add(X.x + zz, S.w[k] * d);
        }
    }
  }
  __syncwarp();
}

template <typename Acc>
__global__ void __launch_bounds__(kPackedWarps * 32) back_packed_kernel(ProjParams p, const int* __restrict__ bin_list,
                                                                       int nbins, const float* __restrict__ pd, Acc img,
                                                                       int zero_ends) {
  __shared__ PackedStage stage[kPackedWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bi = blockIdx.x * kPackedWarps + warp;
  if (bi >= nbins) return;
  back_packed_bin<Acc>(p, p.bins[bin_list[bi]], stage[warp], pd, img, zero_ends, lane);
}

// ---- batched (several reconstructions in one launch) ------------------------
// A persistent grid takes work items (frame, basic bin) from a queue in list order: the list is
// frame-major, so at any time the CTAs work on one or two frames and their images stay in L2.
// The current item's frame, geometry and basic bin, copied to shared memory by the CTA so that the
// projection loops read them like kernel parameters instead of holding them in registers.
struct BatchStage {
  ProjParams p;
  BatchFrameDev f;
  ProjBinDev pb;
};
static_assert(sizeof(ProjParams) % 4 == 0 && sizeof(BatchFrameDev) % 4 == 0 && sizeof(ProjBinDev) % 4 == 0,
              "staged structures are copied as 32-bit words");

__device__ __forceinline__ bool next_item(unsigned* counter, const BatchItem* __restrict__ items, int nitems,
                                          const ProjParams* __restrict__ geoms, const BatchFrameDev* __restrict__ frames,
                                          BatchStage& st) {
  __shared__ int s_item;
  __syncthreads();  // every thread has finished with the previous item (shared row, stage, s_item)
  if (threadIdx.x == 0) s_item = static_cast<int>(atomicAdd(counter, 1u));
  __syncthreads();
  const int it = s_item;
  if (it >= nitems) return false;
  const BatchItem wi = items[it];
  const int g = frames[wi.frame].geom;
  constexpr int nf = sizeof(BatchFrameDev) / 4, np = sizeof(ProjParams) / 4, nb = sizeof(ProjBinDev) / 4;
  static_assert(nf + np + nb <= kThreads, "one word per thread");
  const int t = threadIdx.x;
  if (t < nf) {
    reinterpret_cast<uint32_t*>(&st.f)[t] = reinterpret_cast<const uint32_t*>(frames + wi.frame)[t];
  } else if (t < nf + np) {
    reinterpret_cast<uint32_t*>(&st.p)[t - nf] = reinterpret_cast<const uint32_t*>(geoms + g)[t - nf];
  } else if (t < nf + np + nb) {
    reinterpret_cast<uint32_t*>(&st.pb)[t - nf - np] = reinterpret_cast<const uint32_t*>(geoms[g].bins + wi.bin)[t - nf - np];
  }
  __syncthreads();
  return true;
}

template <int NPA>
__global__ void __launch_bounds__(kThreads, kMinCtasForward) forward_batch_kernel(const ProjParams* __restrict__ geoms,
                                                                           const BatchFrameDev* __restrict__ frames,
                                                                           const BatchItem* __restrict__ items,
                                                                           int nitems, unsigned* counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchStage st;
  const int lane = threadIdx.x & 31;
  while (next_item(counter, items, nitems, geoms, frames, st)) {
    double ll = 0.0;
    unsigned ncancel = 0;
    forward_bin<NPA, kEpiRatio>(st.p, st.pb, smem, st.f.x, st.f.ratio, st.f.ep, ll, ncancel);
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if (lane == 0 && ncancel && st.f.ep.cancelled) atomicAdd(st.f.ep.cancelled, ncancel);
  }
}

template <int NPA>
__global__ void __launch_bounds__(kThreads, kMinCtasBack) back_batch_kernel(const ProjParams* __restrict__ geoms,
                                                                        const BatchFrameDev* __restrict__ frames,
                                                                        const BatchItem* __restrict__ items,
                                                                        int nitems, unsigned* counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchStage st;
  while (next_item(counter, items, nitems, geoms, frames, st))
    back_bin<NPA, FloatAcc>(st.p, st.pb, smem, st.f.ratio, FloatAcc{st.f.u}, 0);
}

// out[c * ld_out + r] = in[r * ld_in + c] for r < rows, c < cols: the image [z][y][x] <-> [y][x][z] and
// projection data [axial][view, tangential] <-> [view, tangential][axial] layout changes, whole or a column range
__global__ void transpose_kernel(const float* __restrict__ in, float* __restrict__ out, int rows, int64_t cols,
                                 int64_t ld_in, int64_t ld_out) {
  __shared__ float tile[32][33];
  const int64_t c0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int r0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int i = ty; i < 32; i += 8) {
    const int r = r0 + i;
    const int64_t c = c0 + tx;
    if (r < rows && c < cols) tile[i][tx] = in[static_cast<int64_t>(r) * ld_in + c];
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int64_t c = c0 + i;
    const int r = r0 + tx;
    if (r < rows && c < cols) out[c * ld_out + r] = tile[tx][i];
  }
}

// the layout change of columns [c0, c0 + nc) of every (timing bin, segment): blockIdx.z = timing bin x segment; the
// same 32 x 32 tiles as transpose_kernel (STIR order: rows = axial positions, columns = views x tangential
// positions, leading dimension nvt; device layout: rows = views x tangential, columns = axial positions)
__global__ void projdata_layout_kernel(const float* __restrict__ in, float* __restrict__ out, const int64_t* __restrict__ tab,
                                       int nsegs, int64_t tof_stride, int64_t nvt, int64_t c0, int64_t nc, int to_dev) {
  __shared__ float tile[32][33];
  const int k = blockIdx.z / nsegs, si = blockIdx.z % nsegs;
  const int nax = static_cast<int>(tab[3 * si + 2]);
  const int64_t so = k * tof_stride + tab[3 * si] + c0;
  const int64_t dv = k * tof_stride + tab[3 * si + 1] + c0 * nax;
  // rows x cols of the input, and its leading dimensions in and out
  const int64_t rows = to_dev ? nax : nc, cols = to_dev ? nc : nax;
  const int64_t ld_in = to_dev ? nvt : nax, ld_out = to_dev ? nax : nvt;
  const float* src = in + (to_dev ? so : dv);
  float* dst = out + (to_dev ? dv : so);
  const int64_t cb = static_cast<int64_t>(blockIdx.x) * 32, rb = static_cast<int64_t>(blockIdx.y) * 32;
  if (cb >= cols || rb >= rows) return;  // a tile past this segment's extent
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int i = ty; i < 32; i += 8) {
    const int64_t r = rb + i, c = cb + tx;
    if (r < rows && c < cols) tile[i][tx] = src[r * ld_in + c];
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int64_t c = cb + i, r = rb + tx;
    if (r < rows && c < cols) dst[c * ld_out + r] = tile[tx][i];
  }
}

cudaError_t transpose(const float* in, float* out, int rows, int64_t cols, cudaStream_t st) {
  return launch_transpose(in, out, rows, cols, cols, rows, st);
}

}  // namespace

size_t proj_smem_bytes(int max_row_len) {
  return sizeof(XElem) * kWarps * kChunk + sizeof(RowElem) * static_cast<size_t>(max_row_len > 0 ? max_row_len : 1);
}

// ---- TOF-grouped packed kernels ------------------------------------------------
// With TOF, every timing bin of a basic bin has its own row: the basic row's elements weighted by the timing
// bin's kernel.  Here a warp takes a basic bin with all its timing bins: it walks the non-TOF row once per group of
// KG timing bins, gathers each voxel once, and applies the group's weights (staged per batch of 32
// elements in shared memory) from registers.  Forward: each (line, axial position, timing bin) sum adds the same
// products in the same order as the TOF row (elements outside the TOF row have weight 0 and add +-0), so the
// results are bit-identical.  Back: the contributions of the group's timing bins to a voxel are summed before the
// one atomic (float), or, in fixed point, summed in float in that fixed order and rounded once to an integer.
constexpr int kTofWarps = 4;
constexpr int kTofMinCtas = 8;  // 64 registers: 32 warps per SM (79 registers left 24)
constexpr int kTofGroupMax = 32;  // timing bins per pass: KG in {8, 16, 20, 24, 32}, chosen from their number
template <int KG>
struct TofStage {
  int2 xs[kPackedMaxLines][33];
  float4 w[32][KG / 4];
};

// transforms and weights of elements [e0, e0 + cnt) of the basic row for the lines l0.. (ng of them) and the
// timing bins [k0, k0 + KG)
template <int KG>
__device__ __forceinline__ void tof_stage_batch(const ProjParams& p, const ProjBinDev& pb, const RowElem* row,
                                                const float* wrow, int K, int l0, int ng, int e0, int cnt, int k0,
                                                TofStage<KG>& S, int lane) {
  __syncwarp();
  if (lane < cnt) {
    const RowElem e = row[e0 + lane];
    int z, y, x;
    unpack_zyx(e.zyx, z, y, x);
    for (int g = 0; g < ng; ++g) {
      const LineDev L = p.lines[pb.first_line + l0 + g];
      const int swap = L.flags & 1;
      const int xt = (swap ? y : x) * ((L.flags & 2) ? -1 : 1);
      const int yt = (swap ? x : y) * ((L.flags & 4) ? -1 : 1);
      const int zt = ((L.flags & 8) ? static_cast<int>(L.q) - z : z) - p.min_z;
      S.xs[g][lane] = make_int2(((yt - p.min_y) * p.nx + (xt - p.min_x)) * p.nz, zt);
    }
  }
  // weights: the batch's elements x timing bins are contiguous ([element][timing bin]); coalesced loads
  float* sw = reinterpret_cast<float*>(S.w);
  const float* src = wrow + static_cast<int64_t>(e0) * K;
  for (int i = lane; i < 32 * KG; i += 32) {
    const int e = i / KG, kk = i % KG;
    sw[e * KG + kk] = (e < cnt && k0 + kk < K) ? __ldg(src + static_cast<int64_t>(e) * K + k0 + kk) : 0.f;
  }
  __syncwarp();
}

template <int KG, int EPI>
__device__ __forceinline__ void forward_tof_grouped_body(const ProjParams& p, const ProjBinDev& pb, TofStage<KG>& S,
                                                         const float* __restrict__ img, float* __restrict__ out,
                                                         const FwdEpilogue& ep, double& ll, unsigned& ncancel,
                                                         int lane) {
  const RowElem* row = p.tof_basic_rows + pb.row_offset;
  const int K = p.num_tof;
  const float* wrow = p.tof_w + pb.row_offset * K;
  const int nax = packed_nax(p, pb);
  const bool blocked = nax > kPackedMaxNax;
  const int G = blocked ? 1 : min(32 / nax, kPackedMaxLines);
  const int gi = blocked ? 0 : lane / nax;
  for (int l0 = 0; l0 < pb.num_lines; l0 += G)
  for (int a0 = 0; a0 < (blocked ? nax : 1); a0 += 32) {
    const PackedLane t = tof_lane(p, pb, l0, G, nax, a0, lane);
    const int ng = min(G, pb.num_lines - l0);
    const int zoff = t.a * t.s.npa;
    for (int k0 = 0; k0 < K; k0 += KG) {
      float acc[KG];
#pragma unroll
      for (int kk = 0; kk < KG; ++kk) acc[kk] = 0.f;
      for (int e0 = 0; e0 < pb.row_len; e0 += 32) {
        const int cnt = min(32, pb.row_len - e0);
        tof_stage_batch<KG>(p, pb, row, wrow, K, l0, ng, e0, cnt, k0, S, lane);
        if (t.act)
          for (int k = 0; k < cnt; ++k) {
            const int2 X = S.xs[gi][k];
            const int zz = X.y + zoff;
            if (zz < 0 || zz >= p.nz) continue;
            const float xv = __ldg(img + X.x + zz);
#pragma unroll
            for (int q = 0; q < KG / 4; ++q) {
              const float4 w = S.w[k][q];
              acc[4 * q] += xv * w.x;
              acc[4 * q + 1] += xv * w.y;
              acc[4 * q + 2] += xv * w.z;
              acc[4 * q + 3] += xv * w.w;
            }
          }
      }
      if (t.act)
#pragma unroll
        for (int kk = 0; kk < KG; ++kk)
          if (k0 + kk < K)
            forward_store<EPI>(p, t.L.seg, t.L.view, k0 + kk, t.s.nax,
                               t.s.out_base + static_cast<int64_t>(k0 + kk) * p.tof_stride + t.a, t.a, acc[kk], out, ep,
                               ll, ncancel);
    }
  }
  __syncwarp();
}

template <int KG, int EPI>
__global__ void __launch_bounds__(kTofWarps * 32, kTofMinCtas) forward_tof_grouped_kernel(ProjParams p, const int* __restrict__ items,
                                                                            int nitems, const float* __restrict__ img,
                                                                            float* __restrict__ out, FwdEpilogue ep) {
  __shared__ TofStage<KG> stage[kTofWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bi = blockIdx.x * kTofWarps + warp;
  if (bi >= nitems) return;
  double ll = 0.0;
  unsigned ncancel = 0;
  forward_tof_grouped_body<KG, EPI>(p, p.tof_basic[items[bi]], stage[warp], img, out, ep, ll, ncancel, lane);
  if (EPI == kEpiRatio || EPI == kEpiGradient) {
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if (lane == 0 && ncancel && ep.cancelled) atomicAdd(ep.cancelled, ncancel);
  }
  if (EPI == kEpiLoglik) {
    // one partial per basic bin (all its timing bins), reduced in a fixed order by the caller
    for (int o = 16; o > 0; o >>= 1) ll += __shfl_xor_sync(0xffffffffu, ll, o);
    if (lane == 0) ep.partials[bi] = ll;
  }
}

// sum of a voxel's contributions over the group's timing bins, then one addition to the image
struct TofFloatSum {
  float* img;
  using T = float;
  __device__ __forceinline__ T term(float v) const { return v; }
  __device__ __forceinline__ void flush(int64_t i, T v) const {
    if (v != 0.f) atomicAdd(img + i, v);
  }
};
// the group's contributions to a voxel summed in float in a fixed order (the timing bins of the group), the sum
// rounded once to the fixed-point grid (a power-of-two scale: exact) and added as a 64-bit integer
struct TofFixedSum {
  unsigned long long* acc;
  float scale;
  using T = float;
  __device__ __forceinline__ T term(float v) const { return v; }
  __device__ __forceinline__ void flush(int64_t i, T v) const {
    if (v != 0.f) atomicAdd(acc + i, static_cast<unsigned long long>(__float2ll_rn(v * scale)));
  }
};

template <int KG, typename Sum>
__device__ __forceinline__ void back_tof_grouped_body(const ProjParams& p, const ProjBinDev& pb, TofStage<KG>& S,
                                                      const float* __restrict__ pd, const Sum& out, int zero_ends,
                                                      int lane) {
  const RowElem* row = p.tof_basic_rows + pb.row_offset;
  const int K = p.num_tof;
  const float* wrow = p.tof_w + pb.row_offset * K;
  const int nax = packed_nax(p, pb);
  const bool blocked = nax > kPackedMaxNax;
  const int G = blocked ? 1 : min(32 / nax, kPackedMaxLines);
  const int gi = blocked ? 0 : lane / nax;
  for (int l0 = 0; l0 < pb.num_lines; l0 += G)
  for (int a0 = 0; a0 < (blocked ? nax : 1); a0 += 32) {
    const PackedLane t = tof_lane(p, pb, l0, G, nax, a0, lane);
    const int ng = min(G, pb.num_lines - l0);
    const int zoff = t.a * t.s.npa;
    const bool zend = zero_ends && t.L.seg == 0 && (t.a == 0 || t.a == t.s.nax - 1);
    for (int k0 = 0; k0 < K; k0 += KG) {
      float d[KG];
      bool any = false;
#pragma unroll
      for (int kk = 0; kk < KG; ++kk) {
        d[kk] = 0.f;
        if (t.act && !zend && k0 + kk < K)
          d[kk] = pd ? __ldg(pd + t.s.out_base + static_cast<int64_t>(k0 + kk) * p.tof_stride + t.a) : 1.f;
        any |= d[kk] != 0.f;
      }
      if (!__any_sync(0xffffffffu, any)) continue;
      for (int e0 = 0; e0 < pb.row_len; e0 += 32) {
        const int cnt = min(32, pb.row_len - e0);
        tof_stage_batch<KG>(p, pb, row, wrow, K, l0, ng, e0, cnt, k0, S, lane);
        if (any)
          for (int k = 0; k < cnt; ++k) {
            const int2 X = S.xs[gi][k];
            const int zz = X.y + zoff;
            if (zz < 0 || zz >= p.nz) continue;
            // zero bins and zero weights add 0: the same sum as the per-timing-bin back projection's terms
            typename Sum::T sum = 0;
#pragma unroll
            for (int q = 0; q < KG / 4; ++q) {
              const float4 w = S.w[k][q];
              sum += out.term(w.x * d[4 * q]);
              sum += out.term(w.y * d[4 * q + 1]);
              sum += out.term(w.z * d[4 * q + 2]);
              sum += out.term(w.w * d[4 * q + 3]);
            }
            out.flush(X.x + zz, sum);
          }
      }
    }
  }
}

template <int KG, typename Sum>
__global__ void __launch_bounds__(kTofWarps * 32, kTofMinCtas) back_tof_grouped_kernel(ProjParams p, const int* __restrict__ items,
                                                                         int nitems, const float* __restrict__ pd,
                                                                         Sum out, const double* __restrict__ scale,
                                                                         int zero_ends) {
  __shared__ TofStage<KG> stage[kTofWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bi = blockIdx.x * kTofWarps + warp;
  if (bi >= nitems) return;
  Sum o = out;
  if constexpr (std::is_same<Sum, TofFixedSum>::value) o.scale = static_cast<float>(*scale);
  back_tof_grouped_body<KG, Sum>(p, p.tof_basic[items[bi]], stage[warp], pd, o, zero_ends, lane);
}

// Batched packed kernels: a persistent grid whose warps take (frame, basic bin) items from the queue one at a time
// and project them as forward_packed_bin / back_packed_bin; each warp stages its item's frame, geometry and bin.
struct WarpStage {
  ProjParams p;
  BatchFrameDev f;
  ProjBinDev pb;
};

__device__ __forceinline__ bool next_item_warp(unsigned* counter, const BatchItem* __restrict__ items, int nitems,
                                               const ProjParams* __restrict__ geoms,
                                               const BatchFrameDev* __restrict__ frames, WarpStage& st, int lane,
                                               bool tof_basic = false) {
  __syncwarp();  // the warp has finished with the previous item
  int it = 0;
  if (lane == 0) it = static_cast<int>(atomicAdd(counter, 1u));
  it = __shfl_sync(0xffffffffu, it, 0);
  if (it >= nitems) return false;
  const BatchItem wi = items[it];
  const int g = frames[wi.frame].geom;
  constexpr int nf = sizeof(BatchFrameDev) / 4, np = sizeof(ProjParams) / 4, nb = sizeof(ProjBinDev) / 4;
  for (int t = lane; t < nf + np + nb; t += 32) {
    if (t < nf)
      reinterpret_cast<uint32_t*>(&st.f)[t] = reinterpret_cast<const uint32_t*>(frames + wi.frame)[t];
    else if (t < nf + np)
      reinterpret_cast<uint32_t*>(&st.p)[t - nf] = reinterpret_cast<const uint32_t*>(geoms + g)[t - nf];
    else
      reinterpret_cast<uint32_t*>(&st.pb)[t - nf - np] =
          reinterpret_cast<const uint32_t*>((tof_basic ? geoms[g].tof_basic : geoms[g].bins) + wi.bin)[t - nf - np];
  }
  __syncwarp();
  return true;
}

__global__ void __launch_bounds__(kPackedWarps * 32) forward_batch_packed_kernel(const ProjParams* __restrict__ geoms,
                                                                                const BatchFrameDev* __restrict__ frames,
                                                                                const BatchItem* __restrict__ items,
                                                                                int nitems, unsigned* counter) {
  __shared__ WarpStage wst[kPackedWarps];
  __shared__ PackedStage stage[kPackedWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpStage& st = wst[warp];
  while (next_item_warp(counter, items, nitems, geoms, frames, st, lane)) {
    double ll = 0.0;
    unsigned ncancel = 0;
    forward_packed_bin<kEpiRatio>(st.p, st.pb, stage[warp], st.f.x, st.f.ratio, st.f.ep, ll, ncancel, lane);
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if (lane == 0 && ncancel && st.f.ep.cancelled) atomicAdd(st.f.ep.cancelled, ncancel);
  }
}

__global__ void __launch_bounds__(kPackedWarps * 32) back_batch_packed_kernel(const ProjParams* __restrict__ geoms,
                                                                             const BatchFrameDev* __restrict__ frames,
                                                                             const BatchItem* __restrict__ items,
                                                                             int nitems, unsigned* counter) {
  __shared__ WarpStage wst[kPackedWarps];
  __shared__ PackedStage stage[kPackedWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpStage& st = wst[warp];
  while (next_item_warp(counter, items, nitems, geoms, frames, st, lane))
    back_packed_bin<FloatAcc>(st.p, st.pb, stage[warp], st.f.ratio, FloatAcc{st.f.u}, 0, lane);
}

// batched TOF-grouped kernels: items are (frame, basic bin) over the frames' TOF basic-bin tables
template <int KG>
__global__ void __launch_bounds__(kTofWarps * 32) forward_batch_tof_kernel(const ProjParams* __restrict__ geoms,
                                                                          const BatchFrameDev* __restrict__ frames,
                                                                          const BatchItem* __restrict__ items, int nitems,
                                                                          unsigned* counter) {
  __shared__ WarpStage wst[kTofWarps];
  __shared__ TofStage<KG> stage[kTofWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpStage& st = wst[warp];
  while (next_item_warp(counter, items, nitems, geoms, frames, st, lane, true)) {
    double ll = 0.0;
    unsigned ncancel = 0;
    forward_tof_grouped_body<KG, kEpiRatio>(st.p, st.pb, stage[warp], st.f.x, st.f.ratio, st.f.ep, ll, ncancel, lane);
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if (lane == 0 && ncancel && st.f.ep.cancelled) atomicAdd(st.f.ep.cancelled, ncancel);
  }
}

template <int KG>
__global__ void __launch_bounds__(kTofWarps * 32) back_batch_tof_kernel(const ProjParams* __restrict__ geoms,
                                                                       const BatchFrameDev* __restrict__ frames,
                                                                       const BatchItem* __restrict__ items, int nitems,
                                                                       unsigned* counter) {
  __shared__ WarpStage wst[kTofWarps];
  __shared__ TofStage<KG> stage[kTofWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpStage& st = wst[warp];
  while (next_item_warp(counter, items, nitems, geoms, frames, st, lane, true)) {
    back_tof_grouped_body<KG, TofFloatSum>(st.p, st.pb, stage[warp], st.f.ratio, TofFloatSum{st.f.u}, 0, lane);
    __syncwarp();
  }
}

static size_t proj_smem_bytes(const ProjParams& p) { return proj_smem_bytes(p.max_row_len); }

static cudaError_t prepare_smem(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  return cudaSuccess;
}

size_t projector_smem_bytes(const ProjParams& p) { return proj_smem_bytes(p); }

template <typename K, typename... A>
static cudaError_t launch_proj(K kernel, const ProjParams& p, int nbins, cudaStream_t st, A... args) {
  const size_t sm = proj_smem_bytes(p);
  cudaError_t e = prepare_smem(reinterpret_cast<const void*>(kernel), sm);
  if (e != cudaSuccess) return e;
  kernel<<<nbins, kThreads, sm, st>>>(p, args...);
  return cudaGetLastError();
}

template <int EPI>
static cudaError_t launch_forward_epi(const ProjParams& p, const int* list, int nbins, const float* image, float* out,
                                      const FwdEpilogue& ep, cudaStream_t st) {
  if (p.max_nax <= kPackedMaxNax) {
    forward_packed_kernel<EPI><<<(nbins + kPackedWarps - 1) / kPackedWarps, kPackedWarps * 32, 0, st>>>(
        p, list, nbins, image, out, ep);
    return cudaGetLastError();
  }
  switch (p.uniform_npa) {
    case 1: return launch_proj(forward_kernel<1, EPI>, p, nbins, st, list, image, out, ep);
    case 2: return launch_proj(forward_kernel<2, EPI>, p, nbins, st, list, image, out, ep);
    default: return launch_proj(forward_kernel<0, EPI>, p, nbins, st, list, image, out, ep);
  }
}

cudaError_t launch_forward(const ProjParams& p, const int* bin_list, int nbins, const float* image, float* projdata,
                           cudaStream_t st, const FwdEpilogue* ep) {
  if (nbins <= 0) return cudaSuccess;
  FwdEpilogue none{};
  if (!ep || ep->mode == kEpiNone) return launch_forward_epi<kEpiNone>(p, bin_list, nbins, image, projdata, none, st);
  if (ep->mode == kEpiRatio) return launch_forward_epi<kEpiRatio>(p, bin_list, nbins, image, projdata, *ep, st);
  if (ep->mode == kEpiGradient) return launch_forward_epi<kEpiGradient>(p, bin_list, nbins, image, projdata, *ep, st);
  return launch_forward_epi<kEpiLoglik>(p, bin_list, nbins, image, projdata, *ep, st);
}

template <typename Acc>
static cudaError_t launch_back_acc(const ProjParams& p, const int* bin_list, int nbins, const float* projdata, Acc acc,
                                   cudaStream_t st, int zero_ends) {
  if (nbins <= 0) return cudaSuccess;
  if (p.max_nax <= kPackedMaxNax) {
    back_packed_kernel<Acc><<<(nbins + kPackedWarps - 1) / kPackedWarps, kPackedWarps * 32, 0, st>>>(
        p, bin_list, nbins, projdata, acc, zero_ends);
    return cudaGetLastError();
  }
  switch (p.uniform_npa) {
    case 1: return launch_proj(back_atomic_kernel<1, Acc>, p, nbins, st, bin_list, projdata, acc, zero_ends);
    case 2: return launch_proj(back_atomic_kernel<2, Acc>, p, nbins, st, bin_list, projdata, acc, zero_ends);
    default: return launch_proj(back_atomic_kernel<0, Acc>, p, nbins, st, bin_list, projdata, acc, zero_ends);
  }
}

cudaError_t launch_back_atomic(const ProjParams& p, const int* bin_list, int nbins, const float* projdata, float* image,
                               cudaStream_t st, int zero_ends) {
  return launch_back_acc(p, bin_list, nbins, projdata, FloatAcc{image}, st, zero_ends);
}

cudaError_t launch_back_fixed(const ProjParams& p, const int* bin_list, int nbins, const float* projdata,
                              unsigned long long* acc, const double* scale, cudaStream_t st, int zero_ends) {
  return launch_back_acc(p, bin_list, nbins, projdata, FixedAcc{acc, scale}, st, zero_ends);
}

cudaError_t launch_forward_batch(const ProjParams* geoms, int npa, size_t smem_bytes, const BatchFrameDev* frames,
                                 const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  const void* fn = npa == 1 ? reinterpret_cast<const void*>(forward_batch_kernel<1>)
                 : npa == 2 ? reinterpret_cast<const void*>(forward_batch_kernel<2>)
                            : reinterpret_cast<const void*>(forward_batch_kernel<0>);
  cudaError_t e = prepare_smem(fn, smem_bytes);
  if (e != cudaSuccess) return e;
  if (npa == 1)
    forward_batch_kernel<1><<<grid, kThreads, smem_bytes, st>>>(geoms, frames, items, nitems, counter);
  else if (npa == 2)
    forward_batch_kernel<2><<<grid, kThreads, smem_bytes, st>>>(geoms, frames, items, nitems, counter);
  else
    forward_batch_kernel<0><<<grid, kThreads, smem_bytes, st>>>(geoms, frames, items, nitems, counter);
  return cudaGetLastError();
}

cudaError_t launch_back_batch(const ProjParams* geoms, int npa, size_t smem_bytes, const BatchFrameDev* frames,
                              const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  const void* fn = npa == 1 ? reinterpret_cast<const void*>(back_batch_kernel<1>)
                 : npa == 2 ? reinterpret_cast<const void*>(back_batch_kernel<2>)
                            : reinterpret_cast<const void*>(back_batch_kernel<0>);
  cudaError_t e = prepare_smem(fn, smem_bytes);
  if (e != cudaSuccess) return e;
  if (npa == 1)
    back_batch_kernel<1><<<grid, kThreads, smem_bytes, st>>>(geoms, frames, items, nitems, counter);
  else if (npa == 2)
    back_batch_kernel<2><<<grid, kThreads, smem_bytes, st>>>(geoms, frames, items, nitems, counter);
  else
    back_batch_kernel<0><<<grid, kThreads, smem_bytes, st>>>(geoms, frames, items, nitems, counter);
  return cudaGetLastError();
}

cudaError_t launch_forward_batch_packed(const ProjParams* geoms, const BatchFrameDev* frames, const BatchItem* items,
                                        int nitems, unsigned* counter, int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  forward_batch_packed_kernel<<<grid, kPackedWarps * 32, 0, st>>>(geoms, frames, items, nitems, counter);
  return cudaGetLastError();
}

cudaError_t launch_back_batch_packed(const ProjParams* geoms, const BatchFrameDev* frames, const BatchItem* items,
                                     int nitems, unsigned* counter, int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  back_batch_packed_kernel<<<grid, kPackedWarps * 32, 0, st>>>(geoms, frames, items, nitems, counter);
  return cudaGetLastError();
}

int batch_packed_max_ctas_per_sm(bool forward) {
  const void* fn = forward ? reinterpret_cast<const void*>(forward_batch_packed_kernel)
                           : reinterpret_cast<const void*>(back_batch_packed_kernel);
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kPackedWarps * 32, 0) != cudaSuccess) return 0;
  return n;
}

// timing bins per pass: the fewest passes of at most 32 bins, spread evenly, rounded up to an instantiated size
int tof_group_size(int K) {
  const int passes = (K + kTofGroupMax - 1) / kTofGroupMax;
  const int per = (K + passes - 1) / passes;
  return per <= 8 ? 8 : per <= 16 ? 16 : per <= 20 ? 20 : per <= 24 ? 24 : 32;
}

#define TOF_KG_SWITCH(K, CALL)                       \
  switch (tof_group_size(K)) {                       \
    case 8: { constexpr int KG = 8; CALL; break; }   \
    case 16: { constexpr int KG = 16; CALL; break; } \
    case 20: { constexpr int KG = 20; CALL; break; } \
    case 24: { constexpr int KG = 24; CALL; break; } \
    default: { constexpr int KG = 32; CALL; break; } \
  }

cudaError_t launch_forward_tof_grouped(const ProjParams& p, const int* items, int nitems, const float* image,
                                       float* projdata, cudaStream_t st, const FwdEpilogue* ep) {
  if (nitems <= 0) return cudaSuccess;
  const int grid = (nitems + kTofWarps - 1) / kTofWarps;
  FwdEpilogue none{};
  if (!ep || ep->mode == kEpiNone) {
    TOF_KG_SWITCH(p.num_tof, (forward_tof_grouped_kernel<KG, kEpiNone><<<grid, kTofWarps * 32, 0, st>>>(
                                 p, items, nitems, image, projdata, none)));
  } else if (ep->mode == kEpiRatio) {
    TOF_KG_SWITCH(p.num_tof, (forward_tof_grouped_kernel<KG, kEpiRatio><<<grid, kTofWarps * 32, 0, st>>>(
                                 p, items, nitems, image, projdata, *ep)));
  } else if (ep->mode == kEpiGradient) {
    TOF_KG_SWITCH(p.num_tof, (forward_tof_grouped_kernel<KG, kEpiGradient><<<grid, kTofWarps * 32, 0, st>>>(
                                 p, items, nitems, image, projdata, *ep)));
  } else {
    TOF_KG_SWITCH(p.num_tof, (forward_tof_grouped_kernel<KG, kEpiLoglik><<<grid, kTofWarps * 32, 0, st>>>(
                                 p, items, nitems, image, projdata, *ep)));
  }
  return cudaGetLastError();
}

cudaError_t launch_back_tof_grouped(const ProjParams& p, const int* items, int nitems, const float* projdata,
                                    float* image, unsigned long long* acc, const double* scale, cudaStream_t st,
                                    int zero_ends) {
  if (nitems <= 0) return cudaSuccess;
  const int grid = (nitems + kTofWarps - 1) / kTofWarps;
  if (acc) {
    TOF_KG_SWITCH(p.num_tof, (back_tof_grouped_kernel<KG, TofFixedSum><<<grid, kTofWarps * 32, 0, st>>>(
                                 p, items, nitems, projdata, TofFixedSum{acc, 0.f}, scale, zero_ends)));
  } else {
    TOF_KG_SWITCH(p.num_tof, (back_tof_grouped_kernel<KG, TofFloatSum><<<grid, kTofWarps * 32, 0, st>>>(
                                 p, items, nitems, projdata, TofFloatSum{image}, scale, zero_ends)));
  }
  return cudaGetLastError();
}

cudaError_t launch_forward_batch_tof(const ProjParams* geoms, int num_tof, const BatchFrameDev* frames,
                                     const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  TOF_KG_SWITCH(num_tof, (forward_batch_tof_kernel<KG><<<grid, kTofWarps * 32, 0, st>>>(geoms, frames, items, nitems,
                                                                                        counter)));
  return cudaGetLastError();
}

cudaError_t launch_back_batch_tof(const ProjParams* geoms, int num_tof, const BatchFrameDev* frames,
                                  const BatchItem* items, int nitems, unsigned* counter, int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  TOF_KG_SWITCH(num_tof, (back_batch_tof_kernel<KG><<<grid, kTofWarps * 32, 0, st>>>(geoms, frames, items, nitems,
                                                                                     counter)));
  return cudaGetLastError();
}

int batch_tof_max_ctas_per_sm(int num_tof, bool forward) {
  const void* fn = nullptr;
  TOF_KG_SWITCH(num_tof, (fn = forward ? reinterpret_cast<const void*>(forward_batch_tof_kernel<KG>)
                                       : reinterpret_cast<const void*>(back_batch_tof_kernel<KG>)));
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kTofWarps * 32, 0) != cudaSuccess) return 0;
  return n;
}

int batch_max_ctas_per_sm(int npa, size_t smem_bytes, bool forward) {
  const void* fn;
  if (forward)
    fn = npa == 1 ? reinterpret_cast<const void*>(forward_batch_kernel<1>)
       : npa == 2 ? reinterpret_cast<const void*>(forward_batch_kernel<2>)
                  : reinterpret_cast<const void*>(forward_batch_kernel<0>);
  else
    fn = npa == 1 ? reinterpret_cast<const void*>(back_batch_kernel<1>)
       : npa == 2 ? reinterpret_cast<const void*>(back_batch_kernel<2>)
                  : reinterpret_cast<const void*>(back_batch_kernel<0>);
  if (prepare_smem(fn, smem_bytes) != cudaSuccess) return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kThreads, smem_bytes) != cudaSuccess) return 0;
  return n;
}

cudaError_t launch_image_to_dev(const float* stir, float* dev, int nz, int ny, int nx, cudaStream_t st) {
  return transpose(stir, dev, nz, static_cast<int64_t>(ny) * nx, st);
}
cudaError_t launch_image_from_dev(const float* dev, float* stir, int nz, int ny, int nx, cudaStream_t st) {
  return transpose(dev, stir, ny * nx, nz, st);  // dev is (ny*nx) x nz
}
cudaError_t launch_projdata_to_dev(const float* stir, float* dev, int nax, int64_t nvt, cudaStream_t st) {
  return transpose(stir, dev, nax, nvt, st);
}
cudaError_t launch_projdata_from_dev(const float* dev, float* stir, int nax, int64_t nvt, cudaStream_t st) {
  return transpose(dev, stir, static_cast<int>(nvt), nax, st);
}

cudaError_t launch_projdata_layout_views(const float* in, float* out, const int64_t* tab, int nsegs, int ntof,
                                         int max_nax, int64_t tof_stride, int64_t nvt, int64_t c0, int64_t nc,
                                         bool to_dev, cudaStream_t st) {
  if (nc <= 0 || nsegs <= 0 || ntof <= 0 || max_nax <= 0) return cudaSuccess;
  // the grid covers the segment with the most axial positions; tiles past a smaller segment's extent return at once
  const int64_t rows = to_dev ? max_nax : nc, cols = to_dev ? nc : max_nax;
  const int64_t gx = (cols + 31) / 32, gy = (rows + 31) / 32;
  const int64_t gz = static_cast<int64_t>(nsegs) * ntof;
  if (gy > 65535 || gz > 65535 || gx > 2147483647LL) return cudaErrorInvalidValue;
  projdata_layout_kernel<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(gy), static_cast<unsigned>(gz)),
                           dim3(32, 8), 0, st>>>(in, out, tab, nsegs, tof_stride, nvt, c0, nc, to_dev ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_transpose(const float* in, float* out, int rows, int64_t cols, int64_t ld_in, int64_t ld_out,
                             cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  const int64_t gx = (cols + 31) / 32;
  const int64_t gy = (rows + 31) / 32;
  if (gy > 65535 || gx > 2147483647LL) return cudaErrorInvalidValue;
  transpose_kernel<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(gy)), dim3(32, 8), 0, st>>>(in, out, rows,
                                                                                                      cols, ld_in, ld_out);
  return cudaGetLastError();
}

}  // namespace b200
