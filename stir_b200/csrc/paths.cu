// Column-staged forward and back projection.
//
// All basic bins with the same basic view and tangential position -- one per segment -- trace the same
// transaxial path (the x/y crossings of STIR's Siddon tracer, RayTraceVoxelsOnCartesianGrid.cxx:51-269,
// do not depend on the ring difference), so their rows cross the same voxel columns (x, y) at different
// z.  A path item is such a path with one transaxial symmetry operation T (swap x/y, negate x, negate y;
// SymmetryOperations_PET_CartesianGrid.h:48-482): its lines are the related lines of every segment
// (both z orientations) that use T.  One CTA per item, over chunks of K columns of the path:
//
//   forward: the image columns T(x, y) -- all nz planes, contiguous in the [y][x][z] layout -- are copied
//     to shared memory (one L2 read per column and item instead of one per line and row element); every
//     (line, part) unit, one warp each, walks the part of its row in the chunk (rows are stored sorted by
//     path slot, then z) with its lanes on the axial positions, as the per-basic-bin kernel does but
//     gathering from shared memory; the parts of a line are added in a fixed order and go through the
//     same epilogue as the per-basic-bin kernel;
//   back: a warp owns a column and its lanes the planes z; it sums, in registers, the contributions of
//     every line of the item to its voxels and adds them to the image once (a gather instead of a
//     scatter: no shared-memory atomics, and a fixed order within the item).
//
// Sums are taken in path order rather than in the stored row order of ProjMatrixElemsForOneBin, so the
// results differ from the per-basic-bin kernels by float rounding only.  The fixed-point back projection sums
// each item's contributions to a voxel in float in a fixed order and adds the rounded sums as integers, so its
// image does not depend on the order of the items (the per-basic-bin kernels round every contribution instead).
#include "internal.hpp"
#include "epilogue.cuh"

namespace b200 {

namespace {

constexpr int kPathWarps = 8;
constexpr int kPathThreads = kPathWarps * 32;
constexpr int kPathMinCtas = 4;      // forward: shared memory allows 4 CTAs per SM on the clinical geometry
constexpr int kPathMinCtasBack = 5;  // back projection: 5 measured fastest (4: +4 %, 6: +21 % with spills)
static_assert(kPathWarps == kPathWarpsH, "shared-memory layout and kernels agree on the warps per CTA");

// line set-up of the item's lines (one thread per line)
__device__ __forceinline__ void setup_path_lines(const ProjParams& p, const PathParams& pp, const PathItemDev& it,
                                                 PathLineSmem* ls) {
  for (int l = threadIdx.x; l < it.num_lines; l += blockDim.x) {
    const PathLineDev pl = pp.lines[it.first_line + l];
    const LineDev L = p.lines[pl.line];
    const ProjBinDev pb = p.bins[pl.bin];
    PathLineSmem s{};
    const int tang = static_cast<int>(L.tang_sign) * pb.tang;
    // the line's view in the data's layout: a view shard holds some views only, the others' lines are inactive
    const int slot = p.view_slot ? __ldg(p.view_slot + L.view) : L.view;
    s.active = tang >= p.min_tang && tang <= p.max_tang && slot >= 0;
    const SegDev sd = p.segs[L.seg + p.S];
    s.nax = sd.nax;
    s.npa = sd.npa;
    s.tofi = pb.tof - p.min_tof;
    s.out_base = static_cast<int64_t>(s.tofi) * p.tof_stride + sd.dev_offset +
                 (static_cast<int64_t>(max(slot, 0)) * p.num_tang + (tang - p.min_tang)) * sd.nax;
    s.elem_off = pl.elem_off;
    s.chunk_off = pl.chunk_off;
    // z index in the image of element z (stored as z + 512): zq ? q - z : z, minus min_z
    if (L.flags & 8) {
      s.zsign = -1;
      s.zadd = static_cast<int>(L.q) + 512 - p.min_z;
    } else {
      s.zsign = 1;
      s.zadd = -512 - p.min_z;
    }
    s.seg = L.seg;
    s.view = L.view;
    s.member = pl.member;
    ls[l] = s;
  }
}

// image offset of path column `col` under the item's symmetry operation (-1 outside the image)
__device__ __forceinline__ int column_image_offset(const ProjParams& p, const PathParams& pp, const PathItemDev& it,
                                                   int col) {
  const int swap = it.flags & 1;
  const int sx = (it.flags & 2) ? -1 : 1;
  const int sy = (it.flags & 4) ? -1 : 1;
  const uint32_t pk = __ldg(pp.cols + it.col_offset + col);
  const int x = static_cast<int>(pk & 2047u) - 1024;
  const int y = static_cast<int>((pk >> 11) & 2047u) - 1024;
  const int xi = (swap ? y : x) * sx - p.min_x;
  const int yi = (swap ? x : y) * sy - p.min_y;
  return (xi >= 0 && xi < p.nx && yi >= 0 && yi < p.ny) ? (yi * p.nx + xi) * p.nz : -1;
}

// image offsets of the chunk's columns (-1 outside the image)
__device__ __forceinline__ void chunk_columns(const ProjParams& p, const PathParams& pp, const PathItemDev& it, int c0,
                                              int kc, int* colbase) {
  for (int i = threadIdx.x; i < kc; i += blockDim.x) colbase[i] = column_image_offset(p, pp, it, c0 + i);
}

// the element range of unit (line, part) in chunk c; P = 1 << lgP parts
__device__ __forceinline__ void unit_range(const PathParams& pp, const PathLineSmem& L, int c, int part, int lgP, int& e0,
                                           int& e1) {
  const int lo = __ldg(pp.chunks + L.chunk_off + c);
  const int n = __ldg(pp.chunks + L.chunk_off + c + 1) - lo;
  e0 = lo + ((n * part) >> lgP);
  e1 = lo + ((n * (part + 1)) >> lgP);
}

__device__ __forceinline__ int log2_parts(int P) { return P == 2 ? 1 : (P == 4 ? 2 : 3); }

// a * b + c on two float lanes at once (sm_100's packed FP32 FMA): each lane rounds as fmaf does
__device__ __forceinline__ void fma2(float& c0, float& c1, float a0, float a1, float b0, float b1) {
  unsigned long long r;
  const unsigned long long a = (static_cast<unsigned long long>(__float_as_uint(a1)) << 32) | __float_as_uint(a0);
  const unsigned long long b = (static_cast<unsigned long long>(__float_as_uint(b1)) << 32) | __float_as_uint(b0);
  const unsigned long long c = (static_cast<unsigned long long>(__float_as_uint(c1)) << 32) | __float_as_uint(c0);
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  c0 = __uint_as_float(static_cast<unsigned>(r));
  c1 = __uint_as_float(static_cast<unsigned>(r >> 32));
}

// 4-byte asynchronous copy global -> shared (completed by cp_async_wait)
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---- bulk staging: one cp.async.bulk (the TMA unit's 1-D copy) per image column, completed on an mbarrier ----
// Source and destination are this GPU's memory only (the image and the CTA's shared memory); no multicast.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n .reg .b64 state;\n mbarrier.arrive.shared::cta.b64 state, [%0];\n}\n" ::"r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Waits for the phase with the given parity to complete, at most kStageWaitLimit polls (each poll may itself
// suspend the thread for a while); false when the limit ran out.
constexpr int kStageWaitLimit = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  for (int i = 0; i < kStageWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_copy_to_smem(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// orders this thread's earlier generic-proxy accesses to shared memory before later async-proxy (bulk copy) ones
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// one packed element of the padded path: staged indices (16-bit, signed) of axial position 0 for both lines
template <int NJ, bool TWO>
__device__ __forceinline__ void padded_fma(const float* cols, uint32_t idx, float v, int zo0, int npa, float* acc1,
                                           float* acc2) {
  const float* q1 = cols + (static_cast<int>(static_cast<int16_t>(idx & 0xffffu)) + zo0);
  const float* q2 = cols + ((static_cast<int>(idx) >> 16) + zo0);
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    if (TWO)
      fma2(acc1[j], acc2[j], q1[j * 32 * npa], q2[j * 32 * npa], v, v);  // both lines' sums in one instruction
    else
      acc1[j] += q1[j * 32 * npa] * v;
  }
}

// One pass of one unit over elements [e0, e1) of its row: NJ groups of 32 axial positions from a0.
// The warp's lanes transform 32 elements at a time (column slot -> staged index, z reflection) into
// the warp's buffer; then every element costs one broadcast read and NJ shared loads and FMAs.
// colstart: with padded staging, the staged index of plane 0 of each column of the chunk.
template <int NPA, int NJ, bool TWO, bool PADDED>
__device__ __forceinline__ void gather_pass(const PathElem* __restrict__ E, int e0, int e1, int c0, const float* cols,
                                            const int* colstart, int nz, int cstride, int coff,
                                            const PathLineSmem& L1,
                                            const PathLineSmem& L2, int a0, int nact, int lane, float* acc_row1,
                                            float* acc_row2, PathXElem* xb) {
  const int npa = NPA ? NPA : L1.npa;
  // lane's plane offset of group j: zo0 + 32 j npa.  In the full path inactive lanes (axial positions past
  // the line's end) read up to 127 npa floats past the staged columns, into the padding of the staging
  // buffer, and their sums are dropped: the full path needs no per-lane tests.
  const int zo0 = (a0 + lane) * npa;
  bool act[NJ];
  float acc1[NJ], acc2[NJ];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    act[j] = j * 32 + lane < nact;
    acc1[j] = act[j] ? acc_row1[a0 + j * 32 + lane] : 0.f;
    acc2[j] = (TWO && act[j]) ? acc_row2[a0 + j * 32 + lane] : 0.f;
  }
  const int zlo = a0 * npa, zhi = (a0 + nact - 1) * npa;
  // padded staging: every read stays inside the staging buffer (fewer than 2^14 floats), so the two staged
  // indices fit 16 bits each and an element is 8 bytes; one 16-byte broadcast read serves two elements
  uint2* xp = reinterpret_cast<uint2*>(xb);
  for (int k0 = e0; k0 < e1; k0 += 32) {
    const int cnt = min(32, e1 - k0);
    __syncwarp();
    if (lane < cnt) {
      // x = (staged index of axial position 0 for line 1, for line 2, value, column slot | full flags)
      const PathElem m = E[k0 + lane];
      const int zr = static_cast<int>(m.sz >> 16);
      const int sl = static_cast<int>(m.sz & 0xffffu) - c0;
      const int zt1 = L1.zsign * zr + L1.zadd;
      const int zt2 = TWO ? L2.zsign * zr + L2.zadd : 0;
      if (PADDED) {
        const int s0 = colstart[sl];
        const int b1 = s0 + zt1, b2 = TWO ? s0 + zt2 : 0;
        xp[lane] = make_uint2((static_cast<uint32_t>(b1) & 0xffffu) | (static_cast<uint32_t>(b2) << 16),
                              __float_as_uint(m.v));
      } else {
        const int f1 = (zt1 + zlo >= 0) && (zt1 + zhi < nz);
        const int f2 = TWO ? ((zt2 + zlo >= 0) && (zt2 + zhi < nz)) : 1;
        PathXElem x;
        x.base = sl * cstride + coff + zt1;
        x.zt = sl * cstride + coff + zt2;
        x.v = m.v;
        x.full = sl | ((f1 & f2) << 30);
        xb[lane] = x;
      }
    }
    __syncwarp();
    if constexpr (PADDED) {
      const uint4* xq = reinterpret_cast<const uint4*>(xb);
      int i = 0;
      for (; i + 1 < cnt; i += 2) {
        const uint4 w = xq[i >> 1];
        padded_fma<NJ, TWO>(cols, w.x, __uint_as_float(w.y), zo0, npa, acc1, acc2);
        padded_fma<NJ, TWO>(cols, w.z, __uint_as_float(w.w), zo0, npa, acc1, acc2);
      }
      if (i < cnt) {
        const uint2 w = xp[i];
        padded_fma<NJ, TWO>(cols, w.x, __uint_as_float(w.y), zo0, npa, acc1, acc2);
      }
    } else {
      for (int i = 0; i < cnt; ++i) {
        const PathXElem e = xb[i];
        const float* q1 = cols + (e.base + zo0);
        const float* q2 = cols + (e.zt + zo0);
        if (e.full >> 30) {
#pragma unroll
          for (int j = 0; j < NJ; ++j) {
            acc1[j] += q1[j * 32 * npa] * e.v;
            if (TWO) acc2[j] += q2[j * 32 * npa] * e.v;
          }
        } else {
          const int sb = (e.full & 0xffff) * cstride + coff;  // column start in the staging buffer
#pragma unroll
          for (int j = 0; j < NJ; ++j) {
            const int zz1 = e.base - sb + zo0 + j * 32 * npa;
            if (act[j] && static_cast<unsigned>(zz1) < static_cast<unsigned>(nz)) acc1[j] += q1[j * 32 * npa] * e.v;
            if (TWO) {
              const int zz2 = e.zt - sb + zo0 + j * 32 * npa;
              if (act[j] && static_cast<unsigned>(zz2) < static_cast<unsigned>(nz)) acc2[j] += q2[j * 32 * npa] * e.v;
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j)
    if (act[j]) {
      acc_row1[a0 + j * 32 + lane] = acc1[j];
      if (TWO) acc_row2[a0 + j * 32 + lane] = acc2[j];
    }
}

// the lines of an item processed together: consecutive active lines of one basic bin (its two z
// orientations), in pairs, and the remaining active lines alone (thread 0; lines of a bin are consecutive)
__device__ __forceinline__ int pair_lines(const PathLineSmem* ls, int nl, int2* pairs) {
  int n = 0;
  for (int l = 0; l < nl; ++l) {
    if (!ls[l].active) continue;
    if (l + 1 < nl && ls[l + 1].active && ls[l + 1].member == ls[l].member && ls[l + 1].nax == ls[l].nax &&
        ls[l + 1].npa == ls[l].npa) {
      pairs[n++] = make_int2(l, l + 1);
      ++l;
    } else {
      pairs[n++] = make_int2(l, -1);
    }
  }
  return n;
}

// one gather pass, with the padded staging or with per-lane range tests
#define GATHER(NJ, TWO, LA, LB, ...)                                                                             \
  (pp.zpad >= 0                                                                                                  \
       ? gather_pass<NPA, NJ, TWO, true>(E, e0, e1, c0, cols, colbase, nz, cstride, coff, LA, LB, __VA_ARGS__)    \
       : gather_pass<NPA, NJ, TWO, false>(E, e0, e1, c0, cols, colbase, nz, cstride, coff, LA, LB, __VA_ARGS__))

// One path item.  With padded staging the columns are copied by bulk copies completed on `bar` (initialised for an
// arrival by every thread of the CTA; phase parity `phase`, flipped once per chunk); false when a copy was not seen
// to complete within the wait limit: the item is then abandoned (no output written) and the projector's status
// word records it.
template <int NPA, int EPI>
__device__ __forceinline__ bool forward_path_item(const ProjParams& p, const PathParams& pp, const PathItemDev& it,
                                                  unsigned char* smem, const float* __restrict__ img,
                                                  float* __restrict__ out, const FwdEpilogue& ep, double& ll,
                                                  unsigned& ncancel, uint64_t* bar, unsigned& phase) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nz = p.nz;
  const PathSmemFwd lay = path_smem_fwd(pp.K, nz, pp.zpad, pp.max_lines, pp.max_acc, pp.npa_max);
  const int cstride = path_col_stride(nz, pp.zpad), coff = path_col_offset(pp.zpad);
  float* cols = reinterpret_cast<float*>(smem);
  int* colbase = reinterpret_cast<int*>(smem + lay.colbase);
  PathLineSmem* ls = reinterpret_cast<PathLineSmem*>(smem + lay.lines);
  int2* pairs = reinterpret_cast<int2*>(smem + lay.pairs);
  int* rowoff = reinterpret_cast<int*>(smem + lay.rowoff);
  PathXElem* xb = reinterpret_cast<PathXElem*>(smem + lay.xbuf) + warp * 32;
  float* lacc = reinterpret_cast<float*>(smem + lay.acc);
  __shared__ int s_npairs, s_nacc;
  const int nl = it.num_lines;
  // units: (pair of lines, part of the elements); the accumulators are per (line, part): nax floats each
  const int P = path_parts(nl), lgP = log2_parts(P);
  setup_path_lines(p, pp, it, ls);
  __syncthreads();
  if (threadIdx.x == 0) {
    s_npairs = pair_lines(ls, nl, pairs);
    int o = 0;
    for (int l = 0; l < nl; ++l) {
      rowoff[l] = o;
      o += P * ls[l].nax;
    }
    s_nacc = o;
  }
  __syncthreads();
  const int U = s_npairs * P;
  for (int i = threadIdx.x; i < s_nacc; i += blockDim.x) lacc[i] = 0.f;
  // the staging buffer starts as zeros: with padded staging the planes between the columns stay zero
  if (pp.zpad > 0)
    for (int i = threadIdx.x; i < lay.colbase / 4; i += blockDim.x) cols[i] = 0.f;
  const bool bulk = pp.zpad >= 0;
  const int nch = (it.ncols + pp.K - 1) / pp.K;
  for (int c = 0; c < nch; ++c) {
    const int c0 = c * pp.K, kc = min(pp.K, it.ncols - c0);
    // every thread's generic accesses to the staging buffer (the previous chunk's reads, the zeroing) come before
    // the bulk copies that any thread issues after the barrier
    if (bulk) fence_proxy_async_smem();
    __syncthreads();  // previous chunk done (and the zeroing visible)
    if (bulk) {
      // Thread t owns columns t, t + blockDim.x, ...: one bulk copy each, of the whole 16-byte blocks that hold its
      // nz planes, to its slot's 16-byte boundary, so plane 0 lands at the column's phase (its address mod 16, in
      // floats), which colbase[ci] records as the column's staged start; a column outside the image is zeroed
      // instead.  Every thread then arrives on the barrier (after its byte counts), so the phase completes when all
      // the chunk's copies have landed.
      const int ext = (nz + 6) & ~3;  // a slot's copies reach at most round_up4(nz + 3) floats from its start
      for (int ci = threadIdx.x; ci < kc; ci += blockDim.x) {
        const int b = column_image_offset(p, pp, it, c0 + ci);
        const int d = ci * cstride + coff;
        float* slot = cols + d;
        int start = d;
        if (b >= 0) {
          const float* src = img + b;
          const int ph = static_cast<int>((reinterpret_cast<uintptr_t>(src) >> 2) & 3u);
          const unsigned bytes = static_cast<unsigned>((ph + nz + 3) & ~3) * 4u;
          mbar_expect_tx(bar, bytes);
          bulk_copy_to_smem(slot, src - ph, bytes, bar);
          start += ph;
        } else {
          for (int z = 0; z < ext; ++z) slot[z] = 0.f;
        }
        colbase[ci] = start;
      }
      mbar_arrive(bar);
      const bool done = mbar_wait_bounded(bar, phase);
      if (done) {
        // the owner puts back to zeros everything of its slots' [0, ext) that is not this chunk's column (the
        // neighbouring planes copied with the blocks, and what an earlier chunk's column with another phase left
        // there): at most 3 planes below plane 0, 6 above nz - 1
        for (int ci = threadIdx.x; ci < kc; ci += blockDim.x) {
          const int d = ci * cstride + coff, ph = colbase[ci] - d;
          for (int k = 0; k < ph; ++k) cols[d + k] = 0.f;
          for (int z = ph + nz; z < ext; ++z) cols[d + z] = 0.f;
        }
      }
      if (!__syncthreads_and(done)) {
        // not seen to complete: record it, give the copies in flight one more bounded wait, abandon the item
        if (threadIdx.x == 0 && pp.status) atomicOr(pp.status, 1u);
        mbar_wait_bounded(bar, phase);
        return false;
      }
      phase ^= 1u;
      // every column and its zeros are visible (the barrier above): the gather follows
    } else {
      chunk_columns(p, pp, it, c0, kc, colbase);
      __syncthreads();
      for (int ci = warp; ci < kc; ci += kPathWarps) {
        const int b = colbase[ci];
        float* dst = cols + ci * cstride + coff;
        if (b >= 0) {
          for (int z = lane; z < nz; z += 32) cp_async4(dst + z, img + b + z);
        } else {
          for (int z = lane; z < nz; z += 32) dst[z] = 0.f;
        }
      }
      cp_async_wait();
      __syncthreads();
    }
    for (int u = warp; u < U; u += kPathWarps) {
      const int pr = u >> lgP, part = u & (P - 1);
      const int2 pl = pairs[pr];
      const PathLineSmem L1 = ls[pl.x];
      int e0, e1;
      unit_range(pp, L1, c, part, lgP, e0, e1);
      if (e0 >= e1) continue;
      const PathElem* E = pp.elems + L1.elem_off;
      float* row1 = lacc + rowoff[pl.x] + part * L1.nax;
      if (pl.y >= 0) {
        const PathLineSmem L2 = ls[pl.y];
        float* row2 = lacc + rowoff[pl.y] + part * L2.nax;
        for (int a0 = 0; a0 < L1.nax; a0 += 128) {
          const int nact = min(L1.nax - a0, 128);
          switch ((nact + 31) >> 5) {
            case 1: GATHER(1, true, L1, L2, a0, nact, lane, row1, row2, xb); break;
            case 2: GATHER(2, true, L1, L2, a0, nact, lane, row1, row2, xb); break;
            case 3: GATHER(3, true, L1, L2, a0, nact, lane, row1, row2, xb); break;
            default: GATHER(4, true, L1, L2, a0, nact, lane, row1, row2, xb); break;
          }
        }
      } else {
        for (int a0 = 0; a0 < L1.nax; a0 += 128) {
          const int nact = min(L1.nax - a0, 128);
          switch ((nact + 31) >> 5) {
            case 1: GATHER(1, false, L1, L1, a0, nact, lane, row1, row1, xb); break;
            case 2: GATHER(2, false, L1, L1, a0, nact, lane, row1, row1, xb); break;
            case 3: GATHER(3, false, L1, L1, a0, nact, lane, row1, row1, xb); break;
            default: GATHER(4, false, L1, L1, a0, nact, lane, row1, row1, xb); break;
          }
        }
      }
    }
  }
  __syncthreads();
  // the parts of each line, added in order, through the epilogue
  for (int l = warp; l < nl; l += kPathWarps) {
    const PathLineSmem L = ls[l];
    if (!L.active) continue;
    for (int a = lane; a < L.nax; a += 32) {
      float v = 0.f;
      for (int q = 0; q < P; ++q) v += lacc[rowoff[l] + q * L.nax + a];
      forward_store<EPI>(p, L.seg, L.view, L.tofi, L.nax, L.out_base + a, a, v, out, ep, ll, ncancel);
    }
  }
  return true;
}

// Back projection as a gather over the voxels of each column: image[col][z] += the sum, over the path's
// elements e in the column and the item's lines l of e's basic bin, of w_e * d_l[a] with z = zt + npa a.
// A warp owns a column at a time (the path's elements are also stored in column order) and its lanes the
// planes z; the sums stay in registers (no shared-memory atomics, a fixed order within the item) and
// are added to the image once per column and item.  Each line's data is kept in shared memory padded
// with zeros, so that every lane reads d at F + z - zt without range tests.
struct FloatCols {
  using T = float;
  float* img;
  __device__ __forceinline__ void load() {}
  __device__ __forceinline__ void offset(int64_t o) { img += o; }
  __device__ __forceinline__ T term(float v) const { return v; }
  __device__ __forceinline__ void flush(int64_t i, float v) const {
    if (v != 0.f) atomicAdd(img + i, v);
  }
};
struct FixedCols {
  using T = float;
  unsigned long long* acc;
  const double* scale_ptr;  // 2^k of the fixed-point format, computed on the device
  double scale;
  float scale_f;  // the same power of two as a float
  __device__ __forceinline__ void load() {
    scale = *scale_ptr;
    scale_f = static_cast<float>(scale);
  }
  __device__ __forceinline__ void offset(int64_t) {}  // one image per launch
  // An item's contributions to a voxel are summed in float in a fixed order (the elements of the voxel's column in
  // the item, one warp per column), and the sum is rounded once to the fixed-point grid and added as a 64-bit
  // integer: integer addition is associative, so the image does not depend on the order of the items.  The scale
  // is a power of two of at most 2^126 and every partial sum times it is at most 2^62, so the product is exact.
  __device__ __forceinline__ T term(float v) const { return v; }
  __device__ __forceinline__ void flush(int64_t i, float v) const {
    if (v != 0.f) atomicAdd(acc + i, static_cast<unsigned long long>(__float2ll_rn(v * scale_f)));
  }
};

// Planes [zp, zp + 128) of the columns whose elements are [e_begin, e_end) of the path in column order, when every
// window of every (element, line) meets the image (checked at set-up, PathParams::zpad >= 0; an inactive line's
// data are all zero).  One warp streams through the elements of a contiguous range of columns, 32 at a time: each
// lane stages one element with the data offsets of its basic bin's first two lines (the z orientations) and
// whether it starts a new column, so that in the loop an element costs one 16-byte broadcast read and, per line,
// the plane loads and FMAs; the column's sums are added to the image when the next column starts.  Further lines
// of a basic bin (rare) read their line entries.
template <typename Cols>
__device__ __forceinline__ void back_span(const ProjParams& p, const PathParams& pp, const PathItemDev& it,
                                          const PathCElem* __restrict__ E, int e_begin, int e_end, const int4* lz,
                                          const int2* members, const float* dl, int zp, int lane, const Cols& acc,
                                          int4* eb) {
  const int nz = p.nz;
  typename Cols::T sum[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) sum[j] = typename Cols::T(0);
  int b = -1;          // image offset of the current column
  int prev_slot = -1;  // column of the last element staged
  auto flush = [&]() {
    if (b >= 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int z = zp + 32 * j + lane;
        if (z < nz) acc.flush(static_cast<int64_t>(b) + z, sum[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) sum[j] = typename Cols::T(0);
  };
  auto line = [&](float v, int off) {
    const float* q = dl + (off + lane);
#pragma unroll
    for (int j = 0; j < 4; ++j) sum[j] += acc.term(v * q[32 * j]);
  };
  for (int kb = e_begin; kb < e_end; kb += 32) {
    const int cnt = min(32, e_end - kb);
    __syncwarp();
    int slot = -1, off1 = 0, off2 = 0, nlines = 0;
    float v = 0.f;
    if (lane < cnt) {
      const PathCElem e = E[kb + lane];
      const int zr = static_cast<int>(e.mz & 2047u);
      const int2 mem = members[(e.mz >> 11) & 31u];
      slot = static_cast<int>(e.mz >> 16);
      v = e.v;
      nlines = mem.y;
      if (mem.y > 0) {
        const int4 L = lz[mem.x];
        off1 = L.w + zp - (L.x * zr + L.y);
      }
      if (mem.y > 1) {
        const int4 L = lz[mem.x + 1];
        off2 = L.w + zp - (L.x * zr + L.y);
      }
    }
    const int up = __shfl_up_sync(0xffffffffu, slot, 1);
    const int prev = lane == 0 ? prev_slot : up;
    prev_slot = __shfl_sync(0xffffffffu, slot, cnt - 1);
    if (lane < cnt) {
      // (value, data offset of line 1, of line 2, min(lines, 3) | new column << 2 | column << 3)
      const unsigned pk = static_cast<unsigned>(min(nlines, 3)) | (static_cast<unsigned>(slot != prev) << 2) |
                          (static_cast<unsigned>(slot) << 3);
      eb[lane] = make_int4(__float_as_int(v), off1, off2, static_cast<int>(pk));
    }
    __syncwarp();
    auto element = [&](const int4 w, int i) {
      const unsigned pk = static_cast<unsigned>(w.w);
      if (pk & 4u) {
        flush();
        b = column_image_offset(p, pp, it, static_cast<int>(pk >> 3));
      }
      const float ev = __int_as_float(w.x);
      const unsigned n = pk & 3u;
      if (n >= 2) {
        line(ev, w.y);
        line(ev, w.z);
        if (n == 3) {
          const PathCElem e = E[kb + i];
          const int zr = static_cast<int>(e.mz & 2047u);
          const int2 mem = members[(e.mz >> 11) & 31u];
          for (int l = mem.x + 2; l < mem.x + mem.y; ++l) {
            const int4 L = lz[l];
            line(ev, L.w + zp - (L.x * zr + L.y));
          }
        }
      } else if (n == 1) {
        line(ev, w.y);
      }
    };
    // two elements at a time: when neither starts a column and each has its basic bin's two lines (the common
    // case) their four lines run without branches between them; the order of the terms is unchanged
    int i = 0;
    for (; i + 1 < cnt; i += 2) {
      const int4 w0 = eb[i], w1 = eb[i + 1];
      if ((static_cast<unsigned>(w0.w) & 7u) == 2u && (static_cast<unsigned>(w1.w) & 7u) == 2u) {
        const float v0 = __int_as_float(w0.x), v1 = __int_as_float(w1.x);
        line(v0, w0.y);
        line(v0, w0.z);
        line(v1, w1.y);
        line(v1, w1.z);
      } else {
        element(w0, i);
        element(w1, i + 1);
      }
    }
    if (i < cnt) element(eb[i], i);
  }
  flush();
}

// the first element of the first column that starts at or after element t (col_starts cs, ncols + 1 entries)
__device__ __forceinline__ int column_boundary(const int* cs, int ncols, int t) {
  int lo = 0, hi = ncols;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(cs + mid) < t)
      lo = mid + 1;
    else
      hi = mid;
  }
  return __ldg(cs + lo);
}

// the same where a window may miss the image (PathParams::zpad < 0): such (element, line) pairs read the zero
// padding, and every line reads its line entry
template <typename Cols, bool HIT>
__device__ __forceinline__ void back_column(const PathCElem* __restrict__ E, int k0, int k1, const int4* lz,
                                            const int2* members, const float* dl, int zp, int nz, int lane, int b,
                                            const Cols& acc, int4* eb) {
  typename Cols::T sum[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) sum[j] = typename Cols::T(0);
  // the warp's 32 elements at a time go through its shared buffer as (z, value, first line and number of lines
  // of the element's basic bin): one 16-byte broadcast read per element
  auto element = [&](int zr, float v, int2 mem) {
      auto line = [&](int l) {
        const int4 L = lz[l];  // (z sign, z offset, window length, data offset)
        int zt = L.x * zr + L.y;
        // a window that misses the image (or an inactive line) reads the zero padding [0, F)
        if (!HIT && !(zt < nz && zt + L.z >= 0)) zt = zp + 128 + nz;
        const float* q = dl + (L.w + zp + lane - zt);
#pragma unroll
        for (int j = 0; j < 4; ++j) sum[j] += acc.term(v * q[32 * j]);
      };
      // a basic bin's lines are usually its two z orientations
      if (mem.y > 0) line(mem.x);
      if (mem.y > 1) line(mem.x + 1);
      for (int l = mem.x + 2; l < mem.x + mem.y; ++l) line(l);
  };
  for (int kb = k0; kb < k1; kb += 32) {
    const int cnt = min(32, k1 - kb);
    __syncwarp();
    if (lane < cnt) {
      const PathCElem e = E[kb + lane];
      const int2 mem = members[(e.mz >> 11) & 31u];
      eb[lane] = make_int4(static_cast<int>(e.mz & 2047u), __float_as_int(e.v), mem.x, mem.y);
    }
    __syncwarp();
    for (int i = 0; i < cnt; ++i) {
      const int4 w = eb[i];
      element(w.x, __int_as_float(w.y), make_int2(w.z, w.w));
    }
  }
  if (b < 0) return;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int z = zp + 32 * j + lane;
    if (z < nz) acc.flush(static_cast<int64_t>(b) + z, sum[j]);
  }
}

template <typename Cols>
__device__ __forceinline__ void back_path_item(const ProjParams& p, const PathParams& pp, const PathItemDev& it,
                                               unsigned char* smem, const float* __restrict__ pd, const Cols& acc,
                                               int zero_ends) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nz = p.nz;
  const PathSmemBack lay = path_smem_back(nz, pp.max_lines, pp.max_members, pp.nax_max, pp.npa_max);
  const int dl_len = path_dl_len(nz, pp.nax_max, pp.npa_max), front = path_dl_front(nz);
  PathLineSmem* ls = reinterpret_cast<PathLineSmem*>(smem + lay.lines);
  int4* lz = reinterpret_cast<int4*>(smem + lay.lz);
  int2* members = reinterpret_cast<int2*>(smem + lay.members);
  float* dl = reinterpret_cast<float*>(smem + lay.dl);
  int4* eb = reinterpret_cast<int4*>(smem + lay.ebuf) + warp * 32;
  const int nl = it.num_lines;
  setup_path_lines(p, pp, it, ls);
  for (int m = threadIdx.x; m < pp.max_members; m += blockDim.x) members[m] = make_int2(0, 0);
  __syncthreads();
  if (threadIdx.x == 0) {  // the lines of one member are consecutive
    for (int l = 0; l < nl; ++l) {
      int2& m = members[ls[l].member];
      if (m.y == 0) m.x = l;
      ++m.y;
    }
  }
  for (int l = threadIdx.x; l < nl; l += blockDim.x) {
    const PathLineSmem& L = ls[l];
    // an inactive line gets an empty window (zt + window < 0 for every zt < nz)
    lz[l] = make_int4(L.zsign, L.zadd, L.active ? (L.nax - 1) * L.npa : -(1 << 30), l * dl_len + front);
  }
  // padded line data: dl[l][front + a npa] = d(a), zero elsewhere and for skipped bins
  for (int l = warp; l < nl; l += kPathWarps) {
    const PathLineSmem L = ls[l];
    for (int t = lane; t < dl_len; t += 32) {
      const int r = t - front;
      float d = 0.f;
      if (L.active && r >= 0 && (L.npa == 1 || r % L.npa == 0)) {
        const int a = L.npa == 1 ? r : r / L.npa;
        if (a < L.nax && !(zero_ends && L.seg == 0 && (a == 0 || a == L.nax - 1)))
          d = pd ? __ldg(pd + L.out_base + a) : 1.f;  // pd == nullptr back-projects ones
      }
      dl[l * dl_len + t] = d;
    }
  }
  __syncthreads();
  const PathCElem* E = pp.cmaj + it.cmaj_off;
  const int* cs = pp.col_starts + it.col_starts;
  if (pp.zpad >= 0) {
    // every window meets the image: each warp streams through an equal share of the elements, cut at columns
    const int ne = __ldg(cs + it.ncols);
    const int e0 = column_boundary(cs, it.ncols, static_cast<int>(static_cast<int64_t>(ne) * warp / kPathWarps));
    const int e1 = column_boundary(cs, it.ncols, static_cast<int>(static_cast<int64_t>(ne) * (warp + 1) / kPathWarps));
    for (int zp = 0; zp < nz; zp += 128) back_span<Cols>(p, pp, it, E, e0, e1, lz, members, dl, zp, lane, acc, eb);
    return;
  }
  for (int ci = warp; ci < it.ncols; ci += kPathWarps) {
    const int b = column_image_offset(p, pp, it, ci);
    const int k0 = __ldg(cs + ci), k1 = __ldg(cs + ci + 1);
    for (int zp = 0; zp < nz; zp += 128) back_column<Cols, false>(E, k0, k1, lz, members, dl, zp, nz, lane, b, acc, eb);
  }
}

template <int NPA, int EPI>
__global__ void __launch_bounds__(kPathThreads, kPathMinCtas)
    forward_paths_kernel(ProjParams p, PathParams pp, const int* __restrict__ list, const float* __restrict__ img,
                         int64_t img_stride, float* __restrict__ out, int64_t out_stride, FwdEpilogue ep) {
  extern __shared__ __align__(16) unsigned char smem[];
  const PathItemDev it = pp.items[list[blockIdx.x]];
  if (blockIdx.y > 0) {  // image blockIdx.y of a batch
    const int64_t b = blockIdx.y;
    img += b * img_stride;
    if (out) out += b * out_stride;
    ep.y += b * ep.y_stride;
    if (ep.add) ep.add += b * ep.add_stride;
    if (ep.mult) ep.mult += b * ep.mult_stride;
    if (ep.small_value) ep.small_value += b * ep.sv_stride;
  }
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, blockDim.x);
  __syncthreads();
  double ll = 0.0;
  unsigned ncancel = 0;
  unsigned phase = 0;
  if (!forward_path_item<NPA, EPI>(p, pp, it, smem, img, out, ep, ll, ncancel, &bar, phase)) {
    // abandoned (the status word says so): the item's log-likelihood partial is NaN rather than stale
    if ((EPI == kEpiLoglik || EPI == kEpiLoglikRatio) && threadIdx.x == 0)
      ep.partials[static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x] = __longlong_as_double(-1ll);
    return;
  }
  if (EPI == kEpiRatio || EPI == kEpiGradient || EPI == kEpiLoglikRatio) {
    // cancelled singularities (distributable.cxx:590-594)
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if ((threadIdx.x & 31) == 0 && ncancel && ep.cancelled) atomicAdd(ep.cancelled, ncancel);
  }
  if (EPI == kEpiLoglik || EPI == kEpiLoglikRatio) {
    // per-CTA partial sums, reduced in a fixed order by the caller: deterministic
    __shared__ double red[kPathWarps];
    for (int o = 16; o > 0; o >>= 1) ll += __shfl_xor_sync(0xffffffffu, ll, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ll;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kPathWarps; ++w) t += red[w];
      ep.partials[static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x] = t;
    }
  }
}

template <typename Cols>
__global__ void __launch_bounds__(kPathThreads, kPathMinCtasBack)
    back_paths_kernel(ProjParams p, PathParams pp, const int* __restrict__ list, const float* __restrict__ pd,
                      int64_t pd_stride, Cols acc, int64_t img_stride, int zero_ends) {
  extern __shared__ __align__(16) unsigned char smem[];
  const PathItemDev it = pp.items[list[blockIdx.x]];
  Cols a = acc;
  a.load();
  if (blockIdx.y > 0) {  // image blockIdx.y of a batch
    if (pd) pd += static_cast<int64_t>(blockIdx.y) * pd_stride;
    a.offset(static_cast<int64_t>(blockIdx.y) * img_stride);
  }
  back_path_item<Cols>(p, pp, it, smem, pd, a, zero_ends);
}

// ---- batched reconstructions: a persistent grid over (frame, path item) work items ----------------
// The current item's frame, geometry (projector and path tables) and path item, copied to shared memory
// by the CTA so that the loops read them like kernel parameters.
struct BatchPathStage {
  ProjParams p;
  PathParams pp;
  BatchFrameDev f;
  PathItemDev it;
};
static_assert(sizeof(ProjParams) % 4 == 0 && sizeof(PathParams) % 4 == 0 && sizeof(BatchFrameDev) % 4 == 0 &&
                  sizeof(PathItemDev) % 4 == 0,
              "staged structures are copied as 32-bit words");

__device__ __forceinline__ bool next_path_item(unsigned* counter, const BatchItem* __restrict__ items, int nitems,
                                               const ProjParams* __restrict__ geoms,
                                               const PathParams* __restrict__ pgeoms,
                                               const BatchFrameDev* __restrict__ frames, BatchPathStage& st) {
  __shared__ int s_item;
  __syncthreads();  // every thread has finished with the previous item
  if (threadIdx.x == 0) s_item = static_cast<int>(atomicAdd(counter, 1u));
  __syncthreads();
  const int it = s_item;
  if (it >= nitems) return false;
  const BatchItem wi = items[it];
  const int g = frames[wi.frame].geom;
  constexpr int nf = sizeof(BatchFrameDev) / 4, np = sizeof(ProjParams) / 4, npp = sizeof(PathParams) / 4,
                ni = sizeof(PathItemDev) / 4;
  static_assert(nf + np + npp + ni <= kPathThreads, "one word per thread");
  const int t = threadIdx.x;
  if (t < nf) {
    reinterpret_cast<uint32_t*>(&st.f)[t] = reinterpret_cast<const uint32_t*>(frames + wi.frame)[t];
  } else if (t < nf + np) {
    reinterpret_cast<uint32_t*>(&st.p)[t - nf] = reinterpret_cast<const uint32_t*>(geoms + g)[t - nf];
  } else if (t < nf + np + npp) {
    reinterpret_cast<uint32_t*>(&st.pp)[t - nf - np] = reinterpret_cast<const uint32_t*>(pgeoms + g)[t - nf - np];
  } else if (t < nf + np + npp + ni) {
    reinterpret_cast<uint32_t*>(&st.it)[t - nf - np - npp] =
        reinterpret_cast<const uint32_t*>(pgeoms[g].items + wi.bin)[t - nf - np - npp];
  }
  __syncthreads();
  return true;
}

template <int NPA>
__global__ void __launch_bounds__(kPathThreads, kPathMinCtas)
    forward_batch_paths_kernel(const ProjParams* __restrict__ geoms, const PathParams* __restrict__ pgeoms,
                               const BatchFrameDev* __restrict__ frames, const BatchItem* __restrict__ items, int nitems,
                               unsigned* counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchPathStage st;
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, blockDim.x);
  unsigned phase = 0;  // next_path_item synchronises the CTA before the barrier's first use
  while (next_path_item(counter, items, nitems, geoms, pgeoms, frames, st)) {
    double ll = 0.0;
    unsigned ncancel = 0;
    // an abandoned item (status word set) ends this CTA: its copies may still be in flight
    if (!forward_path_item<NPA, kEpiRatio>(st.p, st.pp, st.it, smem, st.f.x, st.f.ratio, st.f.ep, ll, ncancel, &bar,
                                           phase))
      return;
    for (int o = 16; o > 0; o >>= 1) ncancel += __shfl_xor_sync(0xffffffffu, ncancel, o);
    if ((threadIdx.x & 31) == 0 && ncancel && st.f.ep.cancelled) atomicAdd(st.f.ep.cancelled, ncancel);
  }
}

__global__ void __launch_bounds__(kPathThreads, kPathMinCtasBack)
    back_batch_paths_kernel(const ProjParams* __restrict__ geoms, const PathParams* __restrict__ pgeoms,
                            const BatchFrameDev* __restrict__ frames, const BatchItem* __restrict__ items, int nitems,
                            unsigned* counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchPathStage st;
  while (next_path_item(counter, items, nitems, geoms, pgeoms, frames, st)) {
    if (st.f.acc64) {  // a deterministic frame: the same fixed-point integers as its own back projection
      FixedCols acc{st.f.acc64, st.f.fixed_scale, 0.0, 0.f};
      acc.load();
      back_path_item<FixedCols>(st.p, st.pp, st.it, smem, st.f.ratio, acc, 0);
    } else {
      back_path_item<FloatCols>(st.p, st.pp, st.it, smem, st.f.ratio, FloatCols{st.f.u}, 0);
    }
  }
}

const void* forward_batch_paths_fn(int npa) {
  return npa == 1 ? reinterpret_cast<const void*>(forward_batch_paths_kernel<1>)
       : npa == 2 ? reinterpret_cast<const void*>(forward_batch_paths_kernel<2>)
                  : reinterpret_cast<const void*>(forward_batch_paths_kernel<0>);
}

cudaError_t prepare_path_smem(const void* fn, int bytes) {
  if (bytes > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return cudaSuccess;
}

template <typename K, typename... A>
cudaError_t launch_path(K kernel, int nitems, int batch, int smem_bytes, cudaStream_t st, A... args) {
  if (nitems <= 0 || batch <= 0) return cudaSuccess;
  if (batch > 65535) return cudaErrorInvalidValue;
  cudaError_t e = prepare_path_smem(reinterpret_cast<const void*>(kernel), smem_bytes);
  if (e != cudaSuccess) return e;
  kernel<<<dim3(nitems, batch), kPathThreads, smem_bytes, st>>>(args...);
  return cudaGetLastError();
}

template <int EPI>
cudaError_t launch_forward_paths_epi(const ProjParams& p, const PathParams& pp, const int* list, int n, const float* image,
                                     int64_t img_stride, float* out, int64_t out_stride, int batch, cudaStream_t st,
                                     const FwdEpilogue& ep) {
  const int sm = path_smem_fwd(pp.K, p.nz, pp.zpad, pp.max_lines, pp.max_acc, pp.npa_max).total;
  switch (p.uniform_npa) {
    case 1:
      return launch_path(forward_paths_kernel<1, EPI>, n, batch, sm, st, p, pp, list, image, img_stride, out, out_stride,
                         ep);
    case 2:
      return launch_path(forward_paths_kernel<2, EPI>, n, batch, sm, st, p, pp, list, image, img_stride, out, out_stride,
                         ep);
    default:
      return launch_path(forward_paths_kernel<0, EPI>, n, batch, sm, st, p, pp, list, image, img_stride, out, out_stride,
                         ep);
  }
}

template <typename Cols>
cudaError_t launch_back_paths(const ProjParams& p, const PathParams& pp, const int* list, int n, const float* pd,
                              int64_t pd_stride, const Cols& acc, int64_t img_stride, int batch, cudaStream_t st,
                              int zero_ends) {
  const int sm = path_smem_back(p.nz, pp.max_lines, pp.max_members, pp.nax_max, pp.npa_max).total;
  return launch_path(back_paths_kernel<Cols>, n, batch, sm, st, p, pp, list, pd, pd_stride, acc, img_stride, zero_ends);
}

}  // namespace

cudaError_t launch_forward_paths_batch(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                       const float* images, int64_t img_stride, float* projdata, int64_t pd_stride,
                                       int batch, cudaStream_t st, const FwdEpilogue* ep) {
  FwdEpilogue e{};
  if (ep) e = *ep;
  switch (e.mode) {
    case kEpiNone:
      return launch_forward_paths_epi<kEpiNone>(p, pp, items, nitems, images, img_stride, projdata, pd_stride, batch, st,
                                                e);
    case kEpiRatio:
      return launch_forward_paths_epi<kEpiRatio>(p, pp, items, nitems, images, img_stride, projdata, pd_stride, batch,
                                                 st, e);
    case kEpiGradient:
      return launch_forward_paths_epi<kEpiGradient>(p, pp, items, nitems, images, img_stride, projdata, pd_stride, batch,
                                                    st, e);
    case kEpiLoglik:
      return launch_forward_paths_epi<kEpiLoglik>(p, pp, items, nitems, images, img_stride, projdata, pd_stride, batch,
                                                  st, e);
    case kEpiLoglikRatio:
      return launch_forward_paths_epi<kEpiLoglikRatio>(p, pp, items, nitems, images, img_stride, projdata, pd_stride,
                                                       batch, st, e);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_forward_paths(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                 const float* image, float* projdata, cudaStream_t st, const FwdEpilogue* ep) {
  return launch_forward_paths_batch(p, pp, items, nitems, image, 0, projdata, 0, 1, st, ep);
}

cudaError_t launch_forward_batch_paths(const ProjParams* geoms, const PathParams* pgeoms, int npa, int smem_bytes,
                                       const BatchFrameDev* frames, const BatchItem* items, int nitems, unsigned* counter,
                                       int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  cudaError_t e = prepare_path_smem(forward_batch_paths_fn(npa), smem_bytes);
  if (e != cudaSuccess) return e;
  if (npa == 1)
    forward_batch_paths_kernel<1><<<grid, kPathThreads, smem_bytes, st>>>(geoms, pgeoms, frames, items, nitems, counter);
  else if (npa == 2)
    forward_batch_paths_kernel<2><<<grid, kPathThreads, smem_bytes, st>>>(geoms, pgeoms, frames, items, nitems, counter);
  else
    forward_batch_paths_kernel<0><<<grid, kPathThreads, smem_bytes, st>>>(geoms, pgeoms, frames, items, nitems, counter);
  return cudaGetLastError();
}

cudaError_t launch_back_batch_paths(const ProjParams* geoms, const PathParams* pgeoms, int smem_bytes,
                                    const BatchFrameDev* frames, const BatchItem* items, int nitems, unsigned* counter,
                                    int grid, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  cudaError_t e = prepare_path_smem(reinterpret_cast<const void*>(back_batch_paths_kernel), smem_bytes);
  if (e != cudaSuccess) return e;
  back_batch_paths_kernel<<<grid, kPathThreads, smem_bytes, st>>>(geoms, pgeoms, frames, items, nitems, counter);
  return cudaGetLastError();
}

int batch_paths_max_ctas_per_sm(int npa, int smem_bytes, bool forward) {
  const void* fn = forward ? forward_batch_paths_fn(npa) : reinterpret_cast<const void*>(back_batch_paths_kernel);
  if (prepare_path_smem(fn, smem_bytes) != cudaSuccess) return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kPathThreads, smem_bytes) != cudaSuccess) return 0;
  return n;
}

cudaError_t launch_back_paths_atomic(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                     const float* projdata, float* image, cudaStream_t st, int zero_ends) {
  return launch_back_paths(p, pp, items, nitems, projdata, 0, FloatCols{image}, 0, 1, st, zero_ends);
}

cudaError_t launch_back_paths_atomic_batch(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                           const float* projdata, int64_t pd_stride, float* images, int64_t img_stride,
                                           int batch, cudaStream_t st, int zero_ends) {
  return launch_back_paths(p, pp, items, nitems, projdata, pd_stride, FloatCols{images}, img_stride, batch, st,
                           zero_ends);
}

cudaError_t launch_back_paths_fixed(const ProjParams& p, const PathParams& pp, const int* items, int nitems,
                                    const float* projdata, unsigned long long* acc, const double* scale,
                                    cudaStream_t st, int zero_ends) {
  return launch_back_paths(p, pp, items, nitems, projdata, 0, FixedCols{acc, scale, 0.0, 0.f}, 0, 1, st, zero_ends);
}

}  // namespace b200
