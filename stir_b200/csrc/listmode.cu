// List-mode Poisson objective with the ray-tracing matrix: per event, the row of its bin (the basic row with the
// event's symmetry operation and axial shift, as ProjMatrixByBin::get_proj_matrix_elems_for_one_bin gives it),
// after LM_gradient_and_value / LM_Hessian
// (src/recon_buildblock/PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin.cxx:750-820)
// and the subset rule of LM_distributable_computation (src/include/stir/recon_buildblock/distributable.txx:36-140):
//   gradient:  out += A_e^T (y_e / (A_e x + c_e))            (the reference's gradient has no cancellation test)
//   value:     -sum_e y_e log(A_e x + c_e)                   (-y_e log(y_e / 1e4) for a cancelled event)
//   Hessian:   out += A_e^T (-y_e / (A_e x + c_e)^2 A_e rhs)  unless cancelled or A_e rhs = 0
// One warp per event: the lanes split the row's elements (coalesced reads of the cached basic row), transform them
// by the event's line (swap / negate x, y; z -> q - z; + planes per axial position times the axial position),
// gather the image, reduce across the warp in a fixed order, and scatter the back projection with float atomics.
#include "internal.hpp"

namespace b200 {

namespace {

constexpr int kLmWarps = 8;
constexpr int kLmThreads = kLmWarps * 32;
constexpr float kMaxQuotient = 10000.F;

// the image index of row element e under line L at axial position a, or -1 outside [0, nz)
__device__ __forceinline__ int lm_voxel(const ProjParams& p, const RowElem& e, const LineDev& L, int zadd) {
  int z, y, x;
  unpack_zyx(e.zyx, z, y, x);
  const int swap = L.flags & 1;
  const int xt = (swap ? y : x) * ((L.flags & 2) ? -1 : 1);
  const int yt = (swap ? x : y) * ((L.flags & 4) ? -1 : 1);
  const int zt = ((L.flags & 8) ? static_cast<int>(L.q) - z : z) + zadd;
  if (zt < 0 || zt >= p.nz) return -1;
  return ((yt - p.min_y) * p.nx + (xt - p.min_x)) * p.nz + zt;
}

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sum over the row of img[voxel] * weight, each lane over elements lane, lane + 32, ... in order, kLmBatch
// elements' loads in flight at a time
constexpr int kLmBatch = 4;

__device__ __forceinline__ float lm_forward(const ProjParams& p, const RowElem* __restrict__ row, int len,
                                            const LineDev& L, int zadd, const float* __restrict__ img, int lane) {
  float f = 0.f;
  int k = lane;
  for (; k + 32 * (kLmBatch - 1) < len; k += 32 * kLmBatch) {
    RowElem e[kLmBatch];
    int v[kLmBatch];
    float xv[kLmBatch];
#pragma unroll
    for (int u = 0; u < kLmBatch; ++u) e[u] = row[k + 32 * u];
#pragma unroll
    for (int u = 0; u < kLmBatch; ++u) {
      v[u] = lm_voxel(p, e[u], L, zadd);
      xv[u] = v[u] >= 0 ? __ldg(img + v[u]) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kLmBatch; ++u)
      if (v[u] >= 0) f += xv[u] * e[u].v;
  }
  for (; k < len; k += 32) {
    const RowElem e = row[k];
    const int v = lm_voxel(p, e, L, zadd);
    if (v >= 0) f += __ldg(img + v) * e.v;
  }
  return warp_sum(f);
}

__device__ __forceinline__ void lm_back(const ProjParams& p, const RowElem* __restrict__ row, int len, const LineDev& L,
                                        int zadd, float data, float* __restrict__ out, int lane) {
  int k = lane;
  for (; k + 32 * (kLmBatch - 1) < len; k += 32 * kLmBatch) {
    RowElem e[kLmBatch];
#pragma unroll
    for (int u = 0; u < kLmBatch; ++u) e[u] = row[k + 32 * u];
#pragma unroll
    for (int u = 0; u < kLmBatch; ++u) {
      const int v = lm_voxel(p, e[u], L, zadd);
      if (v >= 0) atomicAdd(out + v, e[u].v * data);
    }
  }
  for (; k < len; k += 32) {
    const RowElem e = row[k];
    const int v = lm_voxel(p, e, L, zadd);
    if (v >= 0) atomicAdd(out + v, e.v * data);
  }
}

// A warp takes 32 consecutive events at a time: each lane resolves one event (bin lookup, basic bin, line) so the
// dependent loads of 32 events overlap, then the warp projects the events one after the other with the lane's
// results broadcast by shuffles.
template <int OP>  // 0 gradient, 1 value, 2 Hessian times rhs
__global__ void __launch_bounds__(kLmThreads) listmode_kernel(const ProjParams p, const int4* __restrict__ table,
                                                             const LmEventDev* __restrict__ ev, int64_t n,
                                                             const float* __restrict__ x, const float* __restrict__ rhs,
                                                             int subset, int nsub, int has_add, float* __restrict__ out,
                                                             double* __restrict__ partial, unsigned* __restrict__ invalid) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kLmWarps;
  double val = 0.0;
  for (int64_t base = (static_cast<int64_t>(blockIdx.x) * kLmWarps + warp) * 32; base < n; base += nwarps * 32) {
    // this lane's event: 0 = skip, 1 = project (row, line, z offset), invalid ones counted
    int state = 0, row_len = 0, line_bits = 0, zadd = 0;
    int64_t row_off = 0;
    float y = 0.f, corr = 0.f;
    if (base + lane < n) {
      const LmEventDev e = ev[base + lane];
      if (e.value != 0.0f) {
        const int s = e.seg + p.S, tofi = e.tof - p.min_tof, ti = e.tang - p.min_tang;
        bool ok = s >= 0 && s <= 2 * p.S && tofi >= 0 && tofi < p.num_tof && e.view >= 0 && e.view < p.num_views &&
                  ti >= 0 && ti < p.num_tang;
        int4 t = make_int4(-1, 0, 0, 0);
        if (ok) t = table[((static_cast<int64_t>(tofi) * (2 * p.S + 1) + s) * p.num_views + e.view) * p.num_tang + ti];
        SegDev sd{};
        if (ok) sd = p.segs[s];
        ok = ok && t.x >= 0 && e.axial >= 0 && e.axial < sd.nax;
        if (!ok) {
          atomicAdd(invalid, 1u);
        } else if (nsub <= 1 || t.z % nsub == subset) {
          const ProjBinDev pb = p.bins[t.x];
          const LineDev L = p.lines[pb.first_line + t.y];
          state = 1;
          row_off = pb.row_offset;
          row_len = pb.row_len;
          line_bits = (static_cast<int>(static_cast<uint8_t>(L.flags)) << 16) | static_cast<uint16_t>(L.q);
          zadd = e.axial * sd.npa - p.min_z;
          y = e.value;
          corr = has_add ? e.corr : 0.f;
        }
      }
    }
    for (int j = 0; j < 32; ++j) {
      if (!__shfl_sync(0xffffffffu, state, j)) continue;
      const int64_t off = __shfl_sync(0xffffffffu, row_off, j);
      const int len = __shfl_sync(0xffffffffu, row_len, j);
      const int lb = __shfl_sync(0xffffffffu, line_bits, j);
      const int za = __shfl_sync(0xffffffffu, zadd, j);
      const float yj = __shfl_sync(0xffffffffu, y, j);
      const float cj = __shfl_sync(0xffffffffu, corr, j);
      LineDev L;
      L.flags = static_cast<int8_t>(lb >> 16);
      L.q = static_cast<int16_t>(lb & 0xffff);
      const RowElem* row = p.rows + off;
      const float fwd = lm_forward(p, row, len, L, za, x, lane) + cj;
      const bool cancel = yj > kMaxQuotient * fwd;
      if (OP == 1) {
        if (lane == 0)
          val -= cancel ? yj * log(static_cast<double>(yj / kMaxQuotient)) : yj * log(static_cast<double>(fwd));
        continue;
      }
      if (OP == 2 && cancel) continue;
      float data;
      if (OP == 0) {
        data = yj / fwd;
      } else {
        const float r = lm_forward(p, row, len, L, za, rhs, lane);
        if (r == 0.f) continue;
        data = (-yj / (fwd * fwd)) * r;
      }
      if (data == 0.f) continue;
      lm_back(p, row, len, L, za, data, out, lane);
    }
  }
  if (OP == 1) {
    // per-block sum in a fixed order (warps in order), one partial per block
    __shared__ double red[kLmWarps];
    if (lane == 0) red[warp] = val;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kLmWarps; ++w) t += red[w];
      partial[blockIdx.x] = t;
    }
  }
}

// Binned form of the same three sums.  The rows of all events of one bin are the same row, so
//   sum_e A_e^T t_e = A^T h,  h[bin] = sum over the bin's events of t_e,
// and A_e x is entry `bin` of the forward projection A x of the subset.  One thread per event reads its bin's
// A x (and A rhs), applies the event's term exactly as the per-event kernel does, and adds it to h (device
// layout, float atomics); the projection kernels then take A x before and A^T h after.  Per event this costs a
// few bytes instead of a walk over ~400 row elements, so once the events number a fair fraction of the bins
// the two whole-subset projections are cheaper than the per-event rows.
constexpr int kLmBinThreads = 256;

template <int OP>
__global__ void __launch_bounds__(kLmBinThreads) listmode_binned_kernel(
    const ProjParams p, const int4* __restrict__ table, const LmEventDev* __restrict__ ev, int64_t n,
    const float* __restrict__ fwd, const float* __restrict__ fwd_rhs, int subset, int nsub, int has_add,
    float* __restrict__ hist, double* __restrict__ partial, unsigned* __restrict__ invalid) {
  double val = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(kLmBinThreads) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * kLmBinThreads) {
    const LmEventDev e = ev[i];
    if (e.value == 0.0f) continue;
    const int s = e.seg + p.S, tofi = e.tof - p.min_tof, ti = e.tang - p.min_tang;
    bool ok = s >= 0 && s <= 2 * p.S && tofi >= 0 && tofi < p.num_tof && e.view >= 0 && e.view < p.num_views &&
              ti >= 0 && ti < p.num_tang;
    int4 t = make_int4(-1, 0, 0, 0);
    if (ok) t = table[((static_cast<int64_t>(tofi) * (2 * p.S + 1) + s) * p.num_views + e.view) * p.num_tang + ti];
    SegDev sd{};
    if (ok) sd = p.segs[s];
    ok = ok && t.x >= 0 && e.axial >= 0 && e.axial < sd.nax;
    if (!ok) {
      atomicAdd(invalid, 1u);
      continue;
    }
    if (nsub > 1 && t.z % nsub != subset) continue;
    const int64_t bin = static_cast<int64_t>(tofi) * p.tof_stride + sd.dev_offset +
                        (static_cast<int64_t>(e.view) * p.num_tang + ti) * sd.nax + e.axial;
    const float y = e.value;
    const float f = fwd[bin] + (has_add ? e.corr : 0.f);
    const bool cancel = y > kMaxQuotient * f;
    if (OP == 1) {
      val -= cancel ? y * log(static_cast<double>(y / kMaxQuotient)) : y * log(static_cast<double>(f));
      continue;
    }
    if (OP == 2 && cancel) continue;
    float data;
    if (OP == 0) {
      data = y / f;
    } else {
      const float r = fwd_rhs[bin];
      if (r == 0.f) continue;
      data = (-y / (f * f)) * r;
    }
    if (data == 0.f) continue;
    atomicAdd(hist + bin, data);
  }
  if (OP == 1) {
    // fixed order: a shuffle tree per warp, then the warps in order; one partial per block
    for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
    __shared__ double red[kLmBinThreads / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = val;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kLmBinThreads / 32; ++w) t += red[w];
      partial[blockIdx.x] = t;
    }
  }
}

__global__ void subtract_kernel(float* __restrict__ out, const float* __restrict__ s, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] -= s[i];
}

__global__ void add_kernel(float* __restrict__ out, const float* __restrict__ s, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] += s[i];
}

}  // namespace

cudaError_t launch_add(float* out, const float* s, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t want = (n + 255) / 256;
  add_kernel<<<static_cast<int>(want > 148 * 32 ? 148 * 32 : want), 256, 0, st>>>(out, s, n);
  return cudaGetLastError();
}

int listmode_binned_num_blocks(int64_t n) {
  const int64_t want = (n + kLmBinThreads - 1) / kLmBinThreads;
  return static_cast<int>(want < 1 ? 1 : (want > 148 * 8 ? 148 * 8 : want));
}

cudaError_t launch_listmode_binned(const ProjParams& p, const int4* table, const LmEventDev* events, int64_t n, int op,
                                   const float* fwd, const float* fwd_rhs, int subset, int nsub, int has_add,
                                   float* hist, double* partial, unsigned* invalid, cudaStream_t st) {
  const int blocks = listmode_binned_num_blocks(n);
  switch (op) {
    case 0:
      listmode_binned_kernel<0><<<blocks, kLmBinThreads, 0, st>>>(p, table, events, n, fwd, fwd_rhs, subset, nsub,
                                                                  has_add, hist, partial, invalid);
      break;
    case 1:
      listmode_binned_kernel<1><<<blocks, kLmBinThreads, 0, st>>>(p, table, events, n, fwd, fwd_rhs, subset, nsub,
                                                                  has_add, hist, partial, invalid);
      break;
    default:
      listmode_binned_kernel<2><<<blocks, kLmBinThreads, 0, st>>>(p, table, events, n, fwd, fwd_rhs, subset, nsub,
                                                                  has_add, hist, partial, invalid);
      break;
  }
  return cudaGetLastError();
}

cudaError_t launch_subtract(float* out, const float* s, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t want = (n + 255) / 256;
  subtract_kernel<<<static_cast<int>(want > 148 * 32 ? 148 * 32 : want), 256, 0, st>>>(out, s, n);
  return cudaGetLastError();
}

int listmode_num_blocks(int64_t n) {
  const int64_t want = (n + 32 * kLmWarps - 1) / (32 * kLmWarps);
  return static_cast<int>(want < 1 ? 1 : (want > 148 * 16 ? 148 * 16 : want));
}

cudaError_t launch_listmode(const ProjParams& p, const int4* table, const LmEventDev* events, int64_t n, int op,
                            const float* x, const float* rhs, int subset, int nsub, int has_add, float* out,
                            double* partial, unsigned* invalid, cudaStream_t st) {
  const int blocks = listmode_num_blocks(n);
  switch (op) {
    case 0:
      listmode_kernel<0><<<blocks, kLmThreads, 0, st>>>(p, table, events, n, x, rhs, subset, nsub, has_add, out, partial,
                                                       invalid);
      break;
    case 1:
      listmode_kernel<1><<<blocks, kLmThreads, 0, st>>>(p, table, events, n, x, rhs, subset, nsub, has_add, out, partial,
                                                       invalid);
      break;
    default:
      listmode_kernel<2><<<blocks, kLmThreads, 0, st>>>(p, table, events, n, x, rhs, subset, nsub, has_add, out, partial,
                                                       invalid);
      break;
  }
  return cudaGetLastError();
}

}  // namespace b200
