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

template <int OP>  // 0 gradient, 1 value, 2 Hessian times rhs
__global__ void __launch_bounds__(kLmThreads) listmode_kernel(const ProjParams p, const int4* __restrict__ table,
                                                             const LmEventDev* __restrict__ ev, int64_t n,
                                                             const float* __restrict__ x, const float* __restrict__ rhs,
                                                             int subset, int nsub, int has_add, float* __restrict__ out,
                                                             double* __restrict__ partial, unsigned* __restrict__ invalid) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kLmWarps;
  double val = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kLmWarps + warp; i < n; i += nwarps) {
    const LmEventDev e = ev[i];
    if (e.value == 0.0f) continue;
    const int s = e.seg + p.S, tofi = e.tof - p.min_tof, ti = e.tang - p.min_tang;
    if (s < 0 || s > 2 * p.S || tofi < 0 || tofi >= p.num_tof || e.view < 0 || e.view >= p.num_views || ti < 0 ||
        ti >= p.num_tang) {
      if (lane == 0) atomicAdd(invalid, 1u);
      continue;
    }
    const int4 t = table[((static_cast<int64_t>(tofi) * (2 * p.S + 1) + s) * p.num_views + e.view) * p.num_tang + ti];
    const SegDev sd = p.segs[s];
    if (t.x < 0 || e.axial < 0 || e.axial >= sd.nax) {
      if (lane == 0) atomicAdd(invalid, 1u);
      continue;
    }
    if (nsub > 1 && t.z % nsub != subset) continue;
    const ProjBinDev pb = p.bins[t.x];
    const LineDev L = p.lines[pb.first_line + t.y];
    const int zadd = e.axial * sd.npa - p.min_z;
    const RowElem* row = p.rows + pb.row_offset;
    float f = 0.f;
    for (int k = lane; k < pb.row_len; k += 32) {
      const RowElem el = row[k];
      const int v = lm_voxel(p, el, L, zadd);
      if (v >= 0) f += __ldg(x + v) * el.v;
    }
    const float fwd = warp_sum(f) + (has_add ? e.corr : 0.f);
    const float y = e.value;
    const bool cancel = y > kMaxQuotient * fwd;
    if (OP == 1) {
      if (lane == 0) val -= cancel ? y * log(static_cast<double>(y / kMaxQuotient)) : y * log(static_cast<double>(fwd));
      continue;
    }
    if (OP == 2 && cancel) continue;
    float data;
    if (OP == 0) {
      data = y / fwd;
    } else {
      const float c = -y / (fwd * fwd);
      float r = 0.f;
      for (int k = lane; k < pb.row_len; k += 32) {
        const RowElem el = row[k];
        const int v = lm_voxel(p, el, L, zadd);
        if (v >= 0) r += __ldg(rhs + v) * el.v;
      }
      r = warp_sum(r);
      if (r == 0.f) continue;
      data = c * r;
    }
    if (data == 0.f) continue;
    for (int k = lane; k < pb.row_len; k += 32) {
      const RowElem el = row[k];
      const int v = lm_voxel(p, el, L, zadd);
      if (v >= 0) atomicAdd(out + v, el.v * data);
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

__global__ void subtract_kernel(float* __restrict__ out, const float* __restrict__ s, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] -= s[i];
}

}  // namespace

cudaError_t launch_subtract(float* out, const float* s, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t want = (n + 255) / 256;
  subtract_kernel<<<static_cast<int>(want > 148 * 32 ? 148 * 32 : want), 256, 0, st>>>(out, s, n);
  return cudaGetLastError();
}

int listmode_num_blocks(int64_t n) {
  const int64_t want = (n + kLmWarps - 1) / kLmWarps;
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
