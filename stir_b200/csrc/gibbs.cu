// Gibbs penalties on device-resident images: GibbsPenalty<float, Potential>
// (src/include/stir/recon_buildblock/GibbsPenalty.inl) with the Quadratic potential (GibbsQuadraticPenalty.h:50-80)
// or the Relative Difference potential (GibbsRelativeDifferencePenalty.h:60-120), i.e. the operations of
// GibbsQuadraticPenalty / GibbsRelativeDifferencePenalty and of their CUDA versions
// (src/include/stir/recon_buildblock/CUDA/CudaGibbsPenalty.cuh), without the host copies.
//
// One thread per voxel, in memory order, for either image layout; the neighbourhood (weights of any size up to
// 7x7x7, kernel parameters) is walked in STIR's order (dz, dy, dx) and every sum is taken in the type and order of
// GibbsPenalty.inl (double for the value, gradient and Hessian diagonal, float for the Hessian times an input), so
// each voxel's result is that of the host loop.  Scalars (value, gradient times input) are summed per block in a
// fixed order and the block sums reduced in a fixed order: deterministic.  Compiled with -fmad=false, so float and
// double expressions round as the host build evaluates them.
#include "internal.hpp"

namespace b200 {

namespace {

constexpr int kGibbsThreads = 256;

struct QuadPot {
  __device__ __forceinline__ double value(float c, float n) const {
    const float diff = c - n;
    return static_cast<double>(diff * diff) / 4.0;
  }
  __device__ __forceinline__ double d10(float c, float n) const { return static_cast<double>(c - n) / 2.0; }
  __device__ __forceinline__ double d20(float, float) const { return 0.5; }
  __device__ __forceinline__ double d11(float, float) const { return -0.5; }
};

// The reference evaluates with float operands, the double literals 0.5 and 1.0 making those operations double
// and the results assigned to floats rounded back.  Each such double step equals a float step here:
//  - (float)(1.0 / (double)v) is the correctly rounded float reciprocal of v (division of two floats rounded first
//    to 53 bits, then to 24: double rounding is innocuous when 53 >= 2*24 + 2, Figueroa 1995), __frcp_rn(v);
//  - (float)(0.5 * (double)a * (double)b) with float a, b is (0.5f * a) * b: 0.5 a is exact, the double product of
//    two floats is exact, so one rounding to float remains, as in the float product;
//  - (float)(0.5 * (double)(d * d)) is 0.5f * (d * d) (exact scaling).
// so every value is bit-identical to the reference's expression without double divisions.
struct RDPot {
  float gamma, epsilon;
  __device__ __forceinline__ double value(float c, float n) const {
    const float diff = c - n;
    const float add = c + n;
    const float num = 0.5f * (diff * diff);
    const float den = __frcp_rn(add + gamma * fabsf(diff) + epsilon);
    return static_cast<double>(num * den);
  }
  __device__ __forceinline__ double d10(float c, float n) const {
    const float diff = c - n;
    const float factor = c + n + gamma * fabsf(diff) + epsilon;
    const float num = (0.5f * diff) * (factor + 2 * n + epsilon);
    const float den = __frcp_rn(factor * factor);
    return static_cast<double>(num * den);
  }
  __device__ __forceinline__ double d20(float c, float n) const {
    const float num = 2 * n + epsilon;
    const float den = __frcp_rn(c + n + gamma * fabsf(c - n) + epsilon);
    return static_cast<double>(num * num * den * den * den);
  }
  __device__ __forceinline__ double d11(float c, float n) const {
    const float num = -(2 * c + epsilon) * (2 * n + epsilon);
    const float den = __frcp_rn(c + n + gamma * fabsf(c - n) + epsilon);
    return static_cast<double>(num * den * den * den);
  }
};

// the voxel (z, y, x) of memory index i
__device__ __forceinline__ void gibbs_coords(const GibbsDev& g, int i, int& z, int& y, int& x) {
  if (g.layout == 0) {  // [y][x][z]
    z = i % g.nz;
    const int t = i / g.nz;
    x = t % g.nx;
    y = t / g.nx;
  } else {  // [z][y][x]
    x = i % g.nx;
    const int t = i / g.nx;
    y = t % g.ny;
    z = t / g.ny;
  }
}

struct Range {
  int z0, z1, y0, y1, x0, x1;
};
__device__ __forceinline__ Range gibbs_range(const GibbsDev& g, int z, int y, int x) {
  Range r;
  r.z0 = max(-(g.wz / 2), -z);
  r.z1 = min(g.wz - 1 - g.wz / 2, g.nz - 1 - z);
  r.y0 = max(-(g.wy / 2), -y);
  r.y1 = min(g.wy - 1 - g.wy / 2, g.ny - 1 - y);
  r.x0 = max(-(g.wx / 2), -x);
  r.x1 = min(g.wx - 1 - g.wx / 2, g.nx - 1 - x);
  return r;
}
__device__ __forceinline__ float gibbs_w(const GibbsDev& g, int dz, int dy, int dx) {
  return g.w[((dz + g.wz / 2) * g.wy + (dy + g.wy / 2)) * g.wx + (dx + g.wx / 2)];
}

// fixed-order block sum of one double per thread; thread 0 gets the total
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[kGibbsThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kGibbsThreads / 32; ++w) t += red[w];
  return t;
}

// one neighbour's term of the per-voxel sums, in the reference's types
template <typename Pot, int OP>
__device__ __forceinline__ void gibbs_term(const Pot& pot, float w, double wd, float c, float nk, float kk, float inj,
                                           float ink, bool centre, const float* kappa, double& sum, float& result) {
  if (OP == 4) {
    float current = w;
    if (centre)
      current = static_cast<float>(current * (pot.d20(c, nk) * inj));
    else
      current = static_cast<float>(current * (pot.d20(c, nk) * inj + pot.d11(c, nk) * ink));
    if (kappa) current *= kk;
    result += current;
  } else {
    if (centre) return;
    const double f = OP == 0 ? pot.value(c, nk) : (OP == 3 ? pot.d20(c, nk) : pot.d10(c, nk));
    double current = wd * f;  // wd = (double)w: the product is the reference's w * f
    if (kappa) current *= kk;
    sum += current;
  }
}

// OP: 0 value, 1 gradient, 2 gradient times input, 3 Hessian diagonal, 4 accumulate Hessian times input.
// Voxels whose whole neighbourhood lies in the image take an unrolled path when the weights are 3x3x3 or 1x3x3
// (the default weights and STIR's usual explicit ones), with the same order of terms as the general loop.
template <typename Pot, int OP>
__global__ void __launch_bounds__(kGibbsThreads) gibbs_kernel(const GibbsDev g, const Pot pot,
                                                              const float* __restrict__ x,
                                                              const float* __restrict__ in, float* __restrict__ out,
                                                              double* __restrict__ partial) {
  const int n = g.nz * g.ny * g.nx;  // < 2^31, checked at set-up
  const int j = blockIdx.x * kGibbsThreads + threadIdx.x;
  double acc = 0.0;
  if (j < n) {
    int z, y, xx;
    gibbs_coords(g, j, z, y, xx);
    const int sz = static_cast<int>(g.sz), sy = static_cast<int>(g.sy), sx = static_cast<int>(g.sx);
    const float c = __ldg(x + j);
    const float kj = g.kappa ? __ldg(g.kappa + j) : 1.f;
    const float inj = (OP == 4) ? __ldg(in + j) : 0.f;
    double sum = 0.0;
    float result = 0.f;
    const bool in3 = y >= 1 && y + 1 < g.ny && xx >= 1 && xx + 1 < g.nx;
    if (g.wy == 3 && g.wx == 3 && g.wz == 3 && in3 && z >= 1 && z + 1 < g.nz) {
#pragma unroll
      for (int t = 0; t < 27; ++t) {
        const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
        const int k = j + dz * sz + dy * sy + dx * sx;
        const float kk = g.kappa ? kj * __ldg(g.kappa + k) : 1.f;
        gibbs_term<Pot, OP>(pot, g.w[t], g.wd[t], c, __ldg(x + k), kk, inj, OP == 4 ? __ldg(in + k) : 0.f, t == 13,
                            g.kappa, sum, result);
      }
    } else if (g.wy == 3 && g.wx == 3 && g.wz == 1 && in3) {
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const int dy = t / 3 - 1, dx = t % 3 - 1;
        const int k = j + dy * sy + dx * sx;
        const float kk = g.kappa ? kj * __ldg(g.kappa + k) : 1.f;
        gibbs_term<Pot, OP>(pot, g.w[t], g.wd[t], c, __ldg(x + k), kk, inj, OP == 4 ? __ldg(in + k) : 0.f, t == 4,
                            g.kappa, sum, result);
      }
    } else {
      const Range r = gibbs_range(g, z, y, xx);
      for (int dz = r.z0; dz <= r.z1; ++dz)
        for (int dy = r.y0; dy <= r.y1; ++dy)
          for (int dx = r.x0; dx <= r.x1; ++dx) {
            const int k = j + dz * sz + dy * sy + dx * sx;
            const float kk = g.kappa ? kj * __ldg(g.kappa + k) : 1.f;
            const float w = gibbs_w(g, dz, dy, dx);
            gibbs_term<Pot, OP>(pot, w, static_cast<double>(w), c, __ldg(x + k), kk, inj,
                                OP == 4 ? __ldg(in + k) : 0.f, dz == 0 && dy == 0 && dx == 0, g.kappa, sum, result);
          }
    }
    if (OP == 4)
      out[j] += 2 * result * g.beta;
    else if (OP == 1 || OP == 3)
      out[j] = 2 * static_cast<float>(sum * g.beta);
    else if (OP == 0)
      acc = sum;
    else
      acc = 2 * sum * __ldg(in + j);
  }
  if (OP == 0 || OP == 2) {
    const double t = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
  }
}

// compute_Hessian of voxel (z, y, x): out (zeroed by the caller) gets the voxel's row of the Hessian; one thread
// per neighbour
template <typename Pot>
__global__ void gibbs_hessian_voxel_kernel(const GibbsDev g, const Pot pot, const float* __restrict__ x, int z, int y,
                                           int xx, float* __restrict__ out) {
  const Range r = gibbs_range(g, z, y, xx);
  const int ny = r.y1 - r.y0 + 1, nx = r.x1 - r.x0 + 1;
  const int t = threadIdx.x;
  if (t >= (r.z1 - r.z0 + 1) * ny * nx) return;
  const int dz = r.z0 + t / (ny * nx), dy = r.y0 + (t / nx) % ny, dx = r.x0 + t % nx;
  const int64_t j = static_cast<int64_t>(z) * g.sz + static_cast<int64_t>(y) * g.sy + static_cast<int64_t>(xx) * g.sx;
  const float c = x[j];
  float current = 0.f;
  if (dz == 0 && dy == 0 && dx == 0) {
    for (int ddz = r.z0; ddz <= r.z1; ++ddz)
      for (int ddy = r.y0; ddy <= r.y1; ++ddy)
        for (int ddx = r.x0; ddx <= r.x1; ++ddx) {
          const int64_t k = j + ddz * g.sz + ddy * g.sy + ddx * g.sx;
          float dc = static_cast<float>(gibbs_w(g, ddz, ddy, ddx) * 2 * pot.d20(c, x[k]));
          if (g.kappa) dc *= g.kappa[j] * g.kappa[k];
          current += dc;
        }
  } else {
    const int64_t k = j + dz * g.sz + dy * g.sy + dx * g.sx;
    current = static_cast<float>(gibbs_w(g, dz, dy, dx) * 2 * pot.d11(c, x[k]));
    if (g.kappa) current *= g.kappa[j] * g.kappa[k];
  }
  out[j + dz * g.sz + dy * g.sy + dx * g.sx] = current * g.beta;
}

__global__ void gibbs_reduce_kernel(const double* __restrict__ partial, int n, double beta, double* __restrict__ out) {
  // fixed order: thread t sums t, t + 256, ...; then the block sum in a fixed order
  __shared__ double s[256];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) v += partial[i];
  s[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < 256; ++i) t += s[i];
    *out = t * beta;
  }
}

// ---- the gradient with the arithmetic of STIR's CUDA build (CudaGibbsPenalty_gradient_kernel,
// CudaGibbsPenalty.cuh:141-206): a float sum per voxel over the whole neighbourhood (the centre included) of
// weight x derivative_10 (x kappa_j kappa_k), and the float of sum x 2 x beta.  nvcc compiles the reference's
// source with contraction on and folds a double step between floats to the float step when that rounds the same
// (an operation of two floats carried out in double and rounded back: double holds more than 2 x 24 + 2 bits);
// so a term whose last operation becomes a float product is fused into the sum (one fused multiply-add), and the
// other float expressions are contracted as written.  Each step is written here with an explicit round-to-nearest
// operation so that the result does not depend on this file's compilation flags:
//   Quadratic: the term w ((double)(c - n) / 2.0) stays a double product rounded to float, added to the sum;
//              with kappa that float times (kappa_j kappa_k) is fused into the sum;
//   Relative Difference (GibbsRelativeDifferencePenalty.h:81-91): factor = fma(gamma, |c - n|, c + n) + epsilon,
//              num = (0.5 (c - n)) (fma(2, n, factor) + epsilon), den = 1 / (factor factor) (the double reciprocal
//              rounded to float is the correctly rounded float reciprocal), d = num den; the term w d is fused into
//              the sum, or with kappa w d rounded and (w d) (kappa_j kappa_k) fused into the sum.
struct QuadPotCuda {
  template <bool KAPPA>
  __device__ __forceinline__ float add(float sum, float w, float c, float n, float kk) const {
    const float cur = __fmul_rn(w, 0.5f * __fsub_rn(c, n));
    return KAPPA ? __fmaf_rn(cur, kk, sum) : __fadd_rn(sum, cur);
  }
};
struct RDPotCuda {
  float gamma, epsilon;
  template <bool KAPPA>
  __device__ __forceinline__ float add(float sum, float w, float c, float n, float kk) const {
    const float diff = __fsub_rn(c, n);
    const float factor = __fadd_rn(__fmaf_rn(gamma, fabsf(diff), __fadd_rn(c, n)), epsilon);
    const float num = __fmul_rn(0.5f * diff, __fadd_rn(__fmaf_rn(2.f, n, factor), epsilon));
    const float d = __fmul_rn(num, __frcp_rn(__fmul_rn(factor, factor)));
    return KAPPA ? __fmaf_rn(__fmul_rn(w, d), kk, sum) : __fmaf_rn(w, d, sum);
  }
};

template <typename Pot, bool KAPPA>
__global__ void __launch_bounds__(kGibbsThreads) gibbs_gradient_cuda_kernel(const GibbsDev g, const Pot pot,
                                                                            const float* __restrict__ x,
                                                                            float* __restrict__ out) {
  const int n = g.nz * g.ny * g.nx;
  const int j = blockIdx.x * kGibbsThreads + threadIdx.x;
  if (j >= n) return;
  int z, y, xx;
  gibbs_coords(g, j, z, y, xx);
  const int sz = static_cast<int>(g.sz), sy = static_cast<int>(g.sy), sx = static_cast<int>(g.sx);
  const float c = __ldg(x + j);
  const float kj = KAPPA ? __ldg(g.kappa + j) : 1.f;
  float sum = 0.f;
  if (g.wy == 3 && g.wx == 3 && g.wz == 3 && y >= 1 && y + 1 < g.ny && xx >= 1 && xx + 1 < g.nx && z >= 1 &&
      z + 1 < g.nz) {
#pragma unroll
    for (int t = 0; t < 27; ++t) {
      const int k = j + (t / 9 - 1) * sz + ((t / 3) % 3 - 1) * sy + (t % 3 - 1) * sx;
      sum = pot.template add<KAPPA>(sum, g.w[t], c, __ldg(x + k), KAPPA ? __fmul_rn(kj, __ldg(g.kappa + k)) : 1.f);
    }
  } else {
    const Range r = gibbs_range(g, z, y, xx);
    for (int dz = r.z0; dz <= r.z1; ++dz)
      for (int dy = r.y0; dy <= r.y1; ++dy)
        for (int dx = r.x0; dx <= r.x1; ++dx) {
          const int k = j + dz * sz + dy * sy + dx * sx;
          sum = pot.template add<KAPPA>(sum, gibbs_w(g, dz, dy, dx), c, __ldg(x + k),
                                        KAPPA ? __fmul_rn(kj, __ldg(g.kappa + k)) : 1.f);
        }
  }
  out[j] = __fmul_rn(sum * 2.f, g.beta);
}

// ---- the gradient with 3x3x3 weights, tiled: a block of 32 x 8 threads covers a tile of the two fastest memory
// axes and walks the slowest one, keeping three planes of the tile with a one-voxel halo (and of kappa) in shared
// memory, so each image value is read from memory about once instead of 27 times through L1.  Every voxel's terms
// are taken in STIR's (dz, dy, dx) order with the same arithmetic as the kernels above (the host or the CUDA
// build's), so the results are those kernels' bit for bit.
constexpr int kTile0 = 32, kTile1 = 8, kTileChunk = 16;
constexpr int kHalo0 = kTile0 + 2, kHalo1 = kTile1 + 2, kPlane = kHalo0 * kHalo1;

// the per-voxel sum of one arithmetic: HostSum keeps GibbsPenalty.inl's double sum (gibbs_term, gradient), CudaSum
// the CUDA build's float sum (RDPotCuda / QuadPotCuda)
template <typename Pot>
struct HostSum {
  Pot pot;
  using T = double;
  __device__ __forceinline__ void add(T& sum, float w, double wd, float c, float n, float kk, bool kappa,
                                      bool centre) const {
    float unused = 0.f;
    gibbs_term<Pot, 1>(pot, w, wd, c, n, kk, 0.f, 0.f, centre, kappa ? &unused : nullptr, sum, unused);
  }
  __device__ __forceinline__ float result(T sum, float beta) const { return 2 * static_cast<float>(sum * beta); }
};
template <typename Pot, bool KAPPA>
struct CudaSum {
  Pot pot;
  using T = float;
  __device__ __forceinline__ void add(T& sum, float w, double, float c, float n, float kk, bool, bool) const {
    sum = pot.template add<KAPPA>(sum, w, c, n, kk);
  }
  __device__ __forceinline__ float result(T sum, float beta) const { return __fmul_rn(sum * 2.f, beta); }
};

// LAYOUT 0: device [y][x][z] (axes 0, 1, 2 = z, x, y); 1: STIR [z][y][x] (axes 0, 1, 2 = x, y, z)
template <int LAYOUT, typename Sum, bool KAPPA>
__global__ void __launch_bounds__(kTile0 * kTile1) gibbs_gradient_tiled_kernel(const GibbsDev g, const Sum sum_op,
                                                                               const float* __restrict__ x,
                                                                               float* __restrict__ out) {
  __shared__ float tile[3][kPlane];
  __shared__ float ktile[KAPPA ? 3 : 1][KAPPA ? kPlane : 1];
  const int n0 = LAYOUT == 0 ? g.nz : g.nx, n1 = LAYOUT == 0 ? g.nx : g.ny, n2 = LAYOUT == 0 ? g.ny : g.nz;
  const int64_t s1 = n0, s2 = static_cast<int64_t>(n0) * n1;
  const int t0 = threadIdx.x, t1 = threadIdx.y;
  const int i0 = blockIdx.x * kTile0 + t0, i1 = blockIdx.y * kTile1 + t1;
  const int c0 = blockIdx.z * kTileChunk, c1 = min(c0 + kTileChunk, n2);
  const int tid = t1 * kTile0 + t0;
  // plane c of the tile with its halo into ring slot c mod 3 (zeros outside the image: never read)
  auto load = [&](int c) {
    float* dst = tile[(c + 3) % 3];
    float* kdst = ktile[KAPPA ? (c + 3) % 3 : 0];
    for (int q = tid; q < kPlane; q += kTile0 * kTile1) {
      const int h0 = blockIdx.x * kTile0 + q % kHalo0 - 1, h1 = blockIdx.y * kTile1 + q / kHalo0 - 1;
      const bool in = c >= 0 && c < n2 && h0 >= 0 && h0 < n0 && h1 >= 0 && h1 < n1;
      const int64_t k = in ? c * s2 + h1 * s1 + h0 : 0;
      dst[q] = in ? __ldg(x + k) : 0.f;
      if (KAPPA) kdst[q] = in ? __ldg(g.kappa + k) : 0.f;
    }
  };
  load(c0 - 1);
  load(c0);
  for (int c = c0; c < c1; ++c) {
    load(c + 1);
    __syncthreads();
    if (i0 < n0 && i1 < n1) {
      // (z, y, x) of the voxel and the neighbourhood clipped to the image
      const int z = LAYOUT == 0 ? i0 : c, y = LAYOUT == 0 ? c : i1, xx = LAYOUT == 0 ? i1 : i0;
      const int ctr = (t1 + 1) * kHalo0 + (t0 + 1);
      const float cv = tile[c % 3][ctr];
      const float kj = KAPPA ? ktile[c % 3][ctr] : 1.f;
      typename Sum::T sum = 0;
      const bool interior = z >= 1 && z + 1 < g.nz && y >= 1 && y + 1 < g.ny && xx >= 1 && xx + 1 < g.nx;
      auto term = [&](int dz, int dy, int dx, int t) {
        // memory-axis offsets of (dz, dy, dx)
        const int d0 = LAYOUT == 0 ? dz : dx, d1 = LAYOUT == 0 ? dx : dy, d2 = LAYOUT == 0 ? dy : dz;
        const int slot = (c + d2 + 3) % 3, q = ctr + d1 * kHalo0 + d0;
        const float kk = KAPPA ? __fmul_rn(kj, ktile[slot][q]) : 1.f;
        sum_op.add(sum, g.w[t], g.wd[t], cv, tile[slot][q], kk, KAPPA, t == 13);
      };
      if (interior) {
#pragma unroll
        for (int t = 0; t < 27; ++t) term(t / 9 - 1, (t / 3) % 3 - 1, t % 3 - 1, t);
      } else {
        const Range r = gibbs_range(g, z, y, xx);
        for (int dz = r.z0; dz <= r.z1; ++dz)
          for (int dy = r.y0; dy <= r.y1; ++dy)
            for (int dx = r.x0; dx <= r.x1; ++dx) term(dz, dy, dx, (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
      }
      out[static_cast<int64_t>(c) * s2 + static_cast<int64_t>(i1) * s1 + i0] = sum_op.result(sum, g.beta);
    }
    __syncthreads();  // plane c - 1's slot is overwritten by the next load
  }
}

template <typename Sum, bool KAPPA>
cudaError_t launch_tiled(const GibbsDev& g, const Sum& s, const float* x, float* out, cudaStream_t st) {
  const int n0 = g.layout == 0 ? g.nz : g.nx, n1 = g.layout == 0 ? g.nx : g.ny, n2 = g.layout == 0 ? g.ny : g.nz;
  const dim3 grid((n0 + kTile0 - 1) / kTile0, (n1 + kTile1 - 1) / kTile1, (n2 + kTileChunk - 1) / kTileChunk);
  const dim3 block(kTile0, kTile1);
  if (g.layout == 0)
    gibbs_gradient_tiled_kernel<0, Sum, KAPPA><<<grid, block, 0, st>>>(g, s, x, out);
  else
    gibbs_gradient_tiled_kernel<1, Sum, KAPPA><<<grid, block, 0, st>>>(g, s, x, out);
  return cudaGetLastError();
}

// the tiled gradient applies to 3x3x3 weights (the default and STIR's usual explicit ones)
bool gibbs_tiled(const GibbsDev& g) { return g.wz == 3 && g.wy == 3 && g.wx == 3; }

template <typename Pot>
cudaError_t gibbs_launch_pot(const GibbsDev& g, const Pot& pot, int op, const float* x, const float* in, float* out,
                             double* partial, double* result, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(g.nz) * g.ny * g.nx;
  const int64_t blocks = (n + kGibbsThreads - 1) / kGibbsThreads;
  if (blocks > 2147483647LL) return cudaErrorInvalidValue;
  const unsigned nb = static_cast<unsigned>(blocks);
  switch (op) {
    case 0: gibbs_kernel<Pot, 0><<<nb, kGibbsThreads, 0, st>>>(g, pot, x, in, out, partial); break;
    case 1: gibbs_kernel<Pot, 1><<<nb, kGibbsThreads, 0, st>>>(g, pot, x, in, out, partial); break;
    case 2: gibbs_kernel<Pot, 2><<<nb, kGibbsThreads, 0, st>>>(g, pot, x, in, out, partial); break;
    case 3: gibbs_kernel<Pot, 3><<<nb, kGibbsThreads, 0, st>>>(g, pot, x, in, out, partial); break;
    case 4: gibbs_kernel<Pot, 4><<<nb, kGibbsThreads, 0, st>>>(g, pot, x, in, out, partial); break;
    default: return cudaErrorInvalidValue;
  }
  if (op == 0 || op == 2) gibbs_reduce_kernel<<<1, 256, 0, st>>>(partial, static_cast<int>(blocks), g.beta, result);
  return cudaGetLastError();
}

}  // namespace

int64_t gibbs_num_partials(const GibbsDev& g) {
  return (static_cast<int64_t>(g.nz) * g.ny * g.nx + kGibbsThreads - 1) / kGibbsThreads;
}

cudaError_t launch_gibbs(const GibbsDev& g, int op, const float* x, const float* in, float* out, double* partial,
                         double* result, cudaStream_t st) {
  if (op == 1 && gibbs_tiled(g)) {
    if (g.potential == 1)
      return g.kappa ? launch_tiled<HostSum<QuadPot>, true>(g, HostSum<QuadPot>{QuadPot{}}, x, out, st)
                     : launch_tiled<HostSum<QuadPot>, false>(g, HostSum<QuadPot>{QuadPot{}}, x, out, st);
    const HostSum<RDPot> s{RDPot{g.gamma, g.epsilon}};
    return g.kappa ? launch_tiled<HostSum<RDPot>, true>(g, s, x, out, st)
                   : launch_tiled<HostSum<RDPot>, false>(g, s, x, out, st);
  }
  if (g.potential == 1) return gibbs_launch_pot(g, QuadPot{}, op, x, in, out, partial, result, st);
  return gibbs_launch_pot(g, RDPot{g.gamma, g.epsilon}, op, x, in, out, partial, result, st);
}

cudaError_t launch_gibbs_gradient_cuda(const GibbsDev& g, const float* x, float* out, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(g.nz) * g.ny * g.nx;
  const unsigned nb = static_cast<unsigned>((n + kGibbsThreads - 1) / kGibbsThreads);
  const RDPotCuda rdp{g.gamma, g.epsilon};
  if (gibbs_tiled(g)) {
    if (g.potential == 1)
      return g.kappa ? launch_tiled<CudaSum<QuadPotCuda, true>, true>(g, {QuadPotCuda{}}, x, out, st)
                     : launch_tiled<CudaSum<QuadPotCuda, false>, false>(g, {QuadPotCuda{}}, x, out, st);
    return g.kappa ? launch_tiled<CudaSum<RDPotCuda, true>, true>(g, {rdp}, x, out, st)
                   : launch_tiled<CudaSum<RDPotCuda, false>, false>(g, {rdp}, x, out, st);
  }
  if (g.potential == 1 && g.kappa)
    gibbs_gradient_cuda_kernel<QuadPotCuda, true><<<nb, kGibbsThreads, 0, st>>>(g, QuadPotCuda{}, x, out);
  else if (g.potential == 1)
    gibbs_gradient_cuda_kernel<QuadPotCuda, false><<<nb, kGibbsThreads, 0, st>>>(g, QuadPotCuda{}, x, out);
  else if (g.kappa)
    gibbs_gradient_cuda_kernel<RDPotCuda, true><<<nb, kGibbsThreads, 0, st>>>(g, rdp, x, out);
  else
    gibbs_gradient_cuda_kernel<RDPotCuda, false><<<nb, kGibbsThreads, 0, st>>>(g, rdp, x, out);
  return cudaGetLastError();
}

cudaError_t launch_gibbs_hessian_voxel(const GibbsDev& g, const float* x, int z, int y, int xx, float* out,
                                       cudaStream_t st) {
  const int threads = ((g.wz * g.wy * g.wx + 31) / 32) * 32;
  if (g.potential == 1)
    gibbs_hessian_voxel_kernel<<<1, threads, 0, st>>>(g, QuadPot{}, x, z, y, xx, out);
  else
    gibbs_hessian_voxel_kernel<<<1, threads, 0, st>>>(g, RDPot{g.gamma, g.epsilon}, x, z, y, xx, out);
  return cudaGetLastError();
}

}  // namespace b200
