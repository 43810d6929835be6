// Elementwise parts of the OSMAPOSL sub-iteration on device-resident images, and the
// reductions around the fused forward-projection epilogue.
//
//   viewgram thresholds  divide_and_truncate's small_value per viewgram (recon_array_functions.cxx:185)
//   prior gradient       QuadraticPrior::compute_gradient (QuadraticPrior.cxx:303-372),
//                        RelativeDifferencePrior::compute_gradient (RelativeDifferencePrior.cxx:376-452)
//   update               OSMAPOSLReconstruction::update_estimate (OSMAPOSLReconstruction.cxx:371-516):
//                        division by the (MAP) denominator with divide()'s threshold (numerics/divide.inl:26-48),
//                        threshold_upper_lower, multiplicative update
//
// Images use the device layout [y][x][z] (z fastest).
#include "internal.hpp"

namespace b200 {

namespace {

__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// one block per (segment, view) of the subset: max over the viewgram of y with segment 0 end planes zeroed
__global__ void viewgram_small_value_kernel(const float* __restrict__ y, const SegDev* __restrict__ segs, int S, int num_views,
                                            int num_tang, const int* __restrict__ views, int zero_ends, int64_t tof_stride,
                                            float* __restrict__ out, const int* __restrict__ view_slot) {
  const int seg = static_cast<int>(blockIdx.y) - S;
  const int view = views[blockIdx.x];
  const int tofi = blockIdx.z;
  const SegDev sd = segs[seg + S];
  // the viewgram's block in the data's layout (a view shard holds its views at their slots; the caller lists only
  // held views)
  const int slot = view_slot ? view_slot[view] : view;
  const int64_t base = tofi * tof_stride + sd.dev_offset + static_cast<int64_t>(slot) * num_tang * sd.nax;
  const int n = num_tang * sd.nax;
  float m = -INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int a = i % sd.nax;
    float v = y[base + i];
    if (zero_ends && seg == 0 && (a == 0 || a == sd.nax - 1)) v = 0.f;
    m = fmaxf(m, v);
  }
  __shared__ float red[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
    m = warp_max(m);
    if (threadIdx.x == 0) out[(tofi * (2 * S + 1) + seg + S) * num_views + view] = fmaxf(m * 0.000001F, 0.F);  // SMALL_NUM
  }
}

struct PriorDev {
  int type;
  float beta, gamma, epsilon;
  int dzmin, dzmax;
  float w[27];  // [dz+1][dy+1][dx+1]
  const float* kappa;
};

__device__ __forceinline__ void prior_dev_from(const BatchUpdateDev& f, PriorDev& pr) {
  pr.type = f.prior_type;
  pr.beta = f.beta;
  pr.gamma = f.gamma;
  pr.epsilon = f.epsilon;
  pr.dzmin = f.dzmin;
  pr.dzmax = f.dzmax;
  for (int k = 0; k < 27; ++k) pr.w[k] = f.w[k];
  pr.kappa = f.kappa;
}

// RelativeDifferencePrior::derivative_10 (RelativeDifferencePrior.cxx:287-300)
__device__ __forceinline__ float rdp_derivative_10(float x, float y, float gamma, float epsilon) {
  if (epsilon == 0.0f && x == 0 && y == 0) return 0.f;
  const double num = static_cast<double>(x - y) * (gamma * fabsf(x - y) + x + 3 * y + 2 * epsilon);
  const double ds = static_cast<double>(x + y) + gamma * fabsf(x - y) + epsilon;
  return static_cast<float>(num / (ds * ds));
}

// prior gradient of one voxel (double accumulation as STIR), device layout indices
__device__ __forceinline__ float prior_gradient_at(const float* __restrict__ x, const PriorDev& pr, int yi, int xi, int zi,
                                                   int ny, int nx, int nz) {
  const int64_t i = (static_cast<int64_t>(yi) * nx + xi) * nz + zi;
  const float xc = x[i];
  double g = 0.0;
  const int dz0 = max(pr.dzmin, -zi), dz1 = min(pr.dzmax, nz - 1 - zi);
  const int dy0 = max(-1, -yi), dy1 = min(1, ny - 1 - yi);
  const int dx0 = max(-1, -xi), dx1 = min(1, nx - 1 - xi);
  for (int dz = dz0; dz <= dz1; ++dz)
    for (int dy = dy0; dy <= dy1; ++dy)
      for (int dx = dx0; dx <= dx1; ++dx) {
        const int64_t j = i + (static_cast<int64_t>(dy) * nx + dx) * nz + dz;
        const float xn = x[j];
        const float w = pr.w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
        double cur = (pr.type == 1) ? static_cast<double>(w * (xc - xn)) : static_cast<double>(w * rdp_derivative_10(xc, xn, pr.gamma, pr.epsilon));
        if (pr.kappa) cur *= pr.kappa[i] * pr.kappa[j];
        g += cur;
      }
  return static_cast<float>(g * pr.beta);
}

// pass 1: per-block max of the update image u, and the prior gradient (if any) into g
__device__ __forceinline__ void update_prepare_body(int blk, int nblk, const float* __restrict__ u,
                                                    const float* __restrict__ x, float* __restrict__ g, const PriorDev& pr,
                                                    int ny, int nx, int nz, float* __restrict__ partial_max) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  float m = -INFINITY;
  for (int64_t i = blk * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<int64_t>(nblk) * blockDim.x) {
    m = fmaxf(m, u[i]);
    if (pr.type != 0) {
      const int zi = static_cast<int>(i % nz);
      const int64_t c = i / nz;
      const int xi = static_cast<int>(c % nx), yi = static_cast<int>(c / nx);
      g[i] = prior_gradient_at(x, pr, yi, xi, zi, ny, nx, nz);
    }
  }
  __shared__ float red[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
    m = warp_max(m);
    if (threadIdx.x == 0) partial_max[blk] = m;
  }
}

__global__ void update_prepare_kernel(const float* __restrict__ u, const float* __restrict__ x, float* __restrict__ g, PriorDev pr,
                                      int ny, int nx, int nz, float* __restrict__ partial_max) {
  update_prepare_body(blockIdx.x, gridDim.x, u, x, g, pr, ny, nx, nz, partial_max);
}

__device__ __forceinline__ void reduce_max_body(const float* __restrict__ partial, int n, float* __restrict__ out) {
  float m = -INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, partial[i]);
  __shared__ float red[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
    m = warp_max(m);
    if (threadIdx.x == 0) *out = m;
  }
}

__global__ void reduce_max_kernel(const float* __restrict__ partial, int n, float* __restrict__ out) {
  reduce_max_body(partial, n, out);
}

// pass 2: u /= denominator with divide()'s threshold, clamp, x *= u -- one voxel
__device__ __forceinline__ void update_apply_one(float& uv, float& xv, float s, float gv, int prior, int map_model,
                                                 float num_subsets, float sv, int clamp, float min_rel, float max_rel) {
  float den;
  if (!prior) {
    den = s;
  } else if (map_model == 0) {
    // additive MAP model (OSMAPOSLReconstruction.cxx:415-433)
    den = gv / num_subsets + s;
    den = fmaxf(fminf(den, s * 10), s / 10);
  } else {
    // multiplicative MAP model (:436-453)
    den = gv + 1;
    den = fmaxf(fminf(den, 10.F), 1 / 10.F);
    den *= s;
  }
  float v = uv;
  if (fabsf(den) <= sv && fabsf(v) <= sv)
    v = 0;
  else
    v /= den;
  if (clamp) {
    // threshold_upper_lower (thresholding.h:45-54)
    if (v > max_rel)
      v = max_rel;
    else if (min_rel > v)
      v = min_rel;
  }
  uv = v;
  xv *= v;
}

// pass 2 over the image: 16-byte loads and stores where every array allows them (elementwise, so the same results)
__device__ __forceinline__ void update_apply_body(int blk, int nblk, float* __restrict__ u, float* __restrict__ x,
                                                  const float* __restrict__ sens, const float* __restrict__ g, int prior,
                                                  int map_model, float num_subsets, const float* __restrict__ umax,
                                                  float small_num, int clamp, float min_rel, float max_rel, int64_t n) {
  // divide()'s threshold small_num x max(u); without a prior small_num is 0 and max(u) is not needed (or computed)
  float sv = 0.f;
  if (small_num > 0.f) {
    sv = *umax * small_num;
    sv = sv > 0 ? sv : 0;
  }
  const int64_t stride = static_cast<int64_t>(nblk) * blockDim.x;
  const int64_t t0 = blk * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const uintptr_t al = reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(x) |
                       reinterpret_cast<uintptr_t>(sens) | (prior ? reinterpret_cast<uintptr_t>(g) : 0);
  int64_t i0 = 0;
  if ((al & 15) == 0) {
    const int64_t n4 = n / 4;
    float4* u4 = reinterpret_cast<float4*>(u);
    float4* x4 = reinterpret_cast<float4*>(x);
    const float4* s4 = reinterpret_cast<const float4*>(sens);
    const float4* g4 = reinterpret_cast<const float4*>(g);
    for (int64_t i = t0; i < n4; i += stride) {
      float4 U = u4[i], X = x4[i];
      const float4 S = s4[i];
      const float4 G = prior ? g4[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      update_apply_one(U.x, X.x, S.x, G.x, prior, map_model, num_subsets, sv, clamp, min_rel, max_rel);
      update_apply_one(U.y, X.y, S.y, G.y, prior, map_model, num_subsets, sv, clamp, min_rel, max_rel);
      update_apply_one(U.z, X.z, S.z, G.z, prior, map_model, num_subsets, sv, clamp, min_rel, max_rel);
      update_apply_one(U.w, X.w, S.w, G.w, prior, map_model, num_subsets, sv, clamp, min_rel, max_rel);
      u4[i] = U;
      x4[i] = X;
    }
    i0 = n4 * 4;
  }
  for (int64_t i = i0 + t0; i < n; i += stride) {
    float uv = u[i], xv = x[i];
    update_apply_one(uv, xv, sens[i], prior ? g[i] : 0.f, prior, map_model, num_subsets, sv, clamp, min_rel, max_rel);
    u[i] = uv;
    x[i] = xv;
  }
}

__global__ void update_apply_kernel(float* __restrict__ u, float* __restrict__ x, const float* __restrict__ sens,
                                    const float* __restrict__ g, int prior, int map_model, float num_subsets,
                                    const float* __restrict__ umax, float small_num, int clamp, float min_rel, float max_rel,
                                    int64_t n) {
  update_apply_body(blockIdx.x, gridDim.x, u, x, sens, g, prior, map_model, num_subsets, umax, small_num, clamp, min_rel,
                    max_rel, n);
}

// the same three passes for several frames in one launch each (grid.y = frame); every frame keeps the block
// count of its own launch, so the results are those of launch_update frame by frame
__global__ void batch_update_prepare_kernel(const BatchUpdateDev* __restrict__ frames) {
  const BatchUpdateDev& f = frames[blockIdx.y];
  // frames without a prior need neither the prior gradient nor max(u) (divide()'s threshold is 0 for them)
  if (static_cast<int>(blockIdx.x) >= f.nblocks || f.prior_type == 0) return;
  PriorDev pr;
  prior_dev_from(f, pr);
  update_prepare_body(blockIdx.x, f.nblocks, f.u, f.x, f.g, pr, f.ny, f.nx, f.nz, f.partial_max);
}
__global__ void batch_reduce_max_kernel(const BatchUpdateDev* __restrict__ frames) {
  const BatchUpdateDev& f = frames[blockIdx.x];
  if (f.prior_type == 0) return;
  reduce_max_body(f.partial_max, f.nblocks, f.umax);
}
__global__ void batch_update_apply_kernel(const BatchUpdateDev* __restrict__ frames) {
  const BatchUpdateDev& f = frames[blockIdx.y];
  if (static_cast<int>(blockIdx.x) >= f.nblocks) return;
  update_apply_body(blockIdx.x, f.nblocks, f.u, f.x, f.sens, f.g, f.prior, f.map_model, f.num_subsets, f.umax,
                    f.small_num, f.clamp, f.min_rel, f.max_rel, static_cast<int64_t>(f.ny) * f.nx * f.nz);
}

__global__ void reduce_sum_kernel(const double* __restrict__ partial, int n, double* __restrict__ out) {
  // one block, fixed order per thread and a fixed tree: deterministic
  __shared__ double red[256];
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t += partial[i];
  red[threadIdx.x] = t;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// RelativeDifferencePrior::value (RelativeDifferencePrior.cxx:278-285)
__device__ __forceinline__ double rdp_value(float x, float y, float gamma, float epsilon) {
  const double d = static_cast<double>(x - y);
  return 0.5 * (d * d / (x + y + gamma * fabsf(x - y) + epsilon));
}

// per-block FP64 partial sums of the prior value over voxels (grid-stride, fixed assignment: deterministic)
__global__ void prior_value_kernel(const float* __restrict__ x, PriorDev pr, int ny, int nx, int nz,
                                   double* __restrict__ partial) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  double t = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int zi = static_cast<int>(i % nz);
    const int64_t c = i / nz;
    const int xi = static_cast<int>(c % nx), yi = static_cast<int>(c / nx);
    const float xc = x[i];
    const int dz0 = max(pr.dzmin, -zi), dz1 = min(pr.dzmax, nz - 1 - zi);
    const int dy0 = max(-1, -yi), dy1 = min(1, ny - 1 - yi);
    const int dx0 = max(-1, -xi), dx1 = min(1, nx - 1 - xi);
    for (int dz = dz0; dz <= dz1; ++dz)
      for (int dy = dy0; dy <= dy1; ++dy)
        for (int dx = dx0; dx <= dx1; ++dx) {
          const int64_t j = i + (static_cast<int64_t>(dy) * nx + dx) * nz + dz;
          const float xn = x[j];
          const float w = pr.w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
          double cur;
          if (pr.type == 1) {
            const float d = xc - xn;
            cur = static_cast<double>(w * (d * d) / 4);  // QuadraticPrior.cxx:283-286 (float expression)
          } else if (pr.epsilon == 0.0f && xc == 0.0f && xn == 0.0f) {
            cur = 0.0;
          } else {
            cur = w * rdp_value(xc, xn, pr.gamma, pr.epsilon);  // RelativeDifferencePrior.cxx:340-349
          }
          if (pr.kappa) cur *= pr.kappa[i] * pr.kappa[j];
          t += cur;
        }
  }
  __shared__ double red[256];
  red[threadIdx.x] = t;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// per-block max |x| (data == nullptr stands for ones)
__global__ void absmax_kernel(const float* __restrict__ data, int64_t n, float* __restrict__ partial) {
  float m = 0.f;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    m = fmaxf(m, data ? fabsf(data[i]) : 1.f);
  __shared__ float red[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    m = warp_max(m);
    if (threadIdx.x == 0) partial[blockIdx.x] = m;
  }
}

// scale = 2^floor(62 - log2(bound)): every partial sum of |w d| over a voxel is at most
// max|d| * max column sum of A, so the int64 accumulator cannot overflow.  The exponent is capped at 126 so that
// the scale is also a normal float (data whose bound is under 2^-64 keep 62 bits above 2^-126)
__global__ void fixed_scale_kernel(const float* __restrict__ partial, int n, const float* __restrict__ colmax,
                                   double* __restrict__ scale) {
  float m = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, partial[i]);
  __shared__ float red[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (blockDim.x >> 5); ++w) t = fmaxf(t, red[w]);
    const double bound = static_cast<double>(t) * static_cast<double>(*colmax) * 1.01 + 1e-30;
    *scale = exp2(fmin(floor(62.0 - log2(bound)), 126.0));
  }
}

__global__ void fixed_to_float_kernel(const unsigned long long* __restrict__ acc, const double* __restrict__ scale,
                                      float* __restrict__ img, int64_t n) {
  const double inv = 1.0 / *scale;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    img[i] = static_cast<float>(static_cast<double>(static_cast<long long>(acc[i])) * inv);
}

}  // namespace

cudaError_t launch_max(const float* data, int64_t n, float* partial, float* out, cudaStream_t st) {
  const int blocks = update_num_blocks(n);
  absmax_kernel<<<blocks, 256, 0, st>>>(data, n, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  reduce_max_kernel<<<1, 1024, 0, st>>>(partial, blocks, out);
  return cudaGetLastError();
}

cudaError_t launch_fixed_scale(const float* projdata, int64_t n, const float* colmax, float* partial, double* scale,
                               cudaStream_t st) {
  const int blocks = update_num_blocks(n);
  absmax_kernel<<<blocks, 256, 0, st>>>(projdata, n, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  fixed_scale_kernel<<<1, 1024, 0, st>>>(partial, blocks, colmax, scale);
  return cudaGetLastError();
}

cudaError_t launch_fixed_to_float(const unsigned long long* acc, const double* scale, float* image, int64_t n,
                                  cudaStream_t st) {
  fixed_to_float_kernel<<<update_num_blocks(n), 256, 0, st>>>(acc, scale, image, n);
  return cudaGetLastError();
}

// BinNormalisationFromAttenuationImage (BinNormalisationFromAttenuationImage.cxx:138-170) given the line
// integrals A mu: apply multiplies by exp(A mu), undo divides by it; factors = undo of ones
__global__ void attenuation_kernel(const float* __restrict__ line_integrals, float* __restrict__ pd, int64_t n,
                                   int mode) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float e = expf(line_integrals[i]);
    if (mode == B200RT_ATTENUATION_FACTORS)
      pd[i] = 1.F / e;
    else if (mode == B200RT_ATTENUATION_APPLY)
      pd[i] *= e;
    else
      pd[i] /= e;
  }
}

// BinNormalisationFromProjData (BinNormalisationFromProjData.cxx:131-150): apply multiplies by the factors, undo
// divides by them (no guard, as the viewgram division); factors of non-TOF data serve every timing bin (period
// fstride), factors = undo of ones
__global__ void norm_projdata_kernel(const float* __restrict__ f, float* __restrict__ pd, int64_t n, int64_t fstride,
                                     int mode) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float v = f[fstride > 0 ? i % fstride : i];
    if (mode == B200RT_NORM_FACTORS)
      pd[i] = 1.F / v;
    else if (mode == B200RT_NORM_APPLY)
      pd[i] *= v;
    else
      pd[i] /= v;
  }
}

cudaError_t launch_norm_projdata(const float* factors, float* projdata, int64_t n, int64_t fstride, int mode,
                                 cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  norm_projdata_kernel<<<update_num_blocks(n), 256, 0, st>>>(factors, projdata, n, fstride, mode);
  return cudaGetLastError();
}

cudaError_t launch_attenuation(const float* line_integrals, float* projdata, int64_t n, int mode, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  attenuation_kernel<<<update_num_blocks(n), 256, 0, st>>>(line_integrals, projdata, n, mode);
  return cudaGetLastError();
}

// ---- prior Hessian times an image (QuadraticPrior.cxx:603-688, RelativeDifferencePrior.cxx:535-621) ----

namespace {

// RelativeDifferencePrior::derivative_20 / derivative_11 (RelativeDifferencePrior.cxx:623-641): the powers of
// the float arguments are taken in double (STIR's pow(float, int)), the quotient returned as float
__device__ __forceinline__ float rdp_derivative_20(float xj, float xk, float gamma, float epsilon) {
  if (xj > 0.0f || xk > 0.0f || epsilon > 0.0f) {
    const double a = static_cast<double>(2 * xk + epsilon);
    const double b = static_cast<double>(xj + xk + gamma * fabsf(xj - xk) + epsilon);
    return static_cast<float>(2 * (a * a) / (b * b * b));
  }
  return INFINITY;
}
__device__ __forceinline__ float rdp_derivative_11(float xj, float xk, float gamma, float epsilon) {
  if (xj > 0.0f || xk > 0.0f || epsilon > 0.0f) {
    const float num = -2 * (2 * xj + epsilon) * (2 * xk + epsilon);
    const double b = static_cast<double>(xj + xk + gamma * fabsf(xj - xk) + epsilon);
    return static_cast<float>(num / (b * b * b));
  }
  return INFINITY;
}

__global__ void hessian_times_input_kernel(float* __restrict__ out, const float* __restrict__ x,
                                           const float* __restrict__ in, PriorDev pr, int ny, int nx, int nz) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int zi = static_cast<int>(i % nz);
    const int64_t c = i / nz;
    const int xi = static_cast<int>(c % nx), yi = static_cast<int>(c / nx);
    const int dz0 = max(pr.dzmin, -zi), dz1 = min(pr.dzmax, nz - 1 - zi);
    const int dy0 = max(-1, -yi), dy1 = min(1, ny - 1 - yi);
    const int dx0 = max(-1, -xi), dx1 = min(1, nx - 1 - xi);
    const float xj = x[i], inj = in[i];
    float result = 0.f;
    for (int dz = dz0; dz <= dz1; ++dz)
      for (int dy = dy0; dy <= dy1; ++dy)
        for (int dx = dx0; dx <= dx1; ++dx) {
          float current = pr.w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
          if (current == 0.f) continue;
          const int64_t k = i + (static_cast<int64_t>(dy) * nx + dx) * nz + dz;
          float f20, f11;
          if (pr.type == B200RT_PRIOR_QUADRATIC) {
            f20 = 1.0f;
            f11 = -1.0f;
          } else {
            f20 = rdp_derivative_20(xj, x[k], pr.gamma, pr.epsilon);
            f11 = rdp_derivative_11(xj, x[k], pr.gamma, pr.epsilon);
          }
          if (dz == 0 && dy == 0 && dx == 0)
            current *= f20 * inj;
          else
            current *= (f20 * inj + f11 * in[k]);
          if (pr.kappa) current *= pr.kappa[i] * pr.kappa[k];
          result += current;
        }
    out[i] += result * pr.beta;
  }
}

}  // namespace

cudaError_t launch_prior_hessian_times_input(float* out, const float* x, const float* in, const b200rt_prior* prior,
                                             const float prior_weights[27], int ny, int nx, int nz, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  if (!prior || prior->type == B200RT_PRIOR_NONE || prior->penalisation_factor == 0 || n <= 0) return cudaSuccess;
  PriorDev pr{};
  pr.type = prior->type;
  pr.beta = prior->penalisation_factor;
  pr.gamma = prior->gamma;
  pr.epsilon = prior->epsilon;
  pr.dzmin = prior->only_2D ? 0 : -1;
  pr.dzmax = prior->only_2D ? 0 : 1;
  for (int k = 0; k < 27; ++k) pr.w[k] = prior_weights[k];
  pr.kappa = prior->kappa_dev;
  hessian_times_input_kernel<<<update_num_blocks(n), 256, 0, st>>>(out, x, in, pr, ny, nx, nz);
  return cudaGetLastError();
}

// ---- OSSPS (OSSPSReconstruction.cxx) ----------------------------------------------------------------

namespace {

__global__ void fill_kernel(float* __restrict__ p, int64_t n, float v) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = v;
}

// one block per (segment, view) of the data: divide_and_truncate(A 1, (y n) n) in place on the forward
// projection (...AndProjData.cxx:1021-1046), small value from the forward projection's viewgram maximum
__global__ void hessian_ratio_kernel(float* __restrict__ fp, const float* __restrict__ y, const float* __restrict__ norm,
                                     const SegDev* __restrict__ segs, int S, int num_views, int num_tang,
                                     const int* __restrict__ views, int64_t tof_stride,
                                     const float* __restrict__ small_value) {
  const int seg = static_cast<int>(blockIdx.y) - S;
  const int view = views[blockIdx.x];
  const int tofi = blockIdx.z;
  const SegDev sd = segs[seg + S];
  const int64_t base = tofi * tof_stride + sd.dev_offset + static_cast<int64_t>(view) * num_tang * sd.nax;
  const int n = num_tang * sd.nax;
  const float sv = small_value[(tofi * (2 * S + 1) + seg + S) * num_views + view];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float num = fp[base + i];
    float den = y[base + i];
    if (norm) {
      den *= norm[base + i];
      den *= norm[base + i];
    }
    if (num <= sv)
      num = 0.f;
    else
      num = (num > 10000.F * den) ? 10000.F : num / den;
    fp[base + i] = num;
  }
}

// x = 0 where the sensitivity is 0 (fill_nonidentifiable_target_parameters,
// PoissonLogLikelihoodWithLinearModelForMean.cxx:459-471)
__global__ void zero_unidentifiable_kernel(float* __restrict__ x, const float* __restrict__ sens, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (sens[i] == 0) x[i] = 0.f;
}

// den = curvature * 2 + den with the Quadratic prior's parabolic surrogate curvature
// (QuadraticPrior.cxx:460-522; OSSPSReconstruction.cxx:330-339), and the block minimum of its positive values
__global__ void ossps_denominator_kernel(float* __restrict__ den, PriorDev pr, int ny, int nx, int nz,
                                         float* __restrict__ partial_min) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  float m = INFINITY;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float d = den[i];
    if (pr.type != 0) {
      const int zi = static_cast<int>(i % nz);
      const int64_t c = i / nz;
      const int xi = static_cast<int>(c % nx), yi = static_cast<int>(c / nx);
      const int dz0 = max(pr.dzmin, -zi), dz1 = min(pr.dzmax, nz - 1 - zi);
      const int dy0 = max(-1, -yi), dy1 = min(1, ny - 1 - yi);
      const int dx0 = max(-1, -xi), dx1 = min(1, nx - 1 - xi);
      float cv = 0.f;
      for (int dz = dz0; dz <= dz1; ++dz)
        for (int dy = dy0; dy <= dy1; ++dy)
          for (int dx = dx0; dx <= dx1; ++dx) {
            float cur = pr.w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] * 1;
            if (pr.kappa) {
              const int64_t j = i + (static_cast<int64_t>(dy) * nx + dx) * nz + dz;
              cur *= pr.kappa[i] * pr.kappa[j];
            }
            cv += cur;
          }
      d = (cv * pr.beta) * 2 + d;
      den[i] = d;
    }
    if (d > 0) m = fminf(m, d);
  }
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : INFINITY;
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) partial_min[blockIdx.x] = m;
  }
}

__global__ void reduce_min_kernel(const float* __restrict__ partial, int n, float* __restrict__ out) {
  float m = INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fminf(m, partial[i]);
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : INFINITY;
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) *out = m;
  }
}

// threshold_min_to_small_positive_value(den, small) (thresholding.h:99-109) given the smallest positive value
__global__ void threshold_small_positive_kernel(float* __restrict__ den, int64_t n, const float* __restrict__ minpos,
                                                float small) {
  const float mp = *minpos;
  const bool none = !(mp < INFINITY);
  const float lo = mp * small;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (none)
      den[i] = small;
    else if (den[i] < lo)
      den[i] = lo;
  }
}

// the update of OSSPSReconstruction::update_estimate (:314-407) given the sub-gradient g, the prior gradient pg
// (or nullptr) and the denominator
__global__ void ossps_update_kernel(float* __restrict__ x, const float* __restrict__ g, const float* __restrict__ pg,
                                    const float* __restrict__ den, int64_t n, int num_subsets, float relax,
                                    float upper) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float num = g[i];
    if (pg) num -= pg[i] / num_subsets;
    num = num * num_subsets;
    num = num / den[i];
    num = num * relax * 1.F;
    float v = x[i] + num;
    if (v > upper)
      v = upper;
    else if (0.F > v)
      v = 0.F;
    x[i] = v;
  }
}

}  // namespace

cudaError_t launch_zero_unidentifiable(float* x, const float* sens, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  zero_unidentifiable_kernel<<<update_num_blocks(n), 256, 0, st>>>(x, sens, n);
  return cudaGetLastError();
}

cudaError_t launch_fill(float* p, int64_t n, float v, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  fill_kernel<<<update_num_blocks(n), 256, 0, st>>>(p, n, v);
  return cudaGetLastError();
}

cudaError_t launch_hessian_ratio(float* fp, const float* y, const float* norm, const SegDev* segs, int S, int num_views,
                                 int num_tang, const int* views, int nviews, int num_tof, int64_t tof_stride,
                                 const float* small_value, cudaStream_t st) {
  if (nviews <= 0) return cudaSuccess;
  hessian_ratio_kernel<<<dim3(nviews, 2 * S + 1, num_tof), 256, 0, st>>>(fp, y, norm, segs, S, num_views, num_tang, views,
                                                                          tof_stride, small_value);
  return cudaGetLastError();
}

cudaError_t launch_ossps_update(float* x, float* den, const float* g, float* pg, const float* sens, const b200rt_prior* prior,
                                const float prior_weights[27], int ny, int nx, int nz, int num_subsets, int first,
                                float relax, float upper, float* partial, float* minpos, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  const int blocks = update_num_blocks(n);
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  PriorDev pr{};
  if (has_prior) {
    pr.type = prior->type;
    pr.beta = prior->penalisation_factor;
    pr.gamma = prior->gamma;
    pr.epsilon = prior->epsilon;
    pr.dzmin = prior->only_2D ? 0 : -1;
    pr.dzmax = prior->only_2D ? 0 : 1;
    for (int k = 0; k < 27; ++k) pr.w[k] = prior_weights[k];
    pr.kappa = prior->kappa_dev;
  }
  cudaError_t e;
  (void)sens;
  if (has_prior) {
    update_prepare_kernel<<<blocks, 256, 0, st>>>(x, x, pg, pr, ny, nx, nz, partial);  // prior gradient into pg
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (first) {
    PriorDev pc = pr;  // the curvature term is added for the Quadratic prior only
    if (pc.type != B200RT_PRIOR_QUADRATIC) pc.type = 0;
    ossps_denominator_kernel<<<blocks, 256, 0, st>>>(den, pc, ny, nx, nz, partial);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    reduce_min_kernel<<<1, 1024, 0, st>>>(partial, blocks, minpos);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    threshold_small_positive_kernel<<<blocks, 256, 0, st>>>(den, n, minpos, 10.E-6F);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  ossps_update_kernel<<<blocks, 256, 0, st>>>(x, g, has_prior ? pg : nullptr, den, n, num_subsets, relax, upper);
  return cudaGetLastError();
}

cudaError_t launch_viewgram_small_values(const float* y, const SegDev* segs, int S, int num_views, int num_tang,
                                         const int* views, int nviews, int zero_ends, int num_tof, int64_t tof_stride,
                                         float* out, cudaStream_t st, const int* view_slot) {
  if (nviews <= 0) return cudaSuccess;
  viewgram_small_value_kernel<<<dim3(nviews, 2 * S + 1, num_tof), 256, 0, st>>>(y, segs, S, num_views, num_tang, views,
                                                                                  zero_ends, tof_stride, out, view_slot);
  return cudaGetLastError();
}

int update_num_blocks(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return static_cast<int>(b < 148 * 16 ? b : 148 * 16);
}

cudaError_t launch_update(float* u, float* x, const float* sens, float* g, const b200rt_prior* prior,
                          const float prior_weights[27], int num_subsets, int subiteration_num, float min_rel, float max_rel,
                          int ny, int nx, int nz, float* partial_max, float* umax, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  const int blocks = update_num_blocks(n);
  PriorDev pr{};
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  pr.type = has_prior ? prior->type : 0;
  if (has_prior) {
    pr.beta = prior->penalisation_factor;
    pr.gamma = prior->gamma;
    pr.epsilon = prior->epsilon;
    pr.dzmin = prior->only_2D ? 0 : -1;
    pr.dzmax = prior->only_2D ? 0 : 1;
    for (int k = 0; k < 27; ++k) pr.w[k] = prior_weights[k];
    pr.kappa = prior->kappa_dev;
  }
  cudaError_t e;
  if (has_prior) {  // the prior gradient and max(u) for divide()'s threshold (0 without a prior: not needed)
    update_prepare_kernel<<<blocks, 256, 0, st>>>(u, x, g, pr, ny, nx, nz, partial_max);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    reduce_max_kernel<<<1, 1024, 0, st>>>(partial_max, blocks, umax);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  update_apply_kernel<<<blocks, 256, 0, st>>>(u, x, sens, g, has_prior ? 1 : 0, has_prior ? prior->map_model : 0,
                                               static_cast<float>(num_subsets), umax, has_prior ? 0.000001F : 0.F,
                                               subiteration_num != 1, min_rel, max_rel, n);
  return cudaGetLastError();
}

void fill_batch_update(BatchUpdateDev& d, float* u, float* x, const float* sens, float* g, const b200rt_prior* prior,
                       const float prior_weights[27], int num_subsets, int subiteration_num, float min_rel, float max_rel,
                       int ny, int nx, int nz, float* partial_max, float* umax) {
  d = BatchUpdateDev{};
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  d.u = u;
  d.x = x;
  d.sens = sens;
  d.g = has_prior ? g : nullptr;
  d.prior_type = has_prior ? prior->type : 0;
  if (has_prior) {
    d.beta = prior->penalisation_factor;
    d.gamma = prior->gamma;
    d.epsilon = prior->epsilon;
    d.dzmin = prior->only_2D ? 0 : -1;
    d.dzmax = prior->only_2D ? 0 : 1;
    for (int k = 0; k < 27; ++k) d.w[k] = prior_weights[k];
    d.kappa = prior->kappa_dev;
  }
  d.ny = ny;
  d.nx = nx;
  d.nz = nz;
  d.nblocks = update_num_blocks(static_cast<int64_t>(ny) * nx * nz);
  d.partial_max = partial_max;
  d.umax = umax;
  d.prior = has_prior ? 1 : 0;
  d.map_model = has_prior ? prior->map_model : 0;
  d.num_subsets = static_cast<float>(num_subsets);
  d.small_num = has_prior ? 0.000001F : 0.F;
  d.clamp = subiteration_num != 1;
  d.min_rel = min_rel;
  d.max_rel = max_rel;
}

cudaError_t launch_batch_update(const BatchUpdateDev* frames_dev, int nframes, int max_blocks, bool any_prior,
                                cudaStream_t st) {
  if (nframes <= 0) return cudaSuccess;
  cudaError_t e;
  if (any_prior) {  // prior gradients and max(u) of the frames with a prior
    batch_update_prepare_kernel<<<dim3(max_blocks, nframes), 256, 0, st>>>(frames_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    batch_reduce_max_kernel<<<nframes, 1024, 0, st>>>(frames_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  batch_update_apply_kernel<<<dim3(max_blocks, nframes), 256, 0, st>>>(frames_dev);
  return cudaGetLastError();
}

cudaError_t launch_prior_gradient(const float* x, float* g, const b200rt_prior* prior, const float prior_weights[27], int ny,
                                  int nx, int nz, float* partial_max, cudaStream_t st) {
  const int64_t n = static_cast<int64_t>(ny) * nx * nz;
  PriorDev pr{};
  pr.type = prior->type;
  pr.beta = prior->penalisation_factor;
  pr.gamma = prior->gamma;
  pr.epsilon = prior->epsilon;
  pr.dzmin = prior->only_2D ? 0 : -1;
  pr.dzmax = prior->only_2D ? 0 : 1;
  for (int k = 0; k < 27; ++k) pr.w[k] = prior_weights[k];
  pr.kappa = prior->kappa_dev;
  update_prepare_kernel<<<update_num_blocks(n), 256, 0, st>>>(x, x, g, pr, ny, nx, nz, partial_max);
  return cudaGetLastError();
}

cudaError_t launch_prior_value(const float* x, const b200rt_prior* prior, const float prior_weights[27], int ny, int nx,
                               int nz, double* partial, int npartial, double* out, cudaStream_t st) {
  PriorDev pr{};
  pr.type = prior->type;
  pr.beta = prior->penalisation_factor;
  pr.gamma = prior->gamma;
  pr.epsilon = prior->epsilon;
  pr.dzmin = prior->only_2D ? 0 : -1;
  pr.dzmax = prior->only_2D ? 0 : 1;
  for (int k = 0; k < 27; ++k) pr.w[k] = prior_weights[k];
  pr.kappa = prior->kappa_dev;
  prior_value_kernel<<<npartial, 256, 0, st>>>(x, pr, ny, nx, nz, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  reduce_sum_kernel<<<1, 256, 0, st>>>(partial, npartial, out);
  return cudaGetLastError();
}

cudaError_t launch_reduce_sum(const double* partial, int n, double* out, cudaStream_t st) {
  reduce_sum_kernel<<<1, 256, 0, st>>>(partial, n, out);
  return cudaGetLastError();
}

}  // namespace b200
