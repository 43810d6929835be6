// C ABI: Gibbs penalties.
#include "capi.hpp"

using namespace b200;

struct b200rt_gibbs {
  int device = 0;
  GibbsDev d{};
  std::vector<float> host_w;
  DevBuf<double> partial, result;
  int arithmetic = B200RT_GIBBS_ARITH_HOST;
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
    if (op == 1 && g->arithmetic == B200RT_GIBBS_ARITH_CUDA)
      ck(launch_gibbs_gradient_cuda(g->d, x, out, st), "Gibbs penalty");
    else
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

int b200rt_gibbs_set_arithmetic(b200rt_gibbs* g, int arithmetic) {
  if (!g) return B200RT_ERR_INVALID_ARGUMENT;
  if (arithmetic != B200RT_GIBBS_ARITH_HOST && arithmetic != B200RT_GIBBS_ARITH_CUDA)
    return gfail(g, B200RT_ERR_INVALID_ARGUMENT, "unknown Gibbs arithmetic");
  g->arithmetic = arithmetic;
  return B200RT_OK;
}

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
