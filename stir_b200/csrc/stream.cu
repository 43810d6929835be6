// Projection data in a stream (a file's bytes already copied to the device) <-> the device layout: the element
// addressing of ProjDataFromStream::get_offset (src/buildblock/ProjDataFromStream.cxx:415-500) for the
// Segment_AxialPos_View_TangPos and Segment_View_AxialPos_TangPos storage orders (and their Timing_ variants),
// with the number type, byte order and scale factor of the stream.  One segment (and timing position) per launch
// group: a tiled transpose from the stream's [axial][view, tangential] (or, per view, [axial][tangential]) rows
// to the device layout's [view, tangential][axial], staged in shared memory so that both sides are coalesced.
// Elements are read byte by byte, so a stream of any alignment is safe.
#include "internal.hpp"

namespace b200 {

namespace {

__device__ __forceinline__ uint64_t load_bytes(const unsigned char* p, int size, bool swap) {
  uint64_t v = 0;
  for (int b = 0; b < size; ++b) {
    const uint64_t byte = p[swap ? size - 1 - b : b];
    v |= byte << (8 * b);
  }
  return v;
}

// one element of the stream as float (NumericType conversion as a C++ cast, then times the scale factor)
__device__ __forceinline__ float stream_value(const unsigned char* p, int type, bool swap, float scale) {
  switch (type) {
    case kNumSChar: return static_cast<float>(static_cast<signed char>(p[0])) * scale;
    case kNumUChar: return static_cast<float>(p[0]) * scale;
    case kNumShort: return static_cast<float>(static_cast<int16_t>(load_bytes(p, 2, swap))) * scale;
    case kNumUShort: return static_cast<float>(static_cast<uint16_t>(load_bytes(p, 2, swap))) * scale;
    case kNumInt: return static_cast<float>(static_cast<int32_t>(load_bytes(p, 4, swap))) * scale;
    case kNumUInt: return static_cast<float>(static_cast<uint32_t>(load_bytes(p, 4, swap))) * scale;
    case kNumFloat: return __uint_as_float(static_cast<uint32_t>(load_bytes(p, 4, swap))) * scale;
    default: return static_cast<float>(__longlong_as_double(static_cast<long long>(load_bytes(p, 8, swap)))) * scale;
  }
}

__device__ __forceinline__ void store_value(unsigned char* p, float v, int type, bool swap) {
  uint64_t bits;
  int size;
  if (type == kNumFloat) {
    bits = __float_as_uint(v);
    size = 4;
  } else {
    bits = static_cast<uint64_t>(__double_as_longlong(static_cast<double>(v)));
    size = 8;
  }
  for (int b = 0; b < size; ++b) p[swap ? size - 1 - b : b] = static_cast<unsigned char>(bits >> (8 * b));
}

// batch z of rows x cols: stream element (r, c) at in_elem + z * in_batch + r * ld_in + c <-> device value at
// out + z * out_batch + c * rows + r
__global__ void stream_to_dev_kernel(const unsigned char* __restrict__ in, int64_t in_elem, int64_t in_batch,
                                     int64_t ld_in, int type, int size, int swap, float scale, float* __restrict__ out,
                                     int64_t out_batch, int rows, int cols) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int64_t zi = in_elem + static_cast<int64_t>(blockIdx.z) * in_batch;
  float* o = out + static_cast<int64_t>(blockIdx.z) * out_batch;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols)
      tile[i][threadIdx.x] = stream_value(in + (zi + static_cast<int64_t>(r) * ld_in + c) * size, type, swap != 0, scale);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) o[static_cast<int64_t>(c) * rows + r] = tile[threadIdx.x][i];
  }
}

__global__ void dev_to_stream_kernel(const float* __restrict__ in, int64_t in_batch, int type, int size, int swap,
                                     unsigned char* __restrict__ out, int64_t out_elem, int64_t out_batch,
                                     int64_t ld_out, int rows, int cols) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const float* src = in + static_cast<int64_t>(blockIdx.z) * in_batch;
  const int64_t zo = out_elem + static_cast<int64_t>(blockIdx.z) * out_batch;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) tile[threadIdx.x][i] = src[static_cast<int64_t>(c) * rows + r];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) store_value(out + (zo + static_cast<int64_t>(r) * ld_out + c) * size, tile[i][threadIdx.x], type, swap != 0);
  }
}

}  // namespace

int numeric_type_size(int type) {
  switch (type) {
    case kNumSChar:
    case kNumUChar: return 1;
    case kNumShort:
    case kNumUShort: return 2;
    case kNumInt:
    case kNumUInt:
    case kNumFloat: return 4;
    case kNumDouble: return 8;
    default: return 0;
  }
}

cudaError_t launch_stream_segment(const StreamSegment& s, bool to_dev, const void* in, void* out, cudaStream_t st) {
  const int size = numeric_type_size(s.type);
  // segment_axial_view_tang: one (nax) x (nv nt) transpose; segment_view_axial_tang: nv transposes of nax x nt
  const bool savt = s.order == kStorageSegmentAxialViewTang;
  const int rows = s.nax;
  const int cols = savt ? s.nv * s.nt : s.nt;
  const int batches = savt ? 1 : s.nv;
  const int64_t ld = savt ? static_cast<int64_t>(s.nv) * s.nt : s.nt;
  const int64_t sbatch = static_cast<int64_t>(s.nax) * s.nt;  // stream elements per view (view-major order)
  const int64_t dbatch = static_cast<int64_t>(s.nt) * s.nax;  // device floats per view
  const dim3 grid((cols + 31) / 32, (rows + 31) / 32, batches);
  if (grid.y > 65535 || batches > 65535) return cudaErrorInvalidValue;
  if (to_dev)
    stream_to_dev_kernel<<<grid, dim3(32, 8), 0, st>>>(static_cast<const unsigned char*>(in), s.stream_elem, sbatch, ld,
                                                      s.type, size, s.swap, s.scale, static_cast<float*>(out) + s.dev_off,
                                                      dbatch, rows, cols);
  else
    dev_to_stream_kernel<<<grid, dim3(32, 8), 0, st>>>(static_cast<const float*>(in) + s.dev_off, dbatch, s.type, size,
                                                      s.swap, static_cast<unsigned char*>(out), s.stream_elem, sbatch, ld,
                                                      rows, cols);
  return cudaGetLastError();
}

}  // namespace b200
