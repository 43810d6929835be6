// Row builder: traces the rays of every basic bin on the device and assembles
// the rows of STIR's ray-tracing matrix (ProjMatrixByBinUsingRayTracing).
//
// This translation unit is compiled with -fmad=false: every float expression is
// evaluated unfused, in the order STIR writes it, so the rows agree with STIR's
// float arithmetic element for element.
//
// One thread builds one basic bin in its own scratch slice:
//   1. Siddon traversal of each ray            RayTraceVoxelsOnCartesianGrid.cxx:51-269
//   2. merge of the tangential rays            ProjMatrixByBinUsingRayTracing.cxx:765-781, merge :162-277
//   3. add_adjacent_z for direct bins          ProjMatrixByBinUsingRayTracing.cxx:785-795, 831-954
//      or the z copies of oblique bins         ProjMatrixByBinUsingRayTracing.cxx:796-827
// Merges are done as a sort by (z,y,x,tag) followed by a left-to-right sum of
// equal coordinates, which adds duplicates in the order STIR's merges do.
#include "internal.hpp"

namespace b200 {

namespace {

__device__ __forceinline__ int round_half_away(float x) {
  return x >= 0 ? static_cast<int>(x + 0.5F) : -static_cast<int>(-x + 0.5F);
}
__device__ __forceinline__ bool is_half_integer(float a) { return fabsf(floorf(a) + .5F - a) < .0001F; }
__device__ __forceinline__ double norm3(float z, float y, float x) {
  float s = 0.f;
  s = s + z * z;
  s = s + y * y;
  s = s + x * x;
  return sqrt(static_cast<double>(s));
}
__device__ __forceinline__ uint64_t make_key(int z, int y, int x, int tag) {
  return (static_cast<uint64_t>(z + 32768) << 40) | (static_cast<uint64_t>(y + 32768) << 24) |
         (static_cast<uint64_t>(x + 32768) << 8) | static_cast<uint64_t>(tag & 255);
}
__device__ __forceinline__ void key_zyx(uint64_t k, int& z, int& y, int& x) {
  z = static_cast<int>((k >> 40) & 0xFFFF) - 32768;
  y = static_cast<int>((k >> 24) & 0xFFFF) - 32768;
  x = static_cast<int>((k >> 8) & 0xFFFF) - 32768;
}

struct Job {
  float st[3], sp[3], nc;
};

// RayTraceVoxelsOnCartesianGrid, with the recursion of :105-131 unrolled onto a small stack.
__device__ void siddon(const float* st0, const float* sp0, float nc0, float vz, float vy, float vx, int tag, RowKV* out,
                       int& n, int cap, int& err) {
  Job stack[8];
  int top = 0;
  for (int k = 0; k < 3; ++k) {
    stack[0].st[k] = st0[k];
    stack[0].sp[k] = sp0[k];
  }
  stack[0].nc = nc0;
  top = 1;
  while (top > 0) {
    const Job j = stack[--top];
    const float dz = j.sp[0] - j.st[0], dy = j.sp[1] - j.st[1], dx = j.sp[2] - j.st[2];
    if (norm3(dz, dy, dx) <= .00001F) continue;
    const bool zx = fabsf(dx) <= 1.E-4F, zy = fabsf(dy) <= 1.E-4F, zz = fabsf(dz) <= 1.E-4F;
    {
      float inc[3] = {0.f, 0.f, 0.f};
      if (zz && is_half_integer(j.st[0]))
        inc[0] = .5F;
      else if (zy && is_half_integer(j.st[1]))
        inc[1] = .5F;
      else if (zx && is_half_integer(j.st[2]))
        inc[2] = .5F;
      if (norm3(inc[0], inc[1], inc[2]) > .1) {
        if (top + 2 > 8) {
          err = 1;
          return;
        }
        Job a, b;
        for (int k = 0; k < 3; ++k) {
          a.st[k] = j.st[k] + inc[k];
          a.sp[k] = j.sp[k] + inc[k];
          b.st[k] = j.st[k] - inc[k];
          b.sp[k] = j.sp[k] - inc[k];
        }
        a.nc = j.nc / 2;
        b.nc = j.nc / 2;
        stack[top++] = a;
        stack[top++] = b;
        continue;
      }
    }
    // d12 = |difference * voxel_size| * normalisation_constant (:76-79)
    const float d12 = static_cast<float>(norm3(dz * vz, dy * vy, dx * vx) * static_cast<double>(j.nc));
    const int sx = dx >= 0 ? 1 : -1, sy = dy >= 0 ? 1 : -1, sz = dz >= 0 ? 1 : -1;
    const float inc_x = zx ? d12 * 1000000.F : d12 / fabsf(dx);
    const float inc_y = zy ? d12 * 1000000.F : d12 / fabsf(dy);
    const float inc_z = zz ? d12 * 1000000.F : d12 / fabsf(dz);
    const float xmax = static_cast<float>(round_half_away(j.sp[2])) + static_cast<float>(sx) * 0.5F;
    const float ymax = static_cast<float>(round_half_away(j.sp[1])) + static_cast<float>(sy) * 0.5F;
    const float zmax = static_cast<float>(round_half_away(j.sp[0])) + static_cast<float>(sz) * 0.5F;
    const float axend = zx ? d12 * 1000000.F : (xmax - j.st[2]) * inc_x * static_cast<float>(sx) * .9999F;
    const float ayend = zy ? d12 * 1000000.F : (ymax - j.st[1]) * inc_y * static_cast<float>(sy) * .9999F;
    const float azend = zz ? d12 * 1000000.F : (zmax - j.st[0]) * inc_z * static_cast<float>(sz) * .9999F;
    const float amax = fminf(axend, fminf(ayend, azend));
    int cz = round_half_away(j.st[0]), cy = round_half_away(j.st[1]), cx = round_half_away(j.st[2]);
    float az = zz ? -inc_z : ((static_cast<float>(cz) - j.st[0]) - static_cast<float>(sz) * 0.5F) * inc_z * static_cast<float>(sz);
    float ax = zx ? -inc_x : ((static_cast<float>(cx) - j.st[2]) - static_cast<float>(sx) * 0.5F) * inc_x * static_cast<float>(sx);
    float ay = zy ? -inc_y : ((static_cast<float>(cy) - j.st[1]) - static_cast<float>(sy) * 0.5F) * inc_y * static_cast<float>(sy);
    float a = fmaxf(ax, fmaxf(ay, az));
    ax = zx ? axend : ax + inc_x;
    ay = zy ? ayend : ay + inc_y;
    az = zz ? azend : az + inc_z;
    while (a < amax) {
      float len;
      const int oz = cz, oy = cy, ox = cx;
      if (ax < ay) {
        if (ax < az) {
          len = ax - a;
          a = ax;
          ax += inc_x;
          cx += sx;
        } else {
          len = az - a;
          a = az;
          az += inc_z;
          cz += sz;
        }
      } else if (ay < az) {
        len = ay - a;
        a = ay;
        ay += inc_y;
        cy += sy;
      } else {
        len = az - a;
        a = az;
        az += inc_z;
        cz += sz;
      }
      if (n >= cap) {
        err = 2;
        return;
      }
      out[n].key = make_key(oz, oy, ox, tag);
      out[n].v = len;
      ++n;
    }
  }
}

// bottom-up merge sort of a[0..n) by key, using tmp[0..n); result in a
__device__ void sort_kv(RowKV* a, RowKV* tmp, int n) {
  RowKV* src = a;
  RowKV* dst = tmp;
  for (int width = 1; width < n; width *= 2) {
    for (int lo = 0; lo < n; lo += 2 * width) {
      const int mid = min(lo + width, n), hi = min(lo + 2 * width, n);
      int i = lo, j = mid, k = lo;
      while (i < mid && j < hi) dst[k++] = (src[j].key < src[i].key) ? src[j++] : src[i++];
      while (i < mid) dst[k++] = src[i++];
      while (j < hi) dst[k++] = src[j++];
    }
    RowKV* t = src;
    src = dst;
    dst = t;
  }
  if (src != a)
    for (int i = 0; i < n; ++i) a[i] = src[i];
}

// sum equal coordinates left to right (tags ascending), keep one element per coordinate with tag 0
__device__ int reduce_kv(RowKV* a, int n) {
  int m = 0;
  for (int i = 0; i < n; ++i) {
    const uint64_t c = a[i].key >> 8;
    if (m > 0 && (a[m - 1].key >> 8) == c) {
      a[m - 1].v = a[m - 1].v + a[i].v;
    } else {
      a[m].key = c << 8;
      a[m].v = a[i].v;
      ++m;
    }
  }
  return m;
}

__global__ void build_rows_kernel(const RayDev* rays, const BuildBinDev* bins, int nbins, float vz, float vy, float vx,
                                  RowKV* scratch, int* counts) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  const BuildBinDev bb = bins[b];
  RowKV* buf = scratch + bb.scratch_offset;
  RowKV* tmp = buf + bb.capacity;
  int n = 0, err = 0;
  for (int r = 0; r < bb.num_rays && !err; ++r) {
    const RayDev ray = rays[bb.first_ray + r];
    siddon(ray.start, ray.stop, ray.norm_const, vz, vy, vx, r, buf, n, bb.capacity, err);
  }
  if (!err && bb.num_rays > 1 && n > 0) {
    sort_kv(buf, tmp, n);
    n = reduce_kv(buf, n);
  }
  if (!err && n > 0) {
    if (bb.direct) {
      // add_adjacent_z (ProjMatrixByBinUsingRayTracing.cxx:831-954)
      int z0, y0, x0;
      key_zyx(buf[0].key, z0, y0, x0);
      const float zfv = (static_cast<float>(z0) + bb.z_origin_in_planes) - bb.z_centre;
      const float zf = zfv - bb.left_edge;
      const float right = bb.tor_width;
      const int org = n;
      for (int zi = 1;; ++zi) {
        const float overlap = fminf(right, zf + static_cast<float>(zi) + .5F) - fmaxf(0.F, zf + static_cast<float>(zi) - .5F);
        if (static_cast<double>(overlap) <= 0.0001) break;
        if (n + org > bb.capacity) {
          err = 3;
          break;
        }
        for (int k = 0; k < org; ++k) {
          int z, y, x;
          key_zyx(buf[k].key, z, y, x);
          buf[n].key = make_key(z0 + zi, y, x, 0);
          buf[n].v = static_cast<double>(overlap) > .9999 ? buf[k].v : buf[k].v * overlap;
          ++n;
        }
      }
      if (!err && static_cast<double>(zf) > 0.5) {
        const float overlap = zf - .5F;
        if (n + org > bb.capacity) {
          err = 3;
        } else {
          for (int k = 0; k < org; ++k) {
            int z, y, x;
            key_zyx(buf[k].key, z, y, x);
            buf[n].key = make_key(z0 - 1, y, x, 0);
            buf[n].v = static_cast<double>(overlap) > .9999 ? buf[k].v : buf[k].v * overlap;
            ++n;
          }
        }
      }
      if (!err) {
        const float overlap = fminf(right, zf + .5F) - fmaxf(0.F, zf - .5F);
        if (static_cast<double>(overlap) < .9999)
          for (int k = 0; k < org; ++k) buf[k].v *= overlap;
      }
    } else if (bb.nlz > 1) {
      // copies at z+1 .. z+nlz-1 merged in order (ProjMatrixByBinUsingRayTracing.cxx:796-827)
      const int org = n;
      if (org * bb.nlz > bb.capacity) {
        err = 4;
      } else {
        for (int zi = 1; zi < bb.nlz; ++zi)
          for (int k = 0; k < org; ++k) {
            int z, y, x;
            key_zyx(buf[k].key, z, y, x);
            buf[n].key = make_key(z + zi, y, x, zi);
            buf[n].v = buf[k].v;
            ++n;
          }
        sort_kv(buf, tmp, n);
        n = reduce_kv(buf, n);
      }
    }
  }
  // the packed storage covers z in [-512,511] and x,y in [-1024,1023]
  if (!err)
    for (int k = 0; k < n; ++k) {
      int z, y, x;
      key_zyx(buf[k].key, z, y, x);
      if (z < -512 || z > 511 || y < -1024 || y > 1023 || x < -1024 || x > 1023) {
        err = 5;
        break;
      }
    }
  counts[b] = err ? -err : n;
}

__global__ void compact_rows_kernel(const BuildBinDev* bins, int nbins, const RowKV* scratch, const int64_t* out_offsets,
                                    RowElem* rows) {
  const int b = blockIdx.y;
  if (b >= nbins) return;
  const int64_t o = out_offsets[b];
  const int n = static_cast<int>(out_offsets[b + 1] - o);
  const RowKV* src = scratch + bins[b].scratch_offset;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    int z, y, x;
    key_zyx(src[k].key, z, y, x);
    RowElem e;
    e.zyx = pack_zyx(z, y, x);
    e.v = src[k].v;
    rows[o + k] = e;
  }
}

// FastErf::get_erf_linear_interpolation (numerics/FastErf.inl:46-66)
__device__ __forceinline__ double fast_erf(const TofParams& tp, double xp) {
  xp = fmax(fmin(tp.erf_max, xp), -tp.erf_max);
  const double xi = (xp + tp.erf_max) / tp.erf_period;
  const int lower = static_cast<int>(floor(xi));
  return tp.erf_table[lower] + (xi - lower) * (tp.erf_table[lower + 1] - tp.erf_table[lower]);
}

// ProjMatrixByBin::get_tof_value (ProjMatrixByBin.inl:187-197); with trunc_n > 0 the kernel truncated at
// +-trunc_n: the bin's ends clamped to that range (a bin wholly outside it gets 0)
__device__ __forceinline__ float tof_value(const TofParams& tp, float d1, float d2) {
  float d1n = d1 * tp.r_sqrt2_sigma, d2n = d2 * tp.r_sqrt2_sigma;
  if (tp.trunc_n > 0.f) {
    d1n = fminf(fmaxf(d1n, -tp.trunc_n), tp.trunc_n);
    d2n = fminf(fmaxf(d2n, -tp.trunc_n), tp.trunc_n);
  } else if ((d1n >= 4.f && d2n >= 4.f) || (d1n <= -4.f && d2n <= -4.f)) {
    return 0.f;
  }
  return static_cast<float>(0.5 * (fast_erf(tp, static_cast<double>(d2n)) - fast_erf(tp, static_cast<double>(d1n))));
}

// one thread per (basic bin, timing bin): out == nullptr counts, otherwise fills at out_offsets[job]
__global__ void tof_rows_kernel(const RowElem* __restrict__ src, const TofJobDev* __restrict__ jobs, int njobs, TofParams tp,
                                const int64_t* __restrict__ out_offsets, RowElem* __restrict__ out, int* __restrict__ counts) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  const TofJobDev job = jobs[j];
  const float low = tp.low[job.tof_index], high = tp.high[job.tof_index];
  int n = 0;
  int64_t o = out ? out_offsets[j] : 0;
  for (int k = 0; k < job.src_len; ++k) {
    const RowElem e = src[job.src_offset + k];
    int z, y, x;
    unpack_zyx(e.zyx, z, y, x);
    // get_physical_coordinates_for_indices, minus the scanner centre in z
    const float pz = (static_cast<float>(z) * tp.vox[0] + tp.origin[0]) - tp.scanner_z_offset;
    const float py = (static_cast<float>(y) * tp.vox[1] + tp.origin[1]) - 0.0f;
    const float px = (static_cast<float>(x) * tp.vox[2] + tp.origin[2]) - 0.0f;
    float ip = 0.f;
    ip = ip + (pz - job.mid[0]) * job.unit[0];
    ip = ip + (py - job.mid[1]) * job.unit[1];
    ip = ip + (px - job.mid[2]) * job.unit[2];
    const float d2 = -ip;
    const float kv = tof_value(tp, low - d2, high - d2);
    if (kv > 0 && e.v != 0) {
      if (out) {
        RowElem r;
        r.zyx = e.zyx;
        r.v = e.v * kv;
        out[o + n] = r;
      }
      ++n;
    }
  }
  if (!out) counts[j] = n;
}

// one thread per (basic bin, timing bin): the weight of every element of the non-TOF row for this timing bin,
// w[(src_offset + e) * ntof + tof_index] = the TOF row's value (e.v * kernel value), 0 where the TOF row has no
// element (the same arithmetic as tof_rows_kernel, so the weights equal the TOF rows' values)
__global__ void tof_weights_kernel(const RowElem* __restrict__ src, const TofJobDev* __restrict__ jobs, int njobs,
                                   TofParams tp, int ntof, float* __restrict__ w) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  const TofJobDev job = jobs[j];
  const float low = tp.low[job.tof_index], high = tp.high[job.tof_index];
  for (int k = 0; k < job.src_len; ++k) {
    const RowElem e = src[job.src_offset + k];
    int z, y, x;
    unpack_zyx(e.zyx, z, y, x);
    const float pz = (static_cast<float>(z) * tp.vox[0] + tp.origin[0]) - tp.scanner_z_offset;
    const float py = (static_cast<float>(y) * tp.vox[1] + tp.origin[1]) - 0.0f;
    const float px = (static_cast<float>(x) * tp.vox[2] + tp.origin[2]) - 0.0f;
    float ip = 0.f;
    ip = ip + (pz - job.mid[0]) * job.unit[0];
    ip = ip + (py - job.mid[1]) * job.unit[1];
    ip = ip + (px - job.mid[2]) * job.unit[2];
    const float d2 = -ip;
    const float kv = tof_value(tp, low - d2, high - d2);
    w[(job.src_offset + k) * ntof + job.tof_index] = (kv > 0 && e.v != 0) ? e.v * kv : 0.f;
  }
}

}  // namespace

cudaError_t launch_tof_weights(const RowElem* src, const TofJobDev* jobs, int njobs, const TofParams& tp, int ntof,
                               float* w, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  tof_weights_kernel<<<(njobs + 127) / 128, 128, 0, st>>>(src, jobs, njobs, tp, ntof, w);
  return cudaGetLastError();
}

cudaError_t launch_tof_rows(const RowElem* src, const TofJobDev* jobs, int njobs, const TofParams& tp,
                            const int64_t* out_offsets, RowElem* out, int* counts, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  tof_rows_kernel<<<(njobs + 127) / 128, 128, 0, st>>>(src, jobs, njobs, tp, out_offsets, out, counts);
  return cudaGetLastError();
}

cudaError_t launch_build_rows(const RayDev* rays, const BuildBinDev* bins, int nbins, const float voxel_zyx[3],
                              RowKV* scratch, int* counts, cudaStream_t st) {
  if (nbins <= 0) return cudaSuccess;
  const int threads = 64;
  build_rows_kernel<<<(nbins + threads - 1) / threads, threads, 0, st>>>(rays, bins, nbins, voxel_zyx[0], voxel_zyx[1],
                                                                          voxel_zyx[2], scratch, counts);
  return cudaGetLastError();
}

cudaError_t launch_compact_rows(const BuildBinDev* bins, int nbins, const RowKV* scratch, const int64_t* out_offsets,
                                RowElem* rows, cudaStream_t st) {
  if (nbins <= 0) return cudaSuccess;
  int done = 0;
  while (done < nbins) {
    const int chunk = nbins - done < 65535 ? nbins - done : 65535;
    compact_rows_kernel<<<dim3(2, chunk), 256, 0, st>>>(bins + done, chunk, scratch, out_offsets + done, rows);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    done += chunk;
  }
  return cudaSuccess;
}

}  // namespace b200
