"""ctypes wrapper of the CPU oracle (liboracle.so) and of oracle/_ref.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, as the checker.  The product
(stir_b200) never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from stir_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_raytrace.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_F = ctypes.c_float


def build():
    """Compile liboracle.so (and oracle/_ref when STIR's sources are present)."""
    subprocess.run(["make", "-C", HERE, "-s", "all"], check=True)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    sig = {
        "or_create": (_P, [ctypes.POINTER(_abi.Geometry), _I, ctypes.c_char_p, _I]),
        "or_destroy": (None, [_P]),
        "or_projdata_size": (_I64, [_P]),
        "or_image_size": (_I64, [_P]),
        "or_num_tof_bins": (_I, [_P]),
        "or_symmetries_used": (_I, [_P]),
        "or_num_basic_views": (_I, [_P]),
        "or_get_row": (_I64, [_P, _I, _I, _I, _I, _I, _P, _P, _I64]),
        "or_total_nnz": (_I64, [_P, _I]),
        "or_basic_row_elements": (_I64, [_P, _I, ctypes.POINTER(_I64)]),
        "or_forward_project_f32": (_I, [_P, _P, _P, _I, _I, _I]),
        "or_back_project_f32": (_I, [_P, _P, _P, _I, _I, _I]),
        "or_forward_project_f64": (_I, [_P, _P, _P, _I, _I, _I]),
        "or_back_project_f64": (_I, [_P, _P, _P, _I, _I, _I]),
        "or_sensitivity_f32": (_I, [_P, _P, _P, _I, _I, _I, _I]),
        "or_osmaposl_update_f32": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(_abi.Prior), _P, _F, _F, _I,
                                        ctypes.POINTER(_I)]),
        "or_sensitivity_f64": (_I, [_P, _P, _P, _I, _I, _I, _I]),
        "or_osmaposl_update_f64": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(_abi.Prior), _D, _D, _I]),
        "or_log_likelihood_f32": (_D, [_P, _P, _P, _P, _P, _I, _I, _I, _I]),
        "or_osmaposl_numerator_f32": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _P, ctypes.POINTER(_I)]),
        "or_osmaposl_apply_f32": (_I, [_P, _P, _P, _P, _I, _I, ctypes.POINTER(_abi.Prior), _P, _F, _F]),
        "or_loglik_gradient_f32": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _P]),
        "or_prior_gradient_f32": (_I, [ctypes.POINTER(_abi.Prior), _P, _P, _I, _I, _I, _F, _F, _F, _P]),
        "or_prior_value_f32": (_D, [ctypes.POINTER(_abi.Prior), _P, _P, _I, _I, _I, _F, _F, _F]),
        "or_ray_trace": (_I64, [_P, _P, _P, _F, _P, _P, _I64]),
        "or_ossps_denominator_f32": (_I, [_P, _P, _P, _I, _P]),
        "or_prior_hessian_times_input_f32": (_I, [ctypes.POINTER(_abi.Prior), _P, _P, _P, _I, _I, _I, _F, _F, _F, _P]),
        "or_listmode_f32": (_D, [_P, _I, _P, _P, _P, _I64, _P, _P, _I, _I, _I, _P, ctypes.POINTER(_I64)]),
        "or_gibbs_f32": (_D, [_I, _I, _F, _F, _F, _P, _I, _I, _I, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
        "or_gibbs_default_weights": (_I, [_F, _F, _F, _I, _P]),
        "or_prior_curvature_f32": (_I, [ctypes.POINTER(_abi.Prior), _P, _I, _I, _I, _F, _F, _F, _P]),
        "or_ossps_update_f32": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, ctypes.POINTER(_abi.Prior), _P,
                                     _F, _F, _F, _I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def default_threads():
    return os.cpu_count() or 1


class Oracle:
    """CPU restatement of STIR's ray-tracing projector pair for one geometry."""

    def __init__(self, geometry: _abi.Geometry, precision: int = 32):
        self.precision = precision
        err = ctypes.create_string_buffer(512)
        self.h = lib().or_create(ctypes.byref(geometry), precision, err, 512)
        if not self.h:
            raise ValueError(f"oracle geometry rejected: {err.value.decode()}")
        self.geometry = geometry
        self.dtype = np.float64 if precision == 64 else np.float32

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().or_destroy(h)
            self.h = None

    @property
    def projdata_size(self):
        return lib().or_projdata_size(self.h)

    @property
    def image_shape(self):
        g = self.geometry
        return (g.nz, g.ny, g.nx)

    @property
    def symmetries_used(self):
        return lib().or_symmetries_used(self.h)

    @property
    def num_tof_bins(self):
        return lib().or_num_tof_bins(self.h)

    def row(self, seg, view, ax, tang, tof=0, capacity=1 << 16):
        c = np.zeros((capacity, 3), np.int32)
        v = np.zeros(capacity, np.float64)
        n = lib().or_get_row(self.h, seg, view, ax, tang, tof, _ptr(c), _ptr(v), capacity)
        if n < 0:
            raise RuntimeError("oracle row failed")
        n = min(n, capacity)
        return c[:n].copy(), v[:n].copy()

    def total_nnz(self, nthreads=None):
        return lib().or_total_nnz(self.h, nthreads or default_threads())

    def basic_row_elements(self, nthreads=None):
        n = _I64(0)
        e = lib().or_basic_row_elements(self.h, nthreads or default_threads(), ctypes.byref(n))
        return n.value, e

    def forward(self, image, subset=0, nsub=1, nthreads=None, out=None):
        image = np.ascontiguousarray(image, self.dtype).reshape(self.image_shape)
        pd = np.zeros(self.projdata_size, self.dtype) if out is None else out
        f = lib().or_forward_project_f64 if self.precision == 64 else lib().or_forward_project_f32
        if f(self.h, _ptr(image), _ptr(pd), subset, nsub, nthreads or default_threads()) != 0:
            raise RuntimeError("oracle forward projection failed")
        return pd

    def back(self, projdata, subset=0, nsub=1, nthreads=None):
        projdata = np.ascontiguousarray(projdata, self.dtype).ravel()
        img = np.zeros(self.image_shape, self.dtype)
        f = lib().or_back_project_f64 if self.precision == 64 else lib().or_back_project_f32
        if f(self.h, _ptr(projdata), _ptr(img), subset, nsub, nthreads or default_threads()) != 0:
            raise RuntimeError("oracle back projection failed")
        return img

    def sensitivity(self, mult=None, subset=0, nsub=1, zero_seg0_end_planes=False, nthreads=None):
        m = None if mult is None else np.ascontiguousarray(mult, np.float32).ravel()
        img = np.zeros(self.image_shape, self.dtype)
        f = lib().or_sensitivity_f64 if self.precision == 64 else lib().or_sensitivity_f32
        if f(self.h, _ptr(m), _ptr(img), subset, nsub, int(zero_seg0_end_planes),
                                    nthreads or default_threads()) != 0:
            raise RuntimeError("oracle sensitivity failed")
        return img

    def osmaposl_update(self, estimate, y, additive, sens, subset, nsub, subiteration_num, prior=None, kappa=None,
                        min_rel=0.0, max_rel=1e37, zero_seg0_end_planes=False, nthreads=None):
        """One OSMAPOSL sub-iteration; returns (estimate, number of cancelled ratios).  A precision-64 oracle runs
        the FP64 restatement (no kappa; the cancelled count is not reported: -1)."""
        if self.precision == 64:
            x = np.ascontiguousarray(estimate, np.float64).copy().reshape(self.image_shape)
            y = np.ascontiguousarray(y, np.float32).ravel()
            a = None if additive is None else np.ascontiguousarray(additive, np.float32).ravel()
            s = np.ascontiguousarray(sens, np.float64).ravel()
            p = prior if prior is not None else _abi.Prior(type=_abi.PRIOR_NONE)
            if kappa is not None:
                raise ValueError("the FP64 OSMAPOSL restatement has no kappa")
            if lib().or_osmaposl_update_f64(self.h, _ptr(x), _ptr(y), _ptr(a), _ptr(s), subset, nsub, subiteration_num,
                                            int(zero_seg0_end_planes), ctypes.byref(p), float(min_rel), float(max_rel),
                                            nthreads or default_threads()) != 0:
                raise RuntimeError("oracle FP64 OSMAPOSL update failed")
            return x, -1
        x = np.ascontiguousarray(estimate, np.float32).copy().reshape(self.image_shape)
        y = np.ascontiguousarray(y, np.float32).ravel()
        a = None if additive is None else np.ascontiguousarray(additive, np.float32).ravel()
        s = np.ascontiguousarray(sens, np.float32).ravel()
        k = None if kappa is None else np.ascontiguousarray(kappa, np.float32).ravel()
        p = prior if prior is not None else _abi.Prior(type=_abi.PRIOR_NONE)
        cancelled = ctypes.c_int(0)
        st = lib().or_osmaposl_update_f32(self.h, _ptr(x), _ptr(y), _ptr(a), _ptr(s), subset, nsub, subiteration_num,
                                          int(zero_seg0_end_planes), ctypes.byref(p), _ptr(k), float(min_rel),
                                          float(max_rel), nthreads or default_threads(), ctypes.byref(cancelled))
        if st != 0:
            raise RuntimeError("oracle OSMAPOSL update failed")
        return x, cancelled.value

    def osmaposl_numerator(self, estimate, y, additive, subset, nsub, zero_seg0_end_planes=False, nthreads=None):
        x = np.ascontiguousarray(estimate, np.float32).ravel()
        y = np.ascontiguousarray(y, np.float32).ravel()
        a = None if additive is None else np.ascontiguousarray(additive, np.float32).ravel()
        u = np.zeros(self.image_shape, np.float32)
        c = ctypes.c_int(0)
        if lib().or_osmaposl_numerator_f32(self.h, _ptr(x), _ptr(y), _ptr(a), subset, nsub, int(zero_seg0_end_planes),
                                           nthreads or default_threads(), _ptr(u), ctypes.byref(c)) != 0:
            raise RuntimeError("oracle numerator failed")
        return u

    def osmaposl_apply(self, estimate, u, sens, nsub, subiteration_num, prior=None, kappa=None, min_rel=0.0, max_rel=1e37):
        x = np.ascontiguousarray(estimate, np.float32).copy().reshape(self.image_shape)
        uu = np.ascontiguousarray(u, np.float32).copy().reshape(self.image_shape)
        s = np.ascontiguousarray(sens, np.float32).ravel()
        k = None if kappa is None else np.ascontiguousarray(kappa, np.float32).ravel()
        p = prior if prior is not None else _abi.Prior(type=_abi.PRIOR_NONE)
        if lib().or_osmaposl_apply_f32(self.h, _ptr(x), _ptr(uu), _ptr(s), nsub, subiteration_num, ctypes.byref(p), _ptr(k),
                                       float(min_rel), float(max_rel)) != 0:
            raise RuntimeError("oracle update failed")
        return x

    def ossps_denominator(self, y, norm=None, nthreads=None):
        """OSSPS precomputed denominator A^T divide_and_truncate(A 1, (y n) n) (STIR order image)."""
        y = np.ascontiguousarray(y, np.float32).ravel()
        n = None if norm is None else np.ascontiguousarray(norm, np.float32).ravel()
        d = np.zeros(self.image_shape, np.float32)
        if lib().or_ossps_denominator_f32(self.h, _ptr(y), _ptr(n), nthreads or default_threads(), _ptr(d)) != 0:
            raise RuntimeError("oracle OSSPS denominator failed")
        return d

    def ossps_update(self, estimate, denom, y, additive, mult, sens, subset, nsub, subiteration_num,
                     start_subiteration_num=1, zero_seg0_end_planes=False, prior=None, kappa=None,
                     relaxation_parameter=1.0, relaxation_gamma=0.1, upper_bound=3.4028234663852886e38, nthreads=None):
        """One OSSPS sub-iteration; returns (estimate, denominator) after it."""
        x = np.ascontiguousarray(estimate, np.float32).copy().reshape(self.image_shape)
        d = np.ascontiguousarray(denom, np.float32).copy().reshape(self.image_shape)
        y = np.ascontiguousarray(y, np.float32).ravel()
        a = None if additive is None else np.ascontiguousarray(additive, np.float32).ravel()
        m = None if mult is None else np.ascontiguousarray(mult, np.float32).ravel()
        s = np.ascontiguousarray(sens, np.float32).ravel()
        k = None if kappa is None else np.ascontiguousarray(kappa, np.float32).ravel()
        p = prior if prior is not None else _abi.Prior(type=_abi.PRIOR_NONE)
        if lib().or_ossps_update_f32(self.h, _ptr(x), _ptr(d), _ptr(y), _ptr(a), _ptr(m), _ptr(s), subset, nsub,
                                     subiteration_num, start_subiteration_num, int(zero_seg0_end_planes),
                                     ctypes.byref(p), _ptr(k), float(relaxation_parameter), float(relaxation_gamma),
                                     float(upper_bound), nthreads or default_threads()) != 0:
            raise RuntimeError("oracle OSSPS update failed")
        return x, d

    def log_likelihood_gradient(self, image, y, additive=None, mult=None, subset=0, nsub=1, zero_seg0_end_planes=False,
                                nthreads=None):
        x = np.ascontiguousarray(image, np.float32).ravel()
        y = np.ascontiguousarray(y, np.float32).ravel()
        a = None if additive is None else np.ascontiguousarray(additive, np.float32).ravel()
        m = None if mult is None else np.ascontiguousarray(mult, np.float32).ravel()
        g = np.zeros(self.image_shape, np.float32)
        if lib().or_loglik_gradient_f32(self.h, _ptr(x), _ptr(y), _ptr(a), _ptr(m), subset, nsub,
                                        int(zero_seg0_end_planes), nthreads or default_threads(), _ptr(g)) != 0:
            raise RuntimeError("oracle gradient failed")
        return g

    def listmode(self, op, bins, values, image, corr=None, rhs=None, subset=0, nsub=1, has_add=False, out=None):
        """List-mode objective over events: bins (n, 5) ints (segment, view, axial, tangential, timing), values (n,),
        corr (n,) additive terms.  op "gradient" / "hessian" return out + the sum; "value" returns (value, invalid)."""
        bins = np.ascontiguousarray(bins, np.int32).reshape(-1, 5)
        values = np.ascontiguousarray(values, np.float32)
        c = None if corr is None else np.ascontiguousarray(corr, np.float32)
        img = np.ascontiguousarray(image, np.float32)
        r = None if rhs is None else np.ascontiguousarray(rhs, np.float32)
        o = np.zeros(img.shape, np.float32) if out is None else np.ascontiguousarray(out, np.float32).copy()
        bad = ctypes.c_int64()
        code = {"gradient": 0, "value": 1, "hessian": 2}[op]
        v = lib().or_listmode_f32(self.h, code, _ptr(bins), _ptr(values), _ptr(c), bins.shape[0], _ptr(img), _ptr(r),
                                  subset, nsub, int(bool(has_add)), _ptr(o), ctypes.byref(bad))
        return (v, bad.value) if code == 1 else o

    def log_likelihood(self, image, y, additive=None, mult=None, subset=0, nsub=1, zero_seg0_end_planes=False,
                       nthreads=None):
        x = np.ascontiguousarray(image, np.float32).ravel()
        y = np.ascontiguousarray(y, np.float32).ravel()
        a = None if additive is None else np.ascontiguousarray(additive, np.float32).ravel()
        m = None if mult is None else np.ascontiguousarray(mult, np.float32).ravel()
        return lib().or_log_likelihood_f32(self.h, _ptr(x), _ptr(y), _ptr(a), _ptr(m), subset, nsub,
                                           int(zero_seg0_end_planes), nthreads or default_threads())


def prior_gradient(prior: _abi.Prior, image, voxel_size, kappa=None):
    image = np.ascontiguousarray(image, np.float32)
    nz, ny, nx = image.shape
    g = np.zeros_like(image)
    k = None if kappa is None else np.ascontiguousarray(kappa, np.float32)
    lib().or_prior_gradient_f32(ctypes.byref(prior), _ptr(image), _ptr(k), nz, ny, nx, *map(float, voxel_size), _ptr(g))
    return g


def prior_value(prior: _abi.Prior, image, voxel_size, kappa=None):
    image = np.ascontiguousarray(image, np.float32)
    nz, ny, nx = image.shape
    k = None if kappa is None else np.ascontiguousarray(kappa, np.float32)
    return lib().or_prior_value_f32(ctypes.byref(prior), _ptr(image), _ptr(k), nz, ny, nx, *map(float, voxel_size))


def prior_hessian_times_input(prior: _abi.Prior, image, input_image, voxel_size, kappa=None, out=None):
    """out + the prior's Hessian at `image` times `input_image` ([z][y][x])."""
    image = np.ascontiguousarray(image, np.float32)
    nz, ny, nx = image.shape
    inp = np.ascontiguousarray(input_image, np.float32)
    k = None if kappa is None else np.ascontiguousarray(kappa, np.float32).ravel()
    o = np.zeros(image.shape, np.float32) if out is None else np.ascontiguousarray(out, np.float32).copy()
    lib().or_prior_hessian_times_input_f32(ctypes.byref(prior), _ptr(image), _ptr(inp), _ptr(k), nz, ny, nx,
                                           *map(float, voxel_size), _ptr(o))
    return o


def prior_curvature(prior: _abi.Prior, shape, voxel_size, kappa=None):
    """QuadraticPrior::parabolic_surrogate_curvature of an image of `shape` [z][y][x]."""
    nz, ny, nx = shape
    k = None if kappa is None else np.ascontiguousarray(kappa, np.float32).ravel()
    c = np.zeros(shape, np.float32)
    if lib().or_prior_curvature_f32(ctypes.byref(prior), _ptr(k), nz, ny, nx, *map(float, voxel_size), _ptr(c)) != 0:
        raise RuntimeError("oracle curvature failed")
    return c


GIBBS_OPS = {"value": 0, "gradient": 1, "gradient_times_input": 2, "hessian_diagonal": 3,
             "hessian_times_input": 4, "hessian": 5}


def gibbs_default_weights(voxel_size, only_2D=False):
    """GibbsPenalty::compute_default_weights: [wz][3][3] floats, x voxel size / distance."""
    w = np.zeros(27, np.float32)
    wz = lib().or_gibbs_default_weights(*map(float, voxel_size), int(bool(only_2D)), _ptr(w))
    return w[:wz * 9].reshape(wz, 3, 3).copy()


def gibbs(op, potential, beta, weights, image, input_image=None, kappa=None, gamma=2.0, epsilon=1e-7, voxel=(0, 0, 0),
          out=None):
    """GibbsPenalty<float, potential> (potential 1 Quadratic, 2 Relative Difference) on [z][y][x] images.

    op: "value" and "gradient_times_input" return a float; "gradient", "hessian_diagonal" and "hessian"
    (of voxel `voxel`) return an image; "hessian_times_input" returns out + H input."""
    image = np.ascontiguousarray(image, np.float32)
    nz, ny, nx = image.shape
    w = np.ascontiguousarray(weights, np.float32)
    assert w.ndim == 3
    k = None if kappa is None else np.ascontiguousarray(kappa, np.float32)
    inp = None if input_image is None else np.ascontiguousarray(input_image, np.float32)
    o = np.zeros(image.shape, np.float32) if out is None else np.ascontiguousarray(out, np.float32).copy()
    code = GIBBS_OPS[op]
    v = lib().or_gibbs_f32(code, potential, float(beta), float(gamma), float(epsilon), _ptr(w), *w.shape, _ptr(k),
                           _ptr(image), _ptr(inp), nz, ny, nx, *map(int, voxel), _ptr(o))
    return v if code in (0, 2) else o


def ray_trace(start_zyx, stop_zyx, voxel_size_zyx, norm_const, capacity=1 << 14):
    """Oracle restatement of RayTraceVoxelsOnCartesianGrid."""
    return _trace(lib().or_ray_trace, start_zyx, stop_zyx, voxel_size_zyx, norm_const, capacity)


def _trace(fn, start, stop, vox, norm_const, capacity):
    s = np.asarray(start, np.float32)
    e = np.asarray(stop, np.float32)
    v = np.asarray(vox, np.float32)
    c = np.zeros((capacity, 3), np.int32)
    val = np.zeros(capacity, np.float32)
    n = fn(_ptr(s), _ptr(e), _ptr(v), float(norm_const), _ptr(c), _ptr(val), capacity)
    if n < 0:
        raise RuntimeError("capacity exceeded")
    return c[:n].copy(), val[:n].copy()


_ref = None


REF_CUDA_PRIORS_LIB = os.path.join(HERE, "_ref", "libref_cuda_priors.so")
_ref_cuda = None


def ref_cuda_priors_available():
    """STIR's own CUDA prior kernels built by oracle/Makefile (needs the STIR sources when building)."""
    return os.path.exists(REF_CUDA_PRIORS_LIB)


def ref_cuda_priors():
    """ctypes handle of oracle/_ref/libref_cuda_priors.so: STIR's CudaRelativeDifferencePrior gradient kernel and
    CudaGibbsPenalty gradient kernel with its potentials, launched as STIR's host classes launch them, on device
    images in STIR's [z][y][x] order (pointers, a CUDA stream as void*)."""
    global _ref_cuda
    if _ref_cuda is None:
        lib = ctypes.CDLL(REF_CUDA_PRIORS_LIB)
        lib.ref_cuda_rdp_prior_gradient.restype = _I
        lib.ref_cuda_rdp_prior_gradient.argtypes = [_P, _P, _P, _P, _F, _F, _F, _I, _I, _I, _P]
        lib.ref_cuda_gibbs_gradient.restype = _I
        lib.ref_cuda_gibbs_gradient.argtypes = [_I, _P, _P, _P, _I, _I, _I, _P, _F, _F, _F, _I, _I, _I, _I, _I, _P]
        _ref_cuda = lib
    return _ref_cuda


def ref_available():
    return os.path.exists(REF_LIB)


def ref_ray_trace(start_zyx, stop_zyx, voxel_size_zyx, norm_const, capacity=1 << 14):
    """STIR's own RayTraceVoxelsOnCartesianGrid, compiled from the STIR tree into oracle/_ref."""
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_LIB)
        _ref.ref_ray_trace.restype = _I64
        _ref.ref_ray_trace.argtypes = [_P, _P, _P, _F, _P, _P, _I64]
    return _trace(_ref.ref_ray_trace, start_zyx, stop_zyx, voxel_size_zyx, norm_const, capacity)


# ---- projection data streams: ProjDataFromStream::get_offset (src/buildblock/ProjDataFromStream.cxx:415-500) ----
NUMPY_TYPES = {"schar": "i1", "uchar": "u1", "short": "i2", "ushort": "u2", "int": "i4", "uint": "u4", "float": "f4",
               "double": "f8"}


def projdata_from_stream(raw, geometry: _abi.Geometry, storage_order, number_type, big_endian, scale_factor,
                         segment_sequence, num_axial_poss, num_timing_poss=1, timing_poss_sequence=None,
                         min_timing_pos_num=0):
    """The projector's bins in ProjDataInMemory order (segments 0, +1, -1, ..., then axial, view, tangential;
    timing positions outermost) read from the bytes of a stream, element by element as get_offset addresses them."""
    dt = np.dtype(NUMPY_TYPES[number_type]).newbyteorder(">" if big_endian else "<")
    data = np.frombuffer(bytes(raw), dtype=dt)
    nv, nt, S = geometry.num_views, geometry.num_tangential_poss, geometry.max_segment_num
    size3d = sum(num_axial_poss) * nv * nt
    ntof = num_timing_poss
    order = [0] + [s for k in range(1, S + 1) for s in (k, -k)]
    out = []
    for k in range(ntof):
        ti = k if timing_poss_sequence is None else list(timing_poss_sequence).index(min_timing_pos_num + k)
        for s in order:
            i = list(segment_sequence).index(s)
            nax = num_axial_poss[i]
            off = ti * size3d + sum(num_axial_poss[:i]) * nv * nt
            seg = data[off:off + nax * nv * nt].astype(np.float64)
            if storage_order == _abi.STORAGE_SEGMENT_AXIAL_VIEW_TANG:
                seg = seg.reshape(nax, nv, nt)
            else:
                seg = seg.reshape(nv, nax, nt).transpose(1, 0, 2)
            out.append((seg.astype(np.float32) * np.float32(scale_factor)).astype(np.float32).ravel())
    return np.concatenate(out)
