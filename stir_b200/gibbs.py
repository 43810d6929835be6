"""Gibbs penalties on device-resident images, through the C ABI (gibbs.cu).

Mirrors STIR's GibbsQuadraticPenalty / GibbsRelativeDifferencePenalty
(src/include/stir/recon_buildblock/GibbsPenalty.h, GibbsPenalty.inl, GibbsQuadraticPenalty.h,
GibbsRelativeDifferencePenalty.h) and their CUDA versions CudaGibbsQuadraticPenalty /
CudaGibbsRelativeDifferencePenalty (CUDA/CudaGibbsPenalty.h): the same parameters ("penalisation factor",
"only 2D", "weights", kappa, "gamma value", "epsilon value"), the same operations, and STIR's errors for a
penalty used before set_up.  Images are CUDA float32 tensors, shaped (nz, ny, nx) in STIR's [z][y][x] order
(the default) or flat in the projector's device layout [y][x][z] (layout=LAYOUT_DEVICE); they stay on the GPU.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _abi

LAYOUT_STIR = _abi.LAYOUT_STIR
LAYOUT_DEVICE = _abi.LAYOUT_DEVICE


class GibbsPenalty:
    """GibbsPenalty<float, potential>: f = beta sum_{r,dr} w_dr phi(x_r, x_{r+dr}) kappa_r kappa_{r+dr}."""

    potential = 0
    registered_name = ""
    arithmetic = _abi.GIBBS_ARITH_HOST  # the gradient's sums: GibbsPenalty.inl's doubles

    def __init__(self, only_2D: bool = False, penalisation_factor: float = 0.0, device: int = 0):
        self.only_2D = bool(only_2D)
        self.penalisation_factor = float(penalisation_factor)
        self.weights: Optional[np.ndarray] = None
        self.kappa = None
        self.device = device
        self._h = None
        self._lib = _abi.load_library()
        self._shape = None
        self._layout = LAYOUT_STIR

    # --- parameters (GibbsPenalty.h) ---
    def set_penalisation_factor(self, beta: float):
        self.penalisation_factor = float(beta)
        self._release()

    def get_penalisation_factor(self) -> float:
        return self.penalisation_factor

    def set_weights(self, w):
        """Weights [z][y][x]; index ranges -(size/2)..size-1-size/2 (an even size acts as if a 0 were appended)."""
        w = np.ascontiguousarray(w, np.float32)
        if w.ndim != 3 or min(w.shape) < 1 or max(w.shape) > 7:
            raise ValueError("weights must be a 3D array with sizes 1..7")
        self.weights = w
        self._release()

    def get_weights(self) -> np.ndarray:
        if self._h is None:
            if self.weights is None:
                raise RuntimeError(f"{type(self).__name__}: set_up has not been called")
            return self.weights.copy()
        sizes = (ctypes.c_int32 * 3)()
        _abi.check(self._lib.b200rt_gibbs_get_weights(self._h, None, sizes), what="get_weights", gibbs=self._h)
        w = np.zeros(tuple(sizes), np.float32)
        _abi.check(self._lib.b200rt_gibbs_get_weights(self._h, ctypes.c_void_p(w.ctypes.data), sizes),
                   what="get_weights", gibbs=self._h)
        return w

    def set_kappa_sptr(self, kappa):
        """Spatially varying factors (a la Fessler): an image like the estimates, or None."""
        self.kappa = kappa
        if self._h is not None:
            self._check_image(kappa) if kappa is not None else None
            _abi.check(self._lib.b200rt_gibbs_set_kappa(self._h, _ptr(kappa)), what="set_kappa", gibbs=self._h)

    def get_kappa_sptr(self):
        return self.kappa

    @staticmethod
    def is_convex() -> bool:
        return True

    def _potential_params(self):
        return 0.0, 0.0

    # --- set-up ---
    def set_up(self, shape: Sequence[int], voxel_size: Sequence[float] = (1.0, 1.0, 1.0), layout: int = LAYOUT_STIR):
        """GibbsPenalty::set_up for images of `shape` (nz, ny, nx) with voxel sizes (z, y, x) in mm: the default
        weights (x voxel size / distance) unless weights were set."""
        self._release()
        nz, ny, nx = map(int, shape)
        gamma, epsilon = self._potential_params()
        p = _abi.GibbsParams()
        p.potential = self.potential
        p.penalisation_factor = self.penalisation_factor
        p.gamma = gamma
        p.epsilon = epsilon
        p.nz, p.ny, p.nx = nz, ny, nx
        p.layout = layout
        p.voxel_size_z, p.voxel_size_y, p.voxel_size_x = map(float, voxel_size)
        p.only_2D = int(self.only_2D)
        if self.weights is not None:
            p.weights_z, p.weights_y, p.weights_x = self.weights.shape
            p.weights = ctypes.c_void_p(self.weights.ctypes.data)
        if self.kappa is not None:
            self._shape, self._layout = (nz, ny, nx), layout
            self._check_image(self.kappa)
        p.kappa_dev = _ptr(self.kappa)
        h = ctypes.c_void_p()
        st = self._lib.b200rt_gibbs_create(ctypes.byref(p), self.device, ctypes.byref(h))
        if st != _abi.OK:
            msg = self._lib.b200rt_last_error(None)
            raise _abi.B200Error(f"{type(self).__name__}.set_up failed with status {st}: "
                                 f"{msg.decode() if msg else ''}")
        self._h = h
        self._shape = (nz, ny, nx)
        self._layout = layout
        _abi.check(self._lib.b200rt_gibbs_set_arithmetic(self._h, self.arithmetic), what="set_up", gibbs=self._h)

    def _release(self):
        if getattr(self, "_h", None) is not None:
            self._lib.b200rt_gibbs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    def _ready(self):
        if self._h is None:
            raise RuntimeError(f"{type(self).__name__}: set_up has not been called")

    def _check_image(self, t):
        import torch
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous():
            raise TypeError("images must be contiguous float32 CUDA tensors")
        if t.numel() != int(np.prod(self._shape)):
            raise ValueError("image does not have the penalty's size (kappa or estimate of another image?)")
        if self._layout == LAYOUT_STIR and t.dim() == 3 and tuple(t.shape) != tuple(self._shape):
            raise ValueError("image shape differs from the one the penalty was set up for")

    def _empty_like(self, x):
        import torch
        return torch.empty_like(x)

    # --- operations (GibbsPenalty.inl) ---
    def compute_value(self, x) -> float:
        self._ready()
        self._check_image(x)
        v = ctypes.c_double()
        _abi.check(self._lib.b200rt_gibbs_value_dev(self._h, _ptr(x), ctypes.byref(v), _stream()), what="compute_value",
                   gibbs=self._h)
        return v.value

    def compute_gradient(self, x, out=None):
        self._ready()
        self._check_image(x)
        out = self._empty_like(x) if out is None else out
        self._check_image(out)
        _abi.check(self._lib.b200rt_gibbs_gradient_dev(self._h, _ptr(x), _ptr(out), _stream()),
                   what="compute_gradient", gibbs=self._h)
        return out

    def compute_gradient_times_input(self, input_image, x) -> float:
        self._ready()
        self._check_image(x)
        self._check_image(input_image)
        v = ctypes.c_double()
        _abi.check(self._lib.b200rt_gibbs_gradient_times_input_dev(self._h, _ptr(input_image), _ptr(x), ctypes.byref(v),
                                                                   _stream()),
                   what="compute_gradient_times_input", gibbs=self._h)
        return v.value

    def compute_Hessian_diagonal(self, x, out=None):
        self._ready()
        self._check_image(x)
        out = self._empty_like(x) if out is None else out
        self._check_image(out)
        _abi.check(self._lib.b200rt_gibbs_hessian_diagonal_dev(self._h, _ptr(x), _ptr(out), _stream()),
                   what="compute_Hessian_diagonal", gibbs=self._h)
        return out

    def accumulate_Hessian_times_input(self, output, x, input_image):
        """output += H(x) input_image (in place); returns output."""
        self._ready()
        for t in (output, x, input_image):
            self._check_image(t)
        _abi.check(self._lib.b200rt_gibbs_accumulate_hessian_times_input_dev(self._h, _ptr(x), _ptr(input_image),
                                                                             _ptr(output), _stream()),
                   what="accumulate_Hessian_times_input", gibbs=self._h)
        return output

    def compute_Hessian(self, coords, x, out=None):
        """The Hessian row of voxel coords = (z, y, x) (0-based), as an image."""
        self._ready()
        self._check_image(x)
        out = self._empty_like(x) if out is None else out
        self._check_image(out)
        z, y, xx = map(int, coords)
        _abi.check(self._lib.b200rt_gibbs_hessian_dev(self._h, _ptr(x), z, y, xx, _ptr(out), _stream()),
                   what="compute_Hessian", gibbs=self._h)
        return out


class GibbsQuadraticPenalty(GibbsPenalty):
    """phi(a, b) = (a - b)^2 / 4 (QuadraticPotential, GibbsQuadraticPenalty.h); registered as "Gibbs Quadratic"."""

    potential = _abi.GIBBS_QUADRATIC
    registered_name = "Gibbs Quadratic"


class GibbsRelativeDifferencePenalty(GibbsPenalty):
    """phi(a, b) = (a - b)^2 / (2 (a + b + gamma |a - b| + epsilon)) (RelativeDifferencePotential,
    GibbsRelativeDifferencePenalty.h); registered as "Gibbs Relative Difference"."""

    potential = _abi.GIBBS_RELATIVE_DIFFERENCE
    registered_name = "Gibbs Relative Difference"

    def __init__(self, only_2D: bool = False, penalisation_factor: float = 0.0, gamma: float = 2.0,
                 epsilon: float = 1e-7, device: int = 0):
        super().__init__(only_2D, penalisation_factor, device)
        self.gamma = float(gamma)
        self.epsilon = float(epsilon)

    def _potential_params(self):
        return self.gamma, self.epsilon


# The reference's CUDA classes (src/include/stir/recon_buildblock/CUDA/CudaGibbsPenalty.h) run on the same kernels;
# their gradient takes the CUDA build's arithmetic (float sums, CudaGibbsPenalty.cuh:141-206), the other
# operations GibbsPenalty.inl's.
class CudaGibbsQuadraticPenalty(GibbsQuadraticPenalty):
    registered_name = "Cuda Gibbs Quadratic"
    arithmetic = _abi.GIBBS_ARITH_CUDA


class CudaGibbsRelativeDifferencePenalty(GibbsRelativeDifferencePenalty):
    registered_name = "Cuda Gibbs Relative Difference"
    arithmetic = _abi.GIBBS_ARITH_CUDA


REGISTRY = {c.registered_name: c for c in (GibbsQuadraticPenalty, GibbsRelativeDifferencePenalty,
                                          CudaGibbsQuadraticPenalty, CudaGibbsRelativeDifferencePenalty)}


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
