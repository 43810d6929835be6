"""torch.autograd wrappers of the B200 projector pair and of the Poisson objective.

* `forward_project(x, projector)`: A x, whose backward is the hand-written back projector A^T g.
* `back_project(y, projector)`: A^T y, whose backward is A g.
* `PoissonLogLikelihood`: the objective of PoissonLogLikelihoodWithLinearModelForMeanAndProjData
  (value: accumulate_loglikelihood in FP64; gradient: A^T[divide_and_truncate(y, A x + a) - m],
  ...AndProjData.cxx:1421-1515).  Only x is saved for backward: the projection A x is recomputed
  there, so a batch needs no stored sinograms however large it is.
* `Prior`: QuadraticPrior / RelativeDifferencePrior value and gradient on the device.

Images are torch float32 CUDA tensors in the device layout [y][x][z] (or a batch [B][y][x][z]);
projection data in the device layout (flat, or [B][bins]).
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi
from .projectors import RayTracingProjector, _stream_ptr


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _batched(t, per_item):
    return t.dim() > 1 and t.numel() != per_item


class _ForwardProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, proj: RayTracingProjector, subset_num, num_subsets, mode):
        ctx.proj, ctx.subset, ctx.nsub, ctx.mode = proj, subset_num, num_subsets, mode
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        xs = x.detach().contiguous().reshape(-1, n_img)
        out = torch.zeros((xs.shape[0], proj.projdata_size), dtype=torch.float32, device=x.device)
        for b in range(xs.shape[0]):
            proj.forward_dev(xs[b], out=out[b], subset_num=subset_num, num_subsets=num_subsets)
        return out if _batched(x, n_img) else out[0]

    @staticmethod
    def backward(ctx, g):
        proj = ctx.proj
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        gs = g.contiguous().reshape(-1, proj.projdata_size)
        out = torch.empty((gs.shape[0], n_img), dtype=torch.float32, device=g.device)
        for b in range(gs.shape[0]):
            proj.back_dev(gs[b], out=out[b], subset_num=ctx.subset, num_subsets=ctx.nsub, mode=ctx.mode)
        shape = (gs.shape[0],) + proj.device_image_shape if g.dim() > 1 else proj.device_image_shape
        return out.reshape(shape), None, None, None, None


class _BackProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, proj: RayTracingProjector, subset_num, num_subsets, mode):
        ctx.proj, ctx.subset, ctx.nsub = proj, subset_num, num_subsets
        ys = y.detach().contiguous().reshape(-1, proj.projdata_size)
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        out = torch.empty((ys.shape[0], n_img), dtype=torch.float32, device=y.device)
        for b in range(ys.shape[0]):
            proj.back_dev(ys[b], out=out[b], subset_num=subset_num, num_subsets=num_subsets, mode=mode)
        shape = (ys.shape[0],) + proj.device_image_shape if y.dim() > 1 else proj.device_image_shape
        return out.reshape(shape)

    @staticmethod
    def backward(ctx, g):
        proj = ctx.proj
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        gs = g.contiguous().reshape(-1, n_img)
        out = torch.zeros((gs.shape[0], proj.projdata_size), dtype=torch.float32, device=g.device)
        for b in range(gs.shape[0]):
            proj.forward_dev(gs[b], out=out[b], subset_num=ctx.subset, num_subsets=ctx.nsub)
        return (out if gs.shape[0] > 1 or g.dim() > 3 else out[0]), None, None, None, None


def forward_project(x, projector, subset_num=0, num_subsets=1, mode=_abi.BACKPROJECT_ATOMIC):
    return _ForwardProject.apply(x, projector, subset_num, num_subsets, mode)


def back_project(y, projector, subset_num=0, num_subsets=1, mode=_abi.BACKPROJECT_ATOMIC):
    return _BackProject.apply(y, projector, subset_num, num_subsets, mode)


class _LogLikelihood(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, proj, y, additive, mult, subset_num, num_subsets, zero_ends, mode):
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        xs = x.detach().contiguous().reshape(-1, n_img)
        B = xs.shape[0]
        ys = y.reshape(B, -1)
        adds = None if additive is None else additive.reshape(B, -1) if additive.numel() == B * proj.projdata_size else None
        total = 0.0
        out = ctypes.c_double(0.0)
        for b in range(B):
            a = additive if additive is None or additive.numel() == proj.projdata_size else adds[b]
            m = mult if mult is None or mult.numel() == proj.projdata_size else mult.reshape(B, -1)[b]
            _abi.check(proj.lib.b200rt_log_likelihood_dev(proj.h, _p(xs[b]), _p(ys[b]), _p(a), _p(m), subset_num,
                                                          num_subsets, int(zero_ends), ctypes.byref(out),
                                                          _stream_ptr(None)), proj.h, "b200rt_log_likelihood_dev")
            total += out.value
        ctx.save_for_backward(x)
        ctx.args = (proj, y, additive, mult, subset_num, num_subsets, zero_ends, mode)
        return torch.tensor(total, dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx, gout):
        (x,) = ctx.saved_tensors
        proj, y, additive, mult, subset_num, num_subsets, zero_ends, mode = ctx.args
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        xs = x.detach().contiguous().reshape(-1, n_img)
        B = xs.shape[0]
        ys = y.reshape(B, -1)
        grad = torch.empty_like(xs)
        for b in range(B):
            a = additive if additive is None or additive.numel() == proj.projdata_size else additive.reshape(B, -1)[b]
            m = mult if mult is None or mult.numel() == proj.projdata_size else mult.reshape(B, -1)[b]
            _abi.check(proj.lib.b200rt_log_likelihood_gradient_dev(proj.h, _p(xs[b]), _p(ys[b]), _p(a), _p(m), subset_num,
                                                                   num_subsets, int(zero_ends), mode, _p(grad[b]),
                                                                   _stream_ptr(None)), proj.h,
                       "b200rt_log_likelihood_gradient_dev")
        return (grad.reshape(x.shape) * gout.to(torch.float32)), None, None, None, None, None, None, None, None


class PoissonLogLikelihood(torch.nn.Module):
    """Sum over the batch of the subset log-likelihood sum_i y log ybar - ybar, ybar = (A x + a) m, clipped as
    STIR's accumulate_loglikelihood.  Differentiable in x; `forward` returns a float64 scalar tensor."""

    def __init__(self, projector: RayTracingProjector, y, additive=None, mult=None, subset_num=0, num_subsets=1,
                 zero_seg0_end_planes=False, mode=_abi.BACKPROJECT_ATOMIC):
        super().__init__()
        self.proj = projector
        self.y, self.additive, self.mult = y.contiguous(), additive, mult
        self.subset_num, self.num_subsets = subset_num, num_subsets
        self.zero_ends, self.mode = zero_seg0_end_planes, mode

    def forward(self, x):
        return _LogLikelihood.apply(x, self.proj, self.y, self.additive, self.mult, self.subset_num, self.num_subsets,
                                    self.zero_ends, self.mode)


class _Prior(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, proj, prior):
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        xs = x.detach().contiguous().reshape(-1, n_img)
        pa = prior.as_abi()
        total = 0.0
        v = ctypes.c_double(0.0)
        for b in range(xs.shape[0]):
            _abi.check(proj.lib.b200rt_prior_value_dev(proj.h, ctypes.byref(pa), _p(xs[b]), ctypes.byref(v),
                                                       _stream_ptr(None)), proj.h, "b200rt_prior_value_dev")
            total += v.value
        ctx.save_for_backward(x)
        ctx.args = (proj, prior)
        return torch.tensor(total, dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx, gout):
        (x,) = ctx.saved_tensors
        proj, prior = ctx.args
        n_img = proj.geometry.nz * proj.geometry.ny * proj.geometry.nx
        xs = x.detach().contiguous().reshape(-1, n_img)
        grad = torch.empty_like(xs)
        pa = prior.as_abi()
        for b in range(xs.shape[0]):
            _abi.check(proj.lib.b200rt_prior_gradient_dev(proj.h, ctypes.byref(pa), _p(xs[b]), _p(grad[b]),
                                                          _stream_ptr(None)), proj.h, "b200rt_prior_gradient_dev")
        return grad.reshape(x.shape) * gout.to(torch.float32), None, None


class Prior(torch.nn.Module):
    """Penalty R(x) of a QuadraticPrior / RelativeDifferencePrior (stir_b200.osmaposl), summed over the batch."""

    def __init__(self, projector: RayTracingProjector, prior):
        super().__init__()
        self.proj, self.prior = projector, prior

    def forward(self, x):
        return _Prior.apply(x, self.proj, self.prior)
