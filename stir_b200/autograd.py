"""torch.autograd wrappers of the B200 projector pair and of the Poisson objective.

* `forward_project(x, projector)`: A x, whose backward is the hand-written back projector A^T g.
* `back_project(y, projector)`: A^T y, whose backward is A g.
  A batch [B][...] goes through the batch entry points: one launch over (path item, image) per direction.
* `PoissonLogLikelihood`: the objective of PoissonLogLikelihoodWithLinearModelForMeanAndProjData
  (value: accumulate_loglikelihood in FP64; gradient: A^T[divide_and_truncate(y, A x + a) - m],
  ...AndProjData.cxx:1421-1515).  The forward pass projects once and, when the batch's gradient ratios fit in
  free device memory, keeps them for backward, which is then one back projection; otherwise only x is saved and
  backward projects again (`store_ratio`: None decides by the free memory, True / False force either).
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


def _forward_batch(proj, xs, out, subset_num, num_subsets):
    """out[b] = A xs[b] for the images of xs [B][image] (one launch over (path item, image))"""
    n_img, n_pd = xs.shape[1], proj.projdata_size
    _abi.check(proj.lib.b200rt_forward_project_batch_dev(proj.h, _p(xs), n_img, _p(out), n_pd, xs.shape[0], subset_num,
                                                         num_subsets, _stream_ptr(None)), proj.h,
               "b200rt_forward_project_batch_dev")
    return out


def _back_batch(proj, ys, out, subset_num, num_subsets, mode):
    """out[b] = A^T ys[b] for the projection data of ys [B][bins]"""
    n_img, n_pd = out.shape[1], proj.projdata_size
    _abi.check(proj.lib.b200rt_back_project_batch_dev(proj.h, _p(ys), n_pd, _p(out), n_img, ys.shape[0], subset_num,
                                                      num_subsets, mode, _stream_ptr(None)), proj.h,
               "b200rt_back_project_batch_dev")
    return out


def _n_img(proj):
    return proj.geometry.nz * proj.geometry.ny * proj.geometry.nx


class _ForwardProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, proj: RayTracingProjector, subset_num, num_subsets, mode):
        ctx.proj, ctx.subset, ctx.nsub, ctx.mode = proj, subset_num, num_subsets, mode
        n_img = _n_img(proj)
        xs = x.detach().contiguous().reshape(-1, n_img)
        out = torch.zeros((xs.shape[0], proj.projdata_size), dtype=torch.float32, device=x.device)
        _forward_batch(proj, xs, out, subset_num, num_subsets)
        return out if _batched(x, n_img) else out[0]

    @staticmethod
    def backward(ctx, g):
        proj = ctx.proj
        n_img = _n_img(proj)
        gs = g.contiguous().reshape(-1, proj.projdata_size)
        out = torch.empty((gs.shape[0], n_img), dtype=torch.float32, device=g.device)
        _back_batch(proj, gs, out, ctx.subset, ctx.nsub, ctx.mode)
        shape = (gs.shape[0],) + proj.device_image_shape if g.dim() > 1 else proj.device_image_shape
        return out.reshape(shape), None, None, None, None


class _BackProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, proj: RayTracingProjector, subset_num, num_subsets, mode):
        ctx.proj, ctx.subset, ctx.nsub = proj, subset_num, num_subsets
        ys = y.detach().contiguous().reshape(-1, proj.projdata_size)
        out = torch.empty((ys.shape[0], _n_img(proj)), dtype=torch.float32, device=y.device)
        _back_batch(proj, ys, out, subset_num, num_subsets, mode)
        shape = (ys.shape[0],) + proj.device_image_shape if y.dim() > 1 else proj.device_image_shape
        return out.reshape(shape)

    @staticmethod
    def backward(ctx, g):
        proj = ctx.proj
        gs = g.contiguous().reshape(-1, _n_img(proj))
        out = torch.zeros((gs.shape[0], proj.projdata_size), dtype=torch.float32, device=g.device)
        _forward_batch(proj, gs, out, ctx.subset, ctx.nsub)
        return (out if gs.shape[0] > 1 or g.dim() > 3 else out[0]), None, None, None, None


def forward_project(x, projector, subset_num=0, num_subsets=1, mode=_abi.BACKPROJECT_ATOMIC):
    """A x for an image [y][x][z] or a batch [B][y][x][z] (device layout); differentiable, backward A^T g."""
    return _ForwardProject.apply(x, projector, subset_num, num_subsets, mode)


def back_project(y, projector, subset_num=0, num_subsets=1, mode=_abi.BACKPROJECT_ATOMIC):
    """A^T y for projection data [bins] or a batch [B][bins] (device layout); differentiable, backward A g."""
    return _BackProject.apply(y, projector, subset_num, num_subsets, mode)


def _data_strides(proj, B, y, additive, mult):
    """(array, stride) of the data of a batch of B images: one array per image (stride = bins) or one shared by
    the batch (stride 0)."""
    n = proj.projdata_size

    def one(t, name):
        if t is None:
            return None, 0
        t = t.contiguous()
        if t.numel() == n:
            return t, 0
        if t.numel() == B * n:
            return t, n
        raise ValueError(f"{name} must hold the projection data of one image or of each of the {B} images")
    return one(y, "y"), one(additive, "additive"), one(mult, "mult")


def _ratio_fits(proj, B, device):
    """Whether B gradient ratios (projection data of each image) fit in the free device memory with room to spare:
    the driver's free memory plus what torch's caching allocator holds unused."""
    free, _ = torch.cuda.mem_get_info(device)
    free += torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
    need = 4 * B * proj.projdata_size
    return need + need // 4 + (512 << 20) <= free


class _LogLikelihood(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, proj, y, additive, mult, subset_num, num_subsets, zero_ends, mode, store_ratio):
        n_img = _n_img(proj)
        xs = x.detach().contiguous().reshape(-1, n_img)
        B = xs.shape[0]
        (yy, ys), (aa, as_), (mm, ms) = _data_strides(proj, B, y, additive, mult)
        values = (ctypes.c_double * B)()
        ctx.ratio = None
        keep = ctx.needs_input_grad[0] and proj.info.num_tof_bins <= 1 and \
            (store_ratio if store_ratio is not None else _ratio_fits(proj, B, x.device))
        if keep:
            # value and gradient ratios from one projection; zeros where none is written (bins outside the subset and
            # of inactive lines), as in the projection the backward would otherwise make: the deterministic back
            # projection takes its fixed-point scale from the largest |value| of the whole array
            n_pd = proj.projdata_size
            ratio = torch.zeros((B, n_pd), dtype=torch.float32, device=x.device)
            st = proj.lib.b200rt_log_likelihood_and_ratio_batch_dev(
                proj.h, _p(xs), n_img, _p(yy), ys, _p(aa), as_, _p(mm), ms, B, subset_num, num_subsets, int(zero_ends),
                values, _p(ratio), n_pd, _stream_ptr(None))
            if st == _abi.OK:
                ctx.ratio = ratio
            elif st != _abi.ERR_UNSUPPORTED:
                _abi.check(st, proj.h, "b200rt_log_likelihood_and_ratio_batch_dev")
        if ctx.ratio is None:
            _abi.check(proj.lib.b200rt_log_likelihood_batch_dev(proj.h, _p(xs), n_img, _p(yy), ys, _p(aa), as_, _p(mm), ms,
                                                                B, subset_num, num_subsets, int(zero_ends), values,
                                                                _stream_ptr(None)), proj.h, "b200rt_log_likelihood_batch_dev")
        ctx.save_for_backward(x)
        ctx.args = (proj, y, additive, mult, subset_num, num_subsets, zero_ends, mode)
        return torch.tensor(sum(values[b] for b in range(B)), dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx, gout):
        (x,) = ctx.saved_tensors
        proj, y, additive, mult, subset_num, num_subsets, zero_ends, mode = ctx.args
        n_img = _n_img(proj)
        xs = x.detach().contiguous().reshape(-1, n_img)
        B = xs.shape[0]
        if ctx.ratio is not None:
            grad = torch.empty_like(xs)
            _back_batch(proj, ctx.ratio, grad, subset_num, num_subsets, mode)
            ctx.ratio = None
            return ((grad.reshape(x.shape) * gout.to(torch.float32)), None, None, None, None, None, None, None, None,
                    None)
        (yy, ys), (aa, as_), (mm, ms) = _data_strides(proj, B, y, additive, mult)
        grad = torch.empty_like(xs)
        _abi.check(proj.lib.b200rt_log_likelihood_gradient_batch_dev(
            proj.h, _p(xs), n_img, _p(yy), ys, _p(aa), as_, _p(mm), ms, B, subset_num, num_subsets, int(zero_ends), mode,
            _p(grad), n_img, _stream_ptr(None)), proj.h, "b200rt_log_likelihood_gradient_batch_dev")
        return (grad.reshape(x.shape) * gout.to(torch.float32)), None, None, None, None, None, None, None, None, None


class PoissonLogLikelihood(torch.nn.Module):
    """Sum over the batch of the subset log-likelihood sum_i y log ybar - ybar, ybar = (A x + a) m, clipped as
    STIR's accumulate_loglikelihood.  Differentiable in x; `forward` returns a float64 scalar tensor."""

    def __init__(self, projector: RayTracingProjector, y, additive=None, mult=None, subset_num=0, num_subsets=1,
                 zero_seg0_end_planes=False, mode=_abi.BACKPROJECT_ATOMIC, store_ratio=None):
        super().__init__()
        self.proj = projector
        self.y, self.additive, self.mult = y.contiguous(), additive, mult
        self.subset_num, self.num_subsets = subset_num, num_subsets
        self.zero_ends, self.mode = zero_seg0_end_planes, mode
        self.store_ratio = store_ratio

    def forward(self, x):
        return _LogLikelihood.apply(x, self.proj, self.y, self.additive, self.mult, self.subset_num, self.num_subsets,
                                    self.zero_ends, self.mode, self.store_ratio)


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
