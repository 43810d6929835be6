"""List-mode Poisson objective with the B200 ray-tracing matrix, on device-resident events and images.

Mirrors STIR's PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin
(src/recon_buildblock/PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin.cxx): the
events are the objective's cached BinAndCorr records (bin, value, additive term) held on the GPU; the gradient,
value and Hessian-times-input of a subset are one kernel each over the events' rows (listmode.cu), or, once the
events number a fair fraction of the bins, one kernel over the events between the subset's forward and back
projections (the binned method, see set_method).  `ListModeOSEM` runs STIR's
OSMAPOSL update with this objective: x *= (gradient without the sensitivity) / subset sensitivity, with the
sensitivities back-projected from the (binned) multiplicative factors.  Reading vendor list-mode files is not
part of this module: events come as arrays (segment, view, axial, tangential, timing) with values.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _abi
from .projectors import RayTracingProjector, _stream_ptr

EVENT_DTYPE = np.dtype([("segment", "<i4"), ("view", "<i4"), ("axial_pos", "<i4"), ("tangential_pos", "<i4"),
                        ("timing_pos", "<i4"), ("value", "<f4"), ("corr", "<f4")])
assert EVENT_DTYPE.itemsize == ctypes.sizeof(_abi.LmEvent)


def pack_events(bins, values=None, corr=None, device=0):
    """A device tensor of b200rt_lm_event records from bins (n, 5) = (segment, view, axial, tangential, timing),
    values (default 1) and additive terms (default 0)."""
    import torch
    bins = np.asarray(bins, np.int32).reshape(-1, 5)
    ev = np.zeros(bins.shape[0], EVENT_DTYPE)
    for i, k in enumerate(["segment", "view", "axial_pos", "tangential_pos", "timing_pos"]):
        ev[k] = bins[:, i]
    ev["value"] = 1.0 if values is None else np.asarray(values, np.float32)
    ev["corr"] = 0.0 if corr is None else np.asarray(corr, np.float32)
    return torch.from_numpy(ev.view(np.uint8).copy()).to(torch.device("cuda", device))


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin:
    """`events`: a device tensor from pack_events.  Images in the projector's device layout."""

    def __init__(self, projector: RayTracingProjector, events, num_subsets: int = 1, has_add: bool = False):
        self.proj = projector
        self.events = events
        self.num_events = events.numel() // EVENT_DTYPE.itemsize
        self.num_subsets = num_subsets
        self.has_add = bool(has_add)

    def set_method(self, method: int):
        """_abi.LISTMODE_AUTO (default), LISTMODE_PER_EVENT (one row walk per event) or LISTMODE_BINNED (A x of
        the subset read per event, the events' terms summed per bin and back projected once); the method is a
        setting of the projector."""
        _abi.check(self.proj.lib.b200rt_listmode_set_method(self.proj.h, int(method)), self.proj.h,
                   "b200rt_listmode_set_method")

    def compute_sub_gradient_without_penalty(self, x, subset_num: int, subset_sensitivity=None, out=None,
                                             accumulate=False, stream=None):
        """sum over the subset's events of A_e^T y_e / (A_e x + c_e), minus subset_sensitivity when given
        (actual_compute_subset_gradient_without_penalty with add_sensitivity = subset_sensitivity is None)."""
        out = self.proj.empty_image(zero=False) if out is None else out
        _abi.check(self.proj.lib.b200rt_listmode_gradient_dev(self.proj.h, _p(self.events), self.num_events, _p(x),
                                                              subset_num, self.num_subsets, int(self.has_add),
                                                              _p(subset_sensitivity), int(accumulate), _p(out),
                                                              _stream_ptr(stream)),
                   self.proj.h, "b200rt_listmode_gradient_dev")
        return out

    def compute_objective_function_without_penalty(self, x, subset_num: int = 0, stream=None) -> float:
        v = ctypes.c_double()
        _abi.check(self.proj.lib.b200rt_listmode_value_dev(self.proj.h, _p(self.events), self.num_events, _p(x),
                                                           subset_num, self.num_subsets, int(self.has_add),
                                                           ctypes.byref(v), _stream_ptr(stream)),
                   self.proj.h, "b200rt_listmode_value_dev")
        return v.value

    def accumulate_sub_Hessian_times_input_without_penalty(self, output, x, rhs, subset_num: int, stream=None):
        _abi.check(self.proj.lib.b200rt_listmode_hessian_times_input_dev(self.proj.h, _p(self.events), self.num_events,
                                                                         _p(x), _p(rhs), subset_num, self.num_subsets,
                                                                         int(self.has_add), _p(output),
                                                                         _stream_ptr(stream)),
                   self.proj.h, "b200rt_listmode_hessian_times_input_dev")
        return output

    def num_invalid_events(self) -> int:
        n = ctypes.c_int64()
        _abi.check(self.proj.lib.b200rt_listmode_num_invalid(self.proj.h, ctypes.byref(n)), self.proj.h,
                   "b200rt_listmode_num_invalid")
        return n.value


class ListModeOSEM:
    """OSMAPOSL (no prior) with the list-mode objective: x *= grad_S(x) / sens_S per sub-iteration, the
    sensitivities A_S^T m of the binned multiplicative factors m (ones when None)."""

    def __init__(self, objective: PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin,
                 mult=None, min_relative_change: float = 0.0, max_relative_change: float = 3.4028234663852886e38):
        self.obj = objective
        self.proj = objective.proj
        self.mult = mult
        self.min_rel, self.max_rel = min_relative_change, max_relative_change
        self.sens = []
        for s in range(objective.num_subsets):
            t = self.proj.empty_image(zero=False)
            _abi.check(self.proj.lib.b200rt_sensitivity_dev(self.proj.h, _p(mult), _p(t), s, objective.num_subsets, 0,
                                                            _abi.BACKPROJECT_ATOMIC, _stream_ptr(None)),
                       self.proj.h, "b200rt_sensitivity_dev")
            self.sens.append(t)
        self.subiteration = 0

    def update_estimate(self, x):
        self.subiteration += 1
        nsub = self.obj.num_subsets
        subset = (self.subiteration - 1) % nsub
        u = self.obj.compute_sub_gradient_without_penalty(x, subset)
        _abi.check(self.proj.lib.b200rt_osmaposl_apply_update_dev(self.proj.h, _p(x), _p(u), _p(self.sens[subset]), nsub,
                                                                  self.subiteration, None, float(self.min_rel),
                                                                  float(self.max_rel), _stream_ptr(None)),
                   self.proj.h, "b200rt_osmaposl_apply_update_dev")
        return x
