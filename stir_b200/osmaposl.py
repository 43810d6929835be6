"""Device-resident OSMAPOSL / OSEM on the B200 projector pair.

Mirrors STIR's OSMAPOSLReconstruction (src/iterative/OSMAPOSL/OSMAPOSLReconstruction.cxx) driven by
IterativeReconstruction::reconstruct (src/recon_buildblock/IterativeReconstruction.cxx:400-425) with the
PoissonLogLikelihoodWithLinearModelForMeanAndProjData objective: the measured data y, the additive term a,
the multiplicative factors m and the estimate stay in HBM between sub-iterations; each sub-iteration is
one fused forward-projection/ratio kernel, one back projection and two elementwise kernels.

Parameters keep STIR's .par names (as keyword arguments): num_subsets, num_subiterations, start_subset_num,
start_subiteration_num, uniformly_randomise_subset_order (+ subset_order_seed), zero_seg0_end_planes,
use_subset_sensitivities, maximum/minimum_relative_change, enforce_initial_positivity, prior (QuadraticPrior /
RelativeDifferencePrior), MAP_model.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional

from . import _abi
from .projectors import RayTracingProjector, _stream_ptr
from .subsets import SubsetOrder


@dataclasses.dataclass
class QuadraticPrior:
    """QuadraticPrior (src/recon_buildblock/QuadraticPrior.cxx), 3x3x3 weights 1/distance."""
    penalisation_factor: float = 0.0
    only_2D: bool = False
    kappa: Optional[object] = None  # torch tensor, device layout

    def as_abi(self, map_model=_abi.MAP_MULTIPLICATIVE):
        return _abi.Prior(type=_abi.PRIOR_QUADRATIC, penalisation_factor=self.penalisation_factor, gamma=0.0, epsilon=0.0,
                          only_2D=int(self.only_2D), map_model=map_model,
                          kappa_dev=None if self.kappa is None else self.kappa.data_ptr())


@dataclasses.dataclass
class RelativeDifferencePrior:
    """RelativeDifferencePrior (src/recon_buildblock/RelativeDifferencePrior.cxx), defaults gamma=2, epsilon=0."""
    penalisation_factor: float = 0.0
    gamma: float = 2.0
    epsilon: float = 0.0
    only_2D: bool = False
    kappa: Optional[object] = None

    def as_abi(self, map_model=_abi.MAP_MULTIPLICATIVE):
        return _abi.Prior(type=_abi.PRIOR_RELATIVE_DIFFERENCE, penalisation_factor=self.penalisation_factor,
                          gamma=self.gamma, epsilon=self.epsilon, only_2D=int(self.only_2D), map_model=map_model,
                          kappa_dev=None if self.kappa is None else self.kappa.data_ptr())


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class OSMAPOSLReconstruction:
    """OSMAPOSL on device-resident data.  `y`, `additive`, `mult` are device-layout projection data
    (torch float32 CUDA tensors); images are device-layout tensors [y][x][z]."""

    def __init__(self, projector: RayTracingProjector, y, additive=None, mult=None, num_subsets: int = 1,
                 num_subiterations: int = 1, start_subset_num: int = 0, start_subiteration_num: int = 1,
                 zero_seg0_end_planes: bool = False, use_subset_sensitivities: bool = True,
                 maximum_relative_change: float = 3.4028234663852886e38, minimum_relative_change: float = 0.0,
                 enforce_initial_positivity: bool = True, prior=None, MAP_model: str = "multiplicative",
                 back_projection_mode: int = _abi.BACKPROJECT_ATOMIC, stream=None,
                 uniformly_randomise_subset_order: bool = False, subset_order_seed=None,
                 use_tofsens: bool = False, sensitivity_mult=None):
        if num_subsets < 1 or num_subsets > projector.geometry.num_views:
            raise ValueError("number of subsets out of range")
        if MAP_model not in ("additive", "multiplicative"):
            raise ValueError('MAP_model has to be "additive" or "multiplicative"')
        self.proj = projector
        self.y, self.additive, self.mult = y, additive, mult
        self.num_subsets = num_subsets
        self.num_subiterations = num_subiterations
        self.start_subset_num = start_subset_num
        self.start_subiteration_num = start_subiteration_num
        self.zero_seg0_end_planes = zero_seg0_end_planes
        self.use_subset_sensitivities = use_subset_sensitivities
        self.max_rel = maximum_relative_change
        self.min_rel = minimum_relative_change
        self.enforce_initial_positivity = enforce_initial_positivity
        self.prior = prior
        self.map_model = _abi.MAP_ADDITIVE if MAP_model == "additive" else _abi.MAP_MULTIPLICATIVE
        self.mode = back_projection_mode
        self.stream = stream
        self.subiteration_num = start_subiteration_num
        self.subset_order = SubsetOrder(num_subsets, start_subset_num, uniformly_randomise_subset_order,
                                        subset_order_seed)
        self.sensitivities = None
        self.last_num_cancelled = 0
        # TOF data: the sensitivity comes from the non-TOF projector with non-TOF multiplicative factors unless
        # use_tofsens (PoissonLogLikelihoodWithLinearModelForMeanAndProjData.cxx:642-670)
        self.use_tofsens = bool(use_tofsens)
        self.sensitivity_mult = sensitivity_mult
        if projector.info.num_tof_bins > 1 and not use_tofsens and mult is not None and sensitivity_mult is None:
            raise ValueError("TOF data with multiplicative factors: give their non-TOF factors as sensitivity_mult "
                             "(or set use_tofsens)")

    # PoissonLogLikelihoodWithLinearModelForMean::compute_sensitivities / set_total_or_subset_sensitivities
    # (PoissonLogLikelihoodWithLinearModelForMean.cxx:372-455)
    def set_up(self):
        import torch
        tof = self.proj.info.num_tof_bins > 1
        sp = self.proj if (self.use_tofsens or not tof) else self.proj.non_tof_projector()
        mult = self.mult if sp is self.proj else self.sensitivity_mult
        lib, h = sp.lib, sp.h
        subs = []
        for s in range(self.num_subsets):
            t = sp.empty_image(zero=False)
            _abi.check(lib.b200rt_sensitivity_dev(h, _ptr(mult), _ptr(t), s, self.num_subsets,
                                                  int(self.zero_seg0_end_planes), self.mode, _stream_ptr(self.stream)), h,
                       "b200rt_sensitivity_dev")
            subs.append(t)
        if self.use_subset_sensitivities:
            self.sensitivities = subs
        else:
            total = subs[0]
            for t in subs[1:]:
                total += t
            avg = total / self.num_subsets
            self.sensitivities = [avg] * self.num_subsets
        self.total_sensitivity = sum(subs[1:], subs[0].clone()) if self.use_subset_sensitivities else total
        return self

    def get_subset_num(self):
        """IterativeReconstruction::get_subset_num (IterativeReconstruction.cxx:628-640), in order or uniformly
        randomised (subsets.SubsetOrder)."""
        return self.subset_order(self.subiteration_num)

    def _prior_abi(self):
        return None if self.prior is None else ctypes.byref(self.prior.as_abi(self.map_model))

    def update_estimate(self, x, update_out=None):
        lib, h = self.proj.lib, self.proj.h
        subset = self.get_subset_num()
        _abi.check(lib.b200rt_osmaposl_subiteration_dev(
            h, _ptr(x), _ptr(self.y), _ptr(self.additive), _ptr(self.sensitivities[subset]), subset, self.num_subsets,
            self.subiteration_num, int(self.zero_seg0_end_planes), self._prior_abi(), float(self.min_rel),
            float(self.max_rel), self.mode, _ptr(update_out), _stream_ptr(self.stream)), h,
            "b200rt_osmaposl_subiteration_dev")
        return x

    def num_cancelled(self):
        n = ctypes.c_int64(0)
        _abi.check(self.proj.lib.b200rt_get_num_cancelled(self.proj.h, ctypes.byref(n)), self.proj.h, "num_cancelled")
        return n.value

    def reconstruct(self, x):
        """Runs sub-iterations start_subiteration_num..num_subiterations on x (device layout, in place)."""
        if self.sensitivities is None:
            self.set_up()
        if self.enforce_initial_positivity:
            threshold_min_to_small_positive_value(x, 0.000001)
        for self.subiteration_num in range(self.start_subiteration_num, self.num_subiterations + 1):
            self.update_estimate(x)
        return x


def threshold_min_to_small_positive_value(x, small_number: float):
    """thresholding.h:101-109: values below (smallest positive value * small_number) are raised to it."""
    import torch
    pos = x[x > 0]
    if pos.numel() == 0:
        x.fill_(small_number)
    else:
        x.clamp_(min=float(pos.min()) * small_number)
    return x


def log_likelihood(projector: RayTracingProjector, x, y, additive=None, mult=None, subset_num=0, num_subsets=1,
                   zero_seg0_end_planes=False, stream=None) -> float:
    out = ctypes.c_double(0.0)
    _abi.check(projector.lib.b200rt_log_likelihood_dev(projector.h, _ptr(x), _ptr(y), _ptr(additive), _ptr(mult),
                                                       subset_num, num_subsets, int(zero_seg0_end_planes),
                                                       ctypes.byref(out), _stream_ptr(stream)), projector.h,
               "b200rt_log_likelihood_dev")
    return out.value


def prior_gradient(projector: RayTracingProjector, prior, x, out=None, stream=None):
    out = projector.empty_image(zero=False) if out is None else out
    _abi.check(projector.lib.b200rt_prior_gradient_dev(projector.h, ctypes.byref(prior.as_abi()), _ptr(x), _ptr(out),
                                                       _stream_ptr(stream)), projector.h, "b200rt_prior_gradient_dev")
    return out


def prior_hessian_times_input(projector: RayTracingProjector, prior, x, input_image, out=None, stream=None):
    """out += the prior's Hessian at x times input_image (accumulate_Hessian_times_input of QuadraticPrior /
    RelativeDifferencePrior); device-layout images.  out defaults to zeros."""
    out = projector.empty_image() if out is None else out
    _abi.check(projector.lib.b200rt_prior_hessian_times_input_dev(
        projector.h, ctypes.byref(prior.as_abi()), _ptr(x), _ptr(input_image), _ptr(out), _stream_ptr(stream)),
        projector.h, "b200rt_prior_hessian_times_input_dev")
    return out
