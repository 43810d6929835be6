"""Device-resident OSSPS on the B200 projector pair.

Mirrors STIR's OSSPSReconstruction (src/iterative/OSSPS/OSSPSReconstruction.cxx) with the
PoissonLogLikelihoodWithLinearModelForMeanAndProjData objective: the precomputed denominator (minus the
approximate Hessian times ones), then per sub-iteration the sub-gradient (with the prior's gradient / number of
subsets), division by the denominator (completed at the first sub-iteration with the Quadratic prior's parabolic
surrogate curvature), relaxation and clamping to [0, upper bound].  Parameters keep STIR's .par names.
"""
from __future__ import annotations

import ctypes

from . import _abi
from .osmaposl import QuadraticPrior, _ptr
from .subsets import SubsetOrder
from .projectors import RayTracingProjector, _stream_ptr


class OSSPSReconstruction:
    """`y`, `additive`, `mult` (the multiplicative term m), `norm` (the normalisation's correction factors n, used
    by the denominator) are device-layout projection data; images are device-layout tensors."""

    def __init__(self, projector: RayTracingProjector, y, additive=None, mult=None, norm=None, num_subsets: int = 1,
                 num_subiterations: int = 1, start_subset_num: int = 0, start_subiteration_num: int = 1,
                 zero_seg0_end_planes: bool = False, relaxation_parameter: float = 1.0, relaxation_gamma: float = 0.1,
                 upper_bound: float = 3.4028234663852886e38, prior=None,
                 back_projection_mode: int = _abi.BACKPROJECT_ATOMIC, stream=None,
                 uniformly_randomise_subset_order: bool = False, subset_order_seed=None):
        if prior is not None and not isinstance(prior, QuadraticPrior):
            raise ValueError("OSSPS needs a prior with a parabolic surrogate (QuadraticPrior)")
        if relaxation_parameter <= 0:
            raise ValueError("OSSPS: relaxation parameter should be positive")
        self.proj = projector
        self.y, self.additive, self.mult, self.norm = y, additive, mult, norm
        self.num_subsets = num_subsets
        self.num_subiterations = num_subiterations
        self.start_subset_num = start_subset_num
        self.start_subiteration_num = start_subiteration_num
        self.zero_seg0_end_planes = zero_seg0_end_planes
        self.relaxation_parameter = relaxation_parameter
        self.relaxation_gamma = relaxation_gamma
        self.upper_bound = upper_bound
        self.prior = prior
        self.mode = back_projection_mode
        self.stream = stream
        self.subiteration_num = start_subiteration_num
        self.subset_order = SubsetOrder(num_subsets, start_subset_num, uniformly_randomise_subset_order,
                                        subset_order_seed)
        self.denominator = None
        self.sensitivity = None

    def set_up(self):
        lib, h = self.proj.lib, self.proj.h
        self.denominator = self.proj.empty_image(zero=False)
        _abi.check(lib.b200rt_ossps_denominator_dev(h, _ptr(self.y), _ptr(self.norm), _ptr(self.denominator), self.mode,
                                                    _stream_ptr(self.stream)), h, "b200rt_ossps_denominator_dev")
        self.sensitivity = self.proj.empty_image(zero=False)
        _abi.check(lib.b200rt_sensitivity_dev(h, _ptr(self.mult), _ptr(self.sensitivity), 0, 1,
                                              int(self.zero_seg0_end_planes), self.mode, _stream_ptr(self.stream)), h,
                   "b200rt_sensitivity_dev")
        return self

    def get_subset_num(self):
        """IterativeReconstruction::get_subset_num (IterativeReconstruction.cxx:628-640), in order or uniformly
        randomised (subsets.SubsetOrder)."""
        return self.subset_order(self.subiteration_num)

    def update_estimate(self, x):
        lib, h = self.proj.lib, self.proj.h
        prior = None if self.prior is None else ctypes.byref(self.prior.as_abi())
        _abi.check(lib.b200rt_ossps_subiteration_dev(
            h, _ptr(x), _ptr(self.denominator), _ptr(self.y), _ptr(self.additive), _ptr(self.mult),
            _ptr(self.sensitivity), self.get_subset_num(), self.num_subsets, self.subiteration_num,
            self.start_subiteration_num, int(self.zero_seg0_end_planes), prior, float(self.relaxation_parameter),
            float(self.relaxation_gamma), float(self.upper_bound), self.mode, _stream_ptr(self.stream)), h,
            "b200rt_ossps_subiteration_dev")
        return x

    def reconstruct(self, x):
        """Runs sub-iterations start_subiteration_num..num_subiterations on x (device layout, in place)."""
        if self.denominator is None:
            self.set_up()
        for self.subiteration_num in range(self.start_subiteration_num, self.num_subiterations + 1):
            self.update_estimate(x)
        return x
