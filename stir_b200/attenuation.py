"""Attenuation on device-resident projection data.

Mirrors STIR's BinNormalisationFromAttenuationImage (src/recon_buildblock/BinNormalisationFromAttenuationImage.cxx):
set_up forward-projects the attenuation image (mu, 1/mm) with the pair's forward projector; apply multiplies
projection data by exp(A mu) (attenuation correction), undo divides by it.  `factors()` gives undo of ones,
1 / exp(A mu): the multiplicative term m of the Poisson model (norm.undo(1) in
PoissonLogLikelihoodWithLinearModelForMeanAndProjData).  Non-TOF only, as STIR.
"""
from __future__ import annotations

import ctypes

from . import _abi
from .projectors import RayTracingProjector, _stream_ptr


class BinNormalisationFromAttenuationImage:
    """`mu` is a device-layout image tensor ([y][x][z], float32, CUDA) on the projector's grid."""

    def __init__(self, projector: RayTracingProjector, mu):
        self.proj = projector
        self.mu = mu

    def _run(self, projdata, mode, stream):
        _abi.check(self.proj.lib.b200rt_attenuation_dev(self.proj.h, ctypes.c_void_p(self.mu.data_ptr()),
                                                         ctypes.c_void_p(projdata.data_ptr()), mode,
                                                         _stream_ptr(stream)), self.proj.h, "b200rt_attenuation_dev")
        return projdata

    def apply(self, projdata, stream=None):
        """projdata *= exp(A mu), in place (device layout)."""
        return self._run(projdata, _abi.ATTENUATION_APPLY, stream)

    def undo(self, projdata, stream=None):
        """projdata /= exp(A mu), in place (device layout)."""
        return self._run(projdata, _abi.ATTENUATION_UNDO, stream)

    def factors(self, out=None, stream=None):
        """1 / exp(A mu) for every bin (device layout)."""
        out = self.proj.empty_projdata(zero=False) if out is None else out
        return self._run(out, _abi.ATTENUATION_FACTORS, stream)
