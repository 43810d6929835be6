"""Bin normalisations on device-resident projection data (device layout), through b200rt_normalisation_dev.

Mirrors STIR's BinNormalisationFromProjData (src/recon_buildblock/BinNormalisationFromProjData.cxx: apply
multiplies by the factors, undo divides by them; non-TOF factors serve TOF data), ChainedBinNormalisation
(src/recon_buildblock/ChainedBinNormalisation.cxx: apply and undo run "apply first" then "apply second") and,
as a chain term, BinNormalisationFromAttenuationImage (stir_b200.attenuation).  `factors()` is undo of ones: the
multiplicative term of the Poisson model.
"""
from __future__ import annotations

import ctypes

from . import _abi
from .attenuation import BinNormalisationFromAttenuationImage
from .projectors import RayTracingProjector, _stream_ptr


def _terms(norm):
    if norm is None:
        return []
    if isinstance(norm, BinNormalisationFromAttenuationImage):
        return [_abi.NormTerm(kind=_abi.NORM_ATTENUATION, non_tof=0, data_dev=norm.mu.data_ptr())]
    return norm._terms()


def _run(projector: RayTracingProjector, terms, mode, projdata, stream):
    arr = (_abi.NormTerm * max(len(terms), 1))(*terms)
    _abi.check(projector.lib.b200rt_normalisation_dev(projector.h, arr, len(terms), mode,
                                                      ctypes.c_void_p(projdata.data_ptr()), _stream_ptr(stream)),
               projector.h, "b200rt_normalisation_dev")
    return projdata


class _DeviceNormalisation:
    proj: RayTracingProjector

    def _terms(self):
        raise NotImplementedError

    def apply(self, projdata, stream=None):
        """Normalisation correction, in place."""
        return _run(self.proj, self._terms(), _abi.NORM_APPLY, projdata, stream)

    def undo(self, projdata, stream=None):
        """The normalisation's effect on the data (the forward model), in place."""
        return _run(self.proj, self._terms(), _abi.NORM_UNDO, projdata, stream)

    def factors(self, out=None, stream=None):
        """undo of ones for every bin."""
        out = self.proj.empty_projdata(zero=False) if out is None else out
        return _run(self.proj, self._terms(), _abi.NORM_FACTORS, out, stream)


class BinNormalisationFromProjData(_DeviceNormalisation):
    """`factors` in device layout, of this projector's data, or of its non-TOF data (non_tof=True) for TOF data."""

    def __init__(self, projector: RayTracingProjector, factors, non_tof: bool = False):
        self.proj = projector
        self.norm = factors
        self.non_tof = bool(non_tof)

    def _terms(self):
        return [_abi.NormTerm(kind=_abi.NORM_PROJDATA, non_tof=int(self.non_tof), data_dev=self.norm.data_ptr())]


class ChainedBinNormalisation(_DeviceNormalisation):
    """"Bin Normalisation to apply first" and "... to apply second"; either may be None."""

    def __init__(self, apply_first=None, apply_second=None, projector: RayTracingProjector = None):
        self.apply_first = apply_first
        self.apply_second = apply_second
        self.proj = projector or getattr(apply_first, "proj", None) or getattr(apply_second, "proj", None)
        if self.proj is None:
            raise ValueError("ChainedBinNormalisation needs a projector")

    def _terms(self):
        return _terms(self.apply_first) + _terms(self.apply_second)
