"""Batched OSMAPOSL: many reconstructions (dynamic frames, noise realisations) advanced together.

STIR reconstructs the frames of a dynamic study one at a time, one OSMAPOSLReconstruction per frame
(src/iterative/OSMAPOSL/OSMAPOSLReconstruction.cxx:371-516 per sub-iteration).  Here every frame keeps
its own projector (image size), data, sensitivities, subset count and prior, and batched sub-iteration
k advances each frame that has k or more sub-iterations by its own sub-iteration k, with subset
(start_subset_num + k - 1) % num_subsets as IterativeReconstruction::get_subset_num.  Per k the device
runs one persistent forward launch and one persistent back projection over the subsets of all frames,
optionally captured with the per-frame thresholds and updates into one CUDA graph.

The result of each frame equals OSMAPOSLReconstruction.reconstruct: with the atomic back projection up to the
order of float additions in the back projection, with the deterministic one bit for bit.
"""
from __future__ import annotations

import ctypes
from typing import List

from . import _abi
from .osmaposl import OSMAPOSLReconstruction, threshold_min_to_small_positive_value, _ptr
from .projectors import _stream_ptr


class BatchedOSMAPOSL:
    """Frames are OSMAPOSLReconstruction objects (set up or not) with their estimates."""

    def __init__(self, device: int = 0):
        self.lib = _abi.load_library()
        h = ctypes.c_void_p()
        st = self.lib.b200rt_batch_create(int(device), ctypes.byref(h))
        if st != _abi.OK:
            raise _abi.B200Error(f"b200rt_batch_create failed with status {st}")
        self.b = h
        self.frames: List[tuple] = []  # keeps the tensors alive while the batch refers to them

    def _check(self, status, what):
        _abi.check(status, None, what, batch=self.b)

    def add(self, recon: OSMAPOSLReconstruction, x) -> int:
        """Adds recon with estimate x (device layout, updated in place).  recon runs its sub-iterations
        1..num_subiterations; it must start at sub-iteration 1.  A deterministic back projection (recon's
        back_projection_mode) makes the frame bit-reproducible and equal to its own one-frame run (non-TOF
        projectors)."""
        if recon.start_subiteration_num != 1:
            raise ValueError("a batched frame starts at sub-iteration 1")
        if recon.sensitivities is None:
            recon.set_up()
        if recon.enforce_initial_positivity:
            threshold_min_to_small_positive_value(x, 0.000001)
        sens = (ctypes.c_void_p * recon.num_subsets)(*[s.data_ptr() for s in recon.sensitivities])
        prior = recon._prior_abi()
        idx = ctypes.c_int(-1)
        self._check(self.lib.b200rt_batch_add_frame(
            self.b, recon.proj.h, _ptr(x), _ptr(recon.y), _ptr(recon.additive), sens, recon.num_subsets,
            recon.start_subset_num, recon.num_subiterations, int(recon.zero_seg0_end_planes), prior,
            float(recon.min_rel), float(recon.max_rel), ctypes.byref(idx)), "b200rt_batch_add_frame")
        if recon.mode != _abi.BACKPROJECT_ATOMIC:
            self._check(self.lib.b200rt_batch_set_frame_mode(self.b, idx.value, recon.mode), "b200rt_batch_set_frame_mode")
        self.frames.append((recon, x, sens))
        return idx.value

    @property
    def num_subiterations(self) -> int:
        return max((r.num_subiterations for r, _, _ in self.frames), default=0)

    def autotune(self, subiteration: int = 1) -> dict:
        cfg = _abi.BatchConfig()
        self._check(self.lib.b200rt_batch_autotune(self.b, int(subiteration), ctypes.byref(cfg)),
                    "b200rt_batch_autotune")
        return dict(ctas_per_sm_forward=cfg.ctas_per_sm_forward, ctas_per_sm_back=cfg.ctas_per_sm_back,
                    order=cfg.order, kernels=cfg.kernels)

    def set_config(self, ctas_per_sm_forward: int = 0, ctas_per_sm_back: int = 0, order: int = 0,
                   kernels: int = _abi.BATCH_KERNELS_AUTO):
        """kernels: the kernel family (_abi.BATCH_KERNELS_*); AUTO takes the first the frames allow."""
        cfg = _abi.BatchConfig(ctas_per_sm_forward, ctas_per_sm_back, order, kernels)
        self._check(self.lib.b200rt_batch_set_config(self.b, ctypes.byref(cfg)), "b200rt_batch_set_config")

    def get_config(self) -> dict:
        cfg = _abi.BatchConfig()
        self._check(self.lib.b200rt_batch_get_config(self.b, ctypes.byref(cfg)), "b200rt_batch_get_config")
        return dict(ctas_per_sm_forward=cfg.ctas_per_sm_forward, ctas_per_sm_back=cfg.ctas_per_sm_back,
                    order=cfg.order, kernels=cfg.kernels)

    def run(self, first: int = 1, count: int | None = None, use_graph: bool = True, stream=None):
        """Batched sub-iterations first..first+count-1 (default: to the last frame's end)."""
        if count is None:
            count = self.num_subiterations - first + 1
        self._check(self.lib.b200rt_batch_run(self.b, int(first), int(count), int(use_graph), _stream_ptr(stream)),
                    "b200rt_batch_run")

    def reconstruct(self, use_graph: bool = True, stream=None):
        self.run(1, None, use_graph, stream)
        return [x for _, x, _ in self.frames]

    def num_cancelled(self, frame: int) -> int:
        n = ctypes.c_int64(0)
        self._check(self.lib.b200rt_batch_get_num_cancelled(self.b, int(frame), ctypes.byref(n)),
                    "b200rt_batch_get_num_cancelled")
        return n.value

    def close(self):
        if getattr(self, "b", None):
            self.lib.b200rt_batch_destroy(self.b)
            self.b = None
            self.frames = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
