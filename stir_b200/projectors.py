"""Python side of the B200 ray-tracing projector pair.

`RayTracingProjector` owns one `b200rt_projector` handle (C ABI, include/stir_b200.h).
On top of it, `ForwardProjectorByBinB200RayTracing`, `BackProjectorByBinB200RayTracing`
and `ProjectorByBinPairUsingB200RayTracing` mirror the interface of STIR's
ForwardProjectorByBin / BackProjectorByBin / ProjectorByBinPair
(src/include/stir/recon_buildblock/{ForwardProjectorByBin,BackProjectorByBin,ProjectorByBinPair}.h)
with the same method names, argument meaning and error behaviour (errors raise).

Arrays:
  host (numpy)  image [z][y][x], projection data in ProjDataInMemory order (flat)
  device (torch) image [y][x][z], projection data [segment -S..S][view][tangential][axial]
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _abi
from .geometry import ImageGeometry, ProjDataInfo, make_geometry, non_tof


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _stream_ptr(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


class RayTracingProjector:
    """A set-up ray-tracing projection matrix on one CUDA device (STIR's ProjMatrixByBinUsingRayTracing)."""

    def __init__(self, proj_data_info: ProjDataInfo, image: ImageGeometry, num_tangential_LORs: int = 1,
                 restrict_to_cylindrical_FOV: bool = True, symmetries=(True,) * 5, device: int = 0,
                 geometry: Optional[_abi.Geometry] = None, tof_kernel_truncation_sigmas: float = 0.0):
        self.lib = _abi.load_library()
        self.proj_data_info = proj_data_info
        self.image = image
        self.geometry = geometry if geometry is not None else make_geometry(
            proj_data_info, image, num_tangential_LORs, restrict_to_cylindrical_FOV, symmetries,
            tof_kernel_truncation_sigmas)
        self.device = device
        h = ctypes.c_void_p()
        st = self.lib.b200rt_create(ctypes.byref(self.geometry), device, ctypes.byref(h))
        if st != _abi.OK:
            raise _abi.B200Error(f"b200rt_create failed ({st}): {self.lib.b200rt_last_error(None).decode()}")
        self.h = h
        info = _abi.Info()
        _abi.check(self.lib.b200rt_get_info(self.h, ctypes.byref(info)), self.h, "b200rt_get_info")
        self.info = info
        self._non_tof = None
        self.shard_views = None

    def set_view_shard(self, views=None):
        """Hold the projection data of `views` only (b200rt_set_view_shard): projection-data arrays then have the
        shard's size (`projdata_size`), in the device layout with the views in the order given; None restores the
        whole data."""
        import numpy as np
        if views is None or len(views) == 0:
            _abi.check(self.lib.b200rt_set_view_shard(self.h, None, 0), self.h, "b200rt_set_view_shard")
            self.shard_views = None
        else:
            v = np.ascontiguousarray(views, np.int32)
            _abi.check(self.lib.b200rt_set_view_shard(self.h, v.ctypes.data_as(ctypes.c_void_p), len(v)), self.h,
                       "b200rt_set_view_shard")
            self.shard_views = [int(a) for a in v]
        info = _abi.Info()
        _abi.check(self.lib.b200rt_get_info(self.h, ctypes.byref(info)), self.h, "b200rt_get_info")
        self.info = info
        return self

    def non_tof_projector(self) -> "RayTracingProjector":
        """This projector without timing bins (ProjDataInfo::create_non_tof_clone, the same matrix settings); itself
        for non-TOF data.  STIR back-projects a TOF reconstruction's sensitivity with it unless "use time-of-flight
        sensitivities" is set (PoissonLogLikelihoodWithLinearModelForMeanAndProjData.cxx:642-670).  Made once."""
        if self.info.num_tof_bins <= 1:
            return self
        if self._non_tof is None:
            g = _abi.Geometry.from_buffer_copy(self.geometry)
            g.tof_mash_factor = 0
            self._non_tof = RayTracingProjector(non_tof(self.proj_data_info), self.image, device=self.device, geometry=g)
        return self._non_tof

    def close(self):
        if getattr(self, "h", None):
            self.lib.b200rt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # sizes
    @property
    def projdata_size(self) -> int:
        return int(self.info.num_bins)

    @property
    def image_shape(self):
        return (self.geometry.nz, self.geometry.ny, self.geometry.nx)

    @property
    def device_image_shape(self):
        return (self.geometry.ny, self.geometry.nx, self.geometry.nz)

    def device_status(self, clear: bool = False) -> int:
        """The projector's device status word (0: every kernel completed its work; bit STATUS_STAGING_TIMEOUT: a
        forward projection abandoned path items whose staging copies were not seen to complete).  Synchronises."""
        s = ctypes.c_uint32(0)
        _abi.check(self.lib.b200rt_get_device_status(self.h, ctypes.byref(s), int(clear)), self.h,
                   "b200rt_get_device_status")
        return int(s.value)

    def get_row(self, segment, view, axial, tangential, timing=0):
        n = ctypes.c_int64(0)
        _abi.check(self.lib.b200rt_get_row(self.h, segment, view, axial, tangential, timing, None, None, 0, ctypes.byref(n)),
                   self.h, "b200rt_get_row")
        c = np.zeros((max(n.value, 1), 3), np.int32)
        v = np.zeros(max(n.value, 1), np.float32)
        _abi.check(self.lib.b200rt_get_row(self.h, segment, view, axial, tangential, timing, _np_ptr(c), _np_ptr(v),
                                           n.value, ctypes.byref(n)), self.h, "b200rt_get_row")
        return c[:n.value], v[:n.value]

    # host arrays in STIR order
    def forward_host(self, image: np.ndarray, subset_num: int = 0, num_subsets: int = 1) -> np.ndarray:
        img = np.ascontiguousarray(image, np.float32).reshape(self.image_shape)
        out = np.zeros(self.projdata_size, np.float32)
        _abi.check(self.lib.b200rt_forward_project(self.h, _np_ptr(img), _np_ptr(out), subset_num, num_subsets), self.h,
                   "b200rt_forward_project")
        return out

    def back_host(self, projdata: np.ndarray, subset_num: int = 0, num_subsets: int = 1,
                  mode: int = _abi.BACKPROJECT_ATOMIC) -> np.ndarray:
        pd = np.ascontiguousarray(projdata, np.float32).ravel()
        if pd.size != self.projdata_size:
            raise ValueError("projection data has the wrong size")
        out = np.zeros(self.image_shape, np.float32)
        _abi.check(self.lib.b200rt_back_project(self.h, _np_ptr(pd), _np_ptr(out), subset_num, num_subsets, mode), self.h,
                   "b200rt_back_project")
        return out

    # device tensors (torch) in device layout
    def empty_image(self, zero=True):
        import torch
        f = torch.zeros if zero else torch.empty
        return f(self.device_image_shape, dtype=torch.float32, device=f"cuda:{self.device}")

    def empty_projdata(self, zero=True):
        import torch
        f = torch.zeros if zero else torch.empty
        return f(self.projdata_size, dtype=torch.float32, device=f"cuda:{self.device}")

    def forward_dev(self, image_dev, out=None, subset_num=0, num_subsets=1, stream=None):
        if out is None:
            out = self.empty_projdata()
        _check_tensor(image_dev, self.geometry.nz * self.geometry.ny * self.geometry.nx)
        _check_tensor(out, self.projdata_size)
        _abi.check(self.lib.b200rt_forward_project_dev(self.h, ctypes.c_void_p(image_dev.data_ptr()),
                                                       ctypes.c_void_p(out.data_ptr()), subset_num, num_subsets,
                                                       _stream_ptr(stream)), self.h, "b200rt_forward_project_dev")
        return out

    def back_dev(self, projdata_dev, out=None, subset_num=0, num_subsets=1, mode=_abi.BACKPROJECT_ATOMIC, stream=None):
        if out is None:
            out = self.empty_image(zero=False)
        _check_tensor(projdata_dev, self.projdata_size)
        _check_tensor(out, self.geometry.nz * self.geometry.ny * self.geometry.nx)
        _abi.check(self.lib.b200rt_back_project_dev(self.h, ctypes.c_void_p(projdata_dev.data_ptr()),
                                                    ctypes.c_void_p(out.data_ptr()), subset_num, num_subsets, mode,
                                                    _stream_ptr(stream)), self.h, "b200rt_back_project_dev")
        return out

    # layout conversion (device to device)
    def image_to_device_layout(self, stir_dev, out=None, stream=None):
        out = self.empty_image(zero=False) if out is None else out
        _abi.check(self.lib.b200rt_image_to_device_layout(self.h, ctypes.c_void_p(stir_dev.data_ptr()),
                                                          ctypes.c_void_p(out.data_ptr()), _stream_ptr(stream)), self.h,
                   "b200rt_image_to_device_layout")
        return out

    def image_from_device_layout(self, dev, out=None, stream=None):
        import torch
        out = torch.empty(self.image_shape, dtype=torch.float32, device=dev.device) if out is None else out
        _abi.check(self.lib.b200rt_image_from_device_layout(self.h, ctypes.c_void_p(dev.data_ptr()),
                                                            ctypes.c_void_p(out.data_ptr()), _stream_ptr(stream)), self.h,
                   "b200rt_image_from_device_layout")
        return out

    def projdata_to_device_layout(self, stir_dev, out=None, stream=None):
        out = self.empty_projdata(zero=False) if out is None else out
        _abi.check(self.lib.b200rt_projdata_to_device_layout(self.h, ctypes.c_void_p(stir_dev.data_ptr()),
                                                             ctypes.c_void_p(out.data_ptr()), _stream_ptr(stream)), self.h,
                   "b200rt_projdata_to_device_layout")
        return out

    def projdata_from_device_layout(self, dev, out=None, stream=None):
        out = self.empty_projdata(zero=False) if out is None else out
        _abi.check(self.lib.b200rt_projdata_from_device_layout(self.h, ctypes.c_void_p(dev.data_ptr()),
                                                               ctypes.c_void_p(out.data_ptr()), _stream_ptr(stream)), self.h,
                   "b200rt_projdata_from_device_layout")
        return out

    # viewgrams of device-layout projection data ([axial][tangential], STIR's Viewgram order)
    def viewgram_shape(self, segment: int):
        return (self.proj_data_info.get_num_axial_poss(segment), self.proj_data_info.num_tangential_poss)

    def get_viewgram(self, projdata_dev, segment: int, view: int, timing_pos: int = 0, out=None, stream=None):
        """The viewgram (segment, view, timing position) of projdata_dev; `out` a numpy array (default) or a CUDA
        tensor of viewgram_shape(segment)."""
        _check_tensor(projdata_dev, self.projdata_size)
        if out is None:
            out = np.empty(self.viewgram_shape(segment), np.float32)
        ptr = _np_ptr(out) if isinstance(out, np.ndarray) else ctypes.c_void_p(out.data_ptr())
        if isinstance(out, np.ndarray) and (out.dtype != np.float32 or not out.flags.c_contiguous or
                                            out.shape != self.viewgram_shape(segment)):
            raise ValueError("expected a contiguous float32 array of the viewgram's shape")
        _abi.check(self.lib.b200rt_get_viewgram(self.h, ctypes.c_void_p(projdata_dev.data_ptr()), segment, view,
                                                timing_pos, ptr, _stream_ptr(stream)), self.h, "b200rt_get_viewgram")
        return out

    def set_viewgram(self, projdata_dev, viewgram, segment: int, view: int, timing_pos: int = 0,
                     accumulate: bool = False, stream=None):
        """Overwrite (or add to) the viewgram (segment, view, timing position) of projdata_dev."""
        _check_tensor(projdata_dev, self.projdata_size)
        if isinstance(viewgram, np.ndarray):
            viewgram = np.ascontiguousarray(viewgram, np.float32)
            if viewgram.shape != self.viewgram_shape(segment):
                raise ValueError("viewgram shape differs from (axial positions, tangential positions)")
            ptr = _np_ptr(viewgram)
        else:
            ptr = ctypes.c_void_p(viewgram.data_ptr())
        _abi.check(self.lib.b200rt_set_viewgram(self.h, ctypes.c_void_p(projdata_dev.data_ptr()), segment, view,
                                                timing_pos, ptr, int(accumulate), _stream_ptr(stream)), self.h,
                   "b200rt_set_viewgram")
        return projdata_dev


def _check_tensor(t, numel):
    if not t.is_cuda or not t.is_contiguous() or t.numel() != numel or str(t.dtype) != "torch.float32":
        raise ValueError(f"expected a contiguous float32 CUDA tensor with {numel} elements")


class ForwardProjectorByBinB200RayTracing:
    """Mirror of STIR's ForwardProjectorByBin for the B200 pair (ForwardProjectorByBin.h:53-175)."""

    def __init__(self, projector: Optional[RayTracingProjector] = None, **matrix_params):
        self._projector = projector
        self._matrix_params = matrix_params
        self._input = None
        self._cached = None  # device projection of the input, serving forward_project_viewgram

    def set_up(self, proj_data_info: ProjDataInfo, image: ImageGeometry):
        if self._projector is None or self._projector.proj_data_info != proj_data_info or self._projector.image != image:
            self._projector = RayTracingProjector(proj_data_info, image, **self._matrix_params)

    def _check_set_up(self):
        if self._projector is None:
            raise RuntimeError("ForwardProjectorByBin method called without calling set_up first.")

    def set_input(self, image: np.ndarray):
        self._check_set_up()
        self._input = np.ascontiguousarray(image, np.float32)
        self._cached = None

    def forward_project_viewgram(self, segment: int, view: int, timing_pos: int = 0):
        """actual_forward_project for one viewgram (the related set of a projector with trivial symmetries):
        the first call after set_input projects the whole data on the device, later calls copy their viewgram
        out of that projection (ForwardProjectorByBinParallelproj.cxx:128-145, 160-282)."""
        self._check_set_up()
        if self._input is None:
            raise RuntimeError("ForwardProjectorByBin: no input image")
        p = self._projector
        if self._cached is None:
            import torch
            img = p.image_to_device_layout(torch.from_numpy(self._input).to(f"cuda:{p.device}"))
            self._cached = p.forward_dev(img)
        return p.get_viewgram(self._cached, segment, view, timing_pos)

    def forward_project(self, proj_data: np.ndarray, image: Optional[np.ndarray] = None, subset_num: int = 0,
                        num_subsets: int = 1, zero: bool = True):
        """Fill `proj_data` (ProjDataInMemory order) with the projection of `image` (or of set_input's image).
        With zero=False only the subset's bins are overwritten."""
        self._check_set_up()
        img = self._input if image is None else image
        if img is None:
            raise RuntimeError("ForwardProjectorByBin: no input image")
        out = self._projector.forward_host(img, subset_num, num_subsets)
        if zero or num_subsets == 1:
            proj_data[...] = out.reshape(proj_data.shape)
        else:
            proj_data.reshape(-1)[:] = np.where(_subset_mask(self._projector, subset_num, num_subsets), out,
                                                proj_data.reshape(-1))
        return proj_data

    def get_projector(self) -> RayTracingProjector:
        self._check_set_up()
        return self._projector


class BackProjectorByBinB200RayTracing:
    """Mirror of STIR's BackProjectorByBin for the B200 pair (BackProjectorByBin.h:50-205)."""

    def __init__(self, projector: Optional[RayTracingProjector] = None, mode: int = _abi.BACKPROJECT_ATOMIC,
                 **matrix_params):
        self._projector = projector
        self._matrix_params = matrix_params
        self.mode = mode
        self._acc = None
        self._staged = None  # device projection data of back_project_viewgram, back projected by get_output

    def set_up(self, proj_data_info: ProjDataInfo, image: ImageGeometry):
        if self._projector is None or self._projector.proj_data_info != proj_data_info or self._projector.image != image:
            self._projector = RayTracingProjector(proj_data_info, image, **self._matrix_params)

    def _check_set_up(self):
        if self._projector is None:
            raise RuntimeError("BackProjectorByBin method called without calling set_up first.")

    def start_accumulating_in_new_target(self):
        self._check_set_up()
        self._acc = np.zeros(self._projector.image_shape, np.float32)
        self._staged = None

    def back_project_viewgram(self, viewgram: np.ndarray, segment: int, view: int, timing_pos: int = 0):
        """actual_back_project for one viewgram: added to projection data staged on the device, back projected
        by get_output (BackProjectorByBinParallelproj.cxx:161-328)."""
        self._check_set_up()
        if self._acc is None:
            raise RuntimeError("You need to call start_accumulating_in_new_target() before back_project()")
        if self._staged is None:
            self._staged = self._projector.empty_projdata()
        self._projector.set_viewgram(self._staged, viewgram, segment, view, timing_pos, accumulate=True)

    def back_project(self, image_or_proj_data, proj_data=None, subset_num: int = 0, num_subsets: int = 1):
        """back_project(image, proj_data, subset, nsub): overwrite `image` with A^T of the subset;
        back_project(proj_data, subset, nsub) after start_accumulating_in_new_target(): accumulate."""
        self._check_set_up()
        if proj_data is None:
            if self._acc is None:
                raise RuntimeError("You need to call start_accumulating_in_new_target() before back_project()")
            self._acc += self._projector.back_host(image_or_proj_data, subset_num, num_subsets, self.mode)
            return self._acc
        image = image_or_proj_data
        image[...] = self._projector.back_host(proj_data, subset_num, num_subsets, self.mode).reshape(image.shape)
        return image

    def get_output(self, image: np.ndarray):
        if self._acc is None:
            raise RuntimeError("BackProjectorByBin: nothing accumulated")
        if self._staged is not None:
            p = self._projector
            self._acc += p.image_from_device_layout(p.back_dev(self._staged, mode=self.mode)).cpu().numpy()
            self._staged = None
        image[...] = self._acc.reshape(image.shape)
        return image

    def get_projector(self) -> RayTracingProjector:
        self._check_set_up()
        return self._projector


class ProjectorByBinPairUsingB200RayTracing:
    """Mirror of STIR's ProjectorByBinPair (ProjectorByBinPair.h:44-90) for the B200 ray-tracing pair.
    Parsing keyword a STIR plug-in registers for it: "B200 Ray Tracing"."""

    registered_name = "B200 Ray Tracing"

    def __init__(self, num_tangential_LORs: int = 1, restrict_to_cylindrical_FOV: bool = True,
                 symmetries=(True,) * 5, device: int = 0, back_projection_mode: int = _abi.BACKPROJECT_ATOMIC):
        self._params = dict(num_tangential_LORs=num_tangential_LORs,
                            restrict_to_cylindrical_FOV=restrict_to_cylindrical_FOV, symmetries=symmetries,
                            device=device)
        self._mode = back_projection_mode
        self._fwd = None
        self._back = None
        self.projector = None

    def set_up(self, proj_data_info: ProjDataInfo, image: ImageGeometry):
        self.projector = RayTracingProjector(proj_data_info, image, **self._params)
        self._fwd = ForwardProjectorByBinB200RayTracing(self.projector)
        self._back = BackProjectorByBinB200RayTracing(self.projector, self._mode)
        return self

    def get_forward_projector_sptr(self):
        if self._fwd is None:
            raise RuntimeError("ProjectorByBinPair: set_up not called")
        return self._fwd

    def get_back_projector_sptr(self):
        if self._back is None:
            raise RuntimeError("ProjectorByBinPair: set_up not called")
        return self._back


def _subset_mask(projector: RayTracingProjector, subset_num: int, num_subsets: int) -> np.ndarray:
    """Boolean mask (ProjDataInMemory order) of the bins in the subset: views related to basic views
    v with v % num_subsets == subset_num.  Computed by forward projecting a ones image through the
    library would hide zero bins, so the mask is derived from the symmetry structure on the host."""
    from .subsets import views_in_subset
    pdi = projector.proj_data_info
    views = views_in_subset(projector.geometry, subset_num, num_subsets, projector.info.symmetries_used)
    mask = np.zeros(projector.projdata_size, bool)
    per_view = np.zeros(pdi.num_views, bool)
    per_view[views] = True
    off = 0
    for s in pdi.segment_sequence:
        n = pdi.get_num_axial_poss(s) * pdi.num_views * pdi.num_tangential_poss
        blk = np.broadcast_to(per_view[None, :, None], (pdi.get_num_axial_poss(s), pdi.num_views, pdi.num_tangential_poss))
        mask[off:off + n] = blk.reshape(-1)
        off += n
    return mask
