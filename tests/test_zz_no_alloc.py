"""The allocation-free log-likelihood entry point (b200rt_log_likelihood_dev_noalloc).

It exists for callers that must not allocate device memory once set up (for example a service that
gives all device memory to a caching allocator at start-up, or cannot take the device-wide
synchronisation of cudaMalloc/cudaFree mid-frame).  Its scratch is a fixed array inside the library,
shared by all calls.  This file is collected last so that a run stopping at the first failure has run
every other test already; it builds its own data and passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu

TOL = 1e-6  # relative, as the log-likelihood parity test


def _data(proj, img, seed):
    import torch
    rng = np.random.default_rng(seed)
    xt = phantoms.cylinder_with_spheres(img, seed=3)
    xd = proj.image_to_device_layout(torch.from_numpy(xt).cuda())
    ybar = proj.forward_dev(xd)
    y = torch.poisson(ybar * 4.0 + 0.5).div_(4.0).contiguous()
    add = torch.full_like(y, 0.125)
    mult = torch.from_numpy(rng.uniform(0.8, 1.2, proj.projdata_size).astype(np.float32)).cuda()
    x = proj.image_to_device_layout(torch.from_numpy(phantoms.smooth_random_field(img, 2.0, seed=7)).cuda())
    return x, y, add, mult


def _noalloc(proj, x, y, add, mult, subset, nsub, zero_ends, out):
    from stir_b200.projectors import _stream_ptr
    return proj.lib.b200rt_log_likelihood_dev_noalloc(
        proj.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(add.data_ptr()),
        ctypes.c_void_p(mult.data_ptr()), subset, nsub, int(zero_ends), ctypes.c_void_p(out.data_ptr()), _stream_ptr(None))


def _check_against_allocating(proj, x, y, add, mult, cases, cuda_device):
    """Each case is called twice in a row: the shared scratch keeps the previous call's contents, and a
    correct call must not depend on them.  The entry point runs the allocating entry point's kernel on the
    same work items, so beyond the tolerance the two sums are expected to be equal."""
    import torch
    from stir_b200.osmaposl import log_likelihood
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=f"cuda:{cuda_device}")
    for subset, nsub, zero_ends in cases:
        ref = log_likelihood(proj, x, y, add, mult, subset, nsub, zero_ends)
        for _ in range(2):
            out.fill_(float("nan"))
            st = _noalloc(proj, x, y, add, mult, subset, nsub, zero_ends, out)
            assert st == _abi.OK, proj.lib.b200rt_last_error(proj.h)
            torch.cuda.synchronize()
            got = float(out.item())
            assert abs(got - ref) <= TOL * abs(ref), (subset, nsub, got, ref)
            assert got == ref, (subset, nsub, got, ref)


def test_no_alloc_log_likelihood_matches_allocating_entry_point(cuda_device):
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    x, y, add, mult = _data(proj, img, 31)
    _check_against_allocating(proj, x, y, add, mult, [(2, 6, True), (0, 1, False)], cuda_device)

    # arguments are checked before any work
    import torch
    out = torch.zeros(1, dtype=torch.float64, device=f"cuda:{cuda_device}")
    st = proj.lib.b200rt_log_likelihood_dev_noalloc(proj.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                                     None, None, 6, 6, 0, ctypes.c_void_p(out.data_ptr()), None)
    assert st == _abi.ERR_INVALID_ARGUMENT


def test_no_alloc_log_likelihood_tof(cuda_device):
    """The 33-bin TOF geometry (71,280 viewgrams, within the limit): TOF-grouped basic bins as work items.  TOF
    leaves only the z-shift symmetry, so the whole data has 138,240 basic bins, over the 131,072 the array holds:
    half the views (2 subsets) is the largest subset here."""
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=33)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    x, y, add, mult = _data(proj, img, 32)
    _check_against_allocating(proj, x, y, add, mult, [(5, 21, True), (0, 2, False)], cuda_device)


def test_no_alloc_log_likelihood_clinical(cuda_device):
    """The clinical geometry (72.6 M bins): path items as work items, all of them for the whole data."""
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.clinical_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    x, y, add, mult = _data(proj, img, 33)
    _check_against_allocating(proj, x, y, add, mult, [(0, 21, False), (0, 1, True)], cuda_device)


def test_no_alloc_log_likelihood_over_limit(cuda_device):
    """61 timing bins x 15 segments x 144 views = 131,760 viewgrams, over the 131,072 the array holds."""
    import torch
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=61, timing_bin_ps=25.0)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    x = proj.empty_image()
    y = proj.empty_projdata()
    out = torch.full((1,), -1.0, dtype=torch.float64, device=f"cuda:{cuda_device}")
    st = _noalloc(proj, x, y, y, y, 0, 21, False, out)
    assert st == _abi.ERR_TOO_LARGE
    msg = proj.lib.b200rt_last_error(proj.h).decode()
    assert "131760 viewgrams" in msg, msg
    torch.cuda.synchronize()
    assert float(out.item()) == -1.0  # nothing was launched
