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


def test_no_alloc_log_likelihood_matches_allocating_entry_point(cuda_device):
    import torch

    from stir_b200.osmaposl import log_likelihood
    from stir_b200.projectors import RayTracingProjector, _stream_ptr

    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    rng = np.random.default_rng(31)
    xt = phantoms.cylinder_with_spheres(img, seed=3)
    xd = proj.image_to_device_layout(torch.from_numpy(xt).cuda())
    ybar = proj.forward_dev(xd)
    y = torch.poisson(ybar * 4.0 + 0.5).div_(4.0).contiguous()
    add = torch.full_like(y, 0.125)
    mult = torch.from_numpy(rng.uniform(0.8, 1.2, proj.projdata_size).astype(np.float32)).cuda()
    x = proj.image_to_device_layout(torch.from_numpy(phantoms.smooth_random_field(img, 2.0, seed=7)).cuda())
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=f"cuda:{cuda_device}")

    # two subset choices, each called twice in a row: the shared scratch keeps the previous call's
    # contents, and a correct call must not depend on them
    for subset, nsub, zero_ends in [(2, 6, True), (2, 6, True), (0, 1, False), (0, 1, False)]:
        ref = log_likelihood(proj, x, y, add, mult, subset, nsub, zero_ends)
        st = proj.lib.b200rt_log_likelihood_dev_noalloc(
            proj.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(add.data_ptr()),
            ctypes.c_void_p(mult.data_ptr()), subset, nsub, int(zero_ends), ctypes.c_void_p(out.data_ptr()), _stream_ptr(None))
        assert st == _abi.OK, proj.lib.b200rt_last_error(proj.h)
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - ref) <= TOL * abs(ref), (subset, nsub, got, ref)

    # arguments are checked before any work
    st = proj.lib.b200rt_log_likelihood_dev_noalloc(proj.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                                     None, None, 6, 6, 0, ctypes.c_void_p(out.data_ptr()), None)
    assert st == _abi.ERR_INVALID_ARGUMENT
