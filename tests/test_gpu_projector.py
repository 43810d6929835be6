"""Parity of the CUDA projector pair with the oracle (restated STIR), through the C ABI."""
import os

import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))

REL_L2 = 1e-5  # forward/back vs the reference ray tracer (relative L2)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def small(cuda_device, oracle_lib):
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    return pdi, img, proj, orc


@pytest.fixture(scope="module")
def rpt(cuda_device, oracle_lib):
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.rpt_sensitivity_test()
    proj = RayTracingProjector(pdi, img, num_tangential_LORs=2, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    return pdi, img, proj, orc


def _same_row(c1, v1, c2, v2):
    o1 = np.lexsort((c1[:, 2], c1[:, 1], c1[:, 0]))
    o2 = np.lexsort((c2[:, 2], c2[:, 1], c2[:, 0]))
    return np.array_equal(c1[o1], c2[o2]) and np.array_equal(v1[o1].astype(np.float32), v2[o2].astype(np.float32))


@pytest.mark.parametrize("which", ["small", "rpt"])
def test_rows_bit_exact(which, small, rpt):
    """Rows traced on the GPU equal the oracle's rows element for element (same float arithmetic)."""
    pdi, img, proj, orc = small if which == "small" else rpt
    S = pdi.max_segment_num
    rng = np.random.default_rng(21)
    nt = pdi.num_tangential_poss
    for _ in range(400):
        seg = int(rng.integers(-S, S + 1))
        view = int(rng.integers(0, pdi.num_views))
        ax = int(rng.integers(0, pdi.get_num_axial_poss(seg)))
        tang = int(rng.integers(-(nt // 2), nt - nt // 2))
        c1, v1 = proj.get_row(seg, view, ax, tang)
        c2, v2 = orc.row(seg, view, ax, tang)
        assert _same_row(c1, v1, c2, v2), (seg, view, ax, tang)


@pytest.mark.parametrize("which", ["small", "rpt"])
@pytest.mark.parametrize("subset", [(0, 1), (2, 6), (5, 6)])
def test_forward_matches_oracle(which, subset, small, rpt):
    pdi, img, proj, orc = small if which == "small" else rpt
    x = np.random.default_rng(1).uniform(0, 1, img.shape).astype(np.float32)
    got = proj.forward_host(x, *subset)
    ref = orc.forward(x, *subset)
    assert rel_l2(got, ref) <= REL_L2
    assert np.array_equal(got == 0, ref == 0)


@pytest.mark.parametrize("which", ["small", "rpt"])
@pytest.mark.parametrize("subset", [(0, 1), (3, 6)])
def test_back_matches_oracle(which, subset, small, rpt):
    pdi, img, proj, orc = small if which == "small" else rpt
    y = np.random.default_rng(2).uniform(0, 1, proj.projdata_size).astype(np.float32)
    got = proj.back_host(y, *subset)
    ref = orc.back(y, *subset)
    assert rel_l2(got, ref) <= REL_L2


def test_sensitivity_matches_stir_golden(rpt):
    """Back-projection of ones (segment 0 end planes zeroed) vs STIR's RPTsens_seg3_PM.v."""
    pdi, img, proj, orc = rpt
    gold = np.load(os.path.join(HERE, "golden", "rptsens_seg3_pm.npz"))["image"]
    ones = np.ones(proj.projdata_size, np.float32)
    off = 0
    for s in pdi.segment_sequence:
        n_ax = pdi.get_num_axial_poss(s)
        blk = ones[off:off + n_ax * pdi.num_views * pdi.num_tangential_poss].reshape(n_ax, -1)
        if s == 0:
            blk[0] = 0
            blk[-1] = 0
        off += blk.size
    sens = proj.back_host(ones)
    assert np.abs(sens - gold).max() / np.abs(gold).max() <= 0.0005
    assert rel_l2(sens, gold) < 1e-5


def test_adjoint(small):
    pdi, img, proj, orc = small
    rng = np.random.default_rng(9)
    x = rng.uniform(0, 1, img.shape).astype(np.float32)
    y = rng.uniform(0, 1, proj.projdata_size).astype(np.float32)
    lhs = float(proj.forward_host(x).astype(np.float64) @ y)
    rhs = float(proj.back_host(y).astype(np.float64).ravel() @ x.ravel())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_device_api_and_layouts(small):
    import torch
    pdi, img, proj, orc = small
    x = np.random.default_rng(4).uniform(0, 1, img.shape).astype(np.float32)
    xs = torch.from_numpy(x).cuda()
    xd = proj.image_to_device_layout(xs)
    assert torch.equal(proj.image_from_device_layout(xd), xs)
    assert torch.equal(xd, xs.permute(1, 2, 0).contiguous())
    pd = proj.forward_dev(xd)
    stir = proj.projdata_from_device_layout(pd)
    assert torch.equal(proj.projdata_to_device_layout(stir), pd)
    host = proj.forward_host(x)
    assert rel_l2(stir.cpu().numpy(), host) < 1e-6
    back = proj.back_dev(pd)
    ref = proj.back_host(host)
    assert rel_l2(proj.image_from_device_layout(back).cpu().numpy(), ref) < 1e-6


def test_invalid_subset_is_an_error(small):
    pdi, img, proj, orc = small
    with pytest.raises(_abi.B200Error):
        proj.forward_host(np.zeros(img.shape, np.float32), 6, 6)


@pytest.mark.parametrize("which", ["small", "rpt"])
def test_deterministic_back_projection(which, small, rpt):
    """Deterministic mode: same result as the oracle within 1e-5 and bit-identical from run to run."""
    pdi, img, proj, orc = small if which == "small" else rpt
    y = np.random.default_rng(12).uniform(0, 1, proj.projdata_size).astype(np.float32)
    ref = orc.back(y, 1, 6)
    a = proj.back_host(y, 1, 6, _abi.BACKPROJECT_DETERMINISTIC)
    b = proj.back_host(y, 1, 6, _abi.BACKPROJECT_DETERMINISTIC)
    assert rel_l2(a, ref) <= REL_L2
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    full = proj.back_host(y, 0, 1, _abi.BACKPROJECT_DETERMINISTIC)
    assert rel_l2(full, orc.back(y)) <= REL_L2


def test_deterministic_device_api(small):
    import torch
    pdi, img, proj, orc = small
    y = torch.rand(proj.projdata_size, device="cuda")
    a = proj.back_dev(y, mode=_abi.BACKPROJECT_DETERMINISTIC)
    b = proj.back_dev(y, mode=_abi.BACKPROJECT_DETERMINISTIC)
    c = proj.back_dev(y, mode=_abi.BACKPROJECT_ATOMIC)
    assert torch.equal(a, b)
    assert float((a - c).norm() / c.norm()) < 1e-6


SYMMETRY_CASES = {
    "no_90": (False, True, True, True, True),
    "no_180": (True, False, True, True, True),
    "no_swap_segment": (True, True, False, True, True),
    "no_swap_s": (True, True, True, False, True),
    "shift_z_only": (False, False, False, False, True),
}


@pytest.mark.parametrize("case", list(SYMMETRY_CASES))
def test_symmetry_subsets_match_oracle(cuda_device, oracle_lib, case):
    """ProjMatrixByBinUsingRayTracing's do_symmetry_* keys: fewer symmetries mean more basic bins and
    fewer related lines per bin (and other path items); the projections are the same."""
    import torch
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, symmetries=SYMMETRY_CASES[case], device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    rng = np.random.default_rng(31)
    x = rng.uniform(0, 1, img.shape).astype(np.float32)
    y = rng.uniform(0, 1, proj.projdata_size).astype(np.float32)
    for subset, nsub in [(0, 1), (1, 4)]:
        f = proj.forward_host(x, subset, nsub)
        assert rel_l2(f, orc.forward(x, subset, nsub)) < REL_L2
        b = proj.back_host(y, subset, nsub)
        assert rel_l2(b, orc.back(y, subset, nsub)) < REL_L2


def test_unrestricted_fov_matches_oracle(cuda_device, oracle_lib):
    """restrict_to_cylindrical_FOV := 0 traces rays through the square field of view
    (ProjMatrixByBinUsingRayTracing.cxx:488-513)."""
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, restrict_to_cylindrical_FOV=False, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    rng = np.random.default_rng(32)
    x = rng.uniform(0, 1, img.shape).astype(np.float32)
    y = rng.uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.forward_host(x), orc.forward(x)) < REL_L2
    assert rel_l2(proj.back_host(y), orc.back(y)) < REL_L2


@pytest.mark.parametrize("which", ["small", "rpt"])
@pytest.mark.parametrize("subset", [(0, 1), (1, 4)])
def test_host_api_matches_device_api(which, subset, small, rpt):
    """The host-buffer entry points project group by group of views with the copies overlapped: the
    forward projection equals the device entry point's bit for bit, the back projection to float
    rounding; with pageable (numpy) and with pinned host buffers."""
    import ctypes
    import torch
    pdi, img, proj, orc = small if which == "small" else rpt
    rng = np.random.default_rng(41)
    x = rng.uniform(0, 1, img.shape).astype(np.float32)
    y = rng.uniform(0, 1, proj.projdata_size).astype(np.float32)
    xd = proj.image_to_device_layout(torch.from_numpy(x).cuda())
    out = torch.zeros(proj.projdata_size, device="cuda")
    fd = proj.projdata_from_device_layout(proj.forward_dev(xd, out, *subset)).cpu().numpy()
    assert np.array_equal(proj.forward_host(x, *subset), fd)
    yd = proj.projdata_to_device_layout(torch.from_numpy(y).cuda())
    bd = proj.image_from_device_layout(proj.back_dev(yd, None, *subset)).cpu().numpy()
    assert rel_l2(proj.back_host(y, *subset), bd) < 1e-6
    # pinned buffers (asynchronous copies)
    x_pin = torch.from_numpy(x).pin_memory()
    f_pin = torch.full((proj.projdata_size,), -1.0).pin_memory()
    _abi.check(proj.lib.b200rt_forward_project(proj.h, ctypes.c_void_p(x_pin.data_ptr()),
                                               ctypes.c_void_p(f_pin.data_ptr()), *subset), proj.h, "forward")
    assert np.array_equal(f_pin.numpy(), fd)
    y_pin = torch.from_numpy(y).pin_memory()
    b_pin = torch.full(img.shape, -1.0).pin_memory()
    _abi.check(proj.lib.b200rt_back_project(proj.h, ctypes.c_void_p(y_pin.data_ptr()), ctypes.c_void_p(b_pin.data_ptr()),
                                            *subset, _abi.BACKPROJECT_ATOMIC), proj.h, "back")
    assert rel_l2(b_pin.numpy(), bd) < 1e-6


def test_intrinsic_tilt_and_depth_of_interaction(cuda_device, oracle_lib):
    """A scanner with an intrinsic azimuthal tilt (views start at phi = tilt: STIR then disables the 90- and
    180-degree symmetries, DataSymmetriesForBins_PET_CartesianGrid.cxx:302-360) and a non-zero average depth of
    interaction: forward and back projection of a subset against the oracle, and the symmetries used."""
    import dataclasses
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    sc = dataclasses.replace(pdi.scanner, intrinsic_tilt=0.05, average_depth_of_interaction=7.0)
    pdi = dataclasses.replace(pdi, scanner=sc)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    assert proj.info.symmetries_used == orc.symmetries_used
    assert not (proj.info.symmetries_used & 3)  # no 90 / 180 degree symmetry
    x = np.random.default_rng(21).uniform(0, 1, img.shape).astype(np.float32)
    assert rel_l2(proj.forward_host(x, 1, 3), orc.forward(x, 1, 3)) <= 1e-5
    y = np.random.default_rng(22).uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.back_host(y, 1, 3), orc.back(y, 1, 3)) <= 1e-5
    proj.close()
