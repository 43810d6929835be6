"""TOF projection (ProjMatrixByBin::apply_tof_kernel) on the GPU against the oracle."""
import numpy as np
import pytest

from stir_b200 import geometry as G

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def tof(cuda_device, oracle_lib):
    from stir_b200.projectors import RayTracingProjector
    # 48 views (view mashing 3), 7 timing bins of 250 ps, 550 ps FWHM
    pdi, img = G.tof_small_3d_pet(num_tof_bins=7, timing_bin_ps=250.0, num_views=48)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    return pdi, img, proj, orc


def test_tof_symmetries_and_sizes(tof):
    pdi, img, proj, orc = tof
    assert proj.info.num_tof_bins == 7 == orc.num_tof_bins
    assert proj.info.symmetries_used == orc.symmetries_used == 16  # only the z shift, as STIR with TOF
    assert proj.projdata_size == pdi.size == orc.projdata_size


def test_tof_rows_bit_exact(tof):
    pdi, img, proj, orc = tof
    rng = np.random.default_rng(8)
    for _ in range(200):
        seg = int(rng.integers(-7, 8))
        view = int(rng.integers(0, pdi.num_views))
        ax = int(rng.integers(0, pdi.get_num_axial_poss(seg)))
        tang = int(rng.integers(-32, 32))
        k = int(rng.integers(-3, 4))
        c1, v1 = proj.get_row(seg, view, ax, tang, k)
        c2, v2 = orc.row(seg, view, ax, tang, k)
        o1 = np.lexsort((c1[:, 2], c1[:, 1], c1[:, 0]))
        o2 = np.lexsort((c2[:, 2], c2[:, 1], c2[:, 0]))
        assert np.array_equal(c1[o1], c2[o2]), (seg, view, ax, tang, k)
        assert np.array_equal(v1[o1], v2[o2].astype(np.float32)), (seg, view, ax, tang, k)


@pytest.mark.parametrize("subset", [(0, 1), (1, 4)])
def test_tof_forward_back_match_oracle(tof, subset):
    pdi, img, proj, orc = tof
    x = np.random.default_rng(3).uniform(0, 1, img.shape).astype(np.float32)
    assert rel_l2(proj.forward_host(x, *subset), orc.forward(x, *subset)) <= 1e-5
    y = np.random.default_rng(4).uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.back_host(y, *subset), orc.back(y, *subset)) <= 1e-5


def test_tof_sum_over_timing_bins_matches_non_tof(tof, cuda_device):
    """The timing bins partition the LOR: their sum is the non-TOF projection wherever the kernel is
    not truncated by the outermost bins."""
    from stir_b200.projectors import RayTracingProjector
    pdi, img, proj, orc = tof
    nt = RayTracingProjector(G.non_tof(pdi), img, device=cuda_device)
    x = np.zeros(img.shape, np.float32)
    x[:, 28:36, 28:36] = 1.0  # compact object at the centre: far from the outer timing bins
    f = proj.forward_host(x).reshape(7, -1).sum(axis=0)
    g = nt.forward_host(x)
    assert rel_l2(f, g) < 1e-3


def test_tof_33_bins_grouped_kernels(cuda_device, oracle_lib):
    """33 timing bins (the TOF configuration: more than one group of timing bins per pass of the grouped kernels):
    forward and back projection of a subset against the oracle; the deterministic back projection repeats bit for
    bit and agrees with the atomic one."""
    import torch
    from stir_b200 import _abi
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    assert proj.info.num_tof_bins == 33
    sub = (1, 12)
    x = np.random.default_rng(5).uniform(0, 1, img.shape).astype(np.float32)
    assert rel_l2(proj.forward_host(x, *sub), orc.forward(x, *sub)) <= 1e-5
    y = np.random.default_rng(6).uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.back_host(y, *sub), orc.back(y, *sub)) <= 1e-5
    yd = proj.projdata_to_device_layout(torch.from_numpy(y).cuda())
    a = proj.back_dev(yd, None, *sub, mode=_abi.BACKPROJECT_DETERMINISTIC)
    b = proj.back_dev(yd, None, *sub, mode=_abi.BACKPROJECT_DETERMINISTIC)
    c = proj.back_dev(yd, None, *sub, mode=_abi.BACKPROJECT_ATOMIC)
    assert torch.equal(a, b)
    assert float((a - c).norm() / c.norm()) < 1e-6
    proj.close()


@pytest.mark.parametrize("ntof", [13, 23, 29])
def test_tof_group_sizes(cuda_device, oracle_lib, ntof):
    """Timing-bin counts that select the other group sizes of the grouped kernels (16, 24 and 32 bins per pass)."""
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=ntof, timing_bin_ps=1650.0 / ntof, num_views=48)  # 1650 ps in all
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    assert proj.info.num_tof_bins == ntof
    sub = (2, 6)
    x = np.random.default_rng(7).uniform(0, 1, img.shape).astype(np.float32)
    assert rel_l2(proj.forward_host(x, *sub), orc.forward(x, *sub)) <= 1e-5
    y = np.random.default_rng(8).uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.back_host(y, *sub), orc.back(y, *sub)) <= 1e-5
    proj.close()


def test_tof_log_likelihood_matches_oracle(tof):
    """The TOF log-likelihood (TOF-grouped forward with the FP64 epilogue, one partial per basic bin)."""
    import torch
    from stir_b200.osmaposl import log_likelihood
    pdi, img, proj, orc = tof
    rng = np.random.default_rng(11)
    x = rng.uniform(0.5, 1.5, img.shape).astype(np.float32)
    ybar = orc.forward(x)
    y = rng.poisson(ybar * 4.0).astype(np.float32) / np.float32(4.0)
    add = np.full_like(y, np.float32(0.05 * ybar.mean()))
    mult = rng.uniform(0.8, 1.2, y.shape).astype(np.float32)
    dev_pd = lambda a: proj.projdata_to_device_layout(torch.from_numpy(a).cuda())
    xd = proj.image_to_device_layout(torch.from_numpy(x).cuda())
    for sub, nsub, zero in [(0, 1, False), (1, 4, True)]:
        got = log_likelihood(proj, xd, dev_pd(y), dev_pd(add), dev_pd(mult), sub, nsub, zero)
        ref = orc.log_likelihood(x, y, add, mult, sub, nsub, zero)
        assert abs(got - ref) <= 1e-6 * abs(ref), (got, ref)


def test_tof_many_axial_positions(cuda_device, oracle_lib):
    """TOF with more than 16 axial positions per line (24 rings, span 3): the TOF-grouped kernels take one line at
    a time in blocks of 32 axial positions.  Forward, back (atomic and deterministic) and log-likelihood against the
    oracle on a subset."""
    import dataclasses
    import math
    import torch
    from stir_b200 import _abi
    from stir_b200.osmaposl import log_likelihood
    from stir_b200.projectors import RayTracingProjector
    sc = G.Scanner(24, 288, 300.0, 0.0, 4.0, float(np.float32(2 * math.pi * 300.0 / 288 / 2)))
    sc = dataclasses.replace(sc, timing_resolution=550.0, size_of_timing_pos=150.0, max_num_timing_poss=11)
    pdi = dataclasses.replace(G.ProjDataInfoCTI(sc, 3, 10, 48, 64), tof_mash_factor=1)
    img = G.ImageGeometry(47, 64, 64, (2.0, 4.0, 4.0))
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    assert proj.info.num_tof_bins == 11 and max(pdi.get_num_axial_poss(s) for s in pdi.segment_sequence) > 16
    sub = (1, 6)
    rng = np.random.default_rng(12)
    x = rng.uniform(0.5, 1.5, img.shape).astype(np.float32)
    f = proj.forward_host(x, *sub)
    ref = orc.forward(x, *sub)
    assert rel_l2(f, ref) <= 1e-5
    y = rng.uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.back_host(y, *sub), orc.back(y, *sub)) <= 1e-5
    assert rel_l2(proj.back_host(y, *sub, _abi.BACKPROJECT_DETERMINISTIC), orc.back(y, *sub)) <= 1e-5
    xd = proj.image_to_device_layout(torch.from_numpy(x).cuda())
    yd = proj.projdata_to_device_layout(torch.from_numpy((ref + 0.1).astype(np.float32)).cuda())
    got = log_likelihood(proj, xd, yd, None, None, *sub)
    want = orc.log_likelihood(x, (ref + 0.1).astype(np.float32), None, None, *sub)
    assert abs(got - want) <= 1e-6 * abs(want)
    proj.close()


def test_tof_kernel_truncated_at_3_sigma(cuda_device, oracle_lib):
    """The 33-bin TOF geometry with the Gaussian truncated at +-3 sigma instead of STIR's cut-off: rows bit-exact,
    forward and back projection of a subset (TOF-grouped kernels, whose per-element weights take the same cut-off)
    against the oracle, and fewer row elements than with STIR's cut-off."""
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device, tof_kernel_truncation_sigmas=3.0)
    orc = oracle_lib.Oracle(proj.geometry)
    rng = np.random.default_rng(12)
    for _ in range(100):
        seg = int(rng.integers(-7, 8))
        view = int(rng.integers(0, pdi.num_views))
        ax = int(rng.integers(0, pdi.get_num_axial_poss(seg)))
        tang = int(rng.integers(-32, 32))
        k = int(rng.integers(-16, 17))
        c1, v1 = proj.get_row(seg, view, ax, tang, k)
        c2, v2 = orc.row(seg, view, ax, tang, k)
        o1 = np.lexsort((c1[:, 2], c1[:, 1], c1[:, 0]))
        o2 = np.lexsort((c2[:, 2], c2[:, 1], c2[:, 0]))
        assert np.array_equal(c1[o1], c2[o2]), (seg, view, ax, tang, k)
        assert np.array_equal(v1[o1], v2[o2].astype(np.float32)), (seg, view, ax, tang, k)
    sub = (1, 12)
    x = np.random.default_rng(5).uniform(0, 1, img.shape).astype(np.float32)
    assert rel_l2(proj.forward_host(x, *sub), orc.forward(x, *sub)) <= 1e-5
    y = np.random.default_rng(6).uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.back_host(y, *sub), orc.back(y, *sub)) <= 1e-5
    full = RayTracingProjector(pdi, img, device=cuda_device)
    assert proj.info.total_nnz < full.info.total_nnz
    full.close()
    proj.close()


def test_tof_mashing(cuda_device, oracle_lib):
    """TOF mashing (ProjDataInfo.cxx:174-255): 21 unmashed timing positions of 80 ps mashed by 3 into 7 timing bins of
    240 ps; rows bit-exact, forward and back projection of a subset against the oracle."""
    import dataclasses
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=21, timing_bin_ps=80.0, num_views=48)
    pdi = dataclasses.replace(pdi, tof_mash_factor=3)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    assert proj.info.num_tof_bins == 7 == orc.num_tof_bins
    rng = np.random.default_rng(14)
    for _ in range(60):
        seg = int(rng.integers(-7, 8))
        view = int(rng.integers(0, pdi.num_views))
        ax = int(rng.integers(0, pdi.get_num_axial_poss(seg)))
        tang = int(rng.integers(-32, 32))
        k = int(rng.integers(-3, 4))
        c1, v1 = proj.get_row(seg, view, ax, tang, k)
        c2, v2 = orc.row(seg, view, ax, tang, k)
        o1 = np.lexsort((c1[:, 2], c1[:, 1], c1[:, 0]))
        o2 = np.lexsort((c2[:, 2], c2[:, 1], c2[:, 0]))
        assert np.array_equal(c1[o1], c2[o2]), (seg, view, ax, tang, k)
        assert np.array_equal(v1[o1], v2[o2].astype(np.float32)), (seg, view, ax, tang, k)
    sub = (1, 4)
    x = np.random.default_rng(15).uniform(0, 1, img.shape).astype(np.float32)
    assert rel_l2(proj.forward_host(x, *sub), orc.forward(x, *sub)) <= 1e-5
    y = np.random.default_rng(16).uniform(0, 1, proj.projdata_size).astype(np.float32)
    assert rel_l2(proj.back_host(y, *sub), orc.back(y, *sub)) <= 1e-5
    proj.close()
