"""The CPU oracle against STIR's own golden data and compiled code (CPU only)."""
import os

import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G

HERE = os.path.dirname(os.path.abspath(__file__))


def test_ray_tracer_bit_exact_vs_stir_compiled(oracle_lib):
    """The restated Siddon tracer equals STIR's RayTraceVoxelsOnCartesianGrid.cxx compiled from its
    source (oracle/_ref) on random rays, including rays on voxel boundaries and parallel to planes."""
    if not oracle_lib.ref_available():
        pytest.skip("oracle/_ref not built (STIR sources not present)")
    rng = np.random.default_rng(1234)
    for i in range(3000):
        vox = rng.uniform(0.5, 5, 3).astype(np.float32)
        s = rng.uniform(-40, 40, 3).astype(np.float32)
        e = rng.uniform(-40, 40, 3).astype(np.float32)
        k = i % 6
        if k == 1:
            e[0] = s[0]
        elif k == 2:
            e[1] = s[1] = np.float32(np.round(s[1]) + 0.5)
        elif k == 3:
            e[0] = s[0] = np.float32(np.round(s[0]) + 0.5)
        elif k == 4:
            e[2] = s[2] = np.float32(np.round(s[2]) + 0.5)
            e[1] = s[1]
        c1, v1 = oracle_lib.ray_trace(s, e, vox, 0.7)
        c2, v2 = oracle_lib.ref_ray_trace(s, e, vox, 0.7)
        assert np.array_equal(c1, c2) and np.array_equal(v1, v2), (s, e, vox)


def test_oracle_sensitivity_matches_stir_golden(oracle_lib):
    """recon_test_pack: OSMAPOSL_test_PM_for_sensitivity.par -> RPTsens_seg3_PM.v, compared with
    compare_image's criterion (max |diff| / sup-norm <= 0.0005, src/utilities/compare_image.cxx:72,144)."""
    gold = np.load(os.path.join(HERE, "golden", "rptsens_seg3_pm.npz"))["image"]
    pdi, img = G.rpt_sensitivity_test()
    orc = oracle_lib.Oracle(G.make_geometry(pdi, img, num_tangential_LORs=2))
    sens = orc.sensitivity(zero_seg0_end_planes=True)
    err = np.abs(sens - gold).max() / np.abs(gold).max()
    assert err <= 0.0005
    assert err < 1e-5  # in fact the restatement reproduces STIR to float rounding
    assert np.linalg.norm(sens - gold) / np.linalg.norm(gold) < 2e-6


def _rows_equal_stir(c1, v1, c2, v2):
    """ProjMatrixElemsForOneBin::operator== (ProjMatrixElemsForOneBin.cxx:414-475): tolerance 0.2% of the
    row maximum, elements below it may be missing on either side."""
    if len(v1) == 0 and len(v2) == 0:
        return True
    o1 = np.lexsort((c1[:, 2], c1[:, 1], c1[:, 0]))
    o2 = np.lexsort((c2[:, 2], c2[:, 1], c2[:, 0]))
    c1, v1, c2, v2 = c1[o1], v1[o1], c2[o2], v2[o2]
    tol = v1.max() * 0.002 if len(v1) else 0.0
    d1 = {tuple(c): v for c, v in zip(c1, v1)}
    d2 = {tuple(c): v for c, v in zip(c2, v2)}
    for k in set(d1) | set(d2):
        a, b = d1.get(k, 0.0), d2.get(k, 0.0)
        if abs(a - b) > tol and not (k not in d1 and b < tol) and not (k not in d2 and a < tol):
            return False
    return True


def test_symmetry_fold_vs_direct_rows(oracle_lib):
    """test_DataSymmetriesForBins_PET_CartesianGrid.cxx:352-627: rows folded through the symmetries agree
    with rows traced directly (here: only the z-shift symmetry kept) within STIR's 0.2% row tolerance."""
    pdi, img = G.small_3d_pet()
    full = oracle_lib.Oracle(G.make_geometry(pdi, img))
    direct = oracle_lib.Oracle(G.make_geometry(pdi, img, symmetries=(False, False, False, False, True)))
    assert full.symmetries_used == 31 and direct.symmetries_used == 16
    rng = np.random.default_rng(5)
    for _ in range(300):
        seg = int(rng.integers(-7, 8))
        view = int(rng.integers(0, 144))
        ax = int(rng.integers(0, pdi.get_num_axial_poss(seg)))
        tang = int(rng.integers(-32, 32))
        c1, v1 = full.row(seg, view, ax, tang)
        c2, v2 = direct.row(seg, view, ax, tang)
        assert _rows_equal_stir(c1, v1, c2, v2), (seg, view, ax, tang)


@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_adjoint(oracle_lib, precision):
    pdi, img = G.small_3d_pet()
    orc = oracle_lib.Oracle(G.make_geometry(pdi, img), precision)
    rng = np.random.default_rng(7)
    x = rng.uniform(0, 1, img.shape)
    y = rng.uniform(0, 1, orc.projdata_size)
    ax = orc.forward(x).astype(np.float64)
    aty = orc.back(y).astype(np.float64)
    lhs, rhs = float(ax @ y), float(aty.ravel() @ x.ravel())
    assert abs(lhs - rhs) / abs(lhs) < (1e-12 if precision == 64 else 1e-5)


def test_oracle_fp32_close_to_fp64(oracle_lib):
    """STIR's float arithmetic against the same algorithm in double.  The two differ on the few LORs
    whose FOV entry point falls exactly on a voxel boundary (e.g. 30 degrees through the centre of the
    64x64 grid, x = 31*sin(30deg) = 15.5): in float the first voxel rounds to the far side and the tracer
    adds a segment there (RayTraceVoxelsOnCartesianGrid.cxx:178-213), in double it does not."""
    pdi, img = G.small_3d_pet()
    o32 = oracle_lib.Oracle(G.make_geometry(pdi, img), 32)
    o64 = oracle_lib.Oracle(G.make_geometry(pdi, img), 64)
    x = np.random.default_rng(3).uniform(0, 1, img.shape)
    f32, f64 = o32.forward(x), o64.forward(x)
    assert np.linalg.norm(f32 - f64) / np.linalg.norm(f64) < 1e-3
    rel = np.abs(f32 - f64) / np.maximum(np.abs(f64), 1e-9)
    assert (rel > 1e-4).mean() < 1e-3


@pytest.mark.parametrize("ptype", [_abi.PRIOR_QUADRATIC, _abi.PRIOR_RELATIVE_DIFFERENCE])
def test_prior_gradient_vs_numerical(oracle_lib, ptype):
    """test_priors.cxx:151-170 style check: analytic gradient vs central differences of the value."""
    rng = np.random.default_rng(11)
    x = rng.uniform(0.5, 2.0, (5, 6, 7)).astype(np.float32)
    vox = (2.0, 3.0, 3.0)
    p = _abi.Prior(type=ptype, penalisation_factor=0.7, gamma=2.0, epsilon=0.01)
    g = oracle_lib.prior_gradient(p, x, vox)
    for idx in [(0, 0, 0), (2, 3, 4), (4, 5, 6), (1, 2, 3)]:
        h = 1e-2
        xp = x.astype(np.float64).copy()
        xm = xp.copy()
        xp[idx] += h
        xm[idx] -= h
        num = (oracle_lib.prior_value(p, xp.astype(np.float32), vox) - oracle_lib.prior_value(p, xm.astype(np.float32), vox)) / (2 * h)
        assert abs(num - g[idx]) <= 2e-3 * max(1.0, abs(g).max())


@pytest.mark.parametrize("k", [0.0, 3.0])
def test_oracle_tof_kernel_cut_off(oracle_lib, k):
    """The TOF rows of a LOR through the centre summed over the 33 timing bins (50 ps each: they cover +-3.53 sigma
    of the 550 ps kernel): with STIR's cut-off (5.66 sigma, beyond the bins) the voxel at the LOR's middle keeps
    erf(3.53 / sqrt 2) of its non-TOF value; with the kernel truncated at +-3 sigma it keeps erf(3 / sqrt 2) = 0.9973,
    no voxel keeps more, and the rows are shorter."""
    import math
    pdi, img = G.tof_small_3d_pet()
    orc = oracle_lib.Oracle(G.make_geometry(pdi, img, tof_kernel_truncation_sigmas=k))
    nt = oracle_lib.Oracle(G.make_geometry(G.non_tof(pdi), img))
    c0, v0 = nt.row(0, 0, 4, 0)
    key = lambda c: [tuple(r) for r in c]
    total = dict.fromkeys(key(c0), 0.0)
    nnz = 0
    for t in range(-16, 17):
        c, v = orc.row(0, 0, 4, 0, t)
        nnz += len(v)
        for kk, vv in zip(key(c), v):
            total[kk] += vv
    ratio = np.array([total[kk] / vv for kk, vv in zip(key(c0), v0)])
    c_half = 0.299792458 * 0.5  # mm per ps of timing difference
    sigma = 550.0 * c_half / 2.355
    reach = 16.5 * 50.0 * c_half / sigma  # the bins' half range, in sigmas
    expect = math.erf((reach if k == 0 else min(k, reach)) / math.sqrt(2.0))
    assert abs(ratio.max() - expect) < 2e-4
    assert ratio.max() <= expect + 2e-4
    if k:
        full = oracle_lib.Oracle(G.make_geometry(pdi, img))
        assert nnz < sum(len(full.row(0, 0, 4, 0, t)[1]) for t in range(-16, 17))
