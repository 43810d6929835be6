"""The oracle's list-mode objective (LM_gradient_and_value / LM_Hessian over events) against the binned
oracle: events are a sparse sinogram, so sum_e A_e^T y_e / (A_e x + c_e) = A^T (y / (A x + c)) on the bins
that hold events."""
import numpy as np
import pytest

from stir_b200 import geometry as G
from stir_b200.projectors import make_geometry


def stir_index(pdi, seg, view, ax, tang):
    off = 0
    for s in pdi.segment_sequence:
        n = pdi.get_num_axial_poss(s) * pdi.num_views * pdi.num_tangential_poss
        if s == seg:
            return off + (ax * pdi.num_views + view) * pdi.num_tangential_poss + (tang - pdi.min_tangential_pos_num)
        off += n
    raise ValueError(seg)


def random_events(pdi, n, rng):
    S = pdi.max_segment_num
    seg = rng.integers(-S, S + 1, n)
    ax = np.array([rng.integers(0, pdi.get_num_axial_poss(int(s))) for s in seg])
    view = rng.integers(0, pdi.num_views, n)
    tang = rng.integers(pdi.min_tangential_pos_num, pdi.min_tangential_pos_num + pdi.num_tangential_poss, n)
    return np.stack([seg, view, ax, tang, np.zeros(n, int)], 1).astype(np.int32)


@pytest.fixture(scope="module")
def setup(oracle_lib):
    pdi, img = G.small_3d_pet()
    geo = make_geometry(pdi, img)
    orc = oracle_lib.Oracle(geo)
    return pdi, img, orc


@pytest.mark.parametrize("subset", [(0, 1), (1, 3)])
def test_listmode_gradient_value_match_binned(setup, subset):
    pdi, img, orc = setup
    rng = np.random.default_rng(21)
    bins = random_events(pdi, 3000, rng)
    x = rng.uniform(0.5, 1.5, orc.image_shape).astype(np.float32)
    corr = rng.uniform(0.01, 0.1, len(bins)).astype(np.float32)
    # one event per count: bins may repeat
    y = np.zeros(orc.projdata_size, np.float32)
    c = np.zeros(orc.projdata_size, np.float32)
    for b, cc in zip(bins, corr):
        i = stir_index(pdi, *b[:4])
        y[i] += 1
        c[i] = cc
    corr = np.array([c[stir_index(pdi, *b[:4])] for b in bins], np.float32)  # one additive term per bin
    g = orc.listmode("gradient", bins, np.ones(len(bins), np.float32), x, corr=corr, subset=subset[0],
                     nsub=subset[1], has_add=True)
    fwd = orc.forward(x, *subset) + c
    ratio = np.where(y > 0, y / np.where(fwd > 0, fwd, 1), 0).astype(np.float32)
    ref = orc.back(ratio, *subset)
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) < 1e-5
    v, bad = orc.listmode("value", bins, np.ones(len(bins), np.float32), x, corr=corr, subset=subset[0], nsub=subset[1],
                          has_add=True)
    mask = (y > 0) & (orc.forward(np.ones_like(x), *subset) > 0)
    ref_v = -float(np.sum(y[mask].astype(np.float64) * np.log(fwd[mask].astype(np.float64))))
    assert bad == 0 and abs(v - ref_v) <= 1e-5 * abs(ref_v)


def test_listmode_hessian_vs_gradient_differences(setup):
    pdi, img, orc = setup
    rng = np.random.default_rng(22)
    bins = random_events(pdi, 2000, rng)
    vals = np.ones(len(bins), np.float32)
    x = rng.uniform(0.5, 1.5, orc.image_shape).astype(np.float32)
    rhs = rng.uniform(-1, 1, orc.image_shape).astype(np.float32)
    hv = orc.listmode("hessian", bins, vals, x, rhs=rhs)
    h = 1e-3
    gp = orc.listmode("gradient", bins, vals, (x + h * rhs).astype(np.float32)).astype(np.float64)
    gm = orc.listmode("gradient", bins, vals, (x - h * rhs).astype(np.float32)).astype(np.float64)
    assert np.linalg.norm((gp - gm) / (2 * h) - hv) / np.linalg.norm(hv) < 2e-2


def test_listmode_invalid_and_zero_events(setup):
    pdi, img, orc = setup
    x = np.ones(orc.image_shape, np.float32)
    bins = np.array([[0, 0, 0, 0, 0], [pdi.max_segment_num + 1, 0, 0, 0, 0], [0, 0, 0, 0, 0]], np.int32)
    v, bad = orc.listmode("value", bins, np.array([1, 1, 0], np.float32), x)
    assert bad == 1
    g = orc.listmode("gradient", bins[:1], np.array([0], np.float32), x)
    assert not g.any()
