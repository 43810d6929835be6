"""List-mode objective on the GPU (listmode.cu through the C ABI) against the oracle's restatement of
LM_gradient_and_value / LM_Hessian over the same events."""
import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G

pytestmark = pytest.mark.gpu
METHODS = [_abi.LISTMODE_PER_EVENT, _abi.LISTMODE_BINNED]


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def random_events(pdi, n, rng, ntof=1, min_tof=0):
    S = pdi.max_segment_num
    seg = rng.integers(-S, S + 1, n)
    ax = np.array([rng.integers(0, pdi.get_num_axial_poss(int(s))) for s in seg])
    view = rng.integers(0, pdi.num_views, n)
    tang = rng.integers(pdi.min_tangential_pos_num, pdi.min_tangential_pos_num + pdi.num_tangential_poss, n)
    tof = rng.integers(min_tof, min_tof + ntof, n)
    return np.stack([seg, view, ax, tang, tof], 1).astype(np.int32)


@pytest.fixture(scope="module")
def small(cuda_device, oracle_lib):
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    return pdi, img, proj, oracle_lib.Oracle(proj.geometry)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("subset", [(0, 1), (1, 3)])
@pytest.mark.parametrize("has_add", [False, True])
def test_listmode_matches_oracle(small, subset, has_add, method):
    import torch
    from stir_b200.listmode import (PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin as LM,
                                    pack_events)
    pdi, img, proj, orc = small
    rng = np.random.default_rng(31)
    bins = random_events(pdi, 20000, rng)
    vals = rng.integers(1, 3, len(bins)).astype(np.float32)
    corr = rng.uniform(0.01, 0.2, len(bins)).astype(np.float32)
    x = rng.uniform(0.3, 1.5, img.shape).astype(np.float32)
    rhs = rng.uniform(-1, 1, img.shape).astype(np.float32)
    to_dev = lambda a: proj.image_to_device_layout(torch.from_numpy(a).cuda())
    to_host = lambda t: proj.image_from_device_layout(t).cpu().numpy()
    obj = LM(proj, pack_events(bins, vals, corr), num_subsets=subset[1], has_add=has_add)
    obj.set_method(method)
    c = corr if has_add else None
    g = to_host(obj.compute_sub_gradient_without_penalty(to_dev(x), subset[0]))
    ref = orc.listmode("gradient", bins, vals, x, corr=c, subset=subset[0], nsub=subset[1], has_add=has_add)
    assert rel_l2(g, ref) <= 1e-5
    v = obj.compute_objective_function_without_penalty(to_dev(x), subset[0])
    ref_v, bad = orc.listmode("value", bins, vals, x, corr=c, subset=subset[0], nsub=subset[1], has_add=has_add)
    assert bad == 0 and abs(v - ref_v) <= 1e-6 * abs(ref_v)
    out = to_dev(np.ones(img.shape, np.float32))
    obj.accumulate_sub_Hessian_times_input_without_penalty(out, to_dev(x), to_dev(rhs), subset[0])
    ref_h = orc.listmode("hessian", bins, vals, x, corr=c, rhs=rhs, subset=subset[0], nsub=subset[1], has_add=has_add,
                         out=np.ones(img.shape, np.float32))
    assert rel_l2(to_host(out), ref_h) <= 1e-5
    # gradient minus the subset sensitivity, accumulated onto an existing image
    sens = to_dev(rng.uniform(0, 1, img.shape).astype(np.float32))
    base = to_dev(np.full(img.shape, 2.0, np.float32))
    obj.compute_sub_gradient_without_penalty(to_dev(x), subset[0], subset_sensitivity=sens, out=base, accumulate=True)
    assert rel_l2(to_host(base), 2.0 + ref - to_host(sens)) <= 1e-5
    assert obj.num_invalid_events() == 0


@pytest.mark.parametrize("method", METHODS)
def test_listmode_invalid_events_are_counted(small, method):
    import torch
    from stir_b200.listmode import (PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin as LM,
                                    pack_events)
    pdi, img, proj, orc = small
    S = pdi.max_segment_num
    bins = np.array([[0, 3, 2, 0, 0], [S + 1, 0, 0, 0, 0], [0, 0, 99, 0, 0], [0, 1, 1, 1, 0]], np.int32)
    obj = LM(proj, pack_events(bins, [1, 1, 1, 0]))
    obj.set_method(method)
    x = proj.image_to_device_layout(torch.ones(img.shape, device="cuda"))
    obj.compute_sub_gradient_without_penalty(x, 0)
    assert obj.num_invalid_events() == 2
    assert obj.num_invalid_events() == 0  # reset by the read


@pytest.mark.parametrize("method", METHODS)
def test_listmode_tof_matches_oracle(cuda_device, oracle_lib, method):
    import torch
    from stir_b200.listmode import (PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin as LM,
                                    pack_events)
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=5, timing_bin_ps=250.0, num_views=48)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    ntof = proj.info.num_tof_bins
    rng = np.random.default_rng(33)
    bins = random_events(pdi, 5000, rng, ntof, -(ntof // 2))
    vals = np.ones(len(bins), np.float32)
    x = rng.uniform(0.3, 1.5, img.shape).astype(np.float32)
    xd = proj.image_to_device_layout(torch.from_numpy(x).cuda())
    obj = LM(proj, pack_events(bins, vals))
    obj.set_method(method)
    g = proj.image_from_device_layout(obj.compute_sub_gradient_without_penalty(xd, 0)).cpu().numpy()
    assert rel_l2(g, orc.listmode("gradient", bins, vals, x)) <= 1e-5
    v = obj.compute_objective_function_without_penalty(xd, 0)
    ref_v, bad = orc.listmode("value", bins, vals, x)
    assert bad == 0 and abs(v - ref_v) <= 1e-6 * abs(ref_v)
    assert obj.num_invalid_events() == 0


def test_listmode_osem_matches_oracle(small):
    import torch
    from stir_b200.listmode import (PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin as LM,
                                    ListModeOSEM, pack_events)
    pdi, img, proj, orc = small
    rng = np.random.default_rng(34)
    bins = random_events(pdi, 50000, rng)
    nsub = 3
    obj = LM(proj, pack_events(bins), num_subsets=nsub)
    obj.set_method(_abi.LISTMODE_AUTO)
    osem = ListModeOSEM(obj)
    x0 = np.ones(img.shape, np.float32)
    xd = proj.image_to_device_layout(torch.from_numpy(x0).cuda())
    xr = x0.copy()
    for k in range(1, 4):
        osem.update_estimate(xd)
        subset = (k - 1) % nsub
        u = orc.listmode("gradient", bins, np.ones(len(bins), np.float32), xr, subset=subset, nsub=nsub)
        sens = orc.sensitivity(None, subset, nsub)
        xr = orc.osmaposl_apply(xr, u, sens, nsub, k)
    assert rel_l2(proj.image_from_device_layout(xd).cpu().numpy(), xr) <= 1e-4


def test_listmode_methods_agree_on_a_clustered_list(small):
    """Many events in few bins (the binned method sums each bin's terms before the weights): both methods against
    the oracle, and an unknown method is refused."""
    import torch
    from stir_b200.listmode import (PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin as LM,
                                    pack_events)
    pdi, img, proj, orc = small
    rng = np.random.default_rng(35)
    few = random_events(pdi, 40, rng)
    bins = few[rng.integers(0, len(few), 30000)]
    x = rng.uniform(0.3, 1.5, img.shape).astype(np.float32)
    xd = proj.image_to_device_layout(torch.from_numpy(x).cuda())
    obj = LM(proj, pack_events(bins), num_subsets=2)
    ref = orc.listmode("gradient", bins, np.ones(len(bins), np.float32), x, subset=1, nsub=2)
    for method in METHODS:
        obj.set_method(method)
        g = proj.image_from_device_layout(obj.compute_sub_gradient_without_penalty(xd, 1)).cpu().numpy()
        assert rel_l2(g, ref) <= 1e-5
    with pytest.raises(_abi.B200Error):
        obj.set_method(7)
    obj.set_method(_abi.LISTMODE_AUTO)
