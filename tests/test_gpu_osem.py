"""OSMAPOSL on the GPU against the oracle's restatement of STIR's update, through the C ABI."""
import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu

OSEM_TOL = 1e-4  # images after identical sub-iterations (relative L2)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def setup(cuda_device, oracle_lib):
    import torch
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    xt = phantoms.cylinder_with_spheres(img, radius_mm=100.0, n_spheres=2, sphere_radius=(10.0, 10.0), seed=1)
    ybar = orc.forward(xt)
    bg = np.float32(0.1 * ybar.mean())
    rng = np.random.default_rng(2)
    scale = 5e6 / float((ybar + bg).sum())
    y = rng.poisson((ybar + bg) * scale).astype(np.float32) / np.float32(scale)
    add = np.full_like(y, bg)
    mult = rng.uniform(0.8, 1.2, y.shape).astype(np.float32)

    def dev_pd(a):
        return proj.projdata_to_device_layout(torch.from_numpy(a).cuda())

    def dev_img(a):
        return proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda())

    def host_img(t):
        return proj.image_from_device_layout(t).cpu().numpy()

    return dict(pdi=pdi, img=img, proj=proj, orc=orc, y=y, add=add, mult=mult, dev_pd=dev_pd, dev_img=dev_img,
                host_img=host_img)


@pytest.mark.parametrize("zero_ends", [False, True])
def test_sensitivity_with_mult(setup, zero_ends):
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    s = setup
    rec = OSMAPOSLReconstruction(s["proj"], s["dev_pd"](s["y"]), mult=s["dev_pd"](s["mult"]), num_subsets=6,
                                 zero_seg0_end_planes=zero_ends).set_up()
    for sub in (0, 3):
        ref = s["orc"].sensitivity(s["mult"], sub, 6, zero_ends)
        assert rel_l2(s["host_img"](rec.sensitivities[sub]), ref) < 1e-5


CASES = {
    "osem": dict(prior=None, MAP="multiplicative", additive=True, zero_ends=False),
    "osem_zero_ends": dict(prior=None, MAP="multiplicative", additive=True, zero_ends=True),
    "qp_multiplicative": dict(prior=("qp", 0.05), MAP="multiplicative", additive=True, zero_ends=False),
    "qp_additive": dict(prior=("qp", 0.05), MAP="additive", additive=True, zero_ends=False),
    "rdp_additive": dict(prior=("rdp", 0.1), MAP="additive", additive=False, zero_ends=False),
    "rdp_multiplicative": dict(prior=("rdp", 0.1), MAP="multiplicative", additive=True, zero_ends=True),
}


def _make_prior(c):
    from stir_b200.osmaposl import QuadraticPrior, RelativeDifferencePrior
    if not c["prior"]:
        return None
    kind, beta = c["prior"]
    return QuadraticPrior(beta) if kind == "qp" else RelativeDifferencePrior(beta, gamma=2.0, epsilon=0.0)


@pytest.mark.parametrize("case", list(CASES))
def test_osmaposl_subiterations_match_oracle(setup, case):
    import torch
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    c = CASES[case]
    s = setup
    prior = _make_prior(c)
    add = s["add"] if c["additive"] else None
    rec = OSMAPOSLReconstruction(s["proj"], s["dev_pd"](s["y"]), additive=None if add is None else s["dev_pd"](add),
                                 num_subsets=6, num_subiterations=4, zero_seg0_end_planes=c["zero_ends"], prior=prior,
                                 MAP_model=c["MAP"], maximum_relative_change=5.0, minimum_relative_change=0.2)
    rec.set_up()
    x = s["dev_img"](np.ones(s["img"].shape, np.float32))
    xo = np.ones(s["img"].shape, np.float32)
    abi_prior = None if prior is None else prior.as_abi(rec.map_model)
    for it in range(1, 5):
        rec.subiteration_num = it
        sub = rec.get_subset_num()
        rec.update_estimate(x)
        sens = s["host_img"](rec.sensitivities[sub])
        xo, _ = s["orc"].osmaposl_update(xo, s["y"], add, sens, sub, 6, it, prior=abi_prior, min_rel=0.2, max_rel=5.0,
                                         zero_seg0_end_planes=c["zero_ends"])
        err = rel_l2(s["host_img"](x), xo)
        assert err <= OSEM_TOL, (case, it, err)


@pytest.mark.parametrize("case,beta", [("qp_multiplicative", 0.5), ("rdp_additive", 0.1), ("osem", 0.0)])
def test_single_update_from_identical_input(setup, case, beta):
    """One sub-iteration from the same estimate on both sides (no accumulated history): the
    per-step difference, free of the amplification a stiff prior applies over sub-iterations."""
    from stir_b200.osmaposl import OSMAPOSLReconstruction, QuadraticPrior, RelativeDifferencePrior
    c = CASES[case]
    s = setup
    prior = None
    if c["prior"]:
        prior = QuadraticPrior(beta) if c["prior"][0] == "qp" else RelativeDifferencePrior(beta, 2.0, 0.0)
    add = s["add"] if c["additive"] else None
    rec = OSMAPOSLReconstruction(s["proj"], s["dev_pd"](s["y"]), additive=None if add is None else s["dev_pd"](add),
                                 num_subsets=6, zero_seg0_end_planes=c["zero_ends"], prior=prior, MAP_model=c["MAP"],
                                 maximum_relative_change=5.0, minimum_relative_change=0.2).set_up()
    xo = np.ones(s["img"].shape, np.float32)
    abi_prior = None if prior is None else prior.as_abi(rec.map_model)
    for it in range(1, 7):
        rec.subiteration_num = it
        sub = rec.get_subset_num()
        x = s["dev_img"](xo)
        rec.update_estimate(x)
        sens = s["host_img"](rec.sensitivities[sub])
        xo, _ = s["orc"].osmaposl_update(xo, s["y"], add, sens, sub, 6, it, prior=abi_prior, min_rel=0.2, max_rel=5.0,
                                         zero_seg0_end_planes=c["zero_ends"])
        assert rel_l2(s["host_img"](x), xo) <= 1e-5, (case, it)


def test_log_likelihood_matches_oracle(setup):
    from stir_b200.osmaposl import log_likelihood
    s = setup
    x = phantoms.smooth_random_field(s["img"], sigma_vox=2.0, seed=4)
    for sub, nsub, zero in [(0, 1, False), (2, 6, True)]:
        got = log_likelihood(s["proj"], s["dev_img"](x), s["dev_pd"](s["y"]), s["dev_pd"](s["add"]), s["dev_pd"](s["mult"]),
                             sub, nsub, zero)
        ref = s["orc"].log_likelihood(x, s["y"], s["add"], s["mult"], sub, nsub, zero)
        assert abs(got - ref) <= 1e-6 * abs(ref), (got, ref)


@pytest.mark.parametrize("kind", ["qp", "rdp"])
def test_prior_gradient_matches_oracle(setup, oracle_lib, kind):
    from stir_b200.osmaposl import QuadraticPrior, RelativeDifferencePrior, prior_gradient
    s = setup
    x = phantoms.smooth_random_field(s["img"], sigma_vox=2.0, seed=5)
    pr = QuadraticPrior(0.5) if kind == "qp" else RelativeDifferencePrior(0.1, 2.0, 0.01)
    got = s["host_img"](prior_gradient(s["proj"], pr, s["dev_img"](x)))
    ref = oracle_lib.prior_gradient(pr.as_abi(), x, s["img"].voxel_size)
    assert rel_l2(got, ref) < 1e-6


def test_deterministic_osem_is_reproducible(setup):
    """Sub-iterations with the deterministic back projection agree with the oracle and repeat bit for bit."""
    import torch
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    s = setup
    results = []
    for _ in range(2):
        rec = OSMAPOSLReconstruction(s["proj"], s["dev_pd"](s["y"]), additive=s["dev_pd"](s["add"]), num_subsets=6,
                                     num_subiterations=4, back_projection_mode=_abi.BACKPROJECT_DETERMINISTIC).set_up()
        x = s["dev_img"](np.ones(s["img"].shape, np.float32))
        rec.reconstruct(x)
        results.append(x.clone())
    assert torch.equal(results[0], results[1])
    xo = np.ones(s["img"].shape, np.float32)
    rec_sens = OSMAPOSLReconstruction(s["proj"], s["dev_pd"](s["y"]), num_subsets=6).set_up()
    for it in range(1, 5):
        sub = (it - 1) % 6
        sens = s["host_img"](rec_sens.sensitivities[sub])
        xo, _ = s["orc"].osmaposl_update(xo, s["y"], s["add"], sens, sub, 6, it)
    assert rel_l2(s["host_img"](results[0]), xo) <= OSEM_TOL


def test_numerator_and_apply_equal_subiteration(setup):
    """b200rt_osmaposl_numerator_dev + b200rt_osmaposl_apply_update_dev == b200rt_osmaposl_subiteration_dev
    (the split the multi-GPU driver uses), bit for bit with the deterministic back projection."""
    import torch
    from stir_b200.distributed import B200Backend
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    s = setup
    y, add = s["dev_pd"](s["y"]), s["dev_pd"](s["add"])
    mode = _abi.BACKPROJECT_DETERMINISTIC
    rec = OSMAPOSLReconstruction(s["proj"], y, additive=add, num_subsets=6, back_projection_mode=mode,
                                 minimum_relative_change=0.2, maximum_relative_change=5.0).set_up()
    b = B200Backend(s["proj"], y, add, mode=mode)
    x1 = s["dev_img"](np.ones(s["img"].shape, np.float32))
    x2 = x1.clone()
    for it in (1, 2):
        rec.subiteration_num = it
        rec.update_estimate(x1)
        sub = (it - 1) % 6
        u = b.numerator(x2, sub, 6)
        b.apply(x2, u, rec.sensitivities[sub], 6, it, min_rel=0.2, max_rel=5.0)
        assert torch.equal(x1, x2)


def test_randomised_subset_order_matches_oracle(setup):
    """"uniformly randomise subset order": the GPU reconstruction visits a new permutation of the 6 subsets each
    full iteration; the oracle, given the same sequence, reaches the same image (12 sub-iterations)."""
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    s = setup
    rec = OSMAPOSLReconstruction(s["proj"], s["dev_pd"](s["y"]), additive=s["dev_pd"](s["add"]), num_subsets=6,
                                 num_subiterations=12, uniformly_randomise_subset_order=True, subset_order_seed=11,
                                 minimum_relative_change=0.2, maximum_relative_change=5.0).set_up()
    x = s["dev_img"](np.ones(s["img"].shape, np.float32))
    xo = np.ones(s["img"].shape, np.float32)
    seq = []
    for it in range(1, 13):
        rec.subiteration_num = it
        sub = rec.get_subset_num()
        seq.append(sub)
        rec.update_estimate(x)
        sens = s["host_img"](rec.sensitivities[sub])
        xo, _ = s["orc"].osmaposl_update(xo, s["y"], s["add"], sens, sub, 6, it, min_rel=0.2, max_rel=5.0)
    assert sorted(seq[:6]) == sorted(seq[6:]) == list(range(6)) and seq[:6] != list(range(6))
    assert rel_l2(s["host_img"](x), xo) <= OSEM_TOL
