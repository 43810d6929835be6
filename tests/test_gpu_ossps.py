"""OSSPS on the GPU against the oracle's restatement of STIR's OSSPSReconstruction, through the C ABI."""
import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu

OSSPS_TOL = 1e-4  # images after identical sub-iterations (relative L2)


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
    rng = np.random.default_rng(7)
    scale = 5e6 / float((ybar + bg).sum())
    y = rng.poisson((ybar + bg) * scale).astype(np.float32) / np.float32(scale)
    add = np.full_like(y, bg)
    norm = rng.uniform(0.8, 1.25, y.shape).astype(np.float32)

    def dev_pd(a):
        return proj.projdata_to_device_layout(torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda())

    def dev_img(a):
        return proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda())

    def host_img(t):
        return proj.image_from_device_layout(t).cpu().numpy()

    return dict(proj=proj, orc=orc, y=y, add=add, norm=norm, dev_pd=dev_pd, dev_img=dev_img, host_img=host_img)


@pytest.mark.parametrize("with_norm", [False, True])
def test_ossps_denominator_matches_oracle(setup, with_norm):
    from stir_b200.ossps import OSSPSReconstruction
    s = setup
    n = s["norm"] if with_norm else None
    rec = OSSPSReconstruction(s["proj"], s["dev_pd"](s["y"]), norm=None if n is None else s["dev_pd"](n)).set_up()
    ref = s["orc"].ossps_denominator(s["y"], n)
    assert rel_l2(s["host_img"](rec.denominator), ref) < 1e-5


@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_ossps_subiterations_match_oracle(setup, beta):
    from stir_b200.osmaposl import QuadraticPrior
    from stir_b200.ossps import OSSPSReconstruction
    s = setup
    nsub, nit = 4, 5
    prior = QuadraticPrior(beta) if beta else None
    rec = OSSPSReconstruction(s["proj"], s["dev_pd"](s["y"]), additive=s["dev_pd"](s["add"]), num_subsets=nsub,
                              num_subiterations=nit, relaxation_parameter=1.0, relaxation_gamma=0.1, prior=prior)
    x = s["dev_img"](np.ones((15, 64, 64), np.float32))
    rec.set_up()
    d_ref = s["host_img"](rec.denominator)
    sens = s["orc"].sensitivity(None, 0, 1)
    xr = np.ones((15, 64, 64), np.float32)
    p_abi = None if prior is None else prior.as_abi()
    for k in range(1, nit + 1):
        rec.subiteration_num = k
        rec.update_estimate(x)
        xr, d_ref = s["orc"].ossps_update(xr, d_ref, s["y"], s["add"], None, sens, (k - 1) % nsub, nsub, k, 1,
                                          prior=p_abi, relaxation_parameter=1.0, relaxation_gamma=0.1)
        err = rel_l2(s["host_img"](x), xr)
        assert err < OSSPS_TOL, (k, err)
    assert rel_l2(s["host_img"](rec.denominator), d_ref) < 1e-5


def test_ossps_rejects_rdp(setup):
    from stir_b200.osmaposl import RelativeDifferencePrior
    from stir_b200.ossps import OSSPSReconstruction
    with pytest.raises(ValueError):
        OSSPSReconstruction(setup["proj"], setup["dev_pd"](setup["y"]), prior=RelativeDifferencePrior(0.1))
