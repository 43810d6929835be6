"""Prior Hessian times an image on the GPU against the oracle's restatement (QuadraticPrior /
RelativeDifferencePrior accumulate_Hessian_times_input)."""
import numpy as np
import pytest

from stir_b200 import geometry as G

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("kind", ["qp", "rdp", "rdp_eps_kappa_2d"])
def test_prior_hessian_times_input_matches_oracle(cuda_device, oracle_lib, kind):
    import torch
    from oracle.oracle import prior_hessian_times_input as ref_hvp
    from stir_b200.osmaposl import QuadraticPrior, RelativeDifferencePrior, prior_hessian_times_input
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    rng = np.random.default_rng(11)
    x = rng.uniform(0.2, 2.0, img.shape).astype(np.float32)
    x[3, 10:20, 10:20] = 0.0  # zero neighbourhoods exercise the RDP limits
    v = rng.standard_normal(img.shape).astype(np.float32)
    out0 = rng.standard_normal(img.shape).astype(np.float32)  # the result is accumulated
    kappa = None
    if kind == "qp":
        prior = QuadraticPrior(0.7)
    elif kind == "rdp":
        prior = RelativeDifferencePrior(0.4, gamma=2.0, epsilon=0.0)
        x[3, 10:20, 10:20] = 0.5
    else:
        kappa = rng.uniform(0.5, 1.5, img.shape).astype(np.float32)
        prior = RelativeDifferencePrior(0.4, gamma=1.5, epsilon=1e-3, only_2D=True)

    def dev(a):
        return proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(a)).cuda())

    if kappa is not None:
        prior.kappa = dev(kappa)
    out = dev(out0)
    prior_hessian_times_input(proj, prior, dev(x), dev(v), out=out)
    got = proj.image_from_device_layout(out).cpu().numpy()
    p_abi = prior.as_abi()
    p_abi.kappa_dev = None
    ref = ref_hvp(p_abi, x, v, img.voxel_size, kappa=kappa, out=out0)
    assert np.isfinite(got).all()
    assert rel_l2(got - out0, ref - out0) < 1e-5
