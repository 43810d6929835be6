"""The torch.autograd wrappers: adjointness, finite differences, and the gradient against the oracle."""
import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(cuda_device, oracle_lib):
    import torch
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    xt = phantoms.cylinder_with_spheres(img, seed=1)
    ybar = orc.forward(xt)
    rng = np.random.default_rng(5)
    y = (rng.poisson(ybar * 20.0 + 2.0) / 20.0).astype(np.float32)
    add = np.full_like(y, 0.1)
    mult = rng.uniform(0.8, 1.2, y.shape).astype(np.float32)

    def dpd(a):
        return proj.projdata_to_device_layout(torch.from_numpy(a).cuda())

    def dimg(a):
        return proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda())

    return dict(proj=proj, orc=orc, img=img, y=y, add=add, mult=mult, dpd=dpd, dimg=dimg)


def test_autograd_adjoint(env):
    """<A x, y> = <x, A^T y>, with A^T obtained by torch.autograd.grad through forward_project."""
    import torch
    from stir_b200.autograd import back_project, forward_project
    proj = env["proj"]
    x = torch.rand(proj.device_image_shape, device="cuda", requires_grad=True)
    y = torch.rand(proj.projdata_size, device="cuda")
    lhs = (forward_project(x, proj).double() * y.double()).sum()
    (g,) = torch.autograd.grad(lhs, x)
    rhs = (x.detach().double() * g.double()).sum()
    assert abs(float(lhs - rhs)) / abs(float(lhs)) < 1e-5
    # and back_project's backward is the forward projector
    yy = y.clone().requires_grad_(True)
    s = (back_project(yy, proj) * x.detach()).sum()
    (gy,) = torch.autograd.grad(s, yy)
    assert float((gy - forward_project(x.detach(), proj)).norm() / gy.norm()) < 1e-6


def test_batched_forward_matches_single(env):
    import torch
    from stir_b200.autograd import forward_project
    proj = env["proj"]
    xb = torch.rand((3,) + proj.device_image_shape, device="cuda")
    out = forward_project(xb, proj)
    assert out.shape == (3, proj.projdata_size)
    for b in range(3):
        assert torch.allclose(out[b], forward_project(xb[b], proj))


def test_loglik_gradient_matches_oracle(env):
    import torch
    from stir_b200.autograd import PoissonLogLikelihood
    proj, orc = env["proj"], env["orc"]
    xh = phantoms.smooth_random_field(env["img"], 2.0, seed=9)
    x = env["dimg"](xh).requires_grad_(True)
    L = PoissonLogLikelihood(proj, env["dpd"](env["y"]), env["dpd"](env["add"]), env["dpd"](env["mult"]), 1, 4, True)
    val = L(x)
    (g,) = torch.autograd.grad(val, x)
    ref = orc.log_likelihood_gradient(xh, env["y"], env["add"], env["mult"], 1, 4, True)
    got = proj.image_from_device_layout(g).cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5
    ref_val = orc.log_likelihood(xh, env["y"], env["add"], env["mult"], 1, 4, True)
    assert abs(float(val) - ref_val) <= 1e-6 * abs(ref_val)


def test_finite_differences_of_objective(env):
    """Central differences (h=1e-3) of log-likelihood + RDP at 64 seeded voxels vs autograd
    (ObjectiveFunctionTests.h:88-130: tolerance max|g|/1000)."""
    import torch
    from stir_b200.autograd import PoissonLogLikelihood, Prior
    from stir_b200.osmaposl import RelativeDifferencePrior
    proj = env["proj"]
    xh = phantoms.smooth_random_field(env["img"], 2.0, seed=11) + 0.5
    x = env["dimg"](xh).requires_grad_(True)
    L = PoissonLogLikelihood(proj, env["dpd"](env["y"]), env["dpd"](env["add"]))
    R = Prior(proj, RelativeDifferencePrior(0.1, gamma=2.0, epsilon=0.0))

    def obj(t):
        return L(t) - R(t)

    (g,) = torch.autograd.grad(obj(x), x)
    g = g.double()
    rng = np.random.default_rng(12)
    ny, nx, nz = proj.device_image_shape
    # voxels inside the FOV circle (outside it the likelihood does not depend on x)
    picks = []
    while len(picks) < 64:
        yy, xx, zz = rng.integers(16, 48), rng.integers(16, 48), rng.integers(0, nz)
        picks.append((int(yy), int(xx), int(zz)))
    h = 1e-3
    tol = float(g.abs().max()) / 1000
    xd = x.detach()
    for (yy, xx, zz) in picks:
        xp = xd.clone()
        xm = xd.clone()
        xp[yy, xx, zz] += h
        xm[yy, xx, zz] -= h
        num = (float(obj(xp)) - float(obj(xm))) / (2 * h)
        assert abs(num - float(g[yy, xx, zz])) <= tol, (yy, xx, zz, num, float(g[yy, xx, zz]))


@pytest.mark.parametrize("zero_ends", [False, True])
def test_stored_ratio_equals_recomputed_projection(env, zero_ends):
    """The log-likelihood keeps the gradient ratios of its forward projection for backward (one projection per
    step) or projects again in backward: the values agree bit for bit, the gradients bit for bit with the
    deterministic back projection, for a batch of 3 images on a subset."""
    import torch
    from stir_b200.autograd import PoissonLogLikelihood
    proj = env["proj"]
    xs = torch.stack([env["dimg"](phantoms.smooth_random_field(env["img"], 2.0, seed=20 + k)) for k in range(3)])
    args = (proj, env["dpd"](env["y"]), env["dpd"](env["add"]), env["dpd"](env["mult"]), 2, 6, zero_ends,
            _abi.BACKPROJECT_DETERMINISTIC)
    out = []
    for store in (True, False):
        x = xs.clone().requires_grad_(True)
        val = PoissonLogLikelihood(*args, store_ratio=store)(x)
        (g,) = torch.autograd.grad(val, x)
        out.append((float(val), g))
    assert out[0][0] == out[1][0]
    assert torch.equal(out[0][1], out[1][1])
