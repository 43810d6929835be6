"""The five workloads' reconstructions as specified, pinned to the oracle (OSMAPOSLReconstruction.cxx:371-516).

Each test builds the workload's seeded inputs (stir_b200.workloads), runs the GPU reconstruction through the C ABI
and, from the same inputs, the oracle's float restatement of STIR (with its own sensitivities), comparing the images
after every sub-iteration (relative L2 <= 1e-4), and reports the error against the oracle's FP64 restatement
(the float and double algorithms differ where a LOR's field-of-view entry lands on a voxel boundary; the bound
asserted for it is loose and the measured value is printed).
"""
import numpy as np
import pytest

from stir_b200 import geometry as G
from stir_b200 import workloads

pytestmark = pytest.mark.gpu

OSEM_TOL = 1e-4   # images after identical sub-iterations (relative L2)
SENS_TOL = 1e-5   # sensitivities (back projections)
FP64_BOUND = 1e-2  # float algorithm against the double one: reported, loosely bounded


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _host(proj):
    def pd(t):
        return proj.projdata_from_device_layout(t).cpu().numpy()

    def img(t):
        return proj.image_from_device_layout(t).cpu().numpy()

    def dev(a):
        import torch
        return proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda())
    return pd, img, dev


def _report(name, **errs):
    print(f"\n[{name}] " + ", ".join(f"{k} {v:.3e}" for k, v in errs.items()))


@pytest.fixture(scope="module")
def clinical(cuda_device, oracle_lib):
    from stir_b200.projectors import RayTracingProjector
    proj = RayTracingProjector(*G.clinical_3d_pet(), device=cuda_device)
    return proj, oracle_lib.Oracle(proj.geometry)


def test_small_3d_pet_osem_as_specified(cuda_device, oracle_lib):
    """8 rings x 288 detectors, 64x64x15: attenuation factors from mu = 0.0096 /mm through the projector, 10 %
    uniform background, ~5e6 counts (seed 2), OSEM 6 subsets x 2 iterations, every sub-iteration vs the oracle."""
    import torch
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    from stir_b200.projectors import RayTracingProjector
    proj = RayTracingProjector(*G.small_3d_pet(), device=cuda_device)
    orc, o64 = oracle_lib.Oracle(proj.geometry), oracle_lib.Oracle(proj.geometry, 64)
    hpd, himg, _ = _host(proj)
    d = workloads.small_3d_pet_data(proj)
    y, a, m = hpd(d["y"]), hpd(d["additive"]), hpd(d["mult"])
    assert abs(d["events"] - 5e6) < 0.01 * 5e6
    # BinNormalisationFromAttenuationImage: factors = 1 / exp(A mu) with the oracle's projection
    m_ref = np.float32(1.0) / np.exp(orc.forward(d["mu"]).astype(np.float32))
    assert rel_l2(m, m_ref) <= 1e-6
    nsub = 6
    rec = OSMAPOSLReconstruction(proj, d["y"], additive=d["additive"], mult=d["mult"], num_subsets=nsub,
                                 num_subiterations=2 * nsub).set_up()
    sens = [orc.sensitivity(m, s, nsub) for s in range(nsub)]
    sens64 = [o64.sensitivity(m, s, nsub) for s in range(nsub)]
    for s in range(nsub):
        assert rel_l2(himg(rec.sensitivities[s]), sens[s]) <= SENS_TOL
    x = proj.empty_image().fill_(1.0)
    xo = np.ones(proj.image_shape, np.float32)
    x64 = np.ones(proj.image_shape, np.float64)
    errs = []
    for it in range(1, 2 * nsub + 1):
        rec.subiteration_num = it
        sub = rec.get_subset_num()
        rec.update_estimate(x)
        xo, _ = orc.osmaposl_update(xo, y, a, sens[sub], sub, nsub, it, max_rel=3.4028234663852886e38)
        x64, _ = o64.osmaposl_update(x64, y, a, sens64[sub], sub, nsub, it, max_rel=3.4028234663852886e38)
        errs.append(rel_l2(himg(x), xo))
        assert errs[-1] <= OSEM_TOL, (it, errs)
    torch.cuda.synchronize()
    e64 = rel_l2(himg(x), x64)
    _report("small_3d_pet OSEM 6x2", max_vs_oracle=max(errs), vs_fp64_oracle=e64, oracle_vs_fp64=rel_l2(xo, x64))
    assert e64 <= FP64_BOUND


def test_clinical_osem_first_subiterations(clinical, oracle_lib):
    """64 rings x 504 detectors, 344x344x127: normalisation U[0.8, 1.2] x attenuation, smooth 30 % additive term,
    ~3e8 counts; the first 3 sub-iterations of OSEM with 21 subsets vs the oracle."""
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    proj, orc = clinical
    o64 = oracle_lib.Oracle(proj.geometry, 64)
    hpd, himg, _ = _host(proj)
    d = workloads.clinical_data(proj)
    y, a, m = hpd(d["y"]), hpd(d["additive"]), hpd(d["mult"])
    nsub, n = 21, 3
    rec = OSMAPOSLReconstruction(proj, d["y"], additive=d["additive"], mult=d["mult"], num_subsets=nsub,
                                 num_subiterations=n)
    # only the subsets used: the sensitivities of subsets 0..2
    rec.set_up()
    x = proj.empty_image().fill_(1.0)
    xo = np.ones(proj.image_shape, np.float32)
    x64 = np.ones(proj.image_shape, np.float64)
    errs, serrs = [], []
    for it in range(1, n + 1):
        rec.subiteration_num = it
        sub = rec.get_subset_num()
        s32 = orc.sensitivity(m, sub, nsub)
        serrs.append(rel_l2(himg(rec.sensitivities[sub]), s32))
        assert serrs[-1] <= SENS_TOL
        rec.update_estimate(x)
        xo, _ = orc.osmaposl_update(xo, y, a, s32, sub, nsub, it, max_rel=3.4028234663852886e38)
        x64, _ = o64.osmaposl_update(x64, y, a, o64.sensitivity(m, sub, nsub), sub, nsub, it,
                                     max_rel=3.4028234663852886e38)
        errs.append(rel_l2(himg(x), xo))
        assert errs[-1] <= OSEM_TOL, (it, errs)
    e64 = rel_l2(himg(x), x64)
    _report("clinical OSEM 21 subsets, 3 sub-iterations", max_vs_oracle=max(errs), max_sens=max(serrs),
            vs_fp64_oracle=e64, oracle_vs_fp64=rel_l2(xo, x64))
    assert e64 <= FP64_BOUND


def test_tof_osmaposl_quadratic_prior(cuda_device, oracle_lib):
    """33 timing bins of 50 ps, 550 ps FWHM, ~3e8 counts, QuadraticPrior beta 0.5 (26 neighbours), 21 subsets x 3
    iterations.

    STIR's default sensitivity for TOF data comes from the non-TOF projector with the non-TOF symmetries, so its
    subset s holds other views than the TOF data's subset s (here 0, 21, 51, 72, 93, 123 against 0, 21, 42, 63, 84,
    105, 126): near the edge of the field of view some voxels then get a zero sensitivity with a non-zero
    numerator and an infinite update, in STIR's arithmetic as in the oracle and here.  That sensitivity is checked
    against the oracle; the reconstruction uses "use time-of-flight sensitivities" (subsets that agree).  Every one
    of the 63 sub-iterations is checked from identical inputs (the one-step-late update with beta 0.5 amplifies
    float rounding along a trajectory); the independent GPU trajectory's distance to the oracle's is reported."""
    import torch
    from stir_b200.osmaposl import OSMAPOSLReconstruction, QuadraticPrior
    from stir_b200.projectors import RayTracingProjector
    proj = RayTracingProjector(*G.tof_small_3d_pet(num_tof_bins=33), device=cuda_device)
    nt = proj.non_tof_projector()
    orc, orc_nt = oracle_lib.Oracle(proj.geometry), oracle_lib.Oracle(nt.geometry)
    o64 = oracle_lib.Oracle(proj.geometry, 64)
    hpd, himg, dev = _host(proj)
    d = workloads.tof_data(proj)
    y, a, m = hpd(d["y"]), hpd(d["additive"]), hpd(d["mult"])
    m_nt = nt.projdata_from_device_layout(d["sensitivity_mult"]).cpu().numpy()
    assert abs(d["events"] - 3e8) < 0.01 * 3e8
    nsub, n = 21, 63
    prior = QuadraticPrior(0.5)
    # STIR's default: the non-TOF sensitivity
    rec_nt = OSMAPOSLReconstruction(proj, d["y"], additive=d["additive"], mult=d["mult"], num_subsets=nsub,
                                    sensitivity_mult=d["sensitivity_mult"]).set_up()
    for s in (0, 7, 20):
        assert rel_l2(himg(rec_nt.sensitivities[s]), orc_nt.sensitivity(m_nt, s, nsub)) <= SENS_TOL
    del rec_nt
    rec = OSMAPOSLReconstruction(proj, d["y"], additive=d["additive"], mult=d["mult"], num_subsets=nsub,
                                 num_subiterations=n, prior=prior, use_tofsens=True).set_up()
    sens = [orc.sensitivity(m, s, nsub) for s in range(nsub)]
    sens64 = [o64.sensitivity(m, s, nsub) for s in range(nsub)]
    for s in range(nsub):
        assert rel_l2(himg(rec.sensitivities[s]), sens[s]) <= SENS_TOL
    abi_prior = prior.as_abi(rec.map_model)
    step64 = []
    xo = np.ones(proj.image_shape, np.float32)
    x_traj = proj.empty_image().fill_(1.0)
    step_errs = []
    for it in range(1, n + 1):
        rec.subiteration_num = it
        sub = rec.get_subset_num()
        x = dev(xo)
        rec.update_estimate(x)
        rec.update_estimate(x_traj)
        # the same step in double from the same input: the float algorithm's own error
        x64, _ = o64.osmaposl_update(xo.astype(np.float64), y, a, sens64[sub], sub, nsub, it, prior=abi_prior,
                                     max_rel=3.4028234663852886e38)
        xo, _ = orc.osmaposl_update(xo, y, a, sens[sub], sub, nsub, it, prior=abi_prior,
                                    max_rel=3.4028234663852886e38)
        step_errs.append(rel_l2(himg(x), xo))
        step64.append(rel_l2(himg(x), x64))
        assert step_errs[-1] <= 1e-5, (it, step_errs[-1])
    torch.cuda.synchronize()
    _report("TOF OSMAPOSL QP 0.5, 21x3", max_step_vs_oracle=max(step_errs), max_step_vs_fp64_oracle=max(step64),
            trajectory_vs_oracle=rel_l2(himg(x_traj), xo))
    assert max(step64) <= FP64_BOUND


def test_dynamic_frames_batched_vs_oracle(clinical, cuda_device, oracle_lib):
    """Two frames of the 24-frame dynamic study, one per image size (344x344x127 with 21 subsets, 172x172x127 with
    7), reconstructed together by the batched kernels; each frame against the oracle after every batched
    sub-iteration."""
    import torch
    from stir_b200.batch import BatchedOSMAPOSL
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    from stir_b200.projectors import RayTracingProjector
    proj344, orc344 = clinical
    proj172 = RayTracingProjector(*G.clinical_3d_pet_half(), device=cuda_device)
    projs = {344: proj344, 172: proj172}
    orcs = {344: orc344, 172: oracle_lib.Oracle(proj172.geometry)}
    o64s = {344: oracle_lib.Oracle(proj344.geometry, 64), 172: oracle_lib.Oracle(proj172.geometry, 64)}
    frames = workloads.dynamic_frames(projs, cuda_device)
    chosen = [frames[1], frames[21]]
    del frames
    torch.cuda.empty_cache()
    assert [(f["size"], f["nsub"]) for f in chosen] == [(344, 21), (172, 7)]
    n = 3
    batch = BatchedOSMAPOSL(cuda_device)
    state = []
    for f in chosen:
        p = projs[f["size"]]
        rec = OSMAPOSLReconstruction(p, f["y"], additive=f["additive"], num_subsets=f["nsub"], num_subiterations=n)
        rec.set_up()
        x = p.empty_image().fill_(1.0)
        batch.add(rec, x)
        hpd, himg, _ = _host(p)
        state.append(dict(p=p, f=f, rec=rec, x=x, himg=himg, y=hpd(f["y"]), a=hpd(f["additive"]),
                          xo=np.ones(p.image_shape, np.float32), x64=np.ones(p.image_shape, np.float64)))
    errs = {344: [], 172: []}
    for k in range(1, n + 1):
        batch.run(k, 1, use_graph=False)
        torch.cuda.synchronize()
        for s in state:
            size, nsub = s["f"]["size"], s["f"]["nsub"]
            sub = (k - 1) % nsub
            sens = orcs[size].sensitivity(None, sub, nsub)
            assert rel_l2(s["himg"](s["rec"].sensitivities[sub]), sens) <= SENS_TOL
            s["xo"], _ = orcs[size].osmaposl_update(s["xo"], s["y"], s["a"], sens, sub, nsub, k,
                                                    max_rel=3.4028234663852886e38)
            s["x64"], _ = o64s[size].osmaposl_update(s["x64"], s["y"], s["a"], o64s[size].sensitivity(None, sub, nsub),
                                                     sub, nsub, k, max_rel=3.4028234663852886e38)
            errs[size].append(rel_l2(s["himg"](s["x"]), s["xo"]))
            assert errs[size][-1] <= OSEM_TOL, (size, k, errs[size])
    batch.close()
    e64 = {s["f"]["size"]: rel_l2(s["himg"](s["x"]), s["x64"]) for s in state}
    _report("dynamic frames batched, 3 sub-iterations", frame_344=max(errs[344]), frame_172=max(errs[172]),
            frame_344_vs_fp64_oracle=e64[344], frame_172_vs_fp64_oracle=e64[172])
    assert max(e64.values()) <= FP64_BOUND


@pytest.fixture(scope="module")
def half(cuda_device):
    from stir_b200.projectors import RayTracingProjector
    return RayTracingProjector(*G.clinical_3d_pet_half(), device=cuda_device)


def _c3_batch(proj, n=8):
    """8 seeded smooth fields (Gaussian noise blurred with sigma 3 voxels, clipped >= 0; seeds 10..17) and Poisson
    data of each with the attenuation of a water cylinder and a 10 % background."""
    import torch
    from stir_b200 import phantoms
    imgs = [phantoms.smooth_random_field(proj.image, sigma_vox=3.0, seed=10 + k) for k in range(n)]
    x = torch.stack([proj.image_to_device_layout(torch.from_numpy(a).cuda()) for a in imgs])
    mu = phantoms.attenuation_cylinder(proj.image, radius_mm=150.0, mu_per_mm=0.0096)
    m = workloads._attenuation_factors(proj, mu)
    ys, adds = [], []
    for k in range(n):
        ybar = m * proj.forward_dev(x[k])
        b = 0.1 * float(ybar.double().mean())
        y, _ = workloads._poisson(ybar + b, 3e7, 100 + k)
        ys.append(y)
        adds.append(torch.full_like(y, b) / m)
    return x, torch.stack(ys), torch.stack(adds), m


def test_differentiable_projector_batch(half, oracle_lib):
    """The differentiable projector at the workload's size: a batch of 8 images of 172x172x127 on the clinical scanner
    (zoom 0.5), one launch per direction.  Batched projections equal the single-image ones; adjoint test on random
    x, y; Poisson log-likelihood (attenuation, 10 % background) plus RelativeDifferencePrior (beta 0.1, gamma 2):
    central finite differences (h = 1e-3) at 64 seeded voxels within max|g|/1000 (ObjectiveFunctionTests.h:88-130),
    and the log-likelihood and prior gradients against the oracle's."""
    import torch
    from stir_b200.autograd import PoissonLogLikelihood, Prior, back_project, forward_project
    from stir_b200.osmaposl import RelativeDifferencePrior
    proj = half
    x, y, add, m = _c3_batch(proj)
    B = x.shape[0]
    # batched = single-image projections
    fb = forward_project(x, proj)
    for k in (0, 5):
        assert torch.equal(fb[k], proj.forward_dev(x[k]))
    bb = back_project(y, proj)
    for k in (0, 7):
        s = proj.back_dev(y[k])
        assert float((bb[k] - s).norm() / s.norm()) <= 1e-6
    # adjoint on random x, y (through autograd: the backward of forward_project is the back projector)
    g = torch.Generator(device="cuda").manual_seed(21)
    xr = torch.rand(x.shape, device="cuda", generator=g).requires_grad_(True)
    yr = torch.rand(y.shape, device="cuda", generator=g)
    lhs = (forward_project(xr, proj).double() * yr.double()).sum()
    (gx,) = torch.autograd.grad(lhs, xr)
    rhs = (xr.detach().double() * gx.double()).sum()
    assert abs(float(lhs - rhs)) <= 1e-5 * abs(float(lhs))
    # objective: sum over the batch of the log-likelihood minus the prior
    L = PoissonLogLikelihood(proj, y, add, m)
    R = Prior(proj, RelativeDifferencePrior(0.1, gamma=2.0, epsilon=0.0))
    xg = x.clone().requires_grad_(True)
    (grad,) = torch.autograd.grad(L(xg) - R(xg), xg)
    grad = grad.double()
    tol = float(grad.abs().max()) / 1000
    rng = np.random.default_rng(22)
    ny, nx, nz = proj.device_image_shape
    h = 1e-3
    # the fields are clipped at 0, where the Relative Difference prior (epsilon 0) is not differentiable and x - h
    # leaves its domain: the voxels are drawn where the voxel and its 26 neighbours are at least 0.05
    xh = x.cpu().numpy()
    picks = []
    while len(picks) < 64:
        k, yy, xx, zz = int(rng.integers(B)), int(rng.integers(40, ny - 40)), int(rng.integers(40, nx - 40)), \
            int(rng.integers(1, nz - 1))
        if xh[k, yy - 1:yy + 2, xx - 1:xx + 2, zz - 1:zz + 2].min() >= 0.05:
            picks.append((k, yy, xx, zz))
    # The log-likelihood along a voxel's direction is evaluated in double from the float projections A x and A e_v
    # (ybar(x +- h e_v) = m (A x +- h A e_v + a)), with STIR's clipping and thresholds: re-projecting x +- h in
    # float would add rounding noise of about one unit in the last place of A x (~1e-5 of ~150) per LOR against a
    # change of 2e-3, which over the ~1e4 LORs through a voxel is as large as the tolerance.
    S, nvw, nt = proj.proj_data_info.max_segment_num, proj.proj_data_info.num_views, proj.proj_data_info.num_tangential_poss
    def thresholds(yk):  # max over each viewgram x 1e-6 (divide_and_truncate's small value), per bin
        parts, off = [], 0
        for seg in range(-S, S + 1):
            nax = proj.proj_data_info.get_num_axial_poss(seg)
            blk = yk[off:off + nvw * nt * nax].view(nvw, nt * nax)
            parts.append((blk.max(dim=1, keepdim=True).values * 1e-6).clamp(min=0).expand(-1, nt * nax).reshape(-1))
            off += nvw * nt * nax
        return torch.cat(parts)

    def loglik(ybar, yk, sv):
        ne = torch.maximum(ybar, yk / 1e4)
        return float(torch.where(yk <= sv, -ne, yk * torch.log(ne) - ne).sum())
    for k, yy, xx, zz in picks:
        yk = y[k].double()
        sv = thresholds(y[k]).double()
        ax = proj.forward_dev(x[k]).double()
        e = torch.zeros_like(x[k])
        e[yy, xx, zz] = 1.0
        col = proj.forward_dev(e).double()
        sel = col != 0
        md, ad = m.double()[sel], add[k].double()[sel]
        lp = loglik(md * (ax[sel] + h * col[sel] + ad), yk[sel], sv[sel])
        lm = loglik(md * (ax[sel] - h * col[sel] + ad), yk[sel], sv[sel])
        xp, xm = x[k].clone(), x[k].clone()
        xp[yy, xx, zz] += h
        xm[yy, xx, zz] -= h
        num = ((lp - lm) - (float(R(xp)) - float(R(xm)))) / (2 * h)
        assert abs(num - float(grad[k, yy, xx, zz])) <= tol, (k, yy, xx, zz, num, float(grad[k, yy, xx, zz]))
    # gradients against the oracle: the log-likelihood's on subset 0 of 42 (bounded CPU time), the prior's
    orc = oracle_lib.Oracle(proj.geometry)
    hpd, himg, _ = _host(proj)
    Ls = PoissonLogLikelihood(proj, y[:2], add[:2], m, subset_num=0, num_subsets=42)
    xs = x[:2].clone().requires_grad_(True)
    (gs,) = torch.autograd.grad(Ls(xs), xs)
    for k in range(2):
        ref = orc.log_likelihood_gradient(himg(x[k]), hpd(y[k]), hpd(add[k]), hpd(m), 0, 42)
        assert rel_l2(himg(gs[k]), ref) <= 1e-5
    from stir_b200 import _abi as A
    pr = A.Prior(type=A.PRIOR_RELATIVE_DIFFERENCE, penalisation_factor=0.1, gamma=2.0, epsilon=0.0, only_2D=0,
                 map_model=A.MAP_MULTIPLICATIVE, kappa_dev=None)
    xr0 = x[0].clone().requires_grad_(True)
    (gp,) = torch.autograd.grad(R(xr0), xr0)
    assert rel_l2(himg(gp), oracle_lib.prior_gradient(pr, himg(x[0]), proj.image.voxel_size)) <= 1e-6
    _report("differentiable projector, 8 x 172x172x127", fd_tolerance=tol)
