"""Batched OSMAPOSL (several frames per persistent launch) against frame-by-frame OSMAPOSL on the GPU."""
import numpy as np
import pytest

from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu

BATCH_TOL = 1e-4  # relative L2 per frame: only the order of float additions of the back projection differs


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _coarse_image():
    # one plane per axial position (4 mm planes, span 1): a different planes-per-position than small_3d_pet
    return G.ImageGeometry(8, 48, 48, (4.0, 5.0, 5.0))


@pytest.fixture(scope="module")
def frames(cuda_device):
    """Data of three geometries' worth of frames: the small scanner with its default image (2 planes per
    axial position) and with a coarse image (1 plane per axial position)."""
    import torch
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    projs = {"fine": RayTracingProjector(pdi, img, device=cuda_device),
             "coarse": RayTracingProjector(pdi, _coarse_image(), device=cuda_device)}
    data = {}
    for name, proj in projs.items():
        xt = phantoms.cylinder_with_spheres(proj.image, radius_mm=90.0, n_spheres=2, sphere_radius=(10.0, 10.0), seed=1)
        xt_dev = proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(xt, np.float32)).cuda())
        ybar = proj.forward_dev(xt_dev)
        bg = float(0.1 * ybar.mean())
        rng = np.random.default_rng(5)
        scale = 2e6 / float((ybar + bg).sum())
        lam = ((ybar + bg) * scale).cpu().numpy()
        y = torch.from_numpy(rng.poisson(lam).astype(np.float32) / np.float32(scale)).cuda()
        add = torch.full_like(y, bg)
        data[name] = (proj, y, add)
    return data


def _specs():
    from stir_b200.osmaposl import QuadraticPrior, RelativeDifferencePrior
    return [
        dict(geom="fine", nsub=3, start=0, n=5, prior=None, additive=True, zero_ends=False),
        dict(geom="fine", nsub=2, start=1, n=3, prior=QuadraticPrior(0.05), additive=True, zero_ends=True),
        dict(geom="coarse", nsub=4, start=0, n=6, prior=RelativeDifferencePrior(0.1), additive=False, zero_ends=False),
        dict(geom="coarse", nsub=1, start=0, n=2, prior=None, additive=True, zero_ends=False),
    ]


def _recon(data, spec, **kw):
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    proj, y, add = data[spec["geom"]]
    return OSMAPOSLReconstruction(proj, y, additive=add if spec["additive"] else None, num_subsets=spec["nsub"],
                                  num_subiterations=spec["n"], start_subset_num=spec["start"],
                                  zero_seg0_end_planes=spec["zero_ends"], prior=spec["prior"],
                                  MAP_model="multiplicative", **kw)


def _references(data, specs):
    import torch
    out = []
    for sp in specs:
        proj = data[sp["geom"]][0]
        rec = _recon(data, sp)
        x = proj.empty_image().fill_(1.0)
        rec.reconstruct(x)
        torch.cuda.synchronize()
        out.append((rec, x.cpu().numpy()))
    return out


@pytest.mark.parametrize("geoms", ["mixed", "fine_only"])
@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_equals_frame_by_frame(frames, geoms, use_graph):
    import torch
    from stir_b200.batch import BatchedOSMAPOSL
    specs = _specs() if geoms == "mixed" else [s for s in _specs() if s["geom"] == "fine"]
    refs = _references(frames, specs)
    batch = BatchedOSMAPOSL()
    xs = []
    for sp, (rec, _) in zip(specs, refs):
        x = frames[sp["geom"]][0].empty_image().fill_(1.0)
        # reuse the reference's sensitivities: the comparison is of the sub-iterations alone
        brec = _recon(frames, sp)
        brec.sensitivities = rec.sensitivities
        batch.add(brec, x)
        xs.append(x)
    batch.reconstruct(use_graph=use_graph)
    torch.cuda.synchronize()
    for sp, x, (_, ref) in zip(specs, xs, refs):
        err = rel_l2(x.cpu().numpy(), ref)
        assert err < BATCH_TOL, (sp, err)
    batch.close()


def test_batch_runs_in_pieces_and_autotunes(frames):
    """Sub-iterations 1..2 then 3..end, with an autotuned configuration, equal one run; the graph of a
    range is reused when launched again."""
    import torch
    from stir_b200.batch import BatchedOSMAPOSL
    specs = _specs()
    refs = _references(frames, specs)
    batch = BatchedOSMAPOSL()
    xs = []
    for sp, (rec, _) in zip(specs, refs):
        x = frames[sp["geom"]][0].empty_image().fill_(1.0)
        brec = _recon(frames, sp)
        brec.sensitivities = rec.sensitivities
        batch.add(brec, x)
        xs.append(x)
    cfg = batch.autotune(1)
    assert cfg["ctas_per_sm_forward"] >= 1 and cfg["ctas_per_sm_back"] >= 1 and cfg["order"] in (0, 1, 2)
    assert cfg["kernels"] in (1, 2, 3, 4)  # the tuner names the family it chose
    assert batch.get_config() == cfg
    x0 = [x.clone() for x in xs]
    batch.run(1, 2, use_graph=True)
    batch.run(3, None, use_graph=True)
    torch.cuda.synchronize()
    for sp, x, (_, ref) in zip(specs, xs, refs):
        assert rel_l2(x.cpu().numpy(), ref) < BATCH_TOL, sp
    # replay the cached graphs from the initial estimates
    for x, a in zip(xs, x0):
        x.copy_(a)
    batch.run(1, 2, use_graph=True)
    batch.run(3, None, use_graph=True)
    torch.cuda.synchronize()
    for sp, x, (_, ref) in zip(specs, xs, refs):
        assert rel_l2(x.cpu().numpy(), ref) < BATCH_TOL, sp
    assert batch.num_cancelled(0) >= 0
    batch.close()


@pytest.mark.parametrize("kernels", [1, 3, 4])
def test_batch_kernel_families(frames, kernels):
    """Each kernel family the autotuner chooses among (column-staged path items, packed warp per basic bin, CTA per
    basic bin; the 8-ring frames allow all three) reconstructs the frames as frame by frame does."""
    import torch
    from stir_b200.batch import BatchedOSMAPOSL
    specs = _specs()
    refs = _references(frames, specs)
    batch = BatchedOSMAPOSL()
    xs = []
    for sp, (rec, _) in zip(specs, refs):
        x = frames[sp["geom"]][0].empty_image().fill_(1.0)
        brec = _recon(frames, sp)
        brec.sensitivities = rec.sensitivities
        batch.add(brec, x)
        xs.append(x)
    batch.set_config(order=2 if kernels == 1 else 1, kernels=kernels)  # item by item across frames, or longest first
    batch.run(1, None, use_graph=True)
    torch.cuda.synchronize()
    assert batch.get_config()["kernels"] == kernels
    for sp, x, (_, ref) in zip(specs, xs, refs):
        assert rel_l2(x.cpu().numpy(), ref) < BATCH_TOL, (kernels, sp)
    batch.close()


def test_batch_rejects_bad_frames(frames):
    import torch
    from stir_b200 import _abi
    from stir_b200.batch import BatchedOSMAPOSL
    sp = _specs()[0]
    batch = BatchedOSMAPOSL()
    proj = frames[sp["geom"]][0]
    x = proj.empty_image().fill_(1.0)
    rec = _recon(frames, sp, start_subiteration_num=2)
    with pytest.raises(ValueError):
        batch.add(rec, x)
    with pytest.raises(_abi.B200Error):
        batch.set_config(order=5)
    with pytest.raises(_abi.B200Error):
        batch.set_config(kernels=7)
    batch.close()


def test_batch_tof_frames_equal_frame_by_frame(cuda_device):
    """TOF frames go through the per-basic-bin batched kernels (one CTA per timing bin of a basic bin); frame by
    frame they go through the packed kernels: the reconstructions agree to the order of float additions."""
    import torch
    from stir_b200.batch import BatchedOSMAPOSL
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=7, timing_bin_ps=250.0, num_views=48)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    xt = phantoms.cylinder_with_spheres(proj.image, radius_mm=90.0, n_spheres=2, sphere_radius=(10.0, 10.0), seed=3)
    ybar = proj.forward_dev(proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(xt, np.float32)).cuda()))
    bg = float(0.1 * ybar.mean())
    rng = np.random.default_rng(8)
    batch = BatchedOSMAPOSL()
    runs = []
    from stir_b200.osmaposl import QuadraticPrior
    # a strong MAP-OSL prior (beta 0.5 here) multiplies float-rounding differences about tenfold per sub-iteration
    # (the clamped one-step-late denominator), so the comparison uses beta 0.05, where they stay at 1e-7
    for k, (nsub, n, prior) in enumerate([(3, 4, None), (2, 3, None), (7, 9, QuadraticPrior(0.05))]):
        scale = (1e6 * (k + 1)) / float((ybar + bg).sum())
        y = torch.from_numpy(rng.poisson(((ybar + bg) * scale).cpu().numpy()).astype(np.float32) / np.float32(scale)).cuda()
        add = torch.full_like(y, bg)
        ref = OSMAPOSLReconstruction(proj, y, additive=add, num_subsets=nsub, num_subiterations=n, prior=prior,
                                     use_tofsens=True)
        xr = proj.empty_image().fill_(1.0)
        ref.reconstruct(xr)
        rec = OSMAPOSLReconstruction(proj, y, additive=add, num_subsets=nsub, num_subiterations=n, prior=prior)
        rec.sensitivities = ref.sensitivities
        x = proj.empty_image().fill_(1.0)
        batch.add(rec, x)
        runs.append((x, xr))
    batch.reconstruct(use_graph=True)
    torch.cuda.synchronize()
    for x, xr in runs:
        assert rel_l2(x.cpu().numpy(), xr.cpu().numpy()) < BATCH_TOL
    batch.close()


def test_batch_deterministic_strong_prior_is_bit_reproducible(frames):
    """Frames with a strong one-step-late prior (QP beta 0.5, which multiplies float-rounding differences about
    tenfold per sub-iteration) and the deterministic back projection: the batched reconstruction equals each frame's
    own deterministic reconstruction bit for bit, and a second batched run repeats it."""
    import torch
    from stir_b200 import _abi
    from stir_b200.batch import BatchedOSMAPOSL
    from stir_b200.osmaposl import OSMAPOSLReconstruction, QuadraticPrior
    mode = _abi.BACKPROJECT_DETERMINISTIC
    specs = [("fine", 3, 6), ("coarse", 4, 5), ("fine", 2, 4)]
    refs, recs = [], []
    for geom, nsub, n in specs:
        proj, y, add = frames[geom]
        ref = OSMAPOSLReconstruction(proj, y, additive=add, num_subsets=nsub, num_subiterations=n,
                                     prior=QuadraticPrior(0.5), back_projection_mode=mode).set_up()
        xr = proj.empty_image().fill_(1.0)
        ref.reconstruct(xr)
        refs.append(xr)
        recs.append((proj, OSMAPOSLReconstruction(proj, y, additive=add, num_subsets=nsub, num_subiterations=n,
                                                  prior=QuadraticPrior(0.5), back_projection_mode=mode), ref))
    outs = []
    for run in range(2):
        batch = BatchedOSMAPOSL()
        xs = []
        for proj, rec, ref in recs:
            rec.sensitivities = ref.sensitivities
            x = proj.empty_image().fill_(1.0)
            batch.add(rec, x)
            xs.append(x)
        batch.reconstruct(use_graph=bool(run))
        torch.cuda.synchronize()
        outs.append([x.clone() for x in xs])
        batch.close()
    for a, b, r in zip(outs[0], outs[1], refs):
        assert torch.equal(a, b)
        assert torch.equal(a, r)
