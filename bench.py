"""Benchmark of the B200 ray-tracing projector pair (forward + back projection LORs/s).

Default workload: the clinical 3D PET geometry (64 rings x 504 detectors, span 11, max ring
difference 60, 252 views x 344 tangential positions = 72.6M LORs; image 344x344x127), seeded
synthetic phantom.  One step = a forward projection of every LOR followed by a back projection
of every LOR (the projector work of one full OSEM iteration).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N>1) every rank projects its own copy of the workload (independent frames, no
collective): value = all ranks' LORs / the slowest rank's time ("scaling": "weak").
--impl reference times the CPU restatement of STIR's OpenMP path (oracle) on the host cores on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = ("clinical 3D PET: 64 rings x 504 det, R 328 mm, span 11, max ring diff 60, 252 views x 344 tang "
            "(72,557,856 LORs), image 344x344x127 (2.09x2.09x2.03 mm), ray-tracing matrix, 1 tangential LOR")
METRIC = "fwd+back LORs/s"
CPU_SAMPLE_SUBSET = (0, 42)  # views 0, 42 and their symmetry partners: 1/42 of the views
# the column-staged projectors (stir_b200/csrc/paths.cu) that project the clinical workload
FWD_KERNEL, BACK_KERNEL = "forward_paths_kernel", "back_paths_kernel"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mode", default="replicas", choices=["replicas", "split"],
                    help="replicas: an independent copy of the workload per GPU (weak scaling); split: one copy of the "
                         "workload split across the GPUs by views, each holding its share of the projection data, "
                         "the back projections summed by an NCCL all-reduce (strong scaling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched dynamic OSEM measurement")
    ap.add_argument("--batch-iterations", type=int, default=2, help="full OSEM iterations per dynamic frame")
    ap.add_argument("--no-extras", action="store_true", help="skip the list-mode and Gibbs penalty measurements")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region: one nvidia-smi process streaming
    a sample every 50 ms (-lms) from just before the region until its end."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, interval_ms: int = 50):
        self.idx = device_index
        self.interval_ms = interval_ms
        self.samples = []
        self._proc = None
        self._th = None

    def _read(self):
        for line in self._proc.stdout:
            cols = [c.strip() for c in line.split(",")]
            if len(cols) >= 9:
                self.samples.append(cols)

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                           "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._th = threading.Thread(target=self._read, daemon=True)
            self._th.start()
            time.sleep(0.15)  # the first sample precedes the timed region
        except OSError:
            self._proc = None
        return self

    def __exit__(self, *a):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._th:
            self._th.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and "Active" in s[5 + i]
                          and "Not" not in s[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def subset_num_bins(pdi, geometry, bits, subset, nsub):
    from stir_b200.subsets import views_in_subset
    views = views_in_subset(geometry, subset, nsub, bits)
    return len(views) * pdi.num_sinograms * pdi.num_tangential_poss


class CpuBaseline:
    """The oracle (restated STIR OpenMP path) on a bounded sample of the workload: forward + back
    projection of one subset of the clinical geometry with all host threads."""

    def __init__(self, nthreads=None):
        from oracle.oracle import Oracle
        from stir_b200 import geometry as G
        from stir_b200 import phantoms
        self.pdi, self.img = G.clinical_3d_pet()
        self.geo = G.make_geometry(self.pdi, self.img)
        self.orc = Oracle(self.geo)
        self.nthreads = nthreads or os.cpu_count() or 1
        self.x = phantoms.cylinder_with_spheres(self.img, n_spheres=6, sphere_radius=(5, 18), ellipse_axes=(150, 100))
        self.sub, self.nsub = CPU_SAMPLE_SUBSET
        t0 = time.perf_counter()
        y = self.orc.forward(self.x, self.sub, self.nsub, self.nthreads)  # fills the row cache
        self.cache_fill_s = time.perf_counter() - t0
        self.y = (y + np.float32(0.3)).astype(np.float32)
        self.out = np.zeros(self.orc.projdata_size, np.float32)
        self.nbins = subset_num_bins(self.pdi, self.geo, self.orc.symmetries_used, self.sub, self.nsub)

    def step(self):
        t0 = time.perf_counter()
        self.orc.forward(self.x, self.sub, self.nsub, self.nthreads, out=self.out)
        self.orc.back(self.y, self.sub, self.nsub, self.nthreads)
        return time.perf_counter() - t0

    def describe(self, seconds):
        return {"value": self.nbins / seconds, "unit": "LORs/s", "cores": self.nthreads, "kind": "port",
                "sample": f"forward+back of subset {self.sub} of {self.nsub} ({self.nbins} LORs) of the clinical "
                          f"workload with a warm row cache (cache fill {self.cache_fill_s:.2f} s), {self.nthreads} "
                          "OpenMP threads; restated CPU path, not the STIR binary"}


LM_EVENTS = 10_000_000


def random_lm_bins(pdi, n, rng, views=None):
    """n events on uniformly drawn bins (segment, view, axial, tangential, timing 0) of the geometry, optionally
    restricted to `views`."""
    S = pdi.max_segment_num
    seg = rng.integers(-S, S + 1, n)
    nax = np.array([pdi.get_num_axial_poss(int(s)) for s in range(-S, S + 1)])
    ax = (rng.random(n) * nax[seg + S]).astype(np.int64)
    view = rng.integers(0, pdi.num_views, n) if views is None else np.asarray(views)[rng.integers(0, len(views), n)]
    tang = rng.integers(pdi.min_tangential_pos_num, pdi.min_tangential_pos_num + pdi.num_tangential_poss, n)
    return np.stack([seg, view, ax, tang, np.zeros(n, np.int64)], 1).astype(np.int32)


def time_dev(fn, warm=3, reps=5):
    """mean device time of fn() in ms over reps calls (CUDA events on the current stream, after warm calls)"""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def listmode_and_priors(proj, pdi, img, xd, cpu_ref):
    """The list-mode sub-gradient (events/s) and the Gibbs Relative Difference penalty gradient (voxels/s) on the
    clinical geometry, with single-thread oracle baselines on bounded samples (cpu_ref: the CpuBaseline whose row
    cache already holds subset 0 of 42, or None)."""
    import torch
    from stir_b200 import _abi, gibbs
    from stir_b200.listmode import PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin as LM
    from stir_b200.listmode import pack_events
    out = {}
    rng = np.random.default_rng(5)
    bins = random_lm_bins(pdi, LM_EVENTS, rng)
    obj = LM(proj, pack_events(bins, None, np.full(LM_EVENTS, 0.1, np.float32), proj.device), has_add=True)
    g = proj.empty_image(zero=False)
    obj.set_method(_abi.LISTMODE_PER_EVENT)
    ms_ev = time_dev(lambda: obj.compute_sub_gradient_without_penalty(xd, 0, out=g))
    obj.set_method(_abi.LISTMODE_AUTO)
    ms = time_dev(lambda: obj.compute_sub_gradient_without_penalty(xd, 0, out=g))
    lm = {"metric": "list-mode sub-gradient events/s", "value": LM_EVENTS / (ms / 1e3), "unit": "events/s",
          "events": LM_EVENTS, "ms": ms, "gpu_launches": 3,
          "workload": "10M events on uniformly drawn bins of the clinical geometry (seed 5), value 1, additive 0.1, "
                      "one subset",
          "method": "binned (chosen automatically: events >= bins / 16): forward projection of the subset, one "
                    "thread per event adding y / (A x + c) to its bin, back projection of the subset",
          "per_event": {"value": LM_EVENTS / (ms_ev / 1e3), "ms": ms_ev, "gpu_launches": 1,
                        "method": "one warp per event: the event's row gathered, ratio, row scattered"}}
    if cpu_ref is not None:
        from stir_b200.subsets import views_in_subset
        views = views_in_subset(cpu_ref.geo, cpu_ref.sub, cpu_ref.nsub, cpu_ref.orc.symmetries_used)
        sample = random_lm_bins(pdi, 40000, np.random.default_rng(6), views)
        x_host = cpu_ref.x
        t0 = time.perf_counter()
        cpu_ref.orc.listmode("gradient", sample, np.ones(len(sample), np.float32), x_host,
                             corr=np.full(len(sample), 0.1, np.float32), has_add=True)
        dt = time.perf_counter() - t0
        lm["cpu_baseline"] = {"value": len(sample) / dt, "unit": "events/s", "cores": 1, "kind": "port",
                              "sample": f"{len(sample)} events on the bins of subset 0 of 42 (warm row cache), the "
                                        "oracle's sequential LM_gradient_and_value loop"}
    out["listmode"] = lm
    del obj
    # Gibbs Relative Difference penalty gradient on the image
    shape = (img.nz, img.ny, img.nx)
    vox = img.voxel_size
    p = gibbs.GibbsRelativeDifferencePenalty(penalisation_factor=0.1, gamma=2.0, epsilon=1e-7, device=proj.device)
    p.set_up(shape, vox, _abi.LAYOUT_DEVICE)
    gg = proj.empty_image(zero=False)
    ms = time_dev(lambda: p.compute_gradient(xd, gg))
    nvox = int(np.prod(shape))
    hbm, peak_kind = peaks()
    pr = {"metric": "Gibbs RDP gradient voxels/s", "value": nvox / (ms / 1e3), "unit": "voxels/s", "ms": ms,
          "workload": "GibbsRelativeDifferencePenalty (gamma 2, epsilon 1e-7) gradient, 3x3x3 default weights, "
                      "344x344x127 image in the device layout",
          "roofline": {"bound": "issue", "hbm_bytes": 8 * nvox, "achieved_GBs": 8 * nvox / (ms / 1e3) / 1e9,
                       "peak": hbm, "frac_hbm": 8 * nvox / (ms / 1e3) / 1e9 / hbm, "peak_kind": peak_kind}}
    if cpu_ref is not None:
        from oracle import oracle as O
        slab = np.ascontiguousarray(cpu_ref.x[:16])
        w = O.gibbs_default_weights(vox)
        t0 = time.perf_counter()
        O.gibbs("gradient", 2, 0.1, w, slab, gamma=2.0, epsilon=1e-7)
        dt = time.perf_counter() - t0
        pr["cpu_baseline"] = {"value": slab.size / dt, "unit": "voxels/s", "cores": 1, "kind": "port",
                              "sample": "16 planes of the image, the oracle's GibbsPenalty::compute_gradient loop"}
    pr["reference_cuda"] = reference_cuda_priors(p, shape, vox, proj.device)
    out["gibbs_rdp_gradient"] = pr
    del p
    torch.cuda.empty_cache()
    out["tof"] = tof_workload(cpu_ref is not None, proj.device)
    return out


def reference_cuda_priors(p_dev_layout, shape, vox, device):
    """The same gradient by STIR's own CUDA kernels built for this GPU (oracle/_ref: CudaGibbsPenalty's gradient
    kernel with the Relative Difference potential, and CudaRelativeDifferencePrior's), against the B200 kernels in
    both arithmetics, all on one device image in STIR's [z][y][x] order (the reference's layout), no host copies.
    A baseline leg: the reference's kernels are timed, not used."""
    import ctypes
    import torch
    from oracle import oracle as O
    from stir_b200 import _abi, gibbs
    if not O.ref_cuda_priors_available():
        return {"unavailable": "STIR's CUDA prior kernels were not built (oracle/_ref needs the STIR sources)"}
    ref = O.ref_cuda_priors()
    g = torch.Generator(device=f"cuda:{device}").manual_seed(9)
    x = torch.rand(shape, device=f"cuda:{device}", generator=g) + 0.1
    out = torch.empty_like(x)
    w = torch.from_numpy(np.ascontiguousarray(O.gibbs_default_weights(vox), np.float32)).to(x.device)
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    nz, ny, nx = shape
    args = (ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(w.data_ptr()))
    ms_gibbs = time_dev(lambda: ref.ref_cuda_gibbs_gradient(1, *args, 3, 3, 3, None, 0.1, 2.0, 1e-7, nz, ny, nx,
                                                            -(ny // 2), -(nx // 2), sp))
    ref_out = out.clone()
    ms_rdp = time_dev(lambda: ref.ref_cuda_rdp_prior_gradient(*args, None, 2.0, 1e-7, 0.1, nz, ny, nx, sp))
    res = {"layout": "[z][y][x]", "stir_CudaGibbsPenalty_gradient_ms": ms_gibbs,
           "stir_CudaRelativeDifferencePrior_gradient_ms": ms_rdp}
    for name, cls in (("b200_cuda_arithmetic", gibbs.CudaGibbsRelativeDifferencePenalty),
                      ("b200_host_arithmetic", gibbs.GibbsRelativeDifferencePenalty)):
        q = cls(penalisation_factor=0.1, gamma=2.0, epsilon=1e-7, device=device)
        q.set_up(shape, vox, _abi.LAYOUT_STIR)
        ms = time_dev(lambda: q.compute_gradient(x, out))
        res[name + "_ms"] = ms
        if name == "b200_cuda_arithmetic":
            res["b200_cuda_arithmetic_bit_equal_to_stir_cuda"] = bool(torch.equal(out, ref_out))
        del q
    res["speedup_vs_stir_CudaGibbsPenalty"] = ms_gibbs / res["b200_cuda_arithmetic_ms"]
    res["speedup_vs_stir_CudaRelativeDifferencePrior"] = ms_rdp / res["b200_host_arithmetic_ms"]
    return res


def autograd_workload(device, batch=8):
    """The differentiable projector's workload: a batch of 8 seeded smooth fields of 172x172x127 on the clinical
    scanner (zoom 0.5), loss = Poisson log-likelihood (attenuation, 10 % background) + RelativeDifferencePrior (beta
    0.1, gamma 2); one step = the loss's value and its gradient by torch.autograd (forward and back projections of the
    batch, one launch per direction), against the same with one launch per image."""
    import torch
    from stir_b200 import geometry as G
    from stir_b200 import phantoms, workloads
    from stir_b200.autograd import PoissonLogLikelihood, Prior
    from stir_b200.osmaposl import RelativeDifferencePrior
    from stir_b200.projectors import RayTracingProjector
    proj = RayTracingProjector(*G.clinical_3d_pet_half(), device=device)
    imgs = [phantoms.smooth_random_field(proj.image, sigma_vox=3.0, seed=10 + k) for k in range(batch)]
    x = torch.stack([proj.image_to_device_layout(torch.from_numpy(a).cuda(device)) for a in imgs])
    mu = phantoms.attenuation_cylinder(proj.image, radius_mm=150.0, mu_per_mm=0.0096)
    m = workloads._attenuation_factors(proj, mu)
    ys, adds = [], []
    for k in range(batch):
        ybar = m * proj.forward_dev(x[k])
        b = 0.1 * float(ybar.double().mean())
        yk, _ = workloads._poisson(ybar + b, 3e7, 100 + k)
        ys.append(yk)
        adds.append(torch.full_like(yk, b) / m)
    y, add = torch.stack(ys), torch.stack(adds)
    R = Prior(proj, RelativeDifferencePrior(0.1, gamma=2.0, epsilon=0.0))
    L = PoissonLogLikelihood(proj, y, add, m)  # keeps the gradient ratios of its projection when they fit (they do)
    L_rc = PoissonLogLikelihood(proj, y, add, m, store_ratio=False)  # projects again in backward
    singles = [PoissonLogLikelihood(proj, y[k], add[k], m) for k in range(batch)]

    def batched(obj=L):
        xg = x.detach().requires_grad_(True)
        loss = -(obj(xg) - R(xg))
        loss.backward()
        return float(loss)

    def one_by_one():
        total = 0.0
        for k in range(batch):
            xg = x[k].detach().requires_grad_(True)
            loss = -(singles[k](xg) - R(xg))
            loss.backward()
            total += float(loss)
        return total

    ms_b = time_dev(batched, warm=2, reps=5)
    ms_rc = time_dev(lambda: batched(L_rc), warm=2, reps=5)
    ms_1 = time_dev(one_by_one, warm=2, reps=5)
    v_b, v_1 = batched(), one_by_one()
    res = {"metric": "differentiable projector loss+gradient steps/s", "value": 1e3 / ms_b, "unit": "steps/s",
           "ms_per_step": ms_b, "images_per_s": batch * 1e3 / ms_b, "one_launch_per_image_ms": ms_1,
           "speedup_vs_one_launch_per_image": ms_1 / ms_b, "batch": batch,
           "recompute_in_backward_ms": ms_rc, "speedup_vs_recompute_in_backward": ms_rc / ms_b,
           "loss_rel_diff_vs_one_by_one": abs(v_b - v_1) / abs(v_1),
           "workload": "8 x 172x172x127 smooth fields (sigma 3 voxels, seeds 10..17) on the clinical scanner at zoom 0.5; "
                       "loss -log-likelihood (3e7 counts each, attenuation, 10 % background) + RDP beta 0.1; value "
                       "and gradient by torch.autograd, one projection per step (its gradient ratios kept for backward, "
                       "8 x 290 MB) against projecting again in backward; wall clock around CUDA events: the value is "
                       "read on the host"}
    proj.close()
    del proj, x, y, add, m
    torch.cuda.empty_cache()
    return res


def tof_batched_reconstructions(proj, frames=4, nsub=21, iterations=3, beta=0.5):
    """The TOF configuration's reconstructions: `frames` noise realisations (seeds 0..), OSMAPOSL with a
    QuadraticPrior (beta 0.5, 3x3x3 neighbourhood), 21 subsets x 3 iterations, batched in one graph against one
    at a time.  With beta 0.5 the one-step-late update amplifies float-rounding differences, so the two differ by
    far more than rounding after 63 sub-iterations (reported, not a parity check)."""
    import torch
    from stir_b200 import phantoms
    from stir_b200.batch import BatchedOSMAPOSL
    from stir_b200.osmaposl import OSMAPOSLReconstruction, QuadraticPrior
    xt = phantoms.cylinder_with_spheres(proj.image, radius_mm=90.0, n_spheres=2, sphere_radius=(10.0, 10.0), seed=3)
    ybar = proj.forward_dev(proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(xt, np.float32)).cuda()))
    bg = float(0.1 * ybar.mean())
    data = []
    for k in range(frames):
        g = torch.Generator(device=ybar.device).manual_seed(k)
        scale = 3e8 / float((ybar + bg).sum())
        y = torch.poisson((ybar + bg) * scale, generator=g) / scale
        data.append((y, torch.full_like(y, bg)))
    n = nsub * iterations
    objs = [OSMAPOSLReconstruction(proj, y, additive=a, num_subsets=nsub, num_subiterations=n,
                                   prior=QuadraticPrior(beta), use_tofsens=True).set_up() for y, a in data]
    xs = [proj.empty_image() for _ in objs]

    def per_frame():
        for r, x in zip(objs, xs):
            x.fill_(1.0)
            r.reconstruct(x)

    per_frame()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    per_frame()
    torch.cuda.synchronize()
    t_pf = time.perf_counter() - t0
    batch = BatchedOSMAPOSL()
    bx = []
    for (y, a), r0 in zip(data, objs):
        r = OSMAPOSLReconstruction(proj, y, additive=a, num_subsets=nsub, num_subiterations=n, prior=QuadraticPrior(beta),
                                   use_tofsens=True)
        r.sensitivities = r0.sensitivities
        x = proj.empty_image().fill_(1.0)
        batch.add(r, x)
        bx.append(x)
    batch.reconstruct(use_graph=True)  # captures the graph
    for x in bx:
        x.fill_(1.0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch.reconstruct(use_graph=True)
    torch.cuda.synchronize()
    t_b = time.perf_counter() - t0
    batch.close()
    return {"metric": "batched TOF OSMAPOSL reconstructions/s", "value": frames / t_b, "unit": "reconstructions/s",
            "per_frame_value": frames / t_pf, "speedup_vs_per_frame": t_pf / t_b, "frames": frames,
            "subsets": nsub, "sub_iterations": n, "prior": f"QuadraticPrior beta {beta}",
            "workload": "noise realisations (torch Poisson, seeds 0..3, 3e8 counts) of a cylinder with 2 spheres, "
                        "additive background 10 %; wall clock with a device synchronisation on both sides"}


def tof_workload(with_cpu, device):
    """TOF forward + back projection (per-basic-bin kernels with the TOF rows) on the 8-ring scanner with 33 timing
    bins of 50 ps and a 550 ps FWHM kernel (19.5M TOF bins), against the oracle on one subset."""
    import torch
    from stir_b200 import geometry as G
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet()
    t0 = time.perf_counter()
    proj = RayTracingProjector(pdi, img, device=device)
    setup_s = time.perf_counter() - t0
    try:
        n = proj.projdata_size
        x = torch.rand(img.nz * img.ny * img.nx, device=f"cuda:{device}") + 0.5
        pd = proj.empty_projdata()
        y = torch.rand(n, device=f"cuda:{device}") + 0.5
        bk = proj.empty_image(zero=False)
        fms = time_dev(lambda: proj.forward_dev(x, pd))
        bms = time_dev(lambda: proj.back_dev(y, bk))
        res = {"metric": "TOF fwd+back TOF-bin LORs/s", "value": n / ((fms + bms) / 1e3), "unit": "LORs/s",
               "tof_bins_per_step": n, "forward_ms": fms, "back_ms": bms, "setup_s": setup_s, "gpu_launches": 2,
               "workload": "8 rings x 288 det (R 300 mm), span 1, 144 views x 64 tang, 33 timing bins of 50 ps, "
                           "Gaussian 550 ps FWHM (STIR's kernel cut-off), image 64x64x15; TOF-grouped kernels",
               "row_elements": int(proj.info.total_nnz)}
        # the same with the Gaussian truncated at +-3 sigma (the kernel of the TOF configuration) beside STIR's cut-off
        p3 = RayTracingProjector(pdi, img, device=device, tof_kernel_truncation_sigmas=3.0)
        try:
            f3 = time_dev(lambda: p3.forward_dev(x, pd))
            b3 = time_dev(lambda: p3.back_dev(y, bk))
            res["truncated_3_sigma"] = {"value": n / ((f3 + b3) / 1e3), "unit": "LORs/s", "forward_ms": f3,
                                        "back_ms": b3, "row_elements": int(p3.info.total_nnz),
                                        "kernel": "Gaussian truncated at +-3 sigma, bins integrate its inner part"}
        finally:
            p3.close()
        res["batched"] = tof_batched_reconstructions(proj)
        if with_cpu:
            from oracle.oracle import Oracle
            orc = Oracle(proj.geometry)
            xs = np.random.default_rng(2).uniform(0.5, 1.5, (img.nz, img.ny, img.nx)).astype(np.float32)
            nth = os.cpu_count() or 1
            orc.forward(xs, 0, 24, nth)  # fills the subset's TOF rows
            ys = np.random.default_rng(3).uniform(0.5, 1.5, n).astype(np.float32)
            t0 = time.perf_counter()
            orc.forward(xs, 0, 24, nth)
            orc.back(ys, 0, 24, nth)
            dt = time.perf_counter() - t0
            nsb = subset_num_bins(pdi, proj.geometry, orc.symmetries_used, 0, 24) * proj.info.num_tof_bins
            res["cpu_baseline"] = {"value": nsb / dt, "unit": "LORs/s", "cores": nth, "kind": "port",
                                   "sample": "forward+back of subset 0 of 24 (warm TOF row cache), OpenMP"}
        return res
    finally:
        proj.close()


def split_measure(pdi, img, x_host, rank, ws, local, dist, steps, warmup):
    """The clinical workload's forward + back projection split across the ranks: rank r holds the projection data
    of the views of subset r of ws (a view shard: 1/ws of the data) and projects them; the back projections are
    summed by an NCCL all-reduce of the image (the exchange of the multi-GPU reconstruction).  Returns the whole
    job's LORs/s over the slowest rank's device time."""
    import torch
    from stir_b200.distributed import rank_subset, rank_views, shard_projdata
    from stir_b200.projectors import RayTracingProjector
    dev = torch.device("cuda", local)
    proj = RayTracingProjector(pdi, img, device=local)
    nbins = proj.projdata_size
    xd = proj.image_to_device_layout(torch.from_numpy(x_host).to(dev))
    y_full = proj.forward_dev(xd)
    y_full.add_(0.3 * float(y_full.mean()))
    views = rank_views(proj.geometry, 1, rank, ws, proj.info.symmetries_used)
    y = shard_projdata(pdi, y_full, views)
    del y_full
    proj.set_view_shard(views)
    sub, nsub = rank_subset(0, 1, rank, ws)
    pd = proj.empty_projdata()
    bk = proj.empty_image()
    flush = torch.empty(128 * 1024 * 1024, dtype=torch.float32, device=dev)

    def step():
        proj.forward_dev(xd, out=pd, subset_num=sub, num_subsets=nsub)
        proj.back_dev(y, out=bk, subset_num=sub, num_subsets=nsub)
        if dist:
            dist.all_reduce(bk)

    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ar = []
    e0.record()
    for k in range(steps):
        flush.fill_(float(k))
        step()
    e1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # the all-reduce alone, for the record
    if dist:
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(5):
            dist.all_reduce(bk)
        a1.record()
        torch.cuda.synchronize()
        ar.append(a0.elapsed_time(a1) / 5)
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item()) / steps
    res = {"value": nbins / (ms / 1e3), "unit": "LORs/s", "ms_per_step": ms, "scaling": "strong",
           "views_per_rank": len(views), "projdata_bytes_per_rank": 4 * proj.projdata_size,
           "allreduce_ms": ar[0] if ar else 0.0, "image_bytes": 4 * img.nz * img.ny * img.nx,
           "workload": "forward + back projection of all 72.6 M LORs split by views (view shards), NCCL all-reduce "
                       "of the back projection every step"}
    proj.close()
    del pd, bk, flush, y, xd
    torch.cuda.empty_cache()
    return res


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    import datetime
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, ws, local, dist


def reference_main(args):
    rank, ws, local, dist = dist_setup()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cb = CpuBaseline()
    for _ in range(max(0, args.warmup)):
        cb.step()
    times = [cb.step() for _ in range(max(1, args.steps))]
    sec = float(np.mean(times))
    desc = cb.describe(sec)
    v = desc["value"]
    line = {"metric": METRIC, "value": v, "unit": "LORs/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "sample": desc["sample"]},
            "cpu_baseline": desc,
            "e2e": {"value": v, "unit": "LORs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def profile_value(key, kernel_name):
    """`key[kernel_name]: value` from the committed ncu summaries (profiles/), or None."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        try:
            txt = open(path).read()
        except OSError:
            continue
        m = re.search(r"^" + re.escape(key) + r"\[" + re.escape(kernel_name) + r"\]:\s*([0-9.eE+]+)", txt, re.M)
        if m:
            return float(m.group(1))
    return None


def _ratio(nbytes, ms):
    """GB/s of nbytes moved in ms, or None without a byte count"""
    return None if nbytes is None else nbytes / (ms / 1e3) / 1e9


def profile_traffic(kernel_name):
    """DRAM bytes per launch of `kernel_name` from the committed ncu summary (profiles/), or None."""
    return profile_value("traffic_per_launch", kernel_name)


BATCH_WORKLOAD = ("dynamic OSEM: 24 frames on the clinical scanner, 16 at 344x344x127 and 8 at 172x172x127 "
                  "(4.18 mm), counts log-uniform in [1e6, 5e7] (seed 3), 3-region kinetic phantom, 7 or 21 subsets "
                  "per frame (seeded), additive background 10 %")


def batched_dynamic(local, iterations):
    """Dynamic frames reconstructed together (one persistent forward and back launch per batched
    sub-iteration, the whole reconstruction in one CUDA graph) and one at a time (OSMAPOSL per frame)."""
    import torch

    from stir_b200 import geometry as G
    from stir_b200 import phantoms
    from stir_b200.batch import BatchedOSMAPOSL
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    from stir_b200.projectors import RayTracingProjector

    dev = torch.device("cuda", local)
    geoms = {344: G.clinical_3d_pet(), 172: G.clinical_3d_pet_half()}
    projs = {n: RayTracingProjector(*geoms[n], device=local) for n in geoms}
    rng = np.random.default_rng(3)
    counts = np.exp(rng.uniform(np.log(1e6), np.log(5e7), 24))
    nsubs = rng.choice([7, 21], 24)
    sizes = [344] * 16 + [172] * 8
    tac = phantoms.time_activity(np.geomspace(0.25, 60.0, 24))  # frame mid-times in minutes
    regions = {n: torch.from_numpy(phantoms.dynamic_regions(geoms[n][1])).to(dev) for n in geoms}
    gen = torch.Generator(device=dev)
    gen.manual_seed(3)
    frames = []
    for f in range(24):
        p = projs[sizes[f]]
        act = torch.tensordot(torch.tensor(tac[f], dtype=torch.float32, device=dev), regions[sizes[f]], dims=1)
        ybar = p.forward_dev(p.image_to_device_layout(act.contiguous()))
        bg = 0.1 * float(ybar.mean())
        scale = float(counts[f]) / (float(ybar.sum()) + bg * ybar.numel())
        y = torch.poisson((ybar + bg) * scale, generator=gen).div_(scale)
        del ybar
        frames.append(dict(size=sizes[f], nsub=int(nsubs[f]), y=y, add=torch.full_like(y, bg)))
    sens = {}
    for fr in frames:
        key = (fr["size"], fr["nsub"])
        if key not in sens:
            sens[key] = OSMAPOSLReconstruction(projs[fr["size"]], fr["y"], num_subsets=fr["nsub"]).set_up().sensitivities

    def recon(fr):
        r = OSMAPOSLReconstruction(projs[fr["size"]], fr["y"], additive=fr["add"], num_subsets=fr["nsub"],
                                   num_subiterations=iterations * fr["nsub"])
        r.sensitivities = sens[(fr["size"], fr["nsub"])]
        return r

    recs = [recon(fr) for fr in frames]
    x_one = [projs[fr["size"]].empty_image().fill_(1.0) for fr in frames]
    for r, fr in zip(recs, frames):  # warm-up: scratch buffers and subset lists of every frame kind
        r.update_estimate(projs[fr["size"]].empty_image().fill_(1.0))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for r, x in zip(recs, x_one):
        r.reconstruct(x)
    e1.record()
    torch.cuda.synchronize()
    one_ms = e0.elapsed_time(e1)

    batch = BatchedOSMAPOSL(local)
    x_b = [projs[fr["size"]].empty_image().fill_(1.0) for fr in frames]
    for fr, x in zip(frames, x_b):
        batch.add(recon(fr), x)
    t0 = time.perf_counter()
    cfg = batch.autotune(1)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    batch.reconstruct(use_graph=True)  # captures the graph of the whole reconstruction, then runs it
    torch.cuda.synchronize()
    capture_and_run_s = time.perf_counter() - t0
    for x in x_b:
        x.fill_(1.0)
    torch.cuda.synchronize()
    e0.record()
    batch.reconstruct(use_graph=True)
    e1.record()
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1)
    err = max(float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))
              for a, b in zip(x_b, x_one))
    nsub_max = max(fr["nsub"] for fr in frames)
    # per batched sub-iteration: the forward and back projections and the three update launches; once per
    # run: one threshold launch per frame
    launches = 5 * iterations * nsub_max + len(frames)
    batch.close()
    for p in projs.values():
        p.close()
    return {"metric": "batched dynamic OSEM frames/s", "workload": BATCH_WORKLOAD, "frames": 24,
            "iterations_per_frame": iterations, "value": 24 / (batch_ms / 1e3), "unit": "frames/s",
            "ms": batch_ms, "per_frame_value": 24 / (one_ms / 1e3), "per_frame_ms": one_ms,
            "speedup_vs_per_frame": one_ms / batch_ms, "max_rel_l2_vs_per_frame": err, "config": cfg,
            "autotune_s": tune_s, "graph_capture_and_first_run_s": capture_and_run_s,
            "gpu_launches": launches, "batched_sub_iterations": iterations * nsub_max}


def b200_main(args):
    import ctypes

    import torch

    from stir_b200 import _abi
    from stir_b200 import geometry as G
    from stir_b200 import phantoms
    from stir_b200.projectors import RayTracingProjector

    rank, ws, local, dist = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pdi, img = G.clinical_3d_pet()
    t0 = time.perf_counter()
    proj = RayTracingProjector(pdi, img, device=local)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    nbins = proj.projdata_size
    nnz = proj.info.total_nnz

    # seeded phantom per rank (an independent frame per GPU), resident in HBM
    x = phantoms.cylinder_with_spheres(img, n_spheres=6, sphere_radius=(5, 18), ellipse_axes=(150, 100), seed=1 + rank)
    xd = proj.image_to_device_layout(torch.from_numpy(x).to(dev))
    y = proj.forward_dev(xd)
    y.add_(0.3 * float(y.mean()))  # strictly positive data: the back projection skips no bin
    pd = proj.empty_projdata()
    bk = proj.empty_image()
    flush = torch.empty(128 * 1024 * 1024, dtype=torch.float32, device=dev)  # 512 MiB > 126 MB L2

    def step():
        proj.forward_dev(xd, out=pd)
        proj.back_dev(y, out=bk)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        e_start.record()
        for k in range(K):
            flush.fill_(float(k))
            ev[k][0].record()
            proj.forward_dev(xd, out=pd)
            ev[k][1].record()
            proj.back_dev(y, out=bk)
            ev[k][2].record()
        e_end.record()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = e_start.elapsed_time(e_end)
    fwd_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in ev]))
    back_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in ev]))
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    ms_per_step = max_ms / K
    value = nbins * ws / (ms_per_step / 1e3)

    # end to end through the C ABI with host buffers (pinned), copies inside the timed region
    x_pin = torch.from_numpy(x).pin_memory()
    pd_pin = torch.empty(nbins, dtype=torch.float32).pin_memory()
    y_pin = proj.projdata_from_device_layout(y).cpu().pin_memory()
    img_pin = torch.empty(img.shape, dtype=torch.float32).pin_memory()
    lib = proj.lib

    def e2e_step():
        _abi.check(lib.b200rt_forward_project(proj.h, ctypes.c_void_p(x_pin.data_ptr()), ctypes.c_void_p(pd_pin.data_ptr()),
                                              0, 1), proj.h, "b200rt_forward_project")
        _abi.check(lib.b200rt_back_project(proj.h, ctypes.c_void_p(y_pin.data_ptr()), ctypes.c_void_p(img_pin.data_ptr()),
                                           0, 1, _abi.BACKPROJECT_ATOMIC), proj.h, "b200rt_back_project")

    e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ke = max(2, min(K, 5))
    t0 = time.perf_counter()
    for _ in range(ke):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / ke
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = nbins * ws / float(te.item())
    img_bytes = 4 * img.nz * img.ny * img.nx
    pd_bytes = 4 * nbins

    hbm, peak_kind = peaks()
    fwd_bytes = 4.0 * nnz + 4.0 * nbins
    back_bytes = 8.0 * nnz + 4.0 * nbins
    if fwd_ms >= back_ms:
        kname, kms, kbytes = FWD_KERNEL, fwd_ms, fwd_bytes
    else:
        kname, kms, kbytes = BACK_KERNEL, back_ms, back_bytes
    achieved = kbytes / (kms / 1e3) / 1e9
    roof = {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": profile_traffic(kname),
            "algorithmic_bytes_per_launch": kbytes,
            "kernels_ms": {FWD_KERNEL: fwd_ms, BACK_KERNEL: back_ms},
            "frac_forward": fwd_bytes / (fwd_ms / 1e3) / 1e9 / hbm, "frac_back": back_bytes / (back_ms / 1e3) / 1e9 / hbm,
            # the unit that does bound these kernels (the image stays in L2, DRAM moves < 1 GB per launch): the SM's
            # shared-memory data path, as a fraction of its peak wavefront rate, from the committed ncu summaries
            "limiter": {"unit": "shared-memory wavefronts (l1tex data pipe)",
                        "frac_forward": profile_value("smem_wavefront_frac", FWD_KERNEL),
                        "frac_back": profile_value("smem_wavefront_frac", BACK_KERNEL),
                        "issue_active_forward": profile_value("issue_active_frac", FWD_KERNEL),
                        "issue_active_back": profile_value("issue_active_frac", BACK_KERNEL)},
            # compulsory traffic: the image and the projection data once each way (forward reads the image and
            # writes the bins, back reads the bins and writes the image), against the same copy bandwidth
            "compulsory": {"bytes_forward": img_bytes + pd_bytes, "bytes_back": pd_bytes + img_bytes,
                           "frac_forward": (img_bytes + pd_bytes) / (fwd_ms / 1e3) / 1e9 / hbm,
                           "frac_back": (pd_bytes + img_bytes) / (back_ms / 1e3) / 1e9 / hbm},
            # DRAM bytes per launch (committed ncu summaries) over the live kernel time, and the L2 hit rate there
            "dram_GBs": {FWD_KERNEL: _ratio(profile_traffic(FWD_KERNEL), fwd_ms),
                         BACK_KERNEL: _ratio(profile_traffic(BACK_KERNEL), back_ms)},
            "l2_hit_rate": {FWD_KERNEL: profile_value("l2_hit_rate", FWD_KERNEL),
                            BACK_KERNEL: profile_value("l2_hit_rate", BACK_KERNEL)}}

    roof["byte_model"] = ("algorithmic bytes: every (row element, LOR) pair counted as a 4-byte image read "
                          "(forward) or an 8-byte read-modify-write (back); the column staging serves them from shared "
                          "memory and L2, so frac above 1 says the kernel avoids DRAM, not that it beats the copy "
                          "bandwidth; the compulsory-bytes fractions (image and projection data once) and the on-chip "
                          "limiter (ncu) say where the time goes")

    # the deterministic back projection (64-bit fixed point, order-independent) on the same data, beside the atomic one
    bk2 = proj.empty_image()
    proj.back_dev(y, out=bk2, mode=_abi.BACKPROJECT_DETERMINISTIC)
    det_ms = time_dev(lambda: proj.back_dev(y, out=bk2, mode=_abi.BACKPROJECT_DETERMINISTIC), warm=1, reps=3)
    bk3 = proj.back_dev(y, mode=_abi.BACKPROJECT_DETERMINISTIC)
    deterministic = {"back_ms": det_ms, "atomic_back_ms": back_ms, "bit_identical_across_runs": bool(torch.equal(bk2, bk3)),
                     "rel_l2_vs_atomic": float((bk2 - bk).double().norm() / bk.double().norm()),
                     "method": "each item's contributions to a voxel summed in float in a fixed order, the sum rounded "
                               "to a 64-bit fixed-point integer (scale from the data's bound and the largest column "
                               "sum), integers added atomically, converted once"}
    del bk2, bk3

    cpu = None
    cb = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cb = CpuBaseline()
            cpu = cb.describe(cb.step())
        except Exception as e:  # the baseline is reported, never the measured product
            cb = None
            cpu = {"value": None, "unit": "LORs/s", "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {e}"}

    line = {"metric": METRIC, "value": value, "unit": "LORs/s", "n_gpus": ws, "steps": K, "warmup": max(args.warmup, 3),
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "lors_per_step_per_gpu": nbins, "nnz_per_step_per_gpu": nnz,
                       "parallelism": f"replicas{ws}" if ws > 1 else "single",
                       "l2": "512 MiB buffer written between steps; projection data 290 MB > L2",
                       "setup_s": setup_s, "back_projection": "atomic"},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "LORs/s", "h2d_bytes_per_step": img_bytes + pd_bytes,
                    "d2h_bytes_per_step": pd_bytes + img_bytes},
            "clocks": clocks.summary(),
            "gpu_launches": 2 * K,
            "deterministic": deterministic}
    # the secondary workloads and the batched reconstructions are measured on one GPU only (the scaling runs
    # hold every GPU of the node; they report the headline alone)
    if ws > 1 or args.mode == "split":
        # the split of one reconstruction's projections across the GPUs (all ranks take part)
        split = split_measure(pdi, img, x, rank, ws, local, dist, K, args.warmup)
        if args.mode == "split":
            line.update(value=split["value"], ms_per_step=split["ms_per_step"], scaling="strong")
            line["config"]["parallelism"] = f"view split over {ws} GPU(s), NCCL all-reduce of the back projection"
        line["split"] = split
    if not args.no_extras and ws == 1:
        try:
            line.update(listmode_and_priors(proj, pdi, img, xd, cb))
        except Exception as e:  # reported, never hides the headline line
            line["listmode"] = {"error": f"{type(e).__name__}: {e}"}
    if not args.no_extras and ws == 1:
        try:
            line["autograd"] = autograd_workload(local)
        except Exception as e:  # reported, never hides the headline line
            line["autograd"] = {"error": f"{type(e).__name__}: {e}"}
    if not args.no_batch and ws == 1:
        proj.close()
        del pd, bk, flush, y, xd
        torch.cuda.empty_cache()
        try:
            line["batched"] = batched_dynamic(local, args.batch_iterations)
        except Exception as e:  # reported, never hides the headline line
            line["batched"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    proj.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        reference_main(a)
    else:
        b200_main(a)
