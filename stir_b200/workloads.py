"""Seeded synthetic reconstruction inputs of the five workloads (no dataset is used).

Every function builds its data on the device with the given projectors and returns device-layout tensors in
STIR's model convention (PoissonLogLikelihoodWithLinearModelForMeanAndProjData): the mean of the data is
m * (A x + a), with m the multiplicative factors (normalisation times attenuation, norm.undo(1)) and a the
additive term already divided by m.  The OSMAPOSL numerator ignores m (it cancels); the sensitivity is A^T m.

  small_3d_pet_data    8 rings x 288 detectors, 64x64x15 image: water cylinder (r 100 mm) with two hot spheres
                       (r 10 mm, 4:1, seed 1), attenuation of the same cylinder (mu 0.0096 /mm) through the
                       projector, uniform background of 10 % of the mean, Poisson data with ~5e6 counts (seed 2)
  clinical_data        64 rings x 504 detectors, 344x344x127 image: elliptical body 300 x 200 mm with six hot
                       spheres (r 5-18 mm, 4:1), water attenuation, normalisation U[0.8, 1.2] times the
                       attenuation factors, a smooth additive background of 30 % of the mean, ~3e8 counts
  tof_data             the 8-ring scanner with 33 timing bins of 50 ps (550 ps FWHM): the small_3d_pet phantom
                       and attenuation, 10 % background per timing bin, ~3e8 counts; the non-TOF attenuation
                       factors for the sensitivity (STIR computes it with the non-TOF projector)
  dynamic_frames       24 frames on the clinical scanner (16 at 344x344x127, 8 at 172x172x127) of a 3-region
                       kinetic phantom, counts log-uniform in [1e6, 5e7] (seed 3), 7 or 21 subsets (seeded),
                       uniform background of 10 %
"""
from __future__ import annotations

import numpy as np

from . import phantoms


def _dev_img(proj, a):
    import torch
    return proj.image_to_device_layout(torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(f"cuda:{proj.device}"))


def _attenuation_factors(proj, mu):
    from .attenuation import BinNormalisationFromAttenuationImage
    return BinNormalisationFromAttenuationImage(proj, _dev_img(proj, mu)).factors()


def _poisson(mean, total, seed):
    """Poisson counts with about `total` events in all, returned in the units of `mean` (counts / scale), and
    the number of events."""
    import torch
    g = torch.Generator(device=mean.device)
    g.manual_seed(seed)
    scale = float(total) / float(mean.double().sum())
    n = torch.poisson(mean * scale, generator=g)
    events = float(n.double().sum())
    return n.div_(scale), events


def small_3d_pet_data(proj, counts=5e6):
    img = proj.image
    xt = phantoms.cylinder_with_spheres(img, radius_mm=100.0, n_spheres=2, sphere_radius=(10.0, 10.0), seed=1)
    mu = phantoms.attenuation_cylinder(img, radius_mm=100.0, mu_per_mm=0.0096)
    m = _attenuation_factors(proj, mu)
    ybar = m * proj.forward_dev(_dev_img(proj, xt))
    b = 0.1 * float(ybar.double().mean())
    y, events = _poisson(ybar + b, counts, 2)
    return dict(x_true=xt, mu=mu, y=y, additive=b / m, mult=m, events=events)


def clinical_data(proj, counts=3e8, seed=4):
    import torch
    img, pdi = proj.image, proj.proj_data_info
    rng = np.random.default_rng(seed)
    xt = phantoms.cylinder_with_spheres(img, n_spheres=6, sphere_radius=(5.0, 18.0), contrast=4.0, seed=seed,
                                        ellipse_axes=(150.0, 100.0))
    mu = phantoms.attenuation_cylinder(img, mu_per_mm=0.0096, ellipse_axes=(150.0, 100.0))
    acf = _attenuation_factors(proj, mu)
    norm = torch.from_numpy(rng.uniform(0.8, 1.2, proj.projdata_size).astype(np.float32)).to(acf.device)
    m = norm * acf
    del norm, acf
    ybar = m * proj.forward_dev(_dev_img(proj, xt))
    # smooth background: a Gaussian profile over the tangential position (sigma a third of the half-width),
    # constant over views and axial positions, scaled to 30 % of the mean of the data
    nt = pdi.num_tangential_poss
    t = np.arange(nt) - nt // 2
    w = torch.from_numpy(np.exp(-0.5 * (t / (nt / 6.0)) ** 2).astype(np.float32)).to(m.device)
    prof = _tangential_profile(proj, w)
    b = prof * (0.3 * float(ybar.double().mean()) / float(prof.double().mean()))
    y, events = _poisson(ybar + b, counts, seed + 1)
    del ybar
    return dict(x_true=xt, mu=mu, y=y, additive=b / m, mult=m, events=events)


def _tangential_profile(proj, w):
    """Device-layout projection data whose value depends on the tangential position only
    ([timing bin][segment][view][tangential][axial] blocks, axial fastest)."""
    import torch
    pdi = proj.proj_data_info
    parts = []
    S = pdi.max_segment_num
    for _tof in range(pdi.num_tof_bins):
        for seg in range(-S, S + 1):
            nax = pdi.get_num_axial_poss(seg)
            parts.append(w.view(1, -1, 1).expand(pdi.num_views, -1, nax).reshape(-1))
    out = torch.cat(parts)
    assert out.numel() == proj.projdata_size
    return out


def tof_data(proj, counts=3e8):
    """`proj` is a TOF projector; its non-TOF twin gives the attenuation factors."""
    img = proj.image
    nt = proj.non_tof_projector()
    xt = phantoms.cylinder_with_spheres(img, radius_mm=100.0, n_spheres=2, sphere_radius=(10.0, 10.0), seed=1)
    mu = phantoms.attenuation_cylinder(img, radius_mm=100.0, mu_per_mm=0.0096)
    m_nt = _attenuation_factors(nt, mu)
    ntof = proj.info.num_tof_bins
    assert m_nt.numel() * ntof == proj.projdata_size
    m = m_nt.repeat(ntof)  # every timing bin of a LOR has the LOR's attenuation
    ybar = m * proj.forward_dev(_dev_img(proj, xt))
    b = 0.1 * float(ybar.double().mean())
    y, events = _poisson(ybar + b, counts, 2)
    return dict(x_true=xt, mu=mu, y=y, additive=b / m, mult=m, sensitivity_mult=m_nt, events=events)


def dynamic_frames(projs, device, seed=3):
    """`projs` maps the image size (344, 172) to a projector on the clinical scanner.  Returns one dict per frame
    (24): size, nsub, y, additive (uniform background of 10 % of the mean), counts."""
    import torch
    dev = torch.device("cuda", device)
    rng = np.random.default_rng(seed)
    num_frames = 24
    counts = np.exp(rng.uniform(np.log(1e6), np.log(5e7), num_frames))
    nsubs = rng.choice([7, 21], num_frames)
    sizes = [344] * 16 + [172] * 8
    tac = phantoms.time_activity(np.geomspace(0.25, 60.0, num_frames))  # frame mid-times in minutes
    regions = {n: torch.from_numpy(phantoms.dynamic_regions(projs[n].image)).to(dev) for n in set(sizes)}
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    frames = []
    for f in range(num_frames):
        p = projs[sizes[f]]
        act = torch.tensordot(torch.tensor(tac[f], dtype=torch.float32, device=dev), regions[sizes[f]], dims=1)
        ybar = p.forward_dev(p.image_to_device_layout(act.contiguous()))
        bg = 0.1 * float(ybar.mean())
        scale = float(counts[f]) / (float(ybar.sum()) + bg * ybar.numel())
        y = torch.poisson((ybar + bg) * scale, generator=gen).div_(scale)
        del ybar
        frames.append(dict(size=sizes[f], nsub=int(nsubs[f]), y=y, additive=torch.full_like(y, bg),
                           counts=float(counts[f])))
    return frames
