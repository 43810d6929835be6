"""Attenuation factors on the GPU (BinNormalisationFromAttenuationImage) against the oracle's forward projection."""
import numpy as np
import pytest

from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_attenuation_factors_apply_undo(cuda_device, oracle_lib):
    import torch
    from stir_b200.attenuation import BinNormalisationFromAttenuationImage
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    mu = phantoms.attenuation_cylinder(img, radius_mm=100.0, mu_per_mm=0.0096)
    mu_dev = proj.image_to_device_layout(torch.from_numpy(mu).cuda())
    norm = BinNormalisationFromAttenuationImage(proj, mu_dev)
    # undo of ones: 1 / exp(A mu) with the line integrals of the oracle (STIR's float algorithm)
    li = orc.forward(mu)
    ref = (np.float32(1) / np.exp(li.astype(np.float32))).astype(np.float32)
    f = proj.projdata_from_device_layout(norm.factors()).cpu().numpy()
    assert rel_l2(f, ref) < 1e-5
    assert f.min() > 0 and f.max() <= 1
    # apply then undo returns the data; apply multiplies by the inverse factors
    rng = np.random.default_rng(4)
    y = rng.uniform(0.5, 2.0, proj.projdata_size).astype(np.float32)
    y_dev = proj.projdata_to_device_layout(torch.from_numpy(y).cuda())
    a = norm.apply(y_dev.clone())
    assert rel_l2(proj.projdata_from_device_layout(a).cpu().numpy(), y / ref) < 1e-5
    back = norm.undo(a)
    assert rel_l2(back.cpu().numpy(), y_dev.cpu().numpy()) < 1e-6


def test_attenuation_rejects_tof(cuda_device):
    import torch
    from stir_b200 import _abi
    from stir_b200.attenuation import BinNormalisationFromAttenuationImage
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=7, timing_bin_ps=250.0, num_views=48)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    mu_dev = proj.empty_image()
    with pytest.raises(_abi.B200Error, match="non_TOF"):
        BinNormalisationFromAttenuationImage(proj, mu_dev).factors()
