"""BinNormalisationFromProjData and ChainedBinNormalisation on the GPU (b200rt_normalisation_dev)."""
import numpy as np
import pytest

from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_projdata_and_chained_normalisation(cuda_device, oracle_lib):
    import torch
    from stir_b200.attenuation import BinNormalisationFromAttenuationImage
    from stir_b200.normalisation import BinNormalisationFromProjData, ChainedBinNormalisation
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    orc = oracle_lib.Oracle(proj.geometry)
    rng = np.random.default_rng(17)
    n = rng.uniform(0.8, 1.2, proj.projdata_size).astype(np.float32)  # correction factors, STIR order
    n_dev = proj.projdata_to_device_layout(torch.from_numpy(n).cuda())
    y = rng.uniform(0.5, 2.0, proj.projdata_size).astype(np.float32)
    y_dev = proj.projdata_to_device_layout(torch.from_numpy(y).cuda())
    norm = BinNormalisationFromProjData(proj, n_dev)
    host = lambda t: proj.projdata_from_device_layout(t).cpu().numpy()
    # apply multiplies, undo divides: bit for bit the float operations
    assert np.array_equal(host(norm.apply(y_dev.clone())), y * n)
    assert np.array_equal(host(norm.undo(y_dev.clone())), y / n)
    assert np.array_equal(host(norm.factors()), np.float32(1) / n)
    # chained with attenuation: apply = (y n) exp(A mu); undo = (y / n) / exp(A mu); factors = undo of ones
    mu = phantoms.attenuation_cylinder(img, radius_mm=100.0, mu_per_mm=0.0096)
    mu_dev = proj.image_to_device_layout(torch.from_numpy(mu).cuda())
    chain = ChainedBinNormalisation(norm, BinNormalisationFromAttenuationImage(proj, mu_dev))
    e = np.exp(orc.forward(mu).astype(np.float32))
    assert rel_l2(host(chain.apply(y_dev.clone())), (y * n) * e) < 1e-5
    assert rel_l2(host(chain.undo(y_dev.clone())), (y / n) / e) < 1e-5
    assert rel_l2(host(chain.factors()), (np.float32(1) / n) / e) < 1e-5
    # an empty chain leaves the data alone; factors are ones
    empty = ChainedBinNormalisation(None, None, projector=proj)
    assert torch.equal(empty.apply(y_dev.clone()), y_dev)
    assert bool((empty.factors() == 1).all())


def test_non_tof_factors_for_tof_data(cuda_device):
    """Non-TOF factors multiply every timing bin (BinNormalisationFromProjData.cxx:89-96)."""
    import torch
    from stir_b200.normalisation import BinNormalisationFromProjData
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=5, timing_bin_ps=250.0, num_views=48)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    ntof = proj.info.num_tof_bins
    per_tof = proj.projdata_size // ntof
    f = torch.rand(per_tof, device="cuda") + 0.5
    y = torch.rand(proj.projdata_size, device="cuda")
    out = BinNormalisationFromProjData(proj, f, non_tof=True).apply(y.clone())
    assert torch.equal(out, y * f.repeat(ntof))
