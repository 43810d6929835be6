"""Viewgram access to device-resident projection data (b200rt_get_viewgram / b200rt_set_viewgram) and the
viewgram API of the forward and back projector mirrors served from it, as STIR's GPU projector plug-ins serve
actual_forward_project / actual_back_project (ForwardProjectorByBinParallelproj.cxx:128-145,
BackProjectorByBinParallelproj.cxx:161-328)."""
import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G

pytestmark = pytest.mark.gpu


def stir_viewgram(pdi, pd, segment, view):
    """the viewgram of ProjDataInMemory-ordered data: segments 0, +1, -1, ..., each [axial][view][tangential]"""
    off = 0
    for s in pdi.segment_sequence:
        n = pdi.get_num_axial_poss(s) * pdi.num_views * pdi.num_tangential_poss
        if s == segment:
            block = pd[off:off + n].reshape(pdi.get_num_axial_poss(s), pdi.num_views, pdi.num_tangential_poss)
            return block[:, view, :]
        off += n
    raise ValueError(segment)


@pytest.fixture(scope="module")
def setup(cuda_device):
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    rng = np.random.default_rng(41)
    x = rng.uniform(0.2, 1.0, img.shape).astype(np.float32)
    return pdi, img, proj, x


def test_get_viewgram_matches_stir_order(setup):
    import torch
    pdi, img, proj, x = setup
    host = proj.forward_host(x)
    dev = proj.forward_dev(proj.image_to_device_layout(torch.from_numpy(x).cuda()))
    S = pdi.max_segment_num
    for seg in sorted({0, S, -S}):
        for view in (0, pdi.num_views // 3, pdi.num_views - 1):
            ref = stir_viewgram(pdi, host, seg, view)
            np.testing.assert_array_equal(proj.get_viewgram(dev, seg, view), ref)
            out = torch.empty(proj.viewgram_shape(seg), device="cuda")
            proj.get_viewgram(dev, seg, view, out=out)
            np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_set_viewgram_overwrites_and_accumulates(setup):
    import torch
    pdi, img, proj, x = setup
    pd = proj.empty_projdata()
    rng = np.random.default_rng(42)
    seg, view = -pdi.max_segment_num, 5
    v = rng.uniform(-1, 1, proj.viewgram_shape(seg)).astype(np.float32)
    proj.set_viewgram(pd, v, seg, view)
    np.testing.assert_array_equal(proj.get_viewgram(pd, seg, view), v)
    proj.set_viewgram(pd, torch.from_numpy(v).cuda(), seg, view, accumulate=True)
    np.testing.assert_array_equal(proj.get_viewgram(pd, seg, view), v + v)
    # only that viewgram changed
    stir = proj.projdata_from_device_layout(pd).cpu().numpy()
    assert np.count_nonzero(stir) == np.count_nonzero(v)
    np.testing.assert_array_equal(stir_viewgram(pdi, stir, seg, view), v + v)
    with pytest.raises(_abi.B200Error):
        proj.get_viewgram(pd, 0, pdi.num_views, 0)
    with pytest.raises(_abi.B200Error):
        proj.get_viewgram(pd, pdi.max_segment_num + 1, 0, 0, out=torch.empty(4, device="cuda"))
    with pytest.raises(_abi.B200Error):
        proj.set_viewgram(pd, torch.zeros(1, device="cuda"), 0, 0, timing_pos=1)


def test_projector_viewgram_api_matches_projdata_api(setup):
    from stir_b200.projectors import ProjectorByBinPairUsingB200RayTracing
    pdi, img, proj, x = setup
    pair = ProjectorByBinPairUsingB200RayTracing().set_up(pdi, img)
    fwd, back = pair.get_forward_projector_sptr(), pair.get_back_projector_sptr()
    fwd.set_input(x)
    full = np.zeros(fwd.get_projector().projdata_size, np.float32)
    fwd.forward_project(full)
    back.start_accumulating_in_new_target()
    for seg in pdi.segment_sequence:
        for view in range(pdi.num_views):
            v = fwd.forward_project_viewgram(seg, view)
            np.testing.assert_array_equal(v, stir_viewgram(pdi, full, seg, view))
            back.back_project_viewgram(v, seg, view)
    out = np.zeros(img.shape, np.float32)
    back.get_output(out)
    ref = np.zeros(img.shape, np.float32)
    back.back_project(ref, full)
    assert np.linalg.norm(out - ref) <= 1e-5 * np.linalg.norm(ref)
