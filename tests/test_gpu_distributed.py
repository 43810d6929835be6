"""The multi-GPU OSMAPOSL driver on the GPU through NCCL with one rank: the subset split, the all-reduce of the
numerators and the identical update reduce to single-GPU OSMAPOSL."""
import datetime
import socket

import numpy as np
import pytest

from stir_b200 import geometry as G
from stir_b200 import phantoms

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_nccl_single_rank_matches_osmaposl(cuda_device):
    import torch
    import torch.distributed as dist
    from stir_b200.distributed import B200Backend, DistributedOSMAPOSL
    from stir_b200.osmaposl import OSMAPOSLReconstruction
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    xt = proj.image_to_device_layout(torch.from_numpy(phantoms.cylinder_with_spheres(img, seed=1)).cuda())
    y = proj.forward_dev(xt).add_(0.5)
    add = torch.full_like(y, 0.05)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rec = DistributedOSMAPOSL(B200Backend(proj, y, add), num_subsets=6, num_subiterations=4)
        x = rec.reconstruct(proj.empty_image().fill_(1.0))
        ll = rec.log_likelihood(x, 1, 6)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    ref = OSMAPOSLReconstruction(proj, y, additive=add, num_subsets=6, num_subiterations=4)
    xr = ref.reconstruct(proj.empty_image().fill_(1.0))
    a, b = x.cpu().numpy().astype(np.float64), xr.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5
    from stir_b200.osmaposl import log_likelihood
    llr = log_likelihood(proj, xr, y, add, None, 1, 6)
    assert abs(ll - llr) <= 1e-6 * abs(llr)


def test_view_shards_sum_to_the_whole_data(cuda_device):
    """Two view shards (the data of ranks 0 and 1 of 2) on one GPU: their sensitivities, OSMAPOSL numerators of the
    split subsets and log-likelihoods sum to the whole data's, and each holds its share of the data only."""
    import numpy as np
    import torch
    from stir_b200 import geometry as G
    from stir_b200 import phantoms
    from stir_b200.distributed import B200Backend, rank_subset, rank_views, shard_projdata
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    full = RayTracingProjector(pdi, img, device=cuda_device)
    xt = full.image_to_device_layout(torch.from_numpy(phantoms.cylinder_with_spheres(img, seed=1)).cuda())
    y = torch.poisson(full.forward_dev(xt) * 5 + 1) / 5
    add = torch.full_like(y, 0.2)
    mult = torch.from_numpy(np.random.default_rng(3).uniform(0.8, 1.2, full.projdata_size).astype(np.float32)).cuda()
    x = full.image_to_device_layout(torch.from_numpy(phantoms.smooth_random_field(img, 2.0, seed=4)).cuda())
    nsub, world = 6, 2
    whole = B200Backend(full, y, add, mult)
    shards = []
    for r in range(world):
        p = RayTracingProjector(pdi, img, device=cuda_device)
        views = rank_views(p.geometry, nsub, r, world, p.info.symmetries_used)
        p.set_view_shard(views)
        assert p.projdata_size == full.projdata_size * len(views) // pdi.num_views
        shards.append(B200Backend(p, shard_projdata(pdi, y, views), shard_projdata(pdi, add, views),
                                  shard_projdata(pdi, mult, views)))
    assert sum(b.proj.projdata_size for b in shards) == full.projdata_size

    def rel(a, b):
        return float((a - b).double().norm() / b.double().norm())
    for s in (0, 4):
        ref_u = whole.numerator(x, s, nsub)
        u = sum(b.numerator(x, *rank_subset(s, nsub, r, world)) for r, b in enumerate(shards))
        assert rel(u, ref_u) <= 1e-6
        ref_s = whole.sensitivity(s, nsub)
        sens = sum(b.sensitivity(*rank_subset(s, nsub, r, world)) for r, b in enumerate(shards))
        assert rel(sens, ref_s) <= 1e-6
        ref_l = whole.log_likelihood(x, s, nsub)
        ll = sum(b.log_likelihood(x, *rank_subset(s, nsub, r, world)) for r, b in enumerate(shards))
        assert abs(ll - ref_l) <= 1e-9 * abs(ref_l)
    # the whole data's entry points refuse a shard
    import ctypes
    from stir_b200 import _abi
    st = shards[0].proj.lib.b200rt_projdata_to_device_layout(shards[0].proj.h, ctypes.c_void_p(y.data_ptr()),
                                                             ctypes.c_void_p(y.data_ptr()), None)
    assert st == _abi.ERR_STATE
