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
