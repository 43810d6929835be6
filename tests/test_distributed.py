"""Multi-rank logic on CPU (gloo, world size 2): subset splitting across ranks, all-reduce of the
numerators, identical updates; with the oracle as each rank's compute backend."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleBackend:
    """Per-rank compute on the CPU with the oracle (test stand-in for B200Backend)."""

    def __init__(self, orc, y, add):
        self.orc, self.y, self.add = orc, y, add

    def numerator(self, x, subset, nsub):
        return self.orc.osmaposl_numerator(x, self.y, self.add, subset, nsub)

    def apply(self, x, u, sens, nsub, it, prior=None, map_model=1, min_rel=0.0, max_rel=3.4e38):
        pa = None if prior is None else prior
        return self.orc.osmaposl_apply(x, u, sens, nsub, it, pa, min_rel=min_rel, max_rel=max_rel)

    def sensitivity(self, subset, nsub):
        return self.orc.sensitivity(None, subset, nsub)

    def log_likelihood(self, x, subset, nsub):
        return self.orc.log_likelihood(x, self.y, self.add, None, subset, nsub)


def _data():
    from oracle.oracle import Oracle
    from stir_b200 import geometry as G
    from stir_b200 import phantoms
    pdi, img = G.small_3d_pet()
    orc = Oracle(G.make_geometry(pdi, img))
    xt = phantoms.cylinder_with_spheres(img, seed=1)
    y = (np.random.default_rng(2).poisson(orc.forward(xt) * 10 + 1) / 10).astype(np.float32)
    add = np.full_like(y, 0.1)
    return orc, img, y, add


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from stir_b200.distributed import DistributedOSMAPOSL
        orc, img, y, add = _data()
        rec = DistributedOSMAPOSL(OracleBackend(orc, y, add), num_subsets=6, num_subiterations=3,
                                  to_tensor=lambda a: torch.from_numpy(np.ascontiguousarray(a)),
                                  from_tensor=lambda t, like: t.numpy().reshape(like.shape))
        x = rec.reconstruct(np.ones(img.shape, np.float32))
        ll = rec.log_likelihood(x, 1, 6)
        np.save(os.path.join(out_dir, f"x{rank}.npy"), x)
        np.save(os.path.join(out_dir, f"ll{rank}.npy"), np.array([ll]))
    finally:
        dist.destroy_process_group()


def test_split_subsets_cover_each_subset_once():
    from stir_b200.distributed import rank_subset, shard
    from stir_b200.subsets import basic_views_in_subset
    for nsub, world in [(6, 2), (7, 3), (21, 4)]:
        for s in range(nsub):
            parts = [basic_views_in_subset(144, 3, *rank_subset(s, nsub, r, world)) for r in range(world)]
            union = sorted(v for p in parts for v in p)
            assert union == basic_views_in_subset(144, 3, s, nsub)
    assert shard(list(range(24)), 1, 4) == [1, 5, 9, 13, 17, 21]


def test_two_ranks_gloo_match_single_process(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    x0, x1 = np.load(tmp_path / "x0.npy"), np.load(tmp_path / "x1.npy")
    assert np.array_equal(x0, x1)  # every rank applies the identical update
    orc, img, y, add = _data()
    sens = [orc.sensitivity(None, s, 6) for s in range(6)]
    xr = np.ones(img.shape, np.float32)
    for it in range(1, 4):
        s = (it - 1) % 6
        xr, _ = orc.osmaposl_update(xr, y, add, sens[s], s, 6, it)
    assert np.linalg.norm(x0 - xr) / np.linalg.norm(xr) < 1e-5
    ll = float(np.load(tmp_path / "ll0.npy")[0])
    ref = orc.log_likelihood(xr, y, add, None, 1, 6)
    assert abs(ll - ref) <= 1e-6 * abs(ref)


def test_rank_views_partition_the_views():
    """The views each rank holds under the view split of every subset are disjoint and cover every view."""
    from stir_b200 import geometry as G
    from stir_b200.distributed import rank_views
    from stir_b200.subsets import SYM_180, SYM_90
    for pdi, img, nsub, world in [(*G.small_3d_pet(), 6, 2), (*G.clinical_3d_pet(), 21, 4), (*G.clinical_3d_pet(), 7, 3)]:
        geo = G.make_geometry(pdi, img)
        parts = [rank_views(geo, nsub, r, world, SYM_90 | SYM_180) for r in range(world)]
        allv = sorted(v for p in parts for v in p)
        assert allv == list(range(pdi.num_views)), (nsub, world)
        assert all(len(p) > 0 for p in parts)
