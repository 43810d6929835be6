"""Multi-GPU reconstruction: one process per GPU, torch.distributed (NCCL) for the plumbing.

Two ways the hot path shards:
* independent units (dynamic frames, gates, noise realisations): `shard` gives each rank its own units;
  no collective touches the data path;
* one large reconstruction: every rank keeps the whole image and projects part of each subset.  Subset s of n
  is the union over ranks r of subset s + r*n of n*R (the basic views v = s mod n split by v mod n*R), so rank
  r computes the numerator of its part, an all-reduce (sum) combines the numerators (the image-sized exchange
  STIR's MPI version does with MPI_Reduce, distributed_functions.cxx:933,977), and every rank applies the
  identical update (no broadcast needed).  Sensitivities and log-likelihood values are combined the same way.
  Each rank holds the projection data (y, additive term, multiplicative factors) of its own views only: its
  projector is a view shard (`RayTracingProjector.set_view_shard(rank_views(...))`) and its arrays the shard's
  (`shard_projdata`), 1/R of the whole data.

The per-rank compute is a backend with numerator / apply / sensitivity / log_likelihood methods;
`B200Backend` runs them on the GPU through the C ABI.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

from . import _abi
from .projectors import RayTracingProjector, _stream_ptr


def shard(units: Sequence, rank: int, world: int) -> List:
    """The units (frames, realisations) rank `rank` of `world` reconstructs."""
    return list(units[rank::world])


def rank_subset(subset_num: int, num_subsets: int, rank: int, world: int):
    """(subset, number of subsets) of rank `rank`'s part of subset `subset_num` of `num_subsets`."""
    return subset_num + rank * num_subsets, num_subsets * world


def rank_views(geometry, num_subsets: int, rank: int, world: int, bits: int = None) -> List[int]:
    """The views whose projection data rank `rank` of `world` needs when every subset s of `num_subsets` is split as
    subset s + rank * num_subsets of num_subsets * world: the union of those sub-subsets' views (their basic views
    and every view related to them by the symmetries `bits`, b200rt_info.symmetries_used).  The ranks' view sets
    partition the views."""
    from .subsets import views_in_subset
    out = set()
    for s in range(num_subsets):
        out.update(views_in_subset(geometry, *rank_subset(s, num_subsets, rank, world), bits=bits))
    return sorted(out)


def shard_projdata(pdi, data, views):
    """The part of device-layout projection data `data` (non-TOF, [segment -S..S][view][tangential][axial]) that a
    view shard holding `views` (in that order) uses: [segment][slot][tangential][axial]."""
    import torch
    S = pdi.max_segment_num
    nv, nt = pdi.num_views, pdi.num_tangential_poss
    idx = torch.as_tensor(list(views), dtype=torch.long, device=data.device)
    parts, off = [], 0
    for seg in range(-S, S + 1):
        nax = pdi.get_num_axial_poss(seg)
        n = nv * nt * nax
        parts.append(data[off:off + n].view(nv, nt * nax).index_select(0, idx).reshape(-1))
        off += n
    return torch.cat(parts)


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class B200Backend:
    """Per-rank compute on one GPU (device-layout torch tensors)."""

    def __init__(self, projector: RayTracingProjector, y, additive=None, mult=None, zero_seg0_end_planes=False,
                 mode=_abi.BACKPROJECT_ATOMIC):
        self.proj, self.y, self.additive, self.mult = projector, y, additive, mult
        self.zero_ends, self.mode = zero_seg0_end_planes, mode

    def empty_image(self):
        return self.proj.empty_image(zero=False)

    def numerator(self, x, subset, nsub):
        u = self.proj.empty_image(zero=False)
        _abi.check(self.proj.lib.b200rt_osmaposl_numerator_dev(self.proj.h, _p(x), _p(self.y), _p(self.additive), subset,
                                                               nsub, int(self.zero_ends), self.mode, _p(u),
                                                               _stream_ptr(None)), self.proj.h,
                   "b200rt_osmaposl_numerator_dev")
        return u

    def apply(self, x, u, sens, nsub, subiteration_num, prior=None, map_model=_abi.MAP_MULTIPLICATIVE,
              min_rel=0.0, max_rel=3.4028234663852886e38):
        pa = None if prior is None else ctypes.byref(prior.as_abi(map_model))
        _abi.check(self.proj.lib.b200rt_osmaposl_apply_update_dev(self.proj.h, _p(x), _p(u), _p(sens), nsub,
                                                                  subiteration_num, pa, float(min_rel), float(max_rel),
                                                                  _stream_ptr(None)), self.proj.h,
                   "b200rt_osmaposl_apply_update_dev")
        return x

    def sensitivity(self, subset, nsub):
        s = self.proj.empty_image(zero=False)
        _abi.check(self.proj.lib.b200rt_sensitivity_dev(self.proj.h, _p(self.mult), _p(s), subset, nsub, int(self.zero_ends),
                                                        self.mode, _stream_ptr(None)), self.proj.h, "b200rt_sensitivity_dev")
        return s

    def log_likelihood(self, x, subset, nsub):
        out = ctypes.c_double(0.0)
        _abi.check(self.proj.lib.b200rt_log_likelihood_dev(self.proj.h, _p(x), _p(self.y), _p(self.additive),
                                                           _p(self.mult), subset, nsub, int(self.zero_ends),
                                                           ctypes.byref(out), _stream_ptr(None)), self.proj.h,
                   "b200rt_log_likelihood_dev")
        return out.value


class DistributedOSMAPOSL:
    """OSMAPOSL with each subset's projections split across the ranks of a process group.

    `to_tensor` / `from_tensor` convert a backend image to / from the torch tensor the collective
    uses (identity for GPU tensors; numpy <-> CPU tensors for CPU backends)."""

    def __init__(self, backend, num_subsets: int, num_subiterations: int, group=None, prior=None,
                 map_model=_abi.MAP_MULTIPLICATIVE, min_rel=0.0, max_rel=3.4028234663852886e38,
                 use_subset_sensitivities=True, to_tensor=None, from_tensor=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.b = backend
        self.nsub, self.nsubiter = num_subsets, num_subiterations
        self.prior, self.map_model, self.min_rel, self.max_rel = prior, map_model, min_rel, max_rel
        self.use_subset_sensitivities = use_subset_sensitivities
        self.to_tensor = to_tensor or (lambda a: a)
        self.from_tensor = from_tensor or (lambda t, like: t)
        self.sens = None

    def _allreduce_image(self, img):
        t = self.to_tensor(img)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return self.from_tensor(t, img)

    def set_up(self):
        subs = []
        for s in range(self.nsub):
            part = self.b.sensitivity(*rank_subset(s, self.nsub, self.rank, self.world))
            subs.append(self._allreduce_image(part))
        if self.use_subset_sensitivities:
            self.sens = subs
        else:
            total = subs[0]
            for t in subs[1:]:
                total = total + t
            self.sens = [total / self.nsub] * self.nsub
        return self

    def update_estimate(self, x, subiteration_num):
        s = (subiteration_num - 1) % self.nsub
        u = self.b.numerator(x, *rank_subset(s, self.nsub, self.rank, self.world))
        u = self._allreduce_image(u)
        return self.b.apply(x, u, self.sens[s], self.nsub, subiteration_num, self.prior, self.map_model, self.min_rel,
                            self.max_rel)

    def reconstruct(self, x):
        if self.sens is None:
            self.set_up()
        for it in range(1, self.nsubiter + 1):
            x = self.update_estimate(x, it)
        return x

    def log_likelihood(self, x, subset_num=0, num_subsets=1):
        import torch
        v = self.b.log_likelihood(x, *rank_subset(subset_num, num_subsets, self.rank, self.world))
        t = torch.tensor([v], dtype=torch.float64)
        if self.dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return float(t.item())
