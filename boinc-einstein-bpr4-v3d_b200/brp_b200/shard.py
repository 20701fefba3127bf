"""Bank sharding across ranks (one process per GPU).

Templates are independent and the observation is read-only, so a bank splits
into contiguous template ranges, one per rank, with no data-path collective.
The bank-wide toplist is a sequential fold over templates in bank order
(src/workload.cpp:126-141); it is built after the search from every rank's
compact candidate lists, gathered to rank 0.  Because each template's
candidates are compacted against its own (start-of-bank) thresholds and the
toplist re-filters them against its current rows, the final toplist equals the
single-GPU one (batch invariance, src/workunit_main.cpp:85-93).
"""
import numpy as np


def shard_range(count, rank, world):
    """Contiguous [begin, end) of `count` templates for `rank` of `world`."""
    base, extra = divmod(count, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def gather_candidates(per_template, begin, group=None):
    """Gathers {template index: candidates} from every rank to rank 0 over
    torch.distributed (gloo or nccl object collectives).  Returns the merged
    list in bank order on rank 0, None elsewhere."""
    import torch.distributed as dist
    payload = {begin + k: np.asarray(c).tobytes() for k, c in enumerate(per_template)}
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    out = [None] * world if rank == 0 else None
    dist.gather_object(payload, out, dst=0, group=group)
    if rank != 0:
        return None
    from ._lib import CANDIDATE
    merged = {}
    for d in out:
        merged.update(d)
    return [np.frombuffer(merged[t], dtype=CANDIDATE) for t in sorted(merged)]


def search_and_fold(bank, shard_templates, begin, all_templates, all_orbits, out=None, group=None):
    """One end-to-end step of a rank: searches its template shard
    (Bank.run_flat; the series is already on the device) and folds the
    bank-wide toplist of the whole bank in bank order -- directly at world size
    1, else on rank 0 after gathering every rank's kept candidate lists.
    `shard_templates` is the rank's Params array (templates begin..), the
    `all_*` arguments describe the whole bank.  Returns the toplist on rank 0
    and None elsewhere."""
    from .host import Toplist
    flat, offs, counts, status = bank.run_flat(shard_templates, out=out)
    world, rank = 1, 0
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            world, rank = dist.get_world_size(group), dist.get_rank(group)
    except ImportError:
        pass
    if world == 1:
        return Toplist().fold(all_templates, all_orbits, flat, counts)
    merged = gather_candidates([flat[offs[t]:offs[t + 1]] for t in range(len(counts))], begin, group)
    return Toplist().fold(all_templates, all_orbits, merged) if rank == 0 else None


def fold_toplist(toplist, templates, orbits, candidates):
    """Retains every template's candidates in bank order (src/workunit_main.cpp:124)."""
    if hasattr(toplist, "fold"):
        return toplist.fold(templates, orbits, candidates)
    for p, orb, c in zip(templates, orbits, candidates):
        q = toplist.thresholds(p)
        toplist.retain(c, orb[0], orb[1], orb[2], q)
    return toplist
