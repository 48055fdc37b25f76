"""One ATLAS12 model over several GPUs: frequencies sharded across ranks.

The reference iterates one model on one core (atlas12c.f90:496-606).  Its
frequency loop (RUN_RT_PASS, atlas12_modules.f90:3905-3949) only adds into
the mode-2 accumulators of TCORR, RADIAP and ROSS, so the 30,000
frequencies split into contiguous shards, one per rank: each rank runs
LINOP1 (the lines whose +-100-point wing window meets its shard) and the RT
pass over its shard, one all-reduce (sum, 8*72+1 doubles, ~4.6 KB) adds the
shards' accumulators, and every rank runs the same ROSS(3)/RADIAP(3)/TCORR(3)
finish on the total, so the structures stay identical on every rank without
a broadcast.  That all-reduce is the only exchange of the path.

    ctx = _lib.Context(local_rank, stream=torch.cuda.current_stream().cuda_stream)
    m = ShardedAtlasModel(ctx, operators, linedata=lines, waveset=ws, rcoset=rc)
    n, hist = m.iterate(max_iter=60, tol_percent=0.1)

The loop itself (iterate_sharded) takes the begin / all-reduce / end steps
as callables, so the decomposition can be exercised with any backend.
"""
import numpy as np

from . import atlas


def shard_range(numnu, rank, world):
    """Frequencies of `rank` (1-based, inclusive): contiguous, sizes differ by at most one."""
    if not (0 <= rank < world) or numnu < world:
        raise ValueError(f"cannot shard {numnu} frequencies over {world} ranks (rank {rank})")
    base, extra = divmod(numnu, world)
    first = rank * base + min(rank, extra) + 1
    return first, first + base + (1 if rank < extra else 0) - 1


def iterate_sharded(begin, allreduce, end, max_iter, tol_percent):
    """Iterate: begin() produces this rank's frequency sums, allreduce() adds
    every rank's, end() finishes the iteration and returns max |FLXERR|.
    Stops after the first iteration with max |FLXERR| <= tol_percent (every
    rank sees the same value, so every rank stops together).
    Returns (iterations, history)."""
    hist = []
    for _ in range(max_iter):
        begin()
        allreduce()
        e = end()
        hist.append(e)
        if not np.isfinite(e) or (tol_percent > 0 and e <= tol_percent):
            break
    return len(hist), np.array(hist)


class ShardedAtlasModel:
    """An AtlasModel whose frequencies are sharded over the ranks of a
    torch.distributed process group (NCCL); with one rank it is the plain
    device-resident model."""

    def __init__(self, ctx, operators, group=None, **model_kwargs):
        import torch
        import torch.distributed as dist
        self.ctx = ctx
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.model = atlas.AtlasModel(ctx, operators, **model_kwargs)
        numnu = self.model.waveset.size
        self.nu_first, self.nu_last = shard_range(numnu, self.rank, self.world)
        self.model.set_shard(self.nu_first, self.nu_last)
        self.sums = torch.zeros(8 * self.model.nrhox + 1, dtype=torch.float64, device=f"cuda:{ctx.device}")
        self.model.set_sums_buffer(self.sums)

    def _allreduce(self):
        import torch
        import torch.distributed as dist
        if self.world == 1:
            return
        self.ctx.synchronize()  # this rank's sums are complete on the library's stream
        dist.all_reduce(self.sums, op=dist.ReduceOp.SUM, group=self.group)
        torch.cuda.current_stream().synchronize()  # the total is in place before the finish reads it

    def iterate(self, max_iter=60, tol_percent=0.1):
        return iterate_sharded(self.model.iterate_begin, self._allreduce, self.model.iterate_end, max_iter,
                               tol_percent)

    def structure(self):
        return self.model.structure()

    def close(self):
        self.model.set_sums_buffer(None)
        self.model.close()
