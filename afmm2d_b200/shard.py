"""One problem sharded over the ranks of a torch.distributed process group.

Every rank builds the whole problem (setup is deterministic, so every rank
holds the same operators), restricts its handle to its shard with
``AFMM.set_shard(rank, world)`` -- the potentials of its subtrees' points,
zeros elsewhere -- and one all-reduce sums the shards' outputs into the whole
product (exactly: every point has one nonzero contribution).  The reference is
single-process (src/AFMM2DTree.cpp:1099-1225); this is the level-subtree
sharding of one matvec, with the charges replicated on every rank, so the only
exchange is the sum of the outputs.
"""
import torch


def combine(partial, group=None):
    """Sums the shards' outputs in place over `group` and returns the tensor."""
    import torch.distributed as dist

    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


class ShardedMatvec:
    """Matvecs of one assembled AFMM handle split over the ranks of `group`."""

    def __init__(self, afmm, group=None):
        import torch.distributed as dist

        self.afmm = afmm
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        afmm.set_shard(self.rank, self.world)

    def matvec_device(self, q, y, nrhs, precision="mixed"):
        """y = K q for device tensors holding nrhs columns of N values each
        (column-major: column c at offset c * N), on every rank."""
        self.afmm.matvec_device(q.data_ptr(), y.data_ptr(), nrhs, self.afmm.N, precision)  # returns when done
        return combine(y, self.group) if self.world > 1 else y
