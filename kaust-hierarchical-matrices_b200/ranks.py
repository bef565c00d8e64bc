"""Multi-process plumbing of the engine (one process per GPU).

Three ways to spread the work over G ranks:

* independent clouds per rank (the default of bench.py): every rank builds and
  multiplies its own cloud; the only cross-rank steps are the timing
  reduction and the sum of the work (weak scaling);
* a batch's clouds split across ranks (assign_clouds): a size-balanced
  assignment, each rank builds one batch of its clouds, nothing is exchanged
  on the data path;
* one cloud split by block rows (subtree_shards, allgather_rows): every rank
  builds the KD tree and block structure (cheap, identical on all ranks) and
  compresses only the blocks of its row shard (hm_hmatrix_build_rows); a
  product all-gathers X, whose rows are spread like Y's, and writes the rank's
  own rows of Y.  That all-gather is the one exchange per product.
"""
import math


def cloud_seed(base, rank):
    """Seed of rank `rank`'s cloud: independent clouds, reproducible per rank."""
    return int(base) + 7919 * int(rank)


def max_over_ranks(value, world):
    """The maximum of a float over all ranks (identity when world == 1).  Uses
    the initialised process group: a CUDA tensor under NCCL, a CPU tensor
    under gloo."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(bytes_per_rank, ms_max, world):
    """Whole-job throughput in GB/s: every rank moved bytes_per_rank in at most
    ms_max milliseconds."""
    return world * float(bytes_per_rank) / (float(ms_max) * 1e-3) / 1e9


def cloud_cost(n):
    """Relative cost of one cloud of n points: a product reads O(n log n)
    bytes of factors (and a build does O(n log n) work)."""
    return float(n) * max(1.0, math.log2(max(int(n), 2)))


def assign_clouds(sizes, world):
    """Size-balanced assignment of independent clouds to ranks: the longest
    (costliest) cloud first, each to the rank with the least work so far (ties
    to the lower rank).  Returns one list of cloud indices per rank, each in
    increasing order; every rank gets at least one cloud when there are at
    least `world` of them."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-cloud_cost(sizes[i]), i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += cloud_cost(sizes[i])
    return [sorted(x) for x in out]


def subtree_shards(leaf_offsets, world):
    """Block-row shards of one cloud for `world` ranks.

    leaf_offsets: the tree's 2^depth + 1 leaf offsets (tree order).  The 2^L
    subtrees at level L = ceil(log2 world) (at most the leaves) are given out
    as contiguous runs, one run per rank, each run ending at the subtree
    boundary nearest to an equal share of the rows.  Returns one tuple
    (leaf_begin, leaf_end, row_begin, row_end) per rank."""
    leaf_offsets = [int(x) for x in leaf_offsets]
    nleaf = len(leaf_offsets) - 1
    depth = int(round(math.log2(nleaf)))
    if (1 << depth) != nleaf:
        raise ValueError("leaf offsets must cover 2^depth leaves")
    if world < 1 or world > nleaf:
        raise ValueError("need 1 <= world <= number of leaves")
    L = min(depth, max(0, math.ceil(math.log2(world))))
    nsub = 1 << L
    per = nleaf // nsub
    bounds = [leaf_offsets[i * per] for i in range(nsub + 1)]  # rows at subtree boundaries
    n = leaf_offsets[-1]
    cut = [0]
    for r in range(1, world):
        target = n * r / world
        # the subtree boundary nearest the target, leaving at least one subtree
        # for this rank and for every rank after it
        lo_b, hi_b = cut[-1] + 1, nsub - (world - r)
        best = min(range(lo_b, hi_b + 1), key=lambda b: (abs(bounds[b] - target), b))
        cut.append(best)
    cut.append(nsub)
    return [(cut[r] * per, cut[r + 1] * per, bounds[cut[r]], bounds[cut[r + 1]]) for r in range(world)]


class RowGather:
    """All-gather of row blocks: each rank holds rows [row_begin, row_end) of
    an (nrhs, n) array (column-major n x nrhs, i.e. one contiguous row per
    right-hand side); gather() returns the whole (nrhs, n) array on every
    rank.  Buffers are allocated once per shape; shards are padded to the
    widest one for the collective (all_gather_into_tensor), then copied into
    place."""

    def __init__(self, shards, nrhs, dtype, device):
        import torch

        self.shards = shards
        self.world = len(shards)
        self.width = max(r1 - r0 for _, _, r0, r1 in shards)
        self.n = shards[-1][3]
        self.buf = torch.empty((self.world, nrhs, self.width), dtype=dtype, device=device)
        self.send = torch.zeros((nrhs, self.width), dtype=dtype, device=device)
        self.full = torch.empty((nrhs, self.n), dtype=dtype, device=device)

    def gather(self, local, rank):
        """local: this rank's (nrhs, rows) block."""
        import torch.distributed as dist

        r0, r1 = self.shards[rank][2], self.shards[rank][3]
        if local.shape[1] != r1 - r0:
            raise ValueError("rank %d holds rows [%d, %d), got %d" % (rank, r0, r1, local.shape[1]))
        self.send[:, : r1 - r0].copy_(local)
        dist.all_gather_into_tensor(self.buf.view(self.world * self.send.shape[0], self.width), self.send)
        for q, (_, _, a, b) in enumerate(self.shards):
            self.full[:, a:b].copy_(self.buf[q, :, : b - a])
        return self.full


def allgather_rows(local, shards, rank):
    """One-off form of RowGather.gather."""
    return RowGather(shards, local.shape[0], local.dtype, local.device).gather(local, rank).clone()
