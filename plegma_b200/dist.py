"""Running the path on several GPUs: one process per GPU, torch.distributed
for the plumbing.

The contraction is site-local and the projection is a sum over the sites of
one time slice, so the work shards without any exchange while it runs:

  * by source: every rank contracts its own sources (independent requests);
  * by time slab: rank coords[3] holds and computes the slices of its slab
    (p2_local_taus lists them); the other slices of its result stay zero;
  * by space: a rank holds a spatial sub-volume; its projection uses global
    coordinates, so its result is a partial sum over its sites.

One all-reduce (sum) of the [block][group][dataset][tau][mom][comp] result over
the ranks that share a source then gives every rank the full correlator; it
plays the role of the reference's MPI_Allreduce over the spatial
communicator plus the assembly of the time slabs by its writer
(lib/kernels/PLEGMA_baryons.cuh:196-202, lib/PLEGMA_Correlator.cu:810-950).
"""
from __future__ import annotations

from typing import Sequence, Tuple


def rank_coords(procs: Sequence[int], rank: int) -> Tuple[int, int, int, int]:
    """Process-grid coordinates of a rank, x fastest (rank = x + Px (y + Py (z + Pz t)))."""
    c = []
    r = rank
    for p in procs:
        c.append(r % p)
        r //= p
    if r != 0:
        raise ValueError("rank outside the process grid")
    return tuple(c)


def local_extent(L: Sequence[int], procs: Sequence[int]) -> Tuple[int, int, int, int]:
    if any(l % p for l, p in zip(L, procs)):
        raise ValueError("the process grid must divide the lattice")
    return tuple(l // p for l, p in zip(L, procs))


def gather_result(result, group=None):
    """Sum a result tensor over the ranks of `group` in place (zeros outside a
    rank's slices, partial sums over its sites) and return it."""
    import torch.distributed as dist
    dist.all_reduce(result, op=dist.ReduceOp.SUM, group=group)
    return result
