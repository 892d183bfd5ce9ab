"""A process grid of 2 spatial halves x 2 time slabs run on one GPU: one
context per rank (p2_geom procs (2, 1, 1, 2) and that rank's coords), each
holding only its rank's sub-volume and time slab (synthesised from the
global-site-keyed generator), running the real kernels.  The ranks' results
(zeros outside their slices, partial sums over their sites with phases in
global coordinates) summed on the host, as plegma_b200.dist.gather_result
does over NCCL, must match one context over the full lattice and the oracle.
The sums run in a different order than the single context's, so the plain
form is compared at 1e-12 relative, not bitwise; the split form at its
1e-6 per-slice bound against the oracle."""
import numpy as np
import pytest
import torch

from plegma_b200 import dist as pdist
from plegma_b200 import lib as p2

from p2test import oracle_blocks, per_t_error

pytestmark = pytest.mark.gpu

L = (8, 6, 4, 8)
PROCS = (2, 1, 1, 2)
SRC = (3, 2, 1, 6)
W = 6  # slices 6, 7, 0, 1, 2, 3: both time slabs, wrapping through t = 0
WHAT = p2.NUCLEON_CG5 | p2.MESON_G16 | p2.DELTA_ISO12
SEED = 31


def _run_ctx(ctx, nt, t_first, mode, moms):
    V3l = ctx.V3
    bufs = []
    for f in range(2):
        b = torch.empty(144 * V3l * nt, dtype=torch.complex128, device="cuda")
        ctx.synth(b.data_ptr(), True, p2.P2_FP64, SEED, f, SRC[3], 0.5, t_first, nt)
        bufs.append(b)
    props = [ctx.prop(b.data_ptr(), t_first=t_first, nt=nt) for b in bufs]
    _, total = p2.block_info(WHAT, W, len(moms))
    out = torch.zeros(total, dtype=torch.complex128, device="cuda")
    req = ctx.request(SRC, W, WHAT, out.data_ptr(), mode=mode, moms=moms)
    taus = ctx.local_taus(props, req)
    ctx.contract_project(props, [req])
    ctx.sync()
    return out.cpu().numpy(), taus, bufs


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_process_grid_partials_sum_to_the_full_lattice(mode):
    moms = p2.mom_list(2)
    full = p2.Context(L)
    ref, taus_full, fbufs = _run_ctx(full, L[3], 0, mode, moms)
    assert taus_full == list(range(W))
    acc = np.zeros_like(ref)
    Ll = pdist.local_extent(L, PROCS)
    seen = []
    for rank in range(int(np.prod(PROCS))):
        coords = pdist.rank_coords(PROCS, rank)
        ctx = p2.Context(L, procs=PROCS, coords=coords)
        out, taus, _ = _run_ctx(ctx, Ll[3], coords[3] * Ll[3], mode, moms)
        ctx.close()
        # the rank computes exactly the window slices of its time slab
        assert taus == [t for t in range(W) if coords[3] * Ll[3] <= (SRC[3] + t) % L[3] < (coords[3] + 1) * Ll[3]]
        seen += taus
        acc += out
    assert sorted(set(seen)) == list(range(W))
    if mode == p2.P2_PLAIN_FP64:
        assert np.abs(acc - ref).max() / np.abs(ref).max() < 1e-12
    taus = list(range(W))
    orc = oracle_blocks(L, fbufs, SRC, moms, WHAT, taus)
    err = per_t_error(acc, WHAT, W, moms, orc, taus)
    assert err.max() < (1e-12 if mode == p2.P2_PLAIN_FP64 else 1e-6), err
    full.close()
