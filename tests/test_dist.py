"""The multi-rank path on CPU: world_size 2 and 4 with the gloo backend,
rendezvous on 127.0.0.1.  Every rank builds a host-only context for its
place in the process grid, asks the library which time slices it computes
(p2_local_taus), computes its share (the oracle stands in for the GPU on
this CPU test: its sites only, its slices only), and plegma_b200.dist sums
the shares; the result must equal the single-process oracle.  This checks
the slab selection, the global-coordinate phases of a spatial sub-volume and
the gather, which are the host logic of the N > 1 path."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

L = (4, 2, 2, 8)
SRC = (1, 0, 1, 6)
W = 6  # slices 6, 7, 0, 1, 2, 3: wraps through t = 0
WHAT = 1 | 8  # nucleon + 16x16 mesons
MOMS = np.array([[0, 0, 0], [1, 0, 0], [0, 1, -1]], dtype=np.int32)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _props_full():
    """Seeded full-lattice propagators (host generator of the library)."""
    from plegma_b200 import lib as p2
    ctx = p2.Context(L, device=-1)
    V = L[0] * L[1] * L[2] * L[3]
    u = np.zeros(144 * V, dtype=np.complex128)
    d = np.zeros_like(u)
    ctx.synth(u.ctypes.data, False, p2.P2_FP64, 11, 0, SRC[3], 0.5)
    ctx.synth(d.ctypes.data, False, p2.P2_FP64, 11, 1, SRC[3], 0.5)
    ctx.close()
    return u.reshape(144, L[3], L[2], L[1], L[0]), d.reshape(144, L[3], L[2], L[1], L[0])


def _worker(rank, world, procs, port, q):
    try:
        sys.path.insert(0, ROOT)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world)
        import oracle_py as orc
        from plegma_b200 import dist as pdist
        from plegma_b200 import lib as p2

        coords = pdist.rank_coords(procs, rank)
        Ll = pdist.local_extent(L, procs)
        ctx = p2.Context(L, procs=procs, coords=coords, device=-1)
        # this rank's propagator views: its time slab only
        t_first = coords[3] * Ll[3]
        u, d = _props_full()
        props = [ctx.prop(0x1000, location=p2.P2_HOST, t_first=t_first, nt=Ll[3]),
                 ctx.prop(0x1000, location=p2.P2_HOST, t_first=t_first, nt=Ll[3])]
        req = ctx.request(SRC, W, WHAT, 0x1000, p2.P2_HOST, moms=MOMS)
        taus = ctx.local_taus(props, req)
        # this rank's share: the oracle on the full lattice with every other
        # rank's sites zeroed (all contractions are multilinear in the
        # propagators, so zero sites contribute nothing)
        mask = np.zeros((L[3], L[2], L[1], L[0]), dtype=bool)
        sl = [slice(c * n, (c + 1) * n) for c, n in zip(coords, Ll)]
        mask[sl[3], sl[2], sl[1], sl[0]] = True
        um = np.where(mask[None], u, 0).reshape(144, -1)
        dm = np.where(mask[None], d, 0).reshape(144, -1)
        K = orc.components(WHAT)
        full = torch.zeros((W, len(MOMS), K), dtype=torch.complex128)
        if taus:
            out, _, _ = orc.twopt(L, um, dm, SRC, MOMS, WHAT, taus, want_abs=False)
            full[taus] = torch.from_numpy(out)
        pdist.gather_result(full)
        q.put((rank, taus, full.numpy() if rank == 0 else None))
        ctx.close()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None))


def _run(procs):
    world = int(np.prod(procs))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, procs, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
    errs = [r for r in res if isinstance(r[1], str)]
    assert not errs, errs
    return sorted(res, key=lambda r: r[0])


def _reference():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    u, d = _props_full()
    out, _, _ = orc.twopt(L, u.reshape(144, -1), d.reshape(144, -1), SRC, MOMS, WHAT, list(range(W)), want_abs=False)
    return out


@pytest.mark.parametrize("procs", [(1, 1, 1, 2), (2, 1, 1, 2)])
def test_sharded_result_equals_single_process(procs):
    """Time slabs (2 ranks) and time slabs x spatial halves (4 ranks)."""
    res = _run(procs)
    # every window slice is computed by the ranks of exactly one time slab
    Ll = L[3] // procs[3]
    for rank, taus, _ in res:
        t_slab = (rank // (procs[0] * procs[1] * procs[2]))
        assert all(t_slab * Ll <= (SRC[3] + tau) % L[3] < (t_slab + 1) * Ll for tau in taus)
    per_slab = {}
    for rank, taus, _ in res:
        per_slab.setdefault(rank // (procs[0] * procs[1] * procs[2]), set()).update(taus)
    allt = sorted(t for s in per_slab.values() for t in s)
    assert allt == list(range(W))
    ref = _reference()
    got = res[0][2]
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-13
