"""CUDA-graph replays (p2_graph_*) and the launch-shape autotuner
(p2_tune_enable): a replay reproduces the eager call bit for bit, follows
propagators refilled in place, and tuned shapes stay within the form's
tolerance of the oracle."""
import os

import numpy as np
import pytest
import torch

from plegma_b200 import lib as p2

from p2test import device_props, oracle_blocks, per_t_error

pytestmark = pytest.mark.gpu

NUC = p2.NUCLEON_CG5
WHAT = NUC | p2.DELTA_ISO12 | p2.DELTA_ISO32 | p2.MESON_G16
TOL = {p2.P2_PLAIN_FP64: 1e-12, p2.P2_SPLIT_FP16: 1e-6}


def _setup(ctx, mode, nsrc=4, seed=40, q2max=2, what=WHAT):
    rng = np.random.default_rng(seed)
    moms = p2.mom_list(q2max)
    srcs, bufs, props, outs, reqs = [], [], [], [], []
    for i in range(nsrc):
        src = tuple(int(rng.integers(0, ctx.L[d])) for d in range(4))
        W = int(rng.integers(3, ctx.L[3] + 1))
        b = device_props(ctx, [(seed + i, 0), (seed + i, 1)], t0=src[3])
        props += [ctx.prop(t.data_ptr()) for t in b]
        _, total = p2.block_info(what, W, len(moms))
        o = torch.zeros(total, dtype=torch.complex128, device="cuda")
        reqs.append(ctx.request(src, W, what, o.data_ptr(), mode=mode, moms=moms, prop_u=2 * i, prop_d=2 * i + 1))
        srcs.append((src, W))
        bufs.append(b)
        outs.append(o)
    return srcs, bufs, props, outs, reqs, moms


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_graph_replay_matches_eager_and_follows_refills(mode):
    ctx = p2.Context((5, 4, 6, 10))
    srcs, bufs, props, outs, reqs, moms = _setup(ctx, mode)
    ctx.contract_project(props, reqs)
    ctx.sync()
    eager = [o.clone() for o in outs]
    for o in outs:
        o.zero_()
    g = ctx.graph(props, reqs)  # the eager run inside creation writes the results too
    for o in outs:
        o.zero_()
    for _ in range(3):
        g.launch()
    g.sync()
    for a, b in zip(eager, outs):
        assert torch.equal(a, b)
    # refill the propagators in place with new seeds: replays follow the new data
    for i, ((src, W), b) in enumerate(zip(srcs, bufs)):
        for f, t in enumerate(b):
            ctx.synth(t.data_ptr(), True, p2.P2_FP64, 700 + i, f, src[3], 0.5)
    ctx.sync()
    g.launch()
    g.sync()
    for (src, W), b, o in zip(srcs, bufs, outs):
        taus = [0, W - 1]
        ref = oracle_blocks(ctx.L, b, src, moms, WHAT, taus)
        err = per_t_error(o.cpu().numpy(), WHAT, W, moms, ref, taus)
        assert err.max() < TOL[mode], (src, W, err)
    g.close()
    ctx.close()


def test_graph_rejects_host_buffers():
    ctx = p2.Context((4, 4, 4, 8))
    (u,) = device_props(ctx, [(3, 0)], t0=0)
    h = u.cpu().pin_memory()
    out = torch.zeros(p2.block_info(NUC, 8, 1)[1], dtype=torch.complex128, device="cuda")
    req = ctx.request((0, 0, 0, 0), 8, NUC, out.data_ptr(), moms=np.zeros((1, 3), np.int32))
    with pytest.raises(p2.P2Error) as e:
        ctx.graph([ctx.prop(h.data_ptr(), location=p2.P2_HOST)] * 2, [req])
    assert e.value.status == p2.P2_ERR_UNSUPPORTED
    ctx.close()


def test_graph_rejects_two_batches():
    """A graph records one batch (its descriptors and tables are uploaded
    once): requests with different contraction sets are refused, and the
    context still runs them eagerly."""
    ctx = p2.Context((4, 4, 4, 8))
    bufs = device_props(ctx, [(5, 0), (5, 1)], t0=1)
    props = [ctx.prop(b.data_ptr()) for b in bufs]
    moms = p2.mom_list(1)
    outs, reqs = [], []
    for what in (NUC, p2.MESON_G16):
        out = torch.zeros(p2.block_info(what, 8, len(moms))[1], dtype=torch.complex128, device="cuda")
        outs.append(out)
        reqs.append(ctx.request((0, 1, 2, 1), 8, what, out.data_ptr(), moms=moms, mode=p2.P2_SPLIT_FP16))
    with pytest.raises(p2.P2Error) as e:
        ctx.graph(props, reqs)
    assert e.value.status == p2.P2_ERR_UNSUPPORTED
    assert "one batch" in str(e.value)
    ctx.contract_project(props, reqs)
    ctx.sync()
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_tuner_caches_choices_and_stays_accurate(tmp_path, mode):
    path = str(tmp_path / "tune.tsv")
    ctx = p2.Context((6, 6, 4, 8))
    ctx.tune(True, path)
    srcs, bufs, props, outs, reqs, moms = _setup(ctx, mode, nsrc=2, seed=90, what=NUC | p2.MESON_G16)
    ctx.contract_project(props, reqs)
    ctx.sync()
    n = ctx.tune_count()
    assert n >= 1
    lines = open(path).read().strip().splitlines()
    assert len(lines) == n
    kernel = "project_split" if mode == p2.P2_SPLIT_FP16 else "project_fp64"
    assert all(line.startswith(kernel) and len(line.split("\t")) == 3 for line in lines)
    for (src, W), b, o in zip(srcs, bufs, outs):
        taus = list(range(W))
        ref = oracle_blocks(ctx.L, b, src, moms, NUC | p2.MESON_G16, taus)
        err = per_t_error(o.cpu().numpy(), NUC | p2.MESON_G16, W, moms, ref, taus)
        assert err.max() < TOL[mode], (src, W, err)
    first = [o.clone() for o in outs]
    ctx.close()
    # a new context reads the file: same choices, same bits, no new entries
    ctx2 = p2.Context((6, 6, 4, 8))
    ctx2.tune(True, path)
    assert ctx2.tune_count() == n
    srcs2, bufs2, props2, outs2, reqs2, _ = _setup(ctx2, mode, nsrc=2, seed=90, what=NUC | p2.MESON_G16)
    ctx2.contract_project(props2, reqs2)
    ctx2.sync()
    assert ctx2.tune_count() == n
    for a, b in zip(first, outs2):
        assert torch.equal(a, b)
    ctx2.close()
    assert os.path.exists(path)
