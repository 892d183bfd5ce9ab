"""Batched requests: many sources with their own propagators and uneven
time windows in one p2_contract_project call.  Requests that share form,
contraction set and momenta run as one batch (each kernel launches once per
chunk of slices drawn from all of them); every request must still match the
oracle on its own propagators, source and window, and match the same request
run alone."""
import numpy as np
import pytest
import torch

from plegma_b200 import lib as p2

from p2test import device_props, oracle_blocks, per_t_error

pytestmark = pytest.mark.gpu

NUC = p2.NUCLEON_CG5
BATCH_WHAT = NUC | p2.DELTA_ISO12 | p2.DELTA_ISO32 | p2.MESON_G16  # K = 480
TOL = {p2.P2_PLAIN_FP64: 1e-12, p2.P2_SPLIT_FP16: 1e-6}


def _sources(L, n, seed, wmin, wmax):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        src = tuple(int(rng.integers(0, L[d])) for d in range(4))
        out.append((src, int(rng.integers(wmin, wmax + 1))))
    return out


def _run_batch(ctx, sources, what, mode, q2max, seed0, host_props=False, host_out=False, precision=p2.P2_FP64):
    """One propagator pair per source; returns ([flat result], moms, [bufs])."""
    moms = p2.mom_list(q2max)
    props, reqs, outs, bufs, keep = [], [], [], [], []
    for i, (src, W) in enumerate(sources):
        b = device_props(ctx, [(seed0 + i, 0), (seed0 + i, 1)], t0=src[3], precision=precision)
        bufs.append(b)
        for t in b:
            if host_props:
                h = t.cpu().pin_memory()
                keep.append(h)
                props.append(ctx.prop(h.data_ptr(), precision, p2.P2_HOST))
            else:
                props.append(ctx.prop(t.data_ptr(), precision, p2.P2_DEVICE))
        _, total = p2.block_info(what, W, len(moms))
        if host_out:
            o = np.zeros(total, dtype=np.complex128)
            ptr, loc = o.ctypes.data, p2.P2_HOST
        else:
            o = torch.zeros(total, dtype=torch.complex128, device="cuda")
            ptr, loc = o.data_ptr(), p2.P2_DEVICE
        outs.append(o)
        reqs.append(ctx.request(src, W, what, ptr, loc, mode=mode, moms=moms, prop_u=2 * i, prop_d=2 * i + 1))
    ctx.contract_project(props, reqs)
    ctx.sync()
    res = [o if host_out else o.cpu().numpy() for o in outs]
    return res, moms, bufs


def _check_oracle(ctx, sources, bufs, res, moms, what, mode, taus_of):
    for (src, W), b, r in zip(sources, bufs, res):
        taus = taus_of(W)
        ref = oracle_blocks(ctx.L, b, src, moms, what, taus)
        err = per_t_error(r, what, W, moms, ref, taus)
        assert err.max() < TOL[mode], (src, W, err)


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_batch_uneven_windows_match_oracle(mode):
    """6 sources on 6^3 x 16, windows 3..16 (some wrapping through t = 0),
    nucleon + Delta (both isospins) + 16x16 mesons, |n|^2 <= 2."""
    ctx = p2.Context((6, 6, 6, 16))
    sources = _sources(ctx.L, 6, 77, 3, 16)
    res, moms, bufs = _run_batch(ctx, sources, BATCH_WHAT, mode, 2, 500)
    _check_oracle(ctx, sources, bufs, res, moms, BATCH_WHAT, mode, lambda W: sorted({0, W // 2, W - 1}))
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_batch_chunks_cross_requests(mode):
    """A workspace of a few slices forces chunks that span two requests; the
    results agree with one large chunk and with each request run alone."""
    L = (5, 4, 6, 12)
    sources = _sources(L, 4, 91, 3, 9)
    what = NUC | p2.MESON_G16
    ctx = p2.Context(L)
    big, moms, _ = _run_batch(ctx, sources, what, mode, 3, 900)
    K = p2.components(what)
    ctx.set_workspace(3 * K * ctx.V3 * 16)  # 3 slices per chunk (the split form fits 6)
    small, _, _ = _run_batch(ctx, sources, what, mode, 3, 900)
    ctx.close()
    alone = []
    for s in sources:
        c = p2.Context(L)
        r, _, _ = _run_batch(c, [s], what, mode, 3, 900 + sources.index(s))
        alone.append(r[0])
        c.close()
    for (src, W), a, b, c in zip(sources, big, small, alone):
        scale = np.abs(a).max()
        assert np.abs(a - b).max() / scale < TOL[mode], (src, W)
        assert np.abs(a - c).max() / scale < TOL[mode], (src, W)
    _ = moms


def test_batch_host_propagators_and_results_match_device():
    """Host-resident propagators (staged per chunk on the copy stream, runs
    of slices from different sources in one chunk) and host results give the
    same bits as device-resident ones."""
    L = (4, 4, 4, 10)
    sources = _sources(L, 3, 13, 4, 10)
    for mode in (p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16):
        ctx = p2.Context(L)
        ctx.set_workspace(4 * 480 * ctx.V3 * 16)
        a, _, _ = _run_batch(ctx, sources, BATCH_WHAT, mode, 1, 300)
        b, _, _ = _run_batch(ctx, sources, BATCH_WHAT, mode, 1, 300, host_props=True, host_out=True)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        ctx.close()


def test_batch_mixed_forms_and_sets_in_one_call():
    """Requests with different forms, contraction sets and momentum lists in
    one call are grouped; each group still matches the oracle."""
    ctx = p2.Context((4, 5, 3, 8))
    b0 = device_props(ctx, [(61, 0), (61, 1)], t0=2)
    b1 = device_props(ctx, [(62, 0), (62, 1)], t0=6)
    props = [ctx.prop(t.data_ptr()) for t in b0 + b1]
    spec = [  # (bufs index, source, window, what, mode, momenta)
        (0, (1, 2, 0, 2), 8, NUC, p2.P2_SPLIT_FP16, p2.mom_list(1)),
        (1, (3, 0, 2, 6), 5, NUC | p2.MESON_ALL34, p2.P2_PLAIN_FP64, p2.mom_list(2)),
        (1, (3, 0, 2, 6), 4, NUC, p2.P2_SPLIT_FP16, p2.mom_list(1)),
        (0, (0, 4, 1, 2), 6, p2.MESON_DIAG10 | p2.MESON_NEW10, p2.P2_SPLIT_FP16,
         np.array([[0, 0, 0], [1, -1, 0], [0, 0, 2]], dtype=np.int32)),
    ]
    outs, reqs = [], []
    for bi, src, W, what, mode, moms in spec:
        _, total = p2.block_info(what, W, len(moms))
        o = torch.zeros(total, dtype=torch.complex128, device="cuda")
        outs.append(o)
        reqs.append(ctx.request(src, W, what, o.data_ptr(), mode=mode, moms=moms, prop_u=2 * bi, prop_d=2 * bi + 1))
    ctx.contract_project(props, reqs)
    ctx.sync()
    for (bi, src, W, what, mode, moms), o in zip(spec, outs):
        bufs = b0 if bi == 0 else b1
        taus = list(range(W))
        ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
        err = per_t_error(o.cpu().numpy(), what, W, moms, ref, taus)
        assert err.max() < TOL[mode], (src, W, what, err)
    ctx.close()


def test_batch_fp32_propagators_split():
    """FP32 propagators for the whole batch (split form only)."""
    ctx = p2.Context((6, 4, 4, 12))
    sources = _sources(ctx.L, 3, 5, 4, 12)
    res, moms, bufs = _run_batch(ctx, sources, NUC | p2.MESON_G16, p2.P2_SPLIT_FP16, 2, 700,
                                 precision=p2.P2_FP32)
    for (src, W), b, r in zip(sources, bufs, res):
        taus = [0, W - 1]
        ref = oracle_blocks(ctx.L, b, src, moms, NUC | p2.MESON_G16, taus, fp32=True)
        err = per_t_error(r, NUC | p2.MESON_G16, W, moms, ref, taus)
        assert err.max() < 1e-6, (src, W, err)
    ctx.close()
