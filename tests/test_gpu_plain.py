"""Parity of the plain FP64 form (CUDA, through the C ABI) with the FP64
oracle on the same seeded propagators.  Tolerance: err(t) <= 1e-12 relative
to sum_x |c_k(x,t)| for every time slice, momentum and component."""
import numpy as np
import pytest
import torch

from plegma_b200 import lib as p2

from p2test import device_props, oracle_blocks, per_t_error, run

pytestmark = pytest.mark.gpu

NUC = p2.NUCLEON_CG5
MES = p2.MESON_G16 | p2.MESON_ALL34 | p2.MESON_NEW10 | p2.MESON_DIAG10
TOL = 1e-12


@pytest.fixture(scope="module")
def ctx_small():
    c = p2.Context((4, 4, 4, 8))
    yield c
    c.close()


def test_config_small_nucleon(ctx_small):
    """4^3 x 8, one propagator used for u and d, t0 = 0, nucleon C g5, |n|^2 <= 2."""
    ctx = ctx_small
    (u,) = device_props(ctx, [(1001, 0)], t0=0)
    bufs = [u, u]
    out, moms = run(ctx, bufs, (0, 0, 0, 0), 8, NUC, q2max=2)
    taus = list(range(8))
    ref = oracle_blocks(ctx.L, bufs, (0, 0, 0, 0), moms, NUC, taus)
    err = per_t_error(out, NUC, 8, moms, ref, taus)
    assert err.max() < TOL, err
    blk = p2.result_blocks(NUC, 8, len(moms), out)[NUC]
    # u = d: proton and neutron datasets agree
    assert np.allclose(blk[0, 0], blk[0, 1], rtol=1e-13, atol=0)


def test_odd_lattice_window_wrap_all_mesons():
    """V3 = 30 (not a multiple of the 16-site tile), source at t0 = 4 with a
    5-slice window that wraps through t = 0, explicit momentum list, every
    meson block and the nucleon."""
    ctx = p2.Context((3, 5, 2, 6))
    bufs = device_props(ctx, [(7, 0), (7, 1)], t0=4)
    what = NUC | MES
    src = (1, 3, 1, 4)
    moms = np.array([[0, 0, 0], [1, 0, 0], [0, -2, 1], [1, 1, 1], [-1, 2, 0]], dtype=np.int32)
    out, moms = run(ctx, bufs, src, 5, what, moms=moms)
    taus = list(range(5))
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(out, what, 5, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


def test_config_plain_gpu_24():
    """24^3 x 48, independent u and d, t0 from the seed, nucleon + 16x16
    mesons, |n|^2 <= 9 (123 momenta); oracle on a subset of slices."""
    ctx = p2.Context((24, 24, 24, 48))
    rng = np.random.default_rng(1002)
    t0 = int(rng.integers(0, 48))
    src = (int(rng.integers(0, 24)), int(rng.integers(0, 24)), int(rng.integers(0, 24)), t0)
    bufs = device_props(ctx, [(1002, 0), (1002, 1)], t0=t0)
    what = NUC | p2.MESON_G16
    out, moms = run(ctx, bufs, src, 48, what, q2max=9)
    assert len(moms) == 123
    taus = [0, 1, 23, 47]
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(out, what, 48, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


def test_host_propagators_and_host_output_match_device(ctx_small):
    ctx = ctx_small
    bufs = device_props(ctx, [(11, 0), (11, 1)], t0=3)
    what = NUC | p2.MESON_G16
    a, moms = run(ctx, bufs, (1, 2, 3, 3), 8, what, q2max=3)
    b, _ = run(ctx, bufs, (1, 2, 3, 3), 8, what, q2max=3, host_props=True, host_out=True)
    assert np.array_equal(a, b)
    c, _ = run(ctx, bufs, (1, 2, 3, 3), 8, what, q2max=3)
    assert np.array_equal(a, c)  # bitwise reproducible


def test_window_views(ctx_small):
    """Propagators stored only for the window slices (t_first = t0, nt = window)."""
    ctx = ctx_small
    t0, W = 6, 5  # slices 6, 7, 0, 1, 2
    full = device_props(ctx, [(21, 0), (21, 1)], t0=t0)
    win = device_props(ctx, [(21, 0), (21, 1)], t0=t0, t_first=t0, nt=W)
    a, moms = run(ctx, full, (0, 1, 2, t0), W, NUC | p2.MESON_G16, q2max=1)
    b, _ = run(ctx, win, (0, 1, 2, t0), W, NUC | p2.MESON_G16, q2max=1, t_first=t0, nt=W)
    assert np.array_equal(a, b)


def test_position_space_matches_oracle():
    import oracle_py as orc
    ctx = p2.Context((3, 4, 2, 4))
    bufs = device_props(ctx, [(31, 0), (31, 1)], t0=1)
    what = NUC | p2.MESON_G16
    K = p2.components(what)
    out = torch.zeros(4 * K * ctx.V3, dtype=torch.complex128, device="cuda")
    props = [ctx.prop(b.data_ptr(), nt=4) for b in bufs]
    req = ctx.request((0, 0, 0, 1), 4, what, out.data_ptr())
    ctx.contract_position(props, req)
    ctx.sync()
    u = bufs[0].cpu().numpy().reshape(144, -1)
    d = bufs[1].cpu().numpy().reshape(144, -1)
    _, _, pos = orc.twopt(ctx.L, u, d, (0, 0, 0, 1), [[0, 0, 0]], what, [0, 1, 2, 3], want_pos=True)
    g = out.cpu().numpy().reshape(4, K, ctx.V3)
    scale = np.abs(pos).max()
    assert np.abs(g - pos).max() / scale < 1e-13
    ctx.close()


def test_ft_apply_matches_oracle():
    import oracle_py as orc
    ctx = p2.Context((4, 3, 5, 3))
    dof, nt = 7, 3
    rng = np.random.default_rng(5)
    f = rng.standard_normal((dof, ctx.V3 * nt)) + 1j * rng.standard_normal((dof, ctx.V3 * nt))
    fd = torch.from_numpy(f.reshape(-1)).cuda()
    moms = p2.mom_list(4)
    for sign in (-1, 1):
        out = np.zeros(nt * dof * len(moms), dtype=np.complex128)
        ctx.ft_apply(fd.data_ptr(), dof, nt, moms, sign, out.ctypes.data, p2.P2_HOST)
        ref = orc.ft(ctx.L, f, dof, nt, moms, sign)
        assert np.abs(out.reshape(ref.shape) - ref).max() / np.abs(ref).max() < 1e-13
    ctx.close()


def test_invalid_requests_return_status(ctx_small):
    ctx = ctx_small
    (u,) = device_props(ctx, [(1, 0)], t0=0)
    p = ctx.prop(u.data_ptr(), nt=8)
    out = torch.zeros(16, dtype=torch.complex128, device="cuda")
    with pytest.raises(p2.P2Error) as e:
        ctx.contract_project([p, p], [ctx.request((0, 0, 0, 0), 9, NUC, out.data_ptr(), q2max=0)])
    assert e.value.status == p2.P2_ERR_INVALID_ARG
    f32 = ctx.prop(u.data_ptr(), precision=p2.P2_FP32, nt=8)
    with pytest.raises(p2.P2Error) as e:
        ctx.contract_project([f32, f32], [ctx.request((0, 0, 0, 0), 8, NUC, out.data_ptr(), q2max=0)])
    assert e.value.status == p2.P2_ERR_UNSUPPORTED
    # the context stays usable after errors
    (u2,) = device_props(ctx, [(2, 0)], t0=0)
    run(ctx, [u2, u2], (0, 0, 0, 0), 8, NUC, q2max=0)


def test_delta_all_isospins_plain():
    """Delta C g_k, k = 1..3, isospin 1/2 and 3/2, both datasets, with the
    nucleon and the 16x16 mesons in the same request (the batched
    configuration's contraction set, K = 480)."""
    ctx = p2.Context((4, 3, 5, 6))
    bufs = device_props(ctx, [(41, 0), (41, 1)], t0=2)
    what = NUC | p2.DELTA_ISO12 | p2.DELTA_ISO32 | p2.MESON_G16
    assert p2.components(what) == 480
    out, moms = run(ctx, bufs, (1, 2, 3, 2), 6, what, q2max=2)
    taus = list(range(6))
    ref = oracle_blocks(ctx.L, bufs, (1, 2, 3, 2), moms, what, taus)
    err = per_t_error(out, what, 6, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


@pytest.mark.parametrize("what", [p2.DELTA_ISO12, p2.DELTA_ISO32])
@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_delta_single_isospin(what, mode):
    """One Delta isospin block alone (the other block's slots are not part of
    the result), both forms."""
    ctx = p2.Context((3, 4, 5, 6))
    bufs = device_props(ctx, [(43, 0), (43, 1)], t0=1)
    out, moms = run(ctx, bufs, (2, 1, 0, 1), 6, what, q2max=1, mode=mode)
    taus = list(range(6))
    ref = oracle_blocks(ctx.L, bufs, (2, 1, 0, 1), moms, what, taus)
    err = per_t_error(out, what, 6, moms, ref, taus)
    assert err.max() < (TOL if mode == p2.P2_PLAIN_FP64 else 1e-6), err
    ctx.close()


LIGHT = p2.NUCLEON_NTOR | p2.NUCLEON_RTON | p2.NUCLEON_RTOR


@pytest.mark.parametrize("what", [LIGHT, NUC | LIGHT | p2.DELTA_ISO12 | p2.MESON_G16, p2.NUCLEON_RTOR])
@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_second_nucleon_interpolator(what, mode):
    """NtoR, RtoN, RtoR (the reference's light-baryon build), alone and mixed
    with the other blocks, both forms."""
    ctx = p2.Context((4, 3, 2, 6))
    bufs = device_props(ctx, [(45, 0), (45, 1)], t0=3)
    out, moms = run(ctx, bufs, (1, 2, 1, 3), 6, what, q2max=2, mode=mode)
    taus = list(range(6))
    ref = oracle_blocks(ctx.L, bufs, (1, 2, 1, 3), moms, what, taus)
    err = per_t_error(out, what, 6, moms, ref, taus)
    assert err.max() < (TOL if mode == p2.P2_PLAIN_FP64 else 1e-6), err
    ctx.close()


@pytest.mark.parametrize("decay", [0.0, 40.0])
def test_ft_apply_split_matches_oracle(decay):
    """p2_ft_apply_split (tensor-core projection): error per (t, component,
    momentum) <= 1e-6 of sum_x |f(x, t)| of the component, both signs, host
    and device output; with decay 40 the slices span 1e-35 .. 1, which the
    per-slice power-of-two scale keeps inside FP32's range.  The known answer
    of the reference's FT test (plegma/FT.cpp:18-34): a unit field gives
    V3 at p = 0 and 0 elsewhere."""
    import oracle_py as orc
    ctx = p2.Context((4, 6, 5, 3))
    dof, nt = 21, 3
    rng = np.random.default_rng(6)
    f = rng.standard_normal((dof, ctx.V3 * nt)) + 1j * rng.standard_normal((dof, ctx.V3 * nt))
    f *= np.exp(-decay * np.repeat(np.arange(nt), ctx.V3))[None, :]
    fd = torch.from_numpy(f.reshape(-1)).cuda()
    moms = p2.mom_list(5)
    asum = np.abs(f).reshape(dof, nt, ctx.V3).sum(axis=2).T  # [t][dof]
    for sign in (-1, 1):
        ref = orc.ft(ctx.L, f, dof, nt, moms, sign)
        out = np.zeros(nt * dof * len(moms), dtype=np.complex128)
        ctx.ft_apply(fd.data_ptr(), dof, nt, moms, sign, out.ctypes.data, p2.P2_HOST, mode=p2.P2_SPLIT_FP16)
        err = np.abs(out.reshape(ref.shape) - ref).max(axis=2) / asum
        assert err.max() < 1e-6, err.max()
        outd = torch.zeros(nt * dof * len(moms), dtype=torch.complex128, device="cuda")
        ctx.ft_apply(fd.data_ptr(), dof, nt, moms, sign, outd.data_ptr(), mode=p2.P2_SPLIT_FP16)
        ctx.sync()
        assert np.array_equal(outd.cpu().numpy(), out)
    one = torch.ones(ctx.V3 * nt, dtype=torch.complex128, device="cuda")
    out = np.zeros(nt * len(moms), dtype=np.complex128)
    ctx.ft_apply(one.data_ptr(), 1, nt, moms, -1, out.ctypes.data, p2.P2_HOST, mode=p2.P2_SPLIT_FP16)
    out = out.reshape(nt, len(moms))
    assert np.abs(out[:, 0] - ctx.V3).max() < 1e-6 * ctx.V3 and np.abs(out[:, 1:]).max() < 1e-6 * ctx.V3
    ctx.close()


def test_ft_apply_split_odd_volume():
    import oracle_py as orc
    ctx = p2.Context((3, 5, 3, 2))  # V3 = 45
    dof, nt = 5, 2
    rng = np.random.default_rng(8)
    f = rng.standard_normal((dof, ctx.V3 * nt)) + 1j * rng.standard_normal((dof, ctx.V3 * nt))
    fd = torch.from_numpy(f.reshape(-1)).cuda()
    moms = p2.mom_list(3)
    ref = orc.ft(ctx.L, f, dof, nt, moms, -1)
    out = np.zeros(nt * dof * len(moms), dtype=np.complex128)
    ctx.ft_apply(fd.data_ptr(), dof, nt, moms, -1, out.ctypes.data, p2.P2_HOST, mode=p2.P2_SPLIT_FP16)
    asum = np.abs(f).reshape(dof, nt, ctx.V3).sum(axis=2).T
    assert (np.abs(out.reshape(ref.shape) - ref).max(axis=2) / asum).max() < 1e-6
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_window_outside_the_views_is_empty(ctx_small, mode):
    """Views that store none of the request's window slices (the reference
    skips slices outside its time slab the same way): the call succeeds,
    launches nothing and leaves the result untouched; a window that overlaps
    the views in part fills exactly the overlapping slices."""
    ctx = ctx_small
    T = ctx.L[3]
    bufs = device_props(ctx, [(23, 0), (23, 1)], t0=2, t_first=5, nt=2)  # slices 5, 6
    what = NUC | p2.MESON_G16
    out, moms = run(ctx, bufs, (1, 0, 2, 1), 3, what, q2max=1, mode=mode, t_first=5, nt=2)  # slices 1, 2, 3
    assert not np.any(out)
    out, moms = run(ctx, bufs, (1, 0, 2, 4), 3, what, q2max=1, mode=mode, t_first=5, nt=2)  # slices 4, 5, 6
    g = p2.result_blocks(what, 3, len(moms), out)
    for bit in g:
        assert not np.any(g[bit][:, :, 0]), bit  # tau 0 = slice 4: not stored
        assert np.all(np.any(g[bit][:, :, 1:] != 0, axis=(-1, -2))), bit
    assert T == 8
