"""Table-driven baryon two-point functions (p2_contract_udsc, the reference's
contractBaryonsUDSC) against the FP64 oracle, which evaluates the reference's
unfactorised per-entry sum (lib/kernels/PLEGMA_baryons_udsc.cu:85-134) over
the same spin tables.  Tolerance: 1e-12 per time slice relative to
sum_x |c_d(x,t)|, for every dataset and momentum."""
import numpy as np
import pytest
import torch

from plegma_b200 import lib as p2
from plegma_b200 import udsc

from p2test import device_props

import oracle_py as orc

pytestmark = pytest.mark.gpu

TOL = 1e-12
TABLES = dict(udsc.products())


def _check(ctx, flav_bufs, src, W, moms, out, req, t_first=0):
    """Compare a flat [dataset][tau][mom] result with the oracle, product by product."""
    names = p2.udsc_datasets(req)
    res = out.reshape(len(names), W, len(moms))
    off = 0
    taus = list(range(W))
    worst = 0.0
    for key, dss in udsc.products():
        if not names[off:off + len(dss)] == [n for n, _, _ in dss]:
            continue
        props = [flav_bufs[c].cpu().numpy().reshape(144, -1) for c in key]
        ref, asum = orc.udsc_twopt(ctx.L, props, src, moms, dss, taus, t_first=t_first)
        got = res[off:off + len(dss)].transpose(1, 0, 2)  # [tau][dataset][mom]
        err = np.abs(got - ref).max(axis=2) / np.maximum(asum, 1e-300)
        worst = max(worst, float(err.max()))
        off += len(dss)
    assert off == len(names), (off, len(names))
    return worst


def test_light_baryons_u_d():
    """u and d only: proton/neutron and Delta sets (products uud, udd, uuu, ddd)."""
    ctx = p2.Context((3, 4, 2, 6))
    src = (1, 2, 0, 4)
    u, d = device_props(ctx, [(71, 0), (71, 1)], t0=src[3])
    moms = p2.mom_list(1)
    W = 5
    req = ctx.udsc_request(src, W, 0, moms=moms, prop_u=0, prop_d=1)
    n = len(p2.udsc_datasets(req))
    assert n == 28
    out = torch.zeros(n * W * len(moms), dtype=torch.complex128, device="cuda")
    req.out = out.data_ptr()
    ctx.contract_udsc([ctx.prop(u.data_ptr()), ctx.prop(d.data_ptr())], req)
    ctx.sync()
    err = _check(ctx, {"u": u, "d": d}, src, W, moms, out.cpu().numpy(), req)
    assert err < TOL, err
    ctx.close()


def test_all_twenty_products_host_output():
    """u, d, s, c all given: the 20 flavour products and 200 datasets, result on the host."""
    ctx = p2.Context((2, 3, 2, 4))
    src = (1, 0, 1, 2)
    bufs = device_props(ctx, [(81, 0), (81, 1), (82, 0), (82, 1)], t0=src[3])
    flav = dict(zip("udsc", bufs))
    moms = np.array([[0, 0, 0], [1, 0, 0], [0, -1, 1]], dtype=np.int32)
    W = 3
    req = ctx.udsc_request(src, W, 0, p2.P2_HOST, moms=moms, prop_u=0, prop_d=1, prop_s=2, prop_c=3)
    n = len(p2.udsc_datasets(req))
    assert n == 200
    out = np.zeros(n * W * len(moms), dtype=np.complex128)
    req.out = out.ctypes.data
    ctx.contract_udsc([ctx.prop(b.data_ptr()) for b in bufs], req)
    err = _check(ctx, flav, src, W, moms, out, req)
    assert err < TOL, err
    ctx.close()


def test_filters_and_window_views():
    """only_st keeps the products with s; a strange propagator stored for the
    window only (t_first = t0, nt = W) gives the same result as a full one."""
    ctx = p2.Context((2, 2, 3, 6))
    src = (0, 1, 2, 5)
    W = 4
    u, d, s_full = device_props(ctx, [(91, 0), (91, 1), (92, 0)], t0=src[3])
    (s_win,) = device_props(ctx, [(92, 0)], t0=src[3], t_first=src[3], nt=W)
    moms = p2.mom_list(1)
    outs = []
    for s_buf, nt in ((s_full, 6), (s_win, W)):
        req = ctx.udsc_request(src, W, 0, moms=moms, prop_u=0, prop_d=1, prop_s=2, only_st=True)
        names = p2.udsc_datasets(req)
        assert all("s" in key for key, dss in udsc.products() for nm, _, _ in dss if nm in names)
        out = torch.zeros(len(names) * W * len(moms), dtype=torch.complex128, device="cuda")
        req.out = out.data_ptr()
        props = [ctx.prop(u.data_ptr()), ctx.prop(d.data_ptr()),
                 ctx.prop(s_buf.data_ptr(), t_first=0 if nt == 6 else src[3], nt=nt)]
        ctx.contract_udsc(props, req)
        ctx.sync()
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    err = _check(ctx, {"u": u, "d": d, "s": s_full}, src, W, moms, outs[0], req)
    assert err < TOL, err
    ctx.close()


def test_udsc_rejects_fp32_plain_and_host_propagators():
    ctx = p2.Context((2, 2, 2, 4))
    (u,) = device_props(ctx, [(5, 0)], t0=0)
    out = torch.zeros(4 * 4, dtype=torch.complex128, device="cuda")
    req = ctx.udsc_request((0, 0, 0, 0), 4, out.data_ptr(), moms=np.zeros((1, 3), np.int32), prop_u=0)
    with pytest.raises(p2.P2Error) as e:
        ctx.contract_udsc([ctx.prop(u.data_ptr(), precision=p2.P2_FP32)], req)
    assert e.value.status == p2.P2_ERR_UNSUPPORTED
    h = u.cpu().pin_memory()
    with pytest.raises(p2.P2Error) as e:
        ctx.contract_udsc([ctx.prop(h.data_ptr(), location=p2.P2_HOST)], req)
    assert e.value.status == p2.P2_ERR_UNSUPPORTED
    ctx.close()


SPLIT_TOL = 1e-6


def test_split_light_baryons_u_d():
    """Split form (FP32 contraction, hi+lo FP16 tensor-core projection): u and
    d, 28 datasets, window wrapping through t = 0."""
    ctx = p2.Context((4, 4, 2, 6))
    src = (1, 2, 0, 4)
    u, d = device_props(ctx, [(73, 0), (73, 1)], t0=src[3])
    moms = p2.mom_list(2)
    W = 5
    req = ctx.udsc_request(src, W, 0, moms=moms, prop_u=0, prop_d=1, mode=p2.P2_SPLIT_FP16)
    n = len(p2.udsc_datasets(req))
    out = torch.zeros(n * W * len(moms), dtype=torch.complex128, device="cuda")
    req.out = out.data_ptr()
    ctx.contract_udsc([ctx.prop(u.data_ptr()), ctx.prop(d.data_ptr())], req)
    ctx.sync()
    err = _check(ctx, {"u": u, "d": d}, src, W, moms, out.cpu().numpy(), req)
    assert err < SPLIT_TOL, err
    ctx.close()


def test_split_all_products_host_output():
    ctx = p2.Context((2, 3, 2, 4))
    src = (1, 0, 1, 2)
    bufs = device_props(ctx, [(83, 0), (83, 1), (84, 0), (84, 1)], t0=src[3])
    flav = dict(zip("udsc", bufs))
    moms = np.array([[0, 0, 0], [1, 0, 0], [0, -1, 1]], dtype=np.int32)
    W = 3
    req = ctx.udsc_request(src, W, 0, p2.P2_HOST, moms=moms, prop_u=0, prop_d=1, prop_s=2, prop_c=3,
                           mode=p2.P2_SPLIT_FP16)
    n = len(p2.udsc_datasets(req))
    assert n == 200
    out = np.zeros(n * W * len(moms), dtype=np.complex128)
    req.out = out.ctypes.data
    ctx.contract_udsc([ctx.prop(b.data_ptr()) for b in bufs], req)
    err = _check(ctx, flav, src, W, moms, out, req)
    assert err < SPLIT_TOL, err
    ctx.close()


def test_split_fp32_propagators_and_transforms():
    """FP32 propagators (split form only), u rotated with s = +1 and d with
    s = -1 plus the boundary sign, applied on load; the oracle runs on the
    host-transformed FP32 entries."""
    ctx = p2.Context((3, 2, 4, 4))
    src = (2, 1, 3, 1)
    u, d = device_props(ctx, [(75, 0), (75, 1)], t0=src[3], precision=p2.P2_FP32)
    xu, xd = p2.PROP_ROTATE_PLUS | p2.PROP_BOUNDARY, p2.PROP_ROTATE_MINUS | p2.PROP_BOUNDARY
    moms = p2.mom_list(1)
    W = 4
    req = ctx.udsc_request(src, W, 0, moms=moms, prop_u=0, prop_d=1, mode=p2.P2_SPLIT_FP16)
    n = len(p2.udsc_datasets(req))
    out = torch.zeros(n * W * len(moms), dtype=torch.complex128, device="cuda")
    req.out = out.data_ptr()
    ctx.contract_udsc([ctx.prop(u.data_ptr(), precision=p2.P2_FP32, transform=xu, boundary_t0=src[3]),
                       ctx.prop(d.data_ptr(), precision=p2.P2_FP32, transform=xd, boundary_t0=src[3])], req)
    ctx.sync()
    hu = torch.from_numpy(orc.prop_transform(u.cpu().numpy().astype(np.complex128), ctx.V3, 0, 4, 4, xu, src[3]))
    hd = torch.from_numpy(orc.prop_transform(d.cpu().numpy().astype(np.complex128), ctx.V3, 0, 4, 4, xd, src[3]))
    err = _check(ctx, {"u": hu, "d": hd}, src, W, moms, out.cpu().numpy(), req)
    assert err < SPLIT_TOL, err
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_odd_spatial_volume(mode):
    ctx = p2.Context((3, 3, 3, 4))  # V3 = 27
    src = (0, 2, 1, 3)
    u, d = device_props(ctx, [(77, 0), (77, 1)], t0=src[3])
    moms = p2.mom_list(1)
    W = 4
    req = ctx.udsc_request(src, W, 0, moms=moms, prop_u=0, prop_d=1, mode=mode)
    n = len(p2.udsc_datasets(req))
    out = torch.zeros(n * W * len(moms), dtype=torch.complex128, device="cuda")
    req.out = out.data_ptr()
    ctx.contract_udsc([ctx.prop(u.data_ptr()), ctx.prop(d.data_ptr())], req)
    ctx.sync()
    err = _check(ctx, {"u": u, "d": d}, src, W, moms, out.cpu().numpy(), req)
    assert err < (TOL if mode == p2.P2_PLAIN_FP64 else SPLIT_TOL), err
    ctx.close()
