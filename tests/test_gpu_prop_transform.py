"""Propagator pre-processing (the reference's rotateToPhysicalBase,
apply_gamma5 and applyBoundaries): applied in place by p2_prop_transform,
and fused into the contractions' staging through p2_prop::transform.  Both
must give the oracle's result on the host-transformed propagators."""
import numpy as np
import pytest
import torch

from plegma_b200 import lib as p2
from plegma_b200 import udsc

from p2test import device_props, oracle_blocks, per_t_error, run

import oracle_py as orc

pytestmark = pytest.mark.gpu

WHAT = p2.NUCLEON_CG5 | p2.MESON_G16 | p2.NUCLEON_RTON | p2.DELTA_ISO32
XFORMS = [p2.PROP_ROTATE_PLUS | p2.PROP_BOUNDARY, p2.PROP_ROTATE_MINUS, p2.PROP_GAMMA5 | p2.PROP_BOUNDARY]


@pytest.mark.parametrize("xf", XFORMS)
def test_in_place_transform_matches_host(xf):
    ctx = p2.Context((3, 2, 4, 6))
    (u,) = device_props(ctx, [(3, 0)], t0=2)
    host = u.cpu().numpy().reshape(144, -1)
    ctx.prop_transform(u.data_ptr(), xf, boundary_t0=4)
    ctx.sync()
    ref = orc.prop_transform(host, ctx.V3, 0, 6, 6, xf, 4)
    assert np.abs(u.cpu().numpy().reshape(144, -1) - ref).max() <= 1e-15 * np.abs(ref).max()
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_fused_transform_matches_oracle(mode):
    """u rotated with s = +1 and d with s = -1 (the twisted-mass doublet) plus the
    boundary sign at the source time, applied on load; a window that wraps."""
    ctx = p2.Context((4, 3, 2, 8))
    src = (1, 2, 0, 5)
    u, d = device_props(ctx, [(61, 0), (61, 1)], t0=src[3])
    xu = p2.PROP_ROTATE_PLUS | p2.PROP_BOUNDARY
    xd = p2.PROP_ROTATE_MINUS | p2.PROP_BOUNDARY
    moms = p2.mom_list(1)
    _, total = p2.block_info(WHAT, 8, len(moms))
    out = torch.zeros(total, dtype=torch.complex128, device="cuda")
    props = [ctx.prop(u.data_ptr(), transform=xu, boundary_t0=src[3]),
             ctx.prop(d.data_ptr(), transform=xd, boundary_t0=src[3])]
    ctx.contract_project(props, [ctx.request(src, 8, WHAT, out.data_ptr(), mode=mode, moms=moms)])
    ctx.sync()
    hu = torch.from_numpy(orc.prop_transform(u.cpu().numpy(), ctx.V3, 0, 8, 8, xu, src[3]).reshape(-1))
    hd = torch.from_numpy(orc.prop_transform(d.cpu().numpy(), ctx.V3, 0, 8, 8, xd, src[3]).reshape(-1))
    taus = list(range(8))
    ref = oracle_blocks(ctx.L, [hu, hd], src, moms, WHAT, taus)
    err = per_t_error(out.cpu().numpy(), WHAT, 8, moms, ref, taus)
    assert err.max() < (1e-12 if mode == p2.P2_PLAIN_FP64 else 1e-6), err
    if mode == p2.P2_PLAIN_FP64:
        # the same bits as transforming the fields in place first
        ctx.prop_transform(u.data_ptr(), xu, src[3])
        ctx.prop_transform(d.data_ptr(), xd, src[3])
        out2 = torch.zeros_like(out)
        ctx.contract_project([ctx.prop(u.data_ptr()), ctx.prop(d.data_ptr())],
                             [ctx.request(src, 8, WHAT, out2.data_ptr(), mode=mode, moms=moms)])
        ctx.sync()
        assert torch.equal(out, out2)
    ctx.close()


def test_fused_transform_in_table_driven_baryons():
    ctx = p2.Context((2, 3, 2, 4))
    src = (0, 1, 1, 2)
    u, d = device_props(ctx, [(62, 0), (62, 1)], t0=src[3])
    xu, xd = p2.PROP_ROTATE_PLUS | p2.PROP_BOUNDARY, p2.PROP_ROTATE_MINUS | p2.PROP_BOUNDARY
    moms = p2.mom_list(1)
    req = ctx.udsc_request(src, 4, 0, moms=moms, prop_u=0, prop_d=1)
    names = p2.udsc_datasets(req)
    out = torch.zeros(len(names) * 4 * len(moms), dtype=torch.complex128, device="cuda")
    req.out = out.data_ptr()
    ctx.contract_udsc([ctx.prop(u.data_ptr(), transform=xu, boundary_t0=src[3]),
                       ctx.prop(d.data_ptr(), transform=xd, boundary_t0=src[3])], req)
    ctx.sync()
    flav = {"u": orc.prop_transform(u.cpu().numpy(), ctx.V3, 0, 4, 4, xu, src[3]),
            "d": orc.prop_transform(d.cpu().numpy(), ctx.V3, 0, 4, 4, xd, src[3])}
    res = out.cpu().numpy().reshape(len(names), 4, len(moms))
    off = 0
    for key, dss in udsc.products():
        if names[off:off + len(dss)] != [n for n, _, _ in dss]:
            continue
        ref, asum = orc.udsc_twopt(ctx.L, [flav[c] for c in key], src, moms, dss, list(range(4)))
        got = res[off:off + len(dss)].transpose(1, 0, 2)
        assert (np.abs(got - ref).max(axis=2) / np.maximum(asum, 1e-300)).max() < 1e-12
        off += len(dss)
    assert off == len(names)
    ctx.close()


def _vec(rng, n, dtype):
    return torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to(dtype).cuda()


@pytest.mark.parametrize("dtype,prec", [(torch.complex128, p2.P2_FP64), (torch.complex64, p2.P2_FP32)])
def test_absorb_matches_host(dtype, prec):
    """The three forms of absorb (whole 4-D vector; one slice of a 4-D vector;
    a 3-D vector into one slice), on a view of 5 slices from t = 3 of T = 6
    (so it wraps) and with the slice outside the view (column zeroed)."""
    ctx = p2.Context((3, 2, 2, 6))
    V3, nt, t_first = ctx.V3, 5, 3
    rng = np.random.default_rng(7)
    prop = _vec(rng, 144 * nt * V3, dtype)
    v4 = _vec(rng, 12 * nt * V3, dtype)
    v3 = _vec(rng, 12 * V3, dtype)
    cases = [(False, -1, 1, 2), (False, 0, 3, 0), (True, 4, 2, 1), (True, 2, 0, 2)]  # t = 2 is not in the view
    for vec_3d, gt, nu, c2 in cases:
        before = prop.cpu().numpy()
        v = v3 if vec_3d else v4
        ctx.prop_absorb(prop.data_ptr(), v.data_ptr(), nu, c2, prec, t_first, nt, vec_3d, gt)
        ctx.sync()
        ref = orc.prop_absorb(before, v.cpu().numpy(), V3, t_first, nt, 6, nu, c2, vec_3d, gt)
        assert np.array_equal(prop.cpu().numpy().astype(np.complex128).reshape(144, -1), ref)
    with pytest.raises(p2.P2Error) as e:
        ctx.prop_absorb(prop.data_ptr(), v3.data_ptr(), 0, 0, prec, t_first, nt, True, 6)
    assert e.value.status == p2.P2_ERR_INVALID_ARG
    ctx.close()


def test_propagator_from_twelve_columns_contracts_the_same():
    """Twelve solver vectors (the columns of a propagator) absorbed one by one
    give the propagator back bit for bit."""
    ctx = p2.Context((2, 2, 4, 4))
    (u,) = device_props(ctx, [(17, 0)], t0=1)
    V = ctx.V3 * 4
    cols = u.view(4, 4, 3, 3, V).permute(1, 3, 0, 2, 4).contiguous()  # [nu][c2][mu][c1][site]
    rebuilt = torch.empty_like(u)
    for nu in range(4):
        for c2 in range(3):
            ctx.prop_absorb(rebuilt.data_ptr(), cols[nu, c2].data_ptr(), nu, c2)
    ctx.sync()
    assert torch.equal(rebuilt, u)
    ctx.close()
