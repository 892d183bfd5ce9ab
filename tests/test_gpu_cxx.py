"""The C++ drop-in surface (include/plegma/PLEGMA_2pt.h), used by a driver
written like the reference's plegma/Calc_2pt.cpp, checked against the
oracle: reference buffer layouts (including the time rotation of a window
that wraps through t = 0), the binary/JSON writer, the ASCII writer, the
position-space correlator and PLEGMA_FT::apply."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from plegma_b200 import lib as p2

from p2test import device_props, oracle_blocks

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cxx", "_build", "calc_2pt")
L = (6, 4, 4, 8)
SRC = (1, 2, 3, 5)
TOTALT = 6
Q2 = 2


@pytest.fixture(scope="module")
def outputs(tmp_path_factory):
    if not os.path.exists(EXE):
        pytest.fail("tests/cxx/_build/calc_2pt is missing: run __graft_entry__.build()")
    d = tmp_path_factory.mktemp("cxx")
    prefix = str(d / "run")
    args = [EXE] + [str(x) for x in L + SRC] + [str(TOTALT), str(Q2), "0", prefix]
    subprocess.run(args, check=True, timeout=300)
    ctx = p2.Context(L)
    bufs = device_props(ctx, [(2024, 0), (2024, 1)], t0=SRC[3])
    moms = p2.mom_list(Q2)
    yield prefix, ctx, bufs, moms
    ctx.close()


def load(prefix):
    with open(prefix + ".json") as f:
        meta = json.load(f)
    raw = np.fromfile(prefix + ".bin", dtype=np.float64)
    return meta, raw[0::2] + 1j * raw[1::2]


def test_synthetic_fill_matches(outputs):
    prefix, ctx, bufs, _ = outputs
    up = np.fromfile(prefix + "_up.bin", dtype=np.float64)
    up = up[0::2] + 1j * up[1::2]
    assert np.array_equal(up, bufs[0].cpu().numpy())


def test_mesons_all_layout_and_values(outputs):
    prefix, ctx, bufs, moms = outputs
    meta, v = load(prefix + "_mesons_all")
    assert meta["shape"] == [TOTALT, len(moms), 34, 2]
    assert meta["datasets"] == ["mesons/twop_meson"]
    assert np.array_equal(np.array(meta["mvec"]), moms)
    ref = oracle_blocks(L, bufs, SRC, moms, p2.MESON_ALL34, list(range(TOTALT)))[p2.MESON_ALL34][0][0, 0]
    got = v.reshape(TOTALT, len(moms), 34)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12


def test_ascii_writer(outputs):
    prefix, ctx, bufs, moms = outputs
    name = prefix + "_mesons_all_sx%02dsy%02dsz%02dst%02d.dat" % SRC
    lines = open(name).read().strip().split("\n")
    assert len(lines) == TOTALT * len(moms)
    f = lines[len(moms) + 1].split()
    assert [int(x) for x in f[:4]] == [1] + list(moms[1])
    _, v = load(prefix + "_mesons_all")
    got = v.reshape(TOTALT, len(moms), 34)[1, 1, 0]
    assert abs(float(f[4]) - got.real) <= 1e-6 * abs(got) + 1e-300


def test_baryons(outputs):
    prefix, ctx, bufs, moms = outputs
    meta, v = load(prefix + "_baryons")
    assert meta["datasets"] == ["baryons/nucl_nucl/twop_baryon_1", "baryons/nucl_nucl/twop_baryon_2"]
    ref = oracle_blocks(L, bufs, SRC, moms, p2.NUCLEON_CG5, list(range(TOTALT)))[p2.NUCLEON_CG5][0][0]
    got = v.reshape(2, TOTALT, len(moms), 16)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12


def test_mesons10_reference_buffer_layout(outputs):
    """contractMesons keeps the reference's [t][mom][dataset][10] buffer
    (PLEGMA_mesons.cuh:113-120); its writer reads that buffer as
    [dataset][t][mom][10] like the reference's HDF5 writer does."""
    prefix, ctx, bufs, moms = outputs
    meta, v = load(prefix + "_mesons10")
    nm = len(moms)
    # rebuild H_elem from the writer's view, then read it as [slot][mom][ds][10]
    lt = TOTALT
    start = (L[3] - SRC[3]) % L[3]
    start = 0 if start >= TOTALT else start
    per = nm * 10
    h = np.zeros(2 * lt * per, dtype=complex)
    w = v.reshape(2, lt, per)
    for d in range(2):
        for it in range(lt):
            i = (it - start) % TOTALT
            h[(d * lt + i) * per:(d * lt + i + 1) * per] = w[d, it]
    hv = h.reshape(lt, nm, 2, 10)
    ref = oracle_blocks(L, bufs, SRC, moms, p2.MESON_DIAG10, list(range(TOTALT)))[p2.MESON_DIAG10][0][0]
    for i in range(lt):
        tau = (i + start) % TOTALT
        assert np.allclose(hv[i, :, 0, :], ref[0, tau], rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        assert np.allclose(hv[i, :, 1, :], ref[1, tau], rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_position_space_baryons(outputs):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    prefix, ctx, bufs, _ = outputs
    meta, v = load(prefix + "_baryons_pos")
    V3 = L[0] * L[1] * L[2]
    assert meta["shape"] == [TOTALT, V3, 16, 2]
    u = bufs[0].cpu().numpy().reshape(144, -1)
    d = bufs[1].cpu().numpy().reshape(144, -1)
    _, _, pos = orc.twopt(L, u, d, SRC, [[0, 0, 0]], p2.NUCLEON_CG5, list(range(TOTALT)), want_pos=True)
    got = v.reshape(2, TOTALT, V3, 16)
    ref = pos.reshape(TOTALT, 2, 16, V3).transpose(1, 0, 3, 2)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-13


def test_ft_apply(outputs):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    prefix, ctx, bufs, moms = outputs
    raw = np.fromfile(prefix + "_ft_up.bin", dtype=np.float64)
    got = (raw[0::2] + 1j * raw[1::2]).reshape(L[3], 144, len(moms))
    u = bufs[0].cpu().numpy()
    ref = orc.ft(L, u.reshape(144, -1), 144, L[3], moms, -1)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-13
    # FT_SPLIT: error per (t, component, momentum) within 1e-6 of sum_x |u|
    raw = np.fromfile(prefix + "_ft_up_split.bin", dtype=np.float64)
    got = (raw[0::2] + 1j * raw[1::2]).reshape(L[3], 144, len(moms))
    asum = np.abs(u.reshape(144, L[3], -1)).sum(axis=2).T
    assert (np.abs(got - ref).max(axis=2) / asum).max() < 1e-6


def test_udsc_through_the_drop_in(outputs):
    """contractBaryonsUDSC with s and c not allocated: the 28 light datasets,
    empty shape, values equal to the C ABI's on the same propagators."""
    import torch
    prefix, ctx, bufs, moms = outputs
    meta, v = load(prefix + "_udsc")
    req = ctx.udsc_request(SRC, TOTALT, 0, moms=moms, prop_u=0, prop_d=1)
    names = p2.udsc_datasets(req)
    assert meta["shape"] == [TOTALT, len(moms), 2]
    assert meta["datasets"] == ["/" + n for n in names]
    out = torch.zeros(len(names) * TOTALT * len(moms), dtype=torch.complex128, device="cuda")
    req.out = out.data_ptr()
    ctx.contract_udsc([ctx.prop(b.data_ptr()) for b in bufs], req)
    ctx.sync()
    assert np.array_equal(v, out.cpu().numpy())


def test_propagator_preprocessing(outputs):
    """rotateToPhysicalBase_device(+1), applyBoundaries_device(t0) and
    apply_gamma5 against the oracle's restatement; the baryons of the field
    transformed in place equal those of the same transforms applied on load."""
    import oracle_py as orc
    prefix, ctx, bufs, _ = outputs
    rot = np.fromfile(prefix + "_rot.bin", dtype=np.float64)
    rot = (rot[0::2] + 1j * rot[1::2]).reshape(144, -1)
    xf = p2.PROP_ROTATE_PLUS | p2.PROP_BOUNDARY | p2.PROP_GAMMA5
    ref = orc.prop_transform(bufs[0].cpu().numpy(), ctx.V3, 0, L[3], L[3], xf, SRC[3])
    assert np.abs(rot - ref).max() <= 1e-15 * np.abs(ref).max()
    _, a = load(prefix + "_baryons_rot")
    _, b = load(prefix + "_baryons_lazy")
    assert np.array_equal(a, b)


def test_absorb(outputs):
    """PLEGMA_Propagator::absorb of twelve PLEGMA_Vector fields, and of a
    PLEGMA_Vector3D into the source slice of a filled propagator."""
    import oracle_py as orc
    prefix, ctx, bufs, _ = outputs
    V = int(np.prod(L))
    V3 = V // L[3]
    raw = np.fromfile(prefix + "_absorb.bin", dtype=np.float64)
    raw = raw[0::2] + 1j * raw[1::2]
    built, sliced = raw[:144 * V].reshape(144, V), raw[144 * V:].reshape(144, V)
    i = np.arange(12 * V)
    expect = np.zeros((144, V), dtype=np.complex128)
    for k in range(12):
        vec = ((i * 7 + k * 13) % 101) / 16.0 - 3.0 + 1j * (((i * 5 + k * 3) % 67) / 8.0)
        expect = orc.prop_absorb(expect, vec, V3, 0, L[3], L[3], k // 3, k % 3)
    assert np.array_equal(built, expect)
    j = np.arange(12 * V3)
    vec3 = (j % 29) - 14.0 + 1j * ((j % 13) / 4.0)
    (base,) = device_props(ctx, [(5, 0)], t0=0)
    expect = orc.prop_absorb(base.cpu().numpy(), vec3, V3, 0, L[3], L[3], 1, 2, True, SRC[3])
    assert np.array_equal(sliced, expect)


def test_fixed_momentum_vector(outputs):
    """setFixMomVec({1, 0, -1}) (include/PLEGMA_Correlator.h:135-138): one
    momentum, the same values as that momentum of the Q^2 list."""
    prefix, ctx, bufs, moms = outputs
    meta, v = load(prefix + "_baryons_fixmom")
    assert meta["mvec"] == [[1, 0, -1]]
    _, full = load(prefix + "_baryons")
    p = [i for i, m in enumerate(moms.tolist()) if m == [1, 0, -1]][0]
    ref = full.reshape(2, TOTALT, len(moms), 16)[:, :, p, :]
    got = v.reshape(2, TOTALT, 1, 16)[:, :, 0, :]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
