"""Pins of the CPU oracle (no GPU).

1. Against the reference itself: the reference's NtoN and Delta functions,
   compiled from its sources as host code (oracle/_ref), on random sites.
2. Against an independent numpy statement of the physics (einsum over the
   Levi-Civita tensor and the spin matrices of plegma_b200.spin).
3. Known answers of the projection (plegma/FT.cpp:18-34): the transform of a
   unit field is V3 * delta_{p,0}; a shifted source multiplies by the
   constant phase (PLEGMA_FT::mulConstMomentumPhases, lib/PLEGMA_FT.cu:164-182).
"""
import itertools
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle_py as orc  # noqa: E402
from plegma_b200 import spin  # noqa: E402

NUC, D12, D32, G16, A34, N10, DG10 = 1, 2, 4, 8, 16, 32, 64

EPS = np.zeros((3, 3, 3))
for (a, b, c), s in zip(*spin.levi_civita()):
    EPS[a, b, c] = s


def rand_site(rng):
    return rng.standard_normal(144) + 1j * rng.standard_normal(144)


def as_tensor(p):
    return p.reshape(4, 4, 3, 3)


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def rng():
    return np.random.default_rng(1234)


def np_nucleon(u, d):
    """tmp[mu][mu'] for both datasets from the physics formula."""
    out = np.zeros((2, 4, 4), dtype=complex)
    for ds, (A, B) in enumerate(((u, d), (d, u))):
        A = as_tensor(A)
        B = as_tensor(B)
        G = spin.CG5
        Gb = spin.bar(spin.CG5)
        # direct: eps eps' G[nu,lu] Gb[lup,nup] B[lu,lup,b,b'] A[nu,nup,a,a'] A[mu,mup,c,c']
        direct = np.einsum("abc,xyz,nl,pq,lpby,nqax,mrcz->mr", EPS, EPS, G, Gb, B, A, A)
        exch = np.einsum("abc,xyz,nl,pq,lpby,nraz,mqcx->mr", EPS, EPS, G, Gb, B, A, A)
        out[ds] = direct - exch
    return out.reshape(32)


def np_meson(u, d, g1, g2):
    S1 = as_tensor(u)
    S2 = as_tensor(d)
    G1 = spin.GAMMA16[g1]
    G2 = spin.GAMMA16[g2]
    # sum_ab Tr[G1 S1_ab G2 S2_ab^dagger]
    return np.einsum("da,abxy,bz,dzxy->", G1, S1, G2, S2.conj())


def test_oracle_nucleon_matches_reference_build(rng):
    if orc.reference() is None:
        pytest.skip("reference contraction library not built here")
    for _ in range(5):
        u, d = rand_site(rng), rand_site(rng)
        a = orc.site(u, d, NUC)
        b = orc.ref_nucleon(u, d)
        assert rel(a, b) < 1e-13


@pytest.mark.parametrize("g", [0, 1, 2])
def test_oracle_delta_matches_reference_build(rng, g):
    if orc.reference() is None:
        pytest.skip("reference contraction library not built here")
    for _ in range(3):
        u, d = rand_site(rng), rand_site(rng)
        a12 = orc.site(u, d, D12).reshape(3, 32)[g]
        a32 = orc.site(u, d, D32).reshape(3, 32)[g]
        assert rel(a12, orc.ref_delta(u, d, 0, g)) < 1e-13
        assert rel(a32, orc.ref_delta(u, d, 1, g)) < 1e-13


def test_oracle_nucleon_matches_physics(rng):
    u, d = rand_site(rng), rand_site(rng)
    assert rel(orc.site(u, d, NUC), np_nucleon(u, d)) < 1e-12


def test_oracle_mesons_match_physics(rng):
    u, d = rand_site(rng), rand_site(rng)
    g16 = orc.site(u, d, G16).reshape(16, 16)
    ref = np.array([[np_meson(u, d, a, b) for b in range(16)] for a in range(16)])
    assert rel(g16, ref) < 1e-12
    # subsets
    a34 = orc.site(u, d, A34)
    assert np.allclose(a34[0], g16[0, 0]) and np.allclose(a34[1], g16[5, 5])
    assert np.allclose(a34[2:18].reshape(4, 4), g16[1:5, 1:5])
    assert np.allclose(a34[18:34].reshape(4, 4), g16[6:10, 6:10])
    m10 = [0, 5, 1, 2, 3, 4, 6, 7, 8, 9]
    n10 = orc.site(u, d, N10)
    assert np.allclose(n10, [g16[g, g] for g in m10])
    dg = orc.site(u, d, DG10)
    uu = orc.site(u, u, G16).reshape(16, 16)
    dd = orc.site(d, d, G16).reshape(16, 16)
    assert np.allclose(dg[:10], [uu[g, g] for g in m10])
    assert np.allclose(dg[10:], [dd[g, g] for g in m10])


def test_pion_is_trace_s_sdagger(rng):
    """(1,1) with u = d is Tr[S S^dagger] = sum |S|^2 (gamma5-hermiticity pion)."""
    u = rand_site(rng)
    c = orc.site(u, u, G16).reshape(16, 16)
    assert np.isclose(c[0, 0], np.sum(np.abs(u) ** 2))


def test_identity_propagator_closed_forms():
    """S = 1_spin x 1_colour at one site: meson (G1,G2) = 3 Tr[G1 G2]."""
    one = np.zeros((4, 4, 3, 3), dtype=complex)
    for s in range(4):
        for c in range(3):
            one[s, s, c, c] = 1
    one = one.reshape(144)
    g = orc.site(one, one, G16).reshape(16, 16)
    for a in range(16):
        for b in range(16):
            assert np.isclose(g[a, b], 3 * np.trace(spin.GAMMA16[a] @ spin.GAMMA16[b]))


def test_ft_unit_field_known_answer():
    L = (4, 3, 5, 2)
    V3 = 60
    dof, nt = 2, 2
    field = np.ones((dof, V3 * nt), dtype=complex)
    moms = np.array(spin.create_mom(2))
    out = orc.ft(L, field, dof, nt, moms, -1)
    expect = np.zeros_like(out)
    expect[:, :, 0] = V3
    assert np.allclose(out, expect, atol=1e-11)


def test_twopt_source_shift_is_constant_phase(rng):
    """Moving the source spatially multiplies C(p) by exp(+i p.dx)."""
    L = (4, 4, 4, 4)
    V3 = 64
    u = rng.standard_normal((144, V3 * 4)) + 1j * rng.standard_normal((144, V3 * 4))
    d = rng.standard_normal((144, V3 * 4)) + 1j * rng.standard_normal((144, V3 * 4))
    moms = np.array(spin.create_mom(2))
    a, _, _ = orc.twopt(L, u, d, (0, 0, 0, 1), moms, NUC, [0, 2])
    b, _, _ = orc.twopt(L, u, d, (1, 2, 3, 1), moms, NUC, [0, 2])
    ph = np.exp(2j * np.pi * (moms @ np.array([1, 2, 3])) / 4)
    assert np.allclose(b, a * ph[None, :, None], rtol=1e-12, atol=1e-10)


def test_twopt_zero_momentum_is_site_sum(rng):
    L = (3, 2, 2, 3)
    V3 = 12
    u = rng.standard_normal((144, V3 * 3)) + 1j * rng.standard_normal((144, V3 * 3))
    d = rng.standard_normal((144, V3 * 3)) + 1j * rng.standard_normal((144, V3 * 3))
    out, asum, pos = orc.twopt(L, u, d, (1, 0, 1, 2), [[0, 0, 0]], NUC | G16, [0, 1, 2], want_pos=True)
    assert np.allclose(out[:, 0, :], pos.sum(axis=2))
    assert np.allclose(asum, np.abs(pos).sum(axis=2))
    # tau -> global slice (t0 + tau) mod T: tau = 1 is slice 0
    s = np.array([orc.site(u[:, x], d[:, x], NUC | G16) for x in range(V3)])
    assert np.allclose(pos[1].T, s)


@pytest.mark.parametrize("which,bit", [(0, 1 << 7), (1, 1 << 8), (2, 1 << 9)])
def test_oracle_second_nucleon_interpolator_matches_reference_build(rng, which, bit):
    """NtoR, RtoN, RtoR of the oracle against the reference's own functions."""
    if orc.reference() is None:
        pytest.skip("reference contraction library not built here")
    for _ in range(3):
        u, d = rand_site(rng), rand_site(rng)
        assert rel(orc.site(u, d, bit), orc.ref_light(u, d, which)) < 1e-13


# ---- mesons and the projection against the reference's own kernels ----------
# The reference's contract_mesons_device (10 diagonal structures of S1 S1^+
# and S2 S2^+), contract_mesons_all_device (34 Gamma pairs) and
# contract_mesons_new_device (10 structures of S1 S2^+), each followed by its
# in-kernel fourier_transform_3D (source-relative phase, sign -1), compiled
# from the reference sources as host code and summed over sites as its host
# driver does.  The lattice is odd and anisotropic and the source is off the
# origin, so a sign or orientation error in the phase or a transposed Gamma
# index shows.

def _meson_case(seed, L=(3, 4, 5, 3)):
    rng = np.random.default_rng(seed)
    V3 = L[0] * L[1] * L[2]
    u = rng.standard_normal((144, V3 * L[3])) + 1j * rng.standard_normal((144, V3 * L[3]))
    d = rng.standard_normal((144, V3 * L[3])) + 1j * rng.standard_normal((144, V3 * L[3]))
    return L, u, d


REF_MESON_KINDS = [(0, DG10), (1, A34), (2, N10)]


@pytest.mark.parametrize("kind,bit", REF_MESON_KINDS)
def test_oracle_mesons_projected_match_reference_kernels(kind, bit):
    if orc.reference() is None:
        pytest.skip("reference contraction library not built here")
    L, u, d = _meson_case(77 + kind)
    src = (2, 1, 3, 1)
    moms = np.array(spin.create_mom(3))
    for j in range(L[3]):
        tau = (j - src[3]) % L[3]
        mine, _, _ = orc.twopt(L, u, d, src, moms, bit, [tau])
        ref = orc.ref_meson_ft(kind, L, u, d, j, src, moms)
        assert rel(mine[0], ref) < 1e-13, (kind, j)


def test_oracle_g16_covers_reference_pairs_projected():
    """The all-pairs block restricted to the reference's 34 pairs and its 10
    diagonal structures equals the reference kernels' projected output."""
    if orc.reference() is None:
        pytest.skip("reference contraction library not built here")
    L, u, d = _meson_case(91)
    src = (1, 3, 0, 2)
    moms = np.array(spin.create_mom(2))
    j = 1
    tau = (j - src[3]) % L[3]
    g16, _, _ = orc.twopt(L, u, d, src, moms, G16, [tau])
    g16 = g16[0].reshape(len(moms), 16, 16)
    a34 = orc.ref_meson_ft(1, L, u, d, j, src, moms)
    mine = np.concatenate([g16[:, 0, 0:1], g16[:, 5, 5:6], g16[:, 1:5, 1:5].reshape(-1, 16),
                           g16[:, 6:10, 6:10].reshape(-1, 16)], axis=1)
    assert rel(mine, a34) < 1e-13
    n10 = orc.ref_meson_ft(2, L, u, d, j, src, moms)
    m10 = [0, 5, 1, 2, 3, 4, 6, 7, 8, 9]
    assert rel(np.stack([g16[:, g, g] for g in m10], axis=1), n10) < 1e-13


def test_reference_projection_sign_and_source_phase():
    """The reference kernel's projection of a field that is nonzero on one
    site x only is exp(-i p.(x - x0)) times the site value: the sign and the
    source-relative origin, read off the reference itself."""
    if orc.reference() is None:
        pytest.skip("reference contraction library not built here")
    L, u, d = _meson_case(5)
    V3 = L[0] * L[1] * L[2]
    x = (2, 3, 1)
    sid = x[0] + L[0] * (x[1] + L[1] * x[2])
    mask = np.zeros(V3 * L[3])
    mask[sid + V3 * 2] = 1.0
    u1, d1 = u * mask, d * mask
    src = (1, 2, 4, 0)
    moms = np.array(spin.create_mom(2))
    ref = orc.ref_meson_ft(2, L, u1, d1, 2, src, moms)
    site_val = orc.ref_meson_ft(2, L, u1, d1, 2, src, [[0, 0, 0]])[0]
    ph = np.exp(-2j * np.pi * sum(moms[:, i] * (x[i] - src[i]) / L[i] for i in range(3)))
    assert rel(ref, ph[:, None] * site_val[None, :]) < 1e-13
    mine, _, _ = orc.twopt(L, u1, d1, src, moms, N10, [2])
    assert rel(mine[0], ref) < 1e-13
