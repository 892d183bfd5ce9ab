"""Spin tables derived from the gamma matrices, pinned against the reference's
own tables through the digests in tests/golden/ref_table_digests.json
(written by tests/golden/make_golden.py from the reference sources)."""
import json
import os

import numpy as np
import pytest

from plegma_b200 import spin

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_table_digests.json")


@pytest.fixture(scope="module")
def digests():
    with open(GOLD) as f:
        return json.load(f)


def test_gamma_tables_match_reference(digests):
    perms, res, ims = spin.gamma16_tables()
    vals = [[[res[g][r], ims[g][r]] for r in range(4)] for g in range(16)]
    inds = [[[r, perms[g][r]] for r in range(4)] for g in range(16)]
    assert spin.table_digest(vals) == digests["gamma_values"]
    assert spin.table_digest(inds) == digests["gamma_indices"]


def test_nucleon_table_matches_reference(digests):
    t = spin.nucleon_table()
    assert spin.table_digest([r[:4] for r in t]) == digests["nucleon_indices"]
    assert spin.table_digest([r[4] for r in t]) == digests["nucleon_values"]


def test_delta_tables_match_reference(digests):
    t = spin.delta_tables()
    assert spin.table_digest([[r[:4] for r in k] for k in t]) == digests["delta_indices"]
    assert spin.table_digest([[r[4] for r in k] for k in t]) == digests["delta_values"]


def test_levi_civita_matches_reference(digests):
    eps, sgn = spin.levi_civita()
    assert spin.table_digest(eps) == digests["eps"]
    assert spin.table_digest(sgn) == digests["sgn_eps"]
    for p, s in zip(eps, sgn):
        # sign = parity of the permutation
        inv = sum(1 for i in range(3) for j in range(i + 1, 3) if p[i] > p[j])
        assert s == (-1) ** inv


def test_clifford_algebra():
    g = [spin.G1, spin.G2, spin.G3, spin.G4]
    for a in range(4):
        for b in range(4):
            ac = g[a] @ g[b] + g[b] @ g[a]
            assert np.allclose(ac, 2 * (a == b) * np.eye(4))
    assert np.allclose(spin.G5 @ spin.G5, np.eye(4))
    # Tr[G_i G_j^dagger] = 4 delta_ij for the 16 structures
    for i, a in enumerate(spin.GAMMA16):
        for j, b in enumerate(spin.GAMMA16):
            assert np.isclose(np.trace(a @ b.conj().T), 4.0 * (i == j))


def test_momentum_counts_and_order():
    assert len(spin.create_mom(2)) == 19
    assert len(spin.create_mom(9)) == 123
    assert len(spin.create_mom(16)) == 257
    m = spin.create_mom(1)
    assert m[0] == (0, 0, 0) and m[1] == (1, 0, 0) and m[-1] == (-1, 0, 0)
    # closed under p -> -p
    s = set(spin.create_mom(9))
    assert all(tuple(-x for x in p) in s for p in s)


def test_generated_header_is_current():
    path = os.path.join(os.path.dirname(spin.__file__), "csrc", "spin_tables.h")
    with open(path) as f:
        assert f.read() == spin.header_text()


@pytest.mark.parametrize("key,name", [("ntor", "NtoR"), ("rton", "RtoN"), ("rtor", "RtoR")])
def test_second_nucleon_interpolator_tables_match_reference(digests, key, name):
    """NtoR, RtoN, RtoR tables (R = eps (u C d) g5 u) in the reference's column order."""
    rows = spin.light_nucleon_tables()[name]
    assert spin.table_digest([r[:-1] for r in rows]) == digests[key + "_indices"]
    assert spin.table_digest([r[-1] for r in rows]) == digests[key + "_values"]


def test_meson_walsh_stage_matches_direct_sum():
    """The lane-parallel Gamma stages of the mesons (site_contract.cuh
    meson_site): per lane (a, d) the Walsh-Hadamard transform over b of
    M[b][b ^ m2], two butterflies over the lanes l ^ 5 and l ^ 10 with the
    signs of d's bits, then lane l holds C[g1][g2] / (r_g1 r_g2) for g1 of
    spin.meson_lane_table; the phase i^q of the deferred form restores it.
    Checked against C[g1][g2] = sum_d G1[d][pi1(d)] sum_b G2[b][pi2(b)]
    M_{pi1(d) d}[b][pi2(b)] on random M."""
    rng = np.random.default_rng(5)
    M = rng.standard_normal((4, 4, 4, 4)) + 1j * rng.standard_normal((4, 4, 4, 4))  # [a][d][b][z]
    G = [np.array(g) for g in spin.GAMMA16]
    direct = np.zeros((16, 16), dtype=complex)
    for g1 in range(16):
        for g2 in range(16):
            p1, v1 = spin.signed_permutation(G[g1])
            p2, v2 = spin.signed_permutation(G[g2])
            direct[g1, g2] = sum(v1[d] * v2[b] * M[p1[d], d, b, p2[b]] for d in range(4) for b in range(4))
    walsh = [spin.gamma_walsh(g) for g in range(16)]
    chi = lambda s, b: (-1) ** bin(s & b).count("1")
    lanes = spin.meson_lane_table()
    emu = np.zeros((16, 16), dtype=complex)
    for g2 in range(16):
        m2, s2, _ = walsh[g2]
        x = np.array([sum(chi(s2, b) * M[l >> 2, l & 3, b, b ^ m2] for b in range(4)) for l in range(16)])
        s0 = np.array([-1 if (l & 1) else 1 for l in range(16)])
        s1 = np.array([-1 if (l & 2) else 1 for l in range(16)])
        x = s0 * x + x[[l ^ 5 for l in range(16)]]
        x = s1 * x + x[[l ^ 10 for l in range(16)]]
        for l in range(16):
            g1 = lanes[l][0]
            assert complex(lanes[l][1], lanes[l][2]) == walsh[g1][2]
            emu[g1, g2] = x[l] * (1j) ** ((spin_phase_q(walsh, g1) + spin_phase_q(walsh, g2)) % 4)
    assert np.allclose(emu, direct, atol=1e-12)


def spin_phase_q(walsh, g):
    """q with r_g = i^q (the deferred phase code of the projection's reduction)."""
    return {1: 0, 1j: 1, -1: 2, -1j: 3}[complex(np.round(walsh[g][2], 12))]
