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
