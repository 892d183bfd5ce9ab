"""Spin/colour algebra for the hadron two-point contractions, derived from the
gamma-matrix definitions (no tables are copied from the reference).

Basis
-----
PLEGMA works in the Euclidean Dirac--Pauli basis (lib/kernels/PLEGMA_gammas.cuh:6-41,
python/baryons.py:36-54):

    gamma_k = i * [[0, sigma_k], [-sigma_k, 0]]   (k = 1, 2, 3)
    gamma_4 = diag(1, 1, -1, -1)
    gamma_5 = gamma_1 gamma_2 gamma_3 gamma_4
    C       = i gamma_2 gamma_4                    (python/baryons.py:58)

Every table the kernels need is computed here from those four matrices:

* the 16 Dirac structures in PLEGMA's order (1, g1..g4, g5, g5g1..g5g4,
  -i/2[g1,g2], -i/2[g1,g3], -i/2[g2,g3], -i/2[g4,g1], -i/2[g4,g2], -i/2[g4,g3]),
  each as a signed permutation (every one has exactly one non-zero per row);
* the diquark spin tables for the nucleon (C g5 x C g5-bar,
  PLEGMA_baryons_NtoN.cu:3-4) and the Delta (C g_k x C g_k-bar,
  PLEGMA_baryons_deltas.cu:3-4), Gamma-bar = g4 Gamma^dagger g4;
* the Levi-Civita permutation list in the order PLEGMA sums it
  (PLEGMA_kernel_utils.cuh:49-56);
* the momentum list in `createMom` order (lib/PLEGMA_FT.cu:50-72).

`emit_header()` writes these as constexpr tables for the CUDA sources.
"""
from __future__ import annotations

import hashlib
import itertools
import json
from typing import List, Tuple

import numpy as np

I = 1j
NS = 4
NC = 3

_s = [np.array([[0, 1], [1, 0]], dtype=complex),
      np.array([[0, -I], [I, 0]], dtype=complex),
      np.array([[1, 0], [0, -1]], dtype=complex)]
_z = np.zeros((2, 2), dtype=complex)
_e = np.eye(2, dtype=complex)


def _blk(a, b, c, d):
    return np.block([[a, b], [c, d]])


G1 = I * _blk(_z, _s[0], -_s[0], _z)
G2 = I * _blk(_z, _s[1], -_s[1], _z)
G3 = I * _blk(_z, _s[2], -_s[2], _z)
G4 = _blk(_e, _z, _z, -_e)
ONE = np.eye(4, dtype=complex)
G5 = G1 @ G2 @ G3 @ G4
CMAT = I * G2 @ G4
GK = [G1, G2, G3]


def bar(m: np.ndarray) -> np.ndarray:
    """Dirac adjoint of a source structure: g4 M^dagger g4."""
    return G4 @ m.conj().T @ G4


def _sigma(a, b):
    return -0.5 * I * (a @ b - b @ a)


#: The 16 structures in the order of PLEGMA_gammas.cuh (and the GAMMAS enum).
GAMMA16 = [ONE, G1, G2, G3, G4, G5, G5 @ G1, G5 @ G2, G5 @ G3, G5 @ G4,
           _sigma(G1, G2), _sigma(G1, G3), _sigma(G2, G3),
           _sigma(G4, G1), _sigma(G4, G2), _sigma(G4, G3)]
GAMMA16_NAMES = ["1", "g1", "g2", "g3", "g4", "g5", "g5g1", "g5g2", "g5g3", "g5g4",
                 "s12", "s13", "s23", "s41", "s42", "s43"]

CG5 = CMAT @ G5
CGK = [CMAT @ g for g in GK]
P_PLUS = 0.5 * (ONE + G4)
P_MINUS = 0.5 * (ONE - G4)


def signed_permutation(m: np.ndarray) -> Tuple[List[int], List[complex]]:
    """Row r of `m` has its only non-zero at column perm[r] with value phase[r]."""
    perm, phase = [], []
    for r in range(NS):
        nz = [c for c in range(NS) if abs(m[r, c]) > 1e-12]
        if len(nz) != 1:
            raise ValueError("not a signed permutation")
        perm.append(nz[0])
        phase.append(complex(np.round(m[r, nz[0]], 12)))
    return perm, phase


def gamma16_tables():
    """(perm[16][4], re[16][4], im[16][4]) of the 16 Dirac structures."""
    perms, res, ims = [], [], []
    for g in GAMMA16:
        p, v = signed_permutation(g)
        perms.append(p)
        res.append([int(round(x.real)) for x in v])
        ims.append([int(round(x.imag)) for x in v])
    return perms, res, ims


def diquark_table(gamma: np.ndarray):
    """Spin table of a baryon two-point function with interpolator
    eps_abc (q1_a^T Gamma q2_b) q3_c at the sink and its adjoint at the source.

    Entries (nu, lambda, lambda', nu', value) with value = Gamma[nu][lambda] *
    Gamma-bar[lambda'][nu'], enumerated over the non-zeros of Gamma (row major)
    and then of Gamma-bar (row major).  The value is real for C g5 and C g_k.
    """
    gb = bar(gamma)
    rows = []
    for nu, lu in itertools.product(range(NS), range(NS)):
        if abs(gamma[nu, lu]) < 1e-12:
            continue
        for lup, nup in itertools.product(range(NS), range(NS)):
            if abs(gb[lup, nup]) < 1e-12:
                continue
            v = gamma[nu, lu] * gb[lup, nup]
            if abs(v.imag) > 1e-12:
                raise ValueError("complex diquark weight")
            rows.append((nu, lu, lup, nup, int(round(v.real))))
    return rows


def nucleon_table():
    return diquark_table(CG5)


def mixed_diquark_table(ga: np.ndarray, gb: np.ndarray):
    """As diquark_table with G_A at the sink and G_B at the source:
    entries (nu, lambda, lambda', nu', G_A[nu][lambda] G_B-bar[lambda'][nu'])."""
    gbb = bar(gb)
    rows = []
    for nu, lu in itertools.product(range(NS), range(NS)):
        if abs(ga[nu, lu]) < 1e-12:
            continue
        for lup, nup in itertools.product(range(NS), range(NS)):
            if abs(gbb[lup, nup]) < 1e-12:
                continue
            v = ga[nu, lu] * gbb[lup, nup]
            if abs(v.imag) > 1e-12:
                raise ValueError("complex diquark weight")
            rows.append((nu, lu, lup, nup, int(round(v.real))))
    return rows


# Second nucleon interpolator of the reference's light-baryon build:
#   N = eps_abc (u_a^T C g5 d_b) u_c,   R = eps_abc (u_a^T C d_b) g5 u_c.
# NtoR, RtoN, RtoR (lib/kernels/PLEGMA_baryons_NtoR.cu, _RtoN.cu, _RtoR.cu)
# are nucleon-type contractions with G_A / G_B = C g5 or C and a g5 on the open
# spin of the third quark at the sink (R at the sink) and/or the source (R at
# the source).  Their tables, in the reference's column order:
#   NtoR (nu, lambda, lambda', nu', mu', rho): w_AB * g5[rho][mu']
#   RtoN (nu, lambda, lambda', nu', mu, rho):  w_AB * g5[mu][rho]
#   RtoR (nu, lambda, lambda', nu', mu, rho, mu', rho'): w_AB g5[mu][rho] g5[rho'][mu']
def _g5_pairs(transposed: bool):
    out = []
    for a in range(NS):
        for b in range(NS):
            v = G5[b, a] if transposed else G5[a, b]
            if abs(v) > 1e-12:
                out.append((a, b, int(round(v.real))))
    return out


def light_nucleon_tables():
    """{'NtoR': rows, 'RtoN': rows, 'RtoR': rows}, each row the index columns + value."""
    out = {}
    for name, ga, gb in (("NtoR", CG5, CMAT), ("RtoN", CMAT, CG5), ("RtoR", CMAT, CMAT)):
        rows = []
        for nu, lu, lup, nup, w in mixed_diquark_table(ga, gb):
            if name == "NtoR":
                for mup, rho, g in _g5_pairs(True):
                    rows.append((nu, lu, lup, nup, mup, rho, w * g))
            elif name == "RtoN":
                for mu, rho, g in _g5_pairs(False):
                    rows.append((nu, lu, lup, nup, mu, rho, w * g))
            else:
                for mu, rho, g1 in _g5_pairs(False):
                    for mup, rhop, g2 in _g5_pairs(True):
                        rows.append((nu, lu, lup, nup, mu, rho, mup, rhop, w * g1 * g2))
        out[name] = rows
    return out


def light_lane_tables():
    """Lane-parallel form of NtoR, RtoN, RtoR: (sink table of C, lane descriptors
    of the (C g5, C), (C, C g5), (C, C) diquark tables, and per lane the g5
    shuffles): lane (mu, mu') takes T_NR from lane (mu, mu' ^ 2), T_RN from
    (mu ^ 2, mu'), T_RR from (mu ^ 2, mu' ^ 2), with the signs
    -g5[mu'^2][mu'], +g5[mu][mu^2], -g5[mu][mu^2] g5[mu'^2][mu'] (the explicit
    signs of the reference's loops)."""
    sink_c = diquark_lane_tables(diquark_table(CMAT))[0]
    lanes = [diquark_lane_tables(mixed_diquark_table(a, b))[1] for a, b in ((CG5, CMAT), (CMAT, CG5), (CMAT, CMAT))]
    signs = []
    for l in range(16):
        mu, mup = l >> 2, l & 3
        assert abs(G5[mup ^ 2, mup]) > 0 and abs(G5[mu, mu ^ 2]) > 0
        s_nr = -int(round(G5[mup ^ 2, mup].real))
        s_rn = int(round(G5[mu, mu ^ 2].real))
        s_rr = -int(round((G5[mu, mu ^ 2] * G5[mup ^ 2, mup]).real))
        signs.append((s_nr, s_rn, s_rr))
    return sink_c, lanes, signs


def transpose_sign(gamma: np.ndarray) -> int:
    """G^{YX} on lane (y', x') equals sign * G^{XY} on lane (x', y'): -1 for an
    antisymmetric diquark matrix (C g5), +1 for a symmetric one (C g_k)."""
    if np.allclose(gamma, gamma.T):
        return 1
    if np.allclose(gamma, -gamma.T):
        return -1
    raise ValueError("diquark matrix is neither symmetric nor antisymmetric")


def delta_tables():
    return [diquark_table(c) for c in CGK]


def diquark_lane_tables(table):
    """Factorised form of a diquark table for the lane-parallel kernels.

    The weight of entry (iA, iB) (sink pair iA, source pair iB) factorises as
    sA[iA] * sB[iB]; the source pairing lambda' <-> nu' is an involution.
    Returns (sink[4][3] = (nu, lambda, sA), lanes[16][8]) where lane
    l = (x' = l >> 2, y' = l & 3) holds
      z1, sA1, sB1  slot-1 terms: Z spin, sB of the pair with lambda' = y',
                    sB of the pair with nu' = y'
      z2, sA2, sB2  slot-2 terms: same with x'
      sN, sL        type-a terms: sB if (x', y') = (nu', lambda') resp.
                    (lambda', nu') of a pair, else 0.
    """
    vals = [r[4] for r in table]
    sB = [vals[iB] for iB in range(4)]
    sA = [vals[iA * 4] * vals[0] for iA in range(4)]
    assert all(vals[a * 4 + b] == sA[a] * sB[b] for a in range(4) for b in range(4)), "weights do not factorise"
    lamp = [table[iB][2] for iB in range(4)]
    nup = [table[iB][3] for iB in range(4)]
    for iB in range(4):  # involution: the pair whose lambda' is nu'(iB) has nu' = lambda'(iB)
        assert nup[lamp.index(nup[iB])] == lamp[iB], "source pairing is not an involution"
    sink = [(table[iA * 4][0], table[iA * 4][1], sA[iA]) for iA in range(4)]
    lanes = []
    for l in range(16):
        x, y = l >> 2, l & 3
        iA1, iB1 = lamp.index(y), nup.index(y)
        iA2, iB2 = lamp.index(x), nup.index(x)
        sN = next((sB[i] for i in range(4) if (nup[i], lamp[i]) == (x, y)), 0)
        sL = next((sB[i] for i in range(4) if (lamp[i], nup[i]) == (x, y)), 0)
        lanes.append((nup[iA1], sB[iA1], sB[iB1], nup[iA2], sB[iA2], sB[iB2], sN, sL))
    return sink, lanes


def levi_civita():
    """The six colour permutations (a, b, c) and their signs, even ones first:
    the cyclic rotations of (0,1,2), then the transpositions (0<->2), (1<->2),
    (0<->1) of the identity.  This is the summation order PLEGMA uses."""
    base = (0, 1, 2)
    even = [tuple(base[(i - k) % 3] for i in range(3)) for k in range(3)]
    odd = []
    for i, j in ((0, 2), (1, 2), (0, 1)):
        p = list(base)
        p[i], p[j] = p[j], p[i]
        odd.append(tuple(p))
    return even + odd, [1, 1, 1, -1, -1, -1]


def create_mom(q2_max: int, dims: int = 3) -> List[Tuple[int, ...]]:
    """Momentum list in the order of PLEGMA_FT::createMom (lib/PLEGMA_FT.cu:50-72):
    by |n|^2 ascending, each component running from +iQ down to -iQ."""
    out = []
    for iq in range(q2_max + 1):
        rng = range(iq, -iq - 1, -1)
        if dims == 3:
            for nx in rng:
                for ny in rng:
                    for nz in rng:
                        if nx * nx + ny * ny + nz * nz == iq:
                            out.append((nx, ny, nz))
        else:
            for nx in rng:
                for ny in rng:
                    for nz in rng:
                        for nt in rng:
                            if nx * nx + ny * ny + nz * nz + nt * nt == iq:
                                out.append((nx, ny, nz, nt))
    return out


def table_digest(rows) -> str:
    """SHA-256 of a table flattened to integers; used to pin tables against
    the reference's without storing them."""
    flat = [int(round(float(x))) for x in np.asarray(rows, dtype=float).ravel()]
    return hashlib.sha256(json.dumps(flat).encode()).hexdigest()


def _c_array(name, ctype, data, fmt="{}"):
    """A brace-initialiser macro P2_INIT_<name> and a constexpr array using it
    (device code declares local constexpr copies from the macro so that fully
    unrolled loops fold every lookup)."""
    arr = np.asarray(data)
    dims = "".join(f"[{d}]" for d in arr.shape)

    def rec(a):
        if a.ndim == 1:
            return "{" + ",".join(fmt.format(int(x)) for x in a) + "}"
        return "{" + ",".join(rec(x) for x in a) + "}"
    macro = "P2_INIT_" + name[1:] if name.startswith("k") else "P2_INIT_" + name
    return (f"#define {macro} {rec(arr)}\n"
            f"static constexpr {ctype} {name}{dims} = {macro};\n")


def gamma_walsh(g: int):
    """Every Gamma is a signed permutation pi_g(d) = d xor m_g whose
    coefficients are a unit phase times a Walsh character:
        Gamma_g[d][d xor m_g] = r_g * (-1)^{popcount(s_g & d)}.
    Returns (m_g, s_g, r_g)."""
    perm, vals = signed_permutation(GAMMA16[g])
    m = perm[0]
    assert all(perm[d] == d ^ m for d in range(4))
    r = vals[0]
    s = (1 if abs(vals[1] + r) < 1e-12 else 0) | (2 if abs(vals[2] + r) < 1e-12 else 0)
    for d in range(4):
        assert abs(vals[d] - r * (-1) ** bin(s & d).count("1")) < 1e-12, (g, d)
    return m, s, r


def meson_lane_table():
    """Sink-Gamma stage of the lane-parallel mesons as a Walsh-Hadamard transform.

    Lane l = (a, d) = (l >> 2, l & 3) belongs to class m = a xor d; a 4-point
    transform over the lanes of its class (xor masks 5 and 10) leaves on it
    sum_d' (-1)^{popcount(d & d')} N(d'), which by the factorisation of
    gamma_walsh is C[g] / r_g for the Gamma g of class m with s_g = d.
    Returns per lane (g, Re r_g, Im r_g)."""
    lanes = []
    for l in range(16):
        a, d = l >> 2, l & 3
        found = [g for g in range(16) if gamma_walsh(g)[:2] == (a ^ d, d)]
        assert len(found) == 1, (l, found)
        g = found[0]
        r = gamma_walsh(g)[2]
        lanes.append([g, int(round(r.real)), int(round(r.imag))])
    assert sorted(x[0] for x in lanes) == list(range(16))
    return lanes


def header_text() -> str:
    perms, res, ims = gamma16_tables()
    nuc = nucleon_table()
    dl = delta_tables()
    eps, sgn = levi_civita()
    out = ["// Generated by plegma_b200/spin.py from the gamma-matrix definitions.\n",
           "// Do not edit: rerun `python -m plegma_b200.spin` instead.\n",
           "#pragma once\n", "namespace p2 {\n",
           _c_array("kGammaPerm", "int", perms),
           _c_array("kGammaRe", "int", res),
           _c_array("kGammaIm", "int", ims),
           _c_array("kNucIdx", "int", [r[:4] for r in nuc]),
           _c_array("kNucVal", "int", [r[4] for r in nuc]),
           _c_array("kDeltaIdx", "int", [[r[:4] for r in t] for t in dl]),
           _c_array("kDeltaVal", "int", [[r[4] for r in t] for t in dl]),
           _c_array("kNucSink", "int", diquark_lane_tables(nuc)[0]),
           _c_array("kNucLane", "int", diquark_lane_tables(nuc)[1]),
           _c_array("kDeltaSink", "int", [diquark_lane_tables(t)[0] for t in dl]),
           _c_array("kDeltaLane", "int", [diquark_lane_tables(t)[1] for t in dl]),
           _c_array("kMesonLane", "int", meson_lane_table()),
           _c_array("kNtrIdx", "int", [r[:6] for r in light_nucleon_tables()["NtoR"]]),
           _c_array("kNtrVal", "int", [r[6] for r in light_nucleon_tables()["NtoR"]]),
           _c_array("kRtnIdx", "int", [r[:6] for r in light_nucleon_tables()["RtoN"]]),
           _c_array("kRtnVal", "int", [r[6] for r in light_nucleon_tables()["RtoN"]]),
           _c_array("kRtrIdx", "int", [r[:8] for r in light_nucleon_tables()["RtoR"]]),
           _c_array("kRtrVal", "int", [r[8] for r in light_nucleon_tables()["RtoR"]]),
           _c_array("kCSink", "int", light_lane_tables()[0]),
           _c_array("kLightLane", "int", light_lane_tables()[1]),
           _c_array("kLightG5", "int", light_lane_tables()[2]),
           _c_array("kCTransposeSign", "int", [transpose_sign(CMAT)]),
           _c_array("kEps", "int", eps),
           _c_array("kEpsSign", "int", sgn),
           "}  // namespace p2\n"]
    return "".join(out)


def emit_header(path: str) -> bool:
    """Write the generated table header; returns True if the file changed."""
    text = header_text()
    try:
        with open(path) as f:
            if f.read() == text:
                return False
    except FileNotFoundError:
        pass
    with open(path, "w") as f:
        f.write(text)
    return True


if __name__ == "__main__":
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    emit_header(os.path.join(here, "csrc", "spin_tables.h"))
