"""Spin tables of the table-driven baryon two-point functions (the reference's
UDSC set: light, strange and charm octet/decuplet baryons with projected
interpolators), restated from the algorithm of the reference's generator
(python/baryons.py:27-543, output lib/kernels/PLEGMA_baryons_udsc_arrays.cuh).

Each baryon interpolator is J = sum_i k_i eps_abc (f1_a^T G_A f2_b) f3_c.  For
the correlator <J(x) Jbar(0)> with a projector P on the open spin of f3:
  1. list the six fields (three quarks with spin/colour slots 0..2, three
     antiquarks of Jbar = (f3bar, f1bar, f2bar) with slots 3..5);
  2. enumerate the Wick contractions (each quark paired with an antiquark of
     the same flavour; the sign is the parity of the pairing);
  3. move every contraction to the default view: propagators ordered by
     flavour (u, d, s, c), propagator k carrying spins (2k, 2k+1) and colours
     (k, 3+k); the colour relabelling multiplies the term by the parity of
     the colour permutation (the eps eps structure is fixed);
  4. for every non-zero (G_A[s0][s1], P[s2][s3], G_B[s4][s5]) the relabelled
     spin tuple collects value x coefficient;
  5. drop zeros and divide by the norm (sum k_i^2 for spin 1/2; 1/3, 1, 1/2
     for spin-3/2 sets of one, two, three flavour strings).
A site then contributes sum_entries w * sum_{eps eps'} P1[s0][s1][a][a']
P2[s2][s3][b][b'] P3[s4][s5][c][c'] (lib/kernels/PLEGMA_baryons_udsc.cu:85-134).

Weights are kept in single precision, as the reference's float2 tables are.
"""
from __future__ import annotations

import itertools
from typing import Dict, List, Tuple

import numpy as np

from . import spin

I = 1j
ONE = np.eye(4, dtype=complex)
GX, GY, GZ, GT = spin.G1, spin.G2, spin.G3, spin.G4
C = I * GY @ GT
G5 = GX @ GY @ GZ @ GT
CG5 = C @ G5
IGTCG5 = I * GT @ CG5
PP = 0.5 * (ONE + GT)
PM = 0.5 * (ONE - GT)
CGX, CGY, CGZ = C @ GX, C @ GY, C @ GZ

# interpolator sets: name -> list of (projector, G_A at the sink, G_B at the source)
SETS = {
    0.5: [
        ("Pp-Cg5-Cg5", [(PP, CG5, CG5)]),
        ("Pm-Cg5-Cg5", [(PM, CG5, CG5)]),
        ("Pp-igtCg5-igtCg5", [(PP, IGTCG5, IGTCG5)]),
        ("Pm-igtCg5-igtCg5", [(PM, IGTCG5, IGTCG5)]),
        ("g5Ppg5-C-C", [(G5 @ PP @ G5, C, C)]),
        ("g5Pmg5-C-C", [(G5 @ PM @ G5, C, C)]),
    ],
    1.5: [
        ("Pp-Cgi-Cgi", [(PP, CGX, CGX), (PP, CGY, CGY), (PP, CGZ, CGZ)]),
        ("Pm-Cgi-Cgi", [(PM, CGX, CGX), (PM, CGY, CGY), (PM, CGZ, CGZ)]),
        ("Ppgigj-Cgi-Cgj", [(PP @ GX @ GY, CGX, CGY), (PP @ GX @ GZ, CGX, CGZ), (PP @ GY @ GZ, CGY, CGZ),
                            (PP @ GY @ GX, CGY, CGX), (PP @ GZ @ GX, CGZ, CGX), (PP @ GZ @ GY, CGZ, CGY)]),
        ("Pmgigj-Cgi-Cgj", [(PM @ GX @ GY, CGX, CGY), (PM @ GX @ GZ, CGX, CGZ), (PM @ GY @ GZ, CGY, CGZ),
                            (PM @ GY @ GX, CGY, CGX), (PM @ GZ @ GX, CGZ, CGX), (PM @ GZ @ GY, CGZ, CGY)]),
    ],
}

# (name, flavour strings f1-f2-f3, coefficients, spin), in the reference's order
BARYONS: List[Tuple[str, List[str], List[int], float]] = [
    ("Xicc++", ["ch-up-ch"], [1], 0.5),
    ("Xicc+", ["ch-dn-ch"], [1], 0.5),
    ("Omegacc+", ["ch-sr-ch"], [1], 0.5),
    ("Sigmac++", ["up-ch-up"], [1], 0.5),
    ("Sigmac+", ["up-ch-dn", "dn-ch-up"], [1, 1], 0.5),
    ("Sigmac0", ["dn-ch-dn"], [1], 0.5),
    ("Xi'c+", ["up-ch-sr", "sr-ch-up"], [1, 1], 0.5),
    ("Xi'c0", ["dn-ch-sr", "sr-ch-dn"], [1, 1], 0.5),
    ("Omegac0", ["sr-ch-sr"], [1], 0.5),
    ("Lambdac+", ["up-dn-ch", "up-ch-dn", "dn-ch-up"], [2, 1, -1], 0.5),
    ("Xic+", ["sr-up-ch", "sr-ch-up", "up-ch-sr"], [2, 1, -1], 0.5),
    ("Xic0", ["sr-dn-ch", "sr-ch-dn", "dn-ch-sr"], [2, 1, -1], 0.5),
    ("proton", ["up-dn-up"], [1], 0.5),
    ("neutron", ["dn-up-dn"], [1], 0.5),
    ("Lambda", ["up-dn-sr", "up-sr-dn", "dn-sr-up"], [2, 1, -1], 0.5),
    ("Sigma+", ["up-sr-up"], [1], 0.5),
    ("Sigma0", ["up-sr-dn", "dn-sr-up"], [1, 1], 0.5),
    ("Sigma-", ["dn-sr-dn"], [1], 0.5),
    ("Xi0", ["sr-up-sr"], [1], 0.5),
    ("Xi-", ["sr-dn-sr"], [1], 0.5),
    ("Omegaccc++", ["ch-ch-ch"], [1], 1.5),
    ("Xi*cc++", ["ch-up-ch", "ch-ch-up"], [2, 1], 1.5),
    ("Xi*cc+", ["ch-dn-ch", "ch-ch-dn"], [2, 1], 1.5),
    ("Omega*cc+", ["ch-sr-ch", "ch-ch-sr"], [2, 1], 1.5),
    ("Sigma*c++", ["up-up-ch", "ch-up-up"], [1, 2], 1.5),
    ("Sigma*c+", ["up-dn-ch", "dn-ch-up", "ch-up-dn"], [1, 1, 1], 1.5),
    ("Sigma*c0", ["dn-dn-ch", "ch-dn-dn"], [1, 2], 1.5),
    ("Xi*c+", ["up-sr-ch", "sr-ch-up", "ch-up-sr"], [1, 1, 1], 1.5),
    ("Xi*c0", ["dn-sr-ch", "sr-ch-dn", "ch-dn-sr"], [1, 1, 1], 1.5),
    ("Omega*c0", ["sr-ch-sr", "sr-sr-ch"], [2, 1], 1.5),
    ("Delta++", ["up-up-up"], [1], 1.5),
    ("Delta+", ["up-dn-up", "up-up-dn"], [2, 1], 1.5),
    ("Delta0", ["dn-up-dn", "dn-dn-up"], [2, 1], 1.5),
    ("Delta-", ["dn-dn-dn"], [1], 1.5),
    ("Sigma*+", ["up-up-sr", "sr-up-up"], [1, 2], 1.5),
    ("Sigma*0", ["up-dn-sr", "dn-sr-up", "sr-up-dn"], [1, 1, 1], 1.5),
    ("Sigma*-", ["dn-dn-sr", "sr-dn-dn"], [1, 2], 1.5),
    ("Xi*0", ["sr-up-sr", "sr-sr-up"], [2, 1], 1.5),
    ("Xi*-", ["sr-dn-sr", "sr-sr-dn"], [2, 1], 1.5),
    ("Omega-", ["sr-sr-sr"], [1], 1.5),
]

FLAVOUR_ORDER = {"up": 0, "dn": 1, "sr": 2, "ch": 3}

# a field: (flavour, is_antiquark, slot); a propagator: (flavour, quark slot, antiquark slot)
Field = Tuple[str, bool, int]
Prop = Tuple[str, int, int]


def contractions(fields: List[Field]) -> List[Tuple[int, List[Prop]]]:
    """All Wick contractions of the fields as (sign, propagators).  The sign is
    the parity of bringing every (quark, antiquark) pair next to each other,
    quark first, taken pair by pair from the first field."""
    if not fields:
        return [(1, [])]
    head, rest = fields[0], fields[1:]
    out = []
    for i, f in enumerate(rest):
        if f[0] != head[0] or f[1] == head[1]:
            continue
        # moving f next to head crosses i fields; an antiquark-first pair flips once more
        sign = (-1) ** i * (1 if f[1] else -1)
        quark, anti = (head, f) if f[1] else (f, head)
        for s, props in contractions(rest[:i] + rest[i + 1:]):
            out.append((sign * s, [(quark[0], quark[2], anti[2])] + props))
    return out


def parity(perm: List[int]) -> int:
    p, seen = 1, [False] * len(perm)
    for i in range(len(perm)):
        if seen[i]:
            continue
        j, n = i, 0
        while not seen[j]:
            seen[j] = True
            j = perm[j]
            n += 1
        if n % 2 == 0:
            p = -p
    return p


def to_default_view(props: List[Prop]) -> Tuple[Dict[int, int], int]:
    """(spin slot map original -> default, colour sign) of one contraction.
    Default propagator k (flavour-sorted) has quark slot k and antiquark slot
    3 + k for colour, and spins 2k, 2k + 1."""
    flav = sorted((p[0] for p in props), key=lambda f: FLAVOUR_ORDER[f])
    free = list(range(3))
    spin_map, colour = {}, [0] * 6
    for fl, q, a in props:
        k = next(j for j in free if flav[j] == fl)
        free.remove(k)
        spin_map[q], spin_map[a] = 2 * k, 2 * k + 1
        colour[q], colour[a] = k, 3 + k
    return spin_map, parity(colour)


def nonzero_triples(mats):
    """(s0..s5, value) for the non-zero entries of the outer product of three 4x4 matrices."""
    nz = [[(r, c, m[r, c]) for r in range(4) for c in range(4) if abs(m[r, c]) > 1e-12] for m in mats]
    for (a, b, va), (c, d, vb), (e, f, vc) in itertools.product(*nz):
        yield (a, b, c, d, e, f), va * vb * vc


def baryon_tables(name, flavs, coeffs, spin_):
    """{set name: {6-tuple: weight}} and the flavour key of one baryon."""
    terms = []  # (coefficient, spin map)
    for fj, kj in zip(flavs, coeffs):
        q = fj.split("-")
        for fb, kb in zip(flavs, coeffs):
            qb = fb.split("-")
            fields = [(q[0], False, 0), (q[1], False, 1), (q[2], False, 2),
                      (qb[2], True, 3), (qb[0], True, 4), (qb[1], True, 5)]
            for s, props in contractions(fields):
                smap, csign = to_default_view(props)
                terms.append((kj * kb * s * csign, smap))
    if spin_ == 0.5:
        norm = float(sum(k * k for k in coeffs))
    else:
        norm = {3: 0.5, 2: 1.0, 1: 1.0 / 3.0}[len(coeffs)]
    out = {}
    for set_name, triples in SETS[spin_]:
        acc: Dict[Tuple[int, ...], complex] = {}
        for proj, ga, gb in triples:
            nz = list(nonzero_triples([ga, proj, gb]))
            for k, smap in terms:
                for tup, v in nz:
                    new = [0] * 6
                    for src, dst in smap.items():
                        new[dst] = tup[src]
                    key = tuple(new)
                    acc[key] = acc.get(key, 0) + v * k
        out[set_name] = {key: v / norm for key, v in acc.items() if not np.isclose(v, 0)}
    flav0 = sorted(flavs[0].split("-"), key=lambda f: FLAVOUR_ORDER[f])
    return out, "".join(f[0] for f in flav0)


def dataset_name(baryon: str, set_name: str) -> str:
    for a, b in (("+", "Pl"), ("-", "Mn"), ("*", "St"), ("'", "Pr")):
        baryon = baryon.replace(a, b)
    return baryon + "/" + set_name.replace("-", "_")


def products():
    """[(product 'uud', [(dataset name, [(s0..s5)], [complex64 weight])])] in the
    reference's product and dataset order."""
    prods: Dict[str, list] = {}
    for name, flavs, coeffs, sp in BARYONS:
        sets, key = baryon_tables(name, flavs, coeffs, sp)
        lst = prods.setdefault(key, [])
        for set_name, _ in SETS[sp]:
            ent = sets[set_name]
            lst.append((dataset_name(name, set_name), list(ent.keys()),
                        [np.complex64(v) for v in ent.values()]))
    return list(prods.items())


def names_digest(names) -> str:
    import hashlib
    return hashlib.sha256("\n".join(names).encode()).hexdigest()[:16]


def ordered_digest(idx, vals) -> str:
    """Digest of one dataset in entry order: (6 indices, weight rounded to single precision)."""
    import hashlib
    rows = [(tuple(int(x) for x in t), float(np.float32(np.real(v))) + 0.0, float(np.float32(np.imag(v))) + 0.0)
            for t, v in zip(idx, vals)]
    return hashlib.sha256(repr(rows).encode()).hexdigest()[:16]


def table_digest(idx, vals) -> str:
    """Order-independent digest of one dataset: sorted (tuple, weight rounded to 6 digits)."""
    import hashlib
    rows = sorted((tuple(int(x) for x in t), round(float(np.real(v)), 6) + 0.0, round(float(np.imag(v)), 6) + 0.0)
                  for t, v in zip(idx, vals))
    return hashlib.sha256(repr(rows).encode()).hexdigest()[:16]


def emit_header(path: str) -> bool:
    """C header with the tables (generated at build time); True if the file changed."""
    prods = products()
    names, ds_begin, ent_begin, idx, val, pflav = [], [0], [0], [], [], []
    for key, dss in prods:
        pflav.append(key)
        for name, tups, ws in dss:
            names.append(name)
            for t, w in zip(tups, ws):
                idx.append(t)
                val.append((float(np.real(w)), float(np.imag(w))))
            ent_begin.append(len(idx))
        ds_begin.append(len(names))
    L = ["// Generated by plegma_b200/udsc.py: table-driven baryon spin tables.", "#pragma once", "",
         f"constexpr int kUdscProducts = {len(prods)};",
         f"constexpr int kUdscDatasets = {len(names)};",
         f"constexpr int kUdscEntries = {len(idx)};",
         "static const char kUdscProduct[kUdscProducts][4] = {" + ", ".join(f'"{k}"' for k in pflav) + "};",
         "static const int kUdscDsBegin[kUdscProducts + 1] = {" + ", ".join(map(str, ds_begin)) + "};",
         "static const char* const kUdscName[kUdscDatasets] = {" + ", ".join(f'"{n}"' for n in names) + "};",
         "static const int kUdscEntBegin[kUdscDatasets + 1] = {" + ", ".join(map(str, ent_begin)) + "};",
         "static const signed char kUdscIdx[kUdscEntries][6] = {"]
    for i in range(0, len(idx), 12):
        L.append("  " + " ".join("{%d,%d,%d,%d,%d,%d}," % t for t in idx[i:i + 12]))
    L.append("};")
    L.append("static const float kUdscVal[kUdscEntries][2] = {")
    for i in range(0, len(val), 8):
        L.append("  " + " ".join("{%.9ef,%.9ef}," % v for v in val[i:i + 8]))
    L.append("};")
    text = "\n".join(L) + "\n"
    try:
        with open(path) as f:
            if f.read() == text:
                return False
    except FileNotFoundError:
        pass
    with open(path, "w") as f:
        f.write(text)
    return True
