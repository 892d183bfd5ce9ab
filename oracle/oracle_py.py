"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so) and of the
reference's own contraction functions compiled as host code
(oracle/_ref/libplegma_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg; the product never imports it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libplegma_ref.so")

_orc = None
_ref = None


def oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            import importlib.util
            spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(HERE, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build_oracle()
        lib = C.CDLL(ORACLE_LIB)
        lib.orc_components.argtypes = [C.c_uint]
        lib.orc_twopt.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_uint, C.POINTER(C.c_int),
                                  C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_site.argtypes = [C.c_void_p, C.c_void_p, C.c_uint, C.c_void_p]
        lib.orc_ft.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_int,
                               C.c_int, C.c_void_p]
        lib.orc_udsc_site.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
        lib.orc_udsc_twopt.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_int,
                                       C.c_void_p, C.c_void_p]
        _orc = lib
    return _orc


def reference():
    """The reference's baryon functions and meson kernels, or None when not built here."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        lib = C.CDLL(REF_LIB)
        lib.ref_nucleon.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_delta.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        lib.ref_light.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        lib.ref_meson_ft.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_void_p]
        _ref = lib
    return _ref


def _ip(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def components(what):
    return oracle().orc_components(what)


def twopt(L, u, d, src, moms, what, taus, t_first=0, fp32=False, want_abs=True, want_pos=False):
    """Projected two-point functions for the given source-relative times.

    u, d: complex arrays [144][V3*nt] (complex128, or complex64 with fp32).
    Returns (out[ntau][nmom][K], abs_sum[ntau][K] or None, pos[ntau][K][V3] or None).
    """
    lib = oracle()
    L = _ip(L)
    V3 = int(L[0] * L[1] * L[2])
    nt = u.shape[-1] // V3
    moms = _ip(moms).reshape(-1, 3)
    taus = _ip(taus)
    K = lib.orc_components(what)
    out = np.zeros((len(taus), len(moms), K), dtype=np.complex128)
    asum = np.zeros((len(taus), K), dtype=np.float64) if want_abs else None
    pos = np.zeros((len(taus), K, V3), dtype=np.complex128) if want_pos else None
    u = np.ascontiguousarray(u)
    d = np.ascontiguousarray(d)
    st = lib.orc_twopt(L.ctypes.data_as(C.POINTER(C.c_int)), nt, t_first, u.ctypes.data, d.ctypes.data, int(fp32),
                       _ip(src).ctypes.data_as(C.POINTER(C.c_int)), moms.ctypes.data_as(C.POINTER(C.c_int)),
                       len(moms), what, taus.ctypes.data_as(C.POINTER(C.c_int)), len(taus), out.ctypes.data,
                       asum.ctypes.data if asum is not None else None, pos.ctypes.data if pos is not None else None)
    if st != 0:
        raise RuntimeError(f"orc_twopt failed ({st})")
    return out, asum, pos


def site(u1, d1, what):
    """All components of one site from two [144] complex128 arrays."""
    lib = oracle()
    K = lib.orc_components(what)
    out = np.zeros(K, dtype=np.complex128)
    u1 = np.ascontiguousarray(u1, dtype=np.complex128)
    d1 = np.ascontiguousarray(d1, dtype=np.complex128)
    lib.orc_site(u1.ctypes.data, d1.ctypes.data, what, out.ctypes.data)
    return out


def ft(L, field, dof, nt, moms, sign=-1):
    lib = oracle()
    L = _ip(L)
    moms = _ip(moms).reshape(-1, 3)
    out = np.zeros((nt, dof, len(moms)), dtype=np.complex128)
    f = np.ascontiguousarray(field, dtype=np.complex128)
    lib.orc_ft(L.ctypes.data_as(C.POINTER(C.c_int)), nt, f.ctypes.data, dof, moms.ctypes.data_as(C.POINTER(C.c_int)),
               len(moms), sign, out.ctypes.data)
    return out


def udsc_site(p1, p2, p3, idx, w):
    lib = oracle()
    idx = np.ascontiguousarray(idx, dtype=np.int16).reshape(-1, 6)
    w = np.ascontiguousarray(w, dtype=np.complex128)
    out = np.zeros(1, dtype=np.complex128)
    arrs = [np.ascontiguousarray(x, dtype=np.complex128) for x in (p1, p2, p3)]
    lib.orc_udsc_site(arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data, len(idx), idx.ctypes.data,
                      w.ctypes.data, out.ctypes.data)
    return out[0]


def ref_nucleon(u1, d1):
    lib = reference()
    out = np.zeros(32, dtype=np.complex128)
    u1 = np.ascontiguousarray(u1, dtype=np.complex128)
    d1 = np.ascontiguousarray(d1, dtype=np.complex128)
    lib.ref_nucleon(u1.ctypes.data, d1.ctypes.data, out.ctypes.data)
    return out


def ref_light(u1, d1, which):
    """The reference's NtoR (0), RtoN (1), RtoR (2) on one site: [2][4][4]."""
    lib = reference()
    out = np.zeros(32, dtype=np.complex128)
    u1 = np.ascontiguousarray(u1, dtype=np.complex128)
    d1 = np.ascontiguousarray(d1, dtype=np.complex128)
    lib.ref_light(u1.ctypes.data, d1.ctypes.data, int(which), out.ctypes.data)
    return out


def ref_meson_ft(kind, L, u, d, j, src, moms):
    """The reference's meson kernels with their in-kernel projection on local
    slice j (kind 0: contract_mesons_device, 20 components; 1:
    contract_mesons_all_device, 34; 2: contract_mesons_new_device, 10).
    u, d: complex128 [144][V3*nt].  Returns [nmom][ncomp] complex."""
    lib = reference()
    L = _ip(L[:3])
    V3 = int(L[0] * L[1] * L[2])
    u = np.ascontiguousarray(u, dtype=np.complex128).reshape(144, -1)
    d = np.ascontiguousarray(d, dtype=np.complex128).reshape(144, -1)
    nt = u.shape[1] // V3
    moms = _ip(moms).reshape(-1, 3)
    ncomp = {0: 20, 1: 34, 2: 10}[kind]
    out = np.zeros((len(moms), ncomp), dtype=np.complex128)
    rc = lib.ref_meson_ft(int(kind), L.ctypes.data_as(C.POINTER(C.c_int)), nt, u.ctypes.data, d.ctypes.data, int(j),
                          _ip(src[:3]).ctypes.data_as(C.POINTER(C.c_int)), moms.ctypes.data_as(C.POINTER(C.c_int)),
                          len(moms), out.ctypes.data)
    if rc != ncomp:
        raise RuntimeError(f"ref_meson_ft failed ({rc})")
    return out


def ref_delta(u1, d1, iso32, g):
    lib = reference()
    out = np.zeros(32, dtype=np.complex128)
    u1 = np.ascontiguousarray(u1, dtype=np.complex128)
    d1 = np.ascontiguousarray(d1, dtype=np.complex128)
    lib.ref_delta(u1.ctypes.data, d1.ctypes.data, int(iso32), int(g), out.ctypes.data)
    return out


def udsc_twopt(L, props, src, moms, datasets, taus, t_first=0, fp32=False):
    """Table-driven baryon two-point functions of one flavour product.

    props: the product's three propagators (complex arrays [144][V3*nt]);
    datasets: [(name, [(s0..s5)], [complex weight])] as plegma_b200.udsc.products().
    Returns (out[ntau][ndata][nmom], abs_sum[ntau][ndata])."""
    lib = oracle()
    L = _ip(L)
    V3 = int(L[0] * L[1] * L[2])
    nt = props[0].shape[-1] // V3
    moms = _ip(moms).reshape(-1, 3)
    taus = _ip(taus)
    ent = [0]
    idx, w = [], []
    for _, tups, ws in datasets:
        idx += [list(t) for t in tups]
        w += [[np.real(x), np.imag(x)] for x in ws]
        ent.append(len(idx))
    idx = np.ascontiguousarray(idx, dtype=np.int8)
    w = np.ascontiguousarray(w, dtype=np.float32)
    ent = _ip(ent)
    props = [np.ascontiguousarray(p) for p in props]
    out = np.zeros((len(taus), len(datasets), len(moms)), dtype=np.complex128)
    asum = np.zeros((len(taus), len(datasets)), dtype=np.float64)
    rc = lib.orc_udsc_twopt(L.ctypes.data_as(C.POINTER(C.c_int)), nt, t_first, props[0].ctypes.data,
                            props[1].ctypes.data, props[2].ctypes.data, int(fp32),
                            _ip(src).ctypes.data_as(C.POINTER(C.c_int)), moms.ctypes.data_as(C.POINTER(C.c_int)),
                            len(moms), len(datasets), ent.ctypes.data, idx.ctypes.data, w.ctypes.data,
                            taus.ctypes.data_as(C.POINTER(C.c_int)), len(taus), out.ctypes.data, asum.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"orc_udsc_twopt failed ({rc})")
    return out, asum


def prop_transform(p, V3, t_first, nt, T, transform, boundary_t0=0):
    """The reference's propagator pre-processing on a host copy [144][V3*nt]:
    rotateToPhysicalBase (lib/kernels/PLEGMA_propagator_utils.cuh:97-126),
    g5 P (:31-53) and the antiperiodic sign (:64-80), in that order."""
    P = np.array(p, dtype=np.complex128).reshape(4, 4, 9, nt, V3)
    if transform & 3:
        s = 1.0 if transform & 1 else -1.0
        Q = np.empty_like(P)
        for mu in range(4):
            for nu in range(4):
                Q[mu, nu] = 0.5 * (P[mu, nu] - P[(mu + 2) % 4, (nu + 2) % 4] +
                                   s * 1j * (P[mu, (nu + 2) % 4] + P[(mu + 2) % 4, nu]))
        P = Q
    if transform & 4:
        P = P[[2, 3, 0, 1]]
    if transform & 8:
        t = (t_first + np.arange(nt)) % T
        P = np.where((t < boundary_t0)[None, None, None, :, None], -P, P)
    return P.reshape(144, nt * V3)


def prop_absorb(p, vec, V3, t_first, nt, T, nu, c2, vec_3d=False, global_t=-1):
    """PLEGMA_Propagator::absorb (lib/PLEGMA_Propagator.cu:33-95) on host
    copies: prop [144][nt V3], vec [12][nt V3] (or [12][V3] for a 3-D vector)."""
    P = np.array(p, dtype=np.complex128).reshape(4, 4, 3, 3, nt, V3)
    if global_t < 0:
        v = np.asarray(vec).reshape(4, 3, nt, V3)
    else:
        v = np.zeros((4, 3, nt, V3), dtype=np.complex128)
        j = (global_t - t_first) % T
        if j < nt:
            v[:, :, j] = np.asarray(vec).reshape(4, 3, -1, V3)[:, :, 0 if vec_3d else j]
    P[:, nu, :, c2] = v
    return P.reshape(144, nt * V3)
