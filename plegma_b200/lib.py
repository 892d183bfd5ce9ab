"""ctypes binding of the C ABI in include/plegma2pt.h.

The shared library is built in-tree by `python -m plegma_b200.build`
(plegma_b200/lib/libplegma2pt.so).  There is no fallback: if the library is
missing, `load()` raises.
"""
from __future__ import annotations

import ctypes as C
import weakref
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libplegma2pt.so")

P2_OK, P2_ERR_INVALID_ARG, P2_ERR_OOM, P2_ERR_CUDA, P2_ERR_DEVICE_TIMEOUT, P2_ERR_UNSUPPORTED = range(6)
P2_FP64, P2_FP32 = 0, 1
P2_PLAIN_FP64, P2_SPLIT_FP16 = 0, 1
P2_DEVICE, P2_HOST = 0, 1

NUCLEON_CG5 = 1 << 0
DELTA_ISO12 = 1 << 1
DELTA_ISO32 = 1 << 2
MESON_G16 = 1 << 3
MESON_ALL34 = 1 << 4
MESON_NEW10 = 1 << 5
MESON_DIAG10 = 1 << 6
NUCLEON_NTOR = 1 << 7
NUCLEON_RTON = 1 << 8
NUCLEON_RTOR = 1 << 9

#: (bit, groups, datasets, comps, group names, dataset names), the reference's names
#: (lib/PLEGMA_Correlator.cu:43-135).
BLOCKS = [
    (NUCLEON_CG5, 1, 2, 16, ["baryons/nucl_nucl"], ["twop_baryon_1", "twop_baryon_2"]),
    (NUCLEON_NTOR, 1, 2, 16, ["baryons/nucl_nucl2"], ["twop_baryon_1", "twop_baryon_2"]),
    (NUCLEON_RTON, 1, 2, 16, ["baryons/nucl2_nucl"], ["twop_baryon_1", "twop_baryon_2"]),
    (NUCLEON_RTOR, 1, 2, 16, ["baryons/nucl2_nucl2"], ["twop_baryon_1", "twop_baryon_2"]),
    (DELTA_ISO12, 3, 2, 16, ["baryons/deltap_deltaz_11", "baryons/deltap_deltaz_22", "baryons/deltap_deltaz_33"],
     ["twop_baryon_1", "twop_baryon_2"]),
    (DELTA_ISO32, 3, 2, 16, ["baryons/deltapp_deltamm_11", "baryons/deltapp_deltamm_22",
                             "baryons/deltapp_deltamm_33"], ["twop_baryon_1", "twop_baryon_2"]),
    (MESON_G16, 1, 1, 256, ["mesons"], ["twop_meson"]),
    (MESON_ALL34, 1, 1, 34, ["mesons"], ["twop_meson"]),
    (MESON_NEW10, 1, 1, 10, ["mesons"], ["twop_meson"]),
    (MESON_DIAG10, 1, 2, 10, ["mesons"], ["twop_meson_1", "twop_meson_2"]),
]


class P2Geom(C.Structure):
    _fields_ = [("L", C.c_int * 4), ("procs", C.c_int * 4), ("coords", C.c_int * 4), ("device", C.c_int)]


class P2Prop(C.Structure):
    _fields_ = [("data", C.c_void_p), ("precision", C.c_int), ("location", C.c_int), ("t_first", C.c_int),
                ("nt", C.c_int), ("transform", C.c_uint), ("boundary_t0", C.c_int)]


PROP_ROTATE_PLUS = 1 << 0
PROP_ROTATE_MINUS = 1 << 1
PROP_GAMMA5 = 1 << 2
PROP_BOUNDARY = 1 << 3


class P2Request(C.Structure):
    _fields_ = [("source", C.c_int * 4), ("totalT", C.c_int), ("moms", C.POINTER(C.c_int)), ("nmom", C.c_int),
                ("q2max", C.c_int), ("contractions", C.c_uint), ("mode", C.c_int), ("prop_u", C.c_int),
                ("prop_d", C.c_int), ("out", C.c_void_p), ("out_location", C.c_int)]


class P2UdscRequest(C.Structure):
    _fields_ = [("source", C.c_int * 4), ("totalT", C.c_int), ("moms", C.POINTER(C.c_int)), ("nmom", C.c_int),
                ("q2max", C.c_int), ("prop_u", C.c_int), ("prop_d", C.c_int), ("prop_s", C.c_int),
                ("prop_c", C.c_int), ("only_st", C.c_int), ("only_ch", C.c_int), ("out", C.c_void_p),
                ("out_location", C.c_int), ("mode", C.c_int)]


class P2Block(C.Structure):
    _fields_ = [("bit", C.c_uint), ("groups", C.c_int), ("datasets", C.c_int), ("comps", C.c_int),
                ("offset", C.c_size_t)]


class P2KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_longlong), ("ms", C.c_double)]


#: Every entry point declared in include/plegma2pt.h.
EXPORTS = ["p2_ctx_create", "p2_ctx_destroy", "p2_last_error", "p2_sync", "p2_set_stream", "p2_components",
           "p2_mom_list", "p2_block_info", "p2_contract_project", "p2_contract_position", "p2_ft_apply",
           "p2_synth_propagator", "p2_profile_enable", "p2_profile_read", "p2_alloc", "p2_free", "p2_copy",
           "p2_ft_apply_noalloc", "p2_set_workspace", "p2_graph_create", "p2_graph_launch", "p2_graph_sync",
           "p2_graph_destroy", "p2_tune_enable", "p2_tune_count", "p2_udsc_datasets", "p2_contract_udsc", "p2_local_taus", "p2_prop_transform",
           "p2_prop_absorb", "p2_ft_apply_split", "p2_measure_fp64_rate", "p2_debug_wait_timeout"]

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m plegma_b200.build`")
    lib = C.CDLL(path)
    lib.p2_ctx_create.argtypes = [C.POINTER(P2Geom), C.POINTER(C.c_void_p)]
    lib.p2_ctx_destroy.argtypes = [C.c_void_p]
    lib.p2_last_error.argtypes = [C.c_void_p]
    lib.p2_last_error.restype = C.c_char_p
    lib.p2_sync.argtypes = [C.c_void_p]
    lib.p2_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    lib.p2_set_workspace.argtypes = [C.c_void_p, C.c_size_t]
    lib.p2_graph_create.argtypes = [C.c_void_p, C.POINTER(P2Prop), C.c_int, C.POINTER(P2Request), C.c_int,
                                    C.POINTER(C.c_void_p)]
    lib.p2_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
    lib.p2_graph_sync.argtypes = [C.c_void_p]
    lib.p2_graph_destroy.argtypes = [C.c_void_p]
    lib.p2_tune_enable.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
    lib.p2_tune_count.argtypes = [C.c_void_p]
    lib.p2_prop_transform.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint, C.c_int]
    lib.p2_prop_absorb.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_int]
    lib.p2_local_taus.argtypes = [C.c_void_p, C.POINTER(P2Prop), C.c_int, C.POINTER(P2Request),
                                  C.POINTER(C.c_int), C.c_int]
    lib.p2_udsc_datasets.argtypes = [C.POINTER(P2UdscRequest), C.c_char_p, C.c_size_t]
    lib.p2_contract_udsc.argtypes = [C.c_void_p, C.POINTER(P2Prop), C.c_int, C.POINTER(P2UdscRequest)]
    lib.p2_components.argtypes = [C.c_uint]
    lib.p2_mom_list.argtypes = [C.c_int, C.POINTER(C.c_int)]
    lib.p2_block_info.argtypes = [C.c_uint, C.c_int, C.c_int, C.POINTER(P2Block), C.c_int, C.POINTER(C.c_size_t)]
    lib.p2_contract_project.argtypes = [C.c_void_p, C.POINTER(P2Prop), C.c_int, C.POINTER(P2Request), C.c_int]
    lib.p2_contract_position.argtypes = [C.c_void_p, C.POINTER(P2Prop), C.c_int, C.POINTER(P2Request)]
    lib.p2_ft_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int,
                                C.c_void_p, C.c_int]
    lib.p2_synth_propagator.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int,
                                        C.c_double, C.c_int, C.c_int]
    lib.p2_ft_apply_split.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int,
                                      C.c_void_p, C.c_int]
    lib.p2_ft_apply_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int,
                                        C.c_int, C.c_void_p]
    lib.p2_alloc.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]
    lib.p2_free.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.p2_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
    lib.p2_profile_enable.argtypes = [C.c_void_p, C.c_int]
    lib.p2_profile_read.argtypes = [C.c_void_p, C.POINTER(P2KernelTime), C.c_int, C.c_int]
    lib.p2_measure_fp64_rate.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.p2_debug_wait_timeout.argtypes = [C.c_void_p]
    _lib = lib
    return lib


class P2Error(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"plegma2pt status {status}: {msg}")
        self.status = status


def components(contractions: int) -> int:
    return load().p2_components(contractions)


def mom_list(q2max: int) -> np.ndarray:
    lib = load()
    n = lib.p2_mom_list(q2max, None)
    out = np.zeros((n, 3), dtype=np.int32)
    lib.p2_mom_list(q2max, out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def block_info(contractions: int, totalT: int, nmom: int):
    lib = load()
    blocks = (P2Block * 8)()
    total = C.c_size_t(0)
    n = lib.p2_block_info(contractions, totalT, nmom, blocks, 8, C.byref(total))
    return [(b.bit, b.groups, b.datasets, b.comps, b.offset) for b in blocks[:n]], total.value


class Context:
    """One library context (geometry + stream + workspaces) on one device."""

    def __init__(self, L: Sequence[int], procs=(1, 1, 1, 1), coords=(0, 0, 0, 0), device: int = 0):
        self.lib = load()
        g = P2Geom()
        g.L[:] = list(L)
        g.procs[:] = list(procs)
        g.coords[:] = list(coords)
        g.device = device
        self.L = tuple(L)
        self.Ll = tuple(L[i] // procs[i] for i in range(4))
        self.V3 = self.Ll[0] * self.Ll[1] * self.Ll[2]
        h = C.c_void_p()
        st = self.lib.p2_ctx_create(C.byref(g), C.byref(h))
        if st != P2_OK:
            raise P2Error(st, "p2_ctx_create failed")
        self.h = h
        self._graphs = []  # weak references: graphs are destroyed before their context

    def close(self):
        if self.h:
            for ref in self._graphs:
                g = ref()
                if g is not None:
                    g.close()
            self.lib.p2_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st: int):
        if st != P2_OK:
            raise P2Error(st, self.lib.p2_last_error(self.h).decode())

    def sync(self):
        self.check(self.lib.p2_sync(self.h))

    def set_workspace(self, nbytes: int):
        """p2_set_workspace: cap on the per-chunk position-space buffer."""
        self.check(self.lib.p2_set_workspace(self.h, nbytes))

    def set_stream(self, stream_ptr: Optional[int]):
        self.check(self.lib.p2_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def synth(self, ptr: int, on_device: bool, precision: int, seed: int, flavour: int, t0: int, decay: float,
              t_first: int = 0, nt: Optional[int] = None):
        nt = self.Ll[3] if nt is None else nt
        self.check(self.lib.p2_synth_propagator(self.h, C.c_void_p(ptr), int(on_device), precision, seed, flavour,
                                                t0, decay, t_first, nt))

    def prop(self, ptr: int, precision=P2_FP64, location=P2_DEVICE, t_first=0, nt=None, transform=0,
             boundary_t0=0) -> P2Prop:
        """A propagator view; nt defaults to the local time extent; transform = PROP_* bits applied on load."""
        nt = self.Ll[3] if nt is None else nt
        p = P2Prop()
        p.transform = transform
        p.boundary_t0 = boundary_t0
        p.data = ptr
        p.precision = precision
        p.location = location
        p.t_first = t_first
        p.nt = nt
        return p

    def request(self, source, totalT, contractions, out_ptr, out_location=P2_DEVICE, mode=P2_PLAIN_FP64,
                q2max=0, moms: Optional[np.ndarray] = None, prop_u=0, prop_d=1) -> P2Request:
        r = P2Request()
        r.source[:] = list(source)
        r.totalT = totalT
        if moms is not None:
            m = np.ascontiguousarray(moms, dtype=np.int32)
            r._moms_keep = m
            r.moms = m.ctypes.data_as(C.POINTER(C.c_int))
            r.nmom = len(m)
        else:
            r.moms = None
            r.nmom = 0
        r.q2max = q2max
        r.contractions = contractions
        r.mode = mode
        r.prop_u = prop_u
        r.prop_d = prop_d
        r.out = out_ptr
        r.out_location = out_location
        return r

    def contract_project(self, props: Sequence[P2Prop], reqs: Sequence[P2Request]):
        pa = (P2Prop * len(props))(*props)
        ra = (P2Request * len(reqs))(*reqs)
        self.check(self.lib.p2_contract_project(self.h, pa, len(props), ra, len(reqs)))

    def prop_transform(self, ptr: int, transform: int, boundary_t0=0, precision=P2_FP64, t_first=0, nt=None):
        """p2_prop_transform: apply PROP_* transforms in place to a device field."""
        nt = self.Ll[3] if nt is None else nt
        self.check(self.lib.p2_prop_transform(self.h, C.c_void_p(ptr), precision, t_first, nt, transform,
                                              boundary_t0))

    def prop_absorb(self, prop: int, vec: int, nu: int, c2: int, precision=P2_FP64, t_first=0, nt=None,
                    vec_3d=False, global_t=-1):
        """p2_prop_absorb: column (nu, c2) of a device propagator from a spinor field."""
        nt = self.Ll[3] if nt is None else nt
        self.check(self.lib.p2_prop_absorb(self.h, C.c_void_p(prop), C.c_void_p(vec), precision, t_first, nt, nu, c2,
                                           int(vec_3d), global_t))

    def local_taus(self, props: Sequence[P2Prop], req: P2Request):
        """p2_local_taus: source-relative times this rank computes."""
        pa = (P2Prop * len(props))(*props)
        buf = (C.c_int * max(self.L[3], 1))()
        n = self.lib.p2_local_taus(self.h, pa, len(props), C.byref(req), buf, len(buf))
        if n < 0:
            raise P2Error(P2_ERR_INVALID_ARG, "p2_local_taus: invalid request")
        return list(buf[:n])

    def contract_position(self, props: Sequence[P2Prop], req: P2Request):
        pa = (P2Prop * len(props))(*props)
        self.check(self.lib.p2_contract_position(self.h, pa, len(props), C.byref(req)))

    @staticmethod
    def udsc_request(source, totalT, out_ptr, out_location=P2_DEVICE, q2max=0, moms: Optional[np.ndarray] = None,
                     prop_u=-1, prop_d=-1, prop_s=-1, prop_c=-1, only_st=False, only_ch=False,
                     mode=P2_PLAIN_FP64) -> P2UdscRequest:
        """A table-driven baryon request (contractBaryonsUDSC); prop_* index the props list, -1 = not given."""
        r = P2UdscRequest()
        r.source[:] = list(source)
        r.totalT = totalT
        if moms is not None:
            m = np.ascontiguousarray(moms, dtype=np.int32)
            r._moms_keep = m
            r.moms = m.ctypes.data_as(C.POINTER(C.c_int))
            r.nmom = len(m)
        else:
            r.moms = None
            r.nmom = 0
        r.q2max = q2max
        r.prop_u, r.prop_d, r.prop_s, r.prop_c = prop_u, prop_d, prop_s, prop_c
        r.only_st, r.only_ch = int(only_st), int(only_ch)
        r.out = out_ptr
        r.out_location = out_location
        r.mode = mode
        return r

    def contract_udsc(self, props: Sequence[P2Prop], req: P2UdscRequest):
        pa = (P2Prop * len(props))(*props)
        self.check(self.lib.p2_contract_udsc(self.h, pa, len(props), C.byref(req)))

    def graph(self, props: Sequence[P2Prop], reqs: Sequence[P2Request]) -> "Graph":
        """p2_graph_create: record the launch sequence of contract_project(props, reqs)."""
        return Graph(self, props, reqs)

    def tune(self, on: bool = True, cache_path: Optional[str] = None):
        """p2_tune_enable: time candidate launch shapes for new (kernel, shape) keys."""
        self.check(self.lib.p2_tune_enable(self.h, int(on), cache_path.encode() if cache_path else None))

    def tune_count(self) -> int:
        return self.lib.p2_tune_count(self.h)

    def profile(self, on: bool = True):
        self.check(self.lib.p2_profile_enable(self.h, int(on)))

    def profile_read(self, reset: bool = True):
        """{kernel name: (launches, total ms)} since the last reset."""
        buf = (P2KernelTime * 64)()
        n = self.lib.p2_profile_read(self.h, buf, 64, int(reset))
        return {buf[i].name.decode(): (buf[i].launches, buf[i].ms) for i in range(min(n, 64))}

    def debug_wait_timeout(self):
        """p2_debug_wait_timeout: the next tensor-core projection's waits run out (test hook)."""
        self.check(self.lib.p2_debug_wait_timeout(self.h))

    def fp64_rate(self):
        """p2_measure_fp64_rate: (TFLOP/s, ms) of the FP64 FMA-loop kernel."""
        tf, ms = C.c_double(), C.c_double()
        self.check(self.lib.p2_measure_fp64_rate(self.h, C.byref(tf), C.byref(ms)))
        return tf.value, ms.value

    def ft_apply_noalloc(self, field_ptr: int, dof: int, nt: int, moms: np.ndarray, sign: int, out_ptr: int):
        """p2_ft_apply_noalloc: device output, scratch in the library's static device array."""
        m = np.ascontiguousarray(moms, dtype=np.int32)
        self.check(self.lib.p2_ft_apply_noalloc(self.h, C.c_void_p(field_ptr), dof, nt,
                                                m.ctypes.data_as(C.POINTER(C.c_int)), len(m), sign,
                                                C.c_void_p(out_ptr)))

    def ft_apply(self, field_ptr: int, dof: int, nt: int, moms: np.ndarray, sign: int, out_ptr: int,
                 out_location=P2_DEVICE, mode=P2_PLAIN_FP64):
        """p2_ft_apply (FP64), or p2_ft_apply_split (tensor cores) with mode=P2_SPLIT_FP16."""
        m = np.ascontiguousarray(moms, dtype=np.int32)
        fn = self.lib.p2_ft_apply_split if mode == P2_SPLIT_FP16 else self.lib.p2_ft_apply
        self.check(fn(self.h, C.c_void_p(field_ptr), dof, nt, m.ctypes.data_as(C.POINTER(C.c_int)), len(m), sign,
                      C.c_void_p(out_ptr), out_location))


class Graph:
    """A recorded batch (p2_graph_*); keeps the request arrays alive."""

    def __init__(self, ctx: "Context", props: Sequence[P2Prop], reqs: Sequence[P2Request]):
        self.ctx = ctx
        self._props = (P2Prop * len(props))(*props)
        self._reqs = (P2Request * len(reqs))(*reqs)
        self._keep = list(reqs)
        h = C.c_void_p()
        self.h = None
        ctx.check(ctx.lib.p2_graph_create(ctx.h, self._props, len(props), self._reqs, len(reqs), C.byref(h)))
        self.h = h
        ctx._graphs.append(weakref.ref(self))

    def launch(self, stream_ptr: Optional[int] = None):
        self.ctx.check(self.ctx.lib.p2_graph_launch(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def sync(self):
        self.ctx.check(self.ctx.lib.p2_graph_sync(self.h))

    def close(self):
        if self.h:
            self.ctx.lib.p2_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def udsc_datasets(req: P2UdscRequest):
    """Dataset names of a table-driven baryon request, in result order."""
    lib = load()
    n = lib.p2_udsc_datasets(C.byref(req), None, 0)
    buf = C.create_string_buffer(64 * max(n, 1) + 1)
    lib.p2_udsc_datasets(C.byref(req), buf, len(buf))
    names = buf.value.decode().split("\n")
    return [x for x in names if x]


def result_blocks(contractions: int, totalT: int, nmom: int, flat: np.ndarray):
    """Split a flat complex result into {bit: array[groups][datasets][totalT][nmom][comps]}."""
    blocks, total = block_info(contractions, totalT, nmom)
    flat = flat.reshape(-1)
    assert flat.size == total, (flat.size, total)
    out = {}
    for bit, g, d, c, off in blocks:
        n = g * d * totalT * nmom * c
        out[bit] = flat[off:off + n].reshape(g, d, totalT, nmom, c)
    return out
