"""The C-ABI library on a machine without a GPU: it loads, exports every entry
point of include/plegma2pt.h, and its host-side helpers agree with the
reference's conventions (no compute calls here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from plegma_b200 import lib as p2
from plegma_b200 import spin

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_entry_points():
    with open(os.path.join(ROOT, "include", "plegma2pt.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:p2_status|int|const char\*)\s+(p2_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_entry_point():
    lib = p2.load()
    names = header_entry_points()
    assert set(names) == set(p2.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_components_and_blocks():
    assert p2.components(p2.NUCLEON_CG5) == 32
    assert p2.components(p2.NUCLEON_CG5 | p2.MESON_G16) == 288
    assert p2.components(p2.NUCLEON_CG5 | p2.DELTA_ISO12 | p2.DELTA_ISO32 | p2.MESON_G16) == 480
    assert p2.components(1 << 20) == -1
    blocks, total = p2.block_info(p2.NUCLEON_CG5 | p2.MESON_G16, 5, 19)
    assert blocks[0][:4] == (p2.NUCLEON_CG5, 1, 2, 16) and blocks[0][4] == 0
    assert blocks[1][:4] == (p2.MESON_G16, 1, 1, 256) and blocks[1][4] == 2 * 16 * 5 * 19
    assert total == (32 + 256) * 5 * 19


def test_mom_list_matches_createMom_order():
    for q2 in (0, 2, 9, 16):
        assert np.array_equal(p2.mom_list(q2), np.array(spin.create_mom(q2)).reshape(-1, 3))


def test_ctx_create_without_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    with pytest.raises(p2.P2Error):
        p2.Context((4, 4, 4, 8))


def test_host_only_context_generator_and_validation():
    """device = -1 gives a host-only context: the host generator runs, bad
    arguments come back as status codes, device entry points refuse."""
    ctx = p2.Context((4, 3, 2, 6), device=-1)
    V3, nt = 24, 6
    a = np.zeros(144 * V3 * nt, dtype=np.complex128)
    b = np.zeros_like(a)
    ctx.synth(a.ctypes.data, False, p2.P2_FP64, seed=7, flavour=0, t0=2, decay=0.5)
    ctx.synth(b.ctypes.data, False, p2.P2_FP64, seed=7, flavour=0, t0=2, decay=0.5)
    assert np.array_equal(a, b)
    ctx.synth(b.ctypes.data, False, p2.P2_FP64, seed=7, flavour=1, t0=2, decay=0.5)
    assert not np.array_equal(a, b)
    # undo the exp(-0.5|t - t0|) envelope: unit-variance Gaussians
    t = (np.arange(V3 * nt) // V3)
    g = a.reshape(144, V3 * nt) / np.exp(-0.5 * np.abs(t - 2))[None, :]
    assert abs(g.real.mean()) < 0.05 and abs(g.imag.mean()) < 0.05
    assert abs(g.real.var() - 1) < 0.05 and abs(g.imag.var() - 1) < 0.05
    # a window starting at t_first = 4 of 3 slices matches slices 4, 5, 0 of the full field
    w = np.zeros(144 * V3 * 3, dtype=np.complex128)
    ctx.synth(w.ctypes.data, False, p2.P2_FP64, seed=7, flavour=0, t0=2, decay=0.5, t_first=4, nt=3)
    full = a.reshape(144, nt, V3)
    assert np.array_equal(w.reshape(144, 3, V3), full[:, [4, 5, 0], :])
    # fp32 storage rounds the same stream
    f = np.zeros(144 * V3 * nt, dtype=np.complex64)
    ctx.synth(f.ctypes.data, False, p2.P2_FP32, seed=7, flavour=0, t0=2, decay=0.5)
    assert np.array_equal(f, a.astype(np.complex64))
    # argument errors
    with pytest.raises(p2.P2Error) as e:
        ctx.synth(a.ctypes.data, False, p2.P2_FP64, 7, 0, t0=9, decay=0.5)
    assert e.value.status == p2.P2_ERR_INVALID_ARG
    prop = ctx.prop(a.ctypes.data, location=p2.P2_HOST, nt=nt)
    out = np.zeros(10, dtype=np.complex128)
    bad = [ctx.request((0, 0, 0, 0), 0, p2.NUCLEON_CG5, out.ctypes.data, p2.P2_HOST),
           ctx.request((0, 0, 9, 0), 6, p2.NUCLEON_CG5, out.ctypes.data, p2.P2_HOST),
           ctx.request((0, 0, 0, 0), 6, 1 << 12, out.ctypes.data, p2.P2_HOST),
           ctx.request((0, 0, 0, 0), 6, p2.NUCLEON_CG5, out.ctypes.data, p2.P2_HOST, prop_u=3)]
    for r in bad:
        with pytest.raises(p2.P2Error) as e:
            ctx.contract_project([prop, prop], [r])
        assert e.value.status == p2.P2_ERR_INVALID_ARG
    good = ctx.request((0, 0, 0, 0), 6, p2.NUCLEON_CG5, out.ctypes.data, p2.P2_HOST)
    with pytest.raises(p2.P2Error) as e:
        ctx.contract_project([prop, prop], [good])
    assert e.value.status == p2.P2_ERR_UNSUPPORTED
    ctx.close()


def test_tune_cache_file_round_trip(tmp_path):
    """The tuning cache file is read on p2_tune_enable: well-formed lines
    become entries, malformed ones are skipped (host-only context)."""
    path = tmp_path / "tune.tsv"
    path.write_text("project_split V3=32768 K=288 rows=128 n=8\t144,2,37,14\t1.25\n"
                    "project_fp64 V3=64 K=32 nmom=19 n=4\t8,1,64\t0.01\n"
                    "garbage line without tabs\n"
                    "project_fp64 bad\tx,y\t1\n")
    ctx = p2.Context((4, 4, 4, 4), device=-1)
    assert ctx.tune_count() == 0
    ctx.tune(False, str(path))
    assert ctx.tune_count() == 2
    ctx.close()


def test_graph_and_workspace_entry_points_validate_on_host_only_context():
    ctx = p2.Context((4, 4, 4, 4), device=-1)
    with pytest.raises(p2.P2Error) as e:
        ctx.set_workspace(0)
    assert e.value.status == p2.P2_ERR_INVALID_ARG
    ctx.set_workspace(1 << 20)
    a = np.zeros(16, dtype=np.complex128)
    prop = ctx.prop(a.ctypes.data, location=p2.P2_DEVICE, nt=4)
    req = ctx.request((0, 0, 0, 0), 4, p2.NUCLEON_CG5, a.ctypes.data)
    with pytest.raises(p2.P2Error) as e:
        ctx.graph([prop, prop], [req])
    assert e.value.status == p2.P2_ERR_UNSUPPORTED
    ctx.close()


def test_udsc_dataset_selection_follows_the_reference_filters():
    """p2_udsc_datasets: products needing a missing flavour are skipped,
    only_st / only_ch keep the products with s / c, order as the reference's."""
    from plegma_b200 import udsc
    prods = udsc.products()
    R = p2.Context.udsc_request
    assert len(p2.udsc_datasets(R((0, 0, 0, 0), 4, 0, prop_u=0, prop_d=1))) == 28
    allds = p2.udsc_datasets(R((0, 0, 0, 0), 4, 0, prop_u=0, prop_d=1, prop_s=2, prop_c=3))
    assert allds == [n for _, dss in prods for n, _, _ in dss]
    only_ch = p2.udsc_datasets(R((0, 0, 0, 0), 4, 0, prop_u=0, prop_d=1, prop_s=2, prop_c=3, only_ch=True))
    assert only_ch == [n for k, dss in prods if "c" in k for n, _, _ in dss]
    assert p2.udsc_datasets(R((0, 0, 0, 0), 4, 0, prop_s=0, only_ch=True)) == []


def test_header_is_plain_c(tmp_path):
    """include/plegma2pt.h compiles as C99 (the boundary a cgo, JNI or
    N-API stub would include) and links against the library."""
    src = tmp_path / "abi.c"
    src.write_text('#include "plegma2pt.h"\n'
                   "int main(void) {\n"
                   "  int moms[3 * 19];\n"
                   "  if (p2_components(P2_NUCLEON_CG5 | P2_MESON_G16) != 288) return 1;\n"
                   "  if (p2_mom_list(2, moms) != 19) return 2;\n"
                   "  return 0;\n"
                   "}\n")
    exe = tmp_path / "abi"
    libdir = os.path.dirname(p2.LIB_PATH)
    import subprocess
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                        str(exe), "-L", libdir, "-lplegma2pt", "-Wl,-rpath," + libdir],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
