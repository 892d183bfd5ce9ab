"""Parity of the split-FP16 form (FP32 contraction, hi+lo FP16 tensor-core
projection with FP32 accumulation, FP64 cross-block sums) with the FP64
oracle.  Tolerance: err(t) <= 1e-6 relative to sum_x |c_k(x,t)|, per time
slice, over all momenta and components."""
import numpy as np
import pytest

from plegma_b200 import lib as p2

from p2test import device_props, oracle_blocks, per_t_error, run

pytestmark = pytest.mark.gpu

NUC = p2.NUCLEON_CG5
TOL = 1e-6
SPLIT = p2.P2_SPLIT_FP16


def test_split_small_nucleon():
    ctx = p2.Context((4, 4, 4, 8))
    (u,) = device_props(ctx, [(1001, 0)], t0=0)
    bufs = [u, u]
    out, moms = run(ctx, bufs, (0, 0, 0, 0), 8, NUC, q2max=2, mode=SPLIT)
    taus = list(range(8))
    ref = oracle_blocks(ctx.L, bufs, (0, 0, 0, 0), moms, NUC, taus)
    err = per_t_error(out, NUC, 8, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


def test_split_odd_lattice_all_mesons_asymmetric_momenta():
    """V3 = 30 (not a multiple of the 64-site k-step), a wrapping window, and
    a momentum list that is not closed under p -> -p (cos and sin rows of
    unpaired momenta)."""
    ctx = p2.Context((3, 5, 2, 6))
    bufs = device_props(ctx, [(7, 0), (7, 1)], t0=4)
    what = NUC | p2.MESON_G16 | p2.MESON_ALL34 | p2.MESON_NEW10 | p2.MESON_DIAG10
    src = (1, 3, 1, 4)
    moms = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, -2, 1], [1, 1, 1], [-1, 2, 0]], dtype=np.int32)
    out, moms = run(ctx, bufs, src, 5, what, moms=moms, mode=SPLIT)
    taus = list(range(5))
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(out, what, 5, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


def test_split_24_nucleon_mesons_q9():
    """24^3 x 48, u and d, nucleon + 16x16 mesons, 123 momenta; the decay
    exp(-0.5|t - t0|) spans ~10 decades in the baryons over the window."""
    ctx = p2.Context((24, 24, 24, 48))
    rng = np.random.default_rng(1002)
    t0 = int(rng.integers(0, 48))
    src = (int(rng.integers(0, 24)), int(rng.integers(0, 24)), int(rng.integers(0, 24)), t0)
    bufs = device_props(ctx, [(1002, 0), (1002, 1)], t0=t0)
    what = NUC | p2.MESON_G16
    out, moms = run(ctx, bufs, src, 48, what, q2max=9, mode=SPLIT)
    taus = [0, 1, 24, 47]
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(out, what, 48, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


def test_split_fp32_propagators():
    """FP32-stored propagators (the large batched configuration's storage)."""
    ctx = p2.Context((6, 4, 4, 8))
    bufs = device_props(ctx, [(1005, 0), (1005, 1)], t0=2, decay=0.4, precision=p2.P2_FP32)
    what = NUC | p2.MESON_G16
    out, moms = run(ctx, bufs, (1, 1, 1, 2), 8, what, q2max=4, mode=SPLIT, precision=p2.P2_FP32)
    taus = list(range(8))
    ref = oracle_blocks(ctx.L, bufs, (1, 1, 1, 2), moms, what, taus, fp32=True)
    err = per_t_error(out, what, 8, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


def test_split_matches_plain_to_tolerance():
    ctx = p2.Context((8, 8, 8, 8))
    bufs = device_props(ctx, [(3, 0), (3, 1)], t0=5)
    what = NUC | p2.MESON_G16
    a, moms = run(ctx, bufs, (2, 3, 4, 5), 8, what, q2max=3)
    b, _ = run(ctx, bufs, (2, 3, 4, 5), 8, what, q2max=3, mode=SPLIT)
    c, _ = run(ctx, bufs, (2, 3, 4, 5), 8, what, q2max=3, mode=SPLIT)
    assert np.array_equal(b, c)  # deterministic
    ga = p2.result_blocks(what, 8, len(moms), a)
    gb = p2.result_blocks(what, 8, len(moms), b)
    for bit in ga:
        scale = np.abs(ga[bit]).max(axis=(3, 4), keepdims=True)
        assert (np.abs(ga[bit] - gb[bit]) / scale).max() < 1e-5
    ctx.close()


def test_split_delta_batched_set():
    """Nucleon + Delta (both isospins, k = 1..3) + 16x16 mesons, K = 480:
    four N-tiles of the tensor-core projection."""
    ctx = p2.Context((8, 6, 4, 8))
    bufs = device_props(ctx, [(1004, 0), (1004, 1)], t0=6)
    what = NUC | p2.DELTA_ISO12 | p2.DELTA_ISO32 | p2.MESON_G16
    out, moms = run(ctx, bufs, (3, 1, 2, 6), 7, what, q2max=5, mode=SPLIT)
    taus = list(range(7))
    ref = oracle_blocks(ctx.L, bufs, (3, 1, 2, 6), moms, what, taus)
    err = per_t_error(out, what, 7, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()


@pytest.mark.parametrize("decay", [0.5, 15.0])
def test_split_host_propagators_converted_on_host(decay):
    """FP64 propagators on the host are converted to FP32 by the library
    (each slice times an exact power of two) before the upload.  With decay
    15 the entries fall to ~1e-46 across the window, below FP32's normal
    range, so the per-slice scale is what keeps them: the result must equal
    the device-resident FP64 run and meet the 1e-6 bound against the oracle,
    with the window wrapping through t = 0."""
    ctx = p2.Context((4, 3, 2, 8))
    src = (1, 2, 0, 5)
    bufs = device_props(ctx, [(33, 0), (33, 1)], t0=src[3], decay=decay)
    what = p2.NUCLEON_CG5 | p2.MESON_G16
    moms = p2.mom_list(2)
    dev, _ = run(ctx, bufs, src, 8, what, moms=moms, mode=p2.P2_SPLIT_FP16)
    host, _ = run(ctx, bufs, src, 8, what, moms=moms, mode=p2.P2_SPLIT_FP16, host_props=True, host_out=True)
    assert np.array_equal(dev, host)
    taus = list(range(8))
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(host, what, 8, moms, ref, taus)
    assert err.max() < 1e-6, err
    ctx.close()


def test_split_odd_spatial_volume():
    """V3 = 27 (odd): site pairs of the projection are not 16-byte aligned,
    tiles are ragged, and the host conversion writes unaligned rows; device
    and host propagators give the same result within the bound."""
    ctx = p2.Context((3, 3, 3, 6))
    src = (2, 0, 1, 4)
    bufs = device_props(ctx, [(41, 0), (41, 1)], t0=src[3])
    what = p2.NUCLEON_CG5 | p2.MESON_G16 | p2.DELTA_ISO12
    moms = p2.mom_list(2)
    dev, _ = run(ctx, bufs, src, 6, what, moms=moms, mode=p2.P2_SPLIT_FP16)
    host, _ = run(ctx, bufs, src, 6, what, moms=moms, mode=p2.P2_SPLIT_FP16, host_props=True, host_out=True)
    assert np.array_equal(dev, host)
    taus = list(range(6))
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(dev, what, 6, moms, ref, taus)
    assert err.max() < 1e-6, err
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_every_contraction_block_in_one_request(mode):
    """All ten blocks at once (K = 640: both kernel instantiations, the 16 x 16
    mesons beside the 10 diagonal structures, the second nucleon
    interpolator), host output, a window that wraps."""
    ctx = p2.Context((4, 3, 4, 6))
    src = (2, 1, 3, 4)
    bufs = device_props(ctx, [(51, 0), (51, 1)], t0=src[3])
    what = 0
    for b in p2.BLOCKS:
        what |= b[0]
    assert p2.components(what) == 640
    moms = p2.mom_list(1)
    out, _ = run(ctx, bufs, src, 6, what, moms=moms, mode=mode, host_out=True)
    taus = list(range(6))
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(out, what, 6, moms, ref, taus)
    assert err.max() < (1e-12 if mode == p2.P2_PLAIN_FP64 else 1e-6), err
    ctx.close()


@pytest.mark.parametrize("q2max", [0, 16])
def test_split_momentum_list_extremes(q2max):
    """One momentum (a single cos row) and |n|^2 <= 16 (257 momenta: 257 phase
    rows in three 128-row tiles, the batched 64^3 x 128 configuration's
    list) against the oracle."""
    ctx = p2.Context((6, 5, 4, 4))
    src = (3, 1, 2, 1)
    bufs = device_props(ctx, [(61, 0), (61, 1)], t0=src[3])
    what = p2.NUCLEON_CG5 | p2.MESON_G16
    moms = p2.mom_list(q2max)
    assert len(moms) == (1 if q2max == 0 else 257)
    out, _ = run(ctx, bufs, src, 4, what, moms=moms, mode=p2.P2_SPLIT_FP16)
    taus = list(range(4))
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(out, what, 4, moms, ref, taus)
    assert err.max() < 1e-6, err
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_two_site_spatial_volume(mode):
    """L = 1 x 1 x 2 x 4 (V3 = 2): tiles of 16 sites with 14 empty, one k-step
    of the projection, a window of one slice and of all four.  With two sites
    a slice's error is the FP32 rounding of single sites (about 100 terms per
    Delta component, not averaged over a volume), so the split form is held
    to 3e-6 here; the 1e-6 bound of the benchmark volumes is asserted by the
    other tests."""
    import oracle_py as orc
    ctx = p2.Context((1, 1, 2, 4))
    src = (0, 0, 1, 2)
    bufs = device_props(ctx, [(63, 0), (63, 1)], t0=src[3])
    what = p2.NUCLEON_CG5 | p2.MESON_G16 | p2.DELTA_ISO32
    moms = p2.mom_list(1)
    for W in (1, 4):
        out, _ = run(ctx, bufs, src, W, what, moms=moms, mode=mode)
        taus = list(range(W))
        ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
        err = per_t_error(out, what, W, moms, ref, taus)
        assert err.max() < (1e-12 if mode == p2.P2_PLAIN_FP64 else 3e-6), err
    f = bufs[0].cpu().numpy().reshape(144, -1)
    ftd = np.zeros(4 * 144 * len(moms), dtype=np.complex128)
    ctx.ft_apply(bufs[0].data_ptr(), 144, 4, moms, -1, ftd.ctypes.data, p2.P2_HOST, mode=mode)
    ref = orc.ft(ctx.L, f, 144, 4, moms, -1)
    asum = np.abs(f).reshape(144, 4, -1).sum(axis=2).T
    assert (np.abs(ftd.reshape(ref.shape) - ref).max(axis=2) / asum).max() < (1e-12 if mode == p2.P2_PLAIN_FP64 else 1e-6)
    ctx.close()


@pytest.mark.parametrize("what", [
    p2.MESON_G16,                                       # sink Gamma stage in the tile flush
    p2.MESON_G16 | p2.MESON_ALL34 | p2.MESON_NEW10,     # staged, sink stage in the lanes, phases in the reduction
    p2.MESON_G16 | p2.MESON_DIAG10,                     # direct stores with phases
    p2.MESON_ALL34 | p2.MESON_NEW10,                    # no 16 x 16 block
])
def test_split_meson_paths(what):
    """The split kernel's four ways of finishing the 16 x 16 meson Gamma
    stages (which lanes or threads form the sink transform, where the unit
    phases r_g1 r_g2 are applied) against the oracle."""
    ctx = p2.Context((5, 4, 3, 6))
    src = (4, 1, 2, 3)
    bufs = device_props(ctx, [(71, 0), (71, 1)], t0=src[3])
    moms = p2.mom_list(2)
    out, _ = run(ctx, bufs, src, 6, what, moms=moms, mode=SPLIT)
    taus = list(range(6))
    ref = oracle_blocks(ctx.L, bufs, src, moms, what, taus)
    err = per_t_error(out, what, 6, moms, ref, taus)
    assert err.max() < TOL, err
    ctx.close()
