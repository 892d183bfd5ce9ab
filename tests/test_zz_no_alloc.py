"""p2_ft_apply_noalloc, the allocation-free projection for callers that cannot
allocate device memory when they call the library (a framework that owns all
device memory through its own pool, a fixed device-memory budget).

Called through the C ABI twice in a row, it must agree with p2_ft_apply (which
allocates its workspace) within the FP64 tolerance the other projection tests
use; the second call reuses the shared static scratch left by the first.
This file is collected last so a stop-at-first-failure run has already run
every other test; it also passes on its own in a fresh process."""
import numpy as np
import pytest
import torch

from plegma_b200 import lib as p2

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _ref_and_noalloc(ctx, field_d, dof, nt, moms, sign):
    ref = torch.zeros(nt * dof * len(moms), dtype=torch.complex128, device="cuda")
    ctx.ft_apply(field_d.data_ptr(), dof, nt, moms, sign, ref.data_ptr(), p2.P2_DEVICE)
    got = torch.full_like(ref, complex(np.nan, np.nan))
    ctx.ft_apply_noalloc(field_d.data_ptr(), dof, nt, moms, sign, got.data_ptr())
    ctx.sync()
    return ref.cpu().numpy(), got.cpu().numpy()


def test_no_alloc_matches_allocating_projection_twice():
    ctx = p2.Context((6, 5, 4, 4))
    rng = np.random.default_rng(77)
    cases = [(9, 4, p2.mom_list(3), -1), (3, 2, p2.mom_list(1), 1)]
    for dof, nt, moms, sign in cases:  # two calls in a row, different shapes, shared scratch
        f = rng.standard_normal((dof, ctx.V3 * nt)) + 1j * rng.standard_normal((dof, ctx.V3 * nt))
        fd = torch.from_numpy(f.reshape(-1)).cuda()
        ref, got = _ref_and_noalloc(ctx, fd, dof, nt, moms, sign)
        assert np.all(np.isfinite(got))
        assert np.abs(got - ref).max() / np.abs(ref).max() < TOL
    ctx.close()


def test_no_alloc_on_a_spatial_sub_lattice():
    """A rank holding the second half of x (p2_geom coords (1, 0, 0, 0)): the
    phase tables must use global coordinates, as p2_ft_apply's do."""
    ctx = p2.Context((8, 6, 4, 4), procs=(2, 1, 1, 1), coords=(1, 0, 0, 0))
    rng = np.random.default_rng(78)
    dof, nt, moms = 5, 4, p2.mom_list(2)
    f = rng.standard_normal((dof, ctx.V3 * nt)) + 1j * rng.standard_normal((dof, ctx.V3 * nt))
    fd = torch.from_numpy(f.reshape(-1)).cuda()
    for _ in range(2):
        ref, got = _ref_and_noalloc(ctx, fd, dof, nt, moms, -1)
        assert np.abs(got - ref).max() / np.abs(ref).max() < TOL
    ctx.close()


def test_no_alloc_at_the_scratch_limit():
    """Partial sums that fill the scratch to within a few kB (one site split
    fits): accepted, and equal to p2_ft_apply."""
    ctx = p2.Context((8, 8, 8, 1))
    moms = p2.mom_list(9)
    nmom = len(moms)
    tabs = ((3 * nmom * 4 + 255) // 256 + (3 * nmom * 8 * 16 + 255) // 256) * 256
    dof = ((32 << 20) - tabs) // (nmom * 16)
    assert dof * nmom * 16 + tabs <= (32 << 20) < (dof + 1) * nmom * 16 + tabs
    rng = np.random.default_rng(79)
    f = (rng.standard_normal((dof, ctx.V3)) + 1j * rng.standard_normal((dof, ctx.V3))).astype(np.complex128)
    fd = torch.from_numpy(f.reshape(-1)).cuda()
    ref, got = _ref_and_noalloc(ctx, fd, dof, 1, moms, -1)
    assert np.all(np.isfinite(got))
    assert np.abs(got - ref).max() / np.abs(ref).max() < TOL
    ctx.close()


def test_no_alloc_rejects_requests_beyond_the_scratch():
    ctx = p2.Context((4, 4, 4, 8))
    big_dof = (32 << 20) // (8 * 123 * 16) + 1  # nt * nmom * dof * 16 bytes > 32 MiB
    fd = torch.zeros(1, dtype=torch.complex128, device="cuda")
    out = torch.zeros(1, dtype=torch.complex128, device="cuda")
    with pytest.raises(p2.P2Error) as e:
        ctx.ft_apply_noalloc(fd.data_ptr(), big_dof, 8, p2.mom_list(9), -1, out.data_ptr())
    assert e.value.status == p2.P2_ERR_INVALID_ARG
    assert "32 MiB" in str(e.value)
    ctx.close()
