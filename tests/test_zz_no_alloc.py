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
