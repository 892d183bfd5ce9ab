"""Error behaviour of the C ABI on a GPU (the reference aborts through
PLEGMA_error, PLEGMA_prints.hpp:49-81, and returns silently on OOM during
tuning, PLEGMA_mesons.cuh:91-97): allocation failures come back as
P2_ERR_OOM with a message, and the context stays usable.  Nothing here
faults the GPU: the out-of-memory cases are cudaMalloc refusals."""
import ctypes as C

import numpy as np
import pytest
import torch

from plegma_b200 import lib as p2

from p2test import device_props, run

pytestmark = pytest.mark.gpu


def test_alloc_out_of_memory_status():
    ctx = p2.Context((4, 4, 4, 4))
    ptr = C.c_void_p()
    st = ctx.lib.p2_alloc(ctx.h, 1 << 46, p2.P2_DEVICE, C.byref(ptr))  # 64 TiB
    assert st == p2.P2_ERR_OOM
    assert "p2_alloc" in ctx.lib.p2_last_error(ctx.h).decode()
    bufs = device_props(ctx, [(3, 0), (3, 1)], t0=1)
    run(ctx, bufs, (0, 1, 2, 1), 4, p2.NUCLEON_CG5, q2max=1)  # still usable
    ctx.close()


@pytest.mark.parametrize("mode", [p2.P2_PLAIN_FP64, p2.P2_SPLIT_FP16])
def test_workspace_out_of_memory_recovers(mode):
    """The device is filled up to a few MB after the propagators are made; the
    contraction's workspace cannot be allocated, the call returns P2_ERR_OOM,
    and the same request succeeds with the same bits once memory is free."""
    L = (16, 16, 16, 8)
    what = p2.NUCLEON_CG5 | p2.MESON_G16
    ctx = p2.Context(L)
    bufs = device_props(ctx, [(9, 0), (9, 1)], t0=2)
    ref, _ = run(ctx, bufs, (3, 1, 2, 2), 8, what, q2max=2, mode=mode)
    ctx.close()
    ctx = p2.Context(L)  # fresh workspaces
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    hog = torch.empty(max(free - (48 << 20), 0), dtype=torch.uint8, device="cuda")
    with pytest.raises(p2.P2Error) as e:
        run(ctx, bufs, (3, 1, 2, 2), 8, what, q2max=2, mode=mode)
    assert e.value.status in (p2.P2_ERR_OOM,), e.value
    del hog
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    got, _ = run(ctx, bufs, (3, 1, 2, 2), 8, what, q2max=2, mode=mode)
    assert np.array_equal(got, ref)
    ctx.close()


def test_device_wait_timeout_is_reported_and_the_context_recovers():
    """The tensor-core projection's mbarrier waits are bounded.  With the test
    hook armed, its converters never signal their operand stages, every wait
    runs out after a short limit, the kernel drains its own bulk copies, frees
    its TMEM and returns; the call reports P2_ERR_DEVICE_TIMEOUT, and the next
    call on the same context gives the same bits as before.  No fault and no
    hang: the failure is a flag that nothing sets."""
    ctx = p2.Context((8, 8, 8, 4))
    src = (1, 2, 3, 1)
    bufs = device_props(ctx, [(21, 0), (21, 1)], t0=src[3])
    what = p2.NUCLEON_CG5 | p2.MESON_G16
    ref, _ = run(ctx, bufs, src, 4, what, q2max=2, mode=p2.P2_SPLIT_FP16)
    ctx.debug_wait_timeout()
    with pytest.raises(p2.P2Error) as e:
        run(ctx, bufs, src, 4, what, q2max=2, mode=p2.P2_SPLIT_FP16)
    assert e.value.status == p2.P2_ERR_DEVICE_TIMEOUT, e.value
    got, _ = run(ctx, bufs, src, 4, what, q2max=2, mode=p2.P2_SPLIT_FP16)
    assert np.array_equal(got, ref)
    ctx.close()
