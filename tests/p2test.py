"""Helpers shared by the GPU parity tests: synthetic propagators on the
device, a run through the C ABI, the oracle on the same bytes, and the
per-time-slice error of the spec:

    err(t) = max_{p,k} |C_gpu(t,p,k) - C_oracle(t,p,k)| / sum_x |c_k(x,t)|
"""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle_py as orc  # noqa: E402
from plegma_b200 import lib as p2  # noqa: E402


def device_props(ctx, seeds, t0, decay=0.5, precision=p2.P2_FP64, t_first=0, nt=None):
    """One device propagator per (seed, flavour) pair, generated on the GPU."""
    nt = ctx.Ll[3] if nt is None else nt
    dt = torch.complex128 if precision == p2.P2_FP64 else torch.complex64
    out = []
    for seed, flavour in seeds:
        buf = torch.empty(144 * ctx.V3 * nt, dtype=dt, device="cuda")
        ctx.synth(buf.data_ptr(), True, precision, seed, flavour, t0, decay, t_first, nt)
        out.append(buf)
    ctx.sync()
    return out


def run(ctx, bufs, source, totalT, what, q2max=None, moms=None, mode=p2.P2_PLAIN_FP64, precision=p2.P2_FP64,
        t_first=0, nt=None, pu=0, pd=1, host_props=False, host_out=False):
    nt = ctx.Ll[3] if nt is None else nt
    if moms is None:
        moms = p2.mom_list(q2max)
    blocks, total = p2.block_info(what, totalT, len(moms))
    keep = []
    props = []
    for b in bufs:
        if host_props:
            h = b.cpu().pin_memory()
            keep.append(h)
            props.append(ctx.prop(h.data_ptr(), precision, p2.P2_HOST, t_first, nt))
        else:
            props.append(ctx.prop(b.data_ptr(), precision, p2.P2_DEVICE, t_first, nt))
    if host_out:
        out = np.zeros(total, dtype=np.complex128)
        ptr, loc = out.ctypes.data, p2.P2_HOST
    else:
        outd = torch.zeros(total, dtype=torch.complex128, device="cuda")
        ptr, loc = outd.data_ptr(), p2.P2_DEVICE
    req = ctx.request(source, totalT, what, ptr, loc, mode=mode, moms=moms, prop_u=pu, prop_d=pd)
    ctx.contract_project(props, [req])
    ctx.sync()
    if not host_out:
        out = outd.cpu().numpy()
    return out, moms


def oracle_blocks(L, bufs, source, moms, what, taus, t_first=0, pu=0, pd=1, fp32=False):
    """Oracle on the exact device bytes; returns ({bit: [g][d][ntau][nmom][c]}, abs[ntau][K])."""
    u = bufs[pu].cpu().numpy().reshape(144, -1)
    d = bufs[pd].cpu().numpy().reshape(144, -1)
    out, asum, _ = orc.twopt(L, u, d, source, moms, what, taus, t_first=t_first, fp32=fp32)
    res = {}
    k0 = 0
    for bit, g, ds, c, _ in p2.block_info(what, 1, len(moms))[0]:
        n = g * ds * c
        blk = out[:, :, k0:k0 + n].reshape(len(taus), len(moms), g, ds, c).transpose(2, 3, 0, 1, 4)
        res[bit] = (blk, asum[:, k0:k0 + n].reshape(len(taus), g, ds, c).transpose(1, 2, 0, 3))
        k0 += n
    return res


def per_t_error(gpu_flat, what, totalT, moms, ref, taus):
    """max over blocks of err(t) for each tau in taus."""
    g = p2.result_blocks(what, totalT, len(moms), gpu_flat)
    errs = np.zeros(len(taus))
    for bit, (rblk, rabs) in ref.items():
        gb = g[bit][:, :, taus]  # [g][d][ntau][nmom][c]
        diff = np.abs(gb - rblk).max(axis=3)  # [g][d][ntau][c]
        e = (diff / np.maximum(rabs, 1e-300)).max(axis=(0, 1, 3))
        errs = np.maximum(errs, e)
    return errs
