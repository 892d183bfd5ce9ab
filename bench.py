#!/usr/bin/env python
"""Benchmark: hadron two-point contraction + momentum projection at 48^3 x 96.

Workload (one step): one source, both Wick contractions of the nucleon C g5
(2 datasets x 16 open spin) plus all 16 x 16 meson Gamma insertions
(K = 288 components per site), projected onto the 123 momenta |n|^2 <= 9 for
all 96 time slices = 10,616,832 sites.  Propagators u, d: seeded synthetic
FP64 (Gaussian entries x exp(-0.5 |t - t0|)), 24.5 GB each, resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form split|plain]

Under torchrun each rank contracts its own source (seed + rank): the path
shards by source with no data exchange, so scaling is weak and the value is
all ranks' sites over the slowest rank's time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L = (48, 48, 48, 96)
Q2MAX = 9
SEED = 1003
METRIC = "2pt contraction+projection sites/s at 48^3x96"
WORKLOAD = "48^3x96 nucleon Cg5 (2x16) + 16x16 meson Gamma pairs, K=288, |n|^2<=9 (123 momenta), 1 source, 96 slices"


def source_for(seed):
    rng = np.random.default_rng(seed)
    return (int(rng.integers(0, L[0])), int(rng.integers(0, L[1])), int(rng.integers(0, L[2])),
            int(rng.integers(0, L[3])))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.stop = threading.Event()
        self.th = None

    def _run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.th.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 4 + i and r[4 + i].lower().startswith("active"):
                    reasons.add(n)
        pw = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "samples": len(self.rows), "reasons": sorted(reasons)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def cpu_baseline_port(steps=1, slices_per_step=4):
    """The FP64 oracle (faithful restatement of the reference loops, OpenMP on
    all host cores) timed on full 48^3 time slices of the benchmark workload
    (K = 288 components, 123 momenta; 110,592 sites per slice, 255 MB per
    slice and flavour, far larger than the host caches).  Each step
    contracts and projects `slices_per_step` slices; the step's value is its
    sites over its time, the result the median over steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as orc
    from plegma_b200 import spin
    nsl = 4
    Ls = (48, 48, 48, nsl)
    V3 = 48 ** 3
    rng = np.random.default_rng(SEED)
    u = np.empty((144, V3 * nsl), dtype=np.complex128)
    d = np.empty_like(u)
    for a in (u, d):
        a.real = rng.standard_normal(a.shape)
        a.imag = rng.standard_normal(a.shape)
    moms = np.array(spin.create_mom(Q2MAX), dtype=np.int32)
    src = (1, 2, 3, 0)
    orc.twopt((16, 16, 16, 1), u[:, :4096], d[:, :4096], src, moms, 1 | 8, [0], want_abs=False)  # thread pool up
    vals, n = [], 0
    for _ in range(steps):
        t = time.perf_counter()
        for _ in range(slices_per_step):
            orc.twopt(Ls, u, d, src, moms, 1 | 8, [n % nsl], want_abs=False)
            n += 1
        vals.append(slices_per_step * V3 / (time.perf_counter() - t))
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            model = next((l.split(":", 1)[1].strip() for l in f if l.startswith("model name")), "")
    except OSError:
        pass
    return {"value": float(np.median(vals)), "unit": "sites/s", "cores": cores, "cpu_model": model,
            "nproc": os.cpu_count(), "kind": "port",
            "sample": f"full 48^3 time slices ({V3} sites each), K=288, 123 momenta, FP64 oracle: {n} slices in "
                      f"{steps} step(s) of {slices_per_step}, median over steps"}


class SliceChecker:
    """Per-time-slice error of a run's own output against the FP64 oracle,
    evaluated outside the timed region on a few slices (the source slice,
    its neighbours, the middle of the lattice and the slice farthest from
    the source, where the baryons are smallest):
        err(t) = max_{p,k} |C(t,p,k) - C_oracle(t,p,k)| / sum_x |c_k(x,t)|.
    The oracle runs once per slice on a host copy of that slice only."""

    def __init__(self, u, d, src, moms, what, T, V3):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_py as orc
        from plegma_b200 import lib as p2
        self.p2, self.moms, self.what, self.T = p2, moms, what, T
        far = 0 if src[3] >= T - 1 - src[3] else T - 1
        self.taus = sorted({0, 1, T // 2, T - 1, (far - src[3]) % T})
        self.ref = {}
        for tau in self.taus:
            t = (src[3] + tau) % T
            hu = u.view(144, -1, V3)[:, t, :].cpu().numpy()
            hd = d.view(144, -1, V3)[:, t, :].cpu().numpy()
            out, asum, _ = orc.twopt(L, hu, hd, src, moms, what, [tau], t_first=t)
            self.ref[tau] = (out[0], asum[0])

    def errors(self, flat):
        p2 = self.p2
        res = p2.result_blocks(self.what, self.T, len(self.moms), flat)
        errs = []
        for tau in self.taus:
            out, asum = self.ref[tau]
            k0, e = 0, 0.0
            for bit, g, ds, c, _ in p2.block_info(self.what, 1, len(self.moms))[0]:
                n = g * ds * c
                ref = out[:, k0:k0 + n].reshape(len(self.moms), g, ds, c).transpose(1, 2, 0, 3)
                diff = np.abs(res[bit][:, :, tau] - ref).max(axis=2)
                e = max(e, float((diff / np.maximum(asum[k0:k0 + n].reshape(g, ds, c), 1e-300)).max()))
                k0 += n
            errs.append(e)
        return {"taus": self.taus, "err_t": errs, "max_err_t": max(errs)}


def run_reference(args, rank, world):
    if rank != 0:
        return
    # each step one full 48^3 time slice of the workload (about a second on 16
    # host cores), so that --steps 40 ends in about a minute
    if args.warmup > 0:
        cpu_baseline_port(args.warmup, slices_per_step=1)
    t = time.perf_counter()
    cb = cpu_baseline_port(args.steps, slices_per_step=1)
    el = time.perf_counter() - t
    v = cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "sites/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "sample": cb["sample"]},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "sites/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes (read + write) per site of the dominant kernel, measured with ncu
# on the 32^3 x 16 case of the same kernel; traffic grows with the sites a
# launch processes, so it scales to the benchmark's launches
TRAFFIC_PER_SITE = {("contract_f32", "split"): 6864, ("contract_plain_fp64", "plain"): 9129}
# executed FP64 flop per site of the plain site contraction (2 per DFMA, 1 per
# DADD / DMUL, from the ncu instruction counters of the 32^3 x 16 case)
FP64_FLOP_PER_SITE = {"contract_plain_fp64": 50336}
# LSU data-pipe wavefronts per site of the split site contraction (ncu
# l1tex__data_pipe_lsu_wavefronts.sum / sites, 32^3 x 16 case): its binding
# on-chip limit, one wavefront (128 bytes between shared memory and the
# registers) per SM and clock
LSU_WAVEFRONTS_PER_SITE = {"contract_f32": 394.8}

BATCHED = {
    # name: (lattice, sources, window range, |n|^2 max, propagator precision, decay, seed, sources resident at once)
    "batched_32x64": ((32, 32, 32, 64), 16, (8, 20), 9, "fp64", 0.5, 1004, 16),
    # every source over all 128 slices: one FP32 source pair is 77 GB, so the
    # sources are streamed through HBM one at a time (each timed while resident)
    "batched_64x128": ((64, 64, 64, 128), 4, (128, 128), 16, "fp32", 0.4, 1005, 1),
}
BATCH_WORKSPACE = 32 << 30  # position-buffer chunk budget of the batched runs (fewer, larger chunks per graph)


def run_batched(name, stream, steps, warmup, forms=("split",)):
    """Many sources with uneven windows, each group of resident sources
    replayed as one recorded CUDA graph per step: nucleon C g5 + Delta C g_k
    (both isospins) + 16x16 mesons (K = 480).  Propagators are stored for each
    source's window only (t_first = t0, nt = window).  When the sources do not
    fit in HBM together they are streamed: each group is generated (untimed),
    its graph timed over `steps` replays, and a step's time is the sum over
    the groups."""
    import torch
    from plegma_b200 import lib as p2
    Lb, nsrc, (wmin, wmax), q2, prec, decay, seed, resident = BATCHED[name]
    what = p2.NUCLEON_CG5 | p2.DELTA_ISO12 | p2.DELTA_ISO32 | p2.MESON_G16
    K = p2.components(what)
    moms = p2.mom_list(q2)
    ctx = p2.Context(Lb)
    ctx.set_stream(stream.cuda_stream)
    free, _ = torch.cuda.mem_get_info()
    V3 = Lb[0] * Lb[1] * Lb[2]
    rng = np.random.default_rng(seed)
    P = p2.P2_FP32 if prec == "fp32" else p2.P2_FP64
    dt = torch.complex64 if prec == "fp32" else torch.complex128
    esz = 8 if prec == "fp32" else 16
    srcs = []
    for i in range(nsrc):
        src = tuple(int(rng.integers(0, Lb[dd])) for dd in range(4))
        srcs.append((src, int(rng.integers(wmin, wmax + 1))))
    props_bytes = max(2 * 144 * V3 * W * esz for _, W in srcs) * resident
    ctx.set_workspace(int(min(BATCH_WORKSPACE, max(free - props_bytes - (8 << 30), 1 << 30))))
    ctx.tune(True)
    sites = sum(W for _, W in srcs) * V3
    res = {"workload": f"{Lb[0]}^3x{Lb[3]}, {nsrc} sources, windows {wmin}-{wmax} (sum {sites // V3} slices), "
                       f"nucleon Cg5 + Delta Cg_k (iso 1/2, 3/2) + 16x16 mesons, K={K}, |n|^2<={q2} "
                       f"({len(moms)} momenta), {prec} propagators stored per window" +
                       (f", {resident} source(s) resident at a time" if resident < nsrc else ""),
           "sites_per_step": sites,
           "launch": "one CUDA graph per step (p2_graph_launch)" if resident >= nsrc else
                     f"one CUDA graph per resident group of {resident} source(s), {nsrc // resident} groups per step",
           "forms": {}}
    for form in forms:
        mode = p2.P2_SPLIT_FP16 if form == "split" else p2.P2_PLAIN_FP64
        ms_total, prof_tot, clocks, launches = 0.0, {}, [], 0
        for g0 in range(0, nsrc, resident):
            group = srcs[g0:g0 + resident]
            bufs, props, outs, reqs = [], [], [], []
            for i, (src, W) in enumerate(group):
                for f in range(2):
                    b = torch.empty(144 * V3 * W, dtype=dt, device="cuda")
                    ctx.synth(b.data_ptr(), True, P, seed + g0 + i, f, src[3], decay, src[3], W)
                    bufs.append(b)
                    props.append(ctx.prop(b.data_ptr(), P, p2.P2_DEVICE, src[3], W))
                _, total = p2.block_info(what, W, len(moms))
                o = torch.zeros(total, dtype=torch.complex128, device="cuda")
                outs.append(o)
                reqs.append(ctx.request(src, W, what, o.data_ptr(), mode=mode, moms=moms, prop_u=2 * i,
                                        prop_d=2 * i + 1))
            # per-kernel device time from one eager call (graph replays are not split by kernel)
            ctx.profile(True)
            ctx.profile_read(reset=True)
            ctx.contract_project(props, reqs)
            ctx.sync()
            prof = ctx.profile_read(reset=True)
            ctx.profile(False)
            for k, v in prof.items():
                a = prof_tot.setdefault(k, [0, 0.0])
                a[0] += v[0]
                a[1] += v[1]
            g = ctx.graph(props, reqs)
            for _ in range(warmup):
                g.launch()
            g.sync()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            with ClockSampler(torch.cuda.current_device()) as clk:
                ev0.record(stream)
                for _ in range(steps):
                    g.launch()
                ev1.record(stream)
                torch.cuda.synchronize()
            g.sync()
            ms_total += ev0.elapsed_time(ev1) / steps
            clocks.append(clk.summary())
            launches += sum(v[0] for v in prof.values())
            g.close()
            del outs, bufs
            torch.cuda.empty_cache()
        tot = sum(v[1] for v in prof_tot.values()) or 1.0
        sm = [c["sm_mhz"] for c in clocks if c.get("sm_mhz")]
        res["forms"][form] = {"ms_per_step": ms_total, "sites_per_s": sites / (ms_total * 1e-3), "steps": steps,
                              "kernels": {k: {"launches": v[0], "ms": v[1], "share": v[1] / tot}
                                          for k, v in prof_tot.items() if v[0]},
                              "gpu_launches_per_step": launches,
                              "clocks": {"sm_mhz": statistics.median(sm) if sm else None,
                                         "reasons": sorted({r for c in clocks for r in c.get("reasons", [])})}}
    res["tuned_shapes"] = ctx.tune_count()
    res["seed"] = seed
    ctx.close()
    torch.cuda.empty_cache()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="auto", choices=["auto", "split", "plain"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched multi-source graph runs")
    ap.add_argument("--no-check", action="store_true", help="skip the per-slice error check against the oracle")
    ap.add_argument("--tune-cache", default=None,
                    help="tab-separated launch-shape cache: read if present, written after tuning "
                         "(lets a profiler run skip the tuning launches)")
    ap.add_argument("--lattice", default=None,
                    help="Lx,Ly,Lz,Lt override for small profiling cases (not the benchmark workload)")
    ap.add_argument("--what", default="metric", choices=["metric", "delta"],
                    help="contraction set of a profiling case: the metric's (nucleon + 16x16 mesons) or the batched "
                         "configurations' (with both Delta isospins, K = 480)")
    args = ap.parse_args()
    global L
    if args.lattice:
        L = tuple(int(x) for x in args.lattice.split(","))

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    lw = int(os.environ.get("LOCAL_WORLD_SIZE", "1"))
    if lw > 1 and "OMP_NUM_THREADS" not in os.environ:
        # the host-side conversion of the end-to-end run: the node's cores shared between its ranks
        os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or lw) // lw))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from plegma_b200 import lib as p2
    ctx = p2.Context(L, device=local)
    # a dedicated (non-default) stream shared by torch's events and the library
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ctx.tune(True, args.tune_cache)  # launch shapes timed during the warm-up steps, cached in memory

    seed = SEED + rank
    src = source_for(seed)
    V3 = L[0] * L[1] * L[2]
    sites = V3 * L[3]
    what = p2.NUCLEON_CG5 | p2.MESON_G16
    if args.what == "delta":
        if not args.lattice:
            ap.error("--what delta is a profiling case: give --lattice")
        what |= p2.DELTA_ISO12 | p2.DELTA_ISO32
    K = p2.components(what)
    moms = p2.mom_list(Q2MAX)
    nmom = len(moms)
    blocks, total = p2.block_info(what, L[3], nmom)
    u = torch.empty(144 * sites, dtype=torch.complex128, device="cuda")
    d = torch.empty_like(u)
    ctx.synth(u.data_ptr(), True, p2.P2_FP64, seed, 0, src[3], 0.5)
    ctx.synth(d.data_ptr(), True, p2.P2_FP64, seed, 1, src[3], 0.5)
    out = torch.zeros(total, dtype=torch.complex128, device="cuda")
    props = [ctx.prop(u.data_ptr(), nt=L[3]), ctx.prop(d.data_ptr(), nt=L[3])]

    forms = {}
    if args.form in ("auto", "split"):
        forms["split"] = p2.P2_SPLIT_FP16
    if args.form in ("auto", "plain"):
        forms["plain"] = p2.P2_PLAIN_FP64

    def step(mode):
        ctx.contract_project(props, [ctx.request(src, L[3], what, out.data_ptr(), mode=mode, q2max=Q2MAX)])

    results = {}
    hbm, bf16, peak_kind = peaks()
    # FP64 FMA rate of this device (the plain form's FP64 roofline), clocks sampled meanwhile
    with ClockSampler(local) as clk64:
        fp64_tflops, fp64_ms = ctx.fp64_rate()
    fp64 = {"tflops": fp64_tflops, "kernel": "k_fp64_fma_rate (8 FMA chains/thread, 8 x 256 threads/SM)",
            "launch_ms": fp64_ms, "clocks": clk64.summary()}
    checker = SliceChecker(u, d, src, moms, what, L[3], V3) if (rank == 0 and not args.no_check) else None
    for name, mode in forms.items():
        try:
            step(mode)
        except p2.P2Error as e:
            if e.status == p2.P2_ERR_UNSUPPORTED and args.form == "auto":
                continue
            raise
        for _ in range(max(args.warmup - 1, 0)):
            step(mode)
        torch.cuda.synchronize()
        ctx.profile(True)
        ctx.profile_read(reset=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            ev0.record(stream)
            for _ in range(args.steps):
                step(mode)
            ev1.record(stream)
            torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = ev0.elapsed_time(ev1) / args.steps
        prof = ctx.profile_read(reset=True)
        ctx.profile(False)
        if dist:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        results[name] = {"ms": ms, "prof": prof, "clocks": clk.summary()}
        if checker is not None:  # the timed run's own output, checked after the timed region
            results[name]["err"] = checker.errors(out.cpu().numpy())

    head = "split" if "split" in results else "plain"
    r = results[head]
    ms = r["ms"]
    value = sites * world / (ms * 1e-3)
    prof = r["prof"]
    launches = sum(v[0] for v in prof.values())
    tot_ms = sum(v[1] for v in prof.values()) or 1.0
    kernels = {k: {"launches": v[0], "ms_per_step": v[1] / args.steps, "share": v[1] / tot_ms}
               for k, v in prof.items()}
    # roofline of the site-contraction kernel (HBM bound; the spec's figure is
    # the 2 x 144 complex propagator entries per site)
    ck = [k for k in prof if k.startswith("contract")]
    roof = None
    if ck:
        kname = ck[0]
        n, kms = prof[kname]
        bytes_per_site = 2 * 144 * 16  # algorithmic: both FP64 propagators once
        per_launch = sites * args.steps / max(n, 1)
        ach = bytes_per_site * sites * args.steps / (kms * 1e-3) / 1e9
        tps = TRAFFIC_PER_SITE.get((kname, head))
        roof = {"kernel": kname, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "peak_kind": peak_kind,
                "traffic": tps * per_launch if tps else None,
                "traffic_note": "DRAM read+write bytes per site from the ncu capture of the 32^3x16 case, "
                                "times the sites of one launch" if tps else None,
                "algorithmic_bytes_per_launch": bytes_per_site * per_launch, "sites_per_launch": per_launch}
    # the split contraction against its on-chip bound: the LSU data pipe's one
    # wavefront per SM and clock, at the median SM clock sampled in the timed region
    roof_lsu = None
    if ck and LSU_WAVEFRONTS_PER_SITE.get(ck[0]) and r["clocks"].get("sm_mhz"):
        n, kms = prof[ck[0]]
        nsm = torch.cuda.get_device_properties(0).multi_processor_count
        wf = LSU_WAVEFRONTS_PER_SITE[ck[0]]
        floor_ms = wf * sites / (nsm * r["clocks"]["sm_mhz"] * 1e6) * 1e3
        ms_k = kms / args.steps
        roof_lsu = {"kernel": ck[0], "bound": "lsu data pipe (1 wavefront / SM / clock)",
                    "wavefronts_per_site": wf, "wavefronts_source": "ncu, 32^3x16 case",
                    "sm_mhz": r["clocks"]["sm_mhz"], "sms": nsm, "floor_ms_per_step": floor_ms,
                    "ms_per_step": ms_k, "frac": floor_ms / ms_k if ms_k > 0 else None}
    # the projection against the tensor (split) or FP64 (plain) roofline, algorithmic flop = 8 nmom K per site
    roof_proj = None
    pk = [k for k in prof if k.startswith("project")]
    if pk:
        n, kms = prof[pk[0]]
        flop = 8.0 * nmom * K * sites * args.steps
        ach = flop / (kms * 1e-3) / 1e12
        roof_proj = {"kernel": pk[0], "bound": "tensor" if head == "split" else "fp64", "achieved": ach,
                     "unit": "TFLOP/s", "algorithmic_flop_per_launch": flop / max(n, 1)}
        if head == "split":
            roof_proj.update({"peak": bf16, "frac": ach / bf16, "peak_kind": peak_kind + " dense bf16 (= fp16)"})

    # the plain form's FP64 kernels against the measured FP64 FMA rate: the
    # projection's algorithmic 8 nmom K flop per site, and the contraction's
    # executed FP64 flop per site (2 per DFMA, 1 per DADD/DMUL) from ncu
    roof64 = None
    if "plain" in results:
        pp = results["plain"]["prof"]
        roof64 = {"peak": fp64_tflops, "unit": "TFLOP/s", "peak_kind": "measured (p2_measure_fp64_rate)"}
        for kname, kms in pp.items():
            if kname.startswith("project"):
                fl = 8.0 * nmom * K
            elif kname.startswith("contract") and FP64_FLOP_PER_SITE.get(kname):
                fl = FP64_FLOP_PER_SITE[kname]
            else:
                continue
            if kms[1] <= 0:
                continue
            ach = fl * sites * args.steps / (kms[1] * 1e-3) / 1e12
            roof64[kname] = {"achieved": ach, "frac": ach / fp64_tflops, "flop_per_site": fl,
                             "flop_kind": "algorithmic" if kname.startswith("project") else "executed (ncu)"}
        if "contract_plain_fp64" in pp:
            n, kms = pp["contract_plain_fp64"]
            ach = 2 * 144 * 16 * sites * args.steps / (kms * 1e-3) / 1e9
            roof64["contract_plain_fp64_hbm"] = {"achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                                                 "target_frac": 0.7}

    # end to end through the C ABI with host buffers (pinned), copies inside the timed region
    e2e = None
    if not args.no_e2e:
        try:
            import psutil
            avail = psutil.virtual_memory().available
        except Exception:
            avail = 0
        need = 2 * u.numel() * 16 + (8 << 30)
        ok = avail > need * int(os.environ.get("LOCAL_WORLD_SIZE", "1"))
        if dist:  # every rank takes the same collective steps: all run it or none
            flag = torch.tensor([1 if ok else 0], device="cuda")
            dist.all_reduce(flag, op=dist.ReduceOp.MIN)
            ok = bool(flag.item())
        if ok:
            hu = torch.empty(u.numel(), dtype=torch.complex128, pin_memory=True)
            hd = torch.empty(u.numel(), dtype=torch.complex128, pin_memory=True)  # empty_like does not pin
            hu.copy_(u)
            hd.copy_(d)
            del u, d
            torch.cuda.empty_cache()
            hout = np.zeros(total, dtype=np.complex128)
            hprops = [ctx.prop(hu.data_ptr(), location=p2.P2_HOST, nt=L[3]),
                      ctx.prop(hd.data_ptr(), location=p2.P2_HOST, nt=L[3])]

            def estep():
                ctx.contract_project(hprops, [ctx.request(src, L[3], what, hout.ctypes.data, p2.P2_HOST,
                                                          mode=forms[head], q2max=Q2MAX)])
            estep()
            torch.cuda.synchronize()
            ctx.profile(True)
            ctx.profile_read(reset=True)
            if dist:
                dist.barrier()
            t = time.perf_counter()
            n_e = max(1, min(args.steps, 3))
            for _ in range(n_e):
                estep()
            torch.cuda.synchronize()
            el = (time.perf_counter() - t) / n_e
            if dist:  # the slowest rank's wall clock
                te = torch.tensor([el], device="cuda", dtype=torch.float64)
                dist.all_reduce(te, op=dist.ReduceOp.MAX)
                el = float(te.item())
            eprof = ctx.profile_read(reset=True)
            ctx.profile(False)
            e2e = {"value": sites * world / el, "unit": "sites/s", "h2d_bytes_per_step": 2 * hu.numel() * 16,
                   "d2h_bytes_per_step": total * 16, "steps": n_e, "timer": "host wall clock around the C-ABI call",
                   "device_ms_per_step": {k: v[1] / n_e for k, v in eprof.items()}}
        else:
            e2e = {"value": None, "unit": "sites/s",
                   "note": f"host memory {avail >> 30} GiB < {need >> 30} GiB per rank on this node"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:  # the host baseline is reported at N = 1 only
        try:
            cpu = cpu_baseline_port(1, slices_per_step=4)
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "error": str(ex)}

    ctx.close()
    u = d = hu = hd = out = None  # release the headline's buffers before the batched runs
    batched = None
    if not args.no_batched and not args.lattice and world == 1:
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        batched = {}
        for name, forms_b in (("batched_32x64", ("split", "plain")), ("batched_64x128", ("split",))):
            try:
                batched[name] = run_batched(name, stream, max(1, min(args.steps, 3)), max(1, min(args.warmup, 2)),
                                            forms_b)
            except Exception as ex:  # reported, not fatal
                batched[name] = {"error": str(ex)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "sites/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f16x2" if head == "split" else "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "form": head, "L": list(L), "K": K, "nmom": nmom, "seed": SEED,
                           "sites_per_step": sites, "l2": "inputs (49 GB) larger than L2",
                           "parallelism": f"source-sharded x{world}"},
                "forms": {k: {"ms_per_step": v["ms"], "sites_per_s": sites * world / (v["ms"] * 1e-3),
                              "error": v.get("err")} for k, v in results.items()},
                "max_err_t": (r.get("err") or {}).get("max_err_t"),
                "err_note": "max over the checked slices of max_{p,k} |C - C_oracle| / sum_x |c_k(x,t)|, "
                            "FP64 oracle, this run's own output",
                "fp64_peak": fp64, "roofline_fp64": roof64,
                "roofline": roof, "roofline_lsu": roof_lsu, "roofline_projection": roof_proj, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": r["clocks"], "batched": batched}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
