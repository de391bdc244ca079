"""Benchmark of the block-sparse contraction (one JSON line on rank 0).

Workload: C[i,j,a,b] = sum_P A[i,a,P] B[j,b,P] at full size (i,j extent 64 in blocks of
{5,9,13}; a,b 512 in {13,25,32}; P 2048 in {32,48,64}; 15% block occupancy; seeded values).
A step is one full contraction C = A.B on the device: block matching, result pattern, work
list and the tile kernel, inputs resident in HBM.  Metric: effective GFLOP/s =
sum over pairs of 2*m*n*k / step time.  Every available FP64-accurate form is timed and the
fastest is `value`; the others are listed under `forms`.

`--impl reference` times the reference's CPU path of the same contraction (the LAPACK
path of src/Kernel/KernelImpl.cpp:142-208 with the reference's own Utils::reshape, compiled
from its sources into oracle/_ref, and OpenBLAS dgemm, one C block per OpenMP thread) on a
bounded sample of the workload, on the host cores.

Multi-GPU: the contraction does not shard in this build ("replicas only"): with --gpus N
every rank runs the same workload on its own GPU, timing is the max over ranks and `value`
the sum of the ranks' work over that time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "block-sparse contract GFLOP/s (FP64-accurate)"
WORKLOAD = "C[i,j,a,b]=sum_P A[i,a,P]*B[j,b,P]; i,j=64 in {5,9,13}; a,b=512 in {13,25,32}; P=2048 in {32,48,64}; occ 15%"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--forms", default="plain,batched,split")
    ap.add_argument("--split-tol", type=float, default=1e-12,
                    help="relative Frobenius error vs FP64 below which the split form counts as FP64-accurate")
    ap.add_argument("--scale", type=float, default=1.0, help="extent scale of the workload (1.0 = full size)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-count", action="store_true", help="skip the CUPTI launch count (use under ncu)")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--pool-gb", type=float, default=60.0)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-loop phase")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="length of the arrival stream")
    ap.add_argument("--serve-templates", type=int, default=16,
                    help="distinct requests (resident inputs) the stream draws from")
    return ap.parse_args()


# ------------------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reduce_max(x: float) -> float:
    """Max of x over the ranks of the default process group (1 rank: x itself)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(work_per_rank: float, ms_per_rank: float, world: int) -> float:
    """Whole-job rate of `world` independent replicas timed by their slowest rank (work/ms → work/s/1e6)."""
    return world * work_per_rank / reduce_max(ms_per_rank) / 1e6


def build_workload(args):
    from shtensor_b200 import workloads as W
    return W.c1(seed=args.seed, scale=args.scale)


def sample_workload(w, target_flops: float):
    """Restrict A to its first i-blocks so that the sample's pair flops are about target."""
    from shtensor_b200 import workloads as W
    import oracle
    H = lambda t: oracle.HostTensor(t.block_sizes, t.ids, t.offsets, t.data)  # noqa: E731
    idx = w.A.index_lists()
    dims = w.A.block_dims()
    ni = len(w.A.block_sizes[0])
    # flops per i-block, estimated from A block sizes x matching B volume per P block
    Bidx = w.B.index_lists()
    bvol = np.zeros(len(w.B.block_sizes[2]))
    bd = w.B.block_dims()
    np.add.at(bvol, Bidx[2], bd[:, 0] * bd[:, 1])
    per_i = np.zeros(ni)
    np.add.at(per_i, idx[0], 2.0 * dims[:, 0] * dims[:, 1] * dims[:, 2] * bvol[idx[2]])
    k = 1
    while k < ni and per_i[:k].sum() < target_flops:
        k += 1
    keep = idx[0] < k
    sizes = dims.prod(axis=1)
    offs = np.concatenate([[0], np.cumsum(sizes[keep])[:-1]]).astype(np.int64)
    data = np.concatenate([w.A.data[o:o + s] for o, s in zip(w.A.offsets[keep], sizes[keep])])
    A = W.HostBlockSparse(w.A.block_sizes, w.A.ids[keep], offs, data)
    return W.Workload(w.name, w.expr, A, w.B, w.C), k, ni, H


def cpu_reference_run(w, seconds: float, nthreads: int):
    """Time the reference CPU path on a sample sized to run about `seconds`."""
    import oracle
    H = lambda t: oracle.HostTensor(t.block_sizes, t.ids, t.offsets, t.data)  # noqa: E731
    use_ref = oracle.ref_lib() is not None
    kind = "reference" if use_ref else "port"
    # calibrate on a small sample, then size the timed sample
    probe, k, ni, _ = sample_workload(w, 2e9)
    r = oracle.contract(probe.expr, 1.0, H(probe.A), H(probe.B), 0.0, H(probe.C), nthreads=nthreads, ref=use_ref,
                        lapack_blocks=not use_ref)
    rate = r.flops / max(r.seconds, 1e-6)
    samp, k, ni, _ = sample_workload(w, rate * seconds)
    r = oracle.contract(samp.expr, 1.0, H(samp.A), H(samp.B), 0.0, H(samp.C), nthreads=nthreads, ref=use_ref,
                        lapack_blocks=not use_ref)
    desc = (f"A restricted to i-blocks 0..{k - 1} of {ni}: {len(r.pairs)} pairs, {r.flops / 1e9:.2f} GFLOP "
            f"({'reference Utils::reshape + OpenBLAS dgemm per pair' if use_ref else 'oracle LAPACK-path restatement'}, "
            f"OpenMP over C blocks)")
    return r.flops / r.seconds / 1e9, kind, desc, r.seconds


def count_launches(fn):
    """Kernels launched by fn(), counted from the CUDA activity trace (CUPTI via torch)."""
    import torch
    try:
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        names = [e.name for e in prof.events() if e.device_type.name == "CUDA" and "memcpy" not in e.name.lower()
                 and "memset" not in e.name.lower()]
        return len(names), names
    except Exception as ex:  # profiler unavailable
        return None, [str(ex)]


def measure_peak(sht, ctx, which):
    try:
        return sht.measure_peak(ctx, which)
    except Exception:
        return None


def run_serving(args, sht, ctx, upload, server_kwargs=None):
    """Serving phase: a seeded Poisson stream of mixed contractions through sht.Server.

    Requests are drawn from `serve_templates` distinct contractions of the c0..c3 families
    (extents x U(0.25,1), occupancy U(0.05,0.4)), whose inputs stay resident; each request
    writes its own fresh C, released when it completes.  Reported beside it: the same
    requests each run alone on the plain FP64 path (synchronous sht_contract, no queueing),
    a burst of the whole stream submitted at once (the loop's capacity), and a bit-equality
    check of served results against the same requests run alone."""
    from shtensor_b200 import workloads as W
    rng = np.random.default_rng(args.seed + 1000)
    t_gen = time.perf_counter()
    temps = [W.c4_request(rng) for _ in range(args.serve_templates)]
    gen_s = time.perf_counter() - t_gen
    ins = [(upload(w.A), upload(w.B)) for w in temps]
    n = max(1, int(round(args.serve_rate * args.serve_seconds)))
    picks = rng.integers(0, len(temps), n)
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n))

    def fresh_c(w):
        return upload(W.empty_tensor(w.C.block_sizes))

    # each template alone on the plain path: plan + execute to completion, median of 3 after one
    import torch
    alone_ms, tflops = [], []
    for w, (A, B) in zip(temps, ins):
        ts = []
        for r in range(4):
            C = fresh_c(w)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rep = sht.contract(ctx, w.expr, 1.0, A, B, 0.0, C, w.screen_eps, mode=sht.Mode.PLAIN_FP64)
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
            del C
        alone_ms.append(float(np.median(ts[1:])))
        tflops.append(rep["flops"])
    alone_stream = np.array([alone_ms[k] for k in picks])
    stream_flops = float(sum(tflops[k] for k in picks))

    def pct(v, q):
        v = np.sort(np.asarray(v))
        return float(v[min(len(v) - 1, max(0, int(np.ceil(q * len(v))) - 1))])

    out = {"rate_per_s": args.serve_rate, "requests": n, "stream_s": float(arrivals[-1]),
           "templates": [{"family": w.meta["family"], "u": round(w.meta["u"], 3),
                          "occupancy": round(w.meta["occupancy"], 3), "gflop": f / 1e9,
                          "alone_plain_ms": a} for w, f, a in zip(temps, tflops, alone_ms)],
           "template_gen_s": gen_s, "offered_gflops": stream_flops / float(arrivals[-1]) / 1e9}
    out["alone_plain"] = {"p50_ms": pct(alone_stream, 0.5), "p99_ms": pct(alone_stream, 0.99),
                          "gflops": stream_flops / (alone_stream.sum() / 1e3) / 1e9,
                          "busy_s": float(alone_stream.sum() / 1e3)}
    keep_check = {}
    with sht.Server(ctx, **(server_kwargs or {})) as srv:
        # warm-up: every template once
        for w, (A, B) in zip(temps, ins):
            C = fresh_c(w)
            srv.wait(srv.submit(w.expr, 1.0, A, B, 0.0, C, w.screen_eps), 300)
            del C
        for phase in ("stream", "burst"):
            srv.reset_stats()
            pending = {}
            reps = []
            t0 = time.perf_counter()
            i = 0
            while i < n or pending:
                now = time.perf_counter() - t0
                while i < n and (phase == "burst" or arrivals[i] <= now):
                    k = int(picks[i])
                    w, (A, B) = temps[k], ins[k]
                    C = fresh_c(w)
                    t_sub = time.perf_counter() - t0
                    pending[srv.submit(w.expr, 1.0, A, B, 0.0, C, w.screen_eps)] = (C, k, t_sub)
                    i += 1
                for rid in list(pending):
                    if srv.poll(rid):
                        rep = srv.wait(rid, 300)
                        C, k, t_sub = pending.pop(rid)
                        rep.update(template=k, submit_s=round(t_sub, 4))
                        reps.append(rep)
                        if phase == "stream" and k not in keep_check and len(keep_check) < 6:
                            keep_check[k] = C
                        del C
                time.sleep(0.0002)
            st = srv.stats()
            out[phase] = {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
                          "gflops": st["gflops"], "span_s": st["span_s"], "completed": st["completed"],
                          "failed": st["failed"], "launches": st["batches"], "mean_batch": st["mean_batch"],
                          "max_active": st["max_active_seen"], "deferrals": st["deferrals"],
                          "mean_queue_ms": float(np.mean([r["queue_ms"] for r in reps])),
                          "mean_plan_ms": float(np.mean([r["plan_ms"] for r in reps])),
                          "mean_run_ms": float(np.mean([r["run_ms"] for r in reps])),
                          "slowest": [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in r.items()
                                       if k in ("template", "submit_s", "queue_ms", "plan_ms", "run_ms",
                                                "latency_ms", "batch_size")}
                                      for r in sorted(reps, key=lambda r: -r["latency_ms"])[:4]]}
    # served results against the same requests run alone (batched and plain give the same bits)
    same = True
    for k, Cs in keep_check.items():
        w, (A, B) = temps[k], ins[k]
        Cr = fresh_c(w)
        sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cr, w.screen_eps, mode=sht.Mode.PLAIN_FP64)
        mx, _ = sht.compare(Cs, Cr)
        same = same and Cs.nnz == Cr.nnz and mx == 0.0
        del Cr
    out["mix_equals_alone"] = {"checked": len(keep_check), "bit_equal_values": bool(same)}
    keep_check.clear()
    del ins
    return out


# ------------------------------------------------------------------------------ arms
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    w = build_workload(args)
    vals = []
    kind = desc = None
    for _ in range(args.warmup):
        cpu_reference_run(w, max(args.cpu_sample_seconds / 5, 1.0), nthreads)
    for _ in range(args.steps):
        v, kind, desc, secs = cpu_reference_run(w, args.cpu_sample_seconds / max(args.steps, 1), nthreads)
        vals.append(v)
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "scale": args.scale, "seed": args.seed},
        "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": nthreads, "kind": kind, "sample": desc},
        "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    import shtensor_b200 as sht

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    w = build_workload(args)
    ctx = sht.Context(int(args.pool_gb * (1 << 30)), device=dev)
    stream = torch.cuda.current_stream()

    def T(h):
        t = sht.Tensor(ctx, h.block_sizes)
        t.reserve(h.index_lists() if len(h.ids) else [[] for _ in h.block_sizes])
        if h.nnz:
            t.upload(h.data)
        return t

    A, B = T(w.A), T(w.B)
    Cd = T(w.C)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    max_over_ranks = reduce_max

    forms = {"plain": sht.Mode.PLAIN_FP64, "batched": sht.Mode.BATCHED_FP64, "split": sht.Mode.SPLIT}
    results = {}
    clocks = None
    flops = None
    for fname in [f for f in args.forms.split(",") if f]:
        mode = forms[fname]
        rep = None
        if fname == "batched" and not args.no_autotune:
            tuner = sht.Plan(ctx, w.expr, A, B, Cd, mode=mode, stream=stream)
            tuner.autotune(stream=stream)
            tuner.close()
        for _ in range(args.warmup):
            rep = sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cd, mode=mode, stream=stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as cs:
            e0.record(stream)
            for _ in range(args.steps):
                rep = sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cd, mode=mode, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
        flops = rep["flops"]
        results[fname] = {"ms_per_step": ms, "gflops": world * flops / ms / 1e6, "plan_ms": rep["plan_ms"],
                          "npairs": rep["npairs"], "tiles": rep["nwork"]}
        if clocks is None or fname == "batched":
            clocks = cs.summary()
    # error of the split form against the FP64 result (both computed on the device)
    if "split" in results:
        # reference: the plain FP64 form (the drop-in, bit-exact to the XMM order); the batched
        # form must equal it bit for bit, and the split form must be within split_tol of it
        Cref = T(w.C)
        sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cref, mode=sht.Mode.PLAIN_FP64, stream=stream)
        Cb = T(w.C)
        sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cb, mode=sht.Mode.BATCHED_FP64, stream=stream)
        sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cd, mode=sht.Mode.SPLIT, stream=stream)
        mx, fro = sht.compare(Cd, Cref, stream=stream)
        bmx, _ = sht.compare(Cb, Cref, stream=stream)
        results["split"]["error_vs_fp64"] = {"max_abs": mx, "rel_fro": fro, "slices": 7,
                                             "reference": "plain FP64 form"}
        results["split"]["fp64_accurate"] = bool(fro <= args.split_tol)
        if "batched" in results:
            results["batched"]["max_abs_vs_plain"] = bmx
        del Cref, Cb
    eligible = [k for k in results if results[k].get("fp64_accurate", True)]
    best = max(eligible, key=lambda k: results[k]["gflops"])

    # execute-only timing (plan reused) of every form; the best form's kernel gives the roofline
    exec_ms = {}
    for fname in results:
        plan = sht.Plan(ctx, w.expr, A, B, Cd, mode=forms[fname], stream=stream)
        for _ in range(3):
            plan.execute(1.0, 0.0, stream=stream)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for a, b in ev:
            a.record(stream)
            plan.execute(1.0, 0.0, stream=stream)
            b.record(stream)
        torch.cuda.synchronize()
        exec_ms[fname] = float(np.mean([a.elapsed_time(b) for a, b in ev]))
        results[fname]["exec_ms"] = exec_ms[fname]
        results[fname]["exec_gflops"] = flops / exec_ms[fname] / 1e6
        prep = plan.report()
        plan.close()
        del plan
    kern_ms = exec_ms[best]
    c_nnz = Cd.nnz
    # serving runs before the launch count (the CUPTI profiler it uses slows later launches),
    # the CPU baseline (its OpenMP threads) and the end-to-end copies
    serving = None
    if world == 1 and not args.no_serving:
        serving = run_serving(args, sht, ctx, T)
    launches, names = (None, []) if args.no_count else count_launches(
        lambda: sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cd, mode=forms[best], stream=stream))
    peak = measure_peak(sht, ctx, "fp64")
    achieved = prep["flops"] / kern_ms / 1e9  # TFLOP/s
    traffic = None
    try:  # DRAM bytes per launch of the dominant kernel, from the committed ncu summary
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            traffic = json.load(f).get(best, {}).get("traffic_bytes_per_launch")
    except (OSError, ValueError):
        traffic = None
    common = {"traffic": traffic,
              "traffic_source": "profiles/roofline_traffic.json (ncu capture at scale 0.5, scaled to the full workload)",
              "algorithmic_bytes": 8.0 * (c_nnz + w.A.nnz + w.B.nnz), "kernel_ms": kern_ms,
              "kernel": {"plain": "k_contract_tiles", "batched": "k_matform + k_batched",
                         "split": "k_slice + k_split"}.get(best, best)}
    fp64_line = {"achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": (achieved / peak) if peak else None,
                 "peak_source": "measured in this run by the library's FP64 FMA-chain kernel" if peak else "unmeasured"}
    if best == "split":
        # the split kernel's bound is the INT8 tensor core: S(S+1)/2 slice products per FP64 flop
        S = int(results["split"].get("error_vs_fp64", {}).get("slices", 7))
        int8_peak = measure_peak(sht, ctx, "int8")
        int8_ach = prep["flops"] * S * (S + 1) / 2 / kern_ms / 1e9  # TOPS
        roofline = {"bound": "tensor", "pipe": f"int8 (tcgen05 kind::i8, {S} slices) with FP64 reassembly",
                    "achieved": int8_ach, "peak": int8_peak, "unit": "TOPS",
                    "frac": (int8_ach / int8_peak) if int8_peak else None,
                    "peak_source": "measured in this run by the library's tcgen05 kind::i8 kernel" if int8_peak
                    else "unmeasured",
                    "fp64_equivalent": fp64_line, **common}
    else:
        roofline = {"bound": "tensor", "pipe": "fp64 (DFMA / DMMA; B200's FP64 and FP64-tensor peaks are the same figure)",
                    **fp64_line, **common}

    # end to end through the public API: host buffers in pinned memory, copies timed
    e2e = None
    if not args.no_e2e:
        ha = torch.from_numpy(w.A.data).pin_memory()
        hb = torch.from_numpy(w.B.data).pin_memory()
        hc = torch.empty(Cd.nnz, dtype=torch.float64).pin_memory()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ee0.record(stream)
        nrep = max(2, min(args.steps, 4))
        for _ in range(nrep):
            A.upload(ha.numpy(), stream=stream)
            B.upload(hb.numpy(), stream=stream)
            sht.contract(ctx, w.expr, 1.0, A, B, 0.0, Cd, mode=forms[best], stream=stream)
            Cd.download(hc.numpy(), stream=stream)
        ee1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(ee0.elapsed_time(ee1)) / nrep
        e2e = {"value": world * flops / ms / 1e6, "unit": "GFLOP/s",
               "h2d_bytes_per_step": int(ha.numel() * 8 + hb.numel() * 8), "d2h_bytes_per_step": int(hc.numel() * 8),
               "ms_per_step": ms, "wall_ms_per_step": (time.perf_counter() - t0) * 1e3 / nrep}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, kind, desc, secs = cpu_reference_run(w, args.cpu_sample_seconds, os.cpu_count() or 1)
        cpu = {"value": v, "unit": "GFLOP/s", "cores": os.cpu_count(), "kind": kind, "sample": desc,
               "seconds": secs}

    del A, B, Cd

    if rank == 0:
        r = results[best]
        line = {
            "metric": METRIC, "value": r["gflops"], "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "form": best, "scale": args.scale, "seed": args.seed,
                       "npairs": r["npairs"], "gflop_per_step": flops / 1e9,
                       "l2": "inputs and output larger than L2 (A+B 168 MB, C 5.9 GB); no flush",
                       "c_nnz": c_nnz,
                       "parallelism": f"replicas x{world}"},
            "forms": results, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": (launches * args.steps) if launches is not None else None,
            "gpu_launches_per_step": launches, "serving": serving,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
