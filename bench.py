"""Benchmark: states/s of the exhaustive search on the n=36 integer QUBO (6-city TSP with
integer distances, seed 0), tensor-core form, with the plain Gray-code form and the CPU
restatement of the reference timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form tc|gray]

The tensor-core form runs its default kernel (for this problem the 16-bit pair form: one MMA
accumulator per two states); the other tensor-core kernels are timed beside it.

One step = one full exhaustive solve (pass 1 over all 2^36 states, candidate re-evaluation,
tie rule) of the same problem.  For N > 1 (torchrun, one process per GPU) every rank searches
its share of the tiles and the ranks exchange their minima (NCCL); the job is the same
2^36 states ("scaling": "strong").  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic work per state of the contraction: one K = 16 dot product (7 coupling bits x 2
# digits + 2 column-term digits) = 16 multiply-adds, one MMA accumulator element per state.
# The pair kernels execute half of it on the tensor pipe (one accumulator per two states).
FLOPS_PER_STATE_TC = 32
TC_VARIANTS = {"u16": {"tc_one": True}, "fp32": {"tc_no16": True}, "pair": {"tc_pair": True, "tc_no16": True}}
# profiling cases: --form name -> tensor-core kernel options
CASE_FORMS = {"tc_pair": {"tc_pair": True}, "tc_one": {"tc_one": True}, "tc_fp32": {"tc_no16": True},
              "tc_pair_fp32": {"tc_pair": True, "tc_no16": True}}
# tc_kernel name -> (search kernel, states per accumulator)
TC_KERNEL_NAMES = {"pair_u16": ("tc_pair_kernel", 2), "pair": ("tc_pair_fp32_kernel", 2)}
N_VARS = 36
WORKLOAD = "6-city TSP as QUBO, 36 variables, integer distances U{1..100} (seed 0), int32 Q"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["bf16_tflops"]), float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured"
    return 1590.0, 1400.0, "fallback"


def _traffic(kernel: str, states: int):
    """DRAM bytes (read + write) of one launch of `kernel` over `states` states, from the
    committed ncu capture profiles/<kernel>.traffic.json: the captured launch's figure when it
    covered the same number of states, else None."""
    p = os.path.join(ROOT, "profiles", f"{kernel}.traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if int(d.get("states", 0)) == int(states):
            return float(d["dram_bytes_read"]) + float(d["dram_bytes_write"])
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="qb_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            # nvidia-smi needs a moment to start: wait for its first sample before timing
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
                self.f.flush()
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.02)
        except Exception:  # noqa: BLE001
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) >= 9 and parts[1].isdigit():
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [int(r[1]) for r in rows]
        mx = int(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [v for v in sm if v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def _slice_solver(Q):
    """Returns run(m): the CPU restatement of the reference (QBF's prefix loop under
    Parallel's bit fixing, oracle/qbf_port.c) on all host cores over a slice of the
    problem -- the first n - m variables fixed to 0 (one ReducedProblem task of the
    reference's Parallel) and the remaining 2^m states searched -- timed in seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes
    import numpy as np
    import oracle
    cores = len(os.sched_getaffinity(0))
    n = Q.shape[0]
    Qf = np.ascontiguousarray(np.asarray(Q, dtype=np.float64))
    dp = ctypes.POINTER(ctypes.c_double)

    def run(m):
        Qr = np.zeros((m, m))
        oracle.lib().oq_reduce(n, Qf.ctypes.data_as(dp), n - m, 0, Qr.ctypes.data_as(dp))
        splits = 1 << max(0, min(m - 20, (cores - 1).bit_length() + 2))
        t = time.perf_counter()
        oracle.parallel_port(np.rint(Qr).astype(np.int64), splits, nthreads=cores)
        return time.perf_counter() - t, splits

    return run, cores


def _calibrate(run, n, budget_s):
    m = 28
    dt, splits = run(m)
    while dt < budget_s / 4 and m < n:
        m += 2 if dt < budget_s / 16 and m + 2 <= n else 1
        dt, splits = run(m)
    return m, dt, splits


def _sample_text(m, n, splits, dt, reps=1):
    fixed = f"the first {n - m} variables fixed to 0" if m < n else "the whole problem"
    return (f"{reps} x 2^{m} states ({fixed}), Parallel bit fixing into {splits} QBF tasks "
            f"(B = 20 prefix loop), {dt:.1f} s per pass")


def cpu_baseline(Q, budget_s: float = 15.0, min_total_s: float = 10.0) -> dict:
    """The oracle's CPU restatement of the reference on all host cores, timed over about
    10-30 s of work on the same problem."""
    run, cores = _slice_solver(Q)
    n = Q.shape[0]
    m, dt, splits = _calibrate(run, n, budget_s)
    times = [dt]
    while sum(times) < min_total_s:
        times.append(run(m)[0])
    mean = sum(times) / len(times)
    return {"value": (1 << m) / mean, "unit": "states/s", "cores": cores, "kind": "port",
            "sample": _sample_text(m, n, splits, mean, len(times))}


def bench_reference(args):
    """The reference arm: the CPU restatement of the reference's algorithm (the reference is
    a Python/cupy package that is not installed on the GPU host) on all host cores; each
    step searches one bounded slice of the same 36-variable problem."""
    from qubo_b200 import configs
    if int(os.environ.get("RANK", "0")) != 0:
        return
    Q = configs.tsp6_int()
    n = Q.shape[0]
    run, cores = _slice_solver(Q)
    # each step a bounded slice: the whole --steps/--warmup run stays within a few minutes
    step_budget = min(12.0, max(1.0, 4 * 150.0 / max(1, args.steps + args.warmup)))
    m, dt, splits = _calibrate(run, n, step_budget)  # also the warm-up
    for _ in range(max(0, args.warmup - 1)):
        run(m)
    times = [run(m)[0] for _ in range(args.steps)]
    value = (1 << m) * len(times) / sum(times)
    sample = _sample_text(m, n, splits, sum(times) / len(times))
    line = {"metric": "states/s (exhaustive QUBO, exact argmin)", "value": value, "unit": "states/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * sum(times) / len(times), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": n, "sample": sample},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "states/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "states/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bench_ours(args):
    import numpy as np
    import torch
    import qubo_b200  # noqa: F401
    from qubo_b200 import _lib, configs
    from qubo_b200.problems import Just_Q
    from qubo_b200.solvers import QBF

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    Q = configs.tsp6_int()
    n = Q.shape[0]
    states = 1 << n
    Qd = torch.as_tensor(Q, device=f"cuda:{local}")  # inputs resident in HBM
    stream = torch.cuda.current_stream(local)
    h = _lib.handle(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # > 126 MB L2

    def step(form, **kw):
        if world == 1:
            return h.solve_device(Qd.data_ptr(), n, Q.dtype, form=form, tie_rule="qbf", prefix_bits=-1,
                                  stream=stream.cuda_stream, **kw)
        from qubo_b200.distributed import solve_sharded
        return solve_sharded(Q, form=form, device=local, Q_device_ptr=Qd.data_ptr())

    def timed(form, steps, warmup, **kw):
        for _ in range(warmup):
            step(form, **kw)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        res = []
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(stream)
            res.append(step(form, **kw))
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        if dist is not None:
            dist.barrier()
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()) / steps, res

    form = args.form
    if form in CASE_FORMS:
        raise SystemExit(f"--form {form} is a profiling case option (--case cfg2 or n36); the headline times it beside tc")
    with ClockSampler(local) as clk:
        ms, res = timed(form, args.steps, args.warmup)
    clocks = clk.summary()
    gray_ms, gres = timed("gray", max(3, args.steps // 2), 3)
    variants = {}
    if form == "tc":  # the other tensor-core kernels on the same problem
        for name, kw in TC_VARIANTS.items():
            if name == res[-1]["plan"]["tc_kernel"]:
                continue
            v_ms, vres = timed("tc", max(3, args.steps // 2), 3, **kw)
            variants[name] = {"ms_per_step": v_ms, "kernel_ms": statistics.mean(r["kernel_ms"] for r in vres),
                              "tc_kernel": vres[-1]["plan"]["tc_kernel"]}
    r0 = res[-1]
    # e2e: the public API with a host-resident problem, H2D and D2H inside the timed region
    prob = Just_Q(Q)
    e2e_times, h2d, d2h = [], 0, 0
    for k in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if world == 1:
            sol = QBF().solve(prob, device=f"cuda:{local}", form=form)
            rr = sol.search
            h2d_k, d2h_k = rr.get("h2d_bytes", 0), rr.get("d2h_bytes", 0)
        else:
            from qubo_b200.distributed import solve_sharded
            rr = solve_sharded(Q, form=form, device=local)
            h2d_k, d2h_k = rr["h2d_bytes"], rr["d2h_bytes"]
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e_times.append(t1 - t0)
            h2d, d2h = h2d_k, d2h_k
    e2e_s = torch.tensor([sum(e2e_times) / len(e2e_times)], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
    e2e_value = states / float(e2e_s.item())

    kernel_ms = statistics.mean(r["kernel_ms"] for r in res)
    peak, peak_sus, peak_kind = _peaks()
    local_states = r0["states"] if world == 1 else r0["states"]
    achieved = local_states * FLOPS_PER_STATE_TC / (kernel_ms * 1e-3) / 1e12
    tck = r0["plan"]["tc_kernel"] or ""
    kernel_name = ("tc_pair_kernel" if tck.startswith("pair") else "tc_pass1_kernel") if form == "tc" else "gray_pass1_kernel"
    tensor_flops = FLOPS_PER_STATE_TC // 2 if tck.startswith("pair") else FLOPS_PER_STATE_TC
    line = {
        "metric": "states/s (exhaustive QUBO, exact argmin)",
        "value": states / (ms * 1e-3),
        "unit": "states/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32 (f16 digit operands, fp32 accumulate; exact for this integer Q)",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "form": form, "states_per_step": states,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"tile shards x{world}",
                   "answer": {"best_E": r0["best_E"], "best_X": int(r0["best_X_int"])}},
        "e2e": {"value": e2e_value, "unit": "states/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(sum(r["kernels"] for r in res)),
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": _traffic(kernel_name, local_states),
                     "kernel": kernel_name,
                     "peak_kind": f"bf16 dense burst, {peak_kind}", "kernel_ms": kernel_ms,
                     "flops_per_state": FLOPS_PER_STATE_TC, "tensor_flops_per_state": tensor_flops,
                     "frac_tensor_pipe": achieved * tensor_flops / FLOPS_PER_STATE_TC / peak},
        "gray_form": {"value": states / (gray_ms * 1e-3), "ms_per_step": gray_ms,
                      "kernel_ms": statistics.mean(r["kernel_ms"] for r in gres)},
        "tc_over_gray": (gray_ms / ms),
        "tc_kernel": r0["plan"]["tc_kernel"],
        "tc_variants": variants or None,
        "clocks": clocks,
    }
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(Q)
        # the batch configuration (4096 small problems, one graph launch per batch) beside it
        line["batch"] = batch_measure(max(10, min(args.steps, 20)), args.warmup, with_baselines=False)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def bench_case(args):
    """Profiling cases, solved `steps` times with one form, one line per solve: cfg2 = the
    32-variable integer QUBO (RandomQUBO seed 0, entries in [-100, 100], symmetric int16);
    n36 = the headline 36-variable TSP QUBO.  Used for ncu captures of a single kernel (a few
    MB on the device).  --form tc runs the tensor-core form's default kernel, tc_pair the pair
    form, tc_one one state per accumulator, tc_fp32 / tc_pair_fp32 those with fp32 minima."""
    import torch
    import qubo_b200  # noqa: F401
    from qubo_b200 import _lib, configs
    torch.cuda.set_device(0)
    Q = configs.random_i16_n32() if args.case == "cfg2" else configs.tsp6_int()
    name = "random_i16_n32" if args.case == "cfg2" else "tsp6_int_n36"
    h = _lib.handle(0)
    stream = torch.cuda.current_stream(0).cuda_stream
    form, kw = ("tc", CASE_FORMS[args.form]) if args.form in CASE_FORMS else (args.form, {})
    for k in range(args.warmup + args.steps):
        r = h.solve(Q, form=form, stream=stream, **kw)
        if k >= args.warmup:
            print(json.dumps({"case": name, "form": args.form, "best_E": r["best_E"], "states": r["states"],
                              "kernel_ms": r["kernel_ms"], "pass1_ms": r["pass1_ms"], "pass2_ms": r["pass2_ms"],
                              "tc_kernel": r["plan"]["tc_kernel"]}),
                  flush=True)


BATCH_WORKLOAD = "4096 float32 QUBOs, n uniform in [16, 28], Q = (G + G^T)/2, G ~ N(0,1), seeds 0..4095"


def batch_measure(steps: int, warmup: int, with_baselines: bool) -> dict:
    """The 4096-instance batch (n uniform in [16, 28], float Q = (G + G^T) / 2 with G normal,
    seeds 0..4095), solved with qb_solve_batch as one CUDA graph launch per batch.  Device time
    by CUDA events around the graph launch (max of nothing: one GPU); e2e = wall time of the
    public call with host-resident matrices (packing, H2D, the graph, D2H, decoding).  The
    roofline fraction covers the tensor-core pass-1 kernels of the launch-by-launch run (the
    instances with n >= 24; 32 flop per state, of which the batched 16-bit pair kernel runs half
    on the tensor pipe), against the measured bf16 peak and against the int8 dense peak (twice
    the bf16 figure, the B200's nominal ratio)."""
    import torch
    import qubo_b200  # noqa: F401
    from qubo_b200 import _lib, configs
    Qs = configs.batch_f32(4096)
    states = sum(1 << q.shape[0] for q in Qs)
    tc_states = sum(1 << q.shape[0] for q in Qs if q.shape[0] >= 24)
    h = _lib.handle(0)
    stream = torch.cuda.current_stream(0).cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda:0")
    for _ in range(max(3, warmup)):
        h.solve_batch(Qs, stream=stream, graph=True)
        h.solve_batch(Qs, stream=stream)
    g_ms, wall, p_ms, k_ms = [], [], [], []
    res = None
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = h.solve_batch(Qs, stream=stream, graph=True)
        wall.append(time.perf_counter() - t0)
        g_ms.append(res[0]["pass1_ms"])
    for _ in range(steps):
        flush.zero_()
        r2 = h.solve_batch(Qs, stream=stream)
        p_ms.append(r2[0]["pass1_ms"] + r2[0]["pass2_ms"])
        k_ms.append(r2[0]["kernel_ms"])
    ms = statistics.median(g_ms)
    peak, _, peak_kind = _peaks()
    kms = statistics.median(k_ms)
    tflops = tc_states * FLOPS_PER_STATE_TC / (kms * 1e-3) / 1e12
    tck = next((r["plan"]["tc_kernel"] for r in res if r["form"] == "tc"), None)
    per_acc = TC_KERNEL_NAMES.get(tck or "", ("tc_pass1_kernel", 1))[1]
    out = {"metric": "states/s (4096-instance batch, exact FP64 argmin each)", "value": states / (ms * 1e-3),
           "unit": "states/s", "steps": steps, "warmup": max(3, warmup), "ms_per_step": ms,
           "dtype": ("f32 accumulate of f16 integer digits (values rounded to a power-of-two unit, 16-bit minima); "
                     "FP64 re-scoring") if tck == "pair_u16" else "f32 (f16 digit operands, fp32 accumulate; FP64 re-scoring)",
           "config": {"workload": BATCH_WORKLOAD, "states_per_step": states, "instances": len(Qs),
                      "launch": "one CUDA graph (uploads, six kernels, result copy)",
                      "l2": "flushed between steps (256 MiB write)"},
           "e2e": {"value": states / statistics.median(wall), "unit": "states/s",
                   "h2d_bytes_per_step": int(res[0]["h2d_bytes"]), "d2h_bytes_per_step": int(res[0]["d2h_bytes"])},
           "gpu_launches": int(res[0]["kernels"]),
           "launch_by_launch": {"ms_per_step": statistics.median(p_ms), "value": states / (statistics.median(p_ms) * 1e-3)},
           "roofline": {"bound": "tensor", "kernel": "pass-1 kernels (tensor-core items n >= 24, Gray items below)",
                        "kernel_ms": kms, "achieved": tflops, "unit": "TFLOP/s", "tc_states": tc_states,
                        "flops_per_state": FLOPS_PER_STATE_TC, "tc_kernel": tck,
                        "tensor_flops_per_state": FLOPS_PER_STATE_TC // per_acc,
                        "frac_bf16": tflops / peak, "peak_bf16": peak, "peak_bf16_kind": f"bf16 dense burst, {peak_kind}",
                        "frac_int8": tflops / (2 * peak), "peak_int8": 2 * peak,
                        "peak_int8_kind": "2 x the bf16 figure (nominal dense int8 : bf16 ratio)"}}
    if with_baselines:
        sample = Qs[::16]
        s_states = sum(1 << q.shape[0] for q in sample)
        t0 = time.perf_counter()
        for q in sample:
            h.solve(q, stream=stream)
        loop_s = time.perf_counter() - t0
        out["one_call_per_problem"] = {"value": s_states / loop_s, "unit": "states/s",
                                       "sample": f"{len(sample)} instances (every 16th), {loop_s:.2f} s"}
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        cpu = Qs[::256]
        c_states = sum(1 << q.shape[0] for q in cpu)
        t0 = time.perf_counter()
        for q in cpu:
            oracle.qbf_port(q)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": c_states / cpu_s, "unit": "states/s", "cores": 1, "kind": "port",
                               "sample": f"{len(cpu)} instances (every 256th), QBF B = 20 prefix loop, {cpu_s:.1f} s"}
    return out


def bench_batch(args):
    """The 4096-instance batch as its own line (python bench.py --case batch)."""
    import torch
    torch.cuda.set_device(0)
    b = batch_measure(args.steps, args.warmup, with_baselines=True)
    line = dict(b)
    line.update({"n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "data": "synthetic"})
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="tc", choices=["tc", "gray", "auto"] + sorted(CASE_FORMS))
    ap.add_argument("--case", default=None, choices=["cfg2", "n36", "batch"],
                    help="cfg2, n36: profiling cases (one line per solve); batch: the 4096-instance batch line")
    args = ap.parse_args()
    if args.case == "batch":
        bench_batch(args)
    elif args.case:
        bench_case(args)
    elif args.impl == "reference":
        bench_reference(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
