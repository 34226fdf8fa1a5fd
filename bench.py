#!/usr/bin/env python
"""H.v/s of DiagHam's on-the-fly FQHE product on B200, and time-to-E0 FP32+refine vs plain FP64.

Workload (the precision configuration): N = 12 spin-polarised fermions on the sphere, 2S = 33,
total Lz = 0 (dimension 7,764,392), lowest-Landau-level Coulomb pseudopotentials V_m (odd m),
synthetic start vectors from splitmix64.  One step = one H.v through the C ABI with the input
already in HBM: FP32 matrix elements and FP32 per-row accumulation, FP64 in and out (the product
the FP32+refine Lanczos runs).  L2 is flushed (a 256 MiB write) before every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs independent replicas (one process per GPU, launched by torch.distributed.run); the
value is the sum over replicas of their products per second, timed as the max over ranks.
Prints one JSON line on rank 0.
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

N_FERMIONS, TWO_S, TWO_LZ = 12, 33, 0
METRIC = "H·v/sec and time-to-E0 (1e-10) FP32+refine batched vs plain FP64, one B200"
UNIT = "H·v/s"
REF_TOOL = os.path.join(ROOT, "oracle", "_ref", "ref_tool")
FLUSH_BYTES = 256 << 20


def workload_name():
    return ("FermionOnSphere N=12 2S=33 2Lz=0 (dim 7764392), LLL Coulomb V_m odd m, on-the-fly H.v, "
            "FP32 elements + FP32 row accumulation, FP64 vectors")


def pseudopotentials(dh):
    v = dh.coulomb_pseudopotentials(TWO_S)
    v[0::2] = 0.0
    return v


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the FP32 product from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "fqhe_matvec_fp32_n12_2s33.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(self.REASONS, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl" if os.environ.get("DH_BENCH_BACKEND", "nccl") == "nccl" else "gloo",
                                 timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def reduce_max(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as tdist
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()


# ------------------------------------------------------------------ CPU baselines

def reference_cpu_matvec(rows_target_s, reps, hermitian=1):
    """The reference's own SMP product (oracle/_ref/ref_tool bench_fqhe) on all host threads, over
    a bounded sample of rows sized to take about rows_target_s seconds per repetition."""
    import tempfile
    import diagham_b200 as dh
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as tmp:
        vf = os.path.join(tmp, "v.bin")
        pseudopotentials(dh).tofile(vf)
        dim = 7764392
        # calibrate: about 45 us of one thread per row (hermitian product), measured on x86 hosts
        rows = int(min(dim, max(2000, rows_target_s * threads / 45e-6)))
        cmd = [REF_TOOL, "bench_fqhe", N_FERMIONS, TWO_S, TWO_LZ, vf, threads, reps, hermitian, rows]
        out = subprocess.run([str(c) for c in cmd], check=True, capture_output=True, text=True)
        line = [l for l in out.stdout.splitlines() if l.startswith("{")][-1]
        r = json.loads(line)
    per_matvec = r["mean_s"] * r["dim"] / r["rows"]
    return {"value": 1.0 / per_matvec, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": "first %d of %d rows per product, %d repetition(s), SMP %d threads, hermitian %s "
                      "(VectorHamiltonianMultiplyOperation on SMPArchitecture, -m 0)"
                      % (r["rows"], r["dim"], reps, threads, "on" if hermitian else "off"),
            "seconds_per_sample": r["mean_s"]}


def port_cpu_matvec(rows):
    """The oracle's C restatement (single thread) over a bounded row sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import diagham_b200 as dh
    H = oracle.FQHE(N_FERMIONS, TWO_S, TWO_LZ, pseudopotentials(dh))
    x = oracle.random_vector(0, H.dim)
    t0 = time.perf_counter()
    H.push(x, 0, rows)
    dt = time.perf_counter() - t0
    return {"value": (rows / H.dim) / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "first %d of %d rows, oracle push-form product, 1 thread" % (rows, H.dim),
            "seconds_per_sample": dt}


def cpu_baseline():
    if os.path.exists(REF_TOOL):
        try:
            return reference_cpu_matvec(rows_target_s=12.0, reps=1)
        except (subprocess.CalledProcessError, OSError, ValueError, IndexError) as e:
            sys.stderr.write("reference CPU baseline failed (%s); timing the oracle port\n" % e)
    return port_cpu_matvec(20000)


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    if not os.path.exists(REF_TOOL):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_tool was not built (make -C oracle ref)"}))
        return
    budget = 150.0
    per = max(0.05, budget / float(args.steps + args.warmup))
    cb = reference_cpu_matvec(rows_target_s=per, reps=args.steps)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * cb["seconds_per_sample"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name().replace("FP32 elements + FP32 row accumulation, FP64 vectors",
                                                           "FP64 (reference CPU path)")},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------ B200 arm

def time_to_e0(dh, H, dim, max_iter=400):
    """Plain FP64 Lanczos to |dE| < 1e-13 |E| against FP32-product Lanczos + FP64 refinement, same start."""
    import torch
    res = {}
    H.set_precision("fp64")
    lz = dh.BasicLanczosAlgorithm(H, 1, max_iter)
    lz.SetEigenvaluePrecision(1e-13)
    lz.InitializeLanczosAlgorithm(seed=0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r64 = lz.solve(max_iter, graph_batch=16)
    torch.cuda.synchronize()
    t64 = time.perf_counter() - t0
    m64, _ = lz.counters()
    del lz
    lz = dh.BasicLanczosAlgorithm(H, 1, max_iter)
    lz.InitializeLanczosAlgorithm(seed=0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r32 = lz.solve_refined(max_iter, precision=1e-13)
    torch.cuda.synchronize()
    t32 = time.perf_counter() - t0
    del lz
    e64 = float(r64["eigenvalues"][0])
    res = {"fp64": {"seconds": t64, "e0": e64, "iterations": r64["iterations"], "matvecs": m64,
                    "converged": r64["converged"]},
           "fp32_refined": {"seconds": t32, "e0": r32["energy"], "e0_fp32_phase": r32["energy_fp32"],
                            "residual": r32["residual"], "fp32_matvecs": r32["fp32_matvecs"],
                            "fp64_matvecs": r32["fp64_matvecs"]},
           "abs_e_minus_e_fp64": abs(r32["energy"] - e64),
           "rel_e_minus_e_fp64": abs(r32["energy"] - e64) / abs(e64),
           "speedup": t64 / t32 if t32 > 0 else None}
    ref = os.path.join(ROOT, "tests", "golden", "lanczos_n12_2s33_lz0_coulomb_basic.npz")
    if os.path.exists(ref):
        e_ref = float(np.load(ref)["eigenvalues"][0])
        res["reference_e0"] = e_ref
        res["rel_e_minus_reference"] = {"fp64": abs(e64 - e_ref) / abs(e_ref),
                                        "fp32_refined": abs(r32["energy"] - e_ref) / abs(e_ref)}
    return res


def run_b200(args, world, rank, local):
    import torch
    import diagham_b200 as dh
    from diagham_b200 import _build
    _build.build()
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    space = dh.FermionOnSphere(N_FERMIONS, TWO_LZ, TWO_S)
    dim = space.dim
    H = dh.ParticleOnSphereGenericHamiltonian(space, N_FERMIONS, TWO_S, pseudopotentials(dh))
    H.set_stream(stream.cuda_stream)
    moves = H.count_elements()
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.rand(dim, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    x /= torch.linalg.vector_norm(x)
    y = torch.empty_like(x)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    # FP64 product rate (for the record), then the FP32 product (the measured step)
    def timed(precision, steps, warmup):
        H.set_precision(precision)
        for _ in range(warmup):
            flush.zero_()
            H.LowLevelMultiply(x, y)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            H.LowLevelMultiply(x, y)
            ends[i].record(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        total_ms = e0.elapsed_time(e1)
        launch_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
        return total_ms, launch_ms

    if args.kernel_only:
        total_ms, launch_ms = timed("fp32", args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"kernel_only": True, "dim": dim, "elements_per_product": moves, "steps": args.steps,
                              "mean_launch_ms": statistics.mean(launch_ms), "ms_per_step": total_ms / args.steps}))
        return
    fp64_ms, fp64_launch = timed("fp64", max(5, args.steps // 10), 2)
    with ClockSampler(local) as clocks:
        total_ms, launch_ms = timed("fp32", args.steps, args.warmup)
    total_ms = reduce_max(total_ms, world)
    value = world * args.steps / (total_ms / 1000.0)

    # roofline of the FP32 product: algorithmic bytes per launch (basis word + FP64 y + FP32 x per
    # off-diagonal element and for the row itself), over the mean device time of one C-ABI call
    # (FP64->FP32 conversion of x included)
    c_n2 = N_FERMIONS * (N_FERMIONS - 1) // 2
    nnz_off = moves - c_n2 * dim
    alg_bytes = dim * 8 + dim * 8 + (nnz_off + dim) * 4
    launch_mean = statistics.mean(launch_ms) / 1000.0
    peak, peak_kind = peaks()
    achieved = alg_bytes / launch_mean / 1e9
    traffic = profile_traffic()

    # end to end through the public API with pinned host buffers (H2D of x, D2H of y every step)
    hx = torch.empty(dim, dtype=torch.float64, pin_memory=True)
    hy = torch.empty(dim, dtype=torch.float64, pin_memory=True)
    hx.copy_(x.cpu())
    hxn, hyn = hx.numpy(), hy.numpy()
    H.set_precision("fp32")
    e2e_steps = max(3, min(args.steps, 40))
    for _ in range(2):
        H.LowLevelMultiply(hxn, hyn)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        H.LowLevelMultiply(hxn, hyn)
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, world)
    e2e_value = world * e2e_steps / e2e_s

    tte = None
    if not args.no_solve:
        tte = time_to_e0(dh, H, dim)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(), "dim": dim, "elements_per_product": moves,
                       "l2": "flushed: 256 MiB write before every step",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "gpu_launches": 2 * args.steps,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": dim * 8, "d2h_bytes_per_step": dim * 8,
                    "steps": e2e_steps, "buffers": "pinned host"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel": "fqhe_matvec_kernel<float> (+ x FP64->FP32 conversion)",
                         "mean_launch_ms": launch_mean * 1000.0},
            "fp64_product": {"value": len(fp64_launch) / (fp64_ms / 1000.0), "unit": UNIT,
                             "mean_launch_ms": statistics.mean(fp64_launch)},
            "clocks": clocks.summary(),
            "time_to_e0": tte}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only the timed FP32 products (the short command used for ncu captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        else:
            run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
