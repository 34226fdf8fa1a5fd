#!/usr/bin/env python
"""H.v/s of DiagHam's on-the-fly FQHE product on B200, and time-to-E0 FP32+refine vs plain FP64.

Workload (the precision configuration): N = 12 spin-polarised fermions on the sphere, 2S = 33,
total Lz = 0 (dimension 7,764,392), lowest-Landau-level Coulomb pseudopotentials V_m (odd m),
synthetic inputs.  One step = one FP64 block product H X of 4 vectors (4 H.v, the product of
block Lanczos: LowLevelMultipleMultiply) through the C ABI with X already in HBM; X (248 MB) is
larger than L2 and a 256 MiB write also precedes every step.  The reference arm times the same
product with the reference's own SMP code (MultipleVectorHamiltonianMultiplyOperation ->
HermitianLowLevelMultipleMultiply, FP64, all host threads).  The line also carries the FP32 rates,
the time to E0 of the sector (plain FP64 against FP32 products + FP64 refinement), of all 91
sectors of N = 10, 2S = 27 (batched against sector by sector), of the L = 32 J1-J2 chain (block
k = 2, FP32 + FP64 refinement), the adjoint gradients of N = 10, 2S = 27 against the reference's
and finite differences, and secondary product legs; a compact time-to-E0 summary ends the line.

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
BLOCK = 4  # vectors per product in the measured step (the batched form)
KERNEL_FP64_BLOCK4 = "fqhe_split_kernel<double, 4, RANGE=0, LR_SMEM=0, IL=1, W256=1, FORM=autotuned>"


DIM = 7764392
REFERENCE_WINDOWS = 2  # the reference arm alternates two half-basis row windows (two steps = one product)


def workload_config():
    """The config both arms print, identical: the sector, the block and the arithmetic."""
    return {"workload": "FermionOnSphere N=12 2S=33 2Lz=0 (dim 7764392), LLL Coulomb V_m odd m, on-the-fly "
                        "FP64 product H X of blocks of 4 vectors (block Lanczos LowLevelMultipleMultiply)",
            "dim": DIM, "block": BLOCK, "hv_per_step": BLOCK, "arithmetic": "fp64",
            "l2": "X is 248 MB (> 126 MB L2); the GPU arm also writes 256 MiB before every step"}


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


HEADLINE_PROFILE = os.path.join(ROOT, "profiles", "fqhe_block4_fp64_n12_2s33.md")


def profile_field(key, number=True):
    """A field of the committed ncu summary of the measured block product (None if absent)."""
    if not os.path.exists(HEADLINE_PROFILE):
        return None
    for line in open(HEADLINE_PROFILE):
        if line.startswith(key + ":"):
            v = line.split(":", 1)[1].strip()
            return float(v.split()[0]) if number else v
    return None


def profile_traffic():
    """DRAM bytes per launch of the measured block product from the committed ncu summary, if any."""
    return profile_field("dram_bytes_per_launch")


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

def reference_cpu_block(windows, reps, skip=0):
    """The reference's own SMP block product (oracle/_ref/ref_tool bench_fqhe_block:
    MultipleVectorHamiltonianMultiplyOperation on SMPArchitecture -> HermitianLowLevelMultipleMultiply,
    FP64, on the fly, all host threads, pseudopotentials from the reference's EvaluatePseudopotentials)
    on blocks of 4 vectors.  The basis is cut into `windows` equal row windows and repetition r
    multiplies window r mod windows; the first `skip` repetitions are not counted.  Every call pays the
    reference's per-call SMP cost (per-thread destination copies of the whole block and their sum),
    so a windowed product costs slightly more than a whole one."""
    threads = os.cpu_count() or 1
    cmd = [REF_TOOL, "bench_fqhe_block", N_FERMIONS, TWO_S, TWO_LZ, "coulomb", threads, reps + skip, 1, BLOCK,
           windows]
    out = subprocess.run([str(c) for c in cmd], check=True, capture_output=True, text=True)
    r = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    counted = r["reps"][skip:]
    seconds = sum(c["s"] for c in counted)
    products = sum(c["rows"] for c in counted) / float(r["dim"])
    return {"value": BLOCK * products / seconds, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": "%d call(s), each one of %d equal row windows of the %d-row basis in turn (%.2f whole block "
                      "products), SMP %d threads, hermitian (MultipleVectorHamiltonianMultiplyOperation on "
                      "SMPArchitecture, -m 0), FP64 blocks of %d vectors"
                      % (len(counted), windows, r["dim"], products, threads, BLOCK),
            "seconds_per_sample": seconds / len(counted), "seconds_per_block_product": seconds / products,
            "reference_setup_seconds": r["setup_s"]}


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
            # one whole block product, as two half-basis calls
            return reference_cpu_block(REFERENCE_WINDOWS, REFERENCE_WINDOWS)
        except (subprocess.CalledProcessError, OSError, ValueError, IndexError, KeyError) as e:
            sys.stderr.write("reference CPU baseline failed (%s); timing the oracle port\n" % e)
    return port_cpu_matvec(20000)


def run_reference_arm(args, world, rank):
    """The reference's own CPU block product on this arm's workload and metric: each step is one
    half-basis window (two steps = one whole product), the warm-up steps are run and not counted.
    Nothing from the diagham_b200 package is loaded."""
    if rank != 0:
        return
    if not os.path.exists(REF_TOOL):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_tool was not built (make -C oracle ref)"}))
        return
    cb = reference_cpu_block(REFERENCE_WINDOWS, args.steps, skip=args.warmup)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * cb["seconds_per_sample"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(), "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------ B200 arm

def _median_run(fn, runs):
    import torch
    out = []
    for _ in range(runs):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        out.append((time.perf_counter() - t0, r))
    out.sort(key=lambda t: t[0])
    return out[len(out) // 2]


def time_to_e0_single_sector(dh, H, runs=3, max_iter=600, precisions=(1e-10, 1e-13)):
    """The N=12, 2S=33 sector: plain FP64 single-vector Lanczos (CUDA-graph batches) against the
    FP32-product forms with FP64 refinement (single vector, block k = 2, 4), same seeded start, the
    reference's convergence test at each precision (the metric's 1e-10, and 1e-13); median wall time
    of `runs` runs, each from the uploaded start to the refined E0, and the error of every result
    against the reference's E0 of the sector.  Each form runs with the autotuned kernel for its
    precision and block; the *_stored forms have the stored elements (fast multiplication, built
    once before the timed runs) available to the autotuner, which keeps them where they are faster.
    The speed-up is against the faster plain FP64 form."""
    ref = os.path.join(ROOT, "tests", "golden", "lanczos_n12_2s33_lz0_coulomb_basic.npz")
    e_ref = float(np.load(ref)["eigenvalues"][0]) if os.path.exists(ref) else None
    out = {"runs": runs, "reference_e0": e_ref}

    def plain(precision):
        lz = dh.BasicLanczosAlgorithm(H, 1, max_iter)
        lz.SetEigenvaluePrecision(precision)
        lz.InitializeLanczosAlgorithm(seed=0)
        r = lz.solve(max_iter, graph_batch=16)
        return float(r["eigenvalues"][0]), r["iterations"], lz.counters()[0]

    def refined(precision, k):
        if k == 1:
            lz = dh.BasicLanczosAlgorithm(H, 1, max_iter)
        else:
            lz = dh.BasicBlockLanczosAlgorithm(H, 1, max_iter, block_size=k)
        lz.InitializeLanczosAlgorithm(seed=0)
        return lz.solve_refined(max_iter, precision=precision)

    def tuned(precision, k):
        H.set_precision(precision)
        t = H.autotune(block_size=k, repeats=3)
        return {"kernel": "stored elements" if t["stored_in_use"] else "%s LB=%d %s" % (
            t["kernel_variant"], t["low_bits"], t["launch_form"]), "ms_per_product": t["best_ms"]}

    for precision in precisions:
        res = {}
        for stored in (False, True):
            if stored:
                H.EnableFastMultiplication()
            tag = "_stored" if stored else ""
            kern = tuned("fp64", 1)
            t64, (e64, it64, mv64) = _median_run(lambda: plain(precision), runs)
            res["plain_fp64" + tag] = {"seconds": t64, "e0": e64, "iterations": it64, "matvecs": mv64, "product": kern}
            for k in ((1,) if stored else (1, 2, 4)):
                kern = tuned("fp32", k)
                t, r = _median_run(lambda: refined(precision, k), runs)
                res["fp32_refined_k%d%s" % (k, tag)] = {
                    "seconds": t, "e0": r["energy"], "e0_fp32_phase": r["energy_fp32"],
                    "abs_e_minus_e_fp64": abs(r["energy"] - e64), "residual": r["residual"],
                    "fp32_matvecs": r["fp32_matvecs"], "fp64_matvecs": r["fp64_matvecs"], "product": kern}
            if stored:
                H.DisableFastMultiplication()
        if e_ref is not None:
            for v in res.values():
                v["rel_e_minus_reference"] = abs(v["e0"] - e_ref) / abs(e_ref)
        plain_best = min((k for k in res if k.startswith("plain")), key=lambda k: res[k]["seconds"])
        t_plain = res[plain_best]["seconds"]
        for k_, v in res.items():
            if k_.startswith("fp32"):
                v["speedup_vs_best_plain_fp64"] = t_plain / v["seconds"]
        best = min((k for k in res if k.startswith("fp32")), key=lambda k: res[k]["seconds"])
        res["best_fp32_refined"] = {"form": best, "best_plain_fp64": plain_best,
                                    "speedup_vs_best_plain_fp64": t_plain / res[best]["seconds"]}
        out["precision_%g" % precision] = res
    H.set_precision("fp32")
    return out


def splitmix_uniform(seed, n, lo, hi):
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return lo + (hi - lo) * (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def time_to_e0_all_sectors(dh, k=None, runs=3, precisions=(1e-10, 1e-13)):
    """Every Lz sector of N=10, 2S=27 (2Lz = 0..180, 91 sectors) with V1 = 1 and V3, V5, V7 uniform
    in [0, 0.5) from splitmix64 seed 1: the batched block form (FP32 products + FP64 refinement,
    and FP64) against plain FP64 single-vector Lanczos run sector after sector (sectors of
    dimension <= 200 go through the same dense path in both), at each precision; median of `runs`
    (one run at the stricter precision), errors against the plain FP64 energies at 1e-13."""
    import torch
    n, s = 10, 27
    v = np.zeros(s + 1)
    v[1] = 1.0
    v[[3, 5, 7]] = splitmix_uniform(1, 3, 0.0, 0.5)
    sectors = list(range(0, 181, 2))
    dims = [dh.FermionOnSphere(n, lz, s).dim for lz in sectors]
    dense = [lz for lz, d in zip(sectors, dims) if d <= 200]
    tuned = None
    if k is None:
        # the block size from the tuner: time to the refined ground energy of the largest sector
        sp0 = dh.FermionOnSphere(n, 0, s)
        H0 = dh.ParticleOnSphereGenericHamiltonian(sp0, n, s, v)
        k, tk = H0.tune_block_size(max_iter=800, precision=1e-10, refined=True)
        tuned = {"k": k, "seconds_2lz0_by_k": tk}
        del H0, sp0
    out = {"sectors": len(sectors), "total_rows": int(sum(dims)), "largest": int(max(dims)), "block": k,
           "block_tuned": tuned}
    dh.fqhe_sectors_block_lanczos(n, s, sectors[-12:], v, block_size=k, max_iter=400)  # warm-up

    def plain_all(precision):
        plain = dict(zip(dense, dh.fqhe_sectors_block_lanczos(n, s, dense, v, block_size=4, max_iter=800,
                                                              full_diag_limit=200)["energies"]))
        for lz, d in zip(sectors, dims):
            if d <= 200:
                continue
            space = dh.FermionOnSphere(n, lz, s)
            H = dh.ParticleOnSphereGenericHamiltonian(space, n, s, v)
            lzz = dh.BasicLanczosAlgorithm(H, 1, 800)
            lzz.SetEigenvaluePrecision(precision)
            lzz.InitializeLanczosAlgorithm(seed=100)
            plain[lz] = float(lzz.solve(800, graph_batch=16)["eigenvalues"][0])
            del lzz, H, space
        return np.array([plain[lz] for lz in sectors])

    e_strict = None
    for precision in sorted(precisions, reverse=True):
        nr = runs if precision == max(precisions) else 1
        res = {}
        tp, e_plain = _median_run(lambda: plain_all(precision), nr)
        res["plain_fp64_per_sector"] = {"seconds": tp, "energies": e_plain}
        # the batched forms on the fly and with the batch's stored elements (memory = -1: built inside
        # the timed call, one ELL over the concatenated sectors)
        for memory in (0, -1):
            for fp32 in (True, False):
                t, r = _median_run(lambda: dh.fqhe_sectors_block_lanczos(n, s, sectors, v, block_size=k, max_iter=800,
                                                                        precision=precision, fp32=fp32,
                                                                        full_diag_limit=200, memory=memory), nr)
                res["batched_%s%s" % ("fp32_refined" if fp32 else "fp64", "_stored" if memory else "")] = {
                    "seconds": t, "energies": r["energies"], "block_products": r["block_products"],
                    "setup_seconds": r["setup_seconds"], "solve_seconds": r["solve_seconds"],
                    "product_seconds": r["product_seconds"], "fp32_seconds": r["fp32_seconds"],
                    "refine_seconds": r["refine_seconds"], "refined_sectors": r["refined_sectors"],
                    "dense_fallback_sectors": r["dense_fallback_sectors"],
                    "dense_fallback_seconds": r["dense_fallback_seconds"],
                    "stored_bytes": r["stored_bytes"], "store_seconds": r["store_seconds"],
                    "speedup_vs_plain_fp64": tp / t}
        out["precision_%g" % precision] = res
        if precision == min(precisions):
            e_strict = e_plain
    # the reference's lowest energy of every sector (its block Lanczos, k = 4, or full diagonalisation
    # below 300 states; tests/golden/sectors_n10_2s27_block4.npz), when the fixture is present
    ref_path = os.path.join(ROOT, "tests", "golden", "sectors_n10_2s27_block4.npz")
    e_ref = None
    if os.path.exists(ref_path):
        z = np.load(ref_path)
        ref_of = dict(zip((int(t) for t in z["two_lz"]), (float(e) for e in z["e0"])))
        e_ref = np.array([ref_of[lz] for lz in sectors])
    for key in [k_ for k_ in out if k_.startswith("precision_")]:
        for v_ in out[key].values():
            e = np.asarray(v_.pop("energies"))
            v_["max_rel_e_minus_plain_fp64_strict"] = float(np.max(np.abs(e - e_strict) / np.abs(e_strict)))
            if e_ref is not None:
                v_["max_rel_e_minus_reference"] = float(np.max(np.abs(e - e_ref) / np.abs(e_ref)))
    out["ground_state"] = {"two_lz": int(sectors[int(np.argmin(e_strict))]), "e0": float(np.min(e_strict))}
    return out


def spin_chain_product(dh, flush, steps=5, k=2, length=32, warmup=2):
    """The periodic J1-J2 chain, L = 32, Sz = 0 (dimension 601,080,390): FP32 block products of k
    vectors (the config whose x and basis do not fit in L2), with their algorithmic bytes."""
    import torch
    t0 = time.perf_counter()
    chain = dh.Spin1_2Chain(length, 0)
    H = dh.SpinChainJ1J2Hamiltonian(chain, 1.0, 0.5)
    H.set_precision("fp32")
    dim = chain.dim
    setup = time.perf_counter() - t0
    x = torch.empty(dim, k, dtype=torch.float64, device="cuda")
    x.uniform_(-1.0, 1.0)
    y = torch.empty_like(x)
    for _ in range(warmup):
        flush.zero_()
        H.block_multiply(x, y)
    ms = []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        H.block_multiply(x, y)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    flips = H.count_elements()
    alg = dim * 4 + k * dim * 8 + k * (flips + dim) * 4
    mean_s = statistics.mean(ms) / 1000.0
    peak, kind = peaks()
    del x, y, H, chain
    torch.cuda.empty_cache()
    return {"workload": "Spin1_2Chain L=%d Sz=0 periodic J1=1 J2=0.5 (dim %d), FP32 block k=%d" % (length, dim, k),
            "setup_seconds": setup, "mean_launch_ms": mean_s * 1000.0, "hv_per_s": k / mean_s,
            "off_diagonal_flips": flips, "algorithmic_bytes_per_launch": alg,
            "roofline": {"bound": "hbm", "achieved": alg / mean_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / mean_s / 1e9 / peak, "peak_kind": kind,
                         # ncu, one launch at L = 30 (x ten times L2): DRAM bytes against the model
                         "measured_dram": {"profile": "profiles/spin_j1j2_fp32_block2_L30_dram.md",
                                           "dram_over_algorithmic": 0.474, "dram_gbs": 2355.0,
                                           "frac_of_hbm": 0.36,
                                           "limiter": "gather and rank-table latency, not DRAM bandwidth"}}}



def spin_chain_solve(dh, length=32, k=2, precision=1e-10, max_iter=400):
    """The large-spin-chain configuration end to end: periodic J1-J2 chain, L = 32, J2 = J1/2, Sz = 0
    (dimension 601,080,390), block Lanczos with k = 2, FP32 products with FP64 vectors and FP64
    refinement, stopping at the stated precision; the exact E0 = -3L/8 is the check."""
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    chain = dh.Spin1_2Chain(length, 0)
    H = dh.SpinChainJ1J2Hamiltonian(chain, 1.0, 0.5)
    H.set_precision("fp32")
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    lz = dh.BasicBlockLanczosAlgorithm(H, 1, max_iter, block_size=k)
    lz.InitializeLanczosAlgorithm(seed=0)
    r = lz.solve_refined(max_iter, precision=precision)
    torch.cuda.synchronize()
    solve = time.perf_counter() - t0
    exact = -0.375 * length
    out = {"workload": "Spin1_2Chain L=%d Sz=0 periodic J1=1 J2=0.5 (dim %d), block k=%d, FP32 products + FP64 "
                       "refinement" % (length, chain.dim, k),
           "setup_seconds": setup, "seconds": solve, "e0": r["energy"], "e0_fp32_phase": r["energy_fp32"],
           "rel_e0_minus_exact": abs(r["energy"] - exact) / abs(exact), "residual": r["residual"],
           "fp32_block_products": r["fp32_matvecs"], "fp64_products": r["fp64_matvecs"], "precision": precision}
    del lz, H, chain
    torch.cuda.empty_cache()
    return out


def time_to_e0_summary(line):
    """A compact digest of the time-to-E0 legs (seconds, speed-ups, errors) for the end of the line."""
    out = {}
    tte = line.get("time_to_e0")
    if tte:
        p = tte.get("precision_1e-10", {})
        if p:
            best = p["best_fp32_refined"]["form"]
            pb = p["best_fp32_refined"]["best_plain_fp64"]
            out["n12_2s33"] = {"plain_fp64_s": round(p[pb]["seconds"], 4), "plain_form": pb,
                               "fp32_refined_s": round(p[best]["seconds"], 4), "form": best,
                               "speedup": round(p[pb]["seconds"] / p[best]["seconds"], 3),
                               "rel_err_plain": p[pb].get("rel_e_minus_reference"),
                               "rel_err_refined": p[best].get("rel_e_minus_reference")}
    tc = line.get("time_to_e0_all_sectors")
    if tc:
        p = tc.get("precision_1e-10", {})
        if p:
            pl = p["plain_fp64_per_sector"]
            refined = min((k_ for k_ in p if k_.startswith("batched_fp32_refined")), key=lambda k_: p[k_]["seconds"])
            fp64 = min((k_ for k_ in p if k_.startswith("batched_fp64")), key=lambda k_: p[k_]["seconds"])
            out["n10_2s27_91_sectors"] = {
                "block_k": tc.get("block"),
                "plain_fp64_s": round(pl["seconds"], 4),
                "batched_fp32_refined_s": round(p[refined]["seconds"], 4), "refined_form": refined,
                "batched_fp64_s": round(p[fp64]["seconds"], 4), "fp64_form": fp64,
                "speedup": round(p[refined]["speedup_vs_plain_fp64"], 3),
                "max_rel_err_refined": p[refined].get("max_rel_e_minus_plain_fp64_strict"),
                "max_rel_err_vs_reference": p[refined].get("max_rel_e_minus_reference")}
    cs = line.get("spin_chain_l32_solve")
    if cs:
        out["chain_l32"] = {"s": round(cs["seconds"], 3), "e0": cs["e0"], "rel_err": cs["rel_e0_minus_exact"]}
    cb = line.get("cpu_baseline")
    if cb:
        out["headline_fp64_block4"] = {"b200_hv_s": round(line["value"], 2), "reference_cpu_hv_s": round(cb["value"], 4),
                                       "e2e_hv_s": round(line["e2e"]["value"], 2)}
    return out


def long_product(dh, flush, steps=5, warmup=2):
    """FermionOnSphereLong N=6, 2S=63, 2Lz=0 (dimension 671,430: the first 2S above 64-bit words), LLL
    Coulomb V_m with the even m set to zero: FP64 single products and FP32 blocks of 4, with the
    algorithmic bytes (16-byte word and FP64 y per row, one x gather per element), and the same
    products from stored elements."""
    import torch
    n, s = 6, 63
    v = dh.coulomb_pseudopotentials(s)
    v[0::2] = 0.0
    t0 = time.perf_counter()
    sp = dh.FermionOnSphereLong(n, 0, s)
    H = dh.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    dim = sp.dim
    moves = H.count_elements()
    peak, kind = peaks()
    out = {"workload": "FermionOnSphereLong N=%d 2S=%d 2Lz=0 (dim %d), Coulomb V_m odd m" % (n, s, dim),
           "setup_seconds": setup, "elements_per_product": moves}
    def timed(k):
        x = torch.empty(dim, k, dtype=torch.float64, device="cuda")
        x.uniform_(-1.0, 1.0)
        y = torch.empty_like(x)
        for _ in range(warmup):
            flush.zero_()
            H.block_multiply(x, y)
        ms = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            H.block_multiply(x, y)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.mean(ms) / 1000.0

    for prec, k in (("fp64", 1), ("fp32", 4)):
        H.set_precision(prec)
        mean_s = timed(k)
        xb = 4 if prec == "fp32" else 8
        alg = dim * (16 + 8 * k) + moves * xb * k
        out["%s_block_k%d" % (prec, k)] = {
            "mean_launch_ms": mean_s * 1000.0, "hv_per_s": k / mean_s, "elements_per_s": moves * k / mean_s,
            "algorithmic_bytes_per_launch": alg,
            "roofline": {"bound": "hbm", "achieved": alg / mean_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / mean_s / 1e9 / peak, "peak_kind": kind}}
    # stored elements (8 bytes each: target, factor index | sign), streamed once per product
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    on, nbytes = H.EnableFastMultiplication()
    torch.cuda.synchronize()
    stored = {"built": on, "bytes": nbytes, "build_seconds": time.perf_counter() - t0}
    if on:
        for prec, k in (("fp64", 1), ("fp32", 4)):
            H.set_precision(prec)
            t = H.autotune(block_size=k, repeats=3)  # read-ahead depth; keeps the faster form
            st = timed(k)
            stored["%s_block_k%d" % (prec, k)] = {
                "mean_launch_ms": st * 1000.0, "hv_per_s": k / st, "stream_gbs": nbytes / st / 1e9,
                "stored_in_use": t["stored_in_use"], "read_ahead": t["stored_read_ahead"],
                "speedup_vs_on_the_fly": out["%s_block_k%d" % (prec, k)]["mean_launch_ms"] / (st * 1000.0)}
    out["stored"] = stored
    del H, sp
    torch.cuda.empty_cache()
    return out


def reference_cpu_long(rows_target_s=6.0):
    """The reference's own SMP product on the sector of long_product (oracle/_ref/ref_tool bench_lfqhe:
    FermionOnSphereLong + ParticleOnSphereGenericHamiltonian, all host threads) over a row sample."""
    import tempfile
    import diagham_b200 as dh
    if not os.path.exists(REF_TOOL):
        return None
    threads = os.cpu_count() or 1
    v = dh.coulomb_pseudopotentials(63)
    v[0::2] = 0.0
    with tempfile.TemporaryDirectory() as tmp:
        vf = os.path.join(tmp, "v.bin")
        v.tofile(vf)
        # about 50 us of one thread per row (measured on x86 hosts)
        rows = int(min(671430, max(2000, rows_target_s * threads / 50e-6)))
        cmd = [REF_TOOL, "bench_lfqhe", 6, 63, 0, vf, threads, 1, 0, rows]
        out = subprocess.run([str(c) for c in cmd], check=True, capture_output=True, text=True)
        r = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    per_matvec = r["mean_s"] * r["dim"] / r["rows"]
    return {"value": 1.0 / per_matvec, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": "first %d of %d rows per product, SMP %d threads" % (r["rows"], r["dim"], threads),
            "seconds_per_sample": r["mean_s"]}


def momentum_sector(dh, flush, steps=5, k=2, length=32, warmup=2, solve=True):
    """Spin1_2ChainWithTranslations L = 32, Sz = 0, K = 0 with the J1-J2 Hamiltonian at J2 = J1/2
    (dimension 18,784,170): set-up time, FP32 block products of k vectors and FP64 single products
    with their algorithmic bytes (per row: word, orbit size, FP64 y and diagonal x; per element one x
    gather: the flipped words are canonicalised in registers and found among the representatives,
    search probes not counted), and the FP64 Lanczos time to E0 (-3L/8 at this point)."""
    import torch
    t0 = time.perf_counter()
    sp = dh.Spin1_2ChainWithTranslations(length, 0, 0)
    H = dh.SpinChainJ1J2RealHamiltonianWithTranslations(sp, length, 1.0, 0.5)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    dim = sp.dim
    flips = H.count_elements()
    peak, kind = peaks()
    out = {"workload": "Spin1_2ChainWithTranslations L=%d Sz=0 K=0, J1=1 J2=0.5 (dim %d)" % (length, dim),
           "setup_seconds": setup, "off_diagonal_elements": flips}
    for prec, kk in (("fp32", k), ("fp64", 1)):
        H.set_precision(prec)
        x = torch.empty(dim, kk, dtype=torch.float64, device="cuda")
        x.uniform_(-1.0, 1.0)
        y = torch.empty_like(x)
        for _ in range(warmup):
            flush.zero_()
            H.block_multiply(x, y)
        ms = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            H.block_multiply(x, y)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        xb = 4 if prec == "fp32" else 8
        alg = dim * (5 + 16 * kk) + flips * xb * kk
        mean_s = statistics.mean(ms) / 1000.0
        out["%s_block_k%d" % (prec, kk)] = {
            "mean_launch_ms": mean_s * 1000.0, "hv_per_s": kk / mean_s, "algorithmic_bytes_per_launch": alg,
            "roofline": {"bound": "hbm", "achieved": alg / mean_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / mean_s / 1e9 / peak, "peak_kind": kind,
                         "limiter": "issue: the integer work of the canonical forms of the flipped words (ncu "
                                    "at L = 28: issue 69 %, ALU 56 %, DRAM 1.5 %)"}}
        del x, y
    H.set_precision("fp64")
    if not solve:
        del H, sp
        torch.cuda.empty_cache()
        return out
    t0 = time.perf_counter()
    # the stopping test bounds the change of the Ritz value, not its error: 1e-12 leaves a margin
    # under the 1e-10 relative target
    lz = dh.BasicLanczosAlgorithm(H, 1, 600)
    lz.SetEigenvaluePrecision(1e-12)
    lz.InitializeLanczosAlgorithm(seed=0)
    r = lz.solve(600, graph_batch=16)
    out["time_to_e0"] = {"seconds": time.perf_counter() - t0, "e0": float(r["eigenvalues"][0]),
                         "iterations": r["iterations"], "abs_e0_plus_3L_over_8": abs(r["eigenvalues"][0] + 0.375 * length),
                         "rel_e0_minus_exact": abs(r["eigenvalues"][0] + 0.375 * length) / (0.375 * length),
                         "stopping_precision": 1e-12}
    del lz, H, sp
    torch.cuda.empty_cache()
    out["complex_k1"] = complex_momentum_sector(dh, flush, length, 1, steps, warmup)
    return out


def complex_momentum_sector(dh, flush, length, momentum, steps, warmup):
    """The complex Hamiltonian (SpinChainJ1J2HamiltonianWithTranslations) of one momentum sector at
    J2 = J1/2, FP64 products on (Re, Im) vectors, and the FP64 Lanczos time to its E0."""
    import torch
    t0 = time.perf_counter()
    sp = dh.Spin1_2ChainWithTranslations(length, momentum, 0)
    H = dh.SpinChainJ1J2HamiltonianWithTranslations(sp, length, 1.0, 0.5)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    flips = H.count_elements()
    x = torch.empty(2 * sp.dim, dtype=torch.float64, device="cuda")
    x.uniform_(-1.0, 1.0)
    y = torch.empty_like(x)
    for _ in range(warmup):
        flush.zero_()
        H.LowLevelMultiply(x, y)
    ms = []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        H.LowLevelMultiply(x, y)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    del x, y
    mean_s = statistics.mean(ms) / 1000.0
    t0 = time.perf_counter()
    lz = dh.BasicLanczosAlgorithm(H, 1, 600)
    lz.SetEigenvaluePrecision(1e-10)
    lz.InitializeLanczosAlgorithm(seed=0)
    r = lz.solve(600, graph_batch=16)
    out = {"workload": "K=%d (dim %d), complex vectors" % (momentum, sp.dim), "setup_seconds": setup,
           "off_diagonal_elements": flips, "fp64_mean_launch_ms": mean_s * 1000.0, "hv_per_s": 1.0 / mean_s,
           "time_to_e0": {"seconds": time.perf_counter() - t0, "e0": float(r["eigenvalues"][0]),
                          "iterations": r["iterations"], "precision": 1e-10}}
    del lz, H, sp
    torch.cuda.empty_cache()
    return out


def reference_cpu_momentum_sector(length=32, rows_target_s=6.0):
    """The reference's own SMP product on the momentum sector of momentum_sector (oracle/_ref/ref_tool
    bench_spint: Spin1_2ChainWithTranslations + SpinChainJ1J2RealHamiltonianWithTranslations, all host
    threads) over a row sample; its basis set-up is reported beside it."""
    if not os.path.exists(REF_TOOL):
        return None
    threads = os.cpu_count() or 1
    # about 6 us of one thread per row (measured on x86 hosts)
    rows = int(max(2000, rows_target_s * threads / 6e-6))
    cmd = [REF_TOOL, "bench_spint", length, 0, 0, 1.0, 0.5, threads, 1, rows]
    out = subprocess.run([str(c) for c in cmd], check=True, capture_output=True, text=True)
    r = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    per_matvec = r["mean_s"] * r["dim"] / r["rows"]
    return {"value": 1.0 / per_matvec, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": "first %d of %d rows per product, SMP %d threads" % (r["rows"], r["dim"], threads),
            "seconds_per_sample": r["mean_s"], "reference_setup_seconds": r["setup_s"]}


def boson_product(dh, flush, steps=5, k=4, warmup=2, n=12, s=22):
    """BosonOnSphereShort N=12, 2S=22, 2Lz=0 by default (dimension 7,764,392, the size of the fermion
    sector above), LLL Coulomb V_m with the odd m set to zero: FP32 block products of k vectors, their
    algorithmic bytes (basis word, FP64 y, one FP32 x gather per off-diagonal element and per row),
    the same products from stored elements, and, on rank 0 of the default run, the reference's own CPU
    product of the same sector on a row sample."""
    import torch
    v = dh.coulomb_pseudopotentials(s)
    v[1::2] = 0.0
    t0 = time.perf_counter()
    sp = dh.BosonOnSphereShort(n, 0, s)
    H = dh.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    H.set_precision("fp32")
    dim = sp.dim
    setup = time.perf_counter() - t0
    x = torch.empty(dim, k, dtype=torch.float64, device="cuda")
    x.uniform_(-1.0, 1.0)
    y = torch.empty_like(x)
    for _ in range(warmup):
        flush.zero_()
        H.block_multiply(x, y)
    ms = []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        H.block_multiply(x, y)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    moves = H.count_elements()
    off = moves - H.count_diagonal_elements()
    alg = dim * 8 + k * dim * 8 + k * (off + dim) * 4
    mean_s = statistics.mean(ms) / 1000.0
    peak, kind = peaks()
    res = {"workload": "BosonOnSphereShort N=%d 2S=%d 2Lz=0 (dim %d), Coulomb V_m even m, FP32 block k=%d"
                       % (n, s, dim, k),
           "setup_seconds": setup, "mean_launch_ms": mean_s * 1000.0, "hv_per_s": k / mean_s,
           "elements_per_product": moves, "off_diagonal_elements": off, "algorithmic_bytes_per_launch": alg,
           "roofline": {"bound": "hbm", "achieved": alg / mean_s / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / mean_s / 1e9 / peak, "peak_kind": kind}}
    # stored elements (8 bytes each: target, factor index, the two occupation products), streamed once
    # per product; the autotuner then keeps whichever form is faster
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    on, nbytes = H.EnableFastMultiplication()
    torch.cuda.synchronize()
    stored = {"built": on, "bytes": nbytes, "build_seconds": time.perf_counter() - t0}
    if on:
        H.block_multiply(x, y)
        sms = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            H.block_multiply(x, y)
            b.record()
            torch.cuda.synchronize()
            sms.append(a.elapsed_time(b))
        st = statistics.median(sms) / 1000.0
        # bytes that must come from HBM: the structure, y and the FP32 block x once (124 MB, which
        # stays in L2, so the per-element gathers are L2 traffic and set the pace at k = 4)
        dram_st = nbytes + k * dim * 8 + k * dim * 4
        stored.update(mean_launch_ms=st * 1000.0, hv_per_s=k / st, speedup_vs_on_the_fly=mean_s / st,
                      stream_gbs=nbytes / st / 1e9, l2_gathers_per_s=(off + dim) / st,
                      roofline={"bound": "hbm", "achieved": dram_st / st / 1e9, "peak": peak, "unit": "GB/s",
                                "frac": dram_st / st / 1e9 / peak, "peak_kind": kind,
                                "bytes": "structure + y + x once; gathers of x served by L2"})
        t = H.autotune(block_size=k, repeats=3)
        stored["autotuned"] = {"stored_in_use": t["stored_in_use"], "best_ms": t["best_ms"],
                               "read_ahead": t["stored_read_ahead"]}
    res["stored"] = stored
    del x, y, H, sp
    torch.cuda.empty_cache()
    return res


def reference_cpu_bosons(rows_target_s=6.0):
    """The reference's own SMP product on the boson sector of boson_product (oracle/_ref/ref_tool
    bench_bqhe: BosonOnSphereShort + ParticleOnSphereGenericHamiltonian, all host threads; its
    hermitian mode is not implemented for bosons) over a row sample."""
    import tempfile
    import diagham_b200 as dh
    if not os.path.exists(REF_TOOL):
        return None
    threads = os.cpu_count() or 1
    v = dh.coulomb_pseudopotentials(22)
    v[1::2] = 0.0
    with tempfile.TemporaryDirectory() as tmp:
        vf = os.path.join(tmp, "v.bin")
        v.tofile(vf)
        # about 170 us of one thread per row (measured on x86 hosts)
        rows = int(min(7764392, max(2000, rows_target_s * threads / 170e-6)))
        cmd = [REF_TOOL, "bench_bqhe", 12, 22, 0, vf, threads, 1, 0, rows]
        out = subprocess.run([str(c) for c in cmd], check=True, capture_output=True, text=True)
        r = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    per_matvec = r["mean_s"] * r["dim"] / r["rows"]
    return {"value": 1.0 / per_matvec, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": "first %d of %d rows per product, SMP %d threads" % (r["rows"], r["dim"], threads),
            "seconds_per_sample": r["mean_s"]}


def stored_elements(dh, H, flush, dim):
    """The stored-element (fast multiplication) form of the sector's product: build time and size,
    device time per product next to the on-the-fly form, and the autotuner's choice between them."""
    import torch
    res = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    on, nbytes = H.EnableFastMultiplication()
    torch.cuda.synchronize()
    res.update(built=on, bytes=nbytes, build_seconds=time.perf_counter() - t0)
    if not on:
        return res
    stream_bytes = nbytes
    for prec, k in (("fp64", 1), ("fp32", 1), ("fp32", BLOCK), ("fp64", BLOCK)):
        H.set_precision(prec)
        x = torch.rand(dim, k, dtype=torch.float64, device="cuda") - 0.5
        y = torch.empty_like(x)
        H.block_multiply(x, y)
        ms = []
        for _ in range(5):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            H.block_multiply(x, y)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        res["%s_k%d_ms" % (prec, k)] = statistics.median(ms)
        # the stored structure streamed once per product (element targets and indices, the per-row
        # slice data and diagonal), against the measured HBM bandwidth
        res["%s_k%d_stream_gbs" % (prec, k)] = stream_bytes / (statistics.median(ms) / 1000.0) / 1e9
    H.set_precision("fp32")
    t = H.autotune(block_size=BLOCK, repeats=3)
    res["autotuned_k%d" % BLOCK] = {"stored_ms": t["stored_ms"], "best_ms": t["best_ms"],
                                   "stored_in_use": t["stored_in_use"], "read_ahead": t["stored_read_ahead"]}
    # both read-ahead depths of the FP32 single product, for the record
    H.set_precision("fp32")
    t1 = H.autotune(block_size=1, repeats=5)
    res["autotuned_k1"] = {"stored_ms": t1["stored_ms"], "read_ahead": t1["stored_read_ahead"],
                           "stream_gbs": stream_bytes / (t1["stored_ms"] / 1000.0) / 1e9}
    H.DisableFastMultiplication()
    return res


def gradients_two_sectors(dh, h=1e-6):
    """dE0/dV_m and d(neutral gap)/dV_m, odd m = 1..27, for N=10, 2S=27, Lz = 0 and 1 (Coulomb V_m
    plus uniform [-0.05, 0.05) noise from splitmix64 seed 2) by the adjoint kernel (Hellmann-Feynman
    on the GPU ground states), against the reference's FP64 gradient (committed fixture) and
    central finite differences of the GPU E0 with step h."""
    import torch
    from diagham_b200.autograd import ground_state_energy, neutral_gap
    fx = [np.load(os.path.join(ROOT, "tests", "golden", "gradient_n10_2s27_lz%d.npz" % lz)) for lz in (0, 2)]
    v = fx[0]["v"]
    odd = np.arange(1, 28, 2)
    hs = []
    for lz in (0, 2):
        sp = dh.FermionOnSphere(10, lz, 27)
        hs.append((sp, dh.ParticleOnSphereGenericHamiltonian(sp, 10, 27, v)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    V = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    gap = neutral_gap(V, hs[0][1], hs[1][1])
    gap.backward()
    torch.cuda.synchronize()
    t_gap = time.perf_counter() - t0
    g_gap = V.grad.numpy()[odd].copy()
    res = {"workload": "FermionOnSphere N=10 2S=27 2Lz=0,2 (dims %d, %d), Coulomb + U[-0.05,0.05) seed 2"
                       % (hs[0][0].dim, hs[1][0].dim),
           "gap_and_gradient_seconds": t_gap, "gap": float(gap.detach()),
           "gap_reference": float(fx[1]["eigenvalues"][0] - fx[0]["eigenvalues"][0]),
           "max_abs_dgap_minus_reference": float(np.max(np.abs(
               g_gap - (fx[1]["expectation"][odd] - fx[0]["expectation"][odd]))))}
    worst_ref = worst_fd = 0.0
    for (sp, H), z in zip(hs, fx):
        V = torch.tensor(v, dtype=torch.float64, requires_grad=True)
        ground_state_energy(V, H).backward()
        g = V.grad.numpy()[odd]
        worst_ref = max(worst_ref, float(np.max(np.abs(g - z["expectation"][odd]))))
        for i, m in enumerate(odd):
            vp, vm = v.copy(), v.copy()
            vp[m] += h
            vm[m] -= h
            fd = (float(ground_state_energy(torch.tensor(vp), H)) - float(ground_state_energy(torch.tensor(vm), H))) / (2 * h)
            worst_fd = max(worst_fd, abs(fd - g[i]))
    res["max_abs_de0_minus_reference"] = worst_ref
    res["max_abs_de0_minus_central_difference"] = worst_fd
    res["finite_difference_step"] = h
    return res


def run_b200(args, world, rank, local):
    import torch
    import diagham_b200 as dh
    from diagham_b200 import _build
    _build.build()
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    if args.leg:
        flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
        if args.leg == "long":
            r = long_product(dh, flush, steps=args.steps, warmup=args.warmup)
        elif args.leg == "sectors":
            r = time_to_e0_all_sectors(dh, runs=args.steps, precisions=(1e-10,))
        elif args.leg == "stored":
            nf, ts = args.nbr_fermions, args.two_s
            v_ = dh.coulomb_pseudopotentials(ts)
            v_[0::2] = 0.0
            sp_ = dh.FermionOnSphere(nf, 0 if (nf * ts) % 2 == 0 else 1, ts)
            H_ = dh.ParticleOnSphereGenericHamiltonian(sp_, nf, ts, v_)
            H_.set_stream(stream.cuda_stream)
            H_.set_precision("fp32")
            r = stored_elements(dh, H_, flush, sp_.dim)
        elif args.leg == "single":
            v_ = dh.coulomb_pseudopotentials(TWO_S)
            v_[0::2] = 0.0
            sp_ = dh.FermionOnSphere(N_FERMIONS, TWO_LZ, TWO_S)
            H_ = dh.ParticleOnSphereGenericHamiltonian(sp_, N_FERMIONS, TWO_S, v_)
            H_.set_stream(stream.cuda_stream)
            r = time_to_e0_single_sector(dh, H_, runs=args.steps, precisions=(1e-10,))
        elif args.leg == "momentum":
            r = momentum_sector(dh, flush, steps=args.steps, length=args.chain_length or 32, warmup=args.warmup,
                                solve=not args.no_solve)
        else:
            r = boson_product(dh, flush, steps=args.steps, warmup=args.warmup, n=args.nbr_bosons,
                              s=args.boson_two_s)
        if rank == 0:
            print(json.dumps(dict(leg=args.leg, **r)))
        return
    if args.kernel_only and args.chain_length:
        flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
        r = spin_chain_product(dh, flush, steps=args.steps, length=args.chain_length, warmup=args.warmup)
        if rank == 0:
            print(json.dumps(dict(kernel_only=True, **r)))
        return
    space = dh.FermionOnSphere(N_FERMIONS, TWO_LZ, TWO_S)
    dim = space.dim
    assert dim == DIM
    H = dh.ParticleOnSphereGenericHamiltonian(space, N_FERMIONS, TWO_S, pseudopotentials(dh))
    H.set_stream(stream.cuda_stream)
    moves = H.count_elements()
    # the project autotuner picks the kernel form and rank-table split for this sector and block
    # (--no-autotune: the defaults, or DH_FQHE_KERNEL / DH_FQHE_LOW_BITS, as for a short ncu capture)
    H.set_precision("fp64")
    tuning = None if args.no_autotune else H.autotune(block_size=BLOCK, repeats=3)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    xb = torch.rand(dim, BLOCK, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    yb = torch.empty_like(xb)
    x1 = xb[:, 0].contiguous()
    y1 = torch.empty_like(x1)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def timed(precision, k, steps, warmup):
        H.set_precision(precision)
        x, y = (x1, y1) if k == 1 else (xb, yb)
        for _ in range(warmup):
            flush.zero_()
            H.block_multiply(x, y)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            H.block_multiply(x, y)
            ends[i].record(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return e0.elapsed_time(e1), [s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)]

    if args.kernel_only:
        prec = args.precision
        if prec != "fp64" and not args.no_autotune:
            H.set_precision(prec)
            H.autotune(block_size=BLOCK, repeats=3)
        total_ms, launch_ms = timed(prec, BLOCK, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"kernel_only": True, "dim": dim, "block": BLOCK, "precision": prec,
                              "elements_per_product": moves, "steps": args.steps,
                              "mean_launch_ms": statistics.mean(launch_ms), "ms_per_step": total_ms / args.steps}))
        return
    # the headline: FP64 blocks of 4 (the block Lanczos product in the reference's arithmetic)
    with ClockSampler(local) as clocks:
        total_ms, launch_ms = timed("fp64", BLOCK, args.steps, args.warmup)
    total_ms = reduce_max(total_ms, world)
    value = world * BLOCK * args.steps / (total_ms / 1000.0)

    # roofline of the block product: algorithmic bytes per launch (basis word and k FP64 outputs per
    # row, k FP64 inputs per off-diagonal element and for the row itself) over the mean device time
    # of one C-ABI call
    c_n2 = N_FERMIONS * (N_FERMIONS - 1) // 2
    nnz_off = moves - c_n2 * dim

    def alg_bytes(xbytes, k):
        return dim * 8 + k * dim * 8 + k * (nnz_off + dim) * xbytes

    launch_mean = statistics.mean(launch_ms) / 1000.0
    peak, peak_kind = peaks()
    achieved = alg_bytes(8, BLOCK) / launch_mean / 1e9
    traffic = profile_traffic()

    # end to end through the public API with pinned host buffers (H2D of X, D2H of Y every step)
    hx = torch.empty(dim, BLOCK, dtype=torch.float64, pin_memory=True)
    hy = torch.empty(dim, BLOCK, dtype=torch.float64, pin_memory=True)
    hx.copy_(xb.cpu())
    hxn, hyn = hx.numpy(), hy.numpy()
    H.set_precision("fp64")
    e2e_steps = max(3, min(args.steps, 40))
    for _ in range(2):
        H.block_multiply(hxn, hyn)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        H.block_multiply(hxn, hyn)
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, world)
    e2e_value = world * BLOCK * e2e_steps / e2e_s

    # the other arithmetic / widths of the same product, for the record
    other = {}
    for prec, k in (("fp64", 1), ("fp32", 1), ("fp32", BLOCK)):
        if prec == "fp32" and "fp32_tuning" not in other:
            H.set_precision("fp32")
            t = H.autotune(block_size=BLOCK, repeats=3)
            other["fp32_tuning"] = {k_: t[k_] for k_ in ("kernel_variant", "low_bits")}
        t_ms, l_ms = timed(prec, k, max(5, args.steps // 4), 3)
        lm = statistics.mean(l_ms) / 1000.0
        ab = alg_bytes(8 if prec == "fp64" else 4, k)
        other["%s_block%d" % (prec, k)] = {"hv_per_s": k * len(l_ms) / (t_ms / 1000.0), "mean_launch_ms": lm * 1000.0,
                                          "algorithmic_bytes_per_launch": ab,
                                          "roofline_frac": ab / lm / 1e9 / peak}

    tte = tte_c = spin = grads = stored = bosons = momentum = longs = chain_solve = None
    if not args.no_solve:
        H.set_precision("fp32")
        stored = stored_elements(dh, H, flush, dim)
        H.autotune(block_size=BLOCK, repeats=3)
        # medians of 5 runs: the host part of these solves varies on a shared machine
        tte = time_to_e0_single_sector(dh, H, runs=5)
        tte_c = time_to_e0_all_sectors(dh, runs=5)
        grads = gradients_two_sectors(dh)
        del xb, yb, hx, hy, x1, y1
        del H, space
        torch.cuda.empty_cache()
        spin = spin_chain_product(dh, flush)
        chain_solve = spin_chain_solve(dh)
        bosons = boson_product(dh, flush)
        momentum = momentum_sector(dh, flush)
        longs = long_product(dh, flush)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(),
            "gpu_launches": args.steps,
            "autotuned": {k: tuning[k] for k in ("kernel_variant", "low_bits", "candidates")} if tuning else None,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": dim * BLOCK * 8,
                    "d2h_bytes_per_step": dim * BLOCK * 8, "steps": e2e_steps, "buffers": "pinned host"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes(8, BLOCK),
                         "kernel": KERNEL_FP64_BLOCK4, "limiter": profile_field("limiter", number=False),
                         "mean_launch_ms": launch_mean * 1000.0},
            "other_forms": other,
            "clocks": clocks.summary(),
            "time_to_e0": tte,
            "time_to_e0_all_sectors": tte_c,
            "spin_chain_l32_solve": chain_solve,
            "gradients": grads,
            "stored_elements": stored,
            "spin_chain_l32": spin,
            "bosons": bosons,
            "momentum_sector_l32": momentum,
            "fermions_long_2s63": longs}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
        if bosons is not None:
            try:
                bosons["cpu_baseline"] = reference_cpu_bosons()
            except (subprocess.CalledProcessError, OSError, ValueError, IndexError) as e:
                bosons["cpu_baseline"] = {"unavailable": str(e)}
        if momentum is not None:
            try:
                momentum["cpu_baseline"] = reference_cpu_momentum_sector()
            except (subprocess.CalledProcessError, OSError, ValueError, IndexError) as e:
                momentum["cpu_baseline"] = {"unavailable": str(e)}
        if longs is not None:
            try:
                longs["cpu_baseline"] = reference_cpu_long()
            except (subprocess.CalledProcessError, OSError, ValueError, IndexError) as e:
                longs["cpu_baseline"] = {"unavailable": str(e)}
    # last: the compact time-to-E0 summary (the end of the line is what short log tails keep)
    line["time_to_e0_summary"] = time_to_e0_summary(line)
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
    ap.add_argument("--nbr-fermions", type=int, default=N_FERMIONS, help="with --leg stored: N")
    ap.add_argument("--two-s", type=int, default=TWO_S, help="with --leg stored: 2S")
    ap.add_argument("--nbr-bosons", type=int, default=12, help="with --leg bosons: N")
    ap.add_argument("--boson-two-s", type=int, default=22, help="with --leg bosons: 2S")
    ap.add_argument("--no-autotune", action="store_true",
                    help="with --kernel-only: skip the autotuner (kernel form from DH_FQHE_KERNEL / DH_FQHE_LOW_BITS)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="with --kernel-only: the arithmetic of the timed block products")
    ap.add_argument("--chain-length", type=int, default=0,
                    help="with --kernel-only: time the J1-J2 chain block product (k = 2) at this length instead")
    ap.add_argument("--leg", default=None, choices=["long", "momentum", "bosons", "stored", "sectors", "single"],
                    help="run one secondary measurement alone and print its JSON (FermionOnSphereLong N=6 2S=63; "
                         "the momentum sector at --chain-length, 32 by default; BosonOnSphereShort N=12 2S=22; "
                         "the stored-element product of the N=12 2S=33 sector; the 91-sector time to E0 at 1e-10, "
                         "median of --steps runs; the N=12 2S=33 time to E0 at 1e-10, median of --steps runs)")
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
