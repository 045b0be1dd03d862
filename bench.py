"""Benchmark: batched graph-state p(x) on B200 (single-instance throughput workload).

Workload (one "step"): a seeded random 3-regular graph on n = 40 vertices with
Haar-random SU(2) gates, scan order = the seeded random order with the largest
max rank among 2048 seeds (r_max 20); p(x) for 65,536 uniform 40-bit strings in
complex64 (float64 weights and sums), then the FP64 (complex128) recheck of every
result.  Inputs are synthetic (seeded); there is no dataset.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); every rank evaluates its own 65,536
strings (weak scaling, no data-path collective); rank 0 prints one JSON line.
``--impl reference`` times the reference's CPU executor (its NumPy sweep, restated
in ``oracle/``) on all host cores, rank 0 only.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_QUBITS = 40
GRAPH_SEED = 40
BATCH = 65536
ORDER_SEEDS = range(1000, 3048)
TARGET_RANK = 22
BITS_SEED = 1234
# Exact sampling legs: complex64 tables with float32 arithmetic (the bulk), branch masses
# and conditional normalisation summed in float64 (the chain sampler's Gram matrices).
CHAIN_PRECISION = "c64f32"


def build_instance(pkg):
    return pkg.instances.make_instance("reg3", N_QUBITS, GRAPH_SEED, pkg.rank_profile, target_rank=TARGET_RANK,
                                       order_seeds=ORDER_SEEDS)


def _instances_module():
    """The package's seeded instance generator (pure NumPy), loaded from its file alone so
    that the reference arm never imports the package or loads librgs_b200.so."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("rgs_instances_only",
                                                  ROOT / "rgs70-classical-challenge_b200" / "instances.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def build_instance_cpu():
    """The bench instance with the scan order chosen by the oracle's rank profile (the
    reference compiler restated), bit-identical to build_instance's."""
    from oracle import scan_plan as sp
    return _instances_module().make_instance("reg3", N_QUBITS, GRAPH_SEED, sp.rank_profile,
                                             target_rank=TARGET_RANK, order_seeds=ORDER_SEEDS)


def step_bytes(ranks, esize, pairs=()):
    """Compulsory table traffic of one sweep: every input entry read once, every output
    written once (step 0 reads the implicit unit table); a fused pair (j, j + 1) neither
    writes nor reads the table between its two positions."""
    r_in = [0] + list(ranks[:-1])
    total = sum((1 << a) * (j > 0) + (1 << b) for j, (a, b) in enumerate(zip(r_in, ranks)))
    return esize * (total - sum(2 << ranks[j] for j in pairs))


def chain_bytes(plan, esize, fused=True):
    """Compulsory table traffic of one chain-rule sample: per position, one read of its input
    table for the Gram pass (unless the branch masses are analytic: an empty kernel), one
    read of the input and one write of the output for the step; per fused pair (j, j + 1):
    the Gram read of j's input if j needs it, one more read of j's input for j + 1's Gram
    matrix if j + 1 needs it, then one read of j's input and one write of j + 1's output."""
    steps = plan.steps
    pairs = set(plan.pairs) if fused else set()
    total, j = 0, 0
    while j < len(steps):
        st = steps[j]
        gram = j > 0 and len(st.kernel) > 0
        if j in pairs and j + 1 < len(steps):
            total += (1 << st.r_in) * (int(gram) + int(len(steps[j + 1].kernel) > 0) + 1) + (1 << steps[j + 1].r_out)
            j += 2
        else:
            total += (1 << st.r_in) * (int(gram) + int(j > 0)) + (1 << st.r_out)
            j += 1
    return esize * total


def reference_bytes(ranks, esize):
    """Byte model of the reference kernel: every input read twice (each output gathers
    its pre-images), every output written once."""
    r_in = [0] + list(ranks[:-1])
    return esize * sum(2 * (1 << a) + (1 << b) for a, b in zip(r_in, ranks))


# ----------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------- CPU legs
def _cpu_worker(args):
    g, u, order, bits_list = args
    from oracle import scan_plan as sp
    return [sp.amplitude(g, u, order, b) for b in bits_list]


def cpu_oracle_rate(inst, bits, cores, per_core):
    """Amplitudes/s of the reference's NumPy executor (restated in oracle/) on `cores`
    spawned processes, each computing `per_core` amplitudes.  Returns (rate, amplitudes)."""
    import multiprocessing as mp
    sample = bits[:cores * per_core]
    chunks = [(inst.g, inst.u, inst.order, [b.tolist() for b in sample[i::cores]]) for i in range(cores)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_worker, [(inst.g, inst.u, inst.order, [sample[0].tolist()])] * cores)  # import warm-up
        t0 = time.perf_counter()
        out = pool.map(_cpu_worker, chunks)
        dt = time.perf_counter() - t0
    amps = np.empty(len(sample), dtype=np.complex128)
    for i in range(cores):
        amps[i::cores] = out[i]
    return len(sample) / dt, amps


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ----------------------------------------------------------------------------------- arms
def run_reference(args, rank, world):
    if rank != 0:
        return
    inst = build_instance_cpu()
    cores = host_cores()
    rng = np.random.default_rng(BITS_SEED)
    bits = _instances_module().uniform_bits(BATCH, N_QUBITS, rng)
    per_core = 2
    times = []
    for it in range(args.warmup + args.steps):
        rate, _ = cpu_oracle_rate(inst, bits[(it % 64) * cores * per_core:], cores, per_core)
        if it >= args.warmup:
            times.append(cores * per_core / rate)
    value = cores * per_core * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": "amplitudes_per_s (p(x), n=40 3-regular, complex64 + FP64 recheck)",
        "value": value, "unit": "amplitudes/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded)",
        "config": {"workload": "single-instance throughput: n=40 random 3-regular, Haar SU(2), "
                               f"r_max {inst.rmax}, 65536 uniform strings (bounded sample per step)",
                   "rmax": inst.rmax, "sum_states": inst.sum_states, "instance": inst.name},
        "cpu_baseline": {"value": value, "unit": "amplitudes/s", "cores": cores, "kind": "port",
                         "sample": f"{cores * per_core} amplitudes per step on {cores} processes "
                                   "(oracle restatement of scan_plan.sweep_reference, complex128)"},
        "e2e": {"value": value, "unit": "amplitudes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu_kernels": reference_gpu_leg(inst, bits),
    }
    print(json.dumps(line), flush=True)


def reference_gpu_leg(inst, bits):
    """The reference's own GPU scan kernels (K2 complex64, K3 complex128; compiled from its
    source into oracle/_ref/ by oracle/build_ref_gpu.py) driven as its GPUMixin._sweep does,
    on this box: the bench instance (n = 40) and the reference's RGS70 instance with its
    frozen order.  Reported beside the CPU arm; `value` stays the CPU executor's rate."""
    try:
        import torch
        from oracle import ref_gpu
        from oracle import scan_plan as sp
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
        if not (ref_gpu.available("c64") and ref_gpu.available("c128")):
            return {"unavailable": "oracle/_ref not built (needs the reference checkout at build time)"}
        out = {"driver": "one string per sweep, one launch per position, host read of the maximum after "
                         "every launch (GPUMixin._sweep)"}
        sample = bits[:8]
        ref_amp = [sp.amplitude(inst.g, inst.u, inst.order, b.tolist()) for b in sample[:2]]
        for prec in ("c64", "c128"):
            eng = ref_gpu.RefGpuScan(inst.g, inst.u, inst.order, precision=prec)
            eng.amplitude(sample[0])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            amps = [eng.amplitude(b) for b in sample]
            dt = time.perf_counter() - t0
            p_ref = np.abs(np.array(ref_amp)) ** 2
            err = float(np.max(np.abs(np.abs(np.array(amps[:2])) ** 2 - p_ref) / p_ref))
            out[f"n40_{prec}"] = {"amplitudes_per_s": len(sample) / dt, "strings": len(sample),
                                  "max_rel_err_vs_oracle": err}
            del eng
            torch.cuda.empty_cache()
        fx = np.load(ROOT / "tests" / "golden" / "fixtures.npz")
        rec = json.loads((ROOT / "tests" / "golden" / "rgs70_c128.json").read_text())["benchmark_rows"][:2]
        rbits = np.array([[int(c) for c in r["bitstring_q0_left"]] for r in rec], dtype=np.uint8)
        rp = np.array([r["probability_c128"] for r in rec])
        for prec in ("c64", "c128"):
            eng = ref_gpu.RefGpuScan(fx["rgs70/graph"], fx["rgs70/measurement_unitaries"],
                                     fx["rgs70/scan_order"].tolist(), precision=prec)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            amps = np.array([eng.amplitude(b) for b in rbits])
            dt = time.perf_counter() - t0
            out[f"rgs70_frozen_{prec}"] = {"amplitudes_per_s": len(rbits) / dt, "strings": len(rbits),
                                           "max_rel_err_vs_reference_records":
                                               float(np.max(np.abs(np.abs(amps) ** 2 - rp) / rp))}
            del eng
            torch.cuda.empty_cache()
        return out
    except Exception as exc:  # the CPU arm's line must still print
        return {"unavailable": f"{type(exc).__name__}: {exc}"}


def wht_precision_leg(pkg, device, peak, m=30, m_err=20):
    """Config 2's WHT variants: the full Walsh-Hadamard transform of a 2^m complex64 state
    by FP32 butterflies vs 16 x 16 Hadamard blocks on the tensor cores over split-BF16
    values (2 and 3 terms): time per transform (CUDA events, state of 8 GiB at m = 30:
    larger than L2), the achieved HBM rate on 16 bytes per element per pass, the relative
    L2 difference from the FP32 result at m, and the relative L2 error against an FP64
    transform at m_err."""
    import torch
    stream = torch.cuda.current_stream(device)
    out = {"m": m, "bytes_per_element_per_pass": 16}
    rng = np.random.default_rng(30)
    x0 = torch.randn(1 << m, dtype=torch.complex64, device=device)
    ref32 = None
    for prec, passes in (("fp32", None), ("split_bf16x2", None), ("split_bf16x3", None)):
        x = x0.clone()
        pkg.fwht(x, precision=prec)  # warm-up
        x.copy_(x0)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pkg.fwht(x, precision=prec)
        e1.record(stream)
        torch.cuda.synchronize(device)
        t = e0.elapsed_time(e1) / 1e3
        npass = 3 if prec == "fp32" else 1 + math.ceil((m - 12) / 8)
        rec = {"ms": 1e3 * t, "passes": npass,
               "achieved_GBps": 16 * npass * (1 << m) / t / 1e9}
        rec["hbm_frac"] = rec["achieved_GBps"] / peak
        if prec == "fp32":
            ref32 = x
        else:
            rec["rel_l2_vs_fp32"] = float(torch.linalg.vector_norm(x - ref32) / torch.linalg.vector_norm(ref32))
            del x
        out[prec] = rec
    del ref32, x0
    torch.cuda.empty_cache()
    xs = (rng.standard_normal(1 << m_err) + 1j * rng.standard_normal(1 << m_err)).astype(np.complex64)
    ref = xs.astype(np.complex128)
    for q in range(m_err):
        v = ref.reshape(-1, 2, 1 << q)
        ref = np.stack([v[:, 0] + v[:, 1], v[:, 0] - v[:, 1]], axis=1).reshape(-1)
    for prec in ("fp32", "split_bf16x2", "split_bf16x3"):
        d = torch.from_numpy(xs.copy()).to(device)
        pkg.fwht(d, precision=prec)
        got = d.cpu().numpy().astype(np.complex128)
        out[prec][f"rel_l2_err_vs_fp64_m{m_err}"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import __graft_entry__
    pkg = __graft_entry__.package()
    inst = build_instance(pkg)
    cores = host_cores()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    if world > 1:
        dist.init_process_group("nccl", device_id=device)

    plan = pkg.ScanPlan(N_QUBITS, pkg.edges_from_graph(inst.g), inst.order)
    # Replicas: every rank evaluates its own strings from its own seed stream.
    rng = np.random.default_rng(pkg.replicas.rank_seeds(BITS_SEED, world)[rank] if world > 1 else BITS_SEED)
    bits = pkg.instances.uniform_bits(BATCH, N_QUBITS, rng)
    packed = pkg.pack_bits(bits, N_QUBITS)
    # Batch tiles: given, or chosen by the package's autotuner on this GPU (first sweep).
    cap = 1 << max(0, (BATCH - 1).bit_length())
    tile64 = min(args.tile64, cap) if args.tile64 else "tune"
    tile128 = min(args.tile128, cap) if args.tile128 else "tune"
    use64, use128 = args.only in ("both", "c64"), args.only in ("both", "c128")
    eng64 = pkg.ScanEngine(plan, inst.u, device=device, precision=args.bulk, batch_tile=tile64) if use64 else None
    eng128 = pkg.ScanEngine(plan, inst.u, device=device, precision="c128", batch_tile=tile128) if use128 else None
    d_bits = torch.from_numpy(packed.view(np.int64)).to(device)
    v64, l64 = eng64.out_tensors(BATCH) if use64 else (None, None)
    v128, l128 = eng128.out_tensors(BATCH) if use128 else (None, None)
    stream = torch.cuda.current_stream(device)
    side = torch.cuda.Stream(device)

    def queue_step(s):
        # The complex64 bulk and the complex128 recheck are independent sweeps over the
        # same strings: the recheck runs on a second stream (a parallel branch of the step's
        # graph), so each sweep's kernels fill the other's launch tails.
        if use64 and use128 and not args.serial_sweeps:
            side.wait_stream(s)
            eng128.run_bits(d_bits, v128, l128, stream=side)
            eng64.run_bits(d_bits, v64, l64, stream=s)
            s.wait_stream(side)
            return
        if use64:
            eng64.run_bits(d_bits, v64, l64, stream=s)
        if use128:
            eng128.run_bits(d_bits, v128, l128, stream=s)

    # One sweep eagerly (allocates the workspaces), then the step as a CUDA graph: the
    # sweep's launches replay without host launch overhead.
    queue_step(stream)
    torch.cuda.synchronize(device)
    tile64 = eng64.batch_tile if use64 else None
    tile128 = eng128.batch_tile if use128 else None
    tuning = {k: {str(t): r for t, r in e.tuning[1].items()} for k, e in ((args.bulk, eng64), ("c128", eng128))
              if e is not None and e.tuning is not None}
    graphs = {"step": pkg.capture_graph(device, queue_step)}
    if use64:
        graphs["bulk"] = pkg.capture_graph(device, lambda s: eng64.run_bits(d_bits, v64, l64, stream=s))
    if use128:
        graphs["recheck"] = pkg.capture_graph(device, lambda s: eng128.run_bits(d_bits, v128, l128, stream=s))

    def device_step():
        graphs["step"].replay()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return pkg.replicas.max_over_ranks(x, device=device)

    def timed(fn, k):
        barrier()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / 1e3)

    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize(device)
    with ClockSampler(local_rank) as clocks:
        t_step = timed(device_step, args.steps)
    # Split of the step, and the FP64 recheck error (per result: max and quantiles).
    t64 = timed(graphs["bulk"].replay, args.steps) if use64 else None
    t128 = timed(graphs["recheck"].replay, args.steps) if use128 else None
    # The other complex64 recipe (float64 arithmetic on complex64 tables, the reference's
    # own kernel recipe), for comparison: time and error only.
    alt = None
    if use64 and use128 and not args.no_alt:
        alt_prec = "c64" if args.bulk == "c64f32" else "c64f32"
        alt_tile = min(256 if alt_prec == "c64f32" else 128, 1 << max(0, (BATCH - 1).bit_length()))
        eng_alt = pkg.ScanEngine(plan, inst.u, device=device, precision=alt_prec, batch_tile=alt_tile)
        va, la = eng_alt.out_tensors(BATCH)
        eng_alt.run_bits(d_bits, va, la, stream=stream)
        torch.cuda.synchronize(device)
        g_alt = pkg.capture_graph(device, lambda s: eng_alt.run_bits(d_bits, va, la, stream=s))
        t_alt = timed(g_alt.replay, args.steps)
        alt = {"precision": alt_prec, "t": t_alt, "v": va, "l": la}
        del g_alt, eng_alt
    recheck = None
    p128 = None
    if use64 and use128:
        p64 = np.abs(pkg.amplitudes_from(v64.cpu().numpy(), l64.cpu().numpy(), N_QUBITS)) ** 2
        p128 = np.abs(pkg.amplitudes_from(v128.cpu().numpy(), l128.cpu().numpy(), N_QUBITS)) ** 2
        if not (np.all(np.isfinite(p64)) and np.all(np.isfinite(p128))):
            raise ArithmeticError("non-finite probability in the benchmark run")
        def err_stats(p):
            rel = np.abs(p - p128) / p128
            scaled = np.abs(p - p128) * 2.0 ** N_QUBITS
            return {"max_prob_rel_err": float(rel.max()), "median_prob_rel_err": float(np.median(rel)),
                    "p999_prob_rel_err": float(np.quantile(rel, 0.999)),
                    "frac_above_1e-4": float(np.mean(rel > 1e-4)),
                    "max_rel_err_p_ge_0.01_over_2^n": float(rel[p128 * 2.0 ** N_QUBITS >= 0.01].max()),
                    "max_abs_err_times_2^n": float(scaled.max())}
        recheck = {"bulk": args.bulk, **err_stats(p64)}
        if alt is not None:
            pa = np.abs(pkg.amplitudes_from(alt["v"].cpu().numpy(), alt["l"].cpu().numpy(), N_QUBITS)) ** 2
            recheck["other_complex64_recipe"] = {"precision": alt["precision"],
                                                 "amplitudes_per_s": world * BATCH * args.steps / alt["t"],
                                                 **err_stats(pa)}

    # End to end through the public API: pinned host bits in, host probabilities out.
    h_bits = torch.from_numpy(packed.view(np.int64)).pin_memory()
    h_v64 = torch.empty(BATCH, dtype=torch.complex64).pin_memory()
    h_l64 = torch.empty(BATCH, dtype=torch.float64).pin_memory()
    h_v128 = torch.empty(BATCH, dtype=torch.complex128).pin_memory()
    h_l128 = torch.empty(BATCH, dtype=torch.float64).pin_memory()

    def e2e_step():
        d_bits.copy_(h_bits, non_blocking=True)
        device_step()
        if use64:
            h_v64.copy_(v64, non_blocking=True)
            h_l64.copy_(l64, non_blocking=True)
        if use128:
            h_v128.copy_(v128, non_blocking=True)
            h_l128.copy_(l128, non_blocking=True)

    t_e2e = None
    if not args.no_e2e:
        for _ in range(max(1, args.warmup // 2)):
            e2e_step()
        t_e2e = timed(e2e_step, args.steps)
    h2d = packed.nbytes
    d2h = BATCH * ((8 + 8 if use64 else 0) + (16 + 8 if use128 else 0))

    # Roofline of the scan-step kernels (dominant: every launch but the weights and
    # finalisation kernels, one or two per chunk of tiles).
    b64 = step_bytes(inst.ranks, 8, plan.pairs) * BATCH if use64 else 0
    b128 = step_bytes(inst.ranks, 16, plan.pairs) * BATCH if use128 else 0
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peak, peak_src = 6650.0, "fallback"
    if peaks_path.exists():
        peak, peak_src = float(json.loads(peaks_path.read_text())["hbm_gbs"]), "measured"
    achieved = (b64 + b128) / (t_step / args.steps) / 1e9
    # DRAM traffic of one chunk sweep (8192 strings) from one ncu capture, times the chunks
    # of this step (valid for the tile sizes it was captured at).
    traffic = None
    traffic_path = ROOT / "profiles" / "scan_step_traffic.json"
    if traffic_path.exists():
        tr = json.loads(traffic_path.read_text()).get("dram_bytes_per_chunk", {})
        t64r, t128r = tr.get(args.bulk), tr.get("c128")
        if (not use64 or (t64r and t64r["tile"] == tile64)) and (not use128 or (t128r and t128r["tile"] == tile128)):
            traffic = ((BATCH / t64r["items"] * t64r["bytes"] if use64 else 0)
                       + (BATCH / t128r["items"] * t128r["bytes"] if use128 else 0))
    # Kernel launches of one step, from the library's own schedule.
    launches = args.steps * ((eng64.launch_count(BATCH) if use64 else 0)
                             + (eng128.launch_count(BATCH) if use128 else 0))

    # Secondary: exact Born samples/s of the chain sampler on the same instance.
    saved = BATCH
    globals()["BATCH"] = min(BATCH, 16384)
    chain = run_chain(args, rank, world, local_rank, emit=False)
    globals()["BATCH"] = saved
    # The other configurations' headline numbers, bounded (single-GPU measurements, rank 0).
    extra = {}
    if rank == 0 and not args.no_extra:
        peak_extra = 6650.0
        if (ROOT / "MEASURED_PEAKS.json").exists():
            peak_extra = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
        del graphs
        torch.cuda.empty_cache()

        def full_leg():
            fs, fs_inst = full_scale(pkg, device, 64, legs=("random_order",), rescore=64)
            leg = fs["random_order"]
            return dict(leg, workload="config 5: n=70 random degree<=3 graph, seeded random order "
                                      f"(r_max {leg['rmax']}), 64 exact Born samples by the chain rule",
                        instance=fs_inst.name, unit="samples/s", hbm_frac=leg["achieved_GBps"] / peak_extra)

        # Each leg on its own: a failure is reported in the line, not fatal to it.
        for key, fn in (("full_scale_n70", full_leg),
                        ("learned_n56", lambda: learned_comparison(pkg, device, 1024, 1 << 16, 4)),
                        ("wht_fp32_vs_split_bf16", lambda: wht_precision_leg(pkg, device, peak_extra))):
            try:
                extra[key] = fn()
            except Exception as exc:
                extra[key] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.synchronize(device)
            torch.cuda.empty_cache()
    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu_rate, cpu_amps = cpu_oracle_rate(inst, bits, cores, 2)
            cpu = {"value": cpu_rate, "unit": "amplitudes/s", "cores": cores, "kind": "port",
                   "sample": f"{2 * cores} amplitudes (complex128 NumPy sweep restated from the reference) "
                             f"on {cores} spawned processes"}
            p_cpu = np.abs(cpu_amps) ** 2
            if p128 is not None:
                cpu["parity_max_rel_err_vs_fp64"] = float(np.max(np.abs(p128[:len(p_cpu)] - p_cpu) / p_cpu))
        value = world * BATCH * args.steps / t_step
        line = {
            "metric": "amplitudes_per_s (p(x), n=40 3-regular, complex64 + FP64 recheck)",
            "value": value, "unit": "amplitudes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_step / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": ("c64 (fp32 math) + c128 recheck" if args.bulk == "c64f32" else "c64 (fp64 math) + c128 recheck"),
            "data": "synthetic (seeded graph, gates and bitstrings)",
            "config": {"workload": "single-instance throughput: n=40 random 3-regular, Haar SU(2), "
                                   "65536 uniform 40-bit strings, complex64 + FP64 recheck of every result",
                       "instance": inst.name, "rmax": inst.rmax, "sum_states": inst.sum_states,
                       "batch_per_gpu": BATCH, "batch_tile": {args.bulk: tile64, "c128": tile128},
                       "autotune_items_per_s": tuning,
                       "precisions": args.only,
                       "bulk": ("complex64 tables, float32 arithmetic" if args.bulk == "c64f32"
                                else "complex64 tables, float64 arithmetic (the reference recipe)"),
                       "recheck": "complex128 tables, float64 arithmetic, every result",
                       "launch": ("the two sweeps replayed from one CUDA graph, one after the other"
                                  if args.serial_sweeps else
                                  "the two sweeps replayed from one CUDA graph, the recheck on a parallel "
                                  "branch (second stream)"),
                       "l2": "inputs larger than L2 (tables of 2^20 rows x batch tile, >= 2 x 1 GiB)",
                       "parallelism": f"replicas x{world}"},
            "split": {f"{args.bulk}_amplitudes_per_s": world * BATCH * args.steps / t64 if t64 else None,
                      "c128_amplitudes_per_s": world * BATCH * args.steps / t128 if t128 else None},
            "fp64_recheck": recheck,
            "exact_born_samples": {"value": chain["value"], "unit": "samples/s", "samples_per_step": 16384,
                                   "method": "chain rule over the scan (complex64)", "checks": chain["checks"],
                                   "achieved_GBps": chain["roofline"]["achieved"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes_per_step": b64 + b128,
                         "reference_model_bytes_per_step": (reference_bytes(inst.ranks, 8)
                                                            + reference_bytes(inst.ranks, 16)) * BATCH},
            "e2e": {"value": world * BATCH * args.steps / t_e2e if t_e2e else None, "unit": "amplitudes/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            **extra,
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


def fourier_instance(pkg, m, seed=None):
    """Seeded dense graph on 2m vertices with a full-rank balanced cut A = 0..m-1,
    B = m..2m-1; Haar gates, identical on B (the reference's production specialisation)."""
    rng = np.random.default_rng(1000 + m if seed is None else seed)
    while True:
        g = pkg.instances.dense(2 * m, rng)
        A, B = list(range(m)), list(range(m, 2 * m))
        try:
            pkg.samplers.cut_tables(g, np.tile(np.eye(2, dtype=np.complex128), (2 * m, 1, 1)), A, B)
            break
        except ValueError:
            continue
    u = pkg.instances.haar_su2(2 * m, rng)
    u[B] = u[B[0]]
    return g, u, A, B


def run_fourier(args, rank, world, local_rank):
    """One step = one exact conditional Born sample (compute + draw) of the Fourier-cut
    sampler at m conditional qubits (2^m complex64 state on one GPU)."""
    import ctypes
    import torch
    import __graft_entry__
    pkg = __graft_entry__.package()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    m = args.m
    g, u, A, B = fourier_instance(pkg, m)
    L = pkg._lib.lib()
    pkg._lib.check(L.rgs_fourier_set_register_schedule(1 if args.pass_kernel == "registers" else 0))
    pkg._lib.check(L.rgs_fourier_set_tma(1 if args.tma else 0))
    s = pkg.ConditionalSampler(g, u, A, B, [local_rank])
    variant, tune_ms = s.tune()
    stream = torch.cuda.current_stream(device)
    rng = np.random.default_rng(99 + rank)

    def sample():
        ob = rng.integers(0, 2, m)
        mask = int(sum(int(x) << j for j, x in enumerate(ob)))
        pkg._lib.check(L.rgs_fourier_compute(s._h, mask, ctypes.c_void_p(s.state.data_ptr()),
                                             ctypes.c_void_p(s.workspace.data_ptr()), s.workspace.numel(),
                                             ctypes.c_void_p(stream.cuda_stream), None))
        return s.draw(rng)

    for _ in range(args.warmup):
        sample()
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            sample()
        e1.record(stream)
        torch.cuda.synchronize(device)
    t = e0.elapsed_time(e1) / 1e3
    # Pass 0 computes the state and writes it (8 B/element); every other pass reads and
    # writes it (16 B/element).
    bytes_per_sample = (1 << m) * (8 + 16 * (s.passes - 1))
    peak = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]) \
        if (ROOT / "MEASURED_PEAKS.json").exists() else 6650.0
    achieved = bytes_per_sample * args.steps / t / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": f"exact_born_samples_per_s (Fourier-cut conditional sampler, m={m})",
            "value": args.steps / t, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded dense graph)",
            "config": {"workload": f"conditional sampler, dense graph n={2 * m}, full-rank balanced cut m={m}",
                       "passes": s.passes, "specialized": s.specialized, "pass_kernel": args.pass_kernel,
                       "tile_loads": "tma" if args.tma and args.pass_kernel == "registers" else "threads",
                       "tuned_variant": {"chosen": variant, "ms_per_compute": tune_ms,
                                         "variants": "3 or 4 resident blocks per SM"}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "algorithmic_bytes_per_step": bytes_per_sample},
            "gpu_launches": args.steps * (s.passes + 2), "clocks": clocks.summary()}), flush=True)


def run_chain(args, rank, world, local_rank, emit=True):
    """One step = BATCH exact Born samples of the n=40 instance by the chain rule over
    the scan (complex64, float64 weights), each with its probability."""
    import torch
    import torch.distributed as dist
    import __graft_entry__
    pkg = __graft_entry__.package()
    inst = build_instance(pkg)
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    if world > 1 and not dist.is_initialized():
        dist.init_process_group("nccl", device_id=device)
    chain_tile = min(args.tile64 or 128, 128)
    cs = pkg.ChainSampler(inst.g, inst.u, inst.order, device=device, precision=CHAIN_PRECISION,
                          batch_tile=chain_tile)
    stream = torch.cuda.current_stream(device)
    outs = cs._outs(BATCH)
    seed = [1000 + rank]

    def step():
        seed[0] += 1
        return cs.sample_device(BATCH, seed=seed[0], check=False, stream=stream, outs=outs)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(device)
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            res = step()
        e1.record(stream)
        torch.cuda.synchronize(device)
    t = e0.elapsed_time(e1) / 1e3
    if world > 1:
        tt = torch.tensor([t], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    bits, value, logscale, logp = res
    p = np.abs(pkg.amplitudes_from(value.cpu().numpy().astype(np.complex128), logscale.cpu().numpy(), N_QUBITS)) ** 2
    lp = logp.cpu().numpy()
    consistency = float(np.max(np.abs(np.log(p) - lp)))
    xeb = float((2.0 ** N_QUBITS) * p.mean() - 1)
    # Table traffic per sample (compulsory bytes): the sweep, plus the Gram reads.
    bytes_per = chain_bytes(cs.plan, 8)
    line = {"metric": "exact_born_samples_per_s (chain rule over the scan, n=40 3-regular)",
            "value": world * BATCH * args.steps / t, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 (fp32 math, fp64 branch masses)", "data": "synthetic (seeded graph and gates, Philox uniforms)",
            "config": {"workload": f"n=40 random 3-regular, r_max {inst.rmax}, {BATCH} samples per GPU per step",
                       "instance": inst.name, "batch_tile": chain_tile},
            "roofline": {"bound": "hbm", "achieved": bytes_per * BATCH * args.steps / t / 1e9,
                         "algorithmic_bytes_per_step": bytes_per * BATCH},
            "checks": {"max_abs_logp_minus_log_p": consistency, "linear_xeb": xeb},
            "gpu_launches": args.steps * cs.launch_count(BATCH),
            "clocks": clocks.summary()}
    if emit and rank == 0:
        print(json.dumps(line), flush=True)
    return line


BATCH_INSTANCES = 1024
BATCH_STRINGS = 256
BATCH_SAMPLES = 64
BATCH_SEED = 2026


def batched_instances(pkg, count, max_rank):
    """Uneven instances: n uniform in [20, 36], Erdos-Renyi graphs of average degree 3,
    Haar SU(2) gates.  Order: the lowest max rank among 64 seeded random orders (2048 when
    that is above the resident maximum), then 20,000 steps of the package's order search
    (seeded; one host thread per instance)."""
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(BATCH_SEED)
    out = []
    for i in range(count):
        n = int(rng.integers(20, 37))
        inst = pkg.instances.make_instance("er3", n, 300000 + i, pkg.rank_profile, target_rank=0,
                                           order_seeds=range(64))
        if inst.rmax > max_rank:
            inst = pkg.instances.make_instance("er3", n, 300000 + i, pkg.rank_profile, target_rank=0,
                                               order_seeds=range(2048))
        out.append(inst)

    def search(inst):
        order, ranks, _ = pkg.search_order(inst.n, pkg.edges_from_graph(inst.g), inst.order, iterations=20000,
                                           seed=1, threads=1)
        return pkg.instances.Instance(inst.g, inst.u, order, ranks, inst.name + "-searched")
    with ThreadPoolExecutor(max(1, min(16, host_cores()))) as ex:
        return list(ex.map(search, out))


def run_batched(args, rank, world, local_rank):
    """One step = one captured launch over 1024 uneven instances: 256 amplitudes of uniform
    strings + 64 exact chain-rule samples of each (complex64, float64 weights)."""
    import torch
    import torch.distributed as dist
    import __graft_entry__
    pkg = __graft_entry__.package()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    if world > 1 and not dist.is_initialized():
        dist.init_process_group("nccl", device_id=device)
    rmax_res = pkg.batch.max_rank("c64")
    insts = batched_instances(pkg, BATCH_INSTANCES, rmax_res)
    if max(i.rmax for i in insts) > rmax_res:
        raise SystemExit("an instance is above the resident rank limit")
    K, S = BATCH_STRINGS, BATCH_SAMPLES
    nI = len(insts)
    rng = np.random.default_rng(BATCH_SEED + 1 + rank)
    host_bits = np.concatenate([pkg.pack_bits(pkg.instances.uniform_bits(K, i.n, rng), i.n) for i in insts])
    pinned_bits = torch.from_numpy(host_bits.view(np.int64)).pin_memory()
    d_bits = torch.empty((nI * K, 2), dtype=torch.int64, device=device)
    d_bits.copy_(pinned_bits)
    value = torch.empty(nI * K, dtype=torch.complex64, device=device)
    logscale = torch.empty(nI * K, dtype=torch.float64, device=device)
    sbits = torch.empty((nI * S, 2), dtype=torch.int64, device=device)
    svalue = torch.empty(nI * S, dtype=torch.complex64, device=device)
    slogscale = torch.empty(nI * S, dtype=torch.float64, device=device)
    slogp = torch.empty(nI * S, dtype=torch.float64, device=device)
    rb = pkg.ResidentBatch("c64", device=device)
    plans = []
    for k, inst in enumerate(insts):
        plan = pkg.ScanPlan(inst.n, pkg.edges_from_graph(inst.g), inst.order)
        plans.append(plan)
        du = torch.from_numpy(np.asarray(inst.u, dtype=np.complex128).view(np.float64).reshape(-1).copy()).to(device)
        a, b = k * K, (k + 1) * K
        c, d = k * S, (k + 1) * S
        rb.add_device(plan, du, d_bits[a:b], value[a:b], logscale[a:b], S, 5000 + 7919 * k + rank,
                      sbits[c:d], svalue[c:d], slogscale[c:d], slogp[c:d])
    variant, tune_ms = rb.tune()
    rb.capture()
    stream = torch.cuda.current_stream(device)
    for _ in range(args.warmup):
        rb.replay()
    torch.cuda.synchronize(device)
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            rb.replay()
        e1.record(stream)
        torch.cuda.synchronize(device)
    t = e0.elapsed_time(e1) / 1e3
    # End to end through the public API: pinned host bits in, every result out, each step.
    outs = [value, logscale, sbits, svalue, slogscale, slogp]
    host_outs = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in outs]
    h2d = pinned_bits.numel() * 8
    d2h = sum(o.numel() * o.element_size() for o in outs)
    torch.cuda.synchronize(device)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        d_bits.copy_(pinned_bits, non_blocking=True)
        rb.run(check=False, stream=stream)
        for h, o in zip(host_outs, outs):
            h.copy_(o, non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize(device)
    te = f0.elapsed_time(f1) / 1e3
    if world > 1:
        tt = torch.tensor([t, te], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t, te = (float(x) for x in tt.tolist())
    # Checks: every amplitude row of instance 0 against the streaming executor (bitwise),
    # log p of the samples against log |amplitude|^2.
    so = pkg.ScanOracle(insts[0].g, insts[0].u, insts[0].order)
    v0, l0 = so.engine.sweep_bits(pkg.unpack_bits(host_bits[:K], insts[0].n))
    same = bool(np.array_equal(value[:K].cpu().numpy().astype(np.complex128), v0)
                and np.array_equal(logscale[:K].cpu().numpy(), l0))
    ns = np.array([i.n for i in insts for _ in range(S)])
    p = np.abs(pkg.amplitudes_from(svalue.cpu().numpy().astype(np.complex128), slogscale.cpu().numpy(), 0)) ** 2
    p = p * np.exp(-ns * math.log(2.0))
    consistency = float(np.max(np.abs(np.log(p) - slogp.cpu().numpy())))
    items = nI * (K + S)
    # Table traffic in shared memory per step (the streaming executor's compulsory HBM bytes
    # for the same sweeps; samples also read every table once for the branch masses).
    tb = 0
    for inst, plan in zip(insts, plans):
        tb += K * step_bytes(inst.ranks, 8) + S * chain_bytes(plan, 8)
    smem_peak = 148 * 128 * 1.965e9 / 1e9  # nominal: 128 B/clock/SM at the maximum SM clock
    line = {"metric": "batched_items_per_s (amplitudes + exact samples, 1024 uneven instances, one launch)",
            "value": world * items * args.steps / t, "unit": "items/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic (seeded graphs, gates, strings; Philox uniforms)",
            "config": {"workload": f"{nI} Erdos-Renyi instances (avg degree 3, n in [20,36], searched orders, r_max "
                                   f"{min(i.rmax for i in insts)}-{max(i.rmax for i in insts)}): {K} amplitudes + "
                                   f"{S} samples each per step, one persistent launch replayed from a CUDA graph",
                       "instances": nI, "strings_per_instance": K, "samples_per_instance": S,
                       "work_units": rb.units, "l2": "tables live in shared memory; HBM holds only inputs and outputs",
                       "tuned_variant": {"chosen": ["512 threads, 1 block/SM", "256 threads, 2 blocks/SM",
                                                    "128 threads, 4 blocks/SM"][variant],
                                         "ms_per_run": tune_ms}},
            "roofline": {"bound": "smem", "achieved": tb * args.steps / t / 1e9, "peak": smem_peak, "unit": "GB/s",
                         "frac": tb * args.steps / t / 1e9 / smem_peak, "traffic": None,
                         "note": "table bytes through shared memory vs the nominal shared-memory bandwidth"},
            "e2e": {"value": world * items * args.steps / te, "unit": "items/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "amplitudes_per_s": world * nI * K * args.steps / t, "samples_per_s": world * nI * S * args.steps / t,
            "checks": {"instance0_bitwise_equal_streaming": same, "max_abs_logp_minus_log_p": consistency},
            "gpu_launches": args.steps, "clocks": clocks.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)


# Published reference numbers for RGS70 (1x / 2x H200): 32 fixed inputs in 2.986 s (complex64,
# frozen order) and 4.180 s (complex128); exact Born sampling 2.416 s per sample (2x H200).
RGS70_REF_C64_AMP_PER_S = 32 / 2.986
RGS70_REF_C128_AMP_PER_S = 32 / 4.180
RGS70_REF_SAMPLES_PER_S_2GPU = 1 / 2.416


def run_rgs70(args, rank, world, local_rank):
    """The reference's own RGS70 instance (n = 70, 1150 edges, rank 30): p(x) of its 32
    benchmark strings with the frozen order (complex64 and complex128), and exact Born
    samples by the chain rule with the optimised order, each rescored in complex128."""
    import torch
    import torch.distributed as dist
    from scipy import stats
    import __graft_entry__
    pkg = __graft_entry__.package()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    if world > 1 and not dist.is_initialized():
        dist.init_process_group("nccl", device_id=device)
    fx = np.load(ROOT / "tests" / "golden" / "fixtures.npz")
    rec = json.loads((ROOT / "tests" / "golden" / "rgs70_c128.json").read_text())
    born = json.loads((ROOT / "tests" / "golden" / "rgs70_born.json").read_text())["probability_c128"]
    g, u = fx["rgs70/graph"], fx["rgs70/measurement_unitaries"]
    frozen, optimised = fx["rgs70/scan_order"].tolist(), fx["rgs70/scan_order_optimized"].tolist()
    searched = json.loads((ROOT / "tests" / "golden" / "searched_orders.json").read_text())["rgs70"]["order"]
    rows = rec["benchmark_rows"]
    bits = np.array([[int(c) for c in r["bitstring_q0_left"]] for r in rows], dtype=np.uint8)
    ref_p = np.array([r["probability_c128"] for r in rows])
    stream = torch.cuda.current_stream(device)

    def timed(fn, k):
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        return e0.elapsed_time(e1) / 1e3

    def free():
        torch.cuda.synchronize(device)
        torch.cuda.empty_cache()

    plan_f = pkg.ScanPlan(70, pkg.edges_from_graph(g), frozen)
    d_bits = torch.from_numpy(pkg.pack_bits(bits, 70).view(np.int64)).to(device)
    legs = {}
    with ClockSampler(local_rank) as clocks:
        for prec, tile in (("c64", 8), ("c128", 4)):
            eng = pkg.ScanEngine(plan_f, u, device=device, precision=prec, batch_tile=tile)
            val, ls = eng.out_tensors(len(bits))
            for _ in range(args.warmup if prec == "c64" else 1):
                eng.run_bits(d_bits, val, ls, stream=stream)
            t = timed(lambda: eng.run_bits(d_bits, val, ls, stream=stream), args.steps)
            p = np.abs(pkg.amplitudes_from(val.cpu().numpy().astype(np.complex128), ls.cpu().numpy(), 70)) ** 2
            esize = 16 if prec == "c128" else 8
            legs[prec] = {"amplitudes_per_s": len(bits) * args.steps / t, "batch_tile": tile,
                          "max_rel_err_vs_reference_c128": float(np.max(np.abs(p - ref_p) / ref_p)),
                          "achieved_GBps": step_bytes(plan_f.ranks, esize, plan_f.pairs) * len(bits) * args.steps
                          / t / 1e9,
                          "launches_per_sweep": eng.launch_count(len(bits))}
            del eng, val, ls
            free()
        # Exact Born samples, complex64 tables, 8 samples per tile: the reference's optimised
        # order, then the order found by this package's search (tests/golden/searched_orders.json).
        S = 16
        sampled = {}
        for name, sorder in (("reference_optimised", optimised), ("searched", searched)):
            cs = pkg.ChainSampler(g, u, sorder, device=device, precision=CHAIN_PRECISION, batch_tile=8)
            outs = cs._outs(S)
            seed = [70000 + 1000 * rank]

            def sample():
                seed[0] += 1
                return cs.sample_device(S, seed=seed[0], check=False, stream=stream, outs=outs)
            sample()
            ts = timed(sample, args.steps)
            sbits, sval, sls, slogp = sample()
            torch.cuda.synchronize(device)
            sampled[name] = {"t": ts, "plan": cs.plan, "bits": pkg.unpack_bits(sbits.cpu().numpy(), 70),
                             "p64": np.abs(pkg.amplitudes_from(sval.cpu().numpy().astype(np.complex128),
                                                               sls.cpu().numpy(), 70)) ** 2,
                             "logp": slogp.cpu().numpy()}
            del cs, outs, sbits, sval, sls, slogp
            free()
    so = pkg.ScanOracle(g, u, searched, device=device, fp64=True, batch_tile=4)
    for rec_s in sampled.values():
        rec_s["p128"] = so.probabilities(rec_s["bits"])
    del so
    free()
    zref = np.concatenate([born["batch1"], born["batch2"]]) * 2.0 ** 70
    samples_out = {}
    for name, rec_s in sampled.items():
        rate = S * args.steps / rec_s["t"]
        z = rec_s["p128"] * 2.0 ** 70
        ks = stats.ks_2samp(z, zref)
        samples_out[name] = {
            "value": rate, "unit": "samples/s", "sum_states": rec_s["plan"].sum_states,
            "rmax": rec_s["plan"].rmax, "samples_per_step": S,
            "vs_reference_2xH200": rate / RGS70_REF_SAMPLES_PER_S_2GPU,
            "achieved_GBps": chain_bytes(rec_s["plan"], 8) * S * args.steps / rec_s["t"] / 1e9,
            "max_rel_err_c64_vs_c128_rescore": float(np.max(np.abs(rec_s["p64"] - rec_s["p128"]) / rec_s["p128"])),
            "max_abs_logp_minus_log_p128": float(np.max(np.abs(rec_s["logp"] - np.log(rec_s["p128"])))),
            "linear_xeb_of_these_samples": float(z.mean() - 1),
            "ks_vs_reference_born_samples": {"statistic": float(ks.statistic), "pvalue": float(ks.pvalue),
                                             "reference_samples": int(len(zref))}}
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peak = float(json.loads(peaks_path.read_text())["hbm_gbs"]) if peaks_path.exists() else 6650.0
    value = legs["c64"]["amplitudes_per_s"]
    line = {"metric": "amplitudes_per_s (p(x), RGS70 n=70 rank 30, frozen order, complex64)",
            "value": world * value, "unit": "amplitudes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * len(bits) / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / RGS70_REF_C64_AMP_PER_S, "dtype": "c64",
            "data": "the reference's RGS70 instance and its 32 benchmark strings (fixtures from the reference)",
            "config": {"workload": "RGS70 replay: n=70 dense (1150 edges), identical gates, frozen order r_max 30, "
                                   "sum 2^r 9,982,443,517; 32 strings", "sum_states": plan_f.sum_states},
            "roofline": {"bound": "hbm", "achieved": legs["c64"]["achieved_GBps"], "peak": peak, "unit": "GB/s",
                         "frac": legs["c64"]["achieved_GBps"] / peak, "traffic": None},
            "legs": legs,
            "reference_published": {"c64_amplitudes_per_s_1xH200": RGS70_REF_C64_AMP_PER_S,
                                    "c128_amplitudes_per_s_1xH200": RGS70_REF_C128_AMP_PER_S,
                                    "born_samples_per_s_2xH200": RGS70_REF_SAMPLES_PER_S_2GPU},
            "exact_born_samples": samples_out,
            "gpu_launches": args.steps * legs["c64"]["launches_per_sweep"], "clocks": clocks.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)


def full_scale(pkg, device, S, legs=("random_order", "searched_order"), rescore=256, seed=7000):
    """Config 5, full scale on one GPU: n = 70 random degree-<=3 graph, Haar SU(2) gates, the
    seeded random order whose max rank is closest to 30 (two complex64 2^30 tables per
    sample and batch item); S exact Born samples by the chain rule (complex64 tables, float64
    branch masses), `rescore` of them rescored in complex128, linear XEB with the rescored
    p and over all samples; optionally the same instance with the package's order search.
    Returns (legs dict, instance)."""
    import torch
    inst = pkg.instances.make_instance("deg3", 70, 70, pkg.rank_profile, target_rank=30,
                                       order_seeds=range(1000, 1256))
    edges = pkg.edges_from_graph(inst.g)
    orders = {"random_order": inst.order}
    if "searched_order" in legs:
        orders["searched_order"], _, _ = pkg.search_order(70, edges, inst.order, iterations=200000, seed=1,
                                                          threads=max(1, min(16, host_cores())))
    stream = torch.cuda.current_stream(device)
    raw = {}
    for name in legs:
        order = orders[name]
        plan = pkg.ScanPlan(70, edges, order)
        tile = 1
        while tile < 128 and 2 * (2 * tile) * 8 * (1 << plan.rmax) <= 120 * 2 ** 30 and 2 * tile <= S:
            tile *= 2
        cs = pkg.ChainSampler(inst.g, inst.u, order, device=device, precision=CHAIN_PRECISION, batch_tile=tile,
                              plan=plan)
        cs.sample_device(min(S, tile), seed=1, check=True, stream=stream)  # warm-up
        outs = cs._outs(S)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bits, value, logscale, logp = cs.sample_device(S, seed=seed, check=False, stream=stream, outs=outs)
        e1.record(stream)
        torch.cuda.synchronize(device)
        t = e0.elapsed_time(e1) / 1e3
        raw[name] = {"samples_per_s": S / t, "seconds": t, "rmax": plan.rmax, "sum_states": plan.sum_states,
                     "batch_tile": tile, "achieved_GBps": chain_bytes(plan, 8) * S / t / 1e9,
                     "samples": pkg.unpack_bits(bits.cpu().numpy(), 70),
                     "p64": np.abs(pkg.amplitudes_from(value.cpu().numpy().astype(np.complex128),
                                                       logscale.cpu().numpy(), 70)) ** 2,
                     "logp": logp.cpu().numpy()}
        del cs, outs, bits, value, logscale, logp
        torch.cuda.synchronize(device)
        torch.cuda.empty_cache()
    # complex128 rescoring with the cheapest order at hand (any order gives the same p(x)).
    rescore_order = orders.get("searched_order", inst.order)
    so = pkg.ScanOracle(inst.g, inst.u, rescore_order, device=device, fp64=True)
    out = {}
    for name, leg in raw.items():
        k = min(rescore, S)
        p128 = so.probabilities(leg["samples"][:k])
        rel = np.abs(leg["p64"][:k] - p128) / p128
        out[name] = {key: leg[key] for key in ("samples_per_s", "seconds", "rmax", "sum_states", "batch_tile",
                                               "achieved_GBps")}
        out[name].update({"samples": S, "rescored": k, "max_rel_err_c64_vs_c128": float(rel.max()),
                          "max_abs_logp_minus_log_p128": float(np.max(np.abs(leg["logp"][:k] - np.log(p128)))),
                          "linear_xeb_rescored": float((2.0 ** 70) * p128.mean() - 1),
                          "linear_xeb_all_c64": float((2.0 ** 70) * leg["p64"].mean() - 1)})
    del so
    torch.cuda.empty_cache()
    return out, inst


def run_full(args, rank, world, local_rank):
    """Full scale on one GPU (config 5) with `--samples` exact samples, random and searched orders."""
    import torch
    import __graft_entry__
    pkg = __graft_entry__.package()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    S = args.samples
    with ClockSampler(local_rank) as clocks:
        out, inst = full_scale(pkg, device, S, seed=7000 + rank)
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peak = float(json.loads(peaks_path.read_text())["hbm_gbs"]) if peaks_path.exists() else 6650.0
    main = out["random_order"]
    line = {"metric": "exact_born_samples_per_s (n=70 degree<=3, rank 30, chain rule, complex64)",
            "value": main["samples_per_s"], "unit": "samples/s", "n_gpus": world, "steps": 1, "warmup": 1,
            "ms_per_step": 1e3 * main["seconds"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 (fp32 math, fp64 branch masses)", "data": "synthetic (seeded graph, gates, Philox uniforms)",
            "config": {"workload": f"full scale: n=70 random degree<=3 graph, seeded random order with r_max "
                                   f"{main['rmax']}, {S} exact samples, 256 rescored in complex128",
                       "instance": inst.name},
            "roofline": {"bound": "hbm", "achieved": main["achieved_GBps"], "peak": peak, "unit": "GB/s",
                         "frac": main["achieved_GBps"] / peak, "traffic": None},
            "legs": out, "clocks": clocks.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)


def learned_comparison(pkg, device, samples, train_samples, epochs, order_policy="searched", batch_tile=64):
    """Config 4: n=56 random degree<=3 graph (max rank <= 28), MADE 2x512 trained on exact
    samples + their exact conditionals; `samples` accepted samples from (a) rejection with
    the learned proposal (Born-exact under the calibrated envelope), (b) the plain exact
    sampler (chain rule over the scan), (c) the reference's uniform capped rule (cap 1, not
    Born).  order_policy "searched": the package's order search from the seeded order;
    "random": the seeded random order.  Returns a dict of measurements."""
    import torch
    n = 56
    inst = pkg.instances.make_instance("deg3", n, 56, pkg.rank_profile)
    order = inst.order
    if order_policy == "searched":
        order, _, _ = pkg.search_order(n, pkg.edges_from_graph(inst.g), inst.order, iterations=100000, seed=1,
                                       threads=max(1, min(16, host_cores())))
    plan = pkg.ScanPlan(n, pkg.edges_from_graph(inst.g), order)
    if plan.rmax > 28:
        raise SystemExit(f"instance rank {plan.rmax} above 28")
    cs = pkg.ChainSampler(inst.g, inst.u, order, device=device, precision=CHAIN_PRECISION, batch_tile=batch_tile)
    so = pkg.ScanOracle(inst.g, inst.u, order, device=device, precision="c64f32")
    so128 = pkg.ScanOracle(inst.g, inst.u, order, device=device, fp64=True)
    order_a = np.asarray(order)
    inv = np.argsort(order_a)
    t0 = time.perf_counter()
    bits, p, logp, cond = cs.sample(train_samples, seed=1, with_conditionals=True)
    t_data = time.perf_counter() - t0
    net = pkg.MadeProposal(n, hidden=512, device=device, seed=3)
    t0 = time.perf_counter()
    losses = net.fit(bits[:, order_a], cond, epochs=epochs, batch=4096, lr=3e-3)
    torch.cuda.synchronize(device)
    t_train = time.perf_counter() - t0
    c = np.clip(cond.astype(np.float64), 1e-12, 1 - 1e-12)
    floor = float(np.mean(np.sum(-(c * np.log(c) + (1 - c) * np.log(1 - c)), axis=1)))
    # Envelope from held-out exact samples; deficit (TV of the output) on a separate set.
    cal_bits, _, cal_logp = cs.sample(16384, seed=2)
    cal_lq = net.log_q(torch.as_tensor(cal_bits[:, order_a].astype(np.float32)).to(device)).cpu().numpy()
    log_c, _ = pkg.calibrate_envelope(cal_logp, cal_lq, quantile=1.0, slack=1.5)
    val_bits, _, val_logp = cs.sample(16384, seed=3)
    val_lq = net.log_q(torch.as_tensor(val_bits[:, order_a].astype(np.float32)).to(device)).cpu().numpy()
    deficit = float(np.mean(np.maximum(0.0, 1.0 - np.exp(log_c - (val_logp - val_lq)))))
    viol_val = int(np.sum(val_logp - val_lq > log_c))
    # Envelopes calibrated the same way for the defensive mixture (1/2 network, 1/2
    # uniform) and for the uniform proposal alone: acceptance = 1 / c.
    log_c_mix, _ = pkg.calibrate_envelope(cal_logp, net.mixture_log_q(cal_lq, 0.5), quantile=1.0, slack=1.5)
    log_c_uni, _ = pkg.calibrate_envelope(cal_logp, np.full(len(cal_logp), -n * math.log(2.0)), quantile=1.0,
                                          slack=1.5)

    def propose(r):
        x, lq = net.sample(8192, seed=1000 + r)
        scan = x.to(torch.float32).cpu().numpy().astype(np.uint8)
        return scan[:, inv], lq.cpu().numpy()

    rng = np.random.default_rng(4)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    lbits, lp, lst = pkg.rejection_sample(so.probabilities, propose, log_c, samples, rng,
                                          recheck_fn=so128.probabilities)
    torch.cuda.synchronize(device)
    t_learned = time.perf_counter() - t0
    t0 = time.perf_counter()
    cbits, cp, clogp = cs.sample(samples, seed=5)
    torch.cuda.synchronize(device)
    t_chain = time.perf_counter() - t0
    t0 = time.perf_counter()
    recs, usum = pkg.capped_rejection(so, np.random.default_rng(314159), samples, cap=1.0, recheck=so128,
                                      batch=8192, max_proposals=1 << 22)
    torch.cuda.synchronize(device)
    t_uni = time.perf_counter() - t0
    learned, chain = samples / t_learned, samples / t_chain
    return {
        "workload": f"n=56 random degree<=3 graph, {order_policy} order", "rmax": plan.rmax,
        "sum_states": plan.sum_states, "samples": samples, "mlp": "MADE 2x512, bf16 tcgen05 GEMMs, fp32 accumulation",
        "training_samples": train_samples, "epochs": epochs,
        "learned": {"samples_per_s": learned, "acceptance": lst["acceptance"], "proposals": lst["proposals"],
                    "linear_xeb": lst["linear_xeb"], "fp64_rechecked": lst["fp64_rechecked"],
                    "fp64_flips": lst["fp64_flips"], "envelope_violations": lst["envelope_violations"]},
        "plain_chain_rule": {"samples_per_s": chain, "linear_xeb": float((2.0 ** n) * cp.mean() - 1)},
        "uniform_capped_reference_rule": {"samples_per_s": samples / t_uni, "acceptance": usum["acceptance_fraction"],
                                          "xeb": usum["xeb"], "born_exact": False},
        "learned_over_plain": learned / chain,
        "envelope": {"log_c": log_c, "validation_deficit_tv": deficit, "validation_violations": viol_val,
                     "validation_samples": 16384},
        "calibrated_acceptance": {"network": math.exp(-log_c), "mixture_half_uniform": math.exp(-log_c_mix),
                                  "uniform": math.exp(-log_c_uni)},
        "training": {"exact_sample_seconds": t_data, "train_seconds": t_train, "loss_first": losses[0],
                     "loss_last": float(np.mean(losses[-5:])), "entropy_floor": floor,
                     "kl_estimate": float(np.mean(losses[-5:]) - floor)}}


def run_wht(args, rank, world, local_rank):
    """Config 2's WHT variants on their own: FP32 butterflies vs 16 x 16 Hadamard blocks on
    the tensor cores over split-BF16 values, on a 2^m state (`--m`)."""
    import torch
    import __graft_entry__
    pkg = __graft_entry__.package()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peak = float(json.loads(peaks_path.read_text())["hbm_gbs"]) if peaks_path.exists() else 6650.0
    res = wht_precision_leg(pkg, device, peak, m=args.m)
    if rank == 0:
        best = res["fp32"]
        print(json.dumps({"metric": f"full WHT of a 2^{args.m} complex64 state (fp32 vs split-bf16 tensor cores)",
                          "value": best["achieved_GBps"], "unit": "GB/s", "n_gpus": 1, "steps": 1, "warmup": 1,
                          "ms_per_step": best["ms"], "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "c64", "data": "synthetic (Gaussian state)",
                          "config": {"workload": f"WHT on all {args.m} bits"}, "variants": res}), flush=True)


def run_gemm(args, rank, world, local_rank):
    """The proposal network's forward GEMM shape on the tcgen05 kernel: C[8192 x 512] =
    A[8192 x 512] B[512 x 512]^T in BF16 with FP32 accumulation (both operands K-major,
    TMA-loaded), 3 warm-up and 20 timed launches."""
    import ctypes
    import torch
    import __graft_entry__
    pkg = __graft_entry__.package()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    M, N, K = 8192, 512, 512
    a = torch.randn(M, K, device=device).to(torch.bfloat16)
    b = torch.randn(N, K, device=device).to(torch.bfloat16)
    c = torch.empty(M, N, device=device)
    lib = pkg._lib.lib()
    stream = torch.cuda.current_stream(device)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def launch():
        pkg._lib.check(lib.rgs_gemm_bf16(M, N, K, ptr(a), K, 0, ptr(b), K, 1, 1.0, None, 0, None, None, ptr(c),
                                         None, N, ctypes.c_void_p(stream.cuda_stream)))
    for _ in range(3):
        launch()
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(20):
        launch()
    e1.record(stream)
    torch.cuda.synchronize(device)
    t = e0.elapsed_time(e1) / 20 / 1e3
    ref = a[:256].float() @ b.float().T
    err = float((c[:256] - ref).abs().max())
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peak = float(json.loads(peaks_path.read_text())["bf16_tflops"]) if peaks_path.exists() else 1590.0
    tflops = 2 * M * N * K / t / 1e12
    if rank == 0:
        print(json.dumps({"metric": "tflops (tcgen05 bf16 GEMM, MADE forward shape 8192 x 512 x 512)",
                          "value": tflops, "unit": "TFLOP/s", "n_gpus": 1, "steps": 20, "warmup": 3,
                          "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "bf16 (fp32 accumulation)", "data": "synthetic (Gaussian operands)",
                          "config": {"workload": "C = A B^T, M=8192 N=512 K=512, TMA-loaded K-major operands"},
                          "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s",
                                       "frac": tflops / peak},
                          "max_abs_err_vs_torch_fp32": err}), flush=True)


def run_learned(args, rank, world, local_rank):
    """Learned proposal workload (config 4) at full size: 2^16 training samples, `--samples`
    accepted samples; `--order random` keeps the seeded random order (rank 25)."""
    import torch
    import __graft_entry__
    pkg = __graft_entry__.package()
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    res = learned_comparison(pkg, device, args.samples, 1 << 16, args.epochs, order_policy=args.order)
    if rank == 0:
        print(json.dumps({
            "metric": "exact_born_samples_per_s (learned proposal vs plain exact sampler, n=56 degree<=3)",
            "value": res["learned"]["samples_per_s"], "unit": "samples/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": 1e3 * args.samples / res["learned"]["samples_per_s"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 scan, bf16 MLP",
            "data": "synthetic (seeded graph, gates, samples)", "config": res}), flush=True)


def main():
    global BATCH
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--batch", type=int, default=BATCH, help="bitstrings per GPU per step (profiling runs)")
    ap.add_argument("--only", choices=["both", "c64", "c128"], default="both",
                    help="run only one precision (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other configurations' legs of the default line (profiling runs)")
    ap.add_argument("--workload", choices=["amplitudes", "fourier", "chain", "learned", "batched", "rgs70", "full",
                                           "wht", "gemm"], default="amplitudes")
    ap.add_argument("--samples", type=int, default=4096, help="learned: accepted samples; full: exact samples")
    ap.add_argument("--epochs", type=int, default=8, help="training epochs of the learned workload")
    ap.add_argument("--order", choices=["searched", "random"], default="searched",
                    help="scan order of the learned workload's n=56 instance")
    ap.add_argument("--m", type=int, default=30, help="conditional qubits of the fourier workload")
    ap.add_argument("--tma", action="store_true",
                    help="fourier workload: stage tiles with TMA loads in persistent blocks (default: thread loads)")
    ap.add_argument("--pass-kernel", choices=["registers", "rounds"], default="registers",
                    help="fourier workload: register-first pass kernel (default) or one shared-memory "
                         "round per four axes")
    ap.add_argument("--tile64", type=int, default=None, help="complex64 batch tile (default: autotuned)")
    ap.add_argument("--bulk", choices=["c64f32", "c64"], default="c64f32",
                    help="complex64 bulk arithmetic: float32 (default) or float64")
    ap.add_argument("--no-alt", action="store_true", help="skip timing the other complex64 recipe")
    ap.add_argument("--serial-sweeps", action="store_true",
                    help="run the complex64 bulk and the complex128 recheck one after the other")
    ap.add_argument("--tile128", type=int, default=None, help="complex128 batch tile (default: autotuned)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus if args.gpus == 1 else 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.warmup < 3:
        raise SystemExit("warmup must be >= 3")
    BATCH = args.batch
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "fourier":
        run_fourier(args, rank, world, local_rank)
    elif args.workload == "chain":
        run_chain(args, rank, world, local_rank)
    elif args.workload == "learned":
        run_learned(args, rank, world, local_rank)
    elif args.workload == "batched":
        run_batched(args, rank, world, local_rank)
    elif args.workload == "rgs70":
        run_rgs70(args, rank, world, local_rank)
    elif args.workload == "full":
        run_full(args, rank, world, local_rank)
    elif args.workload == "wht":
        run_wht(args, rank, world, local_rank)
    elif args.workload == "gemm":
        run_gemm(args, rank, world, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
