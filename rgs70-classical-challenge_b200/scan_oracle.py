"""Batched p(x) engine and the ``ScanOracle`` drop-in.

``ScanOracle`` keeps the constructor and attributes of ``W/scan_oracle.py:11-29``
(whyihaveyou/rgs70-classical-challenge, ``W/`` = ``work/rgs_attack/``):
``ScanOracle(g, u, order, source, device, gpu, fp64)`` with ``.amplitude(bits)``,
``.steps .ranks .rmax .fut .tables .combos`` and ``.engine._sweep(f, yfix)``.
It adds the batched calls ``.amplitudes(bits)`` / ``.probabilities(bits)`` that
run thousands of bitstrings per launch sequence.

PyTorch provides device memory and streams only; all computation is in
``librgs_b200.so``.  There is no CPU executor here: ``gpu=False`` raises.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from .plan import ScanPlan, edges_from_graph

__all__ = ["ScanEngine", "ScanOracle", "pack_bits", "PRECISIONS", "max_batch_tile", "capture_graph", "autotune_tile"]

PRECISIONS = {"c64": _lib.PREC_C64, "c64f32": _lib.PREC_C64_F32, "c128": _lib.PREC_C128}
LN2 = math.log(2.0)


def pack_bits(bits, n=None):
    """0/1 array [batch, n] (qubit q in column q) -> uint64 [batch, 2] (qubit q = bit q)."""
    b = np.asarray(bits)
    if b.ndim == 1:
        b = b[None, :]
    if n is not None and b.shape[1] != n:
        raise ValueError(f"bitstrings must have {n} entries")
    if b.size and (b.min() < 0 or b.max() > 1):
        raise ValueError("bits must be 0 or 1")
    if b.shape[1] > 128:
        raise ValueError("at most 128 qubits")
    padded = np.zeros((b.shape[0], 128), dtype=np.uint8)
    padded[:, :b.shape[1]] = b
    return np.ascontiguousarray(np.packbits(padded, axis=1, bitorder="little").view("<u8"))


def capture_graph(device, fn):
    """Capture ``fn(stream)`` -- queued library calls on ``stream`` -- into a CUDA graph;
    replay it with ``graph.replay()`` on the current stream.  Workspaces and outputs must
    already exist (a capture allocates nothing); run ``fn`` once eagerly first."""
    device = torch.device(device) if not isinstance(device, torch.device) else device
    g = torch.cuda.CUDAGraph()
    with torch.cuda.device(device):
        s = torch.cuda.Stream(device)
        s.wait_stream(torch.cuda.current_stream(device))
        with torch.cuda.stream(s):
            g.capture_begin()
            fn(s)
            g.capture_end()
        torch.cuda.current_stream(device).wait_stream(s)
    return g


def max_batch_tile(precision):
    """Largest batch tile the step kernel accepts for a precision name."""
    t = ctypes.c_int32()
    _lib.check(_lib.lib().rgs_scan_max_batch_tile(PRECISIONS[precision], ctypes.byref(t)))
    return int(t.value)


def _auto_tile(batch, rmax, esize, budget, cap):
    """Largest power-of-two tile <= cap and <= batch whose two tables fit the budget."""
    bt = 1
    while bt * 2 <= min(cap, max(1, batch)) and 2 * (bt * 2) * esize * (1 << rmax) <= budget:
        bt *= 2
    while bt > 1 and 2 * bt * esize * (1 << rmax) > budget:
        bt //= 2
    return bt


_TUNED = {}


def autotune_tile(engine, d_bits, candidates=None, sample=None, reps=2):
    """Batch tile of ``engine`` chosen by measurement: each candidate (powers of two up to
    the precision's maximum that fit the memory budget) sweeps the same sample of items
    ``reps`` times after one warm-up sweep; the tile with the highest items per second
    wins.  Results are cached per (plan rank profile, precision, device).  Returns
    (tile, {tile: items_per_second})."""
    plan = engine.plan
    key = (plan.n, tuple(plan.ranks), engine.precision, str(engine.device),
           torch.cuda.get_device_name(engine.device))
    if key in _TUNED:
        return _TUNED[key]
    cap = max_batch_tile(engine.precision)
    if candidates is None:
        candidates = [t for t in (8, 16, 32, 64, 128, 256, 512) if t <= cap]
    fits = [t for t in candidates if 2 * t * engine.esize * (1 << plan.rmax) <= engine.memory_budget]
    if not fits:
        fits = [1]
    count = int(d_bits.shape[0])
    sample = min(count, sample if sample is not None else 4 * max(fits))
    bits = d_bits[:sample]
    val, ls = engine.out_tensors(sample)
    s = torch.cuda.current_stream(engine.device)
    rates = {}
    for t in fits:
        engine.run_bits(bits, val, ls, stream=s, tile=t)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            engine.run_bits(bits, val, ls, stream=s, tile=t)
        e1.record(s)
        torch.cuda.synchronize(engine.device)
        rates[t] = sample * reps / (e0.elapsed_time(e1) / 1e3)
    best = max(rates, key=rates.get)
    engine._ws = None  # keep only the chosen tile's workspace
    engine.workspace(best)
    _TUNED[key] = (best, rates)
    return best, rates


class ScanEngine:
    """Executes one compiled plan on one GPU with a caller-visible torch workspace.
    ``batch_tile="tune"`` picks the tile by measurement (``autotune_tile``) at the first
    call with bitstrings."""

    def __init__(self, plan, u, device=0, precision="c64", batch_tile=None, memory_budget=None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        if not plan.executable:
            raise NotImplementedError(f"plan rank {plan.rmax} is too large to execute")
        _lib.lib()
        self.plan = plan
        self.precision = precision
        self.prec_code = PRECISIONS[precision]
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the engine runs on CUDA devices only")
        u = np.asarray(u, dtype=np.complex128)
        if u.shape != (plan.n, 2, 2):
            raise ValueError("u must have shape (n, 2, 2)")
        self.u = u
        self.esize = 16 if precision == "c128" else 8
        with torch.cuda.device(self.device):
            self.d_u = torch.from_numpy(u.view(np.float64).reshape(-1).copy()).to(self.device)
            free, _total = torch.cuda.mem_get_info(self.device)
        self.memory_budget = int(memory_budget if memory_budget is not None else min(0.45 * free, 96 * 2 ** 30))
        self.batch_tile = batch_tile
        self.tuning = None
        self._ws = None
        self._ws_tile = None

    # -------------------------------------------------------------- workspace
    def tile_for(self, batch):
        if self.batch_tile == "tune":
            raise ValueError("the tile is chosen at the first run_bits call (batch_tile='tune')")
        if self.batch_tile is not None:
            return int(self.batch_tile)
        return _auto_tile(batch, self.plan.rmax, self.esize, self.memory_budget, max_batch_tile(self.precision))

    def workspace_bytes(self, tile):
        nb = ctypes.c_size_t()
        _lib.check(_lib.lib().rgs_scan_workspace_bytes(self.plan.handle, int(tile), self.prec_code,
                                                       ctypes.byref(nb)))
        return int(nb.value)

    def launch_count(self, batch, tile=None):
        """Kernel launches of one sweep of ``batch`` items (with the workspace this engine
        allocates for ``tile``, default: the tile in use)."""
        tile = int(tile or self._ws_tile or self.tile_for(batch))
        ws = self._ws.numel() if self._ws is not None and self._ws_tile == tile else self.workspace_bytes(tile)
        out = ctypes.c_int64()
        _lib.check(_lib.lib().rgs_scan_launch_count(self.plan.handle, int(batch), tile, self.prec_code, ws,
                                                    ctypes.byref(out)))
        return int(out.value)

    def workspace(self, tile):
        need = self.workspace_bytes(tile)
        if self._ws is None or self._ws.numel() < need:
            self._ws = None
            with torch.cuda.device(self.device):
                self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        self._ws_tile = tile
        return self._ws

    def out_tensors(self, batch):
        vdt = torch.complex128 if self.precision == "c128" else torch.complex64
        return (torch.empty(batch, dtype=vdt, device=self.device),
                torch.empty(batch, dtype=torch.float64, device=self.device))

    # -------------------------------------------------------------- device-level calls
    def run_bits(self, d_bits, out_value, out_logscale, stream=None, tile=None):
        """Queue the sweep for device bits uint64 [B, 2] into device outputs (no sync)."""
        batch = int(d_bits.shape[0])
        if tile is None and self.batch_tile == "tune":
            self.tuning = autotune_tile(self, d_bits)
            self.batch_tile = self.tuning[0]
        tile = tile or self.tile_for(batch)
        ws = self.workspace(tile)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        _lib.check(_lib.lib().rgs_scan_amplitudes(
            self.plan.handle, ctypes.c_void_p(self.d_u.data_ptr()), ctypes.c_void_p(d_bits.data_ptr()), batch,
            self.prec_code, ctypes.c_void_p(out_value.data_ptr()), ctypes.c_void_p(out_logscale.data_ptr()),
            ctypes.c_void_p(ws.data_ptr()), ws.numel(), tile, ctypes.c_void_p(s.cuda_stream)))

    def run_fvec(self, d_fvec, out_value, out_logscale, stream=None, tile=None):
        """Queue the sweep for device contraction vectors complex128 [B, n, 2]."""
        batch = int(d_fvec.shape[0])
        tile = tile or self.tile_for(batch)
        ws = self.workspace(tile)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        _lib.check(_lib.lib().rgs_scan_contract(
            self.plan.handle, ctypes.c_void_p(d_fvec.data_ptr()), batch, self.prec_code,
            ctypes.c_void_p(out_value.data_ptr()), ctypes.c_void_p(out_logscale.data_ptr()),
            ctypes.c_void_p(ws.data_ptr()), ws.numel(), tile, ctypes.c_void_p(s.cuda_stream)))

    # -------------------------------------------------------------- host-level calls
    def sweep_bits(self, bits):
        """(value, logscale) arrays for host bitstrings [B, n] (copies in and out)."""
        packed = pack_bits(bits, self.plan.n)
        with torch.cuda.device(self.device):
            d_bits = torch.from_numpy(packed.view(np.int64)).to(self.device)
            val, ls = self.out_tensors(len(packed))
            self.run_bits(d_bits, val, ls)
            return val.cpu().numpy().astype(np.complex128), ls.cpu().numpy()

    def sweep_fvec(self, fvec):
        f = np.ascontiguousarray(np.asarray(fvec, dtype=np.complex128))
        if f.ndim != 3 or f.shape[1:] != (self.plan.n, 2):
            raise ValueError("fvec must have shape (batch, n, 2)")
        with torch.cuda.device(self.device):
            d_f = torch.from_numpy(f.view(np.float64)).to(self.device)
            val, ls = self.out_tensors(len(f))
            self.run_fvec(d_f, val, ls)
            return val.cpu().numpy().astype(np.complex128), ls.cpu().numpy()

    def _sweep(self, f, yfix=None):
        """The reference mixin contract (``gpu_kernel.py:125-170``): f maps vertex -> 2-vector.

        ``yfix`` is accepted for signature compatibility; fixed values follow from f
        exactly as the reference derives them (``scan_plan.py:205``)."""
        fv = np.zeros((1, self.plan.n, 2), dtype=np.complex128)
        for q in range(self.plan.n):
            fv[0, q] = np.asarray(f[q], dtype=np.complex128)
        val, ls = self.sweep_fvec(fv)
        return complex(val[0]), float(ls[0])


def amplitudes_from(values, logscale, n):
    """value * exp(logscale) * 2^{-n/2}, as ``ScanOracle.amplitude`` (``W/scan_oracle.py:29``)."""
    return np.asarray(values, dtype=np.complex128) * np.exp(np.asarray(logscale) - 0.5 * n * LN2)


class ScanOracle:
    """p(x) oracle for a graph state measured after per-qubit unitaries (``W/scan_oracle.py:11-29``).

    ``g``: uint8 [n, n] adjacency; ``u``: complex [n, 2, 2]; ``order``: vertex order.
    ``source`` is accepted for signature compatibility and ignored (the engine is
    this package).  ``fp64`` selects complex128 tables (the reference's FP64
    rescoring kernel); otherwise complex64 tables with float64 weights and sums.
    ``fuse=False`` runs every position as its own pass (no fused pairs).
    """

    def __init__(self, g, u, order, source=None, device=0, gpu=True, fp64=False, precision=None,
                 batch_tile=None, memory_budget=None, fuse=True):
        if not gpu:
            raise ValueError("this engine has no CPU executor; the CPU restatement is the test oracle")
        g = np.asarray(g)
        self.n = len(g)
        self.u = np.asarray(u)
        self.order = list(order)
        self.edges = edges_from_graph(g)
        self.plan = ScanPlan(self.n, self.edges, self.order, fuse=fuse)
        self.ranks = self.plan.ranks
        self.rmax = self.plan.rmax
        self.gpu = True
        prec = precision or ("c128" if fp64 else "c64")
        self.engine = ScanEngine(self.plan, self.u, device=device, precision=prec, batch_tile=batch_tile,
                                 memory_budget=memory_budget)

    @property
    def steps(self):
        return self.plan.steps

    @property
    def fut(self):
        return self.plan.fut

    @property
    def tables(self):
        return self.plan.tables

    @property
    def combos(self):
        return self.plan.combos

    def amplitude(self, bits):
        """<x| (x)U |G> for one bitstring (list of n ints, qubit 0 first)."""
        return complex(self.amplitudes(np.asarray(bits)[None, :])[0])

    def amplitudes(self, bits):
        """Amplitudes of a batch of bitstrings [B, n]; complex128 array."""
        val, ls = self.engine.sweep_bits(bits)
        amp = amplitudes_from(val, ls, self.n)
        if not np.all(np.isfinite(amp)):
            raise ArithmeticError("non-finite amplitude from the scan")
        return amp

    def probabilities(self, bits):
        """p(x) in this oracle's precision.  Complex64 results carry the storage rounding
        of the tables, which is relative to each table's maximum, not to the amplitude:
        for p(x) >= 0.01 * 2^-n the relative error stays below 1e-4, for smaller p it can
        exceed it; ``checked_probabilities`` states the error of every result."""
        return np.abs(self.amplitudes(bits)) ** 2

    def checked_probabilities(self, bits, tol=1e-4):
        """p(x) with its error against FP64 stated per result.

        Runs this oracle's precision (the bulk) and the complex128 scan (the recheck) on
        the same strings.  Returns ``(p, rel_err, fp64_used)``: ``rel_err[i]`` =
        |p_bulk - p_fp64| / p_fp64 of result i; ``p[i]`` is the bulk value where
        ``rel_err[i] <= tol`` and the FP64 value elsewhere (``fp64_used[i]`` True), so
        every returned probability is within ``tol`` of the FP64 scan."""
        p_bulk = self.probabilities(bits)
        if self.engine.precision == "c128":
            return p_bulk, np.zeros_like(p_bulk), np.zeros(len(p_bulk), dtype=bool)
        if getattr(self, "_fp64", None) is None:
            self._fp64 = ScanEngine(self.plan, self.u, device=self.engine.device, precision="c128")
        val, ls = self._fp64.sweep_bits(bits)
        p64 = np.abs(amplitudes_from(val, ls, self.n)) ** 2
        if not np.all(np.isfinite(p64)):
            raise ArithmeticError("non-finite probability from the complex128 recheck")
        with np.errstate(divide="ignore", invalid="ignore"):
            rel = np.where(p64 > 0, np.abs(p_bulk - p64) / p64, np.where(p_bulk == 0, 0.0, np.inf))
        use = rel > tol
        return np.where(use, p64, p_bulk), rel, use
