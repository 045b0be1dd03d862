"""Exact conditional Born sampler (Fourier cut) on one GPU, and its production driver.

``ConditionalSampler`` keeps the seam of the reference samplers
(whyihaveyou/rgs70-classical-challenge, ``W/`` = ``work/rgs_attack/``):
``klass(g, u, A, B, devices, chunk_mib=..., fusion_bits=...)`` with ``.compute(outB)
-> stages``, ``.draw(rng) -> (index, pa, norm)`` (exactly three ``rng.random()``
calls), ``.masses()``, ``.probability_at(i)``, ``.host()``, ``.sync()`` and
``.cp.__version__`` (``W/born_production.py:26-58``, ``W/distributed_sampler.py:59-162``,
``W/deferred_global_sampler.py:40-88``, ``W/specialized_deferred_sampler.py:204-238``).

Differences: the whole 2^m state lives on ONE device (m <= 34 on a B200);
``devices`` is accepted and only its first entry is used; ``chunk_mib``,
``fusion_bits``, ``lane_bits``, ``lookup_bits`` are accepted and ignored (the pass
structure is fixed by the kernels).  ``method="permute"`` runs the reference's base
pipeline (product init over b, WHT, index map, products) instead of the covariant one.
"""
import copy
import ctypes
import time
import types

import numpy as np
import torch

from . import _lib

__all__ = ["ConditionalSampler", "ShardedConditionalSampler", "shard_choice", "terminal_pick", "draw_across_shards",
           "draw_distributed", "fwht", "product", "block_mass", "produce", "DrawRecorder", "cut_tables"]


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _create(g, u, A, B, deferred):
    g = np.ascontiguousarray(np.asarray(g, dtype=np.uint8))
    u = np.ascontiguousarray(np.asarray(u, dtype=np.complex128))
    a = np.asarray(A, dtype=np.int32)
    b = np.asarray(B, dtype=np.int32)
    if len(a) != len(b):
        raise ValueError("balanced partition required")
    h = ctypes.c_void_p()
    _lib.check(_lib.lib().rgs_fourier_create(len(g), _lib.ptr(g, ctypes.c_uint8),
                                             _lib.ptr(u.view(np.float64), ctypes.c_double), len(a),
                                             _lib.ptr(a, ctypes.c_int32), _lib.ptr(b, ctypes.c_int32),
                                             1 if deferred else 0, ctypes.byref(h)))
    return h


def _tables(h, m):
    chunks = ctypes.c_int32()
    L = _lib.lib()
    _lib.check(L.rgs_fourier_tables(h, None, None, None, None, ctypes.byref(chunks)))
    c = chunks.value
    lz = np.zeros((c, 256, 2), np.uint64)
    la = np.zeros((c, 256, 2), np.uint64)
    lc = np.zeros((c, 256, 2), np.uint64)
    inv = np.zeros(m, np.uint64)
    _lib.check(L.rgs_fourier_tables(h, _lib.ptr(lz, ctypes.c_uint64), _lib.ptr(la, ctypes.c_uint64),
                                    _lib.ptr(lc, ctypes.c_uint64), _lib.ptr(inv, ctypes.c_uint64),
                                    ctypes.byref(chunks)))
    return {"lut_z": lz, "lut_a": la, "lut_cols": lc, "inv_rows": inv}


def cut_tables(g, u, A, B):
    """Host-only: the GF(2) lookup tables of the cut (A, B) (no GPU needed).  Raises
    ValueError when rank(G[B,A]) < |B| (the reference's uniform-B-marginal assert)."""
    h = _create(g, u, A, B, True)
    try:
        return _tables(h, len(A))
    finally:
        _lib.lib().rgs_fourier_destroy(h)


class ConditionalSampler:
    """Conditional state of A given a uniform x_B, and exact draws from it."""

    def __init__(self, g, u, A, B, devices=(0,), chunk_mib=None, fusion_bits=None, lane_bits=None,
                 lookup_bits=None, deferred=True, method="covariant", host_spill=None):
        g = np.ascontiguousarray(np.asarray(g, dtype=np.uint8))
        u = np.ascontiguousarray(np.asarray(u, dtype=np.complex128))
        self.g, self.u = g, u
        self.A, self.B = [int(a) for a in A], [int(b) for b in B]
        self.m = len(self.A)
        if len(self.B) != self.m:
            raise ValueError("balanced partition required")
        if method not in ("covariant", "permute"):
            raise ValueError("method must be 'covariant' or 'permute'")
        self.method = method
        self.devices = list(devices) if not isinstance(devices, int) else [devices]
        self.device = torch.device("cuda", self.devices[0])
        L = _lib.lib()
        h = _create(g, u, self.A, self.B, deferred)
        self._h = h
        self.deferred = bool(deferred)
        m32, spec, tb, npass = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        nt = ctypes.c_int64()
        _lib.check(L.rgs_fourier_info(h, ctypes.byref(m32), ctypes.byref(spec), ctypes.byref(tb), ctypes.byref(nt),
                                      ctypes.byref(npass)))
        self.specialized, self.tilebits, self.nmass, self.passes = bool(spec.value), tb.value, nt.value, npass.value
        self.n = 1 << self.m                      # elements of the (single-device) state
        self.ng = 1
        self.localbits = self.m
        ws = ctypes.c_size_t()
        _lib.check(L.rgs_fourier_workspace_bytes(h, ctypes.byref(ws)))
        need = (self.n * 8) * (2 if method == "permute" else 1) + ws.value + (64 << 20)
        with torch.cuda.device(self.device):
            free, _ = torch.cuda.mem_get_info(self.device)
            if free < need:
                raise MemoryError(f"GPU {self.devices[0]}: need {need}, free {free}")
            self.state = torch.empty(self.n, dtype=torch.complex64, device=self.device)
            self.scratch = torch.empty(self.n, dtype=torch.complex64, device=self.device) \
                if method == "permute" else None
            self.workspace = torch.empty(ws.value, dtype=torch.uint8, device=self.device)
        self.terminal_unitary = np.asarray(u[self.A[-1]], dtype=np.complex128)
        self.cp = types.SimpleNamespace(__version__=_lib.lib().rgs_version().decode())
        self._result = self.state

    # ------------------------------------------------------------------ helpers
    def _outmask(self, outB):
        bits = np.asarray(outB)
        if bits.shape != (self.m,) or np.any((bits != 0) & (bits != 1)):
            raise ValueError("outB must contain m bits")
        return int(sum(int(x) << j for j, x in enumerate(bits)))

    def sync(self):
        torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------------ reference seam
    def compute(self, outB):
        """Build the conditional state for B outcome ``outB``; returns stage times (s)."""
        mask = self._outmask(outB)
        L = _lib.lib()
        start = time.perf_counter()
        with torch.cuda.device(self.device):
            if self.method == "covariant":
                ms = (ctypes.c_float * 3)()
                _lib.check(L.rgs_fourier_compute(self._h, mask, ctypes.c_void_p(self.state.data_ptr()),
                                                 ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(),
                                                 _stream(self.device), ms))
                self._result = self.state
                return {"initialize_specialized_global" if self.specialized else "initialize_covariant": ms[0] / 1e3,
                        "walsh_fused": ms[1] / 1e3, "product_measurement_fused": ms[2] / 1e3,
                        "linear_permutation_phase": 0.0, "host_seconds": time.perf_counter() - start}
            _lib.check(L.rgs_fourier_compute_permute(self._h, mask, ctypes.c_void_p(self.state.data_ptr()),
                                                     ctypes.c_void_p(self.scratch.data_ptr()),
                                                     ctypes.c_void_p(self.workspace.data_ptr()),
                                                     self.workspace.numel(), _stream(self.device)))
            self._result = self.scratch
            self.sync()
            return {"permute_pipeline": time.perf_counter() - start}

    def tune(self):
        """Times one compute per pass-kernel launch variant on this GPU and keeps the
        faster for this sampler (overwrites the state).  Returns (variant, ms per variant)."""
        v = ctypes.c_int32()
        ms = (ctypes.c_float * 2)()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_fourier_tune(self._h, ctypes.c_void_p(self.state.data_ptr()),
                                                   ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(),
                                                   _stream(self.device), ctypes.byref(v), ms))
        self.variant = int(v.value)
        return self.variant, [float(ms[0]), float(ms[1])]

    def masses(self):
        """(tile masses float64, norm, tilebits, nmass); raises if |norm - 1| > 1e-3."""
        out = np.zeros(self.nmass, dtype=np.float64)
        norm = ctypes.c_double()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_fourier_masses(self._h, ctypes.c_void_p(self._result.data_ptr()),
                                                     ctypes.c_void_p(self.workspace.data_ptr()),
                                                     _lib.ptr(out, ctypes.c_double), ctypes.byref(norm),
                                                     _stream(self.device)))
        if not np.isfinite(norm.value) or abs(norm.value - 1) > 1e-3:
            raise ArithmeticError(f"Conditional norm check failed: {norm.value}")
        return out, norm.value, self.tilebits, self.nmass

    def draw(self, rng):
        """Exact draw: tile (u1), element (u2), terminal bit (u3) -- three rng.random() calls."""
        u1, u2, u3 = float(rng.random()), float(rng.random()), float(rng.random())
        idx, pa, norm = ctypes.c_uint64(), ctypes.c_double(), ctypes.c_double()
        with torch.cuda.device(self.device):
            if self.method == "permute":
                # The permute pipeline leaves masses of the result state in the workspace too.
                pass
            _lib.check(_lib.lib().rgs_fourier_draw(self._h, ctypes.c_void_p(self._result.data_ptr()),
                                                   ctypes.c_void_p(self.workspace.data_ptr()), u1, u2, u3,
                                                   ctypes.byref(idx), ctypes.byref(pa), ctypes.byref(norm),
                                                   _stream(self.device)))
        return int(idx.value), float(pa.value), float(norm.value)

    def transformed_pair(self, local_index):
        """U_last @ (v[local], v[local + 2^{m-1}]) (``deferred_global_sampler.py:65-70``)."""
        half = self.n // 2
        if not 0 <= local_index < half:
            raise ValueError("Local index outside shard")
        raw = np.array([complex(self._result[local_index].item()), complex(self._result[local_index + half].item())])
        return self.terminal_unitary @ raw

    def probability_at(self, index):
        if not 0 <= index < self.n:
            raise ValueError("Bad index")
        if not self.deferred:
            return float(abs(complex(self._result[index].item())) ** 2)
        half = self.n // 2
        return float(abs(self.transformed_pair(index % half)[index // half]) ** 2)

    def host(self):
        """Normalised conditional state (complex128), terminal unitary applied."""
        raw = self._result.cpu().numpy().astype(np.complex128)
        if self.deferred:
            view = raw.reshape(2, -1)
            a, b = view[0].copy(), view[1].copy()
            U = self.terminal_unitary
            view[0] = U[0, 0] * a + U[0, 1] * b
            view[1] = U[1, 0] * a + U[1, 1] * b
        return raw

    def tables(self):
        """GF(2) lookup tables (covariant map, q_A phase, index map) and the rows of N."""
        return _tables(self._h, self.m)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().rgs_fourier_destroy(h)
            except Exception:
                pass
            self._h = None


# ---------------------------------------------------------------------- two shards
def shard_choice(totals, u1):
    """First level of a draw over shards laid end to end: the shard holding the point
    u1 * sum(totals) of the cumulative mass, and the uniform rescaled to that shard's own
    mass (the reference draws one tile index over the concatenated masses of both
    devices, ``distributed_sampler.py:153-157``).  Returns (shard, u1 within it, norm)."""
    totals = [float(t) for t in totals]
    norm = sum(totals)
    if not (norm > 0.0) or not np.isfinite(norm):
        raise ArithmeticError(f"invalid shard masses {totals}")
    target = u1 * norm
    acc = 0.0
    last = max(i for i, t in enumerate(totals) if t > 0.0)
    for i, t in enumerate(totals):
        if t > 0.0 and (target < acc + t or i == last):
            return i, min(max((target - acc) / t, 0.0), np.nextafter(1.0, 0.0)), norm
        acc += t
    raise AssertionError("unreachable")


def terminal_pick(pair, unitary, u3):
    """The deferred terminal unitary on the two values at one local index (one per shard)
    and the output bit (``deferred_global_sampler.py:65-78``): (bit, |(U pair)_bit|^2)."""
    out = np.asarray(unitary, dtype=np.complex128) @ np.asarray(pair, dtype=np.complex128)
    p = np.abs(out) ** 2
    total = float(p.sum())
    if not (total > 0.0) or not np.isfinite(total):
        raise ArithmeticError("Invalid transformed local mass")
    bit = int(u3 * total >= p[0])
    return bit, float(p[bit])


def draw_across_shards(shards, unitary, u1, u2, u3):
    """One exact draw from two shards held in this process (objects with ``mass()``,
    ``local_draw(u1, u2)``, ``value(local)`` and ``half``): shard by mass, local index by
    the shard's two-level inverse CDF, bit by the terminal pair.  Returns (index, pa, norm)."""
    s, u1s, norm = shard_choice([sh.mass() for sh in shards], u1)
    local = shards[s].local_draw(u1s, u2)
    bit, pa = terminal_pick([sh.value(local) for sh in shards], unitary, u3)
    return bit * shards[0].half + local, pa, norm


def draw_distributed(shard, unitary, rng, rank, group=None, device=None):
    """The same draw with one shard per process (rank = shard index, two ranks): rank 0
    draws the three uniforms (the reference's RNG call order) and broadcasts them; the two
    shard masses, the chosen local index and the two terminal values are the only data
    exchanged (collectives on `device` tensors: CPU for gloo, CUDA for NCCL).
    Returns (index, pa, norm) on every rank."""
    import torch.distributed as dist
    dev = device if device is not None else torch.device("cpu")
    u = torch.zeros(3, dtype=torch.float64, device=dev)
    if rank == 0:
        u[:] = torch.tensor([float(rng.random()), float(rng.random()), float(rng.random())], dtype=torch.float64)
    dist.broadcast(u, src=0, group=group)
    u1, u2, u3 = (float(x) for x in u.cpu())
    masses = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(2)]
    dist.all_gather(masses, torch.tensor([shard.mass()], dtype=torch.float64, device=dev), group=group)
    s, u1s, norm = shard_choice([float(m.item()) for m in masses], u1)
    loc = torch.zeros(1, dtype=torch.int64, device=dev)
    if rank == s:
        loc[0] = int(shard.local_draw(u1s, u2))
    dist.broadcast(loc, src=s, group=group)
    local = int(loc.item())
    v = shard.value(local)
    vals = [torch.zeros(2, dtype=torch.float64, device=dev) for _ in range(2)]
    dist.all_gather(vals, torch.tensor([v.real, v.imag], dtype=torch.float64, device=dev), group=group)
    pair = [complex(float(t[0]), float(t[1])) for t in vals]
    bit, pa = terminal_pick(pair, unitary, u3)
    return bit * shard.half + local, pa, norm


class ShardedConditionalSampler:
    """One of two shards of the conditional state on this device: the values whose top A
    bit equals ``shard`` (2^(m-1) complex64), the deferred terminal unitary not applied
    (``DeferredGlobalMixin``, ``W/deferred_global_sampler.py:40-88``).  The top bit's Walsh
    factor is folded into the initialisation, so computing a shard needs no data from the
    other one; a draw exchanges two scalars per shard (``draw_distributed``), or runs on
    two shards of one process (``draw_across_shards``).  m >= 13."""

    def __init__(self, g, u, A, B, shard, device=0):
        g = np.ascontiguousarray(np.asarray(g, dtype=np.uint8))
        u = np.ascontiguousarray(np.asarray(u, dtype=np.complex128))
        self.A, self.B = [int(a) for a in A], [int(b) for b in B]
        self.m = len(self.A)
        if shard not in (0, 1):
            raise ValueError("shard must be 0 or 1")
        self.shard = shard
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        self._h = _create(g, u, self.A, self.B, True)
        self.half = 1 << (self.m - 1)
        ws = ctypes.c_size_t()
        _lib.check(_lib.lib().rgs_fourier_workspace_bytes(self._h, ctypes.byref(ws)))
        with torch.cuda.device(self.device):
            self.state = torch.empty(self.half, dtype=torch.complex64, device=self.device)
            self.workspace = torch.empty(ws.value, dtype=torch.uint8, device=self.device)
        self.terminal_unitary = np.asarray(u[self.A[-1]], dtype=np.complex128)

    def compute(self, outB):
        bits = np.asarray(outB)
        if bits.shape != (self.m,) or np.any((bits != 0) & (bits != 1)):
            raise ValueError("outB must contain m bits")
        mask = int(sum(int(x) << j for j, x in enumerate(bits)))
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_fourier_compute_shard(
                self._h, mask, self.shard, ctypes.c_void_p(self.state.data_ptr()),
                ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(), _stream(self.device)))

    def mass(self):
        out = ctypes.c_double()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_fourier_shard_mass(self._h, ctypes.c_void_p(self.workspace.data_ptr()),
                                                         ctypes.byref(out), _stream(self.device)))
        return float(out.value)

    def local_draw(self, u1, u2):
        idx = ctypes.c_uint64()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_fourier_shard_draw(self._h, ctypes.c_void_p(self.state.data_ptr()),
                                                         ctypes.c_void_p(self.workspace.data_ptr()), float(u1),
                                                         float(u2), ctypes.byref(idx), _stream(self.device)))
        return int(idx.value)

    def value(self, local):
        return complex(self.state[int(local)].item())

    def host(self):
        return self.state.cpu().numpy().astype(np.complex128)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().rgs_fourier_destroy(h)
            except Exception:
                pass
            self._h = None


# ---------------------------------------------------------------------- building blocks
def _state(state):
    """The kernels address raw memory: the state must be a contiguous complex64 CUDA tensor."""
    if state.dtype != torch.complex64 or not state.is_cuda or not state.is_contiguous() or state.dim() != 1:
        raise ValueError("state must be a contiguous 1-D complex64 CUDA tensor")
    if state.numel() & (state.numel() - 1):
        raise ValueError("state length must be a power of two")
    return state


WHT_PRECISIONS = {"fp32": 0, "split_bf16x2": 2, "split_bf16x3": 3}


def fwht(state, lo=0, hi=None, precision="fp32"):
    """In-place Walsh-Hadamard butterflies (x + y, x - y) on bits [lo, hi) of a complex64
    CUDA tensor.  ``precision``: "fp32" (FP32 butterflies), or 16 x 16 Hadamard blocks on the
    tensor cores over a split-BF16 copy of every value, "split_bf16x2" (two BF16 terms,
    about 4e-6 relative error per 4-bit round) or "split_bf16x3" (three terms, FP32 level);
    the tensor-core variants need at least 2^12 values."""
    _state(state)
    if precision not in WHT_PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(WHT_PRECISIONS)}")
    nbits = int(state.numel()).bit_length() - 1
    hi = nbits if hi is None else hi
    with torch.cuda.device(state.device):
        _lib.check(_lib.lib().rgs_fwht_precision(ctypes.c_void_p(state.data_ptr()), nbits, lo, hi,
                                                 WHT_PRECISIONS[precision], _stream(state.device)))


def product(state, unitaries, lo=0, hi=None):
    """In-place per-qubit 2x2 products (unitaries: complex [nbits, 2, 2]) on bits [lo, hi)."""
    _state(state)
    nbits = int(state.numel()).bit_length() - 1
    hi = nbits if hi is None else hi
    u = torch.from_numpy(np.ascontiguousarray(np.asarray(unitaries, np.complex128)).view(np.float64).reshape(-1))
    u = u.to(state.device)
    with torch.cuda.device(state.device):
        _lib.check(_lib.lib().rgs_product(ctypes.c_void_p(state.data_ptr()), nbits, ctypes.c_void_p(u.data_ptr()),
                                          lo, hi, _stream(state.device)))
        torch.cuda.current_stream(state.device).synchronize()


def block_mass(state, tile_bits):
    """Per-tile sum of |state|^2 (float64 CUDA tensor)."""
    _state(state)
    nbits = int(state.numel()).bit_length() - 1
    out = torch.empty(1 << (nbits - tile_bits), dtype=torch.float64, device=state.device)
    with torch.cuda.device(state.device):
        _lib.check(_lib.lib().rgs_block_mass(ctypes.c_void_p(state.data_ptr()), nbits, tile_bits,
                                             ctypes.c_void_p(out.data_ptr()), _stream(state.device)))
    return out


# ---------------------------------------------------------------------- production driver
class DrawRecorder:
    """Records the uniforms a draw consumes (``W/born_production.py:11-14``)."""

    def __init__(self, rng):
        self.rng = rng
        self.uniforms = []

    def random(self):
        v = float(self.rng.random())
        self.uniforms.append(v)
        return v


def _decimal_state(state):
    s = copy.deepcopy(state)
    for k in ("state", "inc"):
        s["state"][k] = str(s["state"][k])
    return s


def produce(sampler, rng, count, n_qubits):
    """Fixed-count exact samples with the reference's RNG schedule: |B| integers for
    x_B, then exactly three uniforms per draw (``W/born_production.py:44-58``).
    Returns the list of records."""
    records = []
    A, B = sampler.A, sampler.B
    for i in range(count):
        before = _decimal_state(rng.bit_generator.state)
        start = time.perf_counter()
        bbits = rng.integers(0, 2, len(B)).tolist()
        stages = sampler.compute(bbits)
        rec = DrawRecorder(rng)
        index, pa, norm = sampler.draw(rec)
        if len(rec.uniforms) != 3:
            raise AssertionError("RNG call schedule changed")
        if not (0 <= index < (1 << len(A)) and np.isfinite(pa) and pa > 0 and abs(norm - 1) < 1e-3):
            raise ArithmeticError("Invalid production result")
        bits = [0] * n_qubits
        for j, q in enumerate(A):
            bits[q] = (index >> j) & 1
        for j, q in enumerate(B):
            bits[q] = bbits[j]
        records.append(dict(sample=i, bitstring_q0_left="".join(map(str, bits)), B_bits=bbits, A_index=index,
                            rngstate_before=before, rngstate_after=_decimal_state(rng.bit_generator.state),
                            draw_uniforms=rec.uniforms, probability_raw=pa * 2.0 ** (-len(B)),
                            probability=pa / norm * 2.0 ** (-len(B)), conditional_norm=norm,
                            elapsed_seconds=time.perf_counter() - start, stages=stages))
    return records
