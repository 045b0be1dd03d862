"""Many small instances in one persistent launch (``rgs_batch_*`` in ``librgs_b200.so``).

``ResidentBatch`` gathers (graph, gates, order) instances of rank at most
``max_rank(precision)`` -- amplitudes of given bitstrings and exact chain-rule
samples of each -- and runs all of them with one kernel whose blocks hold an
instance's whole environment table in shared memory.  Amplitudes equal
``ScanOracle.amplitudes`` bit for bit; samples are those of
``ChainSampler.sample(seed=...)`` (same Philox uniforms), up to decisions whose
uniform falls within rounding of a branch boundary.

This is the batched form of the reference's per-instance loop over
``ScanOracle.amplitude`` (``W/scan_oracle.py:19-28`` of
whyihaveyou/rgs70-classical-challenge).  ``run()`` is two stream operations once
prepared, so it can be captured in a CUDA graph (``capture()``).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .chain import unpack_bits
from .plan import ScanPlan, edges_from_graph
from .scan_oracle import PRECISIONS, amplitudes_from, pack_bits

__all__ = ["ResidentBatch", "max_rank"]


def max_rank(precision="c64"):
    """Largest plan rank the resident executor holds in shared memory."""
    r = ctypes.c_int32()
    _lib.check(_lib.lib().rgs_batch_max_rank(PRECISIONS[precision], ctypes.byref(r)))
    return int(r.value)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class _Entry:
    def __init__(self, plan, n, u, bits, count, nsamples, seed, outs):
        self.plan, self.n, self.u, self.bits, self.count, self.nsamples, self.seed = \
            plan, n, u, bits, count, nsamples, seed
        (self.value, self.logscale, self.sbits, self.svalue, self.slogscale, self.slogp) = outs


class ResidentBatch:
    """A batch of instances on one device; outputs are torch tensors kept by the batch."""

    def __init__(self, precision="c64", device=0):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.precision = precision
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().rgs_batch_create(PRECISIONS[precision], ctypes.byref(h)))
        self._h = h
        self.entries = []
        self._graph = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().rgs_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def add(self, g=None, u=None, order=None, bits=None, nsamples=0, seed=0, plan=None):
        """Adds one instance; returns its index.  ``bits``: 0/1 array [count, n] or None."""
        if plan is None:
            g = np.asarray(g)
            plan = ScanPlan(len(g), edges_from_graph(g), list(order))
        n = plan.n
        u = np.asarray(u, dtype=np.complex128)
        if u.shape != (n, 2, 2):
            raise ValueError("u must have shape (n, 2, 2)")
        d = self.device
        vdt = torch.complex128 if self.precision == "c128" else torch.complex64
        with torch.cuda.device(d):
            du = torch.from_numpy(u.view(np.float64).reshape(-1).copy()).to(d)
            count = 0
            dbits = value = logscale = None
            if bits is not None:
                packed = pack_bits(bits, n)
                count = len(packed)
                dbits = torch.from_numpy(packed.view(np.int64)).to(d)
                value = torch.empty(count, dtype=vdt, device=d)
                logscale = torch.empty(count, dtype=torch.float64, device=d)
            nsamples = int(nsamples)
            sbits = svalue = slogscale = slogp = None
            if nsamples:
                sbits = torch.empty((nsamples, 2), dtype=torch.int64, device=d)
                svalue = torch.empty(nsamples, dtype=vdt, device=d)
                slogscale = torch.empty(nsamples, dtype=torch.float64, device=d)
                slogp = torch.empty(nsamples, dtype=torch.float64, device=d)
        return self.add_device(plan, du, dbits, value, logscale, nsamples, seed, sbits, svalue, slogscale, slogp)

    def add_device(self, plan, du, dbits=None, value=None, logscale=None, nsamples=0, seed=0, sbits=None,
                   svalue=None, slogscale=None, slogp=None):
        """Adds one instance over caller-owned contiguous device tensors (views of larger
        buffers allowed): du float64 [n*8] gates, dbits int64 [count, 2], value/logscale
        [count], sbits int64 [nsamples, 2], svalue/slogscale/slogp [nsamples]."""
        for t in (du, dbits, value, logscale, sbits, svalue, slogscale, slogp):
            if t is not None and (not t.is_cuda or not t.is_contiguous()):
                raise ValueError("batch buffers must be contiguous CUDA tensors")
        count = int(dbits.shape[0]) if dbits is not None else 0
        nsamples = int(nsamples)
        idx = ctypes.c_int32()
        _lib.check(_lib.lib().rgs_batch_add(
            self._h, plan.handle, _p(du), _p(dbits) if count else None, count, _p(value) if count else None,
            _p(logscale) if count else None, nsamples, int(seed) & (2 ** 64 - 1), _p(sbits) if nsamples else None,
            _p(svalue) if nsamples else None, _p(slogscale) if nsamples else None,
            _p(slogp) if nsamples else None, ctypes.byref(idx)))
        self.entries.append(_Entry(plan, plan.n, du, dbits, count, nsamples, seed,
                                   (value, logscale, sbits, svalue, slogscale, slogp)))
        self._graph = None
        return int(idx.value)

    @property
    def units(self):
        k, w = ctypes.c_int32(), ctypes.c_int64()
        _lib.check(_lib.lib().rgs_batch_info(self._h, ctypes.byref(k), ctypes.byref(w)))
        return int(w.value)

    def run(self, check=True, stream=None):
        """Queues every instance's work as one launch (``check`` synchronises)."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_batch_run(self._h, 1 if check else 0, ctypes.c_void_p(s.cuda_stream)))

    def tune(self, stream=None):
        """Runs the batch with each launch variant and keeps the faster (outputs are
        written).  Returns (variant, milliseconds per run of each variant)."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        v = ctypes.c_int32()
        ms = (ctypes.c_float * 3)()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_batch_tune(self._h, ctypes.c_void_p(s.cuda_stream), ctypes.byref(v), ms))
        self._graph = None
        return int(v.value), [float(x) for x in ms]

    def capture(self):
        """Captures ``run()`` into a CUDA graph (after a first, preparing run); returns it."""
        self.run(check=True)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.device(self.device):
            s = torch.cuda.Stream(self.device)
            with torch.cuda.stream(s):
                g.capture_begin()
                self.run(check=False, stream=s)
                g.capture_end()
        torch.cuda.synchronize(self.device)
        self._graph = g
        return g

    def replay(self):
        if self._graph is None:
            self.capture()
        self._graph.replay()

    # ------------------------------------------------------------------ results
    def amplitudes(self, i):
        """(value, logscale) as ``ScanEngine.sweep_bits`` returns them, and the amplitudes."""
        e = self.entries[i]
        if not e.count:
            return np.zeros(0), np.zeros(0), np.zeros(0, dtype=np.complex128)
        val = e.value.cpu().numpy().astype(np.complex128)
        ls = e.logscale.cpu().numpy()
        return val, ls, amplitudes_from(val, ls, e.n)

    def samples(self, i):
        """(bits uint8 [nsamples, n], p(x), log p(x) from the conditionals)."""
        e = self.entries[i]
        bits = unpack_bits(e.sbits.cpu().numpy(), e.n)
        amp = amplitudes_from(e.svalue.cpu().numpy().astype(np.complex128), e.slogscale.cpu().numpy(), e.n)
        return bits, np.abs(amp) ** 2, e.slogp.cpu().numpy()
