"""Exact Born sampling and conditional marginals through the scan (chain rule).

``ChainSampler(g, u, order)`` draws exact samples of p(x) = |<x| (x)U |G>|^2 for any
graph and scan order: position by position, both branches of the next vertex are
contracted from one read of the environment table, x_v is drawn from
p(x_v | prefix) = M_x / (M_0 + M_1), and the chosen branch is one scan step
(``librgs_b200.so``, ``rgs_chain_sample`` / ``rgs_chain_marginals``).  Each sample comes
with its amplitude (as ``ScanOracle.amplitudes``) and log p(x).

This extends the reference's p(x) path (``W/scan_oracle.py``, ``W/upstream_scan/
gpu_kernel.py`` of whyihaveyou/rgs70-classical-challenge) from probabilities to
sampling; the reference's own exact sampler needs a full-rank balanced cut
(``ConditionalSampler`` here) and 2^{n/2} memory.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .plan import ScanPlan, edges_from_graph
from .scan_oracle import PRECISIONS, amplitudes_from, pack_bits

__all__ = ["ChainSampler", "unpack_bits"]


def unpack_bits(words, n):
    """uint64 [count, 2] -> uint8 [count, n] (qubit q = bit q)."""
    w = np.ascontiguousarray(np.asarray(words).astype(np.uint64))
    b = np.unpackbits(w.view(np.uint8).reshape(len(w), 16), axis=1, bitorder="little")
    return b[:, :n].astype(np.uint8)


class ChainSampler:
    """Exact sampler and conditional-marginal oracle for one (graph, gates, order)."""

    def __init__(self, g, u, order, device=0, precision="c64", batch_tile=None, plan=None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        g = np.asarray(g)
        self.n = len(g)
        self.order = list(order)
        self.plan = plan if plan is not None else ScanPlan(self.n, edges_from_graph(g), self.order)
        if not self.plan.executable:
            raise NotImplementedError(f"plan rank {self.plan.rmax} is too large to execute")
        self.u = np.asarray(u, dtype=np.complex128)
        self.precision = precision
        self.prec_code = PRECISIONS[precision]
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        esize = 16 if precision == "c128" else 8
        cap = 64 if precision == "c128" else 128
        if batch_tile is None:
            with torch.cuda.device(self.device):
                free, _ = torch.cuda.mem_get_info(self.device)
            budget = min(0.45 * free, 96 * 2 ** 30)
            batch_tile = 1
            while batch_tile * 2 <= cap and 2 * batch_tile * 2 * esize * (1 << self.plan.rmax) <= budget:
                batch_tile *= 2
        self.batch_tile = int(batch_tile)
        nb = ctypes.c_size_t()
        _lib.check(_lib.lib().rgs_chain_workspace_bytes(self.plan.handle, self.batch_tile, self.prec_code,
                                                        ctypes.byref(nb)))
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(nb.value, dtype=torch.uint8, device=self.device)
            self.d_u = torch.from_numpy(self.u.view(np.float64).reshape(-1).copy()).to(self.device)

    def _outs(self, count):
        vdt = torch.complex128 if self.precision == "c128" else torch.complex64
        return (torch.empty(count, dtype=vdt, device=self.device),
                torch.empty(count, dtype=torch.float64, device=self.device),
                torch.empty(count, dtype=torch.float64, device=self.device))

    def launch_count(self, count, marginals=False, with_logp=True):
        """Kernel launches of one sampling (or marginals) call of ``count`` strings."""
        n = ctypes.c_int64()
        _lib.check(_lib.lib().rgs_chain_launch_count(self.plan.handle, int(count), self.batch_tile,
                                                     1 if marginals else 0, 1 if with_logp else 0, ctypes.byref(n)))
        return int(n.value)

    def sample_device(self, count, seed=0, uniforms=None, check=True, stream=None, outs=None, cond=None):
        """Queue ``count`` samples; returns device tensors (bits, value, logscale, logp).
        ``cond``: optional float32 [count, n] device tensor for the conditionals met."""
        bits = torch.empty((count, 2), dtype=torch.int64, device=self.device)
        value, logscale, logp = outs if outs is not None else self._outs(count)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        uptr = None
        if uniforms is not None:
            uniforms = torch.as_tensor(np.ascontiguousarray(uniforms, dtype=np.float64)).to(self.device)
            if tuple(uniforms.shape) != (count, self.n):
                raise ValueError("uniforms must have shape (count, n)")
            uptr = ctypes.c_void_p(uniforms.data_ptr())
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_chain_sample(
                self.plan.handle, ctypes.c_void_p(self.d_u.data_ptr()), count, int(seed) & (2 ** 64 - 1), uptr,
                self.prec_code, ctypes.c_void_p(bits.data_ptr()), ctypes.c_void_p(value.data_ptr()),
                ctypes.c_void_p(logscale.data_ptr()), ctypes.c_void_p(logp.data_ptr()),
                ctypes.c_void_p(cond.data_ptr()) if cond is not None else None,
                ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(), self.batch_tile,
                1 if check else 0, ctypes.c_void_p(s.cuda_stream)))
        return bits, value, logscale, logp

    def sample(self, count, seed=0, uniforms=None, with_conditionals=False):
        """(bits uint8 [count, n], p(x) float64 [count], log p(x) from the conditionals),
        plus the conditionals p(x_{v_j} = 1 | prefix) [count, n] (scan order) if asked."""
        cond = torch.empty((count, self.n), dtype=torch.float32, device=self.device) if with_conditionals else None
        bits, value, logscale, logp = self.sample_device(count, seed, uniforms, cond=cond)
        b = unpack_bits(bits.cpu().numpy(), self.n)
        amp = amplitudes_from(value.cpu().numpy().astype(np.complex128), logscale.cpu().numpy(), self.n)
        out = (b, np.abs(amp) ** 2, logp.cpu().numpy())
        return out + (cond.cpu().numpy(),) if with_conditionals else out

    def marginals(self, bits):
        """Conditionals p(x_{v_j} = 1 | x_{v_<j}) [count, n] (scan order), log p(x), p(x)."""
        packed = pack_bits(bits, self.n)
        count = len(packed)
        with torch.cuda.device(self.device):
            d_bits = torch.from_numpy(packed.view(np.int64)).to(self.device)
            cond = torch.empty((count, self.n), dtype=torch.float32, device=self.device)
            value, logscale, logp = self._outs(count)
            _lib.check(_lib.lib().rgs_chain_marginals(
                self.plan.handle, ctypes.c_void_p(self.d_u.data_ptr()), ctypes.c_void_p(d_bits.data_ptr()), count,
                self.prec_code, ctypes.c_void_p(cond.data_ptr()), ctypes.c_void_p(logp.data_ptr()),
                ctypes.c_void_p(value.data_ptr()), ctypes.c_void_p(logscale.data_ptr()),
                ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(), self.batch_tile, 1,
                ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))
            amp = amplitudes_from(value.cpu().numpy().astype(np.complex128), logscale.cpu().numpy(), self.n)
            return cond.cpu().numpy(), logp.cpu().numpy(), np.abs(amp) ** 2
