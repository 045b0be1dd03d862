"""The reference's own GPU scan kernels, run on this box (test and baseline
infrastructure; the package never imports this).

``oracle/build_ref_gpu.py`` compiles the reference's K2 (complex64 tables, float64
weights and sums) and K3 (complex128) kernel sources into ``oracle/_ref/``; this module
drives them the way the reference's ``GPUMixin._sweep`` does
(work/rgs_attack/upstream_scan/gpu_kernel.py:125-170): one string at a time, one launch
per scan position, a host read of the table maximum after every launch.  Plans, byte
tables and kernel combos come from the oracle's restatement of the reference compiler
(bit-exact with it), so the kernel sees exactly the reference's inputs.
"""
import ctypes
import math
from pathlib import Path

import numpy as np

from . import scan_plan as sp

REF_DIR = Path(__file__).resolve().parent / "_ref"


def available(precision="c64"):
    return (REF_DIR / f"libref_scan_{precision}.so").exists()


class RefGpuScan:
    """p(x) of one (graph, gates, order) through the reference kernel of one precision."""

    def __init__(self, g, u, order, precision="c64", device=0):
        import torch

        self.lib = ctypes.CDLL(str(REF_DIR / f"libref_scan_{precision}.so"))
        self.lib.ref_sweep.restype = ctypes.c_int
        g = np.asarray(g)
        self.n = len(g)
        self.u = np.asarray(u, dtype=np.complex128)
        edges = [(i, j) for i in range(self.n) for j in range(i + 1, self.n) if g[i][j]]
        self.steps, self.ranks = sp.make_plan(self.n, edges, list(order))
        if any(not st.free for st in self.steps):
            raise ValueError("the reference-kernel driver supports free vertices only")
        self.rmax = max(self.ranks)
        tables = [sp.byte_tables(st.Lcols, st.r_out) for st in self.steps]
        combos = [np.array(sp.kernel_combos(st.kernel), dtype=np.uint64) for st in self.steps]
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        self.r_in = i32([st.r_in for st in self.steps])
        self.r_out = i32([st.r_out for st in self.steps])
        self.nbytes = i32([t.shape[0] for t in tables])
        self.ncombos = i32([len(c) for c in combos])
        self.beta = np.ascontiguousarray([st.beta for st in self.steps], dtype=np.uint64)
        self.table_off = np.ascontiguousarray(np.cumsum([0] + [t.size for t in tables[:-1]]), dtype=np.int64)
        self.combo_off = np.ascontiguousarray(np.cumsum([0] + [c.size for c in combos[:-1]]), dtype=np.int64)
        self.device = torch.device("cuda", device)
        esize = 16 if precision == "c128" else 8
        with torch.cuda.device(self.device):
            self.d_tables = torch.from_numpy(np.concatenate([t.reshape(-1) for t in tables]).view(np.int64)).to(
                self.device)
            self.d_combos = torch.from_numpy(np.concatenate(combos).view(np.int64)).to(self.device)
            self.bufs = [torch.empty((1 << self.rmax) * esize, dtype=torch.uint8, device=self.device)
                         for _ in range(2)]
            self.d_max = torch.zeros(1, dtype=torch.int64, device=self.device)
            self.grid = 32 * torch.cuda.get_device_properties(self.device).multi_processor_count

    def sweep(self, bits):
        """(value, logscale) of one bitstring, as GPUMixin._sweep returns them."""
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        f = np.empty((self.n, 4))
        for j, st in enumerate(self.steps):
            row = self.u[st.v][int(bits[st.v])]
            f[j] = (row[0].real, row[0].imag, row[1].real, row[1].imag)
        f = np.ascontiguousarray(f)
        value = np.zeros(2)
        logscale = ctypes.c_double()
        rc = self.lib.ref_sweep(
            ctypes.c_int(self.n), p(self.r_in), p(self.r_out), p(self.nbytes), p(self.ncombos), p(self.beta),
            p(self.table_off), p(self.combo_off), ctypes.c_void_p(self.d_tables.data_ptr()),
            ctypes.c_void_p(self.d_combos.data_ptr()), ctypes.c_void_p(self.bufs[0].data_ptr()),
            ctypes.c_void_p(self.bufs[1].data_ptr()), ctypes.c_void_p(self.d_max.data_ptr()), p(f),
            ctypes.c_int(self.grid), p(value), ctypes.byref(logscale))
        if rc != 0:
            raise RuntimeError(f"reference kernel sweep failed with CUDA error {rc}")
        return complex(value[0], value[1]), logscale.value

    def amplitude(self, bits):
        """<x| (x)U |G>, as ScanOracle.amplitude of the reference (W/scan_oracle.py:25-29)."""
        value, logscale = self.sweep(bits)
        return value * math.exp(logscale) * 2.0 ** (-self.n / 2)
