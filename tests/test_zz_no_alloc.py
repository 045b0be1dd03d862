"""The allocation-free scan entry point agrees with the allocating one.

rgs_scan_amplitudes_noalloc exists for callers that cannot let the library allocate
device memory (hosts that fix the library's memory budget, integrations whose
allocator must own every byte of the GPU): it takes only inputs and outputs and
keeps its scratch in a static device array.  This file is collected
last so a failure here does not hide the rest of the suite.  Each test calls the
new entry point through the C ABI twice in a row (different batches, so stale
scratch from the first call would show) and compares with rgs_scan_amplitudes.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(pkg, plan, d_u, d_bits, batch, prec, out_v, out_l):
    import torch

    lib = pkg._lib.lib()
    stream = torch.cuda.current_stream()
    return lib.rgs_scan_amplitudes_noalloc(plan.handle, ctypes.c_void_p(d_u.data_ptr()),
                                           ctypes.c_void_p(d_bits.data_ptr()), batch, prec,
                                           ctypes.c_void_p(out_v.data_ptr()), ctypes.c_void_p(out_l.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("precision,tol", [("c64", 1e-4), ("c128", 1e-12)])
def test_noalloc_matches_workspace_entry_point(pkg, precision, tol):
    import torch

    inst = pkg.instances.make_instance("reg3", 26, 77, pkg.rank_profile)
    plan = pkg.ScanPlan(inst.n, pkg.edges_from_graph(inst.g), inst.order)
    eng = pkg.ScanEngine(plan, inst.u, precision=precision)
    prec = pkg.PRECISIONS[precision]
    vdt = torch.complex128 if precision == "c128" else torch.complex64
    for batch, seed in ((300, 1), (37, 2)):
        bits = pkg.instances.uniform_bits(batch, inst.n, np.random.default_rng(seed))
        ref_v, ref_l = eng.sweep_bits(bits)
        d_bits = torch.from_numpy(pkg.pack_bits(bits, inst.n).view(np.int64)).cuda()
        out_v = torch.empty(batch, dtype=vdt, device="cuda")
        out_l = torch.empty(batch, dtype=torch.float64, device="cuda")
        pkg._lib.check(_noalloc(pkg, plan, eng.d_u, d_bits, batch, prec, out_v, out_l))
        torch.cuda.synchronize()
        got = pkg.amplitudes_from(out_v.cpu().numpy(), out_l.cpu().numpy(), inst.n)
        ref = pkg.amplitudes_from(ref_v, ref_l, inst.n)
        rel = np.abs(np.abs(got) ** 2 - np.abs(ref) ** 2) / np.abs(ref) ** 2
        assert rel.max() < tol


def test_noalloc_fixed_vertices(pkg):
    """A plan with structurally fixed vertices: the per-item flag bytes and affine
    offsets live in the shared scratch too (diagonal / anti-diagonal gates)."""
    import torch
    from oracle import scan_plan as sp

    rng = np.random.default_rng(41)
    n = 20
    g = pkg.instances.regular3(n, rng)
    u = pkg.instances.haar_su2(n, rng)
    for k, q in enumerate(rng.choice(n, size=6, replace=False)):
        ph = np.exp(1j * rng.uniform(0, 2 * np.pi, 2))
        u[q] = np.diag(ph) if k % 2 == 0 else np.array([[0, ph[0]], [ph[1], 0]])
    fixed = sp.structurally_fixed(u, n)
    assert len(fixed) == 6
    plan = pkg.ScanPlan(n, pkg.edges_from_graph(g), rng.permutation(n).tolist(), fixed)
    for precision, tol in (("c64", 1e-4), ("c128", 1e-12)):
        eng = pkg.ScanEngine(plan, u, precision=precision)
        vdt = torch.complex128 if precision == "c128" else torch.complex64
        for batch, seed in ((129, 5), (64, 6)):
            bits = pkg.instances.uniform_bits(batch, n, np.random.default_rng(seed))
            ref = pkg.amplitudes_from(*eng.sweep_bits(bits), n)
            d_bits = torch.from_numpy(pkg.pack_bits(bits, n).view(np.int64)).cuda()
            out_v = torch.empty(batch, dtype=vdt, device="cuda")
            out_l = torch.empty(batch, dtype=torch.float64, device="cuda")
            pkg._lib.check(_noalloc(pkg, plan, eng.d_u, d_bits, batch, pkg.PRECISIONS[precision], out_v, out_l))
            torch.cuda.synchronize()
            got = pkg.amplitudes_from(out_v.cpu().numpy(), out_l.cpu().numpy(), n)
            nz = np.abs(ref) > 1e-12
            assert nz.any()
            assert np.all(np.abs(got[~nz]) < 1e-12)
            rel = np.abs(np.abs(got[nz]) ** 2 - np.abs(ref[nz]) ** 2) / np.abs(ref[nz]) ** 2
            assert rel.max() < tol


def test_noalloc_rejects_plans_beyond_its_scratch(pkg):
    import torch

    rng = np.random.default_rng(3)
    g = pkg.instances.dense(48, rng)
    u = pkg.instances.haar_su2(48, rng)
    plan = pkg.ScanPlan(48, pkg.edges_from_graph(g), list(range(48)))
    assert plan.rmax >= 23
    d_u = torch.from_numpy(u.view(np.float64).reshape(-1).copy()).cuda()
    d_bits = torch.zeros((2, 2), dtype=torch.int64, device="cuda")
    out_v = torch.empty(2, dtype=torch.complex64, device="cuda")
    out_l = torch.empty(2, dtype=torch.float64, device="cuda")
    rc = _noalloc(pkg, plan, d_u, d_bits, 2, pkg.PRECISIONS["c64"], out_v, out_l)
    assert rc == pkg._lib.RGS_ERR_OOM
    assert b"scratch" in pkg._lib.lib().rgs_last_error()
