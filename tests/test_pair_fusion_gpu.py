"""Fused pairs on the GPU: scan_pair_kernel against the position-by-position sweep, the
FP64 statevector and itself under other schedules.

* Fused sweeps match the statevector (probability relative error 1e-4 complex64,
  1e-12 complex128) and the unfused sweep to rounding (1e-5 complex64 with float64
  arithmetic, 1e-4 with float32 arithmetic, 1e-13 complex128), for plans that use every
  pair code the compiler produced on these graphs, at batch tiles 1 to the maximum.
* The chunked schedule (low-rank positions once per chunk of tiles) and the
  tile-by-tile schedule (a workspace of one tile) give bitwise-equal results.
* The fused pass keeps the intermediate table out of the launch list: a sweep has one
  launch per pair instead of two.
"""
import ctypes

import numpy as np
import pytest

from oracle import graph_state as gs

pytestmark = pytest.mark.gpu

TOL = {"c64": 1e-4, "c64f32": 1e-4, "c128": 1e-12}


def _prob(pkg, val, ls, n):
    return np.abs(pkg.amplitudes_from(val, ls, n)) ** 2


def _cases(pkg):
    rng = np.random.default_rng(77)
    out = []
    for kind, n in (("reg3", 16), ("reg3", 20), ("er3", 18), ("deg3", 19), ("dense", 12), ("dense", 14)):
        for s in range(2):
            if kind == "dense":
                g = pkg.instances.dense(n, rng)
                u = pkg.instances.haar_su2(n, rng)
                out.append((g, u, rng.permutation(n).tolist()))
            else:
                inst = pkg.instances.make_instance(kind, n, int(rng.integers(1 << 30)), pkg.rank_profile)
                out.append((inst.g, inst.u, inst.order))
                out.append((inst.g, inst.u, rng.permutation(n).tolist()))
    return out


@pytest.mark.parametrize("precision", ["c64", "c64f32", "c128"])
def test_fused_matches_statevector_and_unfused(pkg, precision):
    rng = np.random.default_rng(3)
    codes = set()
    cap = pkg.max_batch_tile(precision)
    for g, u, order in _cases(pkg):
        n = len(g)
        edges = pkg.edges_from_graph(g)
        plan = pkg.ScanPlan(n, edges, order)
        assert plan.pairs, "expected fused pairs"
        for k in range(len(plan.pairs)):
            info = plan.pair_info(k)
            codes.add((info.code_a, info.code_b))
        bits = pkg.instances.uniform_bits(257, n, rng)
        full = gs.statevector(g, u)
        ref = np.abs(full[(bits.astype(np.int64) << np.arange(n)).sum(axis=1)]) ** 2
        off = pkg.ScanEngine(pkg.ScanPlan(n, edges, order, fuse=False), u, precision=precision)
        p_off = _prob(pkg, *off.sweep_bits(bits), n)
        for tile in (1, 8, cap):
            eng = pkg.ScanEngine(plan, u, precision=precision, batch_tile=tile)
            p = _prob(pkg, *eng.sweep_bits(bits), n)
            assert np.max(np.abs(p - ref) / ref) < TOL[precision], (n, tile)
            assert np.max(np.abs(p - p_off) / p_off) < {"c64": 1e-5, "c64f32": 1e-4, "c128": 1e-13}[precision], \
                (n, tile)
    assert {(0, 0), (0, 3), (3, 3), (3, 4), (4, 4)} <= codes, codes


def test_fused_tile_invariance(pkg):
    """Bitwise equal (value, logscale) at every tile: the pair kernel's per-item arithmetic
    does not depend on how items are laid out."""
    inst = pkg.instances.make_instance("reg3", 24, 5, pkg.rank_profile)
    plan = pkg.ScanPlan(24, pkg.edges_from_graph(inst.g), inst.order)
    assert plan.pairs
    bits = pkg.instances.uniform_bits(300, 24, np.random.default_rng(5))
    for precision in ("c64", "c64f32", "c128"):
        outs = []
        for tile in (1, 2, 16, 64, pkg.max_batch_tile(precision)):
            eng = pkg.ScanEngine(plan, inst.u, precision=precision, batch_tile=tile)
            outs.append(eng.sweep_bits(bits))
        for val, ls in outs[1:]:
            assert np.array_equal(val, outs[0][0]) and np.array_equal(ls, outs[0][1]), precision


def _one_tile_workspace(plan, tile, esize):
    n = plan.n

    def up(x):
        return (x + 255) // 256 * 256

    return 2 * up((tile << plan.rmax) * esize) + up(n * tile * 32) + up(n * tile) + up(n * tile * 8)


@pytest.mark.parametrize("precision", ["c64f32", "c128"])
def test_chunked_and_tile_schedules_bitwise(pkg, precision):
    import torch
    # A plan with low-rank head and tail and a middle of higher rank (rmax above 12).
    inst = pkg.instances.make_instance("reg3", 34, 11, pkg.rank_profile, target_rank=15)
    plan = pkg.ScanPlan(inst.n, pkg.edges_from_graph(inst.g), inst.order)
    assert plan.rmax > 12 and plan.pairs
    bits = pkg.instances.uniform_bits(700, inst.n, np.random.default_rng(2))
    tile = 32
    eng = pkg.ScanEngine(plan, inst.u, precision=precision, batch_tile=tile)
    val, ls = eng.sweep_bits(bits)
    # The same sweep through the C ABI with a workspace of one tile (tile by tile).
    esize = 16 if precision == "c128" else 8
    ws_bytes = _one_tile_workspace(plan, tile, esize)
    launches = ctypes.c_int64()
    pkg._lib.check(pkg._lib.lib().rgs_scan_launch_count(plan.handle, len(bits), tile, eng.prec_code, ws_bytes,
                                                        ctypes.byref(launches)))
    nseg = inst.n - len(plan.pairs)
    assert launches.value == -(-len(bits) // tile) * (nseg + 2)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=eng.device)
    d_bits = torch.from_numpy(pkg.pack_bits(bits, inst.n).view(np.int64)).to(eng.device)
    v2, l2 = eng.out_tensors(len(bits))
    s = torch.cuda.current_stream(eng.device)
    pkg._lib.check(pkg._lib.lib().rgs_scan_amplitudes(
        plan.handle, ctypes.c_void_p(eng.d_u.data_ptr()), ctypes.c_void_p(d_bits.data_ptr()), len(bits),
        eng.prec_code, ctypes.c_void_p(v2.data_ptr()), ctypes.c_void_p(l2.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
        ws_bytes, tile, ctypes.c_void_p(s.cuda_stream)))
    torch.cuda.synchronize()
    assert np.array_equal(val, v2.cpu().numpy()) and np.array_equal(ls, l2.cpu().numpy())


def test_launch_count_with_pairs(pkg):
    inst = pkg.instances.make_instance("reg3", 30, 4, pkg.rank_profile)
    on = pkg.ScanEngine(pkg.ScanPlan(30, pkg.edges_from_graph(inst.g), inst.order), inst.u, precision="c64f32",
                        batch_tile=64)
    off = pkg.ScanEngine(pkg.ScanPlan(30, pkg.edges_from_graph(inst.g), inst.order, fuse=False), inst.u,
                         precision="c64f32", batch_tile=64)
    assert on.launch_count(64) == off.launch_count(64) - len(on.plan.pairs)


def test_rare_pair_codes_on_gpu(pkg):
    """The four pair codes the graphs above do not produce, on small seeded plans that do
    (the same plans as the CPU emulation test), against the statevector."""
    from test_pair_fusion import RARE_CODES, rare_code_plans
    plans = rare_code_plans(pkg)
    assert set(plans) == RARE_CODES
    rng = np.random.default_rng(8)
    for code, (g, order) in plans.items():
        n = len(g)
        u = pkg.instances.haar_su2(n, rng)
        plan = pkg.ScanPlan(n, pkg.edges_from_graph(g), order)
        bits = pkg.instances.uniform_bits(100, n, rng)
        ref = np.abs(gs.statevector(g, u)[(bits.astype(np.int64) << np.arange(n)).sum(axis=1)]) ** 2
        for precision in ("c64", "c64f32", "c128"):
            for tile in (1, 8, pkg.max_batch_tile(precision)):
                eng = pkg.ScanEngine(plan, u, precision=precision, batch_tile=tile)
                p = _prob(pkg, *eng.sweep_bits(bits), n)
                assert np.max(np.abs(p - ref) / ref) < TOL[precision], (code, precision, tile)
