"""GPU parity of the conditional (Fourier-cut) sampler against the CPU oracle.

State: L2 error of the normalised conditional state < 1e-5 (the reference's
validation bar, W/specialized_deferred_sampler.py:311).  Draws: chi-square over 64
equal-mass groups and linear XEB bias (the design of W/cpu_draw_test/run_all.py:14-38).
Building blocks: WHT, products, phase, index map and masses against NumPy.
"""
import numpy as np
import pytest
import torch
from scipy import stats

from oracle import graph_state as gs

pytestmark = pytest.mark.gpu


def _fixture(fixtures, name):
    return (fixtures[f"{name}/graph"], fixtures[f"{name}/measurement_unitaries"], fixtures[f"{name}/A"].tolist(),
            fixtures[f"{name}/B"].tolist())


def _synthetic(pkg, m, seed):
    rng = np.random.default_rng(seed)
    while True:
        g = pkg.instances.dense(2 * m, rng)
        perm = rng.permutation(2 * m)
        A, B = perm[:m].tolist(), perm[m:].tolist()
        if gs.gf2rank(g[np.ix_(B, A)]) == m:
            return g, pkg.instances.haar_su2(2 * m, rng), A, B


def _check_state(sampler, g, u, A, B, ob, tol=1e-5):
    ref = gs.cpu_covariant(g, u, A, B, ob)
    got = sampler.host()
    l2 = float(np.linalg.norm(got - ref))
    assert l2 < tol, l2
    return l2


@pytest.mark.parametrize("name", ["induced_12q", "induced_24q", "induced_32q", "induced_40q"])
def test_reference_fixtures(pkg, fixtures, name):
    g, u, A, B = _fixture(fixtures, name)
    s = pkg.ConditionalSampler(g, u, A, B, [0, 1], chunk_mib=1, fusion_bits=5)
    assert s.specialized  # identical B unitaries, as in the reference's production instance
    rng = np.random.default_rng(len(A))
    for _ in range(2):
        ob = rng.integers(0, 2, len(B)).tolist()
        stages = s.compute(ob)
        assert all(v >= 0 for v in stages.values())
        _check_state(s, g, u, A, B, ob)
        _, norm, _, _ = s.masses()
        assert abs(norm - 1) < 1e-5


@pytest.mark.parametrize("m,seed", [(5, 1), (13, 2), (14, 3), (19, 4), (24, 5)])
def test_synthetic_cuts_generic_unitaries(pkg, m, seed):
    """Haar B unitaries (generic chunk weights); m across the one/two/three-pass schedules."""
    g, u, A, B = _synthetic(pkg, m, seed)
    s = pkg.ConditionalSampler(g, u, A, B)
    assert not s.specialized
    ob = np.random.default_rng(seed).integers(0, 2, m).tolist()
    s.compute(ob)
    _check_state(s, g, u, A, B, ob)


@pytest.mark.parametrize("deferred", [True, False])
def test_permute_pipeline_and_deferral(pkg, fixtures, deferred):
    g, u, A, B = _fixture(fixtures, "induced_32q")
    ob = np.random.default_rng(7).integers(0, 2, len(B)).tolist()
    cov = pkg.ConditionalSampler(g, u, A, B, deferred=deferred)
    cov.compute(ob)
    per = pkg.ConditionalSampler(g, u, A, B, deferred=deferred, method="permute")
    per.compute(ob)
    _check_state(cov, g, u, A, B, ob)
    _check_state(per, g, u, A, B, ob)
    idx = np.random.default_rng(1).integers(0, 1 << len(A), 16)
    full = cov.host()
    for i in idx:
        assert abs(cov.probability_at(int(i)) - abs(full[i]) ** 2) < 1e-7
        assert abs(per.probability_at(int(i)) - abs(full[i]) ** 2) < 1e-7


def _grouped_chi2(idx, p, G=64):
    order = np.argsort(p, kind="stable")
    cm = np.cumsum(p[order])
    grp = np.empty(len(p), np.int64)
    grp[order] = np.minimum((cm * G).astype(np.int64), G - 1)
    e = np.bincount(grp, weights=p, minlength=G) * len(idx)
    c = np.bincount(grp[idx], minlength=G)
    return float(stats.chi2.sf(((c - e) ** 2 / e).sum(), G - 1))


def test_draws_follow_born_distribution(pkg, fixtures):
    g, u, A, B = _fixture(fixtures, "induced_24q")
    s = pkg.ConditionalSampler(g, u, A, B)
    rng = np.random.default_rng(20261203)
    pvals, diffs, ses = [], [], []
    for trial in range(3):
        ob = rng.integers(0, 2, len(B)).tolist()
        s.compute(ob)
        p = np.abs(s.host()) ** 2
        p /= p.sum()
        draws = np.array([s.draw(rng)[0] for _ in range(4000)])
        pvals.append(_grouped_chi2(draws, p))
        z = (1 << len(A)) * p[draws]
        exact = (1 << len(A)) * (p ** 2).sum() - 1
        diffs.append(z.mean() - 1 - exact)
        ses.append(z.std(ddof=1) / np.sqrt(len(z)))
    assert min(pvals) > 1e-4, pvals
    assert abs(np.mean(diffs)) < 6 * np.sqrt(np.sum(np.square(ses))) / len(ses)


def test_draw_matches_host_inverse_cdf(pkg, fixtures):
    """Same uniforms -> same index as the reference's two-level searchsorted on the
    pre-terminal tile masses plus the terminal pair (deferred_global_sampler.py:72-78)."""
    g, u, A, B = _fixture(fixtures, "induced_32q")
    s = pkg.ConditionalSampler(g, u, A, B)
    ob = [1, 0] * 8
    s.compute(ob)
    raw = s._result.cpu().numpy().astype(np.complex128)
    pre = np.abs(raw) ** 2
    tb = s.tilebits
    mass = pre.reshape(-1, 1 << tb).sum(axis=1)

    class Fixed:
        def __init__(self, us):
            self.us = list(us)

        def random(self):
            return self.us.pop(0)

    rng = np.random.default_rng(3)
    half = 1 << (len(A) - 1)
    for _ in range(20):
        us = rng.random(3)
        idx, pa, norm = s.draw(Fixed(us))
        block = int(np.searchsorted(np.cumsum(mass), us[0] * mass.sum(), side="right"))
        p = pre[block << tb:(block + 1) << tb]
        within = int(np.searchsorted(np.cumsum(p), us[1] * p.sum(), side="right"))
        local = ((block << tb) + within) % half
        pair = s.terminal_unitary @ np.array([raw[local], raw[local + half]])
        q = np.abs(pair) ** 2
        bit = int(us[2] * q.sum() >= q[0])
        assert idx == bit * half + local
        assert abs(pa - q[bit]) < 1e-12 and abs(norm - mass.sum()) < 1e-9


def test_produce_records(pkg, fixtures):
    g, u, A, B = _fixture(fixtures, "induced_24q")
    s = pkg.ConditionalSampler(g, u, A, B)
    rng = np.random.Generator(np.random.PCG64(178471532066333289424900750257149666881))
    recs = pkg.produce(s, rng, 3, len(g))
    for r in recs:
        assert len(r["draw_uniforms"]) == 3 and len(r["B_bits"]) == len(B)
        bits = r["bitstring_q0_left"]
        assert all(int(bits[q]) == r["B_bits"][j] for j, q in enumerate(B))
        assert abs(r["probability"] - r["probability_raw"] / r["conditional_norm"]) < 1e-15
        full = gs.statevector(g, u)
        idx = sum(int(c) << q for q, c in enumerate(bits))
        assert abs(r["probability"] - abs(full[idx]) ** 2) / abs(full[idx]) ** 2 < 1e-4


@pytest.mark.parametrize("nbits", [4, 9, 13, 14, 20, 24])
def test_building_blocks(pkg, nbits):
    rng = np.random.default_rng(nbits)
    x = (rng.standard_normal(1 << nbits) + 1j * rng.standard_normal(1 << nbits)).astype(np.complex64)
    d = torch.from_numpy(x.copy()).cuda()
    lo, hi = (1, nbits - 1) if nbits > 5 else (0, nbits)
    pkg.fwht(d, lo, hi)
    ref = x.astype(np.complex128)
    for q in range(lo, hi):
        gs.apply_one(ref, gs.HADAMARD, q)
    assert np.abs(d.cpu().numpy() - ref).max() < 1e-4 * np.abs(ref).max()
    u = pkg.instances.haar_su2(nbits, rng)
    d2 = torch.from_numpy(x.copy()).cuda()
    pkg.product(d2, u)
    ref2 = x.astype(np.complex128)
    for q in range(nbits):
        gs.apply_one(ref2, u[q], q)
    assert np.abs(d2.cpu().numpy() - ref2).max() < 1e-5 * np.abs(ref2).max()
    tb = min(nbits, 6)
    masses = pkg.block_mass(d2, tb).cpu().numpy()
    got = d2.cpu().numpy().astype(np.complex128)
    assert np.allclose(masses, (np.abs(got) ** 2).reshape(-1, 1 << tb).sum(1), rtol=1e-12)


def test_index_map_and_phase(pkg, fixtures):
    import ctypes
    g, u, A, B = _fixture(fixtures, "induced_24q")
    s = pkg.ConditionalSampler(g, u, A, B)
    m = len(A)
    rng = np.random.default_rng(5)
    x = (rng.standard_normal(1 << m) + 1j * rng.standard_normal(1 << m)).astype(np.complex64)
    src = torch.from_numpy(x.copy()).cuda()
    dst = torch.empty_like(src)
    lib = pkg._lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    pkg._lib.check(lib.rgs_fourier_index_map(s._h, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()),
                                             stream))
    ida = np.arange(1 << m, dtype=np.uint64)
    mapped = np.zeros_like(ida)
    for i, a in enumerate(A):
        mask = np.uint64(sum(1 << j for j, b in enumerate(B) if g[a, b]))
        mapped ^= ((ida >> np.uint64(i)) & np.uint64(1)) * mask
    phase = gs.phase_for_ids(ida, g[np.ix_(A, A)])
    ref = x[mapped.astype(np.int64)].astype(np.complex128) * phase * 2.0 ** (-m / 2)
    assert np.abs(dst.cpu().numpy() - ref).max() < 1e-6 * np.abs(ref).max()
    pkg._lib.check(lib.rgs_fourier_quadphase(s._h, ctypes.c_void_p(src.data_ptr()), stream))
    assert np.array_equal(src.cpu().numpy(), (x * phase).astype(np.complex64))


@pytest.mark.parametrize("nbits,lo,hi", [(12, 0, 12), (14, 1, 13), (17, 0, 17), (21, 3, 20), (22, 0, 22)])
def test_tensor_core_wht_precision(pkg, nbits, lo, hi):
    """16 x 16 Hadamard blocks on the tensor cores (tcgen05) over split-BF16 values
    against the FP64 oracle: relative L2 error <= 3e-5 with two BF16 terms, <= 1e-6 with
    three (FP32 butterflies: <= 1e-6); the GEMM flag of a bounded wait stays clear."""
    import ctypes
    rng = np.random.default_rng(nbits + lo)
    x = (rng.standard_normal(1 << nbits) + 1j * rng.standard_normal(1 << nbits)).astype(np.complex64)
    ref = x.astype(np.complex128)
    for q in range(lo, hi):  # butterfly (x + y, x - y) on bit q of the flat index, as gs.apply_one
        v = ref.reshape(-1, 2, 1 << q)
        ref = np.stack([v[:, 0] + v[:, 1], v[:, 0] - v[:, 1]], axis=1).reshape(-1)
    errs = {}
    for prec in ("fp32", "split_bf16x2", "split_bf16x3"):
        d = torch.from_numpy(x.copy()).cuda()
        pkg.fwht(d, lo, hi, precision=prec)
        got = d.cpu().numpy().astype(np.complex128)
        errs[prec] = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert errs["fp32"] < 1e-6, errs
    assert errs["split_bf16x3"] < 1e-6, errs
    assert errs["split_bf16x2"] < 3e-5, errs
    flag = ctypes.c_int32(-1)
    pkg._lib.check(pkg._lib.lib().rgs_tensor_core_status(ctypes.byref(flag)))
    assert flag.value == 0


def test_tensor_core_wht_rejects_small_states(pkg):
    d = torch.zeros(1 << 10, dtype=torch.complex64, device="cuda")
    with pytest.raises(NotImplementedError):
        pkg.fwht(d, precision="split_bf16x3")


@pytest.mark.parametrize("m", [13, 16, 21, 22, 26, 29])
@pytest.mark.parametrize("identical_b", [True, False])
def test_register_schedule_matches_rounds(pkg, m, identical_b):
    """The register-first pass kernel (default) and the one-round-per-four-axes kernel
    give the same conditional state and tile masses.  m covers strided groups of 1 (m=13),
    4, 9, 5+5, 7+7 and 9+8 target bits; identical B unitaries take the table init, Haar
    ones the generic chunk init."""
    g, u, A, B = _synthetic(pkg, m, 100 + m)
    if identical_b:
        u[B] = u[B[0]]
    s = pkg.ConditionalSampler(g, u, A, B)
    assert s.specialized == identical_b
    ob = np.random.default_rng(m).integers(0, 2, m).tolist()
    lib = pkg._lib.lib()
    try:
        pkg._lib.check(lib.rgs_fourier_set_register_schedule(0))
        s.compute(ob)
        ref = s.state.clone()
        _, ref_norm, _, _ = s.masses()
        pkg._lib.check(lib.rgs_fourier_set_register_schedule(1))
        s.compute(ob)
        _, norm, _, _ = s.masses()
    finally:
        pkg._lib.check(lib.rgs_fourier_set_register_schedule(1))
    rel = float(torch.linalg.norm((s.state - ref).to(torch.complex128)) / torch.linalg.norm(ref.to(torch.complex128)))
    assert rel < 1e-5, rel
    assert abs(norm - ref_norm) < 1e-5 and abs(norm - 1) < 1e-4


@pytest.mark.parametrize("m", [13, 21, 26, 29])
def test_tma_staging_is_bit_identical(pkg, m):
    """TMA-staged tile loads and thread loads (default) read the same values into the
    same registers: the conditional state is bit-identical, and no bounded wait gave up."""
    import ctypes
    g, u, A, B = _synthetic(pkg, m, 200 + m)
    u[B] = u[B[0]]
    s = pkg.ConditionalSampler(g, u, A, B)
    ob = np.random.default_rng(m).integers(0, 2, m).tolist()
    lib = pkg._lib.lib()
    try:
        pkg._lib.check(lib.rgs_fourier_set_tma(0))
        s.compute(ob)
        ref = s.state.clone()
        pkg._lib.check(lib.rgs_fourier_set_tma(1))
        s.compute(ob)
    finally:
        pkg._lib.check(lib.rgs_fourier_set_tma(0))
    assert torch.equal(s.state, ref)
    flag = ctypes.c_int32()
    pkg._lib.check(lib.rgs_tensor_core_status(ctypes.byref(flag)))
    assert flag.value == 0
