"""Proposal network on the GPU: BF16 GEMM, gradients against the FP64 CPU oracle,
training on exact samples and marginals, and rejection sampling against p(x)."""
import ctypes

import numpy as np
import pytest
import torch
from scipy import stats

from oracle import graph_state as gs
from oracle import made as omade

pytestmark = pytest.mark.gpu


def _bf(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda().to(torch.bfloat16)


def test_inputs_of_any_layout(pkg):
    """Column-permuted (non-contiguous) inputs give the same log q as their copies."""
    net = pkg.MadeProposal(10, hidden=64, seed=2)
    x = np.random.default_rng(0).integers(0, 2, (64, 10)).astype(np.float32)
    view = torch.as_tensor(np.ascontiguousarray(x.T)).cuda().T  # (64, 10), column-major view
    assert not view.is_contiguous()
    a = net.log_q(view).cpu().numpy().copy()
    b = net.log_q(torch.as_tensor(x).cuda()).cpu().numpy()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("M,N,K,tA,tB", [(64, 64, 32, 0, 0), (100, 70, 45, 0, 1), (33, 130, 200, 1, 0),
                                         (512, 40, 4096, 1, 0), (257, 512, 512, 0, 1)])
def test_gemm_bf16(pkg, M, N, K, tA, tB):
    rng = np.random.default_rng(M + N + K)
    A = rng.normal(size=(K, M) if tA else (M, K))
    B = rng.normal(size=(N, K) if tB else (K, N))
    bias = rng.normal(size=N).astype(np.float32)
    mask = (rng.random((M, N)) < 0.7).astype(np.uint8)
    gate = rng.normal(size=(M, N))
    dA, dB, dG = _bf(A), _bf(B), _bf(gate)
    C = torch.empty((M, N), dtype=torch.float32, device="cuda")
    db, dm = torch.from_numpy(bias).cuda(), torch.from_numpy(mask).cuda()
    lib = pkg._lib.lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    pkg._lib.check(lib.rgs_gemm_bf16(M, N, K, p(dA), dA.shape[1], tA, p(dB), dB.shape[1], tB, 0.5, p(db), 1, p(dm),
                                     p(dG), p(C), None, N, s))
    a = dA.to(torch.float32).cpu().numpy().astype(np.float64)
    b = dB.to(torch.float32).cpu().numpy().astype(np.float64)
    g = dG.to(torch.float32).cpu().numpy()
    ref = 0.5 * ((a.T if tA else a) @ (b.T if tB else b)) + bias
    ref = np.maximum(ref, 0) * mask * (g > 0)
    assert np.abs(C.cpu().numpy() - ref).max() < 1e-4 * np.sqrt(K) * 4


@pytest.mark.parametrize("M,N,K", [(256, 512, 56), (4096, 512, 512), (300, 56, 512)])
def test_gemm_tma_and_staged_operands_agree(pkg, M, N, K):
    """K-major operands with 16-byte aligned rows (the forward GEMMs) load by TMA with a
    128-byte swizzle; the thread-staged path issues the same MMAs in the same order, so
    the two results are bitwise equal; the tensor-core wait flag stays clear."""
    rng = np.random.default_rng(M + K)
    dA, dB = _bf(rng.normal(size=(M, K))), _bf(rng.normal(size=(N, K)))
    lib = pkg._lib.lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    out = []
    try:
        for tma in (1, 0):
            pkg._lib.check(lib.rgs_gemm_set_tma(tma))
            C = torch.empty((M, N), dtype=torch.float32, device="cuda")
            pkg._lib.check(lib.rgs_gemm_bf16(M, N, K, p(dA), K, 0, p(dB), K, 1, 1.0, None, 0, None, None, p(C), None,
                                             N, s))
            out.append(C.cpu().numpy())
    finally:
        pkg._lib.check(lib.rgs_gemm_set_tma(1))
    assert np.array_equal(out[0], out[1])
    ref = dA.to(torch.float32).cpu().numpy().astype(np.float64) @ dB.to(torch.float32).cpu().numpy().T
    assert np.abs(out[0] - ref).max() < 1e-4 * np.sqrt(K) * 4
    flag = ctypes.c_int32(-1)
    pkg._lib.check(lib.rgs_tensor_core_status(ctypes.byref(flag)))
    assert flag.value == 0


def test_gradients_match_cpu_oracle(pkg):
    n, hidden, B = 14, 64, 256
    net = pkg.MadeProposal(n, hidden=hidden, seed=3)
    rng = np.random.default_rng(4)
    x = rng.integers(0, 2, (B, n)).astype(np.float32)
    target = rng.random((B, n)).astype(np.float32)
    loss, g = net.gradients(_bf(x), torch.from_numpy(target).cuda())
    st = net.state()
    ref_loss, ref = omade.loss_and_grads(x.astype(np.float64), target.astype(np.float64),
                                         [w.astype(np.float64) for w in st["wb"]],
                                         [b.astype(np.float64) for b in st["b"]], st["masks"])
    assert abs(loss - ref_loss) < 1e-2 * abs(ref_loss)
    for got, want in zip(g, ref):
        got = got.cpu().numpy()
        err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-12)
        assert err < 5e-2, err  # BF16 activations and gradients; FP32 accumulation
    # The autoregressive masks hold on the gradients.
    assert np.all(g[0].cpu().numpy()[st["masks"][0] == 0] == 0)
    assert np.all(g[4].cpu().numpy()[st["masks"][2] == 0] == 0)


@pytest.fixture(scope="module")
def trained(pkg):
    inst = pkg.instances.make_instance("reg3", 14, 21, pkg.rank_profile)
    cs = pkg.ChainSampler(inst.g, inst.u, inst.order)
    bits, p, logp = cs.sample(2 ** 15, seed=5)
    cond, _, _ = cs.marginals(bits)
    scan_bits = bits[:, inst.order]
    net = pkg.MadeProposal(inst.n, hidden=256, seed=1)
    losses = net.fit(scan_bits, cond, epochs=40, batch=1024, lr=5e-3)
    c = np.clip(cond.astype(np.float64), 1e-12, 1 - 1e-12)
    floor = float(np.mean(np.sum(-(c * np.log(c) + (1 - c) * np.log(1 - c)), axis=1)))  # = H(p) by the chain rule
    return inst, cs, net, (losses, floor)


def test_training_learns_the_distribution(pkg, trained):
    """Soft-target cross entropy has the floor H(p); training closes most of the gap."""
    inst, cs, net, (losses, floor) = trained
    assert np.mean(losses[-5:]) - floor < 0.5 * (np.mean(losses[:3]) - floor)
    probs = np.abs(gs.statevector(inst.g, inst.u)) ** 2
    allx = ((np.arange(1 << inst.n)[:, None] >> np.arange(inst.n)) & 1).astype(np.float32)
    lq = net.log_q(_bf(allx[:, inst.order])).cpu().numpy()
    q = np.exp(lq)
    assert abs(q.sum() - 1) < 1e-3                         # a normalised distribution
    kl = float(np.sum(probs * (np.log(probs) - lq)))
    kl_uniform = float(np.sum(probs * (np.log(probs) + inst.n * np.log(2))))
    assert kl < 0.5 * kl_uniform, (kl, kl_uniform)


def test_proposal_samples_follow_q(pkg, trained):
    inst, cs, net, _ = trained
    x, logq = net.sample(4096, seed=7)
    lq2 = net.log_q(x.clone()).cpu().numpy()
    assert np.abs(lq2 - logq.cpu().numpy()).max() < 1e-3
    xs = x.to(torch.float32).cpu().numpy()
    assert set(np.unique(xs)) <= {0.0, 1.0}


def test_learned_rejection_is_born_exact_with_envelope(pkg, trained):
    inst, cs, net, _ = trained
    n = inst.n
    probs = np.abs(gs.statevector(inst.g, inst.u)) ** 2
    allx = ((np.arange(1 << n)[:, None] >> np.arange(n)) & 1).astype(np.float32)
    lq_all = net.log_q(_bf(allx[:, inst.order])).cpu().numpy()
    log_c = float(np.max(np.log(probs) - lq_all))        # exact envelope (small n)
    so = pkg.ScanOracle(inst.g, inst.u, inst.order)
    so128 = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True)
    inv = np.argsort(inst.order)

    def propose(r):
        x, lq = net.sample(4096, seed=100 + r)
        scan = x.to(torch.float32).cpu().numpy().astype(np.uint8)
        return scan[:, inv], lq.cpu().numpy()

    rng = np.random.default_rng(8)
    bits, p, st = pkg.proposal.rejection_sample(so.probabilities, propose, log_c, 6000, rng,
                                                recheck_fn=so128.probabilities)
    assert st["envelope_violations"] == 0
    idx = (bits.astype(np.int64) << np.arange(n)).sum(1)
    G = 32
    order = np.argsort(probs, kind="stable")
    cm = np.cumsum(probs[order])
    grp = np.empty(len(probs), np.int64)
    grp[order] = np.minimum((cm * G).astype(np.int64), G - 1)
    e = np.bincount(grp, weights=probs, minlength=G) * len(idx)
    c = np.bincount(grp[idx], minlength=G)
    assert stats.chi2.sf(((c - e) ** 2 / e).sum(), G - 1) > 1e-4
    learned_acc = float(np.exp(-log_c))
    assert abs(st["acceptance"] - learned_acc) < 5 * np.sqrt(learned_acc / st["proposals"]) + 0.01
    # An envelope below max p/q is reported as violations (output then follows min(p, cq)).
    _, _, st2 = pkg.proposal.rejection_sample(so.probabilities, propose, log_c - 2.0, 1000, rng)
    assert st2["envelope_violations"] > 0


def test_learned_mixture_gains_over_uniform(pkg, trained):
    """What the trained network gains over the method without it (uniform proposals):
    exact rejection with a proposal q accepts 1 / max_x (p / q) of its proposals -- with
    the uniform proposal 1 / (2^n max p).  KL training fits the bulk of p, and the worst
    ratio p / q of the bare network sits in its tail; the defensive mixture
    q_mix = (1 - 1/2) q + 1/2 2^-n bounds that tail.  Both envelopes are exact (all 2^n
    strings), so the comparison carries no sampling noise; draws with the mixture are
    Born-exact (grouped chi-square)."""
    inst, cs, net, _ = trained
    n = inst.n
    probs = np.abs(gs.statevector(inst.g, inst.u)) ** 2
    allx = ((np.arange(1 << n)[:, None] >> np.arange(n)) & 1).astype(np.float32)
    lq_all = net.log_q(_bf(allx[:, inst.order])).cpu().numpy()
    uniform_acc = 1.0 / ((2.0 ** n) * probs.max())
    bare_acc = float(np.exp(-np.max(np.log(probs) - lq_all)))
    mix = 0.5
    log_c = float(np.max(np.log(probs) - net.mixture_log_q(lq_all, mix)))
    mix_acc = float(np.exp(-log_c))
    print(f"exact-envelope acceptance: network {bare_acc:.4f}, mixture {mix_acc:.4f}, uniform {uniform_acc:.4f}")
    assert mix_acc > uniform_acc
    so = pkg.ScanOracle(inst.g, inst.u, inst.order)
    so128 = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True)
    inv = np.argsort(inst.order)

    def propose(r):
        x, lq = net.sample_mixture(4096, mix, seed=500 + r)
        scan = x.to(torch.float32).cpu().numpy().astype(np.uint8)
        return scan[:, inv], lq.cpu().numpy()

    bits, p, st = pkg.proposal.rejection_sample(so.probabilities, propose, log_c, 6000, np.random.default_rng(9),
                                                recheck_fn=so128.probabilities)
    assert st["envelope_violations"] == 0
    assert abs(st["acceptance"] - mix_acc) < 5 * np.sqrt(mix_acc / st["proposals"]) + 0.01
    idx = (bits.astype(np.int64) << np.arange(n)).sum(1)
    G = 32
    order = np.argsort(probs, kind="stable")
    cm = np.cumsum(probs[order])
    grp = np.empty(len(probs), np.int64)
    grp[order] = np.minimum((cm * G).astype(np.int64), G - 1)
    e = np.bincount(grp, weights=probs, minlength=G) * len(idx)
    c = np.bincount(grp[idx], minlength=G)
    assert stats.chi2.sf(((c - e) ** 2 / e).sum(), G - 1) > 1e-4


def test_capped_rejection_reference_rule(pkg):
    """Uniform proposals + accept iff u < min(2^n p / cap, 1) give min(2^n p, cap)
    (W/rejection_selfcheck.py: TV < 0.05, XEB within 6 SE)."""
    inst = pkg.instances.make_instance("dense", 10, 4, pkg.rank_profile)
    n = inst.n
    probs = np.abs(gs.statevector(inst.g, inst.u)) ** 2
    so = pkg.ScanOracle(inst.g, inst.u, inst.order)
    so128 = pkg.ScanOracle(inst.g, inst.u, inst.order, fp64=True)
    rng = np.random.default_rng(314159)
    recs, summary = pkg.proposal.capped_rejection(so, rng, 4000, cap=1.0, recheck=so128)
    assert summary["completed"]
    target = np.minimum((2.0 ** n) * probs, 1.0)
    target /= target.sum()
    acc = np.array([int(r["bitstring_q0_left"][::-1], 2) for r in recs if r["accepted"]])
    # Grouped chi-square against min(2^n p, cap) (2^10 outcomes are too many for a raw TV at 4000 draws).
    G = 32
    order = np.argsort(target, kind="stable")
    cm = np.cumsum(target[order])
    grp = np.empty(len(target), np.int64)
    grp[order] = np.minimum((cm * G).astype(np.int64), G - 1)
    e = np.bincount(grp, weights=target, minlength=G) * len(acc)
    c = np.bincount(grp[acc], minlength=G)
    assert stats.chi2.sf(((c - e) ** 2 / e).sum(), G - 1) > 1e-4
    # Grouped TV well below the gap between the capped and the Born distribution.
    born = np.bincount(grp, weights=probs, minlength=G)
    assert 0.5 * np.abs(c / len(acc) - e / len(acc)).sum() < 0.5 * 0.5 * np.abs(born - e / len(acc)).sum() + 0.03
    # Same RNG call order as the reference: first proposal = first 10 bits of the stream.
    first = np.random.default_rng(314159).integers(0, 2, n)
    assert recs[0]["bitstring_q0_left"] == "".join(map(str, first))
