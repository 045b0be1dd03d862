"""Two-shard conditional sampler on one GPU: both shards computed on the device (one
after the other, separate buffers, as two devices would hold them) against the oracle's
shard-local restatement, against the single-device sampler's state, and draws across the
two shards against the single-device draws with the same uniforms."""
import numpy as np
import pytest
import torch

from oracle import graph_state as gs

pytestmark = pytest.mark.gpu


def _dense_cut(pkg, m, seed, identical_b):
    rng = np.random.default_rng(seed)
    while True:
        g = pkg.instances.dense(2 * m, rng)
        perm = rng.permutation(2 * m)
        A, B = perm[:m].tolist(), perm[m:].tolist()
        if gs.gf2rank(g[np.ix_(B, A)]) == m:
            break
    u = pkg.instances.haar_su2(2 * m, rng)
    if identical_b:
        u[B] = u[B[0]]
    return g, u, A, B, rng


@pytest.mark.parametrize("m,identical_b", [(13, True), (16, False), (21, True)])
def test_gpu_shards_match_oracle_and_single_device(pkg, m, identical_b):
    g, u, A, B, rng = _dense_cut(pkg, m, 100 + m, identical_b)
    ob = rng.integers(0, 2, m).tolist()
    ref = gs.cpu_shards(g, u, A, B, ob)
    shards = [pkg.ShardedConditionalSampler(g, u, A, B, s) for s in (0, 1)]
    for s, sh in enumerate(shards):
        sh.compute(ob)
        got = sh.host()
        assert np.linalg.norm(got - ref[s]) / np.linalg.norm(ref[s]) < 1e-5
    single = pkg.ConditionalSampler(g, u, A, B)
    single.compute(ob)
    whole = single._result.cpu().numpy().astype(np.complex128)
    both = np.concatenate([sh.host() for sh in shards])
    assert np.linalg.norm(both - whole) / np.linalg.norm(whole) < 1e-5
    assert abs(sum(sh.mass() for sh in shards) - 1.0) < 1e-4
    # Draws over the two shards vs the single-device draw with the same uniforms.
    U = np.asarray(u[A[-1]])
    same = 0
    draws = 200
    for _ in range(draws):
        u1, u2, u3 = rng.random(), rng.random(), rng.random()
        idx, pa, norm = pkg.samplers.draw_across_shards(shards, U, u1, u2, u3)
        idx1, pa1, _ = single.draw(iter_rng([u1, u2, u3]))
        same += idx == idx1
        assert abs(pa - pa1) <= 1e-5 * pa1 or idx != idx1
    assert same >= 0.98 * draws


class iter_rng:
    """An rng stand-in returning given uniforms in order."""

    def __init__(self, values):
        self.values = list(values)

    def random(self):
        return self.values.pop(0)


def test_shard_schedule_needs_13_bits(pkg):
    g, u, A, B, _ = _dense_cut(pkg, 12, 5, True)
    with pytest.raises(NotImplementedError):
        pkg.ShardedConditionalSampler(g, u, A, B, 0).compute([0] * 12)
