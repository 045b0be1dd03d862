"""Host GF(2) set-up of the conditional sampler (C++ through the C ABI, no GPU):
bit-exact against the reference's tables and the oracle's maps and phases."""
import numpy as np
import pytest

from oracle import graph_state as gs

NAMES = ["induced_12q", "induced_24q", "induced_32q", "induced_40q", "rgs70"]


def _instance(fixtures, name):
    return (fixtures[f"{name}/graph"], fixtures[f"{name}/measurement_unitaries"], fixtures[f"{name}/A"].tolist(),
            fixtures[f"{name}/B"].tolist())


@pytest.mark.parametrize("name", NAMES)
def test_cut_tables_match_reference(pkg, fixtures, name):
    g, u, A, B = _instance(fixtures, name)
    t = pkg.samplers.cut_tables(g, u, A, B)
    # Rows of N = G[B,A]^{-T} (fourier_covariant_sampler.py:105) and the packed chunk tables
    # of the reference's specialisation (init_specialization.py:160-189), bit for bit.
    assert np.array_equal(t["inv_rows"], gs.row_masks(fixtures[f"{name}/inverse_transpose"]))
    if f"{name}/spec_tables" in fixtures:
        assert np.array_equal(t["lut_z"], fixtures[f"{name}/spec_tables"])
    ids = fixtures[f"{name}/probe_ids"]
    b, phase = gs.specialization_map_and_phase(t["lut_z"], ids)
    assert np.array_equal(b, fixtures[f"{name}/probe_mapped"])
    assert np.array_equal(phase, fixtures[f"{name}/probe_phase_B"])
    # q_A phase table against the reference's phase_for_ids on the same ids.
    zero, phase_a = gs.specialization_map_and_phase(t["lut_a"], ids)
    assert not zero.any()
    assert np.array_equal(phase_a, fixtures[f"{name}/probe_phase_A"])
    # Index map of the permutation path (graph_sampler.py:101-104).
    y, ph0 = gs.specialization_map_and_phase(t["lut_cols"], ids)
    expect = np.zeros_like(ids)
    for i, a in enumerate(A):
        mask = np.uint64(sum(1 << j for j, bb in enumerate(B) if g[a, bb]))
        expect ^= ((ids >> np.uint64(i)) & np.uint64(1)) * mask
    assert np.array_equal(y, expect) and np.all(ph0 == 1.0)


def test_random_cuts_against_oracle(pkg):
    rng = np.random.default_rng(11)
    done = 0
    while done < 12:
        m = int(rng.integers(4, 30))
        n = 2 * m
        g = pkg.instances.dense(n, rng)
        perm = rng.permutation(n)
        A, B = perm[:m].tolist(), perm[m:].tolist()
        if gs.gf2rank(g[np.ix_(B, A)]) < m:
            with pytest.raises(ValueError):
                pkg.samplers.cut_tables(g, pkg.instances.haar_su2(n, rng), A, B)
            continue
        t = pkg.samplers.cut_tables(g, pkg.instances.haar_su2(n, rng), A, B)
        N = gs.gf2_inverse(g[np.ix_(B, A)]).T
        ids = rng.integers(0, 1 << m, 2000, dtype=np.uint64)
        b, ph = gs.specialization_map_and_phase(t["lut_z"], ids)
        assert np.array_equal(b, gs.map_indices(ids, N))
        assert np.array_equal(ph, gs.phase_for_ids(b, g[np.ix_(B, B)]))
        _, pa = gs.specialization_map_and_phase(t["lut_a"], ids)
        assert np.array_equal(pa, gs.phase_for_ids(ids, g[np.ix_(A, A)]))
        done += 1


def test_cut_errors(pkg):
    rng = np.random.default_rng(2)
    n = 12
    g = np.zeros((n, n), dtype=np.uint8)  # empty graph: rank 0
    u = pkg.instances.haar_su2(n, rng)
    with pytest.raises(ValueError, match="not uniform"):
        pkg.samplers.cut_tables(g, u, list(range(6)), list(range(6, 12)))
    with pytest.raises(ValueError):
        pkg.samplers.cut_tables(pkg.instances.dense(n, rng), u, list(range(6)), list(range(5, 11)))
    with pytest.raises(ValueError):
        pkg.samplers.cut_tables(pkg.instances.dense(6, rng), u[:6], [0, 1, 2], [3, 4, 5])  # m < 4
