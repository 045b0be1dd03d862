"""Two-shard conditional sampler on CPU: the shard-local computation (top bit's Walsh
factor folded into the initialisation, every other operation local) restated in the
oracle and pinned to the reference's deferred state and the conditional vector, and the
cross-shard draw protocol in one process and over two gloo ranks (127.0.0.1)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp
from scipy import stats

from oracle import graph_state as gs

ROOT = Path(__file__).resolve().parent.parent


class HostShard:
    """A shard held as a host array, with the GPU shard's draw rule: tiles of 2^12 values
    (or the whole shard), tile by u1 over the tile masses, element by u2 inside."""

    def __init__(self, v, tile_bits=12):
        self.v = np.asarray(v, dtype=np.complex128)
        self.half = len(self.v)
        self.tb = min(tile_bits, int(np.log2(self.half)))
        p = np.abs(self.v) ** 2
        self.tile_mass = p.reshape(-1, 1 << self.tb).sum(axis=1)

    def mass(self):
        return float(self.tile_mass.sum())

    def local_draw(self, u1, u2):
        t = int(np.searchsorted(np.cumsum(self.tile_mass), u1 * self.mass(), side="right"))
        p = np.abs(self.v[t << self.tb:(t + 1) << self.tb]) ** 2
        w = int(np.searchsorted(np.cumsum(p), u2 * p.sum(), side="right"))
        return (t << self.tb) + w

    def value(self, local):
        return complex(self.v[local])


def _instance(fixtures, name):
    return (fixtures[f"{name}/graph"], fixtures[f"{name}/measurement_unitaries"], fixtures[f"{name}/A"].tolist(),
            fixtures[f"{name}/B"].tolist())


@pytest.mark.parametrize("name", ["induced_24q", "induced_32q", "induced_40q"])
def test_shards_from_local_operations(fixtures, name):
    g, u, A, B = _instance(fixtures, name)
    rng = np.random.default_rng(len(A))
    for _ in range(2):
        ob = rng.integers(0, 2, len(B)).tolist()
        shards = gs.cpu_shards(g, u, A, B, ob)
        raw, final = gs.cpu_deferred(g, u, A, B, ob)
        assert np.max(np.abs(np.concatenate(shards) - raw)) < 1e-12
        ref, pb = gs.conditional(g, u, A, B, ob)
        assert np.max(np.abs(final - ref / np.sqrt(pb))) < 1e-12


def test_draw_across_shards_is_born_exact(pkg, fixtures):
    g, u, A, B = _instance(fixtures, "induced_24q")
    ob = [0, 1] * (len(B) // 2)
    shards = [HostShard(v, tile_bits=5) for v in gs.cpu_shards(g, u, A, B, ob)]
    _, final = gs.cpu_deferred(g, u, A, B, ob)
    probs = np.abs(final) ** 2
    probs /= probs.sum()
    U = np.asarray(u[A[-1]])
    rng = np.random.default_rng(11)
    draws = []
    for _ in range(20000):
        idx, pa, norm = pkg.samplers.draw_across_shards(shards, U, rng.random(), rng.random(), rng.random())
        assert abs(pa - abs(final[idx]) ** 2) < 1e-12 and abs(norm - 1.0) < 1e-9
        draws.append(idx)
    G = 64
    order = np.argsort(probs, kind="stable")
    cm = np.cumsum(probs[order])
    grp = np.empty(len(probs), np.int64)
    grp[order] = np.minimum((cm * G).astype(np.int64), G - 1)
    e = np.bincount(grp, weights=probs, minlength=G) * len(draws)
    c = np.bincount(grp[np.array(draws)], minlength=G)
    assert stats.chi2.sf(((c - e) ** 2 / e).sum(), G - 1) > 1e-4


def test_shard_choice_edges(pkg):
    sc = pkg.samplers.shard_choice
    assert sc([0.25, 0.75], 0.0)[0] == 0 and sc([0.25, 0.75], 0.2499)[0] == 0
    s, u, norm = sc([0.25, 0.75], 0.5)
    assert s == 1 and abs(u - (0.5 - 0.25) / 0.75) < 1e-15 and norm == 1.0
    assert sc([0.0, 1.0], 0.0)[0] == 1 and sc([1.0, 0.0], 0.999999)[0] == 0
    with pytest.raises(ArithmeticError):
        sc([0.0, 0.0], 0.5)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, port, out_dir, count):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    import __graft_entry__
    pkg = __graft_entry__.package()
    fx = np.load(ROOT / "tests" / "golden" / "fixtures.npz")
    g, u, A, B = (fx["induced_32q/graph"], fx["induced_32q/measurement_unitaries"], fx["induced_32q/A"].tolist(),
                  fx["induced_32q/B"].tolist())
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        ob = [1, 0] * (len(B) // 2)
        shard = HostShard(gs.cpu_shards(g, u, A, B, ob)[rank])
        rng = np.random.default_rng(7) if rank == 0 else None
        out = [pkg.samplers.draw_distributed(shard, np.asarray(u[A[-1]]), rng, rank) for _ in range(count)]
        np.save(Path(out_dir) / f"draws{rank}.npy", np.array(out, dtype=np.float64))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_draw_distributed_over_gloo(pkg, fixtures, tmp_path):
    """Two ranks, one shard each; only scalars cross: every rank returns the same draws,
    equal to the single-process draw over both shards with the same uniforms."""
    count = 64
    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path), count), nprocs=2, join=True, start_method="spawn")
    g, u, A, B = _instance(fixtures, "induced_32q")
    ob = [1, 0] * (len(B) // 2)
    shards = [HostShard(v) for v in gs.cpu_shards(g, u, A, B, ob)]
    rng = np.random.default_rng(7)
    ref = np.array([pkg.samplers.draw_across_shards(shards, np.asarray(u[A[-1]]), rng.random(), rng.random(),
                                                    rng.random()) for _ in range(count)])
    for rank in (0, 1):
        got = np.load(tmp_path / f"draws{rank}.npy")
        assert np.array_equal(got[:, 0], ref[:, 0])
        assert np.allclose(got[:, 1:], ref[:, 1:], rtol=1e-15, atol=0)
