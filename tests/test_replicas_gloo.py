"""Replica parallelism on CPU: two ranks over gloo (127.0.0.1) split the bitstrings of an
instance, evaluate their shards with the CPU oracle, reduce their times (max over ranks)
and gather the results; the gathered amplitudes equal one process evaluating all of them.
Also the shard and seed-stream helpers on their own."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, size, port, out_dir):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    import __graft_entry__
    from oracle import scan_plan as sp
    pkg = __graft_entry__.package()
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=60))
    try:
        r, n = pkg.replicas.world()
        assert (r, n) == (rank, size)
        inst = pkg.instances.make_instance("reg3", 10, 5, pkg.rank_profile)
        bits = pkg.instances.uniform_bits(37, 10, np.random.default_rng(5))
        lo, hi = pkg.replicas.shard(len(bits), rank, size)
        amps = [sp.amplitude(inst.g, inst.u, inst.order, b.tolist()) for b in bits[lo:hi]]
        t = pkg.replicas.max_over_ranks(1.0 + rank)
        parts = pkg.replicas.gather((lo, hi, amps))
        if rank == 0:
            np.save(Path(out_dir) / "gathered.npy", np.array([a for _, _, a in parts for a in a], dtype=complex))
            np.save(Path(out_dir) / "bounds.npy", np.array([(a, b) for a, b, _ in parts]))
            np.save(Path(out_dir) / "t.npy", np.array([t]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_over_gloo(pkg, tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    from oracle import scan_plan as sp
    inst = pkg.instances.make_instance("reg3", 10, 5, pkg.rank_profile)
    bits = pkg.instances.uniform_bits(37, 10, np.random.default_rng(5))
    ref = np.array([sp.amplitude(inst.g, inst.u, inst.order, b.tolist()) for b in bits])
    got = np.load(tmp_path / "gathered.npy")
    assert np.array_equal(got, ref)
    assert np.load(tmp_path / "bounds.npy").tolist() == [[0, 19], [19, 37]]
    assert float(np.load(tmp_path / "t.npy")[0]) == 2.0


def test_shards_and_seed_streams(pkg):
    for count in (0, 1, 7, 64, 65537):
        for size in (1, 2, 3, 8):
            bounds = [pkg.replicas.shard(count, r, size) for r in range(size)]
            assert bounds[0][0] == 0 and bounds[-1][1] == count
            assert all(bounds[i][1] == bounds[i + 1][0] for i in range(size - 1))
            sizes = [b - a for a, b in bounds]
            assert max(sizes) - min(sizes) <= 1
    seeds = pkg.replicas.rank_seeds(20261030, 8)
    assert len(set(seeds)) == 8 and seeds == pkg.replicas.rank_seeds(20261030, 8)
    assert pkg.replicas.rank_seeds(20261030, 2) == seeds[:2]
    with pytest.raises(ValueError):
        pkg.replicas.shard(10, 2, 2)
    assert pkg.replicas.world() == (0, 1) and pkg.replicas.max_over_ranks(3.5) == 3.5
