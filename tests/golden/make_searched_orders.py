"""Scan orders found by this package's own order search (not reference data), stored so
benchmarks can use them without spending the search time.  Deterministic: the search is
seeded and iteration-bounded.

    python tests/golden/make_searched_orders.py      (from the repository root; ~40 s)
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import __graft_entry__  # noqa: E402

SEARCHES = {"rgs70": {"start": "rgs70/scan_order", "max_rank": 30, "iterations": 2000000, "seed": 5, "threads": 16}}


def main():
    pkg = __graft_entry__.package()
    fx = np.load(ROOT / "tests" / "golden" / "fixtures.npz")
    out = {}
    for name, cfg in SEARCHES.items():
        g = fx[f"{name}/graph"]
        edges = pkg.edges_from_graph(g)
        start = fx[cfg["start"]].tolist()
        order, ranks, cost = pkg.search_order(len(g), edges, start, max_rank=cfg["max_rank"],
                                              iterations=cfg["iterations"], seed=cfg["seed"], threads=cfg["threads"])
        out[name] = dict(cfg, order=order, ranks=ranks, sum_states=int(cost))
        print(name, int(cost), max(ranks))
    (ROOT / "tests" / "golden" / "searched_orders.json").write_text(json.dumps(out))


if __name__ == "__main__":
    main()
