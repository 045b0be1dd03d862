"""Seeded synthetic instances: graphs, Haar SU(2) gates, scan orders, bitstrings.

All randomness flows from ``numpy.random.default_rng(seed)``.  The graph kinds are
those of the benchmark workloads: random 3-regular (configuration model, loops and
multi-edges rejected), Erdos-Renyi G(n, 3/(n-1)) and random degree<=3.
"""
import numpy as np

__all__ = ["regular3", "erdos_renyi", "degree_at_most3", "dense", "haar_su2", "uniform_bits", "Instance",
           "make_instance", "order_with_rank"]


def regular3(n, rng):
    if n % 2 or n < 4:
        raise ValueError("3-regular graphs need an even n >= 4")
    while True:
        stubs = rng.permutation(np.repeat(np.arange(n), 3)).reshape(-1, 2)
        if np.any(stubs[:, 0] == stubs[:, 1]):
            continue
        key = np.sort(stubs, axis=1)
        if len(np.unique(key[:, 0] * n + key[:, 1])) != len(key):
            continue
        g = np.zeros((n, n), dtype=np.uint8)
        g[key[:, 0], key[:, 1]] = 1
        return g | g.T


def erdos_renyi(n, rng, avg_degree=3.0):
    p = min(1.0, avg_degree / max(n - 1, 1))
    g = np.triu((rng.random((n, n)) < p).astype(np.uint8), 1)
    return g | g.T


def degree_at_most3(n, rng, edge_fraction=1.0):
    """Random graph with maximum degree 3: random edge insertions that respect the cap."""
    g = np.zeros((n, n), dtype=np.uint8)
    deg = np.zeros(n, dtype=np.int64)
    target = int(edge_fraction * 3 * n / 2)
    tries = 0
    edges = 0
    while edges < target and tries < 50 * n:
        tries += 1
        a, b = rng.integers(0, n, 2)
        if a == b or g[a, b] or deg[a] >= 3 or deg[b] >= 3:
            continue
        g[a, b] = g[b, a] = 1
        deg[a] += 1
        deg[b] += 1
        edges += 1
    return g


def dense(n, rng):
    g = np.triu(rng.integers(0, 2, (n, n), dtype=np.uint8), 1)
    return g | g.T


def haar_su2(n, rng):
    """n Haar-random SU(2) matrices: QR of a complex Gaussian, phase-fixed, det = 1."""
    z = rng.normal(size=(n, 2, 2)) + 1j * rng.normal(size=(n, 2, 2))
    out = np.empty((n, 2, 2), dtype=np.complex128)
    for i in range(n):
        q, r = np.linalg.qr(z[i])
        q = q * (np.diag(r) / np.abs(np.diag(r)))
        out[i] = q / np.sqrt(np.linalg.det(q))
    return out


def uniform_bits(count, n, rng):
    return rng.integers(0, 2, (count, n), dtype=np.uint8)


class Instance:
    """(graph, unitaries, order) with its rank profile."""

    def __init__(self, g, u, order, ranks, name=""):
        self.g, self.u, self.order, self.ranks, self.name = g, u, list(order), list(ranks), name
        self.n = len(g)

    @property
    def rmax(self):
        return max(self.ranks)

    @property
    def sum_states(self):
        return int(sum(1 << r for r in self.ranks))

    def describe(self):
        return {"name": self.name, "n": self.n, "edges": int(self.g.sum() // 2), "rmax": self.rmax,
                "sum_states": self.sum_states}


def order_with_rank(g, target, seeds, rank_fn):
    """Among seeded random orders, the one whose max rank is closest to ``target``
    (ties: larger rank, then lower seed).  Returns (order, ranks, seed)."""
    n = len(g)
    edges = list(zip(*np.nonzero(np.triu(g, 1))))
    best = None
    for s in seeds:
        order = np.random.default_rng(s).permutation(n).tolist()
        ranks = rank_fn(n, edges, order)
        key = (abs(max(ranks) - target), -max(ranks), s)
        if best is None or key < best[0]:
            best = (key, order, ranks, s)
        if max(ranks) == target:
            break
    return best[1], best[2], best[3]


def make_instance(kind, n, seed, rank_fn, target_rank=None, order_seeds=range(1000, 1256)):
    """Seeded instance; the order is a seeded random permutation, or the one closest to
    ``target_rank`` among ``order_seeds`` when a target is given."""
    rng = np.random.default_rng(seed)
    g = {"reg3": regular3, "er3": erdos_renyi, "deg3": degree_at_most3, "dense": dense}[kind](n, rng)
    u = haar_su2(n, rng)
    edges = list(zip(*np.nonzero(np.triu(g, 1))))
    if target_rank is None:
        order = rng.permutation(n).tolist()
        ranks = rank_fn(n, edges, order)
        name = f"{kind}-n{n}-seed{seed}"
    else:
        order, ranks, oseed = order_with_rank(g, target_rank, order_seeds, rank_fn)
        name = f"{kind}-n{n}-seed{seed}-order{oseed}"
    return Instance(g, u, order, ranks, name)
