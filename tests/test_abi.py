"""The C-ABI library loads without a GPU and exports every symbol declared in include/*.h."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(rgs_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_header(pkg):
    lib = pkg._lib.lib()
    names = declared_symbols()
    assert len(names) >= 12
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # Every declared symbol has a ctypes signature in the binding.
    assert names <= set(pkg._lib.SIGNATURES), sorted(names - set(pkg._lib.SIGNATURES))


def test_library_basics_without_gpu(pkg):
    lib = pkg._lib.lib()
    assert lib.rgs_version().decode().startswith("rgs_b200")
    assert lib.rgs_device_count() >= 0
    # Errors are reported as status codes with a message.
    rc = lib.rgs_plan_compile(0, 0, None, None, None, ctypes.byref(ctypes.c_void_p()))
    assert rc == pkg._lib.RGS_ERR_ARG
    assert b"n must be" in lib.rgs_last_error()


def test_library_is_built_for_sm100a(pkg):
    """The library carries sm_100a device code (cuobjdump is not used: check build flags)."""
    text = (ROOT / "rgs70-classical-challenge_b200" / "build.py").read_text()
    assert "arch=compute_100a,code=sm_100a" in text


def test_product_path_does_not_import_oracle():
    pkg_dir = ROOT / "rgs70-classical-challenge_b200"
    for py in pkg_dir.rglob("*.py"):
        src = py.read_text()
        assert "import oracle" not in src and "from oracle" not in src, py


def _launches(pkg, plan, batch, tile, prec, ws):
    out = ctypes.c_int64()
    pkg._lib.check(pkg._lib.lib().rgs_scan_launch_count(plan.handle, batch, tile, prec, ws, ctypes.byref(out)))
    return out.value


def _segments(plan, lo, hi):
    """Launches of positions [lo, hi): one per position, one per fused pair."""
    pairs = set(plan.pairs)
    count, j = 0, lo
    while j < hi:
        j += 2 if (j in pairs and j + 1 < hi) else 1
        count += 1
    return count


def test_scan_launch_schedule(pkg):
    """Launch count of a sweep: with the full workspace, the low-rank leading and trailing
    positions run once per chunk of tiles; with a one-tile workspace, every segment (a
    position or a fused pair) runs once per tile, plus weights and finalisation."""
    inst = pkg.instances.make_instance("reg3", 40, 40, pkg.rank_profile)
    plan = pkg.ScanPlan(inst.n, pkg.edges_from_graph(inst.g), inst.order)
    n, ranks = inst.n, list(plan.ranks)
    r_in = [0] + ranks[:-1]
    small = [max(a, b) <= 12 for a, b in zip(r_in, ranks)]
    h = 0
    while h < n and small[h]:
        h += 1
    t = n
    while t > h and small[t - 1]:
        t -= 1
    prec = pkg._lib.PREC_C64_F32
    for tile in (8, 64, 256):
        ws = ctypes.c_size_t()
        pkg._lib.check(pkg._lib.lib().rgs_scan_workspace_bytes(plan.handle, tile, prec, ctypes.byref(ws)))
        chunk = max(2, 8192 // tile) * tile
        for batch in (1, tile, chunk, 3 * chunk + 5):
            expect = 0
            for first in range(0, batch, chunk):
                tiles = -(-min(chunk, batch - first) // tile)
                expect += 1 + _segments(plan, 0, h)
                if h < t:
                    expect += tiles * _segments(plan, h, t) + (tiles if t == n else 0)
                if t < n or h == n:
                    expect += _segments(plan, max(t, h), n) + 1
            assert _launches(pkg, plan, batch, tile, prec, ws.value) == expect, (tile, batch)
        # One tile's tables only: the tile-by-tile schedule.
        per_tile = 2 * ((tile << max(ranks)) * 8) + n * tile * (32 + 1 + 8)
        got = _launches(pkg, plan, 1000, tile, prec, per_tile + 4096)
        assert got == -(-1000 // tile) * (_segments(plan, 0, n) + 2)
    assert plan.pairs
