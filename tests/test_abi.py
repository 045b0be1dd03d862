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
