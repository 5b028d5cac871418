"""CPU tests of the C-ABI library: it loads, and it exports every entry point
include/*.h declares (no compute calls; there may be no GPU here)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(lcbi_[A-Za-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "lcbi_gpu_binary_mag0" in names
    assert len(names) >= 5


def test_library_loads_and_exports_every_declared_symbol():
    from lcbinint_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.fail("liblcbinint_b200.so is not built (python -m lcbinint_b200.build)")
    L = _lib.lib()
    exported = set(_lib.exported_symbols())
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for n in declared_symbols():
        assert hasattr(L, n)


@pytest.mark.gpu
def test_library_device_code_is_sm100a():
    """The driver reports the library's kernels as built for compute
    capability 10.0 (sm_100a), the only target the build emits."""
    import ctypes as C
    from lcbinint_b200 import _lib
    v = C.c_int32(0)
    assert _lib.lib().lcbi_gpu_kernel_binary_version(C.byref(v)) == _lib.LCBI_OK
    assert v.value == 100
