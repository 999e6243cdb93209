"""CPU tests of the C-ABI library: it loads without a GPU and exports every declared symbol."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(cav_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("cav_bvh_build", "cav_trace_closest", "cav_trace_any", "cav_bvh_export_nodes", "cav_bvh_free"):
        assert required in names


def test_library_exports_every_declared_symbol():
    import cavalry_b200 as cav

    L = cav.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_without_gpu():
    import cavalry_b200 as cav

    L = cav.lib()
    assert L.cav_status_string(0) == b"ok"
    assert L.cav_version() >= 10000


def test_ctx_create_fails_cleanly_without_gpu():
    import torch

    import cavalry_b200 as cav

    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    st = cav.lib().cav_ctx_create(0, ctypes.byref(h))
    assert st != 0 and not h.value
