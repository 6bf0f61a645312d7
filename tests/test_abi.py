"""The C ABI library loads and exports every entry point its headers declare
(no compute calls: these run without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(bo_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    syms = declared_symbols()
    assert "bo_create" in syms and "bo_q1_fact_device" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    from bespokeolap_artifacts_b200 import native

    lib = native.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol():
    from bespokeolap_artifacts_b200 import native

    native.lib()
    missing = [s for s in declared_symbols() if s not in native._SIGNATURES]
    assert not missing, missing


def test_build_info_names_sm100a():
    from bespokeolap_artifacts_b200 import native

    assert b"sm_100a" in native.lib().bo_build_info()


def test_create_without_gpu_reports_unsupported():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from bespokeolap_artifacts_b200 import native

    with pytest.raises(native.BoError) as e:
        native.Context(0)
    assert e.value.status == -7


def test_null_context_is_rejected():
    from bespokeolap_artifacts_b200 import native

    lib = native.lib()
    assert lib.bo_synchronize(None) == -1
    assert lib.bo_q1_fact_device(None, None, 0, 3, 2, None) == -1
    assert lib.bo_last_error(None) == b"null context"


def declared_arities():
    out = {}
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(bo_\w+)\s*\(([^;{]*?)\)\s*;", text, flags=re.M | re.S):
            params = m.group(2).strip()
            out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_binding_arities_match_the_header():
    from bespokeolap_artifacts_b200 import native

    arity = declared_arities()
    assert len(arity) >= 60
    wrong = {name: (n, len(native._SIGNATURES[name][1])) for name, n in arity.items()
             if name in native._SIGNATURES and len(native._SIGNATURES[name][1]) != n}
    assert not wrong, wrong


def test_no_alloc_rejects_group_factors_whose_product_wraps():
    """65536 x 65536 wraps to 0 in 32-bit arithmetic; the entry point bounds
    each factor first, so the call is rejected before any CUDA call (no GPU
    needed)."""
    import ctypes as C

    from bespokeolap_artifacts_b200 import native

    lib = native.lib()
    cols = native.FactCols(*([None] * 7), 16)
    for nfa, nfb in ((65536, 65536), (1 << 16, 1 << 15), (9, 1), (1, 9), (-1, 4)):
        assert lib.bo_q1_fact_device_noalloc(C.byref(cols), 0, nfa, nfb, C.c_void_p(16), None, None) == -1
