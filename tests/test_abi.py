"""The C ABI: the shared library loads without a GPU and exports every entry
point that include/tigergrav_b200.h declares (no compute calls)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "tigergrav_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+char\s*\*|int64_t|int)\s*(tg_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_api():
    names = declared()
    assert len(names) >= 30
    for core in ("tg_create", "tg_solve_gravity", "tg_forward", "tg_backward", "tg_gravity_PP_ewald"):
        assert core in names


def test_library_exports_every_declared_symbol():
    from tigergrav_b200 import _lib
    missing = [n for n in declared() if not hasattr(_lib.lib, n)]
    assert not missing, missing
    assert set(declared()) <= set(_lib.EXPORTS), sorted(set(declared()) - set(_lib.EXPORTS))


def test_error_strings_without_gpu():
    from tigergrav_b200 import _lib
    assert _lib.lib.tg_error_string(_lib.TG_OK) == b"ok"
    assert b"TG_NOALLOC_MAX_N" in _lib.lib.tg_error_string(_lib.TG_ERR_SIZE)
    assert _lib.lib.tg_version().startswith(b"tigergrav_b200")
