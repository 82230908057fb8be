"""C-ABI checks that need no GPU: the library builds, loads, and exports every
entry point declared in include/yannq_b200.h with the binding's signature."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "yannq_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(yq_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from yannq_b200 import api

    L = api.lib()
    names = _declared()
    assert len(names) >= 35
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(api.SIGNATURES), set(names) ^ set(api.SIGNATURES)


def test_version_string():
    from yannq_b200 import api

    assert api.lib().yq_version().decode().startswith("yannq_b200")


def test_errors_are_reported_not_raised_in_c():
    """Bad arguments come back as status codes with a message (no crash, no GPU work)."""
    import ctypes as C

    from yannq_b200 import api

    L = api.lib()
    assert L.yq_rbm_dim(None, None) == api.E_ARG
    assert "null" in api.last_error()
    h = C.c_void_p()
    rc = L.yq_ctx_create(-1, C.byref(h))
    assert rc != api.OK and h.value is None
    assert api.last_error()


def test_no_oracle_in_product_library():
    """The product library links nothing from oracle/ (the checker stays test-only)."""
    from yannq_b200 import api

    data = open(api.LIB_PATH, "rb").read()
    assert b"orc_" not in data
    for fn in os.listdir(os.path.join(ROOT, "yannq_b200", "csrc")):
        txt = open(os.path.join(ROOT, "yannq_b200", "csrc", fn)).read()
        assert not re.search(r'#include\s*[<"][^>"]*oracle', txt), fn
        assert "orc_" not in txt and "orc::" not in txt, fn


@pytest.mark.parametrize("header", ["yannq_b200.h"])
def test_header_compiles_as_c(header, tmp_path):
    import subprocess

    src = tmp_path / "t.c"
    src.write_text(f'#include "{header}"\nint main(void) {{ return YQ_OK; }}\n')
    out = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c",
                          str(src), "-o", str(tmp_path / "t.o")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
