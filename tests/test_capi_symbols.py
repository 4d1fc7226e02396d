"""The C ABI library loads without a GPU and exports every function that
include/*.h declares; the ctypes binding declares each of them.  No compute
calls are made here."""
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "liblightzk_b200", "liblzk_b200.so")


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \t\*]*?\b(lzk_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def built():
    if not os.path.exists(LIB):
        import liblightzk_b200.build as b
        b.build()
    return LIB


def test_header_declares_functions():
    d = declared()
    assert "lzk_msm_g1" in d and "lzk_status_string" in d
    assert len(d) >= 10


def test_library_exports_every_declared_symbol(built):
    out = subprocess.run(["nm", "-D", "--defined-only", built], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = sorted(declared() - exported)
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_ctypes_binding_covers_header(built):
    from liblightzk_b200 import _capi
    lib = _capi.lib()
    for name in declared():
        assert name in _capi.SIGNATURES, f"{name} missing from the ctypes signature table"
        getattr(lib, name)
    assert lib.lzk_version().decode().startswith("liblzk_b200")
    assert lib.lzk_status_string(-2).decode() == "device out of memory"


def test_pure_host_queries(built):
    from liblightzk_b200 import _capi, msm
    lib = _capi.lib()
    assert lib.lzk_msm_precomp_windows(16) == 16
    assert lib.lzk_msm_precomp_windows(12) == 22
    assert lib.lzk_msm_precomp_windows(13) == 20
    c = msm.autotune_window(1, 1 << 20)
    assert 12 <= c <= 20
    assert msm.workspace_bytes(1, 1 << 20) > (1 << 20) * 16 * 4
