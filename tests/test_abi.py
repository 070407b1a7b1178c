"""The C ABI library loads and exports every entry point include/tontofock.h declares
(no device calls: runs without a GPU)."""

import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    import glob
    txt = "".join(open(f).read() for f in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tf_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_core_entry_points():
    syms = declared_symbols()
    for s in ["tf_ctx_create", "tf_build_jk", "tf_build_fock", "tf_set_geometry", "tf_ctx_destroy",
              "tf_error_string", "tf_last_stats", "tf_build_jk_batch", "tf_build_jk_device"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    from tonto_b200 import build
    lib = build.build()
    L = ctypes.CDLL(lib)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_error_strings_without_device():
    from tonto_b200 import fock
    L = fock.load_library()
    assert L.tf_error_string(0) == b"ok"
    assert b"invalid" in L.tf_error_string(-1)
    assert L.tf_version().startswith(b"tontofock")
    o = fock.default_options()
    assert o.eri_schwarz_cutoff == 1e-9 and o.eri_primitive_pair_cutoff == 1e-6
