"""CPU checks of the C ABI: the library builds/loads, exports every symbol
declared in include/*.h, and rejects bad arguments on the host side."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols() -> set[str]:
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(b200d2_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_all_declared_symbols(pkg):
    lib = pkg.lib()
    syms = declared_symbols()
    assert len(syms) >= 7
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_host_side_argument_validation(pkg):
    lib = pkg.lib()
    v = pkg.View()
    # NULL projector / NULL out: rejected before any CUDA call
    assert lib.b200d2_projector_view(None, 17, 32, 1, 16, 0, C.byref(v)) == 1
    assert lib.b200d2_projector_destroy(None) == 1
    assert lib.b200d2_projector_dims(None, None, None) == 1
    # NULL buffers to the drop-in
    assert lib.b200d2_diff2_coarse(C.byref(v), None, None, None, None, None, None, None, 1, 1, 1, None, 0) == 1
    assert lib.b200d2_projector_load_dat(b"/nonexistent/projector.dat", 1, C.byref(C.c_void_p())) == 1
    # coarse weights: empty problems are a no-op, missing buffers are rejected
    assert lib.b200d2_coarse_weights(None, 0, 10, 10, None, None, None, 1, None, None, None, 0, None) == 0
    assert lib.b200d2_coarse_weights(None, 2, 10, 10, None, None, None, 1, None, None, None, 0, None) == 1
    assert lib.b200d2_coarse_weights(None, -1, 10, 10, None, None, None, 1, None, None, None, 0, None) == 1
    assert lib.b200d2_ctf_fold(None, None, 10, 0, 10, 6, 10, 5, 10, 1.5, None, None, 0, None, None, None,
                               None) == 0
    assert lib.b200d2_ctf_fold(None, None, 10, 2, 10, 6, 10, 5, 10, 1.5, None, None, 0, None, None, None,
                               None) == 1
    assert lib.b200d2_set_gemm_variant(96, 0, 0, 0) == 1 and lib.b200d2_set_gemm_variant(0, 192, 0, 0) == 1
    assert lib.b200d2_set_gemm_variant(0, 0, 0, 3) == 1
    assert lib.b200d2_set_gemm_variant(0, 0, 0, 0) == 0
    # significance: nothing to do for no particles; missing outputs, NaN
    # fraction, oversized rows and short workspaces rejected before any launch
    assert lib.b200d2_significance(None, 0, 10, None, 0.999, 0, None, None, None, None, 0, None) == 0
    assert lib.b200d2_significance(None, 2, 10, None, 0.999, 0, None, None, None, None, 0, None) == 1
    assert lib.b200d2_significance(None, 2, 10, None, float("nan"), 0, 8, 8, None, None, 0, None) == 1
    assert lib.b200d2_significance(8, 2, 1 << 27, 8, 0.999, 0, 8, 8, None, 8, 1 << 40, None) == 2
    assert lib.b200d2_significance(8, 2, 10, 8, 0.999, 0, 8, 8, None, 8, 16, None) == 1
    assert lib.b200d2_significance_workspace(0, 10) == 0
    assert lib.b200d2_significance_workspace(2, 1000) >= 2 * 1000 * 8
    assert lib.b200d2_coarse_weights_workspace(0, 100) == 0
    assert lib.b200d2_coarse_weights_workspace(3, 70000) >= 3 * 8 + 3 * 3 * 8 + 3 * 4


def test_no_cpu_fallback_in_product():
    """The product sources never reference the oracle."""
    for path in glob.glob(os.path.join(ROOT, "t2-relion-kernel_b200", "**", "*.*"), recursive=True):
        if path.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
            txt = open(path).read()
            for pat in ("import oracle", "liboracle", "oracle/", "libref_diff2", "orc_"):
                assert pat not in txt, (path, pat)
