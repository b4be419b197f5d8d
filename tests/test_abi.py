"""The C-ABI library: it loads without a GPU, exports every entry point that
include/*.h declares, and its host-only functions behave. No kernel is launched."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols() -> set:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*(?:[\w\*\s]+?)\b(helio_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol(native_built):
    from helio_b200 import native as N

    lib = C.CDLL(str(N.CULL_LIB))
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing, missing
    assert len(declared_symbols()) >= 30
    # the ctypes table covers every declared entry point
    assert declared_symbols() <= set(N.CULL_EXPORTS), declared_symbols() - set(N.CULL_EXPORTS)


def test_host_functions_without_gpu(native_built):
    from helio_b200 import native as N
    from oracle import oracle as O

    lib = N.cull_lib()
    assert lib.helio_abi_version() == 1
    assert lib.helio_status_string(N.HELIO_ERR_CAPACITY) == b"capacity exceeded"
    vp = np.random.default_rng(0).standard_normal(16).astype(np.float32)
    got = np.zeros(24, np.float32)
    lib.helio_extract_frustum_planes(vp.ctypes.data, got.ctypes.data)
    np.testing.assert_array_equal(got.view(np.uint32), O.extract_frustum_planes(vp).view(np.uint32))


def test_invalid_arguments_are_reported_not_raised(native_built):
    from helio_b200 import native as N

    lib = N.cull_lib()
    h = C.c_void_p()
    cfg = N.HizConfig(0, 0, 0)
    assert lib.helio_hiz_create(C.byref(cfg), C.byref(h)) == N.HELIO_ERR_INVALID_ARG
    assert b"1..32768" in lib.helio_last_error()
    vcfg = N.VgConfig(64, 64, 1, 0, 5, 0)
    assert lib.helio_vg_create(C.byref(vcfg), C.byref(h)) == N.HELIO_ERR_INVALID_ARG
    assert lib.helio_vg_prepare(None, None, None) == N.HELIO_ERR_INVALID_ARG
    # Folding a shadow cull pass into a batch needs a batch.
    assert lib.helio_batch_attach_shadow(None, None) == N.HELIO_ERR_INVALID_ARG
    assert lib.helio_shadow_cull_prepare(None, None) == N.HELIO_ERR_INVALID_ARG


def test_noalloc_rejects_misaligned_levels_before_any_launch(native_built):
    """helio_hiz_build_noalloc stores level 1 as float2 pairs, so a levels pointer that
    is not 16-byte aligned is refused before any CUDA call (no GPU needed here)."""
    from helio_b200 import native as N

    lib = N.cull_lib()
    view = (N.HizViewInput * 1)(N.HizViewInput(0x10000, 64, 64, 64, 0))
    pyr = (N.HizPyramid * 1)()
    st = lib.helio_hiz_build_noalloc(1, view, C.c_void_p(0x10000 + 4), 1 << 20, pyr, None)
    assert st == N.HELIO_ERR_INVALID_ARG
    assert b"16-byte aligned" in lib.helio_last_error()
