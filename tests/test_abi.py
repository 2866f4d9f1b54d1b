"""The C-ABI library loads and exports every entry point its header declares
(no compute call: this runs without a GPU)."""
import ctypes
import os
import re

from asohf_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ["asohf_gpu.h"]:
        txt = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"^\s*(?:int|int64_t|const char \*)\s*\*?\s*(asohf_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "asohf_halofind_particles" in names and "asohf_density" in names
    assert len(names) >= 18


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(api.lib_path())
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings():
    build.build()
    L = api.load()
    for code in range(10):
        assert L.asohf_strerror(code).decode()


def test_no_device_fails_loudly():
    """Without a GPU the library refuses to start (ASOHF_ERR_NO_DEVICE): it
    has no CPU fallback."""
    L = api.load()
    ctx = ctypes.c_void_p()
    rc = L.asohf_create(0, ctypes.byref(ctx))
    import torch
    if torch.cuda.is_available():
        assert rc == 0
        L.asohf_destroy(ctx)
    else:
        assert rc == 7  # ASOHF_ERR_NO_DEVICE
        assert "device" in L.asohf_strerror(rc).decode().lower()
        # the context-free entry point reports the same status
        dummy = ctypes.c_float()
        fn = L.asohf_density_base_noalloc
        rc = fn(1, ctypes.c_float(1.0), ctypes.c_float(1.0), ctypes.c_float(1.0), ctypes.c_float(1.0), 2,
                ctypes.c_int64(0), None, None, None, None, ctypes.byref(dummy), None)
        assert rc == 7


def test_cleaning_and_mesh_entry_points_reject_a_null_context():
    """Argument checks of the catalogue cleaning and mesh entry points come
    before any device work (ASOHF_ERR_INVALID = 1)."""
    L = api.load()
    p = ctypes.c_void_p()
    i32 = ctypes.c_int32()
    nh = (ctypes.c_int32 * 2)(1, 1)
    assert L.asohf_check_rubish(None, p, 0, 1, 1, 0, ctypes.byref(i32)) == 1
    assert L.asohf_accidental_substructure(None, p, 0, 0, ctypes.byref(i32)) == 1
    assert L.asohf_overlapping(None, p, 1, nh, ctypes.c_float(0.2), 0, ctypes.byref(i32)) == 1
    assert L.asohf_mesh_base_counts(None, 8, ctypes.c_float(1.0), 8, 1, nh, p, 0) == 1
    assert L.asohf_mesh_patch_counts(None, 8, ctypes.c_float(8.0), ctypes.c_float(1.0), 1, 8, 1, nh, 0,
                                     None, None, None, None, None, None, None, 0) == 1
    assert L.asohf_veinsgrid_reduced(None, 1, ctypes.c_float(1.0), ctypes.c_float(-3.5), 0, None, None, None,
                                     None, None, None, 100, None, None, 0) == 1
