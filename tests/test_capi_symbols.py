"""The C-ABI library loads and exports every entry point include/sbd_tpb.h declares.

Runs without a GPU: it only loads the shared object and resolves symbols (no compute call).
"""
import ctypes
import os
import re

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "sbd_tpb.h")).read()
    return sorted(set(re.findall(r"SBD_TPB_API\s+[\w\s\*]*?\b(sbd_tpb_\w+)\s*\(", text)))


def test_library_exports_header():
    import sbd_tpb
    lib = ctypes.CDLL(sbd_tpb.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(sbd_tpb.EXPORTED) == sorted(n for n in names if n in sbd_tpb.EXPORTED)


def test_binding_declares_every_symbol():
    import sbd_tpb
    assert set(declared_symbols()) <= set(sbd_tpb.EXPORTED)


def test_no_device_returns_status():
    """Without a CUDA device, creating a handle must fail with a status, not crash."""
    import torch
    if torch.cuda.is_available():
        return
    import sbd_tpb
    h = ctypes.c_void_p()
    rc = sbd_tpb.lib().sbd_tpb_create(0, ctypes.byref(h))
    assert rc == sbd_tpb.ERR_NO_DEVICE
    assert b"device" in sbd_tpb.lib().sbd_tpb_last_error()
