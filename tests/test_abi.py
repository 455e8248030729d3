"""The C-ABI library loads and exports every entry point include/melgpu.h declares (no GPU needed)."""
import os
import re

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "melgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mel_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_all_declared_symbols(gpu_lib):
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(gpu_lib, n)]
    assert not missing, missing


def test_abi_version(gpu_lib):
    assert gpu_lib.mel_abi_version() == 2


def test_struct_sizes_match_header():
    """ctypes mirrors must have the C layout (mel_contact is exchanged in bulk)."""
    import ctypes
    from melody2d_b200 import abi
    assert ctypes.sizeof(abi.MelContact) == 4 * 8 + 4 * 8 + 8 * 4 + 8 * 13 + 4 * 2 + 8 * 3
    assert abi.CONTACT_DTYPE.itemsize == ctypes.sizeof(abi.MelContact)


def test_errors_are_reported_without_device(gpu_lib):
    """Invalid input is rejected on the host with a message (no device work is attempted)."""
    import ctypes
    from melody2d_b200 import abi
    d = abi.MelModelDesc()
    d.abi_version = 999
    h = ctypes.c_void_p()
    rc = gpu_lib.mel_create(ctypes.byref(d), None, ctypes.byref(h))
    assert rc == 1
    assert b"abi_version" in gpu_lib.mel_last_error_string()
