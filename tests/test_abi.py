"""CPU checks of the C ABI: the library loads without a GPU and exports every
function that include/*.h declares; the struct layouts agree with the headers."""
import ctypes
import os
import re

import gsn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(gsn_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(gsn.LIB_PATH)
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string_without_gpu():
    assert b"sm_100a" in gsn.lib().gsn_version()


def test_camera_layout_matches_header():
    # gsn_camera: 4 + 9 + 3 + 2 floats, 2 ints, int64, 3 ints (padded to 8)
    assert ctypes.sizeof(gsn.Camera) == 104
    assert gsn.Camera.pixel_offset.offset == 80
    assert gsn.Camera.tile_offset.offset == 96


def test_invalid_arguments_fail_without_touching_the_gpu():
    L = gsn.lib()
    assert L.gsn_renderer_create(None) != 0
    assert L.gsn_solver_create(None) != 0
    assert L.gsn_sort_pairs_workspace(-1, None) != 0
    # the allocation-free sort checks its arguments and its fixed capacity
    # (16,777,216 pairs) before any device work
    fn = L.gsn_sort_pairs_noalloc
    fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    flag = ctypes.c_int(7)
    assert fn(None, None, None, None, (1 << 24) + 1, 0, 32, ctypes.byref(flag), None) == -4  # GSN_ERR_CAPACITY
    assert flag.value == 0
    assert fn(None, None, None, None, 5, 0, 33, ctypes.byref(flag), None) == -1  # end bit past 32
    assert fn(None, None, None, None, 5, 8, 4, ctypes.byref(flag), None) == -1  # end before begin
    assert fn(None, None, None, None, 5, 0, 32, None, None) == -1  # no result flag
    assert fn(None, None, None, None, 5, 0, 32, ctypes.byref(flag), None) == -1  # no buffers
    assert fn(None, None, None, None, 0, 0, 32, ctypes.byref(flag), None) == 0  # nothing to sort
