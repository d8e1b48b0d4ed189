"""The C-ABI library loads and exports every symbol the public headers declare (CPU, no compute calls)."""
import ctypes
import os
import re

from sabertooth_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("sabertooth_b200.h",):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(st_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_the_headers():
    assert declared_functions() <= set(_lib.SIGNATURES)


def test_struct_layouts_match_the_header():
    assert ctypes.sizeof(_lib.st_pair) == 16
    assert ctypes.sizeof(_lib.st_lane) == 16
    assert ctypes.sizeof(_lib.st_hit) == 12
    assert _lib.PAIR_DTYPE.itemsize == 16 and _lib.LANE_DTYPE.itemsize == 16 and _lib.HIT_DTYPE.itemsize == 12


def test_errors_are_reported_not_raised_in_c():
    # st_init on a machine without a usable device (or with a bad ordinal) returns NULL and sets the message
    h = _lib.lib.st_init(1 << 20, 0)
    assert not h
    assert _lib.lib.st_last_error()
    # calls on a null context fail with EINVAL and a message
    assert _lib.lib.st_synchronize(None) == -1
    assert b"null context" in _lib.lib.st_last_error()


def test_tile_classes_are_listed():
    from sabertooth_b200 import tile_classes
    cls = tile_classes()
    assert (32, 16, 2) in cls and (4, 8, 4) in cls
    for g, r, c in cls:
        assert g in (4, 8, 16, 32) and r % 4 == 0 and 8 <= r <= 32 and c in (1, 2, 4)
