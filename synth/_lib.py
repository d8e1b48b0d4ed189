"""ctypes binding of synth/libsynth.so (synth/pssm.h), built on first use with the Makefile beside it."""
import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsynth.so")
_P = C.c_void_p


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load():
    srcs = [os.path.join(HERE, f) for f in ("pssm.cpp", "pssm.h")]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs):
        build()
    lib = C.CDLL(LIB_PATH)
    lib.st_pssm_from_msa.restype = C.c_int
    lib.st_pssm_from_msa.argtypes = [_P, C.c_uint32, C.c_uint32, _P, _P, C.c_float, C.c_float, C.c_float, _P, _P]
    lib.st_pssm_batch.restype = C.c_int
    lib.st_pssm_batch.argtypes = [_P, _P, _P, _P, C.c_uint32, _P, _P, C.c_float, C.c_float, C.c_float, _P, _P,
                                  C.c_int]
    return lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


lib = _load()
