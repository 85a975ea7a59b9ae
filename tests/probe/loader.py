"""ctypes binding of libtb_probe.so (tb_probe.h): the FP64 FMA throughput
probe and the device-math probe, test and measurement helpers that are not
part of the product library.  `load()` builds the library with the Makefile
beside it when it is missing."""
import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, 'libtb_probe.so')
_lib = None


def build():
    subprocess.check_call(['make', '-s', '-C', HERE, 'all'])
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.tb_probe_fp64_fma.argtypes = [C.c_int, C.c_int64, C.c_void_p, C.c_void_p]
        lib.tb_probe_fp64_fma.restype = C.c_int
        lib.tb_probe_math.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_void_p]
        lib.tb_probe_math.restype = C.c_int
        _lib = lib
    return _lib
