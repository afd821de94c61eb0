"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle (oracle/_build/liboracle.so).

The oracle exports the same entry points as the CUDA library with the prefix ``or_``, so tests
drive it through skgpu.abi.Backend exactly like the GPU tracer.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


def library():
    if not os.path.exists(LIB):
        raise RuntimeError(f"oracle not built: {LIB} (make -C oracle)")
    return C.CDLL(LIB)


def backend():
    from skgpu.abi import Backend
    return Backend(library(), prefix="or_")


def philox(ctr, key):
    lib = library()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.or_philox4x32_10(c, k, o)
    return list(o)
