"""skgpu: host side of the B200 photon-packet life-cycle tracer for SKIRT 9.

The compute path is the CUDA library lib/libskgpu.so (C ABI in include/skgpu.h); this package
binds it with ctypes (`abi`), describes scenes in the ABI layout (`scene`), builds the named
workloads (`workloads`), writes ski files for the reference (`ski`) and sums a segment's tallies
over ranks (`sharding`).
"""
from .abi import Backend, SkgpuError, load_library  # noqa: F401
from .scene import Scene, Results  # noqa: F401
