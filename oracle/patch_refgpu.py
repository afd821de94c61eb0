"""Build step of the reference's own GPU program (oracle/ref.mk target `refgpu`): copies
SKIRT/core/GpuAcceleration.cpp into oracle/_ref/patched/ with one change, in its driver-symbol loader
`loadVersionedSymbol`, which resolves an entry point by its unversioned name first and by the
versioned name (`cuCtxCreate_v2`, `cuMemAlloc_v2`, `cuMemcpyHtoD_v2`, ...) only when that fails.
Current drivers still export the unversioned names as the legacy 32-bit-handle entry points of
CUDA 3.x, so on this pool's driver the reference's runtime fails at `cuCtxCreate` ("out of
memory") and runs on the CPU. The copy tries the versioned name first, which is the ABI the
reference's code is written against (64-bit CUdeviceptr, CUcontext pointers); nothing else changes.
The reference tree itself is never modified.

    python3 oracle/patch_refgpu.py <reference root> <output directory>
"""
import os
import re
import sys


def main():
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    src = open(os.path.join(ref, "SKIRT", "core", "GpuAcceleration.cpp")).read()
    pat = r"return loadSymbol\(handle, name, function\) \|\| loadSymbol\(handle, versionedName, function\);"
    new, n = re.subn(pat, "return loadSymbol(handle, versionedName, function) || loadSymbol(handle, name, function);", src)
    if n != 1:
        raise SystemExit(f"patch_refgpu: expected one loadVersionedSymbol body, found {n}")
    with open(os.path.join(out, "GpuAcceleration.cpp"), "w") as f:
        f.write(new)


if __name__ == "__main__":
    main()
