"""GPU test of skgpu_run_primary_noalloc, the entry point for host codes that must not allocate
device memory while a segment runs (their memory manager owns the device between phases, or an
implicit synchronisation of cudaMalloc/cudaFree in mid-segment is not acceptable to them).

It runs the same life cycle with its scratch in the library's static device array, so its tallies
must equal those of skgpu_run_primary on the same histories, call after call (the array keeps the
previous call's contents, which the call itself must reset). Kept in a file of its own that is
collected last.
"""
import numpy as np
import pytest

from skgpu import Scene, SkgpuError, abi

pytestmark = pytest.mark.gpu


def test_noalloc_equals_run_primary_on_two_calls(golden, gpu_backend):
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.instruments[1]["comps"] = 1
    sc.upload(gpu_backend)
    n = 50000  # more histories than the static pool holds: they stream through it
    ref = sc.run(gpu_backend, n, seed=31)
    for _ in range(2):
        gpu_backend.clear_tallies()
        sc.prepare(gpu_backend, n, seed=31)
        abi.run_primary_noalloc(gpu_backend, 0, n, n)
        res = sc.fetch(gpu_backend)
        assert res.counters["histories"] == n
        for a, b in zip(ref.instruments, res.instruments):
            np.testing.assert_allclose(b["total"], a["total"], rtol=1e-9, atol=0)
            np.testing.assert_allclose(b["stats"], a["stats"], rtol=1e-9, atol=0)
            if "components" in a:
                np.testing.assert_allclose(b["components"], a["components"], rtol=1e-9, atol=0)


def test_noalloc_allocates_no_device_memory(golden, gpu_backend):
    """The property the entry point exists for: once the library is loaded and a first call has
    run, a call leaves the device's free memory unchanged."""
    import torch
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.upload(gpu_backend)
    n = 40000
    gpu_backend.clear_tallies()
    sc.prepare(gpu_backend, n, seed=3)
    abi.run_primary_noalloc(gpu_backend, 0, n, n)
    torch.cuda.mem_get_info(0)  # the first query sets up torch's own CUDA state
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    abi.run_primary_noalloc(gpu_backend, 0, n, n)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_noalloc_rejects_scenes_beyond_its_scratch(golden, gpu_backend):
    sc = Scene.from_export(golden("shell_c16.npz"))
    frame = sc.instruments[0]
    extra = []
    for inc in (10, 50, 70, 80):  # four more observers: five groups
        f = dict(frame)
        th = np.radians(inc)
        f["kobs"] = (np.sin(th), 0.0, np.cos(th))
        f["same_observer"] = 0
        extra.append(f)
    sc.instruments = sc.instruments + extra
    sc.upload(gpu_backend)
    sc.prepare(gpu_backend, 1000)
    with pytest.raises(SkgpuError) as e:
        abi.run_primary_noalloc(gpu_backend, 0, 1000, 1000)
    assert e.value.code == abi.ERR_ARG
