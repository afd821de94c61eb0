"""GPU tests of the measurement aids and the tally read-back of the C ABI.

- Stage timing (skgpu_set_stage_timing / skgpu_last_stage_times) brackets the stage kernels with
  CUDA events inside the captured graph; it must not change the results, every stage must report
  one launch per pass, and the stage times must add up to at most the run's device time.
- Tallies larger than one pinned staging chunk (8M doubles) are read back in pipelined chunks and
  added into the caller's arrays; a 512x512x40 frame spans two chunks, and the result must still
  equal the oracle's history by history, and a second fetch into the same array must double it.
"""
import numpy as np
import pytest

from skgpu import Scene, abi

pytestmark = pytest.mark.gpu


def test_stage_timing_does_not_change_results(golden, gpu_backend):
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.upload(gpu_backend)
    n = 20000
    plain = sc.run(gpu_backend, n, seed=5)
    try:
        abi.set_stage_timing(gpu_backend, 2)
        timed = sc.run(gpu_backend, n, seed=5)
        stages = abi.last_stage_times(gpu_backend)
    finally:
        abi.set_stage_timing(gpu_backend, 0)
    for a, b in zip(plain.instruments, timed.instruments):
        np.testing.assert_allclose(b["total"], a["total"], rtol=1e-9, atol=0)
    assert set(stages) == set(abi.STAGES) - {"guide"}  # no guided-scattering stage without guiding
    launches = {k: v[1] for k, v in stages.items()}
    passes = (timed.counters["kernel_launches"] - 1) // 7
    assert all(v == passes for v in launches.values()), launches
    total = sum(v[0] for v in stages.values())
    assert 0 < total <= timed.ms * 1.01
    assert stages["trace"][0] > 0


def test_stage_timing_level_one_times_trace_only(golden, gpu_backend):
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.upload(gpu_backend)
    try:
        abi.set_stage_timing(gpu_backend, 1)
        res = sc.run(gpu_backend, 5000, seed=2)
        stages = abi.last_stage_times(gpu_backend)
    finally:
        abi.set_stage_timing(gpu_backend, 0)
    assert list(stages) == ["trace"]
    # one traversal stage per pass; a pass is 8 kernels with the split traversal of the captured graph
    passes = stages["trace"][1]
    assert res.counters["kernel_launches"] - 1 in (7 * passes, 8 * passes)
    with pytest.raises(abi.SkgpuError):
        abi.set_stage_timing(gpu_backend, 3)


def test_chunked_fetch_of_large_frames_matches_oracle(gpu_backend, oracle_backend):
    from skgpu import workloads
    sc = workloads.galaxy_octree(npix=512, nlambda=40, max_level=5, max_dust_fraction=1e-4)
    n = 1500
    sc.upload(gpu_backend)
    sc.upload(oracle_backend)
    rg = sc.run(gpu_backend, n, seed=23)
    ro = sc.run(oracle_backend, n, seed=23)
    for ig, io in zip(rg.instruments, ro.instruments):
        assert ig["total"].size > 8 * 1024 * 1024  # spans more than one staging chunk
        assert ig["total"].sum() == pytest.approx(io["total"].sum(), rel=1e-6)
        close = np.isclose(ig["total"], io["total"], rtol=1e-9, atol=0)
        assert close.mean() >= 0.999
    # a second fetch adds into the caller's array
    size = sc.instrument_size(0)
    out = np.zeros(size)
    gpu_backend.fetch_instrument(0, size, out=out)
    first = out.copy()
    gpu_backend.fetch_instrument(0, size, out=out)
    np.testing.assert_array_equal(out, 2 * first)
    np.testing.assert_array_equal(first, rg.instruments[0]["total"].ravel())
