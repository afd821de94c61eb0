"""Batched simulations (skgpu_run_batch): several independent scenes traced as one wavefront must
give every scene the tallies of its own solo run (same histories, same random streams; only the
order of the FP64 atomic additions differs), on the reference-order FP64 walkers and on the
production FP32 walkers, for tetrahedral and Cartesian grids; the launch shape changes nothing
but speed; mismatched batches are refused."""
import numpy as np
import pytest

from skgpu import Backend, SkgpuError, abi, batch, workloads

pytestmark = pytest.mark.gpu


def _tetra_scenes():
    spec = workloads.tetra_batch_spec(num=3, seed=7, min_vertices=2e3, max_vertices=8e3, min_packets=2e4,
                                      max_packets=6e4)
    scenes = [workloads.galaxy_tetra(s["num_vertices"], s["tau_v"], s["point_seed"], npix=32, nlambda=8, store_rf=True)
              for s in spec]
    return scenes, [s["packets"] for s in spec], [s["seed"] for s in spec]


def _shell_scenes():
    scenes = []
    for nb, f in ((16, 1.0), (24, 3.0), (32, 0.3)):
        sc = workloads.shell_cartesian(nb, 32)
        sc.density = sc.density * f
        scenes.append(sc)
    return scenes, [30000, 50000, 20000], [11, 12, 13]


def _assert_same(ra, rb, rtol=1e-9):
    for a, b in zip(ra.instruments, rb.instruments):
        assert np.allclose(a["total"], b["total"], rtol=rtol, atol=0)
        if a["stats"] is not None:
            assert np.allclose(a["stats"], b["stats"], rtol=rtol, atol=0)
    if ra.rf is not None:
        assert np.allclose(ra.rf, rb.rf, rtol=rtol, atol=0)


def _check(scenes, packets, seeds, precision):
    bes = [Backend() for _ in scenes]
    try:
        for sc, be in zip(scenes, bes):
            sc.upload(be)
        solo = [sc.run(be, n, seed=s, precision=precision) for sc, be, n, s in zip(scenes, bes, packets, seeds)]
        hist = sum(r.counters["histories"] for r in solo)
        cross = sum(r.counters["crossings"] for r in solo)
        res = batch.run_batch(scenes, bes, packets, seeds, precision)
        for a, b in zip(solo, res):
            _assert_same(a, b)
        c = bes[0].counters()
        assert c["histories"] == hist and c["crossings"] == cross
        # a small pool (many refills) and other block counts: the same tallies
        abi.set_launch_shape(bes[0], 4096, 1, 2)
        res2 = batch.run_batch(scenes, bes, packets, seeds, precision)
        for a, b in zip(solo, res2):
            _assert_same(a, b)
    finally:
        for be in bes:
            be.close()


@pytest.mark.parametrize("precision", [abi.PREC_FP64_EXACT, abi.PREC_FP32])
def test_batched_tetra_scenes_equal_solo_runs(precision):
    _check(*_tetra_scenes(), precision)


@pytest.mark.parametrize("precision", [abi.PREC_FP64_EXACT, abi.PREC_FP32])
def test_batched_cartesian_scenes_equal_solo_runs(precision):
    _check(*_shell_scenes(), precision)


def test_batch_refuses_mixed_grid_kinds():
    a, b = Backend(), Backend()
    try:
        s1 = workloads.shell_cartesian(8, 16)
        s2 = workloads.galaxy_tetra(2000, 1.0, 3, npix=16, nlambda=4)
        s1.upload(a)
        s2.upload(b)
        with pytest.raises(SkgpuError) as e:
            batch.run_batch([s1, s2], [a, b], [1000, 1000], [1, 2])
        assert e.value.code == abi.ERR_ARG
    finally:
        a.close()
        b.close()


def test_autotune_keeps_results_and_returns_a_shape():
    sc = workloads.galaxy_tetra(5000, 2.0, 5, npix=32, nlambda=8)
    be = Backend()
    try:
        sc.upload(be)
        ref = sc.run(be, 40000, seed=3, precision=abi.PREC_FP32)
        run = lambda: sc.run(be, 40000, seed=3, precision=abi.PREC_FP32)
        shape, ms, trials = batch.autotune(be, run, {"pool_slots": [1 << 14, 1 << 16], "trace_blocks_per_sm": [1, 2],
                                                     "shade_blocks_per_sm": [2, 8], "trace_refill": [4, 24]}, rounds=1)
        assert ms > 0 and len(trials) >= 5 and set(shape) == set(batch.KNOBS)
        _assert_same(ref, sc.run(be, 40000, seed=3, precision=abi.PREC_FP32))
    finally:
        be.close()
