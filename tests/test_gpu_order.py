"""Wavelength-ordered launch (skgpu_set_history_order): taking up the histories in order of their
launch wavelength changes which histories share the pool, not any history, so the tallies equal
those of index order up to the order of FP64 additions; on both walker precisions, with the
radiation field and statistics, and in batches."""
import numpy as np
import pytest

from skgpu import Backend, abi, batch, workloads

pytestmark = pytest.mark.gpu


def _same(ra, rb, rtol=1e-9):
    for a, b in zip(ra.instruments, rb.instruments):
        assert np.allclose(a["total"], b["total"], rtol=rtol, atol=0)
        if a["stats"] is not None:
            assert np.allclose(a["stats"], b["stats"], rtol=rtol, atol=0)
    if ra.rf is not None:
        assert np.allclose(ra.rf, rb.rf, rtol=rtol, atol=0)
    assert ra.counters["histories"] == rb.counters["histories"]
    assert ra.counters["crossings"] == rb.counters["crossings"]


@pytest.mark.parametrize("precision", [abi.PREC_FP64_EXACT, abi.PREC_FP32])
def test_wavelength_order_equals_index_order(gpu_backend, precision):
    sc = workloads.galaxy_octree(npix=32, nlambda=20, max_level=5, max_dust_fraction=1e-4, stats=True)
    sc.upload(gpu_backend)
    abi.set_launch_shape(gpu_backend, 8192, 0, 0)  # a pool far smaller than the segment: ordering applies
    n = 60000
    abi.set_history_order(gpu_backend, abi.ORDER_INDEX)
    r0 = sc.run(gpu_backend, n, seed=31, precision=precision)
    abi.set_history_order(gpu_backend, abi.ORDER_WAVELENGTH)
    r1 = sc.run(gpu_backend, n, seed=31, precision=precision)
    _same(r0, r1)
    # a segment of the range, not starting at 0
    abi.set_history_order(gpu_backend, abi.ORDER_INDEX)
    s0 = sc.run(gpu_backend, n, seed=31, precision=precision, first=10000, count=30000)
    abi.set_history_order(gpu_backend, abi.ORDER_WAVELENGTH)
    s1 = sc.run(gpu_backend, n, seed=31, precision=precision, first=10000, count=30000)
    _same(s0, s1)


def test_wavelength_order_in_batches():
    scenes = [workloads.galaxy_tetra(3000 + 1000 * i, 1.0 + i, 40 + i, npix=24, nlambda=8) for i in range(3)]
    packets, seeds = [20000, 35000, 15000], [3, 4, 5]
    bes = [Backend() for _ in scenes]
    try:
        for sc, be in zip(scenes, bes):
            sc.upload(be)
        abi.set_launch_shape(bes[0], 4096, 0, 0)
        abi.set_history_order(bes[0], abi.ORDER_INDEX)
        r0 = batch.run_batch(scenes, bes, packets, seeds, abi.PREC_FP32)
        abi.set_history_order(bes[0], abi.ORDER_WAVELENGTH)
        r1 = batch.run_batch(scenes, bes, packets, seeds, abi.PREC_FP32)
        for a, b in zip(r0, r1):
            for ia, ib in zip(a.instruments, b.instruments):
                assert np.allclose(ia["total"], ib["total"], rtol=1e-9, atol=0)
    finally:
        for be in bes:
            be.close()


def test_history_order_rejects_unknown_modes(gpu_backend):
    with pytest.raises(abi.SkgpuError):
        abi.set_history_order(gpu_backend, 7)
