"""CPU tests of the batched-workload description and the batch entry points (no GPU work)."""
import numpy as np
import pytest

from skgpu import abi, batch, workloads


def test_tetra_batch_spec_is_seeded_and_in_range():
    a = workloads.tetra_batch_spec()
    b = workloads.tetra_batch_spec()
    assert a == b and len(a) == 16
    for s in a:
        assert 1e4 <= s["num_vertices"] <= 4e5
        assert 0.1 <= s["tau_v"] <= 10
        assert 1e6 <= s["packets"] <= 1e7
    assert len({s["seed"] for s in a}) == 16


def test_galaxy_tetra_scene_is_consistent():
    sc = workloads.galaxy_tetra(3000, tau_v=2.0, seed=4, npix=16, nlambda=8)
    g = sc.grid
    assert g["kind"] == abi.GRID_TETRA
    assert len(sc.density) == len(g["tetra"]) and np.all(sc.density >= 0)
    assert len(g["vertices"]) == 3000 + 8
    assert sc.instruments[0]["num_bins"] == 8


def test_run_batch_checks_its_arguments():
    with pytest.raises(ValueError):
        batch.run_batch([object()], [], [1], [1])


def test_batch_symbols_exported():
    lib = abi.load_library()
    for name in ("skgpu_run_batch", "skgpu_set_launch_shape"):
        assert hasattr(lib, name)


def test_autotune_descends_to_the_fastest_shape(monkeypatch):
    """The coordinate descent of skgpu.batch.autotune on a fake timing model: it visits every
    candidate of each knob with the others fixed, keeps the fastest, and leaves that shape set."""
    state = {"shape": (0, 0, 0), "refill": 0}
    monkeypatch.setattr(abi, "set_launch_shape", lambda be, p, t, s: state.update(shape=(p, t, s)))
    monkeypatch.setattr(abi, "set_trace_refill", lambda be, r: state.update(refill=r))

    class Fake:
        def last_run_ms(self):
            p, t, s = state["shape"]
            cost = 100.0
            cost -= {0: 0, 1 << 20: 5, 1 << 21: 8, 1 << 22: 10}[p]
            cost -= {0: 0, 1: -20, 2: 3, 3: 1}[t]
            cost -= {0: 0, 2: 1, 4: 2, 8: -1}[s]
            cost -= {0: 0, 8: 4, 16: 1}[state["refill"]]
            return cost

    be = Fake()
    cand = {"pool_slots": [1 << 20, 1 << 21, 1 << 22], "trace_blocks_per_sm": [1, 2, 3], "shade_blocks_per_sm": [2, 4, 8],
            "trace_refill": [8, 16]}
    shape, ms, trials = batch.autotune(be, lambda: None, cand, rounds=2)
    assert shape == {"pool_slots": 1 << 22, "trace_blocks_per_sm": 2, "shade_blocks_per_sm": 4, "trace_refill": 8}
    assert ms == 100.0 - 10 - 3 - 2 - 4
    assert state["shape"] == (1 << 22, 2, 4) and state["refill"] == 8
    assert be.launch_shape == shape
    assert len(trials) >= 1 + 3 + 3 + 3 + 2

    # tuned once per grid kind, then reused without new trials
    batch._TUNED.clear()
    calls = []
    first, tuned = batch.tuned_shape(be, 3, lambda: calls.append(1), cand)
    n = len(calls)
    again, tuned2 = batch.tuned_shape(be, 3, lambda: calls.append(1), cand)
    assert tuned and not tuned2 and again == first and len(calls) == n
    batch._TUNED.clear()
