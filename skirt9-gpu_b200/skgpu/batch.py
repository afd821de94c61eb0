"""Batched simulations and launch-shape tuning.

Many small SKIRT simulations (a parameter study, a fitting loop) each leave most of a B200 idle:
their packet pools are too small to fill 148 SMs and each run pays its own launch and drain tail.
`run_batch` traces the primary-emission segments of several independent simulations as one
wavefront (skgpu_run_batch): packets of every simulation share the pool, the traversal kernel and
the stage kernels, and each packet reads its own simulation's grid, medium, sources and tallies.
Every history keeps its own simulation's random stream, so each simulation's tallies equal those
of its own skgpu_run_primary. There is no reference counterpart; the reference runs the
simulations one after another (`skirt` per ski file).

`autotune` picks the launch shape (packet slots in flight, resident traversal blocks per SM, stage
blocks per SM) that gives the shortest device time for a given run, by coordinate descent over
the candidates.
"""
from . import abi


def run_batch(scenes, backends, packets, seeds, precision=abi.PREC_FP32, clear=True, fetch=True):
    """One primary-emission segment of every scene (scene i on backends[i], packets[i] histories,
    random seed seeds[i]) as one wavefront on the first backend's device and stream. Returns each
    scene's Results when `fetch`, else None."""
    n = len(scenes)
    if not (len(backends) == len(packets) == len(seeds) == n):
        raise ValueError("one backend, packet count and seed per scene")
    for sc, be, npp, s in zip(scenes, backends, packets, seeds):
        if clear:
            be.clear_tallies()
        sc.prepare(be, int(npp), int(s), precision)
    abi.run_batch(backends, [0] * n, packets, packets)
    if not fetch:
        return None
    return [sc.fetch(be) for sc, be in zip(scenes, backends)]


DEFAULT_CANDIDATES = {
    "pool_slots": [1 << 20, 1 << 21, 1 << 22],
    "trace_blocks_per_sm": [1, 2, 3, 4, 6, 8],
    "shade_blocks_per_sm": [2, 4, 8, 16],
}


def autotune(be, run, candidates=None, repeats=1, rounds=2):
    """Coordinate descent over the launch shape of backend `be`: for each knob in turn, every
    candidate value is tried with the others fixed and the one with the shortest device time
    (skgpu_last_run_ms after `run()`) kept; `rounds` sweeps. Leaves the best shape set and returns
    (shape dict, best ms, trials list)."""
    cand = dict(DEFAULT_CANDIDATES if candidates is None else candidates)
    shape = {"pool_slots": 0, "trace_blocks_per_sm": 0, "shade_blocks_per_sm": 0}
    trials = []

    def measure(s):
        abi.set_launch_shape(be, s["pool_slots"], s["trace_blocks_per_sm"], s["shade_blocks_per_sm"])
        ms = min(_timed(be, run) for _ in range(max(1, repeats)))
        trials.append((dict(s), ms))
        return ms

    best = measure(shape)
    for _ in range(max(1, rounds)):
        changed = False
        for knob, values in cand.items():
            for v in values:
                if v == shape[knob]:
                    continue
                trial = dict(shape)
                trial[knob] = v
                ms = measure(trial)
                if ms < best:
                    best, shape, changed = ms, trial, True
        if not changed:
            break
    abi.set_launch_shape(be, shape["pool_slots"], shape["trace_blocks_per_sm"], shape["shade_blocks_per_sm"])
    return shape, best, trials


def _timed(be, run):
    run()
    return be.last_run_ms()
