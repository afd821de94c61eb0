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
blocks per SM, and the number of waiting lanes at which a traversal warp takes new tasks) that gives
the shortest device time for a given run, by coordinate descent over the candidates.
`tuned_shape` runs it once per grid kind and keeps the result: later calls for a scene of the same
grid kind set the stored shape on the backend without tuning again.
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
    "trace_refill": [4, 8, 12, 16, 24],
}

KNOBS = ("pool_slots", "trace_blocks_per_sm", "shade_blocks_per_sm", "trace_refill")


def apply_shape(be, shape):
    """Sets a launch shape (dict of KNOBS; missing or 0 entries keep the defaults) on a backend."""
    abi.set_launch_shape(be, shape.get("pool_slots", 0), shape.get("trace_blocks_per_sm", 0),
                         shape.get("shade_blocks_per_sm", 0))
    abi.set_trace_refill(be, shape.get("trace_refill", 0))
    be.launch_shape = dict(shape)


def autotune(be, run, candidates=None, repeats=1, rounds=2):
    """Coordinate descent over the launch shape of backend `be`: for each knob in turn, every
    candidate value is tried with the others fixed and the one with the shortest device time
    (skgpu_last_run_ms after `run()`) kept; `rounds` sweeps. Leaves the best shape set and returns
    (shape dict, best ms, trials list)."""
    cand = dict(DEFAULT_CANDIDATES if candidates is None else candidates)
    shape = {k: 0 for k in KNOBS}
    trials = []

    def measure(s):
        apply_shape(be, s)
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
    apply_shape(be, shape)
    return shape, best, trials


_TUNED = {}  # grid kind -> launch shape found by autotune


def tuned_shape(be, grid_kind, run, candidates=None, repeats=1, rounds=2):
    """The launch shape for scenes of `grid_kind`: tuned by `autotune` with `run` the first time a
    grid kind is seen in this process, then reused. Sets it on the backend and returns
    (shape, tuned now)."""
    if grid_kind in _TUNED:
        apply_shape(be, _TUNED[grid_kind])
        return _TUNED[grid_kind], False
    shape, _, _ = autotune(be, run, candidates, repeats, rounds)
    _TUNED[grid_kind] = shape
    return shape, True


def _timed(be, run):
    run()
    return be.last_run_ms()
