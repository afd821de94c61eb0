"""Throughput benchmark of the photon-packet life cycle: packets/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference|reference-gpu] [--workload NAME]

One step = one primary-emission segment of the workload's packets through the C ABI
(skgpu_run_primary): launch, emission peel-off, forced-scattering propagation, radiation-field
storage, scattering peel-off and HG scattering for every history. `value` is device time (CUDA
events on the launch stream, L2 flushed between steps); `e2e` is measured through the same C ABI
with host buffers (medium state uploaded from pinned memory, every instrument tally and the
radiation field added into the caller's host arrays, every step). The roofline is that of the
traversal kernel, whose launches are bracketed by CUDA events inside the timed steps. Under
torchrun each rank traces its own contiguous range of history indices (weak scaling; no
data-path collective).
"""
import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "skirt9-gpu_b200"), os.path.join(ROOT, "oracle")]

REF_SKIRT = os.path.join(ROOT, "oracle", "_ref", "exe", "skirt", "bin", "skirt")
# the reference's own GPU layer (GpuAcceleration, run with -g): the reference program built with its
# driver-symbol loader preferring the versioned CUDA entry points (oracle/patch_refgpu.py)
REF_SKIRT_GPU = os.path.join(ROOT, "oracle", "_ref", "exe", "skirt", "bin", "skirt_refgpu")

WORKLOADS = {
    # name: (description, packets per step per GPU)
    "shell": ("dust shell r^-2 0.1-1 pc on a 64^3 CartesianSpatialGrid, tau_V=1, point source, 0.55 um, "
              "HG g=0.6 albedo 0.5, 256^2 frame at 30 deg + SED, FP64 tallies with statistics", 1_000_000),
    "galaxy": ("stellar exp. disk (hR 4 kpc, hz 0.35 kpc) + Sersic n=4 bulge (Re 1 kpc, B/T 0.2), dust exp. disk "
               "(hR 6 kpc, hz 0.2 kpc, face-on tau_V=1) on a TreeSpatialGrid octree (max level 8, dust fraction 1e-6, "
               "~5.1e5 leaves), 100 log wavelengths 0.1-10 um with power-law dust, three 512^2 frames at 0/60/90 deg, "
               "radiation field stored on 100 bins; one step = the 1e8-packet primary-emission segment", 100_000_000),
    "voronoi": ("the galaxy's sources and 100 wavelengths on a Voronoi mesh of 1e6 sites drawn (seed 1234) from the "
                "dust exp. disk, analytic density per cell, face-on tau_V=2, two 512^2 frames at 0/90 deg, radiation "
                "field on 100 bins; one step = a 1e7-packet segment (a tenth of the 1e8-packet run)", 10_000_000),
    "guided": ("learned path guiding on the edge-on dust disk (stellar disk + bulge in a dust disk of face-on "
               "tau_V=50, 0.55 um, albedo 0.6, g=0.6) on a ~1e6-leaf octree, 512^2 edge-on frame with statistics: "
               "1e7-packet plain pilot with recorded scattering events, training on the GPU, then 1e8-packet plain "
               "and guided runs; value = figure-of-merit ratio guided / plain (FOM = 1 / (R_med^2 t))", 100_000_000),
    "batch": ("16 independent galaxies on Delaunay tetrahedral meshes (TetraMeshSpatialGrid), parameters from "
              "default_rng(2024): vertex counts log-uniform 1e4-4e5 (half uniform in the box, half from the dust "
              "disk), face-on tau_V log-uniform 0.1-10, packets log-uniform 1e6-1e7 (7.1e7 in all), 32 log "
              "wavelengths, one 256^2 frame each; one step = every simulation's full primary-emission segment, "
              "traced as one batched wavefront", 0),
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.samples = []
        self.proc = None
        self.index = index

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons}


def build_scene(name):
    from skgpu import workloads
    if name == "shell":
        return workloads.shell_cartesian(64, 256)
    if name == "galaxy":
        return workloads.galaxy_octree()
    if name == "voronoi":
        return workloads.galaxy_voronoi()
    raise SystemExit(f"unknown workload {name}")


BYTES_PER_CROSSING = {0: 4, 1: 64, 2: 284, 3: 84}  # Cartesian, octree, Voronoi, tetra


def algorithmic_bytes(counters, grid_kind):
    """Bytes of one segment by the unit costs of the measurement plan: per cell crossing the grid's
    record (Cartesian 4 B, octree 64 B, Voronoi 284 B, tetra 84 B), 128 B per interaction event
    (packet state read + write), 16 B per peel-off detection and per radiation-field update."""
    return (BYTES_PER_CROSSING[grid_kind] * counters["crossings"] + 128 * counters["scatterings"]
            + 16 * (counters["peel_detections"] + counters["rf_stores"]))


def trace_algorithmic_bytes(counters, grid_kind):
    """The traversal kernel's share: cell crossings and radiation-field updates."""
    return BYTES_PER_CROSSING[grid_kind] * counters["crossings"] + 16 * counters["rf_stores"]


def reference_run(scene_ski, npp, threads, files=None, gpu=False):
    """Runs the reference CPU code on a ski file (plus input files {name: text} beside it), or with
    `gpu` the reference's own GPU layer (`skirt_refgpu -g`); returns (packets/s of the primary
    segment, secs)."""
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "bench.ski")
        with open(path, "w") as f:
            f.write(scene_ski)
        for fname, text in (files or {}).items():
            with open(os.path.join(tmp, fname), "w") as f:
                f.write(text)
        env = dict(os.environ)
        cmd = [REF_SKIRT, "-t", str(threads), "bench.ski"]
        if gpu:
            cmd = [REF_SKIRT_GPU, "-g", "-t", str(threads), "bench.ski"]
            nvrtc = "/usr/local/cuda/lib64/libnvrtc.so"
            if "SKIRTGPU_NVRTC_LIBRARY" not in env and os.path.exists(nvrtc):
                env["SKIRTGPU_NVRTC_LIBRARY"] = nvrtc
        out = subprocess.run(cmd, cwd=tmp, capture_output=True, text=True, env=env)
        if out.returncode != 0:
            raise RuntimeError("reference run failed: " + out.stdout[-500:] + out.stderr[-500:])
        if gpu:
            with open(os.path.join(tmp, "bench_log.txt")) as f:
                m = re.search(r"GPU acceleration is ([^\n]*)", f.read())
            status = m.group(1).strip() if m else "no status line"
            if not status.startswith("enabled"):
                raise RuntimeError("reference GPU layer not running: " + status)
        # primary-emission segment from the log time stamps (millisecond resolution): from
        # "Launching ... primary emission photon packets" to "Finished primary emission"
        def stamp(pattern):
            m = re.search(r"(\d\d):(\d\d):(\d\d\.\d+)[^\n]*" + pattern, out.stdout)
            return 3600 * int(m.group(1)) + 60 * int(m.group(2)) + float(m.group(3))
        secs = stamp(r"Finished primary emission") - stamp(r"Launching [^\n]* primary emission photon packets")
        if secs < 0:
            secs += 86400
        return npp / max(secs, 1e-3), secs


def reference_inputs(name, npp):
    """The ski file of the workload for the reference's own run and the input files beside it: the
    Voronoi workload's reference reads the GPU arm's seeded sites (VoronoiMeshSpatialGrid policy
    File) instead of drawing its own."""
    from skgpu import ski, workloads
    if name == "shell":
        return ski.shell_cartesian(npp, nbins=64, npix=256), None
    if name == "galaxy":
        return ski.galaxy_octree(npp), None
    if name == "voronoi":
        h = 25.0 * workloads.KPC
        sites = workloads.disk_sites(1_000_000, 6 * workloads.KPC, 0.2 * workloads.KPC, h)
        return ski.galaxy_voronoi(npp, sites_file="sites.txt"), {"sites.txt": ski.vertex_file_text(sites)}
    raise SystemExit(name)


def reference_batch(indices, fraction, cores):
    """The reference on simulations `indices` of the batched workload, each with `fraction` of its
    packets (one skirt run per simulation, as the reference would run the batch); returns (packets/s
    over the primary segments, packets, secs)."""
    from skgpu import ski, workloads
    spec = workloads.tetra_batch_spec()
    tot_n, tot_s = 0, 0.0
    for i in indices:
        sp = spec[i]
        n = max(1000, int(sp["packets"] * fraction))
        pts = workloads.tetra_points(sp["num_vertices"], sp["point_seed"])
        _, secs = reference_run(ski.galaxy_tetra(n, "vertices.txt", sp["tau_v"]), n, cores,
                                {"vertices.txt": ski.vertex_file_text(pts)})
        tot_n += n
        tot_s += secs
    return tot_n / max(tot_s, 1e-3), tot_n, tot_s


def cpu_baseline(name, sample_s=20.0):
    """The reference's own multithreaded CPU path on the host cores, on a bounded sample."""
    cores = os.cpu_count() or 1
    if name == "batch":
        if not os.path.exists(REF_SKIRT):
            return {"value": None, "error": "reference build oracle/_ref missing"}
        idx = [0, 4, 8, 12]
        rate, _, _ = reference_batch(idx[:1], 0.0025, cores)
        frac = min(1.0, rate * sample_s / 71e6 * 4)  # about sample_s of primary emission over 4 simulations
        rate, n, secs = reference_batch(idx, frac, cores)
        return {"value": rate, "unit": "packets/s", "cores": cores, "kind": "reference",
                "sample": f"simulations {idx} of the batch, {frac:.4f} of their packets ({n} in all), one skirt -t "
                          f"{cores} run each, primary-emission segments {secs:.2f} s (setup excluded)"}
    if os.path.exists(REF_SKIRT):
        probe = 20000
        text, files = reference_inputs(name, probe)
        rate, secs = reference_run(text, probe, cores, files)
        npp = int(min(5e7, max(probe, rate * sample_s)))
        text, files = reference_inputs(name, npp)
        rate, secs = reference_run(text, npp, cores, files)
        return {"value": rate, "unit": "packets/s", "cores": cores, "kind": "reference",
                "sample": f"{npp} packets of the same workload, skirt -t {cores}, primary-emission segment "
                          f"{secs:.2f} s (setup excluded)"}
    import oracle
    sc = build_scene(name)
    be = oracle.backend()
    sc.upload(be)
    n = 20000
    t = time.perf_counter()
    sc.run(be, n, seed=1)
    secs = time.perf_counter() - t
    return {"value": n / secs, "unit": "packets/s", "cores": 1, "kind": "port",
            "sample": f"{n} packets of the same workload through the single-threaded C oracle"}


def run_reference_gpu_arm(args, rank, world):
    """The reference's own GPU route on this box (`skirt_refgpu -g -t <cores>`, its default promoted
    configuration) on the workload's ski file: packets/s of the primary segment from its log, each
    step a sample of about 30 s. A second baseline beside the CPU reference arm."""
    if rank != 0:
        return
    name = args.workload
    if not os.path.exists(REF_SKIRT_GPU) or name == "batch" or name not in ("shell", "galaxy", "voronoi"):
        print(json.dumps({"impl": "reference-gpu", "unavailable": "skirt_refgpu missing or workload not a single ski "
                          "file (oracle/ref.mk target refgpu)"}))
        return
    cores = os.cpu_count() or 1
    try:
        # the route has seconds of fixed cost per primary segment (chunk set-up, resident tables):
        # a probe of 1e5 packets, then samples of about 30 s
        probe = 100000
        text, files = reference_inputs(name, probe)
        rate, _ = reference_run(text, probe, cores, files, gpu=True)
        npp = int(min(5e6, max(probe, rate * 30.0)))
        text, files = reference_inputs(name, npp)
        vals = [reference_run(text, npp, cores, files, gpu=True)[0] for _ in range(args.steps)]
    except RuntimeError as e:
        print(json.dumps({"impl": "reference-gpu", "unavailable": str(e)[:300]}))
        return
    value = statistics.median(vals)
    print(json.dumps({"metric": "packets/s on 1 B200", "value": value, "unit": "packets/s", "n_gpus": 1,
                      "steps": args.steps, "warmup": 0, "ms_per_step": 1e3 * npp / value, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "impl": "reference-gpu",
                      "config": {"workload": name, "description": WORKLOADS[name][0], "packets_per_step": npp,
                                 "route": f"reference GpuAcceleration, skirt -g -t {cores}, default (promoted) route"},
                      "samples": vals}))


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    name = args.workload
    if not os.path.exists(REF_SKIRT):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing (build() compiles "
                          "it where the reference sources are present)"}))
        return
    cores = os.cpu_count() or 1
    if name == "batch":
        return run_reference_batch_arm(args, cores)
    probe = 20000
    text, files = reference_inputs(name, probe)
    rate, _ = reference_run(text, probe, cores, files)
    npp = int(min(5e7, max(probe, rate * 8.0)))
    vals = []
    for _ in range(args.warmup):
        text, files = reference_inputs(name, min(npp, probe))
        reference_run(text, min(npp, probe), cores, files)
    text, files = reference_inputs(name, npp)
    for _ in range(args.steps):
        r, _ = reference_run(text, npp, cores, files)
        vals.append(r)
    value = statistics.median(vals)
    line = {"metric": "packets/s on 1 B200", "value": value, "unit": "packets/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * npp / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": name, "description": WORKLOADS[name][0], "packets_per_step": npp,
                       "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": "packets/s", "cores": cores, "kind": "reference",
                             "sample": f"{npp} packets per step, skirt -t {cores}, primary-emission segment"},
            "e2e": {"value": value, "unit": "packets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_reference_batch_arm(args, cores):
    """The batch on the reference: 16 sequential skirt runs per step, each on a sample of its
    packets sized so the primary segments of a step take about 8 s."""
    rate, _, _ = reference_batch([0], 0.0025, cores)
    frac = min(1.0, rate * 8.0 / 71e6)
    reference_batch([1], 0.001, cores)  # warm-up: one small run
    vals, npp = [], 0
    for _ in range(args.steps):
        r, npp, _ = reference_batch(range(16), frac, cores)
        vals.append(r)
    value = statistics.median(vals)
    print(json.dumps({
        "metric": "packets/s on 1 B200", "value": value, "unit": "packets/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": 1, "ms_per_step": 1e3 * npp / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": "batch", "description": WORKLOADS["batch"][0], "packets_per_step": npp,
                   "packet_fraction": frac, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "packets/s", "cores": cores, "kind": "reference",
                         "sample": f"16 sequential skirt -t {cores} runs per step, {frac:.4f} of each simulation's "
                                   f"packets ({npp} in all), primary-emission segments (setup excluded)"},
        "e2e": {"value": value, "unit": "packets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_batch_arm(args, rank, world, local):
    """Our arm on the batched workload: the 16 simulations (one context each) traced as one
    wavefront per step through skgpu_run_batch. Under torchrun every rank runs its own batch (the
    same meshes, rank-dependent random seeds: weak scaling)."""
    import torch
    from skgpu import Backend, abi, workloads

    torch.cuda.set_device(local)
    scenes, spec = workloads.tetra_batch(num=16, first=args.sims)
    n = len(scenes)
    packets = [max(1, int(s["packets"] * args.packet_scale)) for s in spec]
    seeds = [s["seed"] + 1000003 * rank for s in spec]
    prec = abi.PREC_FP64_EXACT if args.precision == "fp64" else abi.PREC_FP32
    bes = [Backend(device=local) for _ in scenes]
    for sc, be, npp, sd in zip(scenes, bes, packets, seeds):
        sc.upload(be)
        sc.prepare(be, npp, sd, prec)
    be0 = bes[0]
    zeros = [0] * n
    per_gpu = sum(packets)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")

    def step():
        abi.run_batch(bes, zeros, packets, packets)
        return be0.last_run_ms()

    # launch shape by the project autotuner (coordinate descent on a tenth of every simulation's
    # histories), kept per grid kind; the timed steps run with it
    shape = None
    if not args.no_tune:
        from skgpu import batch
        part = [max(1, p // 10) for p in packets]
        shape, _ = batch.tuned_shape(be0, abi.GRID_TETRA, lambda: abi.run_batch(bes, zeros, part, packets))
    for _ in range(args.warmup):
        step()
    abi.set_stage_timing(be0, 1)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    ms, trace_ms, trace_launches, counters = [], 0.0, 0, None
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            ms.append(step())
            counters = be0.counters()
            t_ms, t_n = abi.last_stage_times(be0)["trace"]
            trace_ms += t_ms
            trace_launches += t_n
    torch.cuda.synchronize()
    abi.set_stage_timing(be0, 0)
    total_ms = max_over_ranks(float(sum(ms)), world, local)
    value = per_gpu * world * args.steps / (total_ms / 1e3)

    e2e = None
    if not args.no_e2e:
        dens = [torch.from_numpy(np.ascontiguousarray(sc.density)).pin_memory().numpy() for sc in scenes]
        sizes = [sc.instrument_size(0) for sc in scenes]
        host = [np.zeros(k) for k in sizes]
        h2d = sum(d.nbytes for d in dens)
        d2h = 8 * sum(sizes)
        times = []
        for it in range(1 + max(1, min(args.steps, 3))):  # the first call is untimed (pinned buffers)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for be, d in zip(bes, dens):
                be.clear_tallies()
                be.upload_medium(d)
            abi.run_batch(bes, zeros, packets, packets)
            for be, k, hbuf in zip(bes, sizes, host):
                be.fetch_instrument(0, k, stats=False, out=hbuf)
            torch.cuda.synchronize()
            if it > 0:
                times.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(statistics.median(times), world, local)
        e2e = {"value": per_gpu * world / e2e_s, "unit": "packets/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h}

    if rank == 0:
        line = result_line(args, "batch", world, value, total_ms, trace_ms, trace_launches, counters, abi.GRID_TETRA,
                           prec, clk, e2e, per_gpu)
        line["config"]["simulations"] = n
        if n != 16 or args.packet_scale != 1.0:
            line["config"]["subset"] = f"first {n} simulations, {args.packet_scale:g} of their packets (profiling case)"
        line["config"]["launch_shape"] = ({"tuned": shape, "note": "autotuner (skgpu.batch.autotune) on a tenth of the "
                                           "histories; 0 = default"} if shape is not None else
                                          "default (pool 2^22 slots, resident traversal blocks, 4 stage blocks/SM)")
        if not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline("batch")
            except Exception as e:
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line))
    for be in bes:
        be.close()


def max_over_ranks(x, world, local):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def result_line(args, name, world, value, total_ms, trace_ms, trace_launches, counters, kind, prec, clk, e2e,
                per_gpu):
    """The JSON line of our arm; the roofline is that of the traversal kernel: its algorithmic bytes per
    launch over its average launch duration (CUDA events on the launch stream, timed steps)."""
    from skgpu import abi
    peak, peak_kind = peaks()
    trace_bytes_per_launch = trace_algorithmic_bytes(counters, kind) / max(1, trace_launches / args.steps)
    trace_avg_ms = trace_ms / max(1, trace_launches)
    achieved = trace_bytes_per_launch / (trace_avg_ms / 1e3) / 1e9
    traffic, profile = None, {}
    prof = os.path.join(ROOT, "profiles", f"trace_kernel_{name}_{args.precision}.json")
    if os.path.exists(prof):
        with open(prof) as f:
            profile = json.load(f)
        ratio = profile.get("dram_bytes_per_algorithmic_byte")
        if ratio:
            traffic = ratio * trace_bytes_per_launch
    return {
        "metric": "packets/s on 1 B200", "value": value, "unit": "packets/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == abi.PREC_FP64_EXACT else "f32+f64",
        "data": "synthetic",
        "config": {"workload": name, "description": WORKLOADS[name][0], "packets_per_step_per_gpu": per_gpu,
                   "traversal": args.precision, "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"history ranges x{world}" if name != "batch" else f"independent batches x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": profile.get("kernel", "skg::traceKernel"),
                     "launches_per_step": trace_launches / args.steps, "avg_launch_ms": trace_avg_ms,
                     "algorithmic_bytes_per_launch": trace_bytes_per_launch,
                     "share_of_step": trace_ms / max(total_ms, 1e-9),
                     # what ncu shows limits it (profiles/): the algorithmic bytes come mostly from L2
                     "limiter": profile.get("limiter"), "l2_throughput_frac": profile.get("l2_throughput_frac"),
                     "dram_throughput_frac": profile.get("dram_throughput_frac")},
        "clocks": clk.summary(),
        "e2e": e2e,
        "gpu_launches": int(counters["kernel_launches"]) * args.steps,
        "counters_per_step": counters,
    }


def run_guided_arm(args, rank, world, local):
    """C5, the learned path guiding protocol on one GPU: a plain pilot of 1e7 packets records a
    quarter of its scattering events with the downstream luminosity the edge-on frame detects,
    the network trains on the GPU, then plain and guided runs of the same packet count are timed on
    the device. FOM = 1 / (R_med^2 t) with R the per-pixel relative error from the frame's
    per-history statistics, over all lit pixels and over the pixels whose flux is mostly scattered
    light (more than half of it in the scattered component). Two trainings: the plain one
    (importance = the target's detected luminosity) and one restricted to scattered light (a plain
    pre-pilot's scattered-component image gives every scattered-light-dominated pixel the weight
    1 / F_scattered and every other pixel 0). With --truth-packets N a plain run of N packets (in
    segments) is the reference for the median per-pixel error of both runs."""
    import torch
    from skgpu import Backend, abi, guiding, workloads
    if rank != 0:
        return
    torch.cuda.set_device(local)
    sc = workloads.guided_disk()
    sc.instruments[0]["comps"] = 1
    n = args.packets or WORKLOADS["guided"][1]
    pilot = max(1, n // 10)
    be = Backend(device=local)
    sc.upload(be)

    def frame_stats(res):
        ins = res.instruments[0]
        st = np.asarray(ins["stats"]).reshape(5, -1)
        comp = np.asarray(ins["components"]).reshape(3, -1)  # transparent, direct, scattered
        return st, comp

    def scored(res, seconds, n_hist, mask):
        st, _ = frame_stats(res)
        r = guiding.relative_error(st, n_hist)
        lit = (st[1] > 0) & np.isfinite(r)
        out = {"seconds": seconds}
        for key, sel in (("all", lit), ("scattered", lit & mask)):
            rm = float(np.median(r[sel])) if sel.any() else float("nan")
            out[key] = {"pixels": int(sel.sum()), "R_med": rm, "FOM": 1.0 / (rm * rm * seconds) if rm > 0 else None}
        return out

    # plain run (also the classification of the pixels by their scattered fraction)
    for _ in range(max(1, args.warmup)):
        guiding.run(sc, be, pilot, seed=99)
    plain, t_plain = guiding.run(sc, be, n, seed=1)
    _, comp = frame_stats(plain)
    tot = comp[1] + comp[2]
    scat_mask = (tot > 0) & (comp[2] > 0.5 * tot)
    line = {"metric": "figure-of-merit gain of guided over plain runs (edge-on frame)", "unit": "ratio",
            "n_gpus": 1, "higher_is_better": True, "data": "synthetic", "dtype": "f32+f64 (BF16 network)",
            "config": {"workload": "guided", "description": WORKLOADS["guided"][0], "packets": n,
                       "pilot_packets": pilot}}
    line["plain"] = scored(plain, t_plain, n, scat_mask)
    variants = {}
    images = {"plain": np.asarray(plain.instruments[0]["total"]).ravel()}
    for name, restrict in (("plain-importance", False), ("scattered-importance", True)):
        info = {}
        if not restrict:
            info = guiding.train(sc, be, pilot, target=0, seed=7, record_fraction=0.25, steps=2000,
                                 prepilot_packets=0)
        else:
            pre, _ = guiding.run(sc, be, pilot, seed=5)
            _, c = frame_stats(pre)
            t = c[1] + c[2]
            w = guiding.importance_from_image(c[2])
            w = np.where((t > 0) & (c[2] > 0.5 * t), w, 0.0).astype(np.float32)
            abi.guide_init(be, None, 11)
            abi.guide_set_mode(be, abi.GUIDE_RECORD, 0, 0.0, 0.25, 1 << 22)
            abi.guide_set_importance(be, w)
            try:
                guiding.run(sc, be, pilot, seed=7)
            finally:
                abi.guide_set_mode(be, abi.GUIDE_OFF)
            abi.guide_set_training(be, 0)
            info["loss_final"] = abi.guide_train(be, 2000, 16384, 1e-3, 9)
        guided, t_guided = guiding.run_guided(sc, be, n, seed=1, alpha=0.5)
        images[name] = np.asarray(guided.instruments[0]["total"]).ravel()
        events, mean_w = abi.guide_last_weights(be)
        v = scored(guided, t_guided, n, scat_mask)
        v["training_loss"] = info.get("loss_final")
        v["mean_weight_factor"] = mean_w
        v["total_ratio"] = float(np.asarray(guided.instruments[0]["total"]).sum()
                                 / np.asarray(plain.instruments[0]["total"]).sum())
        for key in ("all", "scattered"):
            fp, fg = line["plain"][key]["FOM"], v[key]["FOM"]
            v[key]["FOM_gain"] = fg / fp if fp and fg else None
        variants[name] = v
    line["guided"] = variants
    if args.truth_packets:
        # the plain reference, in segments of 10x the run's packets (one random stream per history)
        done, seg = 0, 10 * n
        be.clear_tallies()
        sc.prepare(be, args.truth_packets, seed=1000)
        while done < args.truth_packets:
            cnt = min(seg, args.truth_packets - done)
            be.run_primary(done, cnt, args.truth_packets)
            done += cnt
        truth = np.asarray(sc.fetch(be).instruments[0]["total"]).ravel()
        line["truth_packets"] = args.truth_packets
        for key, sel in (("all", truth > 0), ("scattered", (truth > 0) & scat_mask)):
            for name, img in images.items():
                e = float(np.median(np.abs(img[sel] - truth[sel]) / truth[sel])) if sel.any() else None
                (line["plain"] if name == "plain" else variants[name])[key]["median_error_vs_truth"] = e
    line["value"] = variants["plain-importance"]["all"]["FOM_gain"]
    print(json.dumps(line))
    be.close()


def fp32_error_report(args):
    """The error of the production precision (FP32 walkers and accumulators) against the FP64
    reference-order life cycle, on one segment of the workload with the same histories (same Philox
    streams): per frame, per wavelength of the frames' integrated SED, per radiation-field entry and
    per cell's absorbed luminosity, the relative difference of the total and the median / 99th
    percentile over the entries above 1e-3 of the largest. Histories whose FP32 decisions differ
    (a different interaction cell or scattering count) diverge afterwards, so the per-entry figures
    include some Monte Carlo noise of those histories."""
    from skgpu import Backend, abi
    name = args.workload
    sc = build_scene(name)
    npp = args.packets or WORKLOADS[name][1]
    be = Backend(device=0)
    sc.upload(be)
    res = {}
    for prec in (abi.PREC_FP64_EXACT, abi.PREC_FP32):
        t0 = time.perf_counter()
        r = sc.run(be, npp, seed=12345, precision=prec)
        res[prec] = (r, time.perf_counter() - t0)
    r64, t64 = res[abi.PREC_FP64_EXACT]
    r32, t32 = res[abi.PREC_FP32]

    def stats(a, b):
        a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
        m = np.abs(b) >= 1e-3 * np.abs(b).max()
        rel = np.abs(a[m] - b[m]) / np.abs(b[m])
        return {"total_rel": float(abs(a.sum() - b.sum()) / abs(b.sum())), "entries": int(m.sum()),
                "median_rel": float(np.median(rel)), "p99_rel": float(np.quantile(rel, 0.99))}

    out = {"mode": "fp32-vs-fp64", "workload": name, "packets": npp, "fp64_s": t64, "fp32_s": t32, "outputs": {}}
    for i, ins in enumerate(sc.instruments):
        a, b = r32[i]["total"], r64[i]["total"]
        key = f"instrument{i}" + ("_frame" if ins["kind"] == abi.INSTR_FRAME else "_sed")
        out["outputs"][key] = stats(a, b)
        if ins["kind"] == abi.INSTR_FRAME:
            out["outputs"][key + "_integrated_sed"] = stats(a.reshape(a.shape[0], -1).sum(axis=1),
                                                            b.reshape(b.shape[0], -1).sum(axis=1))
    if r64.rf is not None:
        out["outputs"]["radiation_field"] = stats(r32.rf, r64.rf)
        sig_abs = np.asarray(sc.mix["sigma_ext"]) - np.asarray(sc.mix["sigma_sca"])
        nb = r64.rf.shape[1]
        sab = sig_abs[:nb] if len(sig_abs) >= nb else np.resize(sig_abs, nb)
        labs = lambda rf: (np.asarray(sc.density)[:, None] * sab[None, :] * rf).sum(axis=1)
        out["outputs"]["absorbed_luminosity"] = stats(labs(r32.rf), labs(r64.rf))
    out["counters_fp64"] = r64.counters
    out["counters_fp32"] = r32.counters
    print(json.dumps(out))
    be.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--workload", default="galaxy", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32"],
                    help="traversal precision: fp32 (production) or fp64 (reference operation order)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--packets", type=int, default=0, help="packets per step per GPU (default: the workload's)")
    ap.add_argument("--sims", type=int, default=16, help="batch workload: the first K simulations (profiling cases)")
    ap.add_argument("--packet-scale", type=float, default=1.0,
                    help="batch workload: fraction of every simulation's packets (profiling cases)")
    ap.add_argument("--no-tune", action="store_true", help="batch workload: default launch shape instead of the "
                                                            "autotuner's")
    ap.add_argument("--truth-packets", type=int, default=0,
                    help="guided workload: packets of a plain reference run for the per-pixel error (0: none)")
    ap.add_argument("--fp32-error", action="store_true",
                    help="instead of timing: one segment of the workload in FP64 (reference operation order) and "
                         "one in FP32 (production) on the same histories; prints the FP32 error of every output")
    args = ap.parse_args()
    if args.fp32_error:
        fp32_error_report(args)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(seconds=300))

    if args.impl in ("reference", "reference-gpu"):
        (run_reference_arm if args.impl == "reference" else run_reference_gpu_arm)(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return

    if args.workload == "guided":
        run_guided_arm(args, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return

    if args.workload == "batch":
        run_batch_arm(args, rank, world, local)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    from skgpu import Backend, abi

    torch.cuda.set_device(local)
    name = args.workload
    sc = build_scene(name)
    per_gpu = args.packets or WORKLOADS[name][1]
    npp_total = per_gpu * world
    first = rank * per_gpu
    prec = abi.PREC_FP64_EXACT if args.precision == "fp64" else abi.PREC_FP32
    be = Backend(device=local)
    sc.upload(be)
    sc.prepare(be, npp_total, seed=12345, precision=prec)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > L2

    def step():
        be.run_primary(first, per_gpu, npp_total)
        return be.last_run_ms()

    for _ in range(args.warmup):
        step()
    abi.set_stage_timing(be, 1)  # CUDA events around every traversal-kernel launch
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = []
    trace_ms, trace_launches = 0.0, 0
    counters = None
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            ms.append(step())
            counters = be.counters()
            t_ms, t_n = abi.last_stage_times(be)["trace"]
            trace_ms += t_ms
            trace_launches += t_n
    torch.cuda.synchronize()
    abi.set_stage_timing(be, 0)
    total_ms = max_over_ranks(float(sum(ms)), world, local)
    value = npp_total * args.steps / (total_ms / 1e3)

    # end to end through the C ABI with host buffers, as the SKIRT bridge uses it: the medium state
    # goes in from pinned host memory, every tally (instrument totals and statistics, radiation
    # field) is added into the caller's preallocated host arrays, every step. With several ranks the
    # segment's tallies are first summed over the ranks on the device (one NCCL all-reduce per tally
    # buffer over NVLink, the segment-end sum of the reference's ProcessManager) and rank 0 fetches
    # the sum.
    e2e = None
    if not args.no_e2e:
        from skgpu import sharding
        dens = torch.from_numpy(np.ascontiguousarray(sc.density)).pin_memory().numpy()
        sizes = [sc.instrument_size(i) for i in range(len(sc.instruments))]
        stats = [bool(sc.instruments[i].get("stats")) for i in range(len(sizes))]
        host = [(np.zeros(n), np.zeros(5 * n) if st else None) for n, st in zip(sizes, stats)]
        rf_len = sc.rf_length()
        rf_host = np.zeros(rf_len) if rf_len else None
        h2d = dens.nbytes
        d2h = sum(8 * n + (40 * n if st else 0) for n, st in zip(sizes, stats)) + 8 * rf_len
        e2e_times = []
        reduced = 0
        # one untimed call first: the fetch's pinned staging buffers are allocated on first use
        for it in range(1 + max(1, min(args.steps, 3))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            be.clear_tallies()
            be.upload_medium(dens)
            be.run_primary(first, per_gpu, npp_total)
            if world > 1:
                reduced = sharding.allreduce_device_tallies(be, f"cuda:{local}")
            if rank == 0:
                for i, n in enumerate(sizes):
                    be.fetch_instrument(i, n, stats=stats[i], out=host[i][0], out_stats=host[i][1])
                if rf_len:
                    be.fetch_radiation_field(rf_len, out=rf_host)
            torch.cuda.synchronize()
            if it > 0:
                e2e_times.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(statistics.median(e2e_times), world, local)
        e2e = {"value": npp_total / e2e_s, "unit": "packets/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
        if world > 1:
            e2e["allreduce_bytes_per_step_per_rank"] = reduced

    if rank == 0:
        line = result_line(args, name, world, value, total_ms, trace_ms, trace_launches, counters, sc.grid["kind"],
                           prec, clk, e2e, per_gpu)
        if not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(name)
            except Exception as e:  # the baseline is reported, never required for the GPU number
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line))
    be.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
