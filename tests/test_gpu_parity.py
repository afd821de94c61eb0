"""GPU parity tests: the CUDA library through its C ABI against the reference golden vectors and
the CPU oracle.

- Path segments and optical depths of the FP64 walkers must equal the reference CPU generators bit
  for bit (golden path fixtures).
- The FP64 life cycle draws the same Philox streams as the oracle, so on identical scenes the two
  must agree history by history up to the last-bit differences of CUDA's and glibc's
  transcendental functions: totals to 1e-9 relative, and all but a tiny fraction of pixels.
- Against the reference's own run, images and SEDs agree within Monte Carlo noise (z-scores).
"""
import numpy as np
import pytest

from conftest import PATH_FIXTURES
from helpers import compare_paths, tetra_hull_edge_exits, zscores
from skgpu import Scene, SkgpuError, abi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", PATH_FIXTURES)
def test_gpu_paths_match_reference(golden, gpu_backend, name):
    z = golden(f"paths_{name}.npz")
    sc = Scene.from_export(z)
    sc.upload(gpu_backend)
    count, m, ds = gpu_backend.trace_paths(z["rays"], 512)
    assert compare_paths(z, count, m, ds) == []
    tau = gpu_backend.optical_depths(z["rays"], 0.55e-6)
    assert np.array_equal(tau, z["ray_tau"])


def run_both(sc, gpu, orc, n, seed):
    sc.upload(gpu)
    sc.upload(orc)
    return sc.run(gpu, n, seed=seed), sc.run(orc, n, seed=seed)


def assert_close_runs(rg, ro, pix_tol=1e-9, frac=0.995):
    for ig, io in zip(rg.instruments, ro.instruments):
        tg, to = ig["total"], io["total"]
        assert tg.sum() == pytest.approx(to.sum(), rel=1e-6)
        close = np.isclose(tg, to, rtol=pix_tol, atol=0)
        assert close.mean() >= frac, f"only {close.mean():.4f} of bins agree"
        if ig.get("stats") is not None:
            assert np.array_equal(ig["stats"][0], io["stats"][0]) or np.mean(ig["stats"][0] == io["stats"][0]) > frac
    assert rg.counters["histories"] == ro.counters["histories"]
    assert rg.counters["scatterings"] == pytest.approx(ro.counters["scatterings"], rel=1e-3)


def test_gpu_lifecycle_matches_oracle_shell(golden, gpu_backend, oracle_backend):
    z = golden("shell_c16.npz")
    sc = Scene.from_export(z)
    sc.instruments[1]["comps"] = 1
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 20000, seed=11)
    assert_close_runs(rg, ro)
    cg, co = rg[1]["components"], ro[1]["components"]
    assert cg[0, 0] == pytest.approx(co[0, 0], rel=1e-12)  # transparent: deterministic
    assert cg[1, 0] == pytest.approx(co[1, 0], rel=1e-12)  # direct: deterministic for a point source


def test_gpu_levels_and_bands_match_oracle(golden, gpu_backend, oracle_backend):
    """Scattering levels and a band wavelength grid (the shell with a levels frame, its SED and a
    band SED of the same observer): GPU FP64 equals the oracle per history, and both the FP64 and
    the FP32 runs show the band and level identities of test_instrument_output_cpu."""
    from test_instrument_output_cpu import check_levels_and_bands, levels_bands_scene
    sc = levels_bands_scene(golden("shell_c16.npz"), levels=3)
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 20000, seed=13)
    assert_close_runs(rg, ro)
    for ig, io in zip(rg.instruments, ro.instruments):
        for key in ("components", "levels"):
            assert np.mean(np.isclose(ig[key], io[key], rtol=1e-9, atol=0)) > 0.995, key
    check_levels_and_bands(sc, rg, 3)
    r32 = sc.run(gpu_backend, 20000, seed=13, precision=abi.PREC_FP32)
    check_levels_and_bands(sc, r32, 3)


def test_gpu_calibration_matches_oracle_and_reference(golden, gpu_backend, oracle_backend):
    """Calibration on the device: every plane scaled by its bin's factor (one multiply, as the
    oracle), the shell's transparent SED flux equal to the reference's written Jy; a frame's total,
    component and scattering-level planes scaled alike."""
    from skgpu.scene import calibration_factors
    from test_instrument_output_cpu import calibrated_shell, levels_bands_scene
    z, f, rawg, calg = calibrated_shell(gpu_backend, golden)
    _, _, rawo, calo = calibrated_shell(oracle_backend, golden)
    assert np.array_equal(calg["total"], rawg["total"] * f[0])
    assert np.array_equal(calg["components"], rawg["components"] * f[0])
    assert calg["components"][0, 0] == pytest.approx(float(z["ref_sed_jy"][1]), rel=1e-9)
    assert np.allclose(calg["total"], calo["total"], rtol=1e-9, atol=0)
    sc = levels_bands_scene(golden("shell_c16.npz"), levels=3)
    sc.upload(gpu_backend)
    raw = sc.run(gpu_backend, 3000, seed=2)[0]
    fr = sc.instruments[0]
    fac = calibration_factors(fr["distance"], [0.55e-6], [1.1e-9], pixel_size=(fr["xp_size"], fr["yp_size"]))
    gpu_backend.calibrate_instrument(0, fac)
    cal = sc.fetch(gpu_backend)[0]
    for key in ("total", "components", "levels"):
        assert np.array_equal(cal[key], raw[key] * fac[0]), key


def test_gpu_observer_redshift_and_aperture_match_oracle(golden, gpu_backend, oracle_backend):
    """Observer-frame redshift and an SED aperture: GPU FP64 equals the oracle per history."""
    from test_instrument_output_cpu import observer_scene
    sc = observer_scene(golden("shell_c16.npz"), 0.3 * 3.0856775814913673e16, 5e-4)
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 20000, seed=9)
    assert_close_runs(rg, ro)
    assert 0 < rg[2]["total"].sum() < rg[1]["total"].sum()


def test_gpu_free_propagation_matches_oracle(golden, gpu_backend, oracle_backend):
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.force_scattering = False
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 20000, seed=5)
    assert_close_runs(rg, ro)


def test_gpu_free_propagation_matches_reference(golden, gpu_backend):
    """Free (non-forced) propagation, both traversal precisions: frame and SED against the
    reference's own run of the same scene (raw per-history statistics)."""
    z = golden("shell_c16.npz")
    f = golden("shell_c16_free.npz")
    sc = Scene.from_export(z)
    sc.force_scattering = False
    sc.upload(gpu_backend)
    n = int(f["ref_npp"])
    for precision in (abi.PREC_FP64_EXACT, abi.PREC_FP32):
        res = sc.run(gpu_backend, n, seed=37, precision=precision)
        st = res[0]["stats"][:, 0].reshape(5, -1)
        ref = f["ref_frame_w"]
        zs = zscores(st[1], st[2], n, ref[1], ref[2], n)
        assert abs(zs.mean()) < 0.1 and 0.9 < zs.std() < 1.1
        sst = res[1]["stats"][:, 0]
        rs = f["ref_sed_w"]
        assert abs(zscores(sst[1:2], sst[2:3], n, rs[1:2, 0], rs[2:3, 0], n)[0]) < 4


@pytest.mark.parametrize("name", ["octree", "voronoi", "tetra", "cartesian_selftest", "sphere1d", "cylinder2d", "sphere2d", "sphere3d", "cylinder3d", "adaptive"])
def test_gpu_lifecycle_matches_oracle_grids(golden, gpu_backend, oracle_backend, name):
    sc = Scene.from_export(golden(f"paths_{name}.npz"))
    sc.instruments[0]["stats"] = 1
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 5000, seed=3)
    assert_close_runs(rg, ro)


def test_gpu_radiation_field_matches_oracle(golden, gpu_backend, oracle_backend):
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.store_rf = True
    sc.rf = dict(num_bins=1, borders=np.array([0.5e-6, 0.6e-6]), ellv=np.array([-1, 0, -1], np.int32))
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 10000, seed=9)
    assert rg.rf.sum() == pytest.approx(ro.rf.sum(), rel=1e-6)
    assert np.mean(np.isclose(rg.rf, ro.rf, rtol=1e-9, atol=0)) > 0.99
    assert rg.counters["rf_stores"] == pytest.approx(ro.counters["rf_stores"], rel=1e-3)


def test_gpu_lifecycle_matches_reference_statistics(golden, gpu_backend):
    z = golden("shell_c16.npz")
    sc = Scene.from_export(z)
    sc.upload(gpu_backend)
    n = int(z["ref_npp"])
    res = sc.run(gpu_backend, n, seed=21)
    st = res[0]["stats"][:, 0]
    ref = z["ref_frame_w"]
    zs = zscores(st[1], st[2], n, ref[1], ref[2], n)
    assert abs(zs.mean()) < 0.1 and 0.9 < zs.std() < 1.1
    rs = z["ref_sedstats"]
    sst = res[1]["stats"][:, 0]
    assert abs(zscores(sst[1:2], sst[2:3], n, rs[1:2], rs[2:3], n)[0]) < 4


def test_gpu_history_ranges_add_up(golden, gpu_backend):
    """Two half segments (histories [0,n/2) and [n/2,n)) give the same tallies as one run."""
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.upload(gpu_backend)
    n = 8000
    full = sc.run(gpu_backend, n, seed=2)
    gpu_backend.clear_tallies()
    sc.prepare(gpu_backend, n, seed=2)
    gpu_backend.run_primary(0, n // 2, n)
    gpu_backend.run_primary(n // 2, n - n // 2, n)
    halves = sc.fetch(gpu_backend)
    for a, b in zip(full.instruments, halves.instruments):
        assert np.allclose(a["total"], b["total"], rtol=1e-12, atol=0)


def test_gpu_edge_cases(golden, gpu_backend):
    sc = Scene.from_export(golden("shell_c16.npz"))
    with pytest.raises(SkgpuError) as e:
        gpu_backend.run_primary(0, 10, 10)  # nothing uploaded yet
    assert e.value.code == abi.ERR_STATE
    sc.upload(gpu_backend)
    sc.prepare(gpu_backend, 100)
    gpu_backend.run_primary(0, 0, 100)  # empty range is fine
    assert gpu_backend.counters()["histories"] == 0
    with pytest.raises(SkgpuError) as e:
        gpu_backend.run_primary(90, 20, 100)  # beyond the segment
    assert e.value.code == abi.ERR_ARG
    bad = sc.density.copy()
    bad[3] = np.nan
    with pytest.raises(SkgpuError):
        gpu_backend.upload_medium(bad)
    with pytest.raises(SkgpuError):
        gpu_backend.upload_grid_cartesian([0, 1], [1, 0], [0, 1])  # descending borders


@pytest.mark.parametrize("name", ["cartesian_selftest", "cartesian_c16", "octree", "adaptive"])
def test_gpu_production_paths_equal_reference(golden, gpu_backend, name):
    """Production Cartesian and octree walkers (the reference's FP64 geometry with the quotient from
    the reciprocal direction, 64-byte octree leaf records with lattice wall tables): cell sequences
    and segment lengths equal the reference generators' bit for bit on every golden ray, including
    the rays through cell corners and along cell walls; optical depths (FP32 accumulation) within
    1e-5 relative."""
    z = golden(f"paths_{name}.npz")
    sc = Scene.from_export(z)
    sc.upload(gpu_backend)
    count, m, ds = gpu_backend.trace_paths(z["rays"], 512, precision=abi.PREC_FP32)
    assert compare_paths(z, count, m, ds) == []
    tau = gpu_backend.optical_depths(z["rays"], 0.55e-6, precision=abi.PREC_FP32)
    assert np.allclose(tau, z["ray_tau"], rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("name", ["voronoi", "tetra"])
def test_gpu_fp32_paths_close_to_reference(golden, gpu_backend, name):
    """Voronoi and tetrahedral production walkers (FP32 face distances with FP64 re-decisions of near
    ties): cell sequences equal the reference's on every golden ray; segment lengths within 1e-5 of
    the path length; optical depths within 1e-5. The one exception is a ray that leaves a
    tetrahedral mesh's hull exactly through a boundary edge or vertex (five rays of the golden set,
    from the origin along the axes and the diagonal): the reference breaks that exact tie by the
    rounding of its FP64 position, which a walk with FP32 steps does not reproduce, so there the
    sequences may differ in the last in-mesh cells only (the FP64 walker matches them exactly)."""
    z = golden(f"paths_{name}.npz")
    sc = Scene.from_export(z)
    sc.upload(gpu_backend)
    count, m, ds = gpu_backend.trace_paths(z["rays"], 512, precision=abi.PREC_FP32)
    off = z["ray_offset"]
    coin = tetra_hull_edge_exits(z) if name == "tetra" else set()
    assert len(coin) <= 5
    for r in range(len(count)):
        rm, rds = z["ray_m"][off[r]:off[r + 1]], z["ray_ds"][off[r]:off[r + 1]]
        if r in coin:
            n = min(count[r], len(rm))
            assert abs(int(count[r]) - len(rm)) <= 4 and np.array_equal(m[r, :n - 1], rm[:n - 1]), r
            continue
        assert count[r] == len(rm) and np.array_equal(m[r, :count[r]], rm), r
        if count[r] > 0:
            scale = max(np.abs(rds).sum(), 1e-300)
            assert np.abs(ds[r, :count[r]] - rds).max() <= 1e-5 * scale, r
    tau = gpu_backend.optical_depths(z["rays"], 0.55e-6, precision=abi.PREC_FP32)
    keep = np.array([r not in coin for r in range(len(tau))])
    assert np.allclose(tau[keep], z["ray_tau"][keep], rtol=1e-5, atol=1e-9)


def test_gpu_statistics_exact_beyond_the_slot_buffer(golden, gpu_backend, oracle_backend):
    """Per-history statistics (FluxRecorder::recordContributions) of histories with more distinct
    (instrument, bin, pixel) keys than a packet slot buffers: 16 frames at different inclinations and
    long histories (albedo 0.95, termination at 1e-8 of the launch weight) spill into the device log,
    which is grouped exactly after the run. GPU statistics equal the oracle's unbounded grouping."""
    sc = Scene.from_export(golden("shell_c16.npz"))
    frame = dict(sc.instruments[0])
    frame["stats"] = 1
    sc.instruments = []
    for inc in np.linspace(5, 175, 16):
        f = dict(frame)
        th = np.radians(inc)
        f["kobs"] = (np.sin(th), 0.0, np.cos(th))
        f["trig"] = (np.cos(th), np.sin(th), 1.0, 0.0, 1.0, 0.0)
        f["same_observer"] = 0
        sc.instruments.append(f)
    sc.mix = dict(sc.mix, sigma_sca=0.95 * np.asarray(sc.mix["sigma_ext"]))
    sc.min_weight_reduction = 1e8
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 1000, seed=23)
    assert rg.counters["stats_spilled"] > 0 and rg.counters["stats_overflows"] == 0
    for ig, io in zip(rg.instruments, ro.instruments):
        for k in range(5):
            a, b = ig["stats"][k], io["stats"][k]
            assert np.mean(np.isclose(a, b, rtol=1e-9, atol=0)) > 0.995, k
            assert a.sum() == pytest.approx(b.sum(), rel=1e-9)


def test_gpu_fp32_lifecycle_close_to_fp64(golden, gpu_backend):
    """The production (FP32-distance) life cycle follows the same histories as the FP64 one except
    where a path grazes a cell edge: tallies agree to well within Monte Carlo noise."""
    sc = Scene.from_export(golden("shell_c16.npz"))
    sc.upload(gpu_backend)
    n = 100000
    r64 = sc.run(gpu_backend, n, seed=13)
    r32 = sc.run(gpu_backend, n, seed=13, precision=abi.PREC_FP32)
    for a, b in zip(r64.instruments, r32.instruments):
        assert b["total"].sum() == pytest.approx(a["total"].sum(), rel=1e-3)
        assert np.mean(np.isclose(a["total"], b["total"], rtol=1e-4, atol=0)) > 0.95
    st64, st32 = r64[0]["stats"][:, 0], r32[0]["stats"][:, 0]
    zs = zscores(st32[1], st32[2], n, st64[1], st64[2], n)
    assert np.abs(zs).max() < 1.0  # same histories: far inside the noise


def test_gpu_galaxy_octree_matches_oracle(gpu_backend, oracle_backend):
    """Panchromatic galaxy scene on a built octree (disk + Sersic sources with wavelength bias,
    100-bin dust tables, three frames, radiation field): GPU FP64 equals the oracle per history."""
    from skgpu import workloads
    sc = workloads.galaxy_octree(npix=64, nlambda=20, max_level=5, max_dust_fraction=1e-4)
    rg, ro = run_both(sc, gpu_backend, oracle_backend, 3000, seed=17)
    assert_close_runs(rg, ro, frac=0.99)
    assert rg.rf.sum() == pytest.approx(ro.rf.sum(), rel=1e-6)


def test_gpu_fp32_voronoi_lifecycle_close_to_fp64(gpu_backend):
    """Production Voronoi walker (FP32 local distances, FP64 near-tie predicate) on a panchromatic
    galaxy mesh: the same histories as the FP64 reference-order walker, tallies far inside the noise."""
    from skgpu import workloads
    sc = workloads.galaxy_voronoi(n_sites=20000, npix=64, nlambda=20)
    sc.upload(gpu_backend)
    n = 40000
    r64 = sc.run(gpu_backend, n, seed=13)
    r32 = sc.run(gpu_backend, n, seed=13, precision=abi.PREC_FP32)
    for a, b in zip(r64.instruments, r32.instruments):
        assert b["total"].sum() == pytest.approx(a["total"].sum(), rel=2e-3)
        assert np.mean(np.isclose(a["total"], b["total"], rtol=1e-3, atol=0)) > 0.9
    assert r32.rf.sum() == pytest.approx(r64.rf.sum(), rel=2e-3)
    assert r32.counters["crossings"] == pytest.approx(r64.counters["crossings"], rel=1e-3)


def test_gpu_fp32_tetra_lifecycle_close_to_fp64(gpu_backend):
    """Production tetrahedral walker (one plane record per tetrahedron, start-cell hints, walking
    point location) on a panchromatic galaxy mesh: the same histories as the reference-order FP64
    walker, tallies far inside the noise."""
    from skgpu import workloads
    sc = workloads.galaxy_tetra(20000, tau_v=3.0, seed=21, npix=64, nlambda=16, store_rf=True)
    sc.upload(gpu_backend)
    n = 40000
    r64 = sc.run(gpu_backend, n, seed=17)
    r32 = sc.run(gpu_backend, n, seed=17, precision=abi.PREC_FP32)
    for a, b in zip(r64.instruments, r32.instruments):
        assert b["total"].sum() == pytest.approx(a["total"].sum(), rel=2e-3)
        assert np.mean(np.isclose(a["total"], b["total"], rtol=1e-3, atol=0)) > 0.9
    assert r32.rf.sum() == pytest.approx(r64.rf.sum(), rel=2e-3)
    c64, c32 = r64.counters, r32.counters
    assert c32["histories"] == c64["histories"] == n
    assert c32["scatterings"] == pytest.approx(c64["scatterings"], rel=1e-3)
    assert c32["crossings"] == pytest.approx(c64["crossings"], rel=1e-3)


def test_gpu_fp32_octree_lifecycle_close_to_fp64(gpu_backend):
    """Production octree walker with FP32 accumulators on the panchromatic galaxy: images and the
    radiation field (whose L * ds products exceed the FP32 range and are formed in FP64) follow the
    FP64 reference-order walker on the same histories."""
    from skgpu import workloads
    sc = workloads.galaxy_octree(npix=64, nlambda=20, max_level=6, max_dust_fraction=1e-5)
    sc.upload(gpu_backend)
    n = 40000
    r64 = sc.run(gpu_backend, n, seed=19)
    r32 = sc.run(gpu_backend, n, seed=19, precision=abi.PREC_FP32)
    for a, b in zip(r64.instruments, r32.instruments):
        assert b["total"].sum() == pytest.approx(a["total"].sum(), rel=2e-3)
    assert np.all(np.isfinite(r32.rf))
    assert r32.rf.sum() == pytest.approx(r64.rf.sum(), rel=2e-3)
    lit = r64.rf > 0
    assert np.median(np.abs(r32.rf[lit] / r64.rf[lit] - 1)) < 1e-3


@pytest.mark.parametrize("name", ["sphere1d", "cylinder2d", "sphere2d", "sphere3d", "cylinder3d", "adaptive"])
def test_gpu_curvilinear_lifecycle_matches_reference_statistics(golden, gpu_backend, name):
    """The dust shell on a Sphere1DSpatialGrid, the dust disk on the cylindrical, spherical and
    adaptive-mesh grids, both traversal precisions: frame and SED against the reference's own run
    of the same scene."""
    z = golden(f"paths_{name}.npz")
    sc = Scene.from_export(z)
    sc.instruments[0]["stats"] = 1
    sc.instruments[1]["stats"] = 1
    sc.upload(gpu_backend)
    n = int(z["ref_npp"])
    for precision in (abi.PREC_FP64_EXACT, abi.PREC_FP32):
        res = sc.run(gpu_backend, n, seed=29, precision=precision)
        st = res[0]["stats"][:, 0]
        ref = z["ref_frame_w"]
        zs = zscores(st[1], st[2], n, ref[1], ref[2], n)
        assert abs(zs.mean()) < 0.1 and 0.85 < zs.std() < 1.15
        sst = res[1]["stats"][:, 0]
        rs = z["ref_sedstats"]
        assert abs(zscores(sst[1:2], sst[2:3], n, rs[1:2], rs[2:3], n)[0]) < 4
