"""The galaxy configuration pinned against the reference's own run on identical inputs.

Fixture stats_galaxy.npz (tests/golden/make_fixtures.py galaxy): the galaxy at reduced size (stellar
exponential disk + Sersic bulge with black-body SEDs and wavelength bias 0.5, dust disk on the
reference's own octree of max level 6, 20 log wavelengths, three 32^2 frames and an SED with
statistics, radiation field stored), exported from the reference's SimulationItem tree, with the raw
detector sums and the primary radiation field MediumSystem::_rf1 of a single-threaded 5e5-packet
reference run, and 2e4 launches of the reference's SourceSystem::launch.

- Launch: the oracle's launch distributions (wavelength with its bias weight, disk R and z, bulge
  radius, direction) equal the reference's (two-sample KS tests); the GPU launch equals the oracle's
  history by history.
- Life cycle: the oracle's frames and SED agree with the reference run per pixel and bin
  (z-scores from the per-history statistics), its radiation field and absorbed luminosity per cell
  and bin (z-scores with the variance from history sub-ranges of an independent run); the GPU FP64
  life cycle equals the oracle's history by history; the production FP32 life cycle agrees with the
  reference run within noise in the same way.
"""
import numpy as np
import pytest
from scipy import stats

from helpers import zscores
from skgpu import Scene, abi

K = 40  # history sub-ranges per source for the per-cell variance of the radiation field (a variance
# estimate from k sub-ranges has k - 1 degrees of freedom: z-scores then spread like Student t)


def galaxy_scene(golden):
    z = golden("stats_galaxy.npz")
    sc = Scene.from_export(z)
    for ins in sc.instruments:
        ins["stats"] = 1
    sc.store_rf = True
    return z, sc


def reference_rf(z):
    return (z["rf1_scaled"].astype(np.float64) * float(z["rf1_scale"])).ravel()


def run_subranges(sc, be, n, seed, precision=abi.PREC_FP64_EXACT, k=K):
    """One segment of n histories run as k consecutive sub-ranges of each source's history range
    (the histories of one source are identically distributed, those of different sources are not):
    the results of the whole segment and, per source, the radiation field of each of its sub-ranges
    (list of k x cells*bins arrays)."""
    be.clear_tallies()
    sc.prepare(be, n, seed, precision)
    prev, parts = 0.0, []
    for s in sc.source_structs(n)[0]:
        a, m = int(s.first_history), int(s.num_histories)
        mine = []
        for i in range(k):
            be.run_primary(a + i * m // k, (i + 1) * m // k - i * m // k, n)
            cum = be.fetch_radiation_field(sc.rf_length())
            mine.append(cum - prev)
            prev = cum
        parts.append(np.array(mine))
    return sc.fetch(be), parts


def segment_variance(parts, f=lambda p: p):
    """Variance of f of a whole segment from the per-source sub-ranges: sum over sources of k times
    the variance over that source's k sub-ranges."""
    return sum(len(p) * np.array([f(q) for q in p]).var(axis=0, ddof=1) for p in parts)


def absorbed_luminosity(sc, rf):
    """Absorbed luminosity per cell, n(m) sum_ell sigma_abs(lambda_ell) * rf(m, ell), with the
    cross sections of the dust-mix entry of each radiation-field bin's centre (rf in W m per cell
    and bin, so the product is in W)."""
    b = sc.rf["borders"]
    centres = np.sqrt(b[:-1] * b[1:])
    lb = sc.mix["lambda_borders"]
    ell = np.clip(np.searchsorted(lb, centres, side="right") - 1, 0, len(lb) - 1)
    sabs = (sc.mix["sigma_ext"] - sc.mix["sigma_sca"])[ell]
    nb = sc.rf["num_bins"]
    return sc.density * (rf.reshape(-1, nb) * sabs[None, :]).sum(axis=1)


def check_detectors(z, res, n):
    """Frames and SED of a run against the reference run: per-pixel and per-bin z-scores."""
    for i in range(3):
        w = z[f"inst{i}_wifu"]
        st = res[i]["stats"].reshape(5, -1)
        zs = zscores(st[1], st[2], n, w[1], w[2], n)
        assert len(zs) > 5000
        assert abs(zs.mean()) < 0.05 and 0.92 < zs.std() < 1.08, (i, zs.mean(), zs.std())
        assert st[1].sum() == pytest.approx(w[1].sum(), rel=0.01)
    w = z["inst3_wsed"]
    st = res[3]["stats"].reshape(5, -1)
    zs = zscores(st[1], st[2], n, w[1], w[2], n)
    assert np.abs(zs).max() < 4.5 and np.mean(zs ** 2) < 2.0


def check_radiation_field(sc, z, parts, parts_indep):
    """Radiation field and absorbed luminosity per cell against the reference run. The variance of a
    cell's segment sum comes from the per-source history sub-ranges of an independent run (a
    variance from the tested run itself correlates with its own deviations)."""
    ref = reference_rf(z)
    rf = sum(p.sum(0) for p in parts)
    var = segment_variance(parts_indep)
    # cells and bins reached in at least 85 % of the sub-ranges: there a sub-range sum is close to
    # normal and its variance well estimated
    hits = sum((p > 0).sum(axis=0) for p in parts_indep)
    lit = (hits >= 0.85 * sum(len(p) for p in parts_indep)) & (var > 0)
    zr = (rf - ref)[lit] / np.sqrt(2 * var[lit])
    assert lit.sum() > 20000
    assert abs(zr.mean()) < 0.05 and 0.95 < zr.std() < 1.1, (zr.mean(), zr.std())
    assert np.mean(np.abs(zr) > 4) < 0.002
    assert rf.sum() == pytest.approx(ref.sum(), rel=0.01)
    # absorbed luminosity per cell
    la, la_ref = absorbed_luminosity(sc, rf), absorbed_luminosity(sc, ref)
    la_var = segment_variance(parts_indep, lambda p: absorbed_luminosity(sc, p))
    lit = (la_var > 0) & (la > 0) & (la_ref > 0)
    zl = (la - la_ref)[lit] / np.sqrt(2 * la_var[lit])
    assert lit.sum() > 5000
    assert abs(zl.mean()) < 0.05 and 0.95 < zl.std() < 1.1, (zl.mean(), zl.std())
    assert la.sum() == pytest.approx(la_ref.sum(), rel=0.01)


def launch_columns(p, nsrc0):
    """Launch statistics per source: the first nsrc0 histories come from the disk, the rest from
    the bulge (SourceSystem's history ranges)."""
    d, b = p[:nsrc0], p[nsrc0:]
    return dict(wavelength=p[:, 0], luminosity=p[:, 1], disk_R=np.hypot(d[:, 2], d[:, 3]), disk_z=d[:, 4],
                bulge_r=np.sqrt((b[:, 2:5] ** 2).sum(axis=1)), kz=p[:, 7], kphi=np.arctan2(p[:, 6], p[:, 5]))


def source_split(sc, npp):
    structs = sc.source_structs(npp)[0]
    return int(structs[1].first_history)


def test_oracle_galaxy_launch_matches_reference(golden, oracle_backend):
    """SourceSystem::launch of the two geometric sources (ExpDiskGeometry, SersicGeometry with its
    log-log cumulative-mass table, BlackBodySED with wavelength bias 0.5) against the reference's
    own launches: two-sample KS tests per quantity."""
    z, sc = galaxy_scene(golden)
    sc.upload(oracle_backend)
    ref = z["src_probe"].astype(np.float64)
    n = 100000
    mine = sc.probe_launch(oracle_backend, n, seed=5)
    a = launch_columns(mine, source_split(sc, n))
    b = launch_columns(ref, source_split(sc, len(ref)))
    for key in a:
        p = stats.ks_2samp(a[key], b[key]).pvalue
        assert p > 1e-3, (key, p)


def test_oracle_galaxy_matches_reference_run(golden, oracle_backend):
    """The oracle's life cycle on the reference's exported galaxy: frames, SED, radiation field and
    absorbed luminosity against the reference's single-threaded run of the same scene."""
    z, sc = galaxy_scene(golden)
    sc.upload(oracle_backend)
    n = int(z["ref_npp"])
    res, parts = run_subranges(sc, oracle_backend, n, seed=31)
    check_detectors(z, res, n)
    _, indep = run_subranges(sc, oracle_backend, n, seed=77)
    check_radiation_field(sc, z, parts, indep)


@pytest.mark.gpu
def test_gpu_galaxy_launch_matches_oracle(golden, gpu_backend, oracle_backend):
    """The GPU launch of the galaxy's sources equals the oracle's history by history (up to the last
    bits of CUDA's and glibc's transcendental functions)."""
    z, sc = galaxy_scene(golden)
    sc.upload(gpu_backend)
    sc.upload(oracle_backend)
    n = 200000
    g = sc.probe_launch(gpu_backend, n, seed=5)
    o = sc.probe_launch(oracle_backend, n, seed=5)
    scale = np.array([1.0, 1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
    size = np.abs(o).max(axis=0) * scale
    assert np.all(np.abs(g - o) <= 1e-9 * np.abs(o) + 1e-12 * size + 1e-12)


@pytest.mark.gpu
def test_gpu_galaxy_matches_oracle(golden, gpu_backend, oracle_backend):
    """GPU FP64 life cycle on the reference's exported galaxy equals the oracle per history:
    frames, SED, statistics and radiation field."""
    z, sc = galaxy_scene(golden)
    sc.upload(gpu_backend)
    sc.upload(oracle_backend)
    n = 20000
    rg = sc.run(gpu_backend, n, seed=17)
    ro = sc.run(oracle_backend, n, seed=17)
    for ig, io in zip(rg.instruments, ro.instruments):
        assert ig["total"].sum() == pytest.approx(io["total"].sum(), rel=1e-6)
        assert np.mean(np.isclose(ig["total"], io["total"], rtol=1e-9, atol=0)) > 0.99
        assert np.mean(np.isclose(ig["stats"][1], io["stats"][1], rtol=1e-9, atol=0)) > 0.99
    assert rg.rf.sum() == pytest.approx(ro.rf.sum(), rel=1e-6)
    assert np.mean(np.isclose(rg.rf, ro.rf, rtol=1e-9, atol=0)) > 0.99
    assert rg.counters["stats_overflows"] == 0


@pytest.mark.gpu
def test_gpu_fp32_galaxy_matches_reference_run(golden, gpu_backend):
    """The production (FP32 traversal) life cycle on the reference's exported galaxy: frames, SED,
    radiation field and absorbed luminosity against the reference's own run of the same scene."""
    z, sc = galaxy_scene(golden)
    sc.upload(gpu_backend)
    n = int(z["ref_npp"])
    res, parts = run_subranges(sc, gpu_backend, n, seed=41, precision=abi.PREC_FP32)
    assert res.counters["stats_overflows"] == 0
    check_detectors(z, res, n)
    _, indep = run_subranges(sc, gpu_backend, n, seed=43, precision=abi.PREC_FP32)
    check_radiation_field(sc, z, parts, indep)
