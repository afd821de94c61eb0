"""Secondary (dust) emission: the oracle pinned against the reference's own runs.

Fixtures dust_shell.npz (16^3 Cartesian dust shell around a 1e5 Lsun black-body point source) and
dust_galaxy.npz (the galaxy's disk + bulge and dust disk on the reference's own octree, max level 6),
both in DustEmission mode (tests/golden/make_fixtures.py dust_fixtures): the reference's
equilibrium-emission tables, the primary radiation field MediumSystem::_rf1 of a single-threaded
reference run, the reference's own per-cell dust luminosity (MediumSystem::dustLuminosity),
temperature (MediumSystem::indicativeDustTemperature) and emission spectra
(MediumSystem::dustEmissionSpectrum) for that radiation field, and the raw detector sums of the
reference's secondary segment alone (MonteCarloSimulation::runSecondaryEmission into cleared
detectors).

- Per cell, from the reference's radiation field: the oracle's dust luminosity equals the
  reference's bit for bit, its temperature to one rounding (the reference reports the mass-weighted
  mean rho T / rho), its emission spectra are the reference's up to the normalisation.
- The oracle's secondary segment from the same radiation field agrees with the reference's per
  pixel and wavelength bin (z-scores from the per-history statistics).
"""
import numpy as np
import pytest

from helpers import zscores
from skgpu import Scene, abi

FIXTURES = ["dust_shell.npz", "dust_galaxy.npz"]


def dust_scene(golden, name):
    z = golden(name)
    return z, Scene.from_export(z)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_dust_cells_pinned(golden, oracle_backend, name):
    z, sc = dust_scene(golden, name)
    sc.upload(oracle_backend)
    oracle_backend.set_options(sc.options(seed=1))
    oracle_backend.upload_radiation_field(z["rf1"])
    s = sc.secondary
    Ltot = oracle_backend.prepare_secondary(1000, s["spatial_bias"], s["source_bias"], s["wavelength_bias"],
                                            s["bias_range"])
    L, T, lam, pdf, cdf = oracle_backend.fetch_dust_emission(len(sc.density))
    assert np.array_equal(L, z["ref_dust_L"])
    rT = z["ref_dust_T"]
    dusty = sc.density > 0
    assert np.all(T[~dusty] == 0) and np.all(rT[~dusty] == 0)
    assert np.max(np.abs(T[dusty] - rT[dusty]) / rT[dusty]) < 4.5e-16  # one rounding of rho T / rho
    assert 3 < np.median(T[dusty]) < 300
    # the emission pdf at the grid points inside the range is the reference's spectrum, normalised
    cells, spec = z["ref_dust_spec_cells"], z["ref_dust_spec"]
    em = sc.dust_emission["em_lambda"]
    assert np.array_equal(lam[1:-1], em[1:len(lam) - 1])
    for r, m in enumerate(cells):
        p, e = pdf[m, 1:-1], spec[r, 1:len(lam) - 1]
        assert np.array_equal(p > 0, e > 0)  # the Wien tail of cold dust underflows to 0 in both
        ratio = p[e > 0] / e[e > 0]
        assert np.ptp(ratio) <= 1e-13 * ratio.mean()
    assert np.allclose(cdf[cells, -1], 1.0, rtol=1e-14, atol=0)
    assert Ltot == pytest.approx(z["ref_dust_L"].sum(), rel=1e-13)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_secondary_pinned(golden, oracle_backend, name):
    z, sc = dust_scene(golden, name)
    sc.upload(oracle_backend)
    npp = int(z["ref_npp"])
    res, L = sc.run_secondary(oracle_backend, npp, seed=7, rf=z["rf1"])
    assert L > 0
    for i, ins in enumerate(sc.instruments):
        ref = z[f"inst{i}_{'wifu' if ins['kind'] == 0 else 'wsed'}_sec"]
        st = res[i]["stats"].reshape(5, -1)
        zz = zscores(st[1], st[2], npp, ref[1], ref[2], npp)
        assert len(zz) > 10
        assert (zz ** 2).mean() < 1.3, (i, (zz ** 2).mean())
        assert np.abs(zz).max() < 5.5, (i, np.abs(zz).max())
        assert st[1].sum() == pytest.approx(ref[1].sum(), rel=0.02)


def test_oracle_secondary_refuses_unprepared(golden, oracle_backend):
    from skgpu.abi import SkgpuError
    z, sc = dust_scene(golden, "dust_shell.npz")
    sc.upload(oracle_backend)
    oracle_backend.set_options(sc.options(seed=1))
    with pytest.raises(SkgpuError):
        oracle_backend.run_secondary(0, 10)


def secondary_on_grid(golden, grid_fixture):
    """The dust shell's emission tables and a seeded radiation field on another grid (the tetrahedral
    or 1D spherical path fixture): a scene whose secondary launch draws positions in tetrahedra or
    spherical shells. Cell volumes are those of the grid's cells."""
    dust = Scene.from_export(golden("dust_shell.npz"))
    z = golden(grid_fixture)
    sc = Scene.from_export(z)
    n = len(sc.density)
    if sc.grid["kind"] == abi.GRID_TETRA:
        v, t = sc.grid["vertices"], sc.grid["tetra"]
        a, b, c, d = (v[t[:, q]] for q in range(4))
        vol = np.abs(np.einsum("ij,ij->i", b - a, np.cross(c - a, d - a))) / 6.0
    elif sc.grid["kind"] == abi.GRID_VORONOI:
        # the domain as every cell's enclosing box: valid for the rejection draw (longer, same result)
        sc.grid = dict(sc.grid, boxes=np.tile(np.asarray(sc.grid["extent"], dtype=np.float64), (n, 1)))
        vol = np.full(n, 1e48)
    elif sc.grid["kind"] == abi.GRID_SPHERE1D:
        r = np.asarray(sc.grid["rv"])
        vol = 4.0 / 3.0 * np.pi * (r[1:] ** 3 - r[:-1] ** 3)
    else:
        vol = np.full(n, 1e48)  # any positive volumes: GPU and oracle share them
    sc.mix = dust.mix
    sc.instruments = dust.instruments
    sc.rf = dust.rf
    sc.store_rf = True
    sc.dust_emission = dict(dust.dust_emission, cell_volume=vol)
    sc.secondary = dust.secondary
    rng = np.random.default_rng(17)
    rf = rng.uniform(0.5, 1.5, (n, dust.rf["num_bins"])) * np.median(golden("dust_shell.npz")["rf1"])
    return sc, rf


OTHER_GRIDS = ["paths_voronoi.npz", "paths_tetra.npz", "paths_sphere1d.npz", "paths_cylinder2d.npz", "paths_sphere2d.npz",
               "paths_sphere3d.npz", "paths_cylinder3d.npz"]


@pytest.mark.parametrize("fixture", OTHER_GRIDS)
def test_oracle_secondary_launch_in_cells(golden, oracle_backend, fixture):
    """The oracle's secondary segment on the tetrahedral, spherical and cylindrical grids (launch
    positions in tetrahedra and in curvilinear cells) runs every history and reaches the instruments; its
    distributions are tested against the reference's runs through the bridge
    (test_bridge_cpu.py), the GPU's launches against these (test_gpu_secondary.py)."""
    sc, rf = secondary_on_grid(golden, fixture)
    sc.upload(oracle_backend)
    res, L = sc.run_secondary(oracle_backend, 4000, seed=3, rf=rf)
    assert L > 0 and res.counters["histories"] == 4000
    assert sum(float(ins["total"].sum()) for ins in res.instruments) > 0


def test_oracle_secondary_stores_its_radiation_field(golden, oracle_backend):
    """With the radiation field stored, a secondary segment tallies its own field (the emission
    radiation field of dust self-absorption, MediumSystem::storeRadiationField(false, ...)): the
    uploaded primary field is consumed by the preparation and does not reappear in the tally."""
    z = golden("dust_shell.npz")
    sc = Scene.from_export(z)
    sc.upload(oracle_backend)
    res, L = sc.run_secondary(oracle_backend, 5000, seed=3, rf=z["rf1"])
    assert L > 0 and res.rf is not None
    assert 0 < res.rf.sum() < 0.05 * z["rf1"].sum()
    sc.store_rf = False
    res2, _ = sc.run_secondary(oracle_backend, 5000, seed=3, rf=z["rf1"])
    assert res2.rf is None
    for a, b in zip(res.instruments, res2.instruments):
        assert np.array_equal(a["total"], b["total"])
