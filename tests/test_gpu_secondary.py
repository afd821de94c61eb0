"""Secondary (dust) emission on the GPU, against the oracle and the reference's own runs.

Fixtures dust_shell.npz (Cartesian) and dust_galaxy.npz (the reference's octree), see
test_dust_emission_cpu.py. From the reference's primary radiation field:
- the device's per-cell dust luminosity and temperature equal the oracle's bit for bit (no FMA
  contraction, the reference's summation order), its normalised emission spectra to 1e-12
  (last-bit differences of CUDA's exp, log and pow);
- the FP64 secondary life cycle equals the oracle's history by history (tallies to 1e-9);
- the production FP32 secondary life cycle agrees with the reference's secondary segment per pixel
  and bin (z-scores);
- the chain primary segment -> device radiation field -> secondary segment runs without leaving the
  device and agrees with the reference's secondary segment.
"""
import numpy as np
import pytest

from helpers import zscores
from skgpu import Scene, abi

pytestmark = pytest.mark.gpu

FIXTURES = ["dust_shell.npz", "dust_galaxy.npz"]


def scene(golden, name):
    z = golden(name)
    return z, Scene.from_export(z)


def prepare(be, sc, z, npp, precision=abi.PREC_FP64_EXACT):
    sc.upload(be)
    be.set_options(sc.options(seed=3, precision=precision))
    be.upload_radiation_field(z["rf1"])
    s = sc.secondary
    return be.prepare_secondary(npp, s["spatial_bias"], s["source_bias"], s["wavelength_bias"], s["bias_range"])


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_dust_cells_equal_oracle(golden, gpu_backend, oracle_backend, name):
    z, sc = scene(golden, name)
    Lg = prepare(gpu_backend, sc, z, 1000)
    Lo = prepare(oracle_backend, sc, z, 1000)
    assert Lg == Lo
    g = gpu_backend.fetch_dust_emission(len(sc.density))
    o = oracle_backend.fetch_dust_emission(len(sc.density))
    assert np.array_equal(g[0], o[0])  # luminosity
    assert np.array_equal(g[1], o[1])  # temperature
    assert np.array_equal(g[2], o[2])  # spectrum axis
    for a, b in ((g[3], o[3]), (g[4], o[4])):  # pdf, cdf
        assert np.array_equal(a > 0, b > 0)
        m = b > 0
        assert np.max(np.abs(a[m] - b[m]) / b[m]) < 1e-12


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_secondary_fp64_equals_oracle(golden, gpu_backend, oracle_backend, name):
    z, sc = scene(golden, name)
    n = 20000
    sc.upload(gpu_backend)
    sc.upload(oracle_backend)
    rg, Lg = sc.run_secondary(gpu_backend, n, seed=11, rf=z["rf1"])
    ro, Lo = sc.run_secondary(oracle_backend, n, seed=11, rf=z["rf1"])
    assert Lg == Lo
    assert rg.counters["histories"] == n
    assert rg.counters["scatterings"] == ro.counters["scatterings"]
    for a, b in zip(rg.instruments, ro.instruments):
        ta, tb = a["total"].ravel(), b["total"].ravel()
        assert tb.sum() > 0
        assert np.allclose(ta, tb, rtol=1e-9, atol=1e-12 * np.abs(tb).max())
        sa, sb = a["stats"].reshape(5, -1), b["stats"].reshape(5, -1)
        assert np.array_equal(sa[0], sb[0])
        assert np.allclose(sa[2], sb[2], rtol=1e-9, atol=1e-12 * np.abs(sb[2]).max())
    # the segment's own radiation field (dust self-absorption: storeEmissionRadiationField)
    assert ro.rf.sum() > 0
    assert rg.rf.sum() == pytest.approx(ro.rf.sum(), rel=1e-9)
    assert np.mean(np.isclose(rg.rf, ro.rf, rtol=1e-9, atol=1e-12 * ro.rf.max())) > 0.995


def check_vs_reference(res, z, sc, npp, chi2_max=1.3, zmax=5.5, tot_rel=0.02):
    for i, ins in enumerate(sc.instruments):
        ref = z[f"inst{i}_{'wifu' if ins['kind'] == 0 else 'wsed'}_sec"]
        st = res[i]["stats"].reshape(5, -1)
        zz = zscores(st[1], st[2], npp, ref[1], ref[2], npp)
        assert len(zz) > 10
        assert (zz ** 2).mean() < chi2_max, (i, (zz ** 2).mean())
        assert np.abs(zz).max() < zmax, (i, np.abs(zz).max())
        assert st[1].sum() == pytest.approx(ref[1].sum(), rel=tot_rel)


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_secondary_fp32_vs_reference(golden, gpu_backend, name):
    z, sc = scene(golden, name)
    npp = int(z["ref_npp"])
    sc.upload(gpu_backend)
    res, L = sc.run_secondary(gpu_backend, npp, seed=5, precision=abi.PREC_FP32, rf=z["rf1"])
    assert L > 0
    check_vs_reference(res, z, sc, npp)


def test_gpu_primary_then_secondary_on_device(golden, gpu_backend):
    """The secondary segment prepared from the radiation field the primary segment left on the
    device (no host round trip); its own radiation-field noise widens the comparison a little."""
    z, sc = scene(golden, "dust_shell.npz")
    sc.upload(gpu_backend)
    npp = int(z["ref_npp"])
    sc.run(gpu_backend, 10 * npp, seed=21, precision=abi.PREC_FP32)
    s = sc.secondary
    L = gpu_backend.prepare_secondary(npp, s["spatial_bias"], s["source_bias"], s["wavelength_bias"], s["bias_range"])
    assert L == pytest.approx(z["ref_dust_L"].sum(), rel=0.02)
    gpu_backend.clear_tallies()  # the prepared segment no longer needs the radiation field
    gpu_backend.run_secondary(0, npp)
    check_vs_reference(sc.fetch(gpu_backend, rf=False), z, sc, npp, chi2_max=1.6, zmax=6.5, tot_rel=0.03)


@pytest.mark.parametrize("fixture", ["paths_voronoi.npz", "paths_tetra.npz", "paths_sphere1d.npz", "paths_cylinder2d.npz",
                                     "paths_sphere2d.npz", "paths_sphere3d.npz", "paths_cylinder3d.npz"])
def test_gpu_secondary_other_grids_equal_oracle(golden, gpu_backend, oracle_backend, fixture):
    """Secondary launches in Voronoi cells (rejection in the cell box, VoronoiMeshSnapshot::generatePosition),
    in tetrahedra (TetraMeshSpatialGrid::Tetra::generatePosition) and in the
    cells of the spherical and cylindrical grids (their randomPositionInCell): the FP64 secondary life
    cycle equals the oracle's history by history (radii and angles through CUDA's cbrt, sqrt, acos,
    cos and sin, to the last bit or so)."""
    from test_dust_emission_cpu import secondary_on_grid
    sc, rf = secondary_on_grid(golden, fixture)
    n = 20000
    sc.upload(gpu_backend)
    sc.upload(oracle_backend)
    rg, Lg = sc.run_secondary(gpu_backend, n, seed=13, rf=rf)
    ro, Lo = sc.run_secondary(oracle_backend, n, seed=13, rf=rf)
    assert Lg == pytest.approx(Lo, rel=1e-12)
    assert rg.counters["histories"] == n
    assert rg.counters["scatterings"] == pytest.approx(ro.counters["scatterings"], rel=1e-3)
    for a, b in zip(rg.instruments, ro.instruments):
        ta, tb = a["total"].ravel(), b["total"].ravel()
        assert tb.sum() > 0
        assert ta.sum() == pytest.approx(tb.sum(), rel=1e-6)
        assert np.mean(np.isclose(ta, tb, rtol=1e-9, atol=1e-12 * np.abs(tb).max())) > 0.99
