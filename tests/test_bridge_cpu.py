"""The SKIRT-side bridge end to end without a GPU.

oracle/_ref/exe/skirt/bin/skirt_oracle is the bridged reference program of tests/test_gpu_bridge.py
with the bridge's C-ABI calls renamed to the CPU oracle's (oracle/ref.mk target skirt_oracle). It
runs the bridge's own code (support checks, flattening of the SimulationItem tree into the upload
calls, the fetch into FluxRecorder and MediumSystem arrays, the secondary-emission hand-over) with
the oracle's life cycle; its outputs agree with the reference program's within Monte Carlo noise.
"""
import os

import numpy as np
import pytest

import test_gpu_bridge as tb
from skgpu import ski

SKIRT_ORACLE = os.path.join(tb.BIN, "skirt_oracle")

needs_build = pytest.mark.skipif(not os.path.exists(SKIRT_ORACLE) or not os.path.exists(tb.SKIRT),
                                 reason="reference build not present (oracle/ref.mk, run by __graft_entry__.build() "
                                        "where the reference sources are)")


def both(tmp_path, text, name, files=None):
    log = tb.run(SKIRT_ORACLE, text, name, str(tmp_path / "bridge"), ["-g", "-t", "1"], files)
    tb.run(tb.SKIRT, text, name, str(tmp_path / "cpu"), ["-t", "1"], files)
    assert "primary histories on the B200" in log
    return log, str(tmp_path / "bridge"), str(tmp_path / "cpu")


@needs_build
def test_bridge_shell_on_oracle(tmp_path):
    log, g, c = both(tmp_path, ski.shell_cartesian(50000, nbins=16, npix=32), "shell")
    z, (a, b) = tb.sed_z(g, c, "shell", "sed")
    tb.check(z, 9.0, 4.0)
    # the direct flux of the central point source is deterministic: equal to rounding
    da, db = (np.loadtxt(os.path.join(d, "shell_sed_sed.dat"))[3] for d in (g, c))
    assert da == pytest.approx(db, rel=1e-9)
    z, _ = tb.frame_z(g, c, "shell", "i30")
    tb.check(z, 1.3, 5.5)


@needs_build
def test_bridge_galaxy_octree_on_oracle(tmp_path):
    text = ski.galaxy_octree(30000, npix=16, nlambda=10, max_level=5, max_dust_fraction=1e-3, stats=True, sed=True)
    log, g, c = both(tmp_path, text, "galaxy")
    z, _ = tb.sed_z(g, c, "galaxy", "sed")
    tb.check(z, 1.8, 4.5)
    for inc in (0, 60, 90):
        z, _ = tb.frame_z(g, c, "galaxy", f"i{inc}")
        tb.check(z, 1.4, 6.0)


@needs_build
def test_bridge_dust_emission_on_oracle(tmp_path):
    log, g, c = both(tmp_path, ski.dust_shell(50000), "dust")
    assert "secondary histories on the B200" in log
    z, (a, b) = tb.sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    tb.check(z, 2.0, 5.0)
    ir = np.loadtxt(os.path.join(g, "dust_sed_sed.dat"))[:, 0] > 20
    assert a[0][ir].sum() == pytest.approx(b[0][ir].sum(), rel=0.04)


@needs_build
def test_bridge_levels_and_bands_on_oracle(tmp_path):
    """Scattering levels (frame, 3 levels; SED, 2 levels) and a band wavelength grid (four
    overlapping ListBands) through the bridge: SKIRT's own level FITS files and band SED agree with
    the reference program's."""
    log, g, c = both(tmp_path, ski.galaxy_levels_bands(200000), "lb")
    tb.check_levels_and_bands(g, c, "lb")


@needs_build
def test_bridge_dust_emission_adaptive_on_oracle(tmp_path):
    """Primary and secondary segments on an adaptive mesh (the secondary launch in its leaf boxes)."""
    text, files = ski.dust_adaptive(50000)
    log, g, c = both(tmp_path, text, "dust", files)
    assert "secondary histories on the B200" in log
    z, (a, b) = tb.sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    tb.check(z, 2.0, 5.0)


@needs_build
@pytest.mark.parametrize("grid", ["voronoi", "tetra", "sphere1d", "sphere2d", "sphere3d", "cylinder2d", "cylinder3d"])
def test_bridge_dust_emission_other_grids_on_oracle(tmp_path, grid):
    """DustEmission on the Voronoi, tetrahedral, spherical and cylindrical grids: secondary launches
    at random positions in Voronoi cells (rejection in the cell box), tetrahedra (barycentric fold)
    and curvilinear cells."""
    text = ski.dust_tetra(20000, num_vertices=1000) if grid == "tetra" else tb.dust_scene(grid, 50000)
    log, g, c = both(tmp_path, text, "dust")
    assert "secondary histories on the B200" in log
    z, _ = tb.sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    tb.check(z, 2.0, 5.0)


@needs_build
@pytest.mark.parametrize("grid", sorted(tb.GRID_SCENES))
def test_bridge_grids_on_oracle(tmp_path, grid):
    """The disk scene on the adaptive-mesh, Voronoi, tetrahedral, spherical and cylindrical grids:
    the bridge's flattening of each grid through the oracle against the reference program."""
    text, files = tb.GRID_SCENES[grid](20000 if grid == "tetra" else 50000)
    log, g, c = both(tmp_path, text, "disk", files)
    tb.check_disk(g, c, "disk")


@needs_build
def test_bridge_off_is_the_reference(tmp_path):
    """Without -g the bridged program is the reference program: identical outputs."""
    text = ski.shell_cartesian(5000, nbins=8, npix=8)
    la = tb.run(SKIRT_ORACLE, text, "s", str(tmp_path / "a"), ["-t", "1"])
    tb.run(tb.SKIRT, text, "s", str(tmp_path / "b"), ["-t", "1"])
    assert "on the B200" not in la
    sa, sb = (np.loadtxt(os.path.join(tmp_path / d, "s_sed_sed.dat")) for d in ("a", "b"))
    assert np.array_equal(sa, sb)


@needs_build
def test_bridge_dust_self_absorption_on_oracle(tmp_path):
    """Dust self-absorption: the secondary emission iterations (MonteCarloSimulation::
    runSecondaryEmissionIterations) and the final secondary segment store the emission radiation
    field, and each segment's dust emission follows the primary plus the previous secondary field.
    Every segment runs through the bridge; the SED agrees with the reference program's."""
    text = ski.dust_shell(50000, self_absorption=(2, 3))
    log, g, c = both(tmp_path, text, "dust")
    assert log.count("secondary histories on the B200") >= 3  # two iterations and the final segment
    z, (a, b) = tb.sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    tb.check(z, 2.0, 5.0)


@needs_build
def test_bridge_merged_iterations_on_oracle(tmp_path):
    """Merged primary and secondary iterations (includePrimaryEmission,
    MonteCarloSimulation::runMergedEmissionIterations): every segment of the iterations and the final
    segments run through the bridge; the SED agrees with the reference program's."""
    text = ski.dust_shell(50000, self_absorption=(2, 2, True))
    log, g, c = both(tmp_path, text, "dust")
    assert log.count("primary histories on the B200") == 3  # two iterations and the final segment
    assert log.count("secondary histories on the B200") == 3
    z, _ = tb.sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    tb.check(z, 2.0, 5.0)


@needs_build
def test_bridge_redshift_and_aperture_on_oracle(tmp_path):
    """The galaxy at redshift 0.5 (flat-universe cosmology, instruments observing in the redshifted
    frame) with a 3 kpc SED aperture: frame and both SEDs against the reference program."""
    log, g, c = both(tmp_path, ski.galaxy_observer(50000, redshift=0.5, aperture_kpc=3), "g")
    tb.check_observer(g, c, "g")
