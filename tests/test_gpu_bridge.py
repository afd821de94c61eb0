"""The drop-in end to end: a ski file run by SKIRT's own program on the B200.

oracle/_ref/exe/skirt/bin/skirt_gpu is the reference's skirt built from its sources with the two
life-cycle hooks (oracle/patch_hooks.py: MonteCarloSimulation::runPrimaryEmission /
runSecondaryEmission hand their segment to SkgpuLifeCycle, and -g switches the bridge on) and the
SKIRT-side bridge skirt9-gpu_b200/bridge/SkgpuLifeCycle.cpp, linked against lib/libskgpu.so. Each
test runs one ski file twice: `skirt_gpu -g` (setup, output and calibration by SKIRT, the life cycle
on the B200) and the unmodified reference `skirt` on the host cores. The SED fluxes (Jy) and frame
surface brightnesses (MJy/sr) that SKIRT writes agree within Monte Carlo noise: z-scores with each
run's relative errors from its own statistics outputs (sum w^k, whose ratio
R = sqrt(sum w^2 / (sum w)^2) is free of the calibration factors).
"""
import os
import subprocess

import numpy as np
import pytest

from skgpu import fits, ski

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "exe", "skirt", "bin")
SKIRT_GPU, SKIRT = os.path.join(BIN, "skirt_gpu"), os.path.join(BIN, "skirt")

needs_build = pytest.mark.skipif(not os.path.exists(SKIRT_GPU) or not os.path.exists(SKIRT),
                                 reason="bridged reference program not built (oracle/ref.mk target bridge, "
                                        "run by __graft_entry__.build() where the reference sources are)")


def run(exe, text, name, cwd, args, files=None):
    os.makedirs(cwd, exist_ok=True)
    with open(os.path.join(cwd, name + ".ski"), "w") as f:
        f.write(text)
    for fn, content in (files or {}).items():
        with open(os.path.join(cwd, fn), "w") as f:
            f.write(content)
    p = subprocess.run([exe] + args + [name + ".ski"], cwd=cwd, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    with open(os.path.join(cwd, name + "_log.txt")) as f:
        return f.read()


def rel_err(s1, s2):
    return np.sqrt(np.maximum(s2, 0)) / np.where(s1 > 0, s1, np.inf)


def z_of(fa, ra, fb, rb):
    m = (fa > 0) & (fb > 0)
    den = np.hypot(ra[m] * fa[m], rb[m] * fb[m])
    ok = den > 0
    return (fa[m][ok] - fb[m][ok]) / den[ok]


def sed_z(da, db, name, instr):
    out = []
    for d in (da, db):
        sed = np.atleast_2d(np.loadtxt(os.path.join(d, f"{name}_{instr}_sed.dat")))
        st = np.atleast_2d(np.loadtxt(os.path.join(d, f"{name}_{instr}_sedstats.dat")))
        out.append((sed[:, 1], rel_err(st[:, 2], st[:, 3])))
    return z_of(out[0][0], out[0][1], out[1][0], out[1][1]), out


def frame_z(da, db, name, instr):
    out = []
    for d in (da, db):
        total = fits.read(os.path.join(d, f"{name}_{instr}_total.fits"))[0].astype(np.float64).ravel()
        s1 = fits.read(os.path.join(d, f"{name}_{instr}_stats1.fits"))[0].astype(np.float64).ravel()
        s2 = fits.read(os.path.join(d, f"{name}_{instr}_stats2.fits"))[0].astype(np.float64).ravel()
        out.append((total, rel_err(s1, s2)))
    return z_of(out[0][0], out[0][1], out[1][0], out[1][1]), out


def both(tmp_path, text, name, files=None):
    # the reference runs single-threaded: its multi-threaded runs sample the cell densities from
    # randomly seeded threads, so their medium differs from run to run (and from the bridge's, which
    # takes the densities of its own single-threaded setup)
    log = run(SKIRT_GPU, text, name, str(tmp_path / "gpu"), ["-g", "-t", "1"], files)
    run(SKIRT, text, name, str(tmp_path / "cpu"), ["-t", "1"], files)
    assert "B200 photon-packet life cycle" in log
    assert "primary histories on the B200" in log
    return log, str(tmp_path / "gpu"), str(tmp_path / "cpu")


def check_levels_and_bands(g, c, name):
    """Band SED (z-scores from the per-band statistics), frame, and the scattering-level outputs of
    ski.galaxy_levels_bands: summed level planes and the SED's level columns within a few per cent
    (no per-plane statistics exist; at 2e5 packets the spread is ~1 % for levels 1-2)."""
    z, _ = sed_z(g, c, name, "bands")
    assert len(z) == 4
    check(z, 4.0, 4.0)
    z, _ = frame_z(g, c, name, "i60")
    check(z, 1.4, 6.0)
    for n, tol in ((1, 0.04), (2, 0.04), (3, 0.08)):
        a, b = (fits.read(os.path.join(d, f"{name}_i60_primaryscattered{n}.fits"))[0].astype(np.float64).sum()
                for d in (g, c))
        assert a > 0 and a == pytest.approx(b, rel=tol), n
    sa, sb = (np.loadtxt(os.path.join(d, f"{name}_bands_sed.dat")) for d in (g, c))
    assert sa.shape == sb.shape == (4, 10)
    assert np.allclose(sa[:, 8:10].sum(axis=0), sb[:, 8:10].sum(axis=0), rtol=0.04)


def check_observer(g, c, name):
    """Frame and SEDs of ski.galaxy_observer: within noise, the aperture SED below the full one, and
    nothing below 0.15 micron (the shortest source wavelength times 1 + z)."""
    for ins in ("sed", "ap"):
        z, _ = sed_z(g, c, name, ins)
        assert len(z) >= 8
        check(z, 4.0, 4.0)
    full, ap = (np.loadtxt(os.path.join(g, f"{name}_{i}_sed.dat"))[:, 1] for i in ("sed", "ap"))
    assert 0 < ap.sum() < full.sum() and full[0] == 0
    z, _ = frame_z(g, c, name, "i60")
    check(z, 1.4, 6.0)


def check(z, chi2_max, zmax):
    """Mean square z below chi2_max; the 99.9th percentile of |z| below zmax (frame pixels see rare
    high-weight contributions, so the largest |z| of ~2e4 pixels is not a good test)."""
    assert len(z) > 0
    assert (z ** 2).mean() < chi2_max, (z ** 2).mean()
    assert np.quantile(np.abs(z), 0.999) < zmax, np.quantile(np.abs(z), 0.999)


@needs_build
def test_bridge_dust_shell_oligochromatic(tmp_path):
    """Cartesian 16^3 dust shell, one wavelength, forced scattering: frame and SED."""
    text = ski.shell_cartesian(200000, nbins=16, npix=32)
    log, g, c = both(tmp_path, text, "shell")
    z, _ = sed_z(g, c, "shell", "sed")
    check(z, 9.0, 4.0)
    z, (a, b) = frame_z(g, c, "shell", "i30")
    check(z, 1.3, 5.5)
    assert a[0].sum() == pytest.approx(b[0].sum(), rel=0.01)


@needs_build
def test_bridge_galaxy_octree(tmp_path):
    """The galaxy on the reference's own octree (max level 6), 20 wavelengths, three frames and an
    SED, radiation field stored."""
    text = ski.galaxy_octree(200000, npix=32, nlambda=20, max_level=6, max_dust_fraction=1e-4, stats=True, sed=True)
    log, g, c = both(tmp_path, text, "galaxy")
    z, _ = sed_z(g, c, "galaxy", "sed")
    check(z, 1.6, 4.5)
    for inc in (0, 60, 90):
        z, _ = frame_z(g, c, "galaxy", f"i{inc}")
        check(z, 1.3, 6.0)


@needs_build
def test_bridge_levels_and_bands(tmp_path):
    """Scattering levels and a band wavelength grid on the B200 through SKIRT's own program."""
    log, g, c = both(tmp_path, ski.galaxy_levels_bands(200000), "lb")
    check_levels_and_bands(g, c, "lb")


# the disk scene on every other grid kind the bridge hands over (name, ski text, input files)
GRID_SCENES = {
    "adaptive": lambda n: (ski.disk_adaptive(n), {"mesh.txt": ski.adaptive_mesh_text()}),
    "voronoi": lambda n: (ski.disk_scene(ski.voronoi_grid(4, "pc", 2000), n), None),
    "tetra": lambda n: (ski.disk_scene(ski.tetra_grid(4, "pc", 2000), n), None),
    "sphere2d": lambda n: (ski.disk_sphere2d(n), None),
    "sphere3d": lambda n: (ski.disk_sphere3d(n), None),
    "cylinder2d": lambda n: (ski.disk_cylinder2d(n), None),
    "cylinder3d": lambda n: (ski.disk_cylinder3d(n), None),
}


def check_disk(g, c, name):
    z, _ = frame_z(g, c, name, "i60")
    check(z, 1.4, 6.0)
    z, _ = sed_z(g, c, name, "sed")
    assert len(z) == 1 and abs(z[0]) < 4.5


@needs_build
def test_bridge_dust_emission_adaptive(tmp_path):
    """DustEmission on an adaptive mesh: both segments on the B200, secondary launches in leaf boxes."""
    text, files = ski.dust_adaptive(200000)
    log, g, c = both(tmp_path, text, "dust", files)
    assert "secondary histories on the B200" in log
    z, (a, b) = sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    check(z, 2.0, 5.0)
    z, _ = frame_z(g, c, "dust", "i30")
    check(z, 1.3, 6.0)


@needs_build
def dust_scene(grid, n):
    """The DustEmission shell on one of the non-box grids."""
    if grid == "tetra":
        return ski.dust_tetra(n)
    if grid == "sphere1d":
        return ski.dust_sphere1d(n)
    if grid == "voronoi":
        return ski.dust_shell(n, grid=ski.voronoi_grid(1, "pc", 2000))
    return ski.dust_curvilinear(n, grid)


@pytest.mark.parametrize("grid", ["voronoi", "tetra", "sphere1d", "sphere2d", "sphere3d", "cylinder2d", "cylinder3d"])
def test_bridge_dust_emission_other_grids(tmp_path, grid):
    """DustEmission on the Voronoi, tetrahedral, spherical and cylindrical grids through skirt_gpu -g."""
    text = dust_scene(grid, 200000)
    log, g, c = both(tmp_path, text, "dust")
    assert "secondary histories on the B200" in log
    z, _ = sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    check(z, 2.0, 5.0)
    z, _ = frame_z(g, c, "dust", "i30")
    check(z, 1.3, 6.0)


@needs_build
@pytest.mark.parametrize("grid", sorted(GRID_SCENES))
def test_bridge_grids(tmp_path, grid):
    """The disk scene on the adaptive-mesh, Voronoi, tetrahedral, spherical and cylindrical grids
    through skirt_gpu -g: frame and SED against the reference program's run."""
    text, files = GRID_SCENES[grid](200000)
    log, g, c = both(tmp_path, text, "disk", files)
    check_disk(g, c, "disk")


@needs_build
def test_bridge_dust_emission(tmp_path):
    """DustEmission mode: primary and secondary (equilibrium dust) segments both on the B200; the SED
    from the ultraviolet to the submillimetre and the frame."""
    text = ski.dust_shell(200000)
    log, g, c = both(tmp_path, text, "dust")
    assert "secondary histories on the B200" in log
    # the secondary emission also inherits the noise of the primary segment's radiation field, which
    # the per-history statistics do not include: a little more room for the mean square z
    z, (a, b) = sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    check(z, 2.0, 5.0)
    fa, fb = a[0], b[0]
    ir = np.loadtxt(os.path.join(g, "dust_sed_sed.dat"))[:, 0] > 20
    assert fa[ir].sum() == pytest.approx(fb[ir].sum(), rel=0.03)  # the dust emission itself
    z, _ = frame_z(g, c, "dust", "i30")
    check(z, 1.3, 6.0)


@needs_build
def test_bridge_dust_self_absorption(tmp_path):
    """Dust self-absorption on the B200: the secondary emission iterations and the final secondary
    segment store the emission radiation field; SED and frame against the reference program."""
    text = ski.dust_shell(200000, self_absorption=(2, 3))
    log, g, c = both(tmp_path, text, "dust")
    assert log.count("secondary histories on the B200") >= 3
    z, _ = sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    check(z, 2.0, 5.0)
    z, _ = frame_z(g, c, "dust", "i30")
    check(z, 1.3, 6.0)


@needs_build
def test_bridge_merged_iterations(tmp_path):
    """Merged primary and secondary iterations on the B200: every segment through the bridge; SED
    and frame against the reference program."""
    text = ski.dust_shell(200000, self_absorption=(2, 2, True))
    log, g, c = both(tmp_path, text, "dust")
    assert log.count("primary histories on the B200") == 3
    z, _ = sed_z(g, c, "dust", "sed")
    assert len(z) > 25
    check(z, 2.0, 5.0)
    z, _ = frame_z(g, c, "dust", "i30")
    check(z, 1.3, 6.0)


@needs_build
def test_bridge_redshift_and_aperture(tmp_path):
    """Redshift 0.5 and a 3 kpc SED aperture on the B200 through skirt_gpu -g."""
    log, g, c = both(tmp_path, ski.galaxy_observer(200000, redshift=0.5, aperture_kpc=3), "g")
    check_observer(g, c, "g")
