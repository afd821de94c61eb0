"""Generates the golden fixtures under tests/golden/ from the reference SKIRT 9 build.

Runs only where the reference sources are present (it needs oracle/_ref, built by
`make -f oracle/ref.mk`): the export harness (oracle/_ref/exe/skirt/bin/skirt_export) loads each
ski file through the reference's own SimulationItem tree and dumps the flattened grid, medium and
instrument state plus the path segments of the reference's CPU generators for a set of rays; the
reference `skirt` program (single-threaded, so that its setup is reproducible) produces the image
and SED statistics of the dust-shell run.

    python tests/golden/make_fixtures.py

Fixtures written:
  paths_<name>.npz   grid + medium export, rays, reference (count, m, ds) per ray, reference tau
  shell_c16.npz      export of the 16^3 dust-shell scene + reference SED/frame statistics of a
                     2e5-packet run
  shell_c16_explicit.npz  reference frame/SED statistics of the same scene with explicit absorption
                     (forced and free propagation), 2e5 packets each; `python
                     tests/golden/make_fixtures.py explicit` writes only this one
  paths_sphere1d.npz, paths_cylinder2d.npz, paths_sphere2d.npz, paths_sphere3d.npz,
  paths_cylinder3d.npz, paths_adaptive.npz  path fixtures that also hold reference frame/SED statistics of the same
                     scene (arguments `sphere1d`, `cylinder2d`, `sphere2d`, `sphere3d`, `cylinder3d`, `adaptive`
                     write only them)
  stats_octree.npz, stats_voronoi.npz, stats_tetra.npz  the disk scene on these grids (scene export)
                     with reference frame/SED statistics (argument `gridstats`)
  shell_c16_free.npz the raw detector sums (w^0, w^1, w^2 of frame and SED) of a single-threaded
                     2e5-packet reference run of the 16^3 shell with free (non-forced) propagation
                     (argument `free`)
  stats_galaxy.npz   the galaxy configuration reduced in size (stellar exponential disk + Sersic
                     bulge with black-body SEDs and wavelength bias 0.5, dust disk on the reference's
                     own octree of max level 6, 20 log wavelengths, three 32^2 frames and an SED with
                     statistics, radiation field stored): scene export, the raw detector sums
                     (w^0, w^1, w^2 per pixel and bin) and the primary radiation field of a
                     single-threaded 5e5-packet reference run, and 2e4 reference launches
                     (argument `galaxy`)
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "skirt9-gpu_b200"))
from skgpu import fits, ski  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "exe", "skirt", "bin")
OUT = os.path.dirname(os.path.abspath(__file__))
PC = 3.08567758e16  # SKIRT's parsec in m


def export(ski_text, tmp, rays=None, max_seg=512, lam=0.55e-6, files=None):
    ski_path = os.path.join(tmp, "scene.ski")
    with open(ski_path, "w") as f:
        f.write(ski_text)
    for name, text in (files or {}).items():
        with open(os.path.join(tmp, name), "w") as f:
            f.write(text)
    exp = os.path.join(tmp, "export")
    os.makedirs(exp, exist_ok=True)
    args = [os.path.join(BIN, "skirt_export"), ski_path, exp]
    if rays is not None:
        np.save(os.path.join(tmp, "rays.npy"), rays)
        args += [os.path.join(tmp, "rays.npy"), str(max_seg), repr(lam)]
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, cwd=tmp)
    data = {}
    for fn in os.listdir(exp):
        if fn.endswith(".npy"):
            data[fn[:-4]] = np.load(os.path.join(exp, fn))
    with open(os.path.join(exp, "meta.txt")) as f:
        data["meta"] = np.array(f.read())
    return data


def random_rays(rng, n, half, out_frac=0.3):
    """Rays starting inside the box and (a fraction) outside it, isotropic directions, plus
    rays along the axes and diagonals through the centre (exact ties with cell walls)."""
    pos = rng.uniform(-half, half, (n, 3))
    nout = int(out_frac * n)
    pos[:nout] *= rng.uniform(1.05, 1.6, (nout, 1))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    special = []
    for k in ([1, 0, 0], [0, -1, 0], [0, 0, 1], [1, 1, 0], [1, 1, 1], [-1, 2, 0.5]):
        k = np.array(k, float) / np.linalg.norm(k)
        special.append(np.r_[0.0, 0.0, 0.0, k])
        special.append(np.r_[0.1 * half, 0.0, -0.2 * half, k])
    return np.vstack([np.hstack([pos, d]), np.array(special)])


def path_fixture(name, ski_text, rays, max_seg=512, files=None):
    with tempfile.TemporaryDirectory() as tmp:
        data = export(ski_text, tmp, rays, max_seg, files=files)
    data["rays"] = rays
    # keep the segments ragged: ray r owns ray_m[off[r]:off[r+1]] (no truncated paths allowed)
    cnt = data["ray_count"]
    assert (cnt >= 0).all(), "a reference path was truncated; raise max_seg"
    data["ray_offset"] = np.r_[0, np.cumsum(cnt)].astype(np.int64)
    data["ray_m"] = np.concatenate([data["ray_m"][r, :c] for r, c in enumerate(cnt)]).astype(np.int32)
    data["ray_ds"] = np.concatenate([data["ray_ds"][r, :c] for r, c in enumerate(cnt)])
    np.savez_compressed(os.path.join(OUT, f"paths_{name}.npz"), **data)
    print(f"paths_{name}: {len(rays)} rays, {np.abs(cnt).sum()} segments, max {np.abs(cnt).max()}")


def main():
    if not os.path.exists(os.path.join(BIN, "skirt_export")):
        sys.exit("reference build missing: run `make -f oracle/ref.mk -j8` first")
    rng = np.random.default_rng(20260101)

    # Cartesian: the reference self-test grid (SKIRT/core/GpuAcceleration.cpp:12753-12755) with
    # its rays (:12951-12953) and random rays, and the 16^3 shell grid
    xb = np.array([-1.2, -0.5, 0.1, 0.7, 1.4, 2.0])
    yb = np.array([-0.8, -0.2, 0.25, 0.9])
    zb = np.array([-0.4, 0.0, 0.35, 0.8, 1.3])
    norm = lambda b: (b - b[0]) / (b[-1] - b[0])
    grid = (f'<CartesianSpatialGrid minX="{xb[0]} pc" maxX="{xb[-1]} pc" minY="{yb[0]} pc" maxY="{yb[-1]} pc" '
            f'minZ="{zb[0]} pc" maxZ="{zb[-1]} pc">'
            + "".join(f'<mesh{a} type="Mesh"><ListMesh points="' + ", ".join(f"{p:.17g}" for p in norm(b))
                      + f'"/></mesh{a}>' for a, b in zip("XYZ", (xb, yb, zb)))
            + '</CartesianSpatialGrid>')
    st = []
    for p, k in (((-2.1, -0.55, 0.2), (1.0, 0.26, 0.08)), ((0.1, -0.2, 0.0), (1.0, 1.0, 1.0))):
        k = np.array(k) / np.linalg.norm(k)
        st.append(np.r_[np.array(p) * PC, k])
    rays = np.vstack([np.array(st), random_rays(rng, 300, 1.6 * PC)])
    rays[2:, :3] += 0.4 * PC
    path_fixture("cartesian_selftest", ski.disk_probe(grid), rays)
    path_fixture("cartesian_c16", ski.shell_cartesian(1e4, nbins=16, npix=64), random_rays(rng, 300, PC))

    # octree (DensityTreePolicy on a flattened exponential disk: many levels, uneven neighbours)
    path_fixture("octree", ski.disk_probe(ski.octree_grid(4, "pc", 6, 1e-3)), random_rays(rng, 300, 4 * PC))
    # Voronoi and tetrahedral meshes built by the reference (voro++ / TetGen) from disk-sampled sites
    path_fixture("voronoi", ski.disk_probe(ski.voronoi_grid(4, "pc", 300)), random_rays(rng, 300, 4 * PC))
    path_fixture("tetra", ski.disk_probe(ski.tetra_grid(4, "pc", 300)), random_rays(rng, 300, 4 * PC))
    sphere1d_fixture(rng)
    cylinder2d_fixture()
    sphere2d_fixture()
    sphere3d_fixture()
    cylinder3d_fixture()
    grid_stats_fixtures()
    galaxy_fixture()
    dust_fixtures()

    # dust shell, 16^3 grid, 64^2 frame + SED: scene export + reference statistics (2e5 packets)
    npp = 200000
    with tempfile.TemporaryDirectory() as tmp:
        text = ski.shell_cartesian(npp, nbins=16, npix=64)
        data = export(text, tmp)
        run = os.path.join(tmp, "run")
        os.makedirs(run)
        with open(os.path.join(run, "c16.ski"), "w") as f:
            f.write(text)
        subprocess.run([os.path.join(BIN, "skirt"), "-t", "1", "c16.ski"], cwd=run, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        sedstats = np.loadtxt(os.path.join(run, "c16_sed_sedstats.dat"))
        sed = np.loadtxt(os.path.join(run, "c16_sed_sed.dat"))
        stats = np.array([fits.read(os.path.join(run, f"c16_i30_stats{k}.fits"))[0][0] for k in range(5)])
        total = fits.read(os.path.join(run, "c16_i30_total.fits"))[0][0]
    # The stats files are scaled by c^k (FluxRecorder.cpp:1216-1236). Recover c from the
    # transparent SED flux, whose raw value (total luminosity per packet summed) is known exactly:
    # frame surface brightness per raw W = (SED Jy per raw W) * 1e-6 / pixel solid angle.
    meta, load, _ = __import__("skgpu").Scene.read_export(data)
    lum = load("src_probe")[0, 1]                     # L * npp of one packet = raw transparent SED sum
    jy_per_w = sed[2] / lum
    pix = float(meta["instr0_xpsiz"]) / float(meta["instr0_distance"])
    mjysr_per_w = jy_per_w * 1e-6 / (pix * pix)
    w1 = total / mjysr_per_w
    c = stats[1].sum() / w1.sum()
    data.update(ref_npp=npp, ref_sedstats=sedstats[1:], ref_sed_jy=sed[1:], ref_frame_w=np.array(
        [stats[0], stats[1] / c, stats[2] / c ** 2]), ref_stats_scale=c, ref_jy_per_w=jy_per_w)
    np.savez_compressed(os.path.join(OUT, "shell_c16.npz"), **data)
    print("shell_c16: stats scale", c)
    explicit_fixture(mjysr_per_w, npp)
    free_fixture()


def sphere1d_fixture(rng=None):
    """Sphere1DSpatialGrid (the dust shell, 24 radial bins between 0.05 and 1 pc, no cell inside
    0.05 pc): scene export and path fixture with random rays plus radial and tangent rays (exact
    shell borders, rays through the centre, rays starting inside and outside)."""
    rng = rng if rng is not None else np.random.default_rng(20260102)
    rays = random_rays(rng, 300, 1.2 * PC)
    extra = []
    for r0 in (0.0, 0.25, 0.5, 1.0 + 1e-9):
        extra.append(np.r_[np.array([r0, 0.0, 0.0]) * PC, [1.0, 0.0, 0.0]])
        extra.append(np.r_[np.array([r0, 0.0, 0.0]) * PC, [-1.0, 0.0, 0.0]])
    for b in (0.1, 0.5, 1.0 / 24 * 7):
        extra.append(np.r_[np.array([-2.0, b, 0.0]) * PC, [1.0, 0.0, 0.0]])
    rays = np.vstack([rays, np.array(extra)])
    path_fixture("sphere1d", ski.shell_sphere1d(1e4, nbins=24, npix=32), rays)
    # reference statistics of the same scene: a single-threaded 2e5-packet run; its stats files are
    # scaled by the run's own c, recovered from the total image (MJy/sr per raw W from the SED's
    # Jy per raw W of the shell_c16 run, same distance, and this frame's pixel)
    npp = 200000
    path = os.path.join(OUT, "paths_sphere1d.npz")
    data = dict(np.load(path))
    meta = __import__("skgpu").Scene.read_export(data)[0]
    pix = float(meta["instr0_xpsiz"]) / float(meta["instr0_distance"])
    mjysr_per_w = float(np.load(os.path.join(OUT, "shell_c16.npz"))["ref_jy_per_w"]) * 1e-6 / (pix * pix)
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "s1.ski"), "w") as f:
            f.write(ski.shell_sphere1d(npp, nbins=24, npix=32))
        subprocess.run([os.path.join(BIN, "skirt"), "-t", "1", "s1.ski"], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        st = np.array([fits.read(os.path.join(tmp, f"s1_i30_stats{k}.fits"))[0][0] for k in range(5)])
        ss = np.loadtxt(os.path.join(tmp, "s1_sed_sedstats.dat"))
        total = fits.read(os.path.join(tmp, "s1_i30_total.fits"))[0][0]
    c = st[1].sum() / (total / mjysr_per_w).sum()
    data.update(ref_npp=npp, ref_frame_w=np.array([st[0], st[1] / c, st[2] / c ** 2]), ref_sedstats=ss[1:])
    np.savez_compressed(path, **data)


def cylinder2d_fixture(rng=None):
    """Cylinder2DSpatialGrid (exponential disk, R 0.05-4 pc in 20 bins, z -1..1 pc in 16 bins):
    scene export and path fixture (random rays, many starting outside in z, plus vertical,
    horizontal and radial rays), and reference statistics of a single-threaded 2e5-packet run."""
    rng = rng if rng is not None else np.random.default_rng(20260103)
    rays = random_rays(rng, 300, 4.5 * PC)
    extra = []
    for k in ((0, 0, 1), (0, 0, -1), (1, 0, 0), (0.6, 0.8, 0.0), (0.3, 0.0, 0.95)):
        k = np.array(k, float) / np.linalg.norm(k)
        for p in ((0.0, 0.0, 0.0), (1.0, 0.5, 0.3), (5.0, 0.0, 0.1), (0.0, 0.0, -2.0), (0.02, 0.0, 0.0)):
            extra.append(np.r_[np.array(p) * PC, k])
    rays = np.vstack([rays, np.array(extra)])
    path_fixture("cylinder2d", ski.disk_cylinder2d(1e4), rays)
    reference_stats("paths_cylinder2d.npz", ski.disk_cylinder2d(200000), "i60", 200000)


def sphere2d_fixture(rng=None):
    """Sphere2DSpatialGrid (the disk scene, r 0.05-4 pc in 20 bins, 15 polar bins plus the equatorial
    border): scene export and path fixture (random rays plus rays along the axis, in the equatorial
    plane and from outside), and reference statistics of a single-threaded 2e5-packet run."""
    rng = rng if rng is not None else np.random.default_rng(20260104)
    rays = random_rays(rng, 300, 3.5 * PC)
    extra = []
    for k in ((0, 0, 1), (0, 0, -1), (1, 0, 0), (0.6, 0.8, 0.0), (0.3, 0.0, 0.95), (-0.5, 0.5, -0.7071067811865476)):
        k = np.array(k, float) / np.linalg.norm(k)
        for p in ((0.0, 0.0, 0.0), (1.0, 0.5, 0.3), (5.0, 0.0, 0.1), (0.0, 0.0, -2.0), (0.02, 0.0, 0.0)):
            extra.append(np.r_[np.array(p) * PC, k])
    rays = np.vstack([rays, np.array(extra)])
    path_fixture("sphere2d", ski.disk_sphere2d(1e4), rays)
    reference_stats("paths_sphere2d.npz", ski.disk_sphere2d(200000), "i60", 200000)


def sphere3d_fixture(rng=None):
    """Sphere3DSpatialGrid (the disk scene, r up to 4 pc in 12 bins with the grid's artificial inner
    hole, 9 polar and 8 azimuthal bins): scene export and path fixture (random rays plus rays along
    the axis, in the equatorial plane, through the centre and from outside), and reference
    statistics of a single-threaded 2e5-packet run."""
    rng = rng if rng is not None else np.random.default_rng(20260105)
    rays = random_rays(rng, 300, 3.5 * PC)
    extra = []
    for k in ((0, 0, 1), (0, 0, -1), (1, 0, 0), (0.6, 0.8, 0.0), (0.3, 0.0, 0.95), (-0.5, 0.5, -0.7071067811865476)):
        k = np.array(k, float) / np.linalg.norm(k)
        for p in ((0.0, 0.0, 0.0), (1.0, 0.5, 0.3), (5.0, 0.0, 0.1), (0.0, 0.0, -2.0), (-0.02, 0.01, 0.0)):
            extra.append(np.r_[np.array(p) * PC, k])
    rays = np.vstack([rays, np.array(extra)])
    path_fixture("sphere3d", ski.disk_sphere3d(1e4), rays)
    reference_stats("paths_sphere3d.npz", ski.disk_sphere3d(200000), "i60", 200000)


def cylinder3d_fixture(rng=None):
    """Cylinder3DSpatialGrid (the disk scene, R up to 4 pc in 12 bins with the grid's artificial inner
    hole, 8 azimuthal bins, z -1..1 pc in 10 bins): scene export and path fixture (random rays plus
    vertical rays through the hole, radial and tangent rays, starts outside), and reference
    statistics of a single-threaded 2e5-packet run."""
    rng = rng if rng is not None else np.random.default_rng(20260106)
    rays = random_rays(rng, 300, 4.5 * PC)
    extra = []
    for k in ((0, 0, 1), (0, 0, -1), (1, 0, 0), (0.6, 0.8, 0.0), (0.3, 0.0, 0.95), (-0.5, 0.5, -0.7071067811865476)):
        k = np.array(k, float) / np.linalg.norm(k)
        for p in ((0.0, 0.0, 0.0), (1.0, 0.5, 0.3), (5.0, 0.0, 0.1), (0.0, 0.0, -2.0), (-0.02, 0.01, 0.0)):
            extra.append(np.r_[np.array(p) * PC, k])
    rays = np.vstack([rays, np.array(extra)])
    path_fixture("cylinder3d", ski.disk_cylinder3d(1e4), rays)
    reference_stats("paths_cylinder3d.npz", ski.disk_cylinder3d(200000), "i60", 200000)


def adaptive_fixture(rng=None):
    """AdaptiveMeshSpatialGrid of an imported AdaptiveMeshMedium (ski.adaptive_mesh_text: a 4x4x2
    root, then 2x2x2, 3x3x1 and 1x2x3 subdivisions near the disk, 5488 leaves, 8 pc box): scene export
    and path fixture (random rays, starts outside, rays along the axes and node walls through the
    centre), and reference statistics of a single-threaded 2e5-packet run."""
    rng = rng if rng is not None else np.random.default_rng(20260107)
    files = {"mesh.txt": ski.adaptive_mesh_text()}
    rays = random_rays(rng, 300, 4.0 * PC)
    extra = []
    for k in ((1, 0, 0), (0, 1, 0), (0, 0, -1), (1, 1, 0), (0.3, 0.0, 0.95), (-0.5, 0.5, -0.7071067811865476)):
        k = np.array(k, float) / np.linalg.norm(k)
        for p in ((0.0, 0.0, 0.0), (1.0, 0.5, 0.0), (0.0, 2.0, 0.5), (-3.0, -1.0, 0.25), (5.0, 0.0, 0.1)):
            extra.append(np.r_[np.array(p) * PC, k])
    rays = np.vstack([rays, np.array(extra)])
    path_fixture("adaptive", ski.disk_adaptive(1e4), rays, files=files)
    reference_stats("paths_adaptive.npz", ski.disk_adaptive(200000), "i60", 200000, files=files)


def grid_stats_fixtures():
    """The disk scene on the octree, Voronoi and tetrahedral grids of the path fixtures (4 pc box):
    scene exports plus the statistics of single-threaded 2e5-packet reference runs
    (stats_<grid>.npz), so that the life cycle on these grids is pinned against the reference's own
    runs and not only through the oracle."""
    grids = {
        "octree": ski.octree_grid(4, "pc", 6, 1e-3),
        "voronoi": ski.voronoi_grid(4, "pc", 2000),
        "tetra": ski.tetra_grid(4, "pc", 2000),
    }
    for name, grid in grids.items():
        with tempfile.TemporaryDirectory() as tmp:
            data = export(ski.disk_scene(grid, 1e4), tmp)
        path = os.path.join(OUT, f"stats_{name}.npz")
        np.savez_compressed(path, **data)
        reference_stats(f"stats_{name}.npz", ski.disk_scene(grid, 200000), "i60", 200000)
        print(f"stats_{name} written")


def run_raw(ski_text, probe=1000):
    """Exports a scene and runs its primary-emission segment in the harness (single-threaded); the
    export arrays including the raw detector sums inst<i>_wifu / inst<i>_wsed and rf1."""
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, SKGPU_EXPORT_RUN="1", SKGPU_PROBE_N=str(probe))
        ski_path = os.path.join(tmp, "scene.ski")
        with open(ski_path, "w") as f:
            f.write(ski_text)
        exp = os.path.join(tmp, "export")
        os.makedirs(exp)
        subprocess.run([os.path.join(BIN, "skirt_export"), ski_path, exp], check=True, env=env,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        data = {}
        for fn in os.listdir(exp):
            if fn.endswith(".npy"):
                data[fn[:-4]] = np.load(os.path.join(exp, fn))
        with open(os.path.join(exp, "meta.txt")) as f:
            data["meta"] = np.array(f.read())
    return data


def free_fixture(npp=200000):
    """The 16^3 shell with free (non-forced) propagation (MonteCarloSimulation::
    simulateNonForcedPropagation): raw w^0..w^2 sums of the frame and the SED of a single-threaded
    reference run."""
    data = run_raw(ski.shell_cartesian(npp, nbins=16, npix=64, force_scattering=False))
    out = dict(ref_npp=npp, ref_frame_w=data["inst0_wifu"][:3], ref_sed_w=data["inst1_wsed"][:3])
    np.savez_compressed(os.path.join(OUT, "shell_c16_free.npz"), **out)
    print("shell_c16_free written")


def galaxy_fixture(npp=500000, probe=20000):
    """The galaxy configuration at reduced size on the reference's own octree: the harness exports the
    scene, runs the primary-emission segment single-threaded and dumps the raw FP64 detector arrays
    and the radiation field MediumSystem::_rf1 (no FITS scaling to undo), and launches `probe`
    packets through SourceSystem::launch."""
    text = ski.galaxy_octree(npp, npix=32, nlambda=20, max_level=6, max_dust_fraction=1e-4, stats=True, sed=True)
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, SKGPU_EXPORT_RUN="1", SKGPU_PROBE_N=str(probe))
        ski_path = os.path.join(tmp, "galaxy.ski")
        with open(ski_path, "w") as f:
            f.write(text)
        exp = os.path.join(tmp, "export")
        os.makedirs(exp)
        subprocess.run([os.path.join(BIN, "skirt_export"), ski_path, exp], check=True, env=env,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        data = {}
        for fn in os.listdir(exp):
            if fn.endswith(".npy"):
                data[fn[:-4]] = np.load(os.path.join(exp, fn))
        with open(os.path.join(exp, "meta.txt")) as f:
            data["meta"] = np.array(f.read())
    # keep w^0..w^2 of the statistics (the z-scores need no higher moments; w^1 is the total); the
    # radiation field and the launch probe are rounded to FP32 for size (they are compared within
    # Monte Carlo noise)
    for k in list(data):
        if k.startswith("inst") and (k.endswith("_wifu") or k.endswith("_wsed")):
            data[k] = data[k][:3]
        elif k.startswith("inst") and (k.endswith("_ifu") or k.endswith("_sed")):
            del data[k]
    rf = data.pop("rf1")
    data["rf1_scale"] = rf.max()
    data["rf1_scaled"] = (rf / rf.max()).astype(np.float32)  # rf1 = rf1_scaled * rf1_scale
    data["src_probe"] = data["src_probe"].astype(np.float32)
    data["ref_npp"] = npp
    np.savez_compressed(os.path.join(OUT, "stats_galaxy.npz"), **data)
    print(f"stats_galaxy: {len(data['medium_density'])} cells, {npp} packets")


def dust_fixtures():
    """Equilibrium dust emission (DustEmission mode): the harness exports the scene, runs the primary
    segment single-threaded, exports the dust-emission tables with the reference's own per-cell dust
    luminosity, temperature and (every 97th emitting cell) emission spectrum for the radiation field of
    that run, then runs the secondary segment into cleared detectors and dumps its raw sums. Two
    scenes: the 16^3 Cartesian dust shell and the galaxy on the reference's octree at reduced size."""
    for name, text, npp in (("dust_shell", ski.dust_shell(200000), 200000),
                            ("dust_galaxy", ski.dust_galaxy(200000), 200000)):
        data = run_raw(text, probe=2000)
        for k in list(data):
            if k.startswith("inst") and ("_wifu" in k or "_wsed" in k):
                data[k] = data[k][:3]
            elif k.startswith("inst") and (k.endswith("_ifu") or k.endswith("_sed") or k.endswith("_ifu_sec")
                                           or k.endswith("_sed_sec")):
                del data[k]
        data["ref_npp"] = npp
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **data)
        print(f"{name}: {len(data['medium_density'])} cells, {npp} packets per segment")


def reference_stats(fixture, ski_text, frame_name, npp, files=None):
    """Adds the frame and SED statistics of a single-threaded reference run of ski_text to a
    fixture; the run's stats scale c is recovered from its total image (MJy/sr per raw W from the
    SED's Jy per raw W of the shell_c16 run, same distance, and this frame's pixel)."""
    path = os.path.join(OUT, fixture)
    data = dict(np.load(path))
    meta = __import__("skgpu").Scene.read_export(data)[0]
    pix = float(meta["instr0_xpsiz"]) / float(meta["instr0_distance"])
    mjysr_per_w = float(np.load(os.path.join(OUT, "shell_c16.npz"))["ref_jy_per_w"]) * 1e-6 / (pix * pix)
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "r.ski"), "w") as f:
            f.write(ski_text)
        for name, text in (files or {}).items():
            with open(os.path.join(tmp, name), "w") as f:
                f.write(text)
        subprocess.run([os.path.join(BIN, "skirt"), "-t", "1", "r.ski"], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        st = np.array([fits.read(os.path.join(tmp, f"r_{frame_name}_stats{k}.fits"))[0][0] for k in range(5)])
        ss = np.loadtxt(os.path.join(tmp, "r_sed_sedstats.dat"))
        total = fits.read(os.path.join(tmp, f"r_{frame_name}_total.fits"))[0][0]
    c = st[1].sum() / (total / mjysr_per_w).sum()
    data.update(ref_npp=npp, ref_frame_w=np.array([st[0], st[1] / c, st[2] / c ** 2]), ref_sedstats=ss[1:])
    np.savez_compressed(path, **data)


def explicit_fixture(mjysr_per_w, npp):
    """The 16^3 shell with explicit absorption (PhotonPacketOptions::explicitAbsorption), forced and
    free propagation: reference frame and SED statistics of single-threaded runs of npp packets. Each
    run scales its statistics files by its own c (from the largest sums); c is recovered per run from
    its total image as for shell_c16 (same instruments, so the same MJy/sr per raw W)."""
    out = {}
    for tag, forced in (("forced", True), ("free", False)):
        with tempfile.TemporaryDirectory() as tmp:
            with open(os.path.join(tmp, "ea.ski"), "w") as f:
                f.write(ski.shell_cartesian(npp, nbins=16, npix=64, explicit_absorption=True, force_scattering=forced))
            subprocess.run([os.path.join(BIN, "skirt"), "-t", "1", "ea.ski"], cwd=tmp, check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            st = np.array([fits.read(os.path.join(tmp, f"ea_i30_stats{k}.fits"))[0][0] for k in range(5)])
            ss = np.loadtxt(os.path.join(tmp, "ea_sed_sedstats.dat"))
            total = fits.read(os.path.join(tmp, "ea_i30_total.fits"))[0][0]
        c = st[1].sum() / (total / mjysr_per_w).sum()
        out[f"ref_{tag}_frame_w"] = np.array([st[0], st[1] / c, st[2] / c ** 2])
        out[f"ref_{tag}_sedstats"] = ss[1:]
    np.savez_compressed(os.path.join(OUT, "shell_c16_explicit.npz"), ref_npp=npp, **out)
    print("shell_c16_explicit written")


if __name__ == "__main__":
    if sys.argv[1:] == ["sphere1d"]:
        sphere1d_fixture()
    elif sys.argv[1:] == ["cylinder2d"]:
        cylinder2d_fixture()
    elif sys.argv[1:] == ["sphere2d"]:
        sphere2d_fixture()
    elif sys.argv[1:] == ["sphere3d"]:
        sphere3d_fixture()
    elif sys.argv[1:] == ["cylinder3d"]:
        cylinder3d_fixture()
    elif sys.argv[1:] == ["adaptive"]:
        adaptive_fixture()
    elif sys.argv[1:] == ["gridstats"]:
        grid_stats_fixtures()
    elif sys.argv[1:] == ["galaxy"]:
        galaxy_fixture()
    elif sys.argv[1:] == ["free"]:
        free_fixture()
    elif sys.argv[1:] == ["explicit"]:
        z = np.load(os.path.join(OUT, "shell_c16.npz"))
        meta = __import__("skgpu").Scene.read_export(z)[0]
        pix = float(meta["instr0_xpsiz"]) / float(meta["instr0_distance"])
        explicit_fixture(float(z["ref_jy_per_w"]) * 1e-6 / (pix * pix), int(z["ref_npp"]))
    else:
        main()
