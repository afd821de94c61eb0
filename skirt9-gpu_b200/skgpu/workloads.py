"""Builders of the named workloads as `Scene`s, without the reference code.

The reference builds these scenes itself (grid construction, density sampling, source and
instrument setup); these builders produce statistically equivalent scenes for standalone runs of
the tracer with seeded synthetic inputs of the same shapes and sizes:

  shell_cartesian   dust shell r^-2 between 0.1 and 1 pc (radial tau_V = 1) on a Cartesian grid of
                    +-1 pc, central point source, 0.55 micron, HG g = 0.6, albedo 0.5, one frame at
                    30 degrees plus an SED instrument sharing its observer
"""
import numpy as np

from . import abi
from .scene import Scene

PC = 3.08567758e16          # m (SKIRT Constants::pc)
MPC = 1e6 * PC
LAMBDA_V = 0.55e-6          # m


def _frame(inclination, azimuth, roll, fov, npix, distance, num_bins, borders, ellv, stats, center=(0.0, 0.0)):
    th, ph, om = np.radians(inclination), np.radians(azimuth), np.radians(roll)
    kobs = (np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th))
    return dict(kind=abi.INSTR_FRAME, same_observer=0, stats=int(stats), num_bins=num_bins, wlg_borders=borders,
                wlg_ellv=ellv, kobs=kobs, nx=npix, ny=npix,
                trig=(np.cos(th), np.sin(th), np.cos(ph), np.sin(ph), np.cos(om), np.sin(om)),
                xp_min=center[0] - 0.5 * fov, xp_size=fov / npix, yp_min=center[1] - 0.5 * fov, yp_size=fov / npix,
                distance=distance)


def _cell_average(density, xb, yb, zb, samples=4, chunk=8):
    """Mean of density(x,y,z) over each Cartesian cell from samples^3 stratified points per cell."""
    nx, ny, nz = len(xb) - 1, len(yb) - 1, len(zb) - 1
    f = (np.arange(samples) + 0.5) / samples
    out = np.zeros((nx, ny, nz))
    yc = (yb[:-1, None] + np.diff(yb)[:, None] * f[None, :])            # (ny, s)
    zc = (zb[:-1, None] + np.diff(zb)[:, None] * f[None, :])            # (nz, s)
    for i0 in range(0, nx, chunk):
        i1 = min(nx, i0 + chunk)
        xc = xb[i0:i1, None] + np.diff(xb)[i0:i1, None] * f[None, :]   # (cx, s)
        X = xc[:, None, None, :, None, None]
        Y = yc[None, :, None, None, :, None]
        Z = zc[None, None, :, None, None, :]
        out[i0:i1] = density(X, Y, Z).mean(axis=(3, 4, 5))
    return out


KPC = 1e3 * PC
LSUN = 3.828e26  # W


def log_wavelength_grid(lmin, lmax, n):
    """LogWavelengthGrid: characteristic wavelengths, border list and bin map of
    DisjointWavelengthGrid::setWavelengthRange (DisjointWavelengthGrid.cpp:22-84)."""
    lam = np.exp(np.linspace(np.log(lmin), np.log(lmax), n))
    borders = np.empty(n + 1)
    borders[0] = np.sqrt(lam[0] ** 3 / lam[1])
    borders[1:n] = np.sqrt(lam[:-1] * lam[1:])
    borders[n] = np.sqrt(lam[-1] ** 3 / lam[-2])
    ellv = np.r_[-1, np.arange(n), -1].astype(np.int32)
    return lam, borders, ellv


def planck_table(T, lmin, lmax, n=400):
    """Normalised black-body pdf on a log grid with its cumulative distribution for log-log
    sampling (Random::cdfLogLog): piecewise power laws between the grid points."""
    h, c, k = 6.62607015e-34, 2.99792458e8, 1.380649e-23
    lam = np.exp(np.linspace(np.log(lmin), np.log(lmax), n))
    p = 1.0 / (lam ** 5 * np.expm1(h * c / (lam * k * T)))
    alpha = np.log(p[1:] / p[:-1]) / np.log(lam[1:] / lam[:-1])
    q = 1.0 + alpha
    t = lam[1:] / lam[:-1]
    seg = np.where(np.abs(q) > 1e-12, (t ** q - 1.0) / np.where(np.abs(q) > 1e-12, q, 1.0), np.log(t)) * p[:-1] * lam[:-1]
    P = np.r_[0.0, np.cumsum(seg)]
    return lam, p / P[-1], P / P[-1]


def sersic_radial_cdf(reff, n, num=600):
    """Cumulative mass of the deprojected Sersic profile (Abel inversion of the surface density
    exp(-b_n ((R/Re)^(1/n) - 1))), on a log radius grid: the radius distribution of SersicGeometry."""
    b = 2.0 * n - 1.0 / 3.0 + 0.009876 / n
    r = np.exp(np.linspace(np.log(1e-5), np.log(200.0), num))   # in units of Re
    u = np.linspace(0.0, 12.0, 3000)                              # R = r cosh(u)
    ch = np.cosh(u)
    R = r[:, None] * ch[None, :]
    dS = -(b / n) * R ** (1.0 / n - 1.0) * np.exp(-b * (R ** (1.0 / n) - 1.0))
    rho = -np.trapezoid(dS, u, axis=1) / np.pi                   # rho(r) = -1/pi int S'(r cosh u) du
    dm = 4 * np.pi * r ** 2 * rho
    M = np.r_[0.0, np.cumsum(0.5 * (dm[1:] + dm[:-1]) * np.diff(r))]
    return np.r_[0.0, r * reff], np.r_[0.0, M / M[-1]]


def galaxy_octree(npix=512, nlambda=100, max_level=8, max_dust_fraction=1e-6, tau_v=1.0, store_rf=True,
                  seed=1, half_size_kpc=25.0, stats=False):
    """Exponential-disk galaxy on an octree: stellar disk (hR 4 kpc, hz 0.35 kpc) + Sersic n=4
    bulge (Re 1 kpc), B/T = 0.2; dust disk (hR 6 kpc, hz 0.2 kpc) with face-on tau_V; octree by
    the dust-mass-fraction policy (max level 8, fraction 1e-6: ~5e5 leaves); 100 log wavelengths
    0.1-10 micron with power-law dust properties; three 512^2 frames at 0, 60, 90 degrees; the
    radiation field stored on the same wavelength grid."""
    sc = Scene()
    h = half_size_kpc * KPC
    ext = [-h, -h, -h, h, h, h]
    hRd, hzd = 6 * KPC, 0.2 * KPC
    tree = abi.build_octree(abi.GEOM_EXPDISK, [hRd, hzd, 0, 0, 0], ext, 2, max_level, max_dust_fraction, seed=seed)
    sc.grid = dict(kind=abi.GRID_OCTREE, bounds=tree["bounds"], cell_index=tree["cell_index"],
                   child_begin=tree["child_begin"], child_count=tree["child_count"],
                   child_index=tree["child_index"], nb_begin=tree["nb_begin"], nb_index=tree["nb_index"],
                   eps=1e-12 * np.sqrt(3) * 2 * h, extent=np.array(ext))
    # dust: power-law properties on the instrument wavelengths; kappa_V = 1 m2/kg
    lam, borders, ellv = log_wavelength_grid(0.1e-6, 10e-6, nlambda)
    kappa = (lam / LAMBDA_V) ** -1.0
    albedo = np.clip(0.5 * (lam / LAMBDA_V) ** -0.2, 0.05, 0.9)
    g = np.clip(0.6 * (lam / LAMBDA_V) ** -0.3, 0.0, 0.9)
    mixb = np.r_[lam[0], np.sqrt(lam[1:] * lam[:-1])]  # DustMix wavelength-index borders (DustMix.cpp:92-97)
    sc.mix = dict(lambda_borders=mixb, sigma_ext=kappa, sigma_sca=albedo * kappa, asymmpar=g)
    # normalisation: face-on optical depth through the centre = tau_V (column 1/(2 pi hR^2) per unit mass)
    mass = tau_v / (1.0 * 1.0 / (2 * np.pi * hRd ** 2))
    sc.density = mass * tree["density"]
    # sources: disk 80 %, bulge 20 %; black bodies; wavelength bias 0.5 with a log-uniform bias
    sc.total_luminosity = 1e10 * LSUN
    xi_src = 0.5
    lf = np.array([0.8, 0.2])
    wv = (1 - xi_src) * lf + xi_src * 0.5
    ld, pd, Pd = planck_table(6000.0, 0.1e-6, 10e-6)
    lb, pb, Pb = planck_table(4000.0, 0.1e-6, 10e-6)
    rr, rP = sersic_radial_cdf(1.0 * KPC, 4.0)
    common = dict(spectral_model=abi.SPEC_TABLE, wavelength_bias=0.5, bias_range=(0.1e-6, 10e-6))
    sc.sources = [
        dict(position_model=abi.SRC_EXPDISK, geometry=(4 * KPC, 0.35 * KPC, 0, 0, 0), lfrac=lf[0], weight=wv[0],
             table_lambda=ld, table_a=pd, table_b=Pd, **common),
        dict(position_model=abi.SRC_RADIAL, lfrac=lf[1], weight=wv[1], table_lambda=lb, table_a=pb, table_b=Pb,
             radial_r=rr, radial_P=rP, **common),
    ]
    sc.instruments = [_frame(inc, 0, 0, 2 * h, npix, 10 * MPC, nlambda, borders, ellv, stats) for inc in (0, 60, 90)]
    sc.rf = dict(num_bins=nlambda, borders=borders, ellv=ellv)
    sc.store_rf = store_rf
    return sc


def shell_cartesian(nbins=64, npix=256, stats=True, luminosity=5.43959963e23):
    sc = Scene()
    b = np.linspace(-PC, PC, nbins + 1)
    sc.grid = dict(kind=abi.GRID_CARTESIAN, xb=b, yb=b.copy(), zb=b.copy(),
                   extent=np.array([-PC, -PC, -PC, PC, PC, PC]))
    rmin, rmax, kappa, tau_x = 0.1 * PC, 1.0 * PC, 1.0, 2.0
    A = tau_x / (kappa * 2 * (1 / rmin - 1 / rmax))         # rho = A r^-2, column along X = tau_x / kappa

    def rho(x, y, z):
        r2 = x * x + y * y + z * z
        return np.where((r2 >= rmin * rmin) & (r2 <= rmax * rmax), A / np.maximum(r2, 1e-300), 0.0)

    # k + nz*j + nz*ny*i ordering (CartesianSpatialGrid::index)
    sc.density = _cell_average(rho, b, b, b).reshape(-1)
    # two table entries bracketing 0.55 micron: kappa = 1 m2/kg, albedo 0.5, g = 0.6
    sc.mix = dict(lambda_borders=np.array([0.3e-6, 0.9e-6]), sigma_ext=np.array([kappa, kappa]),
                  sigma_sca=np.array([0.5 * kappa, 0.5 * kappa]), asymmpar=np.array([0.6, 0.6]))
    sc.total_luminosity = luminosity
    sc.sources = [dict(position_model=abi.SRC_POINT, spectral_model=abi.SPEC_DISCRETE, position=(0.0, 0.0, 0.0),
                       lfrac=1.0, weight=1.0, table_lambda=np.array([LAMBDA_V]), table_a=np.array([1.0]))]
    borders = np.array([LAMBDA_V * 0.999, LAMBDA_V * 1.001])
    ellv = np.array([-1, 0, -1], np.int32)
    frame = _frame(30, 0, 0, 2 * PC, npix, 10 * MPC, 1, borders, ellv, stats)
    sed = dict(kind=abi.INSTR_SED, same_observer=1, stats=int(stats), num_bins=1, wlg_borders=borders,
               wlg_ellv=ellv, kobs=frame["kobs"])
    sc.instruments = [frame, sed]
    return sc


def guided_disk(npix=512, max_level=9, max_dust_fraction=2.5e-6, tau_v=50.0, seed=1, half_size_kpc=25.0,
                stats=True, store_rf=True):
    """Hard case of the learned path guiding: the stellar disk + bulge of `galaxy_octree` inside a
    dust exponential disk (hR 6 kpc, hz 0.2 kpc) with face-on tau_V = 50, oligochromatic at 0.55
    micron (kappa 1 m2/kg, albedo 0.6, g = 0.6), on an octree of about 1e6 leaves (max level 9, dust
    fraction 2.5e-6), seen edge-on by one 512^2 frame with statistics; the radiation field is
    stored on one bin."""
    sc = Scene()
    h = half_size_kpc * KPC
    ext = [-h, -h, -h, h, h, h]
    hRd, hzd = 6 * KPC, 0.2 * KPC
    tree = abi.build_octree(abi.GEOM_EXPDISK, [hRd, hzd, 0, 0, 0], ext, 2, max_level, max_dust_fraction, seed=seed)
    sc.grid = dict(kind=abi.GRID_OCTREE, bounds=tree["bounds"], cell_index=tree["cell_index"],
                   child_begin=tree["child_begin"], child_count=tree["child_count"],
                   child_index=tree["child_index"], nb_begin=tree["nb_begin"], nb_index=tree["nb_index"],
                   eps=1e-12 * np.sqrt(3) * 2 * h, extent=np.array(ext))
    kappa = 1.0
    sc.mix = dict(lambda_borders=np.array([0.3e-6, 0.9e-6]), sigma_ext=np.array([kappa, kappa]),
                  sigma_sca=np.array([0.6 * kappa, 0.6 * kappa]), asymmpar=np.array([0.6, 0.6]))
    mass = tau_v / (kappa / (2 * np.pi * hRd ** 2))
    sc.density = mass * tree["density"]
    sc.total_luminosity = 1e10 * LSUN
    lf = np.array([0.8, 0.2])
    rr, rP = sersic_radial_cdf(1.0 * KPC, 4.0)
    oligo = dict(spectral_model=abi.SPEC_DISCRETE, table_lambda=np.array([LAMBDA_V]), table_a=np.array([1.0]))
    sc.sources = [
        dict(position_model=abi.SRC_EXPDISK, geometry=(4 * KPC, 0.35 * KPC, 0, 0, 0), lfrac=lf[0], weight=lf[0], **oligo),
        dict(position_model=abi.SRC_RADIAL, lfrac=lf[1], weight=lf[1], radial_r=rr, radial_P=rP, **oligo),
    ]
    borders = np.array([LAMBDA_V * 0.999, LAMBDA_V * 1.001])
    ellv = np.array([-1, 0, -1], np.int32)
    sc.instruments = [_frame(90, 0, 0, 2 * h, npix, 10 * MPC, 1, borders, ellv, stats)]
    sc.rf = dict(num_bins=1, borders=borders, ellv=ellv)
    sc.store_rf = store_rf
    return sc


def disk_sites(n, hR, hz, half, seed=1234):
    """n sites drawn from an exponential-disk density (radius ~ Gamma(2, hR), height ~ Laplace(hz)),
    kept inside the cube of half size `half`."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3))
    while len(out) < n:
        m = 2 * (n - len(out)) + 16
        R = rng.gamma(2.0, hR, m)
        phi = rng.uniform(0.0, 2 * np.pi, m)
        z = rng.laplace(0.0, hz, m)
        p = np.stack([R * np.cos(phi), R * np.sin(phi), z], axis=1)
        p = p[np.all(np.abs(p) < half, axis=1)]
        out = np.concatenate([out, p])
    return out[:n]


def galaxy_voronoi(n_sites=1_000_000, npix=512, nlambda=100, tau_v=2.0, store_rf=True, half_size_kpc=25.0,
                   stats=False, threads=0):
    """The galaxy of `galaxy_octree` on a Voronoi mesh: 1e6 sites drawn (seed 1234) from the dust
    exponential disk (hR 6 kpc, hz 0.2 kpc), each cell with the analytic dust density at its site,
    normalised to face-on tau_V = 2; same sources and 100-point wavelength grid as the octree galaxy;
    two 512^2 frames at 0 and 90 degrees; the radiation field stored on the wavelength grid."""
    sc = galaxy_octree(npix=8, nlambda=nlambda, max_level=2, max_dust_fraction=1e-2, store_rf=store_rf,
                       half_size_kpc=half_size_kpc, stats=stats)
    h = half_size_kpc * KPC
    ext = np.array([-h, -h, -h, h, h, h])
    hRd, hzd = 6 * KPC, 0.2 * KPC
    sites = disk_sites(n_sites, hRd, hzd, h)
    begin, index = abi.build_voronoi(sites, ext, threads)
    sc.grid = dict(kind=abi.GRID_VORONOI, sites=sites, nb_begin=begin, nb_index=index, extent=ext,
                   eps=1e-12 * np.sqrt(3) * 2 * h)
    kappa_v = 1.0
    mass = tau_v / (kappa_v / (2 * np.pi * hRd ** 2))
    R = np.hypot(sites[:, 0], sites[:, 1])
    sc.density = mass * np.exp(-R / hRd - np.abs(sites[:, 2]) / hzd) / (4 * np.pi * hRd ** 2 * hzd)
    lam, borders, ellv = log_wavelength_grid(0.1e-6, 10e-6, nlambda)
    sc.instruments = [_frame(inc, 0, 0, 2 * h, npix, 10 * MPC, nlambda, borders, ellv, stats) for inc in (0, 90)]
    return sc


def tetra_points(num_vertices, seed, half_size_kpc=25.0):
    """Mesh vertices of `galaxy_tetra`: half uniform in the box, half from the dust exponential disk
    (hR 6 kpc, hz 0.2 kpc), from numpy default_rng(seed) and default_rng(seed + 1)."""
    h = half_size_kpc * KPC
    rng = np.random.default_rng(seed)
    nu = num_vertices // 2
    return np.concatenate([rng.uniform(-h, h, (nu, 3)), disk_sites(num_vertices - nu, 6 * KPC, 0.2 * KPC, h, seed=seed + 1)])


def galaxy_tetra(num_vertices, tau_v=1.0, seed=1, npix=256, nlambda=32, half_size_kpc=25.0, store_rf=False,
                 stats=False, threads=0):
    """The galaxy of `galaxy_octree` (sources, power-law dust on `nlambda` log wavelengths) on a
    Delaunay tetrahedral mesh of `num_vertices` points plus the box corners, half drawn uniformly in
    the box and half from the dust exponential disk (hR 6 kpc, hz 0.2 kpc), each tetrahedron with the
    analytic dust density at its centroid, normalised to face-on tau_V; one frame at 60 degrees."""
    sc = galaxy_octree(npix=8, nlambda=nlambda, max_level=2, max_dust_fraction=1e-2, store_rf=store_rf,
                       half_size_kpc=half_size_kpc, stats=stats)
    h = half_size_kpc * KPC
    ext = np.array([-h, -h, -h, h, h, h])
    hRd, hzd = 6 * KPC, 0.2 * KPC
    pts = tetra_points(num_vertices, seed, half_size_kpc)
    t = abi.build_tetra(pts, ext, threads)
    sc.grid = dict(kind=abi.GRID_TETRA, vertices=t["vertices"], tetra=t["tetra"], normals=t["normals"],
                   ntetra=t["ntetra"], nface=t["nface"], extent=ext, eps=1e-12 * np.sqrt(3) * 2 * h)
    c = t["vertices"][t["tetra"]].mean(axis=1)
    mass = tau_v / (1.0 / (2 * np.pi * hRd ** 2))
    R = np.hypot(c[:, 0], c[:, 1])
    sc.density = mass * np.exp(-R / hRd - np.abs(c[:, 2]) / hzd) / (4 * np.pi * hRd ** 2 * hzd)
    lam, borders, ellv = log_wavelength_grid(0.1e-6, 10e-6, nlambda)
    sc.instruments = [_frame(60, 0, 0, 2 * h, npix, 10 * MPC, nlambda, borders, ellv, stats)]
    sc.vertex_points = pts
    return sc


def tetra_batch_spec(num=16, seed=2024, min_vertices=1e4, max_vertices=4e5, min_packets=1e6, max_packets=1e7):
    """Parameters of a batch of independent tetrahedral-mesh simulations, drawn with
    numpy default_rng(seed): vertex counts, face-on tau_V (0.1-10) and packet counts, each
    log-uniform; per simulation a point seed and a random-stream seed."""
    rng = np.random.default_rng(seed)
    lu = lambda lo, hi: np.exp(rng.uniform(np.log(lo), np.log(hi), num))
    nv = lu(min_vertices, max_vertices).astype(np.int64)
    tau = lu(0.1, 10.0)
    npp = lu(min_packets, max_packets).astype(np.int64)
    point_seeds = rng.integers(1, 2 ** 31, num)
    run_seeds = rng.integers(1, 2 ** 31, num)
    return [dict(num_vertices=int(nv[i]), tau_v=float(tau[i]), packets=int(npp[i]), point_seed=int(point_seeds[i]),
                 seed=int(run_seeds[i])) for i in range(num)]


def tetra_batch(num=16, seed=2024, npix=256, nlambda=32, min_vertices=1e4, max_vertices=4e5, min_packets=1e6,
                max_packets=1e7, workers=8, first=None):
    """The batched tetrahedral workload: `num` galaxies on Delaunay meshes (`galaxy_tetra`) with the
    parameters of `tetra_batch_spec` (only the first `first` of them when given), meshes built in
    parallel. Returns (scenes, spec)."""
    from concurrent.futures import ThreadPoolExecutor
    spec = tetra_batch_spec(num, seed, min_vertices, max_vertices, min_packets, max_packets)[:first]
    make = lambda s: galaxy_tetra(s["num_vertices"], s["tau_v"], s["point_seed"], npix=npix, nlambda=nlambda, threads=1)
    with ThreadPoolExecutor(max(1, workers)) as ex:
        scenes = list(ex.map(make, spec))
    return scenes, spec
