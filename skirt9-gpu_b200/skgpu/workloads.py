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
