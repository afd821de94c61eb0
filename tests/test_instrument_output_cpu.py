"""Instrument outputs beyond totals and components, on the CPU oracle: scattering levels
(Instrument::numScatteringLevels, FluxRecorder.cpp:430-433) and band wavelength grids
(BandWavelengthGrid::bins and Band::transmission, FluxRecorder.cpp:380-384).

The scenes are the shell fixture (one wavelength, 0.55 micron) with a frame that records components
and scattering levels, its SED instrument, and a second SED instrument of the same observer on four
overlapping bands. Every detection of the band instrument adds L * T_b(lambda) to each band holding
lambda, so the band SED equals T_b(0.55 micron) times the disjoint SED to rounding; the scattering
levels split the scattered plane by the number of scatterings.
"""
import numpy as np
import pytest

from skgpu import Scene, ski
from skgpu.scene import band_transmission, list_bands


def levels_bands_scene(z, levels=3):
    sc = Scene.from_export(z)
    frame, sed = sc.instruments
    frame = dict(frame, comps=1, levels=levels)
    sed = dict(sed, comps=1, levels=2)
    band = dict(sed, same_observer=1, comps=1, levels=2, bands=list_bands(ski.TEST_BANDS))
    sc.instruments = [frame, sed, band]
    return sc


def check_levels_and_bands(sc, res, levels):
    """The properties both the oracle and the CUDA library must show (see the module docstring)."""
    lam = float(sc.sources[0]["table_lambda"][0])
    frame, sed, band = res.instruments
    comps, lv = frame["components"], frame["levels"]
    assert lv.shape[0] == levels and np.all(lv >= 0) and lv[0].sum() > 0
    # levels split the scattered plane: never more than it
    assert np.all(lv.sum(axis=0) <= comps[2] * (1 + 1e-12))
    T = np.array([band_transmission(b, lam) for b in sc.instruments[2]["bands"]])
    assert (T > 0).sum() == 2  # 0.55 micron lies in two of the four bands
    ell = int(np.nonzero(sed["total"])[0][0])
    pairs = [(band["total"], sed["total"])] + [(band["components"][c], sed["components"][c]) for c in range(3)] \
        + [(band["levels"][k], sed["levels"][k]) for k in range(2)]
    for a, b in pairs:
        assert np.allclose(a, T * b[ell], rtol=1e-12, atol=0)
    assert np.all(band["levels"][:, T == 0] == 0)
    return T


def test_levels_and_bands_on_oracle(golden, oracle_backend):
    z = golden("shell_c16.npz")
    sc = levels_bands_scene(z, levels=3)
    sc.upload(oracle_backend)
    res = sc.run(oracle_backend, 4000, seed=5)
    check_levels_and_bands(sc, res, 3)
    # enough levels for every history (forced scattering, albedo 0.5, termination at 1e-4 of the
    # launch weight: at most ~14 scatterings): the levels add up to the scattered plane
    sc2 = levels_bands_scene(z, levels=60)
    sc2.upload(oracle_backend)
    res2 = sc2.run(oracle_backend, 4000, seed=5)
    f2 = res2.instruments[0]
    assert np.allclose(f2["levels"].sum(axis=0), f2["components"][2], rtol=1e-9, atol=1e-300)
    # the first levels do not depend on how many are recorded
    assert np.array_equal(f2["levels"][:3], res.instruments[0]["levels"])


def test_band_tables_follow_the_reference():
    """list_bands: normalised tables (unit integral), effective width 1/max T, pivot order."""
    bands = list_bands(ski.TEST_BANDS)
    assert len(bands) == 4
    for lv, tv, w in bands:
        integral = np.sum(0.5 * (tv[1:] + tv[:-1]) * np.diff(lv))
        assert integral == pytest.approx(1.0, rel=1e-12)
        assert w == pytest.approx(1.0 / tv.max(), rel=1e-15)
    # Band::transmission: zero at and beyond the last table point, the scaled table inside
    lv, tv, w = bands[0]
    assert band_transmission(bands[0], lv[-1]) == 0.0
    assert band_transmission(bands[0], lv[0]) == pytest.approx(tv[0] * w, rel=1e-15)
    assert band_transmission(bands[0], lv[0] * 0.5) == 0.0


def test_band_and_level_arguments_checked(golden, oracle_backend):
    from skgpu import SkgpuError
    sc = levels_bands_scene(golden("shell_c16.npz"))
    sc.upload(oracle_backend)
    with pytest.raises(SkgpuError):
        oracle_backend.set_instrument_scattering_levels(7, 2)  # no such instrument
    with pytest.raises(SkgpuError):
        oracle_backend.set_instrument_bands(1, list_bands(ski.TEST_BANDS))  # 4 bands for a 1-bin grid


def calibrated_shell(backend, golden):
    """The shell's SED through the life cycle of all its packets, calibrated by the backend: the
    transparent flux is the source luminosity over 4 pi d^2 (every packet's weight counted once), the
    same number the reference writes, so it pins the calibration against the reference's output."""
    from skgpu.scene import calibration_factors
    z = golden("shell_c16.npz")
    sc = Scene.from_export(z)
    sc.instruments[1]["comps"] = 1
    sc.upload(backend)
    npp = 4000
    raw = sc.run(backend, npp, seed=7)
    sed = sc.instruments[1]
    b = np.asarray(sed["wlg_borders"])
    f = calibration_factors(sed["distance"], [float(sc.sources[0]["table_lambda"][0])], [b[1] - b[0]])
    backend.calibrate_instrument(1, f)
    cal = sc.fetch(backend)
    return z, f, raw[1], cal[1]


def test_calibration_on_oracle_matches_the_reference(golden, oracle_backend):
    z, f, raw, cal = calibrated_shell(oracle_backend, golden)
    assert f[0] == pytest.approx(float(z["ref_jy_per_w"]), rel=1e-9)
    # calibration multiplies every plane by its bin's factor
    assert np.array_equal(cal["total"], raw["total"] * f[0])
    assert np.array_equal(cal["components"], raw["components"] * f[0])
    # the transparent flux (Jy) equals the reference's written value (10 significant digits)
    assert cal["components"][0, 0] == pytest.approx(float(z["ref_sed_jy"][1]), rel=1e-9)


def observer_scene(z, radius, redshift):
    """The shell with a second SED instrument of the same observer that has an aperture of `radius`
    (projected with the frame's inclination and azimuth, as ApertureInstrument::isInsideAperture)
    and an observer-frame redshift."""
    sc = Scene.from_export(z)
    frame, sed = sc.instruments
    sed = dict(sed, trig=frame["trig"])
    ap = dict(sed, same_observer=1, aperture=radius, redshift=redshift)
    sc.instruments = [frame, sed, ap]
    return sc


def test_observer_redshift_and_aperture_on_oracle(golden, oracle_backend):
    z = golden("shell_c16.npz")
    sc = observer_scene(z, 0.3 * 3.0856775814913673e16, 5e-4)  # 0.55 micron stays in its bin
    sc.upload(oracle_backend)
    res = sc.run(oracle_backend, 4000, seed=9)
    full, ap = res.instruments[1]["total"], res.instruments[2]["total"]
    assert 0 < ap.sum() < full.sum()  # the aperture keeps the inner part of the shell
    # an aperture larger than the domain records everything
    sc2 = observer_scene(z, 1e30, 5e-4)
    sc2.upload(oracle_backend)
    res2 = sc2.run(oracle_backend, 4000, seed=9)
    assert np.array_equal(res2.instruments[2]["total"], res2.instruments[1]["total"])
    # a redshift that moves 0.55 micron out of the bin records nothing
    sc3 = observer_scene(z, 0.0, 0.01)
    sc3.upload(oracle_backend)
    res3 = sc3.run(oracle_backend, 2000, seed=9)
    assert res3.instruments[2]["total"].sum() == 0 and res3.instruments[1]["total"].sum() > 0
