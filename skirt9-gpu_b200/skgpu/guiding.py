"""Learned path guiding on top of the C ABI: plain pilot, training, guided runs and the figure of
merit they are compared by.

The figure of merit of a run is FOM = 1 / (R_med^2 t), with R the per-pixel relative error of the
target frame estimated from its statistics moments, R = sqrt(sum w^2 / (sum w)^2 - 1/N) over the N
histories (FluxRecorder statistics), R_med its median over pixels with flux, and t the device time
of the run.
"""
import numpy as np

from . import abi


def relative_error(stats, n):
    """Per-pixel relative error from the moment planes (stats[k] = sum_h w_h^k, k = 0..4)."""
    s1, s2 = np.asarray(stats[1], float), np.asarray(stats[2], float)
    with np.errstate(divide="ignore", invalid="ignore"):
        r2 = s2 / (s1 * s1) - 1.0 / n
    return np.where(s1 > 0, np.sqrt(np.clip(r2, 0.0, None)), np.nan)


def median_relative_error(stats, n):
    r = relative_error(stats, n)
    r = r[np.isfinite(r) & (np.asarray(stats[1]) > 0)]
    return float(np.median(r)) if r.size else float("nan")


def figure_of_merit(stats, n, seconds):
    r = median_relative_error(stats, n)
    return 1.0 / (r * r * seconds)


def importance_from_image(image, floor_quantile=0.05, cap=100.0):
    """Per-pixel weights 1 / F of a plain estimate F of the target frame (so that the pilot records
    value every pixel's relative error alike), normalised to mean 1 over lit pixels and capped."""
    F = np.asarray(image, float).ravel()
    lit = F > 0
    w = np.zeros_like(F)
    if lit.any():
        floor = np.quantile(F[lit], floor_quantile)
        w[lit] = 1.0 / np.maximum(F[lit], floor)
        w /= w[lit].mean()
        w = np.minimum(w, cap)
    return w.astype(np.float32)


def run(sc, be, n, seed, precision=abi.PREC_FP32, first=0):
    """One segment; returns the results (with stats) and its device time in seconds."""
    res = sc.run(be, n, seed=seed, precision=precision, first=first)
    return res, res.ms / 1e3


def _image(res, target):
    tot = np.asarray(res.instruments[target]["total"])
    return tot.sum(axis=0) if tot.ndim == 3 else tot


def train(sc, be, pilot_packets, target=0, seed=7, record_fraction=0.25, capacity=1 << 22, steps=2000, batch=16384,
          lr=1e-3, prepilot_packets=0, init_seed=11, precision=abi.PREC_FP32, position_bins=0):
    """Plain pilot with recorded scattering events, then training of the network on the GPU.
    With prepilot_packets > 0 a plain run first estimates the target image, whose inverse weights
    the recorded detections per pixel. Returns a dict of what was done."""
    info = {}
    abi.guide_init(be, None, init_seed)
    abi.guide_set_mode(be, abi.GUIDE_OFF)
    weights = None
    if prepilot_packets:
        res, t = run(sc, be, prepilot_packets, seed + 1, precision)
        weights = importance_from_image(_image(res, target))
        info["prepilot_s"] = t
    abi.guide_set_mode(be, abi.GUIDE_RECORD, target, 0.0, record_fraction, capacity)
    abi.guide_set_importance(be, weights)
    try:
        res, t = run(sc, be, pilot_packets, seed, precision)
    finally:
        abi.guide_set_mode(be, abi.GUIDE_OFF)
    info["pilot_s"] = t
    info["pilot"] = res
    rec = abi.guide_records(be)
    info["records"] = len(rec)
    info["records_with_signal"] = int((rec[:, 11] > 0).sum()) if len(rec) else 0
    abi.guide_set_training(be, position_bins)
    info["loss_final"] = abi.guide_train(be, steps, batch, lr, seed + 2)
    return info


def run_guided(sc, be, n, seed, alpha=0.5, target=0, precision=abi.PREC_FP32):
    abi.guide_set_mode(be, abi.GUIDE_SAMPLE, target, alpha)
    try:
        return run(sc, be, n, seed, precision)
    finally:
        abi.guide_set_mode(be, abi.GUIDE_OFF)
