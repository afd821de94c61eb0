"""ctypes binding of the C ABI in include/skgpu.h.

`Backend` wraps one shared library whose entry points follow the skgpu.h signatures, given the
function-name prefix. The product uses the CUDA library (`lib/libskgpu.so`, prefix ``skgpu_``);
the test suite also drives the CPU oracle through the same class (prefix ``or_``), so that the
GPU tracer and the oracle receive byte-identical inputs.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libskgpu.so")

# status codes
OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_TIMEOUT, ERR_DEVICE, ERR_UNSUPPORTED = range(7)
(GRID_CARTESIAN, GRID_OCTREE, GRID_VORONOI, GRID_TETRA, GRID_SPHERE1D, GRID_CYLINDER2D, GRID_SPHERE2D, GRID_SPHERE3D,
 GRID_CYLINDER3D, GRID_ADAPTIVE_MESH) = range(10)
PREC_FP64_EXACT, PREC_FP32 = 0, 1
SRC_POINT, SRC_EXPDISK, SRC_RADIAL, SRC_RADIAL_LOGLOG = 0, 1, 2, 3
SPEC_DISCRETE, SPEC_TABLE = 0, 1
INSTR_FRAME, INSTR_SED = 0, 1


class SkgpuError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"skgpu error {code}: {message}")
        self.code = code


class Source(C.Structure):
    _fields_ = [
        ("position_model", C.c_int32),
        ("spectral_model", C.c_int32),
        ("position", C.c_double * 3),
        ("geometry", C.c_double * 6),
        ("first_history", C.c_uint64),
        ("num_histories", C.c_uint64),
        ("packet_luminosity", C.c_double),
        ("wavelength_bias", C.c_double),
        ("bias_lambda_min", C.c_double),
        ("bias_lambda_max", C.c_double),
        ("table_offset", C.c_int32),
        ("table_size", C.c_int32),
        ("radial_offset", C.c_int32),
        ("radial_size", C.c_int32),
    ]


class Instrument(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("same_observer", C.c_int32),
        ("record_statistics", C.c_int32),
        ("record_components", C.c_int32),
        ("num_pixels_x", C.c_int32),
        ("num_pixels_y", C.c_int32),
        ("num_wavelength_bins", C.c_int32),
        ("wlg_offset", C.c_int32),
        ("wlg_num_borders", C.c_int32),
        ("kobs", C.c_double * 3),
        ("cos_theta", C.c_double),
        ("sin_theta", C.c_double),
        ("cos_phi", C.c_double),
        ("sin_phi", C.c_double),
        ("cos_omega", C.c_double),
        ("sin_omega", C.c_double),
        ("xp_min", C.c_double),
        ("xp_size", C.c_double),
        ("yp_min", C.c_double),
        ("yp_size", C.c_double),
    ]


class Options(C.Structure):
    _fields_ = [
        ("force_scattering", C.c_int32),
        ("min_scatt_events", C.c_int32),
        ("min_weight_reduction", C.c_double),
        ("path_length_bias", C.c_double),
        ("store_radiation_field", C.c_int32),
        ("peel_off", C.c_int32),
        ("precision", C.c_int32),
        ("explicit_absorption", C.c_int32),
        ("seed", C.c_uint64),
    ]


class Counters(C.Structure):
    _fields_ = [
        ("histories", C.c_uint64),
        ("crossings", C.c_uint64),
        ("scatterings", C.c_uint64),
        ("peel_detections", C.c_uint64),
        ("rf_stores", C.c_uint64),
        ("stats_overflows", C.c_uint64),
        ("kernel_launches", C.c_uint64),
        ("stats_spilled", C.c_uint64),
    ]


class SecondaryOptions(C.Structure):
    _fields_ = [
        ("spatial_bias", C.c_double),
        ("source_bias", C.c_double),
        ("wavelength_bias", C.c_double),
        ("bias_lambda_min", C.c_double),
        ("bias_lambda_max", C.c_double),
    ]


_P = C.c_void_p
_I = C.c_int32
_D = C.c_double
_U = C.c_uint64

# name -> argtypes (restype int unless noted); the exported C-ABI of include/skgpu.h
SIGNATURES = {
    "create": [C.c_int, C.POINTER(_P)],
    "destroy": [_P],
    "last_error": [_P],
    "upload_grid_cartesian": [_P, _P, _I, _P, _I, _P, _I],
    "upload_grid_octree": [_P, _I, _P, _P, _P, _P, _P, _I, _P, _P, _I, _D],
    "upload_grid_adaptive_mesh": [_P, _I, _P, _P, _P, _P, _P, _I, _D],
    "upload_grid_voronoi": [_P, _I, _P, _P, _P, _I, _P, _D],
    "upload_voronoi_cell_boxes": [_P, _I, _P],
    "upload_grid_tetra": [_P, _I, _P, _I, _P, _P, _P, _P, _P, _D],
    "upload_grid_sphere1d": [_P, _I, _P],
    "upload_grid_cylinder2d": [_P, _I, _P, _I, _P],
    "upload_grid_sphere2d": [_P, _I, _P, _I, _P, _P],
    "upload_grid_sphere3d": [_P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _D],
    "upload_grid_cylinder3d": [_P, _I, _P, _I, _P, _P, _P, _I, _P, _D, _I],
    "upload_medium": [_P, _I, _P],
    "upload_dust_mix": [_P, _I, _P, _P, _P, _P],
    "upload_rf_grid": [_P, _I, _I, _P, _P],
    "upload_sources": [_P, _I, _P, _I, _P, _P, _P, _I, _P, _P],
    "upload_instruments": [_P, _I, _P, _I, _P, _P],
    "set_instrument_scattering_levels": [_P, _I, _I],
    "set_instrument_bands": [_P, _I, _I, _P, _P, _P, _P],
    "set_instrument_observer": [_P, _I, _D, _D],
    "set_options": [_P, _P],
    "run_primary": [_P, _U, _U, _U],
    "probe_launch": [_P, _U, _U, _U, _P],
    "fetch_instrument": [_P, _I, _P, _P, _P, _P],
    "fetch_instrument_components": [_P, _I, _P, _P],
    "fetch_instrument_levels": [_P, _I, _P, _P],
    "calibrate_instrument": [_P, _I, _P],
    "fetch_radiation_field": [_P, _P],
    "clear_tallies": [_P],
    "get_counters": [_P, _P],
    "last_run_ms": [_P, _P],
    "trace_paths": [_P, _I, _P, _I, _I, _P, _P, _P],
    "optical_depths": [_P, _I, _P, _D, _I, _P],
    "upload_dust_emission": [_P, _I, _P, _P, _P, _P, _I, _P, _P, _I, _P, _P, _P, _I, _P],
    "upload_radiation_field": [_P, _P],
    "prepare_secondary": [_P, _P, _U, _P],
    "fetch_dust_emission": [_P, _P, _P, _P, _P, _P, _P],
    "run_secondary": [_P, _U, _U],
}

# symbols of include/skgpu.h (the CUDA library must export every one)
EXPORTED = ["skgpu_abi_version", "skgpu_device_count"] + ["skgpu_" + n for n in SIGNATURES]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


_LIBS = {}


def load_library(path=LIB_PATH):
    """Load the CUDA tracer library. Raises if it is missing: there is no fallback path."""
    if path not in _LIBS:
        if not os.path.exists(path):
            raise SkgpuError(ERR_STATE, f"CUDA tracer library not built: {path} (run __graft_entry__.build())")
        _LIBS[path] = C.CDLL(path)
    return _LIBS[path]


class Backend:
    """One context of a library with skgpu.h-shaped entry points."""

    def __init__(self, lib=None, prefix="skgpu_", device=0):
        self.lib = lib if lib is not None else load_library()
        self.prefix = prefix
        self.fn = {}
        for name, args in SIGNATURES.items():
            f = getattr(self.lib, prefix + name)
            f.argtypes = args
            f.restype = None if name == "destroy" else (C.c_char_p if name == "last_error" else C.c_int)
            self.fn[name] = f
        self.ctx = C.c_void_p()
        rc = self.fn["create"](device, C.byref(self.ctx))
        if rc != OK:
            msg = self.fn["last_error"](self.ctx).decode() if self.ctx else "create failed"
            self.close()
            raise SkgpuError(rc, msg)

    def close(self):
        if self.ctx:
            self.fn["destroy"](self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        rc = self.fn[name](self.ctx, *args)
        if rc != OK:
            raise SkgpuError(rc, self.fn["last_error"](self.ctx).decode())
        return rc

    # ---- typed helpers ----
    def upload_grid_cylinder3d(self, rv, phiv, sinv, cosv, zv, eps, has_hole):
        rv, pv, sv, kv, zv = f64(rv), f64(phiv), f64(sinv), f64(cosv), f64(zv)
        self.call("upload_grid_cylinder3d", len(rv), _ptr(rv), len(pv), _ptr(pv), _ptr(sv), _ptr(kv), len(zv), _ptr(zv),
                  float(eps), int(has_hole))

    def upload_grid_sphere3d(self, rv, thetav, cv, phiv, sinv, cosv, eps):
        rv, tv, cv, pv, sv, kv = f64(rv), f64(thetav), f64(cv), f64(phiv), f64(sinv), f64(cosv)
        self.call("upload_grid_sphere3d", len(rv), _ptr(rv), len(tv), _ptr(tv), _ptr(cv), len(pv), _ptr(pv), _ptr(sv),
                  _ptr(kv), float(eps))

    def upload_grid_sphere2d(self, rv, thetav, cv):
        rv, tv, cv = f64(rv), f64(thetav), f64(cv)
        self.call("upload_grid_sphere2d", len(rv), _ptr(rv), len(tv), _ptr(tv), _ptr(cv))

    def upload_grid_cylinder2d(self, rv, zv):
        rv, zv = f64(rv), f64(zv)
        self.call("upload_grid_cylinder2d", len(rv), _ptr(rv), len(zv), _ptr(zv))

    def upload_grid_sphere1d(self, rv):
        rv = f64(rv)
        self.call("upload_grid_sphere1d", len(rv), _ptr(rv))

    def upload_grid_cartesian(self, xb, yb, zb):
        xb, yb, zb = f64(xb), f64(yb), f64(zb)
        self.call("upload_grid_cartesian", _ptr(xb), len(xb), _ptr(yb), len(yb), _ptr(zb), len(zb))

    def upload_grid_octree(self, bounds, cell_index, child_begin, child_count, child_index, nb_begin, nb_index, eps):
        b, ci, cb, cc, cx, nbb, nbi = (f64(bounds), i32(cell_index), i32(child_begin), i32(child_count),
                                       i32(child_index), i32(nb_begin), i32(nb_index))
        self.call("upload_grid_octree", len(ci), _ptr(b), _ptr(ci), _ptr(cb), _ptr(cc), _ptr(cx), len(cx),
                  _ptr(nbb), _ptr(nbi), len(nbi), float(eps))

    def upload_grid_adaptive_mesh(self, bounds, cell_index, child_begin, child_count, child_index, eps):
        b, ci, cb, cc, cx = f64(bounds), i32(cell_index), i32(child_begin), i32(child_count), i32(child_index)
        self.call("upload_grid_adaptive_mesh", len(ci), _ptr(b), _ptr(ci), _ptr(cb), _ptr(cc), _ptr(cx), len(cx),
                  float(eps))

    def upload_voronoi_cell_boxes(self, boxes):
        b = f64(boxes).reshape(-1, 6)
        self.call("upload_voronoi_cell_boxes", len(b), _ptr(b))

    def upload_grid_voronoi(self, sites, nb_begin, nb_index, extent, eps):
        s, nbb, nbi, ext = f64(sites), i32(nb_begin), i32(nb_index), f64(extent)
        self.call("upload_grid_voronoi", len(nbb) - 1, _ptr(s), _ptr(nbb), _ptr(nbi), len(nbi), _ptr(ext), float(eps))

    def upload_grid_tetra(self, vertices, tetra, normals, ntetra, nface, extent, eps):
        v, t, n, nt, nf, ext = f64(vertices), i32(tetra), f64(normals), i32(ntetra), i32(nface), f64(extent)
        self.call("upload_grid_tetra", len(v) // 3 if v.ndim == 1 else v.shape[0], _ptr(v), t.size // 4, _ptr(t),
                  _ptr(n), _ptr(nt), _ptr(nf), _ptr(ext), float(eps))

    def upload_medium(self, density):
        d = f64(density).ravel()
        self.call("upload_medium", len(d), _ptr(d))

    def upload_dust_mix(self, lambda_borders, sigma_ext, sigma_sca, asymmpar):
        a, b, c, d = f64(lambda_borders), f64(sigma_ext), f64(sigma_sca), f64(asymmpar)
        self.call("upload_dust_mix", len(a), _ptr(a), _ptr(b), _ptr(c), _ptr(d))

    def upload_rf_grid(self, num_bins, borders, ellv):
        b, e = f64(borders), i32(ellv)
        self.call("upload_rf_grid", int(num_bins), len(b), _ptr(b), _ptr(e))

    def upload_sources(self, sources, table_lambda, table_a, table_b=None, radial_r=None, radial_P=None):
        arr = (Source * len(sources))(*sources)
        tl, ta = f64(table_lambda), f64(table_a)
        tb = f64(table_b) if table_b is not None else np.zeros_like(tl)
        rr = f64(radial_r) if radial_r is not None else np.zeros(1)
        rp = f64(radial_P) if radial_P is not None else np.zeros(1)
        self._keep = (arr, tl, ta, tb, rr, rp)
        self.call("upload_sources", len(sources), C.cast(arr, C.c_void_p), len(tl), _ptr(tl), _ptr(ta), _ptr(tb),
                  len(rr), _ptr(rr), _ptr(rp))

    def upload_instruments(self, instruments, wlg_borders, wlg_ellv):
        arr = (Instrument * max(1, len(instruments)))(*instruments)
        b, e = f64(wlg_borders), i32(wlg_ellv)
        self.call("upload_instruments", len(instruments), C.cast(arr, C.c_void_p), len(e), _ptr(b), _ptr(e))

    def set_instrument_scattering_levels(self, i, levels):
        self.call("set_instrument_scattering_levels", int(i), int(levels))

    def set_instrument_observer(self, i, redshift=0.0, aperture_radius=0.0):
        self.call("set_instrument_observer", int(i), float(redshift), float(aperture_radius))

    def set_instrument_bands(self, i, bands):
        """bands: list of (wavelengths, normalised transmissions, effective width), in bin order."""
        sizes = i32([len(b[0]) for b in bands])
        lam = f64(np.concatenate([np.asarray(b[0], dtype=np.float64) for b in bands]))
        tr = f64(np.concatenate([np.asarray(b[1], dtype=np.float64) for b in bands]))
        wd = f64([b[2] for b in bands])
        self.call("set_instrument_bands", int(i), len(bands), _ptr(sizes), _ptr(lam), _ptr(tr), _ptr(wd))

    def set_options(self, opt):
        self.call("set_options", C.cast(C.pointer(opt), C.c_void_p))

    def run_primary(self, first, count, total):
        self.call("run_primary", int(first), int(count), int(total))

    def probe_launch(self, first, count, total):
        """(count, 8) array: wavelength, luminosity x total, position, direction of the launched
        histories [first, first+count) of a segment of `total` packets (no traversal)."""
        out = np.zeros((int(count), 8))
        self.call("probe_launch", int(first), int(count), int(total), _ptr(out))
        return out

    @staticmethod
    def _into(out, n):
        """The caller's accumulation array (float64, contiguous, n entries) or a new zeroed one."""
        if out is None:
            return np.zeros(n)
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != n:
            raise ValueError(f"tally array must be contiguous float64 of {n} entries")
        return out

    def fetch_instrument(self, i, n, stats=False, out=None, out_stats=None):
        """Adds instrument i's tallies into `out` (and `out_stats`, 5 planes) or into new arrays."""
        total = self._into(out, n)
        st = self._into(out_stats, 5 * n) if stats else None
        self.call("fetch_instrument", i, _ptr(total), _ptr(total), _ptr(st), _ptr(st))
        return total, (st.reshape(5, n) if stats else None)

    def fetch_instrument_components(self, i, n, out=None):
        comp = self._into(out, 3 * n)
        self.call("fetch_instrument_components", i, _ptr(comp), _ptr(comp))
        return comp.reshape(3, n)

    def calibrate_instrument(self, i, factors):
        """Scales instrument i's device tallies by factors[ell] per wavelength bin (in place)."""
        f = f64(factors)
        self.call("calibrate_instrument", int(i), _ptr(f))

    def fetch_instrument_levels(self, i, n, levels, out=None):
        lv = self._into(out, levels * n)
        self.call("fetch_instrument_levels", i, _ptr(lv), _ptr(lv))
        return lv.reshape(levels, n)

    def fetch_radiation_field(self, n, out=None):
        rf = self._into(out, n)
        self.call("fetch_radiation_field", _ptr(rf))
        return rf

    def clear_tallies(self):
        self.call("clear_tallies")

    def counters(self):
        c = Counters()
        self.call("get_counters", C.cast(C.pointer(c), C.c_void_p))
        return {k: getattr(c, k) for k, _ in Counters._fields_}

    def last_run_ms(self):
        v = C.c_double()
        self.call("last_run_ms", C.cast(C.pointer(v), C.c_void_p))
        return v.value

    # ---- secondary (dust) emission ----
    def upload_dust_emission(self, rf_sigma_abs, rf_width, rf_cmb, rf_sigma_abs_lum, T, planck_abs, em_lambda,
                             em_sigma_abs, em_range, cell_volume):
        a = [f64(x) for x in (rf_sigma_abs, rf_width, rf_cmb, rf_sigma_abs_lum, T, planck_abs, em_lambda, em_sigma_abs,
                              em_range, cell_volume)]
        self.call("upload_dust_emission", len(a[0]), _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(a[3]), len(a[4]),
                  _ptr(a[4]), _ptr(a[5]), len(a[6]), _ptr(a[6]), _ptr(a[7]), _ptr(a[8]), len(a[9]), _ptr(a[9]))

    def upload_radiation_field(self, rf):
        r = f64(rf).ravel()
        self.call("upload_radiation_field", _ptr(r))

    def prepare_secondary(self, total_packets, spatial_bias=0.5, source_bias=0.5, wavelength_bias=0.5,
                          bias_range=(0.0, 0.0)):
        """Prepares a secondary-emission segment of `total_packets` packets from the radiation field
        of the context; returns the total dust luminosity."""
        o = SecondaryOptions(float(spatial_bias), float(source_bias), float(wavelength_bias), float(bias_range[0]),
                             float(bias_range[1]))
        L = C.c_double()
        self.call("prepare_secondary", C.cast(C.pointer(o), C.c_void_p), int(total_packets),
                  C.cast(C.pointer(L), C.c_void_p))
        return L.value

    def fetch_dust_emission(self, num_cells):
        """Per-cell dust luminosity and temperature, and the normalised emission spectra (axis, pdf, cdf)."""
        n = C.c_int32()
        L, T = np.zeros(num_cells), np.zeros(num_cells)
        self.call("fetch_dust_emission", _ptr(L), _ptr(T), C.cast(C.pointer(n), C.c_void_p), None, None, None)
        lam = np.zeros(n.value)
        pdf, cdf = np.zeros((num_cells, n.value)), np.zeros((num_cells, n.value))
        self.call("fetch_dust_emission", None, None, None, _ptr(lam), _ptr(pdf), _ptr(cdf))
        return L, T, lam, pdf, cdf

    def run_secondary(self, first, count):
        self.call("run_secondary", int(first), int(count))

    def trace_paths(self, rays, max_segments, precision=PREC_FP64_EXACT):
        r = f64(rays).reshape(-1, 6)
        n = len(r)
        count = np.zeros(n, np.int32)
        m = np.full((n, max_segments), -2, np.int32)
        ds = np.zeros((n, max_segments))
        self.call("trace_paths", n, _ptr(r), int(max_segments), int(precision), _ptr(count), _ptr(m), _ptr(ds))
        return count, m, ds

    def optical_depths(self, rays, lam, precision=PREC_FP64_EXACT):
        r = f64(rays).reshape(-1, 6)
        tau = np.zeros(len(r))
        self.call("optical_depths", len(r), _ptr(r), float(lam), int(precision), _ptr(tau))
        return tau


GEOM_EXPDISK, GEOM_SHELL = 0, 1


class OctreeSpec(C.Structure):
    _fields_ = [
        ("geometry", C.c_int32),
        ("min_level", C.c_int32),
        ("max_level", C.c_int32),
        ("num_subdivision_samples", C.c_int32),
        ("num_density_samples", C.c_int32),
        ("reserved", C.c_int32),
        ("params", C.c_double * 6),
        ("extent", C.c_double * 6),
        ("max_dust_fraction", C.c_double),
        ("seed", C.c_uint64),
    ]


EXPORTED += ["skgpu_octree_build", "skgpu_octree_sizes", "skgpu_octree_export", "skgpu_octree_free"]


def build_octree(geometry, params, extent, min_level, max_level, max_dust_fraction, num_subdivision_samples=100,
                 num_density_samples=100, seed=1, lib=None):
    """Octree of an analytic unit-mass dust geometry (skgpu_octree_build); returns the arrays of
    skgpu_upload_grid_octree plus the mean normalised density per cell."""
    lib = lib if lib is not None else load_library()
    spec = OctreeSpec()
    spec.geometry = geometry
    spec.min_level, spec.max_level = min_level, max_level
    spec.num_subdivision_samples, spec.num_density_samples = num_subdivision_samples, num_density_samples
    spec.params[:] = list(params) + [0.0] * (6 - len(params))
    spec.extent[:] = list(extent)
    spec.max_dust_fraction = max_dust_fraction
    spec.seed = seed
    lib.skgpu_octree_build.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    lib.skgpu_octree_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    lib.skgpu_octree_export.argtypes = [C.c_void_p] + [C.c_void_p] * 8
    lib.skgpu_octree_free.argtypes = [C.c_void_p]
    lib.skgpu_octree_free.restype = None
    tree = C.c_void_p()
    rc = lib.skgpu_octree_build(C.cast(C.pointer(spec), C.c_void_p), C.byref(tree))
    if rc != OK:
        raise SkgpuError(rc, "octree construction failed (bad specification)")
    try:
        nn, nc, nb = C.c_int32(), C.c_int32(), C.c_int64()
        lib.skgpu_octree_sizes(tree, C.byref(nn), C.byref(nc), C.byref(nb))
        nn, nc, nb = nn.value, nc.value, nb.value
        out = dict(bounds=np.zeros((nn, 6)), cell_index=np.zeros(nn, np.int32), child_begin=np.zeros(nn, np.int32),
                   child_count=np.zeros(nn, np.int32), child_index=np.zeros(max(nn, 1), np.int32),
                   nb_begin=np.zeros(6 * nn + 1, np.int32), nb_index=np.zeros(max(nb, 1), np.int32),
                   density=np.zeros(nc))
        lib.skgpu_octree_export(tree, *[_ptr(out[k]) for k in ("bounds", "cell_index", "child_begin", "child_count",
                                                             "child_index", "nb_begin", "nb_index", "density")])
    finally:
        lib.skgpu_octree_free(tree)
    nsub = int((out["child_count"] > 0).sum())
    out["child_index"] = out["child_index"][:8 * nsub]
    out["nb_index"] = out["nb_index"][:nb]
    out["extent"] = np.array(extent, float)
    return out


EXPORTED += ["skgpu_run_primary_noalloc"]


def run_primary_noalloc(be, first, count, total):
    """skgpu_run_primary_noalloc through a Backend of the CUDA library: the same segment as
    run_primary, with its scratch in the library's static device array (no allocation)."""
    f = be.lib.skgpu_run_primary_noalloc
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64]
    f.restype = C.c_int
    rc = f(be.ctx, int(first), int(count), int(total))
    if rc != OK:
        raise SkgpuError(rc, be.fn["last_error"](be.ctx).decode())


EXPORTED += ["skgpu_tally_buffers"]


def tally_buffers(be):
    """[(device pointer, length in doubles)] of the context's device tally buffers (instrument
    buffers in upload order, then the radiation field), for a collective across GPUs."""
    f = be.lib.skgpu_tally_buffers
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    n = C.c_int32()
    rc = f(be.ctx, 0, None, None, C.byref(n))
    if rc != OK:
        raise SkgpuError(rc, be.fn["last_error"](be.ctx).decode())
    ptrs = (C.c_void_p * max(1, n.value))()
    lens = (C.c_uint64 * max(1, n.value))()
    rc = f(be.ctx, n.value, ptrs, lens, C.byref(n))
    if rc != OK:
        raise SkgpuError(rc, be.fn["last_error"](be.ctx).decode())
    return [(int(ptrs[i] or 0), int(lens[i])) for i in range(n.value)]


EXPORTED += ["skgpu_set_stage_timing", "skgpu_last_stage_times"]

STAGES = ("trace", "peel", "prop1", "prop2", "free", "guide", "launch")  # SKGPU_STAGE_* order


def set_stage_timing(be, level):
    """CUDA-event timing of the stage kernels of later runs: 0 off, 1 traversal kernel, 2 all stages."""
    f = be.lib.skgpu_set_stage_timing
    f.argtypes = [C.c_void_p, C.c_int32]
    f.restype = C.c_int
    rc = f(be.ctx, int(level))
    if rc != OK:
        raise SkgpuError(rc, be.fn["last_error"](be.ctx).decode())


def last_stage_times(be):
    """{stage: (device ms summed over the last run, launches)} of the stages that were timed."""
    ms = np.zeros(len(STAGES))
    n = np.zeros(len(STAGES), np.uint64)
    f = be.lib.skgpu_last_stage_times
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    rc = f(be.ctx, _ptr(ms), _ptr(n))
    if rc != OK:
        raise SkgpuError(rc, be.fn["last_error"](be.ctx).decode())
    return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(STAGES) if n[i]}


# ---- learned path guiding ----
GUIDE_OFF, GUIDE_RECORD, GUIDE_SAMPLE = 0, 1, 2
GUIDE_NUM_INPUTS, GUIDE_NUM_OUTPUTS, GUIDE_RECORD_FLOATS = 8, 40, 13
EXPORTED += ["skgpu_guide_num_params", "skgpu_guide_init", "skgpu_guide_get_params", "skgpu_guide_set_mode",
             "skgpu_guide_set_training", "skgpu_guide_last_weights",
             "skgpu_guide_set_importance", "skgpu_guide_record_count", "skgpu_guide_fetch_records",
             "skgpu_guide_train", "skgpu_guide_loss_grad", "skgpu_guide_infer"]


def _guide_call(be, name, argtypes, *args):
    f = getattr(be.lib, "skgpu_" + name)
    f.argtypes = [C.c_void_p] + argtypes
    f.restype = C.c_int
    rc = f(be.ctx, *args)
    if rc != OK:
        raise SkgpuError(rc, be.fn["last_error"](be.ctx).decode())


def guide_num_params(be):
    f = be.lib.skgpu_guide_num_params
    f.restype = C.c_int
    return int(f())


def guide_init(be, params=None, seed=0):
    """Creates the guiding network from FP32 parameters, or a seeded random initialisation."""
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
    _guide_call(be, "guide_init", [C.c_void_p, C.c_uint64], _ptr(p), int(seed))


def guide_get_params(be):
    p = np.zeros(guide_num_params(be), np.float32)
    _guide_call(be, "guide_get_params", [C.c_void_p], _ptr(p))
    return p


def guide_set_mode(be, mode, target=0, alpha=0.5, record_fraction=1.0, record_capacity=1 << 20):
    _guide_call(be, "guide_set_mode", [C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_uint64], int(mode),
                int(target), float(alpha), float(record_fraction), int(record_capacity))


def guide_last_weights(be):
    """(guided events, mean weight factor) of the last run."""
    n, m = C.c_uint64(), C.c_double()
    _guide_call(be, "guide_last_weights", [C.c_void_p, C.c_void_p], C.cast(C.pointer(n), C.c_void_p),
                C.cast(C.pointer(m), C.c_void_p))
    return n.value, m.value


def guide_set_training(be, position_bins=0):
    """Training target: records weighted per position bin (position_bins^3) or globally (0)."""
    _guide_call(be, "guide_set_training", [C.c_int32], int(position_bins))


def guide_set_importance(be, weights=None):
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32).ravel()
    _guide_call(be, "guide_set_importance", [C.c_int32, C.c_void_p], 0 if w is None else len(w), _ptr(w))


def guide_records(be):
    """Recorded pilot events as an (n, 13) array: inputs[8], direction[3], downstream luminosity, L."""
    n = C.c_uint64()
    _guide_call(be, "guide_record_count", [C.c_void_p], C.cast(C.pointer(n), C.c_void_p))
    out = np.zeros((n.value, GUIDE_RECORD_FLOATS), np.float32)
    if n.value:
        _guide_call(be, "guide_fetch_records", [C.c_uint64, C.c_void_p], n.value, _ptr(out))
    return out


def guide_train(be, steps, batch=8192, lr=1e-3, seed=1):
    loss = C.c_float()
    _guide_call(be, "guide_train", [C.c_int32, C.c_int32, C.c_float, C.c_uint64, C.c_void_p], int(steps), int(batch),
                float(lr), int(seed), C.cast(C.pointer(loss), C.c_void_p))
    return loss.value


def guide_loss_grad(be, inputs, directions, weights):
    x = np.ascontiguousarray(inputs, dtype=np.float32)
    k = np.ascontiguousarray(directions, dtype=np.float32)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    loss = C.c_float()
    grad = np.zeros(guide_num_params(be), np.float32)
    _guide_call(be, "guide_loss_grad", [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
                len(w), _ptr(x), _ptr(k), _ptr(w), C.cast(C.pointer(loss), C.c_void_p), _ptr(grad))
    return loss.value, grad


def guide_infer(be, inputs, tensor_cores=True):
    x = np.ascontiguousarray(inputs, dtype=np.float32)
    out = np.zeros((len(x), GUIDE_NUM_OUTPUTS), np.float32)
    _guide_call(be, "guide_infer", [C.c_int32, C.c_void_p, C.c_void_p, C.c_int32], len(x), _ptr(x), _ptr(out),
                1 if tensor_cores else 0)
    return out


EXPORTED += ["skgpu_voronoi_build", "skgpu_voronoi_sizes", "skgpu_voronoi_export", "skgpu_voronoi_free"]


def build_voronoi(sites, extent, threads=0, lib=None):
    """Face neighbours of the Voronoi cells of the sites in the domain box (walls -1..-6): the CSR
    arrays (nb_begin, nb_index) that skgpu_upload_grid_voronoi takes."""
    lib = lib if lib is not None else load_library()
    s = f64(sites).reshape(-1, 3)
    e = f64(extent)
    v = C.c_void_p()
    lib.skgpu_voronoi_build.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]
    lib.skgpu_voronoi_build.restype = C.c_int
    lib.skgpu_voronoi_sizes.argtypes = [C.c_void_p, C.c_void_p]
    lib.skgpu_voronoi_export.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.skgpu_voronoi_free.argtypes = [C.c_void_p]
    lib.skgpu_voronoi_free.restype = None
    rc = lib.skgpu_voronoi_build(_ptr(s), len(s), _ptr(e), int(threads), C.byref(v))
    if rc != OK:
        raise SkgpuError(rc, "voronoi build failed")
    try:
        nb = C.c_int64()
        lib.skgpu_voronoi_sizes(v, C.cast(C.pointer(nb), C.c_void_p))
        begin = np.zeros(len(s) + 1, np.int32)
        index = np.zeros(max(nb.value, 1), np.int32)
        lib.skgpu_voronoi_export(v, _ptr(begin), _ptr(index))
    finally:
        lib.skgpu_voronoi_free(v)
    return begin, index[:nb.value]


EXPORTED += ["skgpu_tetra_build", "skgpu_tetra_sizes", "skgpu_tetra_export", "skgpu_tetra_free"]


def build_tetra(points, extent, threads=0, lib=None):
    """Delaunay tetrahedra of the points and the domain's 8 corners, as the dict of arrays
    skgpu_upload_grid_tetra takes (vertices, tetra, normals, ntetra, nface)."""
    lib = lib if lib is not None else load_library()
    p = f64(points).reshape(-1, 3)
    e = f64(extent)
    t = C.c_void_p()
    lib.skgpu_tetra_build.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]
    lib.skgpu_tetra_build.restype = C.c_int
    lib.skgpu_tetra_sizes.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.skgpu_tetra_export.argtypes = [C.c_void_p] * 6
    lib.skgpu_tetra_free.argtypes = [C.c_void_p]
    lib.skgpu_tetra_free.restype = None
    rc = lib.skgpu_tetra_build(_ptr(p), len(p), _ptr(e), int(threads), C.byref(t))
    if rc != OK:
        raise SkgpuError(rc, "tetra build failed")
    try:
        nv, nt = C.c_int32(), C.c_int32()
        lib.skgpu_tetra_sizes(t, C.cast(C.pointer(nv), C.c_void_p), C.cast(C.pointer(nt), C.c_void_p))
        out = dict(vertices=np.zeros((nv.value, 3)), tetra=np.zeros((nt.value, 4), np.int32),
                   normals=np.zeros((nt.value, 4, 3)), ntetra=np.zeros((nt.value, 4), np.int32),
                   nface=np.zeros((nt.value, 4), np.int32))
        lib.skgpu_tetra_export(t, *[_ptr(out[k]) for k in ("vertices", "tetra", "normals", "ntetra", "nface")])
    finally:
        lib.skgpu_tetra_free(t)
    return out


EXPORTED += ["skgpu_set_launch_shape", "skgpu_set_trace_refill", "skgpu_run_batch"]


def set_launch_shape(be, pool_slots=0, trace_blocks_per_sm=0, shade_blocks_per_sm=0):
    _guide_call(be, "set_launch_shape", [C.c_int32, C.c_int32, C.c_int32], int(pool_slots), int(trace_blocks_per_sm),
                int(shade_blocks_per_sm))


def set_trace_refill(be, lanes=0):
    _guide_call(be, "set_trace_refill", [C.c_int32], int(lanes))


def run_batch(backends, first, count, total):
    """skgpu_run_batch over the contexts of several Backends of the CUDA library (one simulation each)."""
    n = len(backends)
    ctxs = (C.c_void_p * n)(*[b.ctx.value for b in backends])
    arr = lambda v: (C.c_uint64 * n)(*[int(x) for x in v])
    f = backends[0].lib.skgpu_run_batch
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    rc = f(C.cast(ctxs, C.c_void_p), n, C.cast(arr(first), C.c_void_p), C.cast(arr(count), C.c_void_p),
           C.cast(arr(total), C.c_void_p))
    if rc != OK:
        raise SkgpuError(rc, backends[0].fn["last_error"](backends[0].ctx).decode())


EXPORTED += ["skgpu_set_history_order"]
ORDER_INDEX, ORDER_WAVELENGTH = 0, 1


def set_history_order(be, mode):
    _guide_call(be, "set_history_order", [C.c_int32], int(mode))
