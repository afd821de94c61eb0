"""Host-side scene description: the flattened state SKIRT hands to the tracer.

A `Scene` holds exactly the arrays of the C ABI (grid, medium state, dust-mix tables, sources,
instruments, options). It is filled either from the export of a reference simulation (the
`skirt_export` harness writes the SimulationItem tree's flattened arrays as .npy files) or by the
workload builders in `skgpu.workloads`. `Scene.upload` sends it through a `Backend`;
`Scene.run` performs one primary-emission segment and returns the tallies.
"""
import math
import os

import numpy as np

from . import abi


def list_bands(bands, unit=1e-6):
    """Band tables of a BandWavelengthGrid built from ListBand definitions, in the form
    Backend.set_instrument_bands takes: (wavelengths in m, normalised transmissions, effective
    width) per band, sorted by pivot wavelength. bands: (wavelengths, transmissions) pairs with
    wavelengths in units of `unit` (micron by default). Follows TabulatedBand::setupSelfBefore
    (increasing order, normalisation to unit integral, SKIRT/core/TabulatedBand.cpp) and
    Band::setupSelfAfter (pivot wavelength and effective width 1/max T, Band.cpp); the bands are
    ordered as BandWavelengthGrid::setupSelfAfter orders them."""
    out = []
    for lam, tr in bands:
        lv = np.asarray(lam, dtype=np.float64) * unit
        tv = np.asarray(tr, dtype=np.float64).copy()
        if lv[0] > lv[-1]:
            lv, tv = lv[::-1].copy(), tv[::-1].copy()
        norm = 0.0
        for i in range(1, len(lv)):
            norm += 0.5 * (tv[i - 1] + tv[i]) * (lv[i] - lv[i - 1])
        tv /= norm
        integral = 0.0
        for i in range(1, len(lv)):
            lm = 0.5 * (lv[i - 1] + lv[i])
            integral += 0.5 * (tv[i - 1] + tv[i]) * (lv[i] - lv[i - 1]) / lm / lm
        out.append((1.0 / np.sqrt(integral), lv, tv, 1.0 / tv.max()))
    out.sort(key=lambda b: b[0])
    return [(lv, tv, w) for _, lv, tv, w in out]


def calibration_factors(distance, wavelengths, widths, pixel_size=None):
    """FluxRecorder::calibrateAndWrite's factors per wavelength bin (SKIRT/core/FluxRecorder.cpp:891-921)
    for a distant instrument at redshift 0 (luminosity and angular-diameter distance both `distance`)
    with SKIRT's frequency output style: SED flux densities in Jy (Units::ofluxdensity, unit
    `frequencyfluxdensity` Jy = 1e-26), frames in MJy/sr (Units::osurfacebrightness, MJy/sr = 1e-20)
    over the pixel solid angle 4 atan(px / 2d) atan(py / 2d); pixel_size = (px, py) selects the frame
    form. wavelengths and widths are the grid's characteristic wavelengths and effective widths."""
    c = 2.99792458e8  # Constants::c()
    fourpid2 = 4.0 * math.pi * (distance * distance)
    out = []
    for lam, w in zip(wavelengths, widths):
        conv = lam * lam * 1.0 / c
        if pixel_size is None:
            out.append(1.0 / fourpid2 / w * ((conv - 0.0) / 1e-26))
        else:
            px, py = pixel_size
            omega = 4.0 * math.atan(0.5 * px / distance) * math.atan(0.5 * py / distance)
            out.append(1.0 / fourpid2 / omega / w * ((conv - 0.0) / 1e-20))
    return np.array(out)


def band_transmission(band, lam):
    """Band::transmission(lambda) (SKIRT/core/Band.cpp) of a list_bands entry."""
    lv, tv, width = band
    index = int(np.searchsorted(lv, lam, side="right"))
    if index == 0 or index >= len(lv):
        return 0.0
    t = tv[index - 1] + ((lam - lv[index - 1]) / (lv[index] - lv[index - 1])) * (tv[index] - tv[index - 1])
    return t * width


class Results:
    """Tallies of one segment, per instrument in instrument order, plus the radiation field."""

    def __init__(self):
        self.instruments = []
        self.rf = None
        self.counters = None
        self.ms = None

    def __getitem__(self, i):
        return self.instruments[i]


class Scene:
    def __init__(self):
        self.grid = None          # dict: kind + arrays in the ABI layout
        self.density = None       # (num_cells,)
        self.mix = None           # dict: lambda_borders, sigma_ext, sigma_sca, asymmpar
        self.rf = None            # dict: num_bins, borders, ellv
        self.total_luminosity = None
        self.sources = []         # list of dicts (see add_* helpers)
        self.instruments = []     # list of dicts
        self.force_scattering = True
        self.min_weight_reduction = 1e4
        self.min_scatt_events = 0
        self.path_length_bias = 0.5
        self.store_rf = False
        self.source_bias = 0.5
        self.explicit_absorption = False
        self.dust_emission = None  # dict: equilibrium-emission tables (see Backend.upload_dust_emission)
        self.secondary = None      # dict: spatial_bias, source_bias, wavelength_bias, bias_range

    # ------------------------------------------------------------------ uploads
    def upload(self, be):
        g = self.grid
        k = g["kind"]
        if k == abi.GRID_CARTESIAN:
            be.upload_grid_cartesian(g["xb"], g["yb"], g["zb"])
        elif k == abi.GRID_OCTREE:
            be.upload_grid_octree(g["bounds"], g["cell_index"], g["child_begin"], g["child_count"], g["child_index"],
                                  g["nb_begin"], g["nb_index"], g["eps"])
        elif k == abi.GRID_ADAPTIVE_MESH:
            be.upload_grid_adaptive_mesh(g["bounds"], g["cell_index"], g["child_begin"], g["child_count"],
                                         g["child_index"], g["eps"])
        elif k == abi.GRID_VORONOI:
            be.upload_grid_voronoi(g["sites"], g["nb_begin"], g["nb_index"], g["extent"], g["eps"])
            if g.get("boxes") is not None:
                be.upload_voronoi_cell_boxes(g["boxes"])
        elif k == abi.GRID_TETRA:
            be.upload_grid_tetra(g["vertices"], g["tetra"], g["normals"], g["ntetra"], g["nface"], g["extent"], g["eps"])
        elif k == abi.GRID_SPHERE1D:
            be.upload_grid_sphere1d(g["rv"])
        elif k == abi.GRID_CYLINDER2D:
            be.upload_grid_cylinder2d(g["rv"], g["zv"])
        elif k == abi.GRID_SPHERE2D:
            be.upload_grid_sphere2d(g["rv"], g["thetav"], g["cv"])
        elif k == abi.GRID_CYLINDER3D:
            be.upload_grid_cylinder3d(g["rv"], g["phiv"], g["sinv"], g["cosv"], g["zv"], g["eps"], g["has_hole"])
        elif k == abi.GRID_SPHERE3D:
            be.upload_grid_sphere3d(g["rv"], g["thetav"], g["cv"], g["phiv"], g["sinv"], g["cosv"], g["eps"])
        else:
            raise ValueError(f"unknown grid kind {k}")
        if self.density is not None:
            be.upload_medium(self.density)
        if self.mix is not None:
            m = self.mix
            be.upload_dust_mix(m["lambda_borders"], m["sigma_ext"], m["sigma_sca"], m["asymmpar"])
        if self.rf is not None:
            be.upload_rf_grid(self.rf["num_bins"], self.rf["borders"], self.rf["ellv"])
        if self.instruments:
            self._upload_instruments(be)
        if self.dust_emission is not None:
            d = self.dust_emission
            be.upload_dust_emission(d["rf_sigma_abs"], d["rf_width"], d["rf_cmb"], d["rf_sigma_abs_lum"], d["T"],
                                    d["planck_abs"], d["em_lambda"], d["em_sigma_abs"], d["em_range"],
                                    d["cell_volume"])

    def _upload_instruments(self, be):
        structs, borders, ellv = [], [], []
        for ins in self.instruments:
            s = abi.Instrument()
            s.kind = ins["kind"]
            s.same_observer = int(ins.get("same_observer", 0))
            s.record_statistics = int(ins.get("stats", 0))
            s.record_components = int(ins.get("comps", 0))
            if ins.get("bands") is not None:
                # band grid (set after the upload): no disjoint bin
                ins["num_bins"] = len(ins["bands"])
                wb, we = [0.0], [-1, -1]
            else:
                wb, we = list(ins["wlg_borders"]), list(ins["wlg_ellv"])
            s.num_wavelength_bins = int(ins["num_bins"])
            s.wlg_offset = len(ellv)
            s.wlg_num_borders = len(wb)
            borders.extend(wb + [0.0])
            ellv.extend(we)
            s.kobs[:] = list(ins["kobs"])
            if ins.get("trig") is not None:
                # frames; SED instruments with an aperture (its projection)
                (s.cos_theta, s.sin_theta, s.cos_phi, s.sin_phi, s.cos_omega, s.sin_omega) = ins["trig"]
            if s.kind == abi.INSTR_FRAME:
                s.num_pixels_x, s.num_pixels_y = int(ins["nx"]), int(ins["ny"])
                s.xp_min, s.xp_size, s.yp_min, s.yp_size = ins["xp_min"], ins["xp_size"], ins["yp_min"], ins["yp_size"]
            structs.append(s)
        be.upload_instruments(structs, np.array(borders), np.array(ellv, np.int32))
        for i, ins in enumerate(self.instruments):
            if ins.get("levels"):
                be.set_instrument_scattering_levels(i, ins["levels"])
            if ins.get("bands") is not None:
                be.set_instrument_bands(i, ins["bands"])
            if ins.get("redshift") or ins.get("aperture"):
                be.set_instrument_observer(i, ins.get("redshift", 0.0), ins.get("aperture", 0.0))

    def source_structs(self, npp):
        """ABI source records for a segment of npp packets (SourceSystem::prepareForLaunch)."""
        lv = np.array([s["lfrac"] for s in self.sources], float)
        wv = np.array([s["weight"] for s in self.sources], float)
        first = [0]
        W = 0.0
        for h in range(1, len(self.sources)):
            W += wv[h - 1]
            first.append(min(npp, int(np.floor(W * npp + 0.5))))  # std::round
        first.append(npp)
        structs, tl, ta, tb, rr, rp = [], [], [], [], [], []
        for h, src in enumerate(self.sources):
            s = abi.Source()
            s.position_model = src["position_model"]
            s.spectral_model = src["spectral_model"]
            s.position[:] = list(src.get("position", (0.0, 0.0, 0.0)))
            geo = list(src.get("geometry", ())) + [0.0] * 6
            s.geometry[:] = geo[:6]
            s.first_history = first[h]
            s.num_histories = first[h + 1] - first[h]
            s.packet_luminosity = self.total_luminosity / npp * lv[h] / wv[h]
            s.wavelength_bias = src.get("wavelength_bias", 0.0)
            s.bias_lambda_min, s.bias_lambda_max = src.get("bias_range", (0.0, 0.0))
            s.table_offset = len(tl)
            s.table_size = len(src["table_lambda"])
            tl.extend(src["table_lambda"])
            ta.extend(src["table_a"])
            tb.extend(src.get("table_b", np.zeros(len(src["table_lambda"]))))
            if s.position_model in (abi.SRC_RADIAL, abi.SRC_RADIAL_LOGLOG):
                s.radial_offset = len(rr)
                s.radial_size = len(src["radial_r"])
                rr.extend(src["radial_r"])
                rp.extend(src["radial_P"])
            structs.append(s)
        if not rr:
            rr, rp = [0.0], [0.0]
        return structs, np.array(tl), np.array(ta), np.array(tb), np.array(rr), np.array(rp)

    def options(self, seed=0, precision=abi.PREC_FP64_EXACT, peel=True):
        o = abi.Options()
        o.force_scattering = int(self.force_scattering)
        o.min_scatt_events = int(self.min_scatt_events)
        o.min_weight_reduction = float(self.min_weight_reduction)
        o.path_length_bias = float(self.path_length_bias)
        o.store_radiation_field = int(self.store_rf)
        o.peel_off = int(peel)
        o.precision = int(precision)
        o.explicit_absorption = int(self.explicit_absorption)
        o.seed = int(seed)
        return o

    # ------------------------------------------------------------------ run
    def instrument_size(self, i):
        ins = self.instruments[i]
        npix = ins["nx"] * ins["ny"] if ins["kind"] == abi.INSTR_FRAME else 1
        return npix * ins["num_bins"]

    def rf_length(self):
        """Entries of the radiation-field tally (cells x RF bins), 0 when it is not stored."""
        return len(self.density) * self.rf["num_bins"] if self.store_rf and self.rf is not None else 0

    def prepare(self, be, npp, seed=0, precision=abi.PREC_FP64_EXACT):
        be.set_options(self.options(seed, precision))
        structs, tl, ta, tb, rr, rp = self.source_structs(npp)
        be.upload_sources(structs, tl, ta, tb, rr, rp)

    def probe_launch(self, be, npp, count=None, seed=0, first=0):
        """The launch record (wavelength, L x npp, position, direction) of histories [first,
        first+count) of a segment of npp packets, without tracing them."""
        self.prepare(be, npp, seed)
        return be.probe_launch(first, npp if count is None else count, npp)

    def run(self, be, npp, seed=0, precision=abi.PREC_FP64_EXACT, first=0, count=None, clear=True):
        """One primary-emission segment of npp packets (histories [first, first+count))."""
        if clear:
            be.clear_tallies()
        self.prepare(be, npp, seed, precision)
        be.run_primary(first, npp if count is None else count, npp)
        return self.fetch(be)

    def run_secondary(self, be, npp, seed=0, precision=abi.PREC_FP64_EXACT, first=0, count=None, clear=True,
                      rf=None):
        """One secondary (dust) emission segment of npp packets (histories [first, first+count)) from
        the radiation field on the backend (the last primary segment's, or `rf`, cells x bins);
        returns the tallies (with store_rf the segment's own radiation field, as the secondary
        emission iterations store it) and the total dust luminosity."""
        if clear:
            be.clear_tallies()
        be.set_options(self.options(seed, precision))
        if rf is not None:
            be.upload_radiation_field(rf)
        s = self.secondary
        L = be.prepare_secondary(npp, s["spatial_bias"], s["source_bias"], s["wavelength_bias"], s["bias_range"])
        be.run_secondary(first, npp if count is None else count)
        return self.fetch(be, rf=self.store_rf), L

    def fetch(self, be, rf=True):
        res = Results()
        for i, ins in enumerate(self.instruments):
            n = self.instrument_size(i)
            total, stats = be.fetch_instrument(i, n, stats=bool(ins.get("stats")))
            d = {"total": total, "stats": stats}
            if ins.get("comps"):
                d["components"] = be.fetch_instrument_components(i, n)
                if ins.get("levels"):
                    d["levels"] = be.fetch_instrument_levels(i, n, ins["levels"])
            if ins["kind"] == abi.INSTR_FRAME:
                shape = (ins["num_bins"], ins["ny"], ins["nx"])
                d["total"] = total.reshape(shape)
                if stats is not None:
                    d["stats"] = stats.reshape((5,) + shape)
                if "components" in d:
                    d["components"] = d["components"].reshape((3,) + shape)
                if "levels" in d:
                    d["levels"] = d["levels"].reshape((ins["levels"],) + shape)
            res.instruments.append(d)
        if self.store_rf and rf:
            res.rf = be.fetch_radiation_field(len(self.density) * self.rf["num_bins"]).reshape(len(self.density), -1)
        res.counters = be.counters()
        res.ms = be.last_run_ms()
        return res

    # ------------------------------------------------------------------ export loader
    @staticmethod
    def read_export(d):
        """(meta dict, array loader) for an export directory or a mapping (e.g. an .npz) holding the
        same arrays under their file stems plus the meta text under 'meta'."""
        if isinstance(d, str):
            with open(os.path.join(d, "meta.txt")) as f:
                text = f.read()
            load = lambda name: np.load(os.path.join(d, name + ".npy"))
            has = lambda name: os.path.exists(os.path.join(d, name + ".npy"))
        else:
            text = str(d["meta"])
            load = lambda name: np.asarray(d[name])
            has = lambda name: name in d
        meta = {}
        for line in text.splitlines():
            k, _, v = line.strip().partition(" ")
            if k:
                meta[k] = v
        return meta, load, has

    @staticmethod
    def _panchromatic_source(meta, L, h, position=None):
        """A point or geometric source with a black-body SED (panchromatic mode) from the reference's own
        launch tables: the SED's (lambda, p, P) table for Random::cdfLogLog, the wavelength bias and its
        log-uniform range, and the point's position (from the launch probe), the exponential-disk
        parameters or the Sersic cumulative-mass table."""
        p = f"source{h}_"
        if meta.get(p + "type") not in ("GeometricSource", "PointSource") or meta.get(p + "sed") != "blackbody":
            raise ValueError("export loader supports point and geometric sources with black-body SEDs in "
                             "panchromatic mode")
        src = dict(spectral_model=abi.SPEC_TABLE, lfrac=float(meta[p + "lfrac"]), weight=float(meta[p + "weight"]),
                   table_lambda=L(p + "sed_lambda"), table_a=L(p + "sed_p"), table_b=L(p + "sed_P"),
                   wavelength_bias=float(meta.get(p + "xi", 0.0)))
        if src["wavelength_bias"] > 0:
            src["bias_range"] = (float(meta[p + "bias_min"]), float(meta[p + "bias_max"]))
        geo = meta.get(p + "geometry")
        if meta.get(p + "type") == "PointSource":
            src.update(position_model=abi.SRC_POINT, position=tuple(position))
        elif geo == "expdisk":
            src.update(position_model=abi.SRC_EXPDISK,
                       geometry=tuple(float(meta[p + k]) for k in ("hR", "hz", "Rmin", "Rmax", "zmax")))
        elif geo == "sersic":
            src.update(position_model=abi.SRC_RADIAL_LOGLOG, geometry=(float(meta[p + "reff"]),),
                       radial_r=L(p + "sersic_s"), radial_P=L(p + "sersic_M"))
        else:
            raise ValueError(f"export loader: unsupported source geometry {geo}")
        return src

    @classmethod
    def from_export(cls, d):
        """Scene from the arrays the reference export harness wrote (directory or mapping)."""
        meta, L, has = cls.read_export(d)
        sc = cls()
        kind = meta["grid"]
        ext = L("grid_extent")
        if kind == "cartesian":
            sc.grid = dict(kind=abi.GRID_CARTESIAN, xb=L("grid_xb"), yb=L("grid_yb"), zb=L("grid_zb"), extent=ext)
        elif kind == "octree":
            sc.grid = dict(kind=abi.GRID_OCTREE, bounds=L("tree_bounds"), cell_index=L("tree_cell_index"),
                           child_begin=L("tree_child_begin"), child_count=L("tree_child_count"),
                           child_index=L("tree_child_index"), nb_begin=L("tree_nb_begin"),
                           nb_index=L("tree_nb_index"), eps=float(meta["eps"]), extent=ext)
        elif kind == "adaptive":
            sc.grid = dict(kind=abi.GRID_ADAPTIVE_MESH, bounds=L("am_bounds"), cell_index=L("am_cell_index"),
                           child_begin=L("am_child_begin"), child_count=L("am_child_count"),
                           child_index=L("am_child_index"), eps=float(meta["eps"]), extent=ext)
        elif kind == "voronoi":
            sc.grid = dict(kind=abi.GRID_VORONOI, sites=L("vor_sites"), nb_begin=L("vor_nb_begin"),
                           nb_index=L("vor_nb_index"), extent=ext, eps=float(meta["eps"]))
        elif kind == "tetra":
            sc.grid = dict(kind=abi.GRID_TETRA, vertices=L("tet_vertices"), tetra=L("tet_tetra"),
                           normals=L("tet_normals"), ntetra=L("tet_ntetra"), nface=L("tet_nface"), extent=ext,
                           eps=float(meta["eps"]))
        elif kind == "sphere1d":
            sc.grid = dict(kind=abi.GRID_SPHERE1D, rv=L("grid_rv"), extent=ext)
        elif kind == "cylinder2d":
            sc.grid = dict(kind=abi.GRID_CYLINDER2D, rv=L("grid_rv"), zv=L("grid_zv"), extent=ext)
        elif kind == "cylinder3d":
            sc.grid = dict(kind=abi.GRID_CYLINDER3D, rv=L("grid_rv"), phiv=L("grid_phiv"), sinv=L("grid_sinv"),
                           cosv=L("grid_cosv"), zv=L("grid_zv"), eps=float(meta["eps"]),
                           has_hole=int(float(meta["has_hole"])), extent=ext)
        elif kind == "sphere3d":
            sc.grid = dict(kind=abi.GRID_SPHERE3D, rv=L("grid_rv"), thetav=L("grid_thetav"), cv=L("grid_cv"),
                           phiv=L("grid_phiv"), sinv=L("grid_sinv"), cosv=L("grid_cosv"), eps=float(meta["eps"]),
                           extent=ext)
        elif kind == "sphere2d":
            sc.grid = dict(kind=abi.GRID_SPHERE2D, rv=L("grid_rv"), thetav=L("grid_thetav"), cv=L("grid_cv"),
                           extent=ext)
        else:
            raise ValueError(f"unsupported grid in export: {kind}")
        sc.density = L("medium_density")[:, 0].copy()
        sc.mix = dict(lambda_borders=L("mix0_lambda_borders"), sigma_ext=L("mix0_sigma_ext"),
                      sigma_sca=L("mix0_sigma_sca"), asymmpar=L("mix0_asymmpar"))
        sc.force_scattering = bool(int(meta["force_scattering"]))
        sc.min_weight_reduction = float(meta["min_weight_reduction"])
        sc.min_scatt_events = int(float(meta["min_scatt_events"]))
        sc.path_length_bias = float(meta["path_length_bias"])
        if has("rf_wlg_borders"):
            ellv = L("rf_wlg_ellv")
            sc.rf = dict(num_bins=int(ellv.max()) + 1, borders=L("rf_wlg_borders"), ellv=ellv)
        if has("de_T"):
            # equilibrium dust emission (DustEmission mode): the reference's own tables and options
            sc.dust_emission = {k: L("de_" + k) for k in ("rf_sigma_abs", "rf_width", "rf_cmb", "rf_sigma_abs_lum",
                                                           "T", "planck_abs", "em_lambda", "em_sigma_abs",
                                                           "em_range")}
            sc.dust_emission["cell_volume"] = L("cell_volume")
            sc.secondary = dict(spatial_bias=float(meta["secondary_spatial_bias"]),
                                source_bias=float(meta["secondary_source_bias"]),
                                wavelength_bias=float(meta["dust_emission_wavelength_bias"]),
                                bias_range=(float(meta.get("dust_emission_bias_min", 0.0)),
                                            float(meta.get("dust_emission_bias_max", 0.0))))
            sc.store_rf = True
        sc.total_luminosity = float(meta["source_total_luminosity"])
        probe = L("src_probe")
        nsrc = int(meta["num_sources"])
        if meta["oligochromatic"] == "1":
            # oligochromatic point source: the launch probe gives lambda and L*npp of the reference's
            # own launches (one weight per wavelength)
            if nsrc != 1 or meta["source0_type"] != "PointSource":
                raise ValueError("export loader supports a single point source in oligochromatic mode")
            lams = np.unique(probe[:, 0])
            weights = np.array([probe[probe[:, 0] == l, 1][0] for l in lams]) / sc.total_luminosity
            sc.sources = [dict(position_model=abi.SRC_POINT, spectral_model=abi.SPEC_DISCRETE,
                               position=tuple(probe[0, 2:5]), lfrac=float(meta["source0_lfrac"]),
                               weight=float(meta["source0_weight"]), table_lambda=lams, table_a=weights)]
        else:
            sc.sources = [cls._panchromatic_source(meta, L, h, probe[0, 2:5]) for h in range(nsrc)]
        for i in range(int(meta["num_instruments"])):
            p = f"instr{i}_"
            ellv = L(p + "wlg_ellv")
            ins = dict(kind=abi.INSTR_FRAME if meta[p + "kind"] == "frame" else abi.INSTR_SED,
                       same_observer=int(meta[p + "same_observer"]), stats=int(meta[p + "record_statistics"]),
                       num_bins=int(ellv.max()) + 1, wlg_borders=L(p + "wlg_borders"), wlg_ellv=ellv,
                       kobs=(float(meta[p + "kobs_x"]), float(meta[p + "kobs_y"]), float(meta[p + "kobs_z"])))
            if p + "distance" in meta:
                ins["distance"] = float(meta[p + "distance"])
            if ins["kind"] == abi.INSTR_FRAME:
                ins.update(nx=int(meta[p + "nxp"]), ny=int(meta[p + "nyp"]),
                           trig=tuple(float(meta[p + k]) for k in
                                      ("costheta", "sintheta", "cosphi", "sinphi", "cosomega", "sinomega")),
                           xp_min=float(meta[p + "xpmin"]), xp_size=float(meta[p + "xpsiz"]),
                           yp_min=float(meta[p + "ypmin"]), yp_size=float(meta[p + "ypsiz"]))
            sc.instruments.append(ins)
        return sc
