/* skgpu.h -- C ABI of the B200 (sm_100a) photon-packet life-cycle tracer for SKIRT 9.
 *
 * The boundary is segment level: the SKIRT host (C++) flattens its grid, medium state,
 * dust-mix tables, sources and instruments once, hands them over through the upload calls
 * below, and then replaces the per-thread Parallel::call over performLifeCycle with one
 * skgpu_run_primary call per primary-emission segment. Tallies are added into the caller's
 * arrays afterwards. All pointers are plain host pointers owned by the caller; the library
 * copies what it needs into HBM during the call.
 *
 * Every function returns SKGPU_OK (0) or a positive error code; skgpu_last_error() gives the
 * message. There is no CPU fallback: a non-zero status means the caller must stop (the SKIRT
 * bridge turns it into a FatalError). Functions are not re-entrant per context.
 *
 * Reference interfaces replaced (paths relative to the SKIRT9-GPU source tree):
 *   the whole family of GpuAcceleration static bool wrappers, SKIRT/core/GpuAcceleration.hpp:30-607,
 *   and the per-chunk hook MonteCarloSimulation::performLifeCycle, SKIRT/core/MonteCarloSimulation.cpp:614-694.
 */
#ifndef SKGPU_H
#define SKGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SKGPU_ABI_VERSION 1

/* status codes */
#define SKGPU_OK 0
#define SKGPU_ERR_ARG 1       /* invalid argument or size */
#define SKGPU_ERR_CUDA 2      /* CUDA runtime error (message holds the CUDA error string) */
#define SKGPU_ERR_STATE 3     /* call made in the wrong order (e.g. run before uploads) */
#define SKGPU_ERR_TIMEOUT 4   /* a bounded device-side loop gave up (guard exceeded) */
#define SKGPU_ERR_DEVICE 5    /* device-side consistency check failed (bad index, NaN weight) */
#define SKGPU_ERR_UNSUPPORTED 6

/* grid kinds */
#define SKGPU_GRID_CARTESIAN 0
#define SKGPU_GRID_OCTREE 1
#define SKGPU_GRID_VORONOI 2
#define SKGPU_GRID_TETRA 3
#define SKGPU_GRID_SPHERE1D 4
#define SKGPU_GRID_CYLINDER2D 5
#define SKGPU_GRID_SPHERE2D 6
#define SKGPU_GRID_SPHERE3D 7
#define SKGPU_GRID_CYLINDER3D 8
#define SKGPU_GRID_ADAPTIVE_MESH 9

/* traversal precision (path kernels and life cycle) */
#define SKGPU_PREC_FP64_EXACT 0 /* FP64 with the reference generators' operation order, no FMA contraction */
#define SKGPU_PREC_FP32 1       /* FP32 traversal (positions relative to the ray origin / cell site) */

/* source position models */
#define SKGPU_SRC_POINT 0   /* PointSource: fixed position */
#define SKGPU_SRC_EXPDISK 1 /* GeometricSource + ExpDiskGeometry: params hR, hz, Rmin, Rmax, zmax */
#define SKGPU_SRC_RADIAL 2  /* GeometricSource with a spherical geometry (Sersic, Shell, ...): tabulated radial CDF */
/* GeometricSource with a spherical geometry whose radius is drawn by log-log interpolation in a
 * cumulative-mass table, as SersicGeometry::randomRadius does with SersicFunction::inverseMass
 * (SKIRT/core/SersicGeometry.cpp:41-45, SKIRT/utils/SersicFunction.cpp): radial_r holds the
 * dimensionless radii s_i, radial_P the cumulative masses M_i, geometry[0] the scale (r = scale * s) */
#define SKGPU_SRC_RADIAL_LOGLOG 3

/* source spectral models */
#define SKGPU_SPEC_DISCRETE 0 /* oligochromatic: pick one of n wavelengths uniformly, weight per wavelength */
#define SKGPU_SPEC_TABLE 1    /* panchromatic: log-log tabulated CDF + log-uniform bias distribution */

/* instrument kinds */
#define SKGPU_INSTR_FRAME 0
#define SKGPU_INSTR_SED 1

typedef struct skgpu_ctx skgpu_ctx;

/* One primary source, already normalised by the SourceSystem (SourceSystem.cpp setupSelfAfter /
 * prepareForLaunch): histories [first_history, first_history+num_histories) of the segment
 * launch from this source, each with base luminosity `packet_luminosity` (= Lpp * Lv[h]/Wv[h]). */
typedef struct skgpu_source {
    int32_t position_model;     /* SKGPU_SRC_* */
    int32_t spectral_model;     /* SKGPU_SPEC_* */
    double position[3];         /* point source position, or the centre of the geometry */
    double geometry[6];         /* EXPDISK: hR, hz, Rmin, Rmax (0 = none), zmax (0 = none) */
    uint64_t first_history;     /* _Iv[h] */
    uint64_t num_histories;     /* _Iv[h+1] - _Iv[h] */
    double packet_luminosity;   /* _Lpp * _Lv[h] / _Wv[h] */
    double wavelength_bias;     /* xi of NormalizedSource (0 for unbiased, ignored for DISCRETE) */
    double bias_lambda_min;     /* log-uniform bias distribution range (SPEC_TABLE) */
    double bias_lambda_max;
    int32_t table_offset;       /* offset into the shared table arrays (see skgpu_upload_sources) */
    int32_t table_size;         /* number of entries used by this source */
    int32_t radial_offset;      /* RADIAL: offset into the radial CDF arrays */
    int32_t radial_size;
} skgpu_source;

/* One instrument of the InstrumentSystem, in instrument order. Instruments that share the
 * observer of the preceding one (DistantInstrument::determineSameObserverAsPreceding) reuse its
 * peel-off direction and observed optical depth, as FluxRecorder::detect does. */
typedef struct skgpu_instrument {
    int32_t kind;               /* SKGPU_INSTR_* */
    int32_t same_observer;      /* 1 if same observer as the preceding instrument */
    int32_t record_statistics;  /* accumulate sum_w^k, k=0..4, per history (FluxRecorder.cpp:1355-1409) */
    int32_t record_components;  /* also record transparent / direct / scattered planes (FluxRecorder.cpp:412-440) */
    int32_t num_pixels_x;       /* FRAME only */
    int32_t num_pixels_y;
    int32_t num_wavelength_bins;/* number of instrument wavelength bins */
    int32_t wlg_offset;         /* offset into the wavelength-grid arrays (borders, ellv) */
    int32_t wlg_num_borders;    /* K border points; ellv has K+1 entries */
    double kobs[3];             /* DistantInstrument::bfkobs */
    double cos_theta, sin_theta, cos_phi, sin_phi, cos_omega, sin_omega; /* FrameInstrument setup */
    double xp_min, xp_size, yp_min, yp_size;                             /* FrameInstrument setup */
} skgpu_instrument;

/* Photon-packet options and run configuration (PhotonPacketOptions + Configuration flags). */
typedef struct skgpu_options {
    int32_t force_scattering;      /* 1: forced-scattering loop; 0: free (non-forced) propagation */
    int32_t min_scatt_events;
    double min_weight_reduction;   /* terminate when L <= L0 / reduction and nscatt >= min_scatt_events */
    double path_length_bias;       /* xi of the forced-scattering composite distribution */
    int32_t store_radiation_field; /* accumulate L*lnmean*ds per (cell, RF bin) on forced paths */
    int32_t peel_off;              /* emission and scattering peel-off towards the instruments */
    int32_t precision;             /* SKGPU_PREC_* */
    /* 1: explicit absorption (PhotonPacketOptions::explicitAbsorption): interaction points are
     * sampled on the scattering optical depth and the weight carries exp(-tau_abs) instead of the
     * albedo (MonteCarloSimulation.cpp:1492-1546, 1996-2030; MediumSystem.cpp:1881-1915, 2152-2223);
     * peel-off and radiation field still use extinction */
    int32_t explicit_absorption;
    uint64_t seed;                 /* Philox key; packets draw from counter streams keyed by history index */
} skgpu_options;

/* device counters of the last run (all per segment) */
typedef struct skgpu_counters {
    uint64_t histories;
    uint64_t crossings;        /* cell crossings over all traversals */
    uint64_t scatterings;      /* scattering events */
    uint64_t peel_detections;  /* instrument detections (per instrument) */
    uint64_t rf_stores;        /* radiation-field updates */
    uint64_t stats_overflows;  /* statistics contributions lost because the spill log was full (the run then fails) */
    uint64_t kernel_launches;
    uint64_t stats_spilled;    /* statistics contributions of histories with more distinct bins than the
                                  per-slot buffer holds, grouped exactly through the spill log after the run */
} skgpu_counters;

/* ---- context ---- */
int skgpu_create(int device, skgpu_ctx** out);
void skgpu_destroy(skgpu_ctx* ctx);
const char* skgpu_last_error(const skgpu_ctx* ctx);
int skgpu_abi_version(void);
/* Number of CUDA devices visible to this process (the bridge maps process ranks onto them, as the
 * reference's GPU layer does with SKIRTGPU_DEVICE / SKIRTGPU_USE_ALL_DEVICES, GpuAcceleration.cpp). */
int skgpu_device_count(int32_t* count);

/* ---- grids (one per context; a new upload replaces the previous grid) ---- */
/* CartesianSpatialGrid: border arrays _xv,_yv,_zv (CartesianSpatialGrid.hpp:95-97). */
int skgpu_upload_grid_cartesian(skgpu_ctx* ctx, const double* xb, int32_t nxb, const double* yb, int32_t nyb,
                                const double* zb, int32_t nzb);
/* TreeSpatialGrid (octree): per node bounds xmin,ymin,zmin,xmax,ymax,zmax; cell index (-1 for
 * non-leaf); children (8 per subdivided node, in OctTreeNode::createChildren order); per node and
 * wall (BACK,FRONT,LEFT,RIGHT,BOTTOM,TOP) the overlap-sorted neighbour lists of TreeNode
 * (TreeNode.cpp:103-112, :200-209) as CSR with nb_begin[6*num_nodes+1]. */
int skgpu_upload_grid_octree(skgpu_ctx* ctx, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                             const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                             int32_t num_child_index, const int32_t* nb_begin, const int32_t* nb_index,
                             int32_t num_nb_index, double eps);
/* AdaptiveMeshSpatialGrid: the snapshot's traversal arrays (AdaptiveMeshSpatialGrid::traversalNodeBounds,
 * traversalChildBegin, traversalChildCount, traversalChildIndex, traversalCellIndex,
 * AdaptiveMeshSnapshot.cpp:172-199; the data GpuAcceleration::setAdaptiveMeshSpatialGridPath hands to
 * its tree kernel), nodes in depth-first order from the root, children in local Morton order, and
 * the snapshot's eps (1e-12 of the domain diagonal). The library derives each node's subdivision
 * from its children's bounds and each leaf wall's neighbour by Node::addNeighbors
 * (AdaptiveMeshSnapshot.cpp:67-83); paths follow AdaptiveMeshSnapshot::MySegmentGenerator::next
 * (AdaptiveMeshSnapshot.cpp:378-449). */
int skgpu_upload_grid_adaptive_mesh(skgpu_ctx* ctx, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                                    const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                                    int32_t num_child_index, double eps);
/* VoronoiMeshSnapshot: sites (x,y,z) and neighbour CSR with wall ids -1..-6
 * (VoronoiMeshSnapshot.cpp:725-740); extent xmin..zmax; eps = 1e-12 * diagonal. */
int skgpu_upload_grid_voronoi(skgpu_ctx* ctx, int32_t num_sites, const double* sites, const int32_t* nb_begin,
                              const int32_t* nb_index, int32_t num_nb_index, const double* extent, double eps);
/* Enclosing box of every Voronoi cell (VoronoiMeshSnapshot::extent(m), VoronoiMeshSnapshot.hpp:282;
 * xmin, ymin, zmin, xmax, ymax, zmax per cell), for the secondary launch: a position is drawn in the
 * cell's box until it lies closer to the cell's site than to every neighbouring site
 * (VoronoiMeshSnapshot::generatePosition / isPointClosestTo, VoronoiMeshSnapshot.cpp:879-887,
 * 1007-1020; at most 10000 draws). Call after skgpu_upload_grid_voronoi. */
int skgpu_upload_voronoi_cell_boxes(skgpu_ctx* ctx, int32_t num_cells, const double* boxes);
/* Sphere1DSpatialGrid: the num_borders ascending radial border positions r_0 >= 0 .. r_N of its N
 * radial cells (Sphere1DSpatialGrid::radialBorderPositions, Sphere1DSpatialGrid.hpp:101); cell i is
 * the shell r_i <= r < r_{i+1} around the origin. */
int skgpu_upload_grid_sphere1d(skgpu_ctx* ctx, int32_t num_borders, const double* radial_borders);
/* Cylinder2DSpatialGrid: ascending radial borders R_0 >= 0 .. R_NR and vertical borders z_0 .. z_Nz
 * (its _Rv and _zv); cell index k + Nz * i for radial bin i and vertical bin k
 * (Cylinder2DSpatialGrid.cpp:433-437). */
int skgpu_upload_grid_cylinder2d(skgpu_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                                 int32_t num_z_borders, const double* z_borders);
/* Sphere2DSpatialGrid: ascending radial borders r_0 >= 0 .. r_Nr, polar borders theta_0 = 0 ..
 * theta_Nt = pi and their cosines as the grid holds them (its _rv, _thetav, _cv:
 * SphereSpatialGrid::initPolarGrid, SphereSpatialGrid.cpp:27-60); cell index j + Nt * i
 * (Sphere2DSpatialGrid.cpp:326-329). */
int skgpu_upload_grid_sphere2d(skgpu_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                               int32_t num_polar_borders, const double* polar_borders, const double* polar_cosines);
/* Sphere3DSpatialGrid: radial borders (with the artificial inner hole the grid adds when r_min = 0),
 * polar borders and cosines, azimuthal borders phi_0 = -pi .. phi_Nphi = pi with their sines and
 * cosines, and the grid's path step eps, all as the grid holds them (its _rv, _thetav, _cv, _phiv,
 * _sinv, _cosv, _eps: Sphere3DSpatialGrid.cpp:25-70); cell index k + (j + i * Ntheta) * Nphi. */
int skgpu_upload_grid_sphere3d(skgpu_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                               int32_t num_polar_borders, const double* polar_borders, const double* polar_cosines,
                               int32_t num_azimuth_borders, const double* azimuth_borders, const double* azimuth_sines,
                               const double* azimuth_cosines, double eps);
/* Cylinder3DSpatialGrid: radial borders (with the artificial inner hole the grid adds when
 * R_min = 0, has_hole = 0 then), azimuthal borders phi_0 = -pi .. pi with their sines and cosines,
 * vertical borders and the grid's path step eps, as the grid holds them (its _Rv, _phiv, _sinv,
 * _cosv, _zv, _eps, _hasHole: Cylinder3DSpatialGrid.cpp:20-60); cell index k + (j + i * Nphi) * Nz. */
int skgpu_upload_grid_cylinder3d(skgpu_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                                 int32_t num_azimuth_borders, const double* azimuth_borders,
                                 const double* azimuth_sines, const double* azimuth_cosines, int32_t num_z_borders,
                                 const double* z_borders, double eps, int32_t has_hole);
/* TetraMeshSpatialGrid: vertices, per tetrahedron its 4 vertex indices, and per face the outward
 * normal, the neighbouring tetrahedron (-1 on the hull) and its face index
 * (TetraMeshSpatialGrid.hpp:107-133). */
int skgpu_upload_grid_tetra(skgpu_ctx* ctx, int32_t num_vertices, const double* vertices, int32_t num_tetra,
                            const int32_t* tetra_vertices, const double* face_normals, const int32_t* face_ntetra,
                            const int32_t* face_nface, const double* extent, double eps);

/* ---- medium ---- */
/* MediumState number density per cell for a single dust medium (MediumState.hpp:251). */
int skgpu_upload_medium(skgpu_ctx* ctx, int32_t num_cells, const double* number_density);
/* DustMix tables: wavelength-index borders _lambdav (DustMix.cpp:92-97) and per entry the
 * extinction / scattering cross sections and the HG asymmetry parameter. */
int skgpu_upload_dust_mix(skgpu_ctx* ctx, int32_t num_lambda, const double* lambda_borders, const double* sigma_ext,
                          const double* sigma_sca, const double* asymmpar);
/* Radiation-field wavelength grid (DisjointWavelengthGrid borders + ellv map, as the instruments). */
int skgpu_upload_rf_grid(skgpu_ctx* ctx, int32_t num_bins, int32_t num_borders, const double* borders,
                         const int32_t* ellv);

/* ---- sources ----
 * table_lambda/table_a/table_b hold, per source at [table_offset, +table_size):
 *   SPEC_DISCRETE: wavelengths, luminosity weights w_j (= s/b), unused;
 *   SPEC_TABLE:    wavelength grid, normalised pdf p (per m), normalised cdf P.
 * radial_r/radial_P hold the radial CDFs of SKGPU_SRC_RADIAL sources. */
int skgpu_upload_sources(skgpu_ctx* ctx, int32_t num_sources, const skgpu_source* sources, int32_t table_len,
                         const double* table_lambda, const double* table_a, const double* table_b,
                         int32_t radial_len, const double* radial_r, const double* radial_P);

/* ---- instruments ---- */
int skgpu_upload_instruments(skgpu_ctx* ctx, int32_t num_instruments, const skgpu_instrument* instruments,
                             int32_t wlg_len, const double* wlg_borders, const int32_t* wlg_ellv);
/* Scattering levels of an instrument that records components (Instrument::numScatteringLevels,
 * FluxRecorder::setUserFlags, FluxRecorder.cpp:162-170): the flux of primary packets scattered
 * n = 1..levels times also goes to level plane n-1 (the PrimaryScatteredLevel arrays,
 * FluxRecorder.cpp:430-433); secondary packets record no levels. Call after skgpu_upload_instruments;
 * clears the instrument's component planes. levels 0 removes them. */
int skgpu_set_instrument_scattering_levels(skgpu_ctx* ctx, int32_t instrument, int32_t levels);
/* Band wavelength grid of an instrument (BandWavelengthGrid, BandWavelengthGrid.cpp): bin ell is band
 * ell in pivot-wavelength order; a packet of wavelength lambda is recorded in every band whose table
 * range [lambda_0, lambda_last] holds lambda, with luminosity times Band::transmission(lambda)
 * (Band.cpp: linear interpolation of the normalised transmission table times the effective width),
 * as FluxRecorder::detect loops over WavelengthGrid::bins (FluxRecorder.cpp:380-384). band_sizes[b]
 * table points of band b follow one another in lambda and transmission (the normalised
 * TabulatedBand values, increasing wavelengths); width[b] = Band::effectiveWidth().
 * num_bands must equal the instrument's num_wavelength_bins; replaces its disjoint grid. Call after
 * skgpu_upload_instruments. */
int skgpu_set_instrument_bands(skgpu_ctx* ctx, int32_t instrument, int32_t num_bands, const int32_t* band_sizes,
                               const double* lambda, const double* transmission, const double* width);
/* Observer of a distant instrument beyond the defaults (0, 0): the observer-frame redshift z, with
 * which FluxRecorder::detect looks the wavelength bin up at lambda * (1 + z) (FluxRecorder.cpp:377-384;
 * DistantInstrument::setupSelfBefore passes Configuration::redshift when the distance is zero), and
 * for an SED instrument the aperture radius R of ApertureInstrument::isInsideAperture
 * (ApertureInstrument.cpp:25-44): a packet is recorded only when its position, projected with the
 * instrument's inclination and azimuth (the skgpu_instrument cos/sin fields, which the caller fills
 * for such an SED instrument too), lies within R of the centre. Call after skgpu_upload_instruments. */
int skgpu_set_instrument_observer(skgpu_ctx* ctx, int32_t instrument, double redshift, double aperture_radius);

/* ---- run ---- */
int skgpu_set_options(skgpu_ctx* ctx, const skgpu_options* options);
/* Runs the life cycle (launch, emission peel-off, forced or free propagation, radiation-field
 * storage, scattering peel-off, HG scattering) of histories [first, first+count) of a segment
 * of total_packets packets, adding into the device tallies. */
int skgpu_run_primary(skgpu_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets);
/* Source launch only: histories [first, first+count) of a segment of total_packets packets go through
 * the launch of skgpu_run_primary (the device form of SourceSystem::launch -> NormalizedSource::launch
 * -> PointSource / GeometricSource::launchNormalized, SKIRT/core/SourceSystem.cpp,
 * NormalizedSource.cpp:73-110) and are not traced. out receives 8 doubles per history: wavelength,
 * luminosity times total_packets, position (3) and direction (3), the record the reference's launch
 * writes into a PhotonPacket. Needs the sources and options; used to test the launch distributions. */
int skgpu_probe_launch(skgpu_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets, double* out);
/* ---- secondary (dust) emission ----
 * Replaces the secondary-emission segment of MonteCarloSimulation::runSecondaryEmission
 * (SKIRT/core/MonteCarloSimulation.cpp:211-245) for equilibrium dust emission from a single dust
 * medium on a Cartesian or octree grid: DustSecondarySource (DustSecondarySource.cpp) with the
 * AllCellsLibrary, SecondarySourceSystem (SecondarySourceSystem.cpp) with the dust source alone,
 * EquilibriumDustEmissionCalculator (EquilibriumDustEmissionCalculator.cpp), and the reference's
 * GPU layer calls on this path (GpuAcceleration::dustAbsorbedLuminosities, divideValues,
 * compositeLaunchWeights, GpuAcceleration.hpp). */

/* Tables of the equilibrium dust emission of the dust mix, as EquilibriumDustEmissionCalculator::
 * precalculate builds them (EquilibriumDustEmissionCalculator.cpp:17-90), and the cell volumes:
 *   num_rf radiation-field bins: rf_sigma_abs (_rfsigmaabsvv[0]), rf_width (_rfdlambdav, also the
 *     widths of MediumSystem::meanIntensity), rf_cmb (_Bcmbv; zeros without CMB heating) and
 *     rf_sigma_abs_lum, the mix's DustMix::sectionAbs at each bin's wavelength
 *     (MediumSystem::dustLuminosity, MediumSystem.cpp:2752-2762);
 *   num_T temperatures T (_Tv) with the Planck-integrated cross sections planck_abs (_planckabsvv[0]);
 *   num_em dust-emission wavelengths em_lambda (DisjointWavelengthGrid::extlambdav of the dust-emission
 *     grid) with em_sigma_abs (_emsigmaabsvv[0]) and the grid's range em_range[2] (wavelengthRange);
 *   num_cells cell volumes (MediumState::volume). */
int skgpu_upload_dust_emission(skgpu_ctx* ctx, int32_t num_rf, const double* rf_sigma_abs, const double* rf_width,
                               const double* rf_cmb, const double* rf_sigma_abs_lum, int32_t num_T, const double* T,
                               const double* planck_abs, int32_t num_em, const double* em_lambda,
                               const double* em_sigma_abs, const double* em_range, int32_t num_cells,
                               const double* cell_volume);
/* Replaces the device radiation field (the tally of skgpu_run_primary) by rf, cells x bins in the
 * layout of skgpu_fetch_radiation_field (MediumSystem::_rf1, e.g. after the segment-end sum over
 * processes of MediumSystem::communicateRadiationField). */
int skgpu_upload_radiation_field(skgpu_ctx* ctx, const double* rf);

/* Options of the secondary launch (SecondaryEmissionOptions, DustEmissionOptions). */
typedef struct skgpu_secondary_options {
    double spatial_bias;     /* SecondaryEmissionOptions::spatialBias (uniform fraction over emitting cells) */
    double source_bias;      /* SecondaryEmissionOptions::sourceBias */
    double wavelength_bias;  /* DustEmissionOptions::wavelengthBias */
    double bias_lambda_min;  /* its LogWavelengthDistribution range */
    double bias_lambda_max;
} skgpu_secondary_options;

/* Philox key offset of the secondary segment: its histories draw from key seed ^ this value, streams
 * independent of the primary segment's for the same history indices. */
#define SKGPU_SECONDARY_KEY 0x5EC0DA4EB1A5C0DEULL

/* Prepares the secondary-emission segment of total_packets packets from the device radiation field:
 * on the device, per cell the absorbed dust luminosity (MediumSystem::dustLuminosity), the
 * equilibrium temperature (EquilibriumDustEmissionCalculator::equilibriumTemperature) and the
 * normalised emission spectrum (emissivity, NR::cdf<NR::interpolateLogLog>); on the host, the launch
 * weights and history ranges per cell (DustSecondarySource::prepareLuminosities / preparePacketMap,
 * SecondarySourceSystem::prepareForLaunch). *luminosity receives the total dust luminosity; when it
 * is 0 there is nothing to launch and skgpu_run_secondary refuses to run. The uploaded field is
 * consumed: the radiation-field tally is empty afterwards. Grids: all kinds (a Voronoi grid with its
 * cell boxes, skgpu_upload_voronoi_cell_boxes). */
int skgpu_prepare_secondary(skgpu_ctx* ctx, const skgpu_secondary_options* options, uint64_t total_packets,
                            double* luminosity);
/* Results of the last preparation: per cell the dust luminosity and temperature; *num_points the
 * points of the emission-spectrum axis, lambda that axis, pdf / cdf the normalised spectra (cells x
 * num_points). Null outputs are skipped. */
int skgpu_fetch_dust_emission(skgpu_ctx* ctx, double* luminosity, double* temperature, int32_t* num_points,
                              double* lambda, double* pdf, double* cdf);
/* Runs the life cycle of histories [first, first+count) of the prepared secondary segment
 * (MonteCarloSimulation::performLifeCycle with primary = false: the dust source's launch, emission
 * peel-off, forced or free propagation, scattering peel-off and scattering), adding into the
 * instrument tallies. With the options' store_radiation_field the segment also tallies its own
 * radiation field (SecondaryEmissionOptions::storeEmissionRadiationField, the secondary emission
 * iterations: MediumSystem::storeRadiationField(false, ...), MonteCarloSimulation.cpp:391-450), and
 * with peel_off 0 it records no detections (the iterations' performLifeCycle(.., false, false, true)). */
int skgpu_run_secondary(skgpu_ctx* ctx, uint64_t first, uint64_t count);

/* Same life cycle as skgpu_run_primary for callers that must not allocate device memory while it
 * runs: for example a host code that hands the GPU to this library between phases of its own
 * memory manager, or that cannot afford the implicit device synchronisation of cudaMalloc/cudaFree
 * in the middle of a segment. No counterpart in the reference (its GPU wrappers allocate per call).
 * The call allocates nothing: its scratch (packet pool, task queues, per-history statistics
 * buffers, control block) is a file-scope device array of SKGPU_NOALLOC_SCRATCH_BYTES that every
 * GPU loading the library holds until exit, and it launches its passes directly instead of
 * building a CUDA graph. Limits: at most SKGPU_NOALLOC_MAX_SLOTS histories in flight (larger ranges
 * stream through them, only slower) and SKGPU_NOALLOC_MAX_GROUPS observer groups; scenes beyond
 * that are rejected with SKGPU_ERR_ARG. Everything the run reads or writes besides the scratch
 * (scene, tallies, radiation-field tally) must have been set up by the upload calls, skgpu_set_options
 * and skgpu_clear_tallies beforehand. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first call before any stream
 * capture. Every call looks the address up again with the caller's device current (a lookup
 * allocates nothing once the module is loaded), so the address stays right after a device reset or
 * under another context. The histories run in index order (the wavelength-ordered launch of
 * skgpu_set_history_order needs device memory per history) with the context's launch shape. Calls
 * share the one array and the call re-initialises what must start at zero; calls that overlap on the
 * GPU (other threads, other contexts on the same device) race on it. */
#define SKGPU_NOALLOC_MAX_SLOTS 32768
#define SKGPU_NOALLOC_MAX_GROUPS 4
#define SKGPU_NOALLOC_SCRATCH_BYTES (48u * 1024u * 1024u)
int skgpu_run_primary_noalloc(skgpu_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets);
/* Launch shape of later runs (0 keeps a default): packet slots in flight (default and maximum 2^22), resident
 * traversal blocks per SM (capped by what fits) and stage-kernel blocks per SM. Set by the
 * autotuner (skgpu/batch.py autotune); no reference counterpart. */
int skgpu_set_launch_shape(skgpu_ctx* ctx, int32_t pool_slots, int32_t trace_blocks_per_sm, int32_t shade_blocks_per_sm);
/* Number of waiting lanes (1-32) at which a warp of the traversal kernel takes new tasks in later
 * runs; 0 keeps the walker's default (16 for Cartesian grids and octrees, 8 for Voronoi and
 * tetrahedral meshes). Part of the launch shape the autotuner sets; no reference counterpart. */
int skgpu_set_trace_refill(skgpu_ctx* ctx, int32_t lanes);
/* Launch order of the histories of later runs. SKGPU_ORDER_WAVELENGTH (default): histories are
 * taken up in order of their launch wavelength (a counting sort at the start of every run whose
 * range exceeds the pool; 6 bytes of device memory per history), so that the packets in flight
 * update a few wavelength slices of the tallies at a time. SKGPU_ORDER_INDEX: in index order, as
 * the reference's loop. Every history draws its own random stream either way, so the tallies are
 * the same up to the order of floating-point additions. No reference counterpart. */
#define SKGPU_ORDER_INDEX 0
#define SKGPU_ORDER_WAVELENGTH 1
int skgpu_set_history_order(skgpu_ctx* ctx, int32_t mode);
/* Batched run (no reference counterpart): the segments [first[i], first[i] + count[i]) of n
 * independent simulations, one per context (each with its own uploads and options), traced as one
 * wavefront on the first context's device and stream. The contexts must share the device, grid kind
 * and traversal precision, and guiding must be off. Each history draws from its own simulation's
 * random streams, so every simulation's tallies equal those of its own skgpu_run_primary; they land
 * in each context's device tallies. Counters and device time of the batch are those of the first
 * context (skgpu_get_counters, skgpu_last_run_ms). At most 48 contexts. */
int skgpu_run_batch(skgpu_ctx* const* ctxs, int32_t n, const uint64_t* first, const uint64_t* count,
                    const uint64_t* total_packets);
/* Adds the device tallies of one instrument into the caller's arrays and leaves the device
 * tallies untouched. ifu: num_wavelength_bins*npix (index l + ell*npix), sed: num_wavelength_bins,
 * stats (may be NULL): 5 planes of ifu size then 5 planes of sed size (sum w^k, k=0..4). */
int skgpu_fetch_instrument(skgpu_ctx* ctx, int32_t instrument, double* ifu, double* sed, double* ifu_stats,
                           double* sed_stats);
/* Adds the component planes (transparent, direct, scattered) of an instrument with
 * record_components set: ifu3 holds 3 planes of ifu size, sed3 3 planes of sed size (either may be NULL). */
int skgpu_fetch_instrument_components(skgpu_ctx* ctx, int32_t instrument, double* ifu3, double* sed3);
/* Adds the scattering-level planes of an instrument (skgpu_set_instrument_scattering_levels): levels
 * planes of ifu size or of sed size, plane n-1 for n scatterings. */
int skgpu_fetch_instrument_levels(skgpu_ctx* ctx, int32_t instrument, double* ifu_levels, double* sed_levels);
/* Calibration on the device (FluxRecorder::calibrateAndWrite, FluxRecorder.cpp:876-921, with
 * scaleWavelengthArray / scaleFrameWavelengthArray :97-115; replaces GpuAcceleration::
 * scaleWavelengthValues / scaleFrameWavelengthValues, GpuAcceleration.hpp:488-494): multiplies the
 * instrument's device tallies -- total, component and scattering-level planes, not the statistics --
 * by factors[ell] per wavelength bin, in place (frame entries l + ell*npix). The caller computes the
 * factors as FluxRecorder does: 1 / (4 pi d^2) / effectiveWidth(ell) * Units::ofluxdensity(lambda_ell, 1)
 * for an SED, additionally / omega with Units::osurfacebrightness for a frame. */
int skgpu_calibrate_instrument(skgpu_ctx* ctx, int32_t instrument, const double* factors);
/* Adds the radiation-field tally (num_cells * num_rf_bins, index m*num_rf_bins + ell) into rf. */
int skgpu_fetch_radiation_field(skgpu_ctx* ctx, double* rf);
int skgpu_clear_tallies(skgpu_ctx* ctx);
/* The device tally buffers of the context, for a collective across GPUs before one rank fetches
 * (the segment-end sum of MonteCarloSimulation's ProcessManager::sumToAll / sumToRoot over the
 * instruments and MediumSystem::communicateRadiationField, MediumSystem.cpp:2524-2547, done on the
 * device, e.g. one NCCL all-reduce over NVLink): *num_buffers receives their number; when ptrs and
 * lengths hold max_buffers >= that many entries they receive the device pointers (FP64 arrays,
 * instrument buffers in upload order, then the radiation field) and their lengths in doubles. The
 * pointers stay valid until the instruments, medium or radiation-field grid are uploaded again. */
int skgpu_tally_buffers(skgpu_ctx* ctx, int32_t max_buffers, void** ptrs, uint64_t* lengths, int32_t* num_buffers);
int skgpu_get_counters(skgpu_ctx* ctx, skgpu_counters* out);
/* Milliseconds of device time of the last skgpu_run_primary (CUDA events on the launch stream). */
int skgpu_last_run_ms(skgpu_ctx* ctx, double* ms);

/* ---- stage timing (measurement aid; no reference counterpart) ----
 * Level 1 brackets every launch of the traversal kernel of skgpu_run_primary with CUDA events on the
 * launch stream, level 2 every stage kernel; 0 (the default) records nothing. skgpu_last_stage_times
 * returns, per stage of the last skgpu_run_primary, the summed device milliseconds and the number of
 * launches (arrays of SKGPU_NUM_STAGES; either pointer may be NULL). */
#define SKGPU_STAGE_TRACE 0  /* traversal of peel-off and propagation rays (+ radiation-field updates) */
#define SKGPU_STAGE_PEEL 1   /* detection of finished peel-off rays */
#define SKGPU_STAGE_PROP1 2  /* forced sampling of the interaction optical depth */
#define SKGPU_STAGE_PROP2 3  /* forced interaction: weight, position, scattering, peel-off rays */
#define SKGPU_STAGE_FREE 4   /* non-forced interaction */
#define SKGPU_STAGE_GUIDE 5  /* guided scattering: network inference and direction sampling (guiding on) */
#define SKGPU_STAGE_LAUNCH 6 /* refill of free packet slots with new histories */
#define SKGPU_NUM_STAGES 7
int skgpu_set_stage_timing(skgpu_ctx* ctx, int32_t level);
int skgpu_last_stage_times(skgpu_ctx* ctx, double* ms, uint64_t* launches);

/* ---- learned path guiding (no reference counterpart) ----
 * A small network (8 inputs -> 4 x 64 ReLU -> 40 outputs: 8 von Mises-Fisher lobes over the outgoing
 * direction) proposes scattering directions. Mode SKGPU_GUIDE_RECORD makes the next runs record a
 * fraction of their scattering events (inputs, sampled direction, and the luminosity that the target
 * instrument later detects from the history per unit packet luminosity, optionally weighted per
 * pixel); skgpu_guide_train fits the network to them on the GPU (importance-weighted maximum
 * likelihood, Adam). Mode SKGPU_GUIDE_SAMPLE makes the runs sample alpha * q_net + (1 - alpha) * p_HG
 * and weight the packet by p_HG / (alpha * q_net + (1 - alpha) * p_HG): the estimator stays unbiased,
 * and alpha = 0 is plain sampling. Inference runs as BF16 tensor-core layers with FP32 accumulation.
 * Network inputs: position / domain half size (3), incoming direction (3), log10(lambda / 0.55 um),
 * log(1 + tau) / 5 with tau the optical depth of the propagation path that ended at the event.
 * Outputs per lobe j: [5j] weight logit, [5j+1..5j+3] direction (normalised), [5j+4] concentration
 * (softplus + 0.05, at most 2000). Parameters: FP32, per layer W (out x in, row-major) then b.
 * Guiding is not available through skgpu_run_primary_noalloc. */
#define SKGPU_GUIDE_OFF 0
#define SKGPU_GUIDE_RECORD 1
#define SKGPU_GUIDE_SAMPLE 2
#define SKGPU_GUIDE_NUM_INPUTS 8
#define SKGPU_GUIDE_NUM_OUTPUTS 40
#define SKGPU_GUIDE_RECORD_FLOATS 13 /* inputs[8], direction[3], downstream luminosity, packet luminosity */
int skgpu_guide_num_params(void);
/* creates the network with the given parameters, or a seeded random initialisation (params NULL) */
int skgpu_guide_init(skgpu_ctx* ctx, const float* params, uint64_t seed);
int skgpu_guide_get_params(skgpu_ctx* ctx, float* params);
/* mode, target instrument, alpha (SAMPLE, in [0,1)), recorded fraction and record capacity (RECORD;
 * switching to RECORD discards earlier records) */
int skgpu_guide_set_mode(skgpu_ctx* ctx, int32_t mode, int32_t target_instrument, float alpha, float record_fraction,
                         uint64_t record_capacity);
/* per-pixel weights of the target frame's detections in the records (NULL: weight 1) */
int skgpu_guide_set_importance(skgpu_ctx* ctx, int32_t n, const float* weights);
/* training target: with position_bins > 0 each record's weight is its downstream luminosity over the
 * mean of its position bin (position_bins^3 bins over the domain), so that every region of the
 * domain weighs alike; with 0 (default) over the mean of all records */
int skgpu_guide_set_training(skgpu_ctx* ctx, int32_t position_bins);
/* guided events of the last run and the mean of their weight factors (1 in expectation: a mean far
 * from 1 over many events means the network's density and its sampling disagree) */
int skgpu_guide_last_weights(skgpu_ctx* ctx, uint64_t* events, double* mean_weight);
int skgpu_guide_record_count(skgpu_ctx* ctx, uint64_t* n);
int skgpu_guide_fetch_records(skgpu_ctx* ctx, uint64_t n, float* out);
/* steps of Adam on random batches of the records; the loss of the last batch in final_loss */
int skgpu_guide_train(skgpu_ctx* ctx, int32_t steps, int32_t batch, float learning_rate, uint64_t seed, float* final_loss);
/* sum over n samples of -w log q(direction | inputs) and its gradient (FP32 forward / backward) */
int skgpu_guide_loss_grad(skgpu_ctx* ctx, int32_t n, const float* inputs, const float* directions, const float* weights,
                          float* loss, float* grad);
/* raw outputs (n x 40) for n inputs: BF16 tensor cores (tensor_cores != 0) or FP32 CUDA cores */
int skgpu_guide_infer(skgpu_ctx* ctx, int32_t n, const float* inputs, float* outputs, int32_t tensor_cores);

/* ---- path segments (replaces GpuAcceleration::set*SpatialGridPath, GpuAcceleration.hpp) ----
 * For each ray (x,y,z,kx,ky,kz) the segments (m, ds) the grid's PathSegmentGenerator returns,
 * up to max_segments per ray; count[i] < 0 flags truncation (-n segments generated). */
int skgpu_trace_paths(skgpu_ctx* ctx, int32_t num_rays, const double* rays, int32_t max_segments, int32_t precision,
                      int32_t* count, int32_t* m, double* ds);
/* Optical depth to the domain edge (MediumSystem::getExtinctionOpticalDepth, distance = inf)
 * at wavelength lambda for each ray. */
int skgpu_optical_depths(skgpu_ctx* ctx, int32_t num_rays, const double* rays, double lambda, int32_t precision,
                         double* tau);

/* ---- standalone octree construction ----
 * For scenes not built by SKIRT itself: constructs a TreeSpatialGrid-like octree of an analytic
 * dust geometry with the DensityTreePolicy criteria (SKIRT/core/DensityTreePolicy.cpp:88-245) and
 * the overlap-sorted neighbour lists of OctTreeNode/TreeNode, and samples the mean normalised
 * density per leaf. The exported arrays are exactly those skgpu_upload_grid_octree takes. No
 * reference counterpart: in the drop-in case SKIRT's own tree is uploaded. */
#define SKGPU_GEOM_EXPDISK 0 /* params: hR, hz, Rmin, Rmax (0 = none), zmax (0 = none) */
#define SKGPU_GEOM_SHELL 1   /* params: rmin, rmax, power-law exponent */

typedef struct skgpu_octree_spec {
    int32_t geometry;                /* SKGPU_GEOM_* (unit total mass) */
    int32_t min_level;
    int32_t max_level;
    int32_t num_subdivision_samples; /* random samples per node for the mass-fraction criterion */
    int32_t num_density_samples;     /* random samples per leaf for the cell density */
    int32_t reserved;
    double params[6];
    double extent[6];                /* xmin, ymin, zmin, xmax, ymax, zmax */
    double max_dust_fraction;
    uint64_t seed;
} skgpu_octree_spec;

typedef struct skgpu_octree skgpu_octree;
int skgpu_octree_build(const skgpu_octree_spec* spec, skgpu_octree** out);
int skgpu_octree_sizes(const skgpu_octree* tree, int32_t* num_nodes, int32_t* num_cells, int64_t* num_nb);
/* arrays sized by skgpu_octree_sizes: bounds 6*num_nodes, cell_index/child_begin/child_count
 * num_nodes, child_index 8*(subdivided nodes) (<= num_nodes), nb_begin 6*num_nodes+1, nb_index num_nb,
 * cell_density num_cells (normalised geometry density, unit total mass); any may be NULL */
int skgpu_octree_export(const skgpu_octree* tree, double* bounds, int32_t* cell_index, int32_t* child_begin,
                        int32_t* child_count, int32_t* child_index, int32_t* nb_begin, int32_t* nb_index,
                        double* cell_density);
void skgpu_octree_free(skgpu_octree* tree);

/* ---- standalone Voronoi neighbour construction ----
 * For scenes not built by SKIRT itself: the face neighbours of the Voronoi cells of n sites inside
 * the domain box (extent xmin, ymin, zmin, xmax, ymax, zmax), with the domain walls as -1..-6 (xmin,
 * xmax, ymin, ymax, zmin, zmax): exactly the CSR arrays skgpu_upload_grid_voronoi takes. Cells are
 * built by clipping the box with bisector planes (threads <= 0: all host cores). No reference
 * counterpart: in the drop-in case SKIRT's voro++ mesh is uploaded. */
typedef struct skgpu_voronoi skgpu_voronoi;
int skgpu_voronoi_build(const double* sites, int32_t n, const double* extent, int32_t threads, skgpu_voronoi** out);
int skgpu_voronoi_sizes(const skgpu_voronoi* v, int64_t* num_nb);
/* nb_begin: n + 1 entries, nb_index: num_nb entries */
int skgpu_voronoi_export(const skgpu_voronoi* v, int32_t* nb_begin, int32_t* nb_index);
void skgpu_voronoi_free(skgpu_voronoi* v);

/* ---- standalone Delaunay tetrahedralisation ----
 * For scenes not built by SKIRT itself: the Delaunay tetrahedra of the points inside the domain
 * box, joined by the box's 8 corners, in the form skgpu_upload_grid_tetra takes: positively
 * oriented tetrahedra, face f opposite vertex f, per face the neighbouring tetrahedron (-1 on the
 * hull) and its face index, outward unit normals. Coordinates are snapped to a lattice of 2^20 steps
 * per box side; points on or outside the box surface and points on the lattice point of an earlier
 * one are left out (as TetraMeshSpatialGrid::removeInvalid drops them), so the m vertices exported
 * are the m - 8 kept points in input order followed by the corners. Incremental (Bowyer-Watson)
 * with exact integer predicates. No reference counterpart: in the drop-in case SKIRT's TetGen mesh
 * is uploaded. */
typedef struct skgpu_tetra skgpu_tetra;
int skgpu_tetra_build(const double* points, int32_t n, const double* extent, int32_t threads, skgpu_tetra** out);
int skgpu_tetra_sizes(const skgpu_tetra* t, int32_t* num_vertices, int32_t* num_tetra);
/* vertices 3 x num_vertices, tetra 4 x num_tetra, face_normals 12 x num_tetra, face_ntetra and
 * face_nface 4 x num_tetra; any may be NULL */
int skgpu_tetra_export(const skgpu_tetra* t, double* vertices, int32_t* tetra, double* face_normals,
                       int32_t* face_ntetra, int32_t* face_nface);
void skgpu_tetra_free(skgpu_tetra* t);

#ifdef __cplusplus
}
#endif

#endif /* SKGPU_H */
