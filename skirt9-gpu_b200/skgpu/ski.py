"""Writers for SKIRT 9 ski files (the SimulationItem XML the reference reads).

These produce the ski files of the named workloads (dust shell on a Cartesian grid, exponential
disk galaxy on an octree, Voronoi and tetrahedral meshes, the edge-on thick disk) so that the
reference CPU code and this tracer run the same configuration. Element and attribute names are
those of the reference's schema (`skirt -x`, registered in SKIRT/core/SimulationItemRegistry.cpp).
"""
import math

PC = 3.0856775814913673e16  # m, SKIRT Constants::pc()


def _q(v, unit):
    return f"{v:.17g} {unit}" if unit else f"{v:.17g}"


def cartesian_grid(half_size_pc, nbins, points=None):
    """CartesianSpatialGrid on +-half_size; LinMesh, or ListMesh with normalised border points."""
    if points is None:
        mesh = f'<LinMesh numBins="{nbins}"/>'
        meshes = {a: mesh for a in "XYZ"}
    else:
        meshes = {a: '<ListMesh points="' + ", ".join(f"{p:.17g}" for p in points[a]) + '"/>' for a in "XYZ"}
    h = half_size_pc
    return (f'<CartesianSpatialGrid minX="{-h} pc" maxX="{h} pc" minY="{-h} pc" maxY="{h} pc" '
            f'minZ="{-h} pc" maxZ="{h} pc">'
            f'<meshX type="Mesh">{meshes["X"]}</meshX><meshY type="Mesh">{meshes["Y"]}</meshY>'
            f'<meshZ type="Mesh">{meshes["Z"]}</meshZ></CartesianSpatialGrid>')


def octree_grid(half_size, unit, max_level, max_dust_fraction, min_level=2):
    h = half_size
    return (f'<PolicyTreeSpatialGrid minX="{-h} {unit}" maxX="{h} {unit}" minY="{-h} {unit}" maxY="{h} {unit}" '
            f'minZ="{-h} {unit}" maxZ="{h} {unit}" treeType="OctTree">'
            f'<policy type="TreePolicy"><DensityTreePolicy minLevel="{min_level}" maxLevel="{max_level}" '
            f'maxDustFraction="{max_dust_fraction:g}" maxDustOpticalDepth="0" wavelength="0.55 micron" '
            f'maxDustDensityDispersion="0" maxElectronFraction="1e-6" maxGasFraction="1e-6"/></policy>'
            f'</PolicyTreeSpatialGrid>')


def voronoi_grid(half_size, unit, num_sites, policy="DustDensity", filename=None):
    h = half_size
    f = f' filename="{filename}"' if filename else ""
    return (f'<VoronoiMeshSpatialGrid minX="{-h} {unit}" maxX="{h} {unit}" minY="{-h} {unit}" maxY="{h} {unit}" '
            f'minZ="{-h} {unit}" maxZ="{h} {unit}" policy="{policy}" numSites="{num_sites}"{f} relaxSites="false"/>')


def tetra_grid(half_size, unit, num_samples, policy="DustDensity", filename=None):
    h = half_size
    f = f' filename="{filename}"' if filename else ""
    return (f'<TetraMeshSpatialGrid minX="{-h} {unit}" maxX="{h} {unit}" minY="{-h} {unit}" maxY="{h} {unit}" '
            f'minZ="{-h} {unit}" maxZ="{h} {unit}" policy="{policy}" numSamples="{num_samples}"{f} refine="false"/>')


def vertex_file_text(points_m):
    """Text column file of vertex positions in pc, as TetraMeshSpatialGrid's File policy reads it
    (TetraMeshSpatialGrid.cpp:303-312)."""
    lines = ["# column 1: position x (pc)", "# column 2: position y (pc)", "# column 3: position z (pc)"]
    lines += [f"{x / PC:.17g} {y / PC:.17g} {z / PC:.17g}" for x, y, z in points_m]
    return "\n".join(lines) + "\n"


def sphere1d_grid(rmin_pc, rmax_pc, nbins, mesh="LinMesh"):
    """Sphere1DSpatialGrid between rmin and rmax with nbins radial bins."""
    return (f'<Sphere1DSpatialGrid minRadius="{rmin_pc} pc" maxRadius="{rmax_pc} pc">'
            f'<meshRadial type="Mesh"><{mesh} numBins="{nbins}"/></meshRadial></Sphere1DSpatialGrid>')


def shell_sphere1d(num_packets=1e5, nbins=24, npix=64, stats=True, rmin_pc=0.05):
    """The dust shell of shell_cartesian on a Sphere1DSpatialGrid (rmin to 1 pc, nbins radial bins;
    inside rmin no cell), one frame at 30 degrees with statistics plus one SED instrument."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(),
                      shell_medium(0.1, 1, 2, 2, mix), sphere1d_grid(rmin_pc, 1, nbins),
                      frame_instrument("i30", 30, 2, "pc", npix, stats) + sed_instrument("sed", 30, stats))


def cylinder2d_grid(rmin_pc, rmax_pc, zmin_pc, zmax_pc, nr, nz):
    """Cylinder2DSpatialGrid with nr linear radial bins and nz linear vertical bins."""
    return (f'<Cylinder2DSpatialGrid minRadius="{rmin_pc} pc" maxRadius="{rmax_pc} pc" minZ="{zmin_pc} pc" '
            f'maxZ="{zmax_pc} pc"><meshRadial type="Mesh"><LinMesh numBins="{nr}"/></meshRadial>'
            f'<meshZ type="Mesh"><LinMesh numBins="{nz}"/></meshZ></Cylinder2DSpatialGrid>')


def sphere2d_grid(rmin_pc, rmax_pc, nr, ntheta):
    """Sphere2DSpatialGrid with nr linear radial bins and ntheta linear polar bins."""
    return (f'<Sphere2DSpatialGrid minRadius="{rmin_pc} pc" maxRadius="{rmax_pc} pc">'
            f'<meshRadial type="Mesh"><LinMesh numBins="{nr}"/></meshRadial>'
            f'<meshPolar type="Mesh"><LinMesh numBins="{ntheta}"/></meshPolar></Sphere2DSpatialGrid>')


def sphere3d_grid(rmin_pc, rmax_pc, nr, ntheta, nphi):
    """Sphere3DSpatialGrid with linear radial, polar and azimuthal bins."""
    return (f'<Sphere3DSpatialGrid minRadius="{rmin_pc} pc" maxRadius="{rmax_pc} pc">'
            f'<meshRadial type="Mesh"><LinMesh numBins="{nr}"/></meshRadial>'
            f'<meshPolar type="Mesh"><LinMesh numBins="{ntheta}"/></meshPolar>'
            f'<meshAzimuthal type="Mesh"><LinMesh numBins="{nphi}"/></meshAzimuthal></Sphere3DSpatialGrid>')


def disk_sphere3d(num_packets=1e5, npix=32, stats=True, rmin_pc=0.0):
    """The disk scene of disk_cylinder2d on a Sphere3DSpatialGrid (r up to 4 pc in 12 bins, 9 polar and
    8 azimuthal bins; with rmin 0 the grid adds its artificial inner hole), one frame at 60 degrees
    with statistics plus one SED."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(), expdisk_medium(1.0, 0.2, "pc", 1.0, mix),
                      sphere3d_grid(rmin_pc, 4, 12, 9, 8),
                      frame_instrument("i60", 60, 8, "pc", npix, stats) + sed_instrument("sed", 60, stats),
                      num_density_samples=10)


def disk_scene(grid_xml, num_packets=1e5, npix=32, stats=True):
    """The disk scene of disk_cylinder2d (exponential dust disk hR 1 pc, hz 0.2 pc, face-on tau 1,
    central point source, one 60-degree frame of 8 pc with statistics plus one SED) on any grid."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(), expdisk_medium(1.0, 0.2, "pc", 1.0, mix),
                      grid_xml, frame_instrument("i60", 60, 8, "pc", npix, stats) + sed_instrument("sed", 60, stats),
                      num_density_samples=10)


def cylinder3d_grid(rmin_pc, rmax_pc, zmin_pc, zmax_pc, nr, nphi, nz):
    """Cylinder3DSpatialGrid with linear radial, azimuthal and vertical bins."""
    return (f'<Cylinder3DSpatialGrid minRadius="{rmin_pc} pc" maxRadius="{rmax_pc} pc" minZ="{zmin_pc} pc" '
            f'maxZ="{zmax_pc} pc"><meshRadial type="Mesh"><LinMesh numBins="{nr}"/></meshRadial>'
            f'<meshAzimuthal type="Mesh"><LinMesh numBins="{nphi}"/></meshAzimuthal>'
            f'<meshZ type="Mesh"><LinMesh numBins="{nz}"/></meshZ></Cylinder3DSpatialGrid>')


def disk_cylinder3d(num_packets=1e5, npix=32, stats=True, rmin_pc=0.0):
    """The disk scene of disk_cylinder2d on a Cylinder3DSpatialGrid (R up to 4 pc in 12 bins with the
    grid's artificial inner hole, 8 azimuthal bins, z -1..1 pc in 10 bins), one frame at 60 degrees
    with statistics plus one SED."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(), expdisk_medium(1.0, 0.2, "pc", 1.0, mix),
                      cylinder3d_grid(rmin_pc, 4, -1, 1, 12, 8, 10),
                      frame_instrument("i60", 60, 8, "pc", npix, stats) + sed_instrument("sed", 60, stats),
                      num_density_samples=10)


def disk_sphere2d(num_packets=1e5, npix=32, stats=True):
    """The disk scene of disk_cylinder2d on a Sphere2DSpatialGrid (r 0.05-4 pc in 20 bins, 15 polar
    bins; the grid adds the equatorial border), one frame at 60 degrees with statistics plus one SED."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(), expdisk_medium(1.0, 0.2, "pc", 1.0, mix),
                      sphere2d_grid(0.05, 4, 20, 15),
                      frame_instrument("i60", 60, 8, "pc", npix, stats) + sed_instrument("sed", 60, stats),
                      num_density_samples=10)


def disk_cylinder2d(num_packets=1e5, npix=32, stats=True):
    """Oligochromatic exponential dust disk (hR 1 pc, hz 0.2 pc, face-on tau 1) with a central point
    source on a Cylinder2DSpatialGrid (R 0.05-4 pc in 20 bins, z -1..1 pc in 16 bins), one frame at
    60 degrees with statistics plus one SED instrument."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(), expdisk_medium(1.0, 0.2, "pc", 1.0, mix),
                      cylinder2d_grid(0.05, 4, -1, 1, 20, 16),
                      frame_instrument("i60", 60, 8, "pc", npix, stats) + sed_instrument("sed", 60, stats),
                      num_density_samples=10)


def shell_medium(rmin_pc, rmax_pc, exponent, tau_x, mix):
    return (f'<GeometricMedium velocityMagnitude="0 km/s" magneticFieldStrength="0 uG">'
            f'<geometry type="Geometry"><ShellGeometry minRadius="{rmin_pc} pc" maxRadius="{rmax_pc} pc" '
            f'exponent="{exponent}"/></geometry>'
            f'<materialMix type="MaterialMix">{mix}</materialMix>'
            f'<normalization type="MaterialNormalization"><OpticalDepthMaterialNormalization axis="X" '
            f'wavelength="0.55 micron" opticalDepth="{tau_x}"/></normalization></GeometricMedium>')


def expdisk_medium(hR, hz, unit, tau_z, mix):
    return (f'<GeometricMedium velocityMagnitude="0 km/s" magneticFieldStrength="0 uG">'
            f'<geometry type="Geometry"><ExpDiskGeometry scaleLength="{hR} {unit}" scaleHeight="{hz} {unit}" '
            f'minRadius="0 {unit}" maxRadius="0 {unit}" maxZ="0 {unit}"/></geometry>'
            f'<materialMix type="MaterialMix">{mix}</materialMix>'
            f'<normalization type="MaterialNormalization"><OpticalDepthMaterialNormalization axis="Z" '
            f'wavelength="0.55 micron" opticalDepth="{tau_z}"/></normalization></GeometricMedium>')


def mean_list_mix(wavelengths_um, kappa, albedo, g):
    j = lambda v, u="": ", ".join(f"{x:.17g}{(' ' + u) if u else ''}" for x in v)
    return (f'<MeanListDustMix wavelengths="{j(wavelengths_um, "micron")}" '
            f'extinctionCoefficients="{j(kappa, "m2/kg")}" albedos="{j(albedo)}" asymmetryParameters="{j(g)}"/>')


def point_source(temperature=5800, luminosity_lsun=1.0):
    return (f'<PointSource positionX="0 pc" positionY="0 pc" positionZ="0 pc" velocityX="0 km/s" velocityY="0 km/s" '
            f'velocityZ="0 km/s" sourceWeight="1" wavelengthBias="0.5">'
            f'<angularDistribution type="AngularDistribution"><IsotropicAngularDistribution/></angularDistribution>'
            f'<polarizationProfile type="PolarizationProfile"><NoPolarizationProfile/></polarizationProfile>'
            f'<sed type="SED"><BlackBodySED temperature="{temperature} K"/></sed>'
            f'<normalization type="LuminosityNormalization"><IntegratedLuminosityNormalization wavelengthRange="All" '
            f'integratedLuminosity="{luminosity_lsun} Lsun"/></normalization></PointSource>')


def _instrument_tail(tag, wlg):
    """Closing of an instrument element, with its own wavelength grid (an XML wavelength-grid item)
    when one is given."""
    return f'><wavelengthGrid type="WavelengthGrid">{wlg}</wavelengthGrid></{tag}>' if wlg else "/>"


def frame_instrument(name, inclination_deg, fov, unit, npix, stats=True, distance_mpc=10, comps=False, levels=0,
                     wlg=None):
    return (f'<FrameInstrument instrumentName="{name}" distance="{distance_mpc} Mpc" inclination="{inclination_deg} deg" '
            f'azimuth="0 deg" roll="0 deg" fieldOfViewX="{fov} {unit}" numPixelsX="{npix}" centerX="0 {unit}" '
            f'fieldOfViewY="{fov} {unit}" numPixelsY="{npix}" centerY="0 {unit}" '
            f'recordComponents="{"true" if comps else "false"}" numScatteringLevels="{levels}" recordPolarization="false" '
            f'recordStatistics="{"true" if stats else "false"}"' + _instrument_tail("FrameInstrument", wlg))


def sed_instrument(name, inclination_deg, stats=True, distance_mpc=10, comps=True, levels=0, wlg=None):
    return (f'<SEDInstrument instrumentName="{name}" distance="{distance_mpc} Mpc" inclination="{inclination_deg} deg" '
            f'azimuth="0 deg" roll="0 deg" radius="0 pc" recordComponents="{"true" if comps else "false"}" '
            f'numScatteringLevels="{levels}" recordPolarization="false" recordStatistics="{"true" if stats else "false"}"'
            + _instrument_tail("SEDInstrument", wlg))


def band_grid(bands):
    """ConfigurableBandWavelengthGrid of ListBands; bands: list of (wavelengths in micron,
    transmission values)."""
    items = "".join(f'<ListBand wavelengths="{", ".join(f"{l:g} micron" for l in lam)}" '
                    f'transmissionValues="{", ".join(f"{t:g}" for t in tr)}"/>' for lam, tr in bands)
    return f'<ConfigurableBandWavelengthGrid><bands type="Band">{items}</bands></ConfigurableBandWavelengthGrid>'


# four overlapping bands over 0.2-3 micron (triangles and a flat top), for tests of band grids
TEST_BANDS = [([0.2, 0.35, 0.5], [0.1, 1.0, 0.1]),
              ([0.4, 0.45, 0.7, 0.75], [0.2, 1.0, 1.0, 0.2]),
              ([0.5, 1.0, 1.6], [0.3, 0.9, 0.3]),
              ([1.2, 2.0, 3.0], [1.0, 0.5, 0.2])]


def dust_emission_options(em_min_um=1.0, em_max_um=1000.0, num_em=30, spatial_bias=0.5, source_bias=0.5,
                          wavelength_bias=0.5, packets_multiplier=1.0, store_rf=False):
    """SecondaryEmissionOptions and DustEmissionOptions of a DustEmission simulation: equilibrium
    emission, no CMB heating, AllCellsLibrary, a logarithmic dust-emission wavelength grid and a
    log-uniform wavelength bias distribution over the same range."""
    rng = f'minWavelength="{em_min_um:g} micron" maxWavelength="{em_max_um:g} micron"'
    return (f'<secondaryEmissionOptions type="SecondaryEmissionOptions"><SecondaryEmissionOptions '
            f'storeEmissionRadiationField="{"true" if store_rf else "false"}" secondaryPacketsMultiplier="{packets_multiplier:g}" '
            f'spatialBias="{spatial_bias:g}" sourceBias="{source_bias:g}"/></secondaryEmissionOptions>'
            f'<dustEmissionOptions type="DustEmissionOptions"><DustEmissionOptions dustEmissionType="Equilibrium" '
            f'includeHeatingByCMB="false" maxFractionOfPrimary="0.01" maxFractionOfPrevious="0.03" sourceWeight="1" '
            f'wavelengthBias="{wavelength_bias:g}">'
            f'<cellLibrary type="SpatialCellLibrary"><AllCellsLibrary/></cellLibrary>'
            f'<dustEmissionWLG type="DisjointWavelengthGrid"><LogWavelengthGrid {rng} numWavelengths="{num_em}"/>'
            f'</dustEmissionWLG><wavelengthBiasDistribution type="WavelengthDistribution">'
            f'<LogWavelengthDistribution {rng}/></wavelengthBiasDistribution></DustEmissionOptions></dustEmissionOptions>')


def simulation(mode, num_packets, sources, media, grid, instruments, source_wavelengths="0.55 micron",
               instrument_wlg='<ListWavelengthGrid wavelengths="0.55 micron" relativeHalfWidth="0" log="false"/>',
               force_scattering=True, store_rf=False, rf_wlg="", seed=0, num_density_samples=100,
               min_weight_reduction=1e4, path_length_bias=0.5, explicit_absorption=False, emission="",
               secondary_iterations=None, redshift=0.0):
    """A complete MonteCarloSimulation ski document (`emission`: the secondary and dust emission
    options of a DustEmission simulation, see dust_emission_options)."""
    src_attr = f' wavelengths="{source_wavelengths}"' if mode.startswith("Oligo") else ' minWavelength="0.1 micron" maxWavelength="10 micron"'
    rf = ""
    if store_rf or rf_wlg:
        rf = (f'<radiationFieldOptions type="RadiationFieldOptions"><RadiationFieldOptions '
              f'storeRadiationField="{"true" if store_rf else "false"}">'
              + (f'<radiationFieldWLG type="DisjointWavelengthGrid">{rf_wlg}</radiationFieldWLG>' if rf_wlg else "")
              + '</RadiationFieldOptions></radiationFieldOptions>')
    rf += emission
    cosmology = ('<cosmology type="Cosmology"><LocalUniverseCosmology/></cosmology>' if not redshift else
                 f'<cosmology type="Cosmology"><FlatUniverseCosmology redshift="{redshift:g}" '
                 f'reducedHubbleConstant="0.675" matterDensityFraction="0.31"/></cosmology>')
    iterate = "false"
    iteration_xml = ""
    if secondary_iterations:
        iterate = "true"
        lo, hi = secondary_iterations[:2]
        merged = "true" if len(secondary_iterations) > 2 and secondary_iterations[2] else "false"
        iteration_xml = (f'<iterationOptions type="IterationOptions"><IterationOptions minSecondaryIterations="{lo}" '
                         f'maxSecondaryIterations="{hi}" includePrimaryEmission="{merged}" '
                         f'secondaryIterationPacketsMultiplier="1"/></iterationOptions>')
    return f'''<?xml version="1.0" encoding="UTF-8"?>
<skirt-simulation-hierarchy type="MonteCarloSimulation" format="9" producer="skgpu" time="2026-01-01T00:00:00">
<MonteCarloSimulation userLevel="Expert" simulationMode="{mode}" iteratePrimaryEmission="false" iterateSecondaryEmission="{iterate}" numPackets="{num_packets:g}">
<random type="Random"><Random seed="{seed}"/></random>
<units type="Units"><ExtragalacticUnits wavelengthOutputStyle="Wavelength" fluxOutputStyle="Frequency"/></units>
{cosmology}
<sourceSystem type="SourceSystem"><SourceSystem{src_attr} sourceBias="0.5">
<sources type="Source">{sources}</sources></SourceSystem></sourceSystem>
<mediumSystem type="MediumSystem"><MediumSystem>
<photonPacketOptions type="PhotonPacketOptions"><PhotonPacketOptions explicitAbsorption="{"true" if explicit_absorption else "false"}" forceScattering="{"true" if force_scattering else "false"}" minWeightReduction="{min_weight_reduction:g}" minScattEvents="0" pathLengthBias="{path_length_bias:g}"/></photonPacketOptions>
{iteration_xml}
{rf}
<media type="Medium">{media}</media>
<samplingOptions type="SamplingOptions"><SamplingOptions numDensitySamples="{num_density_samples}" numPropertySamples="1" aggregateVelocity="Average"/></samplingOptions>
<grid type="SpatialGrid">{grid}</grid>
</MediumSystem></mediumSystem>
<instrumentSystem type="InstrumentSystem"><InstrumentSystem>
<defaultWavelengthGrid type="WavelengthGrid">{instrument_wlg}</defaultWavelengthGrid>
<instruments type="Instrument">{instruments}</instruments>
</InstrumentSystem></instrumentSystem>
<probeSystem type="ProbeSystem"><ProbeSystem/></probeSystem>
</MonteCarloSimulation>
</skirt-simulation-hierarchy>
'''


def disk_probe(grid_xml, num_packets=1e4, tau_z=1.0, hR=1.0, hz=0.2):
    """Oligochromatic exponential dust disk (scale length hR pc, height hz pc) with a central
    point source and one SED instrument, on the given grid; used to export grids and paths."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(),
                      expdisk_medium(hR, hz, "pc", tau_z, mix), grid_xml, sed_instrument("sed", 30, False),
                      num_density_samples=10)


def geometric_source(geometry_xml, temperature, luminosity_lsun):
    return (f'<GeometricSource velocityMagnitude="0 km/s" sourceWeight="1" wavelengthBias="0.5">'
            f'<geometry type="Geometry">{geometry_xml}</geometry>'
            f'<sed type="SED"><BlackBodySED temperature="{temperature} K"/></sed>'
            f'<normalization type="LuminosityNormalization"><IntegratedLuminosityNormalization '
            f'wavelengthRange="Source" integratedLuminosity="{luminosity_lsun:g} Lsun"/></normalization>'
            f'</GeometricSource>')


def galaxy_octree(num_packets=1e8, npix=512, nlambda=100, max_level=8, max_dust_fraction=1e-6, tau_v=1.0,
                  half_size_kpc=25, store_rf=True, stats=False, sed=False, grid=None, medium=None,
                  num_density_samples=100):
    """Stellar exponential disk (hR 4 kpc, hz 0.35 kpc) + Sersic n=4 bulge (Re 1 kpc), B/T = 0.2,
    black bodies of 6000 K and 4000 K; dust exponential disk (hR 6 kpc, hz 0.2 kpc, face-on tau_V)
    with power-law MeanListDustMix on 100 log wavelengths 0.1-10 micron; octree by the dust-mass
    fraction policy; three frames at 0, 60 and 90 degrees (with statistics when `stats`), plus an
    SED instrument at 60 degrees when `sed`; radiation field on the same grid. `grid` and `medium`
    replace the policy octree and the analytic dust disk (e.g. a FileTreeSpatialGrid and a
    CellMedium holding the same tree and densities as a standalone scene)."""
    lam = [0.1 * (100.0 ** (i / (nlambda - 1))) for i in range(nlambda)]
    kappa = [(l / 0.55) ** -1.0 for l in lam]
    albedo = [min(0.9, max(0.05, 0.5 * (l / 0.55) ** -0.2)) for l in lam]
    g = [min(0.9, max(0.0, 0.6 * (l / 0.55) ** -0.3)) for l in lam]
    mix = mean_list_mix(lam, kappa, albedo, g)
    sources = (geometric_source('<ExpDiskGeometry scaleLength="4 kpc" scaleHeight="0.35 kpc" minRadius="0 kpc" '
                                'maxRadius="0 kpc" maxZ="0 kpc"/>', 6000, 8e9)
               + geometric_source('<SersicGeometry effectiveRadius="1 kpc" index="4"/>', 4000, 2e9))
    wlg = f'<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="10 micron" numWavelengths="{nlambda}"/>'
    fov = 2 * half_size_kpc
    instruments = "".join(frame_instrument(f"i{inc}", inc, fov, "kpc", npix, stats=stats) for inc in (0, 60, 90))
    if sed:
        instruments += sed_instrument("sed", 60, stats, comps=False)
    if grid is None:
        grid = octree_grid(half_size_kpc, "kpc", max_level, max_dust_fraction)
    if medium is None:
        medium = expdisk_medium(6, 0.2, "kpc", tau_v, mix)
    else:
        medium = medium(mix)
    return simulation("ExtinctionOnly", num_packets, sources, medium, grid, instruments,
                      instrument_wlg=wlg, store_rf=store_rf, rf_wlg=wlg, num_density_samples=num_density_samples)


def dust_galaxy(num_packets=1e5, npix=32, nlambda=20, num_em=30, max_level=6, max_dust_fraction=1e-4, tau_v=1.0,
                half_size_kpc=25):
    """The galaxy of galaxy_octree with dust emission (DustEmission mode) at reduced size: power-law
    MeanListDustMix on 40 log wavelengths 0.1-1000 micron, radiation field on `nlambda` log bins 0.1-10
    micron, equilibrium dust emission on `num_em` log bins 1-1000 micron, three frames at 0, 60 and 90
    degrees and an SED instrument at 60 degrees on 30 log bins 0.1-1000 micron (statistics on)."""
    lam = [0.1 * (1e4 ** (i / 39)) for i in range(40)]
    kappa = [(l / 0.55) ** -1.0 for l in lam]
    albedo = [min(0.9, max(0.01, 0.5 * (l / 0.55) ** -0.5)) for l in lam]
    g = [min(0.9, max(0.0, 0.6 * (l / 0.55) ** -0.3)) for l in lam]
    mix = mean_list_mix(lam, kappa, albedo, g)
    sources = (geometric_source('<ExpDiskGeometry scaleLength="4 kpc" scaleHeight="0.35 kpc" minRadius="0 kpc" '
                                'maxRadius="0 kpc" maxZ="0 kpc"/>', 6000, 8e9)
               + geometric_source('<SersicGeometry effectiveRadius="1 kpc" index="4"/>', 4000, 2e9))
    rf_wlg = f'<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="10 micron" numWavelengths="{nlambda}"/>'
    iwlg = '<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="1000 micron" numWavelengths="30"/>'
    fov = 2 * half_size_kpc
    instruments = "".join(frame_instrument(f"i{inc}", inc, fov, "kpc", npix, stats=True) for inc in (0, 60, 90))
    instruments += sed_instrument("sed", 60, True, comps=False)
    return simulation("DustEmission", num_packets, sources, expdisk_medium(6, 0.2, "kpc", tau_v, mix),
                      octree_grid(half_size_kpc, "kpc", max_level, max_dust_fraction), instruments,
                      instrument_wlg=iwlg, store_rf=True, rf_wlg=rf_wlg, emission=dust_emission_options(num_em=num_em))


def galaxy_voronoi(num_packets=1e8, npix=512, nlambda=100, num_sites=1_000_000, tau_v=2.0, half_size_kpc=25,
                   store_rf=True, sites_file=None):
    """The galaxy of galaxy_octree on a VoronoiMeshSpatialGrid with 1e6 sites, face-on tau_V = 2, two
    frames at 0 and 90 degrees. With `sites_file` the reference reads the site positions from that
    text column file (policy File, e.g. the seeded sites of skgpu.workloads.disk_sites written by
    vertex_file_text); otherwise it draws them from the dust density itself."""
    lam = [0.1 * (100.0 ** (i / (nlambda - 1))) for i in range(nlambda)]
    kappa = [(l / 0.55) ** -1.0 for l in lam]
    albedo = [min(0.9, max(0.05, 0.5 * (l / 0.55) ** -0.2)) for l in lam]
    g = [min(0.9, max(0.0, 0.6 * (l / 0.55) ** -0.3)) for l in lam]
    mix = mean_list_mix(lam, kappa, albedo, g)
    sources = (geometric_source('<ExpDiskGeometry scaleLength="4 kpc" scaleHeight="0.35 kpc" minRadius="0 kpc" '
                                'maxRadius="0 kpc" maxZ="0 kpc"/>', 6000, 8e9)
               + geometric_source('<SersicGeometry effectiveRadius="1 kpc" index="4"/>', 4000, 2e9))
    wlg = f'<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="10 micron" numWavelengths="{nlambda}"/>'
    fov = 2 * half_size_kpc
    instruments = "".join(frame_instrument(f"i{inc}", inc, fov, "kpc", npix, stats=False) for inc in (0, 90))
    return simulation("ExtinctionOnly", num_packets, sources, expdisk_medium(6, 0.2, "kpc", tau_v, mix),
                      voronoi_grid(half_size_kpc, "kpc", num_sites, "File" if sites_file else "DustDensity", sites_file), instruments,
                      instrument_wlg=wlg, store_rf=store_rf, rf_wlg=wlg)


def shell_cartesian(num_packets=1e6, nbins=64, npix=256, stats=True, points=None, explicit_absorption=False,
                    force_scattering=True):
    """Dust shell (r^-2 between 0.1 and 1 pc, radial tau_V = 1, i.e. tau_X = 2 through the centre) on a
    Cartesian grid of +-1 pc, isotropic point source at the centre, 0.55 micron, HG g = 0.6,
    albedo 0.5, one frame at inclination 30 degrees plus one SED instrument."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(),
                      shell_medium(0.1, 1, 2, 2, mix), cartesian_grid(1, nbins, points),
                      frame_instrument("i30", 30, 2, "pc", npix, stats) + sed_instrument("sed", 30, stats),
                      explicit_absorption=explicit_absorption, force_scattering=force_scattering)


def dust_shell(num_packets=1e6, nbins=16, npix=32, stats=True, nlambda=20, num_em=30, grid=None, medium=None,
               self_absorption=None):
    """The dust shell of shell_cartesian with dust emission (DustEmission mode): a 5800 K black-body
    point source of 1e5 Lsun (0.1-10 micron), power-law MeanListDustMix on 40 log wavelengths 0.1-1000
    micron, radiation field on `nlambda` log bins 0.1-10 micron, equilibrium dust emission on `num_em`
    log bins 1-1000 micron, a 32^2 frame at 30 degrees and an SED instrument at 30 degrees on 30 log
    bins 0.1-1000 micron (statistics on). `grid` replaces the Cartesian grid, `medium` (a function of
    the mix XML) the shell medium; self_absorption = (min, max) secondary iterations turns on dust
    self-absorption (the emission radiation field stored, iterateSecondaryEmission), (min, max, True)
    with the primary emission in the iterations (includePrimaryEmission: merged iterations)."""
    lam = [0.1 * (1e4 ** (i / 39)) for i in range(40)]
    kappa = [(l / 0.55) ** -1.0 for l in lam]
    albedo = [min(0.9, max(0.01, 0.5 * (l / 0.55) ** -0.5)) for l in lam]
    g = [min(0.9, max(0.0, 0.6 * (l / 0.55) ** -0.3)) for l in lam]
    mix = mean_list_mix(lam, kappa, albedo, g)
    rf_wlg = f'<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="10 micron" numWavelengths="{nlambda}"/>'
    iwlg = '<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="1000 micron" numWavelengths="30"/>'
    med = medium(mix) if medium else shell_medium(0.1, 1, 2, 2, mix)
    return simulation("DustEmission", num_packets, point_source(luminosity_lsun=1e5), med,
                      grid or cartesian_grid(1, nbins), frame_instrument("i30", 30, 2, "pc", npix, stats)
                      + sed_instrument("sed", 30, stats, comps=False), instrument_wlg=iwlg, store_rf=True,
                      rf_wlg=rf_wlg, emission=dust_emission_options(num_em=num_em, store_rf=bool(self_absorption)),
                      secondary_iterations=self_absorption)


def galaxy_tetra(num_packets, vertex_filename, tau_v=1.0, npix=256, nlambda=32, half_size_kpc=25):
    """The galaxy of galaxy_octree with `nlambda` wavelengths on a TetraMeshSpatialGrid whose vertices
    are read from a text column file (policy File), face-on tau_V, one frame at 60 degrees."""
    lam = [0.1 * (100.0 ** (i / (nlambda - 1))) for i in range(nlambda)]
    kappa = [(l / 0.55) ** -1.0 for l in lam]
    albedo = [min(0.9, max(0.05, 0.5 * (l / 0.55) ** -0.2)) for l in lam]
    g = [min(0.9, max(0.0, 0.6 * (l / 0.55) ** -0.3)) for l in lam]
    mix = mean_list_mix(lam, kappa, albedo, g)
    sources = (geometric_source('<ExpDiskGeometry scaleLength="4 kpc" scaleHeight="0.35 kpc" minRadius="0 kpc" '
                                'maxRadius="0 kpc" maxZ="0 kpc"/>', 6000, 8e9)
               + geometric_source('<SersicGeometry effectiveRadius="1 kpc" index="4"/>', 4000, 2e9))
    wlg = f'<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="10 micron" numWavelengths="{nlambda}"/>'
    instruments = frame_instrument("i60", 60, 2 * half_size_kpc, "kpc", npix, stats=False)
    return simulation("ExtinctionOnly", num_packets, sources, expdisk_medium(6, 0.2, "kpc", tau_v, mix),
                      tetra_grid(half_size_kpc, "kpc", 100, policy="File", filename=vertex_filename), instruments,
                      instrument_wlg=wlg, store_rf=False)


def galaxy_levels_bands(num_packets=30000, npix=16, nlambda=10, max_level=5, max_dust_fraction=1e-3, levels=3,
                        bands=None):
    """The galaxy on a small octree with two instruments at 60 degrees that record components: a
    frame on the log wavelength grid with `levels` scattering levels, and an SED on a band
    wavelength grid (TEST_BANDS) with statistics and two scattering levels."""
    lam = [0.1 * (100.0 ** (i / (nlambda - 1))) for i in range(nlambda)]
    kappa = [(l / 0.55) ** -1.0 for l in lam]
    albedo = [min(0.9, max(0.05, 0.5 * (l / 0.55) ** -0.2)) for l in lam]
    g = [min(0.9, max(0.0, 0.6 * (l / 0.55) ** -0.3)) for l in lam]
    mix = mean_list_mix(lam, kappa, albedo, g)
    sources = (geometric_source('<ExpDiskGeometry scaleLength="4 kpc" scaleHeight="0.35 kpc" minRadius="0 kpc" '
                                'maxRadius="0 kpc" maxZ="0 kpc"/>', 6000, 8e9)
               + geometric_source('<SersicGeometry effectiveRadius="1 kpc" index="4"/>', 4000, 2e9))
    wlg = f'<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="10 micron" numWavelengths="{nlambda}"/>'
    instruments = (frame_instrument("i60", 60, 50, "kpc", npix, stats=True, comps=True, levels=levels)
                   + sed_instrument("bands", 60, stats=True, comps=True, levels=2,
                                    wlg=band_grid(bands or TEST_BANDS)))
    return simulation("ExtinctionOnly", num_packets, sources, expdisk_medium(6, 0.2, "kpc", 1.0, mix),
                      octree_grid(25, "kpc", max_level, max_dust_fraction), instruments, instrument_wlg=wlg)


def adaptive_mesh_text(half_pc=4.0, root=(4, 4, 2), max_level=3, rho0=2000.0, hR=1.0, hz=0.2):
    """An adaptive-mesh data file (the text format AdaptiveMeshSnapshot reads: "! nx ny nz" lines for
    subdivided nodes, one density row per leaf, children in local Morton order with x fastest) of an
    exponential disk of mass density rho0 * exp(-R/hR - |z|/hz) Msun/pc3 on the cube of half size
    half_pc. The root is split root = (nx, ny, nz); nodes near the disk are refined up to max_level
    with subdivisions that vary by level (2x2x2, 3x3x1, 1x2x3), so that the mesh exercises
    non-cubic splits."""
    splits = {1: (2, 2, 2), 2: (3, 3, 1), 3: (1, 2, 3)}
    lines = ["# adaptive mesh: exponential disk", "# column 1: mass density (Msun/pc3)"]

    def node(b, level):
        (x0, y0, z0), (x1, y1, z1) = b
        cx, cy, cz = 0.5 * (x0 + x1), 0.5 * (y0 + y1), 0.5 * (z0 + z1)
        size = max(x1 - x0, y1 - y0, z1 - z0)
        near = (cx * cx + cy * cy) ** 0.5 < 2.0 * hR + size and abs(cz) < 3.0 * hz + size
        div = root if level == 0 else (splits.get(level) if near and level <= max_level else None)
        if div is None:
            lines.append(f"{rho0 * math.exp(-((cx * cx + cy * cy) ** 0.5) / hR - abs(cz) / hz):.9e}")
            return
        nx, ny, nz = div
        lines.append(f"! {nx} {ny} {nz}")
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    lo = (x0 + i * (x1 - x0) / nx, y0 + j * (y1 - y0) / ny, z0 + k * (z1 - z0) / nz)
                    hi = (x0 + (i + 1) * (x1 - x0) / nx, y0 + (j + 1) * (y1 - y0) / ny, z0 + (k + 1) * (z1 - z0) / nz)
                    node((lo, hi), level + 1)

    h = half_pc
    node(((-h, -h, -h), (h, h, h)), 0)
    return "\n".join(lines) + "\n"


def adaptive_mesh_medium(filename, half_pc, mix):
    h = half_pc
    return (f'<AdaptiveMeshMedium filename="{filename}" minX="{-h} pc" maxX="{h} pc" minY="{-h} pc" maxY="{h} pc" '
            f'minZ="{-h} pc" maxZ="{h} pc" massType="MassDensity" massFraction="1" importMetallicity="false" '
            f'importTemperature="false" maxTemperature="0 K" importVelocity="false" importMagneticField="false" '
            f'importVariableMixParams="false" useColumns=""><materialMix type="MaterialMix">{mix}</materialMix>'
            f'</AdaptiveMeshMedium>')


def disk_adaptive(num_packets=1e5, filename="mesh.txt", npix=32, stats=True, half_pc=4.0):
    """The disk scene (central point source, one 60-degree frame of 8 pc with statistics plus one SED)
    on an AdaptiveMeshSpatialGrid of an imported AdaptiveMeshMedium (adaptive_mesh_text in
    `filename`, next to the ski file)."""
    mix = mean_list_mix([0.5, 0.6], [1, 1], [0.5, 0.5], [0.6, 0.6])
    return simulation("OligoExtinctionOnly", num_packets, point_source(), adaptive_mesh_medium(filename, half_pc, mix),
                      "<AdaptiveMeshSpatialGrid/>",
                      frame_instrument("i60", 60, 2 * half_pc, "pc", npix, stats) + sed_instrument("sed", 60, stats),
                      num_density_samples=10)


def dust_adaptive(num_packets=1e5):
    """DustEmission (the dust_shell configuration) on an AdaptiveMeshSpatialGrid: an imported
    adaptive-mesh disk (hR 0.25 pc, hz 0.05 pc) in the +-1 pc box around the 1e5 Lsun point source.
    Returns the ski text and its input files."""
    text = dust_shell(num_packets, grid="<AdaptiveMeshSpatialGrid/>",
                      medium=lambda mix: adaptive_mesh_medium("mesh.txt", 1.0, mix))
    return text, {"mesh.txt": adaptive_mesh_text(half_pc=1.0, hR=0.25, hz=0.05, rho0=500.0)}


def dust_tetra(num_packets=1e5, num_vertices=3000):
    """DustEmission (the dust_shell configuration) on a TetraMeshSpatialGrid of the dust shell
    (vertices sampled from the dust density by the reference's own policy) in the +-1 pc box."""
    return dust_shell(num_packets, grid=tetra_grid(1, "pc", num_vertices))


def dust_sphere1d(num_packets=1e5):
    """DustEmission (the dust_shell configuration) on a Sphere1DSpatialGrid of 24 shells 0.05-1 pc."""
    return dust_shell(num_packets, grid=sphere1d_grid(0.05, 1, 24))


def dust_curvilinear(num_packets, kind):
    """DustEmission (the dust_shell configuration) on a spherical or cylindrical grid of the +-1 pc
    shell: kind in sphere2d, sphere3d, cylinder2d, cylinder3d."""
    grid = {"sphere2d": lambda: sphere2d_grid(0.05, 1, 16, 12),
            "sphere3d": lambda: sphere3d_grid(0.05, 1, 12, 8, 8),
            "cylinder2d": lambda: cylinder2d_grid(0.05, 1, -1, 1, 16, 16),
            "cylinder3d": lambda: cylinder3d_grid(0.05, 1, -1, 1, 12, 8, 12)}[kind]()
    return dust_shell(num_packets, grid=grid)


def galaxy_observer(num_packets=30000, npix=16, nlambda=10, redshift=0.0, aperture_kpc=0.0):
    """The galaxy on a small octree with a frame and two SED instruments at 60 degrees: at `redshift`
    (a flat-universe cosmology, instruments at distance 0 so that they observe in the redshifted
    frame), the second SED with an aperture of `aperture_kpc`."""
    lam = [0.1 * (100.0 ** (i / (nlambda - 1))) for i in range(nlambda)]
    kappa = [(l / 0.55) ** -1.0 for l in lam]
    albedo = [min(0.9, max(0.05, 0.5 * (l / 0.55) ** -0.2)) for l in lam]
    g = [min(0.9, max(0.0, 0.6 * (l / 0.55) ** -0.3)) for l in lam]
    mix = mean_list_mix(lam, kappa, albedo, g)
    sources = (geometric_source('<ExpDiskGeometry scaleLength="4 kpc" scaleHeight="0.35 kpc" minRadius="0 kpc" '
                                'maxRadius="0 kpc" maxZ="0 kpc"/>', 6000, 8e9)
               + geometric_source('<SersicGeometry effectiveRadius="1 kpc" index="4"/>', 4000, 2e9))
    wlg = f'<LogWavelengthGrid minWavelength="0.1 micron" maxWavelength="10 micron" numWavelengths="{nlambda}"/>'
    d = 0 if redshift else 10
    aperture = sed_instrument("ap", 60, stats=True, distance_mpc=d, comps=False)
    if aperture_kpc:
        aperture = aperture.replace('radius="0 pc"', f'radius="{aperture_kpc} kpc"')
    instruments = (frame_instrument("i60", 60, 50, "kpc", npix, stats=True, distance_mpc=d)
                   + sed_instrument("sed", 60, stats=True, distance_mpc=d, comps=False) + aperture)
    return simulation("ExtinctionOnly", num_packets, sources, expdisk_medium(6, 0.2, "kpc", 1.0, mix),
                      octree_grid(25, "kpc", 5, 1e-3), instruments, instrument_wlg=wlg, redshift=redshift)
