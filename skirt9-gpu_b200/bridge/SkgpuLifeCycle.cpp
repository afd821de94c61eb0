/* SkgpuLifeCycle: flattens SKIRT's SimulationItem tree into the C ABI of include/skgpu.h, runs the
 * primary and secondary life-cycle segments on the B200 and adds the results into SKIRT's own
 * detector and radiation-field arrays. See SkgpuLifeCycle.hpp.
 *
 * Supported (otherwise the bridge declines and SKIRT runs its CPU life cycle): one dust medium
 * (DustMix, no polarisation, no kinematics, no Lyman-alpha, no dynamic medium state); Cartesian,
 * octree (TreeSpatialGrid) or 1D spherical grids; PointSource and GeometricSource (exponential
 * disk, Sersic) primary sources with a black-body SED (panchromatic) or any continuous SED
 * (oligochromatic); frame and SED instruments (distant, SED aperture radius 0, no scattering levels,
 * no polarisation), with statistics and components; forced or free propagation, explicit
 * absorption, the primary radiation field; equilibrium dust emission (AllCellsLibrary, no storage
 * of the emission radiation field) for the secondary segment on Cartesian and octree grids.
 *
 * The SKIRT members this file reads are private in the reference headers; SKIRT's tree gives them
 * to the bridge with `friend class SkgpuLifeCycle;` in each class. Built out of tree against
 * unmodified headers, the translation unit opens private access for its own includes instead.
 */
#include "SkgpuLifeCycle.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "skgpu.h"

#define private public
#define protected public
#include "AdaptiveMeshSnapshot.hpp"
#include "AdaptiveMeshSpatialGrid.hpp"
#include "BlackBodySED.hpp"
#include "CartesianSpatialGrid.hpp"
#include "Cylinder2DSpatialGrid.hpp"
#include "Cylinder3DSpatialGrid.hpp"
#include "Configuration.hpp"
#include "ContSED.hpp"
#include "DefaultWavelengthDistribution.hpp"
#include "BandWavelengthGrid.hpp"
#include "DisjointWavelengthGrid.hpp"
#include "DustMix.hpp"
#include "EquilibriumDustEmissionCalculator.hpp"
#include "ExpDiskGeometry.hpp"
#include "FatalError.hpp"
#include "FluxRecorder.hpp"
#include "FrameInstrument.hpp"
#include "GeometricSource.hpp"
#include "Instrument.hpp"
#include "InstrumentSystem.hpp"
#include "Log.hpp"
#include "LogWavelengthDistribution.hpp"
#include "MediumSystem.hpp"
#include "MonteCarloSimulation.hpp"
#include "NormalizedSource.hpp"
#include "PointSource.hpp"
#include "ProcessManager.hpp"
#include "Random.hpp"
#include "SEDInstrument.hpp"
#include "SecondarySourceSystem.hpp"
#include "SersicFunction.hpp"
#include "SersicGeometry.hpp"
#include "SourceSystem.hpp"
#include "Sphere1DSpatialGrid.hpp"
#include "Sphere2DSpatialGrid.hpp"
#include "Sphere3DSpatialGrid.hpp"
#include "TetraMeshSpatialGrid.hpp"
#include "TreeNode.hpp"
#include "TreeSpatialGrid.hpp"
#include "VoronoiMeshSnapshot.hpp"
#include "VoronoiMeshSpatialGrid.hpp"
#include "WavelengthDistribution.hpp"
#undef private
#undef protected

namespace
{
    bool g_enabled = false;
    skgpu_ctx* g_ctx = nullptr;
    int g_device = -1;
    const MonteCarloSimulation* g_scene = nullptr;  // the simulation whose scene is on the device
    bool g_dustTables = false;

    bool envTrue(const char* name)
    {
        const char* v = std::getenv(name);
        return v && *v && std::string(v) != "0" && std::string(v) != "false";
    }

    void check(int rc, const char* what)
    {
        if (rc != SKGPU_OK)
            throw FATALERROR(string("B200 life cycle: ") + what + ": " + skgpu_last_error(g_ctx));
    }

    std::vector<double> vec(const Array& a) { return std::vector<double>(begin(a), end(a)); }

    // ---------------------------------------------------------------------------------------------
    // what the library implements

    // the range of a log-uniform wavelength distribution (LogWavelengthDistribution, or the default
    // bias distribution, log-uniform over the source range: DefaultWavelengthDistribution.cpp:17-39)
    bool logUniform(WavelengthDistribution* d)
    {
        return dynamic_cast<LogWavelengthDistribution*>(d) || dynamic_cast<DefaultWavelengthDistribution*>(d);
    }
    Range logUniformRange(WavelengthDistribution* d)
    {
        if (auto l = dynamic_cast<LogWavelengthDistribution*>(d)) return l->range();
        return dynamic_cast<DefaultWavelengthDistribution*>(d)->_range;
    }

    const DustMix* dustMix(MonteCarloSimulation* sim)
    {
        auto ms = sim->mediumSystem();
        return ms && ms->_numMedia == 1 ? dynamic_cast<const DustMix*>(ms->mix(0, 0)) : nullptr;
    }

    bool supported(MonteCarloSimulation* sim, bool secondary, string& why)
    {
        auto config = sim->config();
        if (!config->hasMedium()) return (why = "no medium"), false;
        if (!dustMix(sim)) return (why = "not a single dust medium"), false;
        if (config->hasPolarization() || config->hasMovingMedia() || config->_hasMovingSources
            || config->_hasLymanAlpha || config->hasDynamicState() || config->hasVariableMedia())
            return (why = "polarisation, kinematics, Lyman-alpha or a dynamic medium"), false;
        auto grid = sim->mediumSystem()->grid();
        // grids whose cells are boxes (the secondary launch draws positions in them)
        bool box = dynamic_cast<CartesianSpatialGrid*>(grid) || dynamic_cast<TreeSpatialGrid*>(grid)
                   || dynamic_cast<AdaptiveMeshSpatialGrid*>(grid);
        bool other = dynamic_cast<Sphere1DSpatialGrid*>(grid) || dynamic_cast<Sphere2DSpatialGrid*>(grid)
                     || dynamic_cast<Sphere3DSpatialGrid*>(grid) || dynamic_cast<Cylinder2DSpatialGrid*>(grid)
                     || dynamic_cast<Cylinder3DSpatialGrid*>(grid) || dynamic_cast<VoronoiMeshSpatialGrid*>(grid)
                     || dynamic_cast<TetraMeshSpatialGrid*>(grid);
        if (!box && !other) return (why = "grid type"), false;
        for (Instrument* instr : sim->instrumentSystem()->instruments())
        {
            auto rec = instr->instrumentFluxRecorder();
            if (rec->_recordPolarization || rec->_local) return (why = "instrument options"), false;
            auto sed = dynamic_cast<SEDInstrument*>(instr);
            if (!dynamic_cast<FrameInstrument*>(instr) && !sed) return (why = "instrument type"), false;
            if (!dynamic_cast<const DisjointWavelengthGrid*>(rec->_lambdagrid)
                && !dynamic_cast<const BandWavelengthGrid*>(rec->_lambdagrid))
                return (why = "instrument grid"), false;
        }
        if (!secondary)
        {
            for (Source* s : sim->sourceSystem()->_sources)
            {
                auto ns = dynamic_cast<NormalizedSource*>(s);
                if (!ns) return (why = "source type"), false;
                bool point = dynamic_cast<PointSource*>(s) != nullptr;
                auto gs = dynamic_cast<GeometricSource*>(s);
                if (!point && !(gs && (dynamic_cast<ExpDiskGeometry*>(gs->_geometry)
                                       || dynamic_cast<SersicGeometry*>(gs->_geometry))))
                    return (why = "source geometry"), false;
                if (config->oligochromatic() ? !ns->_contsed : !dynamic_cast<BlackBodySED*>(ns->_sed))
                    return (why = "source SED"), false;
                if (!config->oligochromatic() && ns->_xi > 0 && !logUniform(ns->_biasDistribution))
                    return (why = "wavelength bias distribution"), false;
            }
        }
        else
        {
            // grids whose randomPositionInCell the library reproduces for the secondary launch
            if (!config->hasDustEmission() || config->hasGasEmission() || config->hasStochasticDustEmission()
                || !config->hasPanRadiationField())
                return (why = "secondary emission other than equilibrium dust emission"), false;
            if (config->cellLibrary()->type() != "AllCellsLibrary") return (why = "cell library"), false;
            if (config->dustEmissionWavelengthBias() > 0
                && !dynamic_cast<LogWavelengthDistribution*>(config->dustEmissionWavelengthBiasDistribution()))
                return (why = "dust emission bias distribution"), false;
        }
        return true;
    }

    // ---------------------------------------------------------------------------------------------
    // uploads

    void uploadGrid(MonteCarloSimulation* sim)
    {
        auto grid = sim->mediumSystem()->grid();
        if (auto g = dynamic_cast<CartesianSpatialGrid*>(grid))
        {
            check(skgpu_upload_grid_cartesian(g_ctx, &g->_xv[0], g->_xv.size(), &g->_yv[0], g->_yv.size(), &g->_zv[0],
                                              g->_zv.size()),
                  "Cartesian grid");
            return;
        }
        if (auto g = dynamic_cast<Sphere1DSpatialGrid*>(grid))
        {
            const Array& rv = g->radialBorderPositions();
            check(skgpu_upload_grid_sphere1d(g_ctx, rv.size(), &rv[0]), "1D spherical grid");
            return;
        }
        if (auto g = dynamic_cast<Sphere2DSpatialGrid*>(grid))
        {
            check(skgpu_upload_grid_sphere2d(g_ctx, g->_rv.size(), &g->_rv[0], g->_thetav.size(), &g->_thetav[0],
                                             &g->_cv[0]),
                  "2D spherical grid");
            return;
        }
        if (auto g = dynamic_cast<Sphere3DSpatialGrid*>(grid))
        {
            check(skgpu_upload_grid_sphere3d(g_ctx, g->_rv.size(), &g->_rv[0], g->_thetav.size(), &g->_thetav[0],
                                             &g->_cv[0], g->_phiv.size(), &g->_phiv[0], &g->_sinv[0], &g->_cosv[0],
                                             g->_eps),
                  "3D spherical grid");
            return;
        }
        if (auto g = dynamic_cast<Cylinder2DSpatialGrid*>(grid))
        {
            check(skgpu_upload_grid_cylinder2d(g_ctx, g->_Rv.size(), &g->_Rv[0], g->_zv.size(), &g->_zv[0]),
                  "2D cylindrical grid");
            return;
        }
        if (auto g = dynamic_cast<Cylinder3DSpatialGrid*>(grid))
        {
            check(skgpu_upload_grid_cylinder3d(g_ctx, g->_Rv.size(), &g->_Rv[0], g->_phiv.size(), &g->_phiv[0],
                                               &g->_sinv[0], &g->_cosv[0], g->_zv.size(), &g->_zv[0], g->_eps,
                                               g->_hasHole ? 1 : 0),
                  "3D cylindrical grid");
            return;
        }
        if (auto g = dynamic_cast<AdaptiveMeshSpatialGrid*>(grid))
        {
            // the snapshot's own traversal arrays (AdaptiveMeshSnapshot.cpp:172-199)
            const std::vector<double>& b = g->traversalNodeBounds();
            std::vector<int32_t> cell(g->traversalCellIndex().begin(), g->traversalCellIndex().end()),
                begin(g->traversalChildBegin().begin(), g->traversalChildBegin().end()),
                count(g->traversalChildCount().begin(), g->traversalChildCount().end()),
                child(g->traversalChildIndex().begin(), g->traversalChildIndex().end());
            check(skgpu_upload_grid_adaptive_mesh(g_ctx, cell.size(), b.data(), cell.data(), begin.data(), count.data(),
                                                  child.data(), child.size(), g->_mesh->_eps),
                  "adaptive mesh");
            return;
        }
        if (auto vg = dynamic_cast<VoronoiMeshSpatialGrid*>(grid))
        {
            // the snapshot's traversal arrays: sites and the neighbour CSR with wall ids -1..-6
            // (VoronoiMeshSnapshot.cpp:725-740)
            auto m = vg->_mesh;
            int n = m->_traversalNeighborBegin.size();
            std::vector<int32_t> begin(n + 1), index(m->_traversalNeighborIndex.begin(), m->_traversalNeighborIndex.end());
            for (int c = 0; c != n; ++c) begin[c] = m->_traversalNeighborBegin[c];
            begin[n] = index.size();
            Box e = vg->extent();
            double ext[6] = {e.xmin(), e.ymin(), e.zmin(), e.xmax(), e.ymax(), e.zmax()};
            check(skgpu_upload_grid_voronoi(g_ctx, n, m->_traversalSiteCoordinates.data(), begin.data(), index.data(),
                                            index.size(), ext, m->_eps),
                  "Voronoi mesh");
            // the cells' enclosing boxes, for the secondary launch (VoronoiMeshSnapshot::extent(m))
            std::vector<double> boxes(6 * static_cast<size_t>(n));
            for (int c = 0; c != n; ++c)
            {
                Box b = m->extent(c);
                double* q = &boxes[6 * static_cast<size_t>(c)];
                q[0] = b.xmin(); q[1] = b.ymin(); q[2] = b.zmin(); q[3] = b.xmax(); q[4] = b.ymax(); q[5] = b.zmax();
            }
            check(skgpu_upload_voronoi_cell_boxes(g_ctx, n, boxes.data()), "Voronoi cell boxes");
            return;
        }
        if (auto g = dynamic_cast<TetraMeshSpatialGrid*>(grid))
        {
            // vertices, per tetrahedron its vertex indices and per face the outward normal and the
            // neighbour across it (TetraMeshSpatialGrid.hpp, Tetra / Face)
            int nv = g->_vertices.size(), nt = g->_tetrahedra.size();
            std::vector<double> verts(3 * static_cast<size_t>(nv)), normals(12 * static_cast<size_t>(nt));
            std::vector<int32_t> tv(4 * static_cast<size_t>(nt)), ntet(4 * static_cast<size_t>(nt)),
                nface(4 * static_cast<size_t>(nt));
            for (int i = 0; i != nv; ++i)
            {
                verts[3 * i] = g->_vertices[i].x();
                verts[3 * i + 1] = g->_vertices[i].y();
                verts[3 * i + 2] = g->_vertices[i].z();
            }
            for (int t = 0; t != nt; ++t)
            {
                const auto& tet = g->_tetrahedra[t];
                for (int f = 0; f != 4; ++f)
                {
                    tv[4 * t + f] = tet._vertexIndices[f];
                    ntet[4 * t + f] = tet._faces[f]._ntetra;
                    nface[4 * t + f] = tet._faces[f]._nface;
                    normals[12 * t + 3 * f] = tet._faces[f]._normal.x();
                    normals[12 * t + 3 * f + 1] = tet._faces[f]._normal.y();
                    normals[12 * t + 3 * f + 2] = tet._faces[f]._normal.z();
                }
            }
            Box e = g->extent();
            double ext[6] = {e.xmin(), e.ymin(), e.zmin(), e.xmax(), e.ymax(), e.zmax()};
            check(skgpu_upload_grid_tetra(g_ctx, nv, verts.data(), nt, tv.data(), normals.data(), ntet.data(),
                                          nface.data(), ext, g->_eps),
                  "tetrahedral mesh");
            return;
        }
        auto g = dynamic_cast<TreeSpatialGrid*>(grid);
        int numNodes = g->_nodev.size();
        std::vector<double> bounds(6 * static_cast<size_t>(numNodes));
        std::vector<int32_t> cellIndex(numNodes), childBegin(numNodes), childCount(numNodes), childIndex;
        std::vector<int32_t> nbBegin(6 * static_cast<size_t>(numNodes) + 1), nbIndex;
        for (int l = 0; l != numNodes; ++l)
        {
            TreeNode* node = g->_nodev[l];
            if (node->id() != l) throw FATALERROR("B200 life cycle: octree node ids out of order");
            double* b = &bounds[6 * static_cast<size_t>(l)];
            b[0] = node->xmin(); b[1] = node->ymin(); b[2] = node->zmin();
            b[3] = node->xmax(); b[4] = node->ymax(); b[5] = node->zmax();
            cellIndex[l] = g->_cellindexv[l];
            childBegin[l] = childIndex.size();
            childCount[l] = node->children().size();
            for (auto c : node->children()) childIndex.push_back(c->id());
            // neighbours per wall in the order TreeNode keeps them (largest overlap first)
            for (int w = 0; w != 6; ++w)
            {
                nbBegin[6 * static_cast<size_t>(l) + w] = nbIndex.size();
                for (auto nb : node->_neighbors[w]) nbIndex.push_back(nb->id());
            }
        }
        nbBegin[6 * static_cast<size_t>(numNodes)] = nbIndex.size();
        check(skgpu_upload_grid_octree(g_ctx, numNodes, bounds.data(), cellIndex.data(), childBegin.data(),
                                       childCount.data(), childIndex.data(), childIndex.size(), nbBegin.data(),
                                       nbIndex.data(), nbIndex.size(), g->_eps),
              "octree");
    }

    void uploadWLG(const WavelengthGrid* wlg, std::vector<double>& borders, std::vector<int32_t>& ellv)
    {
        auto d = dynamic_cast<const DisjointWavelengthGrid*>(wlg);
        borders.assign(begin(d->_borderv), end(d->_borderv));
        ellv.assign(d->_ellv.begin(), d->_ellv.end());
    }

    void uploadMedium(MonteCarloSimulation* sim)
    {
        auto ms = sim->mediumSystem();
        int numCells = ms->_state._numCells;
        std::vector<double> n(numCells);
        for (int m = 0; m != numCells; ++m) n[m] = ms->_state.numberDensity(m, 0);
        check(skgpu_upload_medium(g_ctx, numCells, n.data()), "medium");
        const DustMix* mix = dustMix(sim);
        check(skgpu_upload_dust_mix(g_ctx, mix->_lambdav.size(), &mix->_lambdav[0], &mix->_sigmaextv[0],
                                    &mix->_sigmascav[0], &mix->_asymmparv[0]),
              "dust mix");
        if (sim->config()->hasRadiationField())
        {
            std::vector<double> b;
            std::vector<int32_t> e;
            uploadWLG(sim->config()->radiationFieldWLG(), b, e);
            check(skgpu_upload_rf_grid(g_ctx, sim->config()->radiationFieldWLG()->numBins(), b.size(), b.data(), e.data()),
                  "radiation-field grid");
        }
    }

    void uploadInstruments(MonteCarloSimulation* sim)
    {
        std::vector<skgpu_instrument> v;
        std::vector<double> borders;
        std::vector<int32_t> ellv;
        for (Instrument* instr : sim->instrumentSystem()->instruments())
        {
            auto rec = instr->instrumentFluxRecorder();
            skgpu_instrument d{};
            auto f = dynamic_cast<FrameInstrument*>(instr);
            d.kind = f ? SKGPU_INSTR_FRAME : SKGPU_INSTR_SED;
            d.same_observer = instr->isSameObserverAsPreceding() ? 1 : 0;
            d.record_statistics = rec->_recordStatistics ? 1 : 0;
            d.record_components = rec->_recordTotalOnly ? 0 : 1;
            d.num_wavelength_bins = rec->_lambdagrid->numBins();
            std::vector<double> b{0.};
            std::vector<int32_t> e{-1, -1};  // band grids: no disjoint bin (skgpu_set_instrument_bands below)
            if (!dynamic_cast<const BandWavelengthGrid*>(rec->_lambdagrid)) uploadWLG(rec->_lambdagrid, b, e);
            d.wlg_offset = ellv.size();
            d.wlg_num_borders = b.size();
            borders.insert(borders.end(), b.begin(), b.end());
            borders.push_back(0.);  // border list and bin map share the offset; the map has one more entry
            ellv.insert(ellv.end(), e.begin(), e.end());
            Direction k = static_cast<DistantInstrument*>(instr)->bfkobs(Position());
            d.kobs[0] = k.x();
            d.kobs[1] = k.y();
            d.kobs[2] = k.z();
            if (auto sed = dynamic_cast<SEDInstrument*>(instr))
            {
                // the projection of ApertureInstrument::isInsideAperture
                d.cos_theta = sed->_costheta; d.sin_theta = sed->_sintheta;
                d.cos_phi = sed->_cosphi; d.sin_phi = sed->_sinphi;
            }
            if (f)
            {
                d.num_pixels_x = f->_Nxp;
                d.num_pixels_y = f->_Nyp;
                d.cos_theta = f->_costheta; d.sin_theta = f->_sintheta;
                d.cos_phi = f->_cosphi; d.sin_phi = f->_sinphi;
                d.cos_omega = f->_cosomega; d.sin_omega = f->_sinomega;
                d.xp_min = f->_xpmin; d.xp_size = f->_xpsiz;
                d.yp_min = f->_ypmin; d.yp_size = f->_ypsiz;
            }
            v.push_back(d);
        }
        check(skgpu_upload_instruments(g_ctx, v.size(), v.data(), ellv.size(), borders.data(), ellv.data()),
              "instruments");
        int i = 0;
        for (Instrument* instr : sim->instrumentSystem()->instruments())
        {
            auto rec = instr->instrumentFluxRecorder();
            if (!rec->_recordTotalOnly && rec->_numScatteringLevels > 0)
                check(skgpu_set_instrument_scattering_levels(g_ctx, i, rec->_numScatteringLevels), "scattering levels");
            // observer-frame redshift and SED aperture (FluxRecorder::detect, ApertureInstrument)
            double radius = 0.;
            if (auto sed = dynamic_cast<SEDInstrument*>(instr)) radius = sed->radius();
            if (rec->_redshift != 0. || radius > 0.)
                check(skgpu_set_instrument_observer(g_ctx, i, rec->_redshift, radius), "instrument observer");
            if (auto bg = dynamic_cast<const BandWavelengthGrid*>(rec->_lambdagrid))
            {
                // the bands in the grid's (pivot wavelength) order with their normalised tables
                std::vector<int32_t> sizes;
                std::vector<double> lambda, trans, width;
                for (int ell = 0; ell != bg->numBins(); ++ell)
                {
                    const Band* band = bg->band(ell);
                    size_t size = band->transmissionDataSize();
                    sizes.push_back(static_cast<int32_t>(size));
                    lambda.insert(lambda.end(), band->transmissionWavelengthData(), band->transmissionWavelengthData() + size);
                    trans.insert(trans.end(), band->transmissionValueData(), band->transmissionValueData() + size);
                    width.push_back(band->effectiveWidth());
                }
                check(skgpu_set_instrument_bands(g_ctx, i, sizes.size(), sizes.data(), lambda.data(), trans.data(),
                                                 width.data()),
                      "instrument bands");
            }
            ++i;
        }
    }

    // the sources of SourceSystem after prepareForLaunch(Npp): history ranges, packet luminosities,
    // launch tables (SourceSystem.cpp, NormalizedSource.cpp:73-110)
    void uploadSources(MonteCarloSimulation* sim)
    {
        auto ss = sim->sourceSystem();
        auto config = sim->config();
        std::vector<skgpu_source> v;
        std::vector<double> tl, ta, tb, rr, rp;
        for (size_t h = 0; h != ss->_sources.size(); ++h)
        {
            auto ns = dynamic_cast<NormalizedSource*>(ss->_sources[h]);
            skgpu_source s{};
            s.first_history = ss->_Iv[h];
            s.num_histories = ss->_Iv[h + 1] - ss->_Iv[h];
            s.packet_luminosity = ss->_Lpp * ss->_Lv[h] / ss->_Wv[h];
            s.table_offset = tl.size();
            if (config->oligochromatic())
            {
                // oligochromatic: one of the wavelengths of the bias distribution, uniformly, with the
                // composite-bias weight s / b of each (xi = 1)
                s.spectral_model = SKGPU_SPEC_DISCRETE;
                for (double lambda : ss->wavelengths())
                {
                    tl.push_back(lambda);
                    ta.push_back(ns->_contsed->specificLuminosity(lambda) / ns->_biasDistribution->probability(lambda));
                    tb.push_back(0.);
                }
            }
            else
            {
                auto bb = dynamic_cast<BlackBodySED*>(ns->_sed);
                s.spectral_model = SKGPU_SPEC_TABLE;
                tl.insert(tl.end(), begin(bb->_lambdav), end(bb->_lambdav));
                ta.insert(ta.end(), begin(bb->_pv), end(bb->_pv));
                tb.insert(tb.end(), begin(bb->_Pv), end(bb->_Pv));
                s.wavelength_bias = ns->_xi;
                if (ns->_xi > 0)
                {
                    Range r = logUniformRange(ns->_biasDistribution);
                    s.bias_lambda_min = r.min();
                    s.bias_lambda_max = r.max();
                }
            }
            s.table_size = tl.size() - s.table_offset;
            if (auto ps = dynamic_cast<PointSource*>(ns))
            {
                s.position_model = SKGPU_SRC_POINT;
                s.position[0] = ps->positionX();
                s.position[1] = ps->positionY();
                s.position[2] = ps->positionZ();
            }
            else
            {
                auto gs = dynamic_cast<GeometricSource*>(ns);
                if (auto ed = dynamic_cast<ExpDiskGeometry*>(gs->_geometry))
                {
                    s.position_model = SKGPU_SRC_EXPDISK;
                    s.geometry[0] = ed->_hR;
                    s.geometry[1] = ed->_hz;
                    s.geometry[2] = ed->_Rmin;
                    s.geometry[3] = ed->_Rmax;
                    s.geometry[4] = ed->_zmax;
                }
                else
                {
                    auto sg = dynamic_cast<SersicGeometry*>(gs->_geometry);
                    s.position_model = SKGPU_SRC_RADIAL_LOGLOG;
                    s.geometry[0] = sg->_reff;
                    s.radial_offset = rr.size();
                    s.radial_size = sg->_sersicfunction->_sv.size();
                    rr.insert(rr.end(), begin(sg->_sersicfunction->_sv), end(sg->_sersicfunction->_sv));
                    rp.insert(rp.end(), begin(sg->_sersicfunction->_Mv), end(sg->_sersicfunction->_Mv));
                }
            }
            v.push_back(s);
        }
        if (rr.empty()) rr.assign(1, 0.), rp.assign(1, 0.);
        check(skgpu_upload_sources(g_ctx, v.size(), v.data(), tl.size(), tl.data(), ta.data(), tb.data(), rr.size(),
                                   rr.data(), rp.data()),
              "sources");
    }

    // secondary and iteration segments run so far in this simulation: each draws from streams of its own
    uint64_t g_secondarySegments = 0;
    uint64_t g_iterationSegments = 0;

    void setOptions(MonteCarloSimulation* sim, bool storeRF, bool peel = true, uint64_t stream = 0)
    {
        auto config = sim->config();
        skgpu_options o{};
        o.force_scattering = config->forceScattering() ? 1 : 0;
        o.min_scatt_events = config->minScattEvents();
        o.min_weight_reduction = config->minWeightReduction();
        o.path_length_bias = config->pathLengthBias();
        o.store_radiation_field = storeRF ? 1 : 0;
        o.peel_off = peel ? 1 : 0;
        const char* p = std::getenv("SKGPU_PRECISION");
        o.precision = p && std::string(p) == "fp64" ? SKGPU_PREC_FP64_EXACT : SKGPU_PREC_FP32;
        o.explicit_absorption = config->explicitAbsorption() ? 1 : 0;
        o.seed = static_cast<uint64_t>(sim->random()->seed()) * 0x9E3779B97F4A7C15ULL
                 + static_cast<uint64_t>(ProcessManager::rank()) + stream * 0xD1B54A32D192ED03ULL;
        check(skgpu_set_options(g_ctx, &o), "options");
    }

    // (re)creates the context and uploads the scene of `sim` (grid, medium, mix, RF grid, instruments)
    void ensureScene(MonteCarloSimulation* sim)
    {
        if (!g_ctx)
        {
            int dev = 0;
            if (const char* d = std::getenv("SKGPU_DEVICE"))
                dev = std::atoi(d);
            else
            {
                int32_t n = 0;
                if (skgpu_device_count(&n) == SKGPU_OK && n > 0) dev = ProcessManager::rank() % n;
            }
            if (skgpu_create(dev, &g_ctx) != SKGPU_OK)
            {
                string msg = g_ctx ? skgpu_last_error(g_ctx) : "no context";
                skgpu_destroy(g_ctx);
                g_ctx = nullptr;
                throw FATALERROR("B200 life cycle: cannot create a device context: " + msg);
            }
            g_device = dev;
        }
        if (g_scene == sim) return;
        uploadGrid(sim);
        uploadMedium(sim);
        uploadInstruments(sim);
        g_scene = sim;
        g_dustTables = false;
        g_secondarySegments = 0;
        g_iterationSegments = 0;
    }

    // adds the device tallies of the last segment into the FluxRecorder arrays, then the caller
    // clears the device tallies. FluxRecorder keeps either the total alone, or (recording components)
    // only the components, whose sum the output writes as the total (FluxRecorder.cpp:258-300):
    // Transparent, PrimaryDirect, PrimaryScattered for the primary segment and SecondaryTransparent,
    // SecondaryDirect, SecondaryScattered for the secondary one (component indices
    // FluxRecorder.cpp:31-39); the statistics planes sum w^k, k = 0..4, go to _wifu / _wsed
    void fetchInstruments(MonteCarloSimulation* sim, bool primary)
    {
        enum { Total = 0, Transparent, PrimaryDirect, PrimaryScattered, SecondaryDirect, SecondaryScattered,
               SecondaryTransparent };
        int i = 0;
        for (Instrument* instr : sim->instrumentSystem()->instruments())
        {
            auto rec = instr->instrumentFluxRecorder();
            bool frame = dynamic_cast<FrameInstrument*>(instr) != nullptr;
            vector<Array>& arrays = frame ? rec->_ifu : rec->_sed;
            bool comps = !rec->_recordTotalOnly;
            size_t n = arrays[comps ? PrimaryDirect : Total].size();
            if (!n) throw FATALERROR("B200 life cycle: instrument without detector arrays");
            std::vector<double> total(n, 0.), stats(rec->_recordStatistics ? 5 * n : 0, 0.);
            check(skgpu_fetch_instrument(g_ctx, i, frame ? total.data() : nullptr, frame ? nullptr : total.data(),
                                         frame && !stats.empty() ? stats.data() : nullptr,
                                         !frame && !stats.empty() ? stats.data() : nullptr),
                  "instrument tallies");
            if (!stats.empty())
            {
                vector<Array>& w = frame ? rec->_wifu : rec->_wsed;
                for (int k = 0; k != 5; ++k)
                    for (size_t q = 0; q != n; ++q) w[k][q] += stats[k * n + q];
            }
            if (!comps)
            {
                for (size_t q = 0; q != n; ++q) arrays[Total][q] += total[q];
            }
            else
            {
                std::vector<double> comp(3 * n, 0.);
                check(skgpu_fetch_instrument_components(g_ctx, i, frame ? comp.data() : nullptr,
                                                        frame ? nullptr : comp.data()),
                      "instrument components");
                int planes[3] = {Transparent, PrimaryDirect, PrimaryScattered};
                if (!primary) planes[0] = SecondaryTransparent, planes[1] = SecondaryDirect, planes[2] = SecondaryScattered;
                for (int c = 0; c != 3; ++c)
                {
                    if (arrays[planes[c]].size() != n)
                        throw FATALERROR("B200 life cycle: component arrays missing (secondary emission without medium emission?)");
                    for (size_t q = 0; q != n; ++q) arrays[planes[c]][q] += comp[c * n + q];
                }
                // PrimaryScatteredLevel + n - 1 for n = 1..levels, the planes after Total, the six
                // components and the 21 polarisation planes (FluxRecorder.cpp:31-61); the secondary
                // segment records none
                int levels = rec->_numScatteringLevels;
                if (primary && levels > 0)
                {
                    const int PrimaryScatteredLevel = 28;
                    std::vector<double> lv(static_cast<size_t>(levels) * n, 0.);
                    check(skgpu_fetch_instrument_levels(g_ctx, i, frame ? lv.data() : nullptr, frame ? nullptr : lv.data()),
                          "scattering levels");
                    for (int c = 0; c != levels; ++c)
                    {
                        if (arrays[PrimaryScatteredLevel + c].size() != n)
                            throw FATALERROR("B200 life cycle: scattering-level arrays missing");
                        for (size_t q = 0; q != n; ++q) arrays[PrimaryScatteredLevel + c][q] += lv[c * n + q];
                    }
                }
            }
            ++i;
        }
    }
}

////////////////////////////////////////////////////////////////////

void SkgpuLifeCycle::setProcessEnabled(bool enabled)
{
    g_enabled = enabled;
}

bool SkgpuLifeCycle::isProcessEnabled()
{
    return g_enabled || envTrue("SKGPU");
}

std::string SkgpuLifeCycle::status()
{
    if (!isProcessEnabled()) return "off (the B200 life cycle needs -g or SKGPU=1)";
    return "B200 photon-packet life cycle (skgpu C ABI " + std::to_string(skgpu_abi_version()) + ")"
           + (g_device >= 0 ? " on device " + std::to_string(g_device) : "");
}

namespace
{
    // a primary-emission segment: with peel the detections go to the instruments, with storeRF the
    // radiation field to MediumSystem::_rf1; stream 0 for the primary segment, a fresh one for each
    // segment of the merged iterations
    bool runPrimarySegment(MonteCarloSimulation* sim, size_t Npp, bool peel, bool storeRF, uint64_t stream,
                           const char* what)
    {
        if (!SkgpuLifeCycle::isProcessEnabled()) return false;
        string why;
        if (!supported(sim, false, why))
        {
            sim->log()->warning(string("B200 life cycle not used for the ") + what + ": " + why);
            return false;
        }
        ensureScene(sim);
        setOptions(sim, storeRF, peel, stream);
        uploadSources(sim);
        check(skgpu_clear_tallies(g_ctx), "clear");
        // this process's share of the history indices, as Parallel::call distributes them over processes
        size_t first = 0, count = Npp;
        if (ProcessManager::isMultiProc())
        {
            size_t n = ProcessManager::size(), r = ProcessManager::rank();
            first = Npp * r / n;
            count = Npp * (r + 1) / n - first;
        }
        sim->log()->info("Running " + std::to_string(count) + " primary histories on the B200");
        check(skgpu_run_primary(g_ctx, first, count, Npp), "primary segment");
        if (peel) fetchInstruments(sim, true);
        if (storeRF)
        {
            Table<2>& rf = sim->mediumSystem()->_rf1;
            check(skgpu_fetch_radiation_field(g_ctx, &rf.data()[0]), "radiation field");
        }
        check(skgpu_clear_tallies(g_ctx), "clear");
        return true;
    }
}

bool SkgpuLifeCycle::runPrimary(MonteCarloSimulation* sim, size_t Npp)
{
    return runPrimarySegment(sim, Npp, true, sim->config()->hasRadiationField(), 0, "primary emission");
}

bool SkgpuLifeCycle::runPrimaryIteration(MonteCarloSimulation* sim, size_t Npp)
{
    return runPrimarySegment(sim, Npp, false, true, ++g_iterationSegments, "merged primary emission iteration");
}

namespace
{
    // a secondary-emission segment: with peel the detections go to the instruments (runSecondaryEmission),
    // with storeRF the segment's radiation field goes to MediumSystem::_rf2c (storeEmissionRadiationField,
    // and every secondary iteration); the dust emission follows MediumSystem::radiationField, the
    // primary field plus the secondary field of the previous segment (_rf1 + _rf2)
    bool runSecondarySegment(MonteCarloSimulation* sim, size_t Npp, bool peel, bool storeRF, const char* what)
    {
        if (!SkgpuLifeCycle::isProcessEnabled()) return false;
        string why;
        if (!supported(sim, true, why))
        {
            sim->log()->warning(string("B200 life cycle not used for the ") + what + ": " + why);
            return false;
        }
        ensureScene(sim);
        auto config = sim->config();
        auto ms = sim->mediumSystem();
        if (!g_dustTables)
        {
            const EquilibriumDustEmissionCalculator& c = dustMix(sim)->_calc;
            auto rfw = config->radiationFieldWLG();
            std::vector<double> sal(rfw->numBins());
            for (int ell = 0; ell != rfw->numBins(); ++ell) sal[ell] = dustMix(sim)->sectionAbs(rfw->wavelength(ell));
            int numCells = ms->_state._numCells;
            std::vector<double> vol(numCells);
            for (int m = 0; m != numCells; ++m) vol[m] = ms->_state.volume(m);
            Range er = config->dustEmissionWLG()->wavelengthRange();
            double range[2] = {er.min(), er.max()};
            check(skgpu_upload_dust_emission(g_ctx, c._rflambdav.size(), &c._rfsigmaabsvv[0][0], &c._rfdlambdav[0],
                                             &c._Bcmbv[0], sal.data(), c._Tv.size(), &c._Tv[0], &c._planckabsvv[0][0],
                                             c._emlambdav.size(), &c._emlambdav[0], &c._emsigmaabsvv[0][0], range,
                                             numCells, vol.data()),
                  "dust emission tables");
            g_dustTables = true;
        }
        setOptions(sim, storeRF, peel, ++g_secondarySegments);
        // the radiation field as MediumSystem::radiationField sums it (after the communication
        // between processes)
        Table<2>& rf1 = ms->_rf1;
        std::vector<double> rf(rf1.data().size());
        for (size_t q = 0; q != rf.size(); ++q) rf[q] = rf1.data()[q];
        if (ms->_rf2.size())
            for (size_t q = 0; q != rf.size(); ++q) rf[q] += ms->_rf2.data()[q];
        check(skgpu_upload_radiation_field(g_ctx, rf.data()), "radiation field upload");
        skgpu_secondary_options so{};
        so.spatial_bias = config->secondarySpatialBias();
        so.source_bias = config->secondarySourceBias();
        so.wavelength_bias = config->dustEmissionWavelengthBias();
        if (so.wavelength_bias > 0)
        {
            Range r = static_cast<LogWavelengthDistribution*>(config->dustEmissionWavelengthBiasDistribution())->range();
            so.bias_lambda_min = r.min();
            so.bias_lambda_max = r.max();
        }
        double L = 0.;
        check(skgpu_prepare_secondary(g_ctx, &so, Npp, &L), "secondary preparation");
        if (!(L > 0)) return true;  // nothing to launch (SKIRT has already reported zero dust luminosity)
        check(skgpu_clear_tallies(g_ctx), "clear");
        size_t first = 0, count = Npp;
        if (ProcessManager::isMultiProc())
        {
            size_t n = ProcessManager::size(), r = ProcessManager::rank();
            first = Npp * r / n;
            count = Npp * (r + 1) / n - first;
        }
        sim->log()->info("Running " + std::to_string(count) + " secondary histories on the B200");
        check(skgpu_run_secondary(g_ctx, first, count), "secondary segment");
        if (peel) fetchInstruments(sim, false);
        if (storeRF) check(skgpu_fetch_radiation_field(g_ctx, &ms->_rf2c.data()[0]), "secondary radiation field");
        check(skgpu_clear_tallies(g_ctx), "clear");
        return true;
    }
}

bool SkgpuLifeCycle::runSecondary(MonteCarloSimulation* sim, size_t Npp)
{
    return runSecondarySegment(sim, Npp, true, sim->config()->storeEmissionRadiationField(), "secondary emission");
}

bool SkgpuLifeCycle::runSecondaryIteration(MonteCarloSimulation* sim, size_t Npp)
{
    return runSecondarySegment(sim, Npp, false, true, "secondary emission iteration");
}

void SkgpuLifeCycle::release()
{
    if (g_ctx) skgpu_destroy(g_ctx);
    g_ctx = nullptr;
    g_scene = nullptr;
    g_device = -1;
}
