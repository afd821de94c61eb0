// Test infrastructure (oracle side): an export harness linked against the reference SKIRT 9
// libraries built from source by oracle/ref.mk. It is never part of the product path.
//
//   skirt_export <file.ski> <outdir> [rays.npy [maxSegments [lambda_m]]]
//
// The harness reads a ski file through the reference's own SimulationItem machinery
// (XmlHierarchyCreator + MonteCarloSimulation::setupSimulation, as SkirtCommandLineHandler.cpp
// does at SKIRT/main/SkirtCommandLineHandler.cpp:315-380), then writes the flattened state that
// the GPU tracer consumes as .npy files in <outdir>:
//   - the spatial grid (Cartesian borders, octree nodes + overlap-sorted neighbour lists,
//     Voronoi sites + neighbour lists, tetrahedra + faces);
//   - the medium state (number density per cell and medium) and dust-mix tables;
//   - instrument and source parameters (for geometric sources the exponential-disk parameters or the
//     Sersic cumulative-mass table, for black-body SEDs the launch table, and the wavelength bias);
//   - a launch probe: SourceSystem::launch of SKGPU_PROBE_N packets (default 1000), src_probe.npy;
//   - with SKGPU_EXPORT_RUN=1, the raw detector arrays of a single-threaded primary-emission segment
//     (totals and per-history statistics sums, inst<i>_*.npy) and its primary radiation field
//     MediumSystem::_rf1 (rf1.npy);
//   - optionally, for each ray (x,y,z,kx,ky,kz) in rays.npy, the reference path segments
//     (m, ds) produced by SpatialGrid::createPathSegmentGenerator() -> next(), i.e. by the
//     reference's own CPU generators (CartesianSpatialGrid.cpp:77-155, TreeSpatialGrid.cpp:143-228,
//     VoronoiMeshSnapshot.cpp:1089-1222, TetraMeshSpatialGrid.cpp:688-831), and the optical depth
//     to the domain edge from MediumSystem::getExtinctionOpticalDepth (MediumSystem.cpp:2328-2443).
//
// Members that the reference keeps private (octree neighbour lists, tetra faces, dust tables)
// are read by compiling the reference headers with private/protected access opened; the
// reference sources themselves are compiled unchanged.

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include <array>
#include <algorithm>
#include <functional>
#include <mutex>
#include <atomic>
#include <thread>
#include <condition_variable>
#include <unordered_map>
#include <limits>
#include <cmath>

#define private public
#define protected public
#include "BuildInfo.hpp"
#include "BlackBodySED.hpp"
#include "DefaultWavelengthDistribution.hpp"
#include "ExpDiskGeometry.hpp"
#include "GeometricSource.hpp"
#include "LogWavelengthDistribution.hpp"
#include "NormalizedSource.hpp"
#include "SersicFunction.hpp"
#include "SersicGeometry.hpp"
#include "AdaptiveMeshSnapshot.hpp"
#include "AdaptiveMeshSpatialGrid.hpp"
#include "CartesianSpatialGrid.hpp"
#include "Configuration.hpp"
#include "DisjointWavelengthGrid.hpp"
#include "DustMix.hpp"
#include "EquilibriumDustEmissionCalculator.hpp"
#include "SecondarySourceSystem.hpp"
#include "FatalError.hpp"
#include "FilePaths.hpp"
#include "FluxRecorder.hpp"
#include "FrameInstrument.hpp"
#include "Instrument.hpp"
#include "InstrumentSystem.hpp"
#include "Log.hpp"
#include "MediumSystem.hpp"
#include "MonteCarloSimulation.hpp"
#include "PathSegmentGenerator.hpp"
#include "PhotonPacket.hpp"
#include "ProcessManager.hpp"
#include "SEDInstrument.hpp"
#include "SimulationItemRegistry.hpp"
#include "SourceSystem.hpp"
#include "SpatialGrid.hpp"
#include "SpatialGridPath.hpp"
#include "System.hpp"
#include "Cylinder2DSpatialGrid.hpp"
#include "Cylinder3DSpatialGrid.hpp"
#include "Sphere1DSpatialGrid.hpp"
#include "Sphere2DSpatialGrid.hpp"
#include "Sphere3DSpatialGrid.hpp"
#include "TetraMeshSpatialGrid.hpp"
#include "TreeNode.hpp"
#include "TreeSpatialGrid.hpp"
#include "VoronoiMeshSnapshot.hpp"
#include "VoronoiMeshSpatialGrid.hpp"
#include "WavelengthGrid.hpp"
#include "XmlHierarchyCreator.hpp"
#undef private
#undef protected

namespace
{
    // ---- minimal .npy writer (format version 1.0) ----
    template<typename T> const char* npyDescr();
    template<> const char* npyDescr<double>() { return "<f8"; }
    template<> const char* npyDescr<int32_t>() { return "<i4"; }
    template<> const char* npyDescr<int64_t>() { return "<i8"; }

    template<typename T>
    void writeNpy(const std::string& path, const T* data, const std::vector<size_t>& shape)
    {
        std::ostringstream hdr;
        hdr << "{'descr': '" << npyDescr<T>() << "', 'fortran_order': False, 'shape': (";
        size_t n = 1;
        for (size_t i = 0; i < shape.size(); ++i)
        {
            hdr << shape[i] << (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
            n *= shape[i];
        }
        hdr << "), }";
        std::string h = hdr.str();
        size_t total = 10 + h.size() + 1;
        size_t pad = (64 - total % 64) % 64;
        h += std::string(pad, ' ');
        h += '\n';
        std::ofstream out(path, std::ios::binary);
        const char magic[] = "\x93NUMPY";
        out.write(magic, 6);
        char ver[2] = {1, 0};
        out.write(ver, 2);
        uint16_t hl = static_cast<uint16_t>(h.size());
        out.write(reinterpret_cast<const char*>(&hl), 2);
        out.write(h.data(), h.size());
        out.write(reinterpret_cast<const char*>(data), n * sizeof(T));
    }

    template<typename T> void writeVec(const std::string& path, const std::vector<T>& v)
    {
        writeNpy(path, v.data(), {v.size()});
    }

    // ---- minimal .npy reader for a contiguous little-endian f8 array ----
    std::vector<double> readNpyDoubles(const std::string& path, size_t& rows, size_t& cols)
    {
        std::ifstream in(path, std::ios::binary);
        if (!in) throw std::runtime_error("cannot open " + path);
        char pre[10];
        in.read(pre, 10);
        uint16_t hl;
        std::memcpy(&hl, pre + 8, 2);
        std::string h(hl, ' ');
        in.read(&h[0], hl);
        if (h.find("<f8") == std::string::npos) throw std::runtime_error("rays must be float64");
        auto p = h.find("shape");
        auto a = h.find('(', p), b = h.find(')', p);
        std::string s = h.substr(a + 1, b - a - 1);
        std::vector<size_t> dims;
        std::stringstream ss(s);
        std::string tok;
        while (std::getline(ss, tok, ','))
        {
            if (tok.find_first_not_of(' ') == std::string::npos) continue;
            dims.push_back(std::stoul(tok));
        }
        rows = dims.size() > 0 ? dims[0] : 0;
        cols = dims.size() > 1 ? dims[1] : 1;
        std::vector<double> v(rows * cols);
        in.read(reinterpret_cast<char*>(v.data()), v.size() * sizeof(double));
        return v;
    }

    struct Meta
    {
        std::ostringstream s;
        void kv(const std::string& k, const std::string& v) { s << k << " " << v << "\n"; }
        void kv(const std::string& k, double v)
        {
            char buf[64];
            std::snprintf(buf, sizeof buf, "%.17g", v);
            s << k << " " << buf << "\n";
        }
    };

    void exportGrid(SpatialGrid* grid, const std::string& out, Meta& meta)
    {
        Box ext = dynamic_cast<BoxSpatialGrid*>(grid) ? dynamic_cast<BoxSpatialGrid*>(grid)->extent() : Box();
        std::vector<double> extent = {ext.xmin(), ext.ymin(), ext.zmin(), ext.xmax(), ext.ymax(), ext.zmax()};
        writeVec(out + "/grid_extent.npy", extent);

        if (auto g = dynamic_cast<CartesianSpatialGrid*>(grid))
        {
            meta.kv("grid", "cartesian");
            std::vector<double> xb(begin(g->_xv), end(g->_xv)), yb(begin(g->_yv), end(g->_yv)),
                zb(begin(g->_zv), end(g->_zv));
            writeVec(out + "/grid_xb.npy", xb);
            writeVec(out + "/grid_yb.npy", yb);
            writeVec(out + "/grid_zb.npy", zb);
            return;
        }
        if (auto g = dynamic_cast<Cylinder2DSpatialGrid*>(grid))
        {
            meta.kv("grid", "cylinder2d");
            std::vector<double> rv(begin(g->_Rv), end(g->_Rv)), zv(begin(g->_zv), end(g->_zv));
            writeVec(out + "/grid_rv.npy", rv);
            writeVec(out + "/grid_zv.npy", zv);
            return;
        }
        if (auto g = dynamic_cast<Cylinder3DSpatialGrid*>(grid))
        {
            meta.kv("grid", "cylinder3d");
            meta.kv("eps", g->_eps);
            meta.kv("has_hole", g->_hasHole ? 1. : 0.);
            auto vec = [](const Array& a) { return std::vector<double>(begin(a), end(a)); };
            writeVec(out + "/grid_rv.npy", vec(g->_Rv));
            writeVec(out + "/grid_phiv.npy", vec(g->_phiv));
            writeVec(out + "/grid_sinv.npy", vec(g->_sinv));
            writeVec(out + "/grid_cosv.npy", vec(g->_cosv));
            writeVec(out + "/grid_zv.npy", vec(g->_zv));
            return;
        }
        if (auto g = dynamic_cast<Sphere3DSpatialGrid*>(grid))
        {
            meta.kv("grid", "sphere3d");
            meta.kv("eps", g->_eps);
            auto vec = [](const Array& a) { return std::vector<double>(begin(a), end(a)); };
            writeVec(out + "/grid_rv.npy", vec(g->_rv));
            writeVec(out + "/grid_thetav.npy", vec(g->_thetav));
            writeVec(out + "/grid_cv.npy", vec(g->_cv));
            writeVec(out + "/grid_phiv.npy", vec(g->_phiv));
            writeVec(out + "/grid_sinv.npy", vec(g->_sinv));
            writeVec(out + "/grid_cosv.npy", vec(g->_cosv));
            return;
        }
        if (auto g = dynamic_cast<Sphere2DSpatialGrid*>(grid))
        {
            meta.kv("grid", "sphere2d");
            std::vector<double> rv(begin(g->_rv), end(g->_rv)), tv(begin(g->_thetav), end(g->_thetav)),
                cv(begin(g->_cv), end(g->_cv));
            writeVec(out + "/grid_rv.npy", rv);
            writeVec(out + "/grid_thetav.npy", tv);
            writeVec(out + "/grid_cv.npy", cv);
            return;
        }
        if (auto g = dynamic_cast<Sphere1DSpatialGrid*>(grid))
        {
            meta.kv("grid", "sphere1d");
            std::vector<double> rv(begin(g->radialBorderPositions()), end(g->radialBorderPositions()));
            writeVec(out + "/grid_rv.npy", rv);
            return;
        }
        if (auto g = dynamic_cast<TreeSpatialGrid*>(grid))
        {
            meta.kv("grid", "octree");
            meta.kv("eps", g->_eps);
            int numNodes = g->_nodev.size();
            std::vector<double> bounds(6 * static_cast<size_t>(numNodes));
            std::vector<int32_t> cellIndex(numNodes), childBegin(numNodes), childCount(numNodes), childIndex;
            std::vector<int32_t> nbBegin(6 * static_cast<size_t>(numNodes) + 1), nbIndex;
            for (int l = 0; l != numNodes; ++l)
            {
                TreeNode* node = g->_nodev[l];
                if (node->id() != l) throw std::runtime_error("octree node id mismatch");
                bounds[6 * l + 0] = node->xmin();
                bounds[6 * l + 1] = node->ymin();
                bounds[6 * l + 2] = node->zmin();
                bounds[6 * l + 3] = node->xmax();
                bounds[6 * l + 4] = node->ymax();
                bounds[6 * l + 5] = node->zmax();
                cellIndex[l] = g->_cellindexv[l];
                childBegin[l] = childIndex.size();
                childCount[l] = node->children().size();
                for (auto c : node->children()) childIndex.push_back(c->id());
                for (int w = 0; w != 6; ++w)
                {
                    nbBegin[6 * l + w] = nbIndex.size();
                    for (auto nb : node->_neighbors[w]) nbIndex.push_back(nb->id());
                }
            }
            nbBegin[6 * static_cast<size_t>(numNodes)] = nbIndex.size();
            writeNpy(out + "/tree_bounds.npy", bounds.data(), {static_cast<size_t>(numNodes), 6});
            writeVec(out + "/tree_cell_index.npy", cellIndex);
            writeVec(out + "/tree_child_begin.npy", childBegin);
            writeVec(out + "/tree_child_count.npy", childCount);
            writeVec(out + "/tree_child_index.npy", childIndex);
            writeVec(out + "/tree_nb_begin.npy", nbBegin);
            writeVec(out + "/tree_nb_index.npy", nbIndex);
            return;
        }
        if (auto g = dynamic_cast<AdaptiveMeshSpatialGrid*>(grid))
        {
            // the snapshot's traversal arrays (AdaptiveMeshSnapshot.cpp:172-199), depth-first from the root
            meta.kv("grid", "adaptive");
            meta.kv("eps", g->_mesh->_eps);
            Box bb = g->boundingBox();
            std::vector<double> e = {bb.xmin(), bb.ymin(), bb.zmin(), bb.xmax(), bb.ymax(), bb.zmax()};
            writeVec(out + "/grid_extent.npy", e);
            const std::vector<double>& b = g->traversalNodeBounds();
            size_t n = b.size() / 6;
            writeNpy(out + "/am_bounds.npy", b.data(), {n, 6});
            auto i32 = [](const std::vector<int>& v) { return std::vector<int32_t>(v.begin(), v.end()); };
            writeVec(out + "/am_cell_index.npy", i32(g->traversalCellIndex()));
            writeVec(out + "/am_child_begin.npy", i32(g->traversalChildBegin()));
            writeVec(out + "/am_child_count.npy", i32(g->traversalChildCount()));
            writeVec(out + "/am_child_index.npy", i32(g->traversalChildIndex()));
            return;
        }
        if (auto vg = dynamic_cast<VoronoiMeshSpatialGrid*>(grid))
        {
            meta.kv("grid", "voronoi");
            auto g = vg->_mesh;
            meta.kv("eps", g->_eps);
            int n = g->_traversalNeighborBegin.size();
            writeNpy(out + "/vor_sites.npy", g->_traversalSiteCoordinates.data(), {static_cast<size_t>(n), 3});
            std::vector<int32_t> nbBegin(n + 1);
            for (int m = 0; m != n; ++m) nbBegin[m] = g->_traversalNeighborBegin[m];
            nbBegin[n] = g->_traversalNeighborIndex.size();
            std::vector<int32_t> nbIndex(g->_traversalNeighborIndex.begin(), g->_traversalNeighborIndex.end());
            writeVec(out + "/vor_nb_begin.npy", nbBegin);
            writeVec(out + "/vor_nb_index.npy", nbIndex);
            return;
        }
        if (auto g = dynamic_cast<TetraMeshSpatialGrid*>(grid))
        {
            meta.kv("grid", "tetra");
            meta.kv("eps", g->_eps);
            int nv = g->_vertices.size();
            std::vector<double> verts(3 * static_cast<size_t>(nv));
            for (int i = 0; i != nv; ++i)
            {
                verts[3 * i] = g->_vertices[i].x();
                verts[3 * i + 1] = g->_vertices[i].y();
                verts[3 * i + 2] = g->_vertices[i].z();
            }
            int nt = g->_tetrahedra.size();
            std::vector<int32_t> tv(4 * static_cast<size_t>(nt)), ntet(4 * static_cast<size_t>(nt)),
                nface(4 * static_cast<size_t>(nt));
            std::vector<double> normals(12 * static_cast<size_t>(nt));
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
            writeNpy(out + "/tet_vertices.npy", verts.data(), {static_cast<size_t>(nv), 3});
            writeNpy(out + "/tet_tetra.npy", tv.data(), {static_cast<size_t>(nt), 4});
            writeNpy(out + "/tet_ntetra.npy", ntet.data(), {static_cast<size_t>(nt), 4});
            writeNpy(out + "/tet_nface.npy", nface.data(), {static_cast<size_t>(nt), 4});
            writeNpy(out + "/tet_normals.npy", normals.data(), {static_cast<size_t>(nt), 4, 3});
            return;
        }
        meta.kv("grid", "unsupported");
    }

    void exportMedium(MediumSystem* ms, const std::string& out, Meta& meta)
    {
        int numCells = ms->_state._numCells;
        int numMedia = ms->_numMedia;
        meta.kv("num_cells", numCells);
        meta.kv("num_media", numMedia);
        std::vector<double> dens(static_cast<size_t>(numCells) * numMedia);
        for (int m = 0; m != numCells; ++m)
            for (int h = 0; h != numMedia; ++h) dens[static_cast<size_t>(m) * numMedia + h] = ms->_state.numberDensity(m, h);
        writeNpy(out + "/medium_density.npy", dens.data(), {static_cast<size_t>(numCells), static_cast<size_t>(numMedia)});
        for (int h = 0; h != numMedia; ++h)
        {
            auto mix = dynamic_cast<const DustMix*>(ms->mix(0, h));
            if (!mix) continue;
            std::string p = out + "/mix" + std::to_string(h);
            std::vector<double> lb(begin(mix->_lambdav), end(mix->_lambdav));
            std::vector<double> se(begin(mix->_sigmaextv), end(mix->_sigmaextv));
            std::vector<double> ss(begin(mix->_sigmascav), end(mix->_sigmascav));
            std::vector<double> g(begin(mix->_asymmparv), end(mix->_asymmparv));
            writeVec(p + "_lambda_borders.npy", lb);
            writeVec(p + "_sigma_ext.npy", se);
            writeVec(p + "_sigma_sca.npy", ss);
            writeVec(p + "_asymmpar.npy", g);
        }
    }

    // writes <prefix>_borders.npy and <prefix>_ellv.npy: the border list and the phantom-bin to
    // bin-index map that DisjointWavelengthGrid::bin uses (DisjointWavelengthGrid.cpp:333-342)
    void exportWLG(const WavelengthGrid* wlg, const std::string& prefix)
    {
        auto d = dynamic_cast<const DisjointWavelengthGrid*>(wlg);
        if (!d) return;
        std::vector<double> borders(begin(d->_borderv), end(d->_borderv));
        std::vector<int32_t> ellv(d->_ellv.begin(), d->_ellv.end());
        writeVec(prefix + "_borders.npy", borders);
        writeVec(prefix + "_ellv.npy", ellv);
    }

    void exportInstruments(MonteCarloSimulation* sim, const std::string& out, Meta& meta)
    {
        int i = 0;
        for (Instrument* instr : sim->instrumentSystem()->instruments())
        {
            std::string key = "instr" + std::to_string(i);
            auto rec = instr->instrumentFluxRecorder();
            meta.kv(key + "_same_observer", instr->isSameObserverAsPreceding() ? 1 : 0);
            meta.kv(key + "_record_statistics", rec->_recordStatistics ? 1 : 0);
            meta.kv(key + "_inclination", rec->_inclination);
            meta.kv(key + "_azimuth", rec->_azimuth);
            meta.kv(key + "_roll", rec->_roll);
            if (auto d = dynamic_cast<DistantInstrument*>(instr))
            {
                Direction k = d->bfkobs(Position());
                meta.kv(key + "_kobs_x", k.x());
                meta.kv(key + "_kobs_y", k.y());
                meta.kv(key + "_kobs_z", k.z());
                meta.kv(key + "_distance", d->distance());
            }
            if (auto f = dynamic_cast<FrameInstrument*>(instr))
            {
                meta.kv(key + "_kind", "frame");
                meta.kv(key + "_costheta", f->_costheta);
                meta.kv(key + "_sintheta", f->_sintheta);
                meta.kv(key + "_cosphi", f->_cosphi);
                meta.kv(key + "_sinphi", f->_sinphi);
                meta.kv(key + "_cosomega", f->_cosomega);
                meta.kv(key + "_sinomega", f->_sinomega);
                meta.kv(key + "_nxp", f->_Nxp);
                meta.kv(key + "_nyp", f->_Nyp);
                meta.kv(key + "_xpmin", f->_xpmin);
                meta.kv(key + "_xpsiz", f->_xpsiz);
                meta.kv(key + "_ypmin", f->_ypmin);
                meta.kv(key + "_ypsiz", f->_ypsiz);
            }
            else if (dynamic_cast<SEDInstrument*>(instr))
            {
                meta.kv(key + "_kind", "sed");
            }
            else
            {
                meta.kv(key + "_kind", "other");
            }
            exportWLG(rec->_lambdagrid, out + "/" + key + "_wlg");
            ++i;
        }
        meta.kv("num_instruments", i);
    }

    // launches the first `num` primary packets of a segment of `npp` packets through
    // SourceSystem::launch and records (lambda, L*npp, x, y, z, kx, ky, kz) per packet
    void probeLaunch(MonteCarloSimulation* sim, const std::string& out, size_t npp, size_t num)
    {
        auto ss = sim->sourceSystem();
        ss->prepareForLaunch(npp);
        std::vector<double> v;
        PhotonPacket pp;
        for (size_t i = 0; i != num; ++i)
        {
            ss->launch(&pp, i);
            double x, y, z, kx, ky, kz;
            pp.position().cartesian(x, y, z);
            pp.direction().cartesian(kx, ky, kz);
            double row[8] = {pp.wavelength(), pp.luminosity() * npp, x, y, z, kx, ky, kz};
            v.insert(v.end(), row, row + 8);
        }
        writeNpy(out + "/src_probe.npy", v.data(), {num, 8});
    }

    // Per source: type, luminosity fraction and launch weight; for normalised sources the wavelength
    // bias (NormalizedSource::_xi) and the range of a log-uniform bias distribution; for black-body
    // SEDs the launch table BlackBodySED holds (_lambdav, _pv, _Pv: PlanckFunction::cdf) as
    // source<h>_sed_{lambda,p,P}.npy; for geometric sources the exponential-disk parameters
    // (ExpDiskGeometry) or the Sersic index, effective radius and the cumulative-mass table of
    // SersicFunction (_sv, _Mv: source<h>_sersic_{s,M}.npy).
    void exportSources(MonteCarloSimulation* sim, const std::string& out, Meta& meta)
    {
        auto ss = sim->sourceSystem();
        meta.kv("source_total_luminosity", ss->_L);
        meta.kv("num_sources", static_cast<int>(ss->_sources.size()));
        for (size_t h = 0; h != ss->_sources.size(); ++h)
        {
            std::string key = "source" + std::to_string(h);
            meta.kv(key + "_type", ss->_sources[h]->type());
            meta.kv(key + "_lfrac", ss->_Lv[h]);
            meta.kv(key + "_weight", ss->_Wv[h]);
            auto ns = dynamic_cast<NormalizedSource*>(ss->_sources[h]);
            if (!ns) continue;
            meta.kv(key + "_xi", ns->_xi);
            if (auto ld = dynamic_cast<LogWavelengthDistribution*>(ns->_biasDistribution))
            {
                meta.kv(key + "_bias_min", ld->range().min());
                meta.kv(key + "_bias_max", ld->range().max());
            }
            else if (auto dd = dynamic_cast<DefaultWavelengthDistribution*>(ns->_biasDistribution))
            {
                // log-uniform over the source wavelength range (DefaultWavelengthDistribution.cpp:17-39)
                meta.kv(key + "_bias_min", dd->_range.min());
                meta.kv(key + "_bias_max", dd->_range.max());
            }
            if (auto bb = dynamic_cast<BlackBodySED*>(ns->_sed))
            {
                meta.kv(key + "_sed", "blackbody");
                writeVec(out + "/" + key + "_sed_lambda.npy", std::vector<double>(begin(bb->_lambdav), end(bb->_lambdav)));
                writeVec(out + "/" + key + "_sed_p.npy", std::vector<double>(begin(bb->_pv), end(bb->_pv)));
                writeVec(out + "/" + key + "_sed_P.npy", std::vector<double>(begin(bb->_Pv), end(bb->_Pv)));
            }
            auto gs = dynamic_cast<GeometricSource*>(ss->_sources[h]);
            if (!gs) continue;
            if (auto ed = dynamic_cast<ExpDiskGeometry*>(gs->_geometry))
            {
                meta.kv(key + "_geometry", "expdisk");
                meta.kv(key + "_hR", ed->_hR);
                meta.kv(key + "_hz", ed->_hz);
                meta.kv(key + "_Rmin", ed->_Rmin);
                meta.kv(key + "_Rmax", ed->_Rmax);
                meta.kv(key + "_zmax", ed->_zmax);
            }
            else if (auto sg = dynamic_cast<SersicGeometry*>(gs->_geometry))
            {
                meta.kv(key + "_geometry", "sersic");
                meta.kv(key + "_reff", sg->_reff);
                meta.kv(key + "_n", sg->_n);
                auto sf = sg->_sersicfunction;
                writeVec(out + "/" + key + "_sersic_s.npy", std::vector<double>(begin(sf->_sv), end(sf->_sv)));
                writeVec(out + "/" + key + "_sersic_M.npy", std::vector<double>(begin(sf->_Mv), end(sf->_Mv)));
            }
        }
    }

    // the raw detector arrays of every instrument after a primary-emission segment (before
    // calibration): inst<i>_ifu.npy / inst<i>_sed.npy (total, raw W per pixel and bin, index
    // l + ell * npix) and inst<i>_wifu.npy / inst<i>_wsed.npy (sum w^k, k = 0..4, per pixel and bin,
    // FluxRecorder::recordContributions), in FP64 as FluxRecorder holds them
    void exportDetectors(MonteCarloSimulation* sim, const std::string& out, const std::string& suffix = "")
    {
        int i = 0;
        for (Instrument* instr : sim->instrumentSystem()->instruments())
        {
            auto rec = instr->instrumentFluxRecorder();
            std::string key = out + "/inst" + std::to_string(i);
            auto dumpSet = [&](const vector<Array>& arrays, const std::string& name, bool stack) {
                if (arrays.empty() || arrays[0].size() == 0) return;
                if (!stack)
                {
                    writeVec(key + name, std::vector<double>(begin(arrays[0]), end(arrays[0])));
                    return;
                }
                std::vector<double> all;
                for (const Array& a : arrays) all.insert(all.end(), begin(a), end(a));
                writeNpy(key + name, all.data(), {arrays.size(), arrays[0].size()});
            };
            if (rec->_ifu.size()) dumpSet(rec->_ifu, "_ifu" + suffix + ".npy", false);
            if (rec->_sed.size()) dumpSet(rec->_sed, "_sed" + suffix + ".npy", false);
            dumpSet(rec->_wifu, "_wifu" + suffix + ".npy", true);
            dumpSet(rec->_wsed, "_wsed" + suffix + ".npy", true);
            ++i;
        }
    }

    // zeroes every detector sum of every instrument (FluxRecorder totals, components and statistics)
    void clearDetectors(MonteCarloSimulation* sim)
    {
        for (Instrument* instr : sim->instrumentSystem()->instruments())
        {
            auto rec = instr->instrumentFluxRecorder();
            for (auto* set : {&rec->_sed, &rec->_ifu, &rec->_wsed, &rec->_wifu})
                for (Array& a : *set) a = 0.;
        }
    }

    // the primary radiation field MediumSystem::_rf1 (cells x radiation-field bins) after a run
    void exportRadiationField(MonteCarloSimulation* sim, const std::string& out)
    {
        auto ms = sim->mediumSystem();
        Table<2>& rf = ms->_rf1;
        if (rf.size() == 0) return;
        writeNpy(out + "/rf1.npy", &rf.data()[0], {rf.size(0), rf.size(1)});
    }

    // Equilibrium dust emission (DustEmission mode, after a primary segment): the tables that
    // EquilibriumDustEmissionCalculator::precalculate (EquilibriumDustEmissionCalculator.cpp:17-90)
    // built for the single dust mix, the mix's absorption cross section at each radiation-field
    // wavelength (MediumSystem::dustLuminosity, MediumSystem.cpp:2752-2762), the cell volumes, the
    // reference's own per-cell absorbed luminosity and equilibrium temperature
    // (MediumSystem::indicativeDustTemperature) for the radiation field of the run, the emission
    // spectrum MediumSystem::dustEmissionSpectrum of every 97th emitting cell, and the secondary
    // launch configuration
    void exportDustEmission(MonteCarloSimulation* sim, const std::string& out, Meta& meta)
    {
        auto ms = sim->mediumSystem();
        auto config = sim->config();
        auto mix = dynamic_cast<const DustMix*>(ms->mix(0, 0));
        if (!mix || ms->_numMedia != 1) throw std::runtime_error("dust emission export: one dust medium expected");
        const EquilibriumDustEmissionCalculator& c = mix->_calc;
        writeVec(out + "/de_rf_lambda.npy", std::vector<double>(begin(c._rflambdav), end(c._rflambdav)));
        writeVec(out + "/de_rf_width.npy", std::vector<double>(begin(c._rfdlambdav), end(c._rfdlambdav)));
        writeVec(out + "/de_rf_cmb.npy", std::vector<double>(begin(c._Bcmbv), end(c._Bcmbv)));
        writeVec(out + "/de_rf_sigma_abs.npy", std::vector<double>(begin(c._rfsigmaabsvv[0]), end(c._rfsigmaabsvv[0])));
        writeVec(out + "/de_T.npy", std::vector<double>(begin(c._Tv), end(c._Tv)));
        writeVec(out + "/de_planck_abs.npy", std::vector<double>(begin(c._planckabsvv[0]), end(c._planckabsvv[0])));
        writeVec(out + "/de_em_lambda.npy", std::vector<double>(begin(c._emlambdav), end(c._emlambdav)));
        writeVec(out + "/de_em_sigma_abs.npy", std::vector<double>(begin(c._emsigmaabsvv[0]), end(c._emsigmaabsvv[0])));
        Range er = config->dustEmissionWLG()->wavelengthRange();
        writeVec(out + "/de_em_range.npy", std::vector<double>{er.min(), er.max()});
        auto rfw = config->radiationFieldWLG();
        int nrf = rfw->numBins();
        std::vector<double> sal(nrf);
        for (int ell = 0; ell != nrf; ++ell) sal[ell] = mix->sectionAbs(rfw->wavelength(ell));
        writeVec(out + "/de_rf_sigma_abs_lum.npy", sal);
        int numCells = ms->_state._numCells;
        std::vector<double> vol(numCells), L(numCells), T(numCells);
        std::vector<int32_t> cells;
        std::vector<double> spec;
        for (int m = 0; m != numCells; ++m)
        {
            vol[m] = ms->_state.volume(m);
            L[m] = ms->dustLuminosity(m);
            T[m] = ms->indicativeDustTemperature(m);
            if (L[m] > 0 && m % 97 == 0)
            {
                Array ev = ms->dustEmissionSpectrum(m);
                cells.push_back(m);
                spec.insert(spec.end(), begin(ev), end(ev));
            }
        }
        writeVec(out + "/cell_volume.npy", vol);
        writeVec(out + "/ref_dust_L.npy", L);
        writeVec(out + "/ref_dust_T.npy", T);
        writeVec(out + "/ref_dust_spec_cells.npy", cells);
        if (!cells.empty())
            writeNpy(out + "/ref_dust_spec.npy", spec.data(), {cells.size(), spec.size() / cells.size()});
        meta.kv("secondary_spatial_bias", config->secondarySpatialBias());
        meta.kv("secondary_source_bias", config->secondarySourceBias());
        meta.kv("num_secondary_packets", static_cast<double>(config->numSecondaryPackets()));
        meta.kv("dust_emission_wavelength_bias", config->dustEmissionWavelengthBias());
        auto bd = dynamic_cast<const RangeWavelengthDistribution*>(config->dustEmissionWavelengthBiasDistribution());
        if (bd)
        {
            meta.kv("dust_emission_bias_min", bd->range().min());
            meta.kv("dust_emission_bias_max", bd->range().max());
        }
    }

    void dumpRays(MonteCarloSimulation* sim, const std::string& raysPath, int maxSeg, double lambda,
                  const std::string& out)
    {
        size_t rows, cols;
        auto rays = readNpyDoubles(raysPath, rows, cols);
        if (cols != 6) throw std::runtime_error("rays must be (N,6)");
        SpatialGrid* grid = sim->mediumSystem()->grid();
        auto gen = grid->createPathSegmentGenerator();
        std::vector<int32_t> count(rows), segm(rows * maxSeg, -2);
        std::vector<double> segds(rows * maxSeg, 0.), tau(rows, 0.);
        for (size_t r = 0; r != rows; ++r)
        {
            const double* q = &rays[6 * r];
            Position bfr(q[0], q[1], q[2]);
            Direction bfk(q[3], q[4], q[5], false);
            gen->start(bfr, bfk);
            int n = 0;
            bool overflow = false;
            while (gen->next())
            {
                if (n < maxSeg)
                {
                    segm[r * maxSeg + n] = gen->m();
                    segds[r * maxSeg + n] = gen->ds();
                }
                else
                    overflow = true;
                ++n;
            }
            count[r] = overflow ? -n : n;
            // optical depth to the domain edge through the reference's MediumSystem routine
            PhotonPacket pp;
            pp.launch(r, lambda, 1.0, bfr, bfk);
            tau[r] = sim->mediumSystem()->getExtinctionOpticalDepth(&pp, std::numeric_limits<double>::infinity());
        }
        writeVec(out + "/ray_count.npy", count);
        writeNpy(out + "/ray_m.npy", segm.data(), {rows, static_cast<size_t>(maxSeg)});
        writeNpy(out + "/ray_ds.npy", segds.data(), {rows, static_cast<size_t>(maxSeg)});
        writeVec(out + "/ray_tau.npy", tau);
    }
}

int main(int argc, char** argv)
{
    if (argc < 3)
    {
        std::fprintf(stderr, "usage: skirt_export <file.ski> <outdir> [rays.npy [maxSegments]]\n");
        return 2;
    }
    ProcessManager pm(&argc, &argv);
    System system(argc, argv);
    SimulationItemRegistry registry(BuildInfo::projectVersion(), "9");
    std::string ski = argv[1], out = argv[2];
    try
    {
        auto schema = SimulationItemRegistry::getSchemaDef();
        auto topitem = XmlHierarchyCreator::readFile(schema, ski);
        auto sim = dynamic_cast<MonteCarloSimulation*>(topitem.get());
        if (!sim) throw std::runtime_error("not a MonteCarloSimulation");
        sim->filePaths()->setOutputPrefix("export");
        sim->filePaths()->setOutputPath(out);
        sim->parallelFactory()->setMaxThreadCount(1);
        sim->log()->setLowestLevel(Log::Level::Warning);
        sim->parallelFactory()->setup();
        sim->log()->setup();
        sim->setupSimulation();
        // SKGPU_EXPORT_RUN=1: also run the primary-emission segment single-threaded
        // (MonteCarloSimulation::runPrimaryEmission, which ends with the instrument flush) and dump the
        // raw detector arrays and the primary radiation field; the run comes before the launch probe,
        // so its random stream is that of `skirt -t 1`
        const char* runEnv = std::getenv("SKGPU_EXPORT_RUN");
        bool run = runEnv && std::atoi(runEnv) != 0;
        if (run) sim->runPrimaryEmission();
        // SKGPU_PROBE_N: number of packets launched by the launch probe (default 1000)
        const char* probeEnv = std::getenv("SKGPU_PROBE_N");
        size_t probeN = probeEnv ? static_cast<size_t>(std::atoll(probeEnv)) : 1000;

        Meta meta;
        meta.kv("oligochromatic", sim->config()->oligochromatic() ? 1 : 0);
        meta.kv("force_scattering", sim->config()->forceScattering() ? 1 : 0);
        meta.kv("min_weight_reduction", sim->config()->minWeightReduction());
        meta.kv("min_scatt_events", sim->config()->minScattEvents());
        meta.kv("path_length_bias", sim->config()->pathLengthBias());
        meta.kv("has_medium", sim->config()->hasMedium() ? 1 : 0);
        if (sim->config()->hasMedium())
        {
            exportGrid(sim->mediumSystem()->grid(), out, meta);
            exportMedium(sim->mediumSystem(), out, meta);
            exportWLG(sim->config()->radiationFieldWLG(), out + "/rf_wlg");
        }
        exportInstruments(sim, out, meta);
        exportSources(sim, out, meta);
        if (run) exportDetectors(sim, out);
        if (run && sim->config()->hasMedium()) exportRadiationField(sim, out);
        // DustEmission mode: the dust emission tables and reference per-cell values for the primary
        // radiation field of the run, then the secondary-emission segment
        // (MonteCarloSimulation::runSecondaryEmission, single-threaded, continuing the random
        // stream) into cleared detectors, whose sums are the secondary segment's alone
        // (inst<i>_*_sec.npy)
        if (run && sim->config()->hasDustEmission())
        {
            exportDustEmission(sim, out, meta);
            clearDetectors(sim);
            sim->runSecondaryEmission();
            exportDetectors(sim, out, "_sec");
        }
        probeLaunch(sim, out, probeN, probeN);
        if (argc >= 4)
        {
            int maxSeg = argc >= 5 ? std::atoi(argv[4]) : 4096;
            double lambda = argc >= 6 ? std::atof(argv[5]) : 0.55e-6;
            dumpRays(sim, argv[3], maxSeg, lambda, out);
        }
        std::ofstream(out + "/meta.txt") << meta.s.str();
    }
    catch (FatalError& error)
    {
        for (const string& line : error.message()) std::fprintf(stderr, "%s\n", line.c_str());
        return 1;
    }
    catch (std::exception& e)
    {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
