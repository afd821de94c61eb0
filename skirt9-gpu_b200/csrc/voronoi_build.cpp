// Host-side Voronoi neighbour construction for standalone scenes (in the drop-in case SKIRT builds
// its mesh with voro++ and hands VoronoiMeshSnapshot's neighbour lists to skgpu_upload_grid_voronoi).
//
// Each cell starts as the domain box and is clipped by the bisector planes of its nearest sites,
// taken shell by shell from a uniform site grid, until no remaining site can cut it (a site at
// distance d cuts only if d / 2 is below the largest distance from the site to a cell vertex). The
// cell is kept as a simple polytope: every vertex carries the three planes that meet there, two
// vertices share an edge when they share two planes, and a cut replaces the vertices outside the
// plane by the intersections of the new plane with the cut edges. The planes left with vertices are
// the cell's faces; their owners are the neighbours, with the domain walls numbered -1..-6 (xmin,
// xmax, ymin, ymax, zmin, zmax) as in VoronoiMeshSnapshot (VoronoiMeshSnapshot.cpp:725-740).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/skgpu.h"

namespace {

struct Plane
{
    double n[3];  // outward normal (not normalised)
    double c;     // the cell is n . x <= c
    int owner;    // neighbour site, or -1..-6 for a domain wall
};

struct Vertex
{
    double x[3];
    int p[3];  // indices of the three planes through the vertex
};

struct Cell
{
    std::vector<Plane> planes;
    std::vector<Vertex> verts;

    void box(const double* e)
    {
        planes.clear();
        verts.clear();
        planes.push_back({{-1, 0, 0}, -e[0], -1});
        planes.push_back({{1, 0, 0}, e[3], -2});
        planes.push_back({{0, -1, 0}, -e[1], -3});
        planes.push_back({{0, 1, 0}, e[4], -4});
        planes.push_back({{0, 0, -1}, -e[2], -5});
        planes.push_back({{0, 0, 1}, e[5], -6});
        for (int i = 0; i < 8; ++i)
        {
            Vertex v;
            v.x[0] = (i & 1) ? e[3] : e[0];
            v.x[1] = (i & 2) ? e[4] : e[1];
            v.x[2] = (i & 4) ? e[5] : e[2];
            v.p[0] = (i & 1) ? 1 : 0;
            v.p[1] = (i & 2) ? 3 : 2;
            v.p[2] = (i & 4) ? 5 : 4;
            verts.push_back(v);
        }
    }

    double maxDist2(const double* s) const
    {
        double m = 0;
        for (const Vertex& v : verts)
        {
            double dx = v.x[0] - s[0], dy = v.x[1] - s[1], dz = v.x[2] - s[2];
            m = std::max(m, dx * dx + dy * dy + dz * dz);
        }
        return m;
    }

    static int shared(const Vertex& a, const Vertex& b, int* out)
    {
        int k = 0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                if (a.p[i] == b.p[j] && k < 2) out[k++] = a.p[i];
        return k;
    }

    // clips by n . x <= c; returns false if the cell vanished (cannot happen for a bisector of the
    // cell's own site, which stays inside)
    bool cut(const Plane& pl)
    {
        const double tol = 1e-12 * (std::fabs(pl.c) + 1.0);
        std::vector<double> d(verts.size());
        bool any = false;
        for (size_t i = 0; i < verts.size(); ++i)
        {
            const double* x = verts[i].x;
            d[i] = pl.n[0] * x[0] + pl.n[1] * x[1] + pl.n[2] * x[2] - pl.c;
            if (d[i] > tol) any = true;
        }
        if (!any) return true;
        int id = static_cast<int>(planes.size());
        planes.push_back(pl);
        std::vector<Vertex> out;
        out.reserve(verts.size() + 8);
        for (size_t i = 0; i < verts.size(); ++i)
            if (d[i] <= tol) out.push_back(verts[i]);
        // new vertices on the edges from an inside vertex to an outside vertex
        for (size_t i = 0; i < verts.size(); ++i)
        {
            if (d[i] > tol) continue;
            for (size_t j = 0; j < verts.size(); ++j)
            {
                if (d[j] <= tol) continue;
                int sp[2];
                if (shared(verts[i], verts[j], sp) != 2) continue;
                double t = d[i] / (d[i] - d[j]);
                Vertex v;
                for (int a = 0; a < 3; ++a) v.x[a] = verts[i].x[a] + t * (verts[j].x[a] - verts[i].x[a]);
                v.p[0] = sp[0];
                v.p[1] = sp[1];
                v.p[2] = id;
                out.push_back(v);
            }
        }
        verts.swap(out);
        return verts.size() >= 4;
    }

    // owners of the planes that still carry at least three vertices
    void faces(std::vector<int>& nb) const
    {
        std::vector<int> count(planes.size(), 0);
        for (const Vertex& v : verts)
            for (int i = 0; i < 3; ++i) count[v.p[i]]++;
        for (size_t i = 0; i < planes.size(); ++i)
            if (count[i] >= 3) nb.push_back(planes[i].owner);
    }
};
// Builds the Voronoi cell of every site (clipped by clipExt) on `threads` threads and hands each
// finished cell to visit(site, cell, worker). The site-search grid spans searchExt. Returns false
// if a cell degenerated.
template<typename Visit>
bool buildCells(const double* sites, int n, const double* searchExt, const double* clipExt, int threads, Visit visit)
{
    const double* e = searchExt;
    int g = std::max(1, static_cast<int>(std::cbrt(n / 2.0)));
    double sz[3] = {(e[3] - e[0]) / g, (e[4] - e[1]) / g, (e[5] - e[2]) / g};
    auto blockOf = [&](const double* p, int a) {
        int b = static_cast<int>((p[a] - e[a]) / sz[a]);
        return std::min(g - 1, std::max(0, b));
    };
    std::vector<int32_t> blkBegin(static_cast<size_t>(g) * g * g + 1, 0), blkSites(n);
    for (int i = 0; i < n; ++i)
    {
        const double* p = sites + 3 * static_cast<size_t>(i);
        blkBegin[1 + (static_cast<size_t>(blockOf(p, 0)) * g + blockOf(p, 1)) * g + blockOf(p, 2)]++;
    }
    for (size_t b = 0; b + 1 < blkBegin.size(); ++b) blkBegin[b + 1] += blkBegin[b];
    {
        std::vector<int32_t> fill(blkBegin.begin(), blkBegin.end() - 1);
        for (int i = 0; i < n; ++i)
        {
            const double* p = sites + 3 * static_cast<size_t>(i);
            blkSites[fill[(static_cast<size_t>(blockOf(p, 0)) * g + blockOf(p, 1)) * g + blockOf(p, 2)]++] = i;
        }
    }
    double minSz = std::min(sz[0], std::min(sz[1], sz[2]));
    std::atomic<int> next{0};
    std::atomic<bool> bad{false};
    auto work = [&](int worker) {
        Cell cell;
        std::vector<std::pair<double, int>> cand;
        for (;;)
        {
            int i = next.fetch_add(1);
            if (i >= n || bad) break;
            const double* s = sites + 3 * static_cast<size_t>(i);
            cell.box(clipExt);
            int bi[3] = {blockOf(s, 0), blockOf(s, 1), blockOf(s, 2)};
            // shells of blocks at Chebyshev distance r; sites in shell r are at least (r-1) * minSz away
            for (int r = 0; r <= g; ++r)
            {
                double reach = std::max(0, r - 1) * minSz;
                if (r > 0 && reach * reach > 4.0 * cell.maxDist2(s)) break;
                cand.clear();
                for (int a = bi[0] - r; a <= bi[0] + r; ++a)
                    for (int b = bi[1] - r; b <= bi[1] + r; ++b)
                        for (int c = bi[2] - r; c <= bi[2] + r; ++c)
                        {
                            if (a < 0 || b < 0 || c < 0 || a >= g || b >= g || c >= g) continue;
                            if (std::max(std::abs(a - bi[0]), std::max(std::abs(b - bi[1]), std::abs(c - bi[2]))) != r)
                                continue;
                            size_t blk = (static_cast<size_t>(a) * g + b) * g + c;
                            for (int k = blkBegin[blk]; k < blkBegin[blk + 1]; ++k)
                            {
                                int j = blkSites[k];
                                if (j == i) continue;
                                const double* q = sites + 3 * static_cast<size_t>(j);
                                double dx = q[0] - s[0], dy = q[1] - s[1], dz = q[2] - s[2];
                                cand.push_back({dx * dx + dy * dy + dz * dz, j});
                            }
                        }
                std::sort(cand.begin(), cand.end());
                for (const auto& cj : cand)
                {
                    if (cj.first > 4.0 * cell.maxDist2(s)) break;
                    if (cj.first == 0.0) continue;  // coincident sites share no face
                    const double* q = sites + 3 * static_cast<size_t>(cj.second);
                    Plane pl;
                    for (int a = 0; a < 3; ++a) pl.n[a] = q[a] - s[a];
                    pl.c = 0.5 * (pl.n[0] * (q[0] + s[0]) + pl.n[1] * (q[1] + s[1]) + pl.n[2] * (q[2] + s[2]));
                    pl.owner = cj.second;
                    if (!cell.cut(pl))
                    {
                        bad = true;
                        break;
                    }
                }
                if (bad) break;
            }
            if (!bad) visit(i, cell, worker);
        }
    };
    int T = threads > 0 ? threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    T = std::min(T, 64);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) pool.emplace_back(work, t);
    for (std::thread& t : pool) t.join();
    return !bad;
}

}  // namespace

struct skgpu_voronoi
{
    int n = 0;
    std::vector<int32_t> begin;  // n + 1
    std::vector<int32_t> index;
};

extern "C" {

int skgpu_voronoi_build(const double* sites, int32_t n, const double* extent, int32_t threads, skgpu_voronoi** out)
{
    if (!out) return SKGPU_ERR_ARG;
    *out = nullptr;
    if (!sites || !extent || n < 1) return SKGPU_ERR_ARG;
    const double* e = extent;
    if (!(e[3] > e[0] && e[4] > e[1] && e[5] > e[2])) return SKGPU_ERR_ARG;
    for (int64_t i = 0; i < 3 * static_cast<int64_t>(n); ++i)
        if (!std::isfinite(sites[i])) return SKGPU_ERR_ARG;
    std::vector<std::vector<int32_t>> nbs(n);
    bool ok = buildCells(sites, n, e, e, threads, [&](int i, const Cell& cell, int) {
        std::vector<int> f;
        cell.faces(f);
        nbs[i].assign(f.begin(), f.end());
    });
    if (!ok) return SKGPU_ERR_DEVICE;
    skgpu_voronoi* v = new skgpu_voronoi();
    v->n = n;
    v->begin.resize(static_cast<size_t>(n) + 1, 0);
    for (int i = 0; i < n; ++i) v->begin[i + 1] = v->begin[i] + static_cast<int32_t>(nbs[i].size());
    v->index.reserve(v->begin[n]);
    for (int i = 0; i < n; ++i) v->index.insert(v->index.end(), nbs[i].begin(), nbs[i].end());
    *out = v;
    return SKGPU_OK;
}

int skgpu_voronoi_sizes(const skgpu_voronoi* v, int64_t* num_nb)
{
    if (!v || !num_nb) return SKGPU_ERR_ARG;
    *num_nb = static_cast<int64_t>(v->index.size());
    return SKGPU_OK;
}

int skgpu_voronoi_export(const skgpu_voronoi* v, int32_t* nb_begin, int32_t* nb_index)
{
    if (!v) return SKGPU_ERR_ARG;
    if (nb_begin) std::copy(v->begin.begin(), v->begin.end(), nb_begin);
    if (nb_index) std::copy(v->index.begin(), v->index.end(), nb_index);
    return SKGPU_OK;
}

void skgpu_voronoi_free(skgpu_voronoi* v) { delete v; }

}  // extern "C"

