// Host-side Delaunay tetrahedralisation for standalone scenes (in the drop-in case SKIRT builds its
// mesh with TetGen and hands TetraMeshSpatialGrid's tetrahedra to skgpu_upload_grid_tetra).
//
// Incremental construction (Bowyer-Watson) with exact predicates. Coordinates are quantised to an
// integer lattice of 2^20 steps per box side, on which orient3d and insphere are evaluated exactly
// in 128-bit integers. The box's 8 corners are vertices, as in TetraMeshSpatialGrid, and the
// construction starts from a split of the box into 6 tetrahedra, so the hull is the box at every
// step; points (strictly inside the box, in Morton order for short walks) are inserted by locating
// the tetrahedron that contains them (a visibility walk), removing the tetrahedra whose
// circumsphere contains them and connecting the cavity's boundary faces to the new point.
// The result follows the reference's conventions (TetraMeshSpatialGrid.cpp:495-540): positive
// orientation, face f opposite vertex f, the neighbour across each face (-1 on the hull) and its face
// index, and outward unit normals from the clockwise vertices of each face.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/skgpu.h"

namespace {

typedef __int128 i128;
constexpr int64_t QSTEPS = 1 << 20;

struct Mesh
{
    std::vector<int64_t> P;     // 3 per vertex (lattice coordinates)
    std::vector<int32_t> T;     // 4 per tetrahedron
    std::vector<int32_t> N;     // 4 per tetrahedron: neighbour across face f (opposite vertex f)
    std::vector<char> alive;
    std::vector<int32_t> freeList;

    const int64_t* p(int v) const { return &P[3 * static_cast<size_t>(v)]; }

    // sign of (b - a) . ((c - a) x (d - a))
    int orient(int a, int b, int c, int d) const
    {
        const int64_t *A = p(a), *B = p(b), *C = p(c), *D = p(d);
        i128 bx = B[0] - A[0], by = B[1] - A[1], bz = B[2] - A[2];
        i128 cx = C[0] - A[0], cy = C[1] - A[1], cz = C[2] - A[2];
        i128 dx = D[0] - A[0], dy = D[1] - A[1], dz = D[2] - A[2];
        i128 v = bx * (cy * dz - cz * dy) - by * (cx * dz - cz * dx) + bz * (cx * dy - cy * dx);
        return v > 0 ? 1 : (v < 0 ? -1 : 0);
    }

    // true if e lies strictly inside the circumsphere of the positively oriented tetrahedron t
    bool inSphere(int t, int e) const
    {
        const int64_t* E = p(e);
        i128 r[4][4];
        for (int i = 0; i < 4; ++i)
        {
            const int64_t* Q = p(T[4 * static_cast<size_t>(t) + i]);
            i128 x = Q[0] - E[0], y = Q[1] - E[1], z = Q[2] - E[2];
            r[i][0] = x;
            r[i][1] = y;
            r[i][2] = z;
            r[i][3] = x * x + y * y + z * z;
        }
        // expansion along the lifted column
        auto m3 = [&](int i, int j, int k) {
            return r[i][0] * (r[j][1] * r[k][2] - r[j][2] * r[k][1]) - r[i][1] * (r[j][0] * r[k][2] - r[j][2] * r[k][0])
                   + r[i][2] * (r[j][0] * r[k][1] - r[j][1] * r[k][0]);
        };
        i128 det = -r[0][3] * m3(1, 2, 3) + r[1][3] * m3(0, 2, 3) - r[2][3] * m3(0, 1, 3) + r[3][3] * m3(0, 1, 2);
        return det < 0;  // negative for a point inside, with the orientation above
    }

    int newTet(int a, int b, int c, int d)
    {
        int t;
        if (!freeList.empty())
        {
            t = freeList.back();
            freeList.pop_back();
        }
        else
        {
            t = static_cast<int>(alive.size());
            T.resize(T.size() + 4);
            N.resize(N.size() + 4);
            alive.push_back(0);
        }
        int32_t* q = &T[4 * static_cast<size_t>(t)];
        q[0] = a; q[1] = b; q[2] = c; q[3] = d;
        for (int f = 0; f < 4; ++f) N[4 * static_cast<size_t>(t) + f] = -1;
        alive[t] = 1;
        return t;
    }

    // vertices of face f of tetrahedron t ordered so that orient(a, b, c, opposite vertex) > 0
    // (an even permutation of the tetrahedron's vertices)
    void faceVerts(int t, int f, int& a, int& b, int& c) const
    {
        static const int idx[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};
        const int32_t* q = &T[4 * static_cast<size_t>(t)];
        a = q[idx[f][0]];
        b = q[idx[f][1]];
        c = q[idx[f][2]];
    }
};

}  // namespace

struct skgpu_tetra
{
    std::vector<double> vertices;   // 3 per vertex (the points, then the 8 corners)
    std::vector<int32_t> tetra;     // 4 per tetrahedron
    std::vector<double> normals;    // 12 per tetrahedron
    std::vector<int32_t> ntetra;    // 4 per tetrahedron
    std::vector<int32_t> nface;     // 4 per tetrahedron
};

extern "C" {

int skgpu_tetra_build(const double* points, int32_t n, const double* extent, int32_t threads, skgpu_tetra** out)
{
    (void)threads;
    if (!out) return SKGPU_ERR_ARG;
    *out = nullptr;
    if (!points || !extent || n < 1) return SKGPU_ERR_ARG;
    const double* e = extent;
    if (!(e[3] > e[0] && e[4] > e[1] && e[5] > e[2])) return SKGPU_ERR_ARG;
    Mesh m;
    // lattice coordinates. As TetraMeshSpatialGrid::removeInvalid (TetraMeshSpatialGrid.cpp:324-363)
    // drops vertices outside the domain and vertices too near another one, points that quantise onto
    // or outside the box surface, or onto the lattice point of an earlier point, are left out.
    std::vector<int32_t> keep;
    keep.reserve(n);
    std::unordered_set<uint64_t> used;
    used.reserve(2 * static_cast<size_t>(n));
    m.P.reserve(3 * (static_cast<size_t>(n) + 8));
    for (int c = 0; c < 8; ++c)
    {
        m.P.push_back((c & 1) ? QSTEPS : 0);
        m.P.push_back((c & 2) ? QSTEPS : 0);
        m.P.push_back((c & 4) ? QSTEPS : 0);
    }
    for (int i = 0; i < n; ++i)
    {
        int64_t q[3];
        for (int a = 0; a < 3; ++a)
        {
            double x = points[3 * static_cast<size_t>(i) + a];
            if (!std::isfinite(x)) return SKGPU_ERR_ARG;
            double u = (x - e[a]) / (e[3 + a] - e[a]) * QSTEPS;
            q[a] = u > 0 && u < QSTEPS ? static_cast<int64_t>(std::llround(u)) : 0;
        }
        bool inside = true;
        for (int a = 0; a < 3; ++a) inside = inside && q[a] > 0 && q[a] < QSTEPS;
        if (!inside) continue;
        uint64_t code = (static_cast<uint64_t>(q[0]) << 40) | (static_cast<uint64_t>(q[1]) << 20) | static_cast<uint64_t>(q[2]);
        if (!used.insert(code).second) continue;
        m.P.insert(m.P.end(), q, q + 3);
        keep.push_back(i);
    }
    n = static_cast<int32_t>(keep.size());
    if (n < 1) return SKGPU_ERR_ARG;
    int nv = n + 8;
    // insertion order: Morton order of the lattice coordinates (short walks)
    std::vector<std::pair<uint64_t, int>> order(n);
    for (int i = 0; i < n; ++i)
    {
        const int64_t* q = m.p(8 + i);
        uint64_t code = 0;
        for (int bit = 19; bit >= 0; --bit)
            for (int a = 0; a < 3; ++a) code = (code << 1) | ((q[a] >> bit) & 1);
        order[i] = {code, 8 + i};
    }
    std::sort(order.begin(), order.end());
    // 6 tetrahedra around the main diagonal 0-7 of the box
    const int six[6][4] = {{0, 1, 3, 7}, {0, 1, 7, 5}, {0, 4, 5, 7}, {0, 4, 7, 6}, {0, 2, 6, 7}, {0, 2, 7, 3}};
    for (auto& q : six)
    {
        int t = m.newTet(q[0], q[1], q[2], q[3]);
        if (m.orient(q[0], q[1], q[2], q[3]) < 0) std::swap(m.T[4 * static_cast<size_t>(t) + 2], m.T[4 * static_cast<size_t>(t) + 3]);
    }
    // neighbours of the initial split (match faces by their sorted vertex triple)
    auto linkAll = [&]() {
        std::unordered_map<uint64_t, int> open;
        for (int t = 0; t < static_cast<int>(m.alive.size()); ++t)
            for (int f = 0; f < 4; ++f)
            {
                int a, b, c;
                m.faceVerts(t, f, a, b, c);
                int v[3] = {a, b, c};
                std::sort(v, v + 3);
                uint64_t k = (static_cast<uint64_t>(v[0]) * nv + v[1]) * nv + v[2];
                auto it = open.find(k);
                if (it == open.end())
                    open.emplace(k, 4 * t + f);
                else
                {
                    int t2 = it->second / 4, f2 = it->second % 4;
                    m.N[4 * static_cast<size_t>(t) + f] = t2;
                    m.N[4 * static_cast<size_t>(t2) + f2] = t;
                    open.erase(it);
                }
            }
    };
    linkAll();
    int last = 0;
    std::vector<int> cavity, stack, mark(0);
    std::vector<std::pair<int, int>> boundary;  // (cavity tet, face)
    std::unordered_map<uint64_t, int> edgeMap;
    uint32_t rng = 12345u;
    for (const auto& od : order)
    {
        int v = od.second;
        // visibility walk to the tetrahedron containing v
        int t = last;
        for (int steps = 0;; ++steps)
        {
            if (steps > 4 * nv + 100) return SKGPU_ERR_DEVICE;
            int start = static_cast<int>((rng = rng * 1664525u + 1013904223u) >> 30);
            int move = -1;
            for (int k = 0; k < 4; ++k)
            {
                int f = (start + k) & 3;
                int a, b, c;
                m.faceVerts(t, f, a, b, c);
                if (m.orient(a, b, c, v) < 0)
                {
                    move = f;
                    break;
                }
            }
            if (move < 0) break;
            int nt = m.N[4 * static_cast<size_t>(t) + move];
            if (nt < 0) return SKGPU_ERR_DEVICE;  // cannot leave the box: the point is inside
            t = nt;
        }
        // cavity: tetrahedra whose circumsphere holds v, grown from the containing one
        if (mark.size() < m.alive.size()) mark.resize(m.alive.size() + 1024, 0);
        cavity.clear();
        stack.assign(1, t);
        mark[t] = 1;
        while (!stack.empty())
        {
            int c = stack.back();
            stack.pop_back();
            cavity.push_back(c);
            for (int f = 0; f < 4; ++f)
            {
                int nt = m.N[4 * static_cast<size_t>(c) + f];
                if (nt >= 0 && !mark[nt] && m.inSphere(nt, v))
                {
                    mark[nt] = 1;
                    stack.push_back(nt);
                }
            }
        }
        boundary.clear();
        for (int c : cavity)
            for (int f = 0; f < 4; ++f)
            {
                int nt = m.N[4 * static_cast<size_t>(c) + f];
                if (nt < 0 || !mark[nt]) boundary.push_back({c, f});
            }
        // new tetrahedra: each boundary face (a, b, c) with v, which lies on the positive side of the
        // face like the cavity tetrahedron's opposite vertex: (v, a, c, b) is positively oriented
        std::vector<int> created;
        created.reserve(boundary.size());
        struct Face { int a, b, c, out; };
        std::vector<Face> faces;
        faces.reserve(boundary.size());
        for (auto& bf : boundary)
        {
            int a, b, c;
            m.faceVerts(bf.first, bf.second, a, b, c);
            faces.push_back({a, b, c, m.N[4 * static_cast<size_t>(bf.first) + bf.second]});
        }
        for (int c : cavity)
        {
            mark[c] = 0;
            m.alive[c] = 0;
            m.freeList.push_back(c);
        }
        edgeMap.clear();
        for (const Face& fc : faces)
        {
            // tetrahedron (v, a, c, b): face 0 (opposite v) is the boundary face
            int nt = m.newTet(v, fc.a, fc.c, fc.b);
            if (m.orient(v, fc.a, fc.c, fc.b) <= 0) return SKGPU_ERR_DEVICE;  // cavity not star-shaped
            if (mark.size() < m.alive.size()) mark.resize(m.alive.size() + 1024, 0);
            m.N[4 * static_cast<size_t>(nt)] = fc.out;
            if (fc.out >= 0)
            {
                // point the outside tetrahedron's face back at the new one
                for (int f = 0; f < 4; ++f)
                {
                    int a, b, c;
                    m.faceVerts(fc.out, f, a, b, c);
                    int x[3] = {a, b, c}, y[3] = {fc.a, fc.b, fc.c};
                    std::sort(x, x + 3);
                    std::sort(y, y + 3);
                    if (x[0] == y[0] && x[1] == y[1] && x[2] == y[2])
                    {
                        m.N[4 * static_cast<size_t>(fc.out) + f] = nt;
                        break;
                    }
                }
            }
            // faces 1..3 contain v and one edge of (a, b, c): match them through the edge
            for (int f = 1; f < 4; ++f)
            {
                int fv[3];
                m.faceVerts(nt, f, fv[0], fv[1], fv[2]);
                int ev[2], ne = 0;
                for (int x : fv)
                    if (x != v && ne < 2) ev[ne++] = x;
                int lo = std::min(ev[0], ev[1]), hi = std::max(ev[0], ev[1]);
                uint64_t k = static_cast<uint64_t>(lo) * nv + hi;
                auto it = edgeMap.find(k);
                if (it == edgeMap.end())
                    edgeMap.emplace(k, 4 * nt + f);
                else
                {
                    int t2 = it->second / 4, f2 = it->second % 4;
                    m.N[4 * static_cast<size_t>(nt) + f] = t2;
                    m.N[4 * static_cast<size_t>(t2) + f2] = nt;
                    edgeMap.erase(it);
                }
            }
            created.push_back(nt);
        }
        last = created.empty() ? 0 : created.front();
    }
    // export in the reference's form, compacting the live tetrahedra
    skgpu_tetra* r = new skgpu_tetra();
    r->vertices.resize(3 * static_cast<size_t>(nv));
    for (int v = 0; v < nv; ++v)
        for (int a = 0; a < 3; ++a)
        {
            // vertices n..n+7 are the corners (lattice ids 0..7); the kept points keep their order
            int lat = v < n ? 8 + v : v - n;
            r->vertices[3 * static_cast<size_t>(v) + a] = e[a] + (e[3 + a] - e[a]) * static_cast<double>(m.p(lat)[a]) / QSTEPS;
        }
    auto outId = [&](int lat) { return lat < 8 ? n + lat : lat - 8; };
    std::vector<int32_t> newIndex(m.alive.size(), -1);
    int nt = 0;
    for (size_t t = 0; t < m.alive.size(); ++t)
        if (m.alive[t]) newIndex[t] = nt++;
    r->tetra.resize(4 * static_cast<size_t>(nt));
    r->ntetra.resize(4 * static_cast<size_t>(nt));
    r->nface.resize(4 * static_cast<size_t>(nt));
    r->normals.resize(12 * static_cast<size_t>(nt));
    for (size_t t = 0; t < m.alive.size(); ++t)
    {
        if (!m.alive[t]) continue;
        int k = newIndex[t];
        const int32_t* q = &m.T[4 * t];
        for (int f = 0; f < 4; ++f) r->tetra[4 * static_cast<size_t>(k) + f] = outId(q[f]);
    }
    for (size_t t = 0; t < m.alive.size(); ++t)
    {
        if (!m.alive[t]) continue;
        int k = newIndex[t];
        for (int f = 0; f < 4; ++f)
        {
            int nb = m.N[4 * t + f];
            r->ntetra[4 * static_cast<size_t>(k) + f] = nb >= 0 ? newIndex[nb] : -1;
            int nf = -1;
            if (nb >= 0)
                for (int g = 0; g < 4; ++g)
                    if (m.N[4 * static_cast<size_t>(nb) + g] == static_cast<int>(t)) nf = g;
            if (nb >= 0 && nf < 0)
            {
                delete r;
                return SKGPU_ERR_DEVICE;
            }
            r->nface[4 * static_cast<size_t>(k) + f] = nf;
            // outward unit normal from the clockwise vertices of face f (TetraMeshSpatialGrid.cpp:44-50, 525-531)
            int cv[3] = {(f + 3) % 4, (f + 2) % 4, (f + 1) % 4};
            if (f % 2 == 0) std::swap(cv[0], cv[2]);
            const double* A = &r->vertices[3 * static_cast<size_t>(r->tetra[4 * static_cast<size_t>(k) + cv[0]])];
            const double* B = &r->vertices[3 * static_cast<size_t>(r->tetra[4 * static_cast<size_t>(k) + cv[1]])];
            const double* Cc = &r->vertices[3 * static_cast<size_t>(r->tetra[4 * static_cast<size_t>(k) + cv[2]])];
            double u[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]}, w[3] = {Cc[0] - A[0], Cc[1] - A[1], Cc[2] - A[2]};
            double nn[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
            double len = std::sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
            for (int j = 0; j < 3; ++j) r->normals[12 * static_cast<size_t>(k) + 3 * f + j] = len > 0 ? nn[j] / len : 0.0;
        }
    }
    *out = r;
    return SKGPU_OK;
}

int skgpu_tetra_sizes(const skgpu_tetra* t, int32_t* num_vertices, int32_t* num_tetra)
{
    if (!t || !num_vertices || !num_tetra) return SKGPU_ERR_ARG;
    *num_vertices = static_cast<int32_t>(t->vertices.size() / 3);
    *num_tetra = static_cast<int32_t>(t->tetra.size() / 4);
    return SKGPU_OK;
}

int skgpu_tetra_export(const skgpu_tetra* t, double* vertices, int32_t* tetra, double* face_normals, int32_t* face_ntetra,
                       int32_t* face_nface)
{
    if (!t) return SKGPU_ERR_ARG;
    if (vertices) std::copy(t->vertices.begin(), t->vertices.end(), vertices);
    if (tetra) std::copy(t->tetra.begin(), t->tetra.end(), tetra);
    if (face_normals) std::copy(t->normals.begin(), t->normals.end(), face_normals);
    if (face_ntetra) std::copy(t->ntetra.begin(), t->ntetra.end(), face_ntetra);
    if (face_nface) std::copy(t->nface.begin(), t->nface.end(), face_nface);
    return SKGPU_OK;
}

void skgpu_tetra_free(skgpu_tetra* t) { delete t; }

}  // extern "C"
