/* skoracle.c -- TEST INFRASTRUCTURE ONLY: CPU oracle of the photon-packet life cycle.
 *
 * A sequential restatement of the reference algorithm, written from the reference CPU classes
 * (paths relative to the SKIRT9-GPU source tree):
 *   path generators   CartesianSpatialGrid.cpp:77-155, TreeSpatialGrid.cpp:143-228 (TreeNode.cpp:66-112,
 *                     OctTreeNode.cpp:37-42), VoronoiMeshSnapshot.cpp:1037-1222,
 *                     TetraMeshSpatialGrid.cpp:87-138, 615-622, 688-831, PathSegmentGenerator.cpp:11-112
 *   path + tau        SpatialGridPath.cpp:37-45, 161-203; MediumSystem.cpp:1785-1846, 2005-2150, 2328-2443
 *   life cycle        MonteCarloSimulation.cpp:614-715, 888-957, 1492-1546, 1996-2092
 *   scattering        MediumSystem.cpp:793-837, 1545-1655; DustMix.cpp:395-546
 *   detection         FluxRecorder.cpp:372-538, 1355-1409; FrameInstrument.cpp:117-136
 *   sources           SourceSystem.cpp (launch), NormalizedSource.cpp:73-110, SepAxGeometry.cpp:11-19,
 *                     ExpDiskGeometry.cpp:46-69, SpheGeometry.cpp:25-32, Random.cpp:105-207
 * Arithmetic is plain IEEE double with separate roundings (compiled without FMA contraction), as
 * in the reference's x86-64 build. Random numbers are Philox4x32-10 streams keyed by history index
 * instead of the reference's per-thread mt19937_64; histories draw in the reference's order.
 * Mesh cell searches are brute force (nearest site; first containing tetrahedron by index).
 */
#define _GNU_SOURCE
#include "skoracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_E
#define M_E 2.7182818284590452354
#endif

/* ------------------------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon et al. 2011)                                                          */
/* ------------------------------------------------------------------------------------------- */

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r)
    {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

typedef struct
{
    uint32_t key[2], hist[2], ctr;
    int hasSpare;
    double spare;
} Rng;

static double u01(uint32_t hi, uint32_t lo)
{
    uint64_t j = ((((uint64_t)hi) << 32) | lo) >> 12;
    return ((double)j + 0.5) * 2.220446049250313080847e-16;
}

static void rng_start(Rng* r, uint64_t seed, uint64_t hist)
{
    r->key[0] = (uint32_t)seed;
    r->key[1] = (uint32_t)(seed >> 32);
    r->hist[0] = (uint32_t)hist;
    r->hist[1] = (uint32_t)(hist >> 32);
    r->ctr = 0;
    r->hasSpare = 0;
}

static double uniform(Rng* r)
{
    if (r->hasSpare)
    {
        r->hasSpare = 0;
        return r->spare;
    }
    uint32_t c[4] = {r->ctr++, 0u, r->hist[0], r->hist[1]}, o[4];
    or_philox4x32_10(c, r->key, o);
    r->spare = u01(o[2], o[3]);
    r->hasSpare = 1;
    return u01(o[0], o[1]);
}

/* ------------------------------------------------------------------------------------------- */
/* context                                                                                     */
/* ------------------------------------------------------------------------------------------- */

typedef struct
{
    int kind;
    double ext[6];
    double eps;
    int numCells;
    /* cartesian */
    double *xb, *yb, *zb;
    int nx, ny, nz;
    /* octree (and the adaptive mesh: one neighbour per leaf wall) */
    double* tb;
    int *tcell, *tchild, *tnbb, *tnb;
    int tnodes;
    /* adaptive mesh: subdivision nx, ny, nz per node (0 for leaves), children CSR */
    int *adiv, *acb, *ach;
    /* voronoi */
    double* vs;
    double* vbox; /* per cell enclosing box (secondary launch) */
    int *vnbb, *vnb;
    int vn;
    /* tetra */
    double *tev, *ten, *tebox;
    int *tet, *tent, *tenf;
    int ten_n;
    /* sphere1d */
    double* srv;
    int snr;
    /* cylinder2d */
    double *crv, *czv;
    int cnr, cnz;
    /* sphere2d */
    double *s2r, *s2t, *s2c;
    int s2nr, s2nt;
    /* sphere3d */
    double *s3r, *s3t, *s3c, *s3p, *s3s, *s3k;
    int s3nr, s3nt, s3np;
    double s3eps;
    /* cylinder3d */
    double *c3r, *c3p, *c3s, *c3k, *c3z;
    int c3nr, c3np, c3nz, c3hole;
    double c3eps;
} Grid;

typedef struct
{
    skgpu_instrument d;
    double *ifu, *sed, *comp, *stats;
    size_t n;
    int levels;                     /* scattering-level planes after the 3 component planes */
    int nband;                      /* > 0: band wavelength grid */
    int* bandBeg;                   /* nband + 1 table offsets */
    double *bandLam, *bandTr, *bandW;
    double zfac; /* 1 + observer-frame redshift */
    double apR2; /* SED aperture radius squared (0: none) */
} Instr;

struct or_ctx
{
    char err[256];
    Grid g;
    int hasGrid;
    double* dens;
    int numCells;
    double *mixLb, *mixExt, *mixSca, *mixG;
    int nmix;
    double* rfB;
    int *rfEll, nrf, rfNb;
    double* rf;
    size_t rfLen;
    skgpu_source* src;
    int nsrc;
    double *tabL, *tabA, *tabB, *radR, *radP;
    Instr* instr;
    int ninstr;
    double* wlgB;
    int* wlgEll;
    skgpu_options opt;
    skgpu_counters cnt;
    int errFlag;
    /* secondary (dust) emission: tables, per-cell results, launch tables */
    int deNrf, deNT, deNem, deCells;
    double *deRfSig, *deRfW, *deRfCmb, *deRfSigL, *deT, *dePlanck, *deEmL, *deEmSig, *deVol;
    double deEmRange[2];
    int secCells, secNpts;
    double *secL, *secT, *secXv, *secPv, *secCv, *secLv, *secWv;
    uint64_t* secIv;
    int* secCellNode; /* octree: leaf node of each cell */
    uint64_t secPackets;
    double secLpk, secXi, secBmin, secBmax, secLogMin, secLogWidth;
    int secRun; /* set while or_run_secondary runs */
};

static int fail(or_ctx* c, int code, const char* msg)
{
    if (c) snprintf(c->err, sizeof c->err, "%s", msg);
    return code;
}

static void* dup(const void* p, size_t bytes)
{
    if (!p || !bytes) return NULL;
    void* q = malloc(bytes);
    memcpy(q, p, bytes);
    return q;
}

static void free_grid(Grid* g)
{
    free(g->xb); free(g->yb); free(g->zb);
    free(g->tb); free(g->tcell); free(g->tchild); free(g->tnbb); free(g->tnb);
    free(g->adiv); free(g->acb); free(g->ach);
    free(g->vs); free(g->vbox); free(g->vnbb); free(g->vnb);
    free(g->tev); free(g->ten); free(g->tebox); free(g->tet); free(g->tent); free(g->tenf);
    free(g->srv);
    free(g->crv); free(g->czv);
    free(g->s2r); free(g->s2t); free(g->s2c);
    free(g->s3r); free(g->s3t); free(g->s3c); free(g->s3p); free(g->s3s); free(g->s3k);
    free(g->c3r); free(g->c3p); free(g->c3s); free(g->c3k); free(g->c3z);
    memset(g, 0, sizeof *g);
}

static void free_instruments(or_ctx* c)
{
    for (int i = 0; i < c->ninstr; ++i)
    {
        free(c->instr[i].ifu); free(c->instr[i].sed); free(c->instr[i].comp); free(c->instr[i].stats);
        free(c->instr[i].bandBeg); free(c->instr[i].bandLam); free(c->instr[i].bandTr); free(c->instr[i].bandW);
    }
    free(c->instr);
    c->instr = NULL;
    c->ninstr = 0;
    free(c->wlgB); free(c->wlgEll);
    c->wlgB = NULL; c->wlgEll = NULL;
}

int or_create(int device, or_ctx** out)
{
    (void)device;
    or_ctx* c = (or_ctx*)calloc(1, sizeof(or_ctx));
    c->opt.force_scattering = 1;
    c->opt.min_weight_reduction = 1e4;
    c->opt.path_length_bias = 0.5;
    c->opt.peel_off = 1;
    *out = c;
    return SKGPU_OK;
}

void or_destroy(or_ctx* c)
{
    if (!c) return;
    free_grid(&c->g);
    free_instruments(c);
    free(c->dens); free(c->mixLb); free(c->mixExt); free(c->mixSca); free(c->mixG);
    free(c->rfB); free(c->rfEll); free(c->rf);
    free(c->src); free(c->tabL); free(c->tabA); free(c->tabB); free(c->radR); free(c->radP);
    free(c->deRfSig); free(c->deRfW); free(c->deRfCmb); free(c->deRfSigL); free(c->deT); free(c->dePlanck);
    free(c->deEmL); free(c->deEmSig); free(c->deVol);
    free(c->secL); free(c->secT); free(c->secXv); free(c->secPv); free(c->secCv); free(c->secLv); free(c->secWv);
    free(c->secIv); free(c->secCellNode);
    free(c);
}

const char* or_last_error(const or_ctx* c) { return c ? c->err : "null context"; }

int or_abi_version(void) { return SKGPU_ABI_VERSION; }

/* the oracle has one (host) device */
int or_device_count(int32_t* count)
{
    if (!count) return SKGPU_ERR_ARG;
    *count = 1;
    return SKGPU_OK;
}

/* ------------------------------------------------------------------------------------------- */
/* grid uploads                                                                                */
/* ------------------------------------------------------------------------------------------- */

int or_upload_grid_cartesian(or_ctx* c, const double* xb, int32_t nxb, const double* yb, int32_t nyb,
                             const double* zb, int32_t nzb)
{
    if (nxb < 2 || nyb < 2 || nzb < 2) return fail(c, SKGPU_ERR_ARG, "cartesian: borders");
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_CARTESIAN;
    g->xb = dup(xb, nxb * sizeof(double));
    g->yb = dup(yb, nyb * sizeof(double));
    g->zb = dup(zb, nzb * sizeof(double));
    g->nx = nxb - 1; g->ny = nyb - 1; g->nz = nzb - 1;
    g->ext[0] = xb[0]; g->ext[1] = yb[0]; g->ext[2] = zb[0];
    g->ext[3] = xb[nxb - 1]; g->ext[4] = yb[nyb - 1]; g->ext[5] = zb[nzb - 1];
    g->numCells = g->nx * g->ny * g->nz;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_grid_octree(or_ctx* c, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                          const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                          int32_t num_child_index, const int32_t* nb_begin, const int32_t* nb_index,
                          int32_t num_nb_index, double eps)
{
    (void)num_child_index;
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_OCTREE;
    g->tnodes = num_nodes;
    g->tb = dup(bounds, 6 * (size_t)num_nodes * sizeof(double));
    g->tcell = dup(cell_index, num_nodes * sizeof(int));
    g->tchild = (int*)malloc(num_nodes * sizeof(int));
    int numCells = 0;
    for (int l = 0; l < num_nodes; ++l)
    {
        g->tchild[l] = child_count[l] > 0 ? child_index[child_begin[l]] : -1;
        if (cell_index[l] + 1 > numCells) numCells = cell_index[l] + 1;
    }
    g->tnbb = dup(nb_begin, (6 * (size_t)num_nodes + 1) * sizeof(int));
    g->tnb = dup(nb_index, (size_t)num_nb_index * sizeof(int));
    memcpy(g->ext, bounds, 6 * sizeof(double));
    g->eps = eps;
    g->numCells = numCells;
    c->hasGrid = 1;
    return SKGPU_OK;
}

/* AdaptiveMeshSnapshot::Node::leaf and Node::child (AdaptiveMeshSnapshot.cpp:103-145): Box::cellIndices
   estimate (Box.hpp:162-167), one-index correction per axis; -1 outside the root, -2 where the
   reference stops with a FatalError */
static int box_contains(const double* b, double x, double y, double z);
static int am_leaf(const Grid* g, double x, double y, double z)
{
    if (!box_contains(g->tb, x, y, z)) return -1;
    int node = 0;
    for (int guard = 0; guard < 256; ++guard)
    {
        int nx = g->adiv[3 * node], ny = g->adiv[3 * node + 1], nz = g->adiv[3 * node + 2];
        if (nx == 0) return node;
        const double* b = g->tb + 6 * (size_t)node;
        int i = (int)(nx * (x - b[0]) / (b[3] - b[0]));
        int j = (int)(ny * (y - b[1]) / (b[4] - b[1]));
        int k = (int)(nz * (z - b[2]) / (b[5] - b[2]));
        i = i < 0 ? 0 : (i > nx - 1 ? nx - 1 : i);
        j = j < 0 ? 0 : (j > ny - 1 ? ny - 1 : j);
        k = k < 0 ? 0 : (k > nz - 1 ? nz - 1 : k);
        const int* kids = g->ach + g->acb[node];
        int c = kids[(k * ny + j) * nx + i];
        const double* cb = g->tb + 6 * (size_t)c;
        if (!box_contains(cb, x, y, z))
        {
            if (x < cb[0]) i--;
            else if (x > cb[3]) i++;
            if (y < cb[1]) j--;
            else if (y > cb[4]) j++;
            if (z < cb[2]) k--;
            else if (z > cb[5]) k++;
            if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) return -2;
            c = kids[(k * ny + j) * nx + i];
            if (!box_contains(g->tb + 6 * (size_t)c, x, y, z)) return -2;
        }
        node = c;
    }
    return -2;
}

int or_upload_grid_adaptive_mesh(or_ctx* c, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                                 const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                                 int32_t num_child_index, double eps)
{
    if (num_nodes < 1 || !bounds || !cell_index || !child_begin || !child_count) return fail(c, SKGPU_ERR_ARG, "adaptive mesh: missing arrays");
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_ADAPTIVE_MESH;
    g->tnodes = num_nodes;
    g->tb = dup(bounds, 6 * (size_t)num_nodes * sizeof(double));
    g->tcell = dup(cell_index, num_nodes * sizeof(int));
    g->acb = dup(child_begin, num_nodes * sizeof(int));
    g->ach = dup(child_index, (size_t)(num_child_index > 0 ? num_child_index : 1) * sizeof(int));
    g->adiv = (int*)calloc(3 * (size_t)num_nodes, sizeof(int));
    int numCells = 0;
    /* subdivision: children sharing child 0's (y, z), (x, z) and (x, y) lower corners count nx, ny, nz */
    for (int l = 0; l < num_nodes; ++l)
    {
        if (cell_index[l] + 1 > numCells) numCells = cell_index[l] + 1;
        int cnt = child_count[l];
        if (cnt == 0) continue;
        const int* kids = child_index + child_begin[l];
        const double* c0 = bounds + 6 * (size_t)kids[0];
        int nx = 0, ny = 0, nz = 0;
        for (int q = 0; q < cnt; ++q)
        {
            const double* b = bounds + 6 * (size_t)kids[q];
            nx += b[1] == c0[1] && b[2] == c0[2];
            ny += b[0] == c0[0] && b[2] == c0[2];
            nz += b[0] == c0[0] && b[1] == c0[1];
        }
        if (nx * ny * nz != cnt) return fail(c, SKGPU_ERR_ARG, "adaptive mesh: children are not a lattice");
        g->adiv[3 * l] = nx; g->adiv[3 * l + 1] = ny; g->adiv[3 * l + 2] = nz;
    }
    /* Node::addNeighbors (AdaptiveMeshSnapshot.cpp:67-83): the leaf eps beyond each wall centre */
    g->tnbb = (int*)calloc(6 * (size_t)num_nodes + 1, sizeof(int));
    g->tnb = (int*)malloc(6 * (size_t)num_nodes * sizeof(int));
    int n = 0;
    for (int l = 0; l < num_nodes; ++l)
        for (int w = 0; w < 6; ++w)
        {
            g->tnbb[6 * l + w] = n;
            if (child_count[l]) continue;
            const double* b = bounds + 6 * (size_t)l;
            double ctr[3] = {0.5 * (b[0] + b[3]), 0.5 * (b[1] + b[4]), 0.5 * (b[2] + b[5])};
            double d[3] = {0., 0., 0.};
            d[w / 2] = (w % 2) ? eps : -eps;
            int nb = am_leaf(g, ctr[0] + d[0], ctr[1] + d[1], ctr[2] + d[2]);
            if (nb == -2) return fail(c, SKGPU_ERR_ARG, "adaptive mesh: cannot locate a child node");
            if (nb >= 0) g->tnb[n++] = nb;
        }
    g->tnbb[6 * (size_t)num_nodes] = n;
    memcpy(g->ext, bounds, 6 * sizeof(double));
    g->eps = eps;
    g->numCells = numCells;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_voronoi_cell_boxes(or_ctx* c, int32_t num_cells, const double* boxes)
{
    if (!c->hasGrid || c->g.kind != SKGPU_GRID_VORONOI) return fail(c, SKGPU_ERR_STATE, "voronoi boxes: no Voronoi grid");
    if (num_cells != c->g.vn || !boxes) return fail(c, SKGPU_ERR_ARG, "voronoi boxes: one box per cell expected");
    free(c->g.vbox);
    c->g.vbox = dup(boxes, 6 * (size_t)num_cells * sizeof(double));
    return SKGPU_OK;
}

int or_upload_grid_voronoi(or_ctx* c, int32_t num_sites, const double* sites, const int32_t* nb_begin,
                           const int32_t* nb_index, int32_t num_nb_index, const double* extent, double eps)
{
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_VORONOI;
    g->vn = num_sites;
    g->vs = dup(sites, 3 * (size_t)num_sites * sizeof(double));
    g->vnbb = dup(nb_begin, ((size_t)num_sites + 1) * sizeof(int));
    g->vnb = dup(nb_index, (size_t)num_nb_index * sizeof(int));
    memcpy(g->ext, extent, 6 * sizeof(double));
    g->eps = eps;
    g->numCells = num_sites;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_grid_sphere1d(or_ctx* c, int32_t num_borders, const double* rv)
{
    if (num_borders < 2 || !rv || !(rv[0] >= 0.)) return fail(c, SKGPU_ERR_ARG, "sphere1d: need >= 2 borders from r >= 0");
    for (int i = 1; i < num_borders; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(c, SKGPU_ERR_ARG, "sphere1d: borders must ascend");
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_SPHERE1D;
    g->snr = num_borders - 1;
    g->srv = dup(rv, (size_t)num_borders * sizeof(double));
    double r = rv[num_borders - 1];
    double e[6] = {-r, -r, -r, r, r, r};
    memcpy(g->ext, e, sizeof e);
    g->eps = 1e-12 * sqrt(3.) * 2. * r;
    g->numCells = g->snr;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_grid_cylinder2d(or_ctx* c, int32_t nrb, const double* rv, int32_t nzb, const double* zv)
{
    if (nrb < 2 || nzb < 2 || !rv || !zv || !(rv[0] >= 0.)) return fail(c, SKGPU_ERR_ARG, "cylinder2d: bad borders");
    for (int i = 1; i < nrb; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(c, SKGPU_ERR_ARG, "cylinder2d: radial borders must ascend");
    for (int i = 1; i < nzb; ++i)
        if (!(zv[i] > zv[i - 1])) return fail(c, SKGPU_ERR_ARG, "cylinder2d: z borders must ascend");
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_CYLINDER2D;
    g->cnr = nrb - 1;
    g->cnz = nzb - 1;
    g->crv = dup(rv, (size_t)nrb * sizeof(double));
    g->czv = dup(zv, (size_t)nzb * sizeof(double));
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, zv[0], r, r, zv[nzb - 1]};
    memcpy(g->ext, e, sizeof e);
    g->eps = 1e-12 * sqrt(2. * (2. * r) * (2. * r) + (zv[nzb - 1] - zv[0]) * (zv[nzb - 1] - zv[0]));
    g->numCells = g->cnr * g->cnz;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_grid_sphere2d(or_ctx* c, int32_t nrb, const double* rv, int32_t ntb, const double* tv, const double* cv)
{
    if (nrb < 2 || ntb < 2 || !rv || !tv || !cv || !(rv[0] >= 0.)) return fail(c, SKGPU_ERR_ARG, "sphere2d: bad borders");
    for (int i = 1; i < nrb; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(c, SKGPU_ERR_ARG, "sphere2d: radial borders must ascend");
    for (int i = 1; i < ntb; ++i)
        if (!(tv[i] > tv[i - 1])) return fail(c, SKGPU_ERR_ARG, "sphere2d: polar borders must ascend");
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_SPHERE2D;
    g->s2nr = nrb - 1;
    g->s2nt = ntb - 1;
    g->s2r = dup(rv, (size_t)nrb * sizeof(double));
    g->s2t = dup(tv, (size_t)ntb * sizeof(double));
    g->s2c = dup(cv, (size_t)ntb * sizeof(double));
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, -r, r, r, r};
    memcpy(g->ext, e, sizeof e);
    g->eps = 1e-11 * r;
    g->numCells = g->s2nr * g->s2nt;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_grid_sphere3d(or_ctx* c, int32_t nrb, const double* rv, int32_t ntb, const double* tv, const double* cv,
                            int32_t npb, const double* pv, const double* sv, const double* kv, double eps)
{
    if (nrb < 2 || ntb < 2 || npb < 2 || !rv || !tv || !cv || !pv || !sv || !kv || !(rv[0] >= 0.) || !(eps > 0.))
        return fail(c, SKGPU_ERR_ARG, "sphere3d: bad borders");
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_SPHERE3D;
    g->s3nr = nrb - 1;
    g->s3nt = ntb - 1;
    g->s3np = npb - 1;
    g->s3r = dup(rv, (size_t)nrb * sizeof(double));
    g->s3t = dup(tv, (size_t)ntb * sizeof(double));
    g->s3c = dup(cv, (size_t)ntb * sizeof(double));
    g->s3p = dup(pv, (size_t)npb * sizeof(double));
    g->s3s = dup(sv, (size_t)npb * sizeof(double));
    g->s3k = dup(kv, (size_t)npb * sizeof(double));
    g->s3eps = eps;
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, -r, r, r, r};
    memcpy(g->ext, e, sizeof e);
    g->eps = eps;
    g->numCells = g->s3nr * g->s3nt * g->s3np;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_grid_cylinder3d(or_ctx* c, int32_t nrb, const double* rv, int32_t npb, const double* pv, const double* sv,
                              const double* kv, int32_t nzb, const double* zv, double eps, int32_t hole)
{
    if (nrb < 2 || npb < 2 || nzb < 2 || !rv || !pv || !sv || !kv || !zv || !(rv[0] >= 0.) || !(eps > 0.))
        return fail(c, SKGPU_ERR_ARG, "cylinder3d: bad borders");
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_CYLINDER3D;
    g->c3nr = nrb - 1;
    g->c3np = npb - 1;
    g->c3nz = nzb - 1;
    g->c3r = dup(rv, (size_t)nrb * sizeof(double));
    g->c3p = dup(pv, (size_t)npb * sizeof(double));
    g->c3s = dup(sv, (size_t)npb * sizeof(double));
    g->c3k = dup(kv, (size_t)npb * sizeof(double));
    g->c3z = dup(zv, (size_t)nzb * sizeof(double));
    g->c3eps = eps;
    g->c3hole = hole ? 1 : 0;
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, zv[0], r, r, zv[nzb - 1]};
    memcpy(g->ext, e, sizeof e);
    g->eps = eps;
    g->numCells = g->c3nr * g->c3np * g->c3nz;
    c->hasGrid = 1;
    return SKGPU_OK;
}

int or_upload_grid_tetra(or_ctx* c, int32_t num_vertices, const double* vertices, int32_t num_tetra,
                         const int32_t* tetra_vertices, const double* face_normals, const int32_t* face_ntetra,
                         const int32_t* face_nface, const double* extent, double eps)
{
    free_grid(&c->g);
    Grid* g = &c->g;
    g->kind = SKGPU_GRID_TETRA;
    g->ten_n = num_tetra;
    g->tev = dup(vertices, 3 * (size_t)num_vertices * sizeof(double));
    g->tet = dup(tetra_vertices, 4 * (size_t)num_tetra * sizeof(int));
    g->ten = dup(face_normals, 12 * (size_t)num_tetra * sizeof(double));
    g->tent = dup(face_ntetra, 4 * (size_t)num_tetra * sizeof(int));
    g->tenf = dup(face_nface, 4 * (size_t)num_tetra * sizeof(int));
    g->tebox = (double*)malloc(6 * (size_t)num_tetra * sizeof(double));
    for (int t = 0; t < num_tetra; ++t)
    {
        double* b = g->tebox + 6 * (size_t)t;
        b[0] = b[1] = b[2] = DBL_MAX;
        b[3] = b[4] = b[5] = -DBL_MAX;
        for (int v = 0; v < 4; ++v)
        {
            const double* p = vertices + 3 * (size_t)tetra_vertices[4 * t + v];
            for (int a = 0; a < 3; ++a)
            {
                if (p[a] < b[a]) b[a] = p[a];
                if (p[a] > b[3 + a]) b[3 + a] = p[a];
            }
        }
    }
    memcpy(g->ext, extent, 6 * sizeof(double));
    g->eps = eps;
    g->numCells = num_tetra;
    c->hasGrid = 1;
    return SKGPU_OK;
}

/* ------------------------------------------------------------------------------------------- */
/* path segment generators (restatements of the reference CPU generators)                     */
/* ------------------------------------------------------------------------------------------- */

enum { UNKNOWN = 0, INSIDE = 1, OUTSIDE = 2 };

typedef struct
{
    double rx, ry, rz, kx, ky, kz, ds;
    int m, state;
    int i, j, k;  /* cartesian */
    int node;     /* octree */
    int mr, ef;   /* voronoi / tetra */
    double sq, sp; /* sphere1d: projection of the position on the direction, impact parameter */
    int simin, sinw;
    double cR, cz, ckq, ckz, cp, cq; /* cylinder2d: meridional position and direction */
    int cimin, cphase;
} Gen;

static int box_contains(const double* b, double x, double y, double z)
{
    return x >= b[0] && x <= b[3] && y >= b[1] && y <= b[4] && z >= b[2] && z <= b[5];
}

static void gen_start(Gen* s, const double* ray)
{
    memset(s, 0, sizeof *s);
    s->state = UNKNOWN;
    s->rx = ray[0]; s->ry = ray[1]; s->rz = ray[2];
    s->kx = ray[3]; s->ky = ray[4]; s->kz = ray[5];
    s->m = -1;
    s->node = -1;
    s->mr = -1;
    s->ef = -1;
}

static void propagater(Gen* s, double d)
{
    s->rx += s->kx * d;
    s->ry += s->ky * d;
    s->rz += s->kz * d;
}

/* PathSegmentGenerator::moveInside */
static int move_inside(Gen* s, const double* b, double eps)
{
    s->m = -1;
    s->ds = 0.;
    s->state = OUTSIDE;
    double cumds = 0.;
    if (s->rx <= b[0])
    {
        if (s->kx <= 0.0) return 0;
        double d = (b[0] - s->rx) / s->kx;
        s->rx = b[0] + eps; s->ry += s->ky * d; s->rz += s->kz * d; cumds += d;
    }
    else if (s->rx >= b[3])
    {
        if (s->kx >= 0.0) return 0;
        double d = (b[3] - s->rx) / s->kx;
        s->rx = b[3] - eps; s->ry += s->ky * d; s->rz += s->kz * d; cumds += d;
    }
    if (s->ry <= b[1])
    {
        if (s->ky <= 0.0) return 0;
        double d = (b[1] - s->ry) / s->ky;
        s->rx += s->kx * d; s->ry = b[1] + eps; s->rz += s->kz * d; cumds += d;
    }
    else if (s->ry >= b[4])
    {
        if (s->ky >= 0.0) return 0;
        double d = (b[4] - s->ry) / s->ky;
        s->rx += s->kx * d; s->ry = b[4] - eps; s->rz += s->kz * d; cumds += d;
    }
    if (s->rz <= b[2])
    {
        if (s->kz <= 0.0) return 0;
        double d = (b[2] - s->rz) / s->kz;
        s->rx += s->kx * d; s->ry += s->ky * d; s->rz = b[2] + eps; cumds += d;
    }
    else if (s->rz >= b[5])
    {
        if (s->kz >= 0.0) return 0;
        double d = (b[5] - s->rz) / s->kz;
        s->rx += s->kx * d; s->ry += s->ky * d; s->rz = b[5] - eps; cumds += d;
    }
    if (!box_contains(b, s->rx, s->ry, s->rz)) return 0;
    s->m = -1;
    s->ds = cumds;
    s->state = INSIDE;
    return 1;
}

/* NR::locateClip */
/* NR::locate (SKIRT/utils/NR.hpp:168-173): -1 below the first entry, n - 1 above the last, n - 2
   exactly at the last */
static int locate_nr(const double* xv, int n, double x)
{
    if (x == xv[n - 1]) return n - 2;
    int jl = -1, ju = n;
    while (ju - jl > 1)
    {
        int jm = (ju + jl) >> 1;
        if (x < xv[jm])
            ju = jm;
        else
            jl = jm;
    }
    return jl;
}

/* NR::clampedValue<NR::interpolateLogLog> (NR.hpp:349-358, 394-401); a first interval starting at
   x = 0, where the power law is undefined, gives the interval's lower value */
static double clamped_loglog(const double* xv, const double* yv, int n, double x)
{
    int i = locate_nr(xv, n, x);
    if (i < 0) return yv[0];
    if (i >= n - 1) return yv[n - 1];
    double x1 = xv[i], x2 = xv[i + 1], f1 = yv[i], f2 = yv[i + 1];
    if (f1 <= 0 || f2 <= 0)
    {
        if (x == x1) return f1;
        if (x == x2) return f2;
        return 0;
    }
    if (!(x1 > 0)) return f1;
    return f1 * exp(log(x / x1) / log(x2 / x1) * (log(f2 / f1)));
}

static int locate_clip(const double* xv, int n, double x)
{
    if (x < xv[0]) return 0;
    int jl = -1, ju = n - 1;
    while (ju - jl > 1)
    {
        int jm = (ju + jl) >> 1;
        if (x < xv[jm]) ju = jm; else jl = jm;
    }
    return jl;
}

static int cart_next(const Grid* g, Gen* s)
{
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        double dx = g->ext[3] - g->ext[0], dy = g->ext[4] - g->ext[1], dz = g->ext[5] - g->ext[2];
        if (!move_inside(s, g->ext, 1e-12 * sqrt(dx * dx + dy * dy + dz * dz))) return 0;
        s->i = locate_clip(g->xb, g->nx + 1, s->rx);
        s->j = locate_clip(g->yb, g->ny + 1, s->ry);
        s->k = locate_clip(g->zb, g->nz + 1, s->rz);
        if (s->ds > 0.) return 1;
    }
    int m = s->k + g->nz * s->j + g->nz * g->ny * s->i;
    double xE = (s->kx < 0.0) ? g->xb[s->i] : g->xb[s->i + 1];
    double yE = (s->ky < 0.0) ? g->yb[s->j] : g->yb[s->j + 1];
    double zE = (s->kz < 0.0) ? g->zb[s->k] : g->zb[s->k + 1];
    double dsx = (fabs(s->kx) > 1e-15) ? (xE - s->rx) / s->kx : DBL_MAX;
    double dsy = (fabs(s->ky) > 1e-15) ? (yE - s->ry) / s->ky : DBL_MAX;
    double dsz = (fabs(s->kz) > 1e-15) ? (zE - s->rz) / s->kz : DBL_MAX;
    if (dsx <= dsy && dsx <= dsz)
    {
        s->m = m; s->ds = dsx;
        s->rx = xE; s->ry += s->ky * dsx; s->rz += s->kz * dsx;
        s->i += (s->kx < 0.0) ? -1 : 1;
        if (s->i >= g->nx || s->i < 0) s->state = OUTSIDE;
    }
    else if (dsy < dsx && dsy <= dsz)
    {
        s->m = m; s->ds = dsy;
        s->ry = yE; s->rx += s->kx * dsy; s->rz += s->kz * dsy;
        s->j += (s->ky < 0.0) ? -1 : 1;
        if (s->j >= g->ny || s->j < 0) s->state = OUTSIDE;
    }
    else
    {
        s->m = m; s->ds = dsz;
        s->rz = zE; s->rx += s->kx * dsz; s->ry += s->ky * dsz;
        s->k += (s->kz < 0.0) ? -1 : 1;
        if (s->k >= g->nz || s->k < 0) s->state = OUTSIDE;
    }
    return 1;
}

/* TreeNode::leafChild from the root */
static int leaf_child(const Grid* g, double x, double y, double z)
{
    if (!box_contains(g->tb, x, y, z)) return -1;
    int node = 0;
    while (g->tchild[node] >= 0)
    {
        int c0 = g->tchild[node];
        const double* cb = g->tb + 6 * (size_t)c0;
        node = c0 + (x < cb[3] ? 0 : 1) + (y < cb[4] ? 0 : 2) + (z < cb[5] ? 0 : 4);
    }
    return node;
}

/* the leaf search of a tree grid: the octree's, or the adaptive mesh's (-2 counts as outside) */
static int tree_leaf(const Grid* g, double x, double y, double z)
{
    if (g->kind == SKGPU_GRID_ADAPTIVE_MESH)
    {
        int l = am_leaf(g, x, y, z);
        return l < 0 ? -1 : l;
    }
    return leaf_child(g, x, y, z);
}

/* TreeSpatialGrid::MySegmentGenerator::next (TreeSpatialGrid.cpp:143-228) and
   AdaptiveMeshSnapshot::MySegmentGenerator::next (AdaptiveMeshSnapshot.cpp:378-449) */
static int tree_next(const Grid* g, Gen* s)
{
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        if (!move_inside(s, g->ext, g->eps)) return 0;
        s->node = tree_leaf(g, s->rx, s->ry, s->rz);
        if (s->node < 0)
        {
            s->state = OUTSIDE;
            return 0;
        }
        if (s->ds > 0.) return 1;
    }
    const double* b = g->tb + 6 * (size_t)s->node;
    double xnext = (s->kx < 0.0) ? b[0] : b[3];
    double ynext = (s->ky < 0.0) ? b[1] : b[4];
    double znext = (s->kz < 0.0) ? b[2] : b[5];
    double dsx = (fabs(s->kx) > 1e-15) ? (xnext - s->rx) / s->kx : DBL_MAX;
    double dsy = (fabs(s->ky) > 1e-15) ? (ynext - s->ry) / s->ky : DBL_MAX;
    double dsz = (fabs(s->kz) > 1e-15) ? (znext - s->rz) / s->kz : DBL_MAX;
    double ds;
    int wall;
    if (dsx <= dsy && dsx <= dsz) { ds = dsx; wall = (s->kx < 0.0) ? 0 : 1; }
    else if (dsy <= dsx && dsy <= dsz) { ds = dsy; wall = (s->ky < 0.0) ? 2 : 3; }
    else { ds = dsz; wall = (s->kz < 0.0) ? 4 : 5; }
    propagater(s, ds + g->eps);
    s->m = g->tcell[s->node];
    s->ds = ds;
    int old = s->node, nb = -1;
    for (int e = g->tnbb[6 * old + wall]; e < g->tnbb[6 * old + wall + 1]; ++e)
    {
        int cand = g->tnb[e];
        if (box_contains(g->tb + 6 * (size_t)cand, s->rx, s->ry, s->rz))
        {
            nb = cand;
            break;
        }
    }
    if (nb < 0) nb = tree_leaf(g, s->rx, s->ry, s->rz);
    if (nb == old)
    {
        s->rx = nextafter(s->rx, (s->kx < 0.) ? -DBL_MAX : DBL_MAX);
        s->ry = nextafter(s->ry, (s->ky < 0.) ? -DBL_MAX : DBL_MAX);
        s->rz = nextafter(s->rz, (s->kz < 0.) ? -DBL_MAX : DBL_MAX);
        nb = tree_leaf(g, s->rx, s->ry, s->rz);
    }
    s->node = nb;
    if (nb < 0 || nb == old) s->state = OUTSIDE;
    return 1;
}

/* nearest site by brute force (VoronoiMeshSnapshot::cellIndex up to equidistant ties) */
static int vor_cell(const Grid* g, double x, double y, double z)
{
    if (!box_contains(g->ext, x, y, z)) return -1;
    int best = -1;
    double bd = DBL_MAX;
    for (int s = 0; s < g->vn; ++s)
    {
        const double* p = g->vs + 3 * (size_t)s;
        double dx = p[0] - x, dy = p[1] - y, dz = p[2] - z;
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < bd)
        {
            bd = d2;
            best = s;
        }
    }
    return best;
}

static int vor_next(const Grid* g, Gen* s)
{
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        if (!move_inside(s, g->ext, g->eps)) return 0;
        s->mr = vor_cell(g, s->rx, s->ry, s->rz);
        if (s->mr < 0)
        {
            s->state = OUTSIDE;
            return 0;
        }
        if (s->ds > 0.) return 1;
    }
    for (int guard = 0; guard < 1000; ++guard)
    {
        const double* pr = g->vs + 3 * (size_t)s->mr;
        double sq = DBL_MAX;
        int mq = -99;
        for (int e = g->vnbb[s->mr]; e < g->vnbb[s->mr + 1]; ++e)
        {
            int mi = g->vnb[e];
            double si = 0;
            if (mi >= 0)
            {
                const double* pi = g->vs + 3 * (size_t)mi;
                double nx = pi[0] - pr[0], ny = pi[1] - pr[1], nz = pi[2] - pr[2];
                double ndotk = nx * s->kx + ny * s->ky + nz * s->kz;
                if (ndotk > 0)
                {
                    double px = 0.5 * (pi[0] + pr[0]), py = 0.5 * (pi[1] + pr[1]), pz = 0.5 * (pi[2] + pr[2]);
                    si = (nx * (px - s->rx) + ny * (py - s->ry) + nz * (pz - s->rz)) / ndotk;
                }
            }
            else
            {
                switch (mi)
                {
                    case -1: si = (g->ext[0] - s->rx) / s->kx; break;
                    case -2: si = (g->ext[3] - s->rx) / s->kx; break;
                    case -3: si = (g->ext[1] - s->ry) / s->ky; break;
                    case -4: si = (g->ext[4] - s->ry) / s->ky; break;
                    case -5: si = (g->ext[2] - s->rz) / s->kz; break;
                    case -6: si = (g->ext[5] - s->rz) / s->kz; break;
                    default: si = 0; break;
                }
            }
            if (si > 0 && si < sq)
            {
                sq = si;
                mq = mi;
            }
        }
        if (mq == -99)
        {
            propagater(s, g->eps);
            s->mr = vor_cell(g, s->rx, s->ry, s->rz);
            if (s->mr < 0)
            {
                s->state = OUTSIDE;
                return 0;
            }
        }
        else
        {
            propagater(s, sq + g->eps);
            s->m = s->mr;
            s->ds = sq;
            s->mr = mq;
            if (s->mr < 0) s->state = OUTSIDE;
            return 1;
        }
    }
    s->state = OUTSIDE;
    return 0;
}

static const double* te_vertex(const Grid* g, int t, int v) { return g->tev + 3 * (size_t)g->tet[4 * (size_t)t + v]; }

static int te_contains(const Grid* g, int t, double x, double y, double z)
{
    if (!box_contains(g->tebox + 6 * (size_t)t, x, y, z)) return 0;
    const double* n = g->ten + 12 * (size_t)t;
    const double* v = te_vertex(g, t, 3);
    for (int f = 0; f <= 2; ++f)
        if ((v[0] - x) * n[3 * f] + (v[1] - y) * n[3 * f + 1] + (v[2] - z) * n[3 * f + 2] < 0) return 0;
    v = te_vertex(g, t, 0);
    if ((v[0] - x) * n[9] + (v[1] - y) * n[10] + (v[2] - z) * n[11] < 0.) return 0;
    return 1;
}

static int te_cell(const Grid* g, double x, double y, double z)
{
    if (!box_contains(g->ext, x, y, z)) return -1;
    for (int t = 0; t < g->ten_n; ++t)
        if (te_contains(g, t, x, y, z)) return t;
    return -1;
}

static void cross3(const double* a, const double* b, double* c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void cw_vertices(int face, int cv[3])
{
    cv[0] = (face + 3) % 4;
    cv[1] = (face + 2) % 4;
    cv[2] = (face + 1) % 4;
    if (face % 2 == 0)
    {
        int t = cv[0]; cv[0] = cv[2]; cv[2] = t;
    }
}

static int te_entering_face(const Grid* g, int t, const double* pos, const double* dir)
{
    static const int etable[6][2] = {{3, 2}, {1, 3}, {2, 1}, {3, 0}, {0, 2}, {1, 0}};
    int e = 0;
    for (int t1 = 0; t1 < 3; t1++)
        for (int t2 = t1 + 1; t2 < 4; t2++)
        {
            const double* v1 = te_vertex(g, t, t1);
            const double* v2 = te_vertex(g, t, t2);
            double rel[3] = {pos[0] - v1[0], pos[1] - v1[1], pos[2] - v1[2]}, mom[3];
            cross3(dir, rel, mom);
            double edge[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
            double prod = dot3(mom, edge);
            if (prod != 0.) return prod < 0 ? etable[e][0] : etable[e][1];
            e++;
        }
    return -1;
}

static int tet_next(const Grid* g, Gen* s)
{
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        if (!move_inside(s, g->ext, g->eps)) return 0;
        s->mr = te_cell(g, s->rx, s->ry, s->rz);
        s->ef = -1;
        if (s->mr == -1)
        {
            s->state = OUTSIDE;
            return 0;
        }
        if (s->ds > 0.) return 1;
    }
    for (int guard = 0; guard < 1000; ++guard)
    {
        double pos[3] = {s->rx, s->ry, s->rz}, dir[3] = {s->kx, s->ky, s->kz};
        int leaving = -1;
        double d = DBL_MAX;
        if (s->ef == -1) s->ef = te_entering_face(g, s->mr, pos, dir);
        if (s->ef < 0) s->ef = 0;
        const double* ve = te_vertex(g, s->mr, s->ef);
        double rel[3] = {pos[0] - ve[0], pos[1] - ve[1], pos[2] - ve[2]}, mom[3];
        cross3(dir, rel, mom);
        int cv[3];
        cw_vertices(s->ef, cv);
        const double* c0 = te_vertex(g, s->mr, cv[0]);
        double e0[3] = {ve[0] - c0[0], ve[1] - c0[1], ve[2] - c0[2]};
        double prod0 = dot3(mom, e0);
        int clock0 = prod0 < 0;
        int i = clock0 ? 1 : 2;
        const double* ci = te_vertex(g, s->mr, cv[i]);
        double ei[3] = {ve[0] - ci[0], ve[1] - ci[1], ve[2] - ci[2]};
        double prodi = dot3(mom, ei);
        int cclocki = prodi >= 0;
        const double* nrm = g->ten + 12 * (size_t)s->mr;
        double vp[3] = {ve[0] - pos[0], ve[1] - pos[1], ve[2] - pos[2]};
        if (prod0 == 0. || prodi == 0.)
        {
            for (int q = 0; q < 3; ++q)
            {
                const double* n = nrm + 3 * cv[q];
                double ndotk = dot3(n, dir);
                if (ndotk > 0)
                {
                    double dq = dot3(n, vp) / ndotk;
                    if (dq < d)
                    {
                        d = dq;
                        leaving = cv[q];
                    }
                }
            }
        }
        else
        {
            static const int dtable[2][2] = {{1, 0}, {0, 2}};
            leaving = cv[dtable[clock0][cclocki]];
            const double* n = nrm + 3 * leaving;
            d = dot3(n, vp) / dot3(n, dir);
        }
        if (leaving == -1 || d < g->eps)
        {
            propagater(s, g->eps);
            s->mr = te_cell(g, s->rx, s->ry, s->rz);
            if (s->mr < 0)
            {
                s->state = OUTSIDE;
                return 0;
            }
            s->ef = -1;
        }
        else
        {
            propagater(s, d);
            s->m = s->mr;
            s->ds = d;
            int nt = g->tent[4 * (size_t)s->mr + leaving], nf = g->tenf[4 * (size_t)s->mr + leaving];
            s->mr = nt;
            if (s->mr < 0)
            {
                s->state = OUTSIDE;
                return 0;
            }
            s->ef = nf;
            return 1;
        }
    }
    s->state = OUTSIDE;
    return 0;
}

/* NR::locate on an ascending array of n entries (SKIRT/utils/NR.hpp:168-173): -1 below xv[0], n-2 at xv[n-1] */
static int nr_locate(const double* xv, int n, double x)
{
    if (x == xv[n - 1]) return n - 2;
    int jl = -1, ju = n;
    while (ju - jl > 1)
    {
        int jm = (ju + jl) >> 1;
        if (x < xv[jm]) ju = jm; else jl = jm;
    }
    return jl;
}

/* Sphere1DSpatialGrid::MySegmentGenerator::next (Sphere1DSpatialGrid.cpp): radial shells crossed
   inwards down to the impact parameter's shell, then outwards; the position is not advanced (the
   generator tracks q, the position's projection on the direction) */
static int sph_next(const Grid* g, Gen* s)
{
    if (s->state == OUTSIDE) return 0;
    const double* rv = g->srv;
    int nr = g->snr;
    if (s->state == UNKNOWN)
    {
        double rmax = rv[nr], rmin = rv[0];
        double r = sqrt(s->rx * s->rx + s->ry * s->ry + s->rz * s->rz);
        s->sq = s->rx * s->kx + s->ry * s->ky + s->rz * s->kz;
        s->sp = sqrt((r - s->sq) * (r + s->sq));
        if (r > rmax)
        {
            if (s->sq > 0. || s->sp > rmax)
            {
                s->state = OUTSIDE;
                return 0;
            }
            double qmax = -sqrt((rmax - s->sp) * (rmax + s->sp));
            s->m = -1;
            s->ds = qmax - s->sq;
            s->i = nr - 1;
            s->sq = qmax;
            s->state = INSIDE;
            s->simin = nr_locate(rv, nr + 1, s->sp);
            s->sinw = s->i > s->simin;
            return 1;
        }
        else if (r < rmin)
        {
            double qmin = sqrt((rmin - s->sp) * (rmin + s->sp));
            s->m = -1;
            s->ds = qmin - s->sq;
            s->i = 0;
            s->sq = qmin;
            s->state = INSIDE;
            s->sinw = 0;
            return 1;
        }
        else
        {
            s->i = locate_clip(rv, nr + 1, r);
            s->state = INSIDE;
            s->sinw = 0;
            if (s->sq < 0.)
            {
                s->simin = nr_locate(rv, nr + 1, s->sp);
                if (s->i > s->simin) s->sinw = 1;
            }
        }
    }
    if (s->sinw)
    {
        double rN = rv[s->i];
        double qN = -sqrt((rN - s->sp) * (rN + s->sp));
        s->m = s->i;
        s->ds = qN - s->sq;
        s->i--;
        s->sq = qN;
        if (s->i <= s->simin) s->sinw = 0;
        return 1;
    }
    double rN = rv[s->i + 1];
    double qN = sqrt((rN - s->sp) * (rN + s->sp));
    s->m = s->i;
    s->ds = qN - s->sq;
    s->i++;
    s->sq = qN;
    if (s->i >= nr) s->state = OUTSIDE;
    return 1;
}

/* Quadratic::smallestPositiveSolution (SKIRT/utils/Quadratic.hpp:44-68): of x^2 + 2 b x + c = 0, or 0 */
static double quad_sps(double b, double c)
{
    if (b * b > c)
    {
        if (b > 0.)
        {
            if (c < 0.)
            {
                double x1 = -b - sqrt(b * b - c);
                return c / x1;
            }
        }
        else
        {
            double x2 = -b + sqrt(b * b - c);
            if (c > 0.)
            {
                double x1 = c / x2;
                if (x1 < x2) return x1;
            }
            return x2;
        }
    }
    return 0.;
}

/* smallestPositiveSolution of a x^2 + 2 b x + c = 0 (Sphere2DSpatialGrid.cpp:118-125) */
static double quad_sps3(double a, double b, double c)
{
    if (fabs(a) > 1e-9) return quad_sps(b / a, c / a);
    double x = -0.5 * c / b;
    if (x > 0.) return x;
    return 0.;
}

/* firstIntersectionSphere / firstIntersectionCone (Sphere2DSpatialGrid.cpp:130-142) */
static double s2_sphere(const Gen* s, double r)
{
    double dot = s->rx * s->kx + s->ry * s->ky + s->rz * s->kz;
    double n2 = s->rx * s->rx + s->ry * s->ry + s->rz * s->rz;
    return quad_sps(dot, n2 - r * r);
}
static double s2_cone(const Gen* s, double c)
{
    if (c == 0.) return -s->rz / s->kz;
    double dot = s->rx * s->kx + s->ry * s->ky + s->rz * s->kz;
    double n2 = s->rx * s->rx + s->ry * s->ry + s->rz * s->rz;
    return quad_sps3(c * c - s->kz * s->kz, c * c * dot - s->rz * s->kz, c * c * n2 - s->rz * s->rz);
}

/* setCellIndices (Sphere2DSpatialGrid.cpp:160-167, Position::spherical) */
static int s2_indices(const Grid* g, Gen* s)
{
    double radius = sqrt(s->rx * s->rx + s->ry * s->ry + s->rz * s->rz);
    double theta = radius == 0 ? 0. : acos(s->rz / radius);
    s->i = nr_locate(g->s2r, g->s2nr + 1, radius);
    s->j = locate_clip(g->s2t, g->s2nt + 1, theta);
    return s->i < g->s2nr;
}

/* Sphere2DSpatialGrid::MySegmentGenerator::next (Sphere2DSpatialGrid.cpp:176-290) */
static int sph2_next(const Grid* g, Gen* s)
{
    const double* rv = g->s2r;
    const double* cv = g->s2c;
    int Nr = g->s2nr, Nt = g->s2nt;
    double eps = 1e-11 * rv[Nr];
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        double rn = sqrt(s->rx * s->rx + s->ry * s->ry + s->rz * s->rz);
        if (rn > rv[Nr])
        {
            double ds = s2_sphere(s, rv[Nr]);
            if (ds <= 0.) { s->state = OUTSIDE; return 0; }
            propagater(s, ds + eps);
            if (!s2_indices(g, s)) { s->state = OUTSIDE; return 0; }
            s->m = -1;
            s->ds = ds;
            s->state = INSIDE;
            return 1;
        }
        if (rn < eps) propagater(s, eps);
        if (!s2_indices(g, s)) { s->state = OUTSIDE; return 0; }
        s->state = INSIDE;
    }
    for (int guard = 0; guard < 1000; ++guard)
    {
        int icur = s->i, jcur = s->j;
        double ds = DBL_MAX;
        if (icur > 0 || (icur == 0 && rv[0] > 0.))
        {
            double t = s2_sphere(s, rv[icur]);
            if (t > 0 && t < ds) { ds = t; s->i = icur - 1; s->j = jcur; }
        }
        {
            double t = s2_sphere(s, rv[icur + 1]);
            if (t > 0 && t < ds) { ds = t; s->i = icur + 1; s->j = jcur; }
        }
        if (jcur > 0)
        {
            double t = s2_cone(s, cv[jcur]);
            if (t > 0 && t < ds) { ds = t; s->i = icur; s->j = jcur - 1; }
        }
        if (jcur < Nt - 1)
        {
            double t = s2_cone(s, cv[jcur + 1]);
            if (t > 0 && t < ds) { ds = t; s->i = icur; s->j = jcur + 1; }
        }
        if (s->i != icur || s->j != jcur)
        {
            s->m = jcur + Nt * icur;  /* Sphere2DSpatialGrid::index */
            s->ds = ds;
            propagater(s, ds + eps);
            if (s->i >= Nr) s->state = OUTSIDE;
            return 1;
        }
        propagater(s, eps);
        if (!s2_indices(g, s)) { s->state = OUTSIDE; return 0; }
    }
    s->state = OUTSIDE;
    return 0;
}

/* Sphere3DSpatialGrid::MySegmentGenerator (Sphere3DSpatialGrid.cpp:160-370); EPS = 1e-12 (:20) */
static double s3_sps3(double a, double b, double c)
{
    if (fabs(a) > 1e-12) return quad_sps(b / a, c / a);
    double x = -0.5 * c / b;
    if (x > 0.) return x;
    return 0.;
}
static double s3_sphere(const Gen* s, double r)
{
    double dot = s->rx * s->kx + s->ry * s->ky + s->rz * s->kz;
    double n2 = s->rx * s->rx + s->ry * s->ry + s->rz * s->rz;
    return quad_sps(dot, n2 - r * r);
}
static double s3_cone(const Gen* s, double c)
{
    if (c == 0.) return -s->rz / s->kz;
    double dot = s->rx * s->kx + s->ry * s->ky + s->rz * s->kz;
    double n2 = s->rx * s->rx + s->ry * s->ry + s->rz * s->rz;
    return s3_sps3(c * c - s->kz * s->kz, c * c * dot - s->rz * s->kz, c * c * n2 - s->rz * s->rz);
}
static double s3_plane(const Gen* s, double sn, double cs)
{
    double q = s->kx * sn - s->ky * cs;
    if (fabs(q) < 1e-12) return 0.;
    return -(s->rx * sn - s->ry * cs) / q;
}
static int s3_indices(const Grid* g, Gen* s)
{
    double radius = sqrt(s->rx * s->rx + s->ry * s->ry + s->rz * s->rz);
    double theta = 0., phi = 0.;
    if (radius != 0)
    {
        theta = acos(s->rz / radius);
        phi = atan2(s->ry, s->rx);
    }
    s->i = nr_locate(g->s3r, g->s3nr + 1, radius);
    s->j = locate_clip(g->s3t, g->s3nt + 1, theta);
    s->k = locate_clip(g->s3p, g->s3np + 1, phi);
    return s->i < g->s3nr;
}
static int sph3_next(const Grid* g, Gen* s)
{
    const double* rv = g->s3r;
    int Nr = g->s3nr, Nt = g->s3nt, Np = g->s3np;
    double eps = g->s3eps;
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        double rn = sqrt(s->rx * s->rx + s->ry * s->ry + s->rz * s->rz);
        if (rn > rv[Nr])
        {
            double ds = s3_sphere(s, rv[Nr]);
            if (ds <= 0.) { s->state = OUTSIDE; return 0; }
            propagater(s, ds + eps);
            if (!s3_indices(g, s)) { s->state = OUTSIDE; return 0; }
            s->m = -1;
            s->ds = ds;
            s->state = INSIDE;
            return 1;
        }
        if (!s3_indices(g, s)) { s->state = OUTSIDE; return 0; }
        s->state = INSIDE;
    }
    if (s->i >= 0)
    {
        int icur = s->i, jcur = s->j, kcur = s->k;
        double ds = DBL_MAX;
        {
            double t = s3_sphere(s, rv[icur]);
            if (t > 0 && t < ds) { ds = t; s->i = icur - 1; s->j = jcur; s->k = kcur; }
        }
        {
            double t = s3_sphere(s, rv[icur + 1]);
            if (t > 0 && t < ds) { ds = t; s->i = icur + 1; s->j = jcur; s->k = kcur; }
        }
        if (jcur > 0)
        {
            double t = s3_cone(s, g->s3c[jcur]);
            if (t > 0 && t < ds) { ds = t; s->i = icur; s->j = jcur - 1; s->k = kcur; }
        }
        if (jcur < Nt - 1)
        {
            double t = s3_cone(s, g->s3c[jcur + 1]);
            if (t > 0 && t < ds) { ds = t; s->i = icur; s->j = jcur + 1; s->k = kcur; }
        }
        {
            double t = s3_plane(s, g->s3s[kcur], g->s3k[kcur]);
            if (t > 0. && t < ds) { ds = t; s->i = icur; s->j = jcur; s->k = kcur > 0 ? kcur - 1 : Np - 1; }
        }
        {
            double t = s3_plane(s, g->s3s[kcur + 1], g->s3k[kcur + 1]);
            if (t > 0. && t < ds) { ds = t; s->i = icur; s->j = jcur; s->k = (kcur + 1) % Np; }
        }
        if (ds == DBL_MAX) { s->state = OUTSIDE; return 0; }
        s->m = kcur + (jcur + icur * Nt) * Np;  /* Sphere3DSpatialGrid::index */
        s->ds = ds;
        propagater(s, ds + eps);
        if (s->i >= Nr) s->state = OUTSIDE;
    }
    else
    {
        double ds = s3_sphere(s, rv[0]);
        if (ds <= 0.) { s->state = OUTSIDE; return 0; }
        s->m = -1;
        s->ds = ds;
        propagater(s, ds + eps);
        if (!s3_indices(g, s)) { s->state = OUTSIDE; return 0; }
    }
    return 1;
}

/* NR::locateFail (SKIRT/utils/NR.hpp:186-191): -1 outside [xv[0], xv[n-1]] */
static int nr_locate_fail(const double* xv, int n, double x)
{
    if (x > xv[n - 1]) return -1;
    int jl = -1, ju = n - 1;
    while (ju - jl > 1)
    {
        int jm = (ju + jl) >> 1;
        if (x < xv[jm]) ju = jm; else jl = jm;
    }
    return jl;
}

/* Cylinder3DSpatialGrid::MySegmentGenerator (Cylinder3DSpatialGrid.cpp:180-440); EPS = 1e-12 (:19) */
static double c3_cyl(const Grid* g, const Gen* s, double kq2, int i)
{
    if (fabs(kq2) < 1e-12) return 0.;
    double b = s->rx * s->kx + s->ry * s->ky;
    double c = s->rx * s->rx + s->ry * s->ry - g->c3r[i] * g->c3r[i];
    return quad_sps(b / kq2, c / kq2);
}
static double c3_horiz(const Grid* g, const Gen* s, int k)
{
    if (fabs(s->kz) < 1e-12) return 0.;
    return (g->c3z[k] - s->rz) / s->kz;
}
static int c3_indices(const Grid* g, Gen* s)
{
    double R = sqrt(s->rx * s->rx + s->ry * s->ry);
    double phi = atan2(s->ry, s->rx);
    s->i = nr_locate(g->c3r, g->c3nr + 1, R);
    s->j = locate_clip(g->c3p, g->c3np + 1, phi);
    s->k = nr_locate_fail(g->c3z, g->c3nz + 1, s->rz);
    return s->i < g->c3nr && s->k >= 0;
}
static int cyl3_next(const Grid* g, Gen* s)
{
    int NR = g->c3nr, Np = g->c3np, Nz = g->c3nz;
    double eps = g->c3eps;
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        s->cq = s->kx * s->kx + s->ky * s->ky;  /* kq2, kept for the rest of the path */
        double cumds = 0.;
        double R = sqrt(s->rx * s->rx + s->ry * s->ry);
        if (R > g->c3r[NR])
        {
            double ds = c3_cyl(g, s, s->cq, NR);
            if (ds <= 0.) { s->state = OUTSIDE; return 0; }
            propagater(s, ds + eps);
            cumds += ds;
        }
        if (s->rz < g->c3z[0])
        {
            double ds = c3_horiz(g, s, 0);
            if (ds <= 0.) { s->state = OUTSIDE; return 0; }
            propagater(s, ds + eps);
            cumds += ds;
        }
        else if (s->rz > g->c3z[Nz])
        {
            double ds = c3_horiz(g, s, Nz);
            if (ds <= 0.) { s->state = OUTSIDE; return 0; }
            propagater(s, ds + eps);
            cumds += ds;
        }
        if (!c3_indices(g, s)) { s->state = OUTSIDE; return 0; }
        s->state = INSIDE;
        if (cumds != 0.)
        {
            s->m = -1;
            s->ds = cumds;
            return 1;
        }
    }
    double kq2 = s->cq;
    if (s->i >= 0)
    {
        int icur = s->i, jcur = s->j, kcur = s->k;
        double ds = DBL_MAX, t;
        t = c3_cyl(g, s, kq2, icur);
        if (t > 0. && t < ds) { ds = t; s->i = icur - 1; s->j = jcur; s->k = kcur; }
        t = c3_cyl(g, s, kq2, icur + 1);
        if (t > 0. && t < ds) { ds = t; s->i = icur + 1; s->j = jcur; s->k = kcur; }
        t = s3_plane(s, g->c3s[jcur], g->c3k[jcur]);
        if (t > 0. && t < ds) { ds = t; s->i = icur; s->j = jcur > 0 ? jcur - 1 : Np - 1; s->k = kcur; }
        t = s3_plane(s, g->c3s[jcur + 1], g->c3k[jcur + 1]);
        if (t > 0. && t < ds) { ds = t; s->i = icur; s->j = (jcur + 1) % Np; s->k = kcur; }
        t = c3_horiz(g, s, kcur);
        if (t > 0 && t < ds) { ds = t; s->i = icur; s->j = jcur; s->k = kcur - 1; }
        t = c3_horiz(g, s, kcur + 1);
        if (t > 0. && t < ds) { ds = t; s->i = icur; s->j = jcur; s->k = kcur + 1; }
        if (ds == DBL_MAX) { s->state = OUTSIDE; return 0; }
        s->m = kcur + (jcur + icur * Np) * Nz;  /* Cylinder3DSpatialGrid::index */
        s->ds = ds;
        propagater(s, ds + eps);
        if (s->i >= NR || s->k < 0 || s->k >= Nz) s->state = OUTSIDE;
    }
    else if (!g->c3hole)
    {
        int kcur = s->k;
        double ds = DBL_MAX, t;
        t = c3_cyl(g, s, kq2, 0);
        if (t > 0. && t < ds) ds = t;
        t = c3_horiz(g, s, kcur);
        if (t > 0 && t < ds) { ds = t; s->k = kcur - 1; }
        t = c3_horiz(g, s, kcur + 1);
        if (t > 0. && t < ds) { ds = t; s->k = kcur + 1; }
        if (ds == DBL_MAX) { s->state = OUTSIDE; return 0; }
        s->m = kcur + (s->j + 0 * Np) * Nz;  /* index(0, j, kcur) */
        s->ds = ds;
        propagater(s, ds + eps);
        if (s->k == kcur)
        {
            if (!c3_indices(g, s)) { s->state = OUTSIDE; return 0; }
        }
        else if (s->k < 0 || s->k >= Nz)
            s->state = OUTSIDE;
    }
    else
    {
        double ds = c3_cyl(g, s, kq2, 0);
        if (ds <= 0.) { s->state = OUTSIDE; return 0; }
        s->m = -1;
        s->ds = ds;
        propagater(s, ds + eps);
        if (!c3_indices(g, s)) { s->state = OUTSIDE; return 0; }
    }
    return 1;
}

/* Cylinder2DSpatialGrid::MySegmentGenerator::moveInside (Cylinder2DSpatialGrid.cpp:124-198) */
static int cyl_move_inside(const Grid* g, Gen* s)
{
    const double* Rv = g->crv;
    const double* zv = g->czv;
    int NR = g->cnr, Nz = g->cnz;
    s->cR = sqrt(s->rx * s->rx + s->ry * s->ry);
    s->cz = s->rz;
    s->ckq = sqrt(s->kx * s->kx + s->ky * s->ky);
    s->ckz = s->kz;
    if (s->ckq == 0.0) s->ckq = 1e-20;
    if (s->ckz == 0.0) s->ckz = 1e-20;
    s->cq = (s->rx * s->kx + s->ry * s->ky) / s->ckq;
    double pp = (s->cR - s->cq) * (s->cR + s->cq);
    s->cp = sqrt(0. < pp ? pp : 0.);  /* std::max(0., x) */
    double Rmax = Rv[NR], zmin = zv[0], zmax = zv[Nz];
    s->m = -1;
    s->ds = 0.;
    s->state = OUTSIDE;
    double cumds = 0.;
    if (s->cR >= Rmax)
    {
        if (s->cq > 0.0 || s->cp > Rmax) return 0;
        double qmin = -sqrt((Rmax - s->cp) * (Rmax + s->cp));
        double ds = (qmin - s->cq) / s->ckq;
        s->cq = qmin;
        s->cR = Rmax - 1e-8 * (Rv[NR] - Rv[NR - 1]);
        s->cz += s->ckz * ds;
        cumds += ds;
    }
    if (s->cz < zmin)
    {
        if (s->ckz <= 0.0) return 0;
        double ds = (zmin - s->cz) / s->ckz;
        s->cq += s->ckq * ds;
        s->cR = sqrt(s->cp * s->cp + s->cq * s->cq);
        s->cz = zmin + 1e-8 * (zv[1] - zv[0]);
        cumds += ds;
    }
    else if (s->cz > zmax)
    {
        if (s->ckz >= 0.0) return 0;
        double ds = (zmax - s->cz) / s->ckz;
        s->cq += s->ckq * ds;
        s->cR = sqrt(s->cp * s->cp + s->cq * s->cq);
        s->cz = zmax - 1e-8 * (zv[Nz] - zv[Nz - 1]);
        cumds += ds;
    }
    if (isinf(s->cR) || isnan(s->cR) || isinf(s->cz) || isnan(s->cz)) return 0;
    if (s->cR >= Rmax || s->cz <= zmin || s->cz >= zmax) return 0;
    s->m = -1;
    s->ds = cumds;
    s->state = INSIDE;
    return 1;
}

enum { CYL_UP_IN = 0, CYL_UP_OUT = 1, CYL_DOWN_IN = 2, CYL_DOWN_OUT = 3 };

/* Cylinder2DSpatialGrid::MySegmentGenerator::next (Cylinder2DSpatialGrid.cpp:200-391) */
static int cyl_next(const Grid* g, Gen* s)
{
    const double* Rv = g->crv;
    const double* zv = g->czv;
    int NR = g->cnr, Nz = g->cnz;
    if (s->state == OUTSIDE) return 0;
    if (s->state == UNKNOWN)
    {
        if (!cyl_move_inside(g, s)) return 0;
        s->i = nr_locate(Rv, NR + 1, s->cR);
        s->k = locate_clip(zv, Nz + 1, s->cz);
        if (s->ckz >= 0.)
        {
            s->cphase = CYL_UP_OUT;
            if (s->cq < 0.)
            {
                s->cimin = nr_locate(Rv, NR + 1, s->cp);
                if (s->i > s->cimin) s->cphase = CYL_UP_IN;
            }
        }
        else
        {
            s->cphase = CYL_DOWN_OUT;
            if (s->cq < 0.)
            {
                s->cimin = nr_locate(Rv, NR + 1, s->cp);
                if (s->i > s->cimin) s->cphase = CYL_DOWN_IN;
            }
        }
        if (s->ds > 0.) return 1;
    }
    int up = s->cphase == CYL_UP_IN || s->cphase == CYL_UP_OUT;
    int in = s->cphase == CYL_UP_IN || s->cphase == CYL_DOWN_IN;
    double RN = in ? Rv[s->i] : Rv[s->i + 1];
    double qN = in ? -sqrt((RN - s->cp) * (RN + s->cp)) : sqrt((RN - s->cp) * (RN + s->cp));
    double zN = up ? zv[s->k + 1] : zv[s->k];
    int m = s->i < 0 ? -1 : s->k + Nz * s->i;  /* Cylinder2DSpatialGrid::index */
    double dsq = (qN - s->cq) / s->ckq;
    double dsz = (zN - s->cz) / s->ckz;
    if (dsq < dsz)
    {
        double ds = dsq;
        s->m = m;
        s->ds = ds;
        if (in)
        {
            s->i--;
            s->cq = qN;
            s->cz += s->ckz * ds;
            if (s->i <= s->cimin) s->cphase = up ? CYL_UP_OUT : CYL_DOWN_OUT;
        }
        else
        {
            s->i++;
            if (s->i >= NR)
                s->state = OUTSIDE;
            else
            {
                s->cq = qN;
                s->cz += s->ckz * ds;
            }
        }
    }
    else
    {
        double ds = dsz;
        s->m = m;
        s->ds = ds;
        if (up) s->k++; else s->k--;
        if (up ? s->k >= Nz : s->k < 0)
            s->state = OUTSIDE;
        else
        {
            s->cq += s->ckq * ds;
            s->cz = zN;
        }
    }
    return 1;
}

static int gen_next(const Grid* g, Gen* s)
{
    switch (g->kind)
    {
        case SKGPU_GRID_CARTESIAN: return cart_next(g, s);
        case SKGPU_GRID_OCTREE: return tree_next(g, s);
        case SKGPU_GRID_ADAPTIVE_MESH: return tree_next(g, s);
        case SKGPU_GRID_VORONOI: return vor_next(g, s);
        case SKGPU_GRID_TETRA: return tet_next(g, s);
        case SKGPU_GRID_SPHERE1D: return sph_next(g, s);
        case SKGPU_GRID_CYLINDER2D: return cyl_next(g, s);
        case SKGPU_GRID_SPHERE2D: return sph2_next(g, s);
        case SKGPU_GRID_SPHERE3D: return sph3_next(g, s);
        case SKGPU_GRID_CYLINDER3D: return cyl3_next(g, s);
    }
    return 0;
}

int or_trace_paths(or_ctx* c, int32_t num_rays, const double* rays, int32_t max_segments, int32_t precision,
                   int32_t* count, int32_t* m, double* ds)
{
    (void)precision;
    if (!c->hasGrid) return fail(c, SKGPU_ERR_STATE, "trace: no grid");
    for (int r = 0; r < num_rays; ++r)
    {
        Gen s;
        gen_start(&s, rays + 6 * (size_t)r);
        int n = 0, ovf = 0;
        while (gen_next(&c->g, &s))
        {
            if (n < max_segments)
            {
                m[(size_t)r * max_segments + n] = s.m;
                ds[(size_t)r * max_segments + n] = s.ds;
            }
            else
                ovf = 1;
            ++n;
        }
        count[r] = ovf ? -n : n;
    }
    return SKGPU_OK;
}

/* ------------------------------------------------------------------------------------------- */
/* medium, sources, instruments, options                                                       */
/* ------------------------------------------------------------------------------------------- */

int or_upload_medium(or_ctx* c, int32_t num_cells, const double* number_density)
{
    free(c->dens);
    c->dens = dup(number_density, num_cells * sizeof(double));
    c->numCells = num_cells;
    return SKGPU_OK;
}

int or_upload_dust_mix(or_ctx* c, int32_t num_lambda, const double* lb, const double* se, const double* ss,
                       const double* g)
{
    free(c->mixLb); free(c->mixExt); free(c->mixSca); free(c->mixG);
    c->mixLb = dup(lb, num_lambda * sizeof(double));
    c->mixExt = dup(se, num_lambda * sizeof(double));
    c->mixSca = dup(ss, num_lambda * sizeof(double));
    c->mixG = dup(g, num_lambda * sizeof(double));
    c->nmix = num_lambda;
    return SKGPU_OK;
}

int or_upload_rf_grid(or_ctx* c, int32_t num_bins, int32_t num_borders, const double* borders, const int32_t* ellv)
{
    free(c->rfB); free(c->rfEll);
    c->rfB = dup(borders, num_borders * sizeof(double));
    c->rfEll = dup(ellv, (num_borders + 1) * sizeof(int));
    c->nrf = num_bins;
    c->rfNb = num_borders;
    return SKGPU_OK;
}

int or_upload_sources(or_ctx* c, int32_t num_sources, const skgpu_source* sources, int32_t table_len,
                      const double* table_lambda, const double* table_a, const double* table_b, int32_t radial_len,
                      const double* radial_r, const double* radial_P)
{
    free(c->src); free(c->tabL); free(c->tabA); free(c->tabB); free(c->radR); free(c->radP);
    c->src = dup(sources, num_sources * sizeof(skgpu_source));
    c->nsrc = num_sources;
    c->tabL = dup(table_lambda, table_len * sizeof(double));
    c->tabA = dup(table_a, table_len * sizeof(double));
    c->tabB = dup(table_b, table_len * sizeof(double));
    c->radR = dup(radial_r, radial_len * sizeof(double));
    c->radP = dup(radial_P, radial_len * sizeof(double));
    return SKGPU_OK;
}

int or_upload_instruments(or_ctx* c, int32_t num_instruments, const skgpu_instrument* instruments, int32_t wlg_len,
                          const double* wlg_borders, const int32_t* wlg_ellv)
{
    free_instruments(c);
    c->ninstr = num_instruments;
    c->instr = (Instr*)calloc(num_instruments > 0 ? num_instruments : 1, sizeof(Instr));
    for (int i = 0; i < num_instruments; ++i)
    {
        Instr* in = &c->instr[i];
        in->d = instruments[i];
        in->zfac = 1.;
        in->apR2 = 0.;
        size_t npix = in->d.kind == SKGPU_INSTR_FRAME ? (size_t)in->d.num_pixels_x * in->d.num_pixels_y : 1;
        in->n = npix * in->d.num_wavelength_bins;
        if (in->d.kind == SKGPU_INSTR_FRAME)
            in->ifu = (double*)calloc(in->n, sizeof(double));
        else
            in->sed = (double*)calloc(in->n, sizeof(double));
        if (in->d.record_components) in->comp = (double*)calloc(3 * in->n, sizeof(double));
        if (in->d.record_statistics) in->stats = (double*)calloc(5 * in->n, sizeof(double));
    }
    c->wlgB = dup(wlg_borders, wlg_len * sizeof(double));
    c->wlgEll = dup(wlg_ellv, wlg_len * sizeof(int));
    return SKGPU_OK;
}

/* Instrument::numScatteringLevels with recordComponents (FluxRecorder.cpp:270-292) */
int or_set_instrument_scattering_levels(or_ctx* c, int32_t i, int32_t levels)
{
    if (i < 0 || i >= c->ninstr) return fail(c, SKGPU_ERR_ARG, "levels: bad instrument index");
    Instr* in = &c->instr[i];
    if (!in->comp) return fail(c, SKGPU_ERR_STATE, "levels: instrument does not record components");
    if (levels < 0 || levels > 1000) return fail(c, SKGPU_ERR_ARG, "levels: out of range [0, 1000]");
    free(in->comp);
    in->comp = (double*)calloc((size_t)(3 + levels) * in->n, sizeof(double));
    in->levels = levels;
    return SKGPU_OK;
}

/* BandWavelengthGrid with the bands' TabulatedBand tables (BandWavelengthGrid.cpp, Band.cpp) */
int or_set_instrument_bands(or_ctx* c, int32_t i, int32_t num_bands, const int32_t* sizes, const double* lambda,
                            const double* transmission, const double* width)
{
    if (i < 0 || i >= c->ninstr) return fail(c, SKGPU_ERR_ARG, "bands: bad instrument index");
    Instr* in = &c->instr[i];
    if (num_bands != in->d.num_wavelength_bins) return fail(c, SKGPU_ERR_ARG, "bands: count differs from the instrument's wavelength bins");
    if (!sizes || !lambda || !transmission || !width) return fail(c, SKGPU_ERR_ARG, "bands: missing tables");
    int* beg = (int*)calloc((size_t)num_bands + 1, sizeof(int));
    for (int b = 0; b < num_bands; ++b)
    {
        if (sizes[b] < 2 || !(width[b] > 0))
        {
            free(beg);
            return fail(c, SKGPU_ERR_ARG, "bands: bad table");
        }
        beg[b + 1] = beg[b] + sizes[b];
    }
    free(in->bandBeg); free(in->bandLam); free(in->bandTr); free(in->bandW);
    in->bandBeg = beg;
    in->bandLam = (double*)dup(lambda, (size_t)beg[num_bands] * sizeof(double));
    in->bandTr = (double*)dup(transmission, (size_t)beg[num_bands] * sizeof(double));
    in->bandW = (double*)dup(width, (size_t)num_bands * sizeof(double));
    in->nband = num_bands;
    return SKGPU_OK;
}

/* the observer-frame redshift (FluxRecorder.cpp:377-378) and the SED aperture
   (ApertureInstrument.cpp:25-44) */
int or_set_instrument_observer(or_ctx* c, int32_t i, double redshift, double aperture_radius)
{
    if (i < 0 || i >= c->ninstr) return fail(c, SKGPU_ERR_ARG, "observer: bad instrument index");
    if (!(redshift >= 0.) || !(aperture_radius >= 0.)) return fail(c, SKGPU_ERR_ARG, "observer: bad redshift or radius");
    if (aperture_radius > 0. && c->instr[i].d.kind != SKGPU_INSTR_SED)
        return fail(c, SKGPU_ERR_ARG, "observer: apertures belong to SED instruments");
    c->instr[i].zfac = 1. + redshift;
    c->instr[i].apR2 = aperture_radius * aperture_radius;
    return SKGPU_OK;
}

int or_set_options(or_ctx* c, const skgpu_options* o)
{
    c->opt = *o;
    return SKGPU_OK;
}

/* ------------------------------------------------------------------------------------------- */
/* life cycle                                                                                  */
/* ------------------------------------------------------------------------------------------- */

typedef struct
{
    int m;
    double ds, s, tau;  /* tau: cumulative extinction, or scattering under explicit absorption */
    double tauAbs;      /* cumulative absorption optical depth (explicit absorption), else 0 */
} Seg;

typedef struct
{
    Seg* v;
    int n, cap;
} Path;

typedef struct
{
    int instr, ell, l;
    double w;
} Contrib;

typedef struct
{
    double rx, ry, rz, kx, ky, kz, L, lambda;
    int nscatt, ellMix, ellRF;
    double sext, ssca, g;
    Contrib* contrib;
    int ncontrib, capcontrib;
} Packet;

static int upper_bound(const double* xv, int n, double x)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (x < xv[mid]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

static int wlg_bin(const double* b, int nb, const int* ellv, double lambda) { return ellv[upper_bound(b, nb, lambda)]; }

/* Band::transmission (Band.cpp): NR::interpolateLinLin (NR.hpp:328-331) in the normalised table,
   zero outside it, times the effective width */
static double band_transmission(const double* lv, const double* tv, int size, double width, double lambda)
{
    int index = upper_bound(lv, size, lambda);
    if (index == 0 || index >= size) return 0.;
    double T = tv[index - 1] + ((lambda - lv[index - 1]) / (lv[index] - lv[index - 1])) * (tv[index] - tv[index - 1]);
    return T * width;
}

/* SpecialFunctions::gexp */
static double gexp(double p, double x)
{
    const double q = 1.0 - p;
    if (q == 0.0) return exp(x);
    if (fabs(q) < 1e-3)
    {
        double x2 = x * x;
        return exp(x) * (1.0 - 0.5 * x2 * q + 1.0 / 24.0 * x * x2 * (8.0 + 3.0 * x) * q * q
                         - 1.0 / 48.0 * x2 * x2 * (12.0 + 8.0 * x + x2) * q * q * q);
    }
    return pow(1.0 + q * x, 1.0 / q);
}

/* SpecialFunctions::lnmean (4-argument flavour) */
static double lnmean4(double x1, double x2, double lnx1, double lnx2)
{
    if (x1 > x2)
    {
        double t = x1; x1 = x2; x2 = t;
        t = lnx1; lnx1 = lnx2; lnx2 = t;
    }
    if (x1 <= 0) return 0.;
    double x = x2 / x1 - 1.;
    if (x < 1e-3)
        return x1 / (1. - 1. / 2. * x + 1. / 3. * x * x - 1. / 4. * x * x * x + 1. / 5. * x * x * x * x
                     - 1. / 6. * x * x * x * x * x);
    return (x2 - x1) / (lnx2 - lnx1);
}

/* Lambert W, branch -1 (Halley iteration), used by ExpDiskGeometry::randomCylRadius */
static double lambert_wm1(double x)
{
    if (x >= 0.) return -INFINITY;
    if (x <= -1. / M_E) return -1.;
    double w;
    if (x < -0.25)
    {
        double p = -sqrt(2. * (M_E * x + 1.));
        w = -1. + p - p * p / 3. + 11. / 72. * p * p * p;
    }
    else
    {
        double l1 = log(-x), l2 = log(-l1);
        w = l1 - l2 + l2 / l1;
    }
    for (int it = 0; it < 20; ++it)
    {
        double ew = exp(w), f = w * ew - x, wp1 = w + 1.;
        if (wp1 == 0.) break;
        double dw = f / (ew * wp1 - (w + 2.) * f / (2. * wp1));
        w -= dw;
        if (fabs(dw) <= 1e-15 * fabs(w)) break;
    }
    return w;
}

static void iso_direction(Rng* r, double* kx, double* ky, double* kz)
{
    double theta = acos(2.0 * uniform(r) - 1.0);
    double phi = 2.0 * M_PI * uniform(r);
    const double eps = 1e-8;
    if (theta <= eps) { *kx = 0.; *ky = 0.; *kz = 1.; }
    else if (theta >= M_PI - eps) { *kx = 0.; *ky = 0.; *kz = -1.; }
    else
    {
        double st = sin(theta);
        *kx = st * cos(phi);
        *ky = st * sin(phi);
        *kz = cos(theta);
    }
}

static double expon_cutoff(Rng* r, double xmax)
{
    if (xmax == 0.0) return 0.0;
    if (xmax < 1e-10) return uniform(r) * xmax;
    double c = 1.0 - exp(-xmax);
    for (int guard = 0; guard < 64; ++guard)
    {
        double x = -log(1.0 - uniform(r) * c);
        if (x <= xmax) return x;
    }
    return xmax;
}

static double value_hg(double g, double ct)
{
    double t = 1. + g * g - 2. * g * ct;
    return (1. - g) * (1. + g) / sqrt(t * t * t);
}

static double integral_hg(double g, double ca, double cb)
{
    double ta = sqrt(1. + g * g - 2. * g * ca), tb = sqrt(1. + g * g - 2. * g * cb);
    return (1. - g) * (1. + g) / g * ((tb - ta) / (tb * ta));
}

static double mean_hg(double g, double ct)
{
    const double delta = 4. * M_PI / 180.;
    double theta = acos(fmin(1., fmax(-1., ct)));
    double ca = cos(theta - delta), cb = cos(theta + delta);
    if (theta < delta) return (integral_hg(g, 1., ca) + integral_hg(g, 1., cb)) / (2. - ca - cb);
    if (theta > M_PI - delta) return (integral_hg(g, ca, -1.) + integral_hg(g, cb, -1.)) / (2. + ca + cb);
    return integral_hg(g, ca, cb) / (ca - cb);
}

static void add_contrib(Packet* pk, int i, int ell, int l, double w)
{
    if (pk->ncontrib == pk->capcontrib)
    {
        pk->capcontrib = pk->capcontrib ? 2 * pk->capcontrib : 64;
        pk->contrib = (Contrib*)realloc(pk->contrib, pk->capcontrib * sizeof(Contrib));
    }
    Contrib ct = {i, ell, l, w};
    pk->contrib[pk->ncontrib++] = ct;
}

/* FluxRecorder::recordContributions: group the history's contributions per bin, add w^k */
static void record_contributions(or_ctx* c, Packet* pk)
{
    for (int a = 0; a < pk->ncontrib; ++a)
    {
        if (pk->contrib[a].instr < 0) continue;
        Contrib ca = pk->contrib[a];
        double w = ca.w;
        for (int b = a + 1; b < pk->ncontrib; ++b)
        {
            Contrib* cb = &pk->contrib[b];
            if (cb->instr == ca.instr && cb->ell == ca.ell && cb->l == ca.l)
            {
                w += cb->w;
                cb->instr = -1;
            }
        }
        Instr* in = &c->instr[ca.instr];
        size_t idx = ca.l < 0 ? (size_t)ca.ell
                              : (size_t)ca.l + (size_t)ca.ell * in->d.num_pixels_x * in->d.num_pixels_y;
        double wn = 1.;
        for (int k = 0; k <= 4; ++k)
        {
            in->stats[k * in->n + idx] += wn;
            wn *= w;
        }
    }
    pk->ncontrib = 0;
}

/* MediumSystem::getExtinctionOpticalDepth(pp, inf) for the peel-off packet */
static double observed_tau(or_ctx* c, const Packet* pk, const double* kobs, double Lp)
{
    double taumax = log(Lp) + 745;
    double ray[6] = {pk->rx, pk->ry, pk->rz, kobs[0], kobs[1], kobs[2]};
    Gen s;
    gen_start(&s, ray);
    double tau = 0.;
    while (gen_next(&c->g, &s))
    {
        c->cnt.crossings++;
        if (s.m >= 0)
        {
            tau += pk->sext * c->dens[s.m] * s.ds;
            if (tau >= taumax) return INFINITY;
        }
    }
    return tau;
}

static int frame_pixel(const skgpu_instrument* d, const Packet* pk)
{
    double x = pk->rx, y = pk->ry, z = pk->rz;
    double xpp = -d->sin_phi * x + d->cos_phi * y;
    double ypp = -d->cos_phi * d->cos_theta * x - d->sin_phi * d->cos_theta * y + d->sin_theta * z;
    double xp = d->cos_omega * xpp - d->sin_omega * ypp;
    double yp = d->sin_omega * xpp + d->cos_omega * ypp;
    int i = (int)floor((xp - d->xp_min) / d->xp_size);
    int j = (int)floor((yp - d->yp_min) / d->yp_size);
    if (i < 0 || i >= d->num_pixels_x || j < 0 || j >= d->num_pixels_y) return -1;
    return i + d->num_pixels_x * j;
}

/* peelOffEmission / peelOffScattering + Instrument::detect + FluxRecorder::detect */
static void peel_off(or_ctx* c, Packet* pk, int scattering)
{
    double Lp = 0., tau = 0.;
    int tauKnown = 0;
    const double* kobs = NULL;
    int numScatt = pk->nscatt + (scattering ? 1 : 0);
    for (int i = 0; i < c->ninstr; ++i)
    {
        Instr* in = &c->instr[i];
        if (!in->d.same_observer)
        {
            kobs = in->d.kobs;
            if (scattering)
            {
                double ct = pk->kx * kobs[0] + pk->ky * kobs[1] + pk->kz * kobs[2];
                Lp = pk->L * (fabs(pk->g) > 0.95 ? mean_hg(pk->g, ct) : value_hg(pk->g, ct));
            }
            else
                Lp = pk->L;
            tauKnown = 0;
        }
        int l = in->d.kind == SKGPU_INSTR_FRAME ? frame_pixel(&in->d, pk) : -1;
        if (in->d.kind == SKGPU_INSTR_FRAME && l < 0) continue;
        if (in->d.kind == SKGPU_INSTR_SED && in->apR2 > 0.)
        {
            const skgpu_instrument* d = &in->d;
            double xpp = -d->sin_phi * pk->rx + d->cos_phi * pk->ry;
            double ypp = -d->cos_phi * d->cos_theta * pk->rx - d->sin_phi * d->cos_theta * pk->ry + d->sin_theta * pk->rz;
            if (xpp * xpp + ypp * ypp > in->apR2) continue;
        }
        const double lambda = pk->lambda * in->zfac;
        /* WavelengthGrid::bins and ::transmission: one disjoint bin with transmission 1, or every band
           whose table range holds the wavelength (FluxRecorder.cpp:380-384) */
        int nb = in->nband ? in->nband : 1;
        for (int b = 0; b < nb; ++b)
        {
            int ell;
            double L = Lp;
            if (!in->nband)
            {
                ell = wlg_bin(c->wlgB + in->d.wlg_offset, in->d.wlg_num_borders, c->wlgEll + in->d.wlg_offset, lambda);
                if (ell < 0) continue;
            }
            else
            {
                ell = b;
                const double* lv = in->bandLam + in->bandBeg[b];
                int size = in->bandBeg[b + 1] - in->bandBeg[b];
                if (!(lambda >= lv[0] && lambda <= lv[size - 1])) continue;
                L = Lp * band_transmission(lv, in->bandTr + in->bandBeg[b], size, in->bandW[b], lambda);
            }
            if (!tauKnown)
            {
                tau = observed_tau(c, pk, kobs, Lp);
                tauKnown = 1;
            }
            double Lext = L * exp(-tau);
            c->cnt.peel_detections++;
            size_t idx = in->d.kind == SKGPU_INSTR_FRAME ? (size_t)l + (size_t)ell * in->d.num_pixels_x * in->d.num_pixels_y
                                                         : (size_t)ell;
            double* total = in->d.kind == SKGPU_INSTR_FRAME ? in->ifu : in->sed;
            total[idx] += Lext;
            if (in->d.record_components)
            {
                if (numScatt == 0)
                {
                    in->comp[idx] += L;
                    in->comp[in->n + idx] += Lext;
                }
                else
                {
                    in->comp[2 * in->n + idx] += Lext;
                    /* PrimaryScatteredLevel + numScatt - 1, primary packets only (FluxRecorder.cpp:430-433) */
                    if (numScatt <= in->levels && !c->secRun) in->comp[(size_t)(2 + numScatt) * in->n + idx] += Lext;
                }
            }
            if (in->d.record_statistics) add_contrib(pk, i, ell, l, Lext);
        }
    }
}

static void path_build(or_ctx* c, const Packet* pk, Path* path)
{
    double ray[6] = {pk->rx, pk->ry, pk->rz, pk->kx, pk->ky, pk->kz};
    Gen s;
    gen_start(&s, ray);
    path->n = 0;
    double scum = 0., tau = 0., tauAbs = 0.;
    double sabs = pk->sext - pk->ssca;
    while (gen_next(&c->g, &s))
    {
        c->cnt.crossings++;
        if (s.ds > 0.)
        {
            if (path->n == path->cap)
            {
                path->cap = path->cap ? 2 * path->cap : 1024;
                path->v = (Seg*)realloc(path->v, path->cap * sizeof(Seg));
            }
            scum += s.ds;
            if (c->opt.explicit_absorption)
            {
                /* MediumSystem::setScatteringAndAbsorptionOpticalDepths (MediumSystem.cpp:1899-1913) */
                if (s.m >= 0)
                {
                    double ns = c->dens[s.m] * s.ds;
                    tau += pk->ssca * ns;
                    tauAbs += sabs * ns;
                }
            }
            else if (s.m >= 0)
                tau += pk->sext * c->dens[s.m] * s.ds;
            Seg sg = {s.m, s.ds, scum, tau, tauAbs};
            path->v[path->n++] = sg;
        }
    }
}

static void launch_secondary(or_ctx* c, Rng* r, uint64_t hist, Packet* pk);

static void launch(or_ctx* c, Rng* r, uint64_t hist, Packet* pk)
{
    if (c->secRun)
    {
        launch_secondary(c, r, hist, pk);
        return;
    }
    int h = 0;
    for (int q = 1; q < c->nsrc; ++q)
        if (c->src[q].first_history <= hist) h = q;
    const skgpu_source* S = &c->src[h];
    rng_start(r, c->opt.seed, hist);
    pk->nscatt = 0;
    double L = S->packet_luminosity, lambda;
    if (S->spectral_model == SKGPU_SPEC_DISCRETE)
    {
        int j = (int)(uniform(r) * S->table_size);
        if (j > S->table_size - 1) j = S->table_size - 1;
        lambda = c->tabL[S->table_offset + j];
        L *= c->tabA[S->table_offset + j];
    }
    else
    {
        const double* lv = c->tabL + S->table_offset;
        const double* pv = c->tabA + S->table_offset;
        const double* Pv = c->tabB + S->table_offset;
        int n = S->table_size;
        double xi = S->wavelength_bias;
        int fromSed = (xi <= 0.) || (uniform(r) > xi);
        if (fromSed)
        {
            double X = uniform(r);
            int i = locate_clip(Pv, n, X);
            double alpha = log(pv[i + 1] / pv[i]) / log(lv[i + 1] / lv[i]);
            lambda = lv[i] * gexp(-alpha, (X - Pv[i]) / (pv[i] * lv[i]));
        }
        else
        {
            double lmin = log(S->bias_lambda_min), lw = log(S->bias_lambda_max) - log(S->bias_lambda_min);
            lambda = exp(lmin + lw * uniform(r));
        }
        if (xi > 0.)
        {
            double s = 0.;
            if (lambda >= lv[0] && lambda <= lv[n - 1])
            {
                int i = upper_bound(lv, n, lambda) - 1;
                if (i > n - 2) i = n - 2;
                if (i < 0) i = 0;
                double a = log(pv[i + 1] / pv[i]) / log(lv[i + 1] / lv[i]);
                s = pv[i] * pow(lambda / lv[i], a);
            }
            double b = (lambda >= S->bias_lambda_min && lambda <= S->bias_lambda_max)
                           ? 1. / ((log(S->bias_lambda_max) - log(S->bias_lambda_min)) * lambda)
                           : 0.;
            L *= (s > 0.) ? s / ((1 - xi) * s + xi * b) : 0.;
        }
    }
    pk->lambda = lambda;
    pk->L = L;
    if (S->position_model == SKGPU_SRC_POINT)
    {
        pk->rx = S->position[0]; pk->ry = S->position[1]; pk->rz = S->position[2];
    }
    else if (S->position_model == SKGPU_SRC_EXPDISK)
    {
        double hR = S->geometry[0], hz = S->geometry[1], Rmin = S->geometry[2], Rmax = S->geometry[3], zmax = S->geometry[4];
        double R = 0., z = 0.;
        for (int t = 0; t < 1000; ++t)
        {
            double X = uniform(r);
            R = hR * (-1.0 - lambert_wm1((X - 1.0) / M_E));
            if (!((Rmax > 0.0 && R >= Rmax) || R <= Rmin)) break;
        }
        double phi = 2.0 * M_PI * uniform(r);
        for (int t = 0; t < 1000; ++t)
        {
            double X = uniform(r);
            z = (X <= 0.5) ? hz * log(2.0 * X) : -hz * log(2.0 * (1.0 - X));
            if (!(zmax > 0.0 && fabs(z) >= zmax)) break;
        }
        pk->rx = S->position[0] + R * cos(phi);
        pk->ry = S->position[1] + R * sin(phi);
        pk->rz = S->position[2] + z;
    }
    else
    {
        double X = uniform(r);
        const double* rv = c->radR + S->radial_offset;
        const double* Pv = c->radP + S->radial_offset;
        double rr;
        if (S->position_model == SKGPU_SRC_RADIAL_LOGLOG)
        {
            /* SersicGeometry::randomRadius (SersicGeometry.cpp:41-45): reff * SersicFunction::inverseMass(X),
               i.e. NR::clampedValue<NR::interpolateLogLog>(X, _Mv, _sv) (NR.hpp:349-358, 394-401) */
            rr = S->geometry[0] * clamped_loglog(Pv, rv, S->radial_size, X);
        }
        else
        {
            int i = locate_clip(Pv, S->radial_size, X);
            rr = rv[i] + (X - Pv[i]) / (Pv[i + 1] - Pv[i]) * (rv[i + 1] - rv[i]);
        }
        double ux, uy, uz;
        iso_direction(r, &ux, &uy, &uz);
        pk->rx = S->position[0] + rr * ux;
        pk->ry = S->position[1] + rr * uy;
        pk->rz = S->position[2] + rr * uz;
    }
    iso_direction(r, &pk->kx, &pk->ky, &pk->kz);
    pk->ellMix = locate_clip(c->mixLb, c->nmix, lambda);
    if (pk->ellMix < 0) pk->ellMix = 0;
    pk->sext = c->mixExt[pk->ellMix];
    pk->ssca = c->mixSca[pk->ellMix];
    pk->g = c->mixG[pk->ellMix];
    pk->ellRF = c->opt.store_radiation_field ? wlg_bin(c->rfB, c->rfNb, c->rfEll, lambda) : -1;
}

static double albedo(or_ctx* c, const Packet* pk, int m)
{
    double n = c->dens[m];
    double ksca = n > 0. ? n * pk->ssca : 0.;
    double kext = n > 0. ? n * pk->sext : 0.;
    return kext > 0. ? ksca / kext : 0.;
}

static void scatter(or_ctx* c, Rng* r, Packet* pk)
{
    double g = pk->g;
    if (fabs(g) < 1e-6)
        iso_direction(r, &pk->kx, &pk->ky, &pk->kz);
    else
    {
        double f = ((1.0 - g) * (1.0 + g)) / (1.0 - g + 2.0 * g * uniform(r));
        double costheta = (1.0 + g * g - f * f) / (2.0 * g);
        /* Random::direction(bfk, costheta) */
        double phi = 2.0 * M_PI * uniform(r);
        double cosphi = cos(phi), sinphi = sin(phi);
        double sintheta = sqrt(fabs((1.0 - costheta) * (1.0 + costheta)));
        double kx = pk->kx, ky = pk->ky, kz = pk->kz, nx, ny, nz;
        if (kz > 0.99999)
        {
            nx = cosphi * sintheta; ny = sinphi * sintheta; nz = costheta;
        }
        else if (kz < -0.99999)
        {
            nx = cosphi * sintheta; ny = sinphi * sintheta; nz = -costheta;
        }
        else
        {
            double root = sqrt((1.0 - kz) * (1.0 + kz));
            nx = sintheta / root * (-kx * kz * cosphi + ky * sinphi) + kx * costheta;
            ny = -sintheta / root * (ky * kz * cosphi + kx * sinphi) + ky * costheta;
            nz = root * sintheta * cosphi + kz * costheta;
        }
        pk->kx = nx; pk->ky = ny; pk->kz = nz;
    }
    pk->nscatt++;
    c->cnt.scatterings++;
}

static void life_cycle(or_ctx* c, uint64_t hist, Path* path, Packet* pk)
{
    Rng rng;
    launch(c, &rng, hist, pk);
    c->cnt.histories++;
    pk->ncontrib = 0;
    if (!(pk->L > 0)) return;
    int peel = c->opt.peel_off && c->ninstr > 0;
    if (peel) peel_off(c, pk, 0);
    if (c->opt.force_scattering)
    {
        double Lthreshold = pk->L / c->opt.min_weight_reduction;
        while (1)
        {
            path_build(c, pk, path);
            /* storeRadiationField */
            if (c->opt.store_radiation_field && pk->ellRF >= 0)
            {
                double lnExtBeg = 0., extBeg = 1.;
                for (int q = 0; q < path->n; ++q)
                {
                    /* Segment::tauExt = tauExtOrSca + tauAbs (SpatialGridPath.hpp:108) */
                    double lnExtEnd = -(path->v[q].tau + path->v[q].tauAbs), extEnd = exp(lnExtEnd);
                    int m = path->v[q].m;
                    if (m >= 0)
                    {
                        double extMean = lnmean4(extEnd, extBeg, lnExtEnd, lnExtBeg);
                        c->rf[(size_t)m * c->nrf + pk->ellRF] += pk->L * extMean * path->v[q].ds;
                        c->cnt.rf_stores++;
                    }
                    lnExtBeg = lnExtEnd;
                    extBeg = extEnd;
                }
            }
            /* simulateForcedPropagation */
            double taupath = path->n ? path->v[path->n - 1].tau : 0.;
            if (taupath <= 0.)
            {
                pk->L *= 0.;
            }
            else
            {
                double xi = c->opt.path_length_bias, tau;
                if (xi == 0.)
                    tau = expon_cutoff(&rng, taupath);
                else
                {
                    tau = uniform(&rng) < xi ? uniform(&rng) * taupath : expon_cutoff(&rng, taupath);
                    double p = -exp(-tau) / expm1(-taupath);
                    double q = (1.0 - xi) * p + xi / taupath;
                    pk->L *= p / q;
                }
                /* SpatialGridPath::findInteractionPoint */
                int lo = 0, hi = path->n;
                while (lo < hi)
                {
                    int mid = (lo + hi) >> 1;
                    if (tau < path->v[mid].tau) hi = mid; else lo = mid + 1;
                }
                int m;
                double s, tauAbs;
                if (lo < path->n)
                {
                    double t0 = lo ? path->v[lo - 1].tau : 0., s0 = lo ? path->v[lo - 1].s : 0.;
                    double a0 = lo ? path->v[lo - 1].tauAbs : 0.;
                    m = path->v[lo].m;
                    s = s0 + ((tau - t0) / (path->v[lo].tau - t0)) * (path->v[lo].s - s0);
                    tauAbs = a0 + ((tau - t0) / (path->v[lo].tau - t0)) * (path->v[lo].tauAbs - a0);
                }
                else
                {
                    m = path->v[path->n - 1].m;
                    s = path->v[path->n - 1].s;
                    tauAbs = path->v[path->n - 1].tauAbs;
                }
                if (m < 0)
                {
                    c->errFlag |= 2;
                    break;
                }
                /* MonteCarloSimulation.cpp:1529-1540 */
                if (c->opt.explicit_absorption)
                    pk->L *= -expm1(-taupath) * exp(-tauAbs);
                else
                    pk->L *= -expm1(-taupath) * albedo(c, pk, m);
                pk->rx += s * pk->kx;
                pk->ry += s * pk->ky;
                pk->rz += s * pk->kz;
            }
            if (pk->L <= 0 || (pk->L <= Lthreshold && pk->nscatt >= c->opt.min_scatt_events)) break;
            if (peel) peel_off(c, pk, 1);
            scatter(c, &rng, pk);
        }
    }
    else
    {
        while (1)
        {
            /* simulateNonForcedPropagation with setInteractionPointUsingExtinction */
            double tauinteract = -log(uniform(&rng));
            double ray[6] = {pk->rx, pk->ry, pk->rz, pk->kx, pk->ky, pk->kz};
            Gen s;
            gen_start(&s, ray);
            double tau = 0., sc = 0.;
            int found = 0, m = -1;
            double sInt = 0.;
            while (gen_next(&c->g, &s))
            {
                c->cnt.crossings++;
                double t0 = tau, s0 = sc;
                /* explicit absorption: MediumSystem::setInteractionPointUsingScatteringAndAbsorption
                   (MediumSystem.cpp:2203-2222) walks on the scattering optical depth */
                if (s.m >= 0) tau += (c->opt.explicit_absorption ? pk->ssca : pk->sext) * c->dens[s.m] * s.ds;
                sc += s.ds;
                if (tauinteract < tau)
                {
                    m = s.m;
                    sInt = s0 + ((tauinteract - t0) / (tau - t0)) * (sc - s0);
                    found = 1;
                    break;
                }
            }
            if (!found) break;
            if (m < 0)
            {
                c->errFlag |= 2;
                break;
            }
            /* MonteCarloSimulation::simulateNonForcedPropagation (MonteCarloSimulation.cpp:2001-2022) */
            if (c->opt.explicit_absorption)
                pk->L *= exp(-(tauinteract * (pk->sext - pk->ssca) / pk->ssca));
            else
                pk->L *= albedo(c, pk, m);
            pk->rx += sInt * pk->kx;
            pk->ry += sInt * pk->ky;
            pk->rz += sInt * pk->kz;
            if (pk->L <= 0) break;
            if (peel) peel_off(c, pk, 1);
            scatter(c, &rng, pk);
        }
    }
    if (pk->ncontrib) record_contributions(c, pk);
}

/* ------------------------------------------------------------------------------------------------
 * secondary (dust) emission
 * ------------------------------------------------------------------------------------------------ */

static double* dupd(const double* p, size_t n) { return (double*)dup(p, n * sizeof(double)); }

int or_upload_dust_emission(or_ctx* c, int32_t num_rf, const double* rf_sigma_abs, const double* rf_width,
                            const double* rf_cmb, const double* rf_sigma_abs_lum, int32_t num_T, const double* T,
                            const double* planck_abs, int32_t num_em, const double* em_lambda,
                            const double* em_sigma_abs, const double* em_range, int32_t num_cells,
                            const double* cell_volume)
{
    if (num_rf < 1 || num_T < 2 || num_em < 2 || num_cells < 1) return fail(c, SKGPU_ERR_ARG, "dust emission: missing tables");
    free(c->deRfSig); free(c->deRfW); free(c->deRfCmb); free(c->deRfSigL); free(c->deT); free(c->dePlanck);
    free(c->deEmL); free(c->deEmSig); free(c->deVol);
    c->deRfSig = dupd(rf_sigma_abs, num_rf);
    c->deRfW = dupd(rf_width, num_rf);
    c->deRfCmb = dupd(rf_cmb, num_rf);
    c->deRfSigL = dupd(rf_sigma_abs_lum, num_rf);
    c->deT = dupd(T, num_T);
    c->dePlanck = dupd(planck_abs, num_T);
    c->deEmL = dupd(em_lambda, num_em);
    c->deEmSig = dupd(em_sigma_abs, num_em);
    c->deVol = dupd(cell_volume, num_cells);
    c->deEmRange[0] = em_range[0];
    c->deEmRange[1] = em_range[1];
    c->deNrf = num_rf; c->deNT = num_T; c->deNem = num_em; c->deCells = num_cells;
    c->secPackets = 0;
    return SKGPU_OK;
}

int or_upload_radiation_field(or_ctx* c, const double* rf)
{
    if (!c->nrf || !c->numCells) return fail(c, SKGPU_ERR_STATE, "radiation field: no medium or RF grid uploaded");
    size_t len = (size_t)c->numCells * c->nrf;
    if (c->rfLen != len)
    {
        free(c->rf);
        c->rf = (double*)calloc(len, sizeof(double));
        c->rfLen = len;
    }
    memcpy(c->rf, rf, len * sizeof(double));
    return SKGPU_OK;
}

/* NR::interpolateLogLog (SKIRT/utils/NR.hpp:349-358) */
static double interp_loglog(double x, double x1, double x2, double f1, double f2)
{
    if (f1 <= 0 || f2 <= 0)
    {
        if (x == x1) return f1;
        if (x == x2) return f2;
        return 0;
    }
    return f1 * exp(log(x / x1) / log(x2 / x1) * (log(f2 / f1)));
}

/* SpecialFunctions::gln (SKIRT/utils/SpecialFunctions.cpp:798-811) */
static double gln(double p, double x)
{
    const double q = 1.0 - p;
    if (q == 0.0) return log(x);
    if (fabs(q) < 1e-3)
    {
        double lnx = log(x);
        double s = q * lnx;
        return lnx * (1.0 + 0.5 * s + 1.0 / 6.0 * s * s + 1.0 / 24.0 * s * s * s);
    }
    return (pow(x, q) - 1.0) / q;
}

/* PlanckFunction (SKIRT/utils/PlanckFunction.cpp:12-27) with the constants of SKIRT/utils/Constants.hpp */
static double planck_value(double T, double lambda)
{
    const double h = 6.62606957e-34, cc = 2.99792458e8, k = 1.3806488e-23;
    double f1 = h * cc / (k * T);
    double f2 = 2.0 * h * cc * cc;
    return f2 / pow(lambda, 5) / (exp(f1 / lambda) - 1.0);
}

/* std::upper_bound / std::lower_bound indices */
static int ub_index(const double* v, int n, double x)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        int mid = (lo + hi) / 2;
        if (x < v[mid]) hi = mid; else lo = mid + 1;
    }
    return lo;
}
static int lb_index(const double* v, int n, double x)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        int mid = (lo + hi) / 2;
        if (v[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

int or_prepare_secondary(or_ctx* c, const skgpu_secondary_options* opt, uint64_t total_packets, double* luminosity)
{
    if (!opt || total_packets == 0) return fail(c, SKGPU_ERR_ARG, "secondary: missing options or packets");
    if (!c->hasGrid || (c->g.kind != SKGPU_GRID_CARTESIAN && c->g.kind != SKGPU_GRID_OCTREE
                        && c->g.kind != SKGPU_GRID_ADAPTIVE_MESH && c->g.kind != SKGPU_GRID_TETRA
                        && (c->g.kind < SKGPU_GRID_SPHERE1D || c->g.kind > SKGPU_GRID_CYLINDER3D)
                        && !(c->g.kind == SKGPU_GRID_VORONOI && c->g.vbox)))
        return fail(c, SKGPU_ERR_UNSUPPORTED, "secondary: a Voronoi grid needs its cell boxes (or_upload_voronoi_cell_boxes)");
    if (!c->deNrf || c->deCells != c->numCells || c->deNrf != c->nrf)
        return fail(c, SKGPU_ERR_STATE, "secondary: dust emission tables do not match the medium and RF grid");
    if (!c->rf || c->rfLen != (size_t)c->numCells * c->nrf) return fail(c, SKGPU_ERR_STATE, "secondary: no radiation field");
    const int cells = c->numCells, nrf = c->nrf;
    /* the spectrum axis of NR::cdf (NR.hpp:494-520) */
    int minRight = ub_index(c->deEmL, c->deNem, c->deEmRange[0]);
    int maxRight = lb_index(c->deEmL, c->deNem, c->deEmRange[1]);
    int nb = 1 + maxRight - minRight, npts = nb + 1;
    free(c->secL); free(c->secT); free(c->secXv); free(c->secPv); free(c->secCv); free(c->secLv); free(c->secWv);
    free(c->secIv);
    c->secL = (double*)calloc(cells, sizeof(double));
    c->secT = (double*)calloc(cells, sizeof(double));
    c->secXv = (double*)calloc(npts, sizeof(double));
    c->secPv = (double*)calloc((size_t)cells * npts, sizeof(double));
    c->secCv = (double*)calloc((size_t)cells * npts, sizeof(double));
    c->secLv = (double*)calloc(cells, sizeof(double));
    c->secWv = (double*)calloc(cells, sizeof(double));
    c->secIv = (uint64_t*)calloc((size_t)cells + 1, sizeof(uint64_t));
    c->secCells = cells;
    c->secNpts = npts;
    c->secPackets = 0;
    free(c->secCellNode);
    c->secCellNode = NULL;
    if (c->g.kind == SKGPU_GRID_OCTREE || c->g.kind == SKGPU_GRID_ADAPTIVE_MESH)
    {
        c->secCellNode = (int*)calloc(cells, sizeof(int));
        for (int q = 0; q < c->g.tnodes; ++q)
            if (c->g.tcell[q] >= 0 && c->g.tcell[q] < cells) c->secCellNode[c->g.tcell[q]] = q;
    }
    double* xv = c->secXv;
    xv[0] = c->deEmRange[0];
    for (int j = minRight, i = 1; j < maxRight; ++j, ++i) xv[i] = c->deEmL[j];
    xv[nb] = c->deEmRange[1];
    double* ev = (double*)malloc(c->deNem * sizeof(double));
    for (int m = 0; m < cells; ++m)
    {
        double n = c->dens[m];
        /* MediumSystem::dustLuminosity (MediumSystem.cpp:2752-2762) with DustMix::opacityAbs */
        double Labs = 0.;
        for (int ell = 0; ell < nrf; ++ell)
        {
            double op = n > 0. ? n * c->deRfSigL[ell] : 0.;
            Labs += op * c->rf[(size_t)m * nrf + ell];
        }
        c->secL[m] = Labs;
        /* MediumSystem::meanIntensity (MediumSystem.cpp:2670-2680) and
           EquilibriumDustEmissionCalculator::equilibriumTemperature (EquilibriumDustEmissionCalculator.cpp:
           118-128): the valarray expression's sum() runs from the last element to the first */
        double factor = 1. / (4. * M_PI * c->deVol[m]);
        double inputabs = 0.;
        for (int k = nrf - 1; k >= 0; --k)
        {
            double J = c->rf[(size_t)m * nrf + k] * factor / c->deRfW[k];
            double term = c->deRfSig[k] * (J + c->deRfCmb[k]) * c->deRfW[k];
            inputabs = (k == nrf - 1) ? term : inputabs + term;
        }
        double T = 0.;
        if (inputabs > 0.)
        {
            int i = locate_nr(c->dePlanck, c->deNT, inputabs);
            if (i < 0) T = c->deT[0];
            else if (i >= c->deNT - 1) T = c->deT[c->deNT - 1];
            else
            {
                double x1 = c->dePlanck[i], x2 = c->dePlanck[i + 1], f1 = c->deT[i], f2 = c->deT[i + 1];
                T = f1 + ((inputabs - x1) / (x2 - x1)) * (f2 - f1);
            }
        }
        /* the reported temperature is MediumSystem::indicativeDustTemperature's: 0 without dust */
        c->secT[m] = n > 0. ? T : 0.;
        /* emissivity (EquilibriumDustEmissionCalculator.cpp:132-148) times the number density
           (DustMix::emissionSpectrum), then NR::cdf<NR::interpolateLogLog> and NR::cdf2 (NR.cpp:25-53) */
        for (int j = 0; j < c->deNem; ++j) ev[j] = n * (c->deEmSig[j] * planck_value(T, c->deEmL[j]));
        double* p = c->secPv + (size_t)m * npts;
        double* P = c->secCv + (size_t)m * npts;
        p[0] = minRight == 0 ? 0. : interp_loglog(xv[0], c->deEmL[minRight - 1], c->deEmL[minRight], ev[minRight - 1], ev[minRight]);
        for (int i = 1; i < nb; ++i) p[i] = ev[minRight + i - 1];
        p[nb] = maxRight == c->deNem ? 0. : interp_loglog(xv[nb], c->deEmL[maxRight - 1], c->deEmL[maxRight], ev[maxRight - 1], ev[maxRight]);
        P[0] = 0.;
        for (int i = 0; i < nb; ++i)
        {
            double area = 0.;
            if (p[i] > 0 && p[i + 1] > 0)
            {
                double alpha = log(p[i + 1] / p[i]) / log(xv[i + 1] / xv[i]);
                area = p[i] * xv[i] * gln(-alpha, xv[i + 1] / xv[i]);
            }
            P[i + 1] = P[i] + area;
        }
        double norm = P[nb];
        if (norm > 0.)
            for (int i = 0; i <= nb; ++i)
            {
                p[i] /= norm;
                P[i] /= norm;
            }
    }
    free(ev);
    /* DustSecondarySource::prepareLuminosities / preparePacketMap (DustSecondarySource.cpp:27-152) with
       the AllCellsLibrary, SecondarySourceSystem::prepareForLaunch (SecondarySourceSystem.cpp:62-104)
       with the dust source alone */
    double L = c->secL[0];
    for (int m = 1; m < cells; ++m) L += c->secL[m];
    if (luminosity) *luminosity = L;
    if (!(L > 0.)) return SKGPU_OK;
    for (int m = 0; m < cells; ++m) c->secLv[m] = c->secL[m] / L;
    double xi = opt->spatial_bias;
    double* wv = (double*)malloc(cells * sizeof(double));
    for (int m = 0; m < cells; ++m) wv[m] = c->secLv[m] > 0 ? 1. : 0.;
    double ws = wv[0];
    for (int m = 1; m < cells; ++m) ws += wv[m];
    for (int m = 0; m < cells; ++m) wv[m] /= ws;
    for (int m = 0; m < cells; ++m) c->secWv[m] = (1 - xi) * c->secLv[m] + xi * wv[m];
    free(wv);
    uint64_t N = total_packets;
    c->secIv[0] = 0;
    double W = 0.;
    for (int p = 1; p != cells; ++p)
    {
        W += c->secWv[p - 1];
        uint64_t r = (uint64_t)round(W * (double)N);
        c->secIv[p] = r < N ? r : N;
    }
    c->secIv[cells] = N;
    double xs = opt->source_bias;
    double Ws = (1 - xs) * 1. / 1. + xs * 1. / 1.;
    c->secLpk = (L / (double)N) * (1. / Ws);
    c->secXi = opt->wavelength_bias;
    c->secBmin = opt->bias_lambda_min;
    c->secBmax = opt->bias_lambda_max;
    c->secLogMin = opt->wavelength_bias > 0. ? log(c->secBmin) : 0.;
    c->secLogWidth = opt->wavelength_bias > 0. ? log(c->secBmax) - log(c->secBmin) : 0.;
    c->secPackets = N;
    /* the uploaded radiation field is consumed: the tally starts empty for a segment storing its own */
    if (c->rf) memset(c->rf, 0, c->rfLen * sizeof(double));
    return SKGPU_OK;
}

int or_fetch_dust_emission(or_ctx* c, double* luminosity, double* temperature, int32_t* num_points, double* lambda,
                           double* pdf, double* cdf)
{
    if (!c->secCells || c->secCells != c->numCells) return fail(c, SKGPU_ERR_STATE, "fetch: no prepared dust emission");
    size_t cells = c->secCells, rows = cells * c->secNpts;
    if (num_points) *num_points = c->secNpts;
    if (luminosity) memcpy(luminosity, c->secL, cells * sizeof(double));
    if (temperature) memcpy(temperature, c->secT, cells * sizeof(double));
    if (lambda) memcpy(lambda, c->secXv, c->secNpts * sizeof(double));
    if (pdf) memcpy(pdf, c->secPv, rows * sizeof(double));
    if (cdf) memcpy(cdf, c->secCv, rows * sizeof(double));
    return SKGPU_OK;
}

/* SecondarySourceSystem::launch -> DustSecondarySource::launch / launchFromCell
   (SecondarySourceSystem.cpp:118-133, DustSecondarySource.cpp:521-626; Random::cdfLogLog, Random.cpp:199-205;
   Random::position, Random.cpp:168-176; Box::fracPos, Box.hpp:142-145) */
static void launch_secondary(or_ctx* c, Rng* r, uint64_t hist, Packet* pk)
{
    rng_start(r, c->opt.seed ^ SKGPU_SECONDARY_KEY, hist);
    pk->nscatt = 0;
    int cells = c->secCells;
    int m = 0;
    {
        int lo = 0, hi = cells + 1;
        while (lo < hi)
        {
            int mid = (lo + hi) / 2;
            if (hist < c->secIv[mid]) hi = mid; else lo = mid + 1;
        }
        m = lo - 1;
        if (m < 0) m = 0;
        if (m > cells - 1) m = cells - 1;
    }
    double ws = c->secLv[m] / c->secWv[m];
    const int n = c->secNpts;
    const double* xv = c->secXv;
    const double* pv = c->secPv + (size_t)m * n;
    const double* Pv = c->secCv + (size_t)m * n;
    double lambda, w;
    int fromSpectrum = 1;
    if (c->secXi)
        fromSpectrum = uniform(r) > c->secXi;
    if (fromSpectrum)
    {
        double X = uniform(r);
        int i = locate_clip(Pv, n, X);
        double alpha = log(pv[i + 1] / pv[i]) / log(xv[i + 1] / xv[i]);
        lambda = xv[i] * gexp(-alpha, (X - Pv[i]) / (pv[i] * xv[i]));
    }
    else
        lambda = exp(c->secLogMin + c->secLogWidth * uniform(r));
    if (!c->secXi)
        w = 1.;
    else
    {
        /* NR::value<NR::interpolateLogLog> (NR.hpp:371-377) with NR::locateFail */
        double s = 0.;
        if (!(lambda > xv[n - 1]))
        {
            int jl = -1, ju = n - 1;
            while (ju - jl > 1)
            {
                int jm = (ju + jl) >> 1;
                if (lambda < xv[jm]) ju = jm; else jl = jm;
            }
            if (jl >= 0) s = interp_loglog(lambda, xv[jl], xv[jl + 1], pv[jl], pv[jl + 1]);
        }
        if (!s)
            w = 0.;
        else
        {
            double b = (lambda >= c->secBmin * (1 - 1e-14) && lambda <= c->secBmax * (1 + 1e-14)) ? 1. / (c->secLogWidth * lambda) : 0.;
            w = s / ((1 - c->secXi) * s + c->secXi * b);
        }
    }
    /* a random position in cell m (SpatialGrid::randomPositionInCell of the grid kind) */
    if (c->g.kind == SKGPU_GRID_TETRA)
    {
        /* TetraMeshSpatialGrid::Tetra::generatePosition / generateBarycentric (TetraMeshSpatialGrid.cpp:140-173) */
        double s = uniform(r);
        double t = uniform(r);
        double u = uniform(r);
        if (s + t > 1.)
        {
            s = 1. - s;
            t = 1. - t;
        }
        if (t + u > 1.)
        {
            double tmp = u;
            u = 1. - s - t;
            t = 1. - tmp;
        }
        else if (s + t + u > 1.)
        {
            double tmp = u;
            u = s + t + u - 1.;
            s = 1. - t - tmp;
        }
        double b = 1. - u - t - s;
        const double *v0 = te_vertex(&c->g, m, 0), *v1 = te_vertex(&c->g, m, 1), *v2 = te_vertex(&c->g, m, 2),
                     *v3 = te_vertex(&c->g, m, 3);
        pk->rx = b * v0[0] + u * v1[0] + t * v2[0] + s * v3[0];
        pk->ry = b * v0[1] + u * v1[1] + t * v2[1] + s * v3[1];
        pk->rz = b * v0[2] + u * v1[2] + t * v2[2] + s * v3[2];
    }
    else if (c->g.kind == SKGPU_GRID_SPHERE1D)
    {
        /* Sphere1DSpatialGrid::randomPositionInCell (Sphere1DSpatialGrid.cpp:80-91) */
        double ux, uy, uz;
        iso_direction(r, &ux, &uy, &uz);
        double r0 = c->g.srv[m], r1 = c->g.srv[m + 1];
        double rad = cbrt(r0 * r0 * r0 + (r1 - r0) * (r1 * r1 + r1 * r0 + r0 * r0) * uniform(r));
        pk->rx = rad * ux;
        pk->ry = rad * uy;
        pk->rz = rad * uz;
    }
    else if (c->g.kind == SKGPU_GRID_VORONOI)
    {
        /* VoronoiMeshSnapshot::generatePosition / isPointClosestTo (VoronoiMeshSnapshot.cpp:879-887, 1007-1020) */
        const Grid* g = &c->g;
        const double* bb = g->vbox + 6 * (size_t)m;
        const double* sm = g->vs + 3 * (size_t)m;
        for (int tries = 0; tries < 10000; ++tries)
        {
            double fx = uniform(r);
            double fy = uniform(r);
            double fz = uniform(r);
            pk->rx = bb[0] + fx * (bb[3] - bb[0]);
            pk->ry = bb[1] + fy * (bb[4] - bb[1]);
            pk->rz = bb[2] + fz * (bb[5] - bb[2]);
            double dx = pk->rx - sm[0], dy = pk->ry - sm[1], dz = pk->rz - sm[2];
            double target = dx * dx + dy * dy + dz * dz;
            int closest = 1;
            for (int e = g->vnbb[m]; e < g->vnbb[m + 1] && closest; ++e)
            {
                int id = g->vnb[e];
                if (id < 0) continue;
                const double* q = g->vs + 3 * (size_t)id;
                double ex = pk->rx - q[0], ey = pk->ry - q[1], ez = pk->rz - q[2];
                if (ex * ex + ey * ey + ez * ez < target) closest = 0;
            }
            if (closest) break;
        }
    }
    else if (c->g.kind == SKGPU_GRID_CYLINDER2D || c->g.kind == SKGPU_GRID_CYLINDER3D)
    {
        /* Cylinder2DSpatialGrid.cpp:95-106, Cylinder3DSpatialGrid.cpp:133-144; Position.cpp:21-29 */
        const Grid* g = &c->g;
        int i, j = 0, k;
        const double *Rv, *zv;
        if (g->kind == SKGPU_GRID_CYLINDER2D) { i = m / g->cnz; k = m % g->cnz; Rv = g->crv; zv = g->czv; }
        else { i = m / (g->c3np * g->c3nz); j = (m / g->c3nz) % g->c3np; k = m % g->c3nz; Rv = g->c3r; zv = g->c3z; }
        double R0 = Rv[i], R1 = Rv[i + 1], z0 = zv[k], z1 = zv[k + 1];
        double R = sqrt(R0 * R0 + (R1 - R0) * (R1 + R0) * uniform(r));
        double phi = g->kind == SKGPU_GRID_CYLINDER2D ? 2.0 * M_PI * uniform(r)
                                                       : g->c3p[j] + (g->c3p[j + 1] - g->c3p[j]) * uniform(r);
        double z = z0 + (z1 - z0) * uniform(r);
        pk->rx = R * cos(phi);
        pk->ry = R * sin(phi);
        pk->rz = z;
    }
    else if (c->g.kind == SKGPU_GRID_SPHERE2D || c->g.kind == SKGPU_GRID_SPHERE3D)
    {
        /* Sphere2DSpatialGrid.cpp:102-113, Sphere3DSpatialGrid.cpp:146-157; Position.cpp:30-43 */
        const Grid* g = &c->g;
        int i, j, k = 0;
        const double *rv, *tv;
        if (g->kind == SKGPU_GRID_SPHERE2D) { i = m / g->s2nt; j = m % g->s2nt; rv = g->s2r; tv = g->s2t; }
        else { i = m / (g->s3nt * g->s3np); j = (m / g->s3np) % g->s3nt; k = m % g->s3np; rv = g->s3r; tv = g->s3t; }
        double r0 = rv[i], r1 = rv[i + 1];
        double rad = cbrt(r0 * r0 * r0 + (r1 - r0) * (r1 * r1 + r1 * r0 + r0 * r0) * uniform(r));
        double theta = acos(cos(tv[j]) + (cos(tv[j + 1]) - cos(tv[j])) * uniform(r));
        double phi = g->kind == SKGPU_GRID_SPHERE2D ? 2.0 * M_PI * uniform(r)
                                                     : g->s3p[k] + (g->s3p[k + 1] - g->s3p[k]) * uniform(r);
        double st = sin(theta);
        pk->rx = rad * st * cos(phi);
        pk->ry = rad * st * sin(phi);
        pk->rz = rad * cos(theta);
    }
    else
    {
        double b0, b1, b2, b3, b4, b5;
        if (c->g.kind == SKGPU_GRID_CARTESIAN)
        {
            int i = m / (c->g.nz * c->g.ny), j = (m / c->g.nz) % c->g.ny, k = m % c->g.nz;
            b0 = c->g.xb[i]; b1 = c->g.yb[j]; b2 = c->g.zb[k];
            b3 = c->g.xb[i + 1]; b4 = c->g.yb[j + 1]; b5 = c->g.zb[k + 1];
        }
        else
        {
            const double* bb = c->g.tb + 6 * (size_t)c->secCellNode[m];
            b0 = bb[0]; b1 = bb[1]; b2 = bb[2]; b3 = bb[3]; b4 = bb[4]; b5 = bb[5];
        }
        double fx = uniform(r);
        double fy = uniform(r);
        double fz = uniform(r);
        pk->rx = b0 + fx * (b3 - b0);
        pk->ry = b1 + fy * (b4 - b1);
        pk->rz = b2 + fz * (b5 - b2);
    }
    iso_direction(r, &pk->kx, &pk->ky, &pk->kz);
    pk->lambda = lambda;
    pk->L = c->secLpk * ws * w;
    pk->ellMix = locate_clip(c->mixLb, c->nmix, lambda);
    if (pk->ellMix < 0) pk->ellMix = 0;
    pk->sext = c->mixExt[pk->ellMix];
    pk->ssca = c->mixSca[pk->ellMix];
    pk->g = c->mixG[pk->ellMix];
    pk->ellRF = c->opt.store_radiation_field ? wlg_bin(c->rfB, c->rfNb, c->rfEll, lambda) : -1;
}

int or_run_secondary(or_ctx* c, uint64_t first, uint64_t count)
{
    if (!c->secPackets || c->secCells != c->numCells)
        return fail(c, SKGPU_ERR_STATE, "secondary: no prepared segment (or_prepare_secondary)");
    if (!c->nmix) return fail(c, SKGPU_ERR_STATE, "secondary: no dust mix uploaded");
    if (first + count > c->secPackets) return fail(c, SKGPU_ERR_ARG, "secondary: history range outside the segment");
    if (c->opt.store_radiation_field && c->nrf)
    {
        size_t len = (size_t)c->numCells * c->nrf;
        if (c->rfLen != len)
        {
            free(c->rf);
            c->rf = (double*)calloc(len, sizeof(double));
            c->rfLen = len;
        }
    }
    memset(&c->cnt, 0, sizeof c->cnt);
    c->errFlag = 0;
    c->secRun = 1;
    Path path = {NULL, 0, 0};
    Packet pk;
    memset(&pk, 0, sizeof pk);
    for (uint64_t h = first; h < first + count; ++h) life_cycle(c, h, &path, &pk);
    free(path.v);
    free(pk.contrib);
    c->secRun = 0;
    if (c->errFlag) return fail(c, SKGPU_ERR_DEVICE, "run: interaction point outside the grid");
    return SKGPU_OK;
}

int or_probe_launch(or_ctx* c, uint64_t first, uint64_t count, uint64_t total_packets, double* out)
{
    if (!c->nsrc || !c->nmix) return fail(c, SKGPU_ERR_STATE, "probe_launch: no sources or dust mix uploaded");
    if (total_packets == 0 || first + count > total_packets) return fail(c, SKGPU_ERR_ARG, "probe_launch: history range outside the segment");
    Packet pk;
    memset(&pk, 0, sizeof pk);
    for (uint64_t t = 0; t < count; ++t)
    {
        Rng r;
        launch(c, &r, first + t, &pk);
        double* o = out + 8 * t;
        o[0] = pk.lambda;
        o[1] = pk.L * (double)total_packets;
        o[2] = pk.rx; o[3] = pk.ry; o[4] = pk.rz;
        o[5] = pk.kx; o[6] = pk.ky; o[7] = pk.kz;
    }
    free(pk.contrib);
    return SKGPU_OK;
}

int or_run_primary(or_ctx* c, uint64_t first, uint64_t count, uint64_t total_packets)
{
    if (!c->hasGrid || !c->dens || !c->nmix || !c->nsrc) return fail(c, SKGPU_ERR_STATE, "run: incomplete scene");
    if (first + count > total_packets) return fail(c, SKGPU_ERR_ARG, "run: history range outside the segment");
    if (c->opt.store_radiation_field)
    {
        size_t len = (size_t)c->numCells * c->nrf;
        if (c->rfLen != len)
        {
            free(c->rf);
            c->rf = (double*)calloc(len, sizeof(double));
            c->rfLen = len;
        }
    }
    memset(&c->cnt, 0, sizeof c->cnt);
    c->errFlag = 0;
    Path path = {NULL, 0, 0};
    Packet pk;
    memset(&pk, 0, sizeof pk);
    for (uint64_t h = first; h < first + count; ++h) life_cycle(c, h, &path, &pk);
    free(path.v);
    free(pk.contrib);
    c->cnt.kernel_launches = 0;
    if (c->errFlag) return fail(c, SKGPU_ERR_DEVICE, "run: interaction point outside the grid");
    return SKGPU_OK;
}

static void add_into(const double* src, size_t n, double* dst)
{
    if (!src || !dst) return;
    for (size_t i = 0; i < n; ++i) dst[i] += src[i];
}

int or_fetch_instrument(or_ctx* c, int32_t i, double* ifu, double* sed, double* ifu_stats, double* sed_stats)
{
    if (i < 0 || i >= c->ninstr) return fail(c, SKGPU_ERR_ARG, "fetch: bad instrument index");
    Instr* in = &c->instr[i];
    if (in->d.kind == SKGPU_INSTR_FRAME)
    {
        add_into(in->ifu, in->n, ifu);
        add_into(in->stats, 5 * in->n, ifu_stats);
    }
    else
    {
        add_into(in->sed, in->n, sed);
        add_into(in->stats, 5 * in->n, sed_stats);
    }
    return SKGPU_OK;
}

int or_fetch_instrument_components(or_ctx* c, int32_t i, double* ifu3, double* sed3)
{
    if (i < 0 || i >= c->ninstr) return fail(c, SKGPU_ERR_ARG, "fetch: bad instrument index");
    Instr* in = &c->instr[i];
    if (!in->comp) return fail(c, SKGPU_ERR_STATE, "fetch: instrument does not record components");
    add_into(in->comp, 3 * in->n, in->d.kind == SKGPU_INSTR_FRAME ? ifu3 : sed3);
    return SKGPU_OK;
}

/* FluxRecorder::calibrateAndWrite's scaling (FluxRecorder.cpp:97-115, 891-921) */
int or_calibrate_instrument(or_ctx* c, int32_t i, const double* factors)
{
    if (i < 0 || i >= c->ninstr) return fail(c, SKGPU_ERR_ARG, "calibrate: bad instrument index");
    if (!factors) return fail(c, SKGPU_ERR_ARG, "calibrate: missing factors");
    Instr* in = &c->instr[i];
    size_t npix = in->d.kind == SKGPU_INSTR_FRAME ? (size_t)in->d.num_pixels_x * in->d.num_pixels_y : 1;
    size_t n = in->n;
    double* total = in->d.kind == SKGPU_INSTR_FRAME ? in->ifu : in->sed;
    for (size_t q = 0; q < n; ++q) total[q] *= factors[q / npix];
    if (in->comp)
        for (size_t q = 0; q < (size_t)(3 + in->levels) * n; ++q) in->comp[q] *= factors[(q % n) / npix];
    return SKGPU_OK;
}

int or_fetch_instrument_levels(or_ctx* c, int32_t i, double* ifu_levels, double* sed_levels)
{
    if (i < 0 || i >= c->ninstr) return fail(c, SKGPU_ERR_ARG, "fetch: bad instrument index");
    Instr* in = &c->instr[i];
    if (!in->comp || in->levels < 1) return fail(c, SKGPU_ERR_STATE, "fetch: instrument records no scattering levels");
    add_into(in->comp + 3 * in->n, (size_t)in->levels * in->n, in->d.kind == SKGPU_INSTR_FRAME ? ifu_levels : sed_levels);
    return SKGPU_OK;
}

int or_fetch_radiation_field(or_ctx* c, double* rf)
{
    if (!c->rf) return fail(c, SKGPU_ERR_STATE, "fetch: no radiation field recorded");
    add_into(c->rf, c->rfLen, rf);
    return SKGPU_OK;
}

int or_clear_tallies(or_ctx* c)
{
    for (int i = 0; i < c->ninstr; ++i)
    {
        Instr* in = &c->instr[i];
        if (in->ifu) memset(in->ifu, 0, in->n * sizeof(double));
        if (in->sed) memset(in->sed, 0, in->n * sizeof(double));
        if (in->comp) memset(in->comp, 0, (size_t)(3 + in->levels) * in->n * sizeof(double));
        if (in->stats) memset(in->stats, 0, 5 * in->n * sizeof(double));
    }
    if (c->rf) memset(c->rf, 0, c->rfLen * sizeof(double));
    return SKGPU_OK;
}

int or_get_counters(or_ctx* c, skgpu_counters* out)
{
    *out = c->cnt;
    return SKGPU_OK;
}

int or_last_run_ms(or_ctx* c, double* ms)
{
    (void)c;
    *ms = 0.;
    return SKGPU_OK;
}

int or_optical_depths(or_ctx* c, int32_t num_rays, const double* rays, double lambda, int32_t precision, double* tau)
{
    (void)precision;
    if (!c->hasGrid || !c->dens || !c->nmix) return fail(c, SKGPU_ERR_STATE, "optical depths: incomplete scene");
    int ell = locate_clip(c->mixLb, c->nmix, lambda);
    double section = c->mixExt[ell < 0 ? 0 : ell];
    for (int r = 0; r < num_rays; ++r)
    {
        Gen s;
        gen_start(&s, rays + 6 * (size_t)r);
        double t = 0.;
        while (gen_next(&c->g, &s))
        {
            if (s.m >= 0)
            {
                t += section * c->dens[s.m] * s.ds;
                if (t >= 745.)
                {
                    t = INFINITY;
                    break;
                }
            }
        }
        tau[r] = t;
    }
    return SKGPU_OK;
}

/* C struct sizes of the ABI records, for the binding layout test */
int or_sizeof_source(void) { return (int)sizeof(skgpu_source); }
int or_sizeof_instrument(void) { return (int)sizeof(skgpu_instrument); }
int or_sizeof_options(void) { return (int)sizeof(skgpu_options); }
int or_sizeof_counters(void) { return (int)sizeof(skgpu_counters); }
