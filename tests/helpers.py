"""Shared checks for the parity tests."""
import numpy as np

from conftest import segments_of


def compare_paths(z, count, m, ds):
    """Bit-exact comparison of traced segments with a golden path fixture; returns mismatching rays."""
    bad = []
    ref_cnt = z["ray_count"]
    for r in range(len(ref_cnt)):
        rm, rds = segments_of(z, r)
        if count[r] != ref_cnt[r] or not np.array_equal(m[r, :count[r]], rm) or not np.array_equal(ds[r, :count[r]], rds):
            bad.append(r)
    return bad


def zscores(w1a, w2a, na, w1b, w2b, nb, mask=None):
    """Per-bin z-scores of two Monte Carlo estimates given their sums of w and w^2 over histories
    (per-history contributions, FluxRecorder statistics): var(sum w) = sum w^2 - (sum w)^2 / N."""
    va = np.maximum(w2a - w1a * w1a / na, 0)
    vb = np.maximum(w2b - w1b * w1b / nb, 0)
    if mask is None:
        mask = (w1a > 0) | (w1b > 0)
    den = np.sqrt(va + vb)[mask]
    ok = den > 0
    return ((w1a - w1b)[mask][ok]) / den[ok]


def median_relative_error(stats, n):
    """Median over bins with flux of R = sqrt(sum w^2 / (sum w)^2 - 1/N) (FluxRecorder statistics)."""
    w1, w2 = stats[1], stats[2]
    m = w1 > 0
    return float(np.median(np.sqrt(np.maximum(w2[m] / w1[m] ** 2 - 1.0 / n, 0))))


def tetra_hull_edge_exits(z, rel=1e-9):
    """Rays of a tetrahedral path fixture that leave the mesh's convex hull through an edge or a
    vertex of its boundary triangulation: two or more boundary faces hold the exit point. There the
    reference's own exit decision (TetraMeshSpatialGrid.cpp:750-766, the plane fallback when a
    Plucker product is exactly zero) compares two equal distances, and the rounding of its FP64
    position picks the face."""
    V, T, N, NT = z["tet_vertices"], z["tet_tetra"], z["tet_normals"], z["tet_ntetra"]
    ext = z["grid_extent"]
    tol = rel * np.sqrt(((ext[3:] - ext[:3]) ** 2).sum())
    faces = [(t, f) for t, f in zip(*np.nonzero(NT < 0))]
    tri = np.array([[V[T[t, v]] for v in range(4) if v != f] for t, f in faces])
    nrm = np.array([N[t, f] for t, f in faces])
    out = set()
    for r, ray in enumerate(z["rays"]):
        p0, k = ray[:3], ray[3:]
        nk = nrm @ k
        ahead = nk > 0
        dist = np.full(len(faces), np.inf)
        dist[ahead] = np.einsum("ij,ij->i", nrm[ahead], tri[ahead, 0] - p0) / nk[ahead]
        t_exit = dist.min()
        if not np.isfinite(t_exit):
            continue
        p = p0 + k * t_exit
        held = 0
        for q in np.nonzero(np.abs(dist - t_exit) <= tol)[0]:
            a, b, c = tri[q]
            # barycentric containment with a tolerance of rel
            n = np.cross(b - a, c - a)
            area = n @ n
            wa = np.cross(c - b, p - b) @ n / area
            wb = np.cross(a - c, p - c) @ n / area
            wc = 1.0 - wa - wb
            if min(wa, wb, wc) >= -rel:
                held += 1
        if held >= 2:
            out.add(r)
    return out
