"""CPU tests of the standalone Delaunay builder (skgpu_tetra_build): on the reference's own mesh
fixture it gives TetGen's tetrahedra up to the box-face diagonals (the box corners are cocircular,
so either split of a box face is Delaunay), with the reference's conventions; on random points the
tetrahedra fill the box exactly with consistent neighbours."""
import numpy as np

from skgpu import abi


def _volumes(t):
    p = t["vertices"][t["tetra"]]
    return np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0])) / 6


def _conventions(t):
    T, V = t["tetra"], t["vertices"]
    for k in range(0, len(T), max(1, len(T) // 500)):
        for f in range(4):
            cv = [(f + 3) % 4, (f + 2) % 4, (f + 1) % 4]
            if f % 2 == 0:
                cv[0], cv[2] = cv[2], cv[0]
            a = V[T[k, cv[0]]]
            # outward unit normal: the opposite vertex lies behind the face
            assert np.isclose(np.linalg.norm(t["normals"][k, f]), 1.0)
            assert np.dot(V[T[k, f]] - a, t["normals"][k, f]) < 0
            j, g = t["ntetra"][k, f], t["nface"][k, f]
            if j >= 0:
                assert t["ntetra"][j, g] == k and t["nface"][j, g] == f
                assert set(T[k]) - {T[k, f]} == set(T[j]) - {T[j, g]}


def test_matches_the_reference_tetgen_mesh(golden):
    z = golden("paths_tetra.npz")
    V = z["tet_vertices"].reshape(-1, 3)
    ext = z["grid_extent"]
    corner = np.any(np.isclose(np.abs(V), ext[3], rtol=0, atol=1e-6 * ext[3]), axis=1)
    t = abi.build_tetra(V[~corner], ext)
    ref_tets = z["tet_tetra"].reshape(-1, 4)
    assert len(t["tetra"]) == len(ref_tets)
    q = lambda x: tuple(np.round((x - ext[:3]) / (ext[3:] - ext[:3]) * 2 ** 20).astype(np.int64))
    key = lambda verts, tets: {tuple(sorted(q(verts[v]) for v in tt)) for tt in tets}
    ref, our = key(V, ref_tets), key(t["vertices"], t["tetra"])
    assert len(ref ^ our) <= 0.01 * len(ref)  # the box-face diagonals may differ
    vol = _volumes(t)
    assert vol.min() > 0 and np.isclose(vol.sum(), np.prod(ext[3:] - ext[:3]), rtol=1e-12)
    assert (t["ntetra"] < 0).sum() == 12
    _conventions(t)


def test_random_points_fill_the_box():
    rng = np.random.default_rng(4)
    pts = rng.uniform(-0.99, 0.99, size=(20000, 3))
    t = abi.build_tetra(pts, [-1, -1, -1, 1, 1, 1])
    vol = _volumes(t)
    assert vol.min() > 0 and np.isclose(vol.sum(), 8.0, rtol=1e-12)
    assert 6.4 < len(t["tetra"]) / len(pts) < 6.9  # Poisson-Delaunay: 6.77 tetrahedra per point
    assert (t["ntetra"] < 0).sum() == 12
    _conventions(t)


def test_points_outside_or_repeated_are_left_out():
    """As TetraMeshSpatialGrid::removeInvalid: points outside the box (or on its surface) and repeated
    points are dropped; the kept points come first, in input order, then the 8 corners."""
    rng = np.random.default_rng(9)
    pts = rng.uniform(-0.9, 0.9, size=(3000, 3))
    bad = np.array([[1.5, 0, 0], [0, -1.0, 0], [0.2, 0.3, 1.0]])
    allp = np.concatenate([pts[:1000], bad, pts[:10], pts[1000:]])
    t = abi.build_tetra(allp, [-1, -1, -1, 1, 1, 1])
    assert len(t["vertices"]) == len(pts) + 8
    assert np.allclose(t["vertices"][:len(pts)], pts, atol=2.0 / 2 ** 20)
    vol = _volumes(t)
    assert vol.min() > 0 and np.isclose(vol.sum(), 8.0, rtol=1e-12)
    _conventions(t)
