"""CPU tests of the standalone octree builder (skgpu_octree_build): the exported arrays must form a
valid TreeSpatialGrid-like octree whose neighbour lists follow the reference's conventions, and the
oracle must traverse it consistently."""
import numpy as np
import pytest

from skgpu import Scene, abi

PC = 3.08567758e16


@pytest.fixture(scope="module")
def tree():
    h = 4 * PC
    return abi.build_octree(abi.GEOM_EXPDISK, [1 * PC, 0.2 * PC, 0, 0, 0], [-h, -h, -h, h, h, h], 2, 6, 1e-3, seed=3)


def test_leaves_tile_the_domain(tree):
    b = tree["bounds"]
    leaf = tree["cell_index"] >= 0
    vol = np.prod(b[leaf, 3:] - b[leaf, :3], axis=1).sum()
    assert vol == pytest.approx(np.prod(b[0, 3:] - b[0, :3]), rel=1e-12)
    assert sorted(tree["cell_index"][leaf]) == list(range(leaf.sum()))
    assert len(tree["density"]) == leaf.sum()


def test_children_are_consecutive_octants(tree):
    b, cb, cc, ci = tree["bounds"], tree["child_begin"], tree["child_count"], tree["child_index"]
    for l in np.nonzero(cc)[0][:500]:
        kids = ci[cb[l]:cb[l] + 8]
        assert list(kids) == list(range(kids[0], kids[0] + 8))
        c = 0.5 * (b[l, :3] + b[l, 3:])
        assert np.allclose(b[kids[0], 3:], c)  # first child's upper corner is the split point


def test_neighbour_lists_touch_the_wall_and_are_overlap_sorted(tree):
    b, nbb, nbi = tree["bounds"], tree["nb_begin"], tree["nb_index"]
    leaves = np.nonzero(tree["cell_index"] >= 0)[0]
    for l in leaves[:: max(1, len(leaves) // 400)]:
        for wall in range(6):
            axis, upper = wall // 2, wall % 2
            lst = nbi[nbb[6 * l + wall]:nbb[6 * l + wall + 1]]
            u, w = [a for a in range(3) if a != axis]
            areas = []
            for n in lst:
                face = b[l, 3 + axis] if upper else b[l, axis]
                other = b[n, axis] if upper else b[n, 3 + axis]
                assert face == other
                du = max(min(b[l, 3 + u], b[n, 3 + u]) - max(b[l, u], b[n, u]), 0)
                dw = max(min(b[l, 3 + w], b[n, 3 + w]) - max(b[l, w], b[n, w]), 0)
                areas.append(du * dw)
            assert areas == sorted(areas, reverse=True)


def test_oracle_traverses_built_tree(tree, oracle_backend):
    sc = Scene()
    sc.grid = dict(kind=abi.GRID_OCTREE, eps=1e-12 * 8 * PC * np.sqrt(3), **{k: tree[k] for k in (
        "bounds", "cell_index", "child_begin", "child_count", "child_index", "nb_begin", "nb_index")})
    sc.upload(oracle_backend)
    rng = np.random.default_rng(5)
    rays = np.hstack([rng.uniform(-4 * PC, 4 * PC, (200, 3)), rng.normal(size=(200, 3))])
    rays[:, 3:] /= np.linalg.norm(rays[:, 3:], axis=1)[:, None]
    count, m, ds = oracle_backend.trace_paths(rays, 4096)
    assert (count > 0).all()
    for r in range(len(rays)):
        cells = m[r, :count[r]]
        assert (cells[1:] >= 0).all()
        # path length inside the box equals the chord length
        assert ds[r, :count[r]][cells >= 0].sum() > 0
