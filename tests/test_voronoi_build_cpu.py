"""CPU tests of the standalone Voronoi neighbour builder (skgpu_voronoi_build): on the reference's
own mesh fixture it reproduces the neighbour sets that voro++ gave SKIRT, and on random sites the
neighbour relation is symmetric with about 15.5 neighbours per cell (Poisson-Voronoi)."""
import numpy as np

from skgpu import abi


def test_neighbour_sets_equal_the_reference_mesh(golden):
    z = golden("paths_voronoi.npz")
    sites, ext = z["vor_sites"].reshape(-1, 3), z["grid_extent"]
    b, ix = abi.build_voronoi(sites, ext)
    rb, rix = z["vor_nb_begin"], z["vor_nb_index"]
    for i in range(len(sites)):
        assert set(ix[b[i]:b[i + 1]]) == set(rix[rb[i]:rb[i + 1]]), i


def test_random_sites_symmetric_and_poisson_like():
    rng = np.random.default_rng(3)
    n = 20000
    s = rng.uniform(-1, 1, size=(n, 3))
    b, ix = abi.build_voronoi(s, [-1, -1, -1, 1, 1, 1], threads=4)
    owner = np.repeat(np.arange(n), np.diff(b))
    m = ix >= 0
    a = owner[m].astype(np.int64) * n + ix[m]
    rev = ix[m].astype(np.int64) * n + owner[m]
    assert np.isin(rev, a).all()
    interior = np.all(np.abs(s) < 0.7, axis=1)
    mean_nb = (np.diff(b)[interior]).mean()
    assert 15.0 < mean_nb < 16.0  # Poisson-Voronoi cells have 15.54 faces on average
    assert np.all(ix >= -6) and np.all(ix < n)
