"""Mixed-element mesh grouping (host side): cells split by a seeded
permutation into hexes, prism pairs and tet sextets, one collection per
(shape, P), every kept cell in exactly one collection."""
import numpy as np

from nektar_b200.mixed_mesh import MixedMesh


def test_groups_partition_the_kept_cells():
    mm = MixedMesh(n=6, ncells=(60, 50, 40), pmin=2, pmax=5, seed=3)
    per_shape = {"hex": [], "prism": [], "tet": []}
    for shape, p, cells in mm.groups:
        assert 2 <= p <= 5 and len(cells) > 0
        assert np.all(np.diff(cells) > 0)
        per_shape[shape].extend(cells.tolist())
    assert [len(per_shape[s]) for s in ("hex", "prism", "tet")] == [60, 50, 40]
    allc = sum(per_shape.values(), [])
    assert len(set(allc)) == 150 and max(allc) < 216


def test_grouping_is_seeded():
    a = MixedMesh(n=6, ncells=(60, 50, 40), pmin=2, pmax=5, seed=3)
    b = MixedMesh(n=6, ncells=(60, 50, 40), pmin=2, pmax=5, seed=3)
    c = MixedMesh(n=6, ncells=(60, 50, 40), pmin=2, pmax=5, seed=4)
    key = lambda m: [(s, p, tuple(x)) for s, p, x in m.groups]
    assert key(a) == key(b) and key(a) != key(c)


def test_element_counts_per_collection():
    mm = MixedMesh(n=4, ncells=(10, 8, 6), pmin=2, pmax=3, seed=1)
    per = {"hex": 1, "prism": 2, "tet": 6}
    for (shape, p, cells), m in zip(mm.groups, mm.meshes()):
        assert m.nelmt == per[shape] * len(cells)
        assert m.nm == p + 1 and m.nq[0] == p + 2
