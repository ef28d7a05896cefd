"""The synthetic mesh generator against the oracle's restatement of buildMesh
(solver.cc:2185-2418), and the benchmark shapes' sizes."""
import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po


@pytest.mark.parametrize("cells", [(8, 8, 8), (3, 5, 2), (16, 8, 8), (1, 1, 1)])
def test_generator_matches_the_build_mesh_restatement(cells):
    o = po.build_grid(cells, voxel=0.1, jitter=0.01, seed=7)
    p = tb.box_mesh(cells, voxel=0.1, jitter=0.01, seed=7)
    assert np.array_equal(o.tet_nodes, p.tet_nodes)          # node numbering, Kuhn split, orientation
    assert np.array_equal(o.rest, p.rest_positions)           # float-rounded jittered rest positions
    assert np.array_equal(o.anchored, p.anchored)
    assert np.abs(o.rest_inverse - p.rest_inverse).max() <= 1e-12 * np.abs(o.rest_inverse).max()
    assert np.abs(o.volume - p.volume).max() <= 1e-12 * o.volume.max()
    assert np.abs(o.node_mass - p.node_mass).max() <= 1e-12 * o.node_mass.max()
    assert np.array_equal(o.lattice(), p.lattice)


@pytest.mark.parametrize("cells,nodes,tets", [((8, 8, 8), 729, 3072), ((16, 16, 16), 4913, 24576),
                                              ((64, 32, 32), 70785, 393216)])
def test_benchmark_shapes(cells, nodes, tets):
    m = tb.box_mesh(cells)
    assert (m.nodes, m.tets) == (nodes, tets)
    assert np.all(m.volume > 0)
    # the masses add up to rho * volume of the block (rest positions are float-rounded)
    assert m.node_mass.sum() == pytest.approx(1000.0 * np.prod(cells) * 1e-3, rel=1e-6)
    assert m.node_mass.sum() == pytest.approx(1000.0 * m.volume.sum(), rel=1e-12)


def test_kuhn_tets_fill_each_cell_once_with_positive_orientation():
    m = tb.box_mesh((3, 2, 2), voxel=0.1, jitter=0.02, seed=5)
    x = m.rest_positions[m.tet_nodes]
    det = np.linalg.det(np.stack([x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]], axis=2))
    assert np.all(det > 0)
    assert np.allclose(np.linalg.inv(np.stack([x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]], axis=2)),
                       m.rest_inverse)
    # every tet uses the cell's 0-7 diagonal: 6 tets per cell share exactly two nodes
    for c in range(12):
        t = m.tet_nodes[6 * c:6 * c + 6]
        shared = set(t[0])
        for row in t[1:]:
            shared &= set(row)
        assert len(shared) == 2


def test_node_order_is_first_use_in_x_fastest_cell_order():
    m = tb.box_mesh((2, 2, 1))
    lat = [tuple(v) for v in m.lattice[:8]]
    assert lat == [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    assert tuple(m.lattice[8]) == (2, 0, 0)


def test_anchor_faces():
    m = tb.box_mesh((4, 3, 2))
    assert m.anchored.sum() == 5 * 3   # y = 0 face: (4+1) x (2+1) nodes
    assert np.all(m.lattice[m.anchored != 0, 1] == 0)
    assert m.face(1, 1).sum() == 15
