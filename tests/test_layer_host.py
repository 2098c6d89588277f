"""Host-side set-up of the learned absorbing layer (no GPU): the map from
the thin domain's nodes to the thick domain's, and which nodes carry a
correction, with which face frame and network."""

import numpy as np
import pytest

from gfb import layer as gl


@pytest.fixture(scope="module")
def pair():
    p = gl.PairSpec(ni=3, nj=3, nk=2, d=250.0, seed=5, src=(375.0, 375.0, 250.0), nsteps=10, stride=5, n_thick=3)
    thin, thick, m = gl.build_pair(p)
    return p, thin, thick, m


def test_node_map_matches_positions(pair):
    p, thin, thick, m = pair
    a = gl._node_coords(thin) + np.array([(p.n_thick - p.n_thin) * p.d] * 2 + [0.0])
    b = gl._node_coords(thick)[m]
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-6)
    assert np.unique(m).size == m.size  # one thick node per thin node
    assert thin["dt"] == thick["dt"]


def test_layer_nodes_default_is_the_truncation_surface(pair):
    _, thin, _, _ = pair
    node, frame, net, n_net = gl.layer_nodes(thin)
    ng = thin["ngll"]
    X = gl._node_coords(thin)[node]
    b = thin["bounds"]
    on = (np.isclose(X[:, 0], b["xmin"]) | np.isclose(X[:, 0], b["xmax"]) | np.isclose(X[:, 1], b["ymin"])
          | np.isclose(X[:, 1], b["ymax"]) | np.isclose(X[:, 2], b["zmax"]))
    assert on.all()
    # every node of the five absorbing faces, once
    Xa = gl._node_coords(thin)
    all_on = (np.isclose(Xa[:, 0], b["xmin"]) | np.isclose(Xa[:, 0], b["xmax"]) | np.isclose(Xa[:, 1], b["ymin"])
              | np.isclose(Xa[:, 1], b["ymax"]) | np.isclose(Xa[:, 2], b["zmax"]))
    assert node.size == int(all_on.sum()) and np.unique(node).size == node.size
    assert n_net == 2 * ng
    assert set(np.unique(net)) <= {ng - 1, 2 * ng - 1}  # side / bottom at the outer plane
    # the outward normal of the frame points out of the face the node is on
    for q in range(node.size):
        ax = abs(int(frame[q, 0])) - 1
        sgn = np.sign(frame[q, 0])
        lo, hi = b["xmin ymin zmin".split()[ax]], b["xmax ymax zmax".split()[ax]]
        assert np.isclose(X[q, ax], hi if sgn > 0 else lo)
        assert sorted(abs(int(v)) for v in frame[q]) == [1, 2, 3]


def test_layer_nodes_all_planes_take_the_deepest_face(pair):
    _, thin, _, _ = pair
    ng = thin["ngll"]
    node, frame, net, _ = gl.layer_nodes(thin, planes=range(ng))
    plane = net % ng
    bottom = net // ng
    X = gl._node_coords(thin)[node]
    b, d = thin["bounds"], thin["spec"].dx
    # bottom-layer nodes sit in the bottom element, side nodes in a side one
    assert np.all(X[bottom == 1, 2] >= b["zmax"] - d - 1e-9)
    near = np.minimum.reduce([X[:, 0] - b["xmin"], b["xmax"] - X[:, 0], X[:, 1] - b["ymin"], b["ymax"] - X[:, 1]])
    assert np.all(near[bottom == 0] <= d + 1e-9)
    # deeper planes are nearer the truncation surface
    dist_out = np.where(bottom == 1, b["zmax"] - X[:, 2], near)
    for k in range(ng - 1):
        if np.any(plane == k) and np.any(plane == k + 1):
            assert dist_out[plane == k].min() > dist_out[plane == k + 1].max() - 1e-9
