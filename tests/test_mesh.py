"""Host mesh builder: neighbour tables, 2:1 balance, SFC order, geometry and static fields."""
import numpy as np
import pytest

from discrete_adjoint_b200 import inputs
from discrete_adjoint_b200.mesh import Mesh, MeshSpec, Pile


def check_mesh(m: Mesh, lx: float, ly: float):
    n = m.n
    # cells tile the domain
    assert np.isclose((m.dx * m.dy).sum(), lx * ly, rtol=1e-12)
    # neighbours: geometric adjacency and reciprocity
    for s in range(4):
        d = s & 1
        sign = 1 if s < 2 else -1
        for k in (s, s + 4):
            e = m.nbr[k]
            ok = e >= 0
            assert np.array_equal(ok, m.nbr[s] >= 0)
            co, sz = (m.x, m.dx) if d == 0 else (m.y, m.dy)
            ot, osz = (m.y, m.dy) if d == 0 else (m.x, m.dx)
            i = np.nonzero(ok)[0]
            gap = sign * (co[e[i]] - co[i]) - 0.5 * (sz[e[i]] + sz[i])
            assert np.allclose(gap, 0.0, atol=1e-9)
            # overlap along the side
            assert np.all(np.abs(ot[e[i]] - ot[i]) < 0.5 * (osz[e[i]] + osz[i]))
            # 2:1 balance
            assert np.all(np.abs(m.level[e[i]] - m.level[i]) <= 1)
        # two neighbours only when both are finer
        two = (m.nbr[s + 4] != m.nbr[s]) & (m.nbr[s] >= 0)
        i = np.nonzero(two)[0]
        assert np.all(m.level[m.nbr[s][i]] == m.level[i] + 1)
        assert np.all(m.level[m.nbr[s + 4][i]] == m.level[i] + 1)
        # reciprocity: i appears on the opposite side of each neighbour
        o = s ^ 2
        for k in (s, s + 4):
            e = m.nbr[k][m.nbr[k] >= 0]
            src = np.nonzero(m.nbr[k] >= 0)[0]
            assert np.all((m.nbr[o][e] == src) | (m.nbr[o + 4][e] == src))
    # boundary flags only on the domain edge
    b = m.nbr[0] < 0
    assert np.allclose(m.x[b] + 0.5 * m.dx[b], lx)
    b = m.nbr[2] < 0
    assert np.allclose(m.x[b] - 0.5 * m.dx[b], 0.0)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_adaptive_mesh_is_consistent(seed):
    w = inputs.test_case(seed=seed)
    check_mesh(w.mesh, 40.0 * 24, 40.0 * 16)
    assert w.mesh.two_neighbour_sides() > 100


def test_uniform_mesh():
    m = Mesh.build(MeshSpec(0, 0, 10.0, 10.0, 8, 4, 2, uniform=True))
    assert m.n == 8 * 4 * 16
    check_mesh(m, 80.0, 40.0)
    assert m.two_neighbour_sides() == 0


def test_morton_order_is_contiguous_per_subtree():
    w = inputs.test_case(seed=4)
    m = w.mesh
    L = m.max_level
    X = m.ix.astype(np.int64) << (L - m.level)
    Y = m.iy.astype(np.int64) << (L - m.level)

    def spread(v):
        out = np.zeros_like(v)
        for b in range(30):
            out |= ((v >> b) & 1) << (2 * b)
        return out

    key = spread(X) | (spread(Y) << 1)
    assert np.all(np.diff(key) > 0)


def test_gravity_vector_and_pile():
    w = inputs.workload1()
    m = w.mesh
    g = m.gravity
    # |g| = 9.8 everywhere (calc_gravity_vector), downslope component on the 30 deg plane
    assert np.allclose(np.sqrt((g ** 2).sum(0)), 9.8, rtol=1e-6)
    on_plane = (m.x > 50) & (m.x < 1100)
    assert np.allclose(g[0][on_plane], 9.8 * np.sin(np.radians(30.0)), rtol=2e-3)
    assert np.allclose(g[2][m.x > 1300], 9.8)
    # paraboloid pile volume (continuous: pi/2 H R^2) is reproduced by the 9-node average
    vol = (m.h0 * m.dx * m.dy).sum()
    assert abs(vol - 0.5 * np.pi * 30.0 * 100.0 ** 2) / vol < 0.02
    # h0 is linear in the pile height
    assert np.allclose(m.dh0_dpile[0] * 30.0, m.h0, rtol=1e-12, atol=1e-12)


def test_mesh_save_load_roundtrip(tmp_path):
    w = inputs.test_case(seed=5)
    p = tmp_path / "m.npz"
    w.mesh.save(str(p))
    m2 = Mesh.load(str(p))
    for k, v in w.mesh.arrays().items():
        assert np.array_equal(np.asarray(v), np.asarray(getattr(m2, k) if k != "n" else m2.n)), k
