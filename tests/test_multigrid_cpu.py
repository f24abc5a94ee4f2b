"""Host-side planning of the smoothed-aggregation multigrid (ifem_multigrid_plan, amg.cu) on the CPU.

The aggregation follows Vanek, Mandel and Brezina (1996), sec. 3: a node whose strong neighbours are all free
starts an aggregate of itself and them; the remaining nodes join a neighbouring aggregate of that first pass; nodes
left over form their own.  A coupling is strong when |a_ij| >= theta sqrt(|a_ii a_jj|).  The tests restate that
greedy pass in Python and compare aggregate counts with the library's coarse level exactly; the coarse operator's
size follows from the near-null space kept per aggregate.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from ice_fem_2025a_b200 import abi


def _node_graph(A, node, nnodes, theta):
    A = sp.csr_matrix(A)
    d = np.abs(A.diagonal())
    adj = [set() for _ in range(nnodes)]
    for i in range(A.shape[0]):
        for k in range(A.indptr[i], A.indptr[i + 1]):
            j = A.indices[k]
            a, b = node[i], node[j]
            if a == b:
                continue
            if theta > 0 and abs(A.data[k]) < theta * np.sqrt(d[i] * d[j]):
                continue
            adj[a].add(b)
    return [sorted(s) for s in adj]


def _aggregates(adj):
    n = len(adj)
    agg = [-1] * n
    nagg = 0
    for a in range(n):
        if agg[a] >= 0 or any(agg[b] >= 0 for b in adj[a]):
            continue
        agg[a] = nagg
        for b in adj[a]:
            agg[b] = nagg
        nagg += 1
    first = list(agg)
    for a in range(n):
        if agg[a] >= 0:
            continue
        for b in adj[a]:
            if first[b] >= 0:
                agg[a] = first[b]
                break
    for a in range(n):
        if agg[a] < 0:
            agg[a] = nagg
            nagg += 1
    return nagg, agg


def _laplacian_2d(nx, ny, ey=1.0):
    Ix, Iy = sp.identity(nx), sp.identity(ny)
    Tx = sp.diags([-np.ones(nx - 1), 2 * np.ones(nx), -np.ones(nx - 1)], [-1, 0, 1])
    Ty = sp.diags([-np.ones(ny - 1), 2 * np.ones(ny), -np.ones(ny - 1)], [-1, 0, 1])
    return (sp.kron(Iy, Tx) + ey * sp.kron(Ty, Ix)).tocsr()


def test_plan_1d_laplacian(product_lib):
    n = 2000
    A = sp.diags([-np.ones(n - 1), 2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1]).tocsr()
    rows, nnz = abi.multigrid_plan(A, np.arange(n), np.ones(n), lib=product_lib)
    nagg, _ = _aggregates(_node_graph(A, np.arange(n), n, 0.0))
    assert rows == [n, nagg] and nnz[0] == A.nnz
    assert nnz[1] == 3 * nagg - 2            # a chain of aggregates: the coarse operator is tridiagonal


@pytest.mark.parametrize("theta", [0.0, 0.05])
def test_plan_2d_laplacian_and_strength(product_lib, theta):
    """Isotropic: 3 x 3 node aggregates.  Strongly anisotropic (y couplings 1e-2 of x): with a threshold the weak
    couplings leave the graph and the aggregates become 3-node lines, so the coarse level has more rows."""
    nx = ny = 60
    for ey in (1.0, 1.0e-2):
        A = _laplacian_2d(nx, ny, ey)
        n = A.shape[0]
        rows, _ = abi.multigrid_plan(A, np.arange(n), np.ones(n), threshold=theta, lib=product_lib)
        nagg, _ = _aggregates(_node_graph(A, np.arange(n), n, theta))
        assert rows[0] == n and rows[1] == nagg, (ey, theta, rows, nagg)
        if ey < 1.0 and theta > 0.0:
            full, _ = abi.multigrid_plan(A, np.arange(n), np.ones(n), threshold=0.0, lib=product_lib)
            assert rows[1] == nx * ny // 3 and rows[1] > 1.5 * full[1]   # 3-node lines along x


def test_plan_elasticity_rigid_modes(product_lib):
    """The oracle's 2D u-step matrix with its three rigid-body modes: per aggregate of two or more nodes the three
    modes stay independent (3 coarse rows), a one-node aggregate keeps 2 (the rotation is a combination of the
    translations there)."""
    from tests.helpers import make_pair
    mesh, d, o, _, _ = make_pair(0, 0.25, gpu=False)
    o.assemble(0, dt=1.0)
    K = o.matrix(0)
    ux, uy = o.dof_numbers(abi.DOF_UX), o.dof_numbers(abi.DOF_UY)
    n, nn = K.shape[0], mesh.n_nodes
    node = np.empty(n, np.int64)
    node[ux] = np.arange(nn)
    node[uy] = np.arange(nn)
    x, y = mesh.coords[:, 0] - mesh.coords[:, 0].mean(), mesh.coords[:, 1] - mesh.coords[:, 1].mean()
    B = np.zeros((n, 3))
    B[ux, 0] = 1.0
    B[uy, 1] = 1.0
    B[ux, 2] = -y
    B[uy, 2] = x
    rows, _ = abi.multigrid_plan(K, node, B, lib=product_lib)
    nagg, agg = _aggregates(_node_graph(K, node, nn, 0.0))
    sizes = np.bincount(agg, minlength=nagg)
    assert rows[0] == n and len(rows) == 2
    assert rows[1] == 3 * int((sizes >= 2).sum()) + 2 * int((sizes == 1).sum())
    again, _ = abi.multigrid_plan(K, node, B, lib=product_lib)
    assert again == rows


def test_plan_rejects_bad_input(product_lib):
    A = _laplacian_2d(30, 30)
    n = A.shape[0]
    bad = A.copy()
    bad.indices[5] = n + 3                   # column out of range
    with pytest.raises(abi.IfemError) as e:
        abi.multigrid_plan(bad, np.arange(n), np.ones(n), lib=product_lib)
    assert e.value.code == abi.ERR_INVALID
    with pytest.raises(abi.IfemError) as e:
        abi.multigrid_plan(A, np.arange(n), np.ones(n), threshold=1.0, lib=product_lib)
    assert e.value.code == abi.ERR_INVALID
    small, _ = abi.multigrid_plan(_laplacian_2d(20, 20), np.arange(400), np.ones(400), lib=product_lib)
    assert small == [400]                    # at most 800 rows: one level, inverted densely
