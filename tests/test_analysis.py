"""The host analysis (``ss_analyze_host``: condensation, nested dissection and
front tree, the same host code as ``ss_analyze``) on CPU, against independent
restatements:

* the active DOFs equal the oracle's (the reference's fold and prescribed sets,
  sweep.py:283-299 for Q9, bc_solve.py:121-132 for Hex27), from the oracle's own
  boundary sets and from the product's;
* the front tree is a valid multifrontal structure: pivots partition the
  elimination order, children come before parents, every child's update rows
  lie in its parent, levels count the height, and nnz(L+U) and the flops follow
  from the front sizes;
* the fill is exact: each front's update rows equal the rows of L that its
  pivot columns reach in a symbolic elimination of the condensed structural
  pattern (built here from the mesh and the oracle's fold operator) in the
  analysis' order;
* two analyses agree bit for bit, and bad inputs are refused.
CPU only: no device is touched."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import hex27 as oh, q9 as oq9, solver as osol
from sawsim_b200 import _lib as L, cases
from sawsim_b200.analysis import analyze_csr, analyze_hex27, analyze_q9, level_work


def _node_graph(conn, N):
    ne, npe = conn.shape
    E = sp.csr_matrix((np.ones(ne * npe), (np.repeat(np.arange(ne), npe), conn.ravel())), shape=(ne, N))
    return (E.T @ E).tocsr()


def _q9(name, cols, rows):
    c = cases.make_case(name, cols=cols, rows=rows)
    m = oq9.build_model(c.cell.msh())
    ndisp = 3 if c.mode_extension else 2
    bc = osol.bc_periodic(m, c.cell.LINES3, ndisp=ndisp)
    gdof = (ndisp + 1) * c.mesh.N
    T, slaves, _ = osol.merge_transform(gdof, bc[3])
    presc = np.unique(np.concatenate([np.asarray(bc[0], int), slaves, np.asarray(bc[1], int), np.asarray(bc[2], int)]))
    active = np.setdiff1d(np.arange(gdof), presc)
    S = sp.kron(np.ones((ndisp + 1, ndisp + 1)), _node_graph(c.mesh.quads, c.mesh.N)).tocsr()
    return c, bc, T, active, S


def _hex(nx, ny, nz):
    c = cases.make_hex_case('hex_8x4x48', nx=nx, ny=ny, nz=nz, points=3)
    N = c.N
    gdof = 4 * N
    mach, elec = oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * N)
    t_fb = oh._fold(np.concatenate([mach['period_B'], elec['period_B']]),
                    np.concatenate([mach['period_F'], elec['period_F']]), gdof)
    t_lr = oh._fold(np.concatenate([mach['period_R'], elec['period_R']]),
                    np.concatenate([mach['period_L'], elec['period_L']]), gdof)
    presc = np.unique(np.concatenate([mach['fix'], mach['period_B'], mach['period_R'], elec['period_R'],
                                      elec['period_B'], elec['zheng'], elec['fu']]))
    active = np.setdiff1d(np.arange(gdof), presc)
    # structural pattern in the Hex27 DOF layout (u of node n at 3n + c, phi at 3N + n)
    Scm = sp.kron(np.ones((4, 4)), _node_graph(c.hexas, N)).tocsr()
    lay = np.concatenate([3 * np.arange(N) + cc for cc in range(3)] + [3 * N + np.arange(N)])
    P = sp.csr_matrix((np.ones(gdof), (lay, np.arange(gdof))), shape=(gdof, gdof))
    S = (P @ Scm @ P.T).tocsr()
    return c, (t_fb @ t_lr).tocsr(), active, S


def _check_tree(a):
    nf = a.k.size
    p0 = a.rows[a.rows_ptr[:-1]]
    # pivots: each front's first k rows are p0 .. p0 + k - 1, and the ranges tile 0 .. n-1 in front order
    assert p0[0] == 0 and np.array_equal(p0[1:], np.cumsum(a.k)[:-1]) and int(a.k.sum()) == a.n_active
    assert np.array_equal(np.sort(a.order), np.arange(a.n_active))
    lev = np.zeros(nf, int)
    for f in range(nf):
        r = a.rows[a.rows_ptr[f]:a.rows_ptr[f + 1]]
        assert r.size == a.m[f] and np.array_equal(r[:a.k[f]], p0[f] + np.arange(a.k[f]))
        upd = r[a.k[f]:]
        assert np.all(np.diff(upd) > 0) and (upd.size == 0 or upd[0] >= p0[f] + a.k[f])
        p = a.parent[f]
        if p < 0:
            assert upd.size == 0
            continue
        assert p > f
        assert np.isin(upd, a.rows[a.rows_ptr[p]:a.rows_ptr[p + 1]]).all()
        lev[p] = max(lev[p], lev[f] + 1)
    assert np.array_equal(lev, a.level) and a.levels == lev.max() + 1
    k, u = a.k.astype(float), (a.m - a.k).astype(float)
    assert a.nnz_lu == pytest.approx(float(np.sum(k * k + 2 * k * u)), rel=1e-12)
    assert a.flops_per_point == pytest.approx(float(np.sum(8 * (k ** 3 / 3 + k * k * u + k * u * u))), rel=1e-12)
    assert a.max_front == a.m.max() and a.max_pivots == a.k.max()


def _check_fill(a, T, active, S):
    """Symbolic elimination of the condensed structural pattern in the analysis'
    order; each front's update rows must be exactly what its pivots reach."""
    Pc = (T.T @ S @ T).tocsr()[active][:, active]
    n = a.n_active
    perm = sp.csr_matrix((np.ones(n), (a.order, np.arange(n))), shape=(n, n))
    A = (perm @ Pc @ perm.T).tocsc()
    A = (A + A.T).tocsc()
    assert A.nnz <= a.condensed_nnz + n       # the structural pattern (plus its diagonal)
    p0 = a.rows[a.rows_ptr[:-1]]
    front_of = np.repeat(np.arange(a.k.size), a.k)
    reach = [set() for _ in range(a.k.size)]
    pending = {}
    exact_l = 0
    for j in range(n):
        col = A.indices[A.indptr[j]:A.indptr[j + 1]]
        s = pending.pop(j, set())
        s.update(int(i) for i in col if i > j)
        s.discard(j)
        exact_l += len(s)
        f = front_of[j]
        reach[f] |= s
        if s:
            pending.setdefault(min(s), set()).update(s)
    for f in range(a.k.size):
        upd = set(a.rows[a.rows_ptr[f] + a.k[f]:a.rows_ptr[f + 1]].tolist())
        assert reach[f] - set(range(p0[f], p0[f] + a.k[f])) == upd, f
    k, u = a.k.astype(float), (a.m - a.k).astype(float)
    assert exact_l <= np.sum(k * (k - 1) / 2 + k * u)


@pytest.mark.parametrize('name,cols,rows', [('me1_64x256', 8, 16), ('me0_16x64', 8, 16), ('me1_64x256', 16, 24)])
def test_q9_analysis(name, cols, rows):
    c, bc, T, active, S = _q9(name, cols, rows)
    a = analyze_q9(c.mesh.pos_m, c.mesh.quads, bc, c.mode_extension)
    assert np.array_equal(a.active, active)
    b = analyze_q9(c.mesh.pos_m, c.mesh.quads, c.bc, c.mode_extension)      # the product's boundary sets
    assert np.array_equal(b.active, active) and np.array_equal(b.order, a.order)
    _check_tree(a)
    _check_fill(a, T, active, S)
    again = analyze_q9(c.mesh.pos_m, c.mesh.quads, bc, c.mode_extension)
    for key in ('order', 'k', 'm', 'parent', 'level', 'rows_ptr', 'rows'):
        assert np.array_equal(getattr(again, key), getattr(a, key)), key


@pytest.mark.parametrize('nxyz', [(8, 1, 6), (8, 2, 12)])
def test_hex27_analysis(nxyz):
    c, T, active, S = _hex(*nxyz)
    a = analyze_hex27(c.pos_m, c.hexas, c.bc)
    assert np.array_equal(a.active, active)
    _check_tree(a)
    _check_fill(a, T, active, S)


def test_analysis_refuses_bad_input():
    c = cases.make_case('me1_64x256', cols=8, rows=16)
    fix, zheng, fu, groups = c.bc
    with pytest.raises(L.SawsimError):
        analyze_q9(c.mesh.pos_m, np.where(c.mesh.quads == 0, c.mesh.N, c.mesh.quads), c.bc)   # node out of range
    with pytest.raises(L.SawsimError):
        analyze_q9(c.mesh.pos_m, c.mesh.quads, (fix, [], fu, groups))                          # no driven DOFs
    with pytest.raises(L.SawsimError):
        analyze_q9(c.mesh.pos_m, c.mesh.quads, c.bc, mode_extension=0)                         # ME1 sets, ME0 mesh


def test_benchmarked_cell_analysis():
    """The ME1 two-layer 64x256 cell of the benchmark: the oracle's 262,664 active
    DOFs and a valid front tree, analysed on the host in seconds."""
    c = cases.make_case('me1_64x256')
    m = oq9.build_model(c.cell.msh())
    bc = osol.bc_periodic(m, c.cell.LINES3, ndisp=3)
    _, slaves, _ = osol.merge_transform(4 * c.mesh.N, bc[3])
    presc = np.unique(np.concatenate([np.asarray(bc[0], int), slaves, np.asarray(bc[1], int), np.asarray(bc[2], int)]))
    a = analyze_q9(c.mesh.pos_m, c.mesh.quads, c.bc)
    assert a.n_active == 262664 and np.array_equal(a.active, np.setdiff1d(np.arange(4 * c.mesh.N), presc))
    _check_tree(a)
    assert a.front_bytes_per_point['complex128'] < 5e9     # 37 points per chunk in 180 GB


def test_matrix_input_with_node_map_equals_the_mesh_path():
    """From the assembled pattern with the node of every DOF and the node
    coordinates, the analysis is the mesh path's, front for front."""
    c, bc, T, active, S = _q9('me1_64x256', 8, 16)
    a = analyze_q9(c.mesh.pos_m, c.mesh.quads, bc)
    b = analyze_csr(S, bc, dof_node=np.arange(S.shape[0]) % c.mesh.N, node_xyz=c.mesh.pos_m[:, :2])
    for key in ('active', 'order', 'k', 'm', 'parent', 'level', 'rows_ptr', 'rows'):
        assert np.array_equal(getattr(a, key), getattr(b, key)), key


@pytest.mark.parametrize('cell', ['q9', 'hex27'])
def test_graph_nested_dissection_fill_is_exact(cell):
    """Without geometry (a Gmsh-meshed template's assembled matrices): the graph
    nested dissection's front tree is valid and its fill exact."""
    if cell == 'q9':
        c, bc, T, active, S = _q9('me1_64x256', 8, 16)
        a = analyze_csr(S, bc)
    else:
        c, T, active, S = _hex(8, 1, 6)
        fix, zheng, fu, groups, two_stage = c.bc
        a = analyze_csr(S, (fix, zheng, fu, groups), two_stage=two_stage)
    assert np.array_equal(a.active, active)
    _check_tree(a)
    _check_fill(a, T, active, S)


def test_level_work_adds_up():
    c, bc, T, active, S = _q9('me1_64x256', 8, 16)
    a = analyze_q9(c.mesh.pos_m, c.mesh.quads, bc)
    w = level_work(a)
    assert len(w) == a.levels and sum(r['fronts'] for r in w) == a.k.size
    assert sum(r['schur_flops'] + r['other_flops'] for r in w) == pytest.approx(a.flops_per_point, rel=1e-12)
    assert sum(r['lu_bytes'] for r in w) == pytest.approx(16 * a.nnz_lu, rel=1e-12)
    assert sum(r['pivots'] for r in w) == a.n_active
