"""The allocation-free Q9 assembly (ss_assemble_q9_noalloc) against ss_assemble.

ss_assemble_q9_noalloc exists for callers of this library that may not
allocate device memory: a host framework that hands out all device memory from
its own pool.  The tests own every device buffer (allocated here with torch, as
such a caller would through its own pool), call the entry point through the C
ABI and check the results against the matrices of the allocating entry point,
within the block-relative 1e-12 bar of the other assembly tests: twice in a row
on the legacy default stream, once on a side stream, and once with a pattern
that lacks a node pair (SS_EINVAL) followed by a correct call (SS_OK, which
shows the shared mismatch counter starts from zero on every call).  This file
sorts last so that a stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import block_rel_err
from sawsim_b200 import _lib as L, cases
from sawsim_b200.engine import _pml_arrays
from sawsim_b200.materials import pack

pytestmark = pytest.mark.gpu


def _pattern(mesh, nc):
    """Node adjacency (sorted, self included) and component-major row pointers."""
    N = mesh.N
    adj = [set() for _ in range(N)]
    for q in mesh.quads:
        for a in q:
            adj[a].update(int(x) for x in q)
    nadj_ptr = np.zeros(N + 1, dtype=np.int64)
    nadj_ptr[1:] = np.cumsum([len(s) for s in adj])
    nadj = np.concatenate([np.sort(np.fromiter(s, dtype=np.int64)) for s in adj])
    deg = np.diff(nadj_ptr)
    rowlen = np.tile(nc * deg, nc)
    indptr = np.zeros(nc * N + 1, dtype=np.int64)
    indptr[1:] = np.cumsum(rowlen)
    return indptr, nadj_ptr, nadj


def _setup(torch, name, cols, rows):
    case = cases.make_case(name, cols=cols, rows=rows)
    eng = cases.engine_for(case)
    Kref = eng.export(L.SS_MAT_K)
    Mref = eng.export(L.SS_MAT_M)
    eng.close()
    ndisp = 3 if case.mode_extension else 2
    nc = ndisp + 1
    indptr, nadj_ptr, nadj = _pattern(case.mesh, nc)
    assert np.array_equal(indptr, Kref.indptr)
    rho, Cm, em, epsm = pack(case.materials, ndisp)
    nreg, axis, dmax, npow, inner, outer, region = _pml_arrays(case.mesh.elem_tag, case.pml, case.mesh.ne)
    dev = torch.device('cuda:0')

    def d(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)

    bufs = dict(pos=d(case.mesh.pos_m, np.float64), conn=d(case.mesh.quads, np.int64),
                emat=d(case.mat_idx, np.int32), rho=d(rho, np.float64), C=d(Cm, np.float64), e=d(em, np.float64),
                eps=d(epsm, np.float64), region=d(region, np.int32), axis=d(axis, np.int32), dmax=d(dmax, np.float64),
                npow=d(npow, np.int32), inner=d(inner, np.float64), outer=d(outer, np.float64),
                indptr=d(indptr, np.int64), nadj_ptr=d(nadj_ptr, np.int64), nadj=d(nadj, np.int64))
    nnz = int(indptr[-1])
    K = torch.empty(2 * nnz, dtype=torch.float64, device=dev)
    M = torch.empty(2 * nnz, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    comp = np.arange(nc * case.mesh.N) // case.mesh.N
    return dict(case=case, Kref=Kref, Mref=Mref, ndisp=ndisp, nc=nc, nreg=nreg, bufs=bufs, nnz=nnz, K=K, M=M,
                comp=comp, nadj_ptr=nadj_ptr, nadj=nadj, d=d)


def _call(s, p, stream=None):
    c = s['case']
    return L.load().ss_assemble_q9_noalloc(
        s['ndisp'], c.mesh.N, p['pos'], c.mesh.ne, p['conn'], p['emat'], p['rho'], p['C'], p['e'], p['eps'],
        s['nreg'], p['region'], p['axis'], p['dmax'], p['npow'], p['inner'], p['outer'], c.omega_top, p['indptr'],
        p['nadj_ptr'], p['nadj'], s['nnz'], C.c_void_p(s['K'].data_ptr()), C.c_void_p(s['M'].data_ptr()), stream)


def _check(s, tag):
    Kv = s['K'].cpu().numpy().view(np.complex128)
    Mv = s['M'].cpu().numpy().view(np.complex128)
    Kn = s['Kref'].copy()
    Kn.data = Kv
    assert block_rel_err(Kn, s['Kref'], s['comp'], s['comp'], s['nc']) <= 1e-12, tag
    Mfull = s['Kref'].copy()
    Mfull.data = Mv
    Mfull.eliminate_zeros()
    Mfull.sort_indices()
    assert block_rel_err(Mfull, s['Mref'], s['comp'], s['comp'], s['nc']) <= 1e-12, tag


def _ptrs(bufs):
    return {k: C.c_void_p(v.data_ptr()) for k, v in bufs.items()}


@pytest.mark.parametrize('name,cols,rows', [('me1_64x256', 8, 80), ('me0_16x64', 8, 16)])
def test_noalloc_matches_allocating_assembly(built_lib, name, cols, rows):
    torch = pytest.importorskip('torch')
    s = _setup(torch, name, cols, rows)
    assert s['case'].mesh.ne > 512 or name == 'me0_16x64'      # ME1 case spans several scratch batches
    p = _ptrs(s['bufs'])
    for call in range(2):
        rc = _call(s, p)
        assert rc == L.SS_OK, L.STATUS_NAMES.get(rc, rc)
        _check(s, call)


def test_noalloc_side_stream_and_pattern_error(built_lib):
    torch = pytest.importorskip('torch')
    s = _setup(torch, 'me1_64x256', 8, 80)
    p = _ptrs(s['bufs'])
    # one call on a non-default stream
    side = torch.cuda.Stream()
    rc = _call(s, p, C.c_void_p(side.cuda_stream))
    assert rc == L.SS_OK, L.STATUS_NAMES.get(rc, rc)
    _check(s, 'side stream')
    # a node adjacency with one off-diagonal neighbour of node 0 removed: the
    # row pointers shrink by one from node 1 on, so every lookup and every slot
    # stays inside the original pattern; the missing pair is reported
    nadj_ptr, nadj = s['nadj_ptr'], s['nadj']
    row0 = nadj[nadj_ptr[0]:nadj_ptr[1]]
    drop = int(nadj_ptr[0] + np.nonzero(row0 != 0)[0][0])
    bad_adj = np.delete(nadj, drop)
    bad_ptr = nadj_ptr.copy()
    bad_ptr[1:] -= 1
    pb = dict(p)
    t_ptr, t_adj = s['d'](bad_ptr, np.int64), s['d'](bad_adj, np.int64)
    torch.cuda.synchronize()
    pb['nadj_ptr'], pb['nadj'] = C.c_void_p(t_ptr.data_ptr()), C.c_void_p(t_adj.data_ptr())
    rc = _call(s, pb)
    assert rc == L.SS_EINVAL
    # the next correct call starts its mismatch count from zero
    rc = _call(s, p)
    assert rc == L.SS_OK, L.STATUS_NAMES.get(rc, rc)
    _check(s, 'after the pattern error')
