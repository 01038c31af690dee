"""The allocation-free Q9 assembly (ss_assemble_q9_noalloc) against ss_assemble.

ss_assemble_q9_noalloc exists for callers of this library that cannot
allocate device memory (a stream being captured into a CUDA graph, a host
framework that owns all device memory).  The test owns every device buffer
(allocated here with torch, as such a caller would through its own pool),
calls the entry point twice in a row through the C ABI and checks both
results against the matrices of the allocating entry point, within the
block-relative 1e-12 bar of the other assembly tests.  This file sorts last so
that a stop-at-first-failure run has already run every other test.
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


@pytest.mark.parametrize('name,cols,rows', [('me1_64x256', 8, 80), ('me0_16x64', 8, 16)])
def test_noalloc_matches_allocating_assembly(built_lib, name, cols, rows):
    torch = pytest.importorskip('torch')
    case = cases.make_case(name, cols=cols, rows=rows)
    eng = cases.engine_for(case)
    Kref = eng.export(L.SS_MAT_K)
    Mref = eng.export(L.SS_MAT_M)
    eng.close()
    ndisp = 3 if case.mode_extension else 2
    nc = ndisp + 1
    assert case.mesh.ne > 512 or name == 'me0_16x64'      # ME1 case spans several scratch batches
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
    lib = L.load()
    p = {k: C.c_void_p(v.data_ptr()) for k, v in bufs.items()}
    comp = np.arange(nc * case.mesh.N) // case.mesh.N
    for call in range(2):
        rc = lib.ss_assemble_q9_noalloc(ndisp, case.mesh.N, p['pos'], case.mesh.ne, p['conn'], p['emat'], p['rho'],
                                        p['C'], p['e'], p['eps'], nreg, p['region'], p['axis'], p['dmax'], p['npow'],
                                        p['inner'], p['outer'], case.omega_top, p['indptr'], p['nadj_ptr'],
                                        p['nadj'], nnz, C.c_void_p(K.data_ptr()), C.c_void_p(M.data_ptr()), None)
        assert rc == L.SS_OK, L.STATUS_NAMES.get(rc, rc)
        Kv = K.cpu().numpy().view(np.complex128)
        Mv = M.cpu().numpy().view(np.complex128)
        Kn = Kref.copy()
        Kn.data = Kv
        assert block_rel_err(Kn, Kref, comp, comp, nc) <= 1e-12, call
        Mfull = Kref.copy()
        Mfull.data = Mv
        Mfull.eliminate_zeros()
        Mfull.sort_indices()
        assert block_rel_err(Mfull, Mref, comp, comp, nc) <= 1e-12, call
