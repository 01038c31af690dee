"""Shared test helpers: oracle runs and error measures (oracle used only as checker)."""
import numpy as np

from oracle import q9 as oq9, solver as osol


def oracle_engine(case):
    m = oq9.build_model(case.cell.msh())
    pml = [oq9.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp, xa=p.xa, xp=p.xp) for p in case.pml]
    asm = oq9.assemble if case.mode_extension else oq9.assemble_me0
    K, M = asm(m, case.materials, case.mat_idx, pml, case.omega_top)
    ndisp = 3 if case.mode_extension else 2
    eng = osol.FrequencySolver(K, M, *osol.bc_periodic(m, case.cell.LINES3, ndisp=ndisp))
    return K, M, eng


def comp_of(dof, N, nc):
    return np.asarray(dof) // N


def block_rel_err(A, B, comp_r, comp_c, nc):
    """max over component blocks of max|A-B| / max|B| inside the block."""
    A = A.tocoo()
    D = (A - B).tocoo()
    Bc = B.tocoo()
    worst = 0.0
    for a in range(nc):
        for b in range(nc):
            sb = (comp_r[Bc.row] == a) & (comp_c[Bc.col] == b)
            scale = np.abs(Bc.data[sb]).max() if sb.any() else 0.0
            sd = (comp_r[D.row] == a) & (comp_c[D.col] == b)
            err = np.abs(D.data[sd]).max() if sd.any() else 0.0
            if scale == 0.0:
                sa = (comp_r[A.row] == a) & (comp_c[A.col] == b)
                scale = np.abs(A.data[sa]).max() if sa.any() else 1.0
                scale = scale or 1.0
            worst = max(worst, err / scale)
    return worst
