"""CPU-baseline helper (test/benchmark infrastructure): an oracle engine per case,
cached per process."""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

_cache = {}


def oracle_solver_for(case_name, cols, rows):
    key = (case_name, cols, rows)
    if key not in _cache:
        from sawsim_b200 import cases
        from oracle import q9, solver
        c = cases.make_case(case_name, cols=cols, rows=rows)
        m = q9.build_model(c.cell.msh())
        pml = [q9.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp) for p in c.pml]
        asm = q9.assemble if c.mode_extension else q9.assemble_me0
        K, M = asm(m, c.materials, c.mat_idx, pml, c.omega_top)
        ndisp = 3 if c.mode_extension else 2
        _cache[key] = solver.FrequencySolver(K, M, *solver.bc_periodic(m, c.cell.LINES3, ndisp=ndisp))
    return _cache[key]
