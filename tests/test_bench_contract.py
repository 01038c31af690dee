"""Host-side pieces of bench.py's JSON line (no GPU): the roofline kernel naming
from the autotuner's per-level picks and the Schur traffic scaling."""
import importlib.util
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


@pytest.fixture(scope='module')
def bench():
    spec = importlib.util.spec_from_file_location('bench_under_test', REPO / 'bench.py')
    mod = importlib.util.module_from_spec(spec)
    sys.modules['bench_under_test'] = mod
    spec.loader.exec_module(mod)
    return mod


def test_fp64_kernel_name_lists_the_picked_tiles(bench):
    s = dict(schur_candidate0=1.0, schur_candidate1=0.0, schur_candidate2=13.0)
    name = bench.schur_kernel_name(s, 'fp64')
    assert 'front_dmma_kernel<2,2> (FP64 DMMA 64x64) on 13 levels' in name
    assert 'SIMT 128x64 on 1 levels' in name
    assert 'SIMT 64x64' not in name


def test_mixed_kernel_name_lists_the_picked_tiles(bench):
    s = dict(schur_candidate0=5.0, schur_candidate1=1.0, schur_candidate2=7.0)
    name = bench.schur_kernel_name(s, 'mixed')
    assert 'tc::tma_gemm_kernel<128,2>' in name and 'on 5 levels' in name
    assert 'tc::tma_gemm_kernel<64,3>' in name and 'on 1 levels' in name
    assert 'SIMT FP32 128x64) on 7 levels' in name


def test_schur_traffic_is_known_only_for_the_profiled_workload(bench):
    assert set(bench.SCHUR_DRAM_BYTES_PER_POINT) == {'me1_64x256'}
    # per point: the update's own DRAM bytes, a few GB on the 262k-DOF cell
    assert 4e9 < bench.SCHUR_DRAM_BYTES_PER_POINT['me1_64x256'] < 8e9


class _FakeEngine:
    """Stands in for FrequencySolver in the host-side roofline arithmetic."""

    def export(self, which):
        import scipy.sparse as sp
        return sp.identity(10 if which == 0 else 4, format='csr', dtype=complex)


def test_rooflines_fp64_entries(bench):
    from types import SimpleNamespace
    c = SimpleNamespace(name='me1_64x256', mesh=SimpleNamespace(ne=2, N=6))
    s = dict(schur_launches=2.0, schur_gemm_flops=4e12, solve_ms=10.0, schur_candidate2=14.0)
    st0 = dict(n_active=100.0, nnz_lu=1e6, element_kernel_ms=1.0, scatter_kernel_ms=1.0)
    roof = bench.rooflines(_FakeEngine(), c, s, st0, 'fp64', [100.0], 4, dict(hbm_gbs=6500.0), 'measured',
                           {'fp64_dmma': 34.0, 'fp64_dmma_3m': 40.0})
    assert [r['bound'] for r in roof] == ['tensor', 'hbm', 'hbm']
    # 2 TFLOP per launch in 50 ms = 40 TFLOP/s = the measured ceiling
    assert roof[0]['achieved'] == pytest.approx(40.0) and roof[0]['frac'] == pytest.approx(1.0)
    assert roof[0]['traffic'] == pytest.approx(6.16e9 * 4 / 2)
    # solves: 4 points x (1e6 x 16 + 2 x 100 x 16) bytes in 10 ms
    assert roof[1]['achieved'] == pytest.approx(4 * (16e6 + 3200) / 1e-2 / 1e9)
    # assembly: 16 (10 + 4) + 8*2*6 + 8*9*2 + 8*81*2 bytes in 2 ms
    assert roof[2]['bytes'] == 16 * 14 + 96 + 144 + 1296
    assert roof[2]['frac'] == pytest.approx(roof[2]['bytes'] / 2e-3 / 1e9 / 6500.0)


def test_rooflines_mixed_peak_is_tf32(bench):
    from types import SimpleNamespace
    c = SimpleNamespace(name='hex_8x4x48', hexas=[[0] * 27] * 3, N=10)
    s = dict(schur_launches=1.0, schur_gemm_flops=1e12, solve_ms=0.0, schur_candidate0=1.0)
    st0 = dict(n_active=100.0, nnz_lu=1e6, element_kernel_ms=0.0, scatter_kernel_ms=0.0)
    roof = bench.rooflines(_FakeEngine(), c, s, st0, 'mixed', [10.0], 4, dict(bf16_tflops=1600.0), 'measured', {})
    assert len(roof) == 1 and roof[0]['peak'] == 800.0 and roof[0]['traffic'] is None
