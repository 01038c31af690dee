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
    s = dict(schur_tile_simt128=1.0, schur_tile_simt64=0.0, schur_tile_dmma=13.0)
    name = bench.schur_kernel_name(s, 'fp64')
    assert 'front_dmma_kernel<2,2> (FP64 DMMA 64x64) on 13 levels' in name
    assert 'SIMT 128x64 on 1 levels' in name
    assert 'SIMT 64x64' not in name


def test_mixed_kernel_name_lists_the_picked_tiles(bench):
    s = dict(schur_tile_simt128=5.0, schur_tile_simt64=1.0, schur_tile_dmma=7.0)
    name = bench.schur_kernel_name(s, 'mixed')
    assert 'tc::front_tc_gemm_kernel' in name and 'on 5 levels' in name
    assert 'tc::front_tc_gemm_persistent' in name and 'on 1 levels' in name
    assert 'SIMT FP32 128x64) on 7 levels' in name


def test_schur_traffic_is_known_only_for_the_profiled_workload(bench):
    assert set(bench.SCHUR_DRAM_BYTES_PER_POINT) == {'me1_64x256'}
    # per point: the update's own DRAM bytes, a few GB on the 262k-DOF cell
    assert 4e9 < bench.SCHUR_DRAM_BYTES_PER_POINT['me1_64x256'] < 8e9
