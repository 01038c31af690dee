"""Build the in-tree shared library ``libsawsim_b200.so`` for sm_100a with nvcc.

Every CUDA/C++ source under ``csrc/`` is compiled to an object in ``_build/``
(in parallel) and linked into one C-ABI shared library beside this file.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / 'csrc'
OUT = HERE / 'libsawsim_b200.so'
BUILD = HERE / '_build'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC,-O3', '--expt-relaxed-constexpr']


def nvcc() -> str:
    cand = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not Path(cand).exists():
        raise RuntimeError('nvcc not found')
    return cand


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + '.o')
    deps = [src] + list(SRC.glob('*.h')) + list(SRC.glob('*.cuh')) + list((HERE.parent / 'include').glob('*.h'))
    if obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, '-c', str(src), '-o', str(obj)]
    if src.suffix == '.cu' and verbose:
        cmd += ['-Xptxas', '-v']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'nvcc failed for {src.name}:\n{r.stderr}')
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(SRC.glob('*.cu')) + sorted(SRC.glob('*.cpp'))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if OUT.exists() and OUT.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return OUT
    cmd = [nvcc(), *ARCH, '-shared', '-o', str(OUT), *map(str, objs), '-lcudart']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stderr}')
    return OUT


if __name__ == '__main__':
    print(build(verbose='-v' in sys.argv))
