"""Build libgpawb200.so in-tree with nvcc for sm_100a.

Usage: python -m gpaw_b200.build  (or gpaw_b200.build.build()).
The library is written next to this file so it travels with the source tree;
there is no JIT cache and no fallback.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / 'csrc'
INCLUDE = HERE.parent / 'include'
LIB = HERE / 'libgpawb200.so'
STAMP = HERE / '.libgpawb200.stamp'

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ['-O3', '-std=c++17', '-lineinfo',
              '-Xcompiler', '-fPIC', '-Xptxas', '-O3',
              '--expt-relaxed-constexpr']


def sources() -> list[Path]:
    return sorted(CSRC.glob('*.cu'))


def _digest() -> str:
    h = hashlib.sha256()
    for p in sources() + sorted(CSRC.glob('*.cuh')) + sorted(INCLUDE.glob('*.h')):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(' '.join(ARCH + NVCC_FLAGS).encode())
    return h.hexdigest()


def nvcc() -> str:
    exe = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not Path(exe).exists():
        raise RuntimeError('nvcc not found; the CUDA toolkit is required')
    return exe


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile every .cu under csrc/ and link libgpawb200.so (sm_100a)."""
    digest = _digest()
    if (not force and LIB.exists() and STAMP.exists()
            and STAMP.read_text().strip() == digest):
        return LIB
    objdir = HERE / '_build'
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    jobs = jobs or min(8, os.cpu_count() or 1)
    for src in sources():
        obj = objdir / (src.stem + '.o')
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, '-I', str(INCLUDE), '-c', str(src),
               '-o', str(obj)]
        if verbose:
            print(' '.join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
        objs.append(obj)
        if len([p for _, p in procs if p.poll() is None]) >= jobs:
            for s, p in procs:
                p.wait()
    errors = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errors.append(f'--- {src.name}\n{out.decode(errors="replace")}')
        elif verbose and out:
            print(out.decode(errors='replace'), file=sys.stderr)
    if errors:
        raise RuntimeError('nvcc failed:\n' + '\n'.join(errors))
    tmp = LIB.with_suffix('.so.tmp')
    cmd = [nvcc(), *ARCH, '-shared', '-Xcompiler', '-fPIC', *map(str, objs),
           '-o', str(tmp), '-lcudart']
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    STAMP.write_text(digest)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)
