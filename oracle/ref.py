"""ORACLE (test infrastructure): access to GPAW's own C extension `_gpaw`,
built from the reference sources by oracle/Makefile into oracle/_ref/.

Only tests, the smoke check and bench.py's reference / cpu_baseline legs use
this module.  `available()` is False where the build is absent (then the
numpy restatement in oracle/fd.py, pinned by tests/golden/, stands alone).
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / '_ref'
_mod = None


def load():
    """Import oracle/_ref/_gpaw*.so (once); None if it was not built."""
    global _mod
    if _mod is None:
        cands = sorted(REF_DIR.glob('_gpaw*.so'))
        if not cands:
            return None
        spec = importlib.util.spec_from_file_location('_gpaw', cands[0])
        mod = importlib.util.module_from_spec(spec)
        sys.modules.setdefault('_gpaw', mod)
        spec.loader.exec_module(mod)
        _mod = mod
    return _mod


def available() -> bool:
    return load() is not None


def neighbor_cd(pbc_c):
    return np.ascontiguousarray(
        np.where(np.asarray(pbc_c, bool)[:, None], 0, -1) * np.ones((3, 2), int))


def operator(coef_p, offset_pc, n_c, pbc_c, real=True):
    """_gpaw.Operator with the arguments gpaw/fd_operators.py:48-87 builds."""
    g = load()
    offset_pc = np.asarray(offset_pc, int).reshape(-1, 3)
    cfd = all((o != 0).sum() < 2 for o in offset_pc)
    mp = int(np.abs(offset_pc).max())
    n_c = np.asarray(n_c, int)
    M_c = n_c + 2 * mp
    stride_c = np.array([M_c[1] * M_c[2], M_c[2], 1])
    offset_p = np.ascontiguousarray(offset_pc.dot(stride_c))
    return g.Operator(np.ascontiguousarray(coef_p, float), offset_p, n_c, mp,
                      neighbor_cd(pbc_c), bool(real), None, cfd)


def transformer(n_in, n_out, nn, pad, npad, skip, pbc_c, real, interpolate):
    """_gpaw.Transformer with the arguments of gpaw/transformers.py:71-77."""
    g = load()
    return g.Transformer(np.asarray(n_in, int), np.asarray(n_out, int),
                         2 * nn, np.ascontiguousarray(pad, int),
                         np.ascontiguousarray(npad, int),
                         np.ascontiguousarray(skip, int), neighbor_cd(pbc_c),
                         bool(real), None, bool(interpolate))
