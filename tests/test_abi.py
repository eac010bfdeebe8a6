"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/gpawb200.h declares, and its host-side validation behaves like the
reference's argument checks (errors before any launch)."""
import ctypes
import re

import numpy as np
import pytest

from conftest import REPO
from gpaw_b200 import _native as nat


def declared_symbols():
    names = set()
    for h in (REPO / 'include').glob('*.h'):
        text = h.read_text()
        text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
        names |= set(re.findall(r'\b(gb_[a-z0-9_]+)\s*\(', text))
    return sorted(names)


def test_library_builds_and_loads():
    from gpaw_b200.build import build
    build()
    lib = nat.lib()
    assert b'sm_100a' in lib.gb_version()


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(str(nat.LIBPATH))
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_operator_offsets_decode_and_diagonal():
    lib = nat.lib()
    n_c = np.array([5, 6, 7])
    mp = 2
    M = n_c + 2 * mp
    offs = np.array([[0, 0, 0], [2, 0, 0], [0, -2, 0], [0, 0, 1], [-1, 0, 0]])
    offset_p = offs.dot([M[1] * M[2], M[2], 1])
    coef = np.array([-3.0, 1.0, 0.5, 0.25, 2.0])
    h = ctypes.c_void_p()
    rc = lib.gb_operator_new(nat.f64(coef), nat.i64(offset_p), len(coef),
                             nat.i64(n_c), mp, nat.i64(-np.ones(6)), 1, 1,
                             ctypes.byref(h))
    assert rc == 0
    d = ctypes.c_double()
    assert lib.gb_operator_get_diagonal_element(h, ctypes.byref(d)) == 0
    assert d.value == -3.0
    lib.gb_operator_free(h)


def test_operator_rejects_bad_arguments():
    lib = nat.lib()
    h = ctypes.c_void_p()
    # stencil longer than the domain (gpaw/fd_operators.py:53)
    rc = lib.gb_operator_new(nat.f64([1.0]), nat.i64([0]), 1, nat.i64([2, 8, 8]),
                             3, nat.i64(-np.ones(6)), 1, 1, ctypes.byref(h))
    assert rc == -1 and b'longer than domain' in lib.gb_last_error()
    rc = lib.gb_operator_new(nat.f64([]), nat.i64([0]), 0, nat.i64([8, 8, 8]),
                             1, nat.i64(-np.ones(6)), 1, 1, ctypes.byref(h))
    assert rc == -1
    # dtype / real flag mismatch is caught on the host, before any launch
    rc = lib.gb_operator_new(nat.f64([1.0]), nat.i64([0]), 1, nat.i64([8, 8, 8]),
                             1, nat.i64(-np.ones(6)), 1, 1, ctypes.byref(h))
    assert rc == 0
    rc = lib.gb_operator_apply(h, ctypes.c_void_p(16), ctypes.c_void_p(32), 1,
                               2, None, None)
    assert rc == -1 and b'real/complex' in lib.gb_last_error()
    rc = lib.gb_operator_apply(h, ctypes.c_void_p(16), ctypes.c_void_p(32), 1,
                               7, None, None)
    assert rc == -1
    assert lib.gb_operator_apply(h, None, None, 0, 0, None, None) == 0
    lib.gb_operator_free(h)


def test_transformer_geometry_validation():
    from oracle.fd import transformer_geometry
    lib = nat.lib()
    h = ctypes.c_void_p()
    for pbc in (0, 1):
        beg = np.array([0, 0, 0]) if pbc else np.array([1, 1, 1])
        N = np.array([16, 16, 20])
        for nn in (1, 2, 3, 4):
            pad, npad, skip = transformer_geometry(beg, N, beg, N // 2, nn, True)
            rc = lib.gb_transformer_new(nat.i64(N - beg), nat.i64(N // 2 - beg), 2 * nn,
                                        nat.i64(pad), nat.i64(npad), nat.i64(skip),
                                        nat.i64(np.full(6, 0 if pbc else -1)), 1, 0,
                                        ctypes.byref(h))
            assert rc == 0, lib.gb_last_error()
            lib.gb_transformer_free(h)
            pad, npad, skip = transformer_geometry(beg, N // 2, beg, N, nn, False)
            rc = lib.gb_transformer_new(nat.i64(N // 2 - beg), nat.i64(N - beg), 2 * nn,
                                        nat.i64(pad), nat.i64(npad), nat.i64(skip),
                                        nat.i64(np.full(6, 0 if pbc else -1)), 1, 1,
                                        ctypes.byref(h))
            assert rc == 0, lib.gb_last_error()
            lib.gb_transformer_free(h)
            # inconsistent output size is rejected
            rc = lib.gb_transformer_new(nat.i64(N // 2 - beg), nat.i64(N - beg + 1), 2 * nn,
                                        nat.i64(pad), nat.i64(npad), nat.i64(skip),
                                        nat.i64(np.full(6, 0 if pbc else -1)), 1, 1,
                                        ctypes.byref(h))
            assert rc == -1
    rc = lib.gb_transformer_new(nat.i64([8, 8, 8]), nat.i64([4, 4, 4]), 3,
                                nat.i64(np.zeros(6)), nat.i64(np.zeros(6)),
                                nat.i64(np.zeros(6)), nat.i64(np.zeros(6)), 1, 0,
                                ctypes.byref(h))
    assert rc == -1


def test_product_path_fails_loudly_without_cuda_tensors():
    import torch
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    gd = GridDescriptor((8, 8, 8), (2.0, 2.0, 2.0), device='cpu')
    lap = Laplace(gd, -0.5, 2)
    a = torch.zeros(tuple(gd.n_c), dtype=torch.float64)
    with pytest.raises(nat.GPAWB200Error):
        lap.apply(a, torch.zeros_like(a))


def test_fold_fine_refuses_an_output_overlapping_its_inputs():
    """The folded network's fine part writes y before its coarse part reads
    xc and adds into y, so an aliased output is refused on the host, before
    any launch (the check needs no GPU)."""
    lib = nat.lib()
    n_c = np.array([16, 16, 16], np.int64)
    nb = 2
    nf = nb * int(np.prod(n_c))
    xf = np.zeros(nf, np.float32)
    xc = np.zeros(nb * 16 * int(np.prod(n_c // 2)), np.float32)
    F = np.zeros(125, np.float32)
    G = np.zeros(16 * 216, np.float32)
    p = lambda a, off=0: ctypes.c_void_p(a.ctypes.data + 4 * off)
    for out in (p(xf), p(xf, nf // 2), p(xc, 100)):
        rc = lib.gb_learned_fold_fine(p(xf), p(F), 2, p(xc), p(G), 16, out, nb,
                                      nat.i64(n_c), None)
        assert rc == -1 and b'overlaps' in lib.gb_last_error()
