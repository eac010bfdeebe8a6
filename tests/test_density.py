"""Density accumulation nt_G += sum_n f_n |psi_n|^2 (row a9: the role of
_gpaw.add_to_density, c/utilities.c:313-352, called band by band from
gpaw/wavefunctions/fd.py:95-100).

CPU: the golden accumulations made by the reference's own function
(tests/golden/density.npz, inputs regenerated from seed 3) against the
formula, and against the live reference build where it is present.
GPU: gb_add_to_density (one launch for all bands) through the C ABI
against the same golden data -- real and complex, FP64 at 1e-12 and
FP32 / complex64 at 1e-5 (inputs rounded to FP32 first)."""

import numpy as np
import pytest

from conftest import GOLDEN, relerr
from oracle import ref

CASES = {
    'real_4x31': ((31, 31, 31), 4, False),
    'real_7x12x10x14': ((12, 10, 14), 7, False),
    'complex_5x16': ((16, 16, 16), 5, True),
}


def _inputs(name):
    n_c, nb, cplx = CASES[name]
    rng = np.random.default_rng(3)
    psit = rng.standard_normal((nb,) + n_c)
    if cplx:
        psit = psit + 1j * rng.standard_normal(psit.shape)
    return psit, 2.0 - 0.5 * np.arange(nb)


@pytest.fixture(scope='module')
def golden():
    with np.load(GOLDEN / 'density.npz') as f:
        return {k: f[k] for k in f.files}


@pytest.mark.parametrize('name', sorted(CASES))
def test_golden_density_is_the_formula(golden, name):
    psit, f_n = _inputs(name)
    want = 0.25 + np.einsum('n,n...->...', f_n, np.abs(psit)**2)
    assert relerr(golden[name], want) < 1e-14
    if ref.available():
        g = ref.load()
        nt = np.full(psit.shape[1:], 0.25)
        for f, p in zip(f_n, psit):
            g.add_to_density(float(f), np.ascontiguousarray(p), nt)
        assert np.array_equal(nt, golden[name])


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(CASES))
@pytest.mark.parametrize('single', [False, True])
def test_gpu_add_to_density(golden, name, single):
    import torch
    from gpaw_b200 import _native as nat
    psit, f_n = _inputs(name)
    if single:
        psit = psit.astype(np.complex64 if psit.dtype.kind == 'c' else np.float32)
    want = golden[name]
    if single:   # the reference formula on the FP32-rounded inputs
        want = 0.25 + np.einsum('n,n...->...', f_n,
                                np.abs(psit.astype(np.complex128))**2)
    p = torch.from_numpy(psit).cuda()
    f = torch.from_numpy(f_n).cuda()
    nt = torch.full(psit.shape[1:], 0.25, dtype=torch.float64, device='cuda')
    nat.check(nat.lib().gb_add_to_density(
        len(f_n), nat.ptr(f), nat.ptr(p), nat.dtype_code(p),
        int(np.prod(psit.shape[1:])), nat.ptr(nt), nat.stream_of(nt)),
        'gb_add_to_density')
    torch.cuda.synchronize()
    assert relerr(nt.cpu().numpy(), want) < (1e-5 if single else 1e-12)
