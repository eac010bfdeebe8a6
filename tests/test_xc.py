"""XC point kernels and the GGA grid driver.

CPU: the oracle (oracle/xc.py) against golden vectors from the reference's
own C kernels (tests/golden/xc.npz) and, when built, the live extension.
GPU: gb_xc_calculate against the oracle with the input distribution and the
tolerances of gpaw/test/gpu/test_xc_gpu.py (rtol 1e-13), and the GGA
driver (sigma + gradient correction through the Gradient(nn=2) stencils)."""
import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import xc as oxc
from oracle import ref

CODES = (-1, 0, 1, 2)


@pytest.fixture(scope='module')
def golden_xc():
    with np.load(GOLDEN / 'xc.npz') as f:
        return {k: f[k] for k in f.files}


def run_oracle(code, nspins, seed, ng):
    n_sg, sigma_xg = oxc.log_uniform_inputs(seed, nspins, ng)
    e_g = np.zeros(ng)
    v_sg = np.zeros_like(n_sg)
    d_xg = np.zeros_like(sigma_xg)
    oxc.calculate(code, e_g, n_sg, v_sg, sigma_xg if code != -1 else None,
                  d_xg if code != -1 else None)
    return n_sg, sigma_xg, e_g, v_sg, d_xg


@pytest.mark.parametrize('code', CODES)
@pytest.mark.parametrize('nspins', [1, 2])
def test_oracle_xc_matches_golden(golden_xc, code, nspins):
    _, _, e, v, d = run_oracle(code, nspins, 1000 + 10 * code + nspins, 1000)
    key = f'{code}|{nspins}'
    assert np.allclose(e, golden_xc[f'e|{key}'], rtol=1e-13, atol=1e-14)
    assert np.allclose(v, golden_xc[f'v|{key}'], rtol=1e-13, atol=1e-13)
    if code != -1:
        assert np.allclose(d, golden_xc[f'dedsigma|{key}'], rtol=1e-13, atol=1e-13)


@pytest.mark.skipif(not ref.available(), reason='oracle/_ref not built')
@pytest.mark.parametrize('code', CODES)
def test_oracle_xc_matches_live_reference(code):
    g = ref.load()
    for nspins in (1, 2):
        n_sg, sigma_xg, e, v, d = run_oracle(code, nspins, 77, 3000)
        e1 = np.zeros_like(e)
        v1 = np.zeros_like(v)
        d1 = np.zeros_like(d)
        X = g.XCFunctional(code)
        if code == -1:
            X.calculate(e1, n_sg, v1)
        else:
            X.calculate(e1, n_sg, v1, sigma_xg, d1)
        assert np.allclose(e, e1, rtol=1e-13, atol=1e-14)
        assert np.allclose(v, v1, rtol=1e-13, atol=1e-13)
        assert np.allclose(d, d1, rtol=1e-13, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize('code', CODES)
@pytest.mark.parametrize('nspins', [1, 2])
def test_gpu_xc_kernel(golden_xc, code, nspins):
    """gpaw/test/gpu/test_xc_gpu.py tolerances: v, dedsigma atol 1e-7
    rtol 1e-13; e atol 1e-12 rtol 1e-12 (LDA: 1e-13 / 1e-14)."""
    from gpaw_b200.xc import XCKernel
    name = {-1: 'LDA', 0: 'PBE', 1: 'revPBE', 2: 'RPBE'}[code]
    for seed, ng in ((1000 + 10 * code + nspins, 1000), (5, 10000)):
        n_sg, sigma_xg, e, v, d = run_oracle(code, nspins, seed, ng)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        e_g = torch.zeros(ng, dtype=torch.float64, device='cuda')
        v_sg = torch.zeros((nspins, ng), dtype=torch.float64, device='cuda')
        d_xg = torch.zeros((2 * nspins - 1, ng), dtype=torch.float64, device='cuda')
        k = XCKernel(name)
        k.calculate(e_g, t(n_sg), v_sg, t(sigma_xg) if code != -1 else None,
                    d_xg if code != -1 else None)
        tol_v = (1e-13, 1e-13) if code == -1 else (1e-7, 1e-13)
        assert np.allclose(v_sg.cpu().numpy(), v, atol=tol_v[0], rtol=tol_v[1])
        assert np.allclose(e_g.cpu().numpy(), e, atol=1e-12, rtol=1e-12)
        if code != -1:
            assert np.allclose(d_xg.cpu().numpy(), d, atol=1e-7, rtol=1e-13)
        if ng == 1000:
            key = f'{code}|{nspins}'
            assert np.allclose(e_g.cpu().numpy(), golden_xc[f'e|{key}'], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['LDA', 'PBE'])
@pytest.mark.parametrize('nspins', [1, 2])
@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0)])
def test_gpu_gga_driver(name, nspins, pbc):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.xc import XC
    N = np.array((20, 22, 24))
    gd = GridDescriptor(N, 0.2 / 0.529177 * N, pbc)
    rng = np.random.default_rng(2)
    # smooth positive density: sum of Gaussians
    idx = np.indices(tuple(gd.n_c)).astype(float)
    n_sg = np.zeros((nspins,) + tuple(gd.n_c))
    for s in range(nspins):
        for _ in range(3):
            c = rng.random(3) * gd.n_c
            r2 = sum((idx[i] - c[i])**2 for i in range(3))
            n_sg[s] += rng.random() * np.exp(-r2 / 20.0)
        n_sg[s] += 1e-4
    xc = XC(name)
    nt = torch.from_numpy(n_sg).cuda()
    v_sg = torch.zeros_like(nt)
    e_g = gd.empty()
    E = xc.calculate(gd, nt, v_sg, e_g)
    e_ref = np.zeros(tuple(gd.n_c))
    v_ref = np.zeros_like(n_sg)
    if name == 'LDA':
        oxc.calculate(-1, e_ref.reshape(-1), n_sg.reshape(nspins, -1),
                      v_ref.reshape(nspins, -1))
    else:
        oxc.gga_calculate(0, n_sg, gd.h_cv, pbc, v_ref, e_ref)
    assert np.allclose(e_g.cpu().numpy(), e_ref, rtol=1e-12, atol=1e-14)
    assert abs(E - e_ref.sum() * gd.dv) < 1e-11 * abs(E)
    err = np.abs(v_sg.cpu().numpy() - v_ref).max() / np.abs(v_ref).max()
    assert err < 1e-11
