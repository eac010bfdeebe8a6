"""GPU parity of LFC add / integrate / derivative (gb_lfc_* through the C
ABI) against the oracle, the reference's golden vectors, and the reference
test suite's known answers (gpaw/test/lfc/test_lf.py, test_derivatives.py).
FP64: 1e-12 norm-wise relative; FP32: 1e-5."""
import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import lfc as ol

pytestmark = pytest.mark.gpu


def cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location('lfc_cases', GOLDEN / 'lfc_cases.py')
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.LFC_CASES


class KD:
    def __init__(self, k_c):
        self.ibzk_qc = np.array([k_c], float)
        self.gamma = False


def build(name, dtype=None):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    N_c, cell, pbc, spos, spl, k = cases()[name]
    gd = GridDescriptor(N_c, cell, pbc)
    splines = [[Spline.from_data(l, rmax, f) for (l, rmax, f) in sj] for sj in spl]
    lfc = LFC(gd, splines, kd=KD(k) if k is not None else None, cut=True,
              dtype=complex if k is not None else float)
    lfc.set_positions(np.array(spos))
    return gd, lfc


def rel(x, y):
    return np.abs(x - y).max() / np.abs(y).max()


@pytest.mark.parametrize('name', ['zero', 'periodic', 'bloch'])
def test_golden_lfc(name):
    g = np.load(GOLDEN / 'lfc.npz')
    gd, lfc = build(name)
    cplx = cases()[name][5] is not None
    q = 0 if cplx else -1
    rng = np.random.default_rng(7)
    nx, Mmax = 2, lfc.Mmax
    c = rng.standard_normal((nx, Mmax))
    a = rng.standard_normal((nx,) + tuple(gd.n_c))
    if cplx:
        c = c + 1j * rng.standard_normal(c.shape)
        a = a + 1j * rng.standard_normal(a.shape)
    c_axi = {i: torch.from_numpy(c[:, lfc.M_a[i]:lfc.M_a[i] + lfc.sphere_a[i].Mmax].copy()).cuda()
             for i in range(len(lfc.sphere_a))}
    b = torch.zeros((nx,) + tuple(gd.n_c), dtype=torch.complex128 if cplx else torch.float64,
                    device='cuda')
    lfc.add(b, c_axi, q)
    assert rel(b.cpu().numpy(), g[f'{name}|add']) < 1e-12
    ad = torch.from_numpy(a).cuda()
    i_axi = lfc.dict(nx)
    cM = lfc.integrate(ad, i_axi, q)
    assert rel(cM.cpu().numpy(), g[f'{name}|integrate']) < 1e-12
    d_axiv = lfc.dict(nx, derivative=True)
    dM = lfc.derivative(ad, d_axiv, q)
    assert rel(dM.cpu().numpy(), g[f'{name}|derivative']) < 1e-12
    for i, d in d_axiv.items():
        M1 = lfc.M_a[i]
        assert torch.equal(d, dM[:, M1:M1 + lfc.sphere_a[i].Mmax])


@pytest.mark.parametrize('name', ['periodic', 'bloch'])
def test_fp32_lfc(name):
    gd, lfc = build(name)
    cplx = cases()[name][5] is not None
    q = 0 if cplx else -1
    rng = np.random.default_rng(3)
    a = rng.standard_normal((3,) + tuple(gd.n_c))
    c = rng.standard_normal((3, lfc.Mmax))
    if cplx:
        a = a + 1j * rng.standard_normal(a.shape)
        c = c + 1j * rng.standard_normal(c.shape)
    t64 = torch.complex128 if cplx else torch.float64
    t32 = torch.complex64 if cplx else torch.float32
    out = {}
    for t in (t64, t32):
        c_axi = {i: torch.from_numpy(c[:, lfc.M_a[i]:lfc.M_a[i] + lfc.sphere_a[i].Mmax].copy()).to('cuda', t)
                 for i in range(len(lfc.sphere_a))}
        b = torch.zeros((3,) + tuple(gd.n_c), dtype=t, device='cuda')
        lfc.add(b, c_axi, q)
        cM = lfc.integrate(torch.from_numpy(a).to('cuda', t), {}, q)
        out[t] = (b.cpu().numpy().astype(complex if cplx else float),
                  cM.cpu().numpy().astype(complex if cplx else float))
    assert rel(out[t32][0], out[t64][0]) < 1e-5
    assert rel(out[t32][1], out[t64][1]) < 1e-5


def test_lf_reproducible():
    """gpaw/test/lfc/test_lf.py: two identical collections give the same
    integral to 1e-13."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    s = Spline.from_data(0, 1.0, [1.0, 0.5, 0.0])
    n, a = 40, 8.0
    vals = []
    for _ in range(2):
        gd = GridDescriptor((n, n, n), (a, a, a))
        c = LFC(gd, [[s], [s], [s]])
        c.set_positions([(0.5, 0.5, 0.25 + 0.25 * i) for i in [0, 1, 2]])
        b = gd.zeros()
        c.add(b)
        vals.append(gd.integrate(b))
    assert vals[0] == pytest.approx(vals[1], abs=1e-13)


def test_derivatives_known_answers():
    """gpaw/test/lfc/test_derivatives.py: orthogonality of add/integrate,
    the -0.2144 golden derivative, and finite differences of integrate."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    a = 4.0
    gd = GridDescriptor(N_c=[16, 20, 20], cell_cv=[a, a + 1, a + 2], pbc_c=(0, 1, 1))
    spos_ac = np.array([[0.25, 0.15, 0.35], [0.5, 0.5, 0.5]])
    s = Spline.from_data(l=0, rmax=2.0, f_g=np.array([1, 0.9, 0.1, 0.0]))
    p = Spline.from_data(l=1, rmax=2.0, f_g=np.array([1, 0.9, 0.1, 0.0]))
    c = LFC(gd, [[s], [s, p]], cut=True, forces=True)
    c.set_positions(spos_ac)
    C_ani = c.dict(3, zero=True)
    C_ani[1][:, 1:] = torch.eye(3, dtype=torch.float64, device='cuda')
    psi = gd.zeros(3)
    c.add(psi, C_ani)
    c.integrate(psi, C_ani)
    d = C_ani[1][:, 1:].diagonal().cpu().numpy()
    assert np.ptp(d) < 4e-6
    C = C_ani[1][:, 1:].cpu().numpy() - np.diag(d)
    assert abs(C).max() < 5e-17 * 10
    d_aniv = c.dict(3, derivative=True)
    c.derivative(psi, d_aniv)
    D = d_aniv[1].cpu().numpy()
    for v in range(3):
        assert abs(D[v - 1, 0, v] + 0.2144) < 5e-5
        D[v - 1, 0, v] = 0
    assert abs(D).max() < 3e-16 * 10
    eps = 0.0001
    pos_av = np.dot(spos_ac, gd.cell_cv)
    D0 = d_aniv[0].cpu().numpy()
    for v in range(3):
        pos_av[0, v] += eps
        c.set_positions(np.dot(pos_av, gd.icell_cv.T))
        c.integrate(psi, C_ani)
        C0 = C_ani[0][:, 0].cpu().numpy().copy()
        pos_av[0, v] -= 2 * eps
        c.set_positions(np.dot(pos_av, gd.icell_cv.T))
        c.integrate(psi, C_ani)
        C0 -= C_ani[0][:, 0].cpu().numpy()
        C0 /= -2 * eps
        assert abs(C0 - D0[:, 0, v]).max() < 1e-8
        pos_av[0, v] += eps


def microbench_lfc(n=96, natoms=64, h_ang=0.2, seed=0):
    """The kernel-microbench LFC: natoms atom-centred Gaussians
    exp(-(r/0.8 A)^2) with l = 0, 1, 2 (9 functions per atom), cutoff 2.5 A,
    seeded uniform positions on an n^3 periodic grid with h = 0.2 A."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    bohr = 0.52917721
    rc = 2.5 / bohr
    r = np.linspace(0, rc, 101)
    f = np.exp(-(r / (0.8 / bohr))**2)
    L = n * h_ang / bohr
    gd = GridDescriptor((n, n, n), (L, L, L), True)
    spl = [Spline.from_data(l, rc, f) for l in (0, 1, 2)]
    rng = np.random.default_rng(seed)
    spos = rng.random((natoms, 3))
    lfc = LFC(gd, [spl] * natoms)
    lfc.set_positions(spos)
    return gd, lfc, spos, [(l, rc, f) for l in (0, 1, 2)]


def test_microbench_small_vs_oracle():
    gd, lfc, spos, spl = microbench_lfc(n=40, natoms=8)
    Phi = ol.dense_functions(gd.N_c, gd.cell_cv, gd.pbc_c, spos, [spl] * 8)
    rng = np.random.default_rng(1)
    c = rng.standard_normal((4, lfc.Mmax))
    a = rng.standard_normal((4,) + tuple(gd.n_c))
    b = torch.zeros((4,) + tuple(gd.n_c), dtype=torch.float64, device='cuda')
    lfc.add(b, {i: torch.from_numpy(c[:, 9 * i:9 * i + 9].copy()).cuda() for i in range(8)})
    assert rel(b.cpu().numpy(), ol.add(np.zeros_like(a), c, Phi)) < 1e-12
    cM = lfc.integrate(torch.from_numpy(a).cuda(), {})
    assert rel(cM.cpu().numpy(), ol.integrate(a, Phi, gd.dv)) < 1e-12


def test_microbench_full_size_adjoint():
    """96^3, 64 atoms x 9 functions, 256 bands: add and integrate are
    adjoint (<a, add(c)> dv = <integrate(a), c>) band by band, and a batch
    permutation permutes the outputs."""
    gd, lfc, spos, spl = microbench_lfc()
    g = torch.Generator(device='cuda').manual_seed(0)
    nx = 256
    a = torch.randn((nx,) + tuple(gd.n_c), generator=g, device='cuda', dtype=torch.float64)
    c = torch.randn((nx, lfc.Mmax), generator=g, device='cuda', dtype=torch.float64)
    b = torch.zeros_like(a)
    lfc.add(b, {i: c[:, 9 * i:9 * i + 9].contiguous() for i in range(64)})
    cM = lfc.integrate(a, {})
    lhs = (a * b).sum(dim=(1, 2, 3)) * gd.dv
    rhs = (cM * c).sum(dim=1)
    assert ((lhs - rhs).abs() / rhs.abs().clamp_min(1e-3)).max().item() < 1e-11
    perm = torch.randperm(nx, device='cuda')
    cM2 = lfc.integrate(a[perm].contiguous(), {})
    assert torch.equal(cM2, cM[perm])


def _dense_lfc(nfun, natoms=12, n=24, rc_ang=2.2, seed=5):
    """natoms atoms with nfun functions each (l = 0, 1 radial functions
    up to nfun) in a small periodic box, cutoffs large enough that a point
    lies in up to ~natoms spheres."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    bohr = 0.52917721
    rc = rc_ang / bohr
    r = np.linspace(0, rc, 61)
    ls = {1: [0], 4: [0, 1], 8: [0, 1, 0, 1], 9: [0, 1, 0, 1, 0], 12: [0, 1, 0, 1, 0, 1]}[nfun]
    spl = [(l, rc, np.exp(-(r / (0.9 / bohr))**2) * (1 + 0.3 * j)) for j, l in enumerate(ls)]
    L = n * 0.2 / bohr
    gd = GridDescriptor((n, n, n), (L, L, L), True)
    spos = np.random.default_rng(seed).random((natoms, 3))
    lfc = LFC(gd, [[Spline.from_data(*s) for s in spl]] * natoms)
    lfc.set_positions(spos)
    return gd, lfc, spos, spl


@pytest.mark.parametrize('nfun', [1, 4, 8, 9, 12])
def test_add_all_bands_vs_oracle(nfun):
    """The all-band real add (contributions held in registers, the rest
    re-read; full 16-byte coefficient rows or element loads; a band tail)
    against the oracle's dense sum in FP64, FP32 within 1e-5 of it, and an
    unaligned coefficient array (element loads) equal to the aligned one."""
    gd, lfc, spos, spl = _dense_lfc(nfun)
    Phi = ol.dense_functions(gd.N_c, gd.cell_cv, gd.pbc_c, spos, [spl] * len(spos))
    assert lfc.Mmax == nfun * len(spos)
    rng = np.random.default_rng(11)
    nx = 11
    c = rng.standard_normal((nx, lfc.Mmax))
    a0 = rng.standard_normal((nx,) + tuple(gd.n_c))
    want = ol.add(a0.copy(), c, Phi)
    b = torch.from_numpy(a0).cuda()
    lfc.add_M(b, torch.from_numpy(c).cuda())
    assert rel(b.cpu().numpy(), want) < 1e-12
    b32 = torch.from_numpy(a0).cuda().float()
    lfc.add_M(b32, torch.from_numpy(c).cuda().float())
    assert rel(b32.double().cpu().numpy(), want) < 1e-5
    # the same coefficients at an address 4 bytes past a 16-byte boundary
    buf = torch.zeros(nx * lfc.Mmax + 1, dtype=torch.float32, device='cuda')
    cu = buf[1:].view(nx, lfc.Mmax)
    cu.copy_(torch.from_numpy(c))
    b32u = torch.from_numpy(a0).cuda().float()
    lfc.add_M(b32u, cu)
    assert torch.equal(b32u, b32)


def test_add_all_bands_equals_band_blocks():
    """Adding all bands at once equals adding them in blocks of 10 (the
    reference's RMM-DIIS block size), bit for bit."""
    gd, lfc, spos, spl = _dense_lfc(8)
    g = torch.Generator(device='cuda').manual_seed(2)
    nx = 37
    c = torch.randn((nx, lfc.Mmax), generator=g, device='cuda', dtype=torch.float32)
    a0 = torch.randn((nx,) + tuple(gd.n_c), generator=g, device='cuda', dtype=torch.float32)
    b = a0.clone()
    lfc.add_M(b, c)
    b2 = a0.clone()
    for x in range(0, nx, 10):
        lfc.add_M(b2[x:x + 10], c[x:x + 10].contiguous())
    assert torch.equal(b, b2)


def _tiled_case(natoms, n_c, rc_ang, nfun=8, seed=9):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    bohr = 0.52917721
    rc = rc_ang / bohr
    r = np.linspace(0, rc, 61)
    ls = {1: [0], 4: [0, 1], 8: [0, 1, 0, 1]}[nfun]
    spl = [(l, rc, np.exp(-(r / (0.9 / bohr))**2) * (1 + 0.3 * j)) for j, l in enumerate(ls)]
    gd = GridDescriptor(n_c, np.array(n_c) * 0.2 / bohr, True)
    spos = np.random.default_rng(seed).random((natoms, 3))
    lfc = LFC(gd, [[Spline.from_data(*s) for s in spl]] * natoms)
    lfc.set_positions(spos)
    Phi = ol.dense_functions(gd.N_c, gd.cell_cv, gd.pbc_c, spos, [spl] * natoms)
    return gd, lfc, Phi


@pytest.mark.parametrize('natoms,n_c,rc,nfun', [
    (10, (20, 22, 26), 1.6, 8),   # 11440 points: the last 32-point chunk is partial
    (36, (24, 24, 24), 1.1, 4),   # <= 14 groups per chunk, bricks split at 16
    (9, (16, 20, 18), 1.4, 1),    # one function per atom
])
@pytest.mark.parametrize('nx', [1, 37, 300])
def test_fp32_tiled_add_integrate(natoms, n_c, rc, nfun, nx):
    """The chunk-tiled FP32 add / integrate (gb_lfc_tiled objects) against
    the oracle's dense sums within 1e-5, band counts of one pass (1, 37) and
    of two (300 = 256 + 44); deterministic (two integrates are equal), band
    blocks of 10 equal to one call, and add / integrate adjoint."""
    from gpaw_b200 import _native as nat
    gd, lfc, Phi = _tiled_case(natoms, n_c, rc, nfun)
    assert nat.lib().gb_lfc_tiled(lfc.lfc.handle) == 1
    rng = np.random.default_rng(nx)
    c = rng.standard_normal((nx, lfc.Mmax))
    a0 = rng.standard_normal((nx,) + tuple(gd.n_c))
    want_add = ol.add(a0.copy(), c, Phi)
    want_int = ol.integrate(a0, Phi, gd.dv)
    b = torch.from_numpy(a0).cuda().float()
    c32 = torch.from_numpy(c).cuda().float()
    lfc.add_M(b, c32)
    assert rel(b.double().cpu().numpy(), want_add) < 1e-5
    a32 = torch.from_numpy(a0).cuda().float()
    cM = lfc.integrate(a32, {})
    assert rel(cM.double().cpu().numpy(), want_int) < 1e-5
    assert torch.equal(lfc.integrate(a32, {}), cM)
    b2 = torch.from_numpy(a0).cuda().float()
    for x in range(0, nx, 10):
        lfc.add_M(b2[x:x + 10], c32[x:x + 10].contiguous())
    assert torch.equal(b2, b)
    cM2 = torch.cat([lfc.integrate(a32[x:x + 10], {}) for x in range(0, nx, 10)])
    assert torch.equal(cM2, cM)


def test_fp32_tiled_fallback_when_a_chunk_meets_too_many_groups():
    """More than 16 function groups over one 32-point chunk: the object keeps
    the point-major kernels, with the same results."""
    from gpaw_b200 import _native as nat
    gd, lfc, Phi = _tiled_case(40, (16, 16, 16), 3.0, nfun=1)
    assert nat.lib().gb_lfc_tiled(lfc.lfc.handle) == 0
    rng = np.random.default_rng(1)
    c = rng.standard_normal((5, lfc.Mmax))
    a0 = rng.standard_normal((5,) + tuple(gd.n_c))
    b = torch.from_numpy(a0).cuda().float()
    lfc.add_M(b, torch.from_numpy(c).cuda().float())
    assert rel(b.double().cpu().numpy(), ol.add(a0.copy(), c, Phi)) < 1e-5
