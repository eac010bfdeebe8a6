"""Exchange-correlation on the grid (drop-in for gpaw.xc: XC('LDA'),
XC('PBE'), XCKernel, LDA, GGA).

* ``XCKernel(name).calculate(e_g, n_sg, dedn_sg, sigma_xg, dedsigma_xg)``
  (gpaw/xc/kernel.py:38-58): point kernel, e_g and dedsigma overwritten,
  dedn ADDED to -- one gb_xc_calculate launch.
* ``LDA.calculate(gd, n_sg, v_sg, e_g)`` / ``GGA.calculate(...)`` return the
  energy (gpaw/xc/functional.py:40-61); GGA builds sigma from Gradient(nn=2)
  stencils and adds the correction  v -= 2 div(de/dsigma grad n)
  (gpaw/xc/gga.py:106-163, 177-200), all on the GPU.
Arrays are float64 CUDA tensors (XC stays FP64 in every precision mode).
"""
from __future__ import annotations

import torch

from gpaw_b200 import _native as nat

codes = {'LDA': -1, 'PBE': 0, 'revPBE': 1, 'RPBE': 2}


class XCKernel:
    def __init__(self, name):
        if name not in codes:
            raise ValueError(f'unsupported functional {name!r}; this build has '
                             f'{sorted(codes)}')
        self.name = name
        self.type = 'LDA' if name == 'LDA' else 'GGA'
        self.code = codes[name]

    def calculate(self, e_g, n_sg, dedn_sg, sigma_xg=None, dedsigma_xg=None,
                  tau_sg=None, dedtau_sg=None):
        nspins = n_sg.shape[0]
        assert 1 <= nspins <= 2
        G = tuple(n_sg.shape[1:])
        arrays = [e_g, n_sg, dedn_sg]
        assert tuple(e_g.shape) == G and tuple(dedn_sg.shape) == (nspins,) + G
        if self.type == 'GGA':
            assert tuple(sigma_xg.shape) == (2 * nspins - 1,) + G
            assert tuple(dedsigma_xg.shape) == (2 * nspins - 1,) + G
            arrays += [sigma_xg, dedsigma_xg]
        for a in arrays:
            if a.dtype != torch.float64:
                raise ValueError('XC arrays are float64')
        nat.require_cuda(*arrays)
        ng = e_g.numel()
        nat.check(nat.lib().gb_xc_calculate(
            self.code, nspins, ng, nat.ptr(e_g), nat.ptr(n_sg), nat.ptr(dedn_sg),
            nat.ptr(sigma_xg) if sigma_xg is not None else None,
            nat.ptr(dedsigma_xg) if dedsigma_xg is not None else None,
            nat.stream_of(e_g)), 'gb_xc_calculate')


class XCFunctional:
    def __init__(self, name, type):
        self.name = name
        self.type = type
        self.gd = None

    def set_grid_descriptor(self, gd):
        self.gd = gd

    def calculate(self, gd, n_sg, v_sg=None, e_g=None):
        """Energy; v_sg is ADDED to (reference semantics)."""
        if gd is not self.gd:
            self.set_grid_descriptor(gd)
        if e_g is None:
            e_g = gd.empty()
        if v_sg is None:
            v_sg = torch.zeros_like(n_sg)
        self.calculate_impl(gd, n_sg, v_sg, e_g)
        return gd.integrate(e_g)


class LDA(XCFunctional):
    def __init__(self, kernel):
        self.kernel = kernel
        XCFunctional.__init__(self, kernel.name, kernel.type)

    def calculate_impl(self, gd, n_sg, v_sg, e_g):
        self.kernel.calculate(e_g, n_sg, v_sg)


class GGA(XCFunctional):
    def __init__(self, kernel, stencil=2):
        XCFunctional.__init__(self, kernel.name, kernel.type)
        self.kernel = kernel
        self.stencil_range = stencil

    def set_grid_descriptor(self, gd):
        from gpaw_b200.fd_operators import Gradient
        XCFunctional.set_grid_descriptor(self, gd)
        self.grad_v = [Gradient(gd, v, n=self.stencil_range) for v in range(3)]

    def calculate_impl(self, gd, n_sg, v_sg, e_g):
        nspins = n_sg.shape[0]
        # sigma and grad n (gpaw/xc/gga.py:106-133): one stencil launch per
        # Cartesian direction covers both spins
        gradn_vsg = torch.empty((3,) + tuple(n_sg.shape), dtype=n_sg.dtype,
                                device=n_sg.device)
        for v in range(3):
            self.grad_v[v].apply(n_sg, gradn_vsg[v])
        sigma_xg = torch.empty((2 * nspins - 1,) + tuple(n_sg.shape[1:]),
                               dtype=n_sg.dtype, device=n_sg.device)
        sigma_xg[::2] = (gradn_vsg**2).sum(0)
        if nspins == 2:
            sigma_xg[1] = (gradn_vsg[:, 0] * gradn_vsg[:, 1]).sum(0)
        dedsigma_xg = torch.empty_like(sigma_xg)
        self.kernel.calculate(e_g, n_sg, v_sg, sigma_xg, dedsigma_xg)
        # v_s -= 2 div(dedsigma_ss grad n_s) + div(dedsigma_ud grad n_s')
        # (gpaw/xc/gga.py:136-163)
        flux = torch.empty_like(n_sg)
        out = torch.empty_like(n_sg)
        for v in range(3):
            for s in range(nspins):
                flux[s] = 2.0 * dedsigma_xg[2 * s] * gradn_vsg[v, s]
                if nspins == 2:
                    flux[s] += dedsigma_xg[1] * gradn_vsg[v, 1 - s]
            self.grad_v[v].apply(flux, out)
            v_sg -= out


def XC(name, **kwargs):
    kernel = XCKernel(name)
    if kernel.type == 'LDA':
        return LDA(kernel)
    return GGA(kernel, kwargs.get('stencil', 2))
