"""Single-domain uniform real-space grid (mirror of gpaw.grid_descriptor).

Geometry contract kept from the reference (gpaw/grid_descriptor.py:113-157,
gpaw/domain.py:110-138):

* ``N_c`` grid points per axis; on a non-periodic (zero-boundary) axis the
  first point (the boundary itself) is dropped, so ``beg_c = 1`` and
  ``n_c = N_c - 1``; on a periodic axis ``beg_c = 0`` and ``n_c = N_c``.
* ``h_cv = cell_cv / N_c``, ``dv = volume / prod(N_c)`` (Bohr units).
* ``neighbor_cd`` is 0 (this domain) on periodic axes and -1 on zero-boundary
  axes; ``sdisp_cd`` = (+1, -1) on periodic axes, which makes the Bloch phase
  ``phase_cd = exp(2 pi i sdisp_cd k_c)`` (gpaw/kpt_descriptor.py:281-284).

Arrays are torch tensors (CUDA by default).  One process owns the whole grid:
the domain decomposition of the reference is out of scope on one GPU.
"""
from __future__ import annotations

import numbers

import numpy as np
import torch


class SerialCommunicator:
    """Size-1 communicator (the reference's gpaw.mpi.SerialCommunicator)."""
    size = 1
    rank = 0

    def sum(self, a, root=-1):
        return a

    def sum_scalar(self, a, root=-1):
        return a

    def max(self, a, root=-1):
        return a

    def broadcast(self, a, root):
        return a

    def barrier(self):
        pass

    def all_gather(self, a, b):
        b[:] = a

    def get_c_object(self):
        return None


serial_comm = SerialCommunicator()

_DTYPES = {float: torch.float64, complex: torch.complex128,
           np.float64: torch.float64, np.float32: torch.float32,
           np.complex128: torch.complex128, np.complex64: torch.complex64}


def torch_dtype(dtype) -> torch.dtype:
    if isinstance(dtype, torch.dtype):
        return dtype
    if dtype in _DTYPES:
        return _DTYPES[dtype]
    return _DTYPES[np.dtype(dtype).type]


def is_real(dtype) -> bool:
    return not torch_dtype(dtype).is_complex


class GridDescriptor:
    """Uniform grid over a (possibly non-orthogonal) unit cell."""

    ndim = 3

    def __init__(self, N_c, cell_cv=(1, 1, 1), pbc_c=True, comm=None,
                 parsize_c=None, allow_empty_domains=False,
                 device: str | torch.device = 'cuda'):
        if isinstance(pbc_c, (int, bool, np.bool_)):
            pbc_c = (bool(pbc_c),) * 3
        self.N_c = np.array(N_c, int)
        if (self.N_c != np.asarray(N_c)).any():
            raise ValueError('Non-int number of grid points %s' % (N_c,))
        cell = np.array(cell_cv, float)
        self.cell_cv = np.diag(cell) if cell.ndim == 1 else cell
        self.icell_cv = np.linalg.inv(self.cell_cv).T
        self.pbc_c = np.asarray(pbc_c, bool)
        self.comm = serial_comm if comm is None else comm
        if self.comm.size != 1:
            raise NotImplementedError('one domain per GPU: comm.size must be 1')
        self.parsize_c = np.ones(3, int)
        self.parpos_c = np.zeros(3, int)
        self.device = torch.device(device)

        self.beg_c = np.where(self.pbc_c, 0, 1).astype(int)
        self.end_c = self.N_c.copy()
        self.n_c = self.end_c - self.beg_c
        if (self.n_c <= 0).any():
            raise ValueError('Grid %s too small' % self.N_c)
        self.h_cv = self.cell_cv / self.N_c[:, np.newaxis]
        self.volume = abs(np.linalg.det(self.cell_cv))
        self.dv = self.volume / self.N_c.prod()
        self.orthogonal = not (self.cell_cv -
                               np.diag(self.cell_cv.diagonal())).any()
        self.neighbor_cd = np.where(self.pbc_c[:, None], 0, -1) * np.ones(
            (3, 2), int)
        self.neighbor_cd = np.ascontiguousarray(self.neighbor_cd.astype(int))
        self.sdisp_cd = np.zeros((3, 2), int)
        self.sdisp_cd[self.pbc_c, 0] = 1
        self.sdisp_cd[self.pbc_c, 1] = -1

    def __repr__(self):
        return ('GridDescriptor(%s, cell_cv=%s, pbc_c=%s)'
                % (self.N_c.tolist(), self.cell_cv.tolist(),
                   self.pbc_c.astype(int).tolist()))

    # -- descriptors -------------------------------------------------------
    def new_descriptor(self, N_c=None, cell_cv=None, pbc_c=None, comm=None,
                       parsize_c=None, allow_empty_domains=False):
        return self.__class__(self.N_c if N_c is None else N_c,
                              self.cell_cv if cell_cv is None else cell_cv,
                              self.pbc_c if pbc_c is None else pbc_c,
                              self.comm if comm is None else comm,
                              device=self.device)

    def coarsen(self):
        if (self.N_c % 2).any():
            raise ValueError('Grid %s not divisible by 2!' % self.N_c)
        return self.new_descriptor(self.N_c // 2)

    def refine(self):
        return self.new_descriptor(self.N_c * 2)

    def get_grid_spacings(self):
        L_c = (np.linalg.inv(self.cell_cv)**2).sum(0)**-0.5
        return L_c / self.N_c

    def get_size_of_global_array(self, pad=False):
        return self.N_c if pad else self.N_c - 1 + self.pbc_c

    def flat_index(self, G_c):
        g1, g2, g3 = np.asarray(G_c) - self.beg_c
        return g3 + self.n_c[2] * (g2 + g1 * self.n_c[1])

    def phase_factor_cd(self, k_c):
        """Bloch phases exp(2 pi i sdisp_cd k_c) (gpaw/kpt_descriptor.py:283)."""
        k_c = np.asarray(k_c, float)
        return np.exp(2j * np.pi * self.sdisp_cd * k_c[:, np.newaxis])

    # -- arrays ------------------------------------------------------------
    def _new_array(self, n=(), dtype=float, zero=True, global_array=False,
                   pad=False, xp=None):
        shape = (self.get_size_of_global_array(pad) if global_array
                 else self.n_c)
        if isinstance(n, numbers.Integral):
            n = (n,)
        shape = tuple(n) + tuple(int(s) for s in shape)
        device = self.device if xp is None else (
            torch.device('cpu') if xp is np else xp)
        f = torch.zeros if zero else torch.empty
        return f(shape, dtype=torch_dtype(dtype), device=device)

    def zeros(self, n=(), dtype=float, global_array=False, pad=False,
              xp=None):
        return self._new_array(n, dtype, True, global_array, pad, xp)

    def empty(self, n=(), dtype=float, global_array=False, pad=False,
              xp=None):
        return self._new_array(n, dtype, False, global_array, pad, xp)

    def integrate(self, a_xg, b_yg=None, global_integral=True,
                  hermitian=False):
        """Integrals over the cell; with b_yg: <a_x|b_y> = dv sum a^* b."""
        xshape = a_xg.shape[:-3]
        if b_yg is None:
            r = a_xg.reshape(xshape + (-1,)).sum(-1) * self.dv
            return r.item() if r.ndim == 0 else r
        A = a_xg.reshape(-1, int(np.prod(a_xg.shape[-3:])))
        B = b_yg.reshape(-1, int(np.prod(b_yg.shape[-3:])))
        r = (A.conj() @ B.T) * self.dv
        r = r.reshape(xshape + b_yg.shape[:-3])
        return r.item() if r.ndim == 0 else r

    # -- atom-centred boxes (gpaw/grid_descriptor.py:344-411) ---------------
    def get_boxes(self, spos_c, rcut, cut=True):
        """Boxes of grid points enclosing a sphere, with their periodic
        displacements, exactly as GridDescriptor.get_boxes of the reference."""
        N_c = self.N_c
        ncut = rcut * (self.icell_cv**2).sum(axis=1)**0.5 * self.N_c
        npos_c = np.asarray(spos_c) * N_c
        beg_c = np.ceil(npos_c - ncut).astype(int)
        end_c = np.ceil(npos_c + ncut).astype(int)
        if cut:
            for c in range(3):
                if not self.pbc_c[c]:
                    beg_c[c] = max(beg_c[c], 0)
                    end_c[c] = min(end_c[c], N_c[c])
        else:
            for c in range(3):
                if not self.pbc_c[c] and (beg_c[c] < 0 or end_c[c] > N_c[c]):
                    raise GridBoundsError(
                        'Box at %.3f %.3f %.3f crosses boundary.' %
                        tuple(spos_c))
        range_c = ([], [], [])
        for c in range(3):
            b = beg_c[c]
            e = b
            while e < end_c[c]:
                b0 = b % N_c[c]
                e = min(end_c[c], b + N_c[c] - b0)
                b1 = b + self.beg_c[c] - b0 if b0 < self.beg_c[c] else b
                e0 = b0 - b + e
                e1 = e - (e0 - self.end_c[c]) if e0 > self.end_c[c] else e
                if e1 > b1:
                    range_c[c].append((b1, e1))
                b = e
        boxes = []
        for b0, e0 in range_c[0]:
            for b1, e1 in range_c[1]:
                for b2, e2 in range_c[2]:
                    b = np.array((b0, b1, b2))
                    e = np.array((e0, e1, e2))
                    beg = np.array((b0 % N_c[0], b1 % N_c[1], b2 % N_c[2]))
                    end = beg + e - b
                    disp = (b - beg) / N_c
                    beg = np.maximum(beg, self.beg_c)
                    end = np.minimum(end, self.end_c)
                    if (beg < end).all():
                        boxes.append((beg, end, disp))
        return boxes

    def get_rank_from_position(self, spos_c):
        return 0


class GridBoundsError(ValueError):
    pass
