"""Localized functions collection on the GPU (drop-in for gpaw.lfc.LFC).

``LocalizedFunctionsCollection(gd, spline_aj, kd, cut, dtype, integral,
forces)`` with ``set_positions``, ``add``, ``integrate``, ``derivative``,
``dict`` like gpaw/lfc.py:205-724.  Coefficients are dicts of CUDA tensors
keyed by atom index (``c_axi[a]`` of shape xshape + (ni,)), grids are CUDA
tensors (..., n0, n1, n2).

When positions change, every atom-centred function f_j(|r - R|) r^l Y_lm
is tabulated on the grid points of its boxes by the device spline_to_grid
(gb_spline_to_grid, c/lfc.c:887-977; boxes by the rule of
gpaw/grid_descriptor.py:344-411), the boundary events are sorted
(gpaw/lfc.py:259-374) and handed to gb_lfc_new, which builds the device
indices once.  add / integrate / derivative are then one or a few kernel
launches for all bands; the derivative evaluates the splines' slopes on the
device (gb_lfc_derivative).  Grid descriptors on the CPU (host-side set-up
checks only) tabulate with numpy instead.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from gpaw_b200 import _native as nat
from gpaw_b200.spline import rlYlm


def spline_to_grid(spline, beg_c, end_c, pos_v, h_cv, n_c, gdcorner_c, device='cuda'):
    """_gpaw.spline_to_grid on the device: (A_gm, G_B) -- f(r) r^l Y_lm at
    the box points with r < rmax as a CUDA tensor (ng, 2l + 1), rows (g0, g1)
    in order and g2 increasing, and the [start, end) runs of those points
    in the local grid's flat index (int32 numpy array)."""
    beg_c = np.asarray(beg_c, np.int64)
    end_c = np.asarray(end_c, np.int64)
    ext = np.maximum(end_c - beg_c, 0)
    nm = 2 * spline.l + 1
    npts = int(np.prod(ext))
    A = torch.empty((max(npts, 1), nm), dtype=torch.float64, device=device)
    G = torch.empty(max(2 * int(ext[0] * ext[1]), 2), dtype=torch.int32, device=device)
    ng = ctypes.c_int64()
    nB = ctypes.c_int64()
    nat.check(nat.lib().gb_spline_to_grid(
        spline.handle, nat.i64(beg_c), nat.i64(end_c), nat.f64(pos_v),
        nat.f64(np.ascontiguousarray(h_cv)), nat.i64(n_c), nat.i64(gdcorner_c),
        nat.ptr(A), nat.ptr(G), ctypes.byref(ng), ctypes.byref(nB),
        nat.stream_of(A)), 'gb_spline_to_grid')
    return A[:ng.value], G[:nB.value].cpu().numpy()


def _box_functions(spline, beg_c, end_c, pos_v, gd):
    """Values of one radial function on one box: (A_gm, G_b) as
    spline_to_grid returns them (rows in g0, g1, g2 order, runs along g2).
    On a CUDA grid descriptor the values come from the device
    spline_to_grid; on a CPU one (host-side set-up checks) from numpy."""
    if torch.device(gd.device).type == 'cuda':
        A, G_b = spline_to_grid(spline, beg_c, end_c, pos_v, gd.h_cv, gd.n_c,
                                gd.beg_c, gd.device)
        return A.cpu().numpy(), G_b
    l = spline.l
    rcut = spline.rmax
    g = np.indices(tuple(end_c - beg_c)).reshape(3, -1).T + beg_c
    d = g @ gd.h_cv - pos_v
    r = np.sqrt((d**2).sum(1))
    inside = r < rcut
    g = g[inside]
    d = d[inside]
    r = r[inside]
    f, _ = spline.value_and_derivative(r)
    x, y, z = d.T
    A = np.ascontiguousarray((f * rlYlm(l, x, y, z)).T)    # (ng, nm)
    # flat local index and z-runs
    rel = g - gd.beg_c
    G = (rel[:, 0] * gd.n_c[1] + rel[:, 1]) * gd.n_c[2] + rel[:, 2]
    if len(G) == 0:
        return A, np.zeros(0, np.intc)
    brk = np.nonzero(np.diff(G) != 1)[0]
    starts = np.concatenate([[0], brk + 1])
    ends = np.concatenate([brk + 1, [len(G)]])
    G_b = np.empty(2 * len(starts), np.intc)
    G_b[0::2] = G[starts]
    G_b[1::2] = G[ends - 1] + 1
    return A, G_b


def _run_points(G_b):
    """Grid point indices of the runs [G_b[0], G_b[1]), [G_b[2], G_b[3]), ..."""
    return np.concatenate([np.arange(g0, g1) for g0, g1 in zip(G_b[0::2], G_b[1::2])]) \
        if len(G_b) else np.zeros(0, np.int64)


def _point_runs(G):
    """Inverse of _run_points for a sorted index array."""
    if len(G) == 0:
        return np.zeros(0, np.intc)
    brk = np.nonzero(np.diff(G) != 1)[0]
    starts = np.concatenate([[0], brk + 1])
    ends = np.concatenate([brk + 1, [len(G)]])
    G_b = np.empty(2 * len(starts), np.intc)
    G_b[0::2] = G[starts]
    G_b[1::2] = G[ends - 1] + 1
    return G_b


class Sphere:
    def __init__(self, spline_j):
        self.spline_j = spline_j
        self.spos_c = None
        self.rank = 0
        self.ranks = []
        self.Mmax = sum(2 * s.l + 1 for s in spline_j)
        self.A_wgm = None
        self.G_wb = None
        self.M_w = None
        self.sdisp_wc = None
        self.box_w = None
        self.normalized = False

    def set_position(self, spos_c, gd, cut):
        if self.spos_c is not None and not (self.spos_c - spos_c).any():
            return False
        self.A_wgm, self.G_wb, self.M_w, self.sdisp_wc = [], [], [], []
        self.box_w = []
        M = 0
        for j, spline in enumerate(self.spline_j):
            for beg_c, end_c, sdisp_c in gd.get_boxes(spos_c, spline.rmax, cut):
                pos_v = np.dot(spos_c - sdisp_c, gd.cell_cv)
                A_gm, G_b = _box_functions(spline, beg_c, end_c, pos_v, gd)
                if len(G_b) > 0:
                    self.A_wgm.append(A_gm)
                    self.G_wb.append(G_b)
                    self.M_w.append(M)
                    self.sdisp_wc.append(sdisp_c)
                    self.box_w.append((j, beg_c, end_c, pos_v))
            M += 2 * spline.l + 1
        if not self.A_wgm:
            self.A_wgm = self.G_wb = self.M_w = self.sdisp_wc = None
        self.spos_c = np.array(spos_c, float)
        self.normalized = False
        return True

    def normalize(self, integral, dv):
        """gpaw/lfc.py:126-186 for one domain: scale the l=0 function to the
        given integral and make the others integrate to zero."""
        if self.normalized or integral < 1e-15 or self.A_wgm is None:
            self.normalized = True
            return
        I_M = np.zeros(self.Mmax)
        nw = len(self.A_wgm) // len(self.spline_j)
        for M, A_gm in zip(self.M_w, self.A_wgm):
            I_M[M:M + A_gm.shape[1]] += A_gm.sum(axis=0) * dv
        for w, (M, A_gm) in enumerate(zip(self.M_w, self.A_wgm)):
            if M == 0:
                A_gm *= integral / I_M[0]
            else:
                A_gm -= I_M[M:M + A_gm.shape[1]] / integral * self.A_wgm[w % nw]
        self.normalized = True


class _Native:
    """Owns one gb_lfc handle built from flattened volume data."""

    def __init__(self, A_Wgm, M_W, G_B, W_B, dv, phase_qW, nG, nM):
        nW = len(A_Wgm)
        A_all = (np.concatenate([np.ascontiguousarray(A).ravel() for A in A_Wgm])
                 if nW else np.zeros(1))
        self.A_all = np.ascontiguousarray(A_all, float)
        self.ngm = np.array([A.shape[0] for A in A_Wgm], np.int64)
        self.nm = np.array([int(np.prod(A.shape[1:])) for A in A_Wgm], np.intc)
        self.M_W = np.ascontiguousarray(M_W, np.intc)
        self.G_B = np.ascontiguousarray(G_B, np.intc)
        self.W_B = np.ascontiguousarray(W_B, np.intc)
        self.phase = np.ascontiguousarray(
            np.stack([phase_qW.real, phase_qW.imag], -1).ravel()
            if phase_qW.size else np.zeros(2), float)
        h = ctypes.c_void_p()
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        nat.check(nat.lib().gb_lfc_new(
            nW, P(self.A_all), self.ngm.ctypes.data_as(nat.P64), P(self.nm),
            P(self.M_W), len(self.G_B), P(self.G_B), P(self.W_B), float(dv),
            int(phase_qW.shape[0]) if phase_qW.size else 0, P(self.phase),
            int(nG), int(nM), ctypes.byref(h)), 'gb_lfc_new')
        self.handle = h

    def __del__(self):
        h = getattr(self, 'handle', None)
        if h is not None and h.value:
            try:
                nat.lib().gb_lfc_free(h)
            except Exception:
                pass


class BaseLFC:
    def dict(self, shape=(), derivative=False, zero=False):
        if isinstance(shape, int):
            shape = (shape,)
        tdtype = torch.complex128 if self.dtype == complex else torch.float64
        out = {}
        for a in self.my_atom_indices:
            ni = self.get_function_count(a)
            if derivative:
                assert not zero
                out[a] = torch.empty(shape + (ni, 3), dtype=tdtype, device=self.gd.device)
            else:
                f = torch.zeros if zero else torch.empty
                out[a] = f(shape + (ni,), dtype=tdtype, device=self.gd.device)
        return out

    def get_function_count(self, a):
        return self.sphere_a[a].Mmax


class LocalizedFunctionsCollection(BaseLFC):
    def __init__(self, gd, spline_aj, kd=None, cut=False, dtype=float,
                 integral=None, forces=None, xp=None):
        self.gd = gd
        self.kd = kd
        self.sphere_a = [Sphere(spline_j) for spline_j in spline_aj]
        self.cut = cut
        self.dtype = dtype
        self.Mmax = None
        if kd is None:
            self.ibzk_qc = np.zeros((1, 3))
            self.gamma = True
        else:
            self.ibzk_qc = kd.ibzk_qc
            self.gamma = kd.gamma
        if integral is not None:
            self.integral_a = np.empty(len(spline_aj))
            self.integral_a[:] = integral
        else:
            self.integral_a = None
        self.my_atom_indices = None
        self.lfc = None
        self._deriv = None

    def set_positions(self, spos_ac, atom_partition=None):
        spos_ac = np.asarray(spos_ac, float)
        assert len(spos_ac) == len(self.sphere_a)
        movement = False
        for spos_c, sphere in zip(spos_ac, self.sphere_a):
            movement |= sphere.set_position(spos_c, self.gd, self.cut)
        if movement or self.my_atom_indices is None:
            self._update(spos_ac)

    def _update(self, spos_ac):
        self.my_atom_indices = list(range(len(self.sphere_a)))
        self.atom_indices = []
        self.M_a = []
        M = 0
        for a, sphere in enumerate(self.sphere_a):
            self.M_a.append(M)
            if sphere.G_wb:
                self.atom_indices.append(a)
            M += sphere.Mmax
        self.Mmax = M
        if self.integral_a is not None:
            for a in self.atom_indices:
                self.sphere_a[a].normalize(self.integral_a[a], self.gd.dv)
        # one device volume per (atom, periodic image): the radial functions
        # of an atom are merged onto the union of their sphere points (zeros
        # where a shorter function does not reach), so that add / integrate
        # touch each covered grid point once per atom instead of once per
        # radial function
        A_Wgm, M_W, sdisp_W, G_list, W_list, box_W = [], [], [], [], [], []
        W = 0
        for a in self.atom_indices:
            s = self.sphere_a[a]
            images = {}
            for A_gm, G_b, Mw, sd, box in zip(s.A_wgm, s.G_wb, s.M_w,
                                               s.sdisp_wc, s.box_w):
                images.setdefault(tuple(np.round(sd, 12)), []).append(
                    (A_gm, _run_points(G_b), Mw, box))
            for key, parts in images.items():
                G = parts[0][1]
                for part in parts[1:]:
                    G = np.union1d(G, part[1])
                A = np.zeros((len(G), s.Mmax))
                members = []
                for A_gm, Gp, Mw, box in parts:
                    rows = np.searchsorted(G, Gp)
                    A[rows, Mw:Mw + A_gm.shape[1]] = A_gm
                    members.append((box, rows, Mw))
                A_Wgm.append(A)
                M_W.append(self.M_a[a])
                sdisp_W.append(np.array(key))
                box_W.append((a, len(G), members))
                G_b = _point_runs(G)
                G_list.append(G_b)
                w = np.empty(len(G_b), np.intc)
                w[0::2] = W
                w[1::2] = -W - 1
                W_list.append(w)
                W += 1
        G_B = np.concatenate(G_list) if G_list else np.zeros(0, np.intc)
        W_B = np.concatenate(W_list) if W_list else np.zeros(0, np.intc)
        order = np.argsort(G_B, kind='mergesort')
        self.G_B = G_B[order]
        self.W_B = W_B[order]
        self.M_W = np.array(M_W, np.intc)
        self.sdisp_Wc = np.array(sdisp_W).reshape(-1, 3)
        self.box_W = box_W
        if self.gamma or self.dtype == float:
            self.phase_qW = np.empty((0, len(M_W)), complex)
        else:
            self.phase_qW = np.exp(2j * np.pi * np.inner(self.ibzk_qc, self.sdisp_Wc))
        nG = int(np.prod(self.gd.n_c))
        self.lfc = _Native(A_Wgm, self.M_W, self.G_B, self.W_B, self.gd.dv,
                           self.phase_qW, nG, self.Mmax)
        self._deriv = None

    # -- helpers ------------------------------------------------------------
    def _gather(self, c_axi, xshape, tdtype, device):
        parts = []
        for a, sphere in enumerate(self.sphere_a):
            c = c_axi.get(a) if isinstance(c_axi, dict) else None
            if c is None:
                parts.append(torch.zeros(xshape + (sphere.Mmax,), dtype=tdtype, device=device))
            else:
                parts.append(c.to(device=device, dtype=tdtype))
        c_xM = torch.cat(parts, dim=-1) if parts else torch.zeros(
            xshape + (0,), dtype=tdtype, device=device)
        return c_xM.contiguous()

    def _nq(self, a_xG, q):
        if a_xG.dtype.is_complex and q >= 0 and self.phase_qW.shape[0] == 0:
            return -1
        return q

    @staticmethod
    def _kbatch(q):
        """q = range(nk): the rows are nk equal groups, group k at k-point
        q = k (one launch for the batch); returns nk, or 0 for a single q."""
        return len(q) if isinstance(q, range) else 0

    # -- reference interface --------------------------------------------------
    def add(self, a_xG, c_axi=1.0, q=-1):
        """a_xG += sum_a,i c_axi Phi^a_i (gpaw/lfc.py:392-472)."""
        nat.require_cuda(a_xG)
        if q == -1:
            assert not a_xG.dtype.is_complex or self.gamma
        xshape = tuple(a_xG.shape[:-3])
        if isinstance(c_axi, float):
            assert q == -1 and a_xG.ndim == 3
            c_xM = torch.full((self.Mmax,), c_axi, dtype=a_xG.dtype, device=a_xG.device)
        else:
            c_xM = self._gather(c_axi, xshape, a_xG.dtype, a_xG.device)
        nx = int(np.prod(xshape, dtype=np.int64))
        if self.Mmax == 0:
            return
        nat.check(nat.lib().gb_lfc_add(
            self.lfc.handle, nat.ptr(c_xM), nat.ptr(a_xG), nx,
            nat.dtype_code(a_xG), self._nq(a_xG, q), nat.stream_of(a_xG)),
            'gb_lfc_add')

    def add_M(self, a_xG, c_xM, q=-1):
        """add() with the coefficients already concatenated over atoms,
        c_xM of shape xshape + (Mmax,) (no per-atom dict)."""
        if self.Mmax == 0:
            return
        nx = int(np.prod(tuple(a_xG.shape[:-3]), dtype=np.int64))
        c_xM = c_xM.to(a_xG.dtype).contiguous()
        nk = self._kbatch(q)
        if nk:
            assert q.start == 0 and q.step == 1
            nat.check(nat.lib().gb_lfc_add_k(
                self.lfc.handle, nat.ptr(c_xM), nat.ptr(a_xG), nx,
                nat.dtype_code(a_xG), nk, nat.stream_of(a_xG)), 'gb_lfc_add_k')
            return
        nat.check(nat.lib().gb_lfc_add(
            self.lfc.handle, nat.ptr(c_xM), nat.ptr(a_xG), nx,
            nat.dtype_code(a_xG), self._nq(a_xG, q), nat.stream_of(a_xG)),
            'gb_lfc_add')

    def integrate(self, a_xG, c_axi, q=-1):
        """c_axi = dv sum_G a_xG Phi^a_i* (gpaw/lfc.py:552-631)."""
        nat.require_cuda(a_xG)
        xshape = tuple(a_xG.shape[:-3])
        c_xM = torch.zeros(xshape + (self.Mmax,), dtype=a_xG.dtype, device=a_xG.device)
        nx = int(np.prod(xshape, dtype=np.int64))
        if self.Mmax == 0:
            return c_xM
        nk = self._kbatch(q)
        if nk:
            assert q.start == 0 and q.step == 1
            nat.check(nat.lib().gb_lfc_integrate_k(
                self.lfc.handle, nat.ptr(a_xG), nat.ptr(c_xM), nx,
                nat.dtype_code(a_xG), nk, nat.stream_of(a_xG)), 'gb_lfc_integrate_k')
        else:
            nat.check(nat.lib().gb_lfc_integrate(
                self.lfc.handle, nat.ptr(a_xG), nat.ptr(c_xM), nx,
                nat.dtype_code(a_xG), self._nq(a_xG, q), nat.stream_of(a_xG)),
                'gb_lfc_integrate')
        for a in self.my_atom_indices:
            if a in c_axi:
                M1 = self.M_a[a]
                c_axi[a][:] = c_xM[..., M1:M1 + self.sphere_a[a].Mmax]
        return c_xM

    def _derivative_arguments(self):
        """The reference's arguments of LFC.derivative for this object:
        one spline per M (each function's repeated 2l + 1 times) and the
        centre of every device volume (its atom's periodic image)."""
        if self._deriv is None:
            spline_M = []
            for sphere in self.sphere_a:
                for spline in sphere.spline_j:
                    spline_M.extend([spline] * (2 * spline.l + 1))
            spos_a = [sphere.spos_c for sphere in self.sphere_a]
            pos_Wv = np.array([np.dot(spos_a[a] - sd, self.gd.cell_cv)
                               for (a, _, _), sd in zip(self.box_W, self.sdisp_Wc)])
            self._deriv = (spline_M, np.ascontiguousarray(pos_Wv.reshape(-1, 3), float))
        return self._deriv

    def derivative(self, a_xG, c_axiv, q=-1):
        """c_axiv = dv sum_G a_xG dPhi^a_i*/dv (gpaw/lfc.py:633-724);
        d/dR = -d/dr is left to the caller exactly as in the reference.
        Computed on the device from the splines' values and slopes
        (gb_lfc_derivative); functions normalised to a given integral
        (integral=...) are refused, as their derivative needs the chain
        rule of the normalisation."""
        if self.integral_a is not None:
            raise NotImplementedError('derivative of normalized functions')
        nat.require_cuda(a_xG)
        xshape = tuple(a_xG.shape[:-3])
        c_xMv = torch.zeros(xshape + (self.Mmax, 3), dtype=a_xG.dtype, device=a_xG.device)
        nx = int(np.prod(xshape, dtype=np.int64))
        if self.Mmax == 0 or nx == 0:
            return c_xMv
        spline_M, pos_Wv = self._derivative_arguments()
        handles = (ctypes.c_void_p * len(spline_M))(*[sp.handle.value for sp in spline_M])
        gd = self.gd
        nat.check(nat.lib().gb_lfc_derivative(
            self.lfc.handle, nat.ptr(a_xG), nat.ptr(c_xMv), nx,
            nat.f64(np.ascontiguousarray(gd.h_cv)), nat.i64(gd.n_c), handles,
            nat.i64(gd.beg_c), nat.f64(pos_Wv), self._nq(a_xG, q),
            nat.dtype_code(a_xG), nat.stream_of(a_xG)), 'gb_lfc_derivative')
        for a in self.my_atom_indices:
            if a in c_axiv:
                M1 = self.M_a[a]
                c_axiv[a][:] = c_xMv[..., M1:M1 + self.sphere_a[a].Mmax, :]
        return c_xMv


LFC = LocalizedFunctionsCollection
