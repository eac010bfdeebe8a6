"""CPU: the host side of the LFC merges the radial functions of an atom into
one device volume per (atom, periodic image).  The merged volumes, their
boundary events and the derivative volumes must describe exactly the same
function matrix Phi[G, M] (and dPhi[G, 3M]) as the per-radial-function
boxes of gpaw/lfc.py:259-374 -- checked here densely, with the native
builder replaced by a recorder (no device needed)."""
import importlib.util

import numpy as np
import pytest

from conftest import GOLDEN


def cases():
    spec = importlib.util.spec_from_file_location('lfc_cases', GOLDEN / 'lfc_cases.py')
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.LFC_CASES


class Recorder:
    """Stands in for gpaw_b200.lfc._Native and keeps its inputs."""

    def __init__(self, A_Wgm, M_W, G_B, W_B, dv, phase_qW, nG, nM):
        self.A_Wgm, self.M_W, self.G_B, self.W_B = A_Wgm, M_W, G_B, W_B
        self.phase_qW, self.nG, self.nM = phase_qW, nG, nM


def dense(rec, q=None):
    """Phi[G, M] from a recorded volume set, walking the boundary events in
    the order the device builder does (rows consumed in increasing G)."""
    Phi = np.zeros((rec.nG, rec.nM), complex)
    nxt = [0] * len(rec.A_Wgm)
    cur = []
    Ga = 0
    for Gb, W in zip(rec.G_B, rec.W_B):
        for G in range(Ga, Gb):
            for w in cur:
                A = rec.A_Wgm[w]
                ph = rec.phase_qW[q, w] if q is not None else 1.0
                Phi[G, rec.M_W[w]:rec.M_W[w] + A.shape[1]] += ph * A[nxt[w]]
                nxt[w] += 1
        if W >= 0:
            cur.append(W)
        else:
            cur.remove(-1 - W)
        Ga = Gb
    assert all(n == A.shape[0] for n, A in zip(nxt, rec.A_Wgm))
    return Phi


def dense_reference(gd, lfc, spos, q=None):
    """The same matrix from the per-radial-function boxes directly."""
    from gpaw_b200.lfc import _box_functions
    Phi = np.zeros((int(np.prod(gd.n_c)), lfc.Mmax), complex)
    for a, sphere in enumerate(lfc.sphere_a):
        M = 0
        for j, spline in enumerate(sphere.spline_j):
            nm = 2 * spline.l + 1
            for beg_c, end_c, sdisp_c in gd.get_boxes(spos[a], spline.rmax, lfc.cut):
                pos_v = np.dot(spos[a] - sdisp_c, gd.cell_cv)
                A, G_b = _box_functions(spline, beg_c, end_c, pos_v, gd)
                if len(G_b) == 0:
                    continue
                G = np.concatenate([np.arange(g0, g1) for g0, g1 in zip(G_b[0::2], G_b[1::2])])
                ph = (np.exp(2j * np.pi * np.dot(lfc.ibzk_qc[q], sdisp_c))
                      if q is not None else 1.0)
                c0 = lfc.M_a[a] + M
                Phi[G, c0:c0 + nm] += ph * A
            M += nm
    return Phi


@pytest.mark.parametrize('name', ['zero', 'periodic', 'bloch'])
def test_merged_volumes_match_per_function_boxes(name, monkeypatch):
    from gpaw_b200 import lfc as mod
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.spline import Spline
    monkeypatch.setattr(mod, '_Native', Recorder)
    N_c, cell, pbc, spos, spl, k = cases()[name]
    gd = GridDescriptor(N_c, cell, pbc, device='cpu')

    class KD:
        ibzk_qc = np.array([k], float) if k is not None else None
        gamma = False

    splines = [[Spline.from_data(l, rmax, f) for (l, rmax, f) in sj] for sj in spl]
    lfc = mod.LFC(gd, splines, kd=KD() if k is not None else None, cut=True,
                  dtype=complex if k is not None else float)
    spos = np.array(spos)
    lfc.set_positions(spos)
    q = 0 if k is not None else None
    # fewer volumes than per-function boxes whenever an atom has >1 function
    nboxes = sum(len(s.A_wgm) for s in lfc.sphere_a if s.A_wgm)
    assert len(lfc.lfc.A_Wgm) <= nboxes
    got = dense(lfc.lfc, q)
    want = dense_reference(gd, lfc, spos, q)
    assert np.abs(got - want).max() == 0.0
    # the derivative's arguments: one spline per M in M order, and each
    # merged volume centred on its atom's periodic image
    spline_M, pos_Wv = lfc._derivative_arguments()
    assert len(spline_M) == lfc.Mmax
    for a, sphere in enumerate(lfc.sphere_a):
        M = lfc.M_a[a]
        for spline in sphere.spline_j:
            for m in range(2 * spline.l + 1):
                assert spline_M[M + m] is spline
            M += 2 * spline.l + 1
    for W, ((a, _, _), sd) in enumerate(zip(lfc.box_W, lfc.sdisp_Wc)):
        assert np.allclose(pos_Wv[W], (spos[a] - sd) @ gd.cell_cv)
