""".gpw restart files: read a ground state (wave functions and density) for
a warm start, and write one in the same layout.

The layout is the reference's (Calculator._write, gpaw/calculator.py:
309-325; Density.write, gpaw/density.py:632-634; the FD wave functions,
gpaw/wavefunctions/fd.py:221-237 and gpaw/wavefunctions/base.py:461-510)
in the ULM container (gpaw_b200.ulm):

  top level        version (3), gpaw_version, ha (eV), bohr (Angstrom)
  atoms.           positions (Angstrom), numbers, cell (Angstrom), pbc
  density.         density (nspins, n0, n1, n2), pseudo density in 1/Angstrom^3
                   on the coarse grid; atomic_density_matrices
  wave_functions.  version (2), ha, fermi_levels, projections
                   (nspins, nk, nbands, nproj), eigenvalues (nspins, nk,
                   nbands) in eV, occupations (divided by the k-point
                   weight x 2 / nspins), values (nspins, nk, nbands, n0, n1,
                   n2) in 1/Angstrom^1.5 when written with mode='all'

Grids are the global arrays without the boundary point of zero-boundary
axes (GridDescriptor n_c), as the reference's gd.collect gives them."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .ulm import Reader, Writer

ATOMIC_NUMBERS = {'H': 1, 'He': 2, 'Li': 3, 'Be': 4, 'B': 5, 'C': 6, 'N': 7, 'O': 8, 'F': 9,
                  'Ne': 10, 'Na': 11, 'Mg': 12, 'Al': 13, 'Si': 14, 'P': 15, 'S': 16, 'Cl': 17}


@dataclass
class GPWState:
    positions: np.ndarray          # (natoms, 3) Angstrom
    numbers: np.ndarray            # (natoms,)
    cell: np.ndarray               # (3, 3) Angstrom
    pbc: np.ndarray                # (3,)
    density: np.ndarray            # (nspins, n0, n1, n2) electrons / bohr^3
    eigenvalues: np.ndarray | None     # (nspins, nk, nbands) Hartree
    psit: np.ndarray | None        # (nspins, nk, nbands, n0, n1, n2) bohr^-1.5


def read_gpw(path) -> GPWState:
    """The ground state of a .gpw file in atomic units (the reference's
    Density.read / FDWaveFunctions.read conversions: density x bohr^3,
    wave functions x bohr^1.5, energies / ha)."""
    r = Reader(path)
    try:
        bohr, ha = float(r.bohr), float(r.ha)
        a = r.atoms
        d = r.density
        dens = np.asarray(d.density, float) * bohr**3
        if dens.ndim == 3:
            dens = dens[None]
        wf = r.wave_functions if 'wave_functions' in r else None
        eps = psit = None
        if wf is not None:
            if 'eigenvalues' in wf:
                eps = np.asarray(wf.eigenvalues, float) / ha
            name = 'values' if 'values' in wf else ('coefficients' if 'coefficients' in wf else None)
            if name is not None:
                psit = np.asarray(wf[name]) * bohr**1.5
        return GPWState(np.asarray(a.positions, float), np.asarray(a.numbers, int),
                        np.asarray(a.cell, float).reshape(3, 3), np.asarray(a.pbc, bool),
                        dens, eps, psit)
    finally:
        r.close()


def write_gpw(calc, path, mode: str = 'all') -> None:
    """Write calc's state in the reference's layout; mode='all' includes the
    wave functions (as Calculator.write(..., mode='all'))."""
    from .scf import Bohr, Hartree
    w = Writer(path, 'GPAW')
    w.write(version=3, gpaw_version='gpaw_b200', ha=Hartree, bohr=Bohr)
    cell = calc.cell_cv * Bohr
    w.child('atoms').write(positions=calc.spos_ac @ cell,
                           numbers=np.array([ATOMIC_NUMBERS[s] for s in calc.symbols]),
                           cell=cell, pbc=np.asarray(calc.pbc, bool))
    log = getattr(calc, 'log', None)
    w.child('results').write(energy=float(log.energies[-1]) if log is not None and log.energies
                             else None)
    w.child('parameters').write(mode='fd', xc=getattr(calc.xc, 'name', None), nbands=int(calc.nbands))
    nt = calc.nt_G.detach().double().cpu().numpy()
    w.child('density').write(density=(nt / Bohr**3)[None],
                             atomic_density_matrices=np.zeros((1, 0)))
    wf = w.child('wave_functions')
    nk, nb = len(calc.ibz_kc), calc.nbands
    eps = np.asarray(calc.eigenvalues()).reshape(1, nk, nb) * Hartree
    occ = np.zeros((1, nk, nb))
    nocc = calc.nvalence // 2
    occ[..., :nocc] = 1.0
    wf.write(version=2, ha=Hartree, fermi_levels=np.array([np.nan]), eigenvalues=eps, occupations=occ)
    nproj = int(calc.wfs.pt.Mmax)
    proj_dtype = complex if calc.dtype.is_complex else float
    wf.add_array('projections', (1, nk, nb, nproj), proj_dtype)
    for kpt in calc.wfs.kpt_u:
        P = kpt.P_nM
        P = (np.zeros((getattr(kpt, 'nk', 1) * nb, nproj), proj_dtype) if P is None
             else P.detach().cpu().numpy().astype(proj_dtype))
        wf.fill(P)
    if mode == 'all':
        n_c = tuple(int(x) for x in calc.gd.n_c)
        wf.add_array('values', (1, nk, nb) + n_c, proj_dtype)
        for kpt in calc.wfs.kpt_u:
            psit = kpt.psit_nG.detach().cpu().numpy().astype(proj_dtype)
            wf.fill(psit * Bohr**-1.5)
    w.close()


def warm_start(calc, state: GPWState) -> None:
    """Start calc from a stored ground state of the same system and grid:
    the density and the first bands of every k-point (the rest keep their
    initial guess), orthonormalised; the mixer history is reset."""
    import torch
    n_c = tuple(int(x) for x in calc.gd.n_c)
    if state.density.shape[1:] != n_c:
        raise ValueError(f'grid {state.density.shape[1:]} in the file, {n_c} here')
    cell = calc.cell_cv * _bohr()
    if len(state.positions) != len(calc.symbols) or not np.allclose(state.cell, cell, atol=1e-6):
        raise ValueError('the file holds a different system')
    spos = np.linalg.solve(cell.T, state.positions.T).T
    d = spos - calc.spos_ac
    d[:, calc.pbc] -= np.round(d[:, calc.pbc])
    if np.abs(d).max() > 1e-6:
        raise ValueError('the file holds a different geometry')
    dev = calc.gd.device
    calc.nt_G.copy_(torch.from_numpy(state.density[0]).to(dev, calc.nt_G.dtype))
    calc.mixer.reset()
    if state.psit is not None:
        nk = len(calc.ibz_kc)
        if state.psit.shape[1] != nk:
            raise ValueError(f'{state.psit.shape[1]} k-points in the file, {nk} here')
        nb = min(state.psit.shape[2], calc.nbands)
        for kpt in calc.wfs.kpt_u:
            ks = range(nk) if getattr(kpt, 'nk', 1) > 1 else [_k_index(calc, kpt)]
            for i, k in enumerate(ks):
                rows = slice(i * calc.nbands, i * calc.nbands + nb)
                kpt.psit_nG[rows] = torch.from_numpy(state.psit[0, k, :nb]).to(dev, kpt.psit_nG.dtype)
            calc.wfs.orthonormalize(kpt)
    calc.update_hamiltonian()


def _bohr():
    from .scf import Bohr
    return Bohr


def _k_index(calc, kpt):
    k_c = getattr(kpt, 'k_c', None)
    if k_c is None:
        return 0
    d = np.abs(np.asarray(calc.ibz_kc) - np.asarray(k_c)[None]).sum(1)
    return int(np.argmin(d))
