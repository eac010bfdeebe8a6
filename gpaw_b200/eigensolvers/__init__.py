"""Eigensolvers (drop-in for gpaw.eigensolvers): RMM-DIIS."""
from gpaw_b200.eigensolvers.rmmdiis import RMMDIIS


def get_eigensolver(name='rmm-diis', **kwargs):
    if isinstance(name, dict):
        kwargs = {k: v for k, v in name.items() if k != 'name'}
        name = name.get('name', 'rmm-diis')
    if name in ('rmm-diis', 'rmmdiis'):
        return RMMDIIS(**kwargs)
    raise ValueError(f'eigensolver {name!r} is not part of this build (RMM-DIIS only)')
