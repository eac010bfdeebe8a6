"""The per-iteration JSON Lines log of Calculation.run(logfile=...): one
object per iteration with the convergence quantities (CPU: the writer on a
filled log; GPU: an H2 run whose lines match its SCFLog)."""
import json

import pytest

from gpaw_b200.scf import SCFLog, _append_log_line


def test_log_line_fields(tmp_path):
    log = SCFLog(energies=[-31.5], errors=[2e-3], ddens=[0.1], times=[0.25], fallback_at=0)
    p = tmp_path / 'scf.jsonl'
    _append_log_line(p, 1, log, False)
    log.energies.append(-31.6)
    log.errors.append(1e-4)
    log.ddens.append(0.01)
    log.times.append(0.5)
    log.fallback_at = 2
    _append_log_line(p, 2, log, True)
    lines = [json.loads(x) for x in p.read_text().splitlines()]
    assert lines[0] == {'iteration': 1, 'energy_eV': -31.5, 'eigenstate_error': 2e-3,
                        'density_change': 0.1, 'time_s': 0.25, 'graphed': False, 'fallback_at': None}
    assert lines[1]['graphed'] and lines[1]['fallback_at'] == 2 and lines[1]['energy_eV'] == -31.6


@pytest.mark.gpu
def test_run_writes_one_line_per_iteration(tmp_path):
    from gpaw_b200.scf import Calculation, h2
    sym, pos, cell = h2()
    c = Calculation(sym, pos, cell, False, h=0.2, nbands=4, xc='LDA')
    p = tmp_path / 'h2.jsonl'
    log = c.run(maxiter=40, logfile=p)
    lines = [json.loads(x) for x in p.read_text().splitlines()]
    assert len(lines) == log.iterations
    assert [x['energy_eV'] for x in lines] == log.energies
    assert [x['iteration'] for x in lines] == list(range(1, log.iterations + 1))
