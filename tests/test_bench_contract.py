"""CPU: the benchmark's reference arm (GPAW's own C stencil built from the
reference sources, timed on the host cores) prints one JSON line with the
keys the benchmark contract asks for -- or, where that extension has not
been built, its one-line `unavailable` reason."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, 'bench.py', '--impl', 'reference', '--steps', '1',
                        '--warmup', '1'], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith('{')]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d['impl'] == 'reference'
    if 'unavailable' in d:
        assert isinstance(d['unavailable'], str) and d['unavailable']
        return
    assert d['metric'].startswith('FD stencil GB/s')
    assert d['unit'] == 'GB/s' and d['value'] > 0 and d['higher_is_better'] is True
    assert d['config']['workload'] == 'laplace_nn3_f64_periodic_256x96^3'
    assert d['steps'] == 1 and d['warmup'] == 1 and d['n_gpus'] == 1
    cb = d['cpu_baseline']
    assert cb['kind'] == 'reference' and cb['cores'] >= 1 and cb['value'] == d['value'] and cb['sample']
    assert d['e2e']['h2d_bytes_per_step'] == 0 and d['e2e']['d2h_bytes_per_step'] == 0
    assert d['e2e']['value'] == d['value'] and d['e2e']['unit'] == d['unit']
