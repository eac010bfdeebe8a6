""".gpw restart files (row f4): the ULM container (gpaw_b200.ulm) and the
reference's .gpw layout (gpaw_b200.gpw).

The reader is checked against a file assembled byte by byte from the
published ULM layout (independently of the writer), the writer by round
trips, and read_gpw by a file in the reference's layout with its unit
conventions (density / bohr^3, wave functions x bohr^-1.5, energies in eV).
Parity with files written by ASE / GPAW themselves is not checked here
(neither is installed)."""
import json

import numpy as np
import pytest

from gpaw_b200 import ulm
from gpaw_b200.gpw import read_gpw


def handmade(path):
    """A one-item ULM file: tag 'GPAW', an int, a float, a nested child and
    a (2, 3) float64 array at an 8-byte aligned offset."""
    a = np.arange(6.0).reshape(2, 3)
    buf = bytearray(b'- of Ulm' + b'GPAW'.ljust(16) + bytes(24))
    buf += b'##'                                   # arbitrary padding, then align
    while len(buf) % 8:
        buf += b'#'
    off = len(buf)
    buf += a.astype('<f8').tobytes()
    item = {'version': 3, 'bohr': 0.5291772, 'child.': {'x': 'y', 'arr.': {'ndarray': [[2, 3], 'float64', off]}},
            'z': {'__complex__': [1.0, -2.0]}, 'small': {'__ndarray__': [[2], 'int64', [7, 8]]}}
    blob = json.dumps(item).encode()
    ipos = len(buf)
    buf += np.array([len(blob)], '<i8').tobytes() + blob
    while len(buf) % 8:
        buf += b'#'
    table = len(buf)
    buf += np.array([ipos], '<i8').tobytes()
    buf[24:48] = np.array([3, 1, table], '<i8').tobytes()
    with open(path, 'wb') as f:
        f.write(bytes(buf))
    return a


def test_reader_on_the_published_layout(tmp_path):
    p = tmp_path / 'hand.ulm'
    a = handmade(p)
    r = ulm.Reader(p)
    assert r.tag == 'GPAW' and r.format_version == 3 and r.nitems == 1
    assert r.version == 3 and r.bohr == 0.5291772
    assert r.child.x == 'y'
    assert np.array_equal(r.child.arr, a)
    assert r.z == 1 - 2j
    assert np.array_equal(r.small, [7, 8])
    assert 'child' in r and 'nothing' not in r
    r.close()


def test_not_a_ulm_file(tmp_path):
    p = tmp_path / 'x.gpw'
    p.write_bytes(b'hello world, certainly not ULM' + bytes(40))
    with pytest.raises(ulm.ULMError):
        ulm.Reader(p)


def test_writer_round_trip(tmp_path):
    p = tmp_path / 'rt.ulm'
    rng = np.random.default_rng(0)
    big = rng.standard_normal((3, 5, 7))
    cplx = rng.standard_normal((4, 2)) + 1j * rng.standard_normal((4, 2))
    w = ulm.Writer(p, 'GPAW')
    w.write(version=3, name='x', flag=True, nothing=None, c=2 + 1j, small=np.array([1, 2, 3]))
    ch = w.child('wave_functions')
    ch.write(version=2)
    ch.add_array('values', (2, 3, 5, 7), float)
    ch.fill(big)                                   # filled in pieces, as GPAW does per band
    ch.fill(2 * big)
    ch.write(cplx=cplx, ints=np.arange(5, dtype=np.int32))
    w.child('atoms').write(pbc=np.array([True, False, True]))
    w.close()
    raw = p.read_bytes()
    assert raw[:8] == b'- of Ulm' and raw[8:24] == b'GPAW'.ljust(16)
    r = ulm.Reader(p)
    assert (r.version, r.name, r.flag, r.nothing, r.c) == (3, 'x', True, None, 2 + 1j)
    assert np.array_equal(r.small, [1, 2, 3])
    v = r.wave_functions['values']
    assert v.shape == (2, 3, 5, 7) and np.array_equal(v[0], big) and np.array_equal(v[1], 2 * big)
    assert np.array_equal(r.wave_functions.cplx, cplx)
    assert r.wave_functions.ints.dtype == np.int32
    assert np.array_equal(r.atoms.pbc, [True, False, True])
    r.close()


def test_unfilled_array_is_refused(tmp_path):
    w = ulm.Writer(tmp_path / 'u.ulm', 'GPAW')
    w.add_array('a', (4,), float)
    w.fill(np.zeros(2))
    with pytest.raises(ulm.ULMError):
        w.close()


def test_read_gpw_units(tmp_path):
    """A file in the reference's layout: density in 1/Angstrom^3, values in
    1/Angstrom^1.5, eigenvalues in eV -> atomic units."""
    bohr, ha = 0.52917721067, 27.211386024367243
    p = tmp_path / 'state.gpw'
    rng = np.random.default_rng(1)
    nt = rng.random((1, 4, 6, 8))
    psit = rng.standard_normal((1, 1, 3, 4, 6, 8))
    w = ulm.Writer(p, 'GPAW')
    w.write(version=3, ha=ha, bohr=bohr)
    w.child('atoms').write(positions=np.array([[0.5, 0.6, 0.7]]), numbers=np.array([14]),
                           cell=np.diag([2.0, 3.0, 4.0]), pbc=np.array([True] * 3))
    w.child('density').write(density=nt / bohr**3, atomic_density_matrices=np.zeros((1, 0)))
    wf = w.child('wave_functions')
    wf.write(version=2, ha=ha, eigenvalues=np.array([[[-1.0, 0.0, 2.0]]]) * ha)
    wf.add_array('values', psit.shape, float)
    wf.fill(psit * bohr**-1.5)
    w.close()
    s = read_gpw(p)
    assert np.allclose(s.density, nt, rtol=1e-14)
    assert np.allclose(s.psit, psit, rtol=1e-14)
    assert np.allclose(s.eigenvalues, [[[-1.0, 0.0, 2.0]]])
    assert s.numbers.tolist() == [14] and s.pbc.all() and s.cell.shape == (3, 3)
