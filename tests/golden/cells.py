"""Unit cells used by tests/golden/make_golden.py for the stencil lists
(Bohr; 12x12x12 grids).  Shared with the tests that read stencils.json."""
CELLS = {
    'sc': [1.1, 1.02, 1.03],
    'ortho': [3.0, 3.5, 4.0],
    'hexagonal': [(1, 0, 0), (0.5, 3**0.5 / 2, 0), (0, 0, 1.1)],
    'fcc': [(0, 1, 1), (1, 0, 1), (1, 1, 0)],
    'bcc': [(-1, 1, 1), (1, -1, 1), (1, 1, -1)],
    'distorted_sc': [(1, 0, 0), (0.01, 1, 0), (0, 0.02, 1)],
    'MnO': [(1, 0.5, 0.5), (0.5, 1, 0.5), (0.5, 0.5, 1)],
}
