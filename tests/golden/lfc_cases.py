"""LFC golden-vector cases (Bohr): N_c, cell, pbc, scaled positions,
per-atom radial functions (l, rmax, f_g), k-point (None = real)."""
import numpy as np

LFC_CASES = {
    # name: (N_c, cell (Bohr), pbc, spos_ac, splines [(l, rmax, f_g)] per atom, k_c)
    'zero': ((16, 20, 20), (4.0, 5.0, 6.0), (0, 1, 1),
             [(0.25, 0.15, 0.35), (0.5, 0.5, 0.5)],
             [[(0, 2.0, [1, 0.9, 0.1, 0.0])],
              [(0, 2.0, [1, 0.9, 0.1, 0.0]), (1, 2.0, [1, 0.9, 0.1, 0.0])]], None),
    'periodic': ((20, 20, 24), (5.0, 5.0, 6.0), (1, 1, 1),
                 [(0.05, 0.1, 0.95), (0.5, 0.45, 0.5), (0.9, 0.8, 0.3)],
                 [[(0, 2.2, list(np.exp(-np.linspace(0, 2.2, 25)**2)))],
                  [(1, 2.0, list(np.exp(-np.linspace(0, 2.0, 21)**2))),
                   (2, 2.4, list(np.exp(-np.linspace(0, 2.4, 31)**2)))],
                  [(2, 1.8, list(np.exp(-np.linspace(0, 1.8, 19)**2)))]], None),
    'bloch': ((16, 16, 16), (4.5, 4.5, 4.5), (1, 1, 1),
              [(0.1, 0.9, 0.5), (0.6, 0.3, 0.2)],
              [[(0, 2.0, list(np.exp(-np.linspace(0, 2.0, 21)**2))),
                (1, 2.0, list(np.exp(-np.linspace(0, 2.0, 21)**2)))],
               [(2, 1.9, list(np.exp(-np.linspace(0, 1.9, 20)**2)))]], (0.25, -0.25, 0.5)),
}
