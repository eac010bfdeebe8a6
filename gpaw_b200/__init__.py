"""gpaw_b200: B200-native (sm_100a) real-space finite-difference Kohn-Sham
hot path with the Python API of GPAW's grid operators.

Modules mirror the reference layout: ``fd_operators``, ``transformers``,
``preconditioner``, ``lfc``, ``spline``, ``xc``, ``eigensolvers``,
``grid_descriptor``.  All compute runs in libgpawb200.so (built by
``gpaw_b200.build``); there is no CPU fallback.
"""
__version__ = '0.1.0'
