"""Benchmark: FD stencil throughput on the kernel-microbench workload.

Workload ("step"): one application of the order-6 (nn=3, 19-point) kinetic
Laplacian  -1/2 nabla^2  to a batch of 256 grids of 96x96x96 float64 points
(h = 0.2 A, periodic), values from a seeded N(0, 1) -- the
(256, 96, 96, 96) kernel-microbench configuration.  Metric: algorithmic
bytes moved per second, 2 * 256 * 96^3 * 8 B per step (one read + one write
of the array; halos and coefficients excluded).  Inputs (3.6 GB) are larger
than the 126 MB L2, so no flush is needed between steps.

Also reported on the same JSON line:
  suite        the other microbench kernels (FP32, zero boundaries, Gradient,
               restriction / interpolation k=2, 6, the V-cycle), GB/s each
  roofline     the stencil kernel against the measured HBM copy bandwidth
  e2e          the same metric through the public API with host buffers
               (pinned H2D copy + apply + D2H copy inside the timed region)
  cpu_baseline GPAW's own C Operator (built from the reference sources into
               oracle/_ref) on the host cores, the full 256-grid step

`--impl reference` times GPAW's own C implementation of the same step on the
host cores (all threads) and prints the same metric with "impl": "reference".
Multi-GPU (`--gpus N` under torchrun): independent replicas (the path has no
exchange step on one grid per band batch), value = total bytes / max time.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

BOHR = 0.52917721
NB, N = 256, 96
H_ANG = 0.2
METRIC = 'FD stencil GB/s: order-6 Laplacian on (256,96,96,96)'


def peaks():
    p = REPO / 'MEASURED_PEAKS.json'
    if p.exists():
        d = json.loads(p.read_text())
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


# DRAM bytes per 96^3 FP64 grid of one stencil launch
# (dram__bytes_read.sum + dram__bytes_write.sum of an ncu capture of a 64-grid
# launch of the same kernel, divided by 64; the capture is summarised in
# profiles/star_tma_kernel_f64_laplace_96cubed.txt)
STENCIL_TRAFFIC_PER_GRID = 16.35e6


def profiled_traffic(nb):
    """DRAM bytes per launch of the stencil kernel: the per-grid traffic of
    the ncu capture times the grids per launch (traffic grows in proportion
    to the grids per launch)."""
    return round(STENCIL_TRAFFIC_PER_GRID * nb)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')

    def __init__(self, device_index):
        self.lines = []
        self.proc = None
        self.dev = device_index

    def start(self):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            ident = uuid if uuid.startswith('GPU-') else 'GPU-' + uuid
        except Exception:
            ident = str(self.dev)
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', ident, f'--query-gpu={self.FIELDS}',
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        for line in self.lines:
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, v in zip(names, parts[4:8]):
                if v.lower() == 'active':
                    reasons.add(name)
        return {'sm_mhz': float(np.median(sm)) if sm else None,
                'sm_max_mhz': smax, 'reasons': sorted(reasons),
                'samples': len(sm)}


def grid(pbc, n=N):
    from gpaw_b200.grid_descriptor import GridDescriptor
    N_c = np.array([n, n, n]) + (0 if pbc else 1)
    return GridDescriptor(N_c, N_c * H_ANG / BOHR, pbc)


def time_launches(fn, reps, stream):
    """Average device time of `fn` (one launch chain) with CUDA events on the
    launching stream."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(reps)]
    for a, b in ev:
        a.record(stream)
        fn()
        b.record(stream)
    torch.cuda.synchronize()
    return float(np.mean([a.elapsed_time(b) for a, b in ev]))


SUITE_PARTS = ('grid', 'lfc', 'xc', 'vcycle')


def suite(torch, stream, nb=None, parts=SUITE_PARTS):
    """GB/s of the other kernel-microbench kernels (algorithmic bytes); nb
    grids per call (default: the benchmark's 256); parts: any of 'grid'
    (stencils and transfers), 'lfc', 'xc', 'vcycle'."""
    NB = nb or globals()['NB']
    from gpaw_b200.fd_operators import Laplace, Gradient
    from gpaw_b200.transformers import Transformer
    from gpaw_b200.preconditioner import Preconditioner
    out = {}
    g = torch.Generator(device='cuda').manual_seed(1)
    for dtype, dname in ((torch.float64, 'f64'), (torch.float32, 'f32')) if 'grid' in parts else ():
        for pbc in (True, False):
            gd = grid(pbc)
            x = torch.randn((NB,) + tuple(gd.n_c), generator=g, device='cuda', dtype=dtype)
            y = torch.empty_like(x)
            nbytes = 2 * x.numel() * x.element_size()
            bc = 'periodic' if pbc else 'zero'
            lap = Laplace(gd, -0.5, 3)
            lap.apply(x, y)
            t = time_launches(lambda: lap.apply(x, y), 5, stream)
            out[f'laplace_nn3_{dname}_{bc}'] = round(nbytes / t / 1e6, 1)
            grad = Gradient(gd, 0, 1.0, 3)
            grad.apply(x, y)
            t = time_launches(lambda: grad.apply(x, y), 5, stream)
            out[f'gradient_nn3_{dname}_{bc}'] = round(nbytes / t / 1e6, 1)
            if dtype == torch.float64:
                # restrict / interpolate: zero boundaries use n = 95 -> 47
                gdf = grid(pbc) if pbc else grid(False, N - 1)
                gdc = gdf.coarsen()
                xf = x if pbc else torch.randn((NB,) + tuple(gdf.n_c), generator=g,
                                               device='cuda', dtype=dtype)
                xc = torch.empty((NB,) + tuple(gdc.n_c), device='cuda', dtype=dtype)
                yf = torch.empty_like(xf)
                rbytes = (xf.numel() + xc.numel()) * 8
                for nn in (1, 3):
                    r = Transformer(gdf, gdc, nn)
                    r.apply(xf, xc)
                    t = time_launches(lambda: r.apply(xf, xc), 5, stream)
                    out[f'restrict_k{2 * nn}_{dname}_{bc}'] = round(rbytes / t / 1e6, 1)
                    it = Transformer(gdc, gdf, nn)
                    it.apply(xc, yf)
                    t = time_launches(lambda: it.apply(xc, yf), 5, stream)
                    out[f'interpolate_k{2 * nn}_{dname}_{bc}'] = round(rbytes / t / 1e6, 1)
                del xf, xc, yf
            del x, y
    if 'lfc' in parts:
        suite_lfc(torch, stream, NB, g, out)
    if 'xc' in parts:
        suite_xc(torch, stream, g, out)
    if 'vcycle' in parts:
        suite_vcycle(torch, stream, g, out)
    return out


def suite_lfc(torch, stream, NB, g, out):
    # LFC add / integrate: 64 atom-centred Gaussians x (l = 0, 1, 2) with
    # cutoff 2.5 A on the 96^3 grid (h = 0.2 A), 256 bands, FP64
    from gpaw_b200.lfc import LFC
    from gpaw_b200.spline import Spline
    rc = 2.5 / BOHR
    rr = np.linspace(0, rc, 101)
    f = np.exp(-(rr / (0.8 / BOHR))**2)
    gdl = grid(True)
    lfc = LFC(gdl, [[Spline.from_data(l, rc, f) for l in (0, 1, 2)]] * 64)
    lfc.set_positions(np.random.default_rng(0).random((64, 3)))
    a = torch.randn((NB,) + tuple(gdl.n_c), generator=g, device='cuda', dtype=torch.float64)
    cM = torch.randn((NB, lfc.Mmax), generator=g, device='cuda', dtype=torch.float64)
    c_axi = {i: cM[:, 9 * i:9 * i + 9].contiguous() for i in range(64)}
    # grid points covered by at least one sphere (the union over atoms)
    cover = np.zeros(int(np.prod(gdl.n_c)), bool)
    for sp in lfc.sphere_a:
        for G_b in sp.G_wb:
            for g0, g1 in zip(G_b[0::2], G_b[1::2]):
                cover[g0:g1] = True
    npts = int(cover.sum())
    lfc.add(a, c_axi)
    t = time_launches(lambda: lfc.add(a, c_axi), 5, stream)
    # algorithmic bytes: read + write every covered point of every band
    out['lfc_add_f64_64atoms_256bands_ms'] = round(t, 3)
    out['lfc_add_f64_GBps'] = round(NB * 2 * npts * 8 / t / 1e6, 1)
    lfc.integrate(a, {})
    t = time_launches(lambda: lfc.integrate(a, {}), 5, stream)
    out['lfc_integrate_f64_64atoms_256bands_ms'] = round(t, 3)
    out['lfc_integrate_f64_GBps'] = round(NB * npts * 8 / t / 1e6, 1)
    out['lfc_covered_points'] = npts


def suite_xc(torch, stream, g, out):
    # XC on the fine grid of the H2O-cluster config (151^3), FP64
    from gpaw_b200.xc import XCKernel
    ng = 151**3
    n_g = torch.rand((1, ng), generator=g, device='cuda', dtype=torch.float64) + 1e-3
    sig = torch.rand((1, ng), generator=g, device='cuda', dtype=torch.float64)
    e_g = torch.empty(ng, dtype=torch.float64, device='cuda')
    v_g = torch.zeros_like(n_g)
    d_g = torch.empty_like(sig)
    for name, arrays in (('LDA', 4), ('PBE', 6)):
        k = XCKernel(name)
        call = (lambda: k.calculate(e_g, n_g, v_g)) if name == 'LDA' else (
            lambda: k.calculate(e_g, n_g, v_g, sig, d_g))
        call()
        t = time_launches(call, 5, stream)
        out[f'xc_{name}_151cubed_GBps'] = round(arrays * ng * 8 / t / 1e6, 1)


def suite_vcycle(torch, stream, g, out):
    # V-cycle on 160 bands of the Si64 grid (56^3, periodic), FP64
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.preconditioner import Preconditioner
    gd = GridDescriptor((56, 56, 56), (20.52, 20.52, 20.52), True)
    kin = Laplace(gd, -0.5, 3)
    P = Preconditioner(gd, kin, float, block=10)
    R = torch.randn((160, 56, 56, 56), generator=g, device='cuda', dtype=torch.float64)
    d = torch.empty_like(R)
    P(R, out=d)
    t = time_launches(lambda: P(R, out=d), 5, stream)
    out['precond_vcycle_f64_56cubed_160bands_ms'] = round(t, 3)
    out['precond_vcycle_f64_min_bytes_GBps'] = round(2 * R.numel() * 8 / t / 1e6, 1)


def scf_benchmark(train_steps=400):
    """The SCF time-to-solution comparison on the 64-atom Si cell (2x2x2
    conventional diamond cells, a = 10.86 A, seeded displacements of sigma
    0.05 A, h = 0.2 A -> 56^3 grid, 160 bands, LDA, Gamma): the plain FP64
    multigrid form (the reference's RMM-DIIS blocks of 10 bands, eager
    launches) against the batched FP32 form with the learned preconditioner
    (all bands per launch, the step replayed as CUDA graphs), with the
    intermediate forms beside them.  Every run starts from the same seeded
    initial guess in a process that has just run a short warm-up SCF of the
    same form (its graph memory pool then holds blocks of the right shapes),
    so one-time CUDA / library initialisation is excluded from all of them;
    each timed run still captures its own graphs.  Times are
    host wall-clock to the first iteration after which the total energy
    stays within 1e-5 eV per valence electron of the converged value.
    Training data: (residual, multigrid correction) pairs recorded during 6
    ordinary FP32 iterations of the same cell; the network is initialised
    from the V-cycle and trained with the project's own BF16/FP32 kernels."""
    import torch
    from gpaw_b200.scf import Calculation, si_diamond
    from gpaw_b200.learned import (ConvNet, LearnedPreconditioner, collect_pairs,
                                   train_multi)

    def si64(prec, blocksize=None):
        sym, pos, cell = si_diamond(2, 5.43, rattle=0.05, seed=0)
        return Calculation(sym, pos, cell, True, h=0.2, nbands=160, xc='LDA',
                           precision=prec, blocksize=blocksize)

    def time_to(log, nel, tol=1e-5):
        E = np.array(log.energies)
        for i in range(len(E)):
            if np.all(np.abs(E[i:] - E[-1]) / nel < tol):
                return i + 1, log.times[i]
        return None, None

    # warm-up on the timed shapes: a short SCF of every timed form (precision,
    # band blocks, eager or graphed), so one-time costs -- first launches,
    # the stencil autotuner's timing of each layout, the first allocation of
    # a graph's memory pool -- are paid here by every form alike
    for prec, graph, block in (('fp64', False, 10), ('fp32', True, None),
                               ('fp64', True, None), ('fp64', False, None)):
        w = si64(prec, block)
        w.run(maxiter=8, energy_tol=0.0, graph=graph)
        del w
        # a calculation holds reference cycles: collect it now, so that its
        # device buffers (and the graph pool's blocks) are free for the next
        gc.collect()
    t0 = time.perf_counter()
    c = si64('fp32')
    R, T = collect_pairs(c, iterations=6, per_call=8, max_pairs=400)
    net = ConvNet(c.gd, seed=0).init_from_multigrid(c.preconditioner)
    err0 = float(net.relative_error_t(R[-32:], T[-32:]).mean())
    t1 = time.perf_counter()
    train_multi([(net, R[:-32], T[:-32])], steps=train_steps, lr=1e-3, batch=16)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    err1 = float(net.relative_error_t(R[-32:], T[-32:]).mean())
    t_prep = time.perf_counter() - t0
    del c
    gc.collect()
    out = {'workload': 'Si64 diamond (2x2x2 cells, a=10.86 A, sigma=0.05 A), h=0.2 A '
                       '(56^3), 160 bands, LDA, Gamma; SCF to 1e-5 eV/electron',
           'training': {'pairs': int(len(R)), 'steps': train_steps,
                        'train_s': round(t_train, 2), 'collect_and_train_s': round(t_prep, 2),
                        'heldout_energy_norm_relerr_init': round(err0, 4),
                        'heldout_energy_norm_relerr_trained': round(err1, 4)}}
    # plain: the reference's default RMM-DIIS blocks of 10 bands, eager;
    # batched: every band in every launch, the step replayed as CUDA graphs
    runs = [('fp64_multigrid_plain', 'fp64', False, False, 10),
            ('fp32_learned_batched', 'fp32', True, True, None),
            ('fp32_multigrid_batched', 'fp32', True, False, None),
            ('fp64_multigrid_batched', 'fp64', True, False, None),
            ('fp64_multigrid_batched_eager', 'fp64', False, False, None)]
    ref = None
    for name, prec, graph, learned, block in runs:
        # a short untimed SCF of this very form first (the learned one could
        # not be warmed up above: its network is trained only now), so the
        # timed run's graph capture finds the pool blocks of its own shapes,
        # as in a process that has run such a calculation before; the
        # capture itself stays inside the timed run
        for timed in (False, True):
            c = si64(prec, block)
            if learned:
                c.use_preconditioner(LearnedPreconditioner(net.on_grid(c.gd), c.preconditioner))
            if timed:
                break
            c.run(maxiter=8, energy_tol=0.0, graph=graph)
            del c
            gc.collect()
        log = c.run(maxiter=150, graph=graph)
        it, t = time_to(log, c.nvalence)
        eps = c.eigenvalues()[:c.nvalence // 2]
        r = {'converged': log.converged, 'iterations': log.iterations,
             'iterations_to_1e-5': it, 'seconds_to_1e-5': round(t, 4) if t else None,
             'seconds_total': round(log.wall, 4), 'energy_eV': round(log.energies[-1], 6),
             # wall time per iteration: the first (start-up), the median and
             # the slowest (for a graphed form, the one that captures)
             'iteration_ms': dict(zip(('first', 'median', 'max'), (
                 round(float(x), 2) for x in (lambda d: (d[0], np.median(d), d.max()))(
                     1e3 * np.diff(np.r_[0.0, log.times]))))),
             'learned_fallback_at_iteration': log.fallback_at or None}
        if ref is None:
            ref = (log.energies[-1], eps, c.nvalence)
        else:
            r['energy_error_eV_per_electron'] = float(abs(log.energies[-1] - ref[0]) / ref[2])
            r['max_occupied_eigenvalue_error_eV'] = float(np.abs(eps - ref[1]).max())
        out[name] = r
        del c
        gc.collect()
    a = out['fp64_multigrid_plain']
    for name in ('fp32_learned_batched', 'fp32_multigrid_batched', 'fp64_multigrid_batched'):
        b = out[name]
        if a['seconds_to_1e-5'] and b['seconds_to_1e-5']:
            out[f'speedup_{name}_vs_fp64_multigrid_plain'] = round(
                a['seconds_to_1e-5'] / b['seconds_to_1e-5'], 3)
        # the online criterion: each run's own convergence test (energy
        # change over the last three iterations below 1e-5 eV / electron)
        if a['converged'] and b['converged']:
            out[f'speedup_online_{name}_vs_fp64_multigrid_plain'] = round(
                a['seconds_total'] / b['seconds_total'], 3)
    out['cpu_baseline'] = scf_cpu_baseline(si64, a['iterations'])
    return out


def scf_cpu_baseline(make_calc, iterations, sample_iterations=1):
    """The same SCF on the host cores: the oracle SCF (GPAW's own C
    kernels -- stencils, transfers, multigrid, LFC, XC, density -- with the
    reference's RMM-DIIS, subspace and orthonormalisation steps in numpy,
    FP64, OpenMP over every core) from the plain form's start.  A bounded
    sample: the potential set-up plus `sample_iterations` iterations are
    timed, and the time to solution is that per-iteration time times the
    iterations the plain FP64 form took (the oracle runs the same algorithm
    and, in the parity tests, the same number of iterations)."""
    from oracle import ref
    if not ref.available():
        return None
    from oracle import scf as osf
    c = make_calc('fp64', 10)
    o = osf.from_calculation(c, xc='LDA', blocksize=10)
    del c
    gc.collect()
    t0 = time.perf_counter()
    o.update_hamiltonian()
    t1 = time.perf_counter()
    for _ in range(sample_iterations):
        o.iteration()
    t2 = time.perf_counter()
    per_it = (t2 - t1) / sample_iterations
    return {'value': round((t1 - t0) + per_it * iterations, 2), 'unit': 's',
            'cores': int(os.environ.get('OMP_NUM_THREADS', os.cpu_count() or 1)),
            'kind': 'port',
            'seconds_per_iteration': round(per_it, 3),
            'sample': f'potential set-up + {sample_iterations} SCF iteration(s) of the '
                      'Si64 FP64 SCF with GPAW\'s C kernels (oracle/_ref) and the '
                      'reference\'s RMM-DIIS in numpy (10-band blocks), scaled to the '
                      f'{iterations} iterations of the plain FP64 form'}


def precision_benchmark():
    """The precision configuration: 32 H2O molecules (O-H 0.96 A, 104.5 deg,
    seeded orientations, 4 x 4 x 2 lattice of 3.1 A plus 0.1 A jitter) in a
    15 A box with zero boundaries, h = 0.2 A (76^3), 160 bands (128
    occupied), PBE, Pulay mixing 0.1.  The FP64 run and the FP32 run from
    the same start, both converged to 1e-6 in the density (forces are not
    variational); the FP32 errors in total energy (eV per valence
    electron), occupied eigenvalues (eV) and forces (eV / A) against FP64."""
    import torch
    from gpaw_b200.scf import Calculation, h2o_cluster
    sym, pos, cell = h2o_cluster()
    runs = {}
    for prec, tol in (('fp64', 1e-7), ('fp32', 1e-6)):
        c = Calculation(sym, pos, cell, False, h=0.2, nbands=160, xc='PBE',
                        precision=prec, mixer_beta=0.1)
        log = c.run(maxiter=300, energy_tol=tol, density_tol=1e-6, graph=True)
        runs[prec] = dict(converged=log.converged, iterations=log.iterations,
                          seconds=round(log.wall, 3), energy_eV=log.energies[-1],
                          eps=c.eigenvalues()[:128], F=c.forces(), nel=c.nvalence)
        del c
        gc.collect()
        torch.cuda.empty_cache()
    a, b = runs['fp64'], runs['fp32']
    return {'workload': '(H2O)32, 15 A box, zero boundaries, h=0.2 A (76^3), 160 bands, '
                        'PBE, FP32 vs FP64 from the same start',
            'fp64': {k: a[k] for k in ('converged', 'iterations', 'seconds', 'energy_eV')},
            'fp32': {k: b[k] for k in ('converged', 'iterations', 'seconds', 'energy_eV')},
            'energy_error_eV_per_electron': float(abs(a['energy_eV'] - b['energy_eV']) / a['nel']),
            'max_occupied_eigenvalue_error_eV': float(np.abs(a['eps'] - b['eps']).max()),
            'max_force_error_eV_per_A': float(np.abs(a['F'] - b['F']).max()),
            'max_force_eV_per_A': float(np.abs(a['F']).max())}


def lfc_benchmark(args):
    """The projector LFC of the Si64 SCF on its production shape: 64 Si
    atoms (2 s + 2 p radial functions merged into 8 functions per atom), the
    56^3 periodic grid, 160 FP32 bands.  CUDA events around `steps` calls of
    the add (a += sum_a p^a c^a, the nonlocal term of the residuals) and of
    the integrate (the projections <p^a|psi>) after `warmup` untimed ones.
    Algorithmic bytes: the add reads and writes, the integrate reads, every
    covered point of every band once."""
    import torch
    from gpaw_b200.scf import Calculation, si_diamond
    sym, pos, cell = si_diamond(2, 5.43, rattle=0.05, seed=0)
    c = Calculation(sym, pos, cell, True, h=0.2, nbands=160, xc='LDA', precision='fp32')
    pt = c.wfs.pt
    n_c = tuple(c.gd.n_c)
    g = torch.Generator(device='cuda').manual_seed(0)
    a = torch.randn((160,) + n_c, generator=g, device='cuda', dtype=torch.float32)
    b = torch.randn((160,) + n_c, generator=g, device='cuda', dtype=torch.float32)
    cM = torch.randn((160, pt.Mmax), generator=g, device='cuda', dtype=torch.float32)

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps * 1e3
    t_add = timed(lambda: pt.add_M(b, cM))
    t_int = timed(lambda: pt.integrate(a, {}))
    print(json.dumps({'workload': 'Si64 projector LFC, 160 x 56^3 FP32 bands, 64 atoms x 8 functions',
                      'add_us': round(t_add, 1), 'integrate_us': round(t_int, 1)}))


def iteration_profile(args):
    """Kernel-by-kernel device time of one Si64 SCF iteration in the two FP32
    forms (learned and multigrid preconditioner), graph-replayed: the Si64
    FP32 calculation of scf_benchmark, the network initialised from the
    V-cycle (its cost does not depend on the weights), iterations 13-17 of
    a run timed with the torch profiler's CUDA kernel records (graph kernels
    included).  Prints one JSON object: per form the device time per
    iteration, the median wall time per iteration and the 40 costliest
    kernels (microseconds and launches per iteration)."""
    import numpy as np
    import torch
    from torch.profiler import profile, ProfilerActivity
    from gpaw_b200.scf import Calculation, si_diamond
    from gpaw_b200.learned import ConvNet, LearnedPreconditioner
    k0, k = 12, 5
    out = {'workload': 'Si64 (56^3, 160 FP32 bands, LDA, Gamma), one graph-replayed SCF '
                       f'iteration, mean of iterations {k0 + 1}-{k0 + k}'}
    for learned in (True, False):
        sym, pos, cell = si_diamond(2, 5.43, rattle=0.05, seed=0)
        c = Calculation(sym, pos, cell, True, h=0.2, nbands=160, xc='LDA', precision='fp32')
        if learned:
            net = ConvNet(c.gd, seed=0).init_from_multigrid(c.preconditioner)
            c.use_preconditioner(LearnedPreconditioner(net, c.preconditioner))
        prof = profile(activities=[ProfilerActivity.CUDA])

        def window(calc, it, log):
            if it == k0:
                torch.cuda.synchronize()
                prof.start()
            if it == k0 + k:
                torch.cuda.synchronize()
                prof.stop()
        log = c.run(maxiter=k0 + k, energy_tol=0.0, callback=window, graph=True)
        rows = []
        for e in prof.key_averages():
            t = getattr(e, 'self_device_time_total', None)
            if t is None:
                t = e.self_cuda_time_total
            if t > 0:
                rows.append((t / k, e.count / k, e.key))
        rows.sort(reverse=True)
        wall = np.diff(np.r_[0.0, log.times])[k0:]
        out['learned' if learned else 'multigrid'] = {
            'device_us_per_iteration': round(sum(r[0] for r in rows), 1),
            'wall_ms_median': round(float(np.median(wall)) * 1e3, 2),
            'fallback_at': log.fallback_at,
            'kernels': [(round(t, 1), round(n, 2), name) for t, n, name in rows[:40]]}
        del c, prof
        gc.collect()
    print(json.dumps(out))


def network_benchmark(args):
    """The learned preconditioner's forward pass on its production shape:
    160 FP32 residuals of the 56^3 periodic Si64 grid (h = 0.194 A), the
    network initialised from the V-cycle; CUDA events around `steps` passes
    after `warmup` untimed ones: the layer-by-layer form (the one training
    differentiates), the folded inference form (FoldedNet, what the SCF
    runs on periodic grids) and the fused V-cycle on the same data."""
    import torch
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.preconditioner import Preconditioner
    from gpaw_b200.learned import ConvNet, FoldedNet
    cell = 10.86 / BOHR
    gd = GridDescriptor((56, 56, 56), (cell, cell, cell), True)
    mg = Preconditioner(gd, Laplace(gd, -0.5, 3), float)
    net = ConvNet(gd).init_from_multigrid(mg)
    g = torch.Generator(device='cuda').manual_seed(0)
    R = torch.randn((160, 56, 56, 56), generator=g, device='cuda', dtype=torch.float32)

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps
    folded = FoldedNet(net, scale=mg.step)
    out = {'workload': 'learned preconditioner forward, 160 x 56^3 FP32 residuals',
           'network_ms': round(timed(lambda: net.forward(R, scale=mg.step)), 4),
           'network_folded_ms': round(timed(lambda: folded.forward(R)), 4),
           'vcycle_ms': round(timed(lambda: mg(R)), 4)}
    print(json.dumps(out))


def band_gemm_benchmark(args):
    """The eigensolver's band-space GEMMs on their Si64 shape, 160 FP32 bands
    of 56^3 = 175,616 points: the Gram matrix dv psi^T (H psi) (tensor cores,
    three-product TF32 split, FP64-combined partial sums; plus the FP64 dots
    that make its diagonal exact) and the rotation psi <- U psi (identity
    split), each next to the GEMM it replaces (FP64 GEMM of widened operands;
    FP32 SIMT GEMM).  CUDA events around `steps` calls after `warmup`.
    Algorithmic FLOPs: 2 n^2 N per product (8.99 GFLOP); bytes: the operands
    read once and the output written once."""
    import torch
    from gpaw_b200.bandops import gram_tc, rotate_tc, tf32_split
    nb, N = 160, 56 ** 3
    g = torch.Generator(device='cuda').manual_seed(0)
    A = torch.randn((nb, N), generator=g, device='cuda', dtype=torch.float32)
    B = torch.randn((nb, N), generator=g, device='cuda', dtype=torch.float32)
    U = torch.linalg.qr(torch.eye(nb, dtype=torch.float64, device='cuda') +
                        0.05 * torch.randn((nb, nb), generator=g, dtype=torch.float64,
                                           device='cuda'))[0]
    Y = torch.empty_like(A)
    split = tf32_split(U - torch.eye(nb, dtype=torch.float64, device='cuda'))

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return 1e3 * e0.elapsed_time(e1) / args.steps
    flop = 2.0 * nb * nb * N
    t_gram = timed(lambda: gram_tc(A, B))
    t_gram_d = timed(lambda: gram_tc(A, B, exact_diagonal=True))
    t_ovl = timed(lambda: gram_tc(A, A, exact_diagonal=True))
    t_rot = timed(lambda: rotate_tc((split[0], split[1], nb), A, out=Y, identity_split=True))
    Uf = U.to(torch.float32)
    out = {'workload': 'band-space GEMMs, 160 FP32 bands x 56^3 points (Si64)',
           'gram_tc_us': round(t_gram, 1),
           'gram_tc_exact_diagonal_us': round(t_gram_d, 1),
           'overlap_tc_exact_diagonal_us': round(t_ovl, 1),
           'gram_fp64_widened_us': round(timed(lambda: A.double() @ B.double().T), 1),
           'gram_tc_TFLOPs_per_product': round(flop / t_gram / 1e6, 1),
           'rotate_tc_identity_split_us': round(t_rot, 1),
           'rotate_fp32_simt_gemm_us': round(timed(lambda: Uf @ A), 1),
           'rotate_tc_GBps': round(3 * nb * N * 4 / t_rot / 1e3, 1)}
    print(json.dumps(out))


def cpu_reference_run(nb, steps, warmup):
    """GPAW's own C Operator (oracle/_ref, OpenMP over the host cores) on the
    benchmark step: the order-6 Laplacian of `nb` periodic 96^3 FP64 grids,
    seeded N(0, 1).  `warmup` untimed applications, then the mean over
    `steps` timed ones (time.perf_counter).  Both the reference arm and the
    cpu_baseline of this arm use this one method.  Returns (GB/s, seconds
    per step) or None where the reference build is absent."""
    from oracle import ref, fd
    if not ref.available():
        return None
    gd = grid(True)
    coefs, offs = fd.guc_laplace(gd.h_cv, -0.5, 3)
    op = ref.operator(coefs, offs, gd.n_c, (1, 1, 1), True)
    a = np.random.default_rng(0).standard_normal((nb,) + tuple(gd.n_c))
    b = np.zeros_like(a)
    for _ in range(max(warmup, 1)):
        op.apply(a, b)
    t0 = time.perf_counter()
    for _ in range(steps):
        op.apply(a, b)
    t = (time.perf_counter() - t0) / steps
    return 2 * a.nbytes / t / 1e9, t


def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    threads = int(os.environ.get('OMP_NUM_THREADS', os.cpu_count() or 1))
    r = cpu_reference_run(NB, args.steps, args.warmup)
    if r is None:
        print(json.dumps({'impl': 'reference', 'unavailable':
                          'oracle/_ref (GPAW C extension from the reference '
                          'sources) was not built'}))
        return
    value, t = r
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': round(value, 2),
        'unit': 'GB/s', 'n_gpus': args.gpus, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': round(t * 1e3, 3),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64', 'data': 'synthetic N(0,1), seed 0',
        'config': {'workload': f'laplace_nn3_f64_periodic_{NB}x96^3',
                   'sample': f'the full {NB}-grid step, mean of {args.steps} '
                             f'after {max(args.warmup, 1)} warm-up'},
        'cpu_baseline': {'value': round(value, 2), 'unit': 'GB/s',
                         'cores': threads, 'kind': 'reference',
                         'sample': f'{NB} grids of 96^3 per step, mean of '
                                   f'{args.steps} steps'},
        'e2e': {'value': round(value, 2), 'unit': 'GB/s',
                'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-suite', action='store_true')
    ap.add_argument('--no-scf', action='store_true',
                    help='skip the Si64 SCF time-to-solution comparison')
    ap.add_argument('--stencil-path', type=int, default=0,
                    help='0 auto (TMA where possible), 1 cp.async kernel, 2 TMA only')
    ap.add_argument('--bands', type=int, default=NB,
                    help='grids per step (256 is the benchmark workload; smaller '
                         'values give the small case that ncu captures)')
    ap.add_argument('--kernel-only', action='store_true',
                    help='time the stencil step only (no e2e, suite or CPU '
                         'baseline): the command line used for ncu captures')
    ap.add_argument('--network-only', action='store_true',
                    help='time the learned preconditioner network alone: one '
                         'forward pass over 160 FP32 residuals of the 56^3 Si64 '
                         'grid per step (the command line used for ncu captures)')
    ap.add_argument('--iteration-profile', action='store_true',
                    help='kernel-by-kernel device time of one graph-replayed Si64 '
                         'FP32 SCF iteration, learned and multigrid forms (torch '
                         'profiler; the command behind the iteration summary)')
    ap.add_argument('--lfc-only', action='store_true',
                    help='time the projector LFC add and integrate alone on the '
                         'Si64 shape (64 atoms x 8 functions, 160 FP32 bands of '
                         '56^3; the command line used for ncu captures)')
    ap.add_argument('--band-gemm-only', action='store_true',
                    help='time the tensor-core band-space GEMMs alone on the Si64 '
                         'shapes (160 FP32 bands x 56^3 points): Gram matrix and '
                         'subspace rotation, next to the FP64 / SIMT GEMMs they '
                         'replace (the command line used for ncu captures)')
    ap.add_argument('--suite-only', action='store_true',
                    help='run the kernel suite alone with --bands grids per call '
                         '(the command line used for ncu captures of its kernels)')
    ap.add_argument('--suite-part', action='append', choices=SUITE_PARTS,
                    help='with --suite-only: only these parts (repeatable)')
    ap.add_argument('--dtype', default='f64', choices=['f64', 'f32'],
                    help='storage precision of the kernel-only run (the '
                         'benchmark line itself is FP64)')
    args = ap.parse_args()
    if args.dtype != 'f64' and not args.kernel_only:
        ap.error('--dtype f32 is for --kernel-only runs; the benchmark line is FP64')
    # GPAW's C operator (the reference arm and the cpu_baseline) runs OpenMP
    # over every host core; set before the extension is loaded
    os.environ.setdefault('OMP_NUM_THREADS', str(os.cpu_count() or 1))
    if args.impl == 'reference':
        run_reference(args)
        return
    if args.network_only:
        network_benchmark(args)
        return
    if args.iteration_profile:
        iteration_profile(args)
        return
    if args.lfc_only:
        lfc_benchmark(args)
        return
    if args.band_gemm_only:
        band_gemm_benchmark(args)
        return
    if args.suite_only:
        import torch
        parts = tuple(args.suite_part or SUITE_PARTS)
        print(json.dumps({'suite_GBps': suite(torch, torch.cuda.current_stream(), args.bands, parts),
                          'bands': args.bands}))
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group('nccl', timeout=timedelta(seconds=120),
                                device_id=torch.device('cuda', local))
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200 import _native as nat
    nat.check(nat.lib().gb_set_stencil_path(args.stencil_path), 'stencil path')
    stream = torch.cuda.current_stream()
    gd = grid(True)
    lap = Laplace(gd, -0.5, 3)
    g = torch.Generator(device='cuda').manual_seed(0)
    nb = args.bands
    tdt = torch.float64 if args.dtype == 'f64' else torch.float32
    cname = 'double' if args.dtype == 'f64' else 'float'
    x = torch.randn((nb, N, N, N), generator=g, device='cuda', dtype=tdt)
    y = torch.empty_like(x)
    nbytes = 2 * x.numel() * x.element_size()
    # which stencil kernel serves this layout: try the TMA pipeline alone
    nat.check(nat.lib().gb_set_stencil_path(2), 'stencil path')
    try:
        lap.apply(x[:1], y[:1])
        kernel = (f'star_tma_kernel<{cname},H=3,R1=2,R2=2>' if args.dtype == 'f64'
                  else f'star_tma_kernel<{cname},H=3,R1=2,R2=4>')
    except nat.GPAWB200Error:
        kernel = f'star_kernel<{cname},H=3>'
    nat.check(nat.lib().gb_set_stencil_path(args.stencil_path), 'stencil path')
    if args.stencil_path == 1:
        kernel = f'star_kernel<{cname},H=3>'

    for _ in range(max(args.warmup, 3)):
        lap.apply(x, y)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for a, b in ev:
        a.record(stream)
        lap.apply(x, y)
        b.record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    launch_ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    if world > 1:
        t = torch.tensor([total_ms], device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = t.item()
    value = world * nbytes * args.steps / (total_ms / 1e3) / 1e9

    if args.kernel_only:
        if rank == 0:
            print(json.dumps({'metric': METRIC, 'value': round(value, 1), 'unit': 'GB/s',
                              'bands': nb, 'dtype': args.dtype, 'kernel': kernel,
                              'ms_per_step': round(total_ms / args.steps, 4),
                              'launch_ms': round(launch_ms, 4), 'clocks': clk}))
        if world > 1:
            dist.destroy_process_group()
        return

    # e2e through the public API with host buffers (pinned), fewer steps
    e2e_steps = min(args.steps, 3)
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    xd = torch.empty_like(x)
    yd = torch.empty_like(x)
    xd.copy_(xh, non_blocking=True)
    lap.apply(xd, yd)
    yh.copy_(yd, non_blocking=True)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        xd.copy_(xh, non_blocking=True)
        lap.apply(xd, yd)
        yh.copy_(yd, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    del xd, yd
    if world > 1:
        t = torch.tensor([e2e_ms], device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = t.item()
    e2e_value = world * nbytes / (e2e_ms / 1e3) / 1e9

    scf_res = None
    prec_res = None
    if not args.no_scf and rank == 0:
        scf_res = scf_benchmark()
        prec_res = precision_benchmark()
    suite_res = None
    if not args.no_suite:
        del x, y
        torch.cuda.empty_cache()
        suite_res = suite(torch, stream)

    cpu = None
    if rank == 0 and world == 1:
        threads = int(os.environ.get('OMP_NUM_THREADS', os.cpu_count() or 1))
        r = cpu_reference_run(NB, 3, 1)
        if r is not None:
            cpu = {'value': round(r[0], 2), 'unit': 'GB/s', 'cores': threads,
                   'kind': 'reference',
                   'sample': f'the full {NB}-grid step of 96^3 FP64 periodic grids, '
                             'mean of 3 after 1 warm-up (GPAW C Operator from the '
                             f'reference sources, OpenMP {threads} threads)'}

    peak, peak_kind = peaks()
    achieved = nbytes / (launch_ms / 1e3) / 1e9
    traffic = profiled_traffic(nb)
    line = {
        'metric': METRIC, 'value': round(value, 1), 'unit': 'GB/s',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': round(total_ms / args.steps, 4),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64', 'data': 'synthetic N(0,1), seeded (torch.Generator seed 0)',
        'config': {'workload': f'laplace_nn3_f64_periodic_{nb}x96^3',
                   'grid': [nb, N, N, N], 'h_angstrom': H_ANG,
                   'stencil': '19-point order-6 kinetic Laplacian',
                   'l2': 'inputs 1.8 GB > L2, no flush',
                   'parallelism': f'replicas x{world}'},
        'clocks': clk,
        'e2e': {'value': round(e2e_value, 2), 'unit': 'GB/s',
                'h2d_bytes_per_step': nb * N**3 * 8,
                'd2h_bytes_per_step': nb * N**3 * 8,
                'steps': e2e_steps},
        'gpu_launches': args.steps,
        'roofline': {'bound': 'hbm', 'achieved': round(achieved, 1),
                     'peak': peak, 'unit': 'GB/s', 'frac': round(achieved / peak, 4),
                     'peak_kind': peak_kind,
                     'traffic': traffic,
                     'kernel': kernel},
        'cpu_baseline': cpu,
        'suite_GBps': suite_res,
        'scf': scf_res,
        'precision': prec_res,
    }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
