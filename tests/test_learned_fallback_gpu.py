"""GPU: the failure path of the learned preconditioner, with the failure
made on the host.  A network whose composite weights are broken -- a NaN
planted in them, or every weight negated -- runs inside an ordinary Si8
SCF (FP32, 32 bands, 32^3 periodic grid).  The multigrid judge must flag it
on the first judged call, Calculation.run must record the iteration
(log.fallback_at), continue with the multigrid and still converge to the
energy of a run that used the multigrid throughout."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _si8():
    from gpaw_b200.scf import Calculation, si_diamond
    s, p, c = si_diamond(1, 5.43)
    return Calculation(s, p, c, True, h=0.18, nbands=32, precision='fp32')


@pytest.fixture(scope='module')
def reference_energy():
    c = _si8()
    log = c.run(maxiter=80)
    assert log.converged
    return log.energies[-1], c.nvalence


@pytest.mark.parametrize('fault,graph', [('nan', False), ('negated', False), ('nan', True)])
def test_broken_network_falls_back_and_converges(reference_energy, fault, graph):
    from gpaw_b200.learned import ConvNet, LearnedPreconditioner
    c = _si8()
    net = ConvNet(c.gd, seed=0).init_from_multigrid(c.preconditioner)
    pc = LearnedPreconditioner(net, c.preconditioner)
    assert pc.folded is not None
    with torch.no_grad():
        if fault == 'nan':
            pc.folded.W0.view(-1)[13] = float('nan')     # the centre tap
        else:
            for w in (pc.folded.W0, pc.folded.H):
                w.neg_()
    c.use_preconditioner(pc)
    log = c.run(maxiter=80, graph=graph)
    assert log.fallback_at == 1, log.fallback_at
    assert c.preconditioner is pc.fallback
    assert log.converged and np.all(np.isfinite(log.energies))
    E, nel = reference_energy
    assert abs(log.energies[-1] - E) / nel < 3e-5
