"""GPU: the learned preconditioner's forward and backward kernels against
the FP64 oracle (oracle/learned.py) with the same BF16-rounded weights
(tolerance 1e-4 norm-wise relative: FP32 activations and accumulation),
weight gradients that repeat bit for bit, and training on (residual, multigrid correction) pairs lowers the loss."""
import numpy as np
import pytest
import torch

from oracle import fd
from oracle import learned as ol

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize('N,pbc', [((16, 16, 16), (1, 1, 1)), ((16, 12, 20), (0, 0, 0)),
                                   ((24, 16, 16), (1, 0, 1))])
def test_forward_backward_vs_oracle(N, pbc):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.learned import ConvNet
    gd = GridDescriptor(N, 0.35 * np.array(N), pbc)
    net = ConvNet(gd, seed=3)
    params64 = {k: v.to(torch.bfloat16).to(torch.float64).cpu().numpy()
                for k, v in net.params.items()}
    onet = ol.Net(fd.Grid(gd.N_c, gd.cell_cv, gd.pbc_c), params64)
    rng = np.random.default_rng(5)
    R = rng.standard_normal((3,) + tuple(gd.n_c))
    T = rng.standard_normal(R.shape)
    out = net.forward(torch.from_numpy(R).cuda(), keep=True)
    oout = onet.forward(R)
    assert rel(out.double().cpu().numpy(), oout) < 1e-4
    loss, g = net.loss_and_grad(out, torch.from_numpy(T).cuda())
    grads = net.backward(g)
    oloss, og = ol.loss_and_grad(oout, T, onet.g0)
    ograds = onet.backward(og)
    assert abs(loss - oloss) < 1e-4 * abs(oloss)
    for k in grads:
        assert rel(grads[k].double().cpu().numpy(), ograds[k]) < 1e-3, k
    # the weight gradients are reduced in a fixed order: bit-identical repeats
    again = net.backward(g)
    for k in grads:
        assert torch.equal(grads[k], again[k]), k


def test_training_reduces_loss():
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.preconditioner import Preconditioner
    from gpaw_b200.learned import ConvNet
    gd = GridDescriptor((24, 24, 24), (8.0, 8.0, 8.0), True)
    kin = Laplace(gd, -0.5, 3)
    P = Preconditioner(gd, kin, float)
    g = torch.Generator(device='cuda').manual_seed(0)
    # smooth-ish residuals: a few multigrid-preconditioned random fields
    R = torch.randn((64,) + tuple(gd.n_c), generator=g, device='cuda', dtype=torch.float64)
    M = P(R)
    net = ConvNet(gd, seed=1)
    e0 = net.relative_error(R[:16].contiguous(), M[:16]).mean()
    net.train([(R.float(), M.float())], steps=200, lr=3e-3, batch=16, log_every=0)
    e1 = net.relative_error(R[:16].contiguous(), M[:16]).mean()
    assert e1 < 0.5 * e0, (e0, e1)


def test_learned_gain_over_no_preconditioner():
    """Si8 (FP32): a network trained on the (residual, multigrid correction)
    pairs of a few ordinary iterations drives RMM-DIIS far below what the
    same iterations reach without preconditioning, and stays within the
    multigrid judge's tolerance (no fallback)."""
    from gpaw_b200.scf import Calculation, si_diamond
    from gpaw_b200.learned import ConvNet, LearnedPreconditioner, collect_pairs, train_multi

    def si8():
        s, p, c = si_diamond(1, 5.43)
        return Calculation(s, p, c, True, h=0.18, nbands=32, precision='fp32')

    R, T = collect_pairs(si8(), iterations=8, per_call=8, max_pairs=320)
    calc = si8()
    net = ConvNet(calc.gd, seed=0).init_from_multigrid(calc.preconditioner)
    e0 = net.relative_error_t(R[-16:], T[-16:]).mean().item()
    train_multi([(net, R[:-16], T[:-16])], steps=300, lr=1e-3, batch=16)
    e1 = net.relative_error_t(R[-16:], T[-16:]).mean().item()
    assert e1 < e0, (e0, e1)

    class Plain:
        """no preconditioning beyond the multigrid's diagonal scale"""

        def __init__(self, step):
            self.step = step

        def __call__(self, R, kpt=None, ekin=None, out=None):
            y = self.step * R
            if out is not None:
                out.copy_(y)
                return out
            return y

    errs = {}
    for name in ('learned', 'plain', 'multigrid'):
        c = si8()
        if name == 'learned':
            c.use_preconditioner(LearnedPreconditioner(net.on_grid(c.gd), c.preconditioner))
        elif name == 'plain':
            c.use_preconditioner(Plain(c.preconditioner.step))
        log = c.run(maxiter=12, energy_tol=0.0)
        errs[name] = log.errors[-1]
        if name == 'learned':
            assert log.fallback_at == 0, 'the multigrid judge rejected the network'
    plain = errs['plain'] if np.isfinite(errs['plain']) else np.inf
    assert errs['learned'] < 0.1 * plain, errs
    assert errs['learned'] < 100 * errs['multigrid'], errs
