"""Folded inference form of the learned preconditioner (FoldedNet:
gb_learned_fold_stride / gb_learned_fold_fine) against the layer-by-layer
network it is derived from: the same linear map on periodic grids, up to
FP32 rounding (relative 2e-5 of the output's largest value)."""
import numpy as np
import pytest
import torch

from gpaw_b200.grid_descriptor import GridDescriptor
from gpaw_b200.learned import ConvNet, FoldedNet, LearnedPreconditioner
from gpaw_b200.fd_operators import Laplace
from gpaw_b200.preconditioner import Preconditioner

pytestmark = pytest.mark.gpu

BOHR = 0.52917721


def _grid(N, pbc=True):
    return GridDescriptor((N, N, N), np.array([N, N, N]) * 0.2 / BOHR, pbc)


@pytest.mark.parametrize('N,seed,init', [(56, 0, 'mg'), (32, 1, 'random'), (24, 2, 'random'),
                                         (40, 3, 'mg')])
def test_folded_matches_layered(N, seed, init):
    gd = _grid(N)
    mg = Preconditioner(gd, Laplace(gd, -0.5, 3), float)
    net = ConvNet(gd, seed=seed)
    if init == 'mg':
        net.init_from_multigrid(mg)
    g = torch.Generator(device='cuda').manual_seed(seed + 10)
    R = torch.randn((5, N, N, N), generator=g, device='cuda', dtype=torch.float32)
    ref = net.forward(R, scale=mg.step)
    out = FoldedNet(net, scale=mg.step).forward(R)
    err = (out - ref).abs().max().item() / ref.abs().max().item()
    assert err < 2e-5, err


def test_preconditioner_takes_folded_form_on_periodic_grids():
    gd = _grid(32)
    mg = Preconditioner(gd, Laplace(gd, -0.5, 3), float)
    net = ConvNet(gd, seed=4).init_from_multigrid(mg)
    lp = LearnedPreconditioner(net, mg)
    assert lp.folded is not None
    R = torch.randn((3, 32, 32, 32), device='cuda', dtype=torch.float32)
    y = lp(R)
    ref = net.forward(R, scale=mg.step)
    assert (y - ref).abs().max().item() < 2e-5 * ref.abs().max().item()
    # zero boundaries: the layer-by-layer form (folding assumes wrap-around)
    gdz = _grid(32, pbc=False)
    mgz = Preconditioner(gdz, Laplace(gdz, -0.5, 3), float)
    lpz = LearnedPreconditioner(ConvNet(gdz, seed=4).init_from_multigrid(mgz), mgz)
    assert lpz.folded is None
