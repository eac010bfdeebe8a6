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


@pytest.mark.parametrize('N', [(14, 14, 14), (12, 10, 16), (7, 9, 11)])
def test_conv16_periodic_matches_fp64(N):
    # 16 -> 16 convolution on a periodic grid (the level-2 layer; even rows
    # take the staged-plane kernel, odd ones the general tile kernel)
    gd = GridDescriptor(N, 0.35 * np.array(N), True)
    net = ConvNet(_grid(56), seed=6)
    g = torch.Generator(device='cuda').manual_seed(7)
    x = torch.randn((5, 16) + tuple(gd.n_c), generator=g, device='cuda', dtype=torch.float32)
    w = net.params['wb']
    y = net.conv(x, w, gd)
    wk = w.to(torch.bfloat16).double().reshape(16, 16, 3, 3, 3)
    xp = torch.nn.functional.pad(x.double(), (1, 1, 1, 1, 1, 1), mode='circular')
    ref = torch.nn.functional.conv3d(xp, wk)
    assert (y.double() - ref).abs().max().item() < 1e-5 * ref.abs().max().item()


def test_judge_flags_a_bad_network():
    # a sign-flipped network deviates from the multigrid on the probe bands:
    # the first (judged) call sets the device flag, the next two (not judged
    # with probe_every = 3) leave it as it is
    gd = _grid(32)
    mg = Preconditioner(gd, Laplace(gd, -0.5, 3), float)
    net = ConvNet(gd, seed=4).init_from_multigrid(mg)
    for k in net.params:
        net.params[k].neg_()
    lp = LearnedPreconditioner(net, mg)
    assert not bool(lp.failed)
    R = torch.randn((4, 32, 32, 32), device='cuda', dtype=torch.float32)
    lp(R)
    assert bool(lp.failed) and lp.deviation.item() > lp.tolerance
    good = LearnedPreconditioner(ConvNet(gd, seed=4).init_from_multigrid(mg), mg)
    for _ in range(3):
        good(R)
    assert not bool(good.failed)
