"""Batched passes (k-points of the 8-atom cell and independent cells of
uneven size) captured into one CUDA graph against the same passes run one
context at a time, and the launch-configuration autotuner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(chfsi):
    out = []
    for k in [(-0.375, 0.125, 0.375), (0.125, 0.125, 0.125), (0.375, -0.125, -0.375)]:
        out.append(chfsi.SyntheticSystem(config_index=0, kpt=k))
    out.append(chfsi.SyntheticSystem(config_index=0, lattice=2, n_rep=2, a_conv=6.46, seed=7,
                                     ngrid=(0, 0, 0), n_bands=0))
    out.append(chfsi.SyntheticSystem(config_index=0, lattice=1, n_rep=3, a_conv=5.13, seed=9,
                                     ngrid=(0, 0, 0), n_bands=0))
    return out


def _prepared(chfsi, s):
    ctx = chfsi.Context(s, precision=chfsi.PREC_MIXED)
    ctx.build_v_eff(np.full(ctx.ng_density, s.n_elec / s.omega))
    w = ctx.diagonalize(12)
    w = ctx.diagonalize(12, w)
    return ctx, w


def test_batched_graph_matches_sequential_passes(chfsi):
    systems = _systems(chfsi)
    assert len({s.n_pw for s in systems}) >= 4  # uneven sizes
    ref = []
    for s in systems:
        ctx, w = _prepared(chfsi, s)
        for _ in range(2):
            w = ctx.diagonalize(12, w)
        ref.append(w)
        ctx.close()
    ctxs = [_prepared(chfsi, s)[0] for s in systems]
    b = chfsi.Batch(ctxs)
    nodes = b.capture(12)
    assert nodes > 10 * len(ctxs)
    for _ in range(2):
        got = b.run()
    for g, r in zip(got, ref):
        np.testing.assert_allclose(g, r, atol=1e-8)
    print("graph of %d nodes for %d members" % (nodes, len(ctxs)))


def test_autotuner_keeps_results(chfsi):
    torch = pytest.importorskip("torch")
    s = chfsi.SyntheticSystem(config_index=1, n_bands=132)
    ctx = chfsi.Context(s)
    x = torch.from_numpy(np.ascontiguousarray(s.psi0()[:64])).cuda()
    y0 = torch.empty_like(x)
    y1 = torch.empty_like(x)
    torch.cuda.synchronize()
    ctx.apply_h_local(x.data_ptr(), y0.data_ptr(), 64)
    choice, times = ctx.autotune()
    ctx.apply_h_local(x.data_ptr(), y1.data_ptr(), 64)
    torch.cuda.synchronize()
    print("autotune choice %d, times (ms) %s" % (choice, np.round(times, 3)))
    assert 0 <= choice < 18 and (times > 0).all()
    assert times[choice] == times.min()
    a, b = y0.cpu().numpy(), y1.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
