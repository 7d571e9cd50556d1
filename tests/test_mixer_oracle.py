"""CPU checks of the learned-mixer oracle (oracle/mixer_oracle.py): BF16
rounding, the analytic gradient against central finite differences, and the
least-squares targets on residuals built to have a known per-shell answer."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mixer_oracle as mo  # noqa: E402


def test_bf16_round_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    w = np.concatenate([rng.standard_normal(4096).astype(np.float32) * 10.0 ** rng.integers(-6, 6, 4096),
                        np.float32([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -0.0, 65504.0])])
    ref = torch.from_numpy(w).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(mo.bf16_round(w), ref)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    p = (rng.standard_normal(mo.N_PARAMS) * 0.05).astype(np.float32)
    x = rng.standard_normal((4, mo.N_IN)).astype(np.float32)
    t = rng.standard_normal((4, mo.SHELLS, mo.N_T))
    t[:, :, 2] = np.abs(t[:, :, 2]); t[:, :, 4] = np.abs(t[:, :, 4]) + 1.0
    t[:, :, 3] = 0.1 * t[:, :, 3]
    _, g = mo.loss_grad(p, x, t, quantize=False)
    idx = np.concatenate([rng.integers(lo, hi, 6) for lo, hi in
                          [(mo.OFF_W1, mo.OFF_B1), (mo.OFF_B1, mo.OFF_W2), (mo.OFF_W2, mo.OFF_B2),
                           (mo.OFF_B2, mo.OFF_W3), (mo.OFF_W3, mo.OFF_B3), (mo.OFF_B3, mo.N_PARAMS)]])
    pd = p.astype(np.float64)
    for i in idx:
        h = 1e-4
        q1 = pd.copy(); q1[i] += h
        q2 = pd.copy(); q2[i] -= h
        # float64 parameters: evaluate without the float32 cast of unpack
        f1 = _loss64(q1, x, t)
        f2 = _loss64(q2, x, t)
        fd = (f1 - f2) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def _loss64(p, x, t):
    W1 = p[mo.OFF_W1:mo.OFF_B1].reshape(mo.N_HID, mo.N_IN)
    W2 = p[mo.OFF_W2:mo.OFF_B2].reshape(mo.N_HID, mo.N_HID)
    W3 = p[mo.OFF_W3:mo.OFF_B3].reshape(mo.N_OUT, mo.N_HID)
    b1, b2, b3 = p[mo.OFF_B1:mo.OFF_W2], p[mo.OFF_B2:mo.OFF_W3], p[mo.OFF_B3:]
    xx = x.astype(np.float64)
    y = mo.gelu(mo.gelu(xx @ W1.T + b1) @ W2.T + b2) @ W3.T + b3
    B = y.shape[0]
    y = y.reshape(B, mo.SHELLS, 2)
    ea, eb = y[:, :, 0] - t[:, :, 0], y[:, :, 1] - t[:, :, 1]
    return np.sum(ea * ea * t[:, :, 2] + 2 * ea * eb * t[:, :, 3] + eb * eb * t[:, :, 4]) / B


def test_targets_recover_known_per_shell_update():
    """E = a_s R0 + b_s D exactly in every shell -> targets (a_s, b_s)."""
    rng = np.random.default_rng(3)
    ngrid = (12, 12, 12)
    recip = 2 * np.pi / 6.0 * np.eye(3)
    shell = mo.shell_index(ngrid, recip)
    n = shell.size
    r0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    d = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    a = rng.uniform(-1, 1, mo.SHELLS)
    b = rng.uniform(-1, 1, mo.SHELLS)
    s = np.where(shell == 255, 0, shell)
    e = a[s] * r0 + b[s] * d
    e[shell == 255] = 0
    x, t = mo.features_targets(mo.shell_sums(shell, [r0], d, e))
    t = t.reshape(mo.SHELLS, mo.N_T)
    used = np.bincount(shell[shell != 255], minlength=mo.SHELLS)[:mo.SHELLS] > 1
    assert used.sum() > 5
    np.testing.assert_allclose(t[used, 0], a[used], atol=1e-6)
    np.testing.assert_allclose(t[used, 1], b[used], atol=1e-6)
    # the loss of the update (0, 0) is |E|^2 / |E|^2 = 1 (E is fully explained)
    ea, eb = -t[:, 0], -t[:, 1]
    l0 = np.sum(ea * ea * t[:, 2] + 2 * ea * eb * t[:, 3] + eb * eb * t[:, 4])
    assert abs(l0 - 1.0) < 1e-7
    assert x.shape == (mo.N_IN,)


def test_shell_index_g0_and_symmetry():
    ngrid = (10, 12, 8)
    recip = np.diag([2 * np.pi / 5.0, 2 * np.pi / 6.0, 2 * np.pi / 4.0])
    s = mo.shell_index(ngrid, recip).reshape(8, 12, 10)
    assert s[0, 0, 0] == 255
    assert (s[1:, 1:, 1:] == s[1:, 1:, 1:][::-1, ::-1, ::-1]).all()  # |G| = |-G|


def test_training_cells_reproducible_and_dilute_cells_reach_large_edges():
    # cell_params without dilute cells keeps the seeds' historical draws (the
    # shipped weights were trained on them); dilute cells are 64-atom cells
    # whose edge reaches the 216-atom cell's 30.78 bohr
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "chemrust-scf_b200"))
    import learned_mixer as lm
    a = [(p.lattice, p.n_rep, round(p.a_conv, 6), p.z_val)
         for p in (lm.cell_params(sd) for sd in range(10_000, 10_040))]
    b = [(p.lattice, p.n_rep, round(p.a_conv, 6), p.z_val)
         for p in (lm.cell_params(sd, dilute_frac=0.0) for sd in range(10_000, 10_040))]
    assert a == b
    edges = []
    for sd in range(20_000, 20_200):
        p = lm.cell_params(sd, dilute_frac=0.3)
        edge = p.a_conv * p.n_rep
        if edge > 21.0:  # larger than the densest 64-atom cell (20.52 bohr)
            assert (p.lattice, p.n_rep) == lm.CELL_KINDS[lm.DILUTE_KIND][:2]
            edges.append(edge)
    assert 30 <= len(edges) <= 90
    assert max(edges) <= 30.78 + 1e-6 and min(edges) >= 20.52 * 1.5 ** (1 / 3) - 1e-6
