"""Band-parallel Rayleigh-Ritz (chemrust-scf_b200/band_parallel.py): each rank
filters its band block, then all-to-all to a plane-wave split, partial
subspace matrices, one all-reduce, the small eigenproblem on every rank, the
rotation of the local plane waves and the all-to-all back
(PROJECT_ROOT_PLAN.md:213-234); for the ultrasoft overlap the partial
projections beta_r^H psi_r are summed in the same all-reduce.  Two gloo ranks on CPU, the filter and the
small eigenproblem from the oracle, against the oracle's one-process
ChFSI iteration.  Multi-GPU runs are not measured here (one GPU per run)."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "chemrust-scf_b200"))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
import band_parallel as bp  # noqa: E402

NDEG = 10


class NumpyOps:
    """Steps 2, 4, 5 on the host for the CPU test (oracle eigensolver)."""

    def gemm_cn(self, a, b):
        import torch
        return torch.from_numpy(np.conj(a.numpy()) @ b.numpy().T)

    def rotate(self, v, x):
        import torch
        return torch.from_numpy(v.numpy().T @ x.numpy())

    def hegv(self, h, s):
        import oracle
        import torch
        w, v = oracle.hegv(h.numpy(), s.numpy())
        return w, torch.from_numpy(v)


def _system(uspp):
    import synth
    if uspp:
        return synth.System(config_index=2, n_rep=1, ecut=8.0, ngrid=[0, 0, 0], n_bands=24)
    return synth.System(config_index=0, n_shell=1, lmax=1, rc_proj=[1.2, 0, 0, 0], d_min=0.5,
                        d_max=2.0, n_bands=21)


def _start(oracle, uspp=False):
    s = _system(uspp)
    o = oracle.Oracle.from_system(s)
    if uspp:
        o.set_qmat(s.qmat())
    o.set_veff(o.vloc_r())
    w1 = o.diagonalize(NDEG)
    return s, o, w1


def _block_pass(oracle, s, psi1, w1, b0, b1, uspp=False):
    """Filter of one band block (the rank's share) from the Ritz vectors psi1."""
    import torch
    ob = oracle.Oracle(s.ngrid, s.miller(), s.kinetic(), s.beta(), s.proj_offsets(), s.dmat(),
                       psi1[b0:b1], s.occupations()[b0:b1], s.vloc_g(), s.omega, s.gmax,
                       s.e_ewald, s.n_atoms)
    if uspp:
        ob.set_qmat(s.qmat())
    ob.set_veff(ob.vloc_r())
    st, _ = ob.chebyshev_filter(NDEG, np.array([w1.min(), w1.max()]))
    assert st == 0
    return torch.from_numpy(ob.get_psi()), torch.from_numpy(ob.get_hpsi())


def _uspp_args(s, rank, world):
    """This rank's plane-wave slice of the projectors and the dense q."""
    import torch
    pws = bp.offsets(bp.split_counts(s.n_pw, world))
    beta = np.asarray(s.beta()).reshape(-1, s.n_pw)
    return (torch.from_numpy(np.ascontiguousarray(beta[:, pws[rank]:pws[rank + 1]])),
            torch.from_numpy(bp.qmat_dense(s.qmat(), s.proj_offsets())))


def test_single_rank_bandsplit_equals_oracle_iteration():
    import oracle
    s, o, w1 = _start(oracle)
    psi1 = o.get_psi()
    p, hp = _block_pass(oracle, s, psi1, w1, 0, s.n_bands)
    new, w = bp.rayleigh_ritz_bandsplit(p, hp, s.n_bands, s.n_pw, 0, 1, None, NumpyOps())
    w_ref = o.diagonalize(NDEG, w1)
    np.testing.assert_allclose(w, w_ref, atol=1e-10, rtol=0)


def _free_port():
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    p = sk.getsockname()[1]
    sk.close()
    return p


def _worker(rank, world, port, q, uspp=False):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import oracle
        oracle.lib().oracle_set_num_threads(2)
        s, o, w1 = _start(oracle, uspp)
        counts = bp.split_counts(s.n_bands, world)
        b0 = bp.offsets(counts)
        p, hp = _block_pass(oracle, s, o.get_psi(), w1, int(b0[rank]), int(b0[rank + 1]), uspp)
        kw = {}
        if uspp:
            kw["beta_pw"], kw["qmat"] = _uspp_args(s, rank, world)
        new, w = bp.rayleigh_ritz_bandsplit(p, hp, s.n_bands, s.n_pw, rank, world, dist,
                                            NumpyOps(), **kw)
        q.put((rank, w.tolist(), new.numpy()))
    finally:
        dist.destroy_process_group()


def test_single_rank_bandsplit_uspp_equals_oracle_iteration():
    # the generalised problem: S_sub = psi^H psi + C^H q C with C summed first
    import oracle
    s, o, w1 = _start(oracle, uspp=True)
    p, hp = _block_pass(oracle, s, o.get_psi(), w1, 0, s.n_bands, uspp=True)
    beta_pw, qd = _uspp_args(s, 0, 1)
    new, w = bp.rayleigh_ritz_bandsplit(p, hp, s.n_bands, s.n_pw, 0, 1, None, NumpyOps(),
                                        beta_pw=beta_pw, qmat=qd)
    w_ref = o.diagonalize(NDEG, w1)
    np.testing.assert_allclose(w, w_ref, atol=1e-10, rtol=0)


@pytest.mark.parametrize("uspp", [False, True])
def test_two_rank_bandsplit_matches_one_process(uspp):
    import multiprocessing as mp
    import oracle
    s, o, w1 = _start(oracle, uspp)
    w_ref = o.diagonalize(NDEG, w1)
    psi_ref = o.get_psi()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q, uspp)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted([q.get(timeout=600) for _ in ps], key=lambda t: t[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, w, _ in out:
        np.testing.assert_allclose(w, w_ref, atol=1e-10, rtol=0)
    psi = np.concatenate([blk for _, _, blk in out], axis=0)
    assert psi.shape == psi_ref.shape
    # the same Ritz vectors up to a phase per band, S-orthonormal
    sp = o.apply_s(psi) if uspp else psi
    ov = np.abs(np.sum(np.conj(sp) * psi_ref, axis=1))
    np.testing.assert_allclose(ov, 1.0, atol=1e-9)
    np.testing.assert_allclose(np.conj(psi) @ sp.T, np.eye(s.n_bands), atol=1e-10)


def test_qmat_dense_layout():
    # per-ion blocks in chfsi_set_qmat order -> block-diagonal matrix
    off = np.array([0, 2, 5])
    blocks = np.concatenate([np.arange(4) + 1j, np.arange(9) * 2.0 + 0j])
    q = bp.qmat_dense(blocks, off)
    assert q.shape == (5, 5)
    np.testing.assert_array_equal(q[:2, :2], (np.arange(4) + 1j).reshape(2, 2))
    np.testing.assert_array_equal(q[2:, 2:], (np.arange(9) * 2.0).reshape(3, 3))
    assert not q[:2, 2:].any() and not q[2:, :2].any()
