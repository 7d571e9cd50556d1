"""k-point SCF sharded across ranks (chemrust-scf_b200/kpoint_scf.py): the
driver's loop against the oracle's own SCF (one Gamma member), and the same
k-point set run on two gloo ranks (CPU processes driving oracle members)
against one rank.  The ranks exchange only band energies (all-gather) and the
density (all-reduce).  Multi-GPU runs of the device members are not
measured here: every run of this build has one GPU."""
import os
import socket
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "chemrust-scf_b200"))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
import kpoint_scf  # noqa: E402
import sharding  # noqa: E402

KPTS = [(0.125, 0.125, 0.125), (-0.375, 0.125, 0.375), (0.375, -0.375, -0.125),
        (-0.125, 0.375, -0.375)]
CELL = dict(config_index=0, ecut=8.0, ngrid=[0, 0, 0], n_bands=20)


class OracleMember:
    """Test stand-in for a device member: the CPU oracle of one k-point."""

    def __init__(self, s):
        import oracle
        self.o = oracle.Oracle.from_system(s)
        self.n_bands = s.n_bands
        self._vhxc = None

    def build_v_eff(self, rho):
        vh, vx = self.o.build_veff(rho)
        self._vhxc = vh + vx
        e5 = self.o.energy(rho, rho, np.zeros(self.n_bands))
        return float(e5[2]), float(e5[3])

    def v_hxc(self):
        return self._vhxc

    def diagonalize(self, ndeg, eig=None):
        return self.o.diagonalize(ndeg, eig)

    def density(self, occ):
        self.o.set_occ(occ)
        return self.o.density()


def _systems(kpts):
    import synth
    return [synth.System(kpt=k, **CELL) for k in kpts]


def _run(systems, weights, rank, world, dist, iters):
    costs = [sharding.member_cost(s.n_pw, s.n_bands, s.ngrid) for s in systems]
    mine = kpoint_scf.KpointScf.assign(costs, rank, world)
    members = {i: OracleMember(systems[i]) for i in mine}
    s0 = systems[0]
    scf = kpoint_scf.KpointScf(members, weights, s0.n_elec, s0.omega, s0.e_ewald, s0.n_atoms,
                               dist)
    return scf.run(10, np.full(s0.ng, s0.n_elec / s0.omega), max_iter=iters, tol_per_atom=1e-14)


def test_gamma_member_matches_oracle_scf():
    import oracle
    import synth
    s = synth.System(**CELL)
    got = _run([s], [1.0], 0, 1, None, 4)
    ref = oracle.Oracle.from_system(s).run_scf(10, max_iter=4, tol_per_atom=1e-14)
    np.testing.assert_allclose(got["energies"], ref["energies"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(got["eigenvalues"][0], ref["eigenvalues"], atol=1e-9, rtol=0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import oracle
        oracle.lib().oracle_set_num_threads(2)
        r = _run(_systems(KPTS), np.full(len(KPTS), 1.0 / len(KPTS)), rank, world, dist, 4)
        q.put((rank, r["energies"].tolist(), float(r["charge"])))
    finally:
        dist.destroy_process_group()


def test_two_rank_kpoint_scf_matches_one_rank():
    import multiprocessing as mp
    systems = _systems(KPTS)
    s0 = systems[0]
    one = _run(systems, np.full(len(KPTS), 1.0 / len(KPTS)), 0, 1, None, 4)
    assert abs(one["charge"] - s0.n_elec) < 1e-8
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=600) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, energies, charge in out:
        np.testing.assert_allclose(energies, one["energies"], atol=1e-10, rtol=0)
        assert abs(charge - s0.n_elec) < 1e-8
