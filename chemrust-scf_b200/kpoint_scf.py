"""SCF of one cell over a set of k-points, the k-points sharded across ranks
(one process per GPU, torch.distributed; NCCL on GPUs, gloo on CPU).

The loop is run_scf (src/scf.rs:358-376) with the Brillouin-zone sums the
reference's single-k loop leaves out: the k-points share V_eff and nothing
else during a diagonalisation, so each rank diagonalises its own members
(LPT-balanced by sharding.partition) with no data-path collective, and an
iteration has exactly two exchanges:

* the band energies of every member (an all-gather of a few hundred
  doubles), from which every rank computes the same Fermi level and
  occupations f_nk (sum_k w_k sum_n f_nk = N_e);
* the density, sum_k w_k sum_n f_nk |psi_nk(r)|^2 / Omega, one all-reduce
  of the density grid.

Energies, the convergence test (|dE| per atom) and Pulay mixing (alpha,
history; mixing.rs:24-27 as planned) then run identically on every rank.

A member is any object with
    build_v_eff(rho) -> (E_H, E_xc) of rho, and V_eff = V_loc + V_H + V_xc[rho]
    v_hxc() -> V_H + V_xc of the last density given (density grid)
    diagonalize(ndeg, eig) -> eigenvalues (ChFSI pass: filter + Rayleigh-Ritz)
    density(occ) -> sum_n occ_n |psi_n(r)|^2 / Omega (density grid)
`DeviceMember` wraps a chfsi.Context (the CUDA library; no CPU path).
"""
import numpy as np

import sharding


class DeviceMember:
    """One k-point of the cell on this rank's GPU (a chfsi.Context)."""

    def __init__(self, ctx):
        if tuple(ctx.ngrid) != tuple(ctx.ngrid_density):
            raise ValueError("k-point SCF needs the density grid equal to the wavefunction grid")
        self.ctx = ctx
        self.n_bands = ctx.n_bands
        self._vloc = ctx.get_vloc()

    def build_v_eff(self, rho):
        e2 = self.ctx.build_v_eff(rho)
        return float(e2[0]), float(e2[1])

    def v_hxc(self):
        return self.ctx.get_veff() - self._vloc

    def diagonalize(self, ndeg, eig=None):
        return self.ctx.diagonalize(ndeg, eig)

    def density(self, occ):
        self.ctx.set_occupations(occ)
        return self.ctx.construct_density()


def fermi_weighted(eigs, weights, n_elec, kT):
    """Occupations f_nk in [0, 2] with sum_k w_k sum_n f_nk = n_elec
    (Fermi-Dirac, bisection on mu) and the entropy term -kT S.
    eigs: list of per-k eigenvalue arrays."""
    allv = np.concatenate(eigs)
    lo, hi = allv.min() - 40.0 * kT - 1.0, allv.max() + 40.0 * kT + 1.0

    def occ(mu):
        return [2.0 / (1.0 + np.exp(np.clip((e - mu) / kT, -700.0, 700.0))) for e in eigs]

    def count(mu):
        return sum(w * f.sum() for w, f in zip(weights, occ(mu)))

    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if count(mid) < n_elec:
            lo = mid
        else:
            hi = mid
    mu = 0.5 * (lo + hi)
    f = occ(mu)
    ts = 0.0
    for w, fk in zip(weights, f):
        ft = 0.5 * fk
        m = (ft > 1e-300) & (ft < 1.0 - 1e-16)
        ts += w * np.sum(-2.0 * (ft[m] * np.log(ft[m]) + (1.0 - ft[m]) * np.log(1.0 - ft[m])))
    return f, -kT * ts, mu


class Pulay:
    """Pulay / DIIS over (rho_in, rho_out - rho_in) with scalar alpha."""

    def __init__(self, alpha=0.3, history=6):
        self.alpha, self.history = alpha, history
        self.rin, self.res = [], []

    def mix(self, rho_in, rho_out):
        self.rin.append(rho_in.copy())
        self.res.append(rho_out - rho_in)
        self.rin, self.res = self.rin[-self.history:], self.res[-self.history:]
        m = len(self.res)
        A = np.zeros((m + 1, m + 1))
        for i in range(m):
            for j in range(m):
                A[i, j] = self.res[i] @ self.res[j]
        A[:m, m] = A[m, :m] = 1.0
        rhs = np.zeros(m + 1)
        rhs[m] = 1.0
        try:
            c = np.linalg.solve(A, rhs)[:m]
        except np.linalg.LinAlgError:
            c = np.zeros(m)
            c[-1] = 1.0
        return sum(ci * (a + self.alpha * r) for ci, a, r in zip(c, self.rin, self.res))


class KpointScf:
    """members: this rank's members (dict global index -> member); weights:
    every member's k weight (sums to 1); costs: every member's cost for the
    partition (only used by `assign`)."""

    def __init__(self, members, weights, n_elec, omega, e_ewald, n_atoms, dist=None):
        self.members = dict(members)
        self.weights = np.asarray(weights, dtype=np.float64)
        self.n_elec, self.omega, self.e_ewald, self.n_atoms = n_elec, omega, e_ewald, n_atoms
        self.dist = dist

    @staticmethod
    def assign(costs, rank, world):
        """Member indices this rank owns (LPT over all ranks)."""
        parts, _ = sharding.partition(list(costs), world)
        return parts[rank]

    def _gather_eigs(self, local):
        merged = sharding.gather_results(local, self.dist)
        return [merged[i] for i in range(len(self.weights))]

    def run(self, ndeg, rho0, tol_per_atom=1e-6, max_iter=30, alpha=0.3, history=6,
            first_passes=4, kT=0.01):
        rho_in = np.asarray(rho0, dtype=np.float64).ravel().copy()
        ng = rho_in.size
        dv = self.omega / ng
        mixer = Pulay(alpha, history)
        eig = {i: None for i in self.members}
        energies = []
        e_prev = None
        out = {"converged": False}
        for it in range(1, max_iter + 1):
            vhxc = None
            for m in self.members.values():
                m.build_v_eff(rho_in)
            if self.members:
                vhxc = next(iter(self.members.values())).v_hxc()
            for i, m in self.members.items():
                for _ in range(max(1, first_passes) if it == 1 else 1):
                    eig[i] = m.diagonalize(ndeg, eig[i])
            all_eig = self._gather_eigs({i: np.asarray(e) for i, e in eig.items()})
            f, e_ts, mu = fermi_weighted(all_eig, self.weights, self.n_elec, kT)
            rho_loc = np.zeros(ng)
            for i, m in self.members.items():
                rho_loc += m.density(self.weights[i] * f[i])
            rho_out = sharding.reduce_kpoint_density(rho_loc, self.dist)
            if vhxc is None:  # a rank without members still takes part in every exchange
                raise RuntimeError("every rank needs at least one member")
            e_band = sum(w * np.dot(fk, ek) for w, fk, ek in zip(self.weights, f, all_eig))
            dc = float(np.dot(vhxc, rho_out)) * dv
            m0 = next(iter(self.members.values()))
            e_h, e_xc = m0.build_v_eff(rho_out)
            etot = e_band - dc + e_h + e_xc + self.e_ewald + e_ts
            energies.append(etot)
            out = {"converged": False, "n_iter": it, "energies": np.array(energies),
                   "e_total": etot, "mu": mu, "eigenvalues": all_eig, "rho": rho_out,
                   "charge": float(rho_out.sum() * dv)}
            if e_prev is not None and abs(etot - e_prev) / self.n_atoms < tol_per_atom:
                out["converged"] = True
                return out
            e_prev = etot
            rho_in = mixer.mix(rho_in, rho_out)
        return out


def kpoint_systems(chfsi, config_index, kpts, **overrides):
    """Synthetic systems of one cell at the given k-points (reduced coordinates)."""
    return [chfsi.SyntheticSystem(config_index=config_index, kpt=k, **overrides) for k in kpts]


def run_device_kpoint_scf(chfsi, systems, weights, ndeg, rank=0, world=1, dist=None, device=0,
                          precision=None, **scf_args):
    """Build this rank's device members (LPT share of `systems`) and run the
    k-point SCF; every rank returns the same result."""
    costs = [sharding.member_cost(s.n_pw, s.n_bands, s.ngrid) for s in systems]
    mine = KpointScf.assign(costs, rank, world)
    prec = chfsi.PREC_FP64 if precision is None else precision
    members = {i: DeviceMember(chfsi.Context(systems[i], device=device, precision=prec))
               for i in mine}
    s0 = systems[0]
    scf = KpointScf(members, weights, s0.n_elec, s0.omega, s0.e_ewald, s0.n_atoms, dist)
    rho0 = np.full(s0.ng_density, s0.n_elec / s0.omega)
    return scf.run(ndeg, rho0, **scf_args)
