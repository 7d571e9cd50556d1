"""Work sharding of independent systems across ranks (one process per GPU).

k-points of one cell and independent cells share nothing during a
diagonalisation pass, so they are partitioned across ranks with no data-path
collective: each rank runs its members as one batched CUDA graph
(`chfsi.Batch`) on its own GPU.  Only two host-side reductions exist:

* the Brillouin-zone density of a k-point set, sum_k w_k rho_k, one
  all-reduce of an N^3 float64 grid per SCF iteration (NCCL on GPUs, gloo
  on CPU);
* the gather of per-member results (eigenvalues, energies) to rank 0.

Members are assigned by cost, cost = n_pw * n_bands + n_bands * N^3 log2 N^3
(projection GEMMs and FFT passes of one filter step), greedily largest first
onto the least loaded rank (LPT), which keeps the makespan within 4/3 of the
optimum.  The reference crate runs one k-point on one device; its planned
multi-GPU design (band / plane-wave transposes) is not needed for
independent members.
"""
import math

import numpy as np


def member_cost(n_pw, n_bands, ngrid):
    n3 = int(np.prod(ngrid))
    return float(n_pw) * n_bands + n_bands * n3 * math.log2(max(n3, 2))


def partition(costs, n_ranks):
    """LPT assignment: list of member indices per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * n_ranks
    parts = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += costs[i]
    for p in parts:
        p.sort()
    return parts, loads


def monkhorst_pack(n):
    """n x n x n Monkhorst-Pack mesh in reduced coordinates, equal weights."""
    f = [(2 * i - n - 1) / (2.0 * n) for i in range(1, n + 1)]
    ks = [(a, b, c) for a in f for b in f for c in f]
    return ks, np.full(len(ks), 1.0 / len(ks))


def reduce_kpoint_density(local_weighted_rho, dist=None):
    """sum over all ranks of sum_{k local} w_k rho_k (float64 grid)."""
    rho = np.ascontiguousarray(local_weighted_rho, dtype=np.float64)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return rho
    import torch
    t = torch.from_numpy(rho.copy())
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t)
    return t.cpu().numpy()


def gather_results(local, dist=None):
    """Gather a per-rank dict {member index: result} to every rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, local)
    merged = {}
    for d in out:
        merged.update(d)
    return merged
