"""Band-parallel ChFSI of one cell over ranks (one process per GPU).

Each rank owns a contiguous block of the bands, all plane waves
(ColumnDistributed, src/layout.rs:22-40).  The Chebyshev filter is per band,
so each rank filters its block with no communication.  The Rayleigh-Ritz
needs every band: it follows the reference's planned Row/Column design
(PROJECT_ROOT_PLAN.md:213-234, 482-488):

  1. all-to-all from the band split to a plane-wave split (every band, one
     slice of the plane waves per rank), for psi and H psi;
  2. local partial products psi_r^H psi_r and psi_r^H H psi_r over the
     rank's plane-wave slice (n_b x n_b each);
  3. one all-reduce (sum) of the two n_b^2 matrices;
  4. the small generalised eigenproblem, redundantly on every rank;
  5. the rotation psi <- psi V of the rank's plane-wave slice;
  6. all-to-all back to the band split.

The math of steps 2, 4 and 5 goes through an `ops` object: `DeviceOps` uses
the library's own FP64 tensor-path GEMMs (chfsi_zgemm_cn / chfsi_zgemm_tn)
and its Cholesky + Jacobi eigensolver (chfsi_hegv_dev) on CUDA tensors, the
collectives are NCCL.

For the ultrasoft overlap S = 1 + beta q beta^H the subspace overlap is
S_sub = psi^H psi + C^H q C with C = beta^H psi: step 2 also forms the
partial C_r = beta_r^H psi_r over the rank's plane waves, step 3 sums it
with the two n_b^2 matrices (one all-reduce), and C^H q C is formed on every
rank after the sum (it is not a sum of per-rank terms).
"""
import numpy as np

import chfsi


def split_counts(n, parts):
    """Sizes of `parts` contiguous blocks of n items (the first n % parts get one more)."""
    base, extra = divmod(n, parts)
    return [base + (1 if r < extra else 0) for r in range(parts)]


def offsets(counts):
    return np.concatenate([[0], np.cumsum(counts)]).astype(int)


class _CudaView:
    """__cuda_array_interface__ of a device buffer owned by the library."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<c16",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def device_view(ptr, shape):
    """A torch complex128 CUDA tensor aliasing a library device buffer."""
    import torch
    return torch.as_tensor(_CudaView(ptr, shape), device="cuda")


class DeviceOps:
    """Steps 2, 4 and 5 on the GPU with the library's kernels (torch CUDA
    tensors, complex128, row-major)."""

    def __init__(self):
        import torch
        self.torch = torch

    def stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    def gemm_cn(self, a, b):
        """conj(a) b^T: (m x k), (n x k) -> (m x n)."""
        t = self.torch
        m, k = a.shape
        n = b.shape[0]
        c = t.empty((m, n), dtype=t.complex128, device=a.device)
        chfsi.zgemm_cn(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(), self.stream())
        return c

    def rotate(self, v, x):
        """v^T x: (k x m), (k x n) -> (m x n)."""
        t = self.torch
        k, m = v.shape
        n = x.shape[1]
        o = t.empty((m, n), dtype=t.complex128, device=x.device)
        chfsi.zgemm_tn(v.data_ptr(), m, x.data_ptr(), n, o.data_ptr(), n, m, n, k, 1.0, 0.0,
                       self.stream())
        return o

    def hegv(self, h, s):
        t = self.torch
        n = h.shape[0]
        v = t.empty((n, n), dtype=t.complex128, device=h.device)
        w = chfsi.hegv_dev(h.contiguous().data_ptr(), s.contiguous().data_ptr(), n, v.data_ptr(),
                           self.stream())
        return w, v


def _all_to_all(x_blocks, recv_rows, send_cols, recv_cols, dist):
    """Band split -> plane-wave split of complex128 rows: rank r sends to rank
    q its rows restricted to q's column slice (send_cols[q] columns) and
    receives q's recv_rows[q] rows restricted to its own recv_cols columns."""
    import torch
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    c0 = offsets(send_cols)
    pieces = [x_blocks[:, c0[q]:c0[q + 1]].contiguous() for q in range(world)]
    if world == 1:
        return pieces[0]
    inp = torch.cat([torch.view_as_real(p).reshape(-1) for p in pieces])
    out_sizes = [recv_rows[q] * recv_cols * 2 for q in range(world)]
    out = torch.empty(sum(out_sizes), dtype=torch.float64, device=x_blocks.device)
    dist.all_to_all_single(out, inp, output_split_sizes=out_sizes,
                           input_split_sizes=[p.numel() * 2 for p in pieces])
    parts = torch.split(out, out_sizes)
    rows = [torch.view_as_complex(p.reshape(recv_rows[q], recv_cols, 2))
            for q, p in enumerate(parts)]
    return torch.cat(rows, dim=0)


def qmat_dense(qblocks, proj_offsets):
    """The block-diagonal n_proj x n_proj q from its per-ion blocks (the
    layout of chfsi_set_qmat)."""
    off = np.asarray(proj_offsets)
    n = int(off[-1])
    q = np.zeros((n, n), dtype=np.complex128)
    k = 0
    for i in range(len(off) - 1):
        a, b = int(off[i]), int(off[i + 1])
        ne = b - a
        q[a:b, a:b] = np.asarray(qblocks[k:k + ne * ne]).reshape(ne, ne)
        k += ne * ne
    return q


def rayleigh_ritz_bandsplit(psi_blk, hpsi_blk, nb, npw, rank, world, dist, ops, beta_pw=None,
                            qmat=None):
    """Steps 1-6 for this rank's band block (torch complex128 tensors,
    nb_r x npw).  For the ultrasoft overlap, beta_pw is this rank's
    plane-wave slice of the projectors (n_proj x its plane waves) and qmat
    the dense n_proj x n_proj q (torch tensors).  Returns (new band block,
    eigenvalues of all bands)."""
    import torch
    bands = split_counts(nb, world)
    pws = split_counts(npw, world)
    # 1. band split -> plane-wave split (all bands, this rank's plane waves)
    p = _all_to_all(psi_blk, bands, pws, pws[rank], dist)
    hp = _all_to_all(hpsi_blk, bands, pws, pws[rank], dist)
    # 2. partial subspace matrices over this rank's plane waves
    s = ops.gemm_cn(p, p)
    h = ops.gemm_cn(p, hp)
    c = ops.gemm_cn(beta_pw, p) if beta_pw is not None else None
    # 3. sum over ranks
    if world > 1:
        mats = [s, h] + ([c] if c is not None else [])
        flat = torch.cat([torch.view_as_real(m).reshape(-1) for m in mats])
        dist.all_reduce(flat)
        parts = torch.split(flat, [m.numel() * 2 for m in mats])
        mats = [torch.view_as_complex(x.reshape(*m.shape, 2)) for x, m in zip(parts, mats)]
        s, h = mats[0], mats[1]
        if c is not None:
            c = mats[2]
    if c is not None:
        # S_sub = psi^H psi + C^H q C: conj(C^T) (q C)
        qc = qmat @ c
        s = s + ops.gemm_cn(c.T.contiguous(), qc.T.contiguous())
    # 4. the small eigenproblem, redundant on every rank
    w, v = ops.hegv(h, s)
    # 5. rotation of this rank's plane-wave slice
    pn = ops.rotate(v, p)
    # 6. plane-wave split -> band split: rank r sends the rows of band block
    # q (its plane waves) to rank q, and receives its own band rows from
    # every rank
    b0 = offsets(bands)
    pieces = [pn[b0[q]:b0[q + 1], :].contiguous() for q in range(world)]
    if world == 1:
        return pieces[0], np.asarray(w)
    inp = torch.cat([torch.view_as_real(x).reshape(-1) for x in pieces])
    out_sizes = [bands[rank] * pws[q] * 2 for q in range(world)]
    out = torch.empty(sum(out_sizes), dtype=torch.float64, device=pn.device)
    dist.all_to_all_single(out, inp, output_split_sizes=out_sizes,
                           input_split_sizes=[x.numel() * 2 for x in pieces])
    cols = [torch.view_as_complex(x.reshape(bands[rank], pws[q], 2))
            for q, x in enumerate(torch.split(out, out_sizes))]
    return torch.cat(cols, dim=1), np.asarray(w)


class BandParallelChfsi:
    """One cell's bands split over the ranks, one chfsi.Context per rank
    holding its band block (the block's filter runs there)."""

    def __init__(self, system, rank=0, world=1, dist=None, device=0):
        import torch
        self.nb, self.npw = system.n_bands, system.n_pw
        self.rank, self.world, self.dist = rank, world, dist
        counts = split_counts(self.nb, world)
        if min(counts) < 2:
            raise ValueError("every rank needs at least two bands")
        b0 = offsets(counts)
        self.b0, self.b1 = int(b0[rank]), int(b0[rank + 1])
        p = chfsi.SynthParams()
        chfsi.C.memmove(chfsi.C.byref(p), chfsi.C.byref(system.params), chfsi.C.sizeof(p))
        p.n_bands = self.b1 - self.b0
        self.block = chfsi.SyntheticSystem(params=p)
        self.ctx = chfsi.Context(self.block, device=device)
        # the block's start vectors: its rows of the whole cell's psi0
        self.ctx.set_psi(system.psi0()[self.b0:self.b1])
        self.ops = DeviceOps()
        self.torch = torch

    def set_veff(self, v):
        self.ctx.set_veff(v)

    def diagonalize(self, ndeg, eig=None):
        """Filter this rank's block, then the band-split Rayleigh-Ritz;
        returns the eigenvalues of all bands (every rank)."""
        nb_r = self.b1 - self.b0
        bounds = None if eig is None else np.array([np.min(eig), np.max(eig)])
        self.ctx.chebyshev_filter(ndeg, bounds)
        psi = device_view(self.ctx.psi_device_ptr(), (nb_r, self.npw))
        hpsi = device_view(self.ctx.hpsi_device_ptr(), (nb_r, self.npw))
        self.torch.cuda.synchronize()
        new, w = rayleigh_ritz_bandsplit(psi, hpsi, self.nb, self.npw, self.rank, self.world,
                                         self.dist, self.ops)
        psi.copy_(new)
        self.torch.cuda.synchronize()
        return w
