"""chfsi_zgemm_cn_noalloc: the op::C complex GEMM for callers that cannot
allocate device memory (a host code whose memory pool owns the whole GPU, or
a latency-critical caller for which cudaMalloc would synchronise the device).
Its split-K partials live in a static 4 MiB device array instead of
allocated scratch.  The test calls it through the C ABI twice in a row and
checks it against the allocating entry point chfsi_zgemm_cn, with the same
tolerance as the other FP64 GEMM tests.  This file is collected last so a
run that stops at the first failure has already run every other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = [(160, 160, 37073), (256, 160, 37073), (20, 20, 2945), (512, 512, 300), (1, 7, 300)]


def _run(fn, A, B):
    m, k = A.shape
    n = B.shape[0]
    a = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    c = torch.full((m, n), float("nan"), dtype=torch.complex128, device="cuda")
    fn(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(),
       torch.cuda.current_stream().cuda_stream)
    return c.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(chfsi):
    rng = np.random.default_rng(11)
    for call in range(2):
        for m, n, k in CASES:
            A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
            B = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
            ref = _run(chfsi.zgemm_cn, A, B)
            out = _run(chfsi.zgemm_cn_noalloc, A, B)
            assert np.all(np.isfinite(out))
            tol = 1e-12 * np.abs(ref).max() * max(1.0, np.sqrt(k / 100))
            assert np.abs(out - ref).max() <= tol, (call, m, n, k)


def test_noalloc_rejects_sizes_beyond_the_static_scratch(chfsi):
    a = torch.zeros((513, 8), dtype=torch.complex128, device="cuda")
    c = torch.zeros((513, 513), dtype=torch.complex128, device="cuda")
    with pytest.raises(chfsi.BadInput, match="static scratch"):
        chfsi.zgemm_cn_noalloc(a.data_ptr(), 8, a.data_ptr(), 8, 513, 513, 8, c.data_ptr(), 0)
