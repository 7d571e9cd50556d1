"""Standalone complex GEMM of the C ABI (op::C ZGEMM) against numpy and the
reference's own ZGEMM known answer (src/device/blas.rs:258-310)."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def run(chfsi, A, B):
    m, k = A.shape
    n = B.shape[0]
    a = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    c = torch.zeros((m, n), dtype=torch.complex128, device="cuda")
    chfsi.zgemm_cn(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(),
                   torch.cuda.current_stream().cuda_stream)
    return c.cpu().numpy()


def test_reference_zgemm_known_answer(chfsi):
    c = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_known_answers.json")))["zgemm_2x2"]
    A = np.array([[complex(*x) for x in r] for r in c["a"]])
    B = np.array([[complex(*x) for x in r] for r in c["b"]])
    E = np.array([[complex(*x) for x in r] for r in c["expected"]])
    # A B = conj(conj(A)) (B^T)^T: feed conj(A) and B^T to the conj-first form
    out = run(chfsi, np.conj(A), B.T.copy())
    assert np.abs(out - E).max() < c["tol"]


@pytest.mark.parametrize("m,n,k", [(160, 160, 37073), (256, 160, 37073), (20, 20, 2945),
                                   (1, 7, 300), (65, 130, 1000)])
def test_zgemm_cn_matches_numpy(chfsi, m, n, k):
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    B = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    ref = np.conj(A) @ B.T
    out = run(chfsi, A, B)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max() * max(1.0, np.sqrt(k / 100))


def run_bf16x3(chfsi, A, B, shape=None):
    m, k = A.shape
    n = B.shape[0]
    a = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    c = torch.zeros((m, n), dtype=torch.complex128, device="cuda")
    chfsi.zgemm_cn_bf16x3(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(),
                          torch.cuda.current_stream().cuda_stream, shape=shape)
    return c.cpu().numpy()


@pytest.mark.parametrize("shape", [0, 1, 2])
@pytest.mark.parametrize("m,n,k", [(20, 20, 2945), (160, 160, 37073), (256, 160, 37073),
                                   (65, 130, 1000), (1, 7, 300), (40, 300, 500)])
def test_tcgen05_bf16x3_matches_fp64(chfsi, m, n, k, shape):
    """BF16 3-way split on tcgen05: error at the FP32 level (bound 1e-6 relative
    to the product of norms)."""
    rng = np.random.default_rng(m * 7 + n + k)
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    B = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    ref = np.conj(A) @ B.T
    out = run_bf16x3(chfsi, A, B, shape)
    scale = np.sqrt(k) * 2.0  # typical |C| for unit-variance entries
    assert np.abs(out - ref).max() < 1e-6 * scale * 10


def test_tcgen05_known_answer(chfsi):
    c = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_known_answers.json")))["zgemm_2x2"]
    A = np.array([[complex(*x) for x in r] for r in c["a"]])
    B = np.array([[complex(*x) for x in r] for r in c["b"]])
    E = np.array([[complex(*x) for x in r] for r in c["expected"]])
    out = run_bf16x3(chfsi, np.conj(A), B.T.copy())
    assert np.abs(out - E).max() < 1e-6
