"""The segmented-GEMM engine of the factorization against FP64 numpy.

FP32 plans with more than 16 output columns run on the tcgen05 tensor cores
with the 3-term TF32 split (hi*hi + hi*lo + lo*hi); the result must keep
FP32 accuracy: |C - C_ref| <= 1e-5 * (|alpha| |op(A)| |op(B)| + |beta| |C0|)
elementwise (k up to 300 terms of FP32 products; a single TF32 pass would
miss this by two orders of magnitude), the same bound the SIMT kernel
meets.  Covered: the four transpose combinations, ragged tiles (m, n
not multiples of 128, k not a multiple of 32), leading dimensions that are
not multiples of 4 (scalar-load path), several terms per output, alpha and
beta, and tensor cores on versus off.  FP64 plans run on the FP64 tensor
cores (mma.sync m8n8k4, 64 x 64 tiles) over the same cases, or on the SIMT
kernel with tensor cores off, both to 1e-14 of the same magnitude bound.
"""
import ctypes as C

import numpy as np
import pytest

from mxc_b200 import _lib

pytestmark = pytest.mark.gpu


def _colmajor(rng, rows, cols, ld, count, dtype):
    """count column-major rows x cols blocks with leading dimension ld, as a
    flat array with stride ld * cols between blocks."""
    X = np.zeros((count, cols, ld), dtype=np.float64)
    X[:, :, :rows] = rng.standard_normal((count, cols, rows))
    return X.astype(dtype)


def _run(handle, precision, batch, nterms, m, n, k, opA, opB, alpha, beta, lda, ldb, ldc, seed):
    import torch

    dt = np.float32 if precision == _lib.FP32 else np.float64
    rng = np.random.default_rng(seed)
    ar, ac = (k, m) if opA else (m, k)
    br, bc = (n, k) if opB else (k, n)
    A = _colmajor(rng, ar, ac, lda, batch * nterms, dt)
    B = _colmajor(rng, br, bc, ldb, batch * nterms, dt)
    C0 = _colmajor(rng, m, n, ldc, batch, dt)
    dA = torch.from_numpy(A.reshape(-1)).cuda()
    dB = torch.from_numpy(B.reshape(-1)).cuda()
    dC = torch.from_numpy(C0.reshape(-1).copy()).cuda()
    torch.cuda.synchronize()
    rc = _lib.lib().h2dev_batched_gemm_device(
        handle.h, precision, batch, nterms, m, n, k, opA, opB, alpha, C.c_void_p(dA.data_ptr()), lda, lda * ac,
        C.c_void_p(dB.data_ptr()), ldb, ldb * bc, beta, C.c_void_p(dC.data_ptr()), ldc, ldc * n)
    _lib.check(rc, "h2dev_batched_gemm_device")
    handle.synchronize()
    got = dC.cpu().numpy().reshape(batch, n, ldc)[:, :, :m]
    A64 = A.astype(np.float64)[:, :, :ar]
    B64 = B.astype(np.float64)[:, :, :br]
    worst = 0.0
    for b in range(batch):
        ref = beta * C0[b, :, :m].astype(np.float64).T
        mag = abs(beta) * np.abs(C0[b, :, :m].astype(np.float64).T)
        for t in range(nterms):
            a = A64[b * nterms + t].T  # rows x cols
            bb = B64[b * nterms + t].T
            opa = a.T if opA else a
            opb = bb.T if opB else bb
            ref = ref + alpha * opa @ opb
            mag = mag + abs(alpha) * np.abs(opa) @ np.abs(opb)
        err = np.abs(got[b].T.astype(np.float64) - ref)
        worst = max(worst, float(np.max(err / mag)))
    return worst


CASES = [
    # batch, nterms, m, n, k, opA, opB, alpha, beta, lda, ldb, ldc
    (3, 1, 256, 256, 256, 0, 0, 1.0, 0.0, 256, 256, 256),
    (2, 1, 256, 192, 128, 1, 0, 1.0, 1.0, 128, 128, 256),
    (2, 1, 200, 72, 100, 0, 1, -1.0, 1.0, 200, 72, 200),
    (2, 1, 130, 140, 33, 1, 1, 0.5, 2.0, 33, 140, 131),
    (2, 3, 128, 128, 64, 0, 0, 1.0, 0.0, 129, 65, 128),
    (1, 2, 300, 40, 300, 1, 0, -1.0, 1.0, 301, 303, 300),
    (4, 1, 17, 19, 5, 0, 0, 1.0, 0.0, 17, 5, 17),
]


@pytest.mark.parametrize("case", CASES, ids=[str(i) for i in range(len(CASES))])
def test_fp32_tensor_core_gemm_keeps_fp32_accuracy(handle, case):
    worst = _run(handle, _lib.FP32, *case, seed=hash(case) % 1000)
    assert worst < 1e-5, worst


@pytest.mark.parametrize("case", CASES[:4], ids=[str(i) for i in range(4)])
def test_fp32_simt_gemm_same_bound(handle, case):
    handle.set_option(_lib.OPT_TENSOR_CORES, 0)
    try:
        worst = _run(handle, _lib.FP32, *case, seed=7)
    finally:
        handle.set_option(_lib.OPT_TENSOR_CORES, 1)
    assert worst < 1e-5, worst


# Outputs of at most 16 columns with A and B as stored go to the streaming
# kernels of the block-sparse applies (FP32: TF32 mma.sync with the split in
# registers; FP64: mma.sync m8n8k4), rows in 128- and 256-row tiles; long
# single entries are cut along k and their partials summed in order.
SKINNY = [
    # batch, nterms, m, n, k, opA, opB, alpha, beta, lda, ldb, ldc
    (3, 1, 256, 16, 256, 0, 0, 1.0, 0.0, 256, 256, 256),
    (2, 3, 300, 16, 200, 0, 0, -1.0, 1.0, 301, 203, 300),
    (4, 2, 130, 8, 77, 0, 0, 0.5, 2.0, 131, 77, 130),
    (2, 1, 700, 16, 900, 0, 0, 1.0, 1.0, 700, 900, 701),
    (2, 1, 45, 3, 33, 0, 0, 1.0, 0.0, 45, 33, 45),
]


@pytest.mark.parametrize("case", SKINNY, ids=[str(i) for i in range(len(SKINNY))])
def test_fp32_streaming_apply_keeps_fp32_accuracy(handle, case):
    worst = _run(handle, _lib.FP32, *case, seed=11)
    assert worst < 1e-5, worst


@pytest.mark.parametrize("case", SKINNY, ids=[str(i) for i in range(len(SKINNY))])
def test_fp64_streaming_apply(handle, case):
    worst = _run(handle, _lib.FP64, *case, seed=12)
    assert worst < 1e-14, worst


@pytest.mark.parametrize("case", CASES, ids=[str(i) for i in range(len(CASES))])
def test_fp64_tensor_core_gemm(handle, case):
    worst = _run(handle, _lib.FP64, *case, seed=9)
    assert worst < 1e-14, worst


@pytest.mark.parametrize("case", CASES[:2], ids=[str(i) for i in range(2)])
def test_fp64_simt_gemm(handle, case):
    handle.set_option(_lib.OPT_TENSOR_CORES, 0)
    try:
        worst = _run(handle, _lib.FP64, *case, seed=9)
    finally:
        handle.set_option(_lib.OPT_TENSOR_CORES, 1)
    assert worst < 1e-14, worst
