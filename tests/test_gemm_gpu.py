"""The tcgen05 tensor-core GEMM (hzlb_gemm) against an FP64 matmul of the same (BF16 or
TF32-read) inputs, for tile-aligned and ragged shapes, K-contiguous and transposed operands,
and beta accumulation."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(lib, M, N, K, dtype, A, lda, ak, B, ldb, bk, Cm, ldc, alpha=1.0, beta=0.0):
    fn = lib.hzlb_gemm
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_longlong, C.c_int,
                   C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_longlong, C.c_float,
                   C.c_float, C.c_void_p]
    import torch
    rc = fn(M, N, K, dtype, A.data_ptr(), lda, ak, B.data_ptr(), ldb, bk, Cm.data_ptr(), ldc,
            alpha, beta, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.hzlb_last_error().decode()
    torch.cuda.synchronize()


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (200, 72, 100), (1024, 512, 512),
                                   (37, 16, 8), (256, 520, 72)])
@pytest.mark.parametrize("ak,bk", [(1, 1), (0, 1), (1, 0), (0, 0)])
def test_bf16_gemm(hzlb, M, N, K, ak, bk):
    import torch
    lib = hzlb.library()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    a = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    A = a.contiguous() if ak else a.t().contiguous()
    B = b.contiguous() if bk else b.t().contiguous()
    c0 = torch.randn(M, N, device="cuda", generator=g)
    out = c0.clone()
    _gemm(lib, M, N, K, 2, A, K if ak else M, ak, B, K if bk else N, bk, out, N, 0.5, 2.0)
    ref = 0.5 * (a.double() @ b.double().t()) + 2.0 * c0.double()
    err = (out.double() - ref).norm() / ref.norm()
    assert err < 1e-5, float(err)


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 200, 130)])
def test_tf32_gemm(hzlb, M, N, K):
    import torch
    lib = hzlb.library()
    g = torch.Generator(device="cuda").manual_seed(3)
    a = torch.randn(M, K, device="cuda", generator=g)
    b = torch.randn(N, K, device="cuda", generator=g)
    out = torch.zeros(M, N, device="cuda")
    _gemm(lib, M, N, K, 4, a, K, 1, b, K, 1, out, N)
    ref = a.double() @ b.double().t()
    err = (out.double() - ref).norm() / ref.norm()
    assert err < 2e-3, float(err)
