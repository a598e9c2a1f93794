"""The closure network's tcgen05 BF16 GEMM against an fp32 matmul of the
same bf16 operands (torch, as the checker): every tile width (64 / 128 /
256), one- and multi-block K, and split-K (few tiles, long K)."""

import ctypes

import numpy as np
import pytest

from opendynamo_b200 import _native as N


@pytest.mark.gpu
@pytest.mark.parametrize("M,Nn,K", [(128, 256, 64), (128, 128, 128), (256, 384, 896), (384, 256, 320),
                                    (128, 512, 192), (128, 64, 64), (13824, 256, 896), (8192, 384, 256),
                                    (256, 896, 8192), (384, 256, 4096)])
@pytest.mark.parametrize("bias", [False, True])
def test_gemm_bf16_matches_fp32_matmul(M, Nn, K, bias):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M + Nn + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(Nn, K, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(Nn, device="cuda", generator=g) if bias else None
    C = torch.empty(M, Nn, device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    rc = N.lib().od_gemm_bf16(M, Nn, K, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                              ctypes.c_void_p(C.data_ptr()), ctypes.c_void_p(b.data_ptr() if bias else 0), None)
    assert rc == 0
    ref = A.float() @ B.float().T
    if bias:
        ref = ref + b
    err = (C - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-5, err


@pytest.mark.gpu
def test_gemm_rejects_bad_shapes():
    assert N.lib().od_gemm_bf16(100, 128, 64, ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1), None,
                                None) == -1
    assert N.lib().od_gemm_bf16(128, 128, 60, ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1), None,
                                None) == -1
    assert N.lib().od_gemm_bf16(128, 100, 64, ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1), None,
                                None) == -1


@pytest.mark.gpu
def test_bounded_mbarrier_wait_gives_up_and_completes():
    """The tcgen05 kernels' bounded mbarrier wait: on a barrier nothing
    arrives on it returns false after the poll limit (no hang, no fault); the
    same barrier after one arrival completes."""
    import ctypes
    import time
    from opendynamo_b200 import _native as N
    a, b = ctypes.c_int(-1), ctypes.c_int(-1)
    t0 = time.perf_counter()
    assert N.lib().od_mlp_wait_selftest(10000, 0, ctypes.byref(a), ctypes.byref(b)) == 0
    assert time.perf_counter() - t0 < 30.0
    assert a.value == 0 and b.value == 1
