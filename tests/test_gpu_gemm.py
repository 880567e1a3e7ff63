"""The tcgen05 BF16 GEMM of the learned surrogate against a torch fp32 reference.

C = A * Bt^T on bf16 inputs with fp32 accumulation. The reference multiplies
the same bf16 values in fp32, so the only differences are fp32 summation order:
tolerance 1e-4 relative to the largest |C| (plus 1e-2 relative on bf16 outputs).
"""
import ctypes as C

import pytest

import physics_engine_rs as pe

pytestmark = pytest.mark.gpu


def _gemm():
    f = pe.load_library().pe_mlp_gemm_bf16
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 5 + [C.c_int] * 8 + [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]
    return f


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("M,N,K,relu,bias,splits", [
    (128, 128, 64, 0, False, 1),
    (300, 200, 192, 0, False, 1),
    (1000, 128, 272, 1, True, 1),
    (128, 256, 4096, 0, False, 4),
    (77, 40, 16, 1, True, 1),
])
def test_gemm_matches_fp32_reference(M, N, K, relu, bias, splits):
    import torch

    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    dev = "cuda"
    A = torch.randn(M, K, device=dev, generator=g).to(torch.bfloat16)
    Bt = torch.randn(N, K, device=dev, generator=g).to(torch.bfloat16)
    b = torch.randn(N, device=dev, generator=g) if bias else None
    Cf = torch.full((M, N), float("nan"), device=dev)
    Cb = torch.zeros((M, N), device=dev, dtype=torch.bfloat16)
    part = torch.zeros((splits, M, N), device=dev) if splits > 1 else None
    err = C.c_uint32(0)
    torch.cuda.synchronize()
    rc = _gemm()(_ptr(A), _ptr(Bt), _ptr(Cf), _ptr(Cb), _ptr(b), M, N, K, K, K, N, relu, splits, _ptr(part),
                 C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(err))
    assert rc == 0 and err.value == 0, (rc, err.value)
    ref = A.float() @ Bt.float().T
    if bias:
        ref = ref + b
    if relu:
        ref = ref.clamp_min(0)
    scale = ref.abs().max().item()
    assert (Cf - ref).abs().max().item() <= 1e-4 * scale
    assert (Cb.float() - ref).abs().max().item() <= 1e-2 * scale
