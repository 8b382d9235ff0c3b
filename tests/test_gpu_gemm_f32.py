"""The TF32 store GEMM (ebsd_gemm_f32, kind::tf32 on the tcgen05 kernel)
against FP64, on ragged extents that need no padding."""

import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda"


@pytest.mark.parametrize("m,n,k", [(300, 1024, 16384), (37, 5, 100), (128, 256, 32), (1, 1, 4), (1000, 700, 4100)])
def test_gemm_f32_matches_fp64(m, n, k):
    from ebsdtorch_b200 import kernels

    g = torch.Generator(device="cpu").manual_seed(m + n + k)
    A = torch.randn((m, k), generator=g).to(DEV)
    B = torch.randn((n, k), generator=g).to(DEV)
    C = torch.full((m, n + 3), 7.0, device=DEV)  # ldc > n; the extra columns stay untouched
    st = kernels.gemm_f32(A, B, C[:, :n], alpha=0.5)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = 0.5 * (A.double() @ B.double().t())
    scale = (A.double().norm(dim=1)[:, None] * B.double().norm(dim=1)[None, :])
    err = float(((C[:, :n].double() - ref).abs() / scale).max())
    assert err < 2e-3, err  # TF32 inputs (10-bit mantissa), FP32 accumulation
    assert bool((C[:, n:] == 7.0).all())
    # accumulate into the existing values
    kernels.gemm_f32(A, B, C[:, :n], alpha=1.0, accumulate=True, status=st)
    torch.cuda.synchronize()
    err2 = float(((C[:, :n].double() - 3.0 * ref).abs() / scale).max())
    assert err2 < 4e-3, err2


def test_gemm_f32_strided_rows():
    """Row strides larger than k (a column slice of a wider matrix)."""
    from ebsdtorch_b200 import kernels

    g = torch.Generator(device="cpu").manual_seed(5)
    W = torch.randn((200, 260), generator=g).to(DEV)
    A, B = W[:, :96], W[:50, 100:196]
    C = torch.empty((200, 50), device=DEV)
    kernels.gemm_f32(A, B, C)
    torch.cuda.synchronize()
    ref = A.double() @ B.double().t()
    assert float((C.double() - ref).abs().max() / ref.abs().max()) < 2e-3
