"""The split-BF16 tcgen05 GEMM (``dfb_tc_gemm``) against FP64 products.

Three bfloat16 terms per operand with the six cross products of order <= 2^-16 and FP32
accumulation per k span give about 1e-7 relative per element for general products; sums of
squares (the exchange update's diagonal) carry the tensor cores' FP32 accumulation bias, ~1e-6
over 512-long spans.  Two terms (three products) give about 1e-5.
Shapes cover partial tiles in m, n and k, every tile width (32, 48, 64, 128), split-K with
FP64 atomic combination, the symmetric exchange update over a strided (Q, i) k index, and
batched products.
"""

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _rel(a, b):
    return float((a - b).abs().max()) / float(b.abs().max())


@pytest.fixture(autouse=True)
def _no_wait_errors():
    from asuka_b200 import tc

    tc.error_flag(reset=True)
    yield
    torch.cuda.synchronize()
    assert tc.error_flag(reset=True) == 0


@pytest.mark.parametrize("m,k,n", [(300, 416, 40), (1000, 64, 30), (129, 33, 64), (517, 200, 128), (256, 700, 250)])
def test_matmul_matches_fp64(m, k, n):
    from asuka_b200 import tc

    g = torch.Generator(device="cuda").manual_seed(m + k + n)
    A = torch.randn(m, k, generator=g, dtype=torch.float64, device="cuda")
    B = torch.randn(k, n, generator=g, dtype=torch.float64, device="cuda")
    ref = A @ B
    C = tc.matmul(A, B)
    assert _rel(C, ref) < 1e-6
    # strided (transposed) operands read in place
    C2 = tc.matmul(B.T, A.T)
    assert _rel(C2, ref.T) < 1e-6
    # two terms: about 16 significant bits
    C3 = tc.matmul(A, B, nterms=2)
    assert 1e-7 < _rel(C3, ref) < 1e-4


def test_split_k_accumulation():
    from asuka_b200 import tc

    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.randn(200, 5000, generator=g, dtype=torch.float64, device="cuda")
    B = torch.randn(5000, 96, generator=g, dtype=torch.float64, device="cuda")
    assert _rel(tc.matmul(A, B), A @ B) < 2e-6


def test_exchange_update_over_q_blocks():
    """K = sum_{Q,i} W[Q,m,i] W[Q,n,i] with the (Q, i) k index read in place, symmetric tiles."""
    from asuka_b200 import tc

    g = torch.Generator(device="cuda").manual_seed(2)
    W = torch.randn(700, 300, 37, generator=g, dtype=torch.float64, device="cuda")
    ref = torch.einsum("qmi,qni->mn", W, W)
    K = tc.syrk_qblocks(W)
    # the diagonal sums of squares carry the FP32 accumulation bias of 512-long spans (~1e-6)
    assert _rel(K, ref) < 1.5e-6
    assert torch.equal(K, K.T)
    K0 = torch.ones_like(ref)
    tc.syrk_qblocks(W, out=K0)  # adds to the start value
    assert _rel(K0 - 1.0, ref) < 1.5e-6
    A = torch.randn(260, 3000, generator=g, dtype=torch.float64, device="cuda")
    assert _rel(tc.syrk_rows(A), A @ A.T) < 1.5e-6


def test_batched_products():
    from asuka_b200 import tc

    g = torch.Generator(device="cuda").manual_seed(3)
    Cw = torch.randn(150, 40, generator=g, dtype=torch.float64, device="cuda")
    T = torch.randn(37, 40, 150, generator=g, dtype=torch.float64, device="cuda")
    ref = torch.matmul(Cw, T)
    assert _rel(tc.bmm(Cw, T), ref) < 1e-6
    A = torch.randn(37, 70, 40, generator=g, dtype=torch.float64, device="cuda")
    assert _rel(tc.bmm(A, T), torch.matmul(A, T)) < 1e-6
