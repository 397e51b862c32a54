"""The tensor-core RNS GEMM (tcgen05.mma.kind::i8 on residues, CRT) against the exact schoolbook GEMM on the
CUDA cores: both compute the exact integer dot products of the aligned operands and round once, so the
results must be identical bit for bit, for any shape, batch, sign pattern and limb count."""
import pytest
import torch

from blocksvibe_b200 import mpf, rns

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,nb,M,K,N", [
    (10, 1, 4, 3, 5),          # tiny, padded everywhere
    (10, 3, 40, 33, 70),       # M < N: B on the TMEM lanes
    (10, 2, 130, 64, 17),      # several row tiles
    (18, 1, 12, 98, 600),      # numerator-like
    (34, 1, 42, 42, 300),      # write_output-like, 1024 bits
    (34, 5, 12, 12, 50),       # residues a_i[e]-like batch
    (42, 1, 66, 192, 96),      # 1280 bits, K near the limit
    (10, 1, 3, 256, 260),      # K = 256, N > one column tile
])
@pytest.mark.parametrize("crt,split", [("tensor", "tensor"), ("cuda", "cuda"), ("tensor", "cuda")])
def test_rns_gemm_bitwise_equals_schoolbook(cuda, L, nb, M, K, N, crt, split):
    rns.SPLIT = split
    g = torch.Generator().manual_seed(L * 1000 + M + K + N)
    A = mpf.random_mpf((nb, M, K), L, spread=20, device=cuda, generator=g)
    B = mpf.random_mpf((nb, K, N), L, spread=20, device=cuda, generator=g)
    # zeros and exact cancellations
    A.m[:, 0, 0, 0] = 0
    A.e[0, 0, 0] = mpf.EZ
    Aal, Bal = mpf.align_rows(A), mpf.align_cols(B)
    ref = mpf.gemm_aligned(Aal, Bal)
    got = rns.gemm_aligned_rns(Aal, Bal, crt=crt)
    torch.cuda.synchronize()
    rns.check_errors(cuda)
    assert torch.equal(ref.e, got.e)
    assert torch.equal(ref.m, got.m)


def test_rns_gemm_cancellation(cuda):
    """rows that cancel exactly give zero; nearly cancelling sums keep all their bits"""
    L = 10
    g = torch.Generator().manual_seed(5)
    A = mpf.random_mpf((1, 2, 8), L, spread=4, device=cuda, generator=g)
    B = mpf.random_mpf((1, 8, 3), L, spread=4, device=cuda, generator=g)
    A.m[:, 0, 1, :] = A.m[:, 0, 0, :]                  # row 1 = row 0: rows give equal results
    A.e[0, 1, :] = A.e[0, 0, :]
    Aal, Bal = mpf.align_rows(A), mpf.align_cols(B)
    ref = mpf.gemm_aligned(Aal, Bal)
    for crt in ("tensor", "cuda"):
        got = rns.gemm_aligned_rns(Aal, Bal, crt=crt)
        assert torch.equal(ref.m, got.m) and torch.equal(ref.e, got.e)


@pytest.mark.parametrize("lanes", ["a", "b"])
@pytest.mark.parametrize("L,nb,M,K,N", [(10, 2, 40, 33, 70), (34, 1, 66, 98, 300), (42, 3, 28, 28, 50)])
def test_rns_gemm_either_operand_on_the_lanes(cuda, lanes, L, nb, M, K, N):
    rns.SPLIT = "tensor"
    g = torch.Generator().manual_seed(L + M + K + N)
    A = mpf.random_mpf((nb, M, K), L, spread=20, device=cuda, generator=g)
    B = mpf.random_mpf((nb, K, N), L, spread=20, device=cuda, generator=g)
    Aal, Bal = mpf.align_rows(A), mpf.align_cols(B)
    ref = mpf.gemm_aligned(Aal, Bal)
    got = rns.gemm_aligned_rns(Aal, Bal, lanes=lanes)
    rns.check_errors(cuda)
    assert torch.equal(ref.m, got.m) and torch.equal(ref.e, got.e)


def test_autotuned_gemm_equals_schoolbook(cuda):
    """the autotuner times the candidate paths per shape and keeps the fastest; every path gives the same bits"""
    rns.SPLIT = "tensor"
    g = torch.Generator().manual_seed(77)
    shapes = [(34, 1, 21, 21, 3000), (34, 40, 12, 12, 50), (18, 2, 66, 98, 200)]
    try:
        for L, nb, M, K, N in shapes:
            A = mpf.random_mpf((nb, M, K), L, spread=10, device=cuda, generator=g)
            B = mpf.random_mpf((nb, K, N), L, spread=10, device=cuda, generator=g)
            mpf.GEMM_BACKEND, mpf.AUTOTUNE = "schoolbook", True
            ref = mpf.gemm(A, B)
            mpf.GEMM_BACKEND = "auto"
            first = mpf.gemm(A, B)                     # tunes this shape
            again = mpf.gemm(A, B)                     # uses the choice
            assert (L, nb, M, N, K, cuda.index or 0) in mpf.tuned_paths()
            for got in (first, again):
                assert torch.equal(ref.m, got.m) and torch.equal(ref.e, got.e)
    finally:
        mpf.GEMM_BACKEND, mpf.AUTOTUNE = "auto", False


def _extreme(shape, L, neg, device):
    """MPF of the largest NB-bit magnitude, 2^NB - 1, exponent 0, sign neg (a bool tensor of the shape)"""
    NB = 32 * L - 2
    v = (1 << NB) - 1
    pos = [(v >> (32 * k)) & 0xFFFFFFFF for k in range(L)]
    negl = [((1 << (32 * L)) - v >> (32 * k)) & 0xFFFFFFFF for k in range(L)]
    m = torch.empty((L,) + tuple(shape), dtype=torch.int64)
    for k in range(L):
        m[k] = torch.where(neg, negl[k], pos[k])
    m = ((m + (1 << 31)) % (1 << 32) - (1 << 31)).to(torch.int32)
    return mpf.MPF(m.to(device), torch.zeros(shape, dtype=torch.int64, device=device))


@pytest.mark.parametrize("L", [10, 34, 42])
@pytest.mark.parametrize("signs", ["positive", "negative", "alternating"])
@pytest.mark.parametrize("crt", ["tensor", "cuda"])
def test_rns_gemm_largest_products(cuda, L, signs, crt):
    """the largest products the residue GEMM meets: K = 256 terms of two all-ones NB-bit magnitudes, all of one
    sign (|P| = 256 (2^NB - 1)^2, x' far from its reduced value) or alternating; bitwise the schoolbook GEMM"""
    M_, K, N = 6, 256, 9
    if signs == "alternating":
        na = (torch.arange(M_ * K).reshape(1, M_, K) % 2) == 1
        nb = torch.zeros((1, K, N), dtype=torch.bool)
    else:
        na = torch.full((1, M_, K), signs == "negative")
        nb = torch.zeros((1, K, N), dtype=torch.bool)
    A, B = _extreme((1, M_, K), L, na, cuda), _extreme((1, K, N), L, nb, cuda)
    Aal, Bal = mpf.align_rows(A), mpf.align_cols(B)
    ref = mpf.gemm_aligned(Aal, Bal)
    got = rns.gemm_aligned_rns(Aal, Bal, crt=crt)
    torch.cuda.synchronize()
    rns.check_errors(cuda)
    assert torch.equal(ref.e, got.e) and torch.equal(ref.m, got.m)
