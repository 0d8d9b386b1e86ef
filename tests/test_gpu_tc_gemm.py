"""The large-molecule path's tensor-core GEMM (tcgen05.mma, FP32 accumulator in
tensor memory, TMA tile loads) against an FP64 product of the same BF16
terms, through the test harness library tests/csrc/libtc_gemm_probe.so.

C = sum_s T[a_s] T[b_s]^T over stacked Np x Np BF16 terms.  FP32
accumulation of BF16 products: each entry within 1e-5 of the sum of the
absolute products (plus 1e-30).  The kernel's bounded barrier wait is
checked on its own: a wait that nothing completes gives up after its limit
and reports it, with the context still usable."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(ROOT, "csrc", "libtc_gemm_probe.so")


def _lib():
    if not os.path.exists(LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "csrc")])
    return ctypes.CDLL(LIB)


def run_gemm(T, a_terms, b_terms, ldc=None, allow_split=False, want_split=None):
    """T: torch bf16 (nterms, Np, Np) on cuda; returns (C as float64 numpy, err word).
    allow_split: pass the second output, so the launcher may split K (the
    product is then the sum of both); want_split: the split it must choose."""
    import torch
    L = _lib()
    nterms, Np, _ = T.shape
    ldc = Np if ldc is None else ldc
    C = torch.full((Np, ldc), float("nan"), dtype=torch.float32, device=T.device)
    C2 = torch.full((Np, ldc), float("nan"), dtype=torch.float32, device=T.device) if allow_split else None
    err = torch.zeros(1, dtype=torch.int32, device=T.device)
    ks = ctypes.c_int(0)
    a = (ctypes.c_int * len(a_terms))(*a_terms)
    b = (ctypes.c_int * len(b_terms))(*b_terms)
    rc = L.tc_gemm_probe(ctypes.c_void_p(T.data_ptr()), nterms, Np, a, b, len(a_terms), ctypes.c_void_p(C.data_ptr()),
                         ctypes.c_void_p(C2.data_ptr()) if C2 is not None else None, ldc,
                         ctypes.c_void_p(err.data_ptr()), ctypes.byref(ks))
    assert rc == 0, "tc_gemm_probe returned CUDA error %d" % rc
    if want_split is not None:
        assert ks.value == want_split, ks.value
    out = C[:, :Np].double()
    if ks.value == 2:
        out = out + C2[:, :Np].double()
    else:
        assert ks.value == 1
    return out.cpu().numpy(), int(err.item())


def reference(T, a_terms, b_terms):
    Td = T.double().cpu().numpy()
    C = np.zeros(Td.shape[1:])
    A = np.zeros(Td.shape[1:])
    for a, b in zip(a_terms, b_terms):
        C += Td[a] @ Td[b].T
        A += np.abs(Td[a]) @ np.abs(Td[b]).T
    return C, A


SPLIT_A = [0, 0, 0, 1]
SPLIT_B = [3, 1, 2, 4]


@pytest.mark.gpu
@pytest.mark.parametrize("Np", [128, 256, 384, 1536, 2944])
def test_split_product_matches_fp64(Np):
    import torch
    g = torch.Generator(device="cpu").manual_seed(Np)
    T = (torch.rand((5, Np, Np), generator=g, dtype=torch.float64) * 2 - 1).to(torch.bfloat16).cuda()
    C, err = run_gemm(T, SPLIT_A, SPLIT_B)
    assert err == 0
    ref, absref = reference(T, SPLIT_A, SPLIT_B)
    assert np.all(np.isfinite(C))
    assert np.all(np.abs(C - ref) <= 1e-5 * absref + 1e-30), np.max(np.abs(C - ref) / (absref + 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("Np", [384, 1536])
def test_split_k_launch_matches_fp64(Np):
    """Small sizes run 256-wide tiles over half the K range each into two
    outputs; their sum is the product."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(100 + Np)
    T = (torch.rand((5, Np, Np), generator=g, dtype=torch.float64) * 2 - 1).to(torch.bfloat16).cuda()
    C, err = run_gemm(T, SPLIT_A, SPLIT_B, allow_split=True, want_split=2)
    assert err == 0
    ref, absref = reference(T, SPLIT_A, SPLIT_B)
    assert np.all(np.abs(C - ref) <= 1e-5 * absref + 1e-30), np.max(np.abs(C - ref) / (absref + 1e-30))


@pytest.mark.gpu
def test_large_sizes_do_not_split():
    import torch
    Np = 3072
    g = torch.Generator(device="cpu").manual_seed(5)
    T = (torch.rand((2, Np, Np), generator=g, dtype=torch.float64) * 2 - 1).to(torch.bfloat16).cuda()
    C, err = run_gemm(T, [0], [1], allow_split=True, want_split=1)
    assert err == 0
    ref, absref = reference(T, [0], [1])
    assert np.all(np.abs(C - ref) <= 1e-5 * absref + 1e-30)


@pytest.mark.gpu
def test_tile_widths_cover_both_kernels():
    L = _lib()
    widths = {Np: L.tc_gemm_tile_n(Np) for Np in (128, 384, 1536, 2944, 3072, 6144)}
    assert set(widths.values()) == {128, 256}, widths


@pytest.mark.gpu
def test_single_segment_with_padded_leading_dimension():
    import torch
    Np = 256
    g = torch.Generator(device="cpu").manual_seed(7)
    T = torch.randn((2, Np, Np), generator=g, dtype=torch.float64).to(torch.bfloat16).cuda()
    C, err = run_gemm(T, [0], [1], ldc=Np + 4)
    assert err == 0
    ref, absref = reference(T, [0], [1])
    assert np.all(np.abs(C - ref) <= 1e-5 * absref + 1e-30)


@pytest.mark.gpu
def test_split_of_symmetric_matrix_reproduces_its_square():
    """The SP2 use: X = X1 + X2 + X3 in BF16, X X ~ A + A^T to FP32 accuracy."""
    import torch
    Np = 384
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.standard_normal((Np, Np)))
    X = (Q * rng.uniform(0, 1, Np)) @ Q.T
    X = 0.5 * (X + X.T)
    t = torch.tensor(X)
    x1 = t.to(torch.bfloat16)
    r1 = t - x1.double()
    x2 = r1.to(torch.bfloat16)
    x3 = (r1 - x2.double()).to(torch.bfloat16)
    T = torch.stack([x1, x2, x3, x1 * 0.5, x2 * 0.5]).cuda()
    A, err = run_gemm(T, SPLIT_A, SPLIT_B)
    assert err == 0
    X2 = A + A.T
    assert np.max(np.abs(X2 - X @ X)) < 1e-5


def _wait_probe(arrive):
    import torch
    L = _lib()
    out = torch.zeros(2, dtype=torch.int32, device="cuda")
    rc = L.tc_wait_probe(arrive, ctypes.c_void_p(out.data_ptr()))
    assert rc == 0, "tc_wait_probe returned CUDA error %d" % rc
    ok, ms = (int(v) for v in out.cpu())
    return ok, ms


@pytest.mark.gpu
def test_bounded_barrier_wait_gives_up_and_reports():
    """The GEMM's barrier waits are bounded: a wait on a barrier nothing
    arrives at returns 'not completed' after the limit instead of spinning
    for ever, and the context stays usable (a product right after it is
    exact).  A wait whose arrival came first returns at once."""
    import torch
    L = _lib()
    limit = L.tc_wait_limit_ms()
    ok, ms = _wait_probe(0)
    assert ok == 0
    assert limit <= ms <= limit + 2000, (ms, limit)
    ok, ms = _wait_probe(1)
    assert ok == 1 and ms < 100
    Np = 128
    g = torch.Generator(device="cpu").manual_seed(11)
    T = torch.randn((2, Np, Np), generator=g, dtype=torch.float64).to(torch.bfloat16).cuda()
    C, err = run_gemm(T, [0], [1])
    assert err == 0
    ref, absref = reference(T, [0], [1])
    assert np.all(np.abs(C - ref) <= 1e-5 * absref + 1e-30)


def test_launch_plan_on_the_host():
    """The launcher's tile width and K split (host logic, no GPU): 148 SMs,
    the four-segment split-BF16 product."""
    L = _lib()

    def plan(Np, have_c2):
        bn, ks = ctypes.c_int(0), ctypes.c_int(0)
        L.tc_gemm_plan(Np, 148, 4, 1 if have_c2 else 0, ctypes.byref(bn), ctypes.byref(ks))
        return bn.value, ks.value

    # (H2O)_256: 128 x 256 tiles would fill half the SMs, so K is split
    assert plan(1536, True) == (256, 2)
    assert plan(1536, False) == (128, 1)
    # (H2O)_512 and (H2O)_1024: 288 and 1152 tiles of 128 x 256, no split
    assert plan(3072, True) == (256, 1)
    assert plan(6144, True) == (256, 1)

