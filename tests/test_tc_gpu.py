"""tcgen05 tensor-core update c -= a b^T (the mixed-precision LU's trailing
update) against a float64 reference of the same (quantized) operands (GPU)."""
import pytest
import torch

from linearalgebra_b200 import _lib

pytestmark = pytest.mark.gpu

TF32, BF16, FP16 = 0, 1, 2


def tf32_trunc(x: torch.Tensor) -> torch.Tensor:
    """fp32 with the 13 low mantissa bits cleared (the TF32 value the tensor
    core reads from an fp32 container)."""
    return (x.view(torch.int32) & ~0x1FFF).view(torch.float32)


def run(kind, split3, m, n, k, seed=0):
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(seed)
    a32 = torch.randn(m, k, device="cuda", generator=g)
    b32 = torch.randn(n, k, device="cuda", generator=g)
    c = torch.randn(m, n, device="cuda", generator=g)
    c0 = c.clone()
    if kind == TF32:
        a, b = a32, b32
        if split3:
            a_s, b_s = a32 - tf32_trunc(a32), b32 - tf32_trunc(b32)
        else:
            a_s = b_s = None
    else:
        dt = torch.bfloat16 if kind == BF16 else torch.float16
        a, b = a32.to(dt), b32.to(dt)
        a_s = b_s = None
    ws = torch.empty(lib.b200la_tc_update_workspace_size(), dtype=torch.uint8, device="cuda")
    st = lib.b200la_sgemm_tc_update(kind, int(split3), c.data_ptr(), n, m, n, k, a.data_ptr(), b.data_ptr(),
                                    a_s.data_ptr() if a_s is not None else None,
                                    b_s.data_ptr() if b_s is not None else None,
                                    ws.data_ptr(), ws.numel(), torch.cuda.current_stream().cuda_stream)
    _lib.check(st)
    torch.cuda.synchronize()
    if kind == TF32 and not split3:
        ref = c0.double() - tf32_trunc(a32).double() @ tf32_trunc(b32).double().T
        tol = 4 * k * 2.0 ** -10
    elif kind == TF32:
        ref = c0.double() - a32.double() @ b32.double().T
        tol = 4 * k * 2.0 ** -20
    else:
        ref = c0.double() - a.double() @ b.double().T
        tol = 4 * k * 2.0 ** -22
    err = (c.double() - ref).abs().max().item()
    return err, tol


@pytest.mark.parametrize("kind,split3", [(TF32, False), (TF32, True), (BF16, False), (FP16, False)])
@pytest.mark.parametrize("m,n,k", [(128, 128, 128), (300, 200, 256), (1000, 520, 128)])
def test_tc_update_matches_reference(kind, split3, m, n, k):
    err, tol = run(kind, split3, m, n, k)
    assert err <= tol, (err, tol)


def test_tc_update_rejects_bad_depth():
    lib = _lib.load()
    p = torch.empty(1024, device="cuda")
    ws = torch.empty(256, dtype=torch.uint8, device="cuda")
    st = lib.b200la_sgemm_tc_update(BF16, 0, p.data_ptr(), 8, 8, 8, 40, p.data_ptr(), p.data_ptr(), None, None,
                                    ws.data_ptr(), 256, None)
    assert st == _lib.INVALID_ARGUMENT


def pow2_row_scales(x: torch.Tensor):
    """Per-row power-of-two scale s with max|row| * s in [128, 256)."""
    amax = x.abs().amax(dim=1).clamp_min(1e-30)
    e = torch.frexp(amax).exponent
    s = torch.ldexp(torch.ones_like(amax), (8 - e).clamp(-126, 126))
    return s, 1.0 / s


@pytest.mark.parametrize("m,n,k", [(128, 128, 128), (300, 200, 256), (1000, 520, 384)])
def test_tc_update_fp8_matches_reference(m, n, k):
    """E4M3 operands with per-row power-of-two scales: the kernel's result
    equals c - (inv_sa a)(inv_sb b)^T of the same E4M3 values up to FP32
    accumulation rounding."""
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(7)
    a32 = torch.randn(m, k, device="cuda", generator=g) * torch.logspace(-3, 3, m, device="cuda")[:, None]
    b32 = torch.randn(n, k, device="cuda", generator=g)
    c = torch.randn(m, n, device="cuda", generator=g)
    c0 = c.clone()
    sa, ia = pow2_row_scales(a32)
    sb, ib = pow2_row_scales(b32)
    a8 = (a32 * sa[:, None]).to(torch.float8_e4m3fn)
    b8 = (b32 * sb[:, None]).to(torch.float8_e4m3fn)
    ws = torch.empty(lib.b200la_tc_update_workspace_size(), dtype=torch.uint8, device="cuda")
    st = lib.b200la_sgemm_tc_update_fp8(c.data_ptr(), n, m, n, k, a8.data_ptr(), b8.data_ptr(),
                                        ia.contiguous().data_ptr(), ib.contiguous().data_ptr(),
                                        ws.data_ptr(), ws.numel(), torch.cuda.current_stream().cuda_stream)
    _lib.check(st)
    torch.cuda.synchronize()
    ad = a8.double() * ia.double()[:, None]
    bd = b8.double() * ib.double()[:, None]
    ref = c0.double() - ad @ bd.T
    scale = (ad.abs() @ bd.abs().T) + c0.double().abs()
    rel = ((c.double() - ref).abs() / scale.clamp_min(1e-300)).max().item()
    assert rel <= 4 * k * 2.0 ** -24, rel


def test_tc_update_fp8_rejects_missing_scales():
    lib = _lib.load()
    p = torch.empty(4096, device="cuda")
    ws = torch.empty(256, dtype=torch.uint8, device="cuda")
    st = lib.b200la_sgemm_tc_update_fp8(p.data_ptr(), 8, 8, 8, 128, p.data_ptr(), p.data_ptr(), None,
                                        p.data_ptr(), ws.data_ptr(), 256, None)
    assert st == _lib.INVALID_ARGUMENT


@pytest.mark.parametrize("kind,split3", [(TF32, True), (BF16, False)])
@pytest.mark.parametrize("ctas", ["3", "148"])
def test_tc_update_persistent_walks_many_tiles(monkeypatch, kind, split3, ctas):
    """The persistent kernel with 3 CTAs (each walks ~30 tiles through both
    accumulators and the stage ring) and with a full grid over 4 x 12 tile
    rows: same result as the reference."""
    monkeypatch.setenv("B200LA_TC_CTAS", ctas)
    err, tol = run(kind, split3, 1500, 1800, 256, seed=5)
    assert err <= tol, (err, tol)


def test_tc_update_per_tile_kernel_still_matches(monkeypatch):
    monkeypatch.setenv("B200LA_TC_PERSISTENT", "0")
    err, tol = run(TF32, True, 1000, 520, 128)
    assert err <= tol, (err, tol)
