"""transpose on the GPU: pure data movement, so every result is compared bit
for bit with the oracle (numpy's transpose of the same array) and, at the
full order, through size-independent properties (twice is the identity;
sampled entries)."""
import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200 import api

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 2), (63, 63), (64, 64), (65, 65), (127, 127), (129, 129), (1000, 1000), (4097, 4097),
          (1, 9), (7, 1), (100, 300), (300, 100), (1000, 1500), (4097, 63), (64, 4160)]
TYPES = [np.float64, np.float32]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("dt", TYPES)
def test_transpose_in_place_bitwise(port, shape, dt):
    a = np.random.default_rng(shape[0] * 7 + shape[1]).standard_normal(shape).astype(dt)
    m = dev(a)
    t = la.transpose_in_place(m)
    torch.cuda.synchronize()
    assert t.shape == (shape[1], shape[0])
    assert np.array_equal(t.cpu().numpy(), port.transpose(a))


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("dt", TYPES)
def test_transpose_out_bitwise(shape, dt):
    a = np.random.default_rng(shape[1] * 5 + shape[0]).standard_normal(shape).astype(dt)
    src = dev(a)
    dst = la.transpose_out(src)
    torch.cuda.synchronize()
    assert np.array_equal(dst.cpu().numpy(), a.T)
    assert np.array_equal(src.cpu().numpy(), a), "the source is left alone"


def test_transpose_special_values_move_unchanged():
    a = np.array([[np.nan, -0.0, np.inf], [5e-324, -np.inf, 1.0]], dtype=np.float64)
    m = dev(a)
    t = la.transpose_in_place(m).cpu().numpy()
    assert t.tobytes() == np.ascontiguousarray(a.T).tobytes()


@pytest.mark.parametrize("shape", [(16384, 16384), (8192, 24576)])
def test_transpose_full_size_properties(shape):
    rows, cols = shape
    g = torch.Generator(device="cuda").manual_seed(rows + cols)
    a = torch.randn(rows, cols, dtype=torch.float64, device="cuda", generator=g)
    m = a.clone()
    t = la.transpose_in_place(m)
    idx_r = torch.randint(0, rows, (100000,), device="cuda", generator=g)
    idx_c = torch.randint(0, cols, (100000,), device="cuda", generator=g)
    assert torch.equal(t[idx_c, idx_r], a[idx_r, idx_c])
    back = la.transpose_in_place(t)
    assert torch.equal(back, a)


def test_transpose_api_and_errors():
    m = dev(np.arange(12, dtype=np.float64).reshape(3, 4))
    nbytes = api.transpose.workspace_size(3, 4)
    ws = api.workspace(nbytes, m.device)
    api.transpose.apply(3, 4, m, ws, ws.numel())
    torch.cuda.synchronize()
    assert np.array_equal(m.view(4, 3).cpu().numpy(), np.arange(12.0).reshape(3, 4).T)
    with pytest.raises(la.B200InvalidArgument):
        api.transpose.apply(3, 4, m, None, 0)
    with pytest.raises(la.B200InvalidArgument):
        api.transpose.apply(0, 4, m)
