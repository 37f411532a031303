"""GPU parity of the axpby body against the oracle (bit-exact: same (a*x)+(b*y) rounding)."""
import numpy as np
import pytest

import kernels_oracle as O
import xkaapi_b200 as xk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,off", [(0, 0), (1, 0), (7, 1), (1000, 3), (1 << 20, 0), ((1 << 20) + 5, 1)])
def test_axpby_bit_exact(torch_cuda, n, off):
    torch = torch_cuda
    rng = np.random.default_rng(n + off)
    x = rng.uniform(-1, 1, n + off + 1)
    y = rng.uniform(-1, 1, n + off + 1)
    a, b = 1.75, -0.625
    ref = y.copy()
    ref[off:off + n] = O.axpby(a, x[off:off + n], b, y[off:off + n])
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    # offset views exercise the scalar head/tail peeling
    xk.axpby(a, dx[off:off + n], b, dy[off:off + n])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dy.cpu().numpy(), ref)


def test_axpby_mismatched_alignment(torch_cuda):
    torch = torch_cuda
    n = 4097
    x = np.linspace(-1, 1, n + 1); y = np.linspace(2, -3, n + 2)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    ref = y.copy(); ref[1:n + 1] = O.axpby(0.5, x[:n], 3.0, y[1:n + 1])
    xk.axpby(0.5, dx[:n], 3.0, dy[1:n + 1])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dy.cpu().numpy(), ref)
