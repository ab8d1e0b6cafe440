"""Device-side initial states equal the host-built ones bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

wb = pytest.importorskip("wake_b200")
import oracle  # noqa: E402
from wake_b200 import workloads as W  # noqa: E402


def _f0(g):
    return g.f_src_data().copy()


@pytest.mark.parametrize("q,dims", [(9, (70, 33, 1)), (19, (20, 12, 10)), (27, (12, 10, 8))])
def test_noise_init_equals_host_fields(q, dims):
    nx, ny, nz = dims
    cls = {9: wb.LatticeGrid2D, 19: wb.LatticeGrid3D, 27: wb.LatticeGrid3DQ27}[q]
    args = (nx, ny) if q == 9 else (nx, ny, nz)
    case = W.Case(q=q, nx=nx, ny=ny, nz=nz, types=np.zeros(nx * ny * nz, np.uint8),
                  init=("noise", 1.0, (0.05, -0.01, 0.02 if q != 9 else 0.0), 3e-3, 20261203 + 7, 11), tau=0.6,
                  collision=wb.TRT)
    a, b = cls(*args, 0.6), cls(*args, 0.6)
    wb.check(wb.lib.wake_grid_initialize_noise(a.handle, 1.0, *case.init[2], case.init[3], case.init[4], case.init[5]))
    b.initialize_fields(case.rho, case.ux, case.uy, case.uz if q != 9 else None)
    fa, fb = _f0(a), _f0(b)
    assert np.array_equal(fa, fb)
    ref = oracle.equilibrium(q, case.rho, case.ux, case.uy, case.uz if q != 9 else None, prec=32).astype(np.float32)
    assert np.array_equal(fa.reshape(q, -1), ref.reshape(q, -1))


def test_uniform_init_equals_oracle_equilibrium():
    g = wb.LatticeGrid3D(16, 8, 8, 0.6)
    g.initialize(1.01, 0.04, -0.02, 0.01)
    n = 16 * 8 * 8
    ref = oracle.equilibrium(19, np.full(n, 1.01, np.float32), np.full(n, 0.04, np.float32),
                             np.full(n, -0.02, np.float32), np.full(n, 0.01, np.float32), prec=32).astype(np.float32)
    assert np.array_equal(_f0(g).reshape(19, -1), ref.reshape(19, -1))
