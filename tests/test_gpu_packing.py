"""The GPU packing generator (mlbm_generate_packing_gpu) against the host
generator: the same spheres, count, porosity and solid mask, bit for bit,
for cubic and non-cubic boxes, spheres larger than the box (repeated
periodic wrap), porosity targets met after one chunk of candidates or
several, the sphere cap, and a target met before any sphere."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [((64, 64, 64), 2.5, 7.5, 0.5, 1),
         ((48, 80, 32), 2.0, 6.0, 0.35, 2),
         ((33, 17, 9), 5.0, 12.0, 0.5, 3),       # spheres larger than the box
         ((128, 96, 80), 3.0, 9.0, 0.65, 4),
         ((200, 200, 200), 5.0, 15.0, 0.5, 2024),  # the benchmark packing
         ((40, 40, 40), 2.5, 7.5, 0.2, 5)]       # several chunks


@pytest.mark.parametrize("shape,rmin,rmax,por,seed", CASES)
def test_gpu_packing_equals_host(shape, rmin, rmax, por, seed):
    from multiphase_lbm_b200 import host
    f_h, s_h = host.generate_packing(shape, rmin, rmax, por, seed)
    f_g, s_g = host.generate_packing(shape, rmin, rmax, por, seed, device=0)
    assert np.array_equal(s_h, s_g)
    assert np.array_equal(f_h, f_g)


def test_gpu_packing_edges():
    from multiphase_lbm_b200 import host
    shape = (32, 32, 32)
    for kw in (dict(max_spheres=3), dict(max_spheres=0)):
        a = host.generate_packing(shape, 3.0, 6.0, 0.4, 9, **kw)
        b = host.generate_packing(shape, 3.0, 6.0, 0.4, 9, device=0, **kw)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    f, s = host.generate_packing(shape, 3.0, 6.0, 1.0, 9, device=0)
    assert len(s) == 0 and f.all()
