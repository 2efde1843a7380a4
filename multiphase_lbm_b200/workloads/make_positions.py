"""Write the sphere packing of the 200^3 drainage benchmark as a positions
file in the reference's format (one value per line: x, y, z, r of each
sphere, read by the reference's read_positions, src/multiphase_lbm.cu:
1106-1126, and by mlbm_read_positions).

The packing: spheres of radius U[5, 15] at uniform random centres in the
200^3 box (overlap allowed), added until the porosity is at most 0.50, from
libmlbm's seeded generator (seed 2024).  Values are written with 9
significant digits, so reading them back as double and rounding to float
gives the generator's float values exactly, and the voxelised mask is the
generator's, bit for bit.

    python -m multiphase_lbm_b200.workloads.make_positions
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SHAPE = (200, 200, 200)
SEED = 2024
PATH = os.path.join(HERE, "drainage_200_seed2024.positions")


def main() -> int:
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from multiphase_lbm_b200 import host
    fluid, spheres = host.generate_packing(SHAPE, 5.0, 15.0, 0.50, SEED)
    host.write_positions(PATH, spheres)
    back, _, n = host.read_positions(PATH, SHAPE)
    assert n == len(spheres) and (back == fluid).all()
    print(f"{PATH}: {n} spheres, porosity {fluid.mean():.5f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
