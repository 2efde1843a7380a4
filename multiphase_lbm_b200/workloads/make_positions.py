"""Write the sphere packings of the benchmark workloads as positions files
in the reference's format (one value per line: x, y, z, r of each sphere,
read by the reference's read_positions, src/multiphase_lbm.cu:1106-1126,
and by mlbm_read_positions):

  * the 200^3 drainage case: spheres of radius U[5, 15] at uniform random
    centres in the 200^3 box (overlap allowed), added until the porosity is
    at most 0.50 (seed 2024);
  * the 64^3 periodic case: radius U[2.5, 7.5], porosity at most 0.50
    (seed 64).

Both from libmlbm's seeded generator.  Values are written with 9
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
SHAPE_64 = (64, 64, 64)
SEED_64 = 64
PATH_64 = os.path.join(HERE, "periodic_64_seed64.positions")
# (shape, radius range, seed, file)
CASES = [(SHAPE, (5.0, 15.0), SEED, PATH),
         (SHAPE_64, (2.5, 7.5), SEED_64, PATH_64)]


def main() -> int:
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from multiphase_lbm_b200 import host
    for shape, (rmin, rmax), seed, path in CASES:
        fluid, spheres = host.generate_packing(shape, rmin, rmax, 0.50, seed)
        host.write_positions(path, spheres)
        back, _, n = host.read_positions(path, shape)
        assert n == len(spheres) and (back == fluid).all()
        print(f"{path}: {n} spheres, porosity {fluid.mean():.5f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
