"""Run the reference program on the bench's 200^3 packing (timing only).

Writes the bench packing (seed 2024, radii U[5, 15], porosity 0.50) as a
positions file and a command file in the reference's format into --out, then
runs one of the programs that oracle/build_ref.py builds:

* ``cuda``  -- oracle/_ref/multiphaselbm_cuda_200x200x200, the reference with
  its own CUDA kernels (sm_100a);
* ``dropin`` -- oracle/_ref/refdriver_b200_200x200x200, the same reference
  host driver stepping through libmlbm.

Only step 0 computes statistics (statPeriod above step_max).  The device
time per step comes from a launch list of this command under ncu (per-kernel
durations), not from the program's own host timer, which stops while
launches are still queued.

    python oracle/time_ref_cuda.py --out gpurun_out/refcase --steps 20 --exe cuda
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
EXES = {"cuda": "multiphaselbm_cuda_200x200x200",
        "dropin": "refdriver_b200_200x200x200"}


def write_case(out: str, steps: int, tag: str) -> str:
    sys.path.insert(0, ROOT)
    from multiphase_lbm_b200 import host
    os.makedirs(out, exist_ok=True)
    pos = os.path.join(out, "positions.txt")
    if not os.path.exists(pos):
        _, spheres = host.generate_packing((200, 200, 200), 5.0, 15.0, 0.50, 2024)
        host.write_positions(pos, spheres)
    text = f"""! 200^3 bench packing, timing case
result_folder {out}/{tag}_{steps}
statPeriod 1000000
lx 200
ly 200
lz 200
rho0 2.0
IniPerturbRate 0.0
G -6.0
rhos 0.182322
tau 1.0
resize
read_positions {pos}
step_max {steps}
"""
    cmd = os.path.join(out, f"{tag}_{steps}.txt")
    with open(cmd, "w") as fh:
        fh.write(text)
    return cmd


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--exe", choices=sorted(EXES), default="cuda")
    args = ap.parse_args(argv)
    exe = os.path.join(HERE, "_ref", EXES[args.exe])
    if not os.path.exists(exe):
        print(f"{exe} not built (python oracle/build_ref.py)")
        return 1
    out = os.path.abspath(args.out)
    cmd = write_case(out, args.steps, args.exe)
    # the reference labels clusters with a recursive search: unlimited stack
    r = subprocess.run(["bash", "-c", f"ulimit -s unlimited && exec {exe} {cmd}"],
                       cwd=out, capture_output=True, text=True)
    lines = [ln for ln in r.stdout.splitlines() if "GPU time" in ln]
    print(lines[-1] if lines else r.stdout[-500:] + r.stderr[-500:])
    return r.returncode


if __name__ == "__main__":
    sys.exit(main())
