"""Regenerate the golden fixtures from a checkout of the reference tree.

    python tests/golden/make_golden.py <path to the Perrbit/astr_gpu checkout>

state_ref_128.txt: the reference's own committed Taylor-Green history
miniapps/tgv_solver_3d/state.ref_128 (written by tgvsolver.F90:938: nstep, time, tke,
enstrophy at 128^3, dt=1e-3, 100 steps), copied verbatim as data.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    src = os.path.join(sys.argv[1], "miniapps", "tgv_solver_3d", "state.ref_128")
    if not os.path.exists(src):
        sys.exit(f"reference tree not found at {src}")
    shutil.copyfile(src, os.path.join(HERE, "state_ref_128.txt"))
    print("wrote state_ref_128.txt")


if __name__ == "__main__":
    main()
