"""Runs a few steps of one case through the library that CC_LIBRARY names and
saves the states, the residual and the status word (run as a subprocess by
tests/test_bounds_build.py, so that the bounds-checked build and the normal
build each load into a process of their own).

  python bounds_runner.py <case> <variant> <precision> <scheme> <out.npz>
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import combustioncodegpu_b200 as cc  # noqa: E402
from combustioncodegpu_b200 import cases  # noqa: E402


def make_case(name):
    sp = cases.synthetic_species()
    return {
        "box": lambda: cases.case_box(12, species=sp, seed=3),
        "channel": lambda: cases.case_channel((11, 8, 6), species=sp),
        "multiblock": lambda: cases.case_multiblock(([6, 7], [6, 5], [5]), species=sp),
        "sod": lambda: cases.case_sod(40, 6, 6),
        "mixing": lambda: cases.case_mixing_layer(40, 24, 4, h=4e-3 / 39, delta=4e-4, species=sp),
    }[name]()


def main():
    name, variant, precision, scheme, out = sys.argv[1:6]
    case = make_case(name)
    d = cc.Driver.from_case(case, precision)
    d.set_tuning(variant, 3)
    d.initialize_computation()
    d.simulate(2, scheme, residual=True)
    states = {"b%d" % b: d.field[b].get_state()[2] for b in range(len(case["blocks"]))}
    res, status = d.residual(), d.status()
    d.close()
    np.savez(out, res=res, status=status, lib=os.path.basename(cc.LIB_PATH), **states)


if __name__ == "__main__":
    main()
