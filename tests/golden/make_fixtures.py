"""Regenerate the golden fixtures from the reference's own test outputs.

Reads the IDL ascii golden files of the reference (Param/*/TestOutput) and
stores the columns the hot path produces as compact .npz fixtures, so that
the tests never read the reference tree at run time.

    python tests/golden/make_fixtures.py <BATS-R-US source tree>
    (or with the tree in the environment variable BATSRUS_REFERENCE)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from batsrus_b200.idl import read_idl_ascii  # noqa: E402

VARS = ["Rho", "Ux", "Uy", "Uz", "Bx", "By", "Bz", "P"]


def main(ref):
    src = os.path.join(ref, "Param/SHOCKTUBE/TestOutput/mhdhyp_1d_ref.out")
    d = read_idl_ascii(src)
    cols = [d["varnames"].index(v) for v in VARS]
    np.savez_compressed(os.path.join(HERE, "mhdhyp_1d_ref.npz"),
                        x=d["coord"][:, 0], prim=d["var"][:, cols], names=np.array(VARS),
                        nStep=d["nStep"], time=d["time"], gamma=d["params"][0],
                        source="Param/SHOCKTUBE/TestOutput/mhdhyp_1d_ref.out",
                        tolerance_rel=1e-5, tolerance_abs=1e-11)
    print("wrote mhdhyp_1d_ref.npz", d["var"].shape)

    # Param/SHOCKTUBE/PARAM.in.fast_wave (Makefile.test:439-459): the z=0 cut
    # at step 150, t = 75; DiffNum tolerances -r=1e-3 -a=1e-6
    src = os.path.join(ref, "Param/SHOCKTUBE/TestOutput/fast_wave_ref.out")
    d = read_idl_ascii(src)
    cols = [d["varnames"].index(v) for v in VARS]
    np.savez_compressed(os.path.join(HERE, "fast_wave_ref.npz"),
                        xy=d["coord"][:, :2], prim=d["var"][:, cols], names=np.array(VARS),
                        nStep=d["nStep"], time=d["time"], gamma=d["params"][0],
                        source="Param/SHOCKTUBE/TestOutput/fast_wave_ref.out",
                        tolerance_rel=1e-3, tolerance_abs=1e-6)
    print("wrote fast_wave_ref.npz", d["var"].shape)


if __name__ == "__main__":
    # the BATS-R-US source tree: the first argument, else $BATSRUS_REFERENCE
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BATSRUS_REFERENCE")
    if not ref:
        sys.exit("usage: make_fixtures.py <BATS-R-US source tree> (or set BATSRUS_REFERENCE)")
    main(ref)
