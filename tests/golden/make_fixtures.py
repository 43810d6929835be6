"""Generates the committed golden fixtures from the STIR source tree.

  rptsens_seg3_pm.npz : STIR's recon_test_pack/RPTsens_seg3_PM.v, the sensitivity image that
                        recon_test_pack/run_tests.sh compares OSMAPOSL_test_PM_for_sensitivity.par
                        against (ray-tracing matrix, 2 tangential rays, zoom 0.7, 60x60x31).
  scatter_cylinder.npz: STIR's recon_test_pack/scatter_cylinder.hs (the Interfile header text) and the bytes
                        of its data file scatter_cylinder.s, for the Interfile header and stream reader tests.

Run in a tree where STIR is available:  python tests/golden/make_fixtures.py [STIR_ROOT]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(stir_root="/root/reference"):
    src = os.path.join(stir_root, "recon_test_pack", "RPTsens_seg3_PM.v")
    img = np.fromfile(src, "<f4").reshape(31, 60, 60)  # header RPTsens_seg3_PM.hv: x,y 60, z 31, little endian
    np.savez_compressed(os.path.join(HERE, "rptsens_seg3_pm.npz"), image=img)
    print("wrote", os.path.join(HERE, "rptsens_seg3_pm.npz"), img.shape, float(img.sum()))
    pack = os.path.join(stir_root, "recon_test_pack")
    header = open(os.path.join(pack, "scatter_cylinder.hs"), "rb").read()
    data = np.fromfile(os.path.join(pack, "scatter_cylinder.s"), np.uint8)
    out = os.path.join(HERE, "scatter_cylinder.npz")
    np.savez_compressed(out, header=np.frombuffer(header, np.uint8), data=data)
    print("wrote", out, len(header), data.size)


if __name__ == "__main__":
    main(*sys.argv[1:])
