"""Extract the reference's own particle-interpolation known answers.

The reference's ``dertest`` harness (dertest/part_tools.F90:580-582) replaces
the sampled field with u_theta = 0, u_r = r**2, u_z = 1 on the VR2D mesh
(dertest/VR2D/inp.txt: ntheta x nr x nz = 1 x 256 x 512, maxr 1.5, maxz 3.0)
and dumps, per particle visit, the position and the interpolated Cartesian
velocity (fort.300x), its gradient (fort.310x, dvel(i,j) with j fastest) and
the three Hessian slices (fort.321x/322x/323x, ddvel(i,j,l) with l fastest),
x = MPI rank.  This script samples every 25th line of the rank 0, 1 and 3
dumps into dertest_kat.npz.  It reads the reference tree, whose root is its one
required argument, and is run once; the tests only read the .npz it writes.

    python tests/golden/make_golden.py <reference root>
"""
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <reference root>")
REF = sys.argv[1]
SRC = os.path.join(REF, "dertest", "VR2D")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dertest_kat.npz")

pos, vel, dvel, dd1, dd2, dd3 = [], [], [], [], [], []
for rank in (0, 1, 3):
    a = np.loadtxt(os.path.join(SRC, "fort.%d" % (3000 + rank)))
    b = np.loadtxt(os.path.join(SRC, "fort.%d" % (3100 + rank)))
    c1 = np.loadtxt(os.path.join(SRC, "fort.%d" % (3210 + rank)))
    c2 = np.loadtxt(os.path.join(SRC, "fort.%d" % (3220 + rank)))
    c3 = np.loadtxt(os.path.join(SRC, "fort.%d" % (3230 + rank)))
    sel = slice(0, None, 25)
    assert np.array_equal(a[:, :3], b[:, :3]) and np.array_equal(a[:, :3], c3[:, :3])
    pos.append(a[sel, :3])
    vel.append(a[sel, 3:6])
    dvel.append(b[sel, 3:12])
    dd1.append(c1[sel, 3:12])
    dd2.append(c2[sel, 3:12])
    dd3.append(c3[sel, 3:12])
np.savez_compressed(OUT, pos=np.concatenate(pos), vel=np.concatenate(vel),
                    dvel=np.concatenate(dvel), ddvel1=np.concatenate(dd1),
                    ddvel2=np.concatenate(dd2), ddvel3=np.concatenate(dd3),
                    mesh=np.array([1, 256, 512, 1.5, 3.0]))
print("wrote", OUT, sum(len(p) for p in pos), "points")
