"""Write the small xyz fixtures the legacy-interface tests load
(tests/golden/mol24.xyz, tests/golden/NaCl_2x2_L2.xyz), from this package's
seeded generator.  Run from the repository root:  python tests/golden/make_xyz.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from firecore_b200 import systems as S  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
SYM = {0: "H", 1: "C", 2: "N", 3: "O"}


def main():
    b = S.make_systems([24], seed=7, topo_mode=0, sigma=0.0, rotate=False, cell=(11.28, 11.28, 40.0))
    n = int(b.natoms[0])
    q = b.REQs[:n, 2]
    with open(os.path.join(HERE, "mol24.xyz"), "w") as f:
        f.write(f"{n}\nseeded 24-atom molecule (C:N:O:H 10:2:2:10)\n")
        for i in range(n):
            x, y, z = b.pos[i]
            f.write(f"{SYM[int(b.elements[i])]} {x:.6f} {y:.6f} {z:.6f} {q[i]:.6f}\n")
    sub = S.make_slab(ncell=2, layers=2, grid_step=0.2, nz=100)
    L = sub.lvec
    with open(os.path.join(HERE, "NaCl_2x2_L2.xyz"), "w") as f:
        f.write(f"{len(sub.spos)}\nlvs {L[0,0]:.4f} 0 0  0 {L[1,1]:.4f} 0  0 0 {L[2,2]:.4f}\n")
        for p, r in zip(sub.spos, sub.sREQ):
            f.write(f"{'Na' if r[2] > 0 else 'Cl'} {p[0]:.6f} {p[1]:.6f} {p[2]:.6f} {r[2]:.4f}\n")


if __name__ == "__main__":
    main()
