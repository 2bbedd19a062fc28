"""Small parameter tables in FireCore's .dat formats (this project's own
numbers), for tests that must run without the FireCore tree: the builder's
table reader and typing rules, and the legacy init's table lookup on the GPU.

Every atom type the typing rules name (MM::Builder::assignSpecialTypes) is
present.  Columns as FireCore's readers expect them:
  ElementTypes: name iZ neval valence piMax color Rcov RvdW EvdW Quff Uuff Vuff
  AtomTypes:    name parent element epair valence nepair npi sym Ruff RvdW EvdW Qbase Hb
                [Ass Asp Kss Ksp Kep Kpp]
  BondTypes:    type type order l0 k
  AngleTypes:   type type type ang0 k
"""
import os

ELEMENTS = """# name iZ ne nv npi color Rcov RvdW EvdW Quff Uuff Vuff
E   200 0 0 0 0x00FFFF 0.50 0.50 0.0010 0.0 0.0 0.0
H     1 1 1 0 0xFFFFFF 0.33 1.45 0.0020 0.7 0.0 0.0
C     6 4 4 2 0x909090 0.75 1.90 0.0045 1.9 0.0 0.0
N     7 5 3 2 0x3050F8 0.71 1.83 0.0030 2.5 0.0 0.0
O     8 6 2 1 0xFF0D0D 0.66 1.75 0.0026 2.3 0.0 0.0
"""

_T = [
    # name   parent elem epair nv ne npi sym  Ruff  RvdW  EvdW    Qbase Hb     Ass    Asp    Kss  Ksp  Kep  Kpp
    ("*",     "*",   "H", "E", 1, 0, 0, 0, 0.00, 0.00, 0.0007, 0.0, 0.0),
    ("E",     "*",   "E", "*", 0, 0, 0, 0, 0.50, 0.40, 0.0000, -0.4, 0.0),
    ("H",     "*",   "H", "E", 1, 0, 0, 0, 0.35, 1.45, 0.0020, 0.0, 0.0),
    ("C",     "*",   "C", "E", 4, 0, 0, 0, 0.76, 1.90, 0.0045, 0.0, 0.0, 109.5, -19.5, 6.0, 0.0, 0.0, 0.0),
    ("N",     "*",   "N", "E", 3, 1, 0, 0, 0.70, 1.83, 0.0030, 0.0, 0.0, 109.5, -19.5, 5.5, 1.0, 0.0, 0.5),
    ("O",     "*",   "O", "E", 2, 2, 0, 0, 0.66, 1.75, 0.0026, 0.0, 0.0, 109.5, -19.5, 6.0, 1.0, 0.0, 0.5),
    ("C_3",   "C",   "C", "E", 4, 0, 0, 0, 0.76, 1.92, 0.0046, 0.0, 0.0, 109.5, -19.5, 6.3, 1.5, 1.0, 0.0),
    ("C_R",   "C",   "C", "E", 4, 0, 0, 0, 0.73, 1.92, 0.0046, 0.0, 0.0, 120.0, 0.0, 6.3, 1.5, 1.0, 1.2),
    ("C_2",   "C",   "C", "E", 4, 0, 0, 0, 0.73, 1.92, 0.0046, 0.0, 0.0, 120.0, 0.0, 4.2, 1.5, 1.0, 1.9),
    ("C_1",   "C",   "C", "E", 4, 0, 0, 0, 0.70, 1.92, 0.0046, 0.0, 0.0, 180.0, 0.0, 3.9, 1.5, 1.0, 0.0),
    ("N_3",   "N",   "N", "E", 3, 1, 0, 0, 0.70, 1.83, 0.0030, 0.0, -0.9, 107.0, -22.0, 5.6, 1.5, 1.0, 0.4),
    ("N_R",   "N",   "N", "E", 3, 1, 0, 0, 0.70, 1.83, 0.0030, 0.0, 0.9, 120.0, 0.0, 7.4, 1.5, 1.0, 1.2),
    ("N_2",   "N",   "N", "E", 3, 1, 0, 0, 0.68, 1.83, 0.0030, 0.0, -0.9, 111.0, 0.0, 7.4, 1.5, 1.0, 0.9),
    ("N_1",   "N",   "N", "E", 3, 1, 0, 0, 0.66, 1.83, 0.0030, 0.0, 0.0, 180.0, 0.0, 4.8, 1.5, 1.0, 0.0),
    ("O_3",   "O",   "O", "E", 2, 2, 0, 0, 0.66, 1.75, 0.0026, 0.0, -0.9, 104.5, -37.7, 6.0, 1.5, 1.0, 0.4),
    ("O_R",   "O",   "O", "E", 2, 2, 0, 0, 0.68, 1.75, 0.0026, 0.0, -0.9, 110.0, 0.0, 8.0, 1.5, 1.0, 0.9),
    ("O_2",   "O",   "O", "E", 2, 2, 0, 0, 0.63, 1.75, 0.0026, 0.0, -0.9, 120.0, 0.0, 8.0, 1.5, 1.0, 0.0),
    ("O_1",   "O",   "O", "E", 2, 2, 0, 0, 0.64, 1.75, 0.0026, 0.0, 0.0, 180.0, 0.0, 8.0, 1.5, 1.0, 0.0),
    ("C_CH3", "C_3", "C", "E", 4, 0, 0, 0, 0.76, 1.91, 0.0037, 0.0, 0.0, 109.5, -19.5, 6.3, 1.0, 0.0, 0.0),
    ("C_ene", "C_2", "C", "E", 4, 0, 0, 0, 0.76, 1.91, 0.0037, 0.0, 0.0, 120.0, 0.0, 5.9, 2.0, 1.0, 1.0),
    ("C_yne", "C_1", "C", "E", 4, 0, 0, 0, 0.76, 1.91, 0.0037, 0.0, 0.0, 180.0, 0.0, 3.9, 0.0, 0.0, 0.0),
    ("C_ald", "C_2", "C", "E", 4, 0, 0, 0, 0.76, 1.91, 0.0037, 0.0, 0.0, 120.0, 0.0, 5.9, 2.0, 1.0, 1.0),
    ("C_COO", "C_2", "C", "E", 4, 0, 0, 0, 0.76, 1.91, 0.0037, 0.0, 0.0, 120.0, 0.0, 5.9, 2.0, 1.0, 1.0),
    ("O_OH",  "O_3", "O", "E", 2, 2, 0, 0, 0.66, 1.66, 0.0091, 0.0, 0.0, 109.5, -19.5, 6.0, 1.0, 0.0, 0.5),
    ("O_ald", "O_2", "O", "E", 2, 2, 0, 0, 0.66, 1.66, 0.0091, 0.0, 0.0, 120.0, 0.5, 8.0, 2.0, 0.0, 1.0),
    ("O_sCOO", "O_3", "O", "E", 2, 2, 0, 0, 0.66, 1.66, 0.0091, 0.0, 0.0, 109.5, -19.5, 6.0, 1.0, 0.0, 0.5),
    ("O_pCOO", "O_2", "O", "E", 2, 2, 0, 0, 0.66, 1.66, 0.0091, 0.0, 0.0, 120.0, 0.0, 8.0, 2.0, 0.0, 1.0),
    ("H_OH",  "H",   "H", "E", 1, 0, 0, 0, 0.35, 1.49, 0.0007, 0.0, 0.9),
    ("H_NH2", "H",   "H", "E", 1, 0, 0, 0, 0.35, 1.49, 0.0007, 0.0, 0.9),
    ("H_CH3", "H",   "H", "E", 1, 0, 0, 0, 0.35, 1.49, 0.0007, 0.0, 0.9),
    ("H_ene", "H",   "H", "E", 1, 0, 0, 0, 0.35, 1.49, 0.0007, 0.0, 0.9),
    ("H_yne", "H",   "H", "E", 1, 0, 0, 0, 0.35, 1.49, 0.0007, 0.0, 0.9),
    ("H_ald", "H",   "H", "E", 1, 0, 0, 0, 0.35, 1.49, 0.0007, 0.0, 0.9),
    ("H_COO", "H",   "H", "E", 1, 0, 0, 0, 0.35, 1.49, 0.0007, 0.0, 0.9),
]

BONDS = """# type type order l0 k
H C 1 1.09 16.0
H N 1 1.02 22.0
H O 1 0.97 24.0
C C 1 1.54 10.0
C C 2 1.33 21.0
C C 3 1.20 36.0
C N 1 1.47 11.0
C N 2 1.28 22.0
C O 1 1.42 12.5
C O 2 1.22 27.5
N O 1 1.41 7.6
E C 1 0.50 10.0
E N 1 0.50 10.0
E O 1 0.50 10.0
"""

ANGLES = """# a b c ang0 k
*  C  *  109.5 5.1
*  N  *  107.0 5.2
*  O  *  104.5 5.3
H  C_R H 120.0 5.4
"""


def atom_types():
    lines = ["# name parent element epair nv ne npi sym Ruff RvdW EvdW Qbase Hb Ass Asp Kss Ksp Kep Kpp"]
    for r in _T:
        lines.append(" ".join(str(x) for x in r))
    return "\n".join(lines) + "\n"


def write_tables(directory):
    """Write the four tables into ``directory``; returns their paths in the
    order mmff_build_xyz / init take them."""
    os.makedirs(directory, exist_ok=True)
    files = {"ElementTypes.dat": ELEMENTS, "AtomTypes.dat": atom_types(), "BondTypes.dat": BONDS, "AngleTypes.dat": ANGLES}
    for name, text in files.items():
        with open(os.path.join(directory, name), "w") as f:
            f.write(text)
    return tuple(os.path.join(directory, n) for n in ("ElementTypes.dat", "AtomTypes.dat", "BondTypes.dat", "AngleTypes.dat"))


def type_row(name):
    for r in _T:
        if r[0] == name:
            return r
    raise KeyError(name)


# formaldehyde and methanol, charges in the fifth column
FORMALDEHYDE = """4
formaldehyde
C  0.000  0.000  0.000  0.2
O  1.215  0.000  0.000 -0.4
H -0.560  0.935  0.000  0.1
H -0.560 -0.935  0.000  0.1
"""
METHANOL = """6
methanol
C  0.000  0.000  0.000
O  1.420  0.000  0.000 -0.6
H  1.740  0.910  0.000  0.4
H -0.360  1.030  0.000
H -0.360 -0.515  0.890
H -0.360 -0.515 -0.890  0.2
"""


def polyethylene(ncell=4, noise=0.0, seed=0):
    """xyz text of an infinite zigzag C chain along x, 4 CH2 units per cell (the
    chain bonds across the cell wall), in an "lvs" cell of 5.08 x 8 x 20 A."""
    import numpy as np
    rng = np.random.default_rng(seed)
    lines = []
    for i in range(ncell):
        x, z = 1.27 * i, 10.0 + (0.42 if i % 2 else 0.0)
        lines.append(("C", x, 0.0, z, -0.1))
        s = 1.0 if i % 2 else -1.0
        lines.append(("H", x, 0.89, z + 0.52 * s, 0.05))
        lines.append(("H", x, -0.89, z + 0.52 * s, 0.05))
    out = [str(len(lines)), f"lvs {1.27 * ncell:.4f} 0 0   0 8 0   0 0 20"]
    for e, x, y, z, q in lines:
        d = rng.normal(0, noise, 3) if noise > 0 else np.zeros(3)
        out.append(f"{e} {x + d[0]:.6f} {y + d[1]:.6f} {z + d[2]:.6f} {q}")
    return "\n".join(out) + "\n"
