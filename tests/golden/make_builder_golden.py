"""Golden fixtures for the topology builder, from FireCore's own builder.

Run where the reference tree is present (builds oracle/_ref/libref_harness.so
from the reference sources with oracle/Makefile):

    python tests/golden/make_builder_golden.py

For each listed molecule of FireCore's cpp/common_resources/xyz and both
electron-pair settings it runs the reference's MolWorld_sp3::initParams ->
buildMolecule_xyz -> makeFFs on FireCore's own tables (harness function
ref_build_xyz) in a child process -- FireCore exits the process on molecules it
rejects -- and stores the MMFFsp3_loc arrays it produced in
tests/golden/builder_golden.npz.  Molecules the reference rejects are stored
with natoms = -1.
"""
import ctypes
import os
import pickle
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "builder_golden.npz")
REF_ROOT = os.environ.get("REF_ROOT", "/root/reference")
RES = os.path.join(REF_ROOT, "cpp", "common_resources")
TABLES = ("ElementTypes.dat", "AtomTypes.dat", "BondTypes.dat", "AngleTypes.dat", "DihedralTypes.dat")

# small to large, open and periodic ("lvs" cell; polymers bond across it),
# sp / sp2 / sp3 centres, carbonyl / carboxyl / amide / aromatic-N special types
MOLECULES = ["H2O.xyz", "NH3.xyz", "CH2O.xyz", "C2H4.xyz", "CH2NH.xyz", "HCOOH.xyz", "HCONH2.xyz", "HF.xyz",
             "HCl.xyz", "CO.xyz", "O2.xyz", "HCN.xyz", "formic_dimer.xyz", "oxalate.xyz", "pyridine.xyz",
             "adenine.xyz", "guanine.xyz", "citosine.xyz", "thymine.xyz", "uracil.xyz", "xylitol.xyz",
             "deoxyribose.xyz", "butandiol.xyz", "nHexadecan.xyz", "pentacene.xyz", "PTCDA.xyz",
             "polydiacetylene.xyz", "polydiacetylene_OH.xyz", "polymer-2.xyz", "BPBA.xyz", "Si10_H.xyz",
             "backbone_pasivated-R.xyz", "EndGroup_X_1.xyz", "hexan-dicarboxylic.xyz", "N_2edge_assay_1.xyz",
             "H_xline.xyz", "polymer-2_new-COOH.xyz"]
NPBC = (1, 1, 0)


def _ref_child(xyz, epairs, out):
    from oracle import oracle as O
    lib = ctypes.CDLL(O.REF_LIB)
    cap = 1024
    cnt = np.zeros(4, np.int32)
    apos = np.zeros((2 * cap, 3)); REQ = np.zeros((cap, 4)); at = np.zeros(cap, np.int32)
    ng = np.zeros((cap, 4), np.int32); nc = np.zeros((cap, 4), np.int32)
    par = [np.zeros((cap, 4)) for _ in range(5)]
    names = ctypes.create_string_buffer(8 * cap)
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    npbc = np.array(NPBC, np.int32)                 # held for the duration of the call
    n = lib.ref_build_xyz(*(os.path.join(RES, t).encode() for t in TABLES), xyz.encode(), ctypes.c_int(epairs),
                          P(npbc), ctypes.c_int(cap), P(cnt), P(apos), P(REQ), P(at), P(ng), P(nc),
                          *[P(a) for a in par], names)
    na, nn = int(cnt[0]), int(cnt[1])
    d = dict(natoms=na, nnode=nn, pbc=int(cnt[3]), apos=apos[:na + nn], REQs=REQ[:na], neighs=ng[:na],
             neighCell=nc[:na], apars=par[0][:nn], bLs=par[1][:nn], bKs=par[2][:nn], Ksp=par[3][:nn], Kpp=par[4][:nn],
             type_names=np.array([names.raw[8 * i:8 * i + 8].split(b"\0")[0].decode() for i in range(na)]))
    if n < 0:
        d = dict(natoms=-1)
    with open(out, "wb") as f:
        pickle.dump(d, f)


def main():
    if len(sys.argv) == 5 and sys.argv[1] == "child":
        _ref_child(sys.argv[2], int(sys.argv[3]), sys.argv[4])
        return
    from oracle import oracle as O
    O.build_oracle(with_ref=True)
    out = {}
    tmp = os.path.join(ROOT, "_build", "builder_golden_child.pkl")
    os.makedirs(os.path.dirname(tmp), exist_ok=True)
    for m in MOLECULES:
        for ep in (0, 1):
            if os.path.exists(tmp):
                os.remove(tmp)
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "child", os.path.join(RES, "xyz", m), str(ep), tmp],
                               capture_output=True, text=True, timeout=300)
            d = pickle.load(open(tmp, "rb")) if os.path.exists(tmp) else dict(natoms=-1)
            key = f"{m}|{ep}"
            for k, v in d.items():
                out[f"{key}|{k}"] = np.asarray(v)
            print(f"{key:40s} natoms={d['natoms']} (child rc={r.returncode})")
    np.savez_compressed(OUT, molecules=np.array(MOLECULES), nPBC=np.array(NPBC), **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
