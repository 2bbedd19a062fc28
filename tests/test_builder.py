"""The FireCore topology / parameter builder (mmff_build_xyz, host code):
bit-for-bit against FireCore's own builder on FireCore's tables and
molecules (golden fixtures written by tests/golden/make_builder_golden.py
from MolWorld_sp3::initParams -> buildMolecule_xyz -> makeFFs), and against
hand-derived values on this project's own small tables."""
import math
import os

import numpy as np
import pytest

from builder_tables import FORMALDEHYDE, METHANOL, type_row, write_tables

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "builder_golden.npz")
REF_ROOT = os.environ.get("REF_ROOT", "/root/reference")
RES = os.path.join(REF_ROOT, "cpp", "common_resources")
FIELDS = ("apos", "REQs", "neighs", "neighCell", "apars", "bLs", "bKs", "Ksp", "Kpp")

_G = np.load(GOLDEN)
CASES = [(str(m), ep) for m in _G["molecules"] for ep in (0, 1)]
# molecules FireCore's builder itself rejects (an atom without a bond; a
# carbon with five neighbours) -- as opposed to the linear molecules its first
# force evaluation rejects (NaN in the angle term), which only the force field
# of the reference stops on
BUILDER_REJECTS = {"H_xline.xyz", "polymer-2_new-COOH.xyz"}

need_ref = pytest.mark.skipif(not os.path.isfile(os.path.join(RES, "AtomTypes.dat")), reason="FireCore tree not present")


def _build(xyz, tables, ep=False, npbc=(1, 1, 0)):
    from firecore_b200 import topology as T
    return T.build_xyz(xyz, tables, epairs=ep, nPBC=npbc)


@need_ref
@pytest.mark.parametrize("mol,ep", CASES, ids=[f"{m[:-4]}-{'ep' if e else 'noep'}" for m, e in CASES])
def test_builder_matches_firecore(mol, ep):
    from firecore_b200 import topology as T
    key = f"{mol}|{ep}"
    n_ref = int(_G[f"{key}|natoms"])
    tables = T.table_paths(RES)
    xyz = os.path.join(RES, "xyz", mol)
    if n_ref < 0:
        if mol in BUILDER_REJECTS:
            with pytest.raises(RuntimeError):
                _build(xyz, tables, ep, tuple(_G["nPBC"]))
        else:
            pytest.skip("FireCore stops this molecule at its first force evaluation, not in the builder")
        return
    d = _build(xyz, tables, ep, tuple(_G["nPBC"]))
    assert d["natoms"] == n_ref and d["nnode"] == int(_G[f"{key}|nnode"])
    assert int(d["pbc"]) == int(_G[f"{key}|pbc"])
    assert list(d["type_names"]) == [str(s) for s in _G[f"{key}|type_names"]]
    for f in FIELDS:
        ref = _G[f"{key}|{f}"]
        mine = d[f]
        if f == "neighCell" and not d["pbc"]:
            continue
        assert mine.shape == ref.shape, f
        # bit for bit: same inputs, same operation order
        assert np.array_equal(mine, ref), (f, np.abs(mine - ref).max())


def test_own_tables_formaldehyde(tmp_path):
    tables = write_tables(str(tmp_path / "t"))
    xyz = tmp_path / "f.xyz"
    xyz.write_text(FORMALDEHYDE)
    d = _build(str(xyz), tables)
    # C (3 bonds, npi 1) -> C_2 -> C_ald (a C=O neighbour); O (1 bond, 2 pairs, npi 1)
    # -> O_2 -> O_ald; the hydrogens of a C_ald -> H_ald
    assert d["type_names"] == ["C_ald", "O_ald", "H_ald", "H_ald"]
    assert d["natoms"] == 4 and d["nnode"] == 2
    assert d["neighs"][0].tolist() == [1, 2, 3, -1] and d["neighs"][1].tolist() == [0, -1, -1, -1]
    assert d["neighs"][2].tolist() == [0, -1, -1, -1]
    ald = type_row("C_ald")
    a0 = ald[13] * math.pi / 180 / 2
    np.testing.assert_allclose(d["apars"][0], [math.cos(a0), math.sin(a0), 4 * ald[15], math.sin(ald[14] * math.pi / 180)])
    # bond orders from the pi counts, parameters from the input (element) types
    np.testing.assert_allclose(d["bLs"][0], [1.22, 1.09, 1.09, 0])
    np.testing.assert_allclose(d["bKs"][0], [27.5, 16.0, 16.0, 0])
    np.testing.assert_allclose(d["Ksp"][0], [ald[16]] * 3 + [0])
    np.testing.assert_allclose(d["Kpp"][0], [math.sqrt(ald[18] * type_row("O_ald")[18]), 0, 0, 0])
    # non-bonded: the final type's radius and sqrt(depth), the file's charge, Hb = 0
    np.testing.assert_allclose(d["REQs"][1], [type_row("O_ald")[9], math.sqrt(type_row("O_ald")[10]), -0.4, 0])
    # pi axes: normal to the C plane; the O axis from the frame of its one bond,
    # both turned towards (1,1,1) and normalised
    np.testing.assert_allclose(d["apos"][4], [0, 0, 1], atol=1e-15)
    np.testing.assert_allclose(d["apos"][5], [0, 1, 0], atol=1e-15)


def test_own_tables_methanol_and_pairs(tmp_path):
    tables = write_tables(str(tmp_path / "t"))
    xyz = tmp_path / "m.xyz"
    xyz.write_text(METHANOL)
    d = _build(str(xyz), tables)
    assert d["type_names"] == ["C_3", "O_3", "H", "H_CH3", "H_CH3", "H_CH3"]
    np.testing.assert_allclose(d["bLs"][0][:1], [1.42])
    assert d["REQs"][5, 2] == 0.2 and d["REQs"][2, 2] == 0.4
    # with electron pairs: the O (two bonds, two pairs) gets two generated pairs
    # 0.5 A out along its sp3 frame, each carrying -0.2 e taken from the O
    e = _build(str(xyz), tables, ep=True)
    assert e["natoms"] == 8 and e["type_names"][6:] == ["E", "E"]
    o = e["apos"][1]
    for k in (6, 7):
        assert abs(np.linalg.norm(e["apos"][k] - o) - 0.5) < 1e-9   # frame literals carry 11 digits
        assert e["REQs"][k, 2] == pytest.approx(-0.2)
    assert e["REQs"][1, 2] == pytest.approx(-0.6 + 0.4)
    assert e["neighs"][1].tolist()[2:] == [6, 7]
    # formaldehyde: explicit pairs on the terminal O at 120 degrees from the C=O bond
    xf = tmp_path / "f.xyz"
    xf.write_text(FORMALDEHYDE)
    f = _build(str(xf), tables, ep=True)
    assert f["natoms"] == 6 and f["type_names"][4:] == ["E", "E"]
    co = f["apos"][0] - f["apos"][1]
    for k in (4, 5):
        oe = f["apos"][k] - f["apos"][1]
        c = co @ oe / np.linalg.norm(co) / np.linalg.norm(oe)
        assert c == pytest.approx(-0.5, abs=1e-9)


def test_rejections(tmp_path):
    tables = write_tables(str(tmp_path / "t"))
    bad = tmp_path / "b.xyz"
    bad.write_text("2\n\nC 0 0 0\nH 5 0 0\n")
    with pytest.raises(RuntimeError, match="no bond"):
        _build(str(bad), tables)
    with pytest.raises(RuntimeError, match="cannot open"):
        _build(str(bad), (tables[0], str(tmp_path / "missing.dat"), tables[2], tables[3]))
    broken = tmp_path / "t2"
    t2 = write_tables(str(broken))
    with open(t2[1], "a") as f:
        f.write("X_9 Q_7 C E 4 0 0 0 0.7 1.9 0.004 0 0\n")
    with pytest.raises(RuntimeError, match="unknown parent"):
        _build(str(bad), t2)


def test_batch_of_typed_molecule_evaluates_in_the_oracle(tmp_path):
    """The typed molecule feeds the CSR layout (to_batch) and the FP64 oracle."""
    from firecore_b200 import topology as T
    from oracle import oracle as O
    O.build_oracle()
    tables = write_tables(str(tmp_path / "t"))
    xyz = tmp_path / "m.xyz"
    xyz.write_text(METHANOL)
    b = T.to_batch(_build(str(xyz), tables), nsys=2)
    assert b.nsys == 2 and b.pos.shape == (2 * 8, 3)
    F, E = O.eval_forces(b, O.make_params(flags=O.DEFAULT_FLAGS))
    assert np.isfinite(F).all() and np.isfinite(E).all()
    np.testing.assert_array_equal(E[0], E[1])


@pytest.mark.skipif(not os.path.isfile(os.path.join(RES, "AtomTypes.dat")), reason="FireCore tree not present")
@pytest.mark.parametrize("mol", ["polydiacetylene.xyz", "polydiacetylene_OH.xyz", "polymer-2.xyz"])
def test_oracle_matches_firecore_on_periodic_polymers(mol):
    """Bonds across the cell wall (neighCell != central image): FireCore's
    periodic polymers, typed by this builder, evaluated by the FP64 oracle and by
    FireCore's own eval_atom / evalLJQs_ng4_PBC_atom_omp through the reference
    harness agree to rounding."""
    import ctypes
    from firecore_b200 import topology as T
    from oracle import oracle as O
    O.build_oracle(with_ref=True)
    if not O.ref_available():
        pytest.skip("reference harness not built")
    d = _build(os.path.join(RES, "xyz", mol), T.table_paths(RES))
    assert d["pbc"] and (d["neighCell"][d["neighs"] >= 0] != 4).any()     # bonds into the next cells
    b = T.to_batch(d)
    na, nn = d["natoms"], d["nnode"]
    ref = O.ref()
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    pos = np.ascontiguousarray(b.pos)
    arr = [np.ascontiguousarray(x) for x in (b.neighs, b.neighCell, b.REQs)]
    nar = [np.ascontiguousarray(x) for x in (b.apars, b.bLs, b.bKs, b.Ksp, b.Kpp)]
    lv = np.ascontiguousarray(b.lvec[0].reshape(9)); npbc = np.array([1, 1, 0], np.int32)
    gn = np.array([4, 4, 8], np.int32); gp0 = np.zeros(3); gst = np.ones(3); C = np.zeros(4 * 4 * 8 * 3)
    bk = np.zeros((na, 4), np.int32); ng = np.zeros((na, 4), np.int32)
    for fl in (O.DEFAULT_FLAGS & ~O.GRID, O.BONDS | O.ANGLES | O.PISIGMA | O.PIPI | O.PBC):
        ref.ref_setup(na, nn, p(pos), p(arr[0]), p(arr[1]), p(arr[2]), *[p(x) for x in nar], p(lv), p(npbc), fl, 1.5,
                      p(gn), p(gp0), p(gst), p(C), p(bk), p(ng))
        f = np.zeros((na + nn, 3)); e = np.zeros(4)
        ref.ref_eval(p(f), p(e))
        Fo, Eo = O.eval_forces(b, O.make_params(flags=fl, npbc=(1, 1, 0)))
        assert np.abs(Fo - f).max() <= 1e-12 * max(1.0, np.abs(f).max())
        assert np.abs(Eo[0] - e).max() <= 1e-12 * max(1.0, np.abs(e).max())
