"""Seeded workload generator: determinism and topology invariants (CPU)."""
import numpy as np
import pytest

from firecore_b200 import systems as S


def test_deterministic():
    a = S.make_systems([24, 60, 127], seed=4)
    b = S.make_systems([24, 60, 127], seed=4)
    for k in ("pos", "neighs", "bkneighs", "REQs", "apars", "bLs", "bKs", "Ksp", "Kpp"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


@pytest.mark.parametrize("n", [20, 24, 60, 127, 250, 400])
def test_topology_invariants(n):
    b = S.make_systems([n], seed=n)
    nn = int(b.nnode[0])
    assert b.natoms[0] == n and nn == S._lib.load().mmff_gen_nnode(n)
    ng, bk = b.neighs, b.bkneighs
    # back-neighbours are exactly the node slots pointing at each atom (MMFFsp3_loc::makeBackNeighs)
    for i in range(n):
        refs = sorted(ia * 4 + j for ia in range(nn) for j in range(4) if ng[ia, j] == i)
        assert sorted(x for x in bk[i] if x >= 0) == refs
    # caps have exactly one neighbour (their node); composition C:N:O:H = 10:2:2:10
    assert (ng[nn:, 0] >= 0).all() and (ng[nn:, 1:] == -1).all() and (ng[nn:, 0] < nn).all()
    el = b.elements
    assert (el[:nn] > 0).all() and (el[nn:] == 0).all()
    # bonded distances: heavy-heavy 1.40 +- 0.05 (+ noise), X-H 1.09 (+ noise)
    p = b.pos
    L = [np.linalg.norm(p[j] - p[i]) for i in range(nn) for j in ng[i] if j >= 0]
    assert 0.7 < min(L) and max(L) < 2.0
    # charges re-centred to zero net
    assert abs(b.REQs[:, 2].sum()) < 1e-9


def test_slab():
    sub = S.make_slab()
    assert sub.spos.shape == (192, 3)
    assert abs(sub.sREQ[:, 2].sum()) < 1e-12
    assert sub.grid.n == (226, 226, 200)
