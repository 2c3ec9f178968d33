"""Reference-parity multipole mode (sqb200_jk_set_multipole) against the reference's own
GTO_JK_Matrix_Quartet_Parallel over a sequence of SCF visits.

The reference keeps state across the visits of one SCF: per quartet, the base-1.5 exponent of
its monopole error, measured the first time the quartet is computed, and on later visits it
substitutes the monopole values (computeQuartetMPole, src/matrix.c:3945-3949) for uncached
quartets whose 1.5^exponent * maxPShell falls below the fixed cutoff.  The visits here follow
the shape of its 3STEP schedule: a full density at a loose cutoff, then difference densities at
tightening cutoffs.  Every visit must match the reference's element by element at 1e-10 (the
plain-FP64 bar) and at 1e-7 of each visit's own magnitude, which holds only if the substitution
decisions are the same; the same visits without substitution differ by 1e-7 to 1e-4 of their
magnitude, so the mode is exercised."""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden, golden_basis, load_oracle, load_sqb200

TOL = 1e-10
port = load_oracle()


def _visits(n, P0, seed):
    """A full density, then difference densities shrinking as an SCF's do, at the tightening
    fixed cutoffs of a 3STEP schedule."""
    rng = np.random.default_rng(seed)

    def sym(scale):
        A = rng.normal(size=(n, n)) * scale
        return A + A.T

    return [P0, sym(1e-2), sym(1e-4), sym(1e-6), sym(1e-8)], [1e-7, 1e-7, 1e-9, 1e-10, 1e-10]


@pytest.mark.gpu
@pytest.mark.parametrize("case,max_mem", [("water_321g", 0), ("h2co_631gs", 0), ("h2co_631gs", 1)])
def test_multipole_visits_match_reference(case, max_mem):
    sqb = load_sqb200()
    g = golden(case)
    b = golden_basis(g)
    dens, cuts = _visits(b.nbf, g["PA"], 3)
    with tempfile.TemporaryDirectory() as d:
        xyz = os.path.join(d, "m.xyz")
        with open(xyz, "w") as f:
            f.write(sqb.molecules.xyz_text([(int(a[0]), a[1], a[2], a[3]) for a in g["atoms"]]))
        bas = os.path.join(d, "basis.txt")
        with open(bas, "w") as f:
            f.write(sqb.basis.gamess_text(str(g["basis"]), [int(a[0]) for a in g["atoms"]]))
        ref = port.ref_jkseq(xyz, bas, dens, cuts, scf_cutoff=1e-10, max_mem=max_mem)
    eng = sqb.JKEngine(b, schwarz=g["schwarz"])
    memcut = eng.mem_cutoff(cuts[0], max_mem)
    eng.set_multipole(True, memcut)
    substituted = 0.0
    for v, (P, c) in enumerate(zip(dens, cuts)):
        JT, KA, _ = eng.build(P, restricted=True, scf_cutoff=1e-10, fixed_cutoff=c,
                              dscreen_rmax=memcut if v == 0 else float("inf"))
        J0, K0 = ref[v]
        # 1e-10 absolute, and 1e-7 of the visit's own scale: the later visits' difference
        # densities are small, and a substitution decision taken differently moves their J/K
        # by 1e-4 of their size
        scale = max(np.abs(J0).max(), np.abs(K0).max())
        for M, M0 in ((JT, J0), (KA, K0)):
            err = np.abs(M - M0).max()
            assert err <= TOL and err <= 1e-7 * scale, (case, max_mem, v, err, scale)
        if v > 0:
            # the same visit with every quartet exact: the difference, far above the rounding
            # of these matrices, shows that quartets were substituted
            ex = sqb.JKEngine(b, schwarz=g["schwarz"])
            JX, KX, _ = ex.build(P, restricted=True, scf_cutoff=1e-10, fixed_cutoff=c, dscreen_rmax=float("inf"))
            ex.close()
            substituted = max(substituted, max(np.abs(JX - J0).max(), np.abs(KX - K0).max()) / scale)
    if max_mem == 0:
        assert substituted > 1e-12, substituted
    eng.close()
