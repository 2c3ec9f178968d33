"""Reference-parity multipole mode (sqb200_jk_set_multipole) against the reference's own
GTO_JK_Matrix_Quartet_Parallel over a sequence of SCF visits.

The reference keeps state across the visits of one SCF: per quartet, the base-1.5 exponent of
its monopole error, measured the first time the quartet is computed, and on later visits it
substitutes the monopole values (computeQuartetMPole, src/matrix.c:3945-3949) for uncached
quartets whose 1.5^exponent * maxPShell falls below the fixed cutoff.  The visits here follow
the shape of its 3STEP schedule: a full density at a loose cutoff, then difference densities at
tightening cutoffs.  Every visit must match the reference's element by element at 1e-10 (the
plain-FP64 bar), which holds only if the substitution decisions are the same."""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden, golden_basis, load_oracle, load_sqb200

TOL = 1e-10
port = load_oracle()


def _visits(n, P0, seed):
    rng = np.random.default_rng(seed)

    def sym(scale):
        A = rng.normal(size=(n, n)) * scale
        return A + A.T

    return [P0, sym(0.02), sym(0.005), sym(1e-3)], [1e-7, 1e-7, 1e-9, 1e-10]


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
        assert np.abs(JT - J0).max() <= TOL, (case, max_mem, v, np.abs(JT - J0).max())
        assert np.abs(KA - K0).max() <= TOL, (case, max_mem, v, np.abs(KA - K0).max())
        if v > 0:
            # the same visit without substitution differs: the mode is really exercised
            ex = sqb.JKEngine(b, schwarz=g["schwarz"])
            JX, KX, _ = ex.build(P, restricted=True, scf_cutoff=1e-10, fixed_cutoff=c, dscreen_rmax=float("inf"))
            ex.close()
            substituted = max(substituted, np.abs(JX - J0).max())
    if max_mem == 0:
        assert substituted > TOL, substituted
    eng.close()
