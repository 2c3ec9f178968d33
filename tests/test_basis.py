"""Host-side basis builder and geometry generators against the reference's genBasis output
stored in the golden fixtures (function order, exponents, coefficients, normalisation)."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, load_sqb200


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_build_basis_matches_reference_genbasis(case):
    sqb = load_sqb200()
    g = golden(case)
    atoms = [(int(a[0]), a[1], a[2], a[3]) for a in g["atoms"]]
    b = sqb.basis.build_basis(sqb.molecules.to_bohr(atoms), str(g["basis"]))
    assert b.nbf == len(g["nprim"])
    assert np.array_equal(b.nprim, g["nprim"])
    assert np.array_equal(b.lmn, g["lmn"])
    assert np.array_equal(b.exps, g["exps"])
    assert np.array_equal(b.coefs, g["coefs"])
    np.testing.assert_allclose(b.norms, g["norms"], rtol=1e-15, atol=0)
    # centres: the reference parsed the 12-decimal XYZ text; ours are the unrounded floats
    np.testing.assert_allclose(b.center, g["xyz"], rtol=0, atol=2e-12)


def test_c60_geometry():
    sqb = load_sqb200()
    at = np.array([a[1:] for a in sqb.molecules.c60()])
    assert len(at) == 60
    d = np.linalg.norm(at[:, None] - at[None], axis=-1)
    bonds = np.sort(d[np.triu_indices(60, 1)])[:90]
    assert np.allclose(bonds[:60], 1.40, atol=1e-9) or np.allclose(bonds[30:], 1.45, atol=1e-9)
    assert np.isclose(bonds.min(), 1.40) and np.isclose(bonds.max(), 1.45)
    r = np.linalg.norm(at, axis=1)
    assert np.ptp(r) < 1e-9                      # all atoms on one sphere (Ih orbit)
    b = sqb.basis.build_basis(sqb.molecules.to_bohr(sqb.molecules.c60()), "631g")
    assert b.nbf == 540


def test_benzene_and_water_sizes():
    sqb = load_sqb200()
    M, B = sqb.molecules, sqb.basis
    assert B.build_basis(M.to_bohr(M.water()), "321g").nbf == 13
    assert B.build_basis(M.to_bohr(M.benzene()), "631g_star").nbf == 102


def test_random_organics_closed_shell():
    sqb = load_sqb200()
    rng = np.random.default_rng(5)
    for n_heavy in (2, 5, 12, 20):
        atoms = sqb.molecules.random_organic(rng, n_heavy)
        assert sum(1 for a in atoms if a[0] > 1) == n_heavy
        assert sqb.molecules.n_electrons(atoms) % 2 == 0
        heavy = np.array([a[1:] for a in atoms if a[0] > 1])
        d = np.linalg.norm(heavy[:, None] - heavy[None], axis=-1)
        assert d[np.triu_indices(len(heavy), 1)].min() >= 0.99


def test_gamess_text_roundtrip():
    sqb = load_sqb200()
    txt = sqb.basis.gamess_text("631g_star", [1, 6])
    assert txt.startswith("$DATA") and "CARBON" in txt and txt.rstrip().endswith("$END")
