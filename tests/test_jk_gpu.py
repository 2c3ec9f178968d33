"""J/K parity of the CUDA engine against the reference (golden fixtures) and the oracle port.

Tolerance: 1e-10 max-abs on JT, KA, KB (the plain-FP64 bar).  Quartet counts must match the
oracle exactly (integer work: the screening decisions are identical)."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden, golden_basis, load_oracle, load_sqb200

TOL = 1e-10
port = load_oracle()


def _engine(g):
    sqb = load_sqb200()
    return sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
@pytest.mark.parametrize("mode", ["mem", "dir"])
def test_jk_matches_reference(case, mode):
    g = golden(case)
    eng = _engine(g)
    restricted = bool(g["restricted"])
    cut = float(g["cutoff"])
    rmax = eng.mem_cutoff(cut, 250 if mode == "mem" else 0)
    JT, KA, KB = eng.build(g["PA"], None if restricted else g["PB"], restricted=restricted,
                           scf_cutoff=cut, dscreen_rmax=rmax)
    for k, M in (("JT", JT), ("KA", KA), ("KB", KB)):
        err = np.abs(M - g[k + "_" + mode]).max()
        assert err <= TOL, (case, mode, k, err)
        assert np.array_equal(M, M.T), k
    st = eng.stats()
    assert st["quartets"] > 0 and st["prim_quartets"] > 0 and st["flops"] > 0
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["water_321g", "oh_321g_uhf", "h2co_631gs"])
def test_jk_random_density_matches_port(case):
    """Arbitrary symmetric densities (not just converged ones), both screening modes."""
    g = golden(case)
    b = golden_basis(g)
    rng = np.random.default_rng(7)
    n = b.nbf
    A = rng.normal(size=(n, n)); A = 0.3 * (A + A.T)
    B = rng.normal(size=(n, n)); B = 0.3 * (B + B.T)
    eng = _engine(g)
    for restricted in (True, False):
        for rmax in (float("inf"), 0.0):
            PB = None if restricted else B
            JT, KA, KB = eng.build(A, PB, restricted=restricted, scf_cutoff=1e-10, dscreen_rmax=rmax)
            J0, K0, KB0, st = port.jk_build(b, g["schwarz"], A, PB, restricted=restricted,
                                            scf_cutoff=1e-10, dscreen_rmax=rmax)
            assert np.abs(JT - J0).max() <= TOL
            assert np.abs(KA - K0).max() <= TOL
            assert np.abs(KB - KB0).max() <= TOL
            assert eng.stats()["quartets"] == st[1]
            assert eng.stats()["prim_quartets"] == st[2]


def _pd_basis():
    """A synthetic basis with pure p and d shells beside s and sp (the Pople sets used by
    the workloads have no pure p shell): water 3-21G plus a p and a d shell per atom."""
    sqb = load_sqb200()
    B = sqb.basis
    atoms = sqb.molecules.to_bohr(sqb.molecules.water())
    base = B.build_basis(atoms, "321g")
    nprim, lmn, cen, ex, co, nm = list(base.nprim), [tuple(x) for x in base.lmn], [tuple(x) for x in base.center], \
        list(base.exps), list(base.coefs), list(base.norms)
    for (z, x, y, w) in atoms:
        for kind, prims in (("P", [(1.3, 0.6), (0.35, 0.5)]), ("D", [(0.9, 1.0)])):
            for (l, m, n), _ in B.COMPONENTS[kind]:
                nprim.append(len(prims)); lmn.append((l, m, n)); cen.append((x, y, w))
                for e, c in prims:
                    ex.append(e); co.append(c); nm.append(B.prim_norm(e, l, m, n))
    return B.Basis(nprim, lmn, cen, ex, co, nm)


@pytest.mark.gpu
def test_jk_pure_p_and_d_shells_match_port():
    b = _pd_basis()
    S = port.schwarz(b)
    rng = np.random.default_rng(3)
    n = b.nbf
    A = rng.normal(size=(n, n)); A = 0.2 * (A + A.T)
    sqb = load_sqb200()
    eng = sqb.JKEngine(b, schwarz=S)
    JT, KA, KB = eng.build(A, restricted=True, scf_cutoff=1e-10)
    J0, K0, _, st = port.jk_build(b, S, A, scf_cutoff=1e-10)
    assert np.abs(JT - J0).max() <= TOL
    assert np.abs(KA - K0).max() <= TOL
    assert eng.stats()["quartets"] == st[1]


@pytest.mark.gpu
def test_jk_device_api_with_torch_buffers():
    import torch
    g = golden("h2co_631gs")
    eng = _engine(g)
    dev = torch.device("cuda:0")
    PA = torch.tensor(g["PA"], device=dev, dtype=torch.float64).contiguous()
    JT = torch.empty_like(PA); KA = torch.empty_like(PA); KB = torch.empty_like(PA)
    eng.build_device(PA.data_ptr(), PA.data_ptr(), JT.data_ptr(), KA.data_ptr(), KB.data_ptr(),
                     restricted=True, scf_cutoff=1e-10)
    torch.cuda.synchronize()
    eng.stats()   # synchronises the context stream too
    assert np.abs(JT.cpu().numpy() - g["JT_dir"]).max() <= TOL
    assert np.abs(KA.cpu().numpy() - g["KA_dir"]).max() <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_device_schwarz_matches_reference(case):
    """sqrt|(pq|pq)| on the device against the reference's create_Schwarz."""
    g = golden(case)
    sqb = load_sqb200()
    eng = sqb.JKEngine(golden_basis(g))          # no Schwarz given: computed on the device
    S = eng.schwarz()
    np.testing.assert_allclose(S, g["schwarz"], rtol=1e-12, atol=1e-14)
    # and the build from device-computed bounds still matches the reference
    JT, KA, _ = eng.build(g["PA"], None if g["restricted"] else g["PB"], restricted=bool(g["restricted"]),
                          scf_cutoff=1e-10)
    assert np.abs(JT - g["JT_dir"]).max() <= TOL
    assert np.abs(KA - g["KA_dir"]).max() <= TOL


@pytest.mark.gpu
def test_c60_full_size_properties():
    """C60/6-31G (540 functions) at full size: outputs symmetric, J/K linear in the density
    (density screen off), and the Schwarz-survivor count matches the oracle's shell loop."""
    sqb = load_sqb200()
    atoms = sqb.molecules.to_bohr(sqb.molecules.c60())
    b = sqb.basis.build_basis(atoms, "631g")
    eng = sqb.JKEngine(b)                        # device Schwarz
    n = b.nbf
    rng = np.random.default_rng(11)
    D1 = rng.normal(size=(n, n)) * 0.01; D1 = D1 + D1.T
    D2 = rng.normal(size=(n, n)) * 0.01; D2 = D2 + D2.T
    J1, K1, _ = eng.build(D1, scf_cutoff=1e-10, dscreen_rmax=0.0)
    J2, K2, _ = eng.build(D2, scf_cutoff=1e-10, dscreen_rmax=0.0)
    J3, K3, _ = eng.build(D1 + D2, scf_cutoff=1e-10, dscreen_rmax=0.0)
    assert np.array_equal(J3, J3.T) and np.array_equal(K3, K3.T)
    assert np.abs(J3 - J1 - J2).max() < 1e-11 * max(1.0, np.abs(J3).max())
    assert np.abs(K3 - K1 - K2).max() < 1e-11 * max(1.0, np.abs(K3).max())
    st = eng.stats()
    assert st["shells"] == 180 and st["pairs"] == 180 * 181 // 2
    # independent count of unordered shell-pair pairs with Sch(PQ)*Sch(IJ) >= 1e-10
    S = eng.schwarz()
    first, nf, _ = port.shells(b)
    blk = np.array([[S[f0:f0 + n0, g0:g0 + m0].max() for g0, m0 in zip(first, nf)] for f0, n0 in zip(first, nf)])
    pv = np.sort(np.concatenate([blk[P, :P + 1] for P in range(len(first))]))
    cnt = 0
    for i, v in enumerate(pv):   # pairs (i <= j) in sorted order with pv[i]*pv[j] >= cut
        j0 = max(i, np.searchsorted(pv, 1e-10 / v if v > 0 else np.inf, side="left"))
        while j0 > i and pv[j0 - 1] * v >= 1e-10:
            j0 -= 1
        while j0 < len(pv) and pv[j0] * v < 1e-10:
            j0 += 1
        cnt += len(pv) - max(j0, i)
    assert st["quartets"] == cnt, (st["quartets"], cnt)
    assert 30e6 < cnt < 40e6                     # survey: 36.2M survivors for C60/6-31G


def c60_fixture():
    """The C60/6-31G fixture (tests/golden/make_c60_golden.py): the reference's genBasis arrays,
    Schwarz matrix, its converged SCF density and one fresh reference J/K build from it
    (direct mode: density screen on every quartet), split over 8 reference processes as
    uhf_getGMatrix runs it; symmetric matrices come back from their stored upper triangles."""
    g = golden("c60_631g")
    n = len(g["nprim"])
    iu = np.triu_indices(n)
    for k in ("schwarz", "PA", "JT", "KA"):
        M = np.zeros((n, n))
        M[iu] = g.pop(k + "_u")
        g[k] = M + np.triu(M, 1).T
    return g


def test_c60_fixture_is_consistent():
    """CPU check of the C60 fixture: 540 functions in the reference's order, the density traces
    to the 180 occupied orbitals, the outputs are symmetric, J positive and K negative on the
    diagonal."""
    g = c60_fixture()
    b = golden_basis(g)
    assert b.nbf == 540 and int(g["ncpu"]) == 8
    S = load_sqb200().checkpoint.overlap_matrix(b, b)
    assert abs(np.sum(g["PA"] * S) - 180.0) < 1e-6       # tr(PA S) = occupied orbitals
    assert np.array_equal(g["JT"], g["JT"].T) and np.array_equal(g["KA"], g["KA"].T)
    assert (np.diag(g["JT"]) > 0).all() and (np.diag(g["KA"]) < 0).all()
    assert np.allclose(g["schwarz"], g["schwarz"].T)


@pytest.mark.gpu
def test_c60_matches_reference_split_build():
    """C60/6-31G, 540 functions, element by element against the reference's own build (the sum
    of its 8 processes' shares), 1e-10 max-abs, from the reference's converged density with
    its Schwarz matrix; the density screen applies to every quartet as in the reference's
    direct mode."""
    g = c60_fixture()
    eng = _engine(g)
    JT, KA, KB = eng.build(g["PA"], restricted=True, scf_cutoff=float(g["cutoff"]), dscreen_rmax=float("inf"))
    errJ = np.abs(JT - g["JT"]).max()
    errK = np.abs(KA - g["KA"]).max()
    assert errJ <= TOL and errK <= TOL, (errJ, errK)
    assert np.array_equal(KB, KA)
    st = eng.stats()
    assert 30e6 < st["quartets"] < 40e6
    eng.close()


@pytest.mark.gpu
def test_mem_cutoff_equals_the_reference_rule():
    """The in-memory cutoff (getMemCutoff, src/matrix.c:3703) is the reference's exact value:
    the sorted-pair count in the library against the oracle's pass over every quartet, for
    golden molecules and seeded organics, several cutoffs and memory limits."""
    sqb = load_sqb200()
    cases = []
    for c in GOLDEN_CASES:
        g = golden(c)
        cases.append((golden_basis(g), g["schwarz"]))
    rng = np.random.default_rng(5)
    for k in (3, 6, 9):
        b = sqb.basis.build_basis(sqb.molecules.to_bohr(sqb.molecules.random_organic(rng, k)), "631g_star")
        e = sqb.JKEngine(b)
        cases.append((b, e.schwarz()))
        e.close()
    for b, S in cases:
        eng = sqb.JKEngine(b, schwarz=S)
        for cut in (1e-12, 3.7e-11, 1e-9):
            for mb in (0, 1, 20, 250):
                assert eng.mem_cutoff(cut, mb) == port.mem_cutoff(b, S, cut, mb), (b.nbf, cut, mb)
        eng.close()
