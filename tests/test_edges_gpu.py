"""Edge cases of the J/K build against the oracle port: the smallest basis (one s function),
a zero density, a density with a single non-zero pair, a cutoff no quartet passes, an sp-shell
basis with one f shell added (the generic path with L-shell kets), every screen off against the
reference's unscreened quadruple loop, and the inputs the library must refuse (a g function, a
contraction longer than the reference's MAXCONTRACT of 32)."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from conftest import golden, golden_basis, load_oracle, load_sqb200

TOL = 1e-10
port = load_oracle()


def _basis(funcs):
    """Basis from (nprim, (l, m, n), centre, exps, coefs) tuples, normalised as genBasis does."""
    B = load_sqb200().basis
    nprim, lmn, cen, ex, co, nm = [], [], [], [], [], []
    for np_, l, c, e, cf in funcs:
        nprim.append(np_); lmn.append(l); cen.append(c)
        ex.extend(e); co.extend(cf); nm.extend(B.prim_norm(x, *l) for x in e)
    return B.Basis(nprim, lmn, cen, ex, co, nm)


def _check(b, P, restricted=True, PB=None, **kw):
    sqb = load_sqb200()
    S = port.schwarz(b)
    eng = sqb.JKEngine(b, schwarz=S)
    JT, KA, KB = eng.build(P, PB, restricted=restricted, **kw)
    st = eng.stats()
    eng.close()
    J0, K0, KB0, st0 = port.jk_build(b, S, P, PB, restricted=restricted, scf_cutoff=kw.get("scf_cutoff", 1e-10),
                                     dscreen_rmax=kw.get("dscreen_rmax", float("inf")))
    assert np.abs(JT - J0).max() <= TOL and np.abs(KA - K0).max() <= TOL and np.abs(KB - KB0).max() <= TOL
    assert st["quartets"] == st0[1] and st["prim_quartets"] == st0[2]
    return JT, KA, KB, st


@pytest.mark.gpu
def test_one_s_function():
    b = _basis([(3, (0, 0, 0), (0.0, 0.0, 0.0), [3.42525091, 0.62391373, 0.16885540],
                 [0.15432897, 0.53532814, 0.44463454])])
    JT, KA, _, st = _check(b, np.array([[0.7]]))
    assert st["quartets"] == 1 and JT[0, 0] > 0 and KA[0, 0] < 0


@pytest.mark.gpu
def test_zero_and_single_pair_densities():
    g = golden("h2co_631gs")
    b = golden_basis(g)
    n = b.nbf
    JT, KA, KB, _ = _check(b, np.zeros((n, n)), dscreen_rmax=0.0)
    assert not JT.any() and not KA.any() and not KB.any()
    P = np.zeros((n, n))
    P[3, 17] = P[17, 3] = 0.4
    _check(b, P)                                 # no density screen
    _check(b, P, dscreen_rmax=0.0)               # density screen on every quartet


@pytest.mark.gpu
def test_cutoff_that_no_quartet_passes():
    sqb = load_sqb200()
    g = golden("water_321g")
    eng = sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    JT, KA, _ = eng.build(g["PA"], restricted=True, scf_cutoff=1e6)
    assert eng.stats()["quartets"] == 0 and not JT.any() and not KA.any()
    # and the next build at the usual cutoff is whole again (work lists are per cutoff)
    JT, KA, _ = eng.build(g["PA"], restricted=True, scf_cutoff=1e-10)
    assert np.abs(JT - g["JT_dir"]).max() <= TOL
    eng.close()


@pytest.mark.gpu
def test_sp_shells_with_an_f_shell():
    """Formaldehyde 6-31G* (s, sp and d shells) with an f shell on oxygen: the quartets with the
    f shell take the generic path, with every class of the others (sp shells included) as kets;
    restricted and unrestricted, against the port."""
    sqb = load_sqb200()
    g = golden("h2co_631gs")
    base = golden_basis(g)
    off = np.concatenate([[0], np.cumsum(base.nprim)])
    funcs = [(int(base.nprim[i]), tuple(base.lmn[i]), tuple(base.center[i]), list(base.exps[off[i]:off[i + 1]]),
              list(base.coefs[off[i]:off[i + 1]])) for i in range(base.nbf)]
    o = tuple(base.center[np.argmax(base.exps[off[:-1]])])    # the heaviest atom's centre
    funcs += [(1, l, o, [1.4], [1.0]) for l, _ in sqb.basis.COMPONENTS["F"]]
    b = _basis(funcs)
    n = b.nbf
    rng = np.random.default_rng(4)
    A = rng.normal(size=(n, n)); A = 0.2 * (A + A.T)
    B = rng.normal(size=(n, n)); B = 0.2 * (B + B.T)
    _check(b, A)
    _check(b, A, restricted=False, PB=B, dscreen_rmax=0.0)


def _create(b):
    sqb = load_sqb200()
    L = sqb.load_library()
    ctx = ctypes.c_void_p()
    rc = L.sqb200_jk_create(ctypes.byref(ctx), b.nbf, b.nprim, np.ascontiguousarray(b.lmn.ravel()),
                            np.ascontiguousarray(b.center.ravel()), b.exps, b.ncoef, None, 0)
    msg = L.sqb200_last_error()
    if rc == 0:
        L.sqb200_jk_destroy(ctx)
    return rc, msg


@pytest.mark.gpu
def test_g_function_and_long_contraction_refused():
    rc, msg = _create(_basis([(1, (4, 0, 0), (0.0, 0.0, 0.0), [1.0], [1.0])]))
    assert rc == -2 and b"l+m+n = 4" in msg
    rc, msg = _create(_basis([(33, (0, 0, 0), (0.0, 0.0, 0.0), list(np.geomspace(0.1, 100.0, 33)), [0.1] * 33)]))
    assert rc == -2 and b"contraction" in msg


def _ref_inputs(d, g):
    """The molecule and the basis text (written by the package) for a run of the reference."""
    sqb = load_sqb200()
    xyz = os.path.join(d, "m.xyz")
    with open(xyz, "w") as f:
        f.write(sqb.molecules.xyz_text([(int(a[0]), a[1], a[2], a[3]) for a in g["atoms"]]))
    bas = os.path.join(d, "b.txt")
    with open(bas, "w") as f:
        f.write(sqb.basis.gamess_text(str(g["basis"]), [int(a[0]) for a in g["atoms"]]))
    return xyz, bas


@pytest.mark.gpu
@pytest.mark.skipif(not port.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", ["water_321g", "oh_321g_uhf"])
def test_unscreened_build_matches_reference_quadruple_loop(case):
    """With every screen off (cutoff 0, no density screen) the build equals the reference's
    unscreened loop over all function quartets, GTO_JK_Matrix_NoSymm, to 1e-10: the symmetric
    shell-quartet digestion, the degeneracy factors and the J/K signs, with nothing skipped but
    primitive quartets below the 1e-15 prefactor (which that loop keeps)."""
    sqb = load_sqb200()
    g = golden(case)
    restricted = bool(g["restricted"])
    PB = None if restricted else g["PB"]
    with tempfile.TemporaryDirectory() as d:
        xyz, bas = _ref_inputs(d, g)
        GA, GB = port.ref_nosymm(xyz, bas, g["PA"], PB, cutoff=0.0)
    eng = sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    JT, KA, KB = eng.build(g["PA"], PB, restricted=restricted, scf_cutoff=0.0, dscreen_rmax=float("inf"))
    eng.close()
    assert np.abs(JT + KA - GA).max() <= TOL
    assert np.abs(JT + KB - GB).max() <= TOL
