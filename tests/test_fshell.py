"""Bases with f shells: the generic quartet path (csrc/jk_generic.cu) beside the generated class
kernels.

The reference reads f shells from GAMESS basis files (read_GAMESS_BasisSet, src/basis.c:488-499)
and types a ten-function shell TYPEF (genGTOShell, src/matrix.c:2527-2535); its QZP set gives
every heavy atom two f shells and hydrogen one.  The fixtures water_qzp (RHF, 126 functions)
and oh_qzp_uhf (UHF, 91) hold the reference's own basis arrays, Schwarz matrix, converged
densities, one-electron matrices and J/K builds (tests/golden/make_golden.py --fshells).

CPU: the package's basis builder and the oracle port against those fixtures.
GPU: J/K, device Schwarz, one-electron matrices and whole SCF energies against the reference,
quartet counts against the port, at the plain-FP64 bars (1e-10 on J/K, 1e-8 Eh on energies)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden, golden_basis, load_oracle, load_sqb200

TOL = 1e-10
FCASES = ["water_qzp", "oh_qzp_uhf"]
port = load_oracle()
SQREF_GPU = os.path.join(ROOT, "oracle", "_ref", "sqref_b200")


def _atoms(g):
    return [(int(a[0]), float(a[1]), float(a[2]), float(a[3])) for a in g["atoms"]]


@pytest.mark.parametrize("case", FCASES)
def test_basis_builder_matches_reference_with_f_shells(case):
    sqb = load_sqb200()
    g = golden(case)
    b = sqb.basis.build_basis(sqb.molecules.to_bohr(_atoms(g)), str(g["basis"]))
    assert np.array_equal(b.nprim, g["nprim"]) and np.array_equal(b.lmn, g["lmn"])
    assert np.array_equal(b.exps, g["exps"]) and np.array_equal(b.coefs, g["coefs"])
    assert np.abs(b.norms - g["norms"]).max() <= 1e-15 * np.abs(g["norms"]).max()
    assert int((b.lmn.sum(axis=1) == 3).sum()) > 0          # the case has f functions


def test_port_matches_reference_with_f_shells():
    """The oracle port (which handles f shells like the reference, by THO) against the
    reference's own J/K, both screening modes, and its Schwarz matrix."""
    g = golden("oh_qzp_uhf")
    b = golden_basis(g)
    np.testing.assert_allclose(port.schwarz(b), g["schwarz"], rtol=1e-12, atol=1e-14)
    for mode in ("mem", "dir"):
        rmax = port.mem_cutoff(b, g["schwarz"], 1e-10, 250 if mode == "mem" else 0)
        JT, KA, KB, _ = port.jk_build(b, g["schwarz"], g["PA"], g["PB"], restricted=False, scf_cutoff=1e-10,
                                      dscreen_rmax=rmax)
        for k, M in (("JT", JT), ("KA", KA), ("KB", KB)):
            assert np.abs(M - g[k + "_" + mode]).max() <= TOL, (mode, k)


def _engine(g, schwarz=True):
    sqb = load_sqb200()
    return sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"] if schwarz else None)


@pytest.mark.gpu
@pytest.mark.parametrize("case", FCASES)
@pytest.mark.parametrize("mode", ["mem", "dir"])
def test_fshell_jk_matches_reference(case, mode):
    g = golden(case)
    b = golden_basis(g)
    eng = _engine(g)
    restricted = bool(g["restricted"])
    rmax = eng.mem_cutoff(1e-10, 250 if mode == "mem" else 0)
    assert rmax == port.mem_cutoff(b, g["schwarz"], 1e-10, 250 if mode == "mem" else 0)
    PB = None if restricted else g["PB"]
    JT, KA, KB = eng.build(g["PA"], PB, restricted=restricted, scf_cutoff=1e-10, dscreen_rmax=rmax)
    for k, M in (("JT", JT), ("KA", KA), ("KB", KB)):
        err = np.abs(M - g[k + "_" + mode]).max()
        assert err <= TOL, (case, mode, k, err)
        assert np.array_equal(M, M.T), k
    # the same quartets and primitive quartets as the oracle's pass over every quartet
    _, _, _, st = port.jk_build(b, g["schwarz"], g["PA"], PB, restricted=restricted, scf_cutoff=1e-10,
                                dscreen_rmax=rmax)
    assert eng.stats()["quartets"] == st[1]
    assert eng.stats()["prim_quartets"] == st[2]
    eng.close()


@pytest.mark.gpu
def test_fshell_random_density_matches_port():
    """Arbitrary symmetric densities, restricted and unrestricted, both screening modes."""
    g = golden("oh_qzp_uhf")
    b = golden_basis(g)
    n = b.nbf
    rng = np.random.default_rng(11)
    A = rng.normal(size=(n, n)); A = 0.3 * (A + A.T)
    B = rng.normal(size=(n, n)); B = 0.3 * (B + B.T)
    eng = _engine(g)
    for restricted in (True, False):
        for rmax in (float("inf"), 0.0):
            PB = None if restricted else B
            JT, KA, KB = eng.build(A, PB, restricted=restricted, scf_cutoff=1e-10, dscreen_rmax=rmax)
            J0, K0, KB0, st = port.jk_build(b, g["schwarz"], A, PB, restricted=restricted, scf_cutoff=1e-10,
                                            dscreen_rmax=rmax)
            assert np.abs(JT - J0).max() <= TOL
            assert np.abs(KA - K0).max() <= TOL
            assert np.abs(KB - KB0).max() <= TOL
            assert eng.stats()["quartets"] == st[1]
            assert eng.stats()["prim_quartets"] == st[2]
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", FCASES)
def test_fshell_device_schwarz_and_oneint_match_reference(case):
    sqb = load_sqb200()
    g = golden(case)
    eng = _engine(g, schwarz=False)             # Schwarz bounds computed on the device
    np.testing.assert_allclose(eng.schwarz(), g["schwarz"], rtol=1e-12, atol=1e-14)
    restricted = bool(g["restricted"])
    JT, KA, _ = eng.build(g["PA"], None if restricted else g["PB"], restricted=restricted, scf_cutoff=1e-10)
    assert np.abs(JT - g["JT_dir"]).max() <= TOL
    assert np.abs(KA - g["KA_dir"]).max() <= TOL
    atoms = sqb.molecules.to_bohr(_atoms(g))
    S, T, V = eng.oneint([a[0] for a in atoms], [a[1:] for a in atoms])
    eng.close()
    assert np.abs(S - g["S"]).max() <= 1e-12
    assert np.abs(T - g["T"]).max() <= 1e-11
    assert np.abs(V - g["V"]).max() <= 1e-10 * max(1.0, np.abs(g["V"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", FCASES)
def test_fshell_device_scf_energy(case):
    sqb = load_sqb200()
    g = golden(case)
    job = sqb.scf.SCFJob(_atoms(g), str(g["basis"]), restricted=bool(g["restricted"]))
    e = job.run()
    iters = job.iters
    job.close()
    assert job.converged
    assert abs(e - float(g["energy"])) <= 1e-8, (case, e, float(g["energy"]))
    assert abs(iters - int(g["scf_iters"])) <= 1


@pytest.mark.gpu
@pytest.mark.parametrize("case", FCASES)
def test_fshell_gradient_against_finite_differences(case, monkeypatch):
    """Nuclear gradient with f functions (the gradient kernels sized for f: raised indices to g,
    Hermite orders to 13).  The reference's own uhf_force does not pin it: with f shells its
    forces depart from finite differences of its own energy (water/QZP: 8.6e-5 hartree/bohr on
    the oxygen's z, and 2.4e-4 normal to the molecular plane, where the gradient vanishes by
    symmetry; its d-shell forces agree with the same finite differences to 1.4e-6).  So the
    check is the central finite-difference gradient of the reference's SCF energy (fd_grad,
    tests/golden/make_golden.py --fd): with every quartet kept (SQB200_GRAD_SCREEN=0) to 1e-6
    hartree/bohr, with the reference's 1e-10 screens to 5e-5, and zero where symmetry makes it
    zero."""
    sqb = load_sqb200()
    g = golden(case)
    job = sqb.scf.SCFJob(_atoms(g), str(g["basis"]), restricted=bool(g["restricted"]))
    job.run()
    G0 = job.gradient()                                 # the reference's screens
    monkeypatch.setenv("SQB200_GRAD_SCREEN", "0")
    G = job.gradient()                                  # every quartet
    job.close()
    fd = g["fd_grad"]
    assert np.abs(G.sum(axis=0)).max() < 1e-8           # translational invariance
    assert np.abs(G - fd).max() <= 1e-6, np.abs(G - fd).max()
    assert np.abs(G0 - fd).max() <= 5e-5, np.abs(G0 - fd).max()
    xyz = np.array([a[1:] for a in _atoms(g)])
    for ax in range(3):                                 # an axis no atom leaves: zero force along it
        if np.abs(xyz[:, ax]).max() == 0.0:
            assert np.abs(G[:, ax]).max() <= 1e-9 and np.abs(G0[:, ax]).max() <= 1e-9


def _inputs(d, g):
    """The molecule and the basis text (written by the package) for a run of the reference."""
    sqb = load_sqb200()
    xyz = os.path.join(d, "m.xyz")
    with open(xyz, "w") as f:
        f.write(sqb.molecules.xyz_text(_atoms(g)))
    bas = os.path.join(d, "basis.txt")
    with open(bas, "w") as f:
        f.write(sqb.basis.gamess_text(str(g["basis"]), [int(a[0]) for a in g["atoms"]]))
    return xyz, bas


def _dropin(binary, g, opts, env=None):
    with tempfile.TemporaryDirectory() as d:
        xyz, bas = _inputs(d, g)
        r = subprocess.run([binary, "scf", xyz, bas, "-"] + list(opts), capture_output=True, text=True, timeout=900,
                           env=None if env is None else dict(os.environ, **env))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    res = [line for line in r.stderr.splitlines() if line.startswith("RESULT")]
    return float(dict(kv.split("=") for kv in res[-1].split()[1:])["energy"])


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(SQREF_GPU), reason="oracle/_ref/sqref_b200 not built")
@pytest.mark.parametrize("case", FCASES)
def test_fshell_dropin_scf_energy_matches_reference(case):
    """The reference program relinked onto the GPU build, 1STEP schedule."""
    g = golden(case)
    e = _dropin(SQREF_GPU, g, ["-SCFACC=1STEP", "-SCFCONV=1e-8"])
    assert abs(e - float(g["energy"])) <= 1e-8, (case, e, float(g["energy"]))


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(SQREF_GPU), reason="oracle/_ref/sqref_b200 not built")
@pytest.mark.parametrize("maxmem", [None, "0"])
def test_fshell_dropin_default_schedule_multipole_mode(maxmem):
    """The reference's default 3STEP schedule with the reference-parity multipole mode
    (SQB200_MULTIPOLE=1), which the generic path follows too: energies at 1e-8 Eh."""
    g = golden("oh_qzp_uhf")
    opts = ["-SCFCONV=1e-8"] + (["-MAXMEM=" + maxmem] if maxmem else [])
    e_ref = _dropin(port.REF_BIN, g, opts)
    e_gpu = _dropin(SQREF_GPU, g, opts, env={"SQB200_MULTIPOLE": "1"})
    assert abs(e_ref - e_gpu) <= 1e-8, (maxmem, e_ref, e_gpu)


@pytest.mark.gpu
def test_fshell_multipole_visits_match_reference():
    """Reference-parity multipole mode over SCF-like visits (a full density, then shrinking
    difference densities at tightening cutoffs) against the reference's own sequence."""
    sqb = load_sqb200()
    g = golden("oh_qzp_uhf")
    b = golden_basis(g)
    rng = np.random.default_rng(5)

    def sym(scale):
        A = rng.normal(size=(b.nbf, b.nbf)) * scale
        return A + A.T

    dens = [g["PA"], sym(1e-2), sym(1e-4), sym(1e-6)]
    cuts = [1e-7, 1e-7, 1e-9, 1e-10]
    with tempfile.TemporaryDirectory() as d:
        xyz, bas = _inputs(d, g)
        ref = port.ref_jkseq(xyz, bas, dens, cuts, scf_cutoff=1e-10, max_mem=0)
    eng = sqb.JKEngine(b, schwarz=g["schwarz"])
    memcut = eng.mem_cutoff(cuts[0], 0)
    eng.set_multipole(True, memcut)
    for v, (P, c) in enumerate(zip(dens, cuts)):
        JT, KA, _ = eng.build(P, restricted=True, scf_cutoff=1e-10, fixed_cutoff=c,
                              dscreen_rmax=memcut if v == 0 else float("inf"))
        J0, K0 = ref[v]
        scale = max(np.abs(J0).max(), np.abs(K0).max())
        for M, M0 in ((JT, J0), (KA, K0)):
            err = np.abs(M - M0).max()
            assert err <= TOL and err <= 1e-7 * scale, (v, err, scale)
    eng.close()


@pytest.mark.gpu
def test_fshell_unsupported_entry_points_fail_loudly():
    """The allocation-free entry point and batched builds cover s, sp, p and d shells only:
    with f shells they return SQB200_EUNSUPPORTED instead of a wrong build."""
    import ctypes

    import torch
    sqb = load_sqb200()
    g = golden("oh_qzp_uhf")
    eng = _engine(g)
    with pytest.raises(sqb.SQB200Error, match="f shells"):
        sqb.JKBatch([eng])
    n = eng.nbf
    P = torch.zeros((n, n), dtype=torch.float64, device="cuda:0")
    out = [torch.empty_like(P) for _ in range(3)]
    lib = sqb.load_library()
    lib.sqb200_jk_build_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    rc = lib.sqb200_jk_build_noalloc(eng._ctx, P.data_ptr(), P.data_ptr(), 1, 1e-10, 1e-10, 0.0,
                                     out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), None)
    assert rc == -2 and b"f shells" in lib.sqb200_last_error()
    eng.close()


def _perm_d_components(b):
    """The basis with every d shell's six components in reverse order (a layout the class
    kernels do not take: those shells go to the generic path), and the permutation p with
    new function k = old function p[k]."""
    sqb = load_sqb200()
    n = b.nbf
    perm = np.arange(n)
    k = 0
    while k < n:
        if b.lmn[k].sum() == 2 and k + 5 < n and (b.lmn[k:k + 6].sum(axis=1) == 2).all():
            perm[k:k + 6] = perm[k:k + 6][::-1]
            k += 6
        else:
            k += 1
    off = np.concatenate([[0], np.cumsum(b.nprim)])
    ex = np.concatenate([b.exps[off[i]:off[i + 1]] for i in perm])
    co = np.concatenate([b.coefs[off[i]:off[i + 1]] for i in perm])
    nm = np.concatenate([b.norms[off[i]:off[i + 1]] for i in perm])
    return sqb.basis.Basis(b.nprim[perm], b.lmn[perm], b.center[perm], ex, co, nm), perm


@pytest.mark.gpu
def test_reordered_d_components_take_the_generic_path():
    """d shells whose components come in another order than the reference's run on the
    generic path: J/K must equal the class kernels' result on the canonical order, permuted
    (same screening: the block maxima do not change), and the oracle port's on the new order."""
    sqb = load_sqb200()
    g = golden("h2co_631gs")
    b = golden_basis(g)
    bp, perm = _perm_d_components(b)
    assert (perm != np.arange(b.nbf)).any()
    P = g["PA"]
    Pp = P[np.ix_(perm, perm)]
    e0 = sqb.JKEngine(b, schwarz=g["schwarz"])
    J0, K0, _ = e0.build(P, restricted=True, scf_cutoff=1e-10)
    q0 = e0.stats()["quartets"]
    e0.close()
    e1 = sqb.JKEngine(bp)                            # Schwarz bounds from the device, generic pairs included
    np.testing.assert_allclose(e1.schwarz(), g["schwarz"][np.ix_(perm, perm)], rtol=1e-12, atol=1e-14)
    J1, K1, _ = e1.build(Pp, restricted=True, scf_cutoff=1e-10)
    assert e1.stats()["quartets"] == q0
    e1.close()
    assert np.abs(J1 - J0[np.ix_(perm, perm)]).max() <= TOL
    assert np.abs(K1 - K0[np.ix_(perm, perm)]).max() <= TOL
    Jp, Kp, _, _ = port.jk_build(bp, port.schwarz(bp), Pp, scf_cutoff=1e-10)
    assert np.abs(J1 - Jp).max() <= TOL and np.abs(K1 - Kp).max() <= TOL


@pytest.mark.gpu
def test_merged_shell_takes_the_generic_path():
    """An s and a d function with the same exponent on the same centre, adjacent in the basis,
    form one seven-function shell (genGTOShell merges them; the reference types it TYPEX).
    With screening off, its J/K equal those of the same functions placed apart (a separate s
    and d shell, class kernels), up to the order of the functions."""
    sqb = load_sqb200()
    B = sqb.basis
    atoms = sqb.molecules.to_bohr(sqb.molecules.water())
    base = B.build_basis(atoms, "321g")
    o = tuple(base.center[0])
    extra_s = [(1, (0, 0, 0), o, 0.8)]
    extra_d = [(1, lmn, o, 0.8) for lmn, _ in B.COMPONENTS["D"]]

    def make(funcs):
        nprim, lmn, cen, ex, co, nm = [], [], [], [], [], []
        for np_, l, c, e, cf in funcs:
            nprim.append(np_); lmn.append(l); cen.append(c)
            ex.extend(e); co.extend(cf); nm.extend(B.prim_norm(x, *l) for x in e)
        return B.Basis(nprim, lmn, cen, ex, co, nm)

    off = np.concatenate([[0], np.cumsum(base.nprim)])
    orig = [(int(base.nprim[i]), tuple(base.lmn[i]), tuple(base.center[i]), list(base.exps[off[i]:off[i + 1]]),
             list(base.coefs[off[i]:off[i + 1]])) for i in range(base.nbf)]
    new = [(1, l, c, [e], [1.0]) for _, l, c, e in extra_s + extra_d]
    merged = make(orig + new)                        # ... s(0.8) d(0.8): one 7-function shell
    apart = make(new[:1] + orig + new[1:])           # s(0.8) first, d(0.8) last: two shells
    n = merged.nbf
    perm = np.concatenate([np.arange(1, base.nbf + 1), [0], np.arange(base.nbf + 1, n)])   # apart index of merged k
    rng = np.random.default_rng(2)
    A = rng.normal(size=(n, n)); A = 0.2 * (A + A.T)
    em, ea = sqb.JKEngine(merged), sqb.JKEngine(apart)
    Jm, Km, _ = em.build(A, restricted=True, scf_cutoff=0.0, dscreen_rmax=float("inf"))
    Pa = np.empty_like(A)
    Pa[np.ix_(perm, perm)] = A
    Ja, Ka, _ = ea.build(Pa, restricted=True, scf_cutoff=0.0, dscreen_rmax=float("inf"))
    em.close(); ea.close()
    assert np.abs(Jm - Ja[np.ix_(perm, perm)]).max() <= TOL
    assert np.abs(Km - Ka[np.ix_(perm, perm)]).max() <= TOL
