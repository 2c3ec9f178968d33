"""ctypes access to the oracle: our C restatement (_port/liboracle.so) and the reference
harness (_ref/sqref).  TEST INFRASTRUCTURE ONLY -- imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the product.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_port", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "sqref")

_lib = None
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(PORT_SO):
            subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
        L = ctypes.CDLL(PORT_SO)
        L.orc_boys.argtypes = [ctypes.c_int, ctypes.c_double, _f64p]
        L.orc_shells.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _i32p, _i32p, _i32p]
        L.orc_shells.restype = ctypes.c_int
        L.orc_schwarz.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p]
        L.orc_mem_cutoff.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p,
                                     ctypes.c_double, ctypes.c_int]
        L.orc_mem_cutoff.restype = ctypes.c_double
        L.orc_jk_build.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                   _f64p, _f64p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, _f64p, _f64p, _f64p,
                                   np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        L.orc_jk_build.restype = ctypes.c_int
        L.orc_quartet.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p]
        L.orc_quartet.restype = ctypes.c_int
        _lib = L
    return _lib


def _b(basis):
    return (basis.nbf, basis.nprim, np.ascontiguousarray(basis.lmn.ravel()),
            np.ascontiguousarray(basis.center.ravel()), basis.exps)


def boys(mmax, x):
    F = np.zeros(mmax + 1)
    lib().orc_boys(mmax, float(x), F)
    return F


def shells(basis):
    n = basis.nbf
    first = np.zeros(n, np.int32); nf = np.zeros(n, np.int32); ty = np.zeros(n, np.int32)
    ns = lib().orc_shells(*_b(basis), first, nf, ty)
    return first[:ns], nf[:ns], ty[:ns]


def schwarz(basis):
    S = np.zeros(basis.nbf * basis.nbf)
    lib().orc_schwarz(*_b(basis), basis.coefs, basis.norms, S)
    return S.reshape(basis.nbf, basis.nbf)


def mem_cutoff(basis, schwarz_mat, cutoff, max_mem_mb):
    return lib().orc_mem_cutoff(*_b(basis), np.ascontiguousarray(schwarz_mat, dtype=np.float64).ravel(),
                                cutoff, int(max_mem_mb))


def quartet(basis, P, Q, I, J):
    out = np.zeros(50625)
    n = lib().orc_quartet(*_b(basis), basis.coefs, basis.norms, P, Q, I, J, out)
    return out[:n]


def jk_build(basis, schwarz_mat, PA, PB=None, restricted=True, scf_cutoff=1e-10,
             fixed_cutoff=None, dscreen_rmax=float("inf")):
    """Fresh J/K as the reference's GTO_JK_Matrix_Quartet_Parallel; returns JT, KA, KB, stats."""
    n = basis.nbf
    PA = np.ascontiguousarray(PA, dtype=np.float64).reshape(n * n)
    PB = PA if PB is None else np.ascontiguousarray(PB, dtype=np.float64).reshape(n * n)
    if fixed_cutoff is None:
        fixed_cutoff = scf_cutoff
    JT = np.zeros(n * n); KA = np.zeros(n * n); KB = np.zeros(n * n)
    st = np.zeros(4, np.int64)
    rc = lib().orc_jk_build(*_b(basis), basis.coefs, basis.norms,
                            np.ascontiguousarray(schwarz_mat, dtype=np.float64).ravel(),
                            PA, PB, int(bool(restricted)), scf_cutoff, fixed_cutoff,
                            dscreen_rmax, JT, KA, KB, st)
    if rc != 0:
        raise ValueError("oracle: unsupported shell type")
    return JT.reshape(n, n), KA.reshape(n, n), KB.reshape(n, n), st


# ---------------------------------------------------------------- reference harness

def ref_available():
    return os.path.exists(REF_BIN)


def ref_run(args, timeout=3600):
    r = subprocess.run([REF_BIN] + [str(a) for a in args], capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("sqref failed: %s" % r.stderr[-2000:])
    res = {}
    for line in r.stderr.splitlines():
        if line.startswith("RESULT"):
            for kv in line.split()[1:]:
                k, v = kv.split("=")
                res[k] = float(v)
    # SCF iteration lines of uhf() (src/uhf.c:1733: " %5d %20.8f %20.4E")
    its = [t for t in (ln.split() for ln in r.stdout.splitlines())
           if len(t) == 3 and t[0].isdigit() and "E" in t[2]]
    if its:
        res["iters"] = int(its[-1][0])
    return res


def ref_jk(xyz_path, basis_path, PA, PB=None, restricted=True, cutoff=1e-10, max_mem=250):
    n = PA.shape[0]
    with tempfile.TemporaryDirectory() as d:
        pa = os.path.join(d, "pa.bin"); PA.astype(np.float64).tofile(pa)
        pb = "-"
        if PB is not None:
            pb = os.path.join(d, "pb.bin"); PB.astype(np.float64).tofile(pb)
        out = os.path.join(d, "out.bin")
        res = ref_run(["jk", xyz_path, basis_path, pa, pb, int(bool(restricted)), cutoff, max_mem, out])
        m = np.fromfile(out, dtype=np.float64).reshape(3, n, n)
    return m[0], m[1], m[2], res


def ref_nosymm(xyz_path, basis_path, PA, PB=None, cutoff=0.0):
    """The reference's unscreened quadruple loop over basis functions (GTO_JK_Matrix_NoSymm,
    src/matrix.c:5098-5183, contracted integrals by contr_eri): GA = J[PA+PB] - K[PA] and GB
    likewise with PB.  At cutoff 0 no quartet and no primitive is skipped."""
    n = PA.shape[0]
    with tempfile.TemporaryDirectory() as d:
        pa = os.path.join(d, "pa.bin"); np.ascontiguousarray(PA, dtype=np.float64).tofile(pa)
        pb = "-"
        if PB is not None:
            pb = os.path.join(d, "pb.bin"); np.ascontiguousarray(PB, dtype=np.float64).tofile(pb)
        out = os.path.join(d, "out.bin")
        ref_run(["nosymm", xyz_path, basis_path, pa, pb, "%.17g" % cutoff, out])
        m = np.fromfile(out, dtype=np.float64).reshape(2, n, n)
    return m[0], m[1]


def ref_jkseq(xyz_path, basis_path, densities, cutoffs, scf_cutoff=1e-10, max_mem=250):
    """Visits of one reference SCF (sqref jkseq): after a reset, one restricted
    GTO_JK_Matrix_Quartet_Parallel per (density, fixedCutoff), its cached state carried from
    visit to visit.  Returns a list of (JT, KA) per visit."""
    n = densities[0].shape[0]
    with tempfile.TemporaryDirectory() as d:
        args = ["jkseq", xyz_path, basis_path, 1, "%.17g" % scf_cutoff, max_mem, os.path.join(d, "out.bin")]
        for v, (P, c) in enumerate(zip(densities, cutoffs)):
            pth = os.path.join(d, "p%d.bin" % v)
            np.ascontiguousarray(P, dtype=np.float64).tofile(pth)
            args += [pth, "%.17g" % c]
        ref_run(args)
        m = np.fromfile(os.path.join(d, "out.bin")).reshape(len(densities), 3, n, n)
    return [(m[v, 0], m[v, 1]) for v in range(len(densities))]


def ref_scf(xyz_path, basis_path, options=()):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "dens.bin")
        res = ref_run(["scf", xyz_path, basis_path, out] + list(options))
        n = int(res["nbf"])
        m = np.fromfile(out, dtype=np.float64).reshape(2, n, n)
    return res, m[0], m[1]


def ref_schwarz(xyz_path, basis_path, n):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "s.bin")
        ref_run(["schwarz", xyz_path, basis_path, out])
        return np.fromfile(out, dtype=np.float64).reshape(n, n)


def ref_oneint(xyz_path, basis_path, n):
    """S, T, V of the reference's uhf() set-up (GTO_overlap/GTO_kinetic/GTO_nuclei)."""
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "stv.bin")
        ref_run(["oneint", xyz_path, basis_path, out])
        m = np.fromfile(out, dtype=np.float64).reshape(3, n, n)
        return m[0], m[1], m[2]


def ref_force(xyz_path, basis_path, options=()):
    """Forces (natom, 3) of the reference's uhf_force after uhf(), and the energy."""
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "f.bin")
        res = ref_run(["force", xyz_path, basis_path, out] + list(options))
        F = np.fromfile(out, dtype=np.float64).reshape(3, -1).T
    return F, res
