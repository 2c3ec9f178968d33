"""The drop-in: the reference program itself (uhf(), src/uhf.c:1171) relinked so its Fock build
(GTO_JK_Matrix_Quartet_Parallel, src/matrix.c:3773) runs on the GPU through
siam-quantum_b200/csrc/shim/sq_jk_gpu.c.  Whole SCF energies must match the reference's to
1e-8 Eh (plain FP64 bar) with the reference's 1STEP cutoff schedule."""
import os
import subprocess
import tempfile

import pytest

from conftest import GOLDEN_CASES, ROOT, golden, load_oracle, load_sqb200

port = load_oracle()
SQREF_GPU = os.path.join(ROOT, "oracle", "_ref", "sqref_b200")


def _run(binary, atoms, basis_name, opts, env=None):
    sqb = load_sqb200()
    with tempfile.TemporaryDirectory() as d:
        xyz = os.path.join(d, "m.xyz")
        with open(xyz, "w") as f:
            f.write(sqb.molecules.xyz_text([(int(a[0]), a[1], a[2], a[3]) for a in atoms]))
        bas = os.path.join(d, "basis.txt")
        with open(bas, "w") as f:
            f.write(sqb.basis.gamess_text(basis_name, [int(a[0]) for a in atoms]))
        r = subprocess.run([binary, "scf", xyz, bas, "-"] + list(opts), capture_output=True,
                           text=True, timeout=600, env=None if env is None else dict(os.environ, **env))
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        for line in r.stderr.splitlines():
            if line.startswith("RESULT"):
                return float(dict(kv.split("=") for kv in line.split()[1:])["energy"])
    raise AssertionError("no energy reported")


def test_gamess_writer_reproduces_reference_energy():
    """The basis text our package writes gives the reference the very same energy as its own
    basis file (so the drop-in tests feed both programs identical input)."""
    if not port.ref_available():
        pytest.skip("oracle/_ref not built")
    g = golden("water_321g")
    e = _run(port.REF_BIN, g["atoms"], str(g["basis"]), ["-SCFACC=1STEP", "-SCFCONV=1e-8"])
    assert e == float(g["energy"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_dropin_scf_energy_matches_reference(case):
    g = golden(case)
    e = _run(SQREF_GPU, g["atoms"], str(g["basis"]), ["-SCFACC=1STEP", "-SCFCONV=1e-8"])
    assert abs(e - float(g["energy"])) <= 1e-8, (e, float(g["energy"]))


@pytest.mark.gpu
def test_dropin_default_schedule_close_to_reference():
    """Default 3STEP schedule with exact quartets (the drop-in's default): the reference
    substitutes monopole approximations for some uncached quartets on later visits, which the
    GPU path then evaluates exactly, so agreement is checked at 1e-7 Eh."""
    g = golden("h2co_631gs")
    e_ref = _run(port.REF_BIN, g["atoms"], str(g["basis"]), ["-SCFCONV=1e-8"])
    e_gpu = _run(SQREF_GPU, g["atoms"], str(g["basis"]), ["-SCFCONV=1e-8"])
    assert abs(e_ref - e_gpu) <= 1e-7, (e_ref, e_gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
@pytest.mark.parametrize("maxmem", [None, "0"])
def test_dropin_default_schedule_multipole_mode_matches_reference(case, maxmem):
    """Default 3STEP schedule with the reference-parity multipole mode (SQB200_MULTIPOLE=1):
    the GPU takes the same monopole substitutions as the reference, so the energies agree at
    the plain-FP64 bar, 1e-8 Eh, with the default in-memory cache and without one."""
    g = golden(case)
    opts = ["-SCFCONV=1e-8"] + (["-MAXMEM=" + maxmem] if maxmem else [])
    e_ref = _run(port.REF_BIN, g["atoms"], str(g["basis"]), opts)
    e_gpu = _run(SQREF_GPU, g["atoms"], str(g["basis"]), opts, env={"SQB200_MULTIPOLE": "1"})
    assert abs(e_ref - e_gpu) <= 1e-8, (case, maxmem, e_ref, e_gpu)
