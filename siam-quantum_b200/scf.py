"""Device-resident RHF/UHF SCF around the GPU Fock build (the SCF tail of the reference's uhf(),
src/uhf.c:1171-1964, kept on the GPU).

Per job all matrices (S, H, densities, J/K, Fock, DIIS history) live on the device in FP64 and
every step runs on the job's own CUDA stream.  Each iteration builds J/K from the *difference*
density with the reference's screening semantics (uhf.c:1594-1611 accumulates dJT/dKA/dKB the
same way), forms F = H + JT + K, extrapolates with Pulay DIIS on the commutator FDS - SDF, and
diagonalises in an orthonormal basis with a cuSOLVER FP64 eigensolver (torch.linalg.eigh).
Conventions follow the reference: KA = -K[PA]; E = Enn + sum PT.H + 1/2 sum PT.JT
+ 1/2 sum (PA.KA + PB.KB) (uhf_getEtotal, src/uhf.c:222-315); the integral cutoff is the 1STEP
rule SCFConv / (nEA^2 + nEA nEB + nEB^2) / 50 evaluated on the identity-diagonal guess
(src/uhf.c:1384-1399, 1465-1472); nEA/nEB from the multiplicity as get_nEA/get_nEB (src/mol.c).
The first build reproduces the reference's first visit (no density screen above the memory
cutoff); later builds screen every quartet by the difference density, as its direct mode.
"""
import contextlib
import math
import time

import numpy as np

from . import basis as B
from . import molecules as M
from .engine import JKEngine


def electrons(atoms, charge=0, mult=None):
    """(nEA, nEB, multiplicity); multiplicity defaults to singlet/doublet by parity."""
    ne = sum(int(round(a[0])) for a in atoms) - charge
    if mult is None:
        mult = 1 if ne % 2 == 0 else 2
    nea = (ne + mult - 1) // 2
    neb = ne - nea
    if nea - neb != mult - 1 or neb < 0:
        raise ValueError("inconsistent charge/multiplicity")
    return nea, neb, mult


def nuclear_repulsion(atoms_bohr):
    e = 0.0
    for i in range(len(atoms_bohr)):
        for j in range(i):
            zi, *ri = atoms_bohr[i]
            zj, *rj = atoms_bohr[j]
            e += zi * zj / math.dist(ri, rj)
    return e


class SCFJob:
    """One molecule's SCF state, resident on one device.

    `engine` may supply the J/K engine (anything with nbf, oneint, mem_cutoff, set_precision,
    build_tensors and close, e.g. a JKEngine made earlier); by default a JKEngine is created
    on `device` for the job's basis."""

    def __init__(self, atoms_angstrom, basis_name, charge=0, mult=None, restricted=None,
                 scf_conv=1e-8, device=0, fp32_below=0.0, engine=None, diis_size=8):
        import torch
        self.torch = torch
        self.dev = device if isinstance(device, torch.device) else torch.device("cuda", device)
        self.stream = torch.cuda.Stream(self.dev) if self.dev.type == "cuda" else None
        atoms_angstrom = [(int(round(a[0])), float(a[1]), float(a[2]), float(a[3])) for a in atoms_angstrom]
        self.atoms = M.to_bohr(atoms_angstrom)
        self.basis = B.build_basis(self.atoms, basis_name)
        self.nea, self.neb, self.mult = electrons(atoms_angstrom, charge, mult)
        self.restricted = (self.mult == 1) if restricted is None else bool(restricted)
        if self.restricted and self.nea != self.neb:
            raise ValueError("restricted SCF needs a closed shell")
        self.scf_conv = scf_conv
        self.diis_size = diis_size
        self.eng = engine if engine is not None else JKEngine(self.basis, device=self.dev.index)
        if fp32_below > 0:
            self.eng.set_precision(fp32_below)
        n = self.n = self.basis.nbf
        if self.eng.nbf != n:
            raise ValueError("engine basis has %d functions, job basis %d" % (self.eng.nbf, n))
        Z = np.array([a[0] for a in self.atoms], dtype=np.float64)
        XYZ = np.array([a[1:] for a in self.atoms], dtype=np.float64)
        S, T, V = self.eng.oneint(Z, XYZ)
        self.enn = nuclear_repulsion(self.atoms)
        sa, sb = self.nea, self.neb                  # sums of the identity-diagonal guess
        self.cutoff = scf_conv / (sa * sa + sa * sb + sb * sb) / 50.0
        self.rmax_first = self.eng.mem_cutoff(self.cutoff, 250)
        with self._on_stream():
            f64 = dict(dtype=torch.float64, device=self.dev)
            self.S = torch.tensor(S, **f64)
            self.H = torch.tensor(T + V, **f64)
            w, U = torch.linalg.eigh(self.S)
            self.X = U * w.rsqrt()                   # canonical orthogonaliser: X^T S X = 1
            tr = float(torch.trace(self.S))
            eye = torch.eye(n, **f64)
            self.PA = eye * (self.nea / tr)
            self.PB = eye * (self.neb / tr)
            z = lambda: torch.zeros((n, n), **f64)
            self.JT, self.KA, self.KB = z(), z(), z()
            self.dJT, self.dKA, self.dKB = z(), z(), z()
            self.PA_old, self.PB_old = z(), z()
        self.diis_F, self.diis_E = [], []
        self.energy, self.iters, self.converged, self.dE = None, 0, False, None
        self.emax = self.dP = None
        self.first = True
        self.seconds = 0.0

    def _on_stream(self):
        if self.stream is None:
            return contextlib.nullcontext()
        return self.torch.cuda.stream(self.stream)

    # -------------------------------------------------------------- pieces of an iteration
    def build_jk(self):
        """Enqueue J/K of the difference density on the job's stream."""
        with self._on_stream():
            self._dA = (self.PA - self.PA_old).contiguous()
            self._dB = self._dA if self.restricted else (self.PB - self.PB_old).contiguous()
            self.eng.build_tensors(self._dA, self._dB, self.dJT, self.dKA,
                                   None if self.restricted else self.dKB,
                                   restricted=self.restricted, scf_cutoff=self.cutoff,
                                   fixed_cutoff=self.cutoff,
                                   dscreen_rmax=self.rmax_first if self.first else float("inf"),
                                   stream=self.stream)
        self.first = False

    def _density(self, F, nocc):
        Fo = self.X.T @ F @ self.X
        _, C = self.torch.linalg.eigh(Fo)
        C = self.X @ C[:, :nocc]
        return C @ C.T

    def _diis(self, FA, FB, err):
        torch = self.torch
        self.diis_F.append((FA, FB))
        self.diis_E.append(err)
        if len(self.diis_F) > self.diis_size:
            self.diis_F.pop(0)
            self.diis_E.pop(0)
        m = len(self.diis_F)
        if m < 2:
            return FA, FB
        E = torch.stack([e.reshape(-1) for e in self.diis_E])
        Bm = torch.zeros((m + 1, m + 1), dtype=torch.float64, device=self.dev)
        Bm[:m, :m] = E @ E.T
        # scale for conditioning: the solution's coefficients do not change
        Bm[:m, :m] /= Bm[:m, :m].diagonal().max().clamp_min(1e-300)
        Bm[m, :m] = -1.0
        Bm[:m, m] = -1.0
        rhs = torch.zeros((m + 1, 1), dtype=torch.float64, device=self.dev)
        rhs[m, 0] = -1.0
        c = (torch.linalg.pinv(Bm) @ rhs)[:m, 0]
        FA = torch.einsum("k,kij->ij", c, torch.stack([f[0] for f in self.diis_F]))
        FB = FA if self.restricted else torch.einsum("k,kij->ij", c, torch.stack([f[1] for f in self.diis_F]))
        return FA, FB

    def update(self):
        """After build_jk: accumulate J/K, energy, DIIS, new densities (on the job's stream).
        Returns True when converged (|dE| < SCFConv/100, max |commutator| < 1e-6 and
        max |dP| < 1e-6)."""
        torch = self.torch
        with self._on_stream():
            self.JT += self.dJT
            self.KA += self.dKA
            if self.restricted:
                self.KB = self.KA
            else:
                self.KB += self.dKB
            self.PA_old, self.PB_old = self.PA, self.PB
            FA = self.H + self.JT + self.KA
            FB = FA if self.restricted else self.H + self.JT + self.KB
            PT = self.PA + self.PB
            e_t = ((PT * self.H).sum() + 0.5 * (PT * self.JT).sum()
                   + 0.5 * ((self.PA * self.KA).sum() + (self.PB * self.KB).sum()))
            errA = FA @ self.PA @ self.S
            errA = errA - errA.T
            if self.restricted:
                err = errA
            else:
                errB = FB @ self.PB @ self.S
                err = torch.cat([errA, errB - errB.T])
            emax_t = err.abs().max()
            FA, FB = self._diis(FA, FB, err)
            self.PA = self._density(FA, self.nea)
            self.PB = self.PA if self.restricted else self._density(FB, self.neb)
            dP_t = (self.PA - self.PA_old).abs().max()
            E, emax, dP = (float(v) for v in torch.stack([e_t, emax_t, dP_t]).cpu())
        E += self.enn
        self.dE = None if self.energy is None else E - self.energy
        self.energy = E
        self.iters += 1
        self.emax, self.dP = emax, dP
        self.converged = (self.dE is not None and abs(self.dE) < 0.01 * self.scf_conv
                          and emax < 1e-6 and dP < 1e-6)
        return self.converged

    def run(self, max_iter=100):
        t0 = time.perf_counter()
        while self.iters < max_iter:
            self.build_jk()
            if self.update():
                break
        if self.stream is not None:
            self.stream.synchronize()
        self.seconds = time.perf_counter() - t0
        return self.energy

    def close(self):
        self.eng.close()


def scf_energy(atoms_angstrom, basis_name, **kw):
    """Converged SCF energy (Eh) and the finished job."""
    job = SCFJob(atoms_angstrom, basis_name, **kw)
    try:
        return job.run(), job
    finally:
        job.close()
