"""Device-resident RHF/UHF SCF around the GPU Fock build (the SCF tail of the reference's uhf(),
src/uhf.c:1171-1964, kept on the GPU).

Per job all matrices (S, H, densities, J/K, Fock, DIIS history) live on the device in FP64 and
every step runs on the job's own CUDA stream.  The loop is the reference's (src/uhf.c:1591-1783)
with its defaults: J/K of the *difference* density accumulated into JT/KA/KB, F = H + JT + K,
new densities from the lowest orbitals (a cuSOLVER FP64 eigensolve in an S-orthonormal basis in
place of gen_sym_SomeEigen), the energy of those densities with the accumulated J/K, then the
reference's 4-point density DIIS (conv_diis4, drag 0.25); converged when |dE| and the RMS
density change are both <= SCFConv, at most 80 iterations.
Conventions: KA = -K[PA]; E = Enn + sum PT.H + 1/2 sum PT.JT
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
from .engine import JKEngine, syev_batched


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


SCF_DRAG = 0.25     # reference default -SCFDRAG (src/option.c:526)
SCF_MAX = 80        # reference default -SCFMAX (src/option.c:527)


class DensityDIIS4:
    """The reference's 4-point density DIIS, conv_diis4 (src/conv.c:606-844), applied to many
    independent molecules at once.

    Densities are flat vectors holding every molecule's alpha and beta blocks; `seg` gives the
    molecule of each element, `nbf2` each molecule's nbf^2.  Per molecule, as the reference:
    the residual of a step is d = P_new - P_in (P_in = the previous step's output); the first
    three steps return the damped mix alpha P_new + (1 - alpha) P_in; later steps solve the
    5 x 5 DIIS system on the last four residuals (B_xy = sum over both spins of d_x . d_y, rows
    bordered by -1) and return sum_k c_k (P_in,k + d_k), falling back to the damped mix when the
    newest residual grew (B33 > B22).  The RMS deviation sqrt(sum d^2 / nbf^2 / 2) is what
    the reference tests against SCFConv.

    On the GPU the per-molecule sums come from the library's segmented dot products
    (engine.SegmentDots: the ten B entries in one pass, fixed summation order); `segments` =
    (starts, lengths, slots) lists the contiguous runs of the flat vectors and the molecule
    each belongs to.  On the CPU (host-logic tests) they are index_add_ sums over `seg`."""

    PAIRS = [(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]

    def __init__(self, torch, P, seg, nseg, nbf2, alpha=SCF_DRAG, segments=None):
        self.torch = torch
        self.seg, self.nseg, self.alpha = seg, nseg, alpha
        self.nbf2 = nbf2.to(P.dtype)
        self.Pin = [torch.zeros_like(P) for _ in range(3)] + [P.clone()]   # P0, P1, P2, P3
        self.d = [torch.zeros_like(P) for _ in range(4)]                      # dP0 .. dP3
        self.n = 1                                                            # nIter after the first call
        self.dots = None
        if P.is_cuda:
            if segments is None:
                raise ValueError("DensityDIIS4 on the GPU needs the segments of the packed densities")
            from .engine import SegmentDots
            self.dots = SegmentDots(*segments, nseg, P.device.index)

    def _segsum(self, x):
        torch = self.torch
        return torch.zeros(self.nseg, dtype=x.dtype, device=x.device).index_add_(0, self.seg, x)

    def _sums(self, ds, pairs):
        """{(x, y): per-molecule sum of ds[x] * ds[y]}."""
        if self.dots is not None:
            S = self.dots(ds, pairs)
            return {xy: S[:, k] for k, xy in enumerate(pairs)}
        return {xy: self._segsum(ds[xy[0]] * ds[xy[1]]) for xy in pairs}

    def step(self, Pnew):
        """(the next input density, RMS deviation per molecule)."""
        torch = self.torch
        P0, P1, P2, P3 = self.Pin
        d3 = Pnew - P3
        d0, d1, d2 = self.d[0], self.d[1], self.d[2]
        a = self.alpha
        if self.n <= 3:
            avg = torch.sqrt(self._sums([d3], [(0, 0)])[(0, 0)] / self.nbf2 / 2.0)
            out = a * Pnew + (1.0 - a) * P3
        else:
            ds = [d0, d1, d2, d3]
            Bv = self._sums(ds, self.PAIRS)
            avg = torch.sqrt(Bv[(3, 3)] / self.nbf2 / 2.0)
            A = torch.zeros((self.nseg, 5, 5), dtype=Pnew.dtype, device=Pnew.device)
            for (x, y), v in Bv.items():
                A[:, x, y] = v
                A[:, y, x] = v
            A[:, 4, :4] = -1.0
            A[:, :4, 4] = -1.0
            rhs = torch.zeros((self.nseg, 5, 1), dtype=Pnew.dtype, device=Pnew.device)
            rhs[:, 4, 0] = -1.0
            c, info = torch.linalg.solve_ex(A, rhs)
            c = c[:, :4, 0]
            damp = (Bv[(3, 3)] > Bv[(2, 2)]) | (info != 0) | ~torch.isfinite(c).all(dim=1)
            cd = torch.tensor([0.0, 0.0, 1.0 - a, a], dtype=Pnew.dtype, device=Pnew.device)
            c = torch.where(damp[:, None], cd[None, :], c)
            cs = c[self.seg]                                                  # per element
            out = (cs[:, 3] * Pnew + cs[:, 2] * (P2 + d2) + cs[:, 1] * (P1 + d1) + cs[:, 0] * (P0 + d0))
        self.d = [d1, d2, d3, None]          # d0 <- d1, d1 <- d2, d2 <- d3
        self.Pin = [P1, P2, P3, out]
        self.n += 1
        return out, avg


class SCFJob:
    """One molecule's SCF state, resident on one device.

    `engine` may supply the J/K engine (anything with nbf, oneint, mem_cutoff, set_precision,
    build_tensors and close, e.g. a JKEngine made earlier); by default a JKEngine is created
    on `device` for the job's basis."""

    def __init__(self, atoms_angstrom, basis_name, charge=0, mult=None, restricted=None,
                 scf_conv=1e-8, device=0, fp32_below=0.0, engine=None, guess=None):
        """`guess`: None for the reference's identity-diagonal guess, or a checkpoint (a path or
        the dict of checkpoint.read_checkpoint) whose orbitals are projected onto this basis as
        the reference's -GUESS=CHECK does."""
        import torch
        self.torch = torch
        self.dev = device if isinstance(device, torch.device) else torch.device("cuda", device)
        self.stream = torch.cuda.Stream(self.dev) if self.dev.type == "cuda" else None
        atoms_angstrom = [(int(round(a[0])), float(a[1]), float(a[2]), float(a[3])) for a in atoms_angstrom]
        self.atoms = M.to_bohr(atoms_angstrom)
        self.basis = B.build_basis(self.atoms, basis_name)
        self.nea, self.neb, self.mult = electrons(atoms_angstrom, charge, mult)
        self.charge = charge
        self.restricted = (self.mult == 1) if restricted is None else bool(restricted)
        if self.restricted and self.nea != self.neb:
            raise ValueError("restricted SCF needs a closed shell")
        self.scf_conv = scf_conv
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
        PAg = PBg = None
        if guess is not None:
            from . import checkpoint as CK
            chk = CK.read_checkpoint(guess) if isinstance(guess, str) else guess
            if [int(a[0]) for a in chk["atoms"]] != [int(a[0]) for a in self.atoms]:
                raise ValueError("checkpoint holds a different molecule")
            CA, CB = CK.project_orbitals(chk, self.basis, S)
            PAg = CA[:self.nea].T @ CA[:self.nea]
            PBg = CB[:self.neb].T @ CB[:self.neb]
            sa, sb = float(PAg.sum()), float(PBg.sum())
        else:
            sa, sb = self.nea, self.neb              # sums of the identity-diagonal guess
        # the reference's cutoff rule on the sums of all guess-density elements (src/uhf.c:1465-1472)
        self.cutoff = scf_conv / (sa * sa + sa * sb + sb * sb) / 50.0
        self.rmax_first = self.eng.mem_cutoff(self.cutoff, 250)
        with self._on_stream():
            f64 = dict(dtype=torch.float64, device=self.dev)
            self.S = torch.tensor(S, **f64)
            self.H = torch.tensor(T + V, **f64)
            w, U = torch.linalg.eigh(self.S)
            self.X = U * w.rsqrt()                   # canonical orthogonaliser: X^T S X = 1
            if PAg is not None:
                self.PA = torch.tensor(PAg, **f64)
                self.PB = torch.tensor(PBg, **f64)
            else:
                tr = float(torch.trace(self.S))
                eye = torch.eye(n, **f64)
                self.PA = eye * (self.nea / tr)
                self.PB = eye * (self.neb / tr)
            z = lambda: torch.zeros((n, n), **f64)
            self.JT, self.KA, self.KB = z(), z(), z()
            self.dJT, self.dKA, self.dKB = z(), z(), z()
            self.PA_old, self.PB_old = z(), z()
        self.diis = None
        self.energy, self.iters, self.converged, self.dE = None, 0, False, None
        self.avgdP = None
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
        if self.dev.type == "cuda":
            # cuSOLVER without a host synchronisation (torch.linalg.eigh checks its status on
            # the host), so that several jobs' steps can be in flight at once
            _, C = syev_batched(Fo.unsqueeze(0), stream=self.stream)
            C = C[0]
        else:
            _, C = self.torch.linalg.eigh(Fo)
        C = self.X @ C[:, :nocc]
        return C @ C.T

    def update_launch(self):
        """Enqueue, after build_jk, one step of the reference's loop (src/uhf.c:1600-1730):
        accumulate J/K, Fock, new densities from the lowest orbitals, the energy of those
        densities with the accumulated J/K, then conv_diis4.  Nothing is read back."""
        torch = self.torch
        n = self.n
        with self._on_stream():
            self.JT += self.dJT
            self.KA += self.dKA
            if self.restricted:
                self.KB = self.KA
            else:
                self.KB += self.dKB
            self.PA_old, self.PB_old = self.PA, self.PB
            FA = self.H + self.JT + self.KA
            self.FA = FA
            self.FB = FA if self.restricted else self.H + self.JT + self.KB
            PA = self._density(FA, self.nea)
            PB = PA if self.restricted else self._density(self.FB, self.neb)
            e_t = (((self.H + 0.5 * self.JT) * (PA + PB)).sum()
                   + 0.5 * ((self.KA * PA).sum() + (self.KB * PB).sum()))
            if self.diis is None:
                self.diis = DensityDIIS4(torch, torch.cat([self.PA.reshape(-1), self.PB.reshape(-1)]),
                                         torch.zeros(2 * n * n, dtype=torch.int64, device=self.dev), 1,
                                         torch.tensor([n * n], device=self.dev),
                                         segments=([0], [2 * n * n], [0]))
            out, avg = self.diis.step(torch.cat([PA.reshape(-1), PB.reshape(-1)]))
            self.PA = out[:n * n].view(n, n)
            self.PB = self.PA if self.restricted else out[n * n:].view(n, n)
            self._pending = torch.stack([e_t, avg[0]])

    def update_finish(self):
        """Read the step's energy and RMS density change (synchronises the job's stream) and
        apply the reference's test: True when |dE| <= SCFConv and RMS dP <= SCFConv."""
        with self._on_stream():
            E, avgdP = (float(v) for v in self._pending.cpu())
        E += self.enn
        self.dE = E - (0.0 if self.energy is None else self.energy)
        self.energy = E
        self.iters += 1
        self.avgdP = avgdP
        self.converged = abs(self.dE) <= self.scf_conv and avgdP <= self.scf_conv
        return self.converged

    def update(self):
        """update_launch + update_finish."""
        self.update_launch()
        return self.update_finish()

    def run(self, max_iter=SCF_MAX):
        t0 = time.perf_counter()
        while self.iters < max_iter:
            self.build_jk()
            if self.update():
                break
        if self.stream is not None:
            self.stream.synchronize()
        self.seconds = time.perf_counter() - t0
        return self.energy

    def orbitals(self):
        """All orbitals and orbital energies of the last Fock matrices, as the reference saves
        them after its loop (gen_sym_eigen + normalizeC, src/uhf.c:1840-1843): (CA, CB, eA, eB)
        as numpy arrays, orbital i in row i."""
        out = []
        for F in (self.FA, self.FB):
            # the copies to the host run on the job's stream, after the products they read
            # (the default stream is not ordered after it)
            with self._on_stream():
                w, C = self.torch.linalg.eigh(self.X.T @ F @ self.X)
                C = (self.X @ C).T
                out.append((C.cpu().numpy(), w.cpu().numpy()))
        return out[0][0], out[1][0], out[0][1], out[1][1]

    def gradient(self, terms=15):
        """Nuclear gradient (natom, 3), hartree/bohr, of the converged SCF energy, as the
        reference's uhf_force (src/grad.c:2155) forms it after uhf(): densities and the
        energy-weighted density from the orbitals of the last Fock matrices."""
        CA, CB, eA, eB = self.orbitals()
        ca, cb = CA[:self.nea], CB[:self.neb]
        PA = ca.T @ ca
        PB = cb.T @ cb
        W = (ca.T * eA[:self.nea]) @ ca + (cb.T * eB[:self.neb]) @ cb
        Z = np.array([a[0] for a in self.atoms], dtype=np.float64)
        XYZ = np.array([a[1:] for a in self.atoms], dtype=np.float64)
        return self.eng.gradient(Z, XYZ, PA, PB, W, terms)

    def save_checkpoint(self, path):
        """Write the reference's checkpoint file (-SCHECK) for this job."""
        from . import checkpoint as CK
        CA, CB, eA, eB = self.orbitals()
        CK.write_checkpoint(path, self.atoms, self.charge, self.mult, self.basis, self.energy,
                            self.dE if self.dE is not None else 0.0,
                            self.avgdP if self.avgdP is not None else 0.0, CA, CB, eA, eB)

    def close(self):
        if self.diis is not None and self.diis.dots is not None:
            self.diis.dots.close()
        self.eng.close()


def scf_energy(atoms_angstrom, basis_name, **kw):
    """Converged SCF energy (Eh) and the finished job."""
    job = SCFJob(atoms_angstrom, basis_name, **kw)
    try:
        return job.run(), job
    finally:
        job.close()
