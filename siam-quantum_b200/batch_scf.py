"""Batched RHF/UHF SCF of many molecules on one device (uhf(), src/uhf.c:1171-1964, for a set
of independent molecules at once).

Every molecule's J/K comes from ONE batched Fock build per iteration (sqb200_batch_*: one
launch per class kernel over the work of all molecules), captured once as a CUDA graph and
replayed each iteration.  The SCF tail runs batched as well: molecules are grouped into buckets
of equal padded size (multiples of 32 functions); per bucket the Fock matrices, Pulay DIIS,
orthogonalisation, cuSOLVER FP64 eigensolves and densities are stacked tensor operations.  A
padded orbital gets a large diagonal shift so that it is never occupied.  Each molecule follows
the same conventions and cutoff rule as scf.SCFJob (difference-density builds, 1STEP cutoff
SCFConv / (nEA^2 + nEA nEB + nEB^2) / 50, first build without density screening above the
memory cutoff), so each converged energy is the single-molecule result.

Packed layout: molecule m's nbf_m x nbf_m block starts at offsets[m] of every packed array
(the batch's layout); spin-resolved arrays hold the alpha blocks in [0, total) and the beta
blocks in [total, 2 total), with one trailing zero used as the target of padded positions.
"""
import math
import time

import numpy as np

from . import basis as B
from . import molecules as M
from .engine import JKBatch, JKEngine
from .scf import electrons, nuclear_repulsion

PAD = 32            # bucket granularity (functions)
SHIFT = 1.0e4       # Fock shift of padded orbitals (Eh): above every occupied level


class _Bucket:
    """Spin rows (molecule, spin) of one padded size n and their stacked SCF state."""

    def __init__(self, torch, dev, n, rows, mols, total):
        self.n = n
        self.rows = rows                      # list of (molecule index, spin)
        R = len(rows)
        f64 = dict(dtype=torch.float64, device=dev)
        # flat gather index into a spin-packed array (2 * total + 1): padding -> trailing zero
        gi = np.full((R, n, n), 2 * total, dtype=np.int64)
        for r, (m, s) in enumerate(rows):
            mo = mols[m]
            k = mo["nbf"]
            base = mo["off"] + s * total
            gi[r, :k, :k] = base + np.arange(k * k).reshape(k, k)
        self.gidx = torch.tensor(gi.reshape(-1), device=dev)
        valid = gi.reshape(-1) < 2 * total
        self.sidx = torch.tensor(gi.reshape(-1)[valid], device=dev)       # scatter targets
        self.svalid = torch.tensor(np.nonzero(valid)[0], device=dev)      # their stack positions
        self.mol = torch.tensor([m for m, _ in rows], device=dev)
        self.nocc = torch.tensor([mols[m]["nocc"][s] for m, s in rows], device=dev)
        # occupied-column mask and the padding shift
        cols = torch.arange(n, device=dev)
        self.occ = (cols[None, :] < self.nocc[:, None]).to(torch.float64)          # (R, n)
        pad = np.zeros((R, n))
        for r, (m, s) in enumerate(rows):
            pad[r, mols[m]["nbf"]:] = SHIFT
        self.shift = torch.diag_embed(torch.tensor(pad, **f64))
        # orthogonaliser X (padded with zeros) and S per row
        X = np.zeros((R, n, n))
        S = np.zeros((R, n, n))
        for r, (m, s) in enumerate(rows):
            k = mols[m]["nbf"]
            X[r, :k, :k] = mols[m]["X"]
            S[r, :k, :k] = mols[m]["S"]
        self.X = torch.tensor(X, **f64)
        self.S = torch.tensor(S, **f64)
        self.hF, self.hE = [], []             # DIIS history (stacked per iteration)


class BatchSCF:
    """Solve many molecules together.  `jobs` is a list of dicts with keys atoms (angstrom),
    basis, and optionally charge, mult, restricted."""

    def __init__(self, jobs, device=0, scf_conv=1e-8, fp32_below=0.0, diis_size=8, graph=True,
                 autotune=True):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(self.dev)
        self.scf_conv = scf_conv
        self.diis_size = diis_size
        self.use_graph = graph
        self.autotune = autotune
        self.mols = []
        self.engines = []
        t0 = time.perf_counter()
        for j in jobs:
            atoms = [(int(round(a[0])), float(a[1]), float(a[2]), float(a[3])) for a in j["atoms"]]
            ab = M.to_bohr(atoms)
            bas = B.build_basis(ab, j["basis"])
            nea, neb, mult = electrons(atoms, j.get("charge", 0), j.get("mult"))
            restricted = j.get("restricted", mult == 1)
            if restricted and nea != neb:
                raise ValueError("restricted SCF needs a closed shell")
            eng = JKEngine(bas, device=device)
            if fp32_below > 0:
                eng.set_precision(fp32_below)
            Z = np.array([a[0] for a in ab], dtype=np.float64)
            XYZ = np.array([a[1:] for a in ab], dtype=np.float64)
            S, T, V = eng.oneint(Z, XYZ)
            w, U = np.linalg.eigh(S)
            cut = scf_conv / (nea * nea + nea * neb + neb * neb) / 50.0
            self.mols.append({"nbf": bas.nbf, "nocc": (nea, neb), "restricted": bool(restricted),
                              "S": S, "H": T + V, "X": U / np.sqrt(w), "enn": nuclear_repulsion(ab),
                              "cutoff": cut, "rmax": eng.mem_cutoff(cut, 250)})
            self.engines.append(eng)
        self.setup_seconds = time.perf_counter() - t0
        self.batch = JKBatch(self.engines)
        off = self.batch.offsets
        self.total = T_ = self.batch.total
        for m, mo in enumerate(self.mols):
            mo["off"] = off[m]
        nm = len(self.mols)
        f64 = dict(dtype=torch.float64, device=self.dev)
        with torch.cuda.stream(self.stream):
            # spin-packed state (2T + 1): alpha blocks, beta blocks, trailing zero
            z = lambda: torch.zeros(2 * T_ + 1, **f64)
            self.P, self.Pold = z(), z()
            self.dP = z()
            self.K = z()                       # accumulated KA | KB
            self.dK = z()                      # build output KA | KB
            self.JT = torch.zeros(T_, **f64)
            self.dJT = torch.zeros(T_, **f64)
            self.H = torch.zeros(T_, **f64)
            molid = np.zeros(T_, dtype=np.int64)
            Ph = np.zeros(2 * T_ + 1)
            Hh = np.zeros(T_)
            for m, mo in enumerate(self.mols):
                k = mo["nbf"]
                o = mo["off"]
                molid[o:o + k * k] = m
                Hh[o:o + k * k] = mo["H"].reshape(-1)
                tr = float(np.trace(mo["S"]))
                eye = np.eye(k).reshape(-1)
                Ph[o:o + k * k] = eye * (mo["nocc"][0] / tr)
                Ph[T_ + o:T_ + o + k * k] = eye * (mo["nocc"][1] / tr)
            self.H.copy_(torch.tensor(Hh))
            self.P.copy_(torch.tensor(Ph))
            self.molid = torch.tensor(molid, device=self.dev)
            self.enn = torch.tensor([mo["enn"] for mo in self.mols], **f64)
            # buckets of spin rows by padded size (restricted molecules: alpha row only)
            groups = {}
            for m, mo in enumerate(self.mols):
                n = ((mo["nbf"] + PAD - 1) // PAD) * PAD
                for s in ((0,) if mo["restricted"] else (0, 1)):
                    groups.setdefault(n, []).append((m, s))
            self.buckets = [_Bucket(torch, self.dev, n, rows, self.mols, T_) for n, rows in sorted(groups.items())]
        self.restricted = np.array([mo["restricted"] for mo in self.mols])
        self.energy = np.full(nm, np.nan)
        self.dE = np.full(nm, np.inf)
        self.emax = np.full(nm, np.inf)
        self.dPmax = np.full(nm, np.inf)
        self.converged = np.zeros(nm, dtype=bool)
        self.iters = 0
        self.graph = None
        self.first = True
        self.build_seconds = 0.0

    # ------------------------------------------------------------------ the Fock build
    def _build(self):
        """dP -> dJT, dK on the job stream (a CUDA graph replay after the first two builds)."""
        T_ = self.total
        P, dP = self.P, self.dP
        ptr = lambda t, k: t.data_ptr() + 8 * k
        if self.graph is not None:
            self.graph.replay()
            return

        def body():
            self.torch.sub(self.P, self.Pold, out=self.dP)
            self.batch.build_device(ptr(dP, 0), ptr(dP, T_), self.dJT.data_ptr(), ptr(self.dK, 0),
                                    ptr(self.dK, T_), stream=self.stream.cuda_stream)
            self.JT += self.dJT
            self.K[:2 * T_] += self.dK[:2 * T_]

        if self.use_graph and not self.first and self._graph_ready:
            g = self.torch.cuda.CUDAGraph()
            with self.torch.cuda.graph(g, stream=self.stream):
                body()
            self.graph = g
            g.replay()
        else:
            body()

    def _set_step(self, first):
        cut = [mo["cutoff"] for mo in self.mols]
        rmax = [mo["rmax"] if first else float("inf") for mo in self.mols]
        self.batch.set_step(self.restricted, cut, cut, rmax)

    # ------------------------------------------------------------------ the SCF tail
    def _tail(self):
        torch = self.torch
        T_ = self.total
        nm = len(self.mols)
        # energies: E = Enn + sum PT.H + 1/2 sum PT.JT + 1/2 sum (PA.KA + PB.KB)
        PA, PB = self.P[:T_], self.P[T_:2 * T_]
        KA, KB = self.K[:T_], self.K[T_:2 * T_]
        PT = PA + PB
        dens = PT * (self.H + 0.5 * self.JT) + 0.5 * (PA * KA + PB * KB)
        E = torch.zeros(nm, dtype=torch.float64, device=self.dev).index_add_(0, self.molid, dens) + self.enn
        emax = torch.zeros(nm, dtype=torch.float64, device=self.dev)
        self.Pold.copy_(self.P)
        Fbase = torch.cat([self.H + self.JT, self.H + self.JT, torch.zeros(1, dtype=torch.float64, device=self.dev)])
        Ffull = Fbase + self.K
        newP = torch.zeros_like(self.P)
        for b in self.buckets:
            R, n = len(b.rows), b.n
            F = Ffull[b.gidx].view(R, n, n)
            D = self.P[b.gidx].view(R, n, n)
            e = F @ D @ b.S
            e = e - e.transpose(1, 2)
            emax.scatter_reduce_(0, b.mol, e.abs().amax(dim=(1, 2)), reduce="amax")
            # DIIS (common coefficients for the spin rows of one molecule)
            b.hF.append(F)
            b.hE.append(e)
            if len(b.hF) > self.diis_size:
                b.hF.pop(0)
                b.hE.pop(0)
            h = len(b.hF)
            if h >= 2:
                Es = torch.stack(b.hE, 1).reshape(R, h, -1)
                Brow = Es @ Es.transpose(1, 2)                                  # (R, h, h)
                Bm = torch.zeros((nm, h, h), dtype=torch.float64, device=self.dev).index_add_(0, b.mol, Brow)
                Bm = Bm[b.mol]                                                   # back to rows
                scale = Bm.diagonal(dim1=1, dim2=2).amax(dim=1).clamp_min(1e-300)
                A = torch.zeros((R, h + 1, h + 1), dtype=torch.float64, device=self.dev)
                A[:, :h, :h] = Bm / scale[:, None, None]
                A[:, h, :h] = -1.0
                A[:, :h, h] = -1.0
                rhs = torch.zeros((R, h + 1, 1), dtype=torch.float64, device=self.dev)
                rhs[:, h, 0] = -1.0
                c = (torch.linalg.pinv(A) @ rhs)[:, :h, 0]                        # (R, h)
                F = torch.einsum("rk,rkij->rij", c, torch.stack(b.hF, 1))
            Fo = b.X.transpose(1, 2) @ F @ b.X + b.shift
            _, C = torch.linalg.eigh(Fo)
            C = (b.X @ C) * b.occ[:, None, :]
            Dn = C @ C.transpose(1, 2)
            newP.index_copy_(0, b.sidx, Dn.reshape(-1)[b.svalid])
        # restricted molecules: beta = alpha
        rmask = torch.tensor(self.restricted, device=self.dev)[self.molid]
        newP[T_:2 * T_] = torch.where(rmask, newP[:T_], newP[T_:2 * T_])
        dPm = torch.zeros(nm, dtype=torch.float64, device=self.dev)
        dPm.scatter_reduce_(0, self.molid, (newP[:T_] - self.P[:T_]).abs(), reduce="amax")
        self.P.copy_(newP)
        return E, emax, dPm

    def run(self, max_iter=60):
        torch = self.torch
        t0 = time.perf_counter()
        self._graph_ready = False
        with torch.cuda.stream(self.stream):
            self._set_step(True)
            while self.iters < max_iter:
                tb = time.perf_counter()
                self._build()
                if self.first:
                    self.first = False
                    self._set_step(False)     # later builds: density screen everywhere
                elif not self._graph_ready:
                    self._graph_ready = True  # the next build is captured
                E, emax, dPm = self._tail()
                if self.iters == 0 and self.autotune:
                    # tile autotuner on the work of the difference-density builds that follow
                    T_ = self.total
                    torch.sub(self.P, self.Pold, out=self.dP)
                    self.batch.autotune(self.dP.data_ptr(), self.dP.data_ptr() + 8 * T_,
                                        stream=self.stream.cuda_stream)
                h = torch.stack([E, emax, dPm]).cpu().numpy()
                self.build_seconds += time.perf_counter() - tb
                E, emax, dPm = h
                self.dE = E - self.energy
                self.energy = E
                self.emax, self.dPmax = emax, dPm
                self.iters += 1
                conv = (np.abs(self.dE) < 0.01 * self.scf_conv) & (emax < 1e-6) & (dPm < 1e-6)
                self.converged = conv
                if conv.all():
                    break
        self.stream.synchronize()
        self.seconds = time.perf_counter() - t0
        return self.energy

    def close(self):
        self.graph = None
        self.batch.close()
        for e in self.engines:
            e.close()
