"""Batched RHF/UHF SCF of many molecules on one device (uhf(), src/uhf.c:1171-1964, for a set
of independent molecules at once).

Every molecule's J/K comes from ONE batched Fock build per iteration (sqb200_batch_*: one
launch per class kernel over the work of all molecules), captured once as a CUDA graph and
replayed each iteration.  The SCF tail runs batched as well: molecules are grouped into buckets
of equal padded size (multiples of 32 functions); per bucket the Fock matrices,
orthogonalisation, cuSOLVER FP64 eigensolves and densities are stacked tensor operations (a
padded orbital gets a large diagonal shift so that it is never occupied), and the reference's
density DIIS runs on the packed densities of all molecules at once.  Each molecule follows the
loop, conventions and cutoff rule of scf.SCFJob (the reference's uhf() loop with its defaults:
difference-density builds, 1STEP cutoff, conv_diis4, convergence on |dE| and the RMS density
change); a molecule that has converged keeps its density while the others continue.

Packed layout: molecule m's nbf_m x nbf_m block starts at offsets[m] of every packed array
(the batch's layout); spin-resolved arrays hold the alpha blocks in [0, total) and the beta
blocks in [total, 2 total), with one trailing zero used as the target of padded positions.
"""
import math
import time

import numpy as np

from . import basis as B
from . import molecules as M
from .engine import JKBatch, JKEngine, SegmentDots, syev_batched
from .scf import SCF_MAX, DensityDIIS4, electrons, nuclear_repulsion

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
        self.gidx2 = self.gidx.view(R, n * n)
        self.mol_np = np.array([m for m, _ in rows], dtype=np.int64)
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


class BatchSCF:
    """Solve many molecules together.  `jobs` is a list of dicts with keys atoms (angstrom),
    basis, and optionally charge, mult, restricted."""

    def __init__(self, jobs, device=0, scf_conv=1e-8, fp32_below=0.0, graph=True, autotune=True):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(self.dev)
        self.scf_conv = scf_conv
        self.use_graph = graph
        self.autotune = autotune
        self._tuned = False
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
            self.P0 = self.P.clone()
            self.molid = torch.tensor(molid, device=self.dev)
            self.molid2 = torch.cat([self.molid, self.molid])
            # per-molecule sums over the packed blocks (energy): one pass, fixed order
            self.edots = SegmentDots([mo["off"] for mo in self.mols], [mo["nbf"] ** 2 for mo in self.mols],
                                     list(range(nm)), nm, self.dev.index)
            self.nbf2 = torch.tensor([mo["nbf"] ** 2 for mo in self.mols], device=self.dev)
            self.rmask = torch.tensor([mo["restricted"] for mo in self.mols], device=self.dev)[self.molid]
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
        self.avgdP = np.full(nm, np.inf)
        self.converged = np.zeros(nm, dtype=bool)
        self.iter_count = np.zeros(nm, dtype=np.int64)
        self.iters = 0
        self.graph = None
        self.diis = None
        self.first = True
        self.build_seconds = 0.0

    def reset(self):
        """Back to the identity-diagonal guess (same molecules, contexts, tiles and graph), so
        that the same set can be solved again."""
        T_ = self.total
        with self.torch.cuda.stream(self.stream):
            self.P.copy_(self.P0)
            self.Pold.zero_()
            self.K.zero_()
            self.JT.zero_()
        nm = len(self.mols)
        self.energy = np.full(nm, np.nan)
        self.dE = np.full(nm, np.inf)
        self.avgdP = np.full(nm, np.inf)
        self.converged = np.zeros(nm, dtype=bool)
        self.iter_count = np.zeros(nm, dtype=np.int64)
        self.iters = 0
        self.first = True

    # ------------------------------------------------------------------ the Fock build
    def _build(self):
        """dP -> dJT, dK on the job stream (a CUDA graph replay after the first two builds)."""
        T_ = self.total
        P, dP = self.P, self.dP
        ptr = lambda t, k: t.data_ptr() + 8 * k
        if self.graph is not None and not self.first:
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
        """One step of the reference's loop for every molecule (src/uhf.c:1600-1730): Fock from
        the accumulated J/K, new densities from the lowest orbitals, their energy, conv_diis4.
        Molecules that already met the convergence test keep their density (so their difference
        density, and with it their share of the next builds, is zero)."""
        torch = self.torch
        T_ = self.total
        nm = len(self.mols)
        Fbase = self.H + self.JT
        Ffull = torch.cat([Fbase, Fbase, torch.zeros(1, dtype=torch.float64, device=self.dev)]) + self.K
        Pnew = torch.zeros_like(self.P)
        for b in self.buckets:
            n = b.n
            live = np.nonzero(~self.frozen[b.mol_np])[0]       # rows of molecules still iterating
            if len(live) == 0:
                continue
            if len(live) == len(b.rows):
                g, X, sh, occ = b.gidx2, b.X, b.shift, b.occ
            else:
                li = torch.tensor(live, device=self.dev)
                g, X, sh, occ = b.gidx2[li], b.X[li], b.shift[li], b.occ[li]
            R = len(live)
            F = Ffull[g.reshape(-1)].view(R, n, n)
            Fo = X.transpose(1, 2) @ F @ X + sh
            _, C = syev_batched(Fo, stream=self.stream)     # one cuSOLVER call per bucket
            C = (X @ C) * occ[:, None, :]
            Dn = C @ C.transpose(1, 2)
            # padded positions target the trailing slot; their values are exact zeros
            Pnew.index_copy_(0, g.reshape(-1), Dn.reshape(-1))
        Pnew[2 * T_] = 0.0
        # restricted molecules: beta = alpha
        Pnew[T_:2 * T_] = torch.where(self.rmask, Pnew[:T_], Pnew[T_:2 * T_])
        PA, PB = Pnew[:T_], Pnew[T_:2 * T_]
        dens = (self.H + 0.5 * self.JT) * (PA + PB) + 0.5 * (self.K[:T_] * PA + self.K[T_:2 * T_] * PB)
        E = self.edots([dens], [(0, -1)])[:, 0] + self.enn
        out, avg = self.diis.step(Pnew[:2 * T_])
        keep = self.frozen_t[self.molid2]
        self.Pold.copy_(self.P)
        self.P[:2 * T_] = torch.where(keep, self.P[:2 * T_], out)
        return E, avg

    def run(self, max_iter=SCF_MAX):
        torch = self.torch
        t0 = time.perf_counter()
        self._graph_ready = self.graph is not None
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        nm = len(self.mols)
        T_ = self.total
        with torch.cuda.stream(self.stream):
            ev0.record(self.stream)
            self.frozen = np.zeros(nm, dtype=bool)
            self.frozen_t = torch.zeros(nm, dtype=torch.bool, device=self.dev)
            offs = [mo["off"] for mo in self.mols]
            lens = [mo["nbf"] ** 2 for mo in self.mols]
            self.diis = DensityDIIS4(torch, self.P[:2 * T_], self.molid2, nm, self.nbf2,
                                     segments=(offs + [T_ + o for o in offs], lens + lens,
                                               list(range(nm)) * 2))
            self._set_step(True)
            self.t_build = self.t_tail = 0.0
            eb0, eb1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            et1 = torch.cuda.Event(enable_timing=True)
            while self.iters < max_iter:
                tb = time.perf_counter()
                eb0.record(self.stream)
                self._build()
                eb1.record(self.stream)
                if self.first:
                    self.first = False
                    self._set_step(False)     # later builds: density screen everywhere
                elif not self._graph_ready:
                    self._graph_ready = True  # the next build is captured
                E, avg = self._tail()
                et1.record(self.stream)
                if self.iters == 0 and self.autotune and not self._tuned:
                    # tile autotuner on the work of the difference-density builds that follow
                    self._tuned = True
                    torch.sub(self.P, self.Pold, out=self.dP)
                    self.batch.autotune(self.dP.data_ptr(), self.dP.data_ptr() + 8 * T_,
                                        stream=self.stream.cuda_stream)
                h = torch.stack([E, avg]).cpu().numpy()
                self.build_seconds += time.perf_counter() - tb
                self.t_build += eb0.elapsed_time(eb1) / 1e3
                self.t_tail += eb1.elapsed_time(et1) / 1e3
                E, avg = h
                live = ~self.frozen
                prev = np.where(np.isnan(self.energy), 0.0, self.energy)
                self.dE = np.where(live, E - prev, self.dE)
                self.energy = np.where(live, E, self.energy)
                self.avgdP = np.where(live, avg, self.avgdP)
                self.iters += 1
                self.iter_count = np.where(live, self.iters, self.iter_count)
                conv = live & (np.abs(self.dE) <= self.scf_conv) & (avg <= self.scf_conv)
                self.converged = self.converged | conv
                self.frozen = self.frozen | conv
                self.frozen_t.copy_(torch.tensor(self.frozen), non_blocking=False)
                if self.frozen.all():
                    break
            ev1.record(self.stream)
        self.stream.synchronize()
        self.seconds = time.perf_counter() - t0
        self.device_seconds = ev0.elapsed_time(ev1) / 1e3
        return self.energy

    def close(self):
        self.graph = None
        self.edots.close()
        if self.diis is not None and self.diis.dots is not None:
            self.diis.dots.close()
        self.batch.close()
        for e in self.engines:
            e.close()
