"""Served stream of RHF/UHF SCF energy and energy+gradient jobs on one device, with continuous
batching.

Requests arrive over time (e.g. Poisson arrivals, `poisson_requests`).  The server admits a
request once it has arrived, a slot is free (at most `max_active` jobs in flight) and its
estimated device-memory footprint fits the HBM budget next to the jobs already resident.  An
admitted job keeps its whole SCF state on the device (pair data and Schwarz bounds in its
J/K context; S, H, densities, J/K, DIIS history in torch tensors; scf.SCFJob) until it
converges, and runs on its own CUDA stream.  Every round the server enqueues one SCF step of
every active job (difference-density J/K build, Fock, cuSOLVER eigensolve, density DIIS --
nothing read back), and only then reads each job's energy and density change: the steps of
all jobs are in flight on the GPU at once, and a request that arrives meanwhile joins at the
next round.  A job leaves when it meets the reference's convergence test (or its iteration
cap) -- after its nuclear gradient, when the request asks for one (scf.SCFJob.gradient, on the
job's resident state) -- and frees its slot and memory.

Each job runs exactly the single-job algorithm (scf.SCFJob), so its result is the one it gets
alone, up to the order of floating-point atomics in the J/K build.

With batched=True (the default) the difference-density J/K builds of all active jobs are one
batched build (engine.JKBatch: one launch per class kernel over every job's work items, each
job's own cutoffs, spin and first-visit screen in its molecule record), re-formed whenever a job
joins or leaves; each job's SCF tail still runs on its own stream.  The server stream waits for
every job's previous step before it packs the difference densities, and every job's stream waits
for the build before its tail reads its block of the packed J/K.
"""
import time

import numpy as np

from . import basis as B
from . import molecules as M
from .engine import JKBatch
from .scf import SCF_MAX, SCFJob, electrons


def footprint_bytes(atoms_angstrom, basis_name):
    """Estimated device memory of one job: its J/K context (primitive-pair records of every
    shell pair, FP64 and FP32 copies, and ten nbf x nbf matrices) plus the SCF state (about
    thirty nbf x nbf FP64 matrices: S, H, X, densities, J/K and their differences, DIIS
    history).  An estimate for admission; it errs high."""
    b = B.build_basis(M.to_bohr(atoms_angstrom), basis_name)
    n = b.nbf
    nprim = int(np.sum(b.nprim))
    # primitive pairs ~ (sum of primitives)^2 / 2, ~60 doubles per record (Hermite table for d)
    pairs = 0.5 * nprim * nprim * 60 * (8 + 4)
    return int(8 * 40 * n * n + pairs + (1 << 20))


def poisson_requests(seed, count, rate, heavy=(2, 40), doublet_fraction=0.5, basis="631g_star",
                     gradient_fraction=0.5):
    """`count` requests with exponential inter-arrival times of mean 1/rate (seconds): seeded
    random organics (molecules.random_organic); a `doublet_fraction` of them become UHF
    doublets by removing one hydrogen; a `gradient_fraction` ask for the nuclear gradient as
    well as the energy."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        atoms = M.random_organic(rng, int(rng.integers(heavy[0], heavy[1] + 1)))
        uhf = bool(rng.random() < doublet_fraction)
        if uhf:
            atoms = M.remove_one_h(atoms, rng)
        grad = bool(rng.random() < gradient_fraction)
        out.append({"id": i, "atoms": atoms, "basis": basis, "arrival": t, "charge": 0,
                    "mult": 2 if uhf else 1, "gradient": grad})
    return out


class Server:
    """Continuous-batching SCF server on one device (see the module docstring)."""

    def __init__(self, device=0, max_active=32, hbm_budget=None, scf_conv=1e-8, fp32_below=0.0,
                 max_iter=SCF_MAX, job_factory=None, footprint=footprint_bytes, batched=True):
        """`job_factory(request)` may replace the default SCFJob construction (tests use it to
        run the scheduler on the CPU with a stand-in J/K engine, which also turns the batched
        builds off); `footprint(atoms, basis)` the memory estimate; `batched` merges the active
        jobs' J/K builds into one batched build per round."""
        import torch
        self.torch = torch
        self.device = device
        self.batched = bool(batched) and job_factory is None
        self._batch = None
        self._batch_jobs = []
        self.job_factory = job_factory
        self.footprint = footprint
        self.max_active = max_active
        if hbm_budget is None:
            free, _total = torch.cuda.mem_get_info(device)   # GPU servers; tests pass a budget
            hbm_budget = int(0.5 * free)
        self.hbm_budget = hbm_budget
        self.scf_conv = scf_conv
        self.fp32_below = fp32_below
        self.max_iter = max_iter

    def run(self, requests, realtime=True):
        """Serve `requests` (dicts: id, atoms, basis, arrival [s], charge, mult).  With
        realtime=False every request counts as arrived at time 0.  Returns one result dict per
        request (energy, iterations, converged, arrival/admit/finish times, latency) and keeps
        `self.stats` (makespan, peak concurrency and memory in use)."""
        pending = sorted(requests, key=lambda r: r["arrival"])
        active = []                      # (request, job, footprint, admitted time)
        results = {}
        used = 0
        peak_active = 0
        peak_used = 0
        rounds = 0
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        while pending or active:
            now = clock()
            # admission in arrival order: slot, memory budget, arrived
            while pending and (not realtime or pending[0]["arrival"] <= now) and len(active) < self.max_active:
                r = pending[0]
                fp = self.footprint(r["atoms"], r["basis"])
                if used + fp > self.hbm_budget and active:
                    break                # wait for memory; a lone job is always admitted
                pending.pop(0)
                if self.job_factory is not None:
                    job = self.job_factory(r)
                else:
                    nea, neb, mult = electrons(r["atoms"], r.get("charge", 0), r.get("mult"))
                    job = SCFJob(r["atoms"], r["basis"], charge=r.get("charge", 0), mult=mult,
                                 scf_conv=self.scf_conv, device=self.device, fp32_below=self.fp32_below)
                active.append((r, job, fp, clock()))
                used += fp
                now = clock()
            peak_active = max(peak_active, len(active))
            peak_used = max(peak_used, used)
            if not active:
                time.sleep(max(0.0, pending[0]["arrival"] - clock()))
                continue
            # one SCF step of every active job in flight, then read them back
            if self.batched:
                self._batched_builds([job for _r, job, _fp, _ta in active])
                for _r, job, _fp, _ta in active:
                    job.update_launch()
            else:
                for _r, job, _fp, _ta in active:
                    job.build_jk()
                    job.update_launch()
            rounds += 1
            still = []
            for entry in active:
                r, job, fp, ta = entry
                conv = job.update_finish()
                if conv or job.iters >= self.max_iter:
                    grad = job.gradient() if (r.get("gradient") and conv) else None
                    tf = clock()
                    results[r["id"]] = {"id": r["id"], "energy": job.energy, "iters": job.iters, "gradient": grad,
                                        "converged": bool(conv), "nbf": job.n, "restricted": job.restricted,
                                        "arrival": r["arrival"] if realtime else 0.0, "admitted": ta,
                                        "finished": tf,
                                        "latency": tf - (r["arrival"] if realtime else 0.0)}
                    job.close()
                    used -= fp
                else:
                    still.append(entry)
            active = still
        if self.job_factory is None:
            self.torch.cuda.synchronize(self.device)
        self._drop_batch()
        self.stats = {"makespan": clock(), "peak_active": peak_active, "peak_bytes": peak_used,
                      "rounds": rounds, "budget_bytes": self.hbm_budget}
        return [results[r["id"]] for r in sorted(requests, key=lambda r: r["id"])]


    # ------------------------------------------------------------------ batched builds
    def _drop_batch(self):
        if self._batch is not None:
            self._batch.close()
        self._batch, self._batch_jobs = None, []

    def _batched_builds(self, jobs):
        """The difference-density J/K of every job in `jobs` as one batched build on the server
        stream; afterwards each job's dJT/dKA/dKB are views of its blocks of the packed output
        and its stream waits for the build."""
        torch = self.torch
        dev = torch.device("cuda", self.device)
        if [id(j) for j in jobs] != [id(j) for j in self._batch_jobs]:
            # re-form on a job joining or leaving: the old packed buffers may still be read by a
            # job's stream, so everything in flight finishes before they are released
            torch.cuda.synchronize(dev)
            self._drop_batch()
            self._batch = JKBatch([j.eng for j in jobs])
            self._batch_jobs = list(jobs)
            if not hasattr(self, "_stream"):
                self._stream = torch.cuda.Stream(dev)
            T = self._batch.total
            f64 = dict(dtype=torch.float64, device=dev)
            with torch.cuda.stream(self._stream):
                self._dP = torch.zeros(2 * T, **f64)
                self._dJT = torch.zeros(T, **f64)
                self._dKA = torch.zeros(T, **f64)
                self._dKB = torch.zeros(T, **f64)
        b, T, st = self._batch, self._batch.total, self._stream
        # pack every job's difference densities on its own stream, then the build waits for all
        for m, j in enumerate(jobs):
            o, n = b.offsets[m], j.n
            with torch.cuda.stream(j.stream):
                self._dP[o:o + n * n].view(n, n).copy_(j.PA - j.PA_old)
                self._dP[T + o:T + o + n * n].view(n, n).copy_(
                    self._dP[o:o + n * n].view(n, n) if j.restricted else j.PB - j.PB_old)
                ev = torch.cuda.Event()
                ev.record(j.stream)
            st.wait_event(ev)
        b.set_step([j.restricted for j in jobs], [j.cutoff for j in jobs], [j.cutoff for j in jobs],
                   [j.rmax_first if j.first else float("inf") for j in jobs])
        ptr = lambda t, k: t.data_ptr() + 8 * k
        b.build_device(ptr(self._dP, 0), ptr(self._dP, T), self._dJT.data_ptr(), self._dKA.data_ptr(),
                       self._dKB.data_ptr(), stream=st.cuda_stream)
        done = torch.cuda.Event()
        done.record(st)
        for m, j in enumerate(jobs):
            o, n = b.offsets[m], j.n
            j.dJT = self._dJT[o:o + n * n].view(n, n)
            j.dKA = self._dKA[o:o + n * n].view(n, n)
            j.dKB = self._dKB[o:o + n * n].view(n, n)
            j.first = False
            j.stream.wait_event(done)


def solve_alone(request, device=0, scf_conv=1e-8, fp32_below=0.0):
    """The same job by itself (the plain one-at-a-time GPU path): (energy, iterations,
    seconds of its SCF loop and gradient, set-up seconds, gradient or None)."""
    t0 = time.perf_counter()
    job = SCFJob(request["atoms"], request["basis"], charge=request.get("charge", 0), mult=request.get("mult"),
                 scf_conv=scf_conv, device=device, fp32_below=fp32_below)
    t1 = time.perf_counter()
    e = job.run()
    grad = job.gradient() if (request.get("gradient") and job.converged) else None
    t2 = time.perf_counter()
    out = (e, job.iters, t2 - t1, t1 - t0, grad, job.n)
    job.close()
    return out


def fifo_latencies(arrivals, service):
    """Latencies of a one-at-a-time FIFO server with the given arrival and service times."""
    t = 0.0
    lat = []
    for a, s in sorted(zip(arrivals, service)):
        t = max(t, a) + s
        lat.append(t - a)
    return lat
