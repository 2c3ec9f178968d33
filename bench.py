#!/usr/bin/env python
"""J/K builds/s of the B200 two-electron Fock build (Siam Quantum 2 hot path).

One step = one fresh FP64 J/K build (JT = J[PA+PB], KA = -K[PA]) of the workload, the work of
the reference's GTO_JK_Matrix_Quartet_Parallel (src/matrix.c:3773) in its direct mode
(Schwarz cutoff 1e-10, density-weighted screen on every quartet, no integral cache).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c60|benzene|water|h2co|water-qzp|c60-synthetic|organics|serve]

Default workload: RHF/6-31G C60 (Ih, 6:6 bonds 1.40, 6:5 bonds 1.45 angstrom; 540 functions)
from the reference's own converged SCF density (tests/golden/c60_631g.npz, made by running the
reference), Schwarz 1e-10 and the density screen on every quartet, as the reference's direct
mode builds it.  benzene = RHF/6-31G* benzene (D6h, C-C 1.39, C-H 1.09 angstrom; 102
functions) from its converged density; water-qzp = RHF/QZP water (126 functions, f shells on
every atom: the generic quartet kernel) from its converged density; c60-synthetic = C60 with a
seeded synthetic density and the density screen off.  Multi-GPU runs are independent replicas (one molecule's build runs on
one GPU and is not sharded), value = all ranks' builds / max-over-ranks time.

The reference arm (--impl reference) and the cpu_baseline of C60 run the reference's own process
split (oracle/_ref/sqref jkpart: child c of nCPU builds the bra shell pairs PQ with
PQ % nCPU == c, src/matrix.c:3909-3910) on every host thread: nCPU = threads x SLICES, and
step k runs the children of slice k mod SLICES, one per thread, so a step is 1/SLICES of a
build and SLICES consecutive steps make one whole build.
"""
import argparse
import importlib.util
import json
import os
import signal
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "siam-quantum_b200")
METRIC = "J/K builds/s"


def load_sqb200():
    spec = importlib.util.spec_from_file_location("sqb200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sqb200"] = mod
    spec.loader.exec_module(mod)
    return mod


def c60_reference_density():
    """C60/6-31G: atoms and the reference's converged RHF density from the fixture (symmetric,
    stored as its upper triangle)."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "c60_631g.npz"))
    n = len(g["nprim"])
    iu = np.triu_indices(n)
    P = np.zeros((n, n))
    P[iu] = g["PA_u"]
    P = P + np.triu(P, 1).T
    atoms = [(int(round(a[0])), float(a[1]), float(a[2]), float(a[3])) for a in g["atoms"]]
    return atoms, P


def workload(name, sqb):
    """(atoms_angstrom, basis_name, PA, density_screen, description)"""
    M = sqb.molecules
    if name in ("benzene", "water", "h2co"):
        fx = {"benzene": "benzene_631gs", "water": "water_321g", "h2co": "h2co_631gs"}[name]
        g = np.load(os.path.join(ROOT, "tests", "golden", fx + ".npz"))
        atoms = [tuple(a) for a in g["atoms"]]
        atoms = [(int(a[0]), a[1], a[2], a[3]) for a in atoms]
        desc = {"benzene": "benzene RHF/6-31G* (D6h, 102 bf)", "water": "water RHF/3-21G (13 bf)",
                "h2co": "formaldehyde RHF/6-31G* (34 bf)"}[name]
        return atoms, str(g["basis"]), np.array(g["PA"]), True, desc + ", converged density"
    if name == "water-qzp":
        g = np.load(os.path.join(ROOT, "tests", "golden", "water_qzp.npz"))
        atoms = [(int(a[0]), a[1], a[2], a[3]) for a in g["atoms"]]
        return (atoms, str(g["basis"]), np.array(g["PA"]), True,
                "water RHF/QZP (126 bf; two f shells on O, one per H), converged density")
    if name == "c60":
        atoms, PA = c60_reference_density()
        return (atoms, "631g", PA, True,
                "C60 RHF/6-31G (Ih, 1.40/1.45 A, 540 bf), the reference's converged density")
    if name == "c60-synthetic":
        atoms = M.c60()
        b = sqb.basis.build_basis(M.to_bohr(atoms), "631g")
        rng = np.random.default_rng(2024)
        n = b.nbf
        A = rng.normal(size=(n, n)) * 0.02
        PA = 0.5 * (A + A.T) + np.eye(n) * 0.4
        return atoms, "631g", PA, False, "C60 RHF/6-31G (Ih, 1.40/1.45 A, 540 bf), seeded density, density screen off"
    raise SystemExit("unknown workload " + name)


# ------------------------------------------------------------------ clocks

CLOCK_Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + CLOCK_Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.send_signal(signal.SIGTERM)
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            t = [x.strip() for x in line.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1])); smax.append(float(t[2]))
            except ValueError:
                continue
            for nm, v in zip(names, t[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------------ CPU reference runs

def _cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _ref_inputs(d, atoms, basis_name, PA, sqb):
    xyz = os.path.join(d, "m.xyz")
    with open(xyz, "w") as f:
        f.write(sqb.molecules.xyz_text(atoms))
    bas = os.path.join(d, "basis.txt")
    with open(bas, "w") as f:
        f.write(sqb.basis.gamess_text(basis_name, [a[0] for a in atoms]))
    pa = os.path.join(d, "pa.bin")
    np.ascontiguousarray(PA, dtype=np.float64).tofile(pa)
    return xyz, bas, pa


def ref_builds(atoms, basis_name, PA, seconds, procs, sqb):
    """Run `procs` concurrent reference processes, each doing fresh direct J/K builds
    (oracle/_ref/sqref bench, MAXMEM=0) for at least `seconds`.  Returns (builds/s total,
    per-process results)."""
    sqref = os.path.join(ROOT, "oracle", "_ref", "sqref")
    if not os.path.exists(sqref):
        raise FileNotFoundError(sqref)
    with tempfile.TemporaryDirectory() as d:
        xyz, bas, pa = _ref_inputs(d, atoms, basis_name, PA, sqb)
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
        ps = [subprocess.Popen([sqref, "bench", xyz, bas, pa, "1e-10", "0", str(seconds)],
                               stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True, env=env)
              for _ in range(procs)]
        rate = 0.0
        res = []
        for p in ps:
            _, err = p.communicate()
            for line in err.splitlines():
                if line.startswith("RESULT"):
                    kv = dict(x.split("=") for x in line.split()[1:])
                    b, s = float(kv["builds"]), float(kv["seconds"])
                    rate += b / s
                    res.append((b, s))
        if len(res) != procs:
            raise RuntimeError("reference processes failed")
    return rate, res


SLICES = 8                 # steps per whole build in the split reference runs (C60)


def ref_split_step(atoms, basis_name, PA, procs, step, sqb):
    """One step of the reference's own process split of a fresh direct J/K build (MAXMEM=0):
    nCPU = procs * SLICES children, of which this step runs the procs children of slice
    step % SLICES concurrently (oracle/_ref/sqref jkpart, one thread each).  Returns the
    slice's build time: the slowest child's GTO_JK_Matrix_Quartet_Parallel time (reset + build,
    as the harness times it; process start, basis input and the Schwarz matrix, which the
    caller computes once per SCF, are outside it)."""
    sqref = os.path.join(ROOT, "oracle", "_ref", "sqref")
    if not os.path.exists(sqref):
        raise FileNotFoundError(sqref)
    ncpu = procs * SLICES
    sl = step % SLICES
    with tempfile.TemporaryDirectory() as d:
        xyz, bas, pa = _ref_inputs(d, atoms, basis_name, PA, sqb)
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
        ps = [subprocess.Popen([sqref, "jkpart", xyz, bas, pa, "-", "1", "1e-10", "0", str(ncpu),
                                str(sl * procs + t), os.path.join(d, "o%d.bin" % t)],
                               stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True, env=env)
              for t in range(procs)]
        secs = []
        for p in ps:
            _, err = p.communicate()
            for line in err.splitlines():
                if line.startswith("RESULT"):
                    secs.append(float(dict(x.split("=") for x in line.split()[1:])["seconds"]))
        if len(secs) != procs:
            raise RuntimeError("reference processes failed")
    return max(secs)


ORG_SEED = 20240601        # seed of the 256-molecule organic set (molecules.organic_set)


def ref_scf_sample(mols, basis_name, procs, sqb, timeout=600):
    """Reference SCF (oracle/_ref/sqref scf, -SCFACC=1STEP -SCFCONV=1e-8) of every molecule,
    up to `procs` processes at a time.  Returns (wall seconds, energies)."""
    sqref = os.path.join(ROOT, "oracle", "_ref", "sqref")
    if not os.path.exists(sqref):
        raise FileNotFoundError(sqref)
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
    energies = [None] * len(mols)
    with tempfile.TemporaryDirectory() as d:
        bas = os.path.join(d, basis_name + ".txt")
        with open(bas, "w") as f:
            f.write(sqb.basis.gamess_text(basis_name, sorted({a[0] for m in mols for a in m})))
        paths = []
        for i, m in enumerate(mols):
            x = os.path.join(d, "m%d.xyz" % i)
            with open(x, "w") as f:
                f.write(sqb.molecules.xyz_text(m))
            paths.append(x)
        t0 = time.perf_counter()
        running = []
        todo = list(range(len(mols)))
        while todo or running:
            while todo and len(running) < procs:
                i = todo.pop(0)
                running.append((i, subprocess.Popen([sqref, "scf", paths[i], bas, "-", "-SCFACC=1STEP", "-SCFCONV=1e-8"],
                                                    stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True, env=env)))
            i, p = running.pop(0)
            _, err = p.communicate(timeout=timeout)
            for line in err.splitlines():
                if line.startswith("RESULT"):
                    energies[i] = float(dict(x.split("=") for x in line.split()[1:])["energy"])
        wall = time.perf_counter() - t0
    if any(e is None for e in energies):
        raise RuntimeError("reference SCF failed")
    return wall, energies


def ref_scf_iterations(mol, basis_name, sqb, timeout=3600):
    """The reference's own SCF (oracle/_ref/sqref scf, 1STEP, SCFConv 1e-8) of one molecule:
    (iterations it ran, converged) -- uhf() stops at its iteration cap without converging."""
    sqref = os.path.join(ROOT, "oracle", "_ref", "sqref")
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
    with tempfile.TemporaryDirectory() as d:
        bas = os.path.join(d, "b.txt")
        with open(bas, "w") as f:
            f.write(sqb.basis.gamess_text(basis_name, sorted({a[0] for a in mol})))
        x = os.path.join(d, "m.xyz")
        with open(x, "w") as f:
            f.write(sqb.molecules.xyz_text(mol))
        r = subprocess.run([sqref, "scf", x, bas, "-", "-SCFACC=1STEP", "-SCFCONV=1e-8"], capture_output=True,
                           text=True, env=env, timeout=timeout)
    its = [t for t in (ln.split() for ln in r.stdout.splitlines()) if len(t) == 3 and t[0].isdigit() and "E" in t[2]]
    n = int(its[-1][0]) if its else 0
    return n, 0 < n < sqb.scf.SCF_MAX


def run_organics(args, sqb):
    """Batched SCF of the seeded organic set (RHF/6-31G*): SCF solves/s of the whole set."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bname = "631g_star"
    mols = sqb.molecules.organic_set(ORG_SEED, args.nmol)
    nbfs = [sqb.basis.build_basis(sqb.molecules.to_bohr(m), bname).nbf for m in mols]
    jobs = [{"atoms": m, "basis": bname} for m in mols]
    fp64_peak, _ = sqb.engine.peak_fma(local)

    # end to end through the public API: a fresh BatchSCF from geometries to energies on the host
    t0 = time.perf_counter()
    bs = sqb.batch_scf.BatchSCF(jobs, device=local, fp32_below=args.fp32_below)
    E = bs.run()
    torch.cuda.synchronize(dev)
    t_e2e = time.perf_counter() - t0
    tot = sum(n * n for n in nbfs)
    e2e = {"value": len(mols) / t_e2e, "unit": "solves/s",
           "h2d_bytes_per_step": 8 * (4 * tot + sum(b.n * b.n * len(b.rows) for b in bs.buckets) * 2),
           "d2h_bytes_per_step": 8 * (3 * tot + 3 * len(mols) * bs.iters),
           "api": "batch_scf.BatchSCF(jobs).run() from geometries (set-up, one-electron integrals and "
                  "pair data included)", "setup_s": bs.setup_seconds}
    E_ref_first = E.copy()

    for _ in range(args.warmup):
        bs.reset()
        bs.run()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t_dev, iters, conv = 0.0, [], []
    for _ in range(args.steps):
        bs.reset()
        bs.run()
        t_dev += bs.device_seconds
        iters.append(bs.iters)
        conv.append(int(bs.converged.sum()))
    torch.cuda.synchronize(dev)
    t_max = max_over_ranks(dist, t_dev, dev)
    # a solve counts only when it met the convergence test (|dE| and RMS dP <= 1e-8) within the
    # reference's 80 iterations
    value = world * sum(conv) / t_max
    cv = bs.converged
    dE_rerun = float(np.max(np.abs(bs.energy - E_ref_first)[cv])) if cv.any() else None
    bs_iters = bs.iter_count.copy()
    split = {"build_s": bs.t_build, "tail_s": bs.t_tail}

    # batched J/K throughput: the captured build replayed with the full converged density
    jk = None
    if bs.graph is not None:
        with torch.cuda.stream(bs.stream):
            bs.Pold.zero_()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            bs.graph.replay()
            ev0.record(bs.stream)
            reps = 5
            for _ in range(reps):
                bs.graph.replay()
            ev1.record(bs.stream)
        bs.stream.synchronize()
        t_jk = ev0.elapsed_time(ev1) / 1e3 / reps
        st = bs.batch.stats()
        jk = {"molecule_builds_per_s": len(mols) / t_jk, "ms_per_batched_build": 1e3 * t_jk,
              "quartets_per_s": st["quartets"] / t_jk, "prim_quartets_per_s": st["prim_quartets"] / t_jk,
              "fp64_tflops_alg": st["flops"] / t_jk / 1e12, "fp64_frac": st["flops"] / t_jk / 1e12 / fp64_peak,
              "launches_per_build": st["launches"], "screen": "Schwarz 1STEP cutoff + density (full density)"}
    bs.close()

    # the plain FP64 one-at-a-time GPU path on a sample of the set
    sample = list(range(0, len(mols), max(1, len(mols) // 16)))[:16]
    t1 = 0.0
    for i in sample:
        job = sqb.scf.SCFJob(mols[i], bname, device=local)
        job.run()
        t1 += job.seconds
        job.close()
    one = {"solves_per_s": len(sample) / t1, "sample": "%d molecules of the set (every %d-th), SCFJob one "
           "after another (set-up not timed)" % (len(sample), max(1, len(mols) // 16))}
    line = {"metric": "SCF solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.fp32_below <= 0 else "f64+f32",
            "data": "synthetic",
            "config": {"workload": "%d seeded random C/N/O organics (seed %d, 2-20 heavy atoms, H-saturated), "
                                   "RHF/6-31G*, SCFConv 1e-8, 1STEP cutoffs" % (len(mols), ORG_SEED),
                       "nbf_min": min(nbfs), "nbf_max": max(nbfs), "nbf_mean": float(np.mean(nbfs)),
                       "fp32_below": args.fp32_below, "parallelism": "replicas x%d" % world,
                       "step": "one batched SCF solve of the whole set (reset to the guess; contexts, "
                               "tiles and the captured build graph reused)",
                       "l2": "no flush: each step is a whole SCF solve (every iteration rewrites the "
                             "packed %.0f MB density/J/K arrays and the pair data is re-read per class "
                             "launch)" % (8 * tot / 1e6)},
            "iterations": iters, "converged": conv, "unconverged": [len(mols) - c for c in conv],
            "unconverged_molecules": [{"molecule": int(i), "nbf": nbfs[i]} for i in np.nonzero(~cv)[0]],
            "max_abs_dE_between_solves_converged": dE_rerun,
            "last_solve_device_split": split,
            "iterations_per_molecule": {"mean": float(np.mean(bs_iters)), "max": int(np.max(bs_iters))},
            "batched_jk": jk, "one_at_a_time_gpu": one, "e2e": e2e, "gpu_launches": None}
    if world == 1 and not args.no_cpu_baseline:
        # the smallest molecules that did not converge here (at most 3): does the reference's own
        # SCF converge them within its 80 iterations?
        unc = sorted(np.nonzero(~cv)[0], key=lambda i: nbfs[i])[:3]
        try:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(max_workers=max(1, len(unc))) as ex:
                outs = list(ex.map(lambda i: ref_scf_iterations(mols[i], bname, sqb), unc))
            line["reference_on_unconverged"] = [
                {"molecule": int(i), "nbf": nbfs[i], "iterations_here": int(bs_iters[i]),
                 "reference_iterations": it, "reference_converged": ok}
                for i, (it, ok) in zip(unc, outs)]
        except Exception as e:
            line["reference_on_unconverged"] = "failed: %s" % e
        try:
            small = [i for i, n in enumerate(nbfs) if n <= 120][:16]
            smols = [mols[i] for i in small]
            procs = min(_cpu_threads(), len(smols))
            wall, Eref = ref_scf_sample(smols, bname, procs, sqb)
            bsm = sqb.batch_scf.BatchSCF([jobs[i] for i in small], device=local)
            bsm.run()
            bsm.reset()
            Eg = bsm.run()
            gpu_rate = len(small) / bsm.device_seconds
            bsm.close()
            line["cpu_baseline"] = {"value": len(smols) / wall, "unit": "solves/s", "cores": procs,
                                    "kind": "reference",
                                    "sample": "the first %d molecules of the set with nbf <= 120 (mean %.0f), one "
                                              "reference process each (oracle/_ref/sqref scf, 1STEP, SCFConv "
                                              "1e-8)" % (len(smols), np.mean([nbfs[i] for i in small])),
                                    "gpu_value_same_sample": gpu_rate,
                                    "max_abs_dE_vs_reference": float(np.max(np.abs(np.array(Eg) - np.array(Eref))))}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": 0, "kind": "reference",
                                    "sample": "failed: %s" % e}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


SERVE_SEED = 20240607       # seed of the served request stream (serve.poisson_requests)


def run_serve(args, sqb):
    """Served stream: Poisson arrivals of RHF and UHF (doublet) SCF energy and energy+gradient
    jobs, continuous batching on one device, at each mean arrival rate of --rates; solves/s
    (converged solves only) and p50/p99 latency beside the one-at-a-time GPU path (each job
    solved alone, FIFO in the same arrival order).  `value` is the rate with the highest
    arrival rate (the saturated throughput)."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rates = [float(x) for x in args.rates.split(",")]
    # warm-up: one small job through each path (library load, cuSOLVER handles, kernels' first use)
    warm = sqb.serve.poisson_requests(SERVE_SEED + 1, 3, 100.0, heavy=(2, 4))
    sqb.serve.Server(device=local, max_active=args.slots, batched=args.batched).run(warm, realtime=False)
    # the same molecules at every rate (only the arrival times scale)
    base = sqb.serve.poisson_requests(SERVE_SEED, args.nreq, 1.0, heavy=(2, args.max_heavy))
    alone = [sqb.serve.solve_alone(r, device=local) for r in base]
    service = [a[2] + a[3] for a in alone]
    per_rate = []
    for rate in rates:
        reqs = [dict(r, arrival=r["arrival"] / rate) for r in base]
        srv = sqb.serve.Server(device=local, max_active=args.slots, fp32_below=args.fp32_below, batched=args.batched)
        res = srv.run(reqs, realtime=True)
        conv = np.array([r["converged"] for r in res])
        lat = np.array([r["latency"] for r in res])
        fifo = np.array(sqb.serve.fifo_latencies([r["arrival"] for r in reqs], service))
        tf = 0.0
        for a, sv in sorted(zip([r["arrival"] for r in reqs], service)):
            tf = max(tf, a) + sv
        conv_alone = np.array([a[1] < sqb.scf.SCF_MAX for a in alone])
        dE = np.array([abs(r["energy"] - a[0]) for r, a in zip(res, alone)])
        dG = [float(np.abs(r["gradient"] - a[4]).max()) for r, a in zip(res, alone)
              if r["gradient"] is not None and a[4] is not None]
        per_rate.append({
            "rate_per_s": rate, "solves_per_s": float(conv.sum()) / srv.stats["makespan"],
            "converged": int(conv.sum()), "unconverged": int((~conv).sum()), "makespan_s": srv.stats["makespan"],
            "latency_s": {"p50": float(np.percentile(lat[conv], 50)) if conv.any() else None,
                          "p99": float(np.percentile(lat[conv], 99)) if conv.any() else None},
            "one_at_a_time_gpu": {"solves_per_s": float(conv_alone.sum()) / tf,
                                  "p50": float(np.percentile(fifo[conv_alone], 50)) if conv_alone.any() else None,
                                  "p99": float(np.percentile(fifo[conv_alone], 99)) if conv_alone.any() else None},
            "served_vs_alone_max_abs_dE": float(dE[conv].max()) if conv.any() else None,
            "served_vs_alone_max_abs_dgrad": max(dG) if dG else None,
            "peak_active": srv.stats["peak_active"], "rounds": srv.stats["rounds"]})
    top = per_rate[-1]
    nb = [a[5] for a in alone]
    line = {"metric": "served SCF solves/s", "value": top["solves_per_s"], "unit": "solves/s",
            "n_gpus": 1, "steps": len(rates), "warmup": 1, "ms_per_step": 1e3 * top["makespan_s"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.fp32_below <= 0 else "f64+f32", "data": "synthetic",
            "config": {"workload": "%d Poisson arrivals (seed %d, mean rates %s /s) of seeded random organics with "
                                   "2-%d heavy atoms, 6-31G*, half UHF doublets (one H removed), half energy+"
                                   "gradient jobs, SCFConv 1e-8" % (len(base), SERVE_SEED, args.rates, args.max_heavy),
                       "nbf_min": min(nb), "nbf_max": max(nb), "nbf_mean": float(np.mean(nb)),
                       "slots": args.slots, "fp32_below": args.fp32_below,
                       "served_builds": "batched (one launch per class over every active job)" if args.batched
                       else "one build per job on its own stream",
                       "step": "the whole stream at one rate, wall clock from the first arrival's time origin "
                               "to the last completion; only converged solves count",
                       "l2": "no flush (each job rewrites its own state every iteration)"},
            "rates": per_rate,
            "gradient_jobs": int(sum(1 for r in base if r.get("gradient"))),
            "e2e": {"value": top["solves_per_s"], "unit": "solves/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "api": "serve.Server.run(requests) from geometries; latency includes queueing and set-up"}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ arms

def run_reference_organics(args, sqb):
    """Reference arm of the organics workload: the reference's own SCF (oracle/_ref/sqref scf) of
    a bounded sample of the set (molecules with nbf <= 120), one process per host thread."""
    bname = "631g_star"
    mols = sqb.molecules.organic_set(ORG_SEED, args.nmol)
    nbfs = [sqb.basis.build_basis(sqb.molecules.to_bohr(m), bname).nbf for m in mols]
    small = [mols[i] for i, n in enumerate(nbfs) if n <= 120][:16]
    procs = min(_cpu_threads(), len(small))
    rates = []
    for _ in range(args.steps):
        wall, _E = ref_scf_sample(small, bname, procs, sqb)
        rates.append(len(small) / wall)
    value = float(np.mean(rates))
    line = {"metric": "SCF solves/s", "value": value, "unit": "solves/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": 0, "ms_per_step": 1e3 * len(small) / value / len(small),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "first %d molecules with nbf <= 120 of the seeded organic set (seed %d)" % (
                len(small), ORG_SEED), "parallelism": "%d concurrent single-thread reference processes" % procs},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": "reference",
                             "sample": "each step: the %d molecules, oracle/_ref/sqref scf 1STEP 1e-8" % len(small)},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args, sqb):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "organics":
        return run_reference_organics(args, sqb)
    atoms, bname, PA, dscreen, desc = workload(args.workload, sqb)
    procs = _cpu_threads()
    if args.workload == "c60":
        return run_reference_split(args, atoms, bname, PA, desc, procs, sqb)
    for _ in range(args.warmup):
        ref_builds(atoms, bname, PA, 0, procs, sqb)
    rates, walls = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r, _ = ref_builds(atoms, bname, PA, 0, procs, sqb)
        walls.append(time.perf_counter() - t0)
        rates.append(r)
    value = float(np.mean(rates))
    line = {"metric": METRIC, "value": value, "unit": "builds/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(np.mean(walls)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "screen": "Schwarz 1e-10 + density (direct, MAXMEM=0)",
                       "parallelism": "%d concurrent single-thread reference processes" % procs},
            "cpu_baseline": {"value": value, "unit": "builds/s", "cores": procs, "kind": "reference",
                             "sample": "each step: %d processes x 1 fresh J/K build (oracle/_ref/sqref, gcc -O3)" % procs},
            "e2e": {"value": value, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_split(args, atoms, bname, PA, desc, procs, sqb):
    """Reference arm of the C60 build: the reference's own process split (ref_split_step),
    W + K steps, each step 1/SLICES of a whole build on every host thread."""
    for k in range(args.warmup):
        ref_split_step(atoms, bname, PA, procs, k, sqb)
    secs = [ref_split_step(atoms, bname, PA, procs, args.warmup + k, sqb) for k in range(args.steps)]
    value = args.steps / SLICES / sum(secs)
    line = {"metric": METRIC, "value": value, "unit": "builds/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(np.mean(secs)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "screen": "Schwarz 1e-10 + density (direct, MAXMEM=0)",
                       "parallelism": "the reference's own split: %d processes of nCPU=%d per step, "
                                      "%d steps per build" % (procs, procs * SLICES, SLICES)},
            "cpu_baseline": {"value": value, "unit": "builds/s", "cores": procs, "kind": "reference",
                             "sample": "each step: children [s*%d, (s+1)*%d) of nCPU=%d of a fresh direct build "
                                       "(oracle/_ref/sqref jkpart, gcc -O3), s = step %% %d" % (
                                           procs, procs, procs * SLICES, SLICES)},
            "e2e": {"value": value, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the dominant class
# kernel, from one `ncu --set full` capture of the same workload; the summary with its command
# is profiles/<kernel>_<workload>.md.  Kernels without a capture report null.
TRAFFIC = {("benzene", "jk_DL_LL_R"): 970752, ("benzene", "jk_DL_LL_R_w"): 890112,
           ("benzene", "jk_DL_LL_R_s"): 1268992, ("c60-synthetic", "jk_LL_LL_R_w"): 18592768, ("c60", "jk_LL_LL_R_w"): 20667648,
           ("water-qzp", "k_jk_gen"): 1336320}


def max_over_ranks(dist, t_local, device):
    """The job time of N replicas: the maximum of the ranks' device times (every rank takes
    part; without a process group the local time)."""
    if dist is None:
        return t_local
    import torch
    t = torch.tensor([t_local], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, sqb):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    atoms, bname, PA_np, dscreen, desc = workload(args.workload, sqb)
    b = sqb.basis.build_basis(sqb.molecules.to_bohr(atoms), bname)
    n = b.nbf
    fp64_peak, fp32_peak = sqb.engine.peak_fma(local)
    eng = sqb.JKEngine(b, device=local)            # Schwarz bounds computed on the device
    if args.fp32_below > 0:
        eng.set_precision(args.fp32_below)         # mixed FP32/FP64 by Schwarz bound
    rmax = float("inf") if dscreen else 0.0
    kw = dict(restricted=True, scf_cutoff=1e-10, fixed_cutoff=1e-10, dscreen_rmax=rmax)

    PA = torch.tensor(PA_np, dtype=torch.float64, device=dev).contiguous()
    JT = torch.empty_like(PA); KA = torch.empty_like(PA)
    # an explicit stream: the legacy default stream's handle is 0, which the C ABI reads as
    # "the context's own stream"
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > L2 (126 MB)

    def step():
        eng.build_device(PA.data_ptr(), PA.data_ptr(), JT.data_ptr(), KA.data_ptr(), None,
                         stream=stream.cuda_stream, **kw)

    if args.tiles_from:
        # the forms an earlier run chose (a profiler serialises the autotuner's timed launches,
        # so under one it would choose differently from the timed run it explains)
        eng.set_tiles(np.loadtxt(args.tiles_from, dtype=np.int32, ndmin=1))
    elif not args.no_autotune:
        # untimed set-up: per class, the fastest of the narrow, wide and swapped forms on this work
        eng.autotune(PA.data_ptr(), stream=stream.cuda_stream, **kw)
    tiles = eng.tiles()
    if args.save_tiles and rank == 0:
        np.savetxt(args.save_tiles, tiles, fmt="%d")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    st = eng.stats()

    clocks = ClockSampler(local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    for i in range(args.steps):
        flush.zero_()                                  # L2 flush between timed builds (untimed)
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    t_dev = sum(a.elapsed_time(b_) for a, b_ in evs) / 1e3
    # per-class kernel durations for the roofline: a separate profiled pass, in which the build
    # launches its class kernels one after another on its stream with an event pair around each
    # (the timed builds above overlap classes on several streams, so no single kernel can be
    # timed alone there)
    eng.profile(True)
    for _ in range(max(3, min(args.steps, 10))):
        flush.zero_()
        step()
    torch.cuda.synchronize(dev)
    prof = eng.profile_read()
    eng.profile(False)
    # keep the clock sampler on the same load for at least ~1 s
    tail_end = time.perf_counter() + (0.0 if args.profile_run else max(0.0, 1.0 - t_dev))
    while time.perf_counter() < tail_end:
        step()
        torch.cuda.synchronize(dev)
    clk = clocks.stop()

    t_max = max_over_ranks(dist, t_dev, dev)
    value = world * args.steps / t_max

    # ---- end-to-end through the public host API (pinned host buffers, copies included)
    pin = lambda: torch.empty((n, n), dtype=torch.float64, pin_memory=True).numpy()
    hPA = pin(); hPA[:] = PA_np
    outs = (pin(), pin(), pin())
    e2e_steps = 1 if args.profile_run else max(3, min(args.steps, 20))
    eng.build(hPA, out=outs, **kw)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.build(hPA, out=outs, **kw)
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks(dist, t_e2e, dev)
    e2e = {"value": world * e2e_steps / t_e2e, "unit": "builds/s",
           "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": 3 * n * n * 8,
           "api": "sqb200_jk_build (host buffers, pinned)"}

    # ---- roofline of the dominant class kernel (FP64 pipe)
    dom = max(prof, key=lambda r: r["ms"])
    per_launch_s = dom["ms"] / dom["launches"] / 1e3
    achieved = dom["flops"] / per_launch_s / 1e12
    dom32 = dom["class"].endswith(" f32")
    total_flops = sum(r["flops"] for r in prof)
    peak = fp32_peak if dom32 else fp64_peak
    # (the generic kernel of quartets with f shells counts the operations it executes)
    dom_name = "k_jk_gen" if dom["class"].startswith("generic") else "jk_" + dom["class"].replace(" f32", "").replace("|", "_") + (
        "_R_f32" if dom32 else {1: "_R_w", 2: "_R_s"}.get(int(tiles[dom["index"]]) if dom["index"] < len(tiles) else 0, "_R"))
    roof = {"bound": "fp32" if dom32 else "fp64",
            "kernel": dom_name,
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "measured %s FMA peak of this GPU in this run (sqb200_peak_fma); "
                           "MEASURED_PEAKS.json has no FP64/FP32 figure" % ("FP32" if dom32 else "FP64"),
            "traffic": None, "traffic_source": None, "share_of_build": sum(r["ms"] for r in prof if r is dom) / max(1e-12, sum(r["ms"] for r in prof)),
            "build_fp64_frac": total_flops / (t_dev / args.steps) / 1e12 / fp64_peak,
            "fp32_peak": fp32_peak}

    tb = TRAFFIC.get((args.workload, roof["kernel"]))
    if tb is not None and not dom32:
        roof["traffic"] = tb
        roof["traffic_source"] = "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/%s" % (
            {"benzene": "jk_DL_LL_R_forms_benzene_631gs.md", "c60-synthetic": "jk_LL_LL_R_w_c60_631g_synthetic.md",
             "c60": "jk_LL_LL_R_w_c60_631g_refdensity.md", "water-qzp": "k_jk_gen_water_qzp.md"}.get(
                args.workload, args.workload))
    line = {"metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.fp32_below <= 0 else "f64+f32", "data": "synthetic",
            "config": {"workload": desc, "nbf": n, "fp32_below": args.fp32_below, "screen": "Schwarz 1e-10 + density" if dscreen else "Schwarz 1e-10",
                       "parallelism": "replicas x%d" % world, "l2": "256 MB write between timed builds (untimed)",
                       "launch": "persistent work queue" if args.persistent else "one CTA per work unit",
                       "quartets_per_build": st["quartets"], "prim_quartets_per_build": st["prim_quartets"],
                       "tiles": ("autotuned forms per class: %d narrow, %d wide, %d swapped" % (
                           int((tiles == 0).sum()), int((tiles == 1).sum()), int((tiles == 2).sum()))
                                 if not args.no_autotune else "narrow")
                                if not args.tiles_from else "forms per class from %s" % args.tiles_from},
            "quartets_per_s": value * st["quartets"], "prim_quartets_per_s": value * st["prim_quartets"],
            "e2e": e2e, "roofline": roof, "clocks": clk,
            "gpu_launches": args.steps * st["launches"],
            "classes": sorted(({"class": r["class"], "ms_per_build": r["ms"] / r["launches"],
                                "tflops": r["flops"] / (r["ms"] / r["launches"] / 1e3) / 1e12}
                               for r in prof), key=lambda x: -x["ms_per_build"])[:6]}

    if world == 1 and not (args.no_cpu_baseline or args.profile_run) and args.workload == "c60":
        try:
            procs = _cpu_threads()
            nst = 4
            secs = [ref_split_step(atoms, bname, PA_np, procs, k, sqb) for k in range(nst)]
            line["cpu_baseline"] = {"value": nst / SLICES / sum(secs), "unit": "builds/s", "cores": procs,
                                    "kind": "reference",
                                    "sample": "%d of the %d slices of one fresh direct build split over nCPU=%d "
                                              "reference processes (oracle/_ref/sqref jkpart), %d at a time" % (
                                                  nst, SLICES, procs * SLICES, procs)}
        except Exception as e:  # the GPU line is still valid without the baseline
            line["cpu_baseline"] = {"value": None, "unit": "builds/s", "cores": 0, "kind": "reference",
                                    "sample": "failed: %s" % e}
    elif world == 1 and not (args.no_cpu_baseline or args.profile_run):
        try:
            procs = _cpu_threads()
            rate, res = ref_builds(atoms, bname, PA_np, args.cpu_seconds, procs, sqb)
            line["cpu_baseline"] = {"value": rate, "unit": "builds/s", "cores": procs, "kind": "reference",
                                    "sample": "%d concurrent reference processes (oracle/_ref/sqref bench, direct "
                                              "MAXMEM=0 fresh J/K builds) for >= %.0f s each" % (procs, args.cpu_seconds)}
        except Exception as e:  # the GPU line is still valid without the baseline
            line["cpu_baseline"] = {"value": None, "unit": "builds/s", "cores": 0, "kind": "reference",
                                    "sample": "failed: %s" % e}
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 50 builds; 1 batch of solves for organics)")
    ap.add_argument("--warmup", type=int, default=None,
                    help="untimed steps (default 5 builds; 1 batch of solves for organics)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c60",
                    choices=["c60", "benzene", "water", "h2co", "water-qzp", "c60-synthetic", "organics", "serve"])
    ap.add_argument("--nmol", type=int, default=256, help="molecules of the organics workload")
    ap.add_argument("--nreq", type=int, default=32, help="requests of the serve workload")
    ap.add_argument("--rates", default="0.5,1,2", help="mean arrival rates (1/s) of the serve workload")
    ap.add_argument("--batched", type=int, default=1, help="serve: batched Fock builds over the active jobs")
    ap.add_argument("--max-heavy", type=int, default=40, help="largest molecule (heavy atoms) of the serve workload")
    ap.add_argument("--slots", type=int, default=32, help="concurrent jobs of the serve workload")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep every class on its narrow tile")
    ap.add_argument("--save-tiles", default="", help="write the per-class forms the run used to this file")
    ap.add_argument("--tiles-from", default="",
                    help="J/K workloads: take the per-class forms from this file (written by --save-tiles) "
                         "instead of autotuning")
    ap.add_argument("--fp32-below", type=float, default=0.0,
                    help="mixed precision: quartets with Schwarz product below this run in FP32")
    ap.add_argument("--persistent", action="store_true",
                    help="class kernels as persistent work-queue launches (SQB200_PERSISTENT=1)")
    ap.add_argument("--profile-run", action="store_true",
                    help="minimal run for ncu launch lists: no clock tail, 1 e2e step, no CPU baseline")
    args = ap.parse_args()
    # one organics step is a whole batch of SCF solves (about a minute on one B200)
    if args.steps is None:
        args.steps = 1 if args.workload == "organics" else 50
    if args.warmup is None:
        args.warmup = 1 if args.workload == "organics" else 5
    if args.persistent:
        os.environ["SQB200_PERSISTENT"] = "1"       # read by every context at creation
    sqb = load_sqb200()
    if args.impl == "reference":
        return run_reference(args, sqb)
    if args.workload == "organics":
        return run_organics(args, sqb)
    if args.workload == "serve":
        return run_serve(args, sqb)
    return run_ours(args, sqb)


if __name__ == "__main__":
    sys.exit(main())
