"""Python binding of the B200 J/K engine (libsqb200.so, C ABI in include/sqb200.h).

The engine runs only on the GPU: there is no CPU fallback.  Loading fails loudly when the
shared library is missing, and building a context fails when no CUDA device is present.

Mirrors the reference's Fock-build entry point GTO_JK_Matrix_Quartet_Parallel
(src/matrix.c:3773) and its caller uhf_getGMatrix (src/uhf.c:112): given densities PA, PB it
returns JT = J[PA+PB], KA = -K[PA], KB = -K[PB] (KB = KA when restricted), with the same
Schwarz, density and primitive screening.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the library this package loads: the one built beside it, unless SQB200_LIB names another build
LIB_PATH = os.environ.get("SQB200_LIB") or os.path.join(HERE, "libsqb200.so")

_lib = None
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

EXPORTS = ["sqb200_jk_create", "sqb200_jk_destroy", "sqb200_jk_build", "sqb200_jk_build_device",
           "sqb200_jk_stats", "sqb200_jk_profile", "sqb200_jk_profile_read", "sqb200_jk_class_name",
           "sqb200_jk_schwarz", "sqb200_jk_mem_cutoff", "sqb200_jk_set_precision", "sqb200_oneint",
           "sqb200_peak_fma", "sqb200_batch_create", "sqb200_batch_destroy", "sqb200_batch_offsets",
           "sqb200_batch_set_step", "sqb200_batch_build_device", "sqb200_batch_stats",
           "sqb200_batch_autotune", "sqb200_jk_autotune", "sqb200_jk_tiles", "sqb200_jk_set_tiles",
           "sqb200_syev_batched", "sqb200_gradient", "sqb200_gradient_terms",
           "sqb200_segdots_create", "sqb200_segdots_run", "sqb200_segdots_destroy",
           "sqb200_jk_set_multipole", "sqb200_jk_set_persistent", "sqb200_batch_set_persistent",
           "sqb200_boys_eval", "sqb200_last_error"]


class SQB200Error(RuntimeError):
    pass


def load_library(path=LIB_PATH):
    """Load libsqb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SQB200Error("libsqb200.so not built (%s); run `make -C siam-quantum_b200`" % path)
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.sqb200_jk_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, _i32p, _i32p, _f64p, _f64p,
                                   _f64p, vp, ctypes.c_int]
    L.sqb200_jk_destroy.argtypes = [vp]
    L.sqb200_jk_build.argtypes = [vp, _f64p, _f64p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, _f64p, _f64p, _f64p]
    L.sqb200_jk_build_device.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, vp, vp, vp, vp]
    L.sqb200_jk_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    L.sqb200_jk_schwarz.argtypes = [vp, _f64p]
    L.sqb200_jk_mem_cutoff.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.sqb200_jk_profile.argtypes = [vp, ctypes.c_int]
    L.sqb200_jk_profile_read.argtypes = [vp, _f64p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.sqb200_jk_class_name.argtypes = [ctypes.c_int]
    L.sqb200_jk_set_precision.argtypes = [vp, ctypes.c_double]
    L.sqb200_jk_set_multipole.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.sqb200_jk_set_persistent.argtypes = [vp, ctypes.c_int]
    L.sqb200_boys_eval.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p, _f64p]
    L.sqb200_batch_set_persistent.argtypes = [vp, ctypes.c_int]
    L.sqb200_oneint.argtypes = [vp, ctypes.c_int, _f64p, _f64p, _f64p, _f64p, _f64p]
    L.sqb200_peak_fma.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
    L.sqb200_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
    L.sqb200_batch_destroy.argtypes = [vp]
    L.sqb200_batch_offsets.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.sqb200_batch_set_step.argtypes = [vp, _i32p, _f64p, _f64p, _f64p]
    L.sqb200_batch_build_device.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.sqb200_batch_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    L.sqb200_batch_autotune.argtypes = [vp, vp, vp, vp]
    L.sqb200_jk_autotune.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, vp]
    L.sqb200_jk_tiles.argtypes = [vp, _i32p, ctypes.c_int]
    L.sqb200_syev_batched.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]
    L.sqb200_gradient.argtypes = [vp, ctypes.c_int, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]
    L.sqb200_gradient_terms.argtypes = [vp, ctypes.c_int, _f64p, _f64p, _f64p, _f64p, _f64p, ctypes.c_int, _f64p]
    L.sqb200_jk_set_tiles.argtypes = [vp, _i32p, ctypes.c_int]
    _i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
    L.sqb200_segdots_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, _i64p, _i64p, _i32p,
                                        ctypes.c_int]
    L.sqb200_segdots_run.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int, _i32p, _i32p, vp, vp]
    L.sqb200_segdots_destroy.argtypes = [vp]
    for name in EXPORTS:
        getattr(L, name).restype = ctypes.c_int
    L.sqb200_last_error.restype = ctypes.c_char_p
    L.sqb200_jk_class_name.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise SQB200Error("sqb200 error %d: %s" % (rc, _lib.sqb200_last_error().decode()))


class JKEngine:
    """Per-basis device context.  `basis` is a basis.Basis (flat genBasis-order arrays)."""

    def __init__(self, basis, schwarz=None, device=0):
        L = load_library()
        self.nbf = basis.nbf
        self.device = device
        self._ctx = ctypes.c_void_p()
        sch = None
        if schwarz is not None:
            self._sch = np.ascontiguousarray(schwarz, dtype=np.float64).reshape(-1)
            sch = self._sch.ctypes.data_as(ctypes.c_void_p)
        _check(L.sqb200_jk_create(ctypes.byref(self._ctx), basis.nbf, basis.nprim,
                                  np.ascontiguousarray(basis.lmn.reshape(-1)),
                                  np.ascontiguousarray(basis.center.reshape(-1)), basis.exps,
                                  np.ascontiguousarray(basis.ncoef), sch, device))

    def close(self):
        if self._ctx:
            _lib.sqb200_jk_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, PA, PB=None, restricted=True, scf_cutoff=1e-10, fixed_cutoff=None,
              dscreen_rmax=float("inf"), out=None):
        """Host densities in, host JT, KA, KB out (synchronous).  `out` may supply three
        preallocated C-contiguous float64 (n, n) arrays (e.g. pinned buffers)."""
        n = self.nbf
        PA = np.ascontiguousarray(PA, dtype=np.float64).reshape(n * n)
        PBv = PA if PB is None else np.ascontiguousarray(PB, dtype=np.float64).reshape(n * n)
        if fixed_cutoff is None:
            fixed_cutoff = scf_cutoff
        if out is None:
            out = (np.empty((n, n)), np.empty((n, n)), np.empty((n, n)))
        JT, KA, KB = (o.reshape(n * n) for o in out)
        _check(_lib.sqb200_jk_build(self._ctx, PA, PBv, int(bool(restricted)), scf_cutoff,
                                    fixed_cutoff, dscreen_rmax, JT, KA, KB))
        return out

    def build_device(self, dPA, dPB, dJT, dKA, dKB=None, restricted=True, scf_cutoff=1e-10,
                     fixed_cutoff=None, dscreen_rmax=float("inf"), stream=None):
        """Device pointers (ints, e.g. torch tensor.data_ptr()) in and out; asynchronous."""
        if fixed_cutoff is None:
            fixed_cutoff = scf_cutoff
        _check(_lib.sqb200_jk_build_device(self._ctx, dPA, dPB, int(bool(restricted)), scf_cutoff,
                                           fixed_cutoff, dscreen_rmax, dJT, dKA, dKB, stream))

    def build_tensors(self, PA, PB, JT, KA, KB=None, restricted=True, scf_cutoff=1e-10,
                      fixed_cutoff=None, dscreen_rmax=float("inf"), stream=None):
        """build_device on torch tensors (float64, contiguous, (nbf, nbf), on this context's
        device), enqueued on `stream` (a torch.cuda.Stream; default: torch's current stream).
        On the legacy default stream (handle 0, which the C ABI reads as the context's own
        stream) the call synchronises before and after so that torch work stays ordered."""
        import torch
        n = self.nbf
        for t in (PA, PB, JT, KA) + (() if KB is None else (KB,)):
            if (t.dtype != torch.float64 or not t.is_cuda or t.device.index != self.device
                    or tuple(t.shape) != (n, n) or not t.is_contiguous()):
                raise ValueError("build_tensors: need contiguous float64 (%d, %d) tensors on cuda:%d"
                                 % (n, n, self.device))
        st = torch.cuda.current_stream(PA.device) if stream is None else stream
        legacy = st.cuda_stream == 0
        if legacy:
            st.synchronize()
        self.build_device(PA.data_ptr(), PB.data_ptr(), JT.data_ptr(), KA.data_ptr(),
                          None if KB is None else KB.data_ptr(), restricted=restricted,
                          scf_cutoff=scf_cutoff, fixed_cutoff=fixed_cutoff,
                          dscreen_rmax=dscreen_rmax, stream=st.cuda_stream or None)
        if legacy:
            self.stats()                           # synchronises the context stream

    def autotune(self, dPA, dPB=None, restricted=True, scf_cutoff=1e-10, fixed_cutoff=None,
                 dscreen_rmax=float("inf"), stream=None):
        """Time every FP64 form of every class (narrow tile, wide tile, swapped loop roles) on
        this density's work list and keep the fastest per class (device pointers; synchronous)."""
        if fixed_cutoff is None:
            fixed_cutoff = scf_cutoff
        _check(_lib.sqb200_jk_autotune(self._ctx, dPA, dPA if dPB is None else dPB, int(bool(restricted)),
                                       scf_cutoff, fixed_cutoff, dscreen_rmax, stream))

    def tiles(self):
        """Per class kernel: the FP64 form, 0 narrow tile, 1 wide tile, 2 swapped loop roles
        (-1: the class has one form)."""
        out = np.zeros(256, np.int32)
        n = _lib.sqb200_jk_tiles(self._ctx, out, len(out))
        if n < 0:
            _check(n)
        return out[:n].copy()

    def set_tiles(self, wide):
        w = np.ascontiguousarray(wide, dtype=np.int32)
        _check(_lib.sqb200_jk_set_tiles(self._ctx, w, len(w)))

    def stats(self):
        """dict of the last build's counters."""
        out = (ctypes.c_longlong * 6)()
        _check(_lib.sqb200_jk_stats(self._ctx, out, 6))
        return {"quartets": out[0], "prim_quartets": out[1], "flops": out[2], "shells": out[3],
                "pairs": out[4], "launches": out[5]}

    def profile(self, enable=True):
        """Start (or stop) per-class CUDA-event timing of the class kernels."""
        _check(_lib.sqb200_jk_profile(self._ctx, int(bool(enable))))

    def profile_read(self):
        """Per class kernel since profile(True): list of dicts (launches, ms, flops/launch, ...)."""
        rows = np.zeros(6 * 200)
        n = ctypes.c_int()
        _check(_lib.sqb200_jk_profile_read(self._ctx, rows, 200, ctypes.byref(n)))
        out = []
        for r in rows[: 6 * n.value].reshape(-1, 6):
            out.append({"class": _lib.sqb200_jk_class_name(int(r[0])).decode(), "index": int(r[0]),
                        "launches": int(r[1]),
                        "ms": float(r[2]), "flops": float(r[3]), "prim_quartets": int(r[4]),
                        "quartets": int(r[5])})
        return out

    def set_precision(self, fp32_below):
        """Quartets with Schwarz product below fp32_below use the FP32 kernel form (0 = FP64)."""
        _check(_lib.sqb200_jk_set_precision(self._ctx, float(fp32_below)))

    def set_multipole(self, enable, cache_rmax=float("inf")):
        """Reference-parity multipole mode for the following builds (the reference's monopole
        substitution on later visits of quartets below the memory cutoff cache_rmax)."""
        _check(_lib.sqb200_jk_set_multipole(self._ctx, int(bool(enable)), float(cache_rmax)))

    def set_persistent(self, enable=True):
        """Class kernels as persistent work-queue launches (one CTA per resident slot)."""
        _check(_lib.sqb200_jk_set_persistent(self._ctx, int(bool(enable))))

    def oneint(self, charges, coords_bohr):
        """(S, T, V) one-electron matrices for point charges at coords (bohr)."""
        n = self.nbf
        Z = np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)
        A = np.ascontiguousarray(coords_bohr, dtype=np.float64).reshape(-1)
        S = np.empty(n * n); T = np.empty(n * n); V = np.empty(n * n)
        _check(_lib.sqb200_oneint(self._ctx, len(Z), Z if len(Z) else np.zeros(1),
                                  A if len(A) else np.zeros(3), S, T, V))
        return S.reshape(n, n), T.reshape(n, n), V.reshape(n, n)

    def gradient(self, charges, coords_bohr, PA, PB, W, terms=15):
        """Nuclear gradient (natom, 3) in hartree/bohr (sqb200_gradient_terms; terms: bits
        1 nuclear repulsion, 2 PT d(T+V), 4 -W dS, 8 two-electron)."""
        Z = np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)
        A = np.ascontiguousarray(coords_bohr, dtype=np.float64).reshape(-1)
        f = lambda m: np.ascontiguousarray(m, dtype=np.float64).reshape(-1)
        g = np.zeros(3 * len(Z))
        _check(_lib.sqb200_gradient_terms(self._ctx, len(Z), Z, A, f(PA), f(PB), f(W), int(terms), g))
        return g.reshape(-1, 3)

    def mem_cutoff(self, fixed_cutoff, max_mem_mb):
        v = ctypes.c_double()
        _check(_lib.sqb200_jk_mem_cutoff(self._ctx, fixed_cutoff, int(max_mem_mb), ctypes.byref(v)))
        return v.value

    def schwarz(self):
        S = np.empty(self.nbf * self.nbf)
        _check(_lib.sqb200_jk_schwarz(self._ctx, S))
        return S.reshape(self.nbf, self.nbf)


def peak_fma(device=0, iters=4096):
    """Measured non-tensor FMA peaks (TFLOP/s) of the device: (fp64, fp32)."""
    L = load_library()
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(L.sqb200_peak_fma(device, iters, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


class SegmentDots:
    """Per-slot sums of products of packed FP64 CUDA vectors over fixed segments
    (sqb200_segdots_*): the per-molecule reductions of the SCF tail (DIIS matrix, RMS density
    change, energy) for many molecules in one pass, in a fixed summation order."""

    def __init__(self, starts, lengths, slots, nslot, device):
        L = load_library()
        self.starts = np.ascontiguousarray(starts, dtype=np.int64)
        self.lengths = np.ascontiguousarray(lengths, dtype=np.int64)
        self.slots = np.ascontiguousarray(slots, dtype=np.int32)
        self.nslot = int(nslot)
        self.device = device
        self.extent = int((self.starts + self.lengths).max()) if len(self.starts) else 0
        self._plan = ctypes.c_void_p()
        _check(L.sqb200_segdots_create(ctypes.byref(self._plan), device, len(self.starts), self.starts,
                                       self.lengths, self.slots, self.nslot))

    def __call__(self, vecs, pairs, stream=None):
        """(nslot, len(pairs)) tensor: column p sums vecs[i] * vecs[j] for pairs[p] = (i, j), or
        vecs[i] alone for j = -1.  `vecs`: 1-4 contiguous FP64 CUDA tensors on the plan's device,
        each covering every segment; runs on `stream` (default: the current stream)."""
        import torch
        if not 1 <= len(vecs) <= 4 or not 1 <= len(pairs) <= 10:
            raise ValueError("1-4 vectors and 1-10 products")
        for v in vecs:
            if (v.dtype != torch.float64 or not v.is_cuda or v.device.index != self.device
                    or not v.is_contiguous() or v.numel() < self.extent):
                raise ValueError("vectors must be contiguous FP64 CUDA tensors on device %d with at least %d "
                                 "elements" % (self.device, self.extent))
        st = torch.cuda.current_stream(vecs[0].device) if stream is None else stream
        with torch.cuda.stream(st):
            out = torch.empty((self.nslot, len(pairs)), dtype=torch.float64, device=vecs[0].device)
        ptrs = (ctypes.c_void_p * len(vecs))(*[v.data_ptr() for v in vecs])
        pi = np.array([p[0] for p in pairs], dtype=np.int32)
        pj = np.array([p[1] for p in pairs], dtype=np.int32)
        _check(_lib.sqb200_segdots_run(self._plan, len(vecs), ptrs, len(pairs), pi, pj, out.data_ptr(),
                                       st.cuda_stream))
        return out

    def close(self):
        if self._plan:
            _lib.sqb200_segdots_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def syev_batched(A, stream=None):
    """(eigenvalues, eigenvectors as columns) of a stack of symmetric FP64 CUDA matrices
    (B, n, n), by one cusolverDnXsyevBatched call; A is not modified."""
    import torch
    L = load_library()
    B_, n = A.shape[0], A.shape[-1]
    V = A.contiguous().clone()
    W = torch.empty((B_, n), dtype=torch.float64, device=A.device)
    st = torch.cuda.current_stream(A.device) if stream is None else stream
    _check(L.sqb200_syev_batched(A.device.index, n, B_, V.data_ptr(), W.data_ptr(), st.cuda_stream))
    return W, V.transpose(1, 2)


class JKBatch:
    """Batched J/K builds of many molecules (sqb200_batch_*): one launch per class kernel
    carries every molecule's work.  `engines` are JKEngine contexts (kept alive by the batch).
    Matrices are packed: molecule m's (nbf_m, nbf_m) block starts at element offsets[m]."""

    def __init__(self, engines):
        L = load_library()
        self.engines = list(engines)
        self.nmol = len(self.engines)
        self._b = ctypes.c_void_p()
        arr = (ctypes.c_void_p * self.nmol)(*[e._ctx.value for e in self.engines])
        _check(L.sqb200_batch_create(ctypes.byref(self._b), self.nmol, arr))
        off = (ctypes.c_longlong * (self.nmol + 1))()
        _check(L.sqb200_batch_offsets(self._b, off))
        self.offsets = [int(x) for x in off]
        self.total = self.offsets[-1]

    def set_step(self, restricted, scf_cutoff, fixed_cutoff=None, dscreen_rmax=None):
        """Per-molecule spin flags and cutoffs (sequences of nmol; scalars broadcast)."""
        def vec(x, dt):
            a = np.broadcast_to(np.asarray(x, dtype=dt), (self.nmol,))
            return np.ascontiguousarray(a)
        fixed_cutoff = scf_cutoff if fixed_cutoff is None else fixed_cutoff
        dscreen_rmax = float("inf") if dscreen_rmax is None else dscreen_rmax
        _check(_lib.sqb200_batch_set_step(self._b, vec([1 if r else 0 for r in np.broadcast_to(
            np.asarray(restricted), (self.nmol,))], np.int32), vec(scf_cutoff, np.float64),
            vec(fixed_cutoff, np.float64), vec(dscreen_rmax, np.float64)))

    def build_device(self, dPA, dPB, dJT, dKA, dKB, stream=None):
        """Packed device pointers in and out; asynchronous on `stream` (a cudaStream_t handle)."""
        _check(_lib.sqb200_batch_build_device(self._b, dPA, dPB, dJT, dKA, dKB, stream))

    def set_persistent(self, enable=True):
        """Persistent work-queue launches for this batch's builds."""
        _check(_lib.sqb200_batch_set_persistent(self._b, int(bool(enable))))

    def autotune(self, dPA, dPB, stream=None):
        """Tile autotuner over the batch's current work list (after set_step; synchronous)."""
        _check(_lib.sqb200_batch_autotune(self._b, dPA, dPB, stream))

    def stats(self):
        out = (ctypes.c_longlong * 6)()
        _check(_lib.sqb200_batch_stats(self._b, out, 6))
        return {"quartets": out[0], "prim_quartets": out[1], "flops": out[2], "shells": out[3],
                "pairs": out[4], "launches": out[5]}

    def close(self):
        if self._b:
            _lib.sqb200_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def boys_eval(mmax, T, device=0):
    """F_0..F_mmax at each T by the device Boys function of the class kernels (len(T) x (mmax+1))."""
    L = load_library()
    T = np.ascontiguousarray(T, dtype=np.float64)
    F = np.empty((len(T), mmax + 1))
    _check(L.sqb200_boys_eval(int(device), int(mmax), len(T), T, F))
    return F
