"""Generate the per-class J/K CUDA kernels (McMurchie-Davidson ERI + fused digestion).

One kernel per quartet class (bra pair class | ket pair class) and spin mode (R: restricted,
K from PA only; U: unrestricted, K from PA and PB).  A CTA owns one bra shell pair and as many
ket shell pairs as it has threads (the runtime launches 32, 64 or 128; the bra staging strides
by blockDim.x): one shell quartet per thread, or per `isplit` threads that each take a
strided subset of the bra primitives (the digestion is linear, so each thread digests its
partial contraction).  For each quartet the threads evaluate

    (ab|cd) = sum_{bra prims i} sum_{tuv} Eb_i[ab][tuv] *
              sum_{ket prims j} sum_{tau nu phi} (-1)^(tau+nu+phi) Ek_j[cd][tau nu phi] R_ij[t+tau, u+nu, v+phi]

where Eb/Ek are Hermite expansion coefficients (with contraction coefficients, exp(-mu R^2)/p
and 1/q folded in, precomputed per primitive pair on the host) and R are the Hermite Coulomb
integrals built from the Boys function.  The inner sum over ket primitives is accumulated in
Hermite space (G[cd][tuv]); the bra transform runs once per bra primitive.  When the per-thread
state would not fit in registers the ket functions are split into blocks ("passes"); each pass
is a separate CTA (blockIdx.y) that repeats the primitive loop for its block.  The contracted
block is digested at once into

    Jacc[ab] += 2 deg PT[cd] v     Jacc[cd] += 2 deg PT[ab] v
    Kacc[ac] += deg P[bd] v        Kacc[bc] += deg P[ad] v
    Kacc[ad] += deg P[bc] v        Kacc[bd] += deg P[ac] v

(deg = 1/2 per coinciding bra shells, ket shells and bra==ket pair), so J = Jacc + Jacc^T and
K = Kacc + Kacc^T.  This reproduces what the reference's storeQuartetEE (src/matrix.c:2934)
accumulates for the six degeneracy cases.

The generator also counts the floating-point operations it emits per primitive quartet, per
bra-primitive flush and per quartet (FMA = 2) and writes that table (jk_flops.json) as the
algorithmic work W(class) used for roofline reporting.

Usage: python gen_jk_kernels.py <outdir>
"""
import itertools
import json
import os
import sys

COMP = {
    "S": [(0, 0, 0)],
    "L": [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)],
    "P": [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    "D": [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
}
LMAX = {"S": 0, "L": 1, "P": 1, "D": 2}
TYPE_ID = {"S": 0, "L": 1, "P": 2, "D": 3}        # reference sort order (src/matrix.h:238-244)
# pair classes (type of the first shell >= type of the second in the reference order)
PAIRS = [a + b for a in "SLPD" for b in "SLPD" if TYPE_ID[a] >= TYPE_ID[b]]
# bra/ket orientation: the larger pair (by functions, then L) is the bra
PAIR_ORDER = sorted(PAIRS, key=lambda p: (len(COMP[p[0]]) * len(COMP[p[1]]), LMAX[p[0]] + LMAX[p[1]], p))
STATE_MAX = int(os.environ.get("SQB_STATE_MAX", "64"))   # doubles of G + out accumulators per pass
# the mixed (FP32) form: floats of G + out per pass (a float takes one register).  LL|LL: 64
# floats -> 8 passes at 188 registers, 96 -> 6 passes at 242, 128 -> 4 passes at 255 with 132 B
# of spills; on C60 (tau 1e-5) 128 floats took the build from 64.4 to 53.5 ms: as for the FP64
# forms, fewer passes pay more than the spills cost
STATE_MAX_F32 = int(os.environ.get("SQB_STATE_MAX_F32", "128"))
# the wide tile: a second FP64 form of every class whose passes it merges (fewer passes, each
# re-deriving the Boys function and R for more ket functions, at more registers); which form a
# class runs is chosen by measurement (sqb200_jk_autotune)
STATE_MAX_WIDE = int(os.environ.get("SQB_STATE_MAX_WIDE", "128"))
# the wide form keeps its contracted-block accumulators in shared memory instead (one slot per
# thread, thread-fastest): only the Hermite intermediates G (at most G_MAX doubles) stay in
# registers, so a pass can hold more ket functions without spilling
WIDE_SMEM = int(os.environ.get("SQB_WIDE_SMEM", "0"))
# the swapped-role form (outer loop over the thread's ket primitives, inner over the shared bra
# primitives in shared memory): emitted for every class, state budget of its passes
SWAP = int(os.environ.get("SQB_SWAP", "1"))
STATE_MAX_SWAP = int(os.environ.get("SQB_STATE_MAX_SWAP", "128"))
# swapped form with its contracted block in shared memory (slots per thread, touched once per
# ket primitive at the flush): only G and the recursion stay in registers
SWAP_SMEM_O = int(os.environ.get("SQB_SWAP_SMEM", "0"))
G_MAX_SWAP = int(os.environ.get("SQB_G_MAX_SWAP", "40"))   # G doubles per pass of that form
G_MAX = int(os.environ.get("SQB_G_MAX", "48"))
PREFETCH = int(os.environ.get("SQB_PREFETCH", "0"))      # software-pipeline the ket primitive loop
TILE_KETS = int(os.environ.get("SQB_TILE_KETS", "1"))    # passes over (c, d) tiles of the ket functions
# the wide form stages the ket primitive fields a pass reads in shared memory, one record ahead
# (cp.async double buffer, thread-private slots), instead of reading them from global memory
STAGE_WIDE = int(os.environ.get("SQB_STAGE_WIDE", "0"))
# the Boys-function table columns a kernel reads, staged in shared memory once per CTA: the
# Taylor rows are gathered at each lane's own T, which from global memory touches one L1 line
# per lane and load
BOYS_SMEM = int(os.environ.get("SQB_BOYS_SMEM", "0"))
F32_MAX_L = 6               # mixed-precision kernels for classes up to this total angular momentum
MIN_BLOCKS = int(os.environ.get("SQB_MINB", "0"))   # __launch_bounds__ min CTAs per SM (0 = none)
# the same bound for the FP64 narrow-tile form only (its state is smallest, so a register cap
# spills least there); 0 = none
MIN_BLOCKS_NARROW = int(os.environ.get("SQB_MINB_NARROW", "0"))
USE_WS = int(os.environ.get("SQB_WS", "0"))
if USE_WS:
    raise SystemExit("SQB_WS: the warp-specialised form reads primitive records field-contiguously; "
                     "the pair arrays now store each record's fields kstride apart")   # also emit warp-specialised multi-pass kernels (measured slower on B200; opt-in)
CTA = 128
# Register caps (__maxnreg__) for kernels where a cap measured faster on B200: with fewer
# registers per thread more 64-thread CTAs share an SM, which pays where the spills it adds stay
# small.  C60/6-31G build, restricted forms (ms per build, uncapped -> capped): LL|LS wide
# 17.20 -> 16.19 at 128 registers (16.48 at 168, 17.70 at 144, 255 uncapped); LS|LS swapped
# 3.61 -> 3.12 at 128 (144 uncapped, no spills either way; 3.22 at 112).  LL|LL wide stays
# uncapped (40.4 ms; 42.3 at 168, 47.2 at 200).  The unrestricted forms are not capped.
REG_CAP = {"jk_LL_LS_R_w": 128, "jk_LS_LS_R_s": 128}


def kernel_qualifiers(name, bounds):
    """The launch qualifier of kernel `name`: its register cap if it has one, else
    __launch_bounds__(bounds)."""
    if name in REG_CAP:
        return "__maxnreg__(%d)" % REG_CAP[name]
    return "__launch_bounds__(%s)" % bounds


def pair_funcs(pc):
    a, b = pc
    return [(ca, cb) for ca in COMP[a] for cb in COMP[b]]


def nz(f):
    (ax, ay, az), (bx, by, bz) = f
    return [(t, u, v) for t in range(ax + bx + 1) for u in range(ay + by + 1) for v in range(az + bz + 1)]


def etable(pc):
    """E-table layout: list of (function index, (t,u,v)) in storage order, and offsets."""
    fs = pair_funcs(pc)
    off, lay = [], []
    for fi, f in enumerate(fs):
        off.append(len(lay))
        for h in nz(f):
            lay.append((fi, h))
    return fs, off, lay


def pair_L(pc):
    return LMAX[pc[0]] + LMAX[pc[1]]


class Emitter:
    def __init__(self):
        self.lines = []
        self.ind = 1

    def __call__(self, s):
        self.lines.append("  " * self.ind + s)


def gen_R(em, L, need, cons=None, emit_use=None, rt="double", fma="fma"):
    """Emit R^{(0)}_{tuv} for (t,u,v) in need; returns flop count and name map.  When
    emit_use is given it is called right after each R^{(0)} value is produced, so its
    consumers follow it and the value dies early (lower register pressure)."""
    have = {}
    flops = [0]

    def get(n, t, u, v):
        key = (n, t, u, v)
        if key in have:
            return have[key]
        if t == 0 and u == 0 and v == 0:
            have[key] = "b%d" % n
            return have[key]
        name = "r%d_%d_%d_%d" % key
        if t > 0:
            d, ax, lo = t, "X", (n + 1, t - 2, u, v)
            hi = (n + 1, t - 1, u, v)
        elif u > 0:
            d, ax, lo = u, "Y", (n + 1, t, u - 2, v)
            hi = (n + 1, t, u - 1, v)
        else:
            d, ax, lo = v, "Z", (n + 1, t, u, v - 2)
            hi = (n + 1, t, u, v - 1)
        h = get(*hi)
        if d - 1 > 0:
            l_ = get(*lo)
            if d - 1 == 1:
                em("const %s %s = %s(%s, %s, %s);" % (rt, name, fma, ax, h, l_))
                flops[0] += 2
            else:
                em("const %s %s = %s(%s, %s, %d.0%s * %s);" % (rt, name, fma, ax, h, d - 1, "f" if rt == "float" else "", l_))
                flops[0] += 3
        else:
            em("const %s %s = %s * %s;" % (rt, name, ax, h))
            flops[0] += 1
        have[key] = name
        return name

    names = {}
    for (t, u, v) in sorted(need, key=lambda x: (sum(x), x)):
        names[(t, u, v)] = get(0, t, u, v)
        if emit_use is not None:
            emit_use((t, u, v), names[(t, u, v)])
    return names, flops[0]


def boys_flops(M):
    # Taylor Horner (9 terms: 8 fma + 8 mul), downward recursion (fma + mul per order),
    # argument setup not counted here
    return 8 * 3 + M * 3


def alg_prim_flops(fk, Hb, rt, fma):
    """Algorithmic operations per primitive quartet of a class: the pass-free algorithm (primitive
    setup, one Boys evaluation at the class's highest Hermite order, every R value once, every
    ket E contraction once).  Passes that re-derive the Boys function and R for another block
    of ket functions emit more operations than this; those repeats are not counted as work."""
    need, ncons = set(), 0
    for f in fk:
        for (tau, nu, phi) in nz(f):
            for h in Hb:
                need.add((h[0] + tau, h[1] + nu, h[2] + phi))
                ncons += 1
    L = max(sum(x) for x in need)
    _, rf = gen_R(Emitter(), L, need, rt=rt, fma=fma)
    return 9 + 2 + 3 + 5 + boys_flops(L) + 2 + L + (L + 1) + rf + 2 * ncons


def ket_per_pass(bra, ket, state_max, smem_o=False):
    fb, _, _ = etable(bra)
    fk, _, _ = etable(ket)
    Hb = {h for f in fb for h in nz(f)}
    per = max(1, (G_MAX // len(Hb)) if smem_o else state_max // (len(Hb) + len(fb)))
    return min(per, len(fk))


def ket_blocks(ncd, nc, nd, per):
    """The ket function pairs cd = c*nd + d of each pass.  Every pass digests into K rows of the
    bra functions at the columns of its distinct c and its distinct d, one atomic per (bra
    function, column) and pass, so a pass covering a tc x td tile of (c, d) adds (tc + td) x
    (bra functions) instead of (1 + per) for a run of one c: tiles when they need no more passes
    than runs of consecutive pairs (TILE_KETS=0 keeps the runs)."""
    runs = [list(range(s, min(ncd, s + per))) for s in range(0, ncd, per)]
    if not TILE_KETS or nc < 2 or nd < 2 or per < 2:
        return runs
    best = None
    for tc in range(1, nc + 1):
        for td in range(1, nd + 1):
            if tc * td > per:
                continue
            npass = -(-nc // tc) * -(-nd // td)
            key = (npass, tc + td)
            if best is None or key < best[0]:
                best = (key, tc, td)
    (npass, _), tc, td = best
    if npass > len(runs):
        return runs
    return [[c * nd + d for c in range(c0, min(nc, c0 + tc)) for d in range(d0, min(nd, d0 + td))]
            for c0 in range(0, nc, tc) for d0 in range(0, nd, td)]


def n_passes(bra, ket, state_max, smem_o=False):
    fk, _, _ = etable(ket)
    per = ket_per_pass(bra, ket, state_max, smem_o)
    return (len(fk) + per - 1) // per


def gen_class(bra, ket, spin, prec="D", state_max=None, suffix="", smem_o=False, stage=False):
    """Return (kernel source, metadata) for class (bra|ket) and spin 'R' or 'U'.  prec "F"
    emits the mixed form: primitive setup, prefactor cut and Boys function in FP64, Hermite
    integrals, E tables and contracted accumulators in FP32, digestion into the FP64 J/K
    accumulators in FP64."""
    F32 = prec == "F"
    RT = "float" if F32 else "double"
    FMA = "fmaf" if F32 else "fma"
    fb, offb, layb = etable(bra)
    fk, offk, layk = etable(ket)
    nab, ncd = len(fb), len(fk)
    Lb, Lk = pair_L(bra), pair_L(ket)
    Lt = Lb + Lk
    Hb = sorted({h for f in fb for h in nz(f)}, key=lambda x: (sum(x), x))
    hidx = {h: i for i, h in enumerate(Hb)}
    na, nb_ = len(COMP[bra[0]]), len(COMP[bra[1]])
    nc, nd = len(COMP[ket[0]]), len(COMP[ket[1]])
    NB = 5 + len(layb)
    NK = 5 + len(layk)
    per = ket_per_pass(bra, ket, (STATE_MAX_F32 if F32 else STATE_MAX) if state_max is None else state_max, smem_o)
    blocks = ket_blocks(ncd, len(COMP[ket[0]]), len(COMP[ket[1]]), per)
    name = "jk_%s_%s_%s%s%s" % (bra, ket, spin, "_f32" if F32 else "", suffix)
    SO = smem_o and not F32
    ST = stage and not F32 and not SO and not PREFETCH
    MP = not F32 and suffix == "" and not SO   # the narrow FP64 form carries the multipole mode
    # ket fields one pass stages: q, Qx, Qy, Qz, prefactor and the pass's E entries
    nst = 5 + max(sum(len(nz(fk[cd])) for cd in blk) for blk in blocks)
    fl = {"prim": 0, "flush": 0, "quartet": 0, "passes": len(blocks),
          "alg_prim": alg_prim_flops(fk, Hb, RT, FMA),
          "o_dbl": nab * per if SO else (2 * nst if ST else 0)}

    em = Emitter()
    out = []
    # Boys orders of the passes (the highest Hermite order each pass needs)
    lps = []
    for blk in blocks:
        need_ = {(h[0] + t, h[1] + u, h[2] + v) for cd in blk for (t, u, v) in nz(fk[cd]) for h in Hb}
        lps.append(max(sum(x) for x in need_))
    BS = bool(BOYS_SMEM)
    bnt = 6 if F32 else 9                                   # Taylor terms of boysf / boys
    bc0, bnc = min(lps), max(lps) - min(lps) + bnt         # staged table columns
    prologue = []
    if BS:
        prologue = ["__shared__ %s sboys[BOYS_NGRID * %d];   // Boys table columns %d..%d" % (RT, bnc, bc0, bc0 + bnc - 1),
                    "for (int x = threadIdx.x; x < BOYS_NGRID * %d; x += blockDim.x)" % bnc,
                    "  sboys[x] = a.boys_tab%s[(x / %d) * BOYS_NCOL + %d + x %% %d];" % ("_f" if F32 else "", bnc, bc0, bnc),
                    "__syncthreads();"]
    minb = MIN_BLOCKS_NARROW if (MIN_BLOCKS_NARROW and suffix == "" and not F32) else MIN_BLOCKS
    out.append('extern "C" __global__ void %s' % kernel_qualifiers(
        name, "%d, %d" % (CTA, minb) if minb else "%d" % CTA))
    out.append("%s(const sqb::JKArgs a, const sqb::WorkItem* __restrict__ items) {" % name)
    if F32:
        em("extern __shared__ float sbra_f32[];")
        em("float* __restrict__ sbra = sbra_f32;")
    else:
        em("extern __shared__ double sbra[];")
    if SO:
        em("double* __restrict__ so = sbra + a.so_off;    // contracted-block accumulators, thread-fastest")
    if ST:
        em("// ket staging slots [2][%d fields][128 threads], thread-fastest (conflict-free reads)" % nst)
        em("double* __restrict__ stg = sbra + a.so_off + threadIdx.x;")
        em("const unsigned stg_s = (unsigned)__cvta_generic_to_shared(stg);")
    em("const sqb::WorkItem it = items[blockIdx.x];")
    em("const sqb::PairRec bp = a.bra_pairs[it.bra];")
    em("const sqb::MolRec mr = a.mols[it.mol];        // the molecule of this work item")
    em("double* __restrict__ Jacc = a.Jacc + mr.moff;")
    em("double* __restrict__ KAacc = a.KAacc + mr.moff;")
    em("double* __restrict__ KBacc = a.KBacc + mr.moff;")
    em("const int N = mr.nbf;")
    em("for (int x = threadIdx.x; x < bp.nprim * %d; x += blockDim.x) sbra[x] = a.bra_prims%s[bp.poff + (long long)x * bp.kstride];" % (NB, "_f" if F32 else ""))
    em("__syncthreads();")
    em("const int isplit = it.isplit;                 // threads sharing one quartet (bra primitives split)")
    em("const int kl = threadIdx.x / isplit, grp = threadIdx.x - kl * isplit;")
    em("const int pass = blockIdx.y;                   // block of ket functions handled by this CTA")
    em("bool ok = kl < it.cnt;")
    em("sqb::PairRec kp = bp;")
    em("double deg = 0.0;")
    if MP:
        em("bool mpq = false;                            // multipole mode: the quartet takes monopole values")
        em("int erx = -1, erexp = sqb::ERR_UNKNOWN;      // its error-bank slot and stored exponent")
    em("if (ok) {")
    em.ind += 1
    em("kp = a.ket_pairs[it.k0 + kl];")
    em("const double r = bp.schwarz * kp.schwarz;")
    em("ok = !(r < mr.cut_outer) && !(r < mr.cut_fixed);")
    if MP:
        em("if (ok && a.erbank) { erx = a.er_items[blockIdx.x] + kl; erexp = a.erbank[erx]; }")
        em("const bool mpc = erexp != sqb::ERR_UNKNOWN && r < a.mp_rmax;   // substitution candidate")
        em("if (ok && (r < mr.dscreen_rmax || mpc)) {")
    else:
        em("if (ok && r < mr.dscreen_rmax) {")
    em("  const bool bf = (bp.P > kp.P) || (bp.P == kp.P && bp.Q >= kp.Q);")
    em("  const int P = bf ? bp.P : kp.P, Q = bf ? bp.Q : kp.Q, I = bf ? kp.P : bp.P, J = bf ? kp.Q : bp.Q;")
    em("  const double* PM = a.PM + mr.pmoff; const int ns = mr.ns;")
    em("  const double mp = PM[P * ns + Q] + PM[I * ns + J] + PM[P * ns + I] + PM[P * ns + J] + PM[Q * ns + I] + PM[Q * ns + J];")
    if MP:
        em("  if (r < mr.dscreen_rmax) ok = !(r * mp < mr.cut_fixed);")
        em("  if (ok && mpc) mpq = a.pow15[erexp - sqb::ERR_MIN] * mp < mr.cut_fixed;")
    else:
        em("  ok = !(r * mp < mr.cut_fixed);")
    em("}")
    em("deg = (bp.P == bp.Q ? 0.5 : 1.0) * (kp.P == kp.Q ? 0.5 : 1.0) * ((a.same_class && it.bra == it.k0 + kl) ? 0.5 : 1.0);")
    em.ind -= 1
    em("}")
    for ab in range(nab):
        em("double jab%d = 0.0;" % ab)
    em("unsigned long long nprimq = 0, nflush = 0;")
    em("if (ok) {")
    em.ind += 1
    em("const %s* __restrict__ kprim = a.ket_prims%s + kp.poff;" % (RT, "_f" if F32 else ""))
    em("const int kS = kp.kstride;                   // distance between the fields of one ket record")
    em("const int nbp = %sbp.nprim, nkp = kp.nprim;" % ("mpq ? 0 : " if MP else ""))
    em("nflush = pass == 0 ? (unsigned long long)((nbp - grp + isplit - 1) / isplit) : 0ull;")
    em("const double* __restrict__ PA = a.PA + mr.moff;")
    if spin == "U":
        em("const double* __restrict__ PB = a.PB + mr.moff;")
    em("const double* __restrict__ PT = a.PT + mr.moff;")
    em("switch (pass) {")
    for bi, blk in enumerate(blocks):
        em("case %d: {  // ket functions %s" % (bi, blk))
        em.ind += 1
        if SO:
            em("for (int x = 0; x < %d; ++x) so[x * %d + threadIdx.x] = 0.0;" % (nab * per, CTA))
        else:
            for ab in range(nab):
                for cd in blk:
                    em("%s o%d_%d = 0;" % (RT, ab, cd))
        # ket E-table entries this block reads
        kent = []
        for cd in blk:
            for k, (tau, nu, phi) in enumerate(nz(fk[cd])):
                kent.append((cd, k, offk[cd] + k, -1 if (tau + nu + phi) % 2 else 1))
        if ST:
            fields = [0, 1, 2, 3, 4] + [5 + e for (cd, k, e, sg) in kent]
            def stage_code(jexpr, slotexpr):
                parts = ["const double* __restrict__ src = kprim + (long long)(%s) * %d * kS;" % (jexpr, NK),
                         "const unsigned dst = stg_s + (unsigned)(%s) * %du;" % (slotexpr, nst * 128 * 8)]
                for fi, f in enumerate(fields):
                    parts.append('asm volatile("cp.async.ca.shared.global [%%0], [%%1], 8;" :: "r"(dst + %du), "l"(src + %d * kS) : "memory");' % (fi * 128 * 8, f))
                return "{ " + " ".join(parts) + " }"
            # the first record of the sequence (i, j) = (grp, 0), (grp, 1), ..., (grp + isplit, 0), ...
            em("int slot = 0;")
            em("if (grp < nbp && nkp > 0) %s" % stage_code("0", "0"))
            em('asm volatile("cp.async.commit_group;" ::: "memory");')
        em("for (int i = grp; i < nbp; i += isplit) {")
        em.ind += 1
        em("const %s* __restrict__ bi = sbra + i * %d;" % (RT, NB))
        em("const %s p = bi[0], Px = bi[1], Py = bi[2], Pz = bi[3], kpb = bi[4];" % RT)
        for cd in blk:
            for h in Hb:
                em("%s g%d_%d = 0;" % (RT, cd, hidx[h]))
        if PREFETCH:
            # two-stage software pipeline: the record of primitive j+1 is loaded while j is
            # computed, and its Boys-table row is fetched at the end of iteration j
            em("double nq = 0.0, nQx = 0.0, nQy = 0.0, nQz = 0.0, nkq = 0.0;")
            for (cd, k, e, sg) in kent:
                em("%s nek%d_%d = 0;" % (RT, cd, k))
            em("if (nkp > 0) { nq = kprim[0]; nQx = kprim[kS]; nQy = kprim[2 * kS]; nQz = kprim[3 * kS]; nkq = kprim[4 * kS];")
            for (cd, k, e, sg) in kent:
                em("  nek%d_%d = %skprim[%d * kS];" % (cd, k, "-" if sg < 0 else "", 5 + e))
            em("}")
        em("for (int j = 0; j < nkp; ++j) {")
        em.ind += 1
        if ST:
            # the record of the next (i, j) -- it depends on j only -- is copied while this one
            # is computed; wait_group 1 leaves only that copy in flight
            em("if (j + 1 < nkp || i + isplit < nbp) %s" % stage_code("j + 1 < nkp ? j + 1 : 0", "slot ^ 1"))
            em('asm volatile("cp.async.commit_group;" ::: "memory");')
            em('asm volatile("cp.async.wait_group 1;" ::: "memory");')
            em("const double* __restrict__ sv = stg + slot * %d;" % (nst * 128))
            em("slot ^= 1;")
            em("const double q = sv[0];")
            em("const double pq = p + q;")
            em("const double rs = rsqrt(pq);")
            em("if (TWO_PI_2_5 * kpb * sv[%d] * rs < PRIM_CUTOFF) continue;" % (4 * 128))
        elif PREFETCH:
            em("const double q = nq, Qx = nQx, Qy = nQy, Qz = nQz, kq = nkq;")
            for (cd, k, e, sg) in kent:
                em("const %s ek%d_%d = nek%d_%d;" % (RT, cd, k, cd, k))
            em("if (j + 1 < nkp) { const %s* __restrict__ kn = kprim + (long long)(j + 1) * %d * kS;" % (RT, NK))
            em("  nq = kn[0]; nQx = kn[kS]; nQy = kn[2 * kS]; nQz = kn[3 * kS]; nkq = kn[4 * kS];")
            for (cd, k, e, sg) in kent:
                em("  nek%d_%d = %skn[%d * kS];" % (cd, k, "-" if sg < 0 else "", 5 + e))
            em("}")
            em("const double pq = p + q;")
            em("const double rs = rsqrt(pq);")
            em("if (TWO_PI_2_5 * kpb * kq * rs < PRIM_CUTOFF) continue;")
        elif F32:
            # the mixed form: every step in FP32 (records, set-up, Boys function, recursion,
            # contraction); only the digestion adds into the FP64 accumulators
            em("const float* __restrict__ kj = kprim + (long long)j * %d * kS;" % NK)
            em("const float q = kj[0];")
            em("const float pq = p + q;")
            em("const float rs = rsqrtf(pq);")
            em("if (TWO_PI_2_5F * kpb * kj[4 * kS] * rs < PRIM_CUTOFF_F) continue;")
        else:
            em("const %s* __restrict__ kj = kprim + (long long)j * %d * kS;" % (RT, NK))
            em("const double q = kj[0];")
            em("const double pq = p + q;")
            em("const double rs = rsqrt(pq);")
            em("if (TWO_PI_2_5 * kpb * kj[4 * kS] * rs < PRIM_CUTOFF) continue;")
        if bi == 0:
            em("++nprimq;")   # counted by the pass-0 CTAs only
        em("const %s alpha = p * q * (rs * rs);" % RT)
        if ST:
            em("const double X = Px - sv[%d], Y = Py - sv[%d], Z = Pz - sv[%d];" % (128, 256, 384))
        elif PREFETCH:
            em("const double X = Px - Qx, Y = Py - Qy, Z = Pz - Qz;")
        else:
            em("const %s X = Px - kj[kS], Y = Py - kj[2 * kS], Z = Pz - kj[3 * kS];" % RT)
        em("const %s T = alpha * %s(X, X, %s(Y, Y, Z * Z));" % (RT, FMA, FMA))
        need = set()
        for cd in blk:
            for (tau, nu, phi) in nz(fk[cd]):
                for h in Hb:
                    need.add((h[0] + tau, h[1] + nu, h[2] + phi))
        Lp = max(sum(x) for x in need)          # highest Hermite order this pass needs
        if F32:
            em("float F[%d];" % (Lp + 1))
            if BS:
                em("sqb::boys_s<%d, %d>(T, sboys + %d, F);" % (Lp, bnc, Lp - bc0))
            else:
                em("sqb::boysf<%d>(T, a.boys_tab_f, F);" % Lp)
            em("const float s0 = TWO_PI_2_5F * rs;")
            em("const float m2a = -2.0f * alpha;")
            em("float w = s0;")
        else:
            em("double F[%d];" % (Lp + 1))
            if BS:
                em("sqb::boys_s<%d, %d>(T, sboys + %d, F);" % (Lp, bnc, Lp - bc0))
            else:
                em("sqb::boys<%d>(T, a.boys_tab, F);" % Lp)
            em("const double s0 = TWO_PI_2_5 * rs;")
            em("const double m2a = -2.0 * alpha;")
            em("double w = s0;")
        pf = 9 + 2 + 3 + 5 + boys_flops(Lp) + 2  # setup: pq, alpha, XYZ diff, T, s0, m2a
        for n in range(Lp + 1):
            if n > 0:
                em("w *= m2a;")
                pf += 1
            em("const %s b%d = w * F[%d];" % (RT, n, n))
            pf += 1
        # ket E coefficients of this block, signed by (-1)^(tau+nu+phi)
        if ST:
            for fi, (cd, k, e, sg) in enumerate(kent):
                em("const %s ek%d_%d = %ssv[%d];" % (RT, cd, k, "-" if sg < 0 else "", (5 + fi) * 128))
        elif not PREFETCH:
            for (cd, k, e, sg) in kent:
                em("const %s ek%d_%d = %skj[%d * kS];" % (RT, cd, k, "-" if sg < 0 else "", 5 + e))
        # consumers of each R value: (cd, k, h) with h + (tau nu phi) = R index
        cons = {}
        for cd in blk:
            for k, (tau, nu, phi) in enumerate(nz(fk[cd])):
                for h in Hb:
                    cons.setdefault((h[0] + tau, h[1] + nu, h[2] + phi), []).append((cd, k, h))
        rn, rf = gen_R(em, Lp, need, cons=cons, emit_use=lambda key, name: [
            (em("g%d_%d = %s(ek%d_%d, %s, g%d_%d);" % (cd, hidx[h], FMA, cd, k, name, cd, hidx[h])))
            for (cd, k, h) in cons.get(key, [])], rt=RT, fma=FMA)
        pf += rf + 2 * sum(len(v) for v in cons.values())
        em.ind -= 1
        em("}")
        # flush: o[ab][cd] += sum_h Eb[ab][h] g[cd][h]
        ff = 0
        for ab in range(nab):
            if SO:
                hs = list(enumerate(nz(fb[ab])))
                em("{")
                for k, h in hs:
                    em("  const double eb%d = bi[%d];" % (k, 5 + offb[ab] + k))
                for ci, cd in enumerate(blk):
                    slot = "so[%d * %d + threadIdx.x]" % (ab * per + ci, CTA)
                    em("  { double t = %s;" % slot)
                    for k, h in hs:
                        em("    t = fma(eb%d, g%d_%d, t);" % (k, cd, hidx[h]))
                        ff += 2
                    em("    %s = t; }" % slot)
                em("}")
                continue
            for k, h in enumerate(nz(fb[ab])):
                e = offb[ab] + k
                em("{ const %s eb = bi[%d];" % (RT, 5 + e))
                for cd in blk:
                    em("  o%d_%d = %s(eb, g%d_%d, o%d_%d);" % (ab, cd, FMA, cd, hidx[h], ab, cd))
                    ff += 2
                em("}")
        em.ind -= 1
        em("}")
        fl["prim"] += pf
        fl["flush"] += ff
        if MP:
            emit_multipole(em, blk, nab, nb_, nd)
        # digestion of this block
        if SO:
            for ab in range(nab):
                for ci, cd in enumerate(blk):
                    em("const double o%d_%d = so[%d * %d + threadIdx.x];" % (ab, cd, ab * per + ci, CTA))
        qf = emit_digest(em, spin, blk, nab, na, nb_, nd)
        fl["quartet"] += qf
        em.ind -= 1
        em("} break;")
    em("}")
    em.ind -= 1
    em("}")
    # bra J: warp reduce (every lane shares the bra pair)
    em("{")
    em("  const int fP = bp.fP, fQ = bp.fQ;")
    em("  const double s2 = 2.0 * deg;")
    for ab in range(nab):
        aa, bb = divmod(ab, nb_)
        em("  { const double v = sqb::warp_sum(s2 * jab%d); if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(Jacc + (fP + %d) * N + fQ + %d, v); }" % (ab, aa, bb))
    em("}")
    em("sqb::count_add(a.counters + 0, (ok && grp == 0 && pass == 0) ? 1ull : 0ull);")
    em("sqb::count_add(a.counters + 1, nprimq);")
    em("sqb::count_add(a.counters + 2, nflush);")
    em("sqb::count_add(a.counters + 3, (ok && pass == 0) ? 1ull : 0ull);")
    out.extend(persistent_body(em.lines, prologue))
    out.append("}")
    meta = {"name": name, "bra": bra, "ket": ket, "spin": spin, "nab": nab, "ncd": ncd,
            "neb": len(layb), "nek": len(layk), "Lt": Lt, "flops": fl}
    return "\n".join(out) + "\n", meta


def persistent_body(lines, prologue=()):
    """Wrap a class kernel's body in the work loop of the persistent launch.  A work unit is one
    (work item, pass) pair.  With a.queue null the CTA runs the unit (blockIdx.x, blockIdx.y)
    and stops (one CTA per unit); otherwise a grid of about one CTA per resident slot takes
    units from the device counter a.queue until the a.nqueue units are taken.  Unit q is item
    q % nitems of pass q / nitems -- the order in which the hardware hands out the CTAs of a
    (items x passes) grid, heaviest items first in each pass -- so that the CTAs running at one
    time work on different items: the passes of one item digest into the same exchange
    elements, and running them side by side would queue their atomics on the same addresses."""
    body = [l.replace("blockIdx.x", "qi_").replace("blockIdx.y", "qp_") for l in lines]
    out = ["  __shared__ int q_next;"] + ["  " + l for l in prologue] + [
           "  const bool persistent = a.queue != nullptr;",
           "  for (int round = 0;; ++round) {",
           "    int qi_, qp_;",
           "    if (persistent) {",
           "      __syncthreads();                  // the previous unit is done with shared memory",
           "      if (threadIdx.x == 0) q_next = (int)atomicAdd(a.queue, 1ull);",
           "      __syncthreads();",
           "      const int q = q_next;",
           "      if (q >= a.nqueue) break;",
           "      const int nitems = a.nqueue / a.npass;",
           "      qp_ = q / nitems;",
           "      qi_ = q - qp_ * nitems;",
           "    } else {",
           "      if (round > 0) break;",
           "      qi_ = blockIdx.x;",
           "      qp_ = blockIdx.y;",
           "    }",
           "    {"]
    out += ["    " + l for l in body]
    out += ["    }", "  }"]
    return out


def swap_worthwhile(bra, ket):
    """The swapped form is emitted where a pass can hold at least two bra functions (or the only
    one) and the class needs at most 8 passes (beyond that the code size grows past what ptxas
    compiles in reasonable time, and the form repeats the Boys function and R too often to pay)."""
    fb, _, _ = etable(bra)
    fk, _, _ = etable(ket)
    Hk = {h for f in fk for h in nz(f)}
    per = min(len(fb), STATE_MAX_SWAP // (len(Hk) + len(fk)))
    return per >= min(2, len(fb)) and (len(fb) + per - 1) // per <= 8


def gen_class_swap(bra, ket, spin, state_max):
    """The class kernel with the loop roles swapped (suffix _s): the outer loop runs over the
    primitives of the thread's own ket pair (each record read from global memory once per pass),
    the inner loop over the CTA-shared bra pair's primitives in shared memory (broadcast reads).
    The inner loop contracts the bra E tables, G[ab][k] = sum_i sum_h Eb_i[ab][h] R_{h+k}; after
    it, the ket E tables flush, out[ab][cd] += sum_k (-1)^|k| Ek_j[cd][k] G[ab][k].  Passes
    (grid.y) split the bra functions: G + out of one pass <= state_max doubles.  FP64 only."""
    fb, offb, layb = etable(bra)
    fk, offk, layk = etable(ket)
    nab, ncd = len(fb), len(fk)
    Hk = sorted({h for f in fk for h in nz(f)}, key=lambda x: (sum(x), x))
    kidx = {h: i for i, h in enumerate(Hk)}
    na, nb_ = len(COMP[bra[0]]), len(COMP[bra[1]])
    nc, nd = len(COMP[ket[0]]), len(COMP[ket[1]])
    NB = 5 + len(layb)
    NK = 5 + len(layk)
    SO = SWAP_SMEM_O
    per = max(1, min(nab, (G_MAX_SWAP // len(Hk)) if SO else state_max // (len(Hk) + ncd)))
    blocks = [list(range(s0, min(nab, s0 + per))) for s0 in range(0, nab, per)]
    name = "jk_%s_%s_%s_s" % (bra, ket, spin)
    Hb_all = sorted({h for f in fb for h in nz(f)}, key=lambda x: (sum(x), x))
    fl = {"prim": 0, "flush": 0, "quartet": 0, "passes": len(blocks),
          "alg_prim": alg_prim_flops(fk, Hb_all, "double", "fma"), "o_dbl": per * ncd if SO else 0}
    em = Emitter()
    out = ['extern "C" __global__ void %s' % kernel_qualifiers(name, "%d" % CTA),
           "%s(const sqb::JKArgs a, const sqb::WorkItem* __restrict__ items) {" % name]
    em("extern __shared__ double sbra[];")
    if SO:
        em("double* __restrict__ so = sbra + a.so_off;    // contracted-block accumulators, thread-fastest")
    em("const sqb::WorkItem it = items[blockIdx.x];")
    em("const sqb::PairRec bp = a.bra_pairs[it.bra];")
    em("const sqb::MolRec mr = a.mols[it.mol];        // the molecule of this work item")
    em("double* __restrict__ Jacc = a.Jacc + mr.moff;")
    em("double* __restrict__ KAacc = a.KAacc + mr.moff;")
    em("double* __restrict__ KBacc = a.KBacc + mr.moff;")
    em("const int N = mr.nbf;")
    em("for (int x = threadIdx.x; x < bp.nprim * %d; x += blockDim.x) sbra[x] = a.bra_prims[bp.poff + (long long)x * bp.kstride];" % NB)
    em("__syncthreads();")
    em("const int isplit = it.isplit;                 // threads sharing one quartet (ket primitives split)")
    em("const int kl = threadIdx.x / isplit, grp = threadIdx.x - kl * isplit;")
    em("const int pass = blockIdx.y;                   // block of bra functions handled by this CTA")
    em("bool ok = kl < it.cnt;")
    em("sqb::PairRec kp = bp;")
    em("double deg = 0.0;")
    em("if (ok) {")
    em.ind += 1
    em("kp = a.ket_pairs[it.k0 + kl];")
    em("const double r = bp.schwarz * kp.schwarz;")
    em("ok = !(r < mr.cut_outer) && !(r < mr.cut_fixed);")
    em("if (ok && r < mr.dscreen_rmax) {")
    em("  const bool bf = (bp.P > kp.P) || (bp.P == kp.P && bp.Q >= kp.Q);")
    em("  const int P = bf ? bp.P : kp.P, Q = bf ? bp.Q : kp.Q, I = bf ? kp.P : bp.P, J = bf ? kp.Q : bp.Q;")
    em("  const double* PM = a.PM + mr.pmoff; const int ns = mr.ns;")
    em("  const double mp = PM[P * ns + Q] + PM[I * ns + J] + PM[P * ns + I] + PM[P * ns + J] + PM[Q * ns + I] + PM[Q * ns + J];")
    em("  ok = !(r * mp < mr.cut_fixed);")
    em("}")
    em("deg = (bp.P == bp.Q ? 0.5 : 1.0) * (kp.P == kp.Q ? 0.5 : 1.0) * ((a.same_class && it.bra == it.k0 + kl) ? 0.5 : 1.0);")
    em.ind -= 1
    em("}")
    for ab in range(nab):
        em("double jab%d = 0.0;" % ab)
    em("unsigned long long nprimq = 0, nflush = 0;")
    em("if (ok) {")
    em.ind += 1
    em("const double* __restrict__ kprim = a.ket_prims + kp.poff;")
    em("const int kS = kp.kstride;                   // distance between the fields of one ket record")
    em("const int nbp = bp.nprim, nkp = kp.nprim;")
    em("nflush = pass == 0 ? (unsigned long long)((nkp - grp + isplit - 1) / isplit) : 0ull;")
    em("const double* __restrict__ PA = a.PA + mr.moff;")
    if spin == "U":
        em("const double* __restrict__ PB = a.PB + mr.moff;")
    em("const double* __restrict__ PT = a.PT + mr.moff;")
    em("switch (pass) {")
    for bi, blk in enumerate(blocks):
        em("case %d: {  // bra functions %s" % (bi, blk))
        em.ind += 1
        slot = lambda ab, cd: "so[%d * %d + threadIdx.x]" % ((ab - blk[0]) * ncd + cd, CTA)
        if SO:
            em("for (int x = 0; x < %d; ++x) so[x * %d + threadIdx.x] = 0.0;" % (len(blk) * ncd, CTA))
        else:
            for ab in blk:
                for cd in range(ncd):
                    em("double o%d_%d = 0;" % (ab, cd))
        em("for (int j = grp; j < nkp; j += isplit) {")
        em.ind += 1
        em("const double* __restrict__ kj = kprim + (long long)j * %d * kS;" % NK)
        em("const double q = kj[0], Qx = kj[kS], Qy = kj[2 * kS], Qz = kj[3 * kS], kq = kj[4 * kS];")
        for ab in blk:
            for k in Hk:
                em("double g%d_%d = 0;" % (ab, kidx[k]))
        # bra E-table entries this block reads (from shared memory, inside the inner loop)
        bent = []
        for ab in blk:
            for e, h in enumerate(nz(fb[ab])):
                bent.append((ab, e, h))
        em("for (int i = 0; i < nbp; ++i) {")
        em.ind += 1
        em("const double* __restrict__ bi = sbra + i * %d;" % NB)
        em("const double p = bi[0];")
        em("const double pq = p + q;")
        em("const double rs = rsqrt(pq);")
        em("if (TWO_PI_2_5 * bi[4] * kq * rs < PRIM_CUTOFF) continue;")
        if bi == 0:
            em("++nprimq;")
        em("const double alpha = p * q * (rs * rs);")
        em("const double X = bi[1] - Qx, Y = bi[2] - Qy, Z = bi[3] - Qz;")
        em("const double T = alpha * fma(X, X, fma(Y, Y, Z * Z));")
        need = set()
        cons = {}
        for (ab, e, h) in bent:
            for k in Hk:
                key = (h[0] + k[0], h[1] + k[1], h[2] + k[2])
                need.add(key)
                cons.setdefault(key, []).append((ab, e, k))
        Lp = max(sum(x) for x in need)
        em("double F[%d];" % (Lp + 1))
        em("sqb::boys<%d>(T, a.boys_tab, F);" % Lp)
        em("const double s0 = TWO_PI_2_5 * rs;")
        em("const double m2a = -2.0 * alpha;")
        em("double w = s0;")
        pf = 9 + 2 + 3 + 5 + boys_flops(Lp) + 2
        for n in range(Lp + 1):
            if n > 0:
                em("w *= m2a;")
                pf += 1
            em("const double b%d = w * F[%d];" % (n, n))
            pf += 1
        for (ab, e, h) in bent:
            em("const double eb%d_%d = bi[%d];" % (ab, e, 5 + offb[ab] + e))
        rn, rf = gen_R(em, Lp, need, cons=cons, emit_use=lambda key, nm: [
            em("g%d_%d = fma(eb%d_%d, %s, g%d_%d);" % (ab, kidx[k], ab, e, nm, ab, kidx[k]))
            for (ab, e, k) in cons.get(key, [])], rt="double", fma="fma")
        pf += rf + 2 * sum(len(v) for v in cons.values())
        em.ind -= 1
        em("}")
        # flush with the ket E tables (signed by (-1)^(tau+nu+phi))
        ff = 0
        if SO:
            for cd in range(ncd):
                ks = list(enumerate(nz(fk[cd])))
                em("{")
                for e, k in ks:
                    em("  const double ek%d = %skj[%d * kS];" % (e, "-" if sum(k) % 2 else "", 5 + offk[cd] + e))
                for ab in blk:
                    em("  { double t = %s;" % slot(ab, cd))
                    for e, k in ks:
                        em("    t = fma(ek%d, g%d_%d, t);" % (e, ab, kidx[k]))
                        ff += 2
                    em("    %s = t; }" % slot(ab, cd))
                em("}")
        else:
            for cd in range(ncd):
                for e, k in enumerate(nz(fk[cd])):
                    sg = "-" if sum(k) % 2 else ""
                    em("{ const double ek = %skj[%d * kS];" % (sg, 5 + offk[cd] + e))
                    for ab in blk:
                        em("  o%d_%d = fma(ek, g%d_%d, o%d_%d);" % (ab, cd, ab, kidx[k], ab, cd))
                        ff += 2
                    em("}")
        em.ind -= 1
        em("}")
        fl["prim"] += pf
        fl["flush"] += ff
        if SO:
            for ab in blk:
                for cd in range(ncd):
                    em("const double o%d_%d = %s;" % (ab, cd, slot(ab, cd)))
        qf = emit_digest(em, spin, list(range(ncd)), nab, na, nb_, nd, ablk=blk)
        fl["quartet"] += qf
        em.ind -= 1
        em("} break;")
    em("}")
    em.ind -= 1
    em("}")
    em("{")
    em("  const int fP = bp.fP, fQ = bp.fQ;")
    em("  const double s2 = 2.0 * deg;")
    for ab in range(nab):
        aa, bb = divmod(ab, nb_)
        em("  { const double v = sqb::warp_sum(s2 * jab%d); if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(Jacc + (fP + %d) * N + fQ + %d, v); }" % (ab, aa, bb))
    em("}")
    em("sqb::count_add(a.counters + 0, (ok && grp == 0 && pass == 0) ? 1ull : 0ull);")
    em("sqb::count_add(a.counters + 1, nprimq);")
    em("sqb::count_add(a.counters + 2, nflush);")
    em("sqb::count_add(a.counters + 3, (ok && pass == 0) ? 1ull : 0ull);")
    out.extend(persistent_body(em.lines))
    out.append("}")
    meta = {"name": name, "bra": bra, "ket": ket, "spin": spin, "nab": nab, "ncd": ncd,
            "neb": len(layb), "nek": len(layk), "Lt": pair_L(bra) + pair_L(ket), "flops": fl}
    return "\n".join(out) + "\n", meta


def emit_multipole(em, blk, nab, nb_, nd):
    """Multipole mode of the narrow FP64 form: a substituted quartet (mpq) takes the monopole
    values of computeQuartetMPole (reference src/matrix.c:2609-2647) for its block; an exactly
    computed quartet whose exponent is still unknown contributes the largest |exact - monopole|
    over its block (getErrExpQuartetMPole, src/matrix.c:2551-2600) to its error-bank slot,
    combined over the passes by an atomic maximum of the bits (non-negative doubles order as
    integers; bit 63 marks the slot as measured)."""
    em("if (mpq) {")
    em("  const int fP = bp.fP, fQ = bp.fQ, fI = kp.fP, fJ = kp.fQ;")
    for ab in range(nab):
        aa, bb = divmod(ab, nb_)
        for cd in blk:
            c, d = divmod(cd, nd)
            em("  o%d_%d = sqb::mpole_value(a.mpole, N, fP + %d, fQ + %d, fI + %d, fJ + %d);" % (ab, cd, aa, bb, c, d))
    em("} else if (erexp == sqb::ERR_UNKNOWN && a.erbank) {")
    em("  const int fP = bp.fP, fQ = bp.fQ, fI = kp.fP, fJ = kp.fQ;")
    em("  double e = 0.0;")
    for ab in range(nab):
        aa, bb = divmod(ab, nb_)
        for cd in blk:
            c, d = divmod(cd, nd)
            em("  e = fmax(e, fabs(o%d_%d - sqb::mpole_value(a.mpole, N, fP + %d, fQ + %d, fI + %d, fJ + %d)));" % (ab, cd, aa, bb, c, d))
    em("  atomicMax(a.erscr + erx, (unsigned long long)__double_as_longlong(e) | (1ull << 63));")
    em("}")


def emit_digest(em, spin, blk, nab, na, nb_, nd, ablk=None):
    """Digest the contracted block o<ab>_<cd> (cd in blk, ab in ablk -- all bra functions by
    default) into the J/K accumulators.  Expects PA, PB (unrestricted), PT, N, bp, kp, deg and
    jab<ab> in scope; returns flops."""
    abs_ = list(range(nab)) if ablk is None else list(ablk)
    qf = 0
    cset = sorted({cd // nd for cd in blk})
    dset = sorted({cd % nd for cd in blk})
    em("{  // digest")
    em.ind += 1
    em("const int fP = bp.fP, fQ = bp.fQ, fI = kp.fP, fJ = kp.fQ;")
    for cd in blk:
        c, d = divmod(cd, nd)
        em("const double ptk%d = PT[(fI + %d) * N + fJ + %d];" % (cd, c, d))
    for ab in abs_:
        aa, bb = divmod(ab, nb_)
        em("const double ptb%d = PT[(fP + %d) * N + fQ + %d];" % (ab, aa, bb))
    spins = [("A", "PA")] + ([("B", "PB")] if spin == "U" else [])
    for s, P_ in spins:
        for bb in range(nb_):
            for d in dset:
                em("const double %sbd%d_%d = %s[(fQ + %d) * N + fJ + %d];" % (s, bb, d, P_, bb, d))
        for aa in sorted({ab // nb_ for ab in abs_}):
            for d in dset:
                em("const double %sad%d_%d = %s[(fP + %d) * N + fJ + %d];" % (s, aa, d, P_, aa, d))
        for bb in range(nb_):
            for c in cset:
                em("const double %sbc%d_%d = %s[(fQ + %d) * N + fI + %d];" % (s, bb, c, P_, bb, c))
        for aa in range(na):
            for c in cset:
                em("const double %sac%d_%d = %s[(fP + %d) * N + fI + %d];" % (s, aa, c, P_, aa, c))
    for ab in abs_:
        terms = " + ".join("o%d_%d * ptk%d" % (ab, cd, cd) for cd in blk)
        em("jab%d += %s;" % (ab, terms))
        qf += 2 * len(blk)
    for cd in blk:
        c, d = divmod(cd, nd)
        terms = " + ".join("o%d_%d * ptb%d" % (ab, cd, ab) for ab in abs_)
        em("atomicAdd(Jacc + (fI + %d) * N + fJ + %d, 2.0 * deg * (%s));" % (c, d, terms))
        qf += 2 * len(abs_) + 2
    for s, _ in spins:
        acc = "KAacc" if s == "A" else "KBacc"
        tg = {}
        for ab in abs_:
            aa, bb = divmod(ab, nb_)
            for cd in blk:
                c, d = divmod(cd, nd)
                o = "o%d_%d" % (ab, cd)
                tg.setdefault(("P", aa, "I", c), []).append("%s * %sbd%d_%d" % (o, s, bb, d))
                tg.setdefault(("Q", bb, "I", c), []).append("%s * %sad%d_%d" % (o, s, aa, d))
                tg.setdefault(("P", aa, "J", d), []).append("%s * %sbc%d_%d" % (o, s, bb, c))
                tg.setdefault(("Q", bb, "J", d), []).append("%s * %sac%d_%d" % (o, s, aa, c))
        for (rs_, ri, cs_, ci), terms in tg.items():
            em("atomicAdd(%s + (f%s + %d) * N + f%s + %d, deg * (%s));" % (acc, rs_, ri, cs_, ci, " + ".join(terms)))
            qf += 2 * len(terms) + 1
    em.ind -= 1
    em("}")
    return qf


WS_SMEM_MAX = 100 * 1024     # shared-memory budget of the R staging buffer


def ws_plan(bra, ket):
    """(passes, ket blocks, R list) of the warp-specialised form, or None if it does not fit."""
    fb, offb, layb = etable(bra)
    fk, offk, layk = etable(ket)
    nab, ncd = len(fb), len(fk)
    Hb = sorted({h for f in fb for h in nz(f)}, key=lambda x: (sum(x), x))
    per = max(1, STATE_MAX // (len(Hb) + nab))
    blocks = [list(range(s, min(ncd, s + per))) for s in range(0, ncd, per)]
    P = len(blocks)
    need = sorted({(h[0] + t, h[1] + u, h[2] + v) for cd in range(ncd) for (t, u, v) in nz(fk[cd]) for h in Hb},
                  key=lambda x: (sum(x), x))
    if P < 2 or P > 16 or P * len(need) * 32 * 8 > WS_SMEM_MAX:
        return None
    return P, blocks, need


def gen_class_ws(bra, ket, spin):
    """Warp-specialised form for multi-pass classes: one CTA = P warps = P ket-function blocks
    for the same 32 ket pairs (lane = ket).  Each round, warp w evaluates the Boys function and
    the Hermite integrals R of primitive step r0+w for its lane's quartet into shared memory;
    after a barrier every warp consumes the P staged steps for its own block.  R is therefore
    computed once per primitive quartet instead of once per block."""
    P, blocks, need = ws_plan(bra, ket)
    fb, offb, layb = etable(bra)
    fk, offk, layk = etable(ket)
    nab, ncd = len(fb), len(fk)
    Hb = sorted({h for f in fb for h in nz(f)}, key=lambda x: (sum(x), x))
    hidx = {h: i for i, h in enumerate(Hb)}
    na, nb_ = len(COMP[bra[0]]), len(COMP[bra[1]])
    nd = len(COMP[ket[1]])
    NB = 5 + len(layb)
    NK = 5 + len(layk)
    NR = len(need)
    ridx = {r: i for i, r in enumerate(need)}
    Lm = max(sum(x) for x in need)
    NT = 32 * P
    name = "jk_%s_%s_%s_ws" % (bra, ket, spin)
    fl = {"prim": 0, "flush": 0, "quartet": 0, "passes": P, "nr": NR}
    em = Emitter()
    out = ['extern "C" __global__ void __launch_bounds__(%d)' % NT,
           "%s(const sqb::JKArgs a, const sqb::WorkItem* __restrict__ items) {" % name]
    em("extern __shared__ double smem[];")
    em("double* __restrict__ sR = smem;                       // [%d steps][%d R][32 lanes]" % (P, NR))
    em("double* __restrict__ sbra = smem + %d;" % (P * NR * 32))
    em("const sqb::WorkItem it = items[blockIdx.x];")
    em("const sqb::PairRec bp = a.bra_pairs[it.bra];")
    em("const sqb::MolRec mr = a.mols[it.mol];        // the molecule of this work item")
    em("double* __restrict__ Jacc = a.Jacc + mr.moff;")
    em("double* __restrict__ KAacc = a.KAacc + mr.moff;")
    em("double* __restrict__ KBacc = a.KBacc + mr.moff;")
    em("const int N = mr.nbf;")
    em("for (int x = threadIdx.x; x < bp.nprim * %d; x += blockDim.x) sbra[x] = a.bra_prims[bp.poff + (long long)x * bp.kstride];" % NB)
    em("__syncthreads();")
    em("const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;")
    em("bool ok = lane < it.cnt;")
    em("const sqb::PairRec kp = a.ket_pairs[it.k0 + (ok ? lane : 0)];   // idle lanes shadow the first ket")
    em("double deg = 0.0;")
    em("if (ok) {")
    em("  const double r = bp.schwarz * kp.schwarz;")
    em("  ok = !(r < mr.cut_outer) && !(r < mr.cut_fixed);")
    em("  if (ok && r < mr.dscreen_rmax) {")
    em("    const bool bf = (bp.P > kp.P) || (bp.P == kp.P && bp.Q >= kp.Q);")
    em("    const int P = bf ? bp.P : kp.P, Q = bf ? bp.Q : kp.Q, I = bf ? kp.P : bp.P, J = bf ? kp.Q : bp.Q;")
    em("    const double* PM = a.PM + mr.pmoff; const int ns = mr.ns;")
    em("    const double mp = PM[P * ns + Q] + PM[I * ns + J] + PM[P * ns + I] + PM[P * ns + J] + PM[Q * ns + I] + PM[Q * ns + J];")
    em("    ok = !(r * mp < mr.cut_fixed);")
    em("  }")
    em("  deg = (bp.P == bp.Q ? 0.5 : 1.0) * (kp.P == kp.Q ? 0.5 : 1.0) * ((a.same_class && it.bra == it.k0 + lane) ? 0.5 : 1.0);")
    em("}")
    em("const int nbp = bp.nprim, nkp = kp.nprim, S = nbp * nkp;   // uniform over the CTA")
    em("const double* __restrict__ kprim = a.ket_prims + kp.poff;")
    em("const double* __restrict__ PA = a.PA + mr.moff;")
    if spin == "U":
        em("const double* __restrict__ PB = a.PB + mr.moff;")
    em("const double* __restrict__ PT = a.PT + mr.moff;")
    for ab in range(nab):
        em("double jab%d = 0.0;" % ab)
    em("unsigned long long nprimq = 0;")
    prod = Emitter()
    prod.ind = 0
    prod("{  // produce primitive step r0 + wp")
    prod.ind += 1
    prod("const int s = r0 + wp;")
    prod("if (s < S) {")
    prod.ind += 1
    prod("double* __restrict__ dst = sR + wp * %d + lane;" % (NR * 32))
    prod("const int i = s / nkp, j = s - i * nkp;")
    prod("const double* __restrict__ bi = sbra + i * %d;" % NB)
    prod("const double* __restrict__ kj = kprim + j * %d;" % NK)
    prod("const double p = bi[0], q = kj[0];")
    prod("const double pq = p + q;")
    prod("const double rs = rsqrt(pq);")
    prod("if (TWO_PI_2_5 * bi[4] * kj[4] * rs < PRIM_CUTOFF) {")
    for k in range(NR):
        prod("  dst[%d] = 0.0;" % (32 * k))
    prod("} else {")
    prod.ind += 1
    prod("if (ok) ++nprimq;")
    prod("const double alpha = p * q * (rs * rs);")
    prod("const double X = bi[1] - kj[1], Y = bi[2] - kj[2], Z = bi[3] - kj[3];")
    prod("const double T = alpha * fma(X, X, fma(Y, Y, Z * Z));")
    prod("double F[%d];" % (Lm + 1))
    prod("sqb::boys<%d>(T, a.boys_tab, F);" % Lm)
    prod("const double m2a = -2.0 * alpha;")
    prod("double w = TWO_PI_2_5 * rs;")
    pf = 9 + 2 + 3 + 5 + boys_flops(Lm) + 2
    for n in range(Lm + 1):
        if n > 0:
            prod("w *= m2a;")
            pf += 1
        prod("const double b%d = w * F[%d];" % (n, n))
        pf += 1
    rn, rf = gen_R(prod, Lm, set(need), emit_use=lambda key, nm: prod("dst[%d] = %s;" % (32 * ridx[key], nm)))
    pf += rf
    prod.ind -= 1
    prod("}")
    prod.ind -= 1
    prod("}")
    prod.ind -= 1
    prod("}")
    em("switch (wp) {")
    for bi_, blk in enumerate(blocks):
        em("case %d: {  // ket functions %s" % (bi_, blk))
        em.ind += 1
        for ab in range(nab):
            for cd in blk:
                em("double o%d_%d = 0.0;" % (ab, cd))
        for cd in blk:
            for h in Hb:
                em("double g%d_%d = 0.0;" % (cd, hidx[h]))
        em("int cur = 0;")
        em("for (int r0 = 0; r0 < S; r0 += %d) {" % P)
        em.ind += 1
        for line in prod.lines:
            em(line)
        em('asm volatile("bar.sync 1, %d;" ::: "memory");' % NT)
        em("for (int t = 0; t < %d; ++t) {" % P)
        em.ind += 1
        em("const int s = r0 + t;")
        em("if (s >= S) break;")
        em("const int i = s / nkp, j = s - i * nkp;")
        em("if (i != cur) {")
        em.ind += 1
        em("const double* __restrict__ bc = sbra + cur * %d;" % NB)
        ff = 0
        for ab in range(nab):
            for k, h in enumerate(nz(fb[ab])):
                e = offb[ab] + k
                em("{ const double eb = bc[%d];" % (5 + e))
                for cd in blk:
                    em("  o%d_%d = fma(eb, g%d_%d, o%d_%d);" % (ab, cd, cd, hidx[h], ab, cd))
                    ff += 2
                em("}")
        for cd in blk:
            for h in Hb:
                em("g%d_%d = 0.0;" % (cd, hidx[h]))
        em("cur = i;")
        em.ind -= 1
        em("}")
        em("const double* __restrict__ kj = kprim + j * %d;" % NK)
        em("const double* __restrict__ src = sR + t * %d + lane;" % (NR * 32))
        cons = {}
        for cd in blk:
            for k, (tau, nu, phi) in enumerate(nz(fk[cd])):
                sg = -1 if (tau + nu + phi) % 2 else 1
                em("const double ek%d_%d = %skj[%d];" % (cd, k, "-" if sg < 0 else "", 5 + offk[cd] + k))
                for h in Hb:
                    cons.setdefault((h[0] + tau, h[1] + nu, h[2] + phi), []).append((cd, k, h))
        for key in need:
            if key not in cons:
                continue
            em("{ const double r = src[%d];" % (32 * ridx[key]))
            for (cd, k, h) in cons[key]:
                em("  g%d_%d = fma(ek%d_%d, r, g%d_%d);" % (cd, hidx[h], cd, k, cd, hidx[h]))
                pf += 2
            em("}")
        em.ind -= 1
        em("}")
        em('asm volatile("bar.sync 1, %d;" ::: "memory");' % NT)
        em.ind -= 1
        em("}")
        em("if (S > 0) {")
        em.ind += 1
        em("const double* __restrict__ bc = sbra + cur * %d;" % NB)
        for ab in range(nab):
            for k, h in enumerate(nz(fb[ab])):
                e = offb[ab] + k
                em("{ const double eb = bc[%d];" % (5 + e))
                for cd in blk:
                    em("  o%d_%d = fma(eb, g%d_%d, o%d_%d);" % (ab, cd, cd, hidx[h], ab, cd))
                em("}")
        em.ind -= 1
        em("}")
        em("if (ok) {")
        em.ind += 1
        qf = emit_digest(em, spin, blk, nab, na, nb_, nd)
        em.ind -= 1
        em("}")
        fl["flush"] += ff
        fl["quartet"] += qf
        em.ind -= 1
        em("} break;")
    em("}")
    fl["prim"] = pf
    em("{")
    em("  const int fP = bp.fP, fQ = bp.fQ;")
    em("  const double s2 = 2.0 * deg;")
    for ab in range(nab):
        aa, bb = divmod(ab, nb_)
        em("  { const double v = sqb::warp_sum(s2 * jab%d); if (lane == 0 && v != 0.0) atomicAdd(Jacc + (fP + %d) * N + fQ + %d, v); }" % (ab, aa, bb))
    em("}")
    em("sqb::count_add(a.counters + 0, (ok && wp == 0) ? 1ull : 0ull);")
    em("sqb::count_add(a.counters + 1, nprimq);")
    em("sqb::count_add(a.counters + 2, (ok && wp == 0) ? (unsigned long long)nbp : 0ull);")
    em("sqb::count_add(a.counters + 3, (ok && wp == 0) ? 1ull : 0ull);")
    out.extend(em.lines)
    out.append("}")
    return "\n".join(out) + "\n", {"name": name, "flops": fl, "P": P, "NR": NR}


def write_if_changed(path, text):
    if os.path.exists(path) and open(path).read() == text:
        return
    with open(path, "w") as f:
        f.write(text)


def quartet_classes():
    cls = []
    for i, x in enumerate(PAIR_ORDER):
        for y in PAIR_ORDER[: i + 1]:
            cls.append((x, y))
    return cls


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "gen")
    os.makedirs(outdir, exist_ok=True)
    metas = []
    files = []
    head = ['// generated by gen_jk_kernels.py -- do not edit', '#include "../jk_common.cuh"', '']

    def emit(src, meta):
        # one kernel per file: the largest classes' kernels take ptxas minutes each, and
        # separate files compile in parallel
        fn = "%s.cu" % meta["name"]
        write_if_changed(os.path.join(outdir, fn), "\n".join(head + [src]))
        files.append(fn)

    for bra, ket in quartet_classes():
        for spin in ("R", "U"):
            s, m = gen_class(bra, ket, spin)
            emit(s, m)
            m["ws"] = None
            if USE_WS and ws_plan(bra, ket) is not None:
                s2, m2 = gen_class_ws(bra, ket, spin)
                emit(s2, m2)
                m["ws"] = m2
            m["wide"] = None
            if WIDE_SMEM:
                fb_, _, _ = etable(bra)
                if len(fb_) * ket_per_pass(bra, ket, 0, True) >= 8:
                    s4, m4 = gen_class(bra, ket, spin, "D", None, "_w", smem_o=True)
                    emit(s4, m4)
                    m["wide"] = m4
            elif n_passes(bra, ket, STATE_MAX_WIDE) < n_passes(bra, ket, STATE_MAX):
                s4, m4 = gen_class(bra, ket, spin, "D", STATE_MAX_WIDE, "_w", stage=bool(STAGE_WIDE))
                emit(s4, m4)
                m["wide"] = m4
            m["swap"] = None
            if SWAP and swap_worthwhile(bra, ket):
                s5, m5 = gen_class_swap(bra, ket, spin, STATE_MAX_SWAP)
                emit(s5, m5)
                m["swap"] = m5
            m["f32"] = None
            if pair_L(bra) + pair_L(ket) <= F32_MAX_L:
                s3, m3 = gen_class(bra, ket, spin, "F")
                emit(s3, m3)
                m["f32"] = m3
            metas.append(m)
    # registry
    reg = ['// generated by gen_jk_kernels.py -- do not edit', '#include "../jk_common.cuh"',
           '#include "../jk_registry.h"', '']
    for m in metas:
        reg.append('extern "C" __global__ void %s(const sqb::JKArgs, const sqb::WorkItem*);' % m["name"])
        if m["ws"]:
            reg.append('extern "C" __global__ void %s(const sqb::JKArgs, const sqb::WorkItem*);' % m["ws"]["name"])
        if m["f32"]:
            reg.append('extern "C" __global__ void %s(const sqb::JKArgs, const sqb::WorkItem*);' % m["f32"]["name"])
        if m["wide"]:
            reg.append('extern "C" __global__ void %s(const sqb::JKArgs, const sqb::WorkItem*);' % m["wide"]["name"])
        if m["swap"]:
            reg.append('extern "C" __global__ void %s(const sqb::JKArgs, const sqb::WorkItem*);' % m["swap"]["name"])
    reg.append("")
    reg.append("namespace sqb {")
    reg.append("const char* const kPairClassNames[%d] = {%s};" % (len(PAIRS), ", ".join('"%s"' % p for p in PAIRS)))
    reg.append("const ClassKernel kClassKernels[%d] = {" % (len(metas) // 2))
    for i in range(0, len(metas), 2):
        r, u = metas[i], metas[i + 1]
        wr, wu = r["ws"], u["ws"]
        reg.append('  {%d, %d, %d, %d, %d, %d, %d, %d, (const void*)%s, (const void*)%s, %d, %d, %d,' % (
            PAIRS.index(r["bra"]), PAIRS.index(r["ket"]), r["nab"], r["ncd"], r["neb"], r["nek"],
            r["Lt"], r["flops"]["passes"], r["name"], u["name"], r["flops"]["prim"], r["flops"]["flush"],
            r["flops"]["quartet"]))
        if wr:
            reg.append('   %d, %d, (const void*)%s, (const void*)%s, %d, %d, %d,' % (
                wr["P"], wr["NR"], wr["name"], wu["name"], wr["flops"]["prim"], wr["flops"]["flush"],
                wr["flops"]["quartet"]))
        else:
            reg.append('   0, 0, nullptr, nullptr, 0, 0, 0,')
        fr, fu = r["f32"], u["f32"]
        if fr:
            reg.append('   %d, (const void*)%s, (const void*)%s, %d, %d, %d,' % (
                fr["flops"]["passes"], fr["name"], fu["name"], fr["flops"]["prim"], fr["flops"]["flush"],
                fr["flops"]["quartet"]))
        else:
            reg.append('   0, nullptr, nullptr, 0, 0, 0,')
        reg.append('   %d,' % r["flops"]["alg_prim"])
        wr, wu = r["wide"], u["wide"]
        if wr:
            reg.append('   %d, (const void*)%s, (const void*)%s, %d, %d, %d, %d,' % (
                wr["flops"]["passes"], wr["name"], wu["name"], wr["flops"]["prim"], wr["flops"]["flush"],
                wr["flops"]["quartet"], wr["flops"]["o_dbl"]))
        else:
            reg.append('   0, nullptr, nullptr, 0, 0, 0, 0,')
        sr, su = r["swap"], u["swap"]
        if sr:
            reg.append('   %d, (const void*)%s, (const void*)%s, %d, %d, %d, %d},' % (
                sr["flops"]["passes"], sr["name"], su["name"], sr["flops"]["prim"], sr["flops"]["flush"],
                sr["flops"]["quartet"], sr["flops"]["o_dbl"]))
        else:
            reg.append('   0, nullptr, nullptr, 0, 0, 0, 0},')
    reg.append("};")
    reg.append("const int kNumClassKernels = %d;" % (len(metas) // 2))
    reg.append("}  // namespace sqb")
    write_if_changed(os.path.join(outdir, "jk_registry.cu"), "\n".join(reg) + "\n")
    files.append("jk_registry.cu")
    fj = {m["name"]: m["flops"] for m in metas}
    fj.update({m["ws"]["name"]: m["ws"]["flops"] for m in metas if m["ws"]})
    fj.update({m["f32"]["name"]: m["f32"]["flops"] for m in metas if m["f32"]})
    fj.update({m["wide"]["name"]: m["wide"]["flops"] for m in metas if m["wide"]})
    fj.update({m["swap"]["name"]: m["swap"]["flops"] for m in metas if m["swap"]})
    write_if_changed(os.path.join(outdir, "jk_flops.json"), json.dumps(fj, indent=0))
    # sources of an earlier layout that this run did not write
    for fn in os.listdir(outdir):
        if fn.endswith(".cu") and fn not in files:
            os.remove(os.path.join(outdir, fn))
    write_if_changed(os.path.join(outdir, "files.txt"), "\n".join(files) + "\n")
    print("generated %d kernels in %d files" % (len(metas), len(files)))


if __name__ == "__main__":
    main()
