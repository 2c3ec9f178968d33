/*
 * sqb200.h -- C ABI of the B200 two-electron Fock build (Coulomb J and exchange K).
 *
 * Plain C types only: every entry point returns an int status (0 = success, negative =
 * error, see SQB200_E*), never exits, and keeps the last error text for sqb200_last_error().
 *
 * Basis functions are described exactly as the reference's struct GTOBasis_t
 * (src/basis.h:21-32) in genBasis order (src/basis.c:529-623), flattened:
 *   nprim[i]             nContract of function i
 *   lmn[3i..3i+2]        angular indices l, m, n
 *   xyz[3i..3i+2]        centre (bohr)
 *   exps[], ncoefs[]     primitives of all functions concatenated in function order;
 *                        ncoefs = norm[k]*coef[k] (the weight genGTOShell stores,
 *                        src/matrix.c:2510-2512)
 * Density and output matrices are nbf x nbf row-major float64.
 */
#ifndef SQB200_H
#define SQB200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SQB200_OK            0
#define SQB200_EINVAL       -1   /* bad argument                                  */
#define SQB200_EUNSUPPORTED -2   /* function above f (l+m+n > 3), or a mode the basis */
                                 /* does not support (see the entry point)           */
#define SQB200_ENOMEM       -3   /* device or host allocation failed              */
#define SQB200_ECUDA        -4   /* CUDA runtime error                            */
#define SQB200_ENODEV       -5   /* no usable CUDA device                         */

typedef struct sqb200_jk sqb200_jk;   /* opaque per-basis device context */

/* Create a context: shells and shell-pair Hermite data resident on `device`.
 * Replaces the first-visit set-up of GTO_JK_Matrix_Quartet_Parallel (src/matrix.c:3830-3886:
 * genGTOShell, sortGTOShell, shell-level Schwarz).  `schwarz` is the basis-level Schwarz
 * matrix of create_Schwarz (src/matrix.c:389) the caller already holds (the argument
 * `Schwarz` of uhf_getGMatrix, src/uhf.c:112); pass NULL to compute it on the device.
 * Functions up to f (l+m+n <= 3) in shells of up to 16 functions: s, sp, p and d shells in the
 * reference's component order run in the generated class kernels, every other shell (f, as
 * read_GAMESS_BasisSet lays it out, src/basis.c:488-499, or another layout) on the generic
 * path; a function above f returns SQB200_EUNSUPPORTED. */
int sqb200_jk_create(sqb200_jk **ctx, int nbf, const int *nprim, const int *lmn,
                     const double *xyz, const double *exps, const double *ncoefs,
                     const double *schwarz, int device);

/* Release everything the context holds (the reset call nBasis==0 of
 * GTO_JK_Matrix_Quartet_Parallel, src/matrix.c:3818-3828). */
int sqb200_jk_destroy(sqb200_jk *ctx);

/* One J/K build from host densities into host outputs, overwriting JT, KA, KB.
 * Semantics of GTO_JK_Matrix_Quartet_Parallel (src/matrix.c:3773-3986) for one process:
 *   JT = J[PA+PB];  KA = -K[PA];  KB = -K[PB] (KB = KA when restricted);  all symmetric.
 * A shell quartet is skipped when r = Sch(PQ)*Sch(IJ) < scf_cutoff or r < fixed_cutoff
 * (src/matrix.c:3914-3919), and, for r < dscreen_rmax, when r * maxPShell < fixed_cutoff
 * (src/matrix.c:3921-3943).  A primitive quartet is skipped when its prefactor is below
 * 1e-15 (src/int.c:1282).  PB may equal PA.  Synchronous. */
int sqb200_jk_build(sqb200_jk *ctx, const double *PA, const double *PB, int restricted,
                    double scf_cutoff, double fixed_cutoff, double dscreen_rmax,
                    double *JT, double *KA, double *KB);

/* The same build on device buffers (allocated on the context's device) enqueued on
 * `stream` (a cudaStream_t, or NULL for the context's own stream).  Does not synchronise.
 * dPB may equal dPA; dKB may be NULL when restricted. */
int sqb200_jk_build_device(sqb200_jk *ctx, const double *dPA, const double *dPB,
                           int restricted, double scf_cutoff, double fixed_cutoff,
                           double dscreen_rmax, double *dJT, double *dKA, double *dKB,
                           void *stream);

/* The device build of sqb200_jk_build_device for callers that must not allocate GPU memory:
 * a program whose device memory is entirely owned by its own allocator (a framework's
 * caching allocator that has reserved the GPU), or a latency-critical loop that cannot afford
 * the implicit device-wide synchronisation of cudaMalloc/cudaFree.  No counterpart in the
 * reference (an addition of this library).  This call allocates nothing: all its scratch
 * (density sum, block maxima, J/K accumulators, counters, work list) lives in one static
 * device array of about 4 MB that every GPU loading the library keeps until exit; its device
 * address is looked up by sqb200_jk_create, with the context's device current.
 * Limits: nbf <= 256 and at most 65536 work items; larger inputs return SQB200_EINVAL with
 * a message.  A basis with f shells returns SQB200_EUNSUPPORTED.  The context itself (sqb200_jk_create) must already exist.  Every call shares
 * the one array, so calls that overlap on the GPU (other streams, other threads, other
 * contexts on the same device) race; serialise them.  Buffers are device pointers on the
 * context's device, enqueued on `stream` (NULL = the context's stream); not synchronised.
 * The call rebuilds the work list on the host and copies it from host memory on `stream`.
 * It runs the narrow tile form of every class in 128-thread CTAs on one stream (no autotuned
 * forms, no FP32 quartets, no side streams), so it is not the fastest build; its throughput
 * is not measured.  With the CUDA runtime's lazy module loading (the default), the first call
 * may load kernel code that no earlier call used, which takes device memory for that code;
 * CUDA_MODULE_LOADING=EAGER loads it at start-up instead.  Counters of sqb200_jk_stats are
 * not updated by this call. */
int sqb200_jk_build_noalloc(sqb200_jk *ctx, const double *dPA, const double *dPB,
                            int restricted, double scf_cutoff, double fixed_cutoff,
                            double dscreen_rmax, double *dJT, double *dKA, double *dKB,
                            void *stream);

/* Counters of the last build: out[0] shell quartets computed, out[1] primitive quartets
 * evaluated, out[2] algorithmic FP64 operations (per-class operation table),
 * out[3] shells, out[4] shell pairs, out[5] kernels the build enqueued.
 * Synchronises the context stream; after sqb200_jk_build_device on another stream, call it
 * once that stream has finished.  (No reference counterpart: instrumentation.) */
int sqb200_jk_stats(sqb200_jk *ctx, long long *out, int n);

/* Per-class timing: enable (1) or disable (0) CUDA-event timing of every class kernel
 * launch on the build's stream, clearing the accumulators.  (Instrumentation, no
 * reference counterpart.) */
int sqb200_jk_profile(sqb200_jk *ctx, int enable);

/* Rows of 6 doubles per class kernel launched since sqb200_jk_profile(ctx, 1):
 * [class index, launches, total ms, FP64 ops of the last build's launch, primitive
 * quartets of that launch, shell quartets of that launch]; *nrows receives the count. */
int sqb200_jk_profile_read(sqb200_jk *ctx, double *rows, int max_rows, int *nrows);

/* "bra|ket" pair-class name of a class-kernel index, e.g. "LL|LS" ("LL|LS f32" for the
 * mixed-precision form of that class). */
const char *sqb200_jk_class_name(int k);

/* Mixed precision: shell quartets whose Schwarz product Sch(PQ)*Sch(IJ) is below fp32_below
 * evaluate their Hermite integrals and contractions in FP32 (setup, Boys function, screening
 * and every J/K accumulation stay FP64); quartets above it, and the classes of highest angular
 * momentum (total L >= 7), stay FP64.  0 (the default) = plain FP64.  Applies to the
 * following builds of the context (not to sqb200_jk_build_noalloc).  No reference
 * counterpart: the reference computes every quartet in FP64. */
int sqb200_jk_set_precision(sqb200_jk *ctx, double fp32_below);

/* Reference-parity multipole mode (enable = 1) for the following builds of the context: the
 * reference's monopole substitution of GTO_JK_Matrix_Quartet_Parallel (src/matrix.c:3945-3949,
 * computeQuartetMPole :2609, getErrExpQuartetMPole :2551, genMultipole src/multipole.c:33).
 * The context keeps, per shell quartet surviving the outer Schwarz cutoff, the base-1.5
 * exponent of the largest error of the monopole-monopole approximation, measured the first
 * time the quartet is computed; a later build takes the monopole values for a quartet with
 * Sch(PQ)*Sch(IJ) < cache_rmax (the reference's memory cutoff: it never substitutes the
 * quartets it caches) whose 1.5^exponent * maxPShell is below fixed_cutoff.  With the
 * reference's cutoff schedule (-SCFACC=3STEP, its default) this reproduces the reference's
 * energies, approximation included.  Builds run the narrow FP64 form with one thread per
 * quartet (no FP32 quartets, no autotuned forms).  enable = 0 returns to exact quartets. */
int sqb200_jk_set_multipole(sqb200_jk *ctx, int enable, double cache_rmax);

/* Persistent work-queue launches (enable = 1) for the following builds: every class kernel runs
 * as a grid of at most one CTA per resident slot of the GPU (occupancy x SMs) whose CTAs take the
 * launch's work units -- (work item, pass), heaviest items first -- from a device counter until
 * none is left, instead of one CTA per unit.  Results are the same either way (up to the order
 * of floating-point atomics).  Default: the environment variable SQB200_PERSISTENT=1 at context
 * creation, else off.  (No reference counterpart: launch shape.) */
int sqb200_jk_set_persistent(sqb200_jk *ctx, int enable);

/* Tile autotuner.  Every class has up to three FP64 forms: 0 the narrow tile (ket functions
 * split into passes of at most 64 accumulator doubles), 1 the wide tile (fewer, larger passes;
 * classes with several passes only), 2 the swapped loop roles (outer loop over the thread's own
 * ket primitives, inner loop over the CTA's bra primitives in shared memory; passes split the
 * bra functions).  This call runs the build's prologue for the given density and cutoffs (as
 * sqb200_jk_build_device), times every form of every class on the build's own work list (CUDA
 * events, 2 launches each after one untimed) and keeps the fastest per class for the context's
 * following builds.  Leaves the context's accumulators dirty (the next build clears them);
 * synchronous.  No reference counterpart. */
int sqb200_jk_autotune(sqb200_jk *ctx, const double *dPA, const double *dPB, int restricted,
                       double scf_cutoff, double fixed_cutoff, double dscreen_rmax, void *stream);

/* Read (sqb200_jk_tiles) or set (sqb200_jk_set_tiles) the per-class FP64 form: 0, 1 or 2 as
 * above; -1 (read only) class k has one form.  Setting a form a class lacks selects 0.
 * sqb200_jk_tiles returns the number of entries written (at most n). */
int sqb200_jk_tiles(sqb200_jk *ctx, int *form, int n);
int sqb200_jk_set_tiles(sqb200_jk *ctx, const int *form, int n);

/* One-electron integrals of the context's basis on its device: overlap S, kinetic T and
 * nuclear attraction V = -sum_C Z_C <p|1/|r-C||q> for natom point charges Z at axyz (bohr),
 * each written to a host nbf*nbf array (the matrices the reference's uhf() builds with
 * overlap/kinetic/nai, src/uhf.c:1307-1334; H = T + V). */
int sqb200_oneint(sqb200_jk *ctx, int natom, const double *Z, const double *axyz,
                  double *S, double *T, double *V);

/* ---- Batched builds: many molecules' J/K in one launch per class kernel. ----
 * No reference counterpart (the reference builds one molecule per process); each molecule's
 * result is the single-molecule build of its own context (same screening, same sums up to
 * the order of floating-point additions). */
typedef struct sqb200_batch sqb200_batch;

/* Join nmol contexts (sqb200_jk_create, all on one device) into a batch.  The batch copies
 * their pair data into merged per-class arrays; the contexts must outlive the batch (their
 * Boys table, shells and FP32 threshold are read).  Packed layout of every batched matrix:
 * molecule m's nbf_m x nbf_m row-major block starts at element off[m] (sqb200_batch_offsets).
 * A context whose basis has f shells returns SQB200_EUNSUPPORTED. */
int sqb200_batch_create(sqb200_batch **batch, int nmol, sqb200_jk *const *ctxs);
int sqb200_batch_destroy(sqb200_batch *batch);

/* off[0..nmol]: off[m] = sum of nbf_k^2 for k < m; off[nmol] = total elements. */
int sqb200_batch_offsets(sqb200_batch *batch, long long *off);

/* Per-molecule spin and cutoffs of the next builds (arrays of nmol), with the meaning of
 * sqb200_jk_build's restricted / scf_cutoff / fixed_cutoff / dscreen_rmax.  Synchronises the
 * batch's streams and rebuilds the work list when a spin or Schwarz cutoff changed. */
int sqb200_batch_set_step(sqb200_batch *batch, const int *restricted, const double *scf_cutoff,
                          const double *fixed_cutoff, const double *dscreen_rmax);

/* One build of every molecule on packed device arrays, enqueued on `stream` (NULL = the batch's
 * own stream), not synchronised, no host work and no allocation: capturable into a CUDA graph.
 * For a restricted molecule its PB block must equal its PA block (the reference passes PA as
 * both spins) and its KB block receives KA. */
int sqb200_batch_build_device(sqb200_batch *batch, const double *dPA, const double *dPB,
                              double *dJT, double *dKA, double *dKB, void *stream);

/* The tile autotuner of sqb200_jk_autotune on a batch's work list of the current step (each
 * class keeps the form whose summed time over both spins is lower). */
int sqb200_batch_autotune(sqb200_batch *batch, const double *dPA, const double *dPB, void *stream);

/* Persistent work-queue launches for the batch's builds (see sqb200_jk_set_persistent; a new
 * batch starts with the setting of its first context). */
int sqb200_batch_set_persistent(sqb200_batch *batch, int enable);

/* Counters of the last batched build, as sqb200_jk_stats (summed over molecules).
 * Synchronises with the device. */
int sqb200_batch_stats(sqb200_batch *batch, long long *out, int n);

/* Eigenvalues (ascending, W: batch x n) and eigenvectors of `batch` symmetric n x n FP64
 * matrices stored back to back in A (device memory), in one cusolverDnXsyevBatched call on
 * `stream`.  On return eigenvector k of matrix b is row k of A's b-th block (A read row-major).
 * The SCF tail's eigensolve for many molecules of one padded size (in place of the
 * reference's gen_sym_SomeEigen, src/lin.c:195, per molecule).  Asynchronous; keeps one
 * cuSOLVER handle and workspace per (device, stream), grown when needed (synchronising that
 * stream then), so calls on different streams may overlap. */
int sqb200_syev_batched(int device, int n, int batch, double *A, double *W, void *stream);

/* Segmented dot products of packed FP64 vectors, for the SCF tail of many molecules: the
 * density-DIIS matrix B_xy = d_x . d_y of the last four residuals per molecule and the RMS
 * density change (conv_diis4, src/conv.c:606-844), and the energy sums, over every molecule's
 * blocks of the packed arrays at once.  A plan fixes nseg segments [seg_start, seg_start +
 * seg_len) of the vectors and the output slot (0 <= seg_slot < nslot) each one adds to;
 * sqb200_segdots_run computes out[slot * npair + p] = sum over the slot's segments of
 * vecs[pair_i[p]][e] * vecs[pair_j[p]][e] (pair_j[p] < 0: vecs[pair_i[p]][e] alone), for
 * 1 <= nvec <= 4 device vectors (each holding every segment's elements) and 1 <= npair <= 10
 * products, on `stream`, asynchronously.  The sums are taken in a fixed order (chunks of a
 * segment, then the chunks of a slot in segment order), so repeated runs agree bit for bit.
 * Runs of one plan share its scratch: issue them on one stream.  (No reference counterpart:
 * the reference reduces each molecule on the host.) */
typedef struct sqb200_segdots sqb200_segdots;
int sqb200_segdots_create(sqb200_segdots **out, int device, int nseg, const long long *seg_start,
                          const long long *seg_len, const int *seg_slot, int nslot);
int sqb200_segdots_run(sqb200_segdots *plan, int nvec, const double *const *vecs, int npair,
                       const int *pair_i, const int *pair_j, double *out, void *stream);
int sqb200_segdots_destroy(sqb200_segdots *plan);

/* Gradient of the SCF energy with respect to the natom nuclear positions (bohr), written to
 * grad (natom x 3, hartree/bohr; the reference prints forces = -grad): nuclear repulsion,
 * -sum W dS, sum PT d(T + V) with the Hellmann-Feynman terms, and the two-electron term of
 * GradEri_ShellSet_Parallel (src/grad.c:1734) -- as uhf_force (src/grad.c:2155) assembles
 * them.  PA, PB: the densities of the final orbitals; W: the energy-weighted density
 * sum_i e_i C_i C_i^T over the occupied orbitals of both spins (host arrays, nbf*nbf).  Every
 * basis function must sit on one of the nuclei.  Functions up to f in shells of at most 10
 * functions (SQB200_EUNSUPPORTED beyond); at most 65535 shell pairs and about 1800 atoms
 * (SQB200_EINVAL beyond).  The two-electron screens are the reference's (1e-10 on shell
 * quartets and on function quartets of a primitive quartet); the environment variable
 * SQB200_GRAD_SCREEN replaces that threshold (0 keeps every quartet).  Synchronous. */
int sqb200_gradient(sqb200_jk *ctx, int natom, const double *Z, const double *axyz,
                    const double *PA, const double *PB, const double *W, double *grad);

/* One or more terms of sqb200_gradient (bitwise or of SQB200_GRAD_*): nuclear repulsion,
 * sum PT d(T + V) with the Hellmann-Feynman terms, -sum W dS, the two-electron term. */
#define SQB200_GRAD_NUCLEAR 1
#define SQB200_GRAD_HCORE   2
#define SQB200_GRAD_OVERLAP 4
#define SQB200_GRAD_ERI     8
#define SQB200_GRAD_ALL     15
int sqb200_gradient_terms(sqb200_jk *ctx, int natom, const double *Z, const double *axyz,
                          const double *PA, const double *PB, const double *W, int terms, double *grad);

/* Basis-level Schwarz matrix sqrt|(pq|pq)| on the device (create_Schwarz,
 * src/matrix.c:389-440), written to the host array S (nbf*nbf). */
int sqb200_jk_schwarz(sqb200_jk *ctx, double *S);

/* Memory cutoff of getMemCutoff_Parallel (src/matrix.c:3703-3760) for nCPU=1 and maxMem
 * in MB: the Schwarz product above which the reference's first visit skips the density
 * screen (pass it as dscreen_rmax to reproduce a first reference visit). */
int sqb200_jk_mem_cutoff(sqb200_jk *ctx, double fixed_cutoff, int max_mem_mb, double *out);

/* Non-tensor FMA throughput of `device` in TFLOP/s (FMA = 2 flops): 8 independent FP64
 * (then FP32) FMA chains per thread, 8 CTAs x 256 threads per SM, `fp64_iters` x 16 steps
 * per chain, timed with CUDA events.  The denominator for the roofline fraction of the
 * J/K kernels, which run on the FP64 pipe.  (Instrumentation, no reference counterpart.) */
int sqb200_peak_fma(int device, int fp64_iters, double *fp64_tflops, double *fp32_tflops);

/* F_0..F_mmax(T[i]) for n arguments T[i] >= 0 (mmax <= 8), written to F (n x (mmax + 1)), by
 * the device Boys function the class kernels use (the role of the reference's fgamma_set,
 * src/fgamma.c:172-206).  Synchronous; allocates its own device buffers.  (Instrumentation, for
 * checking the device routine against the reference's.) */
int sqb200_boys_eval(int device, int mmax, int n, const double *T, double *F);

/* Text of the last error on this thread. */
const char *sqb200_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
