/*
 * sqport -- CPU restatement of the Siam Quantum 2 two-electron Fock-build path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  Nothing in the product links or calls this; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do, as the checker.
 * Each function restates, in our own code, the reference routine it cites.  It is pinned
 * against the reference compiled from its own sources (oracle/_ref) by tests/test_oracle.py.
 *
 * Basis arguments are flat arrays in the reference's function order (genBasis,
 * src/basis.c:529): per function nprim[i], lmn[3i..3i+2], xyz[3i..3i+2] (bohr); the
 * primitives of function i are exps/coefs/norms[off_i .. off_i+nprim[i]-1] with off_i the
 * running sum of nprim.
 */
#ifndef SQPORT_H
#define SQPORT_H

/* F_m(x), m = 0..mmax, as fgamma_set (src/fgamma.c:172-206). */
void orc_boys(int mmax, double x, double *F);

/* Shell partition and type sort as genGTOShell/sortGTOShell (src/matrix.c:2457-2541,
 * 2415-2427).  Writes per shell (sorted order) its first function, function count and type
 * (0 S, 1 L, 2 P, 3 D, 4 F, 6 other).  Returns the shell count. */
int orc_shells(int nbf, const int *nprim, const int *lmn, const double *xyz,
               const double *exps, int *first, int *nfunc, int *type);

/* sqrt|(pq|pq)| for every function pair, as create_Schwarz (src/matrix.c:389-440). */
void orc_schwarz(int nbf, const int *nprim, const int *lmn, const double *xyz,
                 const double *exps, const double *coefs, const double *norms, double *S);

/* Memory cutoff of getMemCutoff_Parallel (src/matrix.c:3703-3760) for nCPU=1. */
double orc_mem_cutoff(int nbf, const int *nprim, const int *lmn, const double *xyz,
                      const double *exps, const double *schwarz, double fixed_cutoff,
                      int max_mem_mb);

/* One FRESH J/K build as GTO_JK_Matrix_Quartet_Parallel (src/matrix.c:3773-3986) with
 * childID=0, nCPU=1 and no integral cache or multipole substitution:
 *   skip a quartet if r = Sch(PQ)*Sch(IJ) < scf_cutoff or r < fixed_cutoff;
 *   if r < dscreen_rmax also skip it when r*maxPShell < fixed_cutoff.
 * (A first reference visit density-screens only r < memCutoff; later visits screen all.)
 * Outputs overwrite JT, KA, KB (n*n row-major).  stats (may be NULL) receives
 * [shell quartets passing Schwarz, quartets computed, primitive quartets evaluated,
 *  primitive quartets cut by the 1e-15 prefactor test]. */
int orc_jk_build(int nbf, const int *nprim, const int *lmn, const double *xyz,
                 const double *exps, const double *coefs, const double *norms,
                 const double *schwarz, const double *PA, const double *PB, int restricted,
                 double scf_cutoff, double fixed_cutoff, double dscreen_rmax,
                 double *JT, double *KA, double *KB, long long *stats);

/* Contracted block (PQ|IJ) of four shells (sorted-shell indices), row-major over the four
 * shells' functions, as computeQuartetEE (src/matrix.c:2676-2916). Returns the count. */
int orc_quartet(int nbf, const int *nprim, const int *lmn, const double *xyz,
                const double *exps, const double *coefs, const double *norms,
                int P, int Q, int I, int J, double *out);

#endif
