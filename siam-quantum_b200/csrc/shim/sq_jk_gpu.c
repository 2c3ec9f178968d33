/*
 * Drop-in GPU Fock build for Siam Quantum 2.
 *
 * Defines GTO_JK_Matrix_Quartet_Parallel with the reference's exact signature
 * (src/matrix.h:155-166) on top of the C ABI in include/sqb200.h, so the reference's SCF
 * driver (uhf_getGMatrix, src/uhf.c:112-202, called from uhf() at src/uhf.c:1596-1598) runs
 * every J/K build on the GPU unchanged.  Compile this file against the reference's own
 * headers (-I<reference>/src) and link it ahead of, or instead of, matrix.c's definition.
 *
 * Semantics kept from the reference implementation (src/matrix.c:3773-3986):
 *   - nBasis == 0 is the reset call: the device context is released (src/matrix.c:3818).
 *   - First visit after a reset: the context is built from the basis and the caller's
 *     Schwarz matrix; the memory cutoff of getMemCutoff_Parallel (src/matrix.c:3703) for
 *     opt->maxMem decides which quartets skip the density screen on that visit (the ones
 *     the reference would have cached); on later visits every quartet is density-screened.
 *   - The outer Schwarz gate is opt->SCFCutoff, the inner one fixedCutoff.
 *   - restricted (opt->restricted): K from PA only and KB = KA.
 *   - Outputs are written in full (the reference accumulates into the zeroed arrays
 *     uhf_getGMatrix passes and symmetrises them).
 *   - Work is not split over processes: childID 0 builds everything, other children (only
 *     present with -NCPU>1) return zero matrices so uhf_getGMatrix's sum is unchanged.
 * Differences: quartets are evaluated exactly (McMurchie-Davidson in FP64) unless
 * SQB200_MULTIPOLE=1 asks for the reference's monopole approximation of uncached quartets on
 * later visits (src/matrix.c:3945-3949; sqb200_jk_set_multipole with the memory cutoff of the
 * first visit), which reproduces the reference's energies under its default 3STEP cutoff
 * schedule.  Errors print a message and exit(-1), as the reference does.
 * Environment: SQB200_DEVICE selects the CUDA device (default 0); SQB200_FP32_BELOW=<tau>
 * evaluates quartets whose Schwarz product is below tau in FP32 (mixed precision; the
 * reference's SCF passes difference densities, so these errors shrink as SCF converges).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "basis.h"
#include "option.h"
#include "matrix.h"
#include "sqb200.h"

static sqb200_jk *g_ctx = NULL;
static int g_first = 1;
static double g_memcut = 0.0;

static void die(const char *what, int rc) {
	printf("GTO_JK_Matrix_Quartet_Parallel (GPU) - error %d in %s: %s\n", rc, what,
	       sqb200_last_error());
	exit(-1);
}

static void create_context(int nBasis, const struct GTOBasis_t *gto, const double *schwarz) {
	long tot = 0;
	for (int i = 0; i < nBasis; i++) tot += gto[i].nContract;
	int *nprim = malloc(sizeof(int) * nBasis), *lmn = malloc(sizeof(int) * 3 * nBasis);
	double *xyz = malloc(sizeof(double) * 3 * nBasis);
	double *ex = malloc(sizeof(double) * tot), *nc = malloc(sizeof(double) * tot);
	if (!nprim || !lmn || !xyz || !ex || !nc) die("malloc", -3);
	long k = 0;
	for (int i = 0; i < nBasis; i++) {
		nprim[i] = gto[i].nContract;
		lmn[3 * i] = gto[i].l; lmn[3 * i + 1] = gto[i].m; lmn[3 * i + 2] = gto[i].n;
		xyz[3 * i] = gto[i].x0; xyz[3 * i + 1] = gto[i].y0; xyz[3 * i + 2] = gto[i].z0;
		for (int j = 0; j < gto[i].nContract; j++, k++) {
			ex[k] = gto[i].exp[j];
			nc[k] = gto[i].norm[j] * gto[i].coef[j];
		}
	}
	const char *dev = getenv("SQB200_DEVICE");
	int rc = sqb200_jk_create(&g_ctx, nBasis, nprim, lmn, xyz, ex, nc, schwarz, dev ? atoi(dev) : 0);
	free(nprim); free(lmn); free(xyz); free(ex); free(nc);
	if (rc) die("sqb200_jk_create", rc);
	const char *f32 = getenv("SQB200_FP32_BELOW");
	if (f32 && (rc = sqb200_jk_set_precision(g_ctx, atof(f32)))) die("sqb200_jk_set_precision", rc);
}

void GTO_JK_Matrix_Quartet_Parallel(
	int childID, int nBasis, const double *PA, const double *PB,
	const struct GTOBasis_t *gto, const double *schwarz_basis, double fixedCutoff,
	double *JT, double *KA, double *KB, struct option_t *opt) {

	if (nBasis == 0) {                       /* reset call */
		if (g_ctx) sqb200_jk_destroy(g_ctx);
		g_ctx = NULL;
		g_first = 1;
		return;
	}
	size_t nn = (size_t)nBasis * nBasis;
	if (childID != 0) {                      /* the GPU build is not split over processes */
		memset(JT, 0, nn * sizeof(double));
		memset(KA, 0, nn * sizeof(double));
		memset(KB, 0, nn * sizeof(double));
		return;
	}
	if (g_first) {
		create_context(nBasis, gto, schwarz_basis);
		int rc = sqb200_jk_mem_cutoff(g_ctx, fixedCutoff, opt->maxMem, &g_memcut);
		if (rc) die("sqb200_jk_mem_cutoff", rc);
		const char *mpole = getenv("SQB200_MULTIPOLE");
		if (mpole && atoi(mpole) == 1 && (rc = sqb200_jk_set_multipole(g_ctx, 1, g_memcut)))
			die("sqb200_jk_set_multipole", rc);
	}
	double dscreen = g_first ? g_memcut : INFINITY;
	int rc = sqb200_jk_build(g_ctx, PA, PB, opt->restricted, opt->SCFCutoff, fixedCutoff,
	                         dscreen, JT, KA, KB);
	if (rc) die("sqb200_jk_build", rc);
	g_first = 0;
}
