/*
 * sqport.c -- CPU restatement (the oracle) of the reference's two-electron Fock build.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker; never by the product.  Parity of this file with the reference
 * compiled from its own sources (oracle/_ref) is asserted in tests/test_oracle.py.
 *
 * Algorithm (all FP64, as the reference):
 *   Boys function       fgamma_set            src/fgamma.c:172-206 (+ :27, :52, :139, :158)
 *   1-D THO B arrays    eriB_1d general path  src/int.c:647-873, f_coef :40-58, get_H :529-634
 *   primitive quartet   genSetBxyzSxyzF       src/int.c:1237-1371 (B for every corner computed
 *                                             directly instead of by the HRR shortcut)
 *   contracted quartet  computeQuartetEE      src/matrix.c:2676-2916
 *   digestion           storeQuartetEE        src/matrix.c:2934-3396 (six degeneracy cases)
 *   driver              GTO_JK_Matrix_Quartet_Parallel src/matrix.c:3773-3986 (fresh call,
 *                                             nCPU=1, no eeBank cache, no multipole path)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "sqport.h"

#define SH_MAXFN   16   /* MAXBASIS    src/matrix.h:222 */
#define SH_MAXPRIM 32   /* MAXCONTRACT src/matrix.h:223 */
#define LM         4    /* highest angular index per function handled here */
#define KMAX       (4 * LM + 1)
#define PRIM_CUT   1.0e-15            /* PRIMITIVE_CUTOFF src/int.h:19 */
#define TWO_PI_2_5 34.986836655249725 /* 2*pi^(5/2), the reference's literal */

typedef struct {
	double x, y, z;
	int nfunc, nprim, maxL, first, type;
	int l[SH_MAXFN], m[SH_MAXFN], n[SH_MAXFN];
	double exps[SH_MAXPRIM];
	double coef[SH_MAXPRIM][SH_MAXFN];
} shell_t;

/* ------------------------------------------------------------------ Boys function */

/* F_m(x) by the power series e^-x sum (2x)^i / ((2m+1)(2m+3)...(2m+2i+1)), stopping at
 * the first term below 1e-15 (fgamma_s, src/fgamma.c:27-41). */
static double boys_series(int m, double x){
	double denom = 2.0 * m + 1.0, term = 1.0 / denom, sum = 0.0, twox = 2.0 * x;
	for(int i = 1; i < 100; i++){
		sum += term;
		term *= twox / (denom + 2.0 * i);
		if(term < 1.0e-15) break;
	}
	return exp(-x) * sum;
}

/* F_m(x) by the asymptotic value minus a continued-fraction tail evaluated with Steed's
 * method (fgamma_steed, src/fgamma.c:52-84).  0.8862269254528 is the reference's sqrt(pi)/2. */
static double boys_cfrac(int m, double x){
	double a = m + 0.5, bi = x + 1.0 - a, ai = 0.0;
	double D = 1.0 / bi, f = D, df = D;
	for(int i = 1; i <= 100; i++){
		ai += a - 2.0 * i + 1.0;
		bi += 2.0;
		D = 1.0 / (bi + ai * D);
		df *= (bi * D - 1.0);
		f += df;
		if(fabs(df / f) < 1.0e-15) break;
	}
	double lead = 1.0, inv2x = 1.0 / (x + x);
	for(int i = 1; i <= 2 * m - 1; i += 2) lead *= i * inv2x;
	lead *= 0.8862269254528 / sqrt(x);
	return lead - 0.5 * exp(-x) * f;
}

void orc_boys(int mmax, double x, double *F){
	if(x < 0.0005){                      /* three-term small-x series */
		for(int i = 0; i <= mmax; i++)
			F[i] = 1.0 / (2.0 * i + 1.0) - x / (2.0 * i + 3.0) + x * x / (4.0 * i + 10.0);
		return;
	}
	double sx = sqrt(x);
	F[0] = 0.8862269254528 * erf(sx) / sx;
	if(mmax < 1) return;
	/* upward recursion while (2i-1)/(2x) <= 1 */
	double inv2x = 1.0 / (x + x), c = inv2x * exp(-x);
	int i;
	for(i = 1; i <= mmax; i++){
		double b = (2.0 * i - 1.0) * inv2x;
		if(b > 1.0) break;
		F[i] = b * F[i - 1] - c;
	}
	if(mmax < i) return;
	/* top value directly, then downward */
	F[mmax] = (x < mmax + 0.5) ? boys_series(mmax, x) : boys_cfrac(mmax, x);
	double twox = x + x, ex = c * twox;
	for(int j = mmax - 1; j >= i; j--)
		F[j] = (twox * F[j + 1] + ex) / (2.0 * j + 1.0);
}

/* ------------------------------------------------------------------ 1-D THO coefficients */

static const double FACT[17] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0,
	362880.0, 3628800.0, 39916800.0, 479001600.0, 6227020800.0, 87178291200.0,
	1307674368000.0, 20922789888000.0};

/* coefficients of t^k in (t+a)^l (t+b)^m (f_coef, src/int.c:40-58) */
static void poly2(double *f, int l, int m, double a, double b){
	double ca[LM + 1], cb[LM + 1];
	for(int j = 0; j <= l; j++) ca[j] = FACT[l] / (FACT[j] * FACT[l - j]) * pow(a, l - j);
	for(int k = 0; k <= m; k++) cb[k] = FACT[m] / (FACT[k] * FACT[m - k]) * pow(b, m - k);
	for(int i = 0; i <= l + m; i++) f[i] = 0.0;
	for(int j = 0; j <= l; j++)
		for(int k = 0; k <= m; k++) f[j + k] += ca[j] * cb[k];
}

/* H[L] = sum_{i=L,L+2,..} f[i] i!/(r! L!) (eta/4)^(i-r), r=(i-L)/2  (get_H, src/int.c:529) */
static void hpoly(double *H, const double *f, int lsum, double eta){
	double e = 0.25 * eta;
	for(int L = 0; L <= lsum; L++){
		double s = 0.0;
		for(int i = L; i <= lsum; i += 2){
			int r = (i - L) / 2;
			s += f[i] * FACT[i] / (FACT[r] * FACT[L]) * pow(e, i - r);
		}
		H[L] = s;
	}
}

/* B[I], I=0..l1+l2+l3+l4, of the THO 1-D factor (eriB_1d, src/int.c:647-873) */
static void tho_B(double *B, int l1, int l2, int l3, int l4, double P, double A, double Bc,
                  double Q, double C, double D, double eta1, double eta2, double zeta){
	double f1[2 * LM + 1], f2[2 * LM + 1], HL[2 * LM + 1], HM[2 * LM + 1];
	poly2(f1, l1, l2, P - A, P - Bc);
	poly2(f2, l3, l4, Q - C, Q - D);
	hpoly(HL, f1, l1 + l2, eta1);
	hpoly(HM, f2, l3 + l4, eta2);
	double qp = Q - P;
	int top = l1 + l2 + l3 + l4;
	for(int I = 0; I <= top; I++) B[I] = 0.0;
	for(int L = 0; L <= l1 + l2; L++)
		for(int M = 0; M <= l3 + l4; M++)
			for(int u = 0; u <= (L + M) / 2; u++){
				int I = L + M - u, k = L + M - 2 * u;
				double sgn = ((u + M) & 1) ? -1.0 : 1.0;
				B[I] += HL[L] * HM[M] * sgn * FACT[L + M] / FACT[u] * pow(qp, k) / FACT[k]
				        * pow(zeta, I);
			}
}

/* ------------------------------------------------------------------ shells */

static int same_shell(int i, int j, const int *nprim, const long *off, const double *xyz,
                      const double *exps){
	if(xyz[3 * i] != xyz[3 * j] || xyz[3 * i + 1] != xyz[3 * j + 1] ||
	   xyz[3 * i + 2] != xyz[3 * j + 2]) return 0;
	if(nprim[i] != nprim[j]) return 0;
	for(int k = 0; k < nprim[i]; k++) if(exps[off[i] + k] != exps[off[j] + k]) return 0;
	return 1;
}

static long *offsets(int nbf, const int *nprim){
	long *off = malloc(sizeof(long) * (nbf + 1));
	off[0] = 0;
	for(int i = 0; i < nbf; i++) off[i + 1] = off[i] + nprim[i];
	return off;
}

/* genGTOShell (src/matrix.c:2457-2541) then the stable type sort of sortGTOShell (:2415) */
static shell_t *make_shells(int nbf, const int *nprim, const int *lmn, const double *xyz,
                            const double *exps, const double *coefs, const double *norms,
                            int *nsh_out){
	long *off = offsets(nbf, nprim);
	shell_t *sh = calloc(nbf, sizeof(shell_t));
	int ns = 0;
	for(int p = 0; p < nbf; ){
		shell_t *s = sh + ns;
		s->first = p; s->x = xyz[3 * p]; s->y = xyz[3 * p + 1]; s->z = xyz[3 * p + 2];
		s->nprim = nprim[p];
		for(int k = 0; k < nprim[p]; k++) s->exps[k] = exps[off[p] + k];
		int q = p;
		while(q < nbf && same_shell(p, q, nprim, off, xyz, exps) && s->nfunc < SH_MAXFN){
			int L = lmn[3 * q] + lmn[3 * q + 1] + lmn[3 * q + 2];
			if(L > s->maxL) s->maxL = L;
			s->l[s->nfunc] = lmn[3 * q]; s->m[s->nfunc] = lmn[3 * q + 1];
			s->n[s->nfunc] = lmn[3 * q + 2];
			for(int k = 0; k < nprim[q]; k++)
				s->coef[k][s->nfunc] = norms[off[q] + k] * coefs[off[q] + k];
			s->nfunc++;
			q++;
		}
		switch(s->nfunc){
		case 1: s->type = 0; break; case 4: s->type = 1; break; case 3: s->type = 2; break;
		case 6: s->type = 3; break; case 10: s->type = 4; break; default: s->type = 6;
		}
		p = q; ns++;
	}
	/* stable sort by type (equivalent to the reference's adjacent-swap passes) */
	for(int a = 1; a < ns; a++){
		shell_t t = sh[a]; int b = a - 1;
		while(b >= 0 && sh[b].type > t.type){ sh[b + 1] = sh[b]; b--; }
		sh[b + 1] = t;
	}
	free(off);
	*nsh_out = ns;
	return sh;
}

int orc_shells(int nbf, const int *nprim, const int *lmn, const double *xyz,
               const double *exps, int *first, int *nfunc, int *type){
	/* coefficients are irrelevant to the partition; pass dummies */
	long tot = 0;
	for(int i = 0; i < nbf; i++) tot += nprim[i];
	double *one = malloc(sizeof(double) * (tot > 0 ? tot : 1));
	for(long i = 0; i < tot; i++) one[i] = 1.0;
	int ns;
	shell_t *sh = make_shells(nbf, nprim, lmn, xyz, exps, one, one, &ns);
	for(int s = 0; s < ns; s++){ first[s] = sh[s].first; nfunc[s] = sh[s].nfunc; type[s] = sh[s].type; }
	free(sh); free(one);
	return ns;
}

/* ------------------------------------------------------------------ contracted quartet */

/* B tables for every (a,b,c,d) with a<=la, .. per axis; index ((((a*(lb+1)+b)*(lc+1)+c)*(ld+1)+d)*KMAX + k */
static double Bx_[(LM + 1) * (LM + 1) * (LM + 1) * (LM + 1) * KMAX];
static double By_[(LM + 1) * (LM + 1) * (LM + 1) * (LM + 1) * KMAX];
static double Bz_[(LM + 1) * (LM + 1) * (LM + 1) * (LM + 1) * KMAX];

static long long g_prim_eval, g_prim_cut;

/* computeQuartetEE (src/matrix.c:2676-2916) with genSetBxyzSxyzF (src/int.c:1237-1371) */
static int quartet(const shell_t *P, const shell_t *Q, const shell_t *I, const shell_t *J,
                   double *EE, int apply_cut){
	int nP = P->nfunc, nQ = Q->nfunc, nI = I->nfunc, nJ = J->nfunc;
	int n = nP * nQ * nI * nJ;
	int la = P->maxL, lb = Q->maxL, lc = I->maxL, ld = J->maxL;
	int s3 = ld + 1, s2 = s3 * (lc + 1), s1 = s2 * (lb + 1);
	double F[KMAX];
	memset(EE, 0, sizeof(double) * n);
	for(int pc = 0; pc < P->nprim; pc++)
	for(int qc = 0; qc < Q->nprim; qc++)
	for(int ic = 0; ic < I->nprim; ic++)
	for(int jc = 0; jc < J->nprim; jc++){
		double aa = P->exps[pc], ab = Q->exps[qc], ac = I->exps[ic], ad = J->exps[jc];
		double eta1 = 1.0 / (aa + ab), eta2 = 1.0 / (ac + ad);
		double zeta = 4.0 * (aa + ab) * (ac + ad) / (aa + ab + ac + ad);
		double px = (aa * P->x + ab * Q->x) * eta1, py = (aa * P->y + ab * Q->y) * eta1,
		       pz = (aa * P->z + ab * Q->z) * eta1;
		double qx = (ac * I->x + ad * J->x) * eta2, qy = (ac * I->y + ad * J->y) * eta2,
		       qz = (ac * I->z + ad * J->z) * eta2;
		double rab2 = (P->x - Q->x) * (P->x - Q->x) + (P->y - Q->y) * (P->y - Q->y) +
		              (P->z - Q->z) * (P->z - Q->z);
		double rcd2 = (I->x - J->x) * (I->x - J->x) + (I->y - J->y) * (I->y - J->y) +
		              (I->z - J->z) * (I->z - J->z);
		double rpq2 = (px - qx) * (px - qx) + (py - qy) * (py - qy) + (pz - qz) * (pz - qz);
		double t = TWO_PI_2_5 * eta1 * eta2 / sqrt(aa + ab + ac + ad) *
		           exp(-aa * ab * rab2 * eta1 - ac * ad * rcd2 * eta2);
		if(apply_cut && t < PRIM_CUT){ g_prim_cut++; continue; }
		g_prim_eval++;
		orc_boys(la + lb + lc + ld, 0.25 * rpq2 * zeta, F);
		for(int a = 0; a <= la; a++) for(int b = 0; b <= lb; b++)
		for(int c = 0; c <= lc; c++) for(int d = 0; d <= ld; d++){
			long o = (long)(a * s1 + b * s2 + c * s3 + d) * KMAX;
			tho_B(Bx_ + o, a, b, c, d, px, P->x, Q->x, qx, I->x, J->x, eta1, eta2, zeta);
			tho_B(By_ + o, a, b, c, d, py, P->y, Q->y, qy, I->y, J->y, eta1, eta2, zeta);
			tho_B(Bz_ + o, a, b, c, d, pz, P->z, Q->z, qz, I->z, J->z, eta1, eta2, zeta);
		}
		int e = 0;
		for(int p = 0; p < nP; p++) for(int q = 0; q < nQ; q++)
		for(int i = 0; i < nI; i++) for(int j = 0; j < nJ; j++, e++){
			const double *bx = Bx_ + (long)(P->l[p] * s1 + Q->l[q] * s2 + I->l[i] * s3 + J->l[j]) * KMAX;
			const double *by = By_ + (long)(P->m[p] * s1 + Q->m[q] * s2 + I->m[i] * s3 + J->m[j]) * KMAX;
			const double *bz = Bz_ + (long)(P->n[p] * s1 + Q->n[q] * s2 + I->n[i] * s3 + J->n[j]) * KMAX;
			int mx = P->l[p] + Q->l[q] + I->l[i] + J->l[j];
			int my = P->m[p] + Q->m[q] + I->m[i] + J->m[j];
			int mz = P->n[p] + Q->n[q] + I->n[i] + J->n[j];
			double s = 0.0;
			for(int kx = 0; kx <= mx; kx++)
				for(int ky = 0; ky <= my; ky++)
					for(int kz = 0; kz <= mz; kz++)
						s += bx[kx] * by[ky] * bz[kz] * F[kx + ky + kz];
			EE[e] += s * t * P->coef[pc][p] * Q->coef[qc][q] * I->coef[ic][i] * J->coef[jc][j];
		}
	}
	return n;
}

int orc_quartet(int nbf, const int *nprim, const int *lmn, const double *xyz,
                const double *exps, const double *coefs, const double *norms,
                int P, int Q, int I, int J, double *out){
	int ns;
	shell_t *sh = make_shells(nbf, nprim, lmn, xyz, exps, coefs, norms, &ns);
	int n = quartet(sh + P, sh + Q, sh + I, sh + J, out, 1);
	free(sh);
	return n;
}

/* ------------------------------------------------------------------ Schwarz */

void orc_schwarz(int nbf, const int *nprim, const int *lmn, const double *xyz,
                 const double *exps, const double *coefs, const double *norms, double *S){
	/* contr_eri of (pq|pq) per function pair (src/matrix.c:250-292, 389-440): no
	 * primitive cut; computed here through one-function pseudo-shells */
	long *off = offsets(nbf, nprim);
	shell_t *f = calloc(nbf, sizeof(shell_t));
	for(int p = 0; p < nbf; p++){
		f[p].x = xyz[3 * p]; f[p].y = xyz[3 * p + 1]; f[p].z = xyz[3 * p + 2];
		f[p].nfunc = 1; f[p].nprim = nprim[p];
		f[p].l[0] = lmn[3 * p]; f[p].m[0] = lmn[3 * p + 1]; f[p].n[0] = lmn[3 * p + 2];
		f[p].maxL = f[p].l[0] + f[p].m[0] + f[p].n[0];
		for(int k = 0; k < nprim[p]; k++){
			f[p].exps[k] = exps[off[p] + k];
			f[p].coef[k][0] = norms[off[p] + k] * coefs[off[p] + k];
		}
	}
	double v;
	for(int p = 0; p < nbf; p++)
		for(int q = 0; q < nbf; q++){
			quartet(f + p, f + q, f + p, f + q, &v, 0);
			S[p * nbf + q] = sqrt(fabs(v));
		}
	free(f); free(off);
}

/* ------------------------------------------------------------------ digestion */

enum { T_ALLDISTINCT = 0, T_PIQJ = 1, T_IJPAIR = 2, T_PQPAIR = 3, T_2PAIRS = 4, T_ALLSAME = 5 };

/* element (p,q,i,j) of a block stored row-major over shells (P,Q,I,J) */
typedef struct { int sp, sq, si, sj; } strides_t;

/* J part of storeQuartetEE (macros RSTOREJ_*, src/matrix.c:3181-3246):
 * bra (X,Y) receives sum_kl PT[k][l] (xy|kl) * (ket_distinct ? 2 : 1), written to
 * JT[x][y] and, when the bra shells differ, also to JT[y][x]. */
static void store_J(const shell_t *X, const shell_t *Y, const shell_t *K, const shell_t *L,
                    int sx, int sy, int sk, int sl, int bra_distinct, int ket_distinct,
                    int nbf, double *JT, const double *PT, const double *EE){
	for(int x = 0; x < X->nfunc; x++)
	for(int y = 0; y < Y->nfunc; y++){
		double g = 0.0;
		for(int k = 0; k < K->nfunc; k++)
			for(int l = 0; l < L->nfunc; l++){
				double e = EE[x * sx + y * sy + k * sk + l * sl];
				if(ket_distinct) e += e;
				g += PT[(K->first + k) * nbf + L->first + l] * e;
			}
		JT[(x + X->first) * nbf + (y + Y->first)] += g;
		if(bra_distinct) JT[(y + Y->first) * nbf + (x + X->first)] += g;
	}
}

/* K part (macros RSTOREK_* / USTOREK_*, src/matrix.c:3248-3305): for x in X, k in K,
 * G = sum_{y,l} P[y][l] (xy|kl); K[x][k] -= G and, if both, K[k][x] -= G. */
static void store_K(const shell_t *X, const shell_t *Y, const shell_t *K, const shell_t *L,
                    int sx, int sy, int sk, int sl, int both, int nbf, int nspin,
                    double *KA, double *KB, const double *PA, const double *PB,
                    const double *EE){
	for(int x = 0; x < X->nfunc; x++)
	for(int k = 0; k < K->nfunc; k++){
		double ga = 0.0, gb = 0.0;
		for(int y = 0; y < Y->nfunc; y++)
			for(int l = 0; l < L->nfunc; l++){
				double e = EE[x * sx + y * sy + k * sk + l * sl];
				int o = (Y->first + y) * nbf + L->first + l;
				ga += PA[o] * e;
				if(nspin == 2) gb += PB[o] * e;
			}
		int a = (x + X->first) * nbf + (k + K->first), b = (k + K->first) * nbf + (x + X->first);
		KA[a] -= ga; if(both) KA[b] -= ga;
		if(nspin == 2){ KB[a] -= gb; if(both) KB[b] -= gb; }
	}
}

/* storeQuartetEE case table (src/matrix.c:3307-3395) */
static void store_quartet(const shell_t *P, const shell_t *Q, const shell_t *I,
                          const shell_t *J, int type, int restricted, int nbf, double *JT,
                          double *KA, double *KB, const double *PT, const double *PA,
                          const double *PB, const double *EE){
	int jj = 1, ii = J->nfunc, qq = I->nfunc * J->nfunc, pp = Q->nfunc * qq;
	int ns = restricted ? 1 : 2;
	switch(type){
	case T_ALLSAME:
		store_J(P, Q, I, J, pp, qq, ii, jj, 0, 0, nbf, JT, PT, EE);
		store_K(P, Q, I, J, pp, qq, ii, jj, 0, nbf, ns, KA, KB, PA, PB, EE);
		break;
	case T_2PAIRS:
		store_J(P, Q, I, J, pp, qq, ii, jj, 0, 0, nbf, JT, PT, EE);
		store_J(I, J, P, Q, ii, jj, pp, qq, 0, 0, nbf, JT, PT, EE);
		store_K(P, Q, I, J, pp, qq, ii, jj, 1, nbf, ns, KA, KB, PA, PB, EE);
		break;
	case T_PQPAIR:
		store_J(P, Q, I, J, pp, qq, ii, jj, 0, 1, nbf, JT, PT, EE);
		store_J(I, J, P, Q, ii, jj, pp, qq, 1, 0, nbf, JT, PT, EE);
		store_K(P, Q, I, J, pp, qq, ii, jj, 1, nbf, ns, KA, KB, PA, PB, EE);
		store_K(P, Q, J, I, pp, qq, jj, ii, 1, nbf, ns, KA, KB, PA, PB, EE);
		break;
	case T_IJPAIR:
		store_J(P, Q, I, J, pp, qq, ii, jj, 1, 0, nbf, JT, PT, EE);
		store_J(I, J, P, Q, ii, jj, pp, qq, 0, 1, nbf, JT, PT, EE);
		store_K(P, Q, I, J, pp, qq, ii, jj, 1, nbf, ns, KA, KB, PA, PB, EE);
		store_K(Q, P, I, J, qq, pp, ii, jj, 1, nbf, ns, KA, KB, PA, PB, EE);
		break;
	case T_PIQJ:
		store_J(P, Q, I, J, pp, qq, ii, jj, 1, 1, nbf, JT, PT, EE);
		store_K(P, Q, I, J, pp, qq, ii, jj, 0, nbf, ns, KA, KB, PA, PB, EE);
		store_K(P, Q, J, I, pp, qq, jj, ii, 0, nbf, ns, KA, KB, PA, PB, EE);
		store_K(Q, P, I, J, qq, pp, ii, jj, 0, nbf, ns, KA, KB, PA, PB, EE);
		store_K(Q, P, J, I, qq, pp, jj, ii, 0, nbf, ns, KA, KB, PA, PB, EE);
		break;
	default:
		store_J(P, Q, I, J, pp, qq, ii, jj, 1, 1, nbf, JT, PT, EE);
		store_J(I, J, P, Q, ii, jj, pp, qq, 1, 1, nbf, JT, PT, EE);
		store_K(P, Q, I, J, pp, qq, ii, jj, 1, nbf, ns, KA, KB, PA, PB, EE);
		store_K(P, Q, J, I, pp, qq, jj, ii, 1, nbf, ns, KA, KB, PA, PB, EE);
		store_K(Q, P, I, J, qq, pp, ii, jj, 1, nbf, ns, KA, KB, PA, PB, EE);
		store_K(Q, P, J, I, qq, pp, jj, ii, 1, nbf, ns, KA, KB, PA, PB, EE);
	}
}

/* ------------------------------------------------------------------ screening helpers */

static double *shell_max(int ns, const shell_t *sh, int nbf, const double *M, int absval){
	double *r = calloc((size_t)ns * ns, sizeof(double));
	for(int P = 0; P < ns; P++)
		for(int Q = 0; Q < ns; Q++){
			double v = 0.0;
			for(int p = 0; p < sh[P].nfunc; p++)
				for(int q = 0; q < sh[Q].nfunc; q++){
					double x = M[(sh[P].first + p) * nbf + sh[Q].first + q];
					if(absval) x = fabs(x);
					if(v < x) v = x;
				}
			r[P * ns + Q] = v;
		}
	return r;
}

double orc_mem_cutoff(int nbf, const int *nprim, const int *lmn, const double *xyz,
                      const double *exps, const double *schwarz, double fixed_cutoff,
                      int max_mem_mb){
	int ns;
	long tot = 0;
	for(int i = 0; i < nbf; i++) tot += nprim[i];
	double *one = malloc(sizeof(double) * (tot > 0 ? tot : 1));
	for(long i = 0; i < tot; i++) one[i] = 1.0;
	shell_t *sh = make_shells(nbf, nprim, lmn, xyz, exps, one, one, &ns);
	double *S = shell_max(ns, sh, nbf, schwarz, 0);
	unsigned long long maxEE = (unsigned long long)max_mem_mb * 1000000ULL / sizeof(double);
	double cut = fixed_cutoff;
	int coarse = 1;
	for(;;){
		unsigned long long cnt = 0;
		int over = 0;
		for(int P = 0; P < ns && !over; P++)
		for(int Q = 0; Q <= P && !over; Q++)
		for(int I = 0; I <= P && !over; I++){
			int N = (I == P) ? Q : I;
			for(int J = 0; J <= N; J++){
				if(S[P * ns + Q] * S[I * ns + J] < cut) continue;
				cnt += (unsigned long long)sh[P].nfunc * sh[Q].nfunc * sh[I].nfunc * sh[J].nfunc;
				if(cnt > maxEE){ over = 1; break; }
			}
		}
		if(over){ cut *= coarse ? 2.00 : 1.05; continue; }
		if(coarse && cnt < maxEE){ coarse = 0; cut /= 2.0; continue; }
		break;
	}
	if(cut < fixed_cutoff) cut = fixed_cutoff;
	free(S); free(sh); free(one);
	return cut;
}

/* ------------------------------------------------------------------ driver */

int orc_jk_build(int nbf, const int *nprim, const int *lmn, const double *xyz,
                 const double *exps, const double *coefs, const double *norms,
                 const double *schwarz, const double *PA, const double *PB, int restricted,
                 double scf_cutoff, double fixed_cutoff, double dscreen_rmax,
                 double *JT, double *KA, double *KB, long long *stats){
	int ns;
	shell_t *sh = make_shells(nbf, nprim, lmn, xyz, exps, coefs, norms, &ns);
	for(int s = 0; s < ns; s++) if(sh[s].type == 6 || sh[s].maxL > LM){ free(sh); return -1; }
	size_t nn = (size_t)nbf * nbf;
	double *PT = malloc(sizeof(double) * nn);
	for(size_t k = 0; k < nn; k++) PT[k] = PA[k] + PB[k];
	double *S = shell_max(ns, sh, nbf, schwarz, 0);
	/* PM[P][Q] = max |PT|,|PA|,|PB| over the block (src/matrix.c:3894-3904) */
	double *PM = calloc((size_t)ns * ns, sizeof(double));
	for(int P = 0; P < ns; P++) for(int Q = 0; Q < ns; Q++){
		double r = 0.0;
		for(int p = 0; p < sh[P].nfunc; p++) for(int q = 0; q < sh[Q].nfunc; q++){
			int o = (sh[P].first + p) * nbf + sh[Q].first + q;
			if(r < fabs(PT[o])) r = fabs(PT[o]);
			if(r < fabs(PA[o])) r = fabs(PA[o]);
			if(r < fabs(PB[o])) r = fabs(PB[o]);
		}
		PM[P * ns + Q] = r;
	}
	memset(JT, 0, sizeof(double) * nn);
	memset(KA, 0, sizeof(double) * nn);
	memset(KB, 0, sizeof(double) * nn);
	double *EE = malloc(sizeof(double) * 50625);
	long long n_pass = 0, n_comp = 0;
	g_prim_eval = g_prim_cut = 0;
	for(int P = 0; P < ns; P++)
	for(int Q = 0; Q <= P; Q++)
	for(int I = 0; I <= P; I++){
		int N = (I == P) ? Q : I;
		for(int J = 0; J <= N; J++){
			double r = S[P * ns + Q] * S[I * ns + J];
			if(r < scf_cutoff) continue;
			n_pass++;
			if(r < fixed_cutoff) continue;
			double maxP = PM[P * ns + Q] + PM[I * ns + J] + PM[P * ns + I] + PM[P * ns + J] +
			              PM[Q * ns + I] + PM[Q * ns + J];
			if(r < dscreen_rmax && r * maxP < fixed_cutoff) continue;
			quartet(sh + P, sh + Q, sh + I, sh + J, EE, 1);
			n_comp++;
			int type;
			if(P == Q && I == J && P == I) type = T_ALLSAME;
			else if(P == Q && I == J)      type = T_2PAIRS;
			else if(P == Q)                type = T_PQPAIR;
			else if(I == J)                type = T_IJPAIR;
			else if(P == I && Q == J)      type = T_PIQJ;
			else                           type = T_ALLDISTINCT;
			store_quartet(sh + P, sh + Q, sh + I, sh + J, type, restricted, nbf, JT, KA, KB,
			              PT, PA, PB, EE);
		}
	}
	if(restricted) memcpy(KB, KA, sizeof(double) * nn);
	for(int p = 0; p < nbf; p++)
		for(int q = 0; q < p; q++){
			JT[q * nbf + p] = JT[p * nbf + q];
			KA[q * nbf + p] = KA[p * nbf + q];
			KB[q * nbf + p] = KB[p * nbf + q];
		}
	if(stats){ stats[0] = n_pass; stats[1] = n_comp; stats[2] = g_prim_eval; stats[3] = g_prim_cut; }
	free(EE); free(PM); free(S); free(PT); free(sh);
	return 0;
}
