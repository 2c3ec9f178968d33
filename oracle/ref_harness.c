/*
 * sqref -- harness around the UNMODIFIED reference (Siam Quantum 2) J/K path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is ours; it is compiled against the reference's own
 * headers and linked with the reference's own objects by oracle/Makefile, and is used only as
 * a checker (golden-fixture generation, tests) and as the timed CPU baseline of bench.py.
 *
 * Commands (matrices are raw little-endian float64, row-major n*n):
 *   sqref basis   <xyz> <basis>                     print genBasis() output (src/basis.c:529)
 *   sqref schwarz <xyz> <basis> <out>               create_Schwarz() (src/matrix.c:389)
 *   sqref jk      <xyz> <basis> <PA> <PB|-> <restricted> <cutoff> <maxMem> <out>
 *                 one FRESH GTO_JK_Matrix_Quartet_Parallel (src/matrix.c:3773) after the
 *                 nBasis==0 reset (src/matrix.c:3818), nCPU=1, SCFCutoff=fixedCutoff=cutoff;
 *                 writes JT,KA,KB (3*n*n doubles)
 *   sqref jkpart  <xyz> <basis> <PA> <PB|-> <restricted> <cutoff> <maxMem> <nCPU> <childID> <out>
 *                 child childID's share of a fresh build split over nCPU processes, as
 *                 uhf_getGMatrix (src/uhf.c:132-186) runs it; the caller sums the children
 *   sqref jkseq   <xyz> <basis> <restricted> <scfCutoff> <maxMem> <out> <P1> <cut1> [<P2> <cut2> ...]
 *                 visits of one SCF after a reset: one build per (density, fixedCutoff), the
 *                 reference's cached state carried between them; JT,KA,KB per visit
 *   sqref nosymm  <xyz> <basis> <PA> <PB|-> <cutoff> <out>
 *                 GTO_JK_Matrix_NoSymm (src/matrix.c:5098), writes GA,GB
 *   sqref scf     <xyz> <basis> <densout|-> [reference options...]
 *                 uhf() (src/uhf.c:1171) as sq.c:152-415 drives it; prints the total energy
 *                 with 12 decimals on stderr and writes PA,PB of the final orbitals
 *   sqref force   <xyz> <basis> <out> [reference options...]
 *                 uhf() then uhf_force() (src/grad.c:2155): writes the forces Fx, Fy, Fz
 *                 (3*nAtom doubles, hartree/bohr; force = -gradient) and prints the energy
 *   sqref oneint  <xyz> <basis> <out>
 *                 S, T, V as uhf() builds them (src/uhf.c:1307-1334: GTO_overlap,
 *                 GTO_kinetic, GTO_nuclei); writes S,T,V (3*n*n doubles)
 *   sqref bench   <xyz> <basis> <PA> <cutoff> <maxMem> <seconds>
 *                 repeated fresh restricted J/K builds for at least <seconds>; prints count
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "basis.h"
#include "mol.h"
#include "matrix.h"
#include "option.h"
#include "uhf.h"
#include "grad.h"

static double now_s(void){
	struct timespec t; clock_gettime(CLOCK_MONOTONIC, &t);
	return t.tv_sec + 1e-9 * t.tv_nsec;
}

static struct GTOBasis_t *load_basis(const char *xyz, const char *bas, int *n,
                                     struct Molecule_t **molOut){
	FILE *f = fopen(xyz, "r");
	if(!f){ fprintf(stderr, "cannot open %s\n", xyz); exit(2); }
	struct Molecule_t *mol = readMolecule_XYZ(f); fclose(f);
	int nSet;
	f = fopen(bas, "r");
	if(!f){ fprintf(stderr, "cannot open %s\n", bas); exit(2); }
	struct GTOBasisSet_t *db = read_GAMESS_BasisSet(f, (char *)bas, &nSet); fclose(f);
	struct GTOBasis_t *gto = genBasis(mol, n, nSet, db);
	if(molOut) *molOut = mol;
	return gto;
}

static double *read_mat(const char *path, int n){
	double *m = calloc((size_t)n * n, sizeof(double));
	FILE *f = fopen(path, "rb");
	if(!f){ fprintf(stderr, "cannot open %s\n", path); exit(2); }
	if(fread(m, sizeof(double), (size_t)n * n, f) != (size_t)n * n){
		fprintf(stderr, "short read %s\n", path); exit(2);
	}
	fclose(f);
	return m;
}

static void write_mats(const char *path, int n, int k, double **m){
	FILE *f = fopen(path, "wb");
	if(!f){ fprintf(stderr, "cannot write %s\n", path); exit(2); }
	for(int i = 0; i < k; i++) fwrite(m[i], sizeof(double), (size_t)n * n, f);
	fclose(f);
}

static void fresh_jk(int n, const double *PA, const double *PB, struct GTOBasis_t *gto,
                     const double *S, double cutoff, int restricted, int maxMem,
                     double *JT, double *KA, double *KB){
	struct option_t opt;
	char *fa[3] = {"sq", "x", "y"};
	parse_option(&opt, 3, fa);
	opt.nCPU = 1; opt.maxMem = maxMem; opt.SCFCutoff = cutoff; opt.restricted = restricted;
	GTO_JK_Matrix_Quartet_Parallel(0, 0, NULL, NULL, NULL, NULL, 0.0, NULL, NULL, NULL, &opt);
	memset(JT, 0, sizeof(double) * n * n);
	memset(KA, 0, sizeof(double) * n * n);
	memset(KB, 0, sizeof(double) * n * n);
	GTO_JK_Matrix_Quartet_Parallel(0, n, PA, PB, gto, S, cutoff, JT, KA, KB, &opt);
}

int main(int argc, char **argv){
	if(argc < 4){ fprintf(stderr, "usage: see header of ref_harness.c\n"); return 2; }
	const char *cmd = argv[1];
	int n;

	if(!strcmp(cmd, "basis")){
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, NULL);
		printf("%d\n", n);
		for(int i = 0; i < n; i++){
			printf("%d %d %d %d %.17g %.17g %.17g\n", g[i].nContract, g[i].l, g[i].m, g[i].n,
			       g[i].x0, g[i].y0, g[i].z0);
			for(int k = 0; k < g[i].nContract; k++)
				printf("%.17g %.17g %.17g\n", g[i].exp[k], g[i].coef[k], g[i].norm[k]);
		}
		return 0;
	}

	if(!strcmp(cmd, "schwarz")){
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, NULL);
		double *S = create_Schwarz(n, g);
		write_mats(argv[4], n, 1, &S);
		return 0;
	}

	if(!strcmp(cmd, "jk") && argc >= 10){
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, NULL);
		double *PA = read_mat(argv[4], n);
		double *PB = strcmp(argv[5], "-") ? read_mat(argv[5], n) : PA;
		int restricted = atoi(argv[6]);
		double cutoff = atof(argv[7]);
		int maxMem = atoi(argv[8]);
		double *S = create_Schwarz(n, g);
		double *JT = calloc((size_t)n * n, 8), *KA = calloc((size_t)n * n, 8),
		       *KB = calloc((size_t)n * n, 8);
		double t0 = now_s();
		fresh_jk(n, PA, PB, g, S, cutoff, restricted, maxMem, JT, KA, KB);
		double t1 = now_s();
		double *out[3] = {JT, KA, KB};
		write_mats(argv[9], n, 3, out);
		fprintf(stderr, "RESULT nbf=%d seconds=%.6f\n", n, t1 - t0);
		return 0;
	}

	if(!strcmp(cmd, "jkpart") && argc >= 12){
		/* one child's share of a split build, as uhf_getGMatrix (src/uhf.c:132-186) hands it to
		 * process childID of nCPU: the bra shell pairs PQ with PQ % nCPU == childID
		 * (src/matrix.c:3909-3910); the caller sums the children's JT/KA/KB */
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, NULL);
		double *PA = read_mat(argv[4], n);
		double *PB = strcmp(argv[5], "-") ? read_mat(argv[5], n) : PA;
		int restricted = atoi(argv[6]);
		double cutoff = atof(argv[7]);
		int maxMem = atoi(argv[8]);
		int nCPU = atoi(argv[9]), child = atoi(argv[10]);
		if(nCPU < 1 || child < 0 || child >= nCPU){ fprintf(stderr, "bad nCPU/childID\n"); return 2; }
		double *S = create_Schwarz(n, g);
		double *JT = calloc((size_t)n * n, 8), *KA = calloc((size_t)n * n, 8),
		       *KB = calloc((size_t)n * n, 8);
		struct option_t opt;
		char *fa[3] = {"sq", "x", "y"};
		parse_option(&opt, 3, fa);
		opt.nCPU = nCPU; opt.maxMem = maxMem; opt.SCFCutoff = cutoff; opt.restricted = restricted;
		double t0 = now_s();
		GTO_JK_Matrix_Quartet_Parallel(child, 0, NULL, NULL, NULL, NULL, 0.0, NULL, NULL, NULL, &opt);
		GTO_JK_Matrix_Quartet_Parallel(child, n, PA, PB, g, S, cutoff, JT, KA, KB, &opt);
		double t1 = now_s();
		double *out[3] = {JT, KA, KB};
		write_mats(argv[11], n, 3, out);
		fprintf(stderr, "RESULT nbf=%d child=%d ncpu=%d seconds=%.6f\n", n, child, nCPU, t1 - t0);
		return 0;
	}

	if(!strcmp(cmd, "jkseq") && argc >= 10 && (argc - 8) % 2 == 0){
		/* a sequence of visits of one SCF: the reset, then GTO_JK_Matrix_Quartet_Parallel
		 * (nCPU=1) once per (density, fixedCutoff) pair with the reference's state (eeBank,
		 * erBank, firstVisit) carried from visit to visit, as uhf() calls it through
		 * uhf_getGMatrix (src/uhf.c:1596) with the zeroed outputs it passes (src/uhf.c:124-129);
		 * writes JT,KA,KB of every visit */
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, NULL);
		int restricted = atoi(argv[4]);
		double scfcut = atof(argv[5]);
		int maxMem = atoi(argv[6]);
		int nv = (argc - 8) / 2;
		double *S = create_Schwarz(n, g);
		struct option_t opt;
		char *fa[3] = {"sq", "x", "y"};
		parse_option(&opt, 3, fa);
		opt.nCPU = 1; opt.maxMem = maxMem; opt.SCFCutoff = scfcut; opt.restricted = restricted;
		GTO_JK_Matrix_Quartet_Parallel(0, 0, NULL, NULL, NULL, NULL, 0.0, NULL, NULL, NULL, &opt);
		FILE *f = fopen(argv[7], "wb");
		if(!f){ fprintf(stderr, "cannot write %s\n", argv[7]); exit(2); }
		double *JT = calloc((size_t)n * n, 8), *KA = calloc((size_t)n * n, 8),
		       *KB = calloc((size_t)n * n, 8);
		for(int v = 0; v < nv; v++){
			double *PA = read_mat(argv[8 + 2 * v], n);
			double cut = atof(argv[9 + 2 * v]);
			memset(JT, 0, sizeof(double) * n * n);
			memset(KA, 0, sizeof(double) * n * n);
			memset(KB, 0, sizeof(double) * n * n);
			GTO_JK_Matrix_Quartet_Parallel(0, n, PA, PA, g, S, cut, JT, KA, KB, &opt);
			fwrite(JT, sizeof(double), (size_t)n * n, f);
			fwrite(KA, sizeof(double), (size_t)n * n, f);
			fwrite(KB, sizeof(double), (size_t)n * n, f);
			free(PA);
		}
		fclose(f);
		fprintf(stderr, "RESULT nbf=%d visits=%d\n", n, nv);
		return 0;
	}

	if(!strcmp(cmd, "nosymm") && argc >= 8){
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, NULL);
		double *PA = read_mat(argv[4], n);
		double *PB = strcmp(argv[5], "-") ? read_mat(argv[5], n) : PA;
		double cutoff = atof(argv[6]);
		double *S = create_Schwarz(n, g);
		double *GA = calloc((size_t)n * n, 8), *GB = calloc((size_t)n * n, 8);
		GTO_JK_Matrix_NoSymm(n, PA, PB, g, S, cutoff, GA, GB);
		double *out[2] = {GA, GB};
		write_mats(argv[7], n, 2, out);
		return 0;
	}

	if(!strcmp(cmd, "scf") && argc >= 5){
		/* argv for parse_option: sq <xyz> <basis> [options...] as sq.c:183 */
		int na = argc - 2;
		char **pa = calloc(na + 1, sizeof(char *));
		pa[0] = "sq"; pa[1] = argv[2]; pa[2] = argv[3];
		for(int i = 5; i < argc; i++) pa[i - 2] = argv[i];
		struct option_t opt;
		parse_option(&opt, na, pa);
		opt.nCPU = 1;
		struct Molecule_t *mol;
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, &mol);
		mol->Q = opt.molCharge;
		if(opt.multiplicity == 0) opt.multiplicity = (get_nElectron(mol) % 2 == 0) ? 1 : 2;
		if(opt.multiplicity > 1) opt.restricted = 0;
		int nEA = get_nEA(mol, opt.multiplicity), nEB = get_nEB(mol, opt.multiplicity);
		double *CA = calloc((size_t)n * n, 8), *CB = calloc((size_t)n * n, 8);
		double *eA = calloc(n, 8), *eB = calloc(n, 8);
		double t0 = now_s();
		double E = uhf(n, g, mol, nEA, nEB, CA, CB, eA, eB, &opt);
		double t1 = now_s();
		fflush(stdout);
		fprintf(stderr, "RESULT energy=%.12f nbf=%d nEA=%d nEB=%d seconds=%.6f\n",
		        E, n, nEA, nEB, t1 - t0);
		if(strcmp(argv[4], "-")){
			double *PA = calloc((size_t)n * n, 8), *PB = calloc((size_t)n * n, 8);
			uhf_getDMatrix(n, nEA, CA, PA);
			uhf_getDMatrix(n, nEB, CB, PB);
			double *out[2] = {PA, PB};
			write_mats(argv[4], n, 2, out);
		}
		return 0;
	}

	if(!strcmp(cmd, "force") && argc >= 5){
		int na = argc - 2;
		char **pa = calloc(na + 1, sizeof(char *));
		pa[0] = "sq"; pa[1] = argv[2]; pa[2] = argv[3];
		for(int i = 5; i < argc; i++) pa[i - 2] = argv[i];
		struct option_t opt;
		parse_option(&opt, na, pa);
		opt.nCPU = 1;
		struct Molecule_t *mol;
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, &mol);
		mol->Q = opt.molCharge;
		if(opt.multiplicity == 0) opt.multiplicity = (get_nElectron(mol) % 2 == 0) ? 1 : 2;
		if(opt.multiplicity > 1) opt.restricted = 0;
		int nEA = get_nEA(mol, opt.multiplicity), nEB = get_nEB(mol, opt.multiplicity);
		double *CA = calloc((size_t)n * n, 8), *CB = calloc((size_t)n * n, 8);
		double *eA = calloc(n, 8), *eB = calloc(n, 8);
		double E = uhf(n, g, mol, nEA, nEB, CA, CB, eA, eB, &opt);
		double *F = calloc(3 * (size_t)mol->nAtom, 8);
		uhf_force(n, g, mol, nEA, nEB, CA, CB, eA, eB, &opt, F, F + mol->nAtom, F + 2 * mol->nAtom);
		fflush(stdout);
		fprintf(stderr, "RESULT energy=%.12f nbf=%d natom=%d\n", E, n, mol->nAtom);
		double *out[1] = {F};
		FILE *f = fopen(argv[4], "wb");
		if(!f){ fprintf(stderr, "cannot write %s\n", argv[4]); exit(2); }
		fwrite(out[0], sizeof(double), 3 * (size_t)mol->nAtom, f);
		fclose(f);
		return 0;
	}

	if(!strcmp(cmd, "oneint") && argc >= 5){
		struct Molecule_t *mol;
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, &mol);
		double *S = calloc((size_t)n * n, 8), *T = calloc((size_t)n * n, 8),
		       *V = calloc((size_t)n * n, 8);
		for(int i = 0; i < n; i++)
		for(int j = 0; j <= i; j++){
			S[i * n + j] = S[j * n + i] = GTO_overlap(i, j, g);
			T[i * n + j] = T[j * n + i] = GTO_kinetic(i, j, g);
			V[i * n + j] = V[j * n + i] = GTO_nuclei(i, j, g, mol);
		}
		double *out[3] = {S, T, V};
		write_mats(argv[4], n, 3, out);
		return 0;
	}

	if(!strcmp(cmd, "bench") && argc >= 8){
		struct GTOBasis_t *g = load_basis(argv[2], argv[3], &n, NULL);
		double *PA = read_mat(argv[4], n);
		double cutoff = atof(argv[5]);
		int maxMem = atoi(argv[6]);
		double seconds = atof(argv[7]);
		double *S = create_Schwarz(n, g);
		double *JT = calloc((size_t)n * n, 8), *KA = calloc((size_t)n * n, 8),
		       *KB = calloc((size_t)n * n, 8);
		int builds = 0;
		double t0 = now_s(), t1;
		do{
			fresh_jk(n, PA, PA, g, S, cutoff, 1, maxMem, JT, KA, KB);
			builds++;
			t1 = now_s();
		}while(t1 - t0 < seconds);
		fprintf(stderr, "RESULT builds=%d seconds=%.6f nbf=%d\n", builds, t1 - t0, n);
		return 0;
	}

	fprintf(stderr, "bad command\n");
	return 2;
}
