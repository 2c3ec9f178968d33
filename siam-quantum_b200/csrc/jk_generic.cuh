// The generic J/K path: shell quartets that involve a shell outside the generated class
// kernels -- f shells (10 Cartesian functions, read by read_GAMESS_BasisSet, reference
// src/basis.c:488-499) or any other shell layout genGTOShell accepts (src/matrix.c:2527-2535:
// TYPEF for 10 functions, TYPEX otherwise) -- computed by one kernel with run-time angular
// momenta (jk_generic.cu).  Internal to the library.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace sqb {

constexpr int kGenLmax = 3;         // highest l+m+n of one function on the generic path
constexpr int kGenMmax = 4 * kGenLmax;   // highest Boys order, (ff|ff)
constexpr int kGenBoysCols = 22;    // Boys table columns of the generic path: orders to 12 (13 for
                                    // the f gradient) with their 9-term Taylor expansions

// One shell as the generic path sees it.
struct GenShell {
  int first, nfunc, nprim, lmax;
  int gen;                          // 1: its pairs take the generic path
  double x, y, z;
  const double* exps;               // nprim exponents
  const double* coef;               // norm * coefficient of primitive k, function f: coef[k * 16 + f]
  const int* lmn;                   // l, m, n of function f: lmn[3 f .. 3 f + 2]
};

// One shell pair (P >= Q in the sorted shell order), 56 bytes.
struct GenPairRec {
  int P, Q, fP, fQ;
  int nfP, nfQ, lP, lQ;             // function counts and highest l+m+n of each shell
  int nprim, poff;                  // primitive pairs; first record (records of kGenPrimStride)
  int gen;                          // the pair has a generic shell
  int doff;                         // its function pairs' component descriptors in `desc`
  double schwarz;                   // max over the block of the basis-level Schwarz matrix
};

// Fields of one primitive-pair record: p, Px, Py, Pz, kp = exp(-ab|AB|^2/p)/p, PA (3), PB (3),
// the offset of its Hermite tables and weights in `coef` (as a double), padding, and the two
// primitive indices (as doubles): 16.
constexpr int kGenPrimStride = 16;

// A CTA's unit: one generic bra pair and kets k0 .. k0+cnt-1 of the all-pairs list.  er: in
// the multipole mode, the error-bank slot of the bra's ket 0 (ket k has slot er + k), else -1.
struct GenItem {
  int bra, k0, cnt, er;
};

struct GenPath {
  bool on = false;                  // the basis has generic shells
  std::vector<GenPairRec> pairs;    // every shell pair, by decreasing Schwarz bound
  std::vector<double> prims;
  std::vector<double> coef;         // per primitive pair: its 1-D Hermite tables, then its weights
  std::vector<int> desc;            // per pair: one component descriptor per function pair
  std::vector<int> gen_idx;         // positions of the generic pairs in `pairs`
  // device (one allocation)
  void* d_base = nullptr;
  size_t bytes = 0;
  GenPairRec* d_pairs = nullptr;
  double* d_prims = nullptr;
  double* d_coef = nullptr;
  int* d_desc = nullptr;
  int* d_gen_idx = nullptr;
  double* d_boys = nullptr;         // Boys table, BOYS_NGRID x kGenBoysCols
  unsigned long long* d_counters = nullptr;   // quartets, primitive quartets, operations of the last build
};

// Arguments of one generic J/K launch (the accumulators are the build's unsymmetrised ones).
struct GenBuild {
  const double *PA, *PB, *PT, *PM;
  double *J, *KA, *KB;
  int nbf, ns, uhf;
  double cut_outer, cut_fixed, dscreen_rmax;
  // multipole mode (erbank != nullptr): the class kernels' error bank, its scratch, the
  // monopole table, powers of 1.5 and the cache bound (sqb200_jk_set_multipole)
  const signed char* erbank;
  unsigned long long* erscr;
  const double* mpole;
  const double* pow15;
  double mp_rmax;
};

// Pair records and primitive data for every shell pair; `schwarz` is the basis-level matrix.
void gen_build_pairs(GenPath& g, const std::vector<GenShell>& sh, const double* schwarz, int nbf);
// Device copies of the pair data and the generic Boys table.
int gen_upload(GenPath& g, cudaStream_t st);
// Schwarz entries sqrt|(pq|pq)| of the generic pairs' functions into S (nbf x nbf, device).
int gen_schwarz(const GenPath& g, int nbf, double* S, cudaStream_t st);
// Work items of one build at these cutoffs; cost: a relative estimate for launch ordering.
// er_run != nullptr (multipole mode): every generic bra takes error-bank slots for its kets
// that pass the outer cutoff, numbered on from *er_run.
void gen_items(const GenPath& g, double outer, double fixed, std::vector<GenItem>& items, double& cost,
               long long* er_run = nullptr);
// One launch over the items (counters zeroed first).
int gen_launch(const GenPath& g, const GenItem* d_items, int nitems, const GenBuild& b, cudaStream_t st);
void gen_free(GenPath& g);

}  // namespace sqb
