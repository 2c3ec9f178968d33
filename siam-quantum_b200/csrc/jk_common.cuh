// Device-side records and the Boys function shared by every J/K class kernel.
//
// Boys function F_m(T) = int_0^1 u^(2m) exp(-T u^2) du  (role of fgamma_set, reference
// src/fgamma.c:172-206).  Written from the mathematics, not from any library:
//   T <  BOYS_TMAX : the top order F_M(T) by a 9-term Taylor expansion about the nearest grid
//                    point T0 (spacing BOYS_H), F_M(T0+d) = sum_k F_{M+k}(T0) (-d)^k / k!,
//                    then the stable downward recursion F_m = (2T F_{m+1} + e^-T)/(2m+1), with
//                    e^-T = e^-T0 e^-d from a tabulated e^-T0 and the Taylor series of e^-d.
//   T >= BOYS_TMAX : F_0 = sqrt(pi/T)/2 (the erfc tail is below 1e-17 relative there) and the
//                    stable upward recursion F_{m+1} = ((2m+1) F_m - e^-T)/(2T).
// The grid values are computed on the host in extended precision (jk_engine.cu).
#pragma once
#include <cstdint>

#define BOYS_H      0.1
#define BOYS_INV_H  10.0
#define BOYS_TMAX   36.0
#define BOYS_NGRID  361      // grid points T0 = 0, 0.1, ..., 36.0
#define BOYS_MMAX   8        // highest order requested by a kernel ((dd|dd))
#define BOYS_NTAY   9        // Taylor terms
// columns m = 0..17 per grid row: a row is 144 bytes (a multiple of 16), so the Taylor values of
// any order M (columns M..M+8, read from the even column at or below M) come in five 16-byte
// loads; each lane gathers its own row, one L1 sector per load
#define BOYS_NCOL   (BOYS_MMAX + BOYS_NTAY + 1)

#define TWO_PI_2_5  34.986836655249725     // 2 pi^(5/2)
#define PRIM_CUTOFF 1.0e-15                // reference src/int.h:19
#define TWO_PI_2_5F 34.986836655249725f    // the same in FP32 (mixed-precision forms)
#define PRIM_CUTOFF_F 1.0e-15f

namespace sqb {

// One shell pair (P >= Q in the reference's sorted shell order), 32 bytes.
struct PairRec {
  int P, Q;        // sorted shell indices
  int fP, fQ;      // first basis function of each shell
  int nprim;       // primitive pairs
  int poff;        // offset (elements) of field 0 of its first primitive record in the class array
  int kstride;     // elements between consecutive fields of one record: field f of primitive
                   // record j sits at poff + (j * fields + f) * kstride
  int pad_;
  double schwarz;  // max over the block of the basis-level Schwarz matrix
};

// A CTA's unit of work: one bra pair and a contiguous range of cnt ket pairs, each ket
// handled by `isplit` threads (power of two) that split the bra primitives between them.
struct WorkItem {
  int bra, k0, cnt, isplit;
  int mol;         // index of the molecule (MolRec) the pairs belong to
};

// One molecule of a build: where its matrices sit in the packed device arrays, and the
// cutoffs of its current SCF step.  A single-molecule build has one record at offset 0; a
// batched build packs many molecules' nbf x nbf blocks back to back.
struct MolRec {
  long long moff;      // offset (doubles) of its nbf x nbf blocks in PA, PB, PT, Jacc, KAacc, KBacc
  long long pmoff;     // offset of its ns x ns block-maximum matrix in PM
  int nbf, ns;
  double cut_outer, cut_fixed, dscreen_rmax;
  int shoff;           // its first shell in the packed shell tables (batched block maxima)
  int uhf;             // 1 = unrestricted (KB from PB), 0 = restricted (KB = KA)
};

struct JKArgs {
  const PairRec* bra_pairs;
  const double* bra_prims;
  const PairRec* ket_pairs;
  const double* ket_prims;
  const double* PA;
  const double* PB;
  const double* PT;
  const double* PM;            // per molecule ns x ns shell-block max of |PT|,|PA|,|PB|
  double* Jacc;                // per molecule nbf x nbf, J = Jacc + Jacc^T
  double* KAacc;               // per molecule nbf x nbf, K[PA] = KAacc + KAacc^T
  double* KBacc;
  const double* boys_tab;      // BOYS_NGRID x BOYS_NCOL
  const float* boys_tab_f;     // the same table rounded to FP32 (mixed-precision forms)
  unsigned long long* counters;// [0] quartets computed, [1] primitive quartets evaluated,
                               // [2] bra-primitive flushes, [3] digestions
  const MolRec* mols;          // per-molecule offsets, sizes and cutoffs (WorkItem::mol)
  int same_class;              // bra and ket pairs come from one class (pair identity possible)
  int so_off;                  // doubles from the start of dynamic shared memory to the
                               // accumulator slots of the shared-memory wide form
  const float* bra_prims_f;    // FP32 copies of the primitive records (mixed-precision kernels)
  const float* ket_prims_f;
  // Reference-parity multipole mode (erbank == nullptr: off; narrow FP64 form, isplit 1).
  // The reference's GTO_JK_Matrix_Quartet_Parallel (src/matrix.c:3914-3967) keeps, per shell
  // quartet surviving the outer Schwarz cutoff, the base-1.5 exponent of the largest error of
  // the monopole approximation (getErrExpQuartetMPole, src/matrix.c:2551), measured the first
  // time the quartet is computed; on later visits a quartet below its memory cutoff whose
  // 1.5^exponent * maxPShell is below the fixed cutoff takes the monopole values instead
  // (computeQuartetMPole, src/matrix.c:2609).
  signed char* erbank;         // per outer-cutoff survivor: exponent, or ERR_UNKNOWN
  unsigned long long* erscr;   // per survivor: bits of this build's largest error | 1 << 63
  const int* er_items;         // per work item: erbank index of its first ket
  const double* mpole;         // per function pair (p * nbf + q): charge q, centre x, y, z
  const double* pow15;         // 1.5^e, e = -120..120, as the host's pow computes it
  double mp_rmax;              // quartets with Sch(PQ)*Sch(IJ) >= this are never substituted
  // Persistent launch (queue != nullptr): a fixed grid takes the nqueue work units (item, pass)
  // of the launch from this device counter, zeroed before the launch; npass passes per item.
  unsigned long long* queue;
  int nqueue, npass;
};

constexpr int ERR_MIN = -120;      // src/matrix.c:1745-1747
constexpr int ERR_MAX = 120;
constexpr int ERR_UNKNOWN = 121;
#define MULTIPOLE_R2_CUTOFF 1.0    // src/multipole.h:23: below this squared distance the term is 0

// Monopole-monopole value of the function-pair quartet (pq|rs) (computeQuartetMPole): charges
// times the inverse distance between the pairs' charge centres, 0 when the squared distance
// is below MULTIPOLE_R2_CUTOFF; the same operations in the same order, without contractions.
// Not inlined: the multipole mode is rare and its callers are unrolled over whole blocks.
static __device__ __noinline__ double mpole_value(const double* __restrict__ mp, int N, int p, int q, int r, int s) {
  const double* m1 = mp + 4 * ((long long)p * N + q);
  const double* m2 = mp + 4 * ((long long)r * N + s);
  const double dx = __dadd_rn(m1[1], -m2[1]), dy = __dadd_rn(m1[2], -m2[2]), dz = __dadd_rn(m1[3], -m2[3]);
  const double K = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  if (K < MULTIPOLE_R2_CUTOFF) return 0.0;
  return __dmul_rn(__dmul_rn(m1[0], m2[0]), __dsqrt_rn(__ddiv_rn(1.0, K)));
}

// F_0..F_M at T.  M is a compile-time order so the recursion unrolls.
template <int M>
__device__ __forceinline__ void boys(double T, const double* __restrict__ tab, double* F) {
  if (T < BOYS_TMAX) {
    const int g = __double2int_rn(T * BOYS_INV_H);
    const double d = T - g * BOYS_H;          // |d| <= BOYS_H/2
    const double2* r2 = reinterpret_cast<const double2*>(tab + g * BOYS_NCOL + (M & ~1));
    double v[BOYS_NTAY + 1];
#pragma unroll
    for (int q = 0; q < (BOYS_NTAY + 1) / 2; ++q) {
      const double2 t = __ldg(r2 + q);
      v[2 * q] = t.x;
      v[2 * q + 1] = t.y;
    }
    const double* row = v + (M & 1);          // row[k] = F_{M+k}(T0)
    // Horner in -d with 1/k! folded in: sum_k row[k] (-d)^k / k!
    double s = row[BOYS_NTAY - 1];
#pragma unroll
    for (int k = BOYS_NTAY - 2; k >= 0; --k) s = fma(s, -d * (1.0 / (double)(k + 1)), row[k]);
    F[M] = s;
    if (M > 0) {
      // e^-T = e^-T0 e^-d: the grid value (stored after the table's rows) times the Taylor
      // series of e^-d through d^9/9! (|d| <= 0.05: the next term is below 3e-20)
      const double e0 = __ldg(tab + BOYS_NGRID * BOYS_NCOL + g);
      double ed = 1.0;
#pragma unroll
      for (int k = 9; k >= 1; --k) ed = fma(ed, -d * (1.0 / (double)k), 1.0);
      const double e = e0 * ed;
      const double t2 = T + T;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) * (1.0 / (2 * m + 1));
    }
  } else {
    const double it = 1.0 / T;
    F[0] = 0.88622692545275801365 * sqrt(it);   // sqrt(pi)/2 / sqrt(T)
    if (M > 0) {
      const double e = exp(-T);
      const double h = 0.5 * it;
#pragma unroll
      for (int m = 0; m < M; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * h;
    }
  }
}

// F_0..F_M at T in FP32, for the mixed-precision forms (quartets whose Schwarz bound is below
// the FP32 threshold): the scheme of boys<M> with the FP32 table and 6 Taylor terms
// (|d| <= BOYS_H/2: the next term is below 2e-11 of F_M, under FP32 rounding).
template <int M>
__device__ __forceinline__ void boysf(float T, const float* __restrict__ tab, float* F) {
  if (T < (float)BOYS_TMAX) {
    const int g = __float2int_rn(T * (float)BOYS_INV_H);
    const float d = T - g * (float)BOYS_H;
    const float2* r2 = reinterpret_cast<const float2*>(tab + g * BOYS_NCOL + (M & ~1));
    float v[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float2 t = __ldg(r2 + q);
      v[2 * q] = t.x;
      v[2 * q + 1] = t.y;
    }
    const float* row = v + (M & 1);           // row[k] = F_{M+k}(T0), k < 6
    float s = row[5];
#pragma unroll
    for (int k = 4; k >= 0; --k) s = fmaf(s, -d * (1.0f / (float)(k + 1)), row[k]);
    F[M] = s;
    if (M > 0) {
      const float e = expf(-T);
      const float t2 = T + T;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) F[m] = fmaf(t2, F[m + 1], e) * (1.0f / (float)(2 * m + 1));
    }
  } else {
    const float it = 1.0f / T;
    F[0] = 0.886226925f * sqrtf(it);
    if (M > 0) {
      const float e = expf(-T);
      const float h = 0.5f * it;
#pragma unroll
      for (int m = 0; m < M; ++m) F[m + 1] = ((float)(2 * m + 1) * F[m] - e) * h;
    }
  }
}

// F_0..F_M at T, as boys<M> (R = double) or boysf<M> (R = float), reading the Taylor rows from
// a copy of the table's columns in shared memory: s points at column M of a table of NC columns
// per grid row (the staged columns start at some order c0 <= M; s = staged + M - c0).
template <int M, int NC, class R>
__device__ __forceinline__ void boys_s(R T, const R* __restrict__ s, R* F) {
  constexpr int NT = sizeof(R) == 8 ? BOYS_NTAY : 6;
  if (T < (R)BOYS_TMAX) {
    const int g = (int)rint(T * (R)BOYS_INV_H);
    const R d = T - g * (R)BOYS_H;
    const R* row = s + g * NC;
    R acc = row[NT - 1];
#pragma unroll
    for (int k = NT - 2; k >= 0; --k) acc = fma(acc, -d * ((R)1 / (R)(k + 1)), row[k]);
    F[M] = acc;
    if (M > 0) {
      const R e = exp(-T);
      const R t2 = T + T;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) * ((R)1 / (R)(2 * m + 1));
    }
  } else {
    const R it = (R)1 / T;
    F[0] = (R)0.88622692545275801365 * sqrt(it);
    if (M > 0) {
      const R e = exp(-T);
      const R h = (R)0.5 * it;
#pragma unroll
      for (int m = 0; m < M; ++m) F[m + 1] = ((R)(2 * m + 1) * F[m] - e) * h;
    }
  }
}

// Warp-aggregated 64-bit counter increment.
__device__ __forceinline__ void count_add(unsigned long long* c, unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(c, v);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace sqb
