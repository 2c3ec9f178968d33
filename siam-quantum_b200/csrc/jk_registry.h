// Table of generated class kernels (filled in by gen/jk_registry.cu).
#pragma once

namespace sqb {

// Pair classes in generator order: SS LS LL PS PL PP DS DL DP DD.
constexpr int kNumPairClasses = 10;
extern const char* const kPairClassNames[kNumPairClasses];

struct ClassKernel {
  int bra_cls, ket_cls;   // pair class of the CTA-shared bra and of the per-thread ket
  int nab, ncd;           // functions per bra / ket pair
  int neb, nek;           // Hermite E-table entries per primitive pair
  int Lt;                 // total angular momentum
  int passes;             // ket-function blocks = grid.y of a launch
  const void* fn_r;       // restricted kernel
  const void* fn_u;       // unrestricted kernel
  int flops_prim;         // FP64 ops per primitive quartet as emitted (all passes, repeats included)
  int flops_flush;        // FP64 ops per bra primitive and ket pair (all passes)
  int flops_quartet;      // FP64 ops of one digestion (all passes) of a (partial) quartet block
  // warp-specialised form (null when the class has one pass or its R buffer does not fit):
  // one CTA of 32*ws_warps threads = all passes of 32 quartets, R staged in shared memory
  int ws_warps, ws_nr;
  const void* ws_r;
  const void* ws_u;
  int ws_flops_prim, ws_flops_flush, ws_flops_quartet;
  // mixed form (FP32 Hermite integrals and contraction, FP64 Boys/setup/accumulation); null
  // for the classes of highest angular momentum, whose small quartets stay in FP64
  int passes32;
  const void* fn_r32;
  const void* fn_u32;
  int f32_flops_prim, f32_flops_flush, f32_flops_quartet;
  // algorithmic operations per primitive quartet (pass-free: the Boys function and every R
  // value once); the work figure of the roofline, the same for every form of the class
  int alg_flops_prim;
  // wide-tile FP64 form (fewer passes of more ket functions each); null when it would not
  // merge any pass.  sqb200_jk_autotune picks the faster form per class.
  int passes_w;
  const void* fn_rw;
  const void* fn_uw;
  int w_flops_prim, w_flops_flush, w_flops_quartet;
  int w_o_dbl;            // doubles per thread of the wide form's shared-memory accumulators (0: registers)
  // swapped-role FP64 form: outer loop over the thread's ket primitives (global, once per
  // pass), inner loop over the shared bra primitives (shared memory); passes split the bra
  // functions; its flush counter counts ket primitives
  int passes_s;
  const void* fn_rs;
  const void* fn_us;
  int s_flops_prim, s_flops_flush, s_flops_quartet;
  int s_o_dbl;            // doubles per thread of the swapped form's shared-memory accumulators (0: registers)
};

extern const ClassKernel kClassKernels[];
extern const int kNumClassKernels;

}  // namespace sqb
