/*
 * advance_fp64.cu -- the step kernel with its pair terms (LJ, LJ + Coulomb,
 * Born-Mayer-Huggins) in FP64 (mdn_options.force_mode = 1): advance.cu
 * compiled a second time as mdn_advance_fp64.
 */
#define MDN_FP64_PAIRS 1
#include "advance.cu"
