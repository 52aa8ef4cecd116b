/*
 * advance_gg_fp64.cu -- the gas-gas kernel (advance_gg.cu) with FP64 pair
 * terms (mdn_options.force_mode = 1), as mdn_advance_gg_fp64.
 */
#define MDN_GG_TERMS 1
#define MDN_FP64_PAIRS 1
#include "advance.cu"
