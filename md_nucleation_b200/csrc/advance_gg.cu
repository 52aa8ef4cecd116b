/*
 * advance_gg.cu -- the step kernel with the gas-gas term (gg LJ, the
 * corrected PotentialGasGas): advance.cu compiled again as mdn_advance_gg,
 * so that the kernel every configuration without gg uses carries none of
 * its code or registers.  The engine takes it when any replica of the batch
 * has gg on.
 */
#define MDN_GG_TERMS 1
#include "advance.cu"
