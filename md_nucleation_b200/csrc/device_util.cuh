/*
 * device_util.cuh -- small device helpers of the engine: the counter-based
 * generator, fixed-point conversion, deterministic reductions and the
 * reference's Euler rotation.
 *
 * This translation unit is compiled with --fmad=false, so FP64 expressions
 * round exactly like the reference's x86 build (one rounding per + - * / and
 * sqrt).  FP32 pair arithmetic that should fuse uses fmaf() explicitly.
 */
#ifndef MDN_DEVICE_UTIL_CUH
#define MDN_DEVICE_UTIL_CUH

#include <stdint.h>

#include "mdn_types.h"

namespace mdn {

/* Philox4x32-10 (Salmon et al., SC'11): ten rounds of two 32x32->64-bit
 * multiplications with Weyl-bumped round keys.  Counter layout of the
 * effective-domain draws: (molecule, rebuild number, purpose, word). */
struct U4 {
  unsigned v[4];
};

__device__ __forceinline__ U4 philox(U4 c, unsigned k0, unsigned k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    unsigned hi0 = __umulhi(0xD2511F53u, c.v[0]), lo0 = 0xD2511F53u * c.v[0];
    unsigned hi1 = __umulhi(0xCD9E8D57u, c.v[2]), lo1 = 0xCD9E8D57u * c.v[2];
    U4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

__device__ __forceinline__ U4 draw(const RepParams& P, int mol, int rebuild, int purpose, int word) {
  U4 c;
  c.v[0] = (unsigned)mol;
  c.v[1] = (unsigned)rebuild;
  c.v[2] = (unsigned)purpose;
  c.v[3] = (unsigned)word;
  return philox(c, P.key0, P.key1);
}

__device__ __forceinline__ double u01(unsigned u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

__device__ __forceinline__ void box_muller(unsigned a, unsigned b, double& z0, double& z1) {
  double r = sqrt(-2.0 * log(u01(a)));
  double t = 6.283185307179586 * u01(b);
  z0 = r * cos(t);
  z1 = r * sin(t);
}

/* Variables::ROTATION (src/variables.hpp:94-98), same expression order */
__device__ __forceinline__ void rotation(double& X, double& Y, double& Z, double A, double B, double C,
                                         double x, double y, double z) {
  double cA = cos(A), sA = sin(A), cB = cos(B), sB = sin(B), cC = cos(C), sC = sin(C);
  double t = x * cB + y * sA * sB - z * cA * sB;
  double u = y * cA + z * sA;
  X = cC * t + sC * u;
  Y = -sC * t + cC * u;
  Z = x * sB - y * sA * cB + z * cA * cB;
}

/* fixed-point conversion of one term, saturated at +-2^21 kcal/mol/A so that a
 * few saturated terms still sum inside int64 (NaN converts to 0) */
__device__ __forceinline__ long long fixd(double f) {
  return __double2ll_rn(fmin(fmax(f, -2097152.0), 2097152.0) * MDN_FIX_SCALE);
}
__device__ __forceinline__ long long fixf(float f) {
  return __float2ll_rn(fminf(fmaxf(f, -2097152.0f), 2097152.0f) * 1099511627776.0f);
}
__device__ __forceinline__ long long efixd(double e) { return __double2ll_rn(e * MDN_EFIX_SCALE); }
__device__ __forceinline__ long long efixf(float e) { return __float2ll_rn(e * 68719476736.0f); }

__device__ __forceinline__ long long shfl_xor_ll(long long v, int m) {
  int lo = (int)(v & 0xffffffffll);
  int hi = (int)(v >> 32);
  lo = __shfl_xor_sync(0xffffffffu, lo, m);
  hi = __shfl_xor_sync(0xffffffffu, hi, m);
  return ((long long)hi << 32) | (unsigned)lo;
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += shfl_xor_ll(v, m);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}

__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, m));
  return v;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}

/* exclusive prefix sum of `v` over the block; returns the block total in *total.
 * `scratch` holds >= 33 ints.  All threads must call it. */
__device__ __forceinline__ int block_exscan(int v, int* scratch, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) scratch[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < nw ? scratch[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) scratch[lane] = w;  /* inclusive over warps */
    if (lane == nw - 1) scratch[32] = w;
  }
  __syncthreads();
  int before = (wid > 0 ? scratch[wid - 1] : 0) + x - v;
  *total = scratch[32];
  __syncthreads();
  return before;
}

__device__ __forceinline__ int block_sum_i(int v, int* scratch) {
  int t;
  block_exscan(v, scratch, &t);
  return t;
}

/* max over the block of a non-negative double; scratch >= 33 doubles */
__device__ __forceinline__ double block_max_d(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max_d(v);
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double w = lane < nw ? scratch[lane] : 0.0;
    w = warp_max_d(w);
    if (lane == 0) scratch[32] = w;
  }
  __syncthreads();
  double r = scratch[32];
  __syncthreads();
  return r;
}

}  // namespace mdn
#endif
