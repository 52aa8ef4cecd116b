/*
 * place.cu -- mdn_place: initial centres and velocities of the gas and vapor
 * molecules, MD::initialization_gas / MD::initialization_vapor
 * (src/initialization/initializationGas.cpp:24-100,
 * src/initialization/initializationVapor.cpp:14-76), on the GPU.
 *
 * The reference draws a centre uniformly in the cube, measures its minimum
 * image distance to every row of the atom table and keeps it when all are
 * farther than 10 A.  The rows of molecules placed so far all sit at the
 * origin (their atoms are inserted at the first rebuild), so the test is
 * against the ion's atoms and, once one molecule is placed, the origin.  It
 * scans the whole table for every candidate: O(N^2) for N molecules.
 *
 * Here candidate k of a species is a pure function of (seed, species, k):
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11) of the counter (k, species, tag) under the key
 * seed.  One thread tests one candidate against the ion atoms staged in
 * shared memory; an ordered compaction keeps the first n accepted
 * candidates.  The result is that of the sequential loop over the same
 * stream, whatever the launch shape.
 *
 * Arithmetic that decides acceptance is written with explicit round-to-
 * nearest intrinsics (and the unit is compiled without fused multiply-add),
 * so the decision is the one a plain IEEE double evaluation of the
 * reference's expressions makes.
 */
#include <cuda_runtime.h>
#include <limits.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "device_util.cuh"
#include "mdn.h"

__attribute__((visibility("hidden"))) int mdn_error(int code, const char* msg);

namespace {

constexpr int kTestThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kIonTile = 1024;            /* ion atoms per shared-memory tile */
constexpr uint32_t kTag = 0x706c6163u;    /* fourth counter word of every draw */

/* counter (k, k >> 32, purpose, tag) under the key seed; the generator and
 * the (0, 1) map are the engine's (device_util.cuh) */
__device__ __forceinline__ mdn::U4 draw(unsigned long long seed, uint32_t purpose, long long k) {
  mdn::U4 c;
  c.v[0] = (unsigned)k;
  c.v[1] = (unsigned)((unsigned long long)k >> 32);
  c.v[2] = purpose;
  c.v[3] = kTag;
  return mdn::philox(c, (unsigned)seed, (unsigned)(seed >> 32));
}

/* squared minimum-image distance, src/pairList/periodic.cpp:134-142 */
__device__ __forceinline__ double dist2(const double* p, const double* X, double L, double LH) {
  double d[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double v = __dsub_rn(p[c], X[c]);
    if (v < -LH) v = __dadd_rn(v, L);
    if (v > LH) v = __dsub_rn(v, L);
    d[c] = v;
  }
  return __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2]));
}

/* candidates k0 .. k0+K-1: bits bit 0 = clear of every ion atom, bit 1 =
 * clear of the origin; *first = the smallest local index with bit 0 set */
__global__ void __launch_bounds__(kTestThreads) place_test(const double* ion_x, int n_ion, double L, double dis,
                                                            unsigned long long seed, uint32_t purpose, long long k0,
                                                            int K, unsigned char* bits, double* cx, int* first) {
  __shared__ double s_ion[3 * kIonTile];
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = id < K;
  const double LH = L * 0.5;
  double X[3] = {0, 0, 0};
  if (live) {
    const mdn::U4 w = draw(seed, purpose, k0 + id);
#pragma unroll
    for (int c = 0; c < 3; c++) X[c] = __dmul_rn(__dsub_rn(mdn::u01(w.v[c]), 0.5), L);
  }
  /* sqrt(d2) > dis is decided from d2 outside a band of 1e-12 relative
   * around dis^2 (there sqrt, correctly rounded, cannot land on the other
   * side of dis) and by sqrt itself inside it */
  const double dd = __dmul_rn(dis, dis);
  const double lo = dd * (1.0 - 1e-12), hi = dd * (1.0 + 1e-12);
  auto clear = [&](double d2) { return d2 > hi || (d2 >= lo && sqrt(d2) > dis); };
  bool ion_ok = true;
  for (int t0 = 0; t0 < n_ion; t0 += kIonTile) {
    const int nt = min(kIonTile, n_ion - t0);
    __syncthreads();
    for (int q = threadIdx.x; q < 3 * nt; q += blockDim.x) s_ion[q] = ion_x[3 * t0 + q];
    __syncthreads();
    if (live && ion_ok)
      for (int j = 0; j < nt; j++)
        if (!clear(dist2(s_ion + 3 * j, X, L, LH))) {
          ion_ok = false;
          break;
        }
  }
  if (!live) return;
  const double o[3] = {0.0, 0.0, 0.0};
  const bool origin_ok = clear(dist2(o, X, L, LH));
  bits[id] = (unsigned char)((ion_ok ? 1 : 0) | (origin_ok ? 2 : 0));
  cx[3 * id] = X[0];
  cx[3 * id + 1] = X[1];
  cx[3 * id + 2] = X[2];
  if (ion_ok) atomicMin(first, id);
}

/* the acceptance rule: clear of the ion, and of the origin unless this is
 * the species' first molecule with no earlier molecule in the table */
__device__ __forceinline__ bool accepted(unsigned char b, int id, int exempt) {
  return (b & 1) && ((b & 2) || id == exempt);
}

__global__ void __launch_bounds__(kScanThreads) place_count(const unsigned char* bits, int K, int exempt,
                                                             int* counts) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const bool a = id < K && accepted(bits[id], id, exempt);
  const int n = __syncthreads_count(a);
  if (threadIdx.x == 0) counts[blockIdx.x] = n;
}

/* rows in candidate order: row = placed + (accepted candidates before it) */
__global__ void __launch_bounds__(kScanThreads) place_scatter(const unsigned char* bits, const double* cx, int K,
                                                               int exempt, const int* counts, long long placed,
                                                               long long n, double* out_x) {
  __shared__ int s_red[kScanThreads / 32];
  __shared__ int s_base;
  /* this block's offset: the counts of the blocks before it */
  int part = 0;
  for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) part += counts[b];
  for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) s_red[wid] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += s_red[w];
    s_base = s;
  }
  __syncthreads();
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const bool a = id < K && accepted(bits[id], id, exempt);
  const unsigned ball = __ballot_sync(0xffffffffu, a);
  __syncthreads();
  if (lane == 0) s_red[wid] = __popc(ball);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      const int c = s_red[w];
      s_red[w] = s;
      s += c;
    }
  }
  __syncthreads();
  if (!a) return;
  const long long row = placed + s_base + s_red[wid] + __popc(ball & ((1u << lane) - 1u));
  if (row >= n) return;
  out_x[3 * row] = cx[3 * id];
  out_x[3 * row + 1] = cx[3 * id + 1];
  out_x[3 * row + 2] = cx[3 * id + 2];
}

/* Maxwell-Boltzmann centre velocity of molecule i: two Box-Muller pairs
 * from one draw, the fourth deviate unused; sigma * N(0,1) * 1e-5 A/fs */
__global__ void place_velocity(long long n, double sigma, unsigned long long seed, uint32_t purpose, double* v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const mdn::U4 w = draw(seed, purpose, i);
  double z[4];
  mdn::box_muller(w.v[0], w.v[1], z[0], z[1]);
  mdn::box_muller(w.v[2], w.v[3], z[2], z[3]);
  for (int c = 0; c < 3; c++) v[3 * i + c] = sigma * z[c] * 1e-5;
}

struct Dev {
  double* ion = nullptr;
  double* cx = nullptr;
  unsigned char* bits = nullptr;
  int* counts = nullptr;
  int* first = nullptr;
  double* x = nullptr;
  double* v = nullptr;
  cudaStream_t st = nullptr;
  ~Dev() {
    if (st) cudaStreamSynchronize(st);
    cudaFree(ion);
    cudaFree(cx);
    cudaFree(bits);
    cudaFree(counts);
    cudaFree(first);
    cudaFree(x);
    cudaFree(v);
    if (st) cudaStreamDestroy(st);
  }
};

int cuda_fail(const char* what, cudaError_t e) {
  char msg[256];
  snprintf(msg, sizeof msg, "mdn_place: %s: %s", what, cudaGetErrorString(e));
  return mdn_error(MDN_ERR_CUDA, msg);
}

/* one species (0 gas, 1 vapor): n molecules, counter purpose `species` for
 * the centres and 2 + species for the velocities; origin_from_start: an
 * earlier molecule is already in the table */
int place_species(Dev& d, const mdn_place_desc* p, uint32_t species, long long n, double sigma,
                  bool origin_from_start, long long chunk, double* hx, double* hv, const char* what) {
  if (n == 0) return MDN_OK;
  const long long cap = 1000LL * (n + 10);
  long long placed = 0, k0 = 0;
  /* local index of the exempt candidate in the current chunk: -1 none */
  bool pending = !origin_from_start;
  cudaError_t e;
  std::vector<int> counts;
  while (placed < n) {
    if (k0 >= cap) {
      char msg[160];
      snprintf(msg, sizeof msg, "%s placement did not converge (box %.1f A)", what, p->box);
      return mdn_error(MDN_ERR_ARG, msg);
    }
    /* candidates this round: the molecules still wanted plus a quarter
     * (the acceptance is near 1 in the reference's dilute boxes) */
    const long long want = n - placed;
    const int K = (int)std::min(std::min<long long>(chunk, want + want / 4 + 4096), cap - k0);
    const int big = INT_MAX;
    if ((e = cudaMemcpyAsync(d.first, &big, sizeof(int), cudaMemcpyHostToDevice, d.st)) != cudaSuccess)
      return cuda_fail("copy", e);
    place_test<<<(K + kTestThreads - 1) / kTestThreads, kTestThreads, 0, d.st>>>(
        d.ion, p->n_ion, p->box, p->min_dist, p->seed, species, k0, K, d.bits, d.cx, d.first);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail("place_test", e);
    int exempt = -1;
    if (pending) {
      int f = big;
      if ((e = cudaMemcpyAsync(&f, d.first, sizeof(int), cudaMemcpyDeviceToHost, d.st)) != cudaSuccess ||
          (e = cudaStreamSynchronize(d.st)) != cudaSuccess)
        return cuda_fail("copy", e);
      if (f != big) {
        exempt = f;  /* the first molecule: nothing but the ion in the table */
        pending = false;
      }
    }
    const int nb = (K + kScanThreads - 1) / kScanThreads;
    place_count<<<nb, kScanThreads, 0, d.st>>>(d.bits, K, exempt, d.counts);
    place_scatter<<<nb, kScanThreads, 0, d.st>>>(d.bits, d.cx, K, exempt, d.counts, placed, n, d.x);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail("place_scatter", e);
    counts.resize(nb);
    if ((e = cudaMemcpyAsync(counts.data(), d.counts, sizeof(int) * nb, cudaMemcpyDeviceToHost, d.st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(d.st)) != cudaSuccess)
      return cuda_fail("count", e);
    long long got = 0;
    for (int c : counts) got += c;
    placed = std::min(n, placed + got);
    k0 += K;
  }
  const int vt = 256;
  place_velocity<<<(unsigned)((n + vt - 1) / vt), vt, 0, d.st>>>(n, sigma, p->seed, 2 + species, d.v);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail("place_velocity", e);
  if ((e = cudaMemcpyAsync(hx, d.x, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, d.st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(hv, d.v, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, d.st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(d.st)) != cudaSuccess)
    return cuda_fail("copy back", e);
  return MDN_OK;
}

}  // namespace

extern "C" int mdn_place(int device, const mdn_place_desc* p, double* gas_x, double* gas_v, double* vapor_x,
                         double* vapor_v) {
  if (!p) return mdn_error(MDN_ERR_ARG, "mdn_place: null descriptor");
  if (!(p->box > 0) || !(p->min_dist >= 0) || p->n_ion < 0 || p->n_gas < 0 || p->n_vapor < 0 ||
      (p->n_ion > 0 && !p->ion_x) || (p->n_gas > 0 && (!gas_x || !gas_v)) ||
      (p->n_vapor > 0 && (!vapor_x || !vapor_v)) || !(p->gas_sigma >= 0) || !(p->vapor_sigma >= 0))
    return mdn_error(MDN_ERR_ARG, "mdn_place: bad descriptor");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return mdn_error(MDN_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return mdn_error(MDN_ERR_ARG, "mdn_place: device out of range");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail("cudaSetDevice", e);
  const long long nmax = std::max(p->n_gas, p->n_vapor);
  if (nmax == 0) return MDN_OK;
  /* the largest round either species can take */
  const long long chunk = std::min<long long>(nmax + nmax / 4 + 4096, 1LL << 26);
  Dev d;
  if ((e = cudaStreamCreateWithFlags(&d.st, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaMalloc((void**)&d.ion, sizeof(double) * 3 * std::max(1, p->n_ion))) != cudaSuccess ||
      (e = cudaMalloc((void**)&d.cx, sizeof(double) * 3 * chunk)) != cudaSuccess ||
      (e = cudaMalloc((void**)&d.bits, chunk)) != cudaSuccess ||
      (e = cudaMalloc((void**)&d.counts, sizeof(int) * ((chunk + kScanThreads - 1) / kScanThreads))) !=
          cudaSuccess ||
      (e = cudaMalloc((void**)&d.first, sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc((void**)&d.x, sizeof(double) * 3 * nmax)) != cudaSuccess ||
      (e = cudaMalloc((void**)&d.v, sizeof(double) * 3 * nmax)) != cudaSuccess)
    return cuda_fail("allocation", e);
  if (p->n_ion > 0 &&
      (e = cudaMemcpyAsync(d.ion, p->ion_x, sizeof(double) * 3 * p->n_ion, cudaMemcpyHostToDevice, d.st)) !=
          cudaSuccess)
    return cuda_fail("copy", e);
  int rc = place_species(d, p, 0, p->n_gas, p->gas_sigma, false, chunk, gas_x, gas_v, "gas");
  if (rc) return rc;
  return place_species(d, p, 1, p->n_vapor, p->vapor_sigma, p->n_gas > 0, chunk, vapor_x, vapor_v, "vapor");
}
