/*
 * snapshot.cu -- the output path: every replica's in-domain atoms (what
 * MD::export_dump_close writes, src/output/output.cpp:133-170) and energies
 * gathered on the device into one packed staging buffer and copied to the
 * host with one asynchronous copy per array.
 *
 * Layout of a snapshot: replica r owns rows [offset[r], offset[r+1]); inside
 * a replica the ion atoms come first, then the gas atoms of the in-domain
 * molecules (ascending molecule index), then the vapor atoms -- the order of
 * the reference's dump loop over molecules with region[i] set.
 */
#include <cuda_runtime.h>

#include "mdn.h"
#include "mdn_types.h"

namespace {

__global__ void snapshot_counts(const RepParams* P, const RepDyn* D, int R, long long* offset) {
  /* one thread: R is at most a few thousand */
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    long long o = 0;
    for (int r = 0; r < R; r++) {
      offset[r] = o;
      o += P[r].n_ion + (long long)D[r].n_gas_in * P[r].a_g +
           (long long)D[r].n_vap_in * (P[r].n_vap > 0 ? P[r].a_v : 0);
    }
    offset[R] = o;
  }
}

__global__ void snapshot_gather(const RepParams* P, const RepDyn* D, const int* iblob, const long long* offset,
                                long long capacity, const double* ion_x, const double* ion_v, const double* slab_x,
                                const double* slab_v, const double* vslab_x, const double* vslab_v, int* type,
                                double* x, double* v) {
  const int r = blockIdx.x;
  const RepParams& p = P[r];
  const RepDyn& d = D[r];
  const long long base = offset[r];
  const int* ib = iblob + p.iblob_off;
  const int ni = p.n_ion, ag = p.a_g, av = p.a_v;
  const long long ng = (long long)d.n_gas_in * ag;
  const long long nv = p.n_vap > 0 ? (long long)d.n_vap_in * av : 0;
  const long long n = ni + ng + nv;
  for (long long t = threadIdx.x; t < n; t += blockDim.x) {
    const long long row = base + t;
    if (row >= capacity) break;
    const double *sx, *sv;
    int ty;
    if (t < ni) {
      size_t g = (size_t)p.ion_off + t;
      sx = ion_x + 3 * g;
      sv = ion_v + 3 * g;
      ty = ib[p.o_ion_type + t];
    } else if (t < ni + ng) {
      long long u = t - ni;
      int s = (int)(u / ag), a = (int)(u - (long long)s * ag);
      size_t g = (size_t)p.slab_off + ((size_t)d.parity * p.slab_cap + s) * ag + a;
      sx = slab_x + 3 * g;
      sv = slab_v + 3 * g;
      ty = ib[p.o_gas_type + a];
    } else {
      long long u = t - ni - ng;
      int s = (int)(u / av), a = (int)(u - (long long)s * av);
      size_t g = (size_t)p.vslab_off + ((size_t)d.parity * p.vcap + s) * av + a;
      sx = vslab_x + 3 * g;
      sv = vslab_v + 3 * g;
      ty = ib[p.o_vap_type + a];
    }
    type[row] = ty;
    for (int k = 0; k < 3; k++) {
      x[3 * row + k] = sx[k];
      v[3 * row + k] = sv[k];
    }
  }
}

}  // namespace

/* Host side, called from engine.cu and snapshot_noalloc.cu with the
 * handle's device pointers.  Returns the launch error it read (and thereby
 * cleared), cudaSuccess when both kernels were queued. */
cudaError_t mdn_snapshot_device(const RepParams* dP, const RepDyn* dD, const int* d_iblob, int R,
                                const double* ion_x, const double* ion_v, const double* slab_x,
                                const double* slab_v, const double* vslab_x, const double* vslab_v,
                                long long* d_offset, int* d_type, double* d_x, double* d_v, long long d_capacity,
                                cudaStream_t stream) {
  snapshot_counts<<<1, 32, 0, stream>>>(dP, dD, R, d_offset);
  snapshot_gather<<<R, 256, 0, stream>>>(dP, dD, d_iblob, d_offset, d_capacity, ion_x, ion_v, slab_x, slab_v,
                                         vslab_x, vslab_v, d_type, d_x, d_v);
  return cudaGetLastError();
}

/* Loads the snapshot kernels on the current device (under lazy module
 * loading a kernel's module is loaded, and its code memory allocated, when
 * the kernel is first named), so that a later snapshot loads nothing. */
__attribute__((visibility("hidden"))) cudaError_t mdn_snapshot_load_kernels() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, snapshot_counts);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, snapshot_gather);
  return e;
}
