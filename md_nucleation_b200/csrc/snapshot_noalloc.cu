/*
 * snapshot_noalloc.cu -- mdn_snapshot_noalloc: the batch snapshot of
 * mdn_snapshot (every replica's in-domain atoms, the rows of
 * MD::export_dump_close, src/output/output.cpp:133-170) staged in a fixed
 * device array that the library holds on each device, so the call allocates
 * no memory.  The gather kernels are the ones mdn_snapshot launches
 * (snapshot.cu); only their staging differs.
 *
 * The array is one file-scope __device__ symbol, carved as
 *   [0, OFF_BYTES)              offsets, MDN_NOALLOC_MAX_REPLICAS + 1 int64
 *   [TYPE_AT, +4*ROWS)          atom type per row
 *   [X_AT, +24*ROWS)            positions, 3 doubles per row
 *   [V_AT, +24*ROWS)            velocities, 3 doubles per row
 * Nothing in it has to start at zero: snapshot_counts writes offsets
 * 0..R, snapshot_gather writes every row below offset[R] (and none at or
 * beyond MDN_NOALLOC_MAX_ROWS), and only those are copied back.  Every call
 * in the process shares it; calls that overlap in time on one device race.
 *
 * The per-device set-up (the array's device address, found with
 * cudaGetSymbolAddress; the module that holds the array, and the snapshot
 * kernels' module, loaded) runs once per device inside mdn_create, so even
 * under lazy module loading the first snapshot call loads and allocates
 * nothing.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "mdn.h"
#include "mdn_types.h"

cudaError_t mdn_snapshot_device(const RepParams* dP, const RepDyn* dD, const int* d_iblob, int R,
                                const double* ion_x, const double* ion_v, const double* slab_x,
                                const double* slab_v, const double* vslab_x, const double* vslab_v,
                                long long* d_offset, int* d_type, double* d_x, double* d_v, long long d_capacity,
                                cudaStream_t stream);
__attribute__((visibility("hidden"))) void mdn_snapshot_args(const mdn_handle* h, SnapshotArgs* s);
__attribute__((visibility("hidden"))) int mdn_error(int code, const char* msg);
__attribute__((visibility("hidden"))) cudaError_t mdn_snapshot_load_kernels();

namespace {

constexpr size_t ROWS = MDN_NOALLOC_MAX_ROWS;
constexpr size_t round256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t OFF_BYTES = round256(sizeof(long long) * (MDN_NOALLOC_MAX_REPLICAS + 1));
constexpr size_t TYPE_AT = OFF_BYTES;
constexpr size_t X_AT = TYPE_AT + round256(sizeof(int) * ROWS);
constexpr size_t V_AT = X_AT + round256(3 * sizeof(double) * ROWS);
constexpr size_t SCRATCH_BYTES = V_AT + round256(3 * sizeof(double) * ROWS);

/* the devices a process may use, for the per-device set-up below */
constexpr int MAX_DEVICES = 64;

}  // namespace

static __device__ __align__(256) unsigned char g_snapshot_scratch[SCRATCH_BYTES];

namespace {

std::once_flag g_once[MAX_DEVICES];
unsigned char* g_scratch[MAX_DEVICES];
cudaError_t g_setup_rc[MAX_DEVICES];

int error(int code, const char* fmt, long long a, long long b) {
  char buf[320];
  snprintf(buf, sizeof buf, fmt, a, b);
  return mdn_error(code, buf);
}

/* The per-device set-up, once per device with that device current: the
 * device address of the array (looking it up loads the module that holds
 * it, which is where the array's memory is allocated), and the snapshot
 * kernels loaded too.  mdn_create runs it for its device, so a snapshot
 * call finds it done. */
void setup_once(int dev) {
  std::call_once(g_once[dev], [dev] {
    void* p = nullptr;
    g_setup_rc[dev] = cudaGetSymbolAddress(&p, g_snapshot_scratch);
    if (g_setup_rc[dev] == cudaSuccess) g_setup_rc[dev] = mdn_snapshot_load_kernels();
    g_scratch[dev] = g_setup_rc[dev] == cudaSuccess ? (unsigned char*)p : nullptr;
  });
}

/* The device address of the array on `dev` (current device). */
int scratch_on(int dev, unsigned char** out) {
  if (dev < 0 || dev >= MAX_DEVICES)
    return error(MDN_ERR_ARG, "mdn_snapshot_noalloc: device %lld beyond the %lld devices it supports", dev,
                 MAX_DEVICES);
  setup_once(dev);
  if (g_setup_rc[dev] != cudaSuccess || !g_scratch[dev]) {
    char buf[256];
    snprintf(buf, sizeof buf, "mdn_snapshot_noalloc: cudaGetSymbolAddress of the staging array failed: %s",
             cudaGetErrorString(g_setup_rc[dev]));
    return mdn_error(MDN_ERR_CUDA, buf);
  }
  *out = g_scratch[dev];
  return MDN_OK;
}

int cuda_fail(const char* what, cudaError_t e) {
  char buf[256];
  snprintf(buf, sizeof buf, "mdn_snapshot_noalloc: %s: %s", what, cudaGetErrorString(e));
  return mdn_error(MDN_ERR_CUDA, buf);
}

}  // namespace

/* Internal, for mdn_create: the set-up above for the handle's device (the
 * current device).  A failure is kept and reported by mdn_snapshot_noalloc,
 * so creating a handle never fails for it. */
__attribute__((visibility("hidden"))) void mdn_noalloc_setup(int dev) {
  if (dev >= 0 && dev < MAX_DEVICES) setup_once(dev);
}

extern "C" int mdn_snapshot_noalloc(mdn_handle* h, long long* offset, long long capacity, int* type, double* x,
                                    double* v, double* U) {
  if (!h || !offset) return mdn_error(MDN_ERR_ARG, "mdn_snapshot_noalloc: null handle or offset");
  SnapshotArgs s;
  mdn_snapshot_args(h, &s);
  if (s.R > MDN_NOALLOC_MAX_REPLICAS)
    return error(MDN_ERR_CAPACITY,
                 "mdn_snapshot_noalloc: %lld replicas, the fixed staging holds %lld (MDN_NOALLOC_MAX_REPLICAS); "
                 "use mdn_snapshot",
                 s.R, MDN_NOALLOC_MAX_REPLICAS);
  cudaError_t e = cudaSetDevice(s.dev);
  if (e != cudaSuccess) return cuda_fail("cudaSetDevice", e);
  unsigned char* base = nullptr;
  int rc = scratch_on(s.dev, &base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)s.stream;
  long long* d_off = (long long*)base;
  int* d_type = (int*)(base + TYPE_AT);
  double* d_x = (double*)(base + X_AT);
  double* d_v = (double*)(base + V_AT);
  if ((e = mdn_snapshot_device(s.P, s.D, s.iblob, s.R, s.ion_x, s.ion_v, s.slab_x, s.slab_v, s.vslab_x,
                               s.vslab_v, d_off, d_type, d_x, d_v, (long long)ROWS, st)) != cudaSuccess)
    return cuda_fail("snapshot kernels", e);
  if ((e = cudaMemcpyAsync(offset, d_off, sizeof(long long) * (s.R + 1), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return cuda_fail("offset copy", e);
  /* energies: the int64 fixed-point sums land in U itself and are converted
   * in place, so no host buffer is needed either */
  if (U && (e = cudaMemcpyAsync(U, s.energy, sizeof(long long) * 8 * s.R, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return cuda_fail("energy copy", e);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail("snapshot", e);
  if (U)
    for (long long i = 0; i < 8LL * s.R; i++) {
      long long q;
      memcpy(&q, U + i, sizeof q);
      U[i] = (double)q * MDN_EFIX_INV;
    }
  const long long total = offset[s.R];
  if (total > (long long)ROWS)
    return error(MDN_ERR_CAPACITY,
                 "mdn_snapshot_noalloc: the snapshot has %lld rows, the fixed staging holds %lld "
                 "(MDN_NOALLOC_MAX_ROWS); use mdn_snapshot",
                 total, (long long)ROWS);
  if (total > capacity)
    return error(MDN_ERR_CAPACITY, "mdn_snapshot_noalloc: the snapshot needs %lld rows, the buffer holds %lld", total,
                 capacity);
  if (total > 0) {
    if (type && (e = cudaMemcpyAsync(type, d_type, sizeof(int) * total, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return cuda_fail("type copy", e);
    if (x && (e = cudaMemcpyAsync(x, d_x, 3 * sizeof(double) * total, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return cuda_fail("position copy", e);
    if (v && (e = cudaMemcpyAsync(v, d_v, 3 * sizeof(double) * total, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return cuda_fail("velocity copy", e);
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail("snapshot copies", e);
  return MDN_OK;
}
