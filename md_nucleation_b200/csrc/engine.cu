/*
 * engine.cu -- host side of the C ABI declared in include/mdn.h.
 *
 * mdn_create packs every replica descriptor into per-replica blobs (type
 * tables, Lorentz-Berthelot LJ table, topology, SHAKE colouring, AMBER
 * exclusion bitmask), sizes the device pools, uploads them and runs the
 * initial MD::make_pair on the device.  mdn_step launches the persistent
 * kernel of advance.cu.  Everything else moves state between the device
 * pools and host arrays in the reference's layout.
 *
 * No function here falls back to a CPU computation: without a CUDA device
 * mdn_create fails with MDN_ERR_NO_DEVICE.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <functional>
#include <vector>

#include "mdn.h"
#include "mdn_types.h"

extern "C" __global__ void mdn_advance(KArgs a);
extern "C" __global__ void mdn_advance_fp64(KArgs a);
extern "C" __global__ void mdn_advance_gg(KArgs a);
extern "C" __global__ void mdn_advance_gg_fp64(KArgs a);
cudaError_t mdn_snapshot_device(const RepParams* dP, const RepDyn* dD, const int* d_iblob, int R,
                                const double* ion_x, const double* ion_v, const double* slab_x,
                                const double* slab_v, const double* vslab_x, const double* vslab_v,
                                long long* d_offset, int* d_type, double* d_x, double* d_v, long long d_capacity,
                                cudaStream_t stream);

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(MDN_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                    \
  } while (0)

/* constants of src/constants.hpp:28-53, same expressions */
const double Nw = 6.02e23;
const double kb = 1.38e-23;
const double kb_real = kb * Nw / 4184.0;
const double e0 = 8.85e-12;
const double e_ch = 1.602e-19;
const double qqrd2e = e_ch * e_ch / 4.0 / M_PI / e0 * Nw * 1e10 / 4184.0;
const double real_to_kcalmol = 10000 / 4.184;

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
};

/* greedy colouring of constraints: each pair takes the lowest colour not used
 * by an earlier pair sharing an atom (the order the SHAKE sweeps follow) */
int color_rigid(const int* rig, int n, std::vector<int>& color) {
  color.assign(n, 0);
  int nc = 0;
  for (int k = 0; k < n; k++) {
    int c = 0;
    for (;;) {
      bool clash = false;
      for (int p = 0; p < k; p++)
        if (color[p] == c && (rig[3 * p] == rig[3 * k] || rig[3 * p] == rig[3 * k + 1] ||
                              rig[3 * p + 1] == rig[3 * k] || rig[3 * p + 1] == rig[3 * k + 1])) {
          clash = true;
          break;
        }
      if (!clash) break;
      c++;
    }
    color[k] = c;
    nc = std::max(nc, c + 1);
  }
  return nc;
}

/* the constraints' connected groups (constraints sharing an atom, joined
 * transitively): order = constraint indices group by group, start = group
 * starts (n_groups + 1).  Returns the number of groups, or 0 when a group
 * holds more than 3 constraints (the kernel then sweeps). */
int group_rigid(const int* rig, int n, std::vector<int>& order, std::vector<int>& start) {
  order.clear();
  start.clear();
  if (n <= 0) return 0;
  std::vector<int> parent(n);
  for (int k = 0; k < n; k++) parent[k] = k;
  std::function<int(int)> root = [&](int k) { return parent[k] == k ? k : parent[k] = root(parent[k]); };
  for (int a = 0; a < n; a++)
    for (int b = 0; b < a; b++)
      if (rig[3 * a] == rig[3 * b] || rig[3 * a] == rig[3 * b + 1] || rig[3 * a + 1] == rig[3 * b] ||
          rig[3 * a + 1] == rig[3 * b + 1])
        parent[root(a)] = root(b);
  std::vector<int> seen(n, 0);
  for (int a = 0; a < n; a++) {
    const int g = root(a);
    if (seen[g]) continue;
    seen[g] = 1;
    start.push_back((int)order.size());
    for (int k = 0; k < n; k++)
      if (root(k) == g) order.push_back(k);
    if ((int)order.size() - start.back() > 3) {
      order.clear();
      start.clear();
      return 0;
    }
  }
  start.push_back((int)order.size());
  return (int)start.size() - 1;
}

}  // namespace

struct mdn_handle {
  int R = 0;
  mdn_options opt;
  int dev = 0, num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<RepParams> P;
  std::vector<RepDyn> D0;
  std::vector<std::vector<int>> type_names;  /* unused placeholder */
  int nc_cap = 0, nt_cap = 0, excl_cap = 0;
  size_t smem = 0;
  /* device pools */
  RepParams* dP = nullptr;
  RepDyn* dD = nullptr;
  int* d_iblob = nullptr;
  double* d_dblob = nullptr;
  double *ion_x = nullptr, *ion_v = nullptr, *ion_f = nullptr;
  double *mol_x = nullptr, *mol_v = nullptr;
  unsigned char* region = nullptr;
  int* slot = nullptr;
  double *slab_x = nullptr, *slab_v = nullptr, *slab_f = nullptr;
  int* slab_mol = nullptr;
  double *vslab_x = nullptr, *vslab_v = nullptr, *vslab_f = nullptr;
  float* vslab_w = nullptr;
  int* vslab_mol = nullptr;
  int* near_list = nullptr;
  int *near_gi = nullptr, *near_gv = nullptr;
  unsigned short *gil_n = nullptr, *gvl_n = nullptr, *gil = nullptr, *gvl = nullptr;
  int *ggl_start = nullptr, *ggl_n = nullptr, *ggl = nullptr, *slab_ins = nullptr;
  double* slab_fgg = nullptr;
  long long* energy = nullptr;
  DevEvent* events = nullptr;
  int* n_events = nullptr;
  int ev_cap = 65536;
  int* status = nullptr;
  int auto_cluster = 1;  /* cluster size when mdn_options.cluster_size is 0 */
  int* job_order = nullptr;
  int* job_counter = nullptr;
  /* split step launch: the split_n largest replicas in a second, concurrent
   * launch with clusters of split_cluster CTAs (0: one launch) */
  int split_n = 0, split_cluster = 0;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int* job_order2 = nullptr;
  int* job_counter2 = nullptr;
  std::vector<int> order;
  std::vector<int> h_iblob;
  std::vector<int> ctl_mode;
  std::vector<double> ctl_T;
  int* d_ctl_mode = nullptr;
  double* d_ctl_T = nullptr;
  long long* d_prof = nullptr;
  bool prof_on = false;
  /* sizes */
  size_t n_ion_tot = 0, n_mol_tot = 0, n_slab_atoms = 0, n_slab_mols = 0, n_vslab_atoms = 0,
         n_vslab_mols = 0, n_near = 0, n_gil = 0, n_gvl = 0, n_ggl = 0;
  double last_ms = 0;
  long long last_launches = 0;
  /* snapshot staging */
  long long snap_cap = 0;
  long long* snap_off = nullptr;
  int* snap_type = nullptr;
  double *snap_x = nullptr, *snap_v = nullptr;
  std::vector<std::vector<std::string>> names;
};

namespace {

void free_all(mdn_handle* h) {
  void* ptrs[] = {h->dP, h->dD, h->d_iblob, h->d_dblob, h->ion_x, h->ion_v, h->ion_f, h->mol_x, h->mol_v,
                  h->region, h->slot, h->slab_x, h->slab_v, h->slab_f, h->slab_mol, h->vslab_x, h->vslab_v,
                  h->vslab_f, h->vslab_w, h->vslab_mol, h->near_list, h->near_gi, h->near_gv, h->gil_n,
                  h->gvl_n, h->gil, h->gvl, h->energy, h->events, h->n_events, h->status, h->job_order,
                  h->job_counter, h->snap_off, h->snap_type, h->snap_x, h->snap_v, h->d_ctl_mode,
                  h->d_ctl_T, h->d_prof, h->job_order2, h->job_counter2, h->ggl_start, h->ggl_n, h->ggl,
                  h->slab_fgg, h->slab_ins};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->stream2) cudaStreamDestroy(h->stream2);
  if (h->stream) cudaStreamDestroy(h->stream);
}

size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

/* dynamic shared memory of the kernel, carved in this order in advance.cu */
size_t smem_bytes(int nc, int nt, int excl) {
  size_t s = 0;
  s += align16(sizeof(long long) * 3 * nc);
  s += align16(sizeof(unsigned) * 9 * nc);
  s += 3 * align16(sizeof(double) * 3 * nc);
  s += align16(sizeof(float4) * nc);
  s += 3 * align16(sizeof(int) * nc);
  s += align16(sizeof(unsigned) * excl);
  s += 2 * align16(sizeof(float) * nt * nt);
  s += align16(sizeof(double) * nt);
  return s;
}

int check_topology(const mdn_topology& t, int n_types, int nb, int na, int nd, const char* what) {
  if (t.n_atoms < 0) return fail(MDN_ERR_ARG, "%s: negative atom count", what);
  for (int i = 0; i < t.n_atoms; i++)
    if (t.type[i] < 0 || t.type[i] >= n_types) return fail(MDN_ERR_ARG, "%s: atom %d type out of range", what, i);
  auto chk = [&](const int* rows, int n, int w, int tmax, const char* kind) -> int {
    for (int r = 0; r < n; r++) {
      for (int k = 0; k < w - 1; k++)
        if (rows[w * r + k] < 0 || rows[w * r + k] >= t.n_atoms)
          return fail(MDN_ERR_ARG, "%s: %s %d atom index out of range", what, kind, r);
      if (rows[w * r + w - 1] < 0 || rows[w * r + w - 1] >= tmax)
        return fail(MDN_ERR_ARG, "%s: %s %d type out of range", what, kind, r);
    }
    return MDN_OK;
  };
  int rc;
  if ((rc = chk(t.bonds, t.n_bonds, 3, nb, "bond"))) return rc;
  if ((rc = chk(t.rigid, t.n_rigid, 3, nb, "rigid pair"))) return rc;
  if ((rc = chk(t.angles, t.n_angles, 4, na, "angle"))) return rc;
  if ((rc = chk(t.dihedrals, t.n_dihedrals, 5, nd, "dihedral"))) return rc;
  return MDN_OK;
}

/* one launch of the step kernel over jobs[0..n_jobs) with clusters of C
 * CTAs on `stream`, using the given device job list and counter */
cudaError_t launch_one(mdn_handle* h, KArgs a, const int* jobs, int n_jobs, int C, int max_clusters,
                       int* d_order, int* d_counter, cudaStream_t stream) {
  cudaError_t e;
  if ((e = cudaMemcpyAsync(d_order, jobs, sizeof(int) * n_jobs, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(d_counter, 0, sizeof(int), stream)) != cudaSuccess)
    return e;
  a.job_order = d_order;
  a.n_jobs = n_jobs;
  a.job_counter = d_counter;
  const int clusters = std::max(1, std::min(max_clusters, n_jobs));
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(clusters * C);
  cfg.blockDim = dim3(h->opt.threads);
  cfg.dynamicSmemBytes = h->smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  /* the gas-gas kernels only when a replica has gg on (advance_gg.cu) */
  const bool gg = h->n_ggl > 0;
  return cudaLaunchKernelEx(&cfg, h->opt.force_mode ? (gg ? mdn_advance_gg_fp64 : mdn_advance_fp64)
                                                    : (gg ? mdn_advance_gg : mdn_advance), a);
}

long long launch(mdn_handle* h, int mode, long long n_steps, int energy_mode, unsigned term_mask,
                 const std::vector<int>* jobs, int* rc, int keep_com = 0) {
  *rc = MDN_OK;
  const std::vector<int>& J = jobs ? *jobs : h->order;
  cudaError_t e;
  KArgs a;
  memset(&a, 0, sizeof a);
  a.P = h->dP;
  a.D = h->dD;
  a.iblob = h->d_iblob;
  a.dblob = h->d_dblob;
  a.ion_x = h->ion_x; a.ion_v = h->ion_v; a.ion_f = h->ion_f;
  a.mol_x = h->mol_x; a.mol_v = h->mol_v;
  a.region = h->region; a.slot = h->slot;
  a.slab_x = h->slab_x; a.slab_v = h->slab_v; a.slab_f = h->slab_f; a.slab_mol = h->slab_mol;
  a.vslab_x = h->vslab_x; a.vslab_v = h->vslab_v; a.vslab_f = h->vslab_f; a.vslab_w = h->vslab_w;
  a.vslab_mol = h->vslab_mol;
  a.near_list = h->near_list; a.near_gi = h->near_gi; a.near_gv = h->near_gv;
  a.gil_n = h->gil_n; a.gvl_n = h->gvl_n; a.gil = h->gil; a.gvl = h->gvl;
  a.ggl_start = h->ggl_start; a.ggl_n = h->ggl_n; a.ggl = h->ggl;
  a.slab_fgg = h->slab_fgg; a.slab_ins = h->slab_ins;
  a.energy = h->energy;
  a.events = h->events; a.n_events = h->n_events; a.ev_cap = h->ev_cap;
  a.status = h->status;
  a.ctl_mode = h->d_ctl_mode;
  a.ctl_T = h->d_ctl_T;
  a.n_steps = n_steps;
  a.energy_mode = energy_mode;
  a.mode = mode;
  a.term_mask = term_mask;
  a.keep_com = keep_com;
  a.prof = h->prof_on ? h->d_prof : nullptr;
  a.nc_cap = h->nc_cap;
  a.nt_cap = h->nt_cap;
  a.excl_cap = h->excl_cap;
  const int C = std::max(1, std::min(8, h->opt.cluster_size > 0 ? h->opt.cluster_size : h->auto_cluster));
  const int n = (int)J.size();
  const int nb = h->split_n, Cb = h->split_cluster;
  if (mode == MDN_MODE_STEP && !jobs && nb > 0 && nb < n && Cb > 0 && nb * Cb + C <= h->num_sms) {
    /* the nb largest replicas (the head of the largest-first order) on
     * clusters of Cb CTAs, one cluster each, on the second stream; the rest
     * on the SMs left.  The two launches share no replica. */
    if ((e = cudaEventRecord(h->ev_fork, h->stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(h->stream2, h->ev_fork, 0)) != cudaSuccess ||
        (e = launch_one(h, a, J.data(), nb, Cb, nb, h->job_order2, h->job_counter2, h->stream2)) != cudaSuccess ||
        (e = launch_one(h, a, J.data() + nb, n - nb, C, (h->num_sms - nb * Cb) / C, h->job_order, h->job_counter,
                        h->stream)) != cudaSuccess ||
        (e = cudaEventRecord(h->ev_join, h->stream2)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(h->stream, h->ev_join, 0)) != cudaSuccess) {
      *rc = fail(MDN_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
      return 0;
    }
    return 2;
  }
  if ((e = launch_one(h, a, J.data(), n, C, h->num_sms / C, h->job_order, h->job_counter, h->stream)) !=
      cudaSuccess) {
    *rc = fail(MDN_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return 0;
  }
  return 1;
}

int sync_check(mdn_handle* h) {
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(MDN_ERR_CUDA, "kernel failed: %s", cudaGetErrorString(e));
  return MDN_OK;
}

}  // namespace

/* Internal, for snapshot_noalloc.cu: the snapshot kernels' inputs of a
 * handle, and the text mdn_last_error returns. */
__attribute__((visibility("hidden"))) void mdn_snapshot_args(const mdn_handle* h, SnapshotArgs* s) {
  s->P = h->dP;
  s->D = h->dD;
  s->iblob = h->d_iblob;
  s->R = h->R;
  s->dev = h->dev;
  s->ion_x = h->ion_x;
  s->ion_v = h->ion_v;
  s->slab_x = h->slab_x;
  s->slab_v = h->slab_v;
  s->vslab_x = h->vslab_x;
  s->vslab_v = h->vslab_v;
  s->energy = h->energy;
  s->stream = (void*)h->stream;
}

__attribute__((visibility("hidden"))) int mdn_error(int code, const char* msg) { return fail(code, "%s", msg); }

__attribute__((visibility("hidden"))) void mdn_noalloc_setup(int dev);

__attribute__((visibility("hidden"))) unsigned mdn_internal_quirks(const mdn_handle* h) { return h->opt.quirks; }

extern "C" {

int mdn_abi_version(void) { return MDN_ABI_VERSION; }

const char* mdn_last_error(void) { return g_err.c_str(); }

void mdn_default_options(mdn_options* o) {
  memset(o, 0, sizeof *o);
  o->quirks = MDN_Q_ALL;
  o->force_mode = 0;
  o->cluster_size = 0;
  o->threads = 512;
  o->steps_per_launch = 0;
  o->use_graph = 0;
  o->capacity_factor = 1.5;
  o->device = 0;
}

int mdn_device_count(int* n) {
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) c = 0;
  *n = c;
  return MDN_OK;
}

int mdn_create(const mdn_replica_desc* descs, int R, const mdn_options* opt_in, mdn_handle** out) {
  *out = nullptr;
  if (!descs || R <= 0) return fail(MDN_ERR_ARG, "no replicas");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(MDN_ERR_NO_DEVICE, "no CUDA device");
  mdn_options opt;
  mdn_default_options(&opt);
  if (opt_in) opt = *opt_in;
  if (opt.threads <= 0) opt.threads = 512;
  if (opt.threads % 32 || opt.threads > 512) return fail(MDN_ERR_ARG, "threads must be a multiple of 32 <= 512");
  if (opt.capacity_factor < 1.0) opt.capacity_factor = 1.0;
  if (opt.cluster_size < 0 || opt.cluster_size > 8) return fail(MDN_ERR_ARG, "cluster size must be 0..8");
  if (opt.device < 0 || opt.device >= ndev) return fail(MDN_ERR_ARG, "bad device ordinal");

  mdn_handle* h = new mdn_handle();
  h->R = R;
  h->opt = opt;
  h->dev = opt.device;
  cudaSetDevice(h->dev);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->dev);

  std::vector<int> iblob;
  std::vector<double> dblob;
  h->P.resize(R);
  h->D0.resize(R);
  size_t ion_tot = 0, mol_tot = 0, slab_atoms = 0, slab_mols = 0, vslab_atoms = 0, vslab_mols = 0, near_tot = 0,
         gil_tot = 0, gvl_tot = 0, ggl_tot = 0;
  for (int r = 0; r < R; r++) {
    const mdn_replica_desc& d = descs[r];
    RepParams& P = h->P[r];
    memset(&P, 0, sizeof P);
    int nt = d.n_atom_types;
    if (nt <= 0 || nt > MDN_MAX_TYPES) { delete h; return fail(MDN_ERR_CAPACITY, "replica %d: %d atom types (max %d)", r, nt, MDN_MAX_TYPES); }
    if (d.gas.n_atoms < 1 || d.gas.n_atoms > MDN_MAX_GAS_ATOMS) { delete h; return fail(MDN_ERR_CAPACITY, "replica %d: gas molecule of %d atoms (1..%d)", r, d.gas.n_atoms, MDN_MAX_GAS_ATOMS); }
    if (d.n_vapor > 0 && (d.vapor.n_atoms < 1 || d.vapor.n_atoms > MDN_MAX_VAP_ATOMS)) { delete h; return fail(MDN_ERR_CAPACITY, "replica %d: vapor molecule of %d atoms (1..%d)", r, d.vapor.n_atoms, MDN_MAX_VAP_ATOMS); }
    if (d.ion.n_atoms < 1 || d.ion.n_atoms > 65535) { delete h; return fail(MDN_ERR_CAPACITY, "replica %d: ion of %d atoms", r, d.ion.n_atoms); }
    if (!(d.dt > 0) || !(d.box > 0) || !(d.temperature > 0)) { delete h; return fail(MDN_ERR_ARG, "replica %d: dt, box and temperature must be positive", r); }
    int rc;
    if ((rc = check_topology(d.ion, nt, d.n_bond_types, d.n_angle_types, d.n_dihedral_types, "ion")) ||
        (rc = check_topology(d.gas, nt, d.n_bond_types, d.n_angle_types, d.n_dihedral_types, "gas")) ||
        (rc = check_topology(d.vapor, nt, d.n_bond_types, d.n_angle_types, d.n_dihedral_types, "vapor"))) {
      delete h;
      return rc;
    }
    for (int t = 0; t < d.n_dihedral_types; t++)
      if (d.dihedral_multi[t] < 0 || d.dihedral_multi[t] > 3) { delete h; return fail(MDN_ERR_ARG, "dihedral type %d: multi %d", t, d.dihedral_multi[t]); }
    if (d.interactions & MDN_I_BMH)
      for (int i = 0; i < d.ion.n_atoms; i++)
        if (!d.ion_bmh_type || d.ion_bmh_type[i] < 0 || d.ion_bmh_type[i] > 1) { delete h; return fail(MDN_ERR_ARG, "ion atom %d: Born-Mayer-Huggins row must be 0 (Na) or 1 (Cl)", i); }

    P.n_ion = d.ion.n_atoms;
    P.a_g = d.gas.n_atoms;
    P.a_v = d.n_vapor > 0 ? d.vapor.n_atoms : 1;
    P.n_gas = d.n_gas;
    P.n_vap = d.n_vapor;
    P.n_types = nt;
    P.interactions = d.interactions;
    P.quirks = opt.quirks;
    P.gas_kind = d.gas_kind;
    P.force_mode = opt.force_mode;
    P.dt = d.dt;
    P.box = d.box;
    P.ml2 = (d.cutoff + d.margin) * (d.cutoff + d.margin);
    P.ri2 = d.r_inter * d.r_inter;
    P.RI2 = (d.r_inter + d.overlap) * (d.r_inter + d.overlap);
    P.rcenter = d.r_inter - d.overlap * 0.5;
    P.overlap = d.overlap;
    P.margin = d.margin;
    P.coeff = 0.5 * d.dt * 4.184e-4;
    P.gas_com_mass = d.gas_com_mass;
    P.vap_com_mass = d.vapor_com_mass;
    P.gas_sigma = sqrt(kb * d.temperature / d.gas_mb_mass) * 1e-5;
    P.vap_sigma = d.vapor_mb_mass > 0 ? sqrt(kb * d.temperature / d.vapor_mb_mass) * 1e-5 : 0;
    P.qqrd2e = qqrd2e;
    P.kb_real = kb_real;
    P.real_to_kcalmol = real_to_kcalmol;
    for (int k = 0; k < 3; k++) P.efield[k] = d.efield[k];
    P.key0 = (unsigned)(d.seed & 0xffffffffull);
    P.key1 = (unsigned)(d.seed >> 32);

    /* ---- int blob ---- */
    P.iblob_off = (long long)iblob.size();
    auto ipush = [&](const int* p, int n) {
      int o = (int)(iblob.size() - P.iblob_off);
      for (int i = 0; i < n; i++) iblob.push_back(p[i]);
      return o;
    };
    std::vector<int> tmp;
    P.o_ion_type = ipush(d.ion.type, d.ion.n_atoms);
    tmp.assign(d.ion.n_atoms, 0);
    if (d.ion_bmh_type) for (int i = 0; i < d.ion.n_atoms; i++) tmp[i] = d.ion_bmh_type[i];
    P.o_ion_bmh = ipush(tmp.data(), d.ion.n_atoms);
    P.n_ion_bonds = d.ion.n_bonds;
    P.o_ion_bonds = ipush(d.ion.bonds, 3 * d.ion.n_bonds);
    P.n_ion_angles = d.ion.n_angles;
    P.o_ion_angles = ipush(d.ion.angles, 4 * d.ion.n_angles);
    P.n_ion_dih = d.ion.n_dihedrals;
    P.o_ion_dih = ipush(d.ion.dihedrals, 5 * d.ion.n_dihedrals);
    P.n_ion_rigid = d.ion.n_rigid;
    P.o_ion_rigid = ipush(d.ion.rigid, 3 * d.ion.n_rigid);
    std::vector<int> col;
    P.n_ion_colors = color_rigid(d.ion.rigid, d.ion.n_rigid, col);
    P.o_ion_color = ipush(col.data(), (int)col.size());
    {
      std::vector<int> go, gs;
      P.n_ion_groups = group_rigid(d.ion.rigid, d.ion.n_rigid, go, gs);
      P.o_ion_grp = ipush(go.data(), (int)go.size());
      P.o_ion_gstart = ipush(gs.data(), (int)gs.size());
    }
    /* AMBER exclusions: 1-2 (bonds and rigid pairs), 1-3, 1-4 (compute_AMBER.cpp:256-278) */
    P.excl_words = (d.ion.n_atoms + 31) / 32;
    {
      std::vector<int> ex((size_t)d.ion.n_atoms * P.excl_words, 0);
      auto mark = [&](int i, int j) {
        ex[(size_t)i * P.excl_words + (j >> 5)] |= (int)(1u << (j & 31));
        ex[(size_t)j * P.excl_words + (i >> 5)] |= (int)(1u << (i & 31));
      };
      for (int b = 0; b < d.ion.n_bonds; b++) mark(d.ion.bonds[3 * b], d.ion.bonds[3 * b + 1]);
      for (int b = 0; b < d.ion.n_rigid; b++) mark(d.ion.rigid[3 * b], d.ion.rigid[3 * b + 1]);
      for (int b = 0; b < d.ion.n_angles; b++) mark(d.ion.angles[4 * b], d.ion.angles[4 * b + 2]);
      for (int b = 0; b < d.ion.n_dihedrals; b++) mark(d.ion.dihedrals[5 * b], d.ion.dihedrals[5 * b + 3]);
      P.o_excl = ipush(ex.data(), (int)ex.size());
    }
    P.o_gas_type = ipush(d.gas.type, d.gas.n_atoms);
    P.n_gas_bonds = d.gas.n_bonds;
    P.o_gas_bonds = ipush(d.gas.bonds, 3 * d.gas.n_bonds);
    P.n_gas_rigid = d.gas.n_rigid;
    P.o_gas_rigid = ipush(d.gas.rigid, 3 * d.gas.n_rigid);
    if (d.n_vapor > 0) {
      P.o_vap_type = ipush(d.vapor.type, d.vapor.n_atoms);
      P.n_vap_bonds = d.vapor.n_bonds;
      P.o_vap_bonds = ipush(d.vapor.bonds, 3 * d.vapor.n_bonds);
      P.n_vap_angles = d.vapor.n_angles;
      P.o_vap_angles = ipush(d.vapor.angles, 4 * d.vapor.n_angles);
      P.n_vap_dih = d.vapor.n_dihedrals;
      P.o_vap_dih = ipush(d.vapor.dihedrals, 5 * d.vapor.n_dihedrals);
      P.n_vap_rigid = d.vapor.n_rigid;
      P.o_vap_rigid = ipush(d.vapor.rigid, 3 * d.vapor.n_rigid);
      P.n_vap_colors = color_rigid(d.vapor.rigid, d.vapor.n_rigid, col);
      P.o_vap_color = ipush(col.data(), (int)col.size());
      std::vector<int> go, gs;
      P.n_vap_groups = group_rigid(d.vapor.rigid, d.vapor.n_rigid, go, gs);
      P.o_vap_grp = ipush(go.data(), (int)go.size());
      P.o_vap_gstart = ipush(gs.data(), (int)gs.size());
    } else {
      int zero = 0;
      P.o_vap_type = ipush(&zero, 1);
      P.o_vap_bonds = P.o_vap_angles = P.o_vap_dih = P.o_vap_rigid = P.o_vap_color = P.o_vap_type;
      P.o_vap_grp = P.o_vap_gstart = P.o_vap_type;
      P.n_vap_groups = 0;
    }
    P.o_dih_multi = ipush(d.dihedral_multi, d.n_dihedral_types);

    /* ---- double blob ---- */
    P.dblob_off = (long long)dblob.size();
    auto dpush = [&](const double* p, int n) {
      int o = (int)(dblob.size() - P.dblob_off);
      for (int i = 0; i < n; i++) dblob.push_back(p[i]);
      return o;
    };
    /* SHAKE constraint tables: d^2, 1/m_i, 1/m_j of each rigid pair */
    auto cons_table = [&](const mdn_topology& t) {
      std::vector<double> c(3 * (size_t)std::max(t.n_rigid, 1), 0.0);
      for (int k = 0; k < t.n_rigid; k++) {
        const double dk = d.bond_coeff[2 * t.rigid[3 * k + 2] + 1];
        c[3 * k] = dk * dk;
        c[3 * k + 1] = 1.0 / d.atom_mass[t.type[t.rigid[3 * k]]];
        c[3 * k + 2] = 1.0 / d.atom_mass[t.type[t.rigid[3 * k + 1]]];
      }
      return dpush(c.data(), (int)c.size());
    };
    P.d_ion_cons = cons_table(d.ion);
    P.d_gas_cons = cons_table(d.gas);
    P.d_vap_cons = d.n_vapor > 0 ? cons_table(d.vapor) : P.d_ion_cons;
    P.d_bond = dpush(d.bond_coeff, 2 * d.n_bond_types);
    P.d_angle = dpush(d.angle_coeff, 2 * d.n_angle_types);
    P.d_dih = dpush(d.dihedral_coeff, 15 * d.n_dihedral_types);
    {
      /* Variables::setCrossPotentials (src/initialization/setCrossPotential.cpp:4-23) */
      std::vector<double> A((size_t)nt * nt), B((size_t)nt * nt);
      for (int i = 0; i < nt; i++)
        for (int j = 0; j < nt; j++) {
          double epu = d.pair_eps ? d.pair_eps[(size_t)i * nt + j] : sqrt(d.atom_eps[i] * d.atom_eps[j]);
          double sigma = d.pair_sigma ? d.pair_sigma[(size_t)i * nt + j] : (d.atom_sigma[i] + d.atom_sigma[j]) * 0.5;
          A[(size_t)i * nt + j] = 48 * epu * pow(sigma, 12.0);
          B[(size_t)i * nt + j] = 24 * epu * pow(sigma, 6.0);
        }
      P.d_ljA = dpush(A.data(), nt * nt);
      P.d_ljB = dpush(B.data(), nt * nt);
      P.d_mass = dpush(d.atom_mass, nt);
      std::vector<double> c2(nt);
      for (int t = 0; t < nt; t++) c2[t] = P.coeff / d.atom_mass[t];
      P.d_c2 = dpush(c2.data(), nt);
    }
    P.d_ion_q = dpush(d.ion.charge, d.ion.n_atoms);
    P.d_gas_x = dpush(d.gas.x, 3 * d.gas.n_atoms);
    P.d_gas_q = dpush(d.gas.charge, d.gas.n_atoms);
    if (d.n_vapor > 0) {
      P.d_vap_x = dpush(d.vapor.x, 3 * d.vapor.n_atoms);
      P.d_vap_q = dpush(d.vapor.charge, d.vapor.n_atoms);
    } else {
      double z[3] = {0, 0, 0};
      P.d_vap_x = dpush(z, 3);
      P.d_vap_q = P.d_vap_x;
    }
    double msum = 0;
    for (int i = 0; i < d.ion.n_atoms; i++) msum += d.atom_mass[d.ion.type[i]];
    P.ion_msum = msum;

    /* ---- capacities ---- */
    const double V_sphere = 4.0 / 3.0 * M_PI * pow(d.r_inter + d.overlap, 3);
    const double V_box = d.box * d.box * d.box;
    const double frac = std::min(1.0, V_sphere / V_box);
    const double f = opt.capacity_factor;
    double eg = d.n_gas * frac;
    P.slab_cap = (int)std::min<double>(d.n_gas, ceil(eg * f + 6 * sqrt(eg) + 64));
    P.slab_cap = std::max(P.slab_cap, 1);
    /* in-domain vapor: binomial mean + 4 sigma (the core lives in shared memory,
     * 160 B per atom, so this capacity is kept tight; exceeding it raises
     * MDN_ST_CORE_OVERFLOW) */
    double ev = d.n_vapor * frac;
    P.vcap = (int)std::min<double>(d.n_vapor, ceil(ev * (f > 1.0 ? 1.0 + 0.2 * (f - 1.0) : 1.0) +
                                                   4 * sqrt(ev * (1 - frac)) + 8));
    P.vcap = std::max(P.vcap, 1);
    /* the core's 16-bit chunk sums are exact for up to 65,536 terms per
     * atom: one per near molecule at most, plus pair tiles and bonded terms */
    P.near_cap = std::min(P.slab_cap, 64511);
    double rion = 0;
    {
      double c[3] = {0, 0, 0};
      for (int i = 0; i < d.ion.n_atoms; i++)
        for (int k = 0; k < 3; k++) c[k] += d.ion.x[3 * i + k] / d.ion.n_atoms;
      for (int i = 0; i < d.ion.n_atoms; i++) {
        double r2 = 0;
        for (int k = 0; k < 3; k++) r2 += (d.ion.x[3 * i + k] - c[k]) * (d.ion.x[3 * i + k] - c[k]);
        rion = std::max(rion, sqrt(r2));
      }
    }
    const double rlist = d.cutoff + d.margin;
    const double dens = d.n_gas / V_box;
    double near_est = dens * 4.0 / 3.0 * M_PI * pow(rion + rlist + 15.0, 3);
    double gil_est = (near_est * f * 2 + 6 * sqrt(near_est) + 64) * d.ion.n_atoms;
    P.gil_cap = (int)std::min<double>(std::min<double>((double)P.slab_cap * d.ion.n_atoms, gil_est), 2.0e9);
    double gv_est = dens * 4.0 / 3.0 * M_PI * pow(rlist + 5.0, 3) * P.vcap;
    P.gvl_cap = (int)std::min<double>((double)P.slab_cap * P.vcap, gv_est * f * 2 + 64 * P.vcap + 256);
    P.gil_cap = std::max(P.gil_cap, 16);
    P.gvl_cap = std::max(P.gvl_cap, 16);
    /* gas-gas (both directions): partners within the list radius at the
     * in-domain density, 1.5 x plus a margin per molecule */
    P.ggl_cap = 0;
    if (d.interactions & MDN_I_GG) {
      const double partners = eg / V_sphere * 4.0 / 3.0 * M_PI * pow(rlist, 3);
      const double est = (double)P.slab_cap * (partners * f * 1.5 + 6 * sqrt(partners) + 16);
      P.ggl_cap = (int)std::max(16.0, std::min(std::min((double)P.slab_cap * P.slab_cap, est), 2.0e9));
    }

    /* ---- pool offsets ---- */
    P.ion_off = (long long)ion_tot;
    ion_tot += d.ion.n_atoms;
    P.mol_off = (long long)mol_tot;
    mol_tot += 1 + d.n_gas + d.n_vapor;
    P.slab_off = (long long)slab_atoms;
    slab_atoms += (size_t)2 * P.slab_cap * P.a_g;
    P.slab_moff = (long long)slab_mols;
    slab_mols += (size_t)2 * P.slab_cap;
    P.vslab_off = (long long)vslab_atoms;
    vslab_atoms += (size_t)2 * P.vcap * P.a_v;
    P.vslab_moff = (long long)vslab_mols;
    vslab_mols += (size_t)2 * P.vcap;
    P.near_off = (long long)near_tot;
    near_tot += P.near_cap;
    P.gil_off = (long long)gil_tot;
    gil_tot += P.gil_cap;
    P.gvl_off = (long long)gvl_tot;
    gvl_tot += P.gvl_cap;
    P.ggl_off = (long long)ggl_tot;
    ggl_tot += P.ggl_cap;
    P.work = eg * P.a_g + 0.05 * pow(d.ion.n_atoms + P.vcap * P.a_v * 0.5, 2) + near_est * d.ion.n_atoms;

    h->nt_cap = std::max(h->nt_cap, nt);
    h->excl_cap = std::max(h->excl_cap, d.ion.n_atoms * P.excl_words);
    h->nc_cap = std::max(h->nc_cap, d.ion.n_atoms + P.vcap * P.a_v);

    RepDyn& D = h->D0[r];
    memset(&D, 0, sizeof D);
    D.loop_pair = 0;
    D.loop_update = 0;
    D.margin_length = d.margin;
    D.nvt_mode = d.nvt_mode;
    D.nvt_T = d.nvt_temperature;
  }
  h->h_iblob = iblob;
  h->smem = smem_bytes(h->nc_cap, h->nt_cap, h->excl_cap);
  int max_optin = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->dev);
  if (h->smem + 4096 > (size_t)max_optin) {
    size_t need = h->smem;
    int nc = h->nc_cap;
    delete h;
    return fail(MDN_ERR_CAPACITY, "a core of %d atoms needs %zu B of shared memory (device limit %d)",
                nc, need, max_optin);
  }
  h->n_ion_tot = ion_tot;
  h->n_mol_tot = mol_tot;
  h->n_slab_atoms = slab_atoms;
  h->n_slab_mols = slab_mols;
  h->n_vslab_atoms = vslab_atoms;
  h->n_vslab_mols = vslab_mols;
  h->n_near = near_tot;
  h->n_gil = gil_tot;
  h->n_gvl = gvl_tot;
  h->n_ggl = ggl_tot;

  /* job order: largest estimated work first */
  h->order.resize(R);
  for (int r = 0; r < R; r++) h->order[r] = r;
  std::stable_sort(h->order.begin(), h->order.end(), [&](int a, int b) { return h->P[a].work > h->P[b].work; });
  /* automatic cluster size: the smallest power of two that lets the largest
   * replica finish within the time of an even share of the SMs
   * (num_sms * W_max / W_total CTAs), at most 8 */
  {
    double wmax = 0, wsum = 0;
    for (int r = 0; r < R; r++) {
      wmax = std::max(wmax, h->P[r].work);
      wsum += h->P[r].work;
    }
    const double want = wsum > 0 ? h->num_sms * wmax / wsum : 1.0;
    int c = 1;
    while (c < 8 && c < want) c *= 2;
    h->auto_cluster = c;
  }

#define ALLOC(ptr, count)                                                          \
  do {                                                                             \
    cudaError_t e_ = cudaMalloc((void**)&(ptr), sizeof(*(ptr)) * std::max<size_t>(1, (count))); \
    if (e_ != cudaSuccess) {                                                       \
      free_all(h);                                                                 \
      delete h;                                                                    \
      return fail(MDN_ERR_CUDA, "cudaMalloc(%s): %s", #ptr, cudaGetErrorString(e_)); \
    }                                                                              \
  } while (0)
  ALLOC(h->dP, R);
  ALLOC(h->dD, R);
  ALLOC(h->d_iblob, iblob.size());
  ALLOC(h->d_dblob, dblob.size());
  ALLOC(h->ion_x, 3 * ion_tot);
  ALLOC(h->ion_v, 3 * ion_tot);
  ALLOC(h->ion_f, 3 * ion_tot);
  ALLOC(h->mol_x, 3 * mol_tot);
  ALLOC(h->mol_v, 3 * mol_tot);
  ALLOC(h->region, mol_tot);
  ALLOC(h->slot, mol_tot);
  ALLOC(h->slab_x, 3 * slab_atoms);
  ALLOC(h->slab_v, 3 * slab_atoms);
  ALLOC(h->slab_f, 3 * slab_atoms);
  ALLOC(h->slab_mol, slab_mols);
  ALLOC(h->vslab_x, 3 * vslab_atoms);
  ALLOC(h->vslab_v, 3 * vslab_atoms);
  ALLOC(h->vslab_f, 3 * vslab_atoms);
  ALLOC(h->vslab_w, vslab_atoms);
  ALLOC(h->vslab_mol, vslab_mols);
  ALLOC(h->near_list, near_tot);
  ALLOC(h->near_gi, slab_mols);
  ALLOC(h->near_gv, slab_mols);
  ALLOC(h->gil_n, slab_mols);
  ALLOC(h->gvl_n, slab_mols);
  ALLOC(h->gil, gil_tot);
  ALLOC(h->gvl, gvl_tot);
  if (ggl_tot > 0) {
    ALLOC(h->ggl_start, slab_mols);
    ALLOC(h->ggl_n, slab_mols);
    ALLOC(h->ggl, ggl_tot);
    ALLOC(h->slab_fgg, 3 * slab_atoms);
    ALLOC(h->slab_ins, slab_mols);
  }
  ALLOC(h->energy, 8 * (size_t)R);
  ALLOC(h->events, (size_t)h->ev_cap);
  ALLOC(h->n_events, 1);
  ALLOC(h->status, R);
  ALLOC(h->job_order, R);
  ALLOC(h->job_counter, 1);
  ALLOC(h->job_order2, R);
  ALLOC(h->job_counter2, 1);
  ALLOC(h->d_ctl_mode, R);
  ALLOC(h->d_ctl_T, R);
#undef ALLOC
  int rc = MDN_OK;
  auto ck = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == MDN_OK) rc = fail(MDN_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  };
  ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
  ck(cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking), "stream");
  ck(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming), "event");
  ck(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming), "event");
  ck(cudaEventCreate(&h->ev0), "event");
  ck(cudaEventCreate(&h->ev1), "event");
  for (auto kern : {mdn_advance, mdn_advance_fp64, mdn_advance_gg, mdn_advance_gg_fp64}) {
    ck(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->smem), "smem attr");
    ck(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1), "cluster attr");
  }
  ck(cudaMemcpy(h->dP, h->P.data(), sizeof(RepParams) * R, cudaMemcpyHostToDevice), "params");
  ck(cudaMemcpy(h->dD, h->D0.data(), sizeof(RepDyn) * R, cudaMemcpyHostToDevice), "dyn");
  ck(cudaMemcpy(h->d_iblob, iblob.data(), sizeof(int) * iblob.size(), cudaMemcpyHostToDevice), "iblob");
  ck(cudaMemcpy(h->d_dblob, dblob.data(), sizeof(double) * dblob.size(), cudaMemcpyHostToDevice), "dblob");
  ck(cudaMemset(h->region, 0, mol_tot), "region");
  for (int r = 0; r < R && rc == MDN_OK; r++) {
    unsigned char one = 1; /* molecule 0, the ion, is always in the domain (readIonFile.cpp:177) */
    ck(cudaMemcpy(h->region + h->P[r].mol_off, &one, 1, cudaMemcpyHostToDevice), "region");
  }
  ck(cudaMemset(h->slot, 0xff, sizeof(int) * mol_tot), "slot");
  ck(cudaMemset(h->ion_f, 0, sizeof(double) * 3 * ion_tot), "ion_f");
  ck(cudaMemset(h->energy, 0, sizeof(long long) * 8 * R), "energy");
  ck(cudaMemset(h->n_events, 0, sizeof(int)), "events");
  ck(cudaMemset(h->status, 0, sizeof(int) * R), "status");
  ck(cudaMemset(h->near_gi, 0xff, sizeof(int) * slab_mols), "near_gi");
  if (h->slab_ins) ck(cudaMemset(h->slab_ins, 0xff, sizeof(int) * slab_mols), "slab_ins");
  if (h->ggl_n) ck(cudaMemset(h->ggl_n, 0, sizeof(int) * slab_mols), "ggl_n");
  h->ctl_mode.resize(R);
  h->ctl_T.resize(R);
  for (int r = 0; r < R; r++) {
    h->ctl_mode[r] = descs[r].nvt_mode;
    h->ctl_T[r] = descs[r].nvt_temperature;
  }
  ck(cudaMemcpy(h->d_ctl_mode, h->ctl_mode.data(), sizeof(int) * R, cudaMemcpyHostToDevice), "ctl");
  ck(cudaMemcpy(h->d_ctl_T, h->ctl_T.data(), sizeof(double) * R, cudaMemcpyHostToDevice), "ctl");
  /* ion atoms and molecule centres */
  {
    std::vector<double> ix(3 * ion_tot), iv(3 * ion_tot), mx(3 * mol_tot, 0.0), mv(3 * mol_tot, 0.0);
    for (int r = 0; r < R; r++) {
      const mdn_replica_desc& d = descs[r];
      const RepParams& P = h->P[r];
      for (int i = 0; i < 3 * d.ion.n_atoms; i++) {
        ix[3 * P.ion_off + i] = d.ion.x[i];
        iv[3 * P.ion_off + i] = d.ion_v ? d.ion_v[i] : 0.0;
      }
      for (int q = 0; q < d.n_gas; q++)
        for (int k = 0; k < 3; k++) {
          mx[3 * (P.mol_off + 1 + q) + k] = d.gas_x[3 * q + k];
          mv[3 * (P.mol_off + 1 + q) + k] = d.gas_v[3 * q + k];
        }
      for (int q = 0; q < d.n_vapor; q++)
        for (int k = 0; k < 3; k++) {
          mx[3 * (P.mol_off + 1 + d.n_gas + q) + k] = d.vapor_x[3 * q + k];
          mv[3 * (P.mol_off + 1 + d.n_gas + q) + k] = d.vapor_v[3 * q + k];
        }
    }
    ck(cudaMemcpy(h->ion_x, ix.data(), sizeof(double) * ix.size(), cudaMemcpyHostToDevice), "ion_x");
    ck(cudaMemcpy(h->ion_v, iv.data(), sizeof(double) * iv.size(), cudaMemcpyHostToDevice), "ion_v");
    ck(cudaMemcpy(h->mol_x, mx.data(), sizeof(double) * mx.size(), cudaMemcpyHostToDevice), "mol_x");
    ck(cudaMemcpy(h->mol_v, mv.data(), sizeof(double) * mv.size(), cudaMemcpyHostToDevice), "mol_v");
  }
  if (rc != MDN_OK) {
    free_all(h);
    delete h;
    return rc;
  }
  /* MD::MD's initial make_pair (src/initialization/md.cpp:34), classified
   * against the ion centre entry as MD::MD leaves it: (0, 0, 0) */
  launch(h, MDN_MODE_MAKE_PAIR, 0, 0, 0, nullptr, &rc, 1);
  if (rc == MDN_OK) rc = sync_check(h);
  if (rc != MDN_OK) {
    free_all(h);
    delete h;
    return rc;
  }
  /* the allocation-free snapshot's per-device set-up (snapshot_noalloc.cu):
   * its fixed array and kernels are loaded here, not by its first call */
  mdn_noalloc_setup(h->dev);
  *out = h;
  return MDN_OK;
}

void mdn_destroy(mdn_handle* h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  free_all(h);
  delete h;
}

static int check_status(mdn_handle* h) {
  std::vector<int> st(h->R);
  cudaError_t e = cudaMemcpy(st.data(), h->status, sizeof(int) * h->R, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(MDN_ERR_CUDA, "status read: %s", cudaGetErrorString(e));
  for (int r = 0; r < h->R; r++)
    if (st[r] & MDN_ST_FATAL) return fail(MDN_ERR_REPLICA, "replica %d raised status 0x%x", r, st[r]);
  return MDN_OK;
}

int mdn_step(mdn_handle* h, long long n_steps, int energy_mode) {
  if (!h || n_steps < 0) return fail(MDN_ERR_ARG, "bad arguments");
  cudaSetDevice(h->dev);
  CK(cudaMemsetAsync(h->energy, 0, sizeof(long long) * 8 * h->R, h->stream));
  CK(cudaEventRecord(h->ev0, h->stream));
  long long launches = 0;
  long long spl = h->opt.steps_per_launch > 0 ? h->opt.steps_per_launch : n_steps;
  long long done = 0;
  int rc = MDN_OK;
  while (done < n_steps) {
    long long n = std::min(spl, n_steps - done);
    int em = 0;
    if (energy_mode == 2) em = 2;
    if (energy_mode == 1 && done + n == n_steps) em = 1;
    launches += launch(h, MDN_MODE_STEP, n, em, 0, nullptr, &rc);
    if (rc != MDN_OK) return rc;
    done += n;
  }
  CK(cudaEventRecord(h->ev1, h->stream));
  if ((rc = sync_check(h)) != MDN_OK) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last_ms = ms;
  h->last_launches = launches;
  return check_status(h);
}

int mdn_make_pair(mdn_handle* h) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  cudaSetDevice(h->dev);
  int rc;
  launch(h, MDN_MODE_MAKE_PAIR, 0, 0, 0, nullptr, &rc);
  if (rc) return rc;
  if ((rc = sync_check(h))) return rc;
  return check_status(h);
}

int mdn_compute_forces(mdn_handle* h, unsigned term_mask) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  cudaSetDevice(h->dev);
  CK(cudaMemsetAsync(h->energy, 0, sizeof(long long) * 8 * h->R, h->stream));
  int rc;
  launch(h, MDN_MODE_FORCES, 0, 1, term_mask, nullptr, &rc);
  if (rc) return rc;
  if ((rc = sync_check(h))) return rc;
  return check_status(h);
}

int mdn_recenter(mdn_handle* h, int compat) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  cudaSetDevice(h->dev);
  for (int r = 0; r < h->R; r++) {
    const RepParams& P = h->P[r];
    RepDyn D;
    CK(cudaMemcpy(&D, h->dD + r, sizeof D, cudaMemcpyDeviceToHost));
    if (compat) {
      /* src/run.cpp:42-53 subtracts position[0] from every entry while that
       * entry itself is being zeroed: only the ion centre moves */
      double z[3] = {0, 0, 0};
      CK(cudaMemcpy(h->mol_x + 3 * P.mol_off, z, sizeof z, cudaMemcpyHostToDevice));
      for (int k = 0; k < 3; k++) D.ion_com[k] = 0;
      CK(cudaMemcpy(h->dD + r, &D, sizeof D, cudaMemcpyHostToDevice));
    } else {
      double c[3] = {D.ion_com[0], D.ion_com[1], D.ion_com[2]};
      auto shift = [&](double* base, size_t first, size_t count) -> int {
        std::vector<double> v(3 * count);
        CK(cudaMemcpy(v.data(), base + 3 * first, sizeof(double) * v.size(), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < count; i++)
          for (int k = 0; k < 3; k++) v[3 * i + k] -= c[k];
        CK(cudaMemcpy(base + 3 * first, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice));
        return MDN_OK;
      };
      int rc;
      if ((rc = shift(h->ion_x, P.ion_off, P.n_ion))) return rc;
      if ((rc = shift(h->mol_x, P.mol_off, 1 + P.n_gas + P.n_vap))) return rc;
      if ((rc = shift(h->slab_x, P.slab_off, (size_t)2 * P.slab_cap * P.a_g))) return rc;
      if ((rc = shift(h->vslab_x, P.vslab_off, (size_t)2 * P.vcap * P.a_v))) return rc;
      for (int k = 0; k < 3; k++) D.ion_com[k] = 0;
      CK(cudaMemcpy(h->dD + r, &D, sizeof D, cudaMemcpyHostToDevice));
    }
  }
  /* MD::run calls make_pair right after the shift, with the ion centre entry
   * as the shift left it */
  int rc;
  launch(h, MDN_MODE_MAKE_PAIR, 0, 0, 0, nullptr, &rc, 1);
  if (rc) return rc;
  if ((rc = sync_check(h))) return rc;
  return check_status(h);
}

int mdn_set_nvt(mdn_handle* h, int replica, int mode, double T) {
  if (!h || replica >= h->R) return fail(MDN_ERR_ARG, "bad replica");
  if (mode < MDN_NVT_OFF || mode > MDN_NVT_NH) return fail(MDN_ERR_ARG, "bad thermostat mode");
  for (int r = 0; r < h->R; r++) {
    if (replica >= 0 && r != replica) continue;
    h->ctl_mode[r] = mode;
    h->ctl_T[r] = T;
  }
  CK(cudaMemcpy(h->d_ctl_mode, h->ctl_mode.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_ctl_T, h->ctl_T.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice));
  return MDN_OK;
}

int mdn_set_nvt_batch(mdn_handle* h, const int* mode, const double* T) {
  if (!h || !mode || !T) return fail(MDN_ERR_ARG, "bad arguments");
  for (int r = 0; r < h->R; r++) {
    if (mode[r] < MDN_NVT_OFF || mode[r] > MDN_NVT_NH) return fail(MDN_ERR_ARG, "bad thermostat mode");
    h->ctl_mode[r] = mode[r];
    h->ctl_T[r] = T[r];
  }
  cudaSetDevice(h->dev);
  CK(cudaMemcpyAsync(h->d_ctl_mode, mode, sizeof(int) * h->R, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_ctl_T, T, sizeof(double) * h->R, cudaMemcpyHostToDevice, h->stream));
  return MDN_OK;
}

int mdn_energies(mdn_handle* h, double* U) {
  if (!h || !U) return fail(MDN_ERR_ARG, "bad arguments");
  std::vector<long long> e(8 * h->R);
  CK(cudaMemcpy(e.data(), h->energy, sizeof(long long) * e.size(), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < e.size(); i++) U[i] = (double)e[i] * MDN_EFIX_INV;
  return MDN_OK;
}

int mdn_get_status(mdn_handle* h, int* status) {
  if (!h || !status) return fail(MDN_ERR_ARG, "bad arguments");
  CK(cudaMemcpy(status, h->status, sizeof(int) * h->R, cudaMemcpyDeviceToHost));
  return MDN_OK;
}

int mdn_clear_status(mdn_handle* h) {
  if (!h) return fail(MDN_ERR_ARG, "bad arguments");
  CK(cudaMemset(h->status, 0, sizeof(int) * h->R));
  return MDN_OK;
}

int mdn_replica_info_get(mdn_handle* h, int r, mdn_replica_info* info) {
  if (!h || r < 0 || r >= h->R || !info) return fail(MDN_ERR_ARG, "bad arguments");
  RepDyn D;
  int st = 0;
  CK(cudaMemcpy(&D, h->dD + r, sizeof D, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&st, h->status + r, sizeof(int), cudaMemcpyDeviceToHost));
  const RepParams& P = h->P[r];
  memset(info, 0, sizeof *info);
  info->n_ion = P.n_ion;
  info->gas_atoms = P.a_g;
  info->vapor_atoms = P.n_vap > 0 ? P.a_v : 0;
  info->n_gas = P.n_gas;
  info->n_vapor = P.n_vap;
  info->n_gas_in = D.n_gas_in;
  info->n_vapor_in = D.n_vap_in;
  info->loop_pair = D.loop_pair;
  info->loop_update = D.loop_update;
  info->n_rebuilds = D.n_rebuilds;
  info->step = D.step;
  info->status = st;
  info->gi_pairs = D.gi_count;
  info->gv_pairs = D.gv_count;
  info->gg_pairs = D.gg_count;
  return MDN_OK;
}

int mdn_download_state(mdn_handle* h, int r, mdn_state* s) {
  if (!h || r < 0 || r >= h->R || !s) return fail(MDN_ERR_ARG, "bad arguments");
  cudaSetDevice(h->dev);
  const RepParams& P = h->P[r];
  RepDyn D;
  CK(cudaMemcpy(&D, h->dD + r, sizeof D, cudaMemcpyDeviceToHost));
  const size_t ni = P.n_ion, nm = 1 + P.n_gas + P.n_vap;
  if (s->ion_x) CK(cudaMemcpy(s->ion_x, h->ion_x + 3 * P.ion_off, 24 * ni, cudaMemcpyDeviceToHost));
  if (s->ion_v) CK(cudaMemcpy(s->ion_v, h->ion_v + 3 * P.ion_off, 24 * ni, cudaMemcpyDeviceToHost));
  if (s->ion_f) CK(cudaMemcpy(s->ion_f, h->ion_f + 3 * P.ion_off, 24 * ni, cudaMemcpyDeviceToHost));
  if (s->mol_x) CK(cudaMemcpy(s->mol_x, h->mol_x + 3 * P.mol_off, 24 * nm, cudaMemcpyDeviceToHost));
  if (s->mol_v) CK(cudaMemcpy(s->mol_v, h->mol_v + 3 * P.mol_off, 24 * nm, cudaMemcpyDeviceToHost));
  if (s->region) CK(cudaMemcpy(s->region, h->region + P.mol_off, nm, cudaMemcpyDeviceToHost));
  /* gas slab -> rows of the in-domain molecules */
  {
    const int G = D.n_gas_in, ag = P.a_g, par = D.parity;
    std::vector<int> mol(G);
    std::vector<double> x(3 * (size_t)G * ag), v(x.size()), f(x.size());
    if (G > 0) {
      const size_t a0 = (size_t)P.slab_off + (size_t)par * P.slab_cap * ag;
      CK(cudaMemcpy(mol.data(), h->slab_mol + P.slab_moff + (size_t)par * P.slab_cap, sizeof(int) * G, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(x.data(), h->slab_x + 3 * a0, 8 * x.size(), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(v.data(), h->slab_v + 3 * a0, 8 * v.size(), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(f.data(), h->slab_f + 3 * a0, 8 * f.size(), cudaMemcpyDeviceToHost));
    }
    for (int s_ = 0; s_ < G; s_++) {
      size_t dst = 3 * (size_t)mol[s_] * ag, src = 3 * (size_t)s_ * ag;
      for (int q = 0; q < 3 * ag; q++) {
        if (s->gas_ax) s->gas_ax[dst + q] = x[src + q];
        if (s->gas_av) s->gas_av[dst + q] = v[src + q];
        if (s->gas_af) s->gas_af[dst + q] = f[src + q];
      }
    }
  }
  if (P.n_vap > 0) {
    const int V = D.n_vap_in, av = P.a_v, par = D.parity;
    std::vector<int> mol(V);
    std::vector<double> x(3 * (size_t)V * av), v(x.size()), f(x.size());
    std::vector<float> w((size_t)V * av);
    if (V > 0) {
      const size_t a0 = (size_t)P.vslab_off + (size_t)par * P.vcap * av;
      CK(cudaMemcpy(mol.data(), h->vslab_mol + P.vslab_moff + (size_t)par * P.vcap, sizeof(int) * V, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(x.data(), h->vslab_x + 3 * a0, 8 * x.size(), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(v.data(), h->vslab_v + 3 * a0, 8 * v.size(), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(f.data(), h->vslab_f + 3 * a0, 8 * f.size(), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(w.data(), h->vslab_w + a0, 4 * w.size(), cudaMemcpyDeviceToHost));
    }
    for (int s_ = 0; s_ < V; s_++) {
      size_t dst = 3 * (size_t)mol[s_] * av, src = 3 * (size_t)s_ * av;
      for (int q = 0; q < 3 * av; q++) {
        if (s->vap_ax) s->vap_ax[dst + q] = x[src + q];
        if (s->vap_av) s->vap_av[dst + q] = v[src + q];
        if (s->vap_af) s->vap_af[dst + q] = f[src + q];
      }
      if (s->vap_w)
        for (int at = 0; at < av; at++) s->vap_w[(size_t)mol[s_] * av + at] = w[(size_t)s_ * av + at];
    }
  }
  s->loop_pair = D.loop_pair;
  s->loop_update = D.loop_update;
  s->zeta = D.zeta;
  s->margin_length = D.margin_length;
  return MDN_OK;
}

int mdn_upload_state(mdn_handle* h, int r, const mdn_state* s) {
  if (!h || r < 0 || r >= h->R || !s) return fail(MDN_ERR_ARG, "bad arguments");
  if (!s->ion_x || !s->ion_v || !s->ion_f || !s->mol_x || !s->mol_v || !s->region || !s->gas_ax || !s->gas_av ||
      !s->gas_af)
    return fail(MDN_ERR_ARG, "upload needs every ion, molecule and gas array");
  cudaSetDevice(h->dev);
  const RepParams& P = h->P[r];
  RepDyn D;
  CK(cudaMemcpy(&D, h->dD + r, sizeof D, cudaMemcpyDeviceToHost));
  const size_t ni = P.n_ion, nm = 1 + P.n_gas + P.n_vap;
  CK(cudaMemcpy(h->ion_x + 3 * P.ion_off, s->ion_x, 24 * ni, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->ion_v + 3 * P.ion_off, s->ion_v, 24 * ni, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->ion_f + 3 * P.ion_off, s->ion_f, 24 * ni, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->mol_x + 3 * P.mol_off, s->mol_x, 24 * nm, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->mol_v + 3 * P.mol_off, s->mol_v, 24 * nm, cudaMemcpyHostToDevice));
  std::vector<unsigned char> reg(s->region, s->region + nm);
  reg[0] = 1;
  std::vector<int> slot(nm, -1);
  /* gas slab (parity 0), ascending molecule index */
  const int ag = P.a_g, av = P.a_v;
  std::vector<int> gmol_;
  for (int q = 0; q < P.n_gas; q++)
    if (reg[1 + q]) gmol_.push_back(q);
  if ((int)gmol_.size() > P.slab_cap)
    return fail(MDN_ERR_CAPACITY, "replica %d: %zu in-domain gas molecules exceed the slab (%d)", r, gmol_.size(), P.slab_cap);
  std::vector<int> vmol_;
  for (int q = 0; q < P.n_vap; q++)
    if (reg[1 + P.n_gas + q]) vmol_.push_back(q);
  if ((int)vmol_.size() > P.vcap || P.n_ion + (int)vmol_.size() * av > h->nc_cap)
    return fail(MDN_ERR_CAPACITY, "replica %d: %zu in-domain vapor molecules exceed the core", r, vmol_.size());
  if (!vmol_.empty() && (!s->vap_ax || !s->vap_av || !s->vap_af))
    return fail(MDN_ERR_ARG, "upload needs the vapor atom arrays");
  {
    const int G = (int)gmol_.size();
    std::vector<double> x(3 * (size_t)G * ag), v(x.size()), f(x.size());
    for (int i = 0; i < G; i++) {
      slot[1 + gmol_[i]] = i;
      size_t src = 3 * (size_t)gmol_[i] * ag, dst = 3 * (size_t)i * ag;
      for (int q = 0; q < 3 * ag; q++) {
        x[dst + q] = s->gas_ax[src + q];
        v[dst + q] = s->gas_av[src + q];
        f[dst + q] = s->gas_af[src + q];
      }
    }
    if (G > 0) {
      const size_t a0 = (size_t)P.slab_off;
      CK(cudaMemcpy(h->slab_mol + P.slab_moff, gmol_.data(), sizeof(int) * G, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(h->slab_x + 3 * a0, x.data(), 8 * x.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(h->slab_v + 3 * a0, v.data(), 8 * v.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(h->slab_f + 3 * a0, f.data(), 8 * f.size(), cudaMemcpyHostToDevice));
      if (h->slab_ins) CK(cudaMemset(h->slab_ins + P.slab_moff, 0xff, sizeof(int) * G));
    }
    D.n_gas_in = G;
  }
  {
    const int V = (int)vmol_.size();
    std::vector<double> x(3 * (size_t)V * av), v(x.size()), f(x.size());
    std::vector<float> w((size_t)V * av, 0.0f);
    for (int i = 0; i < V; i++) {
      slot[1 + P.n_gas + vmol_[i]] = i;
      size_t src = 3 * (size_t)vmol_[i] * av, dst = 3 * (size_t)i * av;
      for (int q = 0; q < 3 * av; q++) {
        x[dst + q] = s->vap_ax[src + q];
        v[dst + q] = s->vap_av[src + q];
        f[dst + q] = s->vap_af[src + q];
      }
      if (s->vap_w)
        for (int at = 0; at < av; at++) w[(size_t)i * av + at] = (float)s->vap_w[(size_t)vmol_[i] * av + at];
    }
    if (V > 0) {
      const size_t a0 = (size_t)P.vslab_off;
      CK(cudaMemcpy(h->vslab_mol + P.vslab_moff, vmol_.data(), sizeof(int) * V, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(h->vslab_x + 3 * a0, x.data(), 8 * x.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(h->vslab_v + 3 * a0, v.data(), 8 * v.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(h->vslab_f + 3 * a0, f.data(), 8 * f.size(), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(h->vslab_w + a0, w.data(), 4 * w.size(), cudaMemcpyHostToDevice));
    }
    D.n_vap_in = V;
  }
  CK(cudaMemcpy(h->region + P.mol_off, reg.data(), nm, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->slot + P.mol_off, slot.data(), sizeof(int) * nm, cudaMemcpyHostToDevice));
  D.parity = 0;
  D.loop_pair = s->loop_pair;
  D.loop_update = s->loop_update;
  D.zeta = s->zeta;
  if (s->margin_length > 0) D.margin_length = s->margin_length;
  for (int k = 0; k < 3; k++) {
    D.ion_com[k] = s->mol_x[k];
    D.ion_com[3 + k] = s->mol_v[k];
  }
  CK(cudaMemcpy(h->dD + r, &D, sizeof D, cudaMemcpyHostToDevice));
  /* lists from the given centres (no classification) */
  std::vector<int> one(1, r);
  int rc;
  launch(h, MDN_MODE_RELIST, 0, 0, 0, &one, &rc);
  if (rc) return rc;
  return sync_check(h);
}

int mdn_pair_list(mdn_handle* h, int r, int kind, int* pairs, int capacity, int* count) {
  if (!h || r < 0 || r >= h->R || !count) return fail(MDN_ERR_ARG, "bad arguments");
  const RepParams& P = h->P[r];
  RepDyn D;
  CK(cudaMemcpy(&D, h->dD + r, sizeof D, cudaMemcpyDeviceToHost));
  if (kind == 2) {
    /* gas-gas: (molecule, partner molecule) once per unordered pair, the
     * lower slab slot first (ascending molecule indices, as gas_in) */
    int c = 0;
    const int G = D.n_gas_in, par = D.parity;
    if (P.ggl_cap > 0 && G > 0) {
      const size_t m0 = P.slab_moff + (size_t)par * P.slab_cap;
      std::vector<int> mol(G), st(G), n(G);
      CK(cudaMemcpy(mol.data(), h->slab_mol + m0, sizeof(int) * G, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(st.data(), h->ggl_start + m0, sizeof(int) * G, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(n.data(), h->ggl_n + m0, sizeof(int) * G, cudaMemcpyDeviceToHost));
      long long tot = 0;
      for (int i = 0; i < G; i++) tot = std::max<long long>(tot, (long long)st[i] + n[i]);
      std::vector<int> ent(std::max<long long>(tot, 1));
      if (tot > 0) CK(cudaMemcpy(ent.data(), h->ggl + P.ggl_off, sizeof(int) * tot, cudaMemcpyDeviceToHost));
      for (int s_ = 0; s_ < G; s_++)
        for (int q = 0; q < n[s_]; q++) {
          const int t = ent[st[s_] + q];
          if (t <= s_) continue;
          if (c < capacity && pairs) {
            pairs[2 * c] = mol[s_];
            pairs[2 * c + 1] = mol[t];
          }
          c++;
        }
    }
    *count = c;
    return MDN_OK;
  }
  const int G = D.n_gas_in, par = D.parity;
  std::vector<int> mol(G), st(G), vm(D.n_vap_in);
  std::vector<unsigned short> n(G);
  if (G > 0) {
    const size_t m0 = P.slab_moff + (size_t)par * P.slab_cap;
    CK(cudaMemcpy(mol.data(), h->slab_mol + m0, sizeof(int) * G, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(st.data(), (kind == 0 ? h->near_gi : h->near_gv) + m0, sizeof(int) * G, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(n.data(), (kind == 0 ? h->gil_n : h->gvl_n) + m0, sizeof(unsigned short) * G, cudaMemcpyDeviceToHost));
  }
  if (kind == 1 && D.n_vap_in > 0)
    CK(cudaMemcpy(vm.data(), h->vslab_mol + P.vslab_moff + (size_t)par * P.vcap, sizeof(int) * D.n_vap_in, cudaMemcpyDeviceToHost));
  const int tot = kind == 0 ? D.gi_count : D.gv_count;
  std::vector<unsigned short> ent(std::max(tot, 1));
  if (tot > 0)
    CK(cudaMemcpy(ent.data(), (kind == 0 ? h->gil + P.gil_off : h->gvl + P.gvl_off), sizeof(unsigned short) * tot, cudaMemcpyDeviceToHost));
  int c = 0;
  for (int s_ = 0; s_ < G; s_++) {
    if (st[s_] < 0) continue;
    for (int q = 0; q < n[s_]; q++) {
      int partner = ent[st[s_] + q];
      if (kind == 1) partner = vm[partner];
      if (c < capacity && pairs) {
        pairs[2 * c] = mol[s_];
        pairs[2 * c + 1] = partner;
      }
      c++;
    }
  }
  *count = c;
  return MDN_OK;
}

int mdn_in_domain(mdn_handle* h, int r, int capacity, int* count, int* type, double* x, double* v) {
  if (!h || r < 0 || r >= h->R || !count) return fail(MDN_ERR_ARG, "bad arguments");
  /* assembled from the state download, in molecule order (ion, gas, vapor) */
  const RepParams& P = h->P[r];
  const size_t nm = 1 + P.n_gas + P.n_vap;
  std::vector<double> ix(3 * P.n_ion), iv(3 * P.n_ion), mx(3 * nm), mv(3 * nm);
  std::vector<unsigned char> reg(nm);
  std::vector<double> gx(3 * (size_t)P.n_gas * P.a_g), gv(gx.size());
  std::vector<double> vx(3 * (size_t)P.n_vap * P.a_v), vv(vx.size());
  mdn_state s;
  memset(&s, 0, sizeof s);
  s.ion_x = ix.data(); s.ion_v = iv.data(); s.mol_x = mx.data(); s.mol_v = mv.data(); s.region = reg.data();
  s.gas_ax = gx.data(); s.gas_av = gv.data(); s.vap_ax = vx.data(); s.vap_av = vv.data();
  int rc = mdn_download_state(h, r, &s);
  if (rc) return rc;
  const int* IB = h->h_iblob.data() + P.iblob_off;
  int c = 0;
  auto put = [&](int t, const double* px, const double* pv) {
    if (c < capacity) {
      if (type) type[c] = t;
      for (int k = 0; k < 3; k++) {
        if (x) x[3 * c + k] = px[k];
        if (v) v[3 * c + k] = pv[k];
      }
    }
    c++;
  };
  for (int i = 0; i < P.n_ion; i++) put(IB[P.o_ion_type + i], &ix[3 * i], &iv[3 * i]);
  for (int q = 0; q < P.n_gas; q++)
    if (reg[1 + q])
      for (int a = 0; a < P.a_g; a++)
        put(IB[P.o_gas_type + a], &gx[3 * ((size_t)q * P.a_g + a)], &gv[3 * ((size_t)q * P.a_g + a)]);
  for (int q = 0; q < P.n_vap; q++)
    if (reg[1 + P.n_gas + q])
      for (int a = 0; a < P.a_v; a++)
        put(IB[P.o_vap_type + a], &vx[3 * ((size_t)q * P.a_v + a)], &vv[3 * ((size_t)q * P.a_v + a)]);
  *count = c;
  return MDN_OK;
}

int mdn_snapshot(mdn_handle* h, long long* offset, long long capacity, int* type, double* x, double* v,
                 double* U) {
  if (!h || !offset) return fail(MDN_ERR_ARG, "bad arguments");
  cudaSetDevice(h->dev);
  if (!h->snap_off) {
    long long cap = 0;
    for (int r = 0; r < h->R; r++) {
      const RepParams& P = h->P[r];
      cap += P.n_ion + (long long)P.slab_cap * P.a_g + (P.n_vap > 0 ? (long long)P.vcap * P.a_v : 0);
    }
    h->snap_cap = cap;
    CK(cudaMalloc((void**)&h->snap_off, sizeof(long long) * (h->R + 1)));
    CK(cudaMalloc((void**)&h->snap_type, sizeof(int) * std::max<long long>(cap, 1)));
    CK(cudaMalloc((void**)&h->snap_x, 3 * sizeof(double) * std::max<long long>(cap, 1)));
    CK(cudaMalloc((void**)&h->snap_v, 3 * sizeof(double) * std::max<long long>(cap, 1)));
  }
  const cudaError_t le = mdn_snapshot_device(h->dP, h->dD, h->d_iblob, h->R, h->ion_x, h->ion_v, h->slab_x,
                                             h->slab_v, h->vslab_x, h->vslab_v, h->snap_off, h->snap_type, h->snap_x,
                                             h->snap_v, h->snap_cap, h->stream);
  if (le != cudaSuccess) return fail(MDN_ERR_CUDA, "snapshot kernels: %s", cudaGetErrorString(le));
  CK(cudaMemcpyAsync(offset, h->snap_off, sizeof(long long) * (h->R + 1), cudaMemcpyDeviceToHost, h->stream));
  std::vector<long long> e(U ? 8 * h->R : 0);
  if (U) CK(cudaMemcpyAsync(e.data(), h->energy, sizeof(long long) * e.size(), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (U)
    for (size_t i = 0; i < e.size(); i++) U[i] = (double)e[i] * MDN_EFIX_INV;
  const long long total = offset[h->R];
  if (total > capacity) return fail(MDN_ERR_CAPACITY, "snapshot needs %lld rows, buffer holds %lld", total, capacity);
  if (total > 0) {
    if (type) CK(cudaMemcpyAsync(type, h->snap_type, sizeof(int) * total, cudaMemcpyDeviceToHost, h->stream));
    if (x) CK(cudaMemcpyAsync(x, h->snap_x, 3 * sizeof(double) * total, cudaMemcpyDeviceToHost, h->stream));
    if (v) CK(cudaMemcpyAsync(v, h->snap_v, 3 * sizeof(double) * total, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return MDN_OK;
}

int mdn_host_alloc(size_t bytes, void** ptr) {
  if (!ptr) return fail(MDN_ERR_ARG, "null pointer");
  *ptr = nullptr;
  CK(cudaHostAlloc(ptr, std::max<size_t>(bytes, 1), cudaHostAllocDefault));
  return MDN_OK;
}

int mdn_host_free(void* ptr) {
  if (ptr) CK(cudaFreeHost(ptr));
  return MDN_OK;
}

int mdn_events(mdn_handle* h, mdn_event* ev, int capacity, int* count) {
  if (!h || !count) return fail(MDN_ERR_ARG, "bad arguments");
  int n = 0;
  CK(cudaMemcpy(&n, h->n_events, sizeof(int), cudaMemcpyDeviceToHost));
  n = std::min(n, h->ev_cap);
  std::vector<DevEvent> e(std::max(n, 1));
  if (n > 0) CK(cudaMemcpy(e.data(), h->events, sizeof(DevEvent) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n && i < capacity && ev; i++) {
    ev[i].replica = e[i].replica;
    ev[i].molecule = e[i].molecule;
    ev[i].kind = e[i].kind;
    ev[i].pad = 0;
    ev[i].step = e[i].step;
    for (int k = 0; k < 3; k++) {
      ev[i].dx[k] = e[i].dx[k];
      ev[i].dv[k] = e[i].dv[k];
    }
  }
  *count = n;
  CK(cudaMemset(h->n_events, 0, sizeof(int)));
  return MDN_OK;
}

int mdn_kinetic(mdn_handle* h, double* out) {
  if (!h || !out) return fail(MDN_ERR_ARG, "bad arguments");
  for (int r = 0; r < h->R; r++) {
    const RepParams& P = h->P[r];
    const size_t nm = 1 + P.n_gas + P.n_vap;
    std::vector<double> mv(3 * nm), iv(3 * P.n_ion);
    std::vector<int> it(P.n_ion);
    CK(cudaMemcpy(mv.data(), h->mol_v + 3 * P.mol_off, 24 * nm, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(iv.data(), h->ion_v + 3 * P.ion_off, 24 * P.n_ion, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(it.data(), h->d_iblob + P.iblob_off + P.o_ion_type, sizeof(int) * P.n_ion, cudaMemcpyDeviceToHost));
    std::vector<double> mass(P.n_types);
    CK(cudaMemcpy(mass.data(), h->d_dblob + P.dblob_off + P.d_mass, sizeof(double) * P.n_types, cudaMemcpyDeviceToHost));
    /* Observer::computeProps (src/output/observer.cpp:5-36) */
    double Kg = 0, Kv = 0, Ki = 0;
    for (int q = 0; q < P.n_gas; q++) {
      const double* v = &mv[3 * (1 + q)];
      Kg += v[0] * v[0] * P.gas_com_mass;
      Kg += v[1] * v[1] * P.gas_com_mass;
      Kg += v[2] * v[2] * P.gas_com_mass;
    }
    Kg *= (0.5 * real_to_kcalmol);
    for (int q = 0; q < P.n_vap; q++) {
      const double* v = &mv[3 * (1 + P.n_gas + q)];
      Kv += v[0] * v[0] * P.vap_com_mass;
      Kv += v[1] * v[1] * P.vap_com_mass;
      Kv += v[2] * v[2] * P.vap_com_mass;
    }
    Kv *= 0.5 * real_to_kcalmol;
    for (int i = 0; i < P.n_ion; i++) {
      double m = mass[it[i]];
      Ki += iv[3 * i] * iv[3 * i] * m;
      Ki += iv[3 * i + 1] * iv[3 * i + 1] * m;
      Ki += iv[3 * i + 2] * iv[3 * i + 2] * m;
    }
    Ki *= 0.5 * real_to_kcalmol;
    out[4 * r + 0] = Ki;
    out[4 * r + 1] = Kg;
    out[4 * r + 2] = Kv;
    out[4 * r + 3] = Ki / double(P.n_ion) * ((1 / kb_real) / 1.5);
  }
  return MDN_OK;
}

int mdn_last_timing(mdn_handle* h, double* ms, long long* launches) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  if (ms) *ms = h->last_ms;
  if (launches) *launches = h->last_launches;
  return MDN_OK;
}

int mdn_profile(mdn_handle* h, int enable, long long* out) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  cudaSetDevice(h->dev);
  if (!h->d_prof) {
    CK(cudaMalloc((void**)&h->d_prof, sizeof(long long) * MDN_PROF_N * h->R));
    CK(cudaMemset(h->d_prof, 0, sizeof(long long) * MDN_PROF_N * h->R));
  }
  if (out) {
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(out, h->d_prof, sizeof(long long) * MDN_PROF_N * h->R, cudaMemcpyDeviceToHost));
  }
  if (enable && !h->prof_on) CK(cudaMemset(h->d_prof, 0, sizeof(long long) * MDN_PROF_N * h->R));
  h->prof_on = enable != 0;
  return MDN_OK;
}

int mdn_get_launch(mdn_handle* h, int* cluster_size, int* threads, int* steps_per_launch) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  if (cluster_size) *cluster_size = h->opt.cluster_size > 0 ? h->opt.cluster_size : h->auto_cluster;
  if (threads) *threads = h->opt.threads;
  if (steps_per_launch) *steps_per_launch = h->opt.steps_per_launch;
  return MDN_OK;
}

/* One block of n_steps with the cycle accounting on; the job order becomes
 * the replicas by measured cycles, largest first (the estimate from the
 * sizes misses terms such as the gas-vapor lists of a dense gas around many
 * vapor molecules).  The accounting is returned to the state it was in. */
static int order_by_measured(mdn_handle* h, long long n_steps, int* status) {
  const bool was_on = h->prof_on;
  int rc = mdn_profile(h, 0, nullptr);
  if (rc) return rc;
  std::vector<long long> keep;
  if (was_on) {
    keep.resize((size_t)MDN_PROF_N * h->R);
    if ((rc = mdn_profile(h, 1, keep.data()))) return rc;
  }
  CK(cudaMemset(h->d_prof, 0, sizeof(long long) * MDN_PROF_N * h->R));
  h->prof_on = true;
  rc = mdn_step(h, n_steps, 0);
  if (rc == MDN_ERR_REPLICA) *status = rc;
  else if (rc != MDN_OK) return rc;
  std::vector<long long> prof((size_t)MDN_PROF_N * h->R);
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(prof.data(), h->d_prof, sizeof(long long) * prof.size(), cudaMemcpyDeviceToHost));
  std::stable_sort(h->order.begin(), h->order.end(), [&](int a, int b) {
    return prof[(size_t)a * MDN_PROF_N + MDN_PROF_TOTAL] > prof[(size_t)b * MDN_PROF_N + MDN_PROF_TOTAL];
  });
  /* the accounting as it was */
  if (was_on) CK(cudaMemcpy(h->d_prof, keep.data(), sizeof(long long) * keep.size(), cudaMemcpyHostToDevice));
  else CK(cudaMemset(h->d_prof, 0, sizeof(long long) * MDN_PROF_N * h->R));
  h->prof_on = was_on;
  return MDN_OK;
}

int mdn_tune_launch(mdn_handle* h, long long n_steps, int* best) {
  if (!h || n_steps <= 0) return fail(MDN_ERR_ARG, "bad arguments");
  int best_c = 0, status = MDN_OK;
  float best_ms = 0;
  for (int c = 1; c <= 8; c *= 2) {
    h->opt.cluster_size = c;
    int rc = mdn_step(h, n_steps, 0);
    if (rc == MDN_ERR_REPLICA) status = rc;
    else if (rc != MDN_OK) return rc;
    if (best_c == 0 || h->last_ms < best_ms) {
      best_c = c;
      best_ms = h->last_ms;
    }
  }
  h->opt.cluster_size = best_c;
  const int save_n = h->split_n, save_c = h->split_cluster;
  if (save_n == 0) {
    /* the replicas that bound the launch are the ones that take longest:
     * order the jobs by measured cycles, then time the launch with that
     * order */
    int rc = order_by_measured(h, n_steps, &status);
    if (rc) return rc;
    rc = mdn_step(h, n_steps, 0);
    if (rc == MDN_ERR_REPLICA) status = rc;
    else if (rc != MDN_OK) return rc;
    best_ms = h->last_ms;
  }
  /* then the k slowest replicas on larger clusters (2 or 4 times, at most 8
   * CTAs), one each, in a concurrent launch beside the rest */
  int best_n = 0, best_sc = 0;
  if (save_n == 0)
    for (int sc = 2 * best_c; sc <= 8; sc *= 2)
      for (int k = 2; k <= 16 && k < h->R; k *= 2) {
        if (k * sc + best_c > h->num_sms) break;
        h->split_n = k;
        h->split_cluster = sc;
        int rc = mdn_step(h, n_steps, 0);
        if (rc == MDN_ERR_REPLICA) status = rc;
        else if (rc != MDN_OK) {
          h->split_n = save_n;
          h->split_cluster = save_c;
          return rc;
        }
        if (h->last_ms < best_ms) {
          best_n = k;
          best_sc = sc;
          best_ms = h->last_ms;
        }
      }
  if (save_n == 0) {
    h->split_n = best_n;
    h->split_cluster = best_n ? best_sc : 0;
  }
  if (best) *best = best_c;
  return status;
}

int mdn_set_split(mdn_handle* h, int n_largest, int cluster_size) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  if (n_largest < 0 || (n_largest > 0 && (cluster_size < 1 || cluster_size > 8)))
    return fail(MDN_ERR_ARG, "split: n_largest >= 0 and cluster size 1..8");
  h->split_n = n_largest;
  h->split_cluster = n_largest ? cluster_size : 0;
  return MDN_OK;
}

int mdn_get_split(mdn_handle* h, int* n_largest, int* cluster_size) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  if (n_largest) *n_largest = h->split_n;
  if (cluster_size) *cluster_size = h->split_cluster;
  return MDN_OK;
}

int mdn_set_launch(mdn_handle* h, int cluster_size, int threads, int steps_per_launch) {
  if (!h) return fail(MDN_ERR_ARG, "null handle");
  if (cluster_size > 0) {
    if (cluster_size > 8) return fail(MDN_ERR_ARG, "cluster size must be 1..8");
    h->opt.cluster_size = cluster_size;
  }
  if (threads > 0) {
    if (threads % 32 || threads > 512) return fail(MDN_ERR_ARG, "threads must be a multiple of 32 <= 512");
    h->opt.threads = threads;
  }
  if (steps_per_launch >= 0) h->opt.steps_per_launch = steps_per_launch;
  return MDN_OK;
}

}  // extern "C"
