/*
 * advance.cu -- the persistent step kernel of the engine (sm_100a).
 *
 * One launch advances a batch of replicas by n steps.  Thread-block clusters
 * of C CTAs (C = the launch's cluster size, 1..8) pull replicas from a work
 * queue, largest first, and keep a replica on-chip for all n steps:
 *
 *   - the "core" -- the ion (seed) and the in-domain vapor molecules, at most
 *     a few hundred to ~1000 atoms -- lives in shared memory, replicated in
 *     every CTA of the cluster.  All CTAs integrate it identically; its forces
 *     are int64 fixed-point partial sums that the cluster adds over DSMEM, so
 *     every copy receives the same total and the copies never diverge;
 *   - the in-domain gas molecules (up to ~20,000 atoms) live in the gas slab in
 *     global memory (L2-resident while the replica is being stepped) and are
 *     split evenly over the cluster's CTAs;
 *   - gas-gas interactions are absent from the reference's configurations, so
 *     a gas molecule interacts only with the core: molecules whose gas-ion /
 *     gas-vapor lists are empty ("far") are advanced by one thread in a single
 *     pass (kick, drift, intramolecular force, kick); "near" molecules are
 *     handled by one thread each too, walking the molecule's lists (about one
 *     entry per molecule), with shared-memory fixed-point atomics for the
 *     reaction on the core.
 *
 * Each step follows MD::verlet (src/verlet.cpp:20-39) exactly:
 *   kick (MD::velocity_calculation), [MD::velocity_scaling], drift with
 *   optional SHAKE (MD::update_position / updatePositionSHAKE), ion centre and
 *   taper weights, [MD::nosehoover_zeta], MD::check_pairlist -> make_pair on
 *   the device, forces of every enabled Potential, kick, [MD::nosehoover_ion].
 * The rebuild (MD::make_pair, src/pairList/pairlist.cpp:16-49) -- free flight,
 * updateInCenters, in/out classification with periodic wrap and
 * Maxwell-Boltzmann resampling, insertion with a random rotation, pair lists,
 * loop_update -- runs inside the same launch, decided per replica.
 *
 * Precision: FP64 for integration, SHAKE, centres, weights, the rebuild and
 * the bonded terms; FP32 for the pair terms (LJ, Coulomb, Born-Mayer-Huggins)
 * on coordinates taken relative to the ion centre; every sum with more than one
 * writer is an int64 fixed-point sum (units 2^-40 kcal/mol/A for forces,
 * 2^-36 kcal/mol for energies), so results do not depend on the launch shape.
 */
#include <cooperative_groups.h>

#include <type_traits>

#include "device_util.cuh"
#include "mdn_types.h"

namespace cg = cooperative_groups;
using namespace mdn;

namespace {

/* pointers into the dynamic shared memory of a CTA */
struct Core {
  double* x;        /* [3*nc] positions                        */
  double* v;        /* [3*nc] velocities                       */
  double* f;        /* [3*nc] force of the last evaluation     */
  long long* acc;   /* [3*nc] this CTA's fixed-point force sums */
  unsigned* chunk;  /* [9*nc] the same sums in 32-bit chunks (acc_add) */
  float4* pos;      /* [nc] (x - ion centre, charge), FP32     */
  float* w;         /* [nc] taper weight                       */
  int* type;        /* [nc] atom type                          */
  int* mol;         /* [nc] -1 for ion atoms, else vapor slot  */
  unsigned* excl;   /* AMBER exclusions, n_ion rows            */
  float* ljA;       /* [nt*nt] 48 eps s^12                     */
  float* ljB;       /* [nt*nt] 24 eps s^6                      */
  double* c2;       /* [nt] 0.5*dt*4.184e-4 / mass             */
  int* vcolor;      /* scratch                                 */
};

struct Ctx {
  const KArgs* a;
  RepParams* P;
  RepDyn* D;
  Core c;
  int r;            /* replica                          */
  int rank, C;      /* cluster rank and size            */
  int n_core;       /* atoms in the core                */
  int* iscr;        /* >= 64 ints of scratch            */
  int* cand;        /* [MDN_INSERT_MAX_VAPOR + 1] entering vapor molecules, count last */
  double* trial;    /* [3*MDN_MAX_VAP_ATOMS] trial atoms */
  double* dscr;     /* >= 64 doubles of scratch         */
  const int* ib;    /* int blob of the replica          */
  const double* db; /* double blob of the replica       */
};

__device__ __forceinline__ size_t gatom(const RepParams* P, int parity, int s, int a) {
  return (size_t)P->slab_off + ((size_t)parity * P->slab_cap + s) * P->a_g + a;
}
__device__ __forceinline__ size_t gmol(const RepParams* P, int parity, int s) {
  return (size_t)P->slab_moff + (size_t)parity * P->slab_cap + s;
}
__device__ __forceinline__ size_t vatom(const RepParams* P, int parity, int s, int a) {
  return (size_t)P->vslab_off + ((size_t)parity * P->vcap + s) * P->a_v + a;
}
__device__ __forceinline__ size_t vmol(const RepParams* P, int parity, int s) {
  return (size_t)P->vslab_moff + (size_t)parity * P->vcap + s;
}

/* per-phase SM cycles of the current job (thread 0 times phases that end in a
 * block barrier); flushed to KArgs::prof at the end of the job */
__shared__ long long s_prof[MDN_PROF_N];
__shared__ long long s_prof_t0;
__device__ __forceinline__ void prof_start(const Ctx& x) {
  if (x.a->prof && threadIdx.x == 0) s_prof_t0 = clock64();
}
__device__ __forceinline__ void prof_end(const Ctx& x, int phase) {
  if (x.a->prof && threadIdx.x == 0) s_prof[phase] += clock64() - s_prof_t0;
}

__device__ __forceinline__ void set_status(const Ctx& x, int bit) {
  atomicOr(&x.a->status[x.r], bit);
}

/* ------------------------------------------------------------------------- */
/* core load / store                                                          */
/* ------------------------------------------------------------------------- */
__device__ __forceinline__ void load_ion(Ctx& x) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  const int ni = P->n_ion;
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    size_t g = (size_t)P->ion_off + i;
    for (int k = 0; k < 3; k++) {
      x.c.x[3 * i + k] = a->ion_x[3 * g + k];
      x.c.v[3 * i + k] = a->ion_v[3 * g + k];
      x.c.f[3 * i + k] = a->ion_f[3 * g + k];
    }
    x.c.type[i] = x.ib[P->o_ion_type + i];
    x.c.mol[i] = -1;
    x.c.w[i] = 1.0f;
  }
}

/* the vapor part of the core, from the vapor slab of the current parity */
__device__ __forceinline__ void load_vapor(Ctx& x) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  const int ni = P->n_ion, av = P->a_v, nv = x.D->n_vap_in, par = x.D->parity;
  x.n_core = ni + nv * av;
  for (int t = threadIdx.x; t < nv * av; t += blockDim.x) {
    int s = t / av, at = t - s * av;
    size_t g = vatom(P, par, s, at);
    int i = ni + t;
    for (int k = 0; k < 3; k++) {
      x.c.x[3 * i + k] = a->vslab_x[3 * g + k];
      x.c.v[3 * i + k] = a->vslab_v[3 * g + k];
      x.c.f[3 * i + k] = a->vslab_f[3 * g + k];
    }
    x.c.type[i] = x.ib[P->o_vap_type + at];
    x.c.mol[i] = s;
    x.c.w[i] = a->vslab_w[g];
  }
}

__device__ __forceinline__ void store_core(Ctx& x) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  if (x.rank != 0) return;
  const int ni = P->n_ion, av = P->a_v, nv = x.D->n_vap_in, par = x.D->parity;
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    size_t g = (size_t)P->ion_off + i;
    for (int k = 0; k < 3; k++) {
      a->ion_x[3 * g + k] = x.c.x[3 * i + k];
      a->ion_v[3 * g + k] = x.c.v[3 * i + k];
      a->ion_f[3 * g + k] = x.c.f[3 * i + k];
    }
  }
  for (int t = threadIdx.x; t < nv * av; t += blockDim.x) {
    int s = t / av, at = t - s * av;
    size_t g = vatom(P, par, s, at);
    int i = ni + t;
    for (int k = 0; k < 3; k++) {
      a->vslab_x[3 * g + k] = x.c.x[3 * i + k];
      a->vslab_v[3 * g + k] = x.c.v[3 * i + k];
      a->vslab_f[3 * g + k] = x.c.f[3 * i + k];
    }
    a->vslab_w[g] = x.c.w[i];
  }
}

/* ------------------------------------------------------------------------- */
/* integration of the core                                                    */
/* ------------------------------------------------------------------------- */
__device__ __forceinline__ void core_kick(Ctx& x) {
  for (int i = threadIdx.x; i < x.n_core; i += blockDim.x) {
    double c2 = x.c.c2[x.c.type[i]];
    for (int k = 0; k < 3; k++) x.c.v[3 * i + k] += x.c.f[3 * i + k] * c2;
  }
}

/* Observer::computeProps, ion part: Tion.  Warp 0, lane-strided sums then a
 * butterfly, so the result depends on the atom order only. */
__device__ __forceinline__ double ion_temperature(Ctx& x) {
  const RepParams* P = x.P;
  if (threadIdx.x < 32) {
    double K = 0;
    for (int i = threadIdx.x; i < P->n_ion; i += 32) {
      double m = x.db[P->d_mass + x.c.type[i]];
      K += x.c.v[3 * i] * x.c.v[3 * i] * m;
      K += x.c.v[3 * i + 1] * x.c.v[3 * i + 1] * m;
      K += x.c.v[3 * i + 2] * x.c.v[3 * i + 2] * m;
    }
    K = warp_sum_d(K);
    if (threadIdx.x == 0) {
      K *= 0.5 * P->real_to_kcalmol;
      x.dscr[40] = K / double(P->n_ion) * ((1.0 / P->kb_real) / 1.5);
    }
  }
  __syncthreads();
  double T = x.dscr[40];
  __syncthreads();
  return T;
}

/* one SHAKE correction with the constraint's table row c = (d^2, 1/m_i,
 * 1/m_j): the multiplier of shake_pair with one division */
__device__ __forceinline__ void shake_pair_c(double* Xi, double* Xj, const double* Ri, const double* Rj,
                                             const double* c) {
  double r0 = Ri[0] - Rj[0], r1 = Ri[1] - Rj[1], r2 = Ri[2] - Rj[2];
  double s0 = Xi[0] - Xj[0], s1 = Xi[1] - Xj[1], s2 = Xi[2] - Xj[2];
  double ss = s0 * s0 + s1 * s1 + s2 * s2;
  double dot = r0 * s0 + r1 * s1 + r2 * s2;
  if (dot < 1e-10) dot = 1e-10;
  double g = (c[0] - ss) / (2 * (c[1] + c[2]) * dot);
  double gi = g * c[1], gj = g * c[2];
  Xi[0] += r0 * gi; Xi[1] += r1 * gi; Xi[2] += r2 * gi;
  Xj[0] -= r0 * gj; Xj[1] -= r1 * gj; Xj[2] -= r2 * gj;
}

/* (|s|^2 - d^2)^2 of one constraint; the sweeps stop when every residual is
 * <= 1e-20 A^4 (src/shake.cpp:51-90), and a NaN residual counts as not
 * converged, so a sweep that diverged runs into the cap and is reported */
__device__ __forceinline__ double shake_res_c(const double* Xi, const double* Xj, const double* c) {
  double s0 = Xi[0] - Xj[0], s1 = Xi[1] - Xj[1], s2 = Xi[2] - Xj[2];
  double dr = s0 * s0 + s1 * s1 + s2 * s2 - c[0];
  return dr * dr;
}

/* Newton's method on one group of at most three constraints that share
 * atoms (M-SHAKE).  The positions move along the constraints' reference
 * bond vectors r_k exactly as in the sweeps (x_i += l_k r_k / m_i,
 * x_j -= l_k r_k / m_j), and the l_k solve |s_k|^2 = d_k^2 for the whole
 * group at once, so the result is the sweeps' fixed point; the equations
 * are quadratic in l, and a handful of steps reach it where the sweeps of a
 * rigid water take dozens.  For one constraint a step is the sweep's own
 * update.  ks: the group's constraint indices (n of them); ct: the
 * constraint table (d^2, 1/m_i, 1/m_j).  Returns true once every
 * (|s_k|^2 - d_k^2)^2 <= 1e-20 A^4, the sweeps' criterion; false after 50
 * steps or a singular system, and the caller sweeps from there. */
__device__ bool shake_group(double* X, const double* R, const int* rig, const double* ct, const int* ks, int n) {
  int I[3], J[3];
  double r[3][3], d2[3], ci[3], cj[3], w[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int c = ks[k < n ? k : 0];
    I[k] = rig[3 * c];
    J[k] = rig[3 * c + 1];
    d2[k] = ct[3 * c];
    ci[k] = ct[3 * c + 1];
    cj[k] = ct[3 * c + 2];
#pragma unroll
    for (int q = 0; q < 3; q++) r[k][q] = R[3 * I[k] + q] - R[3 * J[k] + q];
  }
  /* d s_k / d l_l = w_kl r_l; rows and columns past n: the identity */
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) {
      const double ai = I[k] == I[l] ? ci[l] : (I[k] == J[l] ? -cj[l] : 0.0);
      const double aj = J[k] == I[l] ? ci[l] : (J[k] == J[l] ? -cj[l] : 0.0);
      w[k][l] = (k < n && l < n) ? ai - aj : 0.0;
    }
  for (int it = 0; it < 50; it++) {
    double s[3][3], f[3];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
      for (int q = 0; q < 3; q++) s[k][q] = X[3 * I[k] + q] - X[3 * J[k] + q];
      const double dr = s[k][0] * s[k][0] + s[k][1] * s[k][1] + s[k][2] * s[k][2] - d2[k];
      f[k] = k < n ? dr : 0.0;
      if (k < n && !(dr * dr <= 1e-20)) ok = false;
    }
    if (ok) return true;
    double A[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++)
        A[k][l] = (k < n && l < n) ? 2.0 * (s[k][0] * r[l][0] + s[k][1] * r[l][1] + s[k][2] * r[l][2]) * w[k][l]
                                   : (k == l ? 1.0 : 0.0);
    /* A d = -f by Cramer's rule */
    const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    const double c01 = A[1][0] * A[2][2] - A[1][2] * A[2][0];
    const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    const double det = A[0][0] * c00 - A[0][1] * c01 + A[0][2] * c02;
    if (!(fabs(det) > 1e-300)) return false;
    const double inv = 1.0 / det;
    const double b0 = -f[0], b1 = -f[1], b2 = -f[2];
    const double D0 = (b0 * c00 - A[0][1] * (b1 * A[2][2] - A[1][2] * b2) + A[0][2] * (b1 * A[2][1] - A[1][1] * b2)) * inv;
    const double D1 = (A[0][0] * (b1 * A[2][2] - A[1][2] * b2) - b0 * c01 + A[0][2] * (A[1][0] * b2 - b1 * A[2][0])) * inv;
    const double D2 = (A[0][0] * (A[1][1] * b2 - b1 * A[2][1]) - A[0][1] * (A[1][0] * b2 - b1 * A[2][0]) + b0 * c02) * inv;
    const double Dl[3] = {D0, D1, D2};
#pragma unroll
    for (int l = 0; l < 3; l++) {
      if (l >= n) break;
#pragma unroll
      for (int q = 0; q < 3; q++) {
        X[3 * I[l] + q] += Dl[l] * ci[l] * r[l][q];
        X[3 * J[l] + q] -= Dl[l] * cj[l] * r[l][q];
      }
    }
  }
  return false;
}

template <int AG>
__device__ __forceinline__ void gas_integrate_t(Ctx& x, bool fused, bool eflag, int tid, int nthr);

__device__ __forceinline__ void gas_integrate(Ctx& x, bool fused, bool eflag, int tid, int nthr);

/* Drift of the core, its constraints, and the gas integration of the step.
 * The constraints and the gas are independent (the gas pass touches only
 * the gas slab), so they run side by side: warp 0 sweeps the ion's
 * constraints, the next warps take one vapor molecule per thread, and the
 * remaining warps integrate the gas molecules. */
__device__ __forceinline__ void core_drift_shake(Ctx& x, bool fused, bool eflag) {
  const RepParams* P = x.P;
  /* positions before the drift (the SHAKE reference vectors) live in the
   * 64-bit sum buffer: core_reduce overwrites it only after this step's
   * forces, and no CTA of the cluster reads it any more (core_reduce ends
   * with a cluster barrier) */
  double* const xold = (double*)x.c.acc;
  const bool sh = (P->interactions & MDN_I_SHAKE) != 0;
  const bool vcorr = !(P->quirks & MDN_Q_SHAKE_NO_VCORR);
  const double dt = P->dt;
  for (int i = threadIdx.x; i < x.n_core; i += blockDim.x) {
    for (int k = 0; k < 3; k++) {
      double xo = x.c.x[3 * i + k];
      xold[3 * i + k] = xo;
      x.c.x[3 * i + k] = xo + x.c.v[3 * i + k] * dt;
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const bool ion_sh = sh && P->n_ion_rigid > 0;
  const int nv = (sh && P->n_vap_rigid > 0) ? x.D->n_vap_in : 0;
  /* warps of the ion constraints, of the vapor molecules, then of the gas */
  const int w_ion = ion_sh ? 1 : 0;
  const int w_vap = nv > 0 ? min((nv + 31) >> 5, max(1, (nwarps - w_ion) / 2)) : 0;
  const int w_gas0 = min(w_ion + w_vap, nwarps - 1);
  if (ion_sh && warp == 0) {
    /* sweeps in colour order (a colour's constraints share no atom, so
     * the lanes may take them in any order) until every constraint holds
     * after a sweep */
    const int* rig = x.ib + P->o_ion_rigid;
    const int* col = x.ib + P->o_ion_color;
    /* the ion's groups (an atom and its constrained hydrogens) share no
     * atom: the lanes solve them independently */
    bool done = false;
    if (P->n_ion_groups > 0) {
      const int* grp = x.ib + P->o_ion_grp;
      const int* gst = x.ib + P->o_ion_gstart;
      bool ok = true;
      for (int g = lane; g < P->n_ion_groups; g += 32)
        ok = shake_group(x.c.x, xold, rig, x.db + P->d_ion_cons, grp + gst[g], gst[g + 1] - gst[g]) && ok;
      done = __all_sync(0xffffffffu, ok);
      __syncwarp();
    }
    int sweeps = 0;
    for (; !done;) {
      for (int c = 0; c < P->n_ion_colors; c++) {
        for (int k = lane; k < P->n_ion_rigid; k += 32) {
          if (col[k] != c) continue;
          int i = rig[3 * k], j = rig[3 * k + 1];
          shake_pair_c(x.c.x + 3 * i, x.c.x + 3 * j, xold + 3 * i, xold + 3 * j, x.db + P->d_ion_cons + 3 * k);
        }
        __syncwarp();
      }
      bool ok = true;
      for (int k = lane; k < P->n_ion_rigid; k += 32)
        if (!(shake_res_c(x.c.x + 3 * rig[3 * k], x.c.x + 3 * rig[3 * k + 1], x.db + P->d_ion_cons + 3 * k) <= 1e-20))
          ok = false;
      if (__all_sync(0xffffffffu, ok)) break;
      if (++sweeps >= MDN_SHAKE_MAX_SWEEPS) {
        if (lane == 0 && x.rank == 0) set_status(x, MDN_ST_SHAKE_NOCONV);
        break;
      }
    }
    if (vcorr)
      for (int i = lane; i < P->n_ion; i += 32)
        for (int k = 0; k < 3; k++) {
          /* displacement by the constraints = x - (xold + v*dt) */
          double xd = xold[3 * i + k] + x.c.v[3 * i + k] * dt;
          x.c.v[3 * i + k] += (x.c.x[3 * i + k] - xd) / dt;
        }
  } else if (nv > 0 && warp >= w_ion && warp < w_ion + w_vap) {
    /* vapor molecules: one thread each, in place in shared memory, sweeps
     * in colour order until every constraint holds after a sweep */
    const int av = P->a_v, nr = P->n_vap_rigid, nco = P->n_vap_colors;
    const int* rig = x.ib + P->o_vap_rigid;
    const int* col = x.ib + P->o_vap_color;
    const double* ct = x.db + P->d_vap_cons;
    for (int s = threadIdx.x - 32 * w_ion; s < nv; s += 32 * w_vap) {
      const int base = P->n_ion + s * av;
      double* X = x.c.x + 3 * base;
      const double* R = xold + 3 * base;
      bool conv = false;
      if (P->n_vap_groups > 0) {
        const int* grp = x.ib + P->o_vap_grp;
        const int* gst = x.ib + P->o_vap_gstart;
        conv = true;
        for (int g = 0; g < P->n_vap_groups; g++)
          conv = shake_group(X, R, rig, ct, grp + gst[g], gst[g + 1] - gst[g]) && conv;
      }
      for (int sweep = 0; sweep < MDN_SHAKE_MAX_SWEEPS && !conv; sweep++) {
        for (int c = 0; c < nco; c++)
          for (int k = 0; k < nr; k++) {
            if (col[k] != c) continue;
            const int i = rig[3 * k], j = rig[3 * k + 1];
            shake_pair_c(X + 3 * i, X + 3 * j, R + 3 * i, R + 3 * j, ct + 3 * k);
          }
        conv = true;
        for (int k = 0; k < nr; k++)
          if (!(shake_res_c(X + 3 * rig[3 * k], X + 3 * rig[3 * k + 1], ct + 3 * k) <= 1e-20)) conv = false;
      }
      if (!conv && x.rank == 0) set_status(x, MDN_ST_SHAKE_NOCONV);
      if (vcorr)
        for (int q = 0; q < 3 * av; q++) {
          /* displacement by the constraints = x - (xold + v*dt) */
          const double xd = R[q] + x.c.v[3 * base + q] * dt;
          x.c.v[3 * base + q] += (X[q] - xd) / dt;
        }
    }
  } else if (warp >= w_gas0) {
    gas_integrate(x, fused, eflag, threadIdx.x - 32 * w_gas0, blockDim.x - 32 * w_gas0);
  }
  __syncthreads();
}

/* ion centre: warp 0, lane-strided partial sums, butterfly, fixed order */
__device__ __forceinline__ void ion_centre(Ctx& x) {
  const RepParams* P = x.P;
  if (threadIdx.x < 32) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < P->n_ion; i += 32) {
      double m = x.db[P->d_mass + x.c.type[i]];
      for (int k = 0; k < 3; k++) {
        s[k] += x.c.x[3 * i + k] * m;
        s[3 + k] += x.c.v[3 * i + k] * m;
      }
    }
    for (int k = 0; k < 6; k++) s[k] = warp_sum_d(s[k]);
    if (threadIdx.x == 0) {
      double mInv = 1 / P->ion_msum;
      for (int k = 0; k < 6; k++) x.D->ion_com[k] = s[k] * mInv;
    }
  }
  __syncthreads();
}

/* the ion centre in the reference's own order (sequential sum), used where a
 * threshold decision depends on it (the in/out classification) */
__device__ __forceinline__ void ion_centre_exact(Ctx& x) {
  const RepParams* P = x.P;
  if (threadIdx.x == 0) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < P->n_ion; i++) {
      double m = x.db[P->d_mass + x.c.type[i]];
      for (int k = 0; k < 3; k++) {
        s[k] += x.c.x[3 * i + k] * m;
        s[3 + k] += x.c.v[3 * i + k] * m;
      }
    }
    double mInv = 1 / P->ion_msum;
    for (int k = 0; k < 6; k++) x.D->ion_com[k] = s[k] * mInv;
  }
  __syncthreads();
}

__device__ __forceinline__ double taper(const RepParams* P, const double* com, const double* xa) {
  double dx = xa[0] - com[0];
  double dy = xa[1] - com[1];
  double dz = xa[2] - com[2];
  double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 < P->ri2) return 1;
  if (r2 > P->RI2) return 0;
  double dr = (sqrt(r2) - P->rcenter);
  double C = cos(3.141592653589793 / P->overlap * 0.5 * dr);
  return C * C;
}

/* taper weights of the vapor atoms (when `weights`) and the FP32 coordinates
 * of the core relative to the ion centre.  A molecule inserted by the rebuild
 * of this step carries w < 0 and gets 0 for this step: MD::update_position
 * ran before the rebuild, while the molecule was still outside
 * (src/verlet.cpp:109-134), so the reference leaves its weights unset. */
__device__ __forceinline__ void core_weights_pos(Ctx& x, bool weights) {
  const RepParams* P = x.P;
  const double* com = x.D->ion_com;
  for (int i = threadIdx.x; i < x.n_core; i += blockDim.x) {
    if (i >= P->n_ion) {
      if (x.c.w[i] < 0.0f) x.c.w[i] = 0.0f;
      else if (weights) x.c.w[i] = (float)taper(P, com, x.c.x + 3 * i);
    }
    double q = i < P->n_ion ? x.db[P->d_ion_q + i] : x.db[P->d_vap_q + (i - P->n_ion) % P->a_v];
    x.c.pos[i] = make_float4((float)(x.c.x[3 * i] - com[0]), (float)(x.c.x[3 * i + 1] - com[1]),
                             (float)(x.c.x[3 * i + 2] - com[2]), (float)q);
  }
  __syncthreads();
}

/* ------------------------------------------------------------------------- */
/* bonded terms (FP64, the reference's expressions)                           */
/* ------------------------------------------------------------------------- */
struct BondOut {
  double f[4][3];
  double e;
};

__device__ __forceinline__ void bond_fd(const double* X, const double* co, int i, int j, BondOut& o) {
  double dx = X[3 * i] - X[3 * j];
  double dy = X[3 * i + 1] - X[3 * j + 1];
  double dz = X[3 * i + 2] - X[3 * j + 2];
  double rsq = (dx * dx + dy * dy + dz * dz);
  double r = sqrt(rsq);
  double dr = (r - co[1]);
  double rk = co[0] * dr;
  double fb = -2.0 * rk / r;
  o.f[0][0] = fb * dx; o.f[0][1] = fb * dy; o.f[0][2] = fb * dz;
  o.f[1][0] = -(fb * dx); o.f[1][1] = -(fb * dy); o.f[1][2] = -(fb * dz);
  o.e = rk * dr;
}

__device__ __forceinline__ void angle_fd(const double* X, const double* co, int i, int j, int k, BondOut& o) {
  double dx1 = X[3 * i] - X[3 * j];
  double dy1 = X[3 * i + 1] - X[3 * j + 1];
  double dz1 = X[3 * i + 2] - X[3 * j + 2];
  double rsq1 = (dx1 * dx1 + dy1 * dy1 + dz1 * dz1);
  double r1 = sqrt(rsq1);
  double dx2 = X[3 * k] - X[3 * j];
  double dy2 = X[3 * k + 1] - X[3 * j + 1];
  double dz2 = X[3 * k + 2] - X[3 * j + 2];
  double rsq2 = (dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
  double r2 = sqrt(rsq2);
  double C = dx1 * dx2 + dy1 * dy2 + dz1 * dz2;
  C /= r1 * r2;
  double Cs = 1 / (sqrt(1.0 - C * C));
  double dtheta = acos(C) - co[1];
  double tk = co[0] * dtheta;
  double a = -2.0 * tk * Cs;
  double a11 = a * C / rsq1;
  double a12 = -a / (r1 * r2);
  double a22 = a * C / rsq2;
  double f1[3] = {a11 * dx1 + a12 * dx2, a11 * dy1 + a12 * dy2, a11 * dz1 + a12 * dz2};
  double f3[3] = {a22 * dx2 + a12 * dx1, a22 * dy2 + a12 * dy1, a22 * dz2 + a12 * dz1};
  for (int q = 0; q < 3; q++) {
    o.f[0][q] = f1[q];
    o.f[1][q] = -(f1[q] + f3[q]);
    o.f[2][q] = f3[q];
  }
  o.e = tk * dtheta;
}

__device__ __forceinline__ void dihedral_fd(const double* X, const double* co, int multi, int i, int j, int k,
                                            int l, BondOut& o) {
  double vb1x = X[3 * i] - X[3 * j];
  double vb1y = X[3 * i + 1] - X[3 * j + 1];
  double vb1z = X[3 * i + 2] - X[3 * j + 2];
  double vb2x = X[3 * k] - X[3 * j];
  double vb2y = X[3 * k + 1] - X[3 * j + 1];
  double vb2z = X[3 * k + 2] - X[3 * j + 2];
  double vb2xm = -vb2x, vb2ym = -vb2y, vb2zm = -vb2z;
  double vb3x = X[3 * l] - X[3 * k];
  double vb3y = X[3 * l + 1] - X[3 * k + 1];
  double vb3z = X[3 * l + 2] - X[3 * k + 2];
  double ax = vb1y * vb2zm - vb1z * vb2ym;
  double ay = vb1z * vb2xm - vb1x * vb2zm;
  double az = vb1x * vb2ym - vb1y * vb2xm;
  double bx = vb3y * vb2zm - vb3z * vb2ym;
  double by = vb3z * vb2xm - vb3x * vb2zm;
  double bz = vb3x * vb2ym - vb3y * vb2xm;
  double rasq = ax * ax + ay * ay + az * az;
  double rbsq = bx * bx + by * by + bz * bz;
  double rgsq = vb2xm * vb2xm + vb2ym * vb2ym + vb2zm * vb2zm;
  double rg = sqrt(rgsq);
  double rginv = 0.0, ra2inv = 0.0, rb2inv = 0.0;
  if (rg > 0) rginv = 1.0 / rg;
  if (rasq > 0) ra2inv = 1.0 / rasq;
  if (rbsq > 0) rb2inv = 1.0 / rbsq;
  double rabinv = sqrt(ra2inv * rb2inv);
  double c = (ax * bx + ay * by + az * bz) * rabinv;
  double s = rg * rabinv * (ax * vb3x + ay * vb3y + az * vb3z);
  double df = 0.0, e = 0.0;
  for (int JJ = 0; JJ < multi; JJ++) {
    int J5 = JJ * 5;
    double p_ = 1.0, df1 = 0.0, ddf1 = 0.0;
    for (int loop = 0; loop < co[J5 + 1]; loop++) {
      ddf1 = p_ * c - df1 * s;
      df1 = p_ * s + df1 * c;
      p_ = ddf1;
    }
    p_ = p_ * co[J5 + 3] + df1 * co[J5 + 4];
    df1 = df1 * co[J5 + 3] - ddf1 * co[J5 + 4];
    df1 *= -co[J5 + 1];
    p_ += 1.0;
    if (co[1] == 0) { /* term 0's periodicity tested for every term (src/potential/compute_AMBER.cpp:199) */
      p_ = 1.0 + co[J5 + 3];
      df1 = 0.0;
    }
    df += (-co[J5] * df1);
    e += co[J5] * p_;
  }
  double fg = vb1x * vb2xm + vb1y * vb2ym + vb1z * vb2zm;
  double hg = vb3x * vb2xm + vb3y * vb2ym + vb3z * vb2zm;
  double fga = fg * ra2inv * rginv;
  double hgb = hg * rb2inv * rginv;
  double gaa = -ra2inv * rg;
  double gbb = rb2inv * rg;
  double dtf[3] = {gaa * ax, gaa * ay, gaa * az};
  double dtg[3] = {fga * ax - hgb * bx, fga * ay - hgb * by, fga * az - hgb * bz};
  double dth[3] = {gbb * bx, gbb * by, gbb * bz};
  for (int q = 0; q < 3; q++) {
    double s2 = df * dtg[q];
    double f1 = df * dtf[q];
    double f4 = df * dth[q];
    o.f[0][q] = f1;
    o.f[1][q] = s2 - f1;
    o.f[2][q] = -s2 - f4;
    o.f[3][q] = f4;
  }
  o.e = e;
}

/* ------------------------------------------------------------------------- */
/* FP32 pair terms                                                            */
/* ------------------------------------------------------------------------- */
/* LJ (+ Coulomb) force factor and energy, the reference's formulas:
 *   f = r^-6 (A r^-6 - B) r^-2 [+ qqrd2e qi qj r^-1 r^-2], times w
 *   U = r^-6 (A/12 r^-6 - B/6) [+ qqrd2e qi qj / r]  (unweighted)          */
__device__ __forceinline__ float lj_coul(float r2, float A, float B, float qq, bool coul, float* e) {
  float rinv = rsqrtf(r2);
  float r2inv = rinv * rinv;
  float r6inv = r2inv * r2inv * r2inv;
  float flj = r6inv * fmaf(A, r6inv, -B);
  float fc = coul ? qq * rinv : 0.0f;
  *e = fmaf(r6inv, fmaf(A * (1.0f / 12.0f), r6inv, -B * (1.0f / 6.0f)), fc);
  return (flj + fc) * r2inv;
}

/* pair energies in FP64 from FP64 coordinates, evaluated only on the steps
 * that request energies: sums of Coulomb terms of both signs cancel by orders
 * of magnitude, which FP32 coordinates cannot resolve */
__device__ __forceinline__ double r2d(const double* a, const double* b) {
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return dx * dx + dy * dy + dz * dz;
}
__device__ __forceinline__ double lj_coul_energy(double r2, double A, double B, double qq) {
  double r2inv = 1 / r2;
  double r6inv = r2inv * r2inv * r2inv;
  return r6inv * (A / 12.0 * r6inv - B / 6.0) + qq * sqrt(r2inv);
}

/* Born-Mayer-Huggins (Tosi-Fumi NaCl, src/potential/BMHFT/potentialBMHFT.hpp:21-39) */
__constant__ float kBorn[2][2][5] = {
    {{25.4435f * 3.1546f / 4.184f, 6.f * 101.1719f / 4.184f, 8.f * 48.1771f / 4.184f, 2.340f, 3.1546f},
     {20.3548f * 3.1546f / 4.184f, 6.f * 674.4793f / 4.184f, 8.f * 837.077f / 4.184f, 2.755f, 3.1546f}},
    {{20.3548f * 3.1546f / 4.184f, 6.f * 674.4793f / 4.184f, 8.f * 837.077f / 4.184f, 2.755f, 3.1546f},
     {15.2661f * 3.1546f / 4.184f, 6.f * 6985.6786f / 4.184f, 8.f * 14031.5785f / 4.184f, 3.170f, 3.1546f}}};

__device__ __forceinline__ double born_energy(double r2, int ti, int tj, double qq) {
  const float* c = kBorn[ti][tj];
  double r2inv = 1 / r2;
  double r6inv = r2inv * r2inv * r2inv;
  double r = sqrt(r2);
  double rexp = exp((double)c[4] * ((double)c[3] - r));
  return qq * sqrt(r2inv) + rexp * c[0] - (double)c[1] / 6.0 * r6inv - (double)c[2] / 8.0 * r6inv * r2inv;
}

__device__ __forceinline__ float born(float r2, int ti, int tj, float qq, float* e) {
  const float* c = kBorn[ti][tj];
  float rinv = rsqrtf(r2);
  float r = r2 * rinv;
  float r2inv = rinv * rinv;
  float r6inv = r2inv * r2inv * r2inv;
  float rexp = expf(c[4] * (c[3] - r));
  float f1 = c[4] * c[0] * r * rexp;
  float f2 = -c[1] * r6inv;
  float f3 = -c[2] * r6inv * r2inv;
  float fc = qq * rinv;
  *e = fc + rexp * c[0] - c[1] * (1.0f / 6.0f) * r6inv - c[2] * (1.0f / 8.0f) * r6inv * r2inv;
  return (f1 + f2 + f3 + fc) * r2inv;
}

/* FP64 forms of the pair terms (mdn_options.force_mode = 1), with the
 * reference's FP64 constants (src/potential/BMHFT/potentialBMHFT.hpp:21-39) */
__constant__ double kBornD[2][2][5] = {
    {{25.4435 * 3.1546 / 4.184, 6. * 101.1719 / 4.184, 8. * 48.1771 / 4.184, 2.340, 3.1546},
     {20.3548 * 3.1546 / 4.184, 6. * 674.4793 / 4.184, 8. * 837.077 / 4.184, 2.755, 3.1546}},
    {{20.3548 * 3.1546 / 4.184, 6. * 674.4793 / 4.184, 8. * 837.077 / 4.184, 2.755, 3.1546},
     {15.2661 * 3.1546 / 4.184, 6. * 6985.6786 / 4.184, 8. * 14031.5785 / 4.184, 3.170, 3.1546}}};

__device__ __forceinline__ double lj_coul_d(double r2, double A, double B, double qq, bool coul) {
  double r2inv = 1 / r2;
  double r6inv = r2inv * r2inv * r2inv;
  double f = r6inv * (A * r6inv - B);
  if (coul) f += qq * sqrt(r2inv);
  return f * r2inv;
}

__device__ __forceinline__ double born_d(double r2, int ti, int tj, double qq) {
  const double* c = kBornD[ti][tj];
  double r2inv = 1 / r2;
  double r6inv = r2inv * r2inv * r2inv;
  double r = sqrt(r2);
  double rexp = exp(c[4] * (c[3] - r));
  return (c[4] * c[0] * r * rexp - c[1] * r6inv - c[2] * r6inv * r2inv + qq * sqrt(r2inv)) * r2inv;
}

/* taper weight of core atom i in FP64: the float copy is exact at 0 and 1 */
__device__ __forceinline__ double weight_d(const Ctx& x, int i) {
  const float w = x.c.w[i];
  if (w == 0.0f || w == 1.0f) return (double)w;
  return taper(x.P, x.D->ion_com, x.c.x + 3 * i);
}

/* charge of core atom i */
__device__ __forceinline__ double charge_d(const Ctx& x, int i) {
  const RepParams* P = x.P;
  return i < P->n_ion ? x.db[P->d_ion_q + i] : x.db[P->d_vap_q + (i - P->n_ion) % P->a_v];
}

/* ------------------------------------------------------------------------- */
/* forces of the core (ion + vapor) among themselves, and the core kick        */
/* ------------------------------------------------------------------------- */
/* One term of the core force sums.  Each 64-bit fixed-point term
 * u = lo16 + 2^16 mid16 + 2^32 hi32 goes into three 32-bit sums (64-bit
 * shared-memory atomics measured far slower than 32-bit ones here).  The two 16-bit
 * sums are exact for up to 65,536 terms per atom and evaluation (one per
 * near gas molecule, whose list holds at most 64,511, plus at most one per
 * pair tile and per bonded term); the high sum only matters modulo 2^32.
 * core_reduce folds the three into the 64-bit sum exactly, so the result
 * does not depend on the order of the adds. */
__device__ __forceinline__ void acc_add(Ctx& x, int i, const long long* f3) {
  unsigned* A = x.c.chunk + 9 * i;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const unsigned long long u = (unsigned long long)f3[k];
    atomicAdd(&A[3 * k], (unsigned)(u & 0xFFFFull));
    atomicAdd(&A[3 * k + 1], (unsigned)((u >> 16) & 0xFFFFull));
    atomicAdd(&A[3 * k + 2], (unsigned)(u >> 32));
  }
}

__device__ __forceinline__ void energy_add(Ctx& x, int bucket, long long e) {
  if (e != 0) atomicAdd((unsigned long long*)&x.a->energy[8 * x.r + bucket], (unsigned long long)e);
}

__device__ __forceinline__ bool term_on(const Ctx& x, unsigned bit) {
  return (x.P->interactions & bit) && (!x.a->term_mask || (x.a->term_mask & bit));
}

/* Core pairs as 32 x 32 tiles (i block ib <= j block jb), one warp each,
 * every unordered pair evaluated once.  Lane l owns atom i = 32 ib + l; at
 * step s it pairs with j = 32 jb + ((l + s) mod 32), so the lanes read 32
 * distinct j (no bank conflicts), and it keeps the reaction on that j in a
 * register that moves one lane down after every step: after 32 steps lane l
 * holds the whole reaction on j = 32 jb + l.  Diagonal tiles take steps
 * 1..15 and half of step 16.  Each side is summed over the tile's steps in
 * the pair precision, in that fixed order, and reaches the core sums once
 * per tile as a 64-bit integer (one conversion per atom and tile instead of
 * one per pair, 32-bit shuffles for the reactions), so the result does not
 * depend on the launch shape. */
template <bool FP64>
__device__ __forceinline__ void core_pairs_t(Ctx& x, bool eflag) {
  const RepParams* P = x.P;
  const int ni = P->n_ion, nc = x.n_core, nt = P->n_types;
  const bool amber = term_on(x, MDN_I_AMBER), bmh = term_on(x, MDN_I_BMH);
  const bool vi = term_on(x, MDN_I_VI), vv = term_on(x, MDN_I_VV);
  if (!(amber || bmh || vi || vv)) return;
  const float qqf = (float)P->qqrd2e;
  const int nblk = (nc + 31) >> 5;
  const int tiles = nblk * (nblk + 1) / 2;
  const int lane = threadIdx.x & 31;
  const int nwb = blockDim.x >> 5;
  const int* bmht = x.ib + P->o_ion_bmh;
  long long e_ion = 0, e_vi = 0, e_vv = 0;
  for (int t = x.rank * nwb + (threadIdx.x >> 5); t < tiles; t += x.C * nwb) {
    int ib = 0, rem = t;
    while (rem >= nblk - ib) {
      rem -= nblk - ib;
      ib++;
    }
    const int jb = ib + rem;
    const bool diag = ib == jb;
    const int i = ib * 32 + lane;
    const bool act = i < nc;
    const int ii = act ? i : 0;
    const float4 pi = x.c.pos[ii];
    const int ti = x.c.type[ii], mi = x.c.mol[ii];
    const float wi = x.c.w[ii];
    const bool iion = ii < ni;
    const int bi = (bmh && iion) ? bmht[ii] : 0;
    double xd[3] = {0, 0, 0}, wid = 1.0, qid = 0.0;
    if constexpr (FP64) {
      for (int k = 0; k < 3; k++) xd[k] = x.c.x[3 * ii + k];
      wid = weight_d(x, ii);
      qid = charge_d(x, ii);
    }
    /* the tile's sums in the pair arithmetic's own precision, in a fixed
     * order (the tile's steps), turned into fixed point once per atom */
    using Acc = typename std::conditional<FP64, double, float>::type;
    Acc F0 = 0, F1 = 0, F2 = 0, R0 = 0, R1 = 0, R2 = 0;
    for (int s = 0; s < 32; s++) {
      const int j = jb * 32 + ((lane + s) & 31);
      bool take = act && j < nc;
      if (diag) take = take && s != 0 && (s < 16 || (s == 16 && lane < 16));
      if (take) {
        const float4 pj = x.c.pos[j];
        const int tj = x.c.type[j], mj = x.c.mol[j];
        const float wj = x.c.w[j];
        const bool jion = j < ni;
        const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        float fp = 0.0f;
        bool any = false;
        int bucket = 0;
        if (iion && jion) {
          const bool ex = amber && ((x.c.excl[i * P->excl_words + (j >> 5)] >> (j & 31)) & 1u);
          if (amber && !ex) {
            float ee;
            fp += lj_coul(r2, x.c.ljA[ti * nt + tj], x.c.ljB[ti * nt + tj], qqf * pi.w * pj.w, true, &ee);
            any = true;
          }
          if (bmh) {
            float ee;
            fp += born(r2, bi, bmht[j], qqf * pi.w * pj.w, &ee);
            any = true;
          }
          bucket = 1;
        } else if (iion != jion) {
          if (vi) {
            float ee;
            fp = lj_coul(r2, x.c.ljA[ti * nt + tj], x.c.ljB[ti * nt + tj], qqf * pi.w * pj.w, true, &ee) * (wi * wj);
            any = true;
            bucket = 2;
          }
        } else if (mi != mj) {
          if (vv) {
            float ee;
            fp = lj_coul(r2, x.c.ljA[ti * nt + tj], x.c.ljB[ti * nt + tj], qqf * pi.w * pj.w, true, &ee) * (wi * wj);
            any = true;
            bucket = 3;
          }
        }
        if (any) {
          Acc fx, fy, fz;
          if constexpr (FP64) {
            /* the same terms in FP64 from the FP64 positions and tables */
            const double ex = xd[0] - x.c.x[3 * j], ey = xd[1] - x.c.x[3 * j + 1], ez = xd[2] - x.c.x[3 * j + 2];
            const double R2d = ex * ex + ey * ey + ez * ez;
            const double qq = P->qqrd2e * qid * charge_d(x, j);
            const double Ad = x.db[P->d_ljA + ti * nt + tj], Bd = x.db[P->d_ljB + ti * nt + tj];
            double fd = 0.0;
            if (bucket == 1) {
              if (amber && !((x.c.excl[i * P->excl_words + (j >> 5)] >> (j & 31)) & 1u))
                fd += lj_coul_d(R2d, Ad, Bd, qq, true);
              if (bmh) fd += born_d(R2d, bi, bmht[j], qq);
            } else {
              fd = lj_coul_d(R2d, Ad, Bd, qq, true) * (wid * weight_d(x, j));
            }
            fx = fd * ex;
            fy = fd * ey;
            fz = fd * ez;
          } else {
            fx = fp * dx;
            fy = fp * dy;
            fz = fp * dz;
          }
          F0 += fx; F1 += fy; F2 += fz;
          R0 -= fx; R1 -= fy; R2 -= fz;
          if (eflag) {
            const double R2e = r2d(x.c.x + 3 * i, x.c.x + 3 * j);
            const double qi = i < ni ? x.db[P->d_ion_q + i] : x.db[P->d_vap_q + (i - ni) % P->a_v];
            const double qj = j < ni ? x.db[P->d_ion_q + j] : x.db[P->d_vap_q + (j - ni) % P->a_v];
            const double qq = P->qqrd2e * qi * qj;
            double ed = 0;
            if (bucket == 1) {
              if (amber && !((x.c.excl[i * P->excl_words + (j >> 5)] >> (j & 31)) & 1u))
                ed += lj_coul_energy(R2e, x.db[P->d_ljA + ti * nt + tj], x.db[P->d_ljB + ti * nt + tj], qq);
              if (bmh) ed += born_energy(R2e, bi, bmht[j], qq);
              e_ion += efixd(ed);
            } else {
              ed = lj_coul_energy(R2e, x.db[P->d_ljA + ti * nt + tj], x.db[P->d_ljB + ti * nt + tj], qq);
              if (bucket == 2) e_vi += efixd(ed);
              else e_vv += efixd(ed);
            }
          }
        }
      }
      R0 = __shfl_sync(0xffffffffu, R0, (lane + 1) & 31);
      R1 = __shfl_sync(0xffffffffu, R1, (lane + 1) & 31);
      R2 = __shfl_sync(0xffffffffu, R2, (lane + 1) & 31);
    }
    auto fix = [](Acc v) -> long long {
      if constexpr (FP64) return fixd(v);
      else return fixf(v);
    };
    if (act && (F0 != 0 || F1 != 0 || F2 != 0)) {
      const long long F[3] = {fix(F0), fix(F1), fix(F2)};
      acc_add(x, i, F);
    }
    const int jj = jb * 32 + lane;
    if (jj < nc && (R0 != 0 || R1 != 0 || R2 != 0)) {
      const long long Rv[3] = {fix(R0), fix(R1), fix(R2)};
      acc_add(x, jj, Rv);
    }
  }
  if (eflag) {
    e_ion = warp_sum_ll(e_ion);
    e_vi = warp_sum_ll(e_vi);
    e_vv = warp_sum_ll(e_vv);
    if (lane == 0) {
      energy_add(x, MDN_U_ION, e_ion);
      energy_add(x, MDN_U_VI, e_vi);
      energy_add(x, MDN_U_VV, e_vv);
    }
  }
}

/* MDN_FP64_PAIRS selects the pair precision of this compilation: the FP64
 * form (mdn_options.force_mode = 1) is compiled into its own kernel,
 * mdn_advance_fp64 (advance_fp64.cu), so that the FP32 kernel's registers
 * and code are not shaped by it */
#ifdef MDN_FP64_PAIRS
constexpr bool kFP64Pairs = true;
#else
constexpr bool kFP64Pairs = false;
#endif

__device__ __forceinline__ void core_pairs(Ctx& x, bool eflag) { core_pairs_t<kFP64Pairs>(x, eflag); }

/* MDN_GG_TERMS selects the gas-gas term: compiled into its own kernels
 * (advance_gg.cu, advance_gg_fp64.cu), absent from the others */
#ifdef MDN_GG_TERMS
constexpr bool kGG = true;
#else
constexpr bool kGG = false;
#endif

__device__ __forceinline__ void core_bonded(Ctx& x, bool eflag) {
  const RepParams* P = x.P;
  const bool amber = term_on(x, MDN_I_AMBER);
  const bool vin = term_on(x, MDN_I_VAPOR_INTRA);
  const bool qb = (P->quirks & MDN_Q_ENERGY_BUCKETS) != 0;
  const int nb = amber ? P->n_ion_bonds : 0, na = amber ? P->n_ion_angles : 0, nd = amber ? P->n_ion_dih : 0;
  const int vterms = vin ? (P->n_vap_bonds + P->n_vap_angles + P->n_vap_dih) : 0;
  const long long total = (long long)nb + na + nd + (long long)vterms * x.D->n_vap_in;
  long long eU[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (long long t = (long long)x.rank * blockDim.x + threadIdx.x; t < total; t += (long long)x.C * blockDim.x) {
    BondOut o;
    int idx[4];
    int n = 0, bucket = MDN_U_ION;
    const double* X = x.c.x;
    int base = 0;
    long long u = t;
    int kind;  /* 0 bond, 1 angle, 2 dihedral */
    const int* row;
    if (u < nb) { kind = 0; row = x.ib + P->o_ion_bonds + 3 * u; }
    else if ((u -= nb) < na) { kind = 1; row = x.ib + P->o_ion_angles + 4 * u; }
    else if ((u -= na) < nd) { kind = 2; row = x.ib + P->o_ion_dih + 5 * u; }
    else {
      u -= nd;
      int s = (int)(u / vterms), q = (int)(u - (long long)s * vterms);
      base = P->n_ion + s * P->a_v;
      if (q < P->n_vap_bonds) { kind = 0; row = x.ib + P->o_vap_bonds + 3 * q; bucket = qb ? MDN_U_GAS : MDN_U_VAP; }
      else if ((q -= P->n_vap_bonds) < P->n_vap_angles) { kind = 1; row = x.ib + P->o_vap_angles + 4 * q; bucket = qb ? MDN_U_GAS : MDN_U_VAP; }
      else { q -= P->n_vap_angles; kind = 2; row = x.ib + P->o_vap_dih + 5 * q; bucket = qb ? MDN_U_ION : MDN_U_VAP; }
    }
    if (kind == 0) {
      idx[0] = base + row[0]; idx[1] = base + row[1];
      bond_fd(X, x.db + P->d_bond + 2 * row[2], idx[0], idx[1], o);
      n = 2;
    } else if (kind == 1) {
      idx[0] = base + row[0]; idx[1] = base + row[1]; idx[2] = base + row[2];
      angle_fd(X, x.db + P->d_angle + 2 * row[3], idx[0], idx[1], idx[2], o);
      n = 3;
    } else {
      idx[0] = base + row[0]; idx[1] = base + row[1]; idx[2] = base + row[2]; idx[3] = base + row[3];
      dihedral_fd(X, x.db + P->d_dih + 15 * row[4], x.ib[P->o_dih_multi + row[4]], idx[0], idx[1], idx[2],
                  idx[3], o);
      n = 4;
    }
    for (int q = 0; q < n; q++) {
      long long F[3] = {fixd(o.f[q][0]), fixd(o.f[q][1]), fixd(o.f[q][2])};
      acc_add(x, idx[q], F);
    }
    if (eflag) eU[bucket] += efixd(o.e);
  }
  if (eflag)
    for (int b = 0; b < 8; b++) {
      long long s = warp_sum_ll(eU[b]);
      if ((threadIdx.x & 31) == 0) energy_add(x, b, s);
    }
  if (term_on(x, MDN_I_EFIELD) && x.rank == 0)
    for (int i = threadIdx.x; i < P->n_ion; i += blockDim.x) {
      double coeff = 5.55e-5 * x.db[P->d_ion_q + i];
      long long F[3] = {fixd(coeff * P->efield[0]), fixd(coeff * P->efield[1]), fixd(coeff * P->efield[2])};
      acc_add(x, i, F);
    }
}

/* ------------------------------------------------------------------------- */
/* gas molecules                                                              */
/* ------------------------------------------------------------------------- */
__device__ __forceinline__ void partition(const Ctx& x, int n, int* lo, int* hi) {
  *lo = (int)(((long long)n * x.rank) / x.C);
  *hi = (int)(((long long)n * (x.rank + 1)) / x.C);
}

/* intramolecular bond force of one gas molecule (PotentialGasIntra), FP64 */
/* Gas molecules have one or two atoms (AG); the bonded and SHAKE terms of a
 * two-atom molecule copy the pair into fixed slots (swapped when a row reads
 * (1, 0)) so that every array index is a compile-time constant and the
 * arrays stay in registers.  The arithmetic is that of bond_fd / shake_pair
 * on the row's own order. */
template <int AG>
__device__ __forceinline__ double gas_intra(const Ctx& x, const double* X, double* F) {
  if constexpr (AG == 1) {
    return 0.0;
  } else {
    const RepParams* P = x.P;
    double e = 0;
    for (int b = 0; b < P->n_gas_bonds; b++) {
      const int* row = x.ib + P->o_gas_bonds + 3 * b;
      const bool sw = row[0] != 0;
      double Y[6];
      for (int k = 0; k < 3; k++) {
        Y[k] = sw ? X[3 + k] : X[k];
        Y[3 + k] = sw ? X[k] : X[3 + k];
      }
      BondOut o;
      bond_fd(Y, x.db + P->d_bond + 2 * row[2], 0, 1, o);
      for (int k = 0; k < 3; k++) {
        F[k] += sw ? o.f[1][k] : o.f[0][k];
        F[3 + k] += sw ? o.f[0][k] : o.f[1][k];
      }
      e += o.e;
    }
    return e;
  }
}

/* SHAKE of a two-atom gas molecule: the sweeps of the vapor SHAKE with one colour */
__device__ __forceinline__ int shake_gas2(const Ctx& x, double* X, const double* R) {
  const RepParams* P = x.P;
  const int* rigid = x.ib + P->o_gas_rigid;
  const int n = P->n_gas_rigid;
  bool converge = false;
  for (int sweep = 0; sweep < MDN_SHAKE_MAX_SWEEPS && !converge; sweep++) {
    for (int k = 0; k < n; k++) {
      const bool sw = rigid[3 * k] != 0;
      double Y[6], RY[6];
      for (int q = 0; q < 3; q++) {
        Y[q] = sw ? X[3 + q] : X[q];
        Y[3 + q] = sw ? X[q] : X[3 + q];
        RY[q] = sw ? R[3 + q] : R[q];
        RY[3 + q] = sw ? R[q] : R[3 + q];
      }
      shake_pair_c(Y, Y + 3, RY, RY + 3, x.db + P->d_gas_cons + 3 * k);
      for (int q = 0; q < 3; q++) {
        X[q] = sw ? Y[3 + q] : Y[q];
        X[3 + q] = sw ? Y[q] : Y[3 + q];
      }
    }
    converge = true;
    for (int k = 0; k < n; k++)
      if (!(shake_res_c(X, X + 3, x.db + P->d_gas_cons + 3 * k) <= 1e-20)) converge = false;
  }
  return converge ? 0 : MDN_ST_SHAKE_NOCONV;
}

/* kick + drift (+SHAKE) of the gas molecules of this CTA; far molecules also
 * get their intramolecular force and the second kick when `fused`. */
/* kick, drift, gas SHAKE and (fused, for molecules without list entries)
 * the intramolecular force and second kick of the gas molecules; thread tid
 * of the nthr (whole warps) that take part */
template <int AG>
__device__ __forceinline__ void gas_integrate_t(Ctx& x, bool fused, bool eflag, int tid, int nthr) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  constexpr int ag = AG;
  const int par = x.D->parity;
  const bool sh = (P->interactions & MDN_I_SHAKE) && P->n_gas_rigid > 0;
  const bool vcorr = !(P->quirks & MDN_Q_SHAKE_NO_VCORR);
  const bool intra = term_on(x, MDN_I_GAS_INTRA) && P->n_gas_bonds > 0;
  const double dt = P->dt;
  int lo, hi;
  partition(x, x.D->n_gas_in, &lo, &hi);
  double m[AG], c2[AG];
#pragma unroll
  for (int at = 0; at < ag; at++) {
    int t = x.ib[P->o_gas_type + at];
    m[at] = x.db[P->d_mass + t];
    c2[at] = x.c.c2[t];
  }
  long long eg = 0;
  for (int s = lo + tid; s < hi; s += nthr) {
    double X[3 * AG], V[3 * AG], F[3 * AG], R[3 * AG];
    for (int at = 0; at < ag; at++) {
      size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) {
        X[3 * at + k] = a->slab_x[3 * g + k];
        V[3 * at + k] = a->slab_v[3 * g + k];
        F[3 * at + k] = a->slab_f[3 * g + k];
      }
    }
    for (int at = 0; at < ag; at++)
      for (int k = 0; k < 3; k++) {
        V[3 * at + k] += F[3 * at + k] * c2[at];
        R[3 * at + k] = X[3 * at + k];
        X[3 * at + k] = X[3 * at + k] + V[3 * at + k] * dt;
        F[3 * at + k] = 0.0;
      }
    if constexpr (AG == 2) {
      if (sh) {
        double Xd[3 * AG];
#pragma unroll
        for (int q = 0; q < 3 * ag; q++) Xd[q] = X[q];
        int st = shake_gas2(x, X, R);
        if (st) set_status(x, st);
        if (vcorr)
#pragma unroll
          for (int q = 0; q < 3 * ag; q++) V[q] += (X[q] - Xd[q]) / dt;
      }
    }
    if (!isfinite(X[0] + X[1] + X[2] + V[0] + V[1] + V[2])) set_status(x, MDN_ST_NONFINITE);
    bool near = fused ? (a->near_gi[gmol(P, par, s)] >= 0) : true;
    if (!near) {
      if (intra) {
        double e = gas_intra<AG>(x, X, F);
        if (eflag) eg += efixd(e);
      }
      for (int at = 0; at < ag; at++)
        for (int k = 0; k < 3; k++) V[3 * at + k] += F[3 * at + k] * c2[at];
    }
    for (int at = 0; at < ag; at++) {
      size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) {
        a->slab_x[3 * g + k] = X[3 * at + k];
        a->slab_v[3 * g + k] = V[3 * at + k];
        a->slab_f[3 * g + k] = F[3 * at + k];
      }
    }
  }
  if (eflag && intra) {
    eg = warp_sum_ll(eg);
    if ((threadIdx.x & 31) == 0) energy_add(x, MDN_U_GAS, eg);
  }
}

__device__ __forceinline__ void gas_integrate(Ctx& x, bool fused, bool eflag, int tid, int nthr) {
  if (x.P->a_g == 1) gas_integrate_t<1>(x, fused, eflag, tid, nthr);
  else gas_integrate_t<2>(x, fused, eflag, tid, nthr);
}

/* after a rebuild: intramolecular force and second kick of the far molecules */
template <int AG>
__device__ __forceinline__ void gas_far_pass_t(Ctx& x, bool eflag, bool kick) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  constexpr int ag = AG;
  const int par = x.D->parity;
  const bool intra = term_on(x, MDN_I_GAS_INTRA) && P->n_gas_bonds > 0;
  const bool gg = kGG && term_on(x, MDN_I_GG) && P->ggl_cap > 0;
  int lo, hi;
  partition(x, x.D->n_gas_in, &lo, &hi);
  double c2[AG];
#pragma unroll
  for (int at = 0; at < ag; at++) c2[at] = x.c.c2[x.ib[P->o_gas_type + at]];
  long long eg = 0;
  for (int s = lo + threadIdx.x; s < hi; s += blockDim.x) {
    if (a->near_gi[gmol(P, par, s)] >= 0) continue;
    double X[3 * AG], F[3 * AG];
    for (int at = 0; at < ag; at++) {
      size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) {
        X[3 * at + k] = a->slab_x[3 * g + k];
        F[3 * at + k] = 0.0;
      }
    }
    if (intra) {
      double e = gas_intra<AG>(x, X, F);
      if (eflag) eg += efixd(e);
    }
    if (gg)
      for (int at = 0; at < ag; at++)
        for (int k = 0; k < 3; k++) F[3 * at + k] += a->slab_fgg[3 * gatom(P, par, s, at) + k];
    for (int at = 0; at < ag; at++) {
      size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) {
        if (kick) a->slab_v[3 * g + k] += F[3 * at + k] * c2[at];
        a->slab_f[3 * g + k] = F[3 * at + k];
      }
    }
  }
  if (eflag && intra) {
    eg = warp_sum_ll(eg);
    if ((threadIdx.x & 31) == 0) energy_add(x, MDN_U_GAS, eg);
  }
}

__device__ __forceinline__ void gas_far_pass(Ctx& x, bool eflag, bool kick) {
  if (x.P->a_g == 1) gas_far_pass_t<1>(x, eflag, kick);
  else gas_far_pass_t<2>(x, eflag, kick);
}

/* gas-gas LJ, the corrected form of PotentialGasGas::compute
 * (src/potential/GasGas.cpp:4-38): every atom pair of two listed in-domain
 * gas molecules, force x w_i w_j with both atoms' taper weights, energy
 * unweighted into Ugg.  The reference's own routine pairs loop indices
 * instead of gas_in entries (:48-57), reads weight[0][jj] (:25), bounds the
 * partner loop by the first molecule's size (:13) and books the energy in
 * Uvg (:34); none of that is reproduced.  One thread per slab molecule of
 * this CTA walks its full (both-direction) partner list and writes its own
 * force, so no reaction is scattered and the sum does not depend on the
 * launch shape.  Weights come from the current positions and ion centre, as
 * MD::update_position sets them (src/verlet.cpp:109-134); molecules the
 * rebuild of this step inserted have weight 0 (`fresh`: this step rebuilt). */
template <int AG, bool FP64>
__device__ __forceinline__ void gas_gg_pass_t(Ctx& x, bool eflag, bool fresh) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  const int par = x.D->parity, nt = P->n_types, nreb = x.D->n_rebuilds;
  int lo, hi;
  partition(x, x.D->n_gas_in, &lo, &hi);
  int gtype[AG];
#pragma unroll
  for (int at = 0; at < AG; at++) gtype[at] = x.ib[P->o_gas_type + at];
  const double* com = x.D->ion_com;
  long long egg = 0;
  for (int s = lo + (int)threadIdx.x; s < hi; s += blockDim.x) {
    const size_t ms = gmol(P, par, s);
    const bool s_new = fresh && __ldcg(a->slab_ins + ms) == nreb;
    double X[3 * AG], w[AG];
#pragma unroll
    for (int at = 0; at < AG; at++) {
      const size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) X[3 * at + k] = a->slab_x[3 * g + k];
      w[at] = s_new ? 0.0 : taper(P, com, X + 3 * at);
    }
    long long F[AG][3];
#pragma unroll
    for (int at = 0; at < AG; at++) F[at][0] = F[at][1] = F[at][2] = 0;
    const int start = a->ggl_start[ms], cnt = a->ggl_n[ms];
    for (int q = 0; q < cnt; q++) {
      const int t = a->ggl[P->ggl_off + start + q];
      const bool t_new = fresh && __ldcg(a->slab_ins + gmol(P, par, t)) == nreb;
#pragma unroll
      for (int b = 0; b < AG; b++) {
        const size_t gt = gatom(P, par, t, b);
        /* another CTA's molecule, moved this step: from L2 */
        const double Y[3] = {__ldcg(a->slab_x + 3 * gt), __ldcg(a->slab_x + 3 * gt + 1),
                             __ldcg(a->slab_x + 3 * gt + 2)};
        const double wb = t_new ? 0.0 : taper(P, com, Y);
        const int tb = gtype[b];
#pragma unroll
        for (int at = 0; at < AG; at++) {
          const int ta = gtype[at];
          long long fx, fy, fz;
          if constexpr (FP64) {
            const double ex = X[3 * at] - Y[0], ey = X[3 * at + 1] - Y[1], ez = X[3 * at + 2] - Y[2];
            const double fd = lj_coul_d(ex * ex + ey * ey + ez * ez, x.db[P->d_ljA + ta * nt + tb],
                                        x.db[P->d_ljB + ta * nt + tb], 0.0, false) * (w[at] * wb);
            fx = fixd(fd * ex); fy = fixd(fd * ey); fz = fixd(fd * ez);
          } else {
            /* the displacement from the FP64 positions: both atoms may sit
             * 100 A from the ion centre, where FP32 coordinates would carry
             * 1e-5 A of rounding into a 3 A separation */
            const float dx = (float)(X[3 * at] - Y[0]), dy = (float)(X[3 * at + 1] - Y[1]),
                        dz = (float)(X[3 * at + 2] - Y[2]);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            float ee;
            const float fp = lj_coul(r2, x.c.ljA[ta * nt + tb], x.c.ljB[ta * nt + tb], 0.0f, false, &ee) *
                             (float)(w[at] * wb);
            fx = fixf(fp * dx); fy = fixf(fp * dy); fz = fixf(fp * dz);
          }
          F[at][0] += fx; F[at][1] += fy; F[at][2] += fz;
          if (eflag && t > s)
            egg += efixd(lj_coul_energy(r2d(X + 3 * at, Y), x.db[P->d_ljA + ta * nt + tb],
                                        x.db[P->d_ljB + ta * nt + tb], 0.0));
        }
      }
    }
#pragma unroll
    for (int at = 0; at < AG; at++) {
      const size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) {
        const double f = (double)F[at][k] * MDN_FIX_INV;
        if (!(fabs(f) < MDN_FIX_LIMIT)) set_status(x, MDN_ST_FIXED_OVERFLOW);
        a->slab_fgg[3 * g + k] = f;
      }
    }
  }
  if (eflag) {
    egg = warp_sum_ll(egg);
    if ((threadIdx.x & 31) == 0) energy_add(x, MDN_U_GG, egg);
  }
}

/* the gas-gas forces of this step, when gg LJ is on: every CTA of the
 * cluster must see the final gas positions first */
__device__ __forceinline__ void gas_gg_pass(Ctx& x, cg::cluster_group& cl, bool eflag, bool fresh) {
  if constexpr (kGG) {
    if (!(term_on(x, MDN_I_GG) && x.P->ggl_cap > 0)) return;
    __threadfence();
    cl.sync();
    if (x.P->a_g == 1) gas_gg_pass_t<1, kFP64Pairs>(x, eflag, fresh);
    else gas_gg_pass_t<2, kFP64Pairs>(x, eflag, fresh);
    __syncthreads();
  }
}

/* LJ force of one (gas atom, core atom j) pair as 64-bit fixed point, the
 * force on the gas atom (PotentialGasIon / PotentialVaporGas: no Coulomb,
 * no taper weight); the near pass adds it to the gas atom and its negative
 * to the core atom's sums. */
template <bool FP64>
__device__ __forceinline__ void gas_core_pair(const Ctx& x, const double* Xa, float3 ga, int ta, int j,
                                              long long* f) {
  const RepParams* P = x.P;
  const int nt = P->n_types, tj = x.c.type[j];
  if constexpr (FP64) {
    const double ex = Xa[0] - x.c.x[3 * j], ey = Xa[1] - x.c.x[3 * j + 1], ez = Xa[2] - x.c.x[3 * j + 2];
    const double fd = lj_coul_d(ex * ex + ey * ey + ez * ez, x.db[P->d_ljA + ta * nt + tj],
                                x.db[P->d_ljB + ta * nt + tj], 0.0, false);
    f[0] = fixd(fd * ex); f[1] = fixd(fd * ey); f[2] = fixd(fd * ez);
  } else {
    const float4 pj = x.c.pos[j];
    const float dx = ga.x - pj.x, dy = ga.y - pj.y, dz = ga.z - pj.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float ee;
    const float fp = lj_coul(r2, x.c.ljA[ta * nt + tj], x.c.ljB[ta * nt + tj], 0.0f, false, &ee);
    f[0] = fixf(fp * dx); f[1] = fixf(fp * dy); f[2] = fixf(fp * dz);
  }
}

/* One core partner j of a near gas molecule: the LJ pairs of its AG atoms
 * with j, their forces added to F (64-bit fixed point), the reaction on j to
 * the core sums (shared 32-bit atomics on exact chunks, acc_add), and with
 * eflag the pair energy to e.  X holds the molecule's FP64 positions (used
 * by the FP64 pairs and the energies), gp its FP32 positions relative to the
 * ion centre. */
template <int AG, bool FP64>
__device__ __forceinline__ void near_partner(Ctx& x, const double* X, const float3* gp, const int* gtype, int j,
                                             bool eflag, long long (*F)[3], long long& e) {
  const RepParams* P = x.P;
  const int nt = P->n_types, tj = x.c.type[j];
  long long R[3] = {0, 0, 0};
#pragma unroll
  for (int at = 0; at < AG; at++) {
    long long f[3];
    gas_core_pair<FP64>(x, X + 3 * at, gp[at], gtype[at], j, f);
    F[at][0] += f[0]; F[at][1] += f[1]; F[at][2] += f[2];
    R[0] -= f[0]; R[1] -= f[1]; R[2] -= f[2];
    if (eflag)
      e += efixd(lj_coul_energy(r2d(X + 3 * at, x.c.x + 3 * j), x.db[P->d_ljA + gtype[at] * nt + tj],
                                x.db[P->d_ljB + gtype[at] * nt + tj], 0.0));
  }
  acc_add(x, j, R);
}

/* A near molecule with more partners than this has them spread over a warp. */
constexpr int kNearHeavy = 16;

/* near molecules (those with a gas-ion or gas-vapor list entry).  Partner
 * counts (gas-ion entries, plus gas-vapor entries times the vapor atoms each
 * reaches) are uneven: the few dozen to few hundred molecules next to a
 * large ion have 30-100 gas-ion entries, the thousands near vapor 1-13
 * gas-vapor partners.  So, first, each warp takes 32 of the CTA's near
 * molecules at a time and spreads the partners of those with more than
 * kNearHeavy over its lanes, one molecule after another, their force summed
 * by shuffles and parked, as 64-bit integers, in the molecule's slab force
 * rows.  Then one thread per near molecule walks the other molecules'
 * lists (the lanes of a warp run through their molecules independently, so
 * uneven light walks even out over a lane's several molecules), takes the
 * parked force of the heavy ones, and finishes each molecule: its force,
 * the gas-gas and intramolecular terms and the second kick.  Each reaction
 * goes to the core sums by shared 32-bit integer atomics on exact chunks
 * (acc_add); all sums are integers, so neither the split nor the order
 * changes the result. */
template <int AG, bool FP64>
__device__ __forceinline__ void gas_near_pass_t(Ctx& x, bool eflag, bool kick) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  constexpr int ag = AG;
  const int av = P->a_v, par = x.D->parity, ni = P->n_ion;
  const bool gi = term_on(x, MDN_I_GI), gv = term_on(x, MDN_I_GV);
  const bool intra = term_on(x, MDN_I_GAS_INTRA) && P->n_gas_bonds > 0;
  const bool gg = kGG && term_on(x, MDN_I_GG) && P->ggl_cap > 0;
  const int nj = (P->quirks & MDN_Q_GV_GAS_COUNT) ? min(ag, av) : av;
  int lo, hi;
  partition(x, x.D->n_gas_in, &lo, &hi);
  /* this CTA's range of the (ascending) near list */
  const int* nl = a->near_list + P->near_off;
  const int nn = x.D->n_near;
  int b0 = 0, b1 = nn;
  {
    int L = 0, H = nn;
    while (L < H) { int M = (L + H) >> 1; if (nl[M] < lo) L = M + 1; else H = M; }
    b0 = L;
    L = b0; H = nn;
    while (L < H) { int M = (L + H) >> 1; if (nl[M] < hi) L = M + 1; else H = M; }
    b1 = L;
  }
  int gtype[AG];
  double c2[AG];
#pragma unroll
  for (int at = 0; at < ag; at++) {
    gtype[at] = x.ib[P->o_gas_type + at];
    c2[at] = x.c.c2[gtype[at]];
  }
  const double* com = x.D->ion_com;
  long long egi = 0, egv = 0, eintra = 0;
  /* heavy molecules, spread over a warp */
  {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    for (int c0 = b0 + (int)(threadIdx.x & ~31u); c0 < b1; c0 += blockDim.x) {
      const int e = c0 + lane;
      int items = 0;
      if (e < b1) {
        const size_t ms = gmol(P, par, nl[e]);
        items = (gi ? (int)a->gil_n[ms] : 0) + (gv ? (int)a->gvl_n[ms] * nj : 0);
      }
      for (unsigned heavy = __ballot_sync(FULL, items > kNearHeavy); heavy; heavy &= heavy - 1) {
        const int so = nl[c0 + __ffs(heavy) - 1];
        const size_t ms = gmol(P, par, so);
        const int ngo = gi ? a->gil_n[ms] : 0, nvo = gv ? a->gvl_n[ms] : 0;
        const int sgo = a->near_gi[ms], svo = a->near_gv[ms];
        float3 gpo[AG];
        double Xo[3 * AG];
#pragma unroll
        for (int at = 0; at < AG; at++) {
          const size_t g = gatom(P, par, so, at);
#pragma unroll
          for (int k = 0; k < 3; k++) Xo[3 * at + k] = a->slab_x[3 * g + k];
          gpo[at] = make_float3((float)(Xo[3 * at] - com[0]), (float)(Xo[3 * at + 1] - com[1]),
                                (float)(Xo[3 * at + 2] - com[2]));
        }
        long long Fo[AG][3];
#pragma unroll
        for (int at = 0; at < AG; at++) Fo[at][0] = Fo[at][1] = Fo[at][2] = 0;
        const int n_it = ngo + nvo * nj;
        for (int it = lane; it < n_it; it += 32) {
          if (it < ngo) {
            near_partner<AG, FP64>(x, Xo, gpo, gtype, (int)a->gil[P->gil_off + sgo + it], eflag, Fo, egi);
          } else {
            const int t = it - ngo, ent = t / nj, b = t - ent * nj;
            near_partner<AG, FP64>(x, Xo, gpo, gtype, ni + (int)a->gvl[P->gvl_off + svo + ent] * av + b, eflag,
                                   Fo, egv);
          }
        }
#pragma unroll
        for (int at = 0; at < AG; at++) {
          const size_t g = gatom(P, par, so, at);
#pragma unroll
          for (int k = 0; k < 3; k++) {
            const long long v = warp_sum_ll(Fo[at][k]);
            if (lane == 0) a->slab_f[3 * g + k] = __longlong_as_double(v);
          }
        }
      }
    }
  }
  __syncthreads();
  for (int e = b0 + (int)threadIdx.x; e < b1; e += blockDim.x) {
    const int s = nl[e];
    const size_t ms = gmol(P, par, s);
    float3 gp[AG];
    double X[3 * AG];
#pragma unroll
    for (int at = 0; at < ag; at++) {
      size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) X[3 * at + k] = a->slab_x[3 * g + k];
      gp[at] = make_float3((float)(X[3 * at] - com[0]), (float)(X[3 * at + 1] - com[1]),
                           (float)(X[3 * at + 2] - com[2]));
    }
    long long F[AG][3];
#pragma unroll
    for (int at = 0; at < AG; at++) F[at][0] = F[at][1] = F[at][2] = 0;
    /* a heavy molecule's force was parked by its warp */
    const int ngi = gi ? a->gil_n[ms] : 0, ngv = gv ? a->gvl_n[ms] : 0;
    const bool heavy = ngi + ngv * nj > kNearHeavy;
    {
      const int sgi = a->near_gi[ms], sgv = a->near_gv[ms];
      const int cgi = heavy ? 0 : ngi, cgv = heavy ? 0 : ngv;
      for (int q = 0; q < cgi; q++)
        near_partner<AG, FP64>(x, X, gp, gtype, (int)a->gil[P->gil_off + sgi + q], eflag, F, egi);
      for (int ent = 0; ent < cgv; ent++) {
        const int vs = a->gvl[P->gvl_off + sgv + ent];
        for (int b = 0; b < nj; b++) near_partner<AG, FP64>(x, X, gp, gtype, ni + vs * av + b, eflag, F, egv);
      }
    }
    double Fd[3 * AG];
#pragma unroll
    for (int at = 0; at < ag; at++)
      for (int k = 0; k < 3; k++) {
        const long long v = heavy ? __double_as_longlong(a->slab_f[3 * gatom(P, par, s, at) + k]) : F[at][k];
        Fd[3 * at + k] = (double)v * MDN_FIX_INV;
        if (!(fabs(Fd[3 * at + k]) < MDN_FIX_LIMIT)) set_status(x, MDN_ST_FIXED_OVERFLOW);
      }
    if (gg)
      for (int at = 0; at < ag; at++)
        for (int k = 0; k < 3; k++) Fd[3 * at + k] += a->slab_fgg[3 * gatom(P, par, s, at) + k];
    if (intra) {
      double ei = gas_intra<AG>(x, X, Fd);
      if (eflag) eintra += efixd(ei);
    }
    for (int at = 0; at < ag; at++) {
      size_t g = gatom(P, par, s, at);
      for (int k = 0; k < 3; k++) {
        if (kick) a->slab_v[3 * g + k] += Fd[3 * at + k] * c2[at];
        a->slab_f[3 * g + k] = Fd[3 * at + k];
      }
    }
  }
  if (eflag) {
    egi = warp_sum_ll(egi);
    egv = warp_sum_ll(egv);
    eintra = warp_sum_ll(eintra);
    if ((threadIdx.x & 31) == 0) {
      energy_add(x, MDN_U_GI, egi);
      energy_add(x, MDN_U_VG, egv);
      energy_add(x, MDN_U_GAS, eintra);
    }
  }
}

__device__ __forceinline__ void gas_near_pass(Ctx& x, bool eflag, bool kick) {
  if (x.P->a_g == 1) gas_near_pass_t<1, kFP64Pairs>(x, eflag, kick);
  else gas_near_pass_t<2, kFP64Pairs>(x, eflag, kick);
}

/* sum of the core partials over the cluster -> f (double), identical in every CTA */
__device__ __forceinline__ void core_reduce(Ctx& x, cg::cluster_group& cl) {
  const int n3 = 3 * x.n_core;
  long long* mine = x.c.acc;
  /* fold the chunk sums into this CTA's 64-bit sums (each thread its own
   * elements) and clear them for the next evaluation */
  for (int q = threadIdx.x; q < n3; q += blockDim.x) {
    unsigned* c = x.c.chunk + 3 * q;
    const unsigned long long s =
        (unsigned long long)c[0] + ((unsigned long long)c[1] << 16) + ((unsigned long long)c[2] << 32);
    c[0] = c[1] = c[2] = 0;
    mine[q] = (long long)s;
  }
  if (x.C > 1) {
    cl.sync();
    for (int q = threadIdx.x; q < n3; q += blockDim.x) {
      long long s = 0;
      for (int k = 0; k < x.C; k++) {
        const long long* other = cl.map_shared_rank(mine, k);
        s += other[q];
      }
      x.c.f[q] = (double)s * MDN_FIX_INV;
    }
    /* every CTA has read this one's sums: the buffer is free again (the
     * next step's SHAKE keeps its reference positions there) */
    cl.sync();
  } else {
    for (int q = threadIdx.x; q < n3; q += blockDim.x) x.c.f[q] = (double)mine[q] * MDN_FIX_INV;
  }
  __syncthreads();
  /* flag saturated forces, and positions that are no longer finite */
  if (x.rank == 0)
    for (int q = threadIdx.x; q < n3; q += blockDim.x) {
      if (!(fabs(x.c.f[q]) < MDN_FIX_LIMIT)) set_status(x, MDN_ST_FIXED_OVERFLOW);
      if (!isfinite(x.c.x[q]) || !isfinite(x.c.v[q])) set_status(x, MDN_ST_NONFINITE);
    }
}

/* all forces of the step (after positions and lists are final) and the second kick */
__device__ __forceinline__ void forces_and_kick(Ctx& x, cg::cluster_group& cl, bool eflag, bool kick) {
  prof_start(x);
  gas_near_pass(x, eflag, kick);
  __syncthreads();
  prof_end(x, MDN_PROF_NEAR);
  prof_start(x);
  core_bonded(x, eflag);
  __syncthreads();
  prof_end(x, MDN_PROF_BONDED);
  prof_start(x);
  core_pairs(x, eflag);
  __syncthreads();
  prof_end(x, MDN_PROF_PAIRS);
  prof_start(x);
  core_reduce(x, cl);
  if (kick) {
    core_kick(x);
    __syncthreads();
  }
  prof_end(x, MDN_PROF_REDUCE);
}

/* ------------------------------------------------------------------------- */
/* the effective-domain rebuild (MD::make_pair)                               */
/* ------------------------------------------------------------------------- */
/* Philox word of insertion draw `t` (word 1 is the N2 spin) */
__device__ __forceinline__ int insert_word(int t) { return t == 0 ? 0 : 1 + t; }

__device__ __forceinline__ void insert_vapor(const Ctx& x, int q, int n_rebuild, int t, double* X, double* V);

/* true when no atom of X[0..n) lies within MDN_INSERT_MIN_DIST of a core atom
 * (ion, vapor in the domain before this rebuild) or of a vapor molecule whose
 * entry this rebuild already accepted; with the gas-gas term on, nor of a gas
 * atom in the domain before this rebuild (gas molecules entering in the same
 * rebuild are not tested against each other) */
__device__ __forceinline__ bool insert_clear(const Ctx& x, const double* X, int n, int n_rebuild) {
  const double d2min = MDN_INSERT_MIN_DIST * MDN_INSERT_MIN_DIST;
  if (kGG && (x.P->interactions & MDN_I_GG)) {
    const RepParams* P = x.P;
    const int G = x.D->n_gas_in, par = x.D->parity;
    for (int u = 0; u < G * P->a_g; u++) {
      const double* gpos = x.a->slab_x + 3 * ((size_t)P->slab_off + (size_t)par * P->slab_cap * P->a_g + u);
      const double g0 = __ldcg(gpos), g1 = __ldcg(gpos + 1), g2 = __ldcg(gpos + 2);
      for (int a = 0; a < n; a++) {
        double dx = X[3 * a] - g0, dy = X[3 * a + 1] - g1, dz = X[3 * a + 2] - g2;
        if (dx * dx + dy * dy + dz * dz < d2min) return false;
      }
    }
  }
  for (int i = 0; i < x.n_core; i++) {
    const double* c = x.c.x + 3 * i;
    for (int a = 0; a < n; a++) {
      double dx = X[3 * a] - c[0], dy = X[3 * a + 1] - c[1], dz = X[3 * a + 2] - c[2];
      if (dx * dx + dy * dy + dz * dz < d2min) return false;
    }
  }
  const int nc = min(x.cand[MDN_INSERT_MAX_VAPOR], MDN_INSERT_MAX_VAPOR);
  for (int k = 0; k < nc; k++) {
    const int mi = x.cand[k];
    const int f = x.a->region[(size_t)x.P->mol_off + mi];
    if (!(f & 1)) continue;
    double Xv[3 * MDN_MAX_VAP_ATOMS], Vv[3 * MDN_MAX_VAP_ATOMS];
    insert_vapor(x, mi - 1 - x.P->n_gas, n_rebuild, f >> 2, Xv, Vv);
    for (int b = 0; b < x.P->a_v; b++)
      for (int a = 0; a < n; a++) {
        double dx = X[3 * a] - Xv[3 * b], dy = X[3 * a + 1] - Xv[3 * b + 1], dz = X[3 * a + 2] - Xv[3 * b + 2];
        if (dx * dx + dy * dy + dz * dz < d2min) return false;
      }
  }
  return true;
}

__device__ __forceinline__ void insert_gas(const Ctx& x, int q, int n_rebuild, int t, double* X, double* V) {
  const RepParams* P = x.P;
  const int ag = P->a_g, mi = 1 + q;
  const double* cx = x.a->mol_x + 3 * ((size_t)P->mol_off + mi);
  const double* cv = x.a->mol_v + 3 * ((size_t)P->mol_off + mi);
  for (int at = 0; at < ag; at++)
    for (int k = 0; k < 3; k++) {
      X[3 * at + k] = x.db[P->d_gas_x + 3 * at + k];
      V[3 * at + k] = 0;
    }
  if (P->gas_kind == MDN_GAS_N2 && ag == 2) {
    U4 s = draw(*P, mi, n_rebuild, 1, 1);
    double vy, vz;
    box_muller(s.v[0], s.v[1], vy, vz);
    vy *= P->gas_sigma;
    vz *= P->gas_sigma;
    double vzu = (P->quirks & MDN_Q_N2_ROT_VYVZ) ? vy : vz;
    V[0] = 0; V[1] = vy; V[2] = vzu;
    V[3] = 0; V[4] = -vy; V[5] = -vzu;
  }
  U4 s = draw(*P, mi, n_rebuild, 1, insert_word(t));
  double A = u01(s.v[0]) * 2 * 3.141592653589793;
  double B = u01(s.v[1]) * 2 * 3.141592653589793;
  double Cc = u01(s.v[2]) * 2 * 3.141592653589793;
  const bool zy = (P->quirks & MDN_Q_GAS_ROT_ZY) != 0;
  for (int at = 0; at < ag; at++) {
    double* p = X + 3 * at;
    rotation(p[0], p[1], p[2], A, B, Cc, p[0], p[1], zy ? p[1] : p[2]);
    for (int k = 0; k < 3; k++) p[k] += cx[k];
  }
  for (int at = 0; at < ag; at++) {
    double* p = V + 3 * at;
    rotation(p[0], p[1], p[2], A, B, Cc, p[0], p[1], zy ? p[1] : p[2]);
    for (int k = 0; k < 3; k++) p[k] += cv[k];
  }
}

__device__ __forceinline__ void insert_vapor(const Ctx& x, int q, int n_rebuild, int t, double* X, double* V) {
  const RepParams* P = x.P;
  const int av = P->a_v, mi = 1 + P->n_gas + q;
  const double* cx = x.a->mol_x + 3 * ((size_t)P->mol_off + mi);
  const double* cv = x.a->mol_v + 3 * ((size_t)P->mol_off + mi);
  U4 s = draw(*P, mi, n_rebuild, 1, insert_word(t));
  double A = u01(s.v[0]) * 2 * 3.141592653589793;
  double B = u01(s.v[1]) * 2 * 3.141592653589793;
  double Cc = u01(s.v[2]) * 2 * 3.141592653589793;
  for (int at = 0; at < av; at++) {
    double* p = X + 3 * at;
    for (int k = 0; k < 3; k++) p[k] = x.db[P->d_vap_x + 3 * at + k];
    rotation(p[0], p[1], p[2], A, B, Cc, p[0], p[1], p[2]);
    for (int k = 0; k < 3; k++) p[k] += cx[k];
    double* u = V + 3 * at;
    u[0] = u[1] = u[2] = 0;
    rotation(u[0], u[1], u[2], A, B, Cc, u[0], u[1], u[2]);
    for (int k = 0; k < 3; k++) u[k] += cv[k];
  }
}

/* free flight, in/out test, wrap and resampling of one molecule; returns
 * (draw << 2) | (was_in << 1) | now_in, draw = the insertion draw that passed
 * the overlap test (0 under MDN_Q_BLIND_INSERT).  A molecule inside the sphere
 * whose draws all overlap stays outside, unwrapped and not resampled, until
 * the next rebuild.  Entering vapor molecules become candidates that
 * vapor_entries() decides. */
__device__ __forceinline__ int classify_one(const Ctx& x, int mi, double sigma, int n_rebuild, int loop_pair,
                                            const double* com, int kind /* 0 gas, 1 vapor */) {
  const RepParams* P = x.P;
  const size_t g = (size_t)P->mol_off + mi;
  double* X = x.a->mol_x + 3 * g;
  double* V = x.a->mol_v + 3 * g;
  const int was = x.a->region[g] & 1;
  if (!was)
    for (int k = 0; k < 3; k++) X[k] += V[k] * P->dt * loop_pair;
  double dx = X[0] - com[0];
  double dy = X[1] - com[1];
  double dz = X[2] - com[2];
  double r2 = (dx * dx + dy * dy + dz * dz);
  int in = r2 < P->RI2 ? 1 : 0;
  int draw_ok = 0;
  if (in && !was && !(P->quirks & MDN_Q_BLIND_INSERT) && kind == 1) {
    /* decided by vapor_entries(): recorded as a candidate, provisionally in;
     * beyond MDN_INSERT_MAX_VAPOR candidates in one rebuild the entry waits
     * for the next */
    int c = atomicAdd(&x.cand[MDN_INSERT_MAX_VAPOR], 1);
    if (c >= MDN_INSERT_MAX_VAPOR) {
      x.a->region[g] = 0;
      return 0;
    }
    x.cand[c] = mi;
    x.a->region[g] = (unsigned char)1;
    return 1;
  }
  if (in && !was && !(P->quirks & MDN_Q_BLIND_INSERT)) {
    double Xt[3 * MDN_MAX_VAP_ATOMS], Vt[3 * MDN_MAX_VAP_ATOMS];
    int t = 0;
    for (; t < MDN_INSERT_TRIES; t++) {
      insert_gas(x, mi - 1, n_rebuild, t, Xt, Vt);
      if (insert_clear(x, Xt, P->a_g, n_rebuild)) break;
    }
    if (t == MDN_INSERT_TRIES) {
      x.a->region[g] = 0; /* the entry waits for the next rebuild */
      return 0;
    }
    draw_ok = t;
  }
  if (!in) {
    double HL = P->box * 0.5;
    if (dx < -HL) X[0] += P->box;
    if (dy < -HL) X[1] += P->box;
    if (dz < -HL) X[2] += P->box;
    if (dx > HL) X[0] -= P->box;
    if (dy > HL) X[1] -= P->box;
    if (dz > HL) X[2] -= P->box;
    U4 s = draw(*P, mi, n_rebuild, 0, 0);
    double z0, z1, z2, z3;
    box_muller(s.v[0], s.v[1], z0, z1);
    box_muller(s.v[2], s.v[3], z2, z3);
    V[0] = z0 * sigma;
    V[1] = z1 * sigma;
    V[2] = z2 * sigma;
  }
  x.a->region[g] = (unsigned char)((draw_ok << 2) | (was << 1) | in);
  return (draw_ok << 2) | (was << 1) | in;
}

/* exchange one int per CTA across the cluster: returns the prefix before this
 * rank and the total */
__device__ __forceinline__ void cluster_prefix(Ctx& x, cg::cluster_group& cl, int* slot_in_smem, int mine, int* before,
                               int* total) {
  if (threadIdx.x == 0) *slot_in_smem = mine;
  cl.sync();
  int b = 0, t = 0;
  for (int k = 0; k < x.C; k++) {
    int v = *cl.map_shared_rank(slot_in_smem, k);
    if (k < x.rank) b += v;
    t += v;
  }
  *before = b;
  *total = t;
  cl.sync();
}

/* gas-gas pair list of the slab (PotentialGasGas::makePair,
 * src/potential/GasGas.cpp:41-62, on the in-domain molecules it was meant
 * for): every other slab molecule whose centre lies within the list radius,
 * both directions, ascending slab slot, CSR by slab slot over the cluster */
__device__ __forceinline__ void relist_gg(Ctx& x, cg::cluster_group& cl) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  const int par = x.D->parity, G = x.D->n_gas_in;
  int lo, hi;
  partition(x, G, &lo, &hi);
  int* sc = x.iscr;
  const double* cen = a->mol_x + 3 * ((size_t)P->mol_off + 1);
  const int* smol = a->slab_mol + gmol(P, par, 0);
  /* centres and slab entries of every CTA's molecules, from L2 */
  auto partners = [&](int s, int* out) {
    const double* c = cen + 3 * (size_t)__ldcg(smol + s);
    const double c0 = __ldcg(c), c1 = __ldcg(c + 1), c2 = __ldcg(c + 2);
    int n = 0;
    for (int t = 0; t < G; t++) {
      if (t == s) continue;
      const double* d = cen + 3 * (size_t)__ldcg(smol + t);
      const double dx = c0 - __ldcg(d), dy = c1 - __ldcg(d + 1), dz = c2 - __ldcg(d + 2);
      if ((dx * dx + dy * dy + dz * dz) < P->ml2) {
        if (out) out[n] = t;
        n++;
      }
    }
    return n;
  };
  int mine = 0;
  for (int s = lo + (int)threadIdx.x; s < hi; s += blockDim.x) mine += partners(s, nullptr);
  mine = block_sum_i(mine, sc);
  int base, tot;
  cluster_prefix(x, cl, &sc[46], mine, &base, &tot);
  const bool over = tot > P->ggl_cap;
  if (over && threadIdx.x == 0 && x.rank == 0) set_status(x, MDN_ST_LIST_OVERFLOW);
  int run = base;
  for (int s0 = lo; s0 < hi; s0 += blockDim.x) {
    const int s = s0 + threadIdx.x;
    const int c = s < hi ? partners(s, nullptr) : 0;
    int t_tot;
    const int off = block_exscan(c, sc, &t_tot);
    if (s < hi) {
      const size_t ms = gmol(P, par, s);
      if (!over) {
        a->ggl_start[ms] = run + off;
        a->ggl_n[ms] = c;
        partners(s, a->ggl + P->ggl_off + run + off);
      } else {
        a->ggl_start[ms] = 0;
        a->ggl_n[ms] = 0;
      }
    }
    run += t_tot;
  }
  if (threadIdx.x == 0) x.D->gg_count = over ? 0 : tot / 2;
  __threadfence();
  cl.sync();
}

/* pair lists of the gas slab (current parity) from the centres: gas-ion
 * (PotentialGasIon::makePair) and gas-vapor (PotentialVaporGas::makePair) */
__device__ __forceinline__ void relist(Ctx& x, cg::cluster_group& cl) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  const int par = x.D->parity, ni = P->n_ion, nv = x.D->n_vap_in;
  const bool gi = (P->interactions & MDN_I_GI) != 0, gv = (P->interactions & MDN_I_GV) != 0;
  int lo, hi;
  partition(x, x.D->n_gas_in, &lo, &hi);
  /* bounding sphere of the ion, exact test below */
  int* sc = x.iscr;
  int gi_tot = 0, gv_tot = 0, nn_tot = 0;
  int gi_base = 0, gv_base = 0, nn_base = 0;
  /* pass 1: counts */
  int my_gi = 0, my_gv = 0, my_nn = 0;
  for (int s0 = lo; s0 < hi; s0 += blockDim.x) {
    int s = s0 + threadIdx.x;
    int cgi = 0, cgv = 0;
    if (s < hi) {
      int m = __ldcg(a->slab_mol + gmol(P, par, s));
      const double* cm = a->mol_x + 3 * ((size_t)P->mol_off + 1 + m);
      /* centres set by whichever CTA classified the molecule: from L2 */
      const double cx0 = __ldcg(cm), cx1 = __ldcg(cm + 1), cx2 = __ldcg(cm + 2);
      if (gi)
        for (int j = 0; j < ni; j++) {
          double dx = cx0 - x.c.x[3 * j], dy = cx1 - x.c.x[3 * j + 1], dz = cx2 - x.c.x[3 * j + 2];
          if ((dx * dx + dy * dy + dz * dz) < P->ml2) cgi++;
        }
      if (gv)
        for (int q = 0; q < nv; q++) {
          int vm = __ldcg(a->vslab_mol + vmol(P, par, q));
          const double* vc = a->mol_x + 3 * ((size_t)P->mol_off + 1 + P->n_gas + vm);
          double dx = cx0 - __ldcg(vc), dy = cx1 - __ldcg(vc + 1), dz = cx2 - __ldcg(vc + 2);
          if ((dx * dx + dy * dy + dz * dz) < P->ml2) cgv++;
        }
    }
    my_gi += cgi;
    my_gv += cgv;
    my_nn += (cgi + cgv) > 0 ? 1 : 0;
  }
  my_gi = block_sum_i(my_gi, sc);
  my_gv = block_sum_i(my_gv, sc);
  my_nn = block_sum_i(my_nn, sc);
  cluster_prefix(x, cl, &sc[40], my_gi, &gi_base, &gi_tot);
  cluster_prefix(x, cl, &sc[41], my_gv, &gv_base, &gv_tot);
  cluster_prefix(x, cl, &sc[42], my_nn, &nn_base, &nn_tot);
  bool over = gi_tot > P->gil_cap || gv_tot > P->gvl_cap || nn_tot > P->near_cap;
  if (over && threadIdx.x == 0 && x.rank == 0) set_status(x, MDN_ST_LIST_OVERFLOW);
  /* pass 2: fill, ascending slab slot */
  int run_gi = gi_base, run_gv = gv_base, run_nn = nn_base;
  for (int s0 = lo; s0 < hi; s0 += blockDim.x) {
    int s = s0 + threadIdx.x;
    int cgi = 0, cgv = 0;
    const double* cm = nullptr;
    double cx0 = 0, cx1 = 0, cx2 = 0;
    if (s < hi) {
      int m = __ldcg(a->slab_mol + gmol(P, par, s));
      cm = a->mol_x + 3 * ((size_t)P->mol_off + 1 + m);
      cx0 = __ldcg(cm);
      cx1 = __ldcg(cm + 1);
      cx2 = __ldcg(cm + 2);
      if (gi)
        for (int j = 0; j < ni; j++) {
          double dx = cx0 - x.c.x[3 * j], dy = cx1 - x.c.x[3 * j + 1], dz = cx2 - x.c.x[3 * j + 2];
          if ((dx * dx + dy * dy + dz * dz) < P->ml2) cgi++;
        }
      if (gv)
        for (int q = 0; q < nv; q++) {
          int vm = __ldcg(a->vslab_mol + vmol(P, par, q));
          const double* vc = a->mol_x + 3 * ((size_t)P->mol_off + 1 + P->n_gas + vm);
          double dx = cx0 - __ldcg(vc), dy = cx1 - __ldcg(vc + 1), dz = cx2 - __ldcg(vc + 2);
          if ((dx * dx + dy * dy + dz * dz) < P->ml2) cgv++;
        }
    }
    int t_gi, t_gv, t_nn;
    int o_gi = block_exscan(cgi, sc, &t_gi);
    int o_gv = block_exscan(cgv, sc, &t_gv);
    int isn = (cgi + cgv) > 0 ? 1 : 0;
    int o_nn = block_exscan(isn, sc, &t_nn);
    if (s < hi) {
      size_t ms = gmol(P, par, s);
      if (isn && !over) {
        int bgi = run_gi + o_gi, bgv = run_gv + o_gv;
        a->near_list[P->near_off + run_nn + o_nn] = s;
        a->near_gi[ms] = bgi;
        a->near_gv[ms] = bgv;
        a->gil_n[ms] = (unsigned short)cgi;
        a->gvl_n[ms] = (unsigned short)cgv;
        int w = 0;
        if (gi)
          for (int j = 0; j < ni; j++) {
            double dx = cx0 - x.c.x[3 * j], dy = cx1 - x.c.x[3 * j + 1], dz = cx2 - x.c.x[3 * j + 2];
            if ((dx * dx + dy * dy + dz * dz) < P->ml2) a->gil[P->gil_off + bgi + w++] = (unsigned short)j;
          }
        w = 0;
        if (gv)
          for (int q = 0; q < nv; q++) {
            int vm = __ldcg(a->vslab_mol + vmol(P, par, q));
            const double* vc = a->mol_x + 3 * ((size_t)P->mol_off + 1 + P->n_gas + vm);
            double dx = cx0 - __ldcg(vc), dy = cx1 - __ldcg(vc + 1), dz = cx2 - __ldcg(vc + 2);
            if ((dx * dx + dy * dy + dz * dz) < P->ml2) a->gvl[P->gvl_off + bgv + w++] = (unsigned short)q;
          }
      } else {
        a->near_gi[ms] = -1;
        a->near_gv[ms] = -1;
        a->gil_n[ms] = 0;
        a->gvl_n[ms] = 0;
      }
    }
    run_gi += t_gi;
    run_gv += t_gv;
    run_nn += t_nn;
  }
  if (threadIdx.x == 0) {
    x.D->gi_count = over ? 0 : gi_tot;
    x.D->gv_count = over ? 0 : gv_tot;
    x.D->n_near = over ? 0 : nn_tot;
  }
  __threadfence();
  cl.sync();
  if (kGG && P->ggl_cap > 0 && (P->interactions & MDN_I_GG)) relist_gg(x, cl);
}

/* The overlap test of entering vapor molecules: against the ion, the vapor
 * already in the domain and every in-domain gas atom (up to ~20,000), so the
 * whole block tests each candidate's draws.  Rank 0 only; returns the number
 * of entries that must wait. */
__device__ __forceinline__ int vapor_entries(Ctx& x, int nreb) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  const int av = P->a_v, ag = P->a_g, par = x.D->parity, G = x.D->n_gas_in;
  const double d2min = MDN_INSERT_MIN_DIST * MDN_INSERT_MIN_DIST;
  const int nc = min(x.cand[MDN_INSERT_MAX_VAPOR], MDN_INSERT_MAX_VAPOR);
  int deferred = 0;
  for (int c = 0; c < nc; c++) {
    const int mi = x.cand[c];
    const int q = mi - 1 - P->n_gas;
    int t = 0;
    for (; t < MDN_INSERT_TRIES; t++) {
      if (threadIdx.x == 0) {
        double V[3 * MDN_MAX_VAP_ATOMS];
        insert_vapor(x, q, nreb, t, x.trial, V);
        x.iscr[51] = 1;
      }
      __syncthreads();
      bool clash = false;
      for (int i = threadIdx.x; i < x.n_core && !clash; i += blockDim.x) {
        const double* cpos = x.c.x + 3 * i;
        for (int k = 0; k < av; k++) {
          double dx = x.trial[3 * k] - cpos[0], dy = x.trial[3 * k + 1] - cpos[1], dz = x.trial[3 * k + 2] - cpos[2];
          if (dx * dx + dy * dy + dz * dz < d2min) clash = true;
        }
      }
      for (int u = threadIdx.x; u < G * ag && !clash; u += blockDim.x) {
        const double* gp = a->slab_x + 3 * ((size_t)P->slab_off + (size_t)par * P->slab_cap * ag + u);
        const double g0 = __ldcg(gp), g1 = __ldcg(gp + 1), g2 = __ldcg(gp + 2);  /* moved this step by any CTA */
        for (int k = 0; k < av; k++) {
          double dx = x.trial[3 * k] - g0, dy = x.trial[3 * k + 1] - g1, dz = x.trial[3 * k + 2] - g2;
          if (dx * dx + dy * dy + dz * dz < d2min) clash = true;
        }
      }
      if (clash) x.iscr[51] = 0;
      __syncthreads();
      int ok = x.iscr[51];
      __syncthreads();
      if (ok) break;
    }
    if (threadIdx.x == 0) {
      size_t g = (size_t)P->mol_off + mi;
      if (t == MDN_INSERT_TRIES) {
        a->region[g] = 0; /* the entry waits for the next rebuild */
        deferred++;
      } else {
        a->region[g] = (unsigned char)((t << 2) | 1);
      }
    }
  }
  if (threadIdx.x == 0) x.iscr[52] = deferred;
  __syncthreads();
  int d = x.iscr[52];
  __syncthreads();
  return d;
}

__device__ __forceinline__ void make_pair(Ctx& x, cg::cluster_group& cl) {
  const RepParams* P = x.P;
  const KArgs* a = x.a;
  const int ag = P->a_g, av = P->a_v, par = x.D->parity, npar = par ^ 1;
  const int loop_pair = x.D->loop_pair, nreb = x.D->n_rebuilds;
  int* sc = x.iscr;
  /* updateInCenters: gas slab partition of this CTA, vapor core by rank 0 */
  {
    int lo, hi;
    partition(x, x.D->n_gas_in, &lo, &hi);
    for (int s = lo + threadIdx.x; s < hi; s += blockDim.x) {
      int m = a->slab_mol[gmol(P, par, s)];
      double sx[3] = {0, 0, 0}, sv[3] = {0, 0, 0};
      for (int at = 0; at < ag; at++) {
        size_t g = gatom(P, par, s, at);
        double mm = x.db[P->d_mass + x.ib[P->o_gas_type + at]];
        for (int k = 0; k < 3; k++) {
          sx[k] += a->slab_x[3 * g + k] * mm;
          sv[k] += a->slab_v[3 * g + k] * mm;
        }
      }
      double massInv = 1 / P->gas_com_mass;
      size_t g = (size_t)P->mol_off + 1 + m;
      for (int k = 0; k < 3; k++) {
        a->mol_x[3 * g + k] = sx[k] * massInv;
        a->mol_v[3 * g + k] = sv[k] * massInv;
      }
    }
    if (x.rank == 0)
      for (int s = threadIdx.x; s < x.D->n_vap_in; s += blockDim.x) {
        int m = a->vslab_mol[vmol(P, par, s)];
        double sx[3] = {0, 0, 0}, sv[3] = {0, 0, 0};
        for (int at = 0; at < av; at++) {
          int i = P->n_ion + s * av + at;
          double mm = x.db[P->d_mass + x.c.type[i]];
          for (int k = 0; k < 3; k++) {
            sx[k] += x.c.x[3 * i + k] * mm;
            sv[k] += x.c.v[3 * i + k] * mm;
          }
        }
        double massInv = 1 / P->vap_com_mass;
        size_t g = (size_t)P->mol_off + 1 + P->n_gas + m;
        for (int k = 0; k < 3; k++) {
          a->mol_x[3 * g + k] = sx[k] * massInv;
          a->mol_v[3 * g + k] = sv[k] * massInv;
        }
      }
  }
  /* the ion centre in the reference's summation order (MD::update_position
   * computed it just before check_pairlist); MD::MD's first make_pair and the
   * re-centring in MD::run use the stored entry instead */
  if (!a->keep_com) ion_centre_exact(x);
  if (x.rank == 0 && threadIdx.x == 0) {
    size_t g = (size_t)P->mol_off;
    for (int k = 0; k < 3; k++) {
      a->mol_x[3 * g + k] = x.D->ion_com[k];
      a->mol_v[3 * g + k] = x.D->ion_com[3 + k];
    }
  }
  __threadfence();
  cl.sync();
  double com[3] = {x.D->ion_com[0], x.D->ion_com[1], x.D->ion_com[2]};
  int mlo, mhi;
  partition(x, P->n_gas, &mlo, &mhi);
  int my_in = 0;
  double vmax2 = 0;
  /* vapor molecules (rank 0; events) */
  int my_vin = 0;
  if (threadIdx.x == 0) x.cand[MDN_INSERT_MAX_VAPOR] = 0;
  __syncthreads();
  if (x.rank == 0)
    for (int q = threadIdx.x; q < P->n_vap; q += blockDim.x) {
      int mi = 1 + P->n_gas + q;
      size_t g = (size_t)P->mol_off + mi;
      int was = a->region[g] & 1;
      if (was) {
        /* MD::Ovin / MD::Ovout log the centre before any change */
        double dx[3], dv[3];
        for (int k = 0; k < 3; k++) {
          dx[k] = a->mol_x[3 * g + k] - com[k];
          dv[k] = a->mol_v[3 * g + k] - x.D->ion_com[3 + k];
        }
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        int e = atomicAdd(a->n_events, 1);
        if (e < a->ev_cap) {
          DevEvent& ev = a->events[e];
          ev.replica = x.r;
          ev.molecule = q;
          ev.kind = r2 < P->RI2 ? 1 : 2;
          ev.step = x.D->step;
          for (int k = 0; k < 3; k++) { ev.dx[k] = dx[k]; ev.dv[k] = dv[k]; }
        } else {
          set_status(x, MDN_ST_EVENT_OVERFLOW);
        }
      }
      int f = classify_one(x, mi, P->vap_sigma, nreb, loop_pair, com, 1);
      my_vin += f & 1;
      const double* V = a->mol_v + 3 * g;
      double v2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2];
      vmax2 = fmax(vmax2, v2);
    }
  /* the vapor decisions (and their accepted draws) before any gas entry is
   * tested against them: every CTA takes rank 0's candidate list */
  my_vin = block_sum_i(my_vin, sc);
  if (x.rank == 0 && !(P->quirks & MDN_Q_BLIND_INSERT)) my_vin -= vapor_entries(x, nreb);
  __threadfence();
  cl.sync();
  if (x.rank != 0) {
    for (int k = threadIdx.x; k <= MDN_INSERT_MAX_VAPOR; k += blockDim.x) x.cand[k] = *cl.map_shared_rank(&x.cand[k], 0);
  }
  __syncthreads();
  /* free flight + classification of the gas molecules of this CTA's range */
  for (int q = mlo + threadIdx.x; q < mhi; q += blockDim.x) {
    int f = classify_one(x, 1 + q, P->gas_sigma, nreb, loop_pair, com, 0);
    my_in += f & 1;
    const double* V = a->mol_v + 3 * ((size_t)P->mol_off + 1 + q);
    double v2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2];
    vmax2 = fmax(vmax2, v2);
  }
  {
    const double* V = x.D->ion_com + 3;
    vmax2 = fmax(vmax2, V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
  }
  my_in = block_sum_i(my_in, sc);
  vmax2 = block_max_d(vmax2, x.dscr);
  __threadfence();
  int gin_base, gin_tot, vin_base, vin_tot;
  cluster_prefix(x, cl, &sc[43], my_in, &gin_base, &gin_tot);
  cluster_prefix(x, cl, &sc[44], my_vin, &vin_base, &vin_tot);
  /* vmax over the cluster */
  if (threadIdx.x == 0) x.dscr[45] = vmax2;
  cl.sync();
  double vm2 = 0;
  for (int k = 0; k < x.C; k++) vm2 = fmax(vm2, *cl.map_shared_rank(&x.dscr[45], k));
  cl.sync();
  const bool slab_over = gin_tot > P->slab_cap;
  const bool core_over = vin_tot > P->vcap || P->n_ion + vin_tot * av > a->nc_cap;
  /* new gas slab, ascending molecule index */
  int run = gin_base;
  for (int q0 = mlo; q0 < mhi; q0 += blockDim.x) {
    int q = q0 + threadIdx.x;
    int f = 0;
    if (q < mhi) f = a->region[(size_t)P->mol_off + 1 + q];
    int in = f & 1, tot;
    int off = block_exscan(in, sc, &tot);
    if (q < mhi) {
      size_t g = (size_t)P->mol_off + 1 + q;
      if (in && !slab_over) {
        int ns = run + off;
        double X[3 * MDN_MAX_GAS_ATOMS], V[3 * MDN_MAX_GAS_ATOMS];
        if (f & 2) {
          int os = a->slot[g];
          for (int at = 0; at < ag; at++) {
            size_t go = gatom(P, par, os, at);
            for (int k = 0; k < 3; k++) {
              /* the old slab slot may belong to another CTA, which moved
               * it this step: from L2 */
              X[3 * at + k] = __ldcg(a->slab_x + 3 * go + k);
              V[3 * at + k] = __ldcg(a->slab_v + 3 * go + k);
            }
          }
        } else {
          insert_gas(x, q, nreb, f >> 2, X, V);
        }
        for (int at = 0; at < ag; at++) {
          size_t gn = gatom(P, npar, ns, at);
          for (int k = 0; k < 3; k++) {
            a->slab_x[3 * gn + k] = X[3 * at + k];
            a->slab_v[3 * gn + k] = V[3 * at + k];
            a->slab_f[3 * gn + k] = 0.0;
          }
        }
        a->slab_mol[gmol(P, npar, ns)] = q;
        if (a->slab_ins) a->slab_ins[gmol(P, npar, ns)] = (f & 2) ? -1 : nreb + 1;
        a->slot[g] = ns;
      } else {
        a->slot[g] = -1;
      }
      a->region[g] = (unsigned char)in;
    }
    run += tot;
  }
  /* new vapor slab (rank 0), from the core copy (current positions); each
   * molecule reads its own old slot before overwriting it */
  if (x.rank == 0) {
    int runv = 0;
    for (int q0 = 0; q0 < P->n_vap; q0 += blockDim.x) {
      int q = q0 + threadIdx.x;
      int f = 0;
      if (q < P->n_vap) f = a->region[(size_t)P->mol_off + 1 + P->n_gas + q];
      int in = f & 1, tot;
      int off = block_exscan(in, sc, &tot);
      if (q < P->n_vap) {
        size_t g = (size_t)P->mol_off + 1 + P->n_gas + q;
        if (in && !core_over) {
          int ns = runv + off;
          double X[3 * MDN_MAX_VAP_ATOMS], V[3 * MDN_MAX_VAP_ATOMS];
          if (f & 2) {
            int os = a->slot[g];
            for (int at = 0; at < av; at++) {
              int i = P->n_ion + os * av + at;
              for (int k = 0; k < 3; k++) {
                X[3 * at + k] = x.c.x[3 * i + k];
                V[3 * at + k] = x.c.v[3 * i + k];
              }
            }
          } else {
            insert_vapor(x, q, nreb, f >> 2, X, V);
          }
          for (int at = 0; at < av; at++) {
            size_t gn = vatom(P, npar, ns, at);
            for (int k = 0; k < 3; k++) {
              a->vslab_x[3 * gn + k] = X[3 * at + k];
              a->vslab_v[3 * gn + k] = V[3 * at + k];
              a->vslab_f[3 * gn + k] = 0.0;
            }
            a->vslab_w[gn] = (f & 2) ? 0.0f : -1.0f;
          }
          a->vslab_mol[vmol(P, npar, ns)] = q;
          a->slot[g] = ns;
        } else {
          a->slot[g] = -1;
        }
        a->region[g] = (unsigned char)in;
      }
      runv += tot;
    }
  }
  __threadfence();
  cl.sync();
  /* new counters, identical in every CTA */
  if (threadIdx.x == 0) {
    if (slab_over && x.rank == 0) set_status(x, MDN_ST_SLAB_OVERFLOW);
    if (core_over && x.rank == 0) set_status(x, MDN_ST_CORE_OVERFLOW);
    x.D->parity = npar;
    x.D->n_gas_in = slab_over ? 0 : gin_tot;
    x.D->n_vap_in = core_over ? 0 : vin_tot;
    double vmax = sqrt(vm2);
    double lu = x.D->margin_length / (vmax * P->dt);
    x.D->loop_update = lu >= 2147483647.0 ? 2147483647 : (int)lu;
    x.D->loop_pair = 0;
    x.D->n_rebuilds = nreb + 1;
  }
  __syncthreads();
  /* reload the vapor part of the core from the new vapor slab */
  load_vapor(x);
  __syncthreads();
  core_weights_pos(x, true);
  relist(x, cl);
}

/* ------------------------------------------------------------------------- */
__device__ __forceinline__ void one_step(Ctx& x, cg::cluster_group& cl, bool eflag) {
  const RepParams* P = x.P;
  prof_start(x);
  core_kick(x);
  __syncthreads();
  if (x.D->nvt_mode == MDN_NVT_SCALE) {
    double T = ion_temperature(x);
    double ratio = sqrt(300.0 / T);
    for (int i = threadIdx.x; i < P->n_ion; i += blockDim.x)
      for (int k = 0; k < 3; k++) x.c.v[3 * i + k] *= ratio;
    __syncthreads();
  }
  const bool rebuild = x.D->loop_pair + 1 > x.D->loop_update;
  /* with gas-gas forces no gas molecule can take its force during its own
   * drift: they need every molecule's new position */
  const bool gg = kGG && (P->interactions & MDN_I_GG) && P->ggl_cap > 0;
  core_drift_shake(x, !rebuild && !gg, eflag);
  ion_centre(x);
  if (x.D->nvt_mode == MDN_NVT_NH) {
    double T = ion_temperature(x);
    if (threadIdx.x == 0) {
      int g = P->n_ion * 3;
      x.D->zeta += (T - x.D->nvt_T) * g * P->kb_real * 0.0001 * P->dt;
    }
    __syncthreads();
  }
  core_weights_pos(x, true);
  prof_end(x, MDN_PROF_CORE_INT);
  prof_start(x);
  if (threadIdx.x == 0) x.D->loop_pair += 1;
  __syncthreads();
  prof_end(x, MDN_PROF_GAS_INT);
  if (rebuild) {
    prof_start(x);
    make_pair(x, cl);
    prof_end(x, MDN_PROF_REBUILD);
  }
  if (gg) gas_gg_pass(x, cl, eflag, rebuild);
  if (rebuild || gg) {
    prof_start(x);
    gas_far_pass(x, eflag, true);
    __syncthreads();
    prof_end(x, MDN_PROF_REBUILD);
  }
  forces_and_kick(x, cl, eflag, true);
  if (x.D->nvt_mode == MDN_NVT_NH) {
    double Coeff = exp(-x.D->zeta * 0.5 * P->dt);
    for (int i = threadIdx.x; i < P->n_ion; i += blockDim.x)
      for (int k = 0; k < 3; k++) x.c.v[3 * i + k] *= Coeff;
    __syncthreads();
  }
  if (threadIdx.x == 0) x.D->step += 1;
  __syncthreads();
}

}  // namespace

#if defined(MDN_GG_TERMS) && defined(MDN_FP64_PAIRS)
#define MDN_ADVANCE_KERNEL mdn_advance_gg_fp64
#elif defined(MDN_GG_TERMS)
#define MDN_ADVANCE_KERNEL mdn_advance_gg
#elif defined(MDN_FP64_PAIRS)
#define MDN_ADVANCE_KERNEL mdn_advance_fp64
#else
#define MDN_ADVANCE_KERNEL mdn_advance
#endif
extern "C" __global__ void __launch_bounds__(512, 1) MDN_ADVANCE_KERNEL(KArgs a) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ RepParams sP;
  __shared__ RepDyn sD;
  __shared__ int s_job;
  __shared__ int iscr[64];
  __shared__ double dscr[64];
  __shared__ int cand[MDN_INSERT_MAX_VAPOR + 1];
  __shared__ double trial[3 * MDN_MAX_VAP_ATOMS];

  Ctx x;
  x.a = &a;
  x.P = &sP;
  x.D = &sD;
  x.rank = (int)cl.block_rank();
  x.C = (int)cl.num_blocks();
  x.iscr = iscr;
  x.dscr = dscr;
  x.cand = cand;
  x.trial = trial;
  /* carve the dynamic shared memory */
  {
    unsigned char* p = dsm;
    const int nc = a.nc_cap;
    auto take = [&](size_t bytes) { unsigned char* q = p; p += (bytes + 15) & ~(size_t)15; return q; };
    x.c.acc = (long long*)take(sizeof(long long) * 3 * nc);
    x.c.chunk = (unsigned*)take(sizeof(unsigned) * 9 * nc);
    x.c.x = (double*)take(sizeof(double) * 3 * nc);
    x.c.v = (double*)take(sizeof(double) * 3 * nc);
    x.c.f = (double*)take(sizeof(double) * 3 * nc);
    x.c.pos = (float4*)take(sizeof(float4) * nc);
    x.c.w = (float*)take(sizeof(float) * nc);
    x.c.type = (int*)take(sizeof(int) * nc);
    x.c.mol = (int*)take(sizeof(int) * nc);
    x.c.excl = (unsigned*)take(sizeof(unsigned) * a.excl_cap);
    x.c.ljA = (float*)take(sizeof(float) * a.nt_cap * a.nt_cap);
    x.c.ljB = (float*)take(sizeof(float) * a.nt_cap * a.nt_cap);
    x.c.c2 = (double*)take(sizeof(double) * a.nt_cap);
  }
  /* the chunk sums start at zero and every core_reduce leaves them so */
  for (int q = threadIdx.x; q < 9 * a.nc_cap; q += blockDim.x) x.c.chunk[q] = 0;
  __syncthreads();
  for (;;) {
    if (x.rank == 0 && threadIdx.x == 0) s_job = atomicAdd(a.job_counter, 1);
    cl.sync();
    const int job = *cl.map_shared_rank(&s_job, 0);
    cl.sync();
    if (job >= a.n_jobs) break;
    const int r = a.job_order[job];
    x.r = r;
    if (threadIdx.x == 0) {
      sP = a.P[r];
      sD = a.D[r];
      sD.nvt_mode = a.ctl_mode[r];
      sD.nvt_T = a.ctl_T[r];
    }
    __syncthreads();
    x.ib = a.iblob + sP.iblob_off;
    x.db = a.dblob + sP.dblob_off;
    const bool fatal = (a.status[r] & MDN_ST_FATAL) != 0;
    const bool fits = sP.n_types <= a.nt_cap && sP.n_ion * sP.excl_words <= a.excl_cap &&
                      sP.n_ion + sD.n_vap_in * sP.a_v <= a.nc_cap;
    if (fatal || !fits) {
      if (!fits && x.rank == 0 && threadIdx.x == 0) atomicOr(&a.status[r], MDN_ST_CORE_OVERFLOW);
      __syncthreads();
      continue;
    }
    /* tables */
    const int nt = sP.n_types;
    for (int q = threadIdx.x; q < nt * nt; q += blockDim.x) {
      x.c.ljA[q] = (float)x.db[sP.d_ljA + q];
      x.c.ljB[q] = (float)x.db[sP.d_ljB + q];
    }
    for (int q = threadIdx.x; q < nt; q += blockDim.x) x.c.c2[q] = x.db[sP.d_c2 + q];
    for (int q = threadIdx.x; q < sP.n_ion * sP.excl_words; q += blockDim.x) x.c.excl[q] = (unsigned)x.ib[sP.o_excl + q];
    load_ion(x);
    load_vapor(x);
    if (threadIdx.x < MDN_PROF_N) s_prof[threadIdx.x] = 0;
    __syncthreads();
    const long long job_t0 = clock64();
    if (a.mode == MDN_MODE_STEP) {
      for (long long s = 0; s < a.n_steps; s++) {
        bool eflag = a.energy_mode == 2 || (a.energy_mode == 1 && s == a.n_steps - 1);
        one_step(x, cl, eflag);
      }
    } else if (a.mode == MDN_MODE_FORCES) {
      /* the ion centre serves only as the origin of the FP32 coordinates here */
      double keep[6];
      for (int k = 0; k < 6; k++) keep[k] = sD.ion_com[k];
      __syncthreads();
      ion_centre(x);
      core_weights_pos(x, false);
      gas_gg_pass(x, cl, true, false);
      gas_far_pass(x, true, false);
      __syncthreads();
      forces_and_kick(x, cl, true, false);
      if (threadIdx.x == 0)
        for (int k = 0; k < 6; k++) sD.ion_com[k] = keep[k];
      __syncthreads();
    } else if (a.mode == MDN_MODE_MAKE_PAIR) {
      core_weights_pos(x, false);
      make_pair(x, cl);
    } else if (a.mode == MDN_MODE_RELIST) {
      relist(x, cl);
    }
    __syncthreads();
    if (a.prof && threadIdx.x == 0) {
      s_prof[MDN_PROF_TOTAL] = clock64() - job_t0;
      for (int k = 0; k < MDN_PROF_N; k++)
        atomicAdd((unsigned long long*)&a.prof[(size_t)r * MDN_PROF_N + k], (unsigned long long)s_prof[k]);
    }
    store_core(x);
    __syncthreads();
    if (x.rank == 0 && threadIdx.x == 0) {
      a.D[r] = sD;
      if (a.mode == MDN_MODE_STEP) {
        size_t g = (size_t)sP.mol_off;
        for (int k = 0; k < 3; k++) {
          a.mol_x[3 * g + k] = sD.ion_com[k];
          a.mol_v[3 * g + k] = sD.ion_com[3 + k];
        }
      }
    }
    __threadfence();
    __syncthreads();
  }
}
