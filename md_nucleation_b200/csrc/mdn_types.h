/*
 * mdn_types.h -- layout shared by the host side (engine.cu) and the device
 * kernels (advance.cu) of the B200 engine.
 *
 * Device memory of a handle holds R replicas in flat pools.  Per replica:
 *   RepParams   read-only sizes, run parameters and offsets into the pools
 *   RepDyn      mutable counters (MD::loopPair, MD::loop_update, zeta, ...)
 *   ion atoms   x, v, f (FP64, xyz interleaved)
 *   molecules   centre x, v (FP64) of molecule 0 (the ion), the gas and the
 *               vapor, in the reference's order; region flag; slab slot
 *   gas slab    the atoms of the in-domain gas molecules, ascending molecule
 *               index (the order of Variables::gas_in), two buffers that the
 *               rebuild ping-pongs between
 *   vapor slab  the atoms of the in-domain vapor molecules (the "core"
 *               together with the ion), two buffers
 *   lists       gas-ion and gas-vapor pair lists of the "near" gas molecules
 *               (those with a non-empty list), CSR by slab slot
 *   blobs       per-replica topology (int) and coefficient (double) tables
 */
#ifndef MDN_TYPES_H
#define MDN_TYPES_H

#include <stdint.h>

#include "mdn.h"

#define MDN_MAX_GAS_ATOMS 2
#define MDN_MAX_VAP_ATOMS 8
#define MDN_MAX_TYPES 64
#define MDN_SHAKE_MAX_SWEEPS 1000

/* forces accumulate as int64 in units of 2^-40 kcal/mol/A (|F| up to 8.4e6 fits;
 * a long-range pair force of 1e-6 keeps 1e-6 relative resolution); energies in
 * 2^-36 kcal/mol (|U| up to 1.3e8 fits) */
#define MDN_FIX_SCALE 1099511627776.0
#define MDN_FIX_INV (1.0 / 1099511627776.0)
#define MDN_EFIX_SCALE 68719476736.0
#define MDN_EFIX_INV (1.0 / 68719476736.0)
#define MDN_FIX_LIMIT 2.0e6 /* |force component| above this flags saturation (a warning) */

/* phases of the per-replica cycle accounting (mdn_profile) */
#define MDN_PROF_TOTAL 0
#define MDN_PROF_CORE_INT 1   /* kick, thermostat, drift, SHAKE, centre, weights */
#define MDN_PROF_GAS_INT 2    /* gas kick/drift (+ far-molecule forces)          */
#define MDN_PROF_REBUILD 3    /* make_pair                                       */
#define MDN_PROF_NEAR 4       /* near gas molecules: gas-ion, gas-vapor          */
#define MDN_PROF_BONDED 5     /* core bonded terms                               */
#define MDN_PROF_PAIRS 6      /* core pair terms                                 */
#define MDN_PROF_REDUCE 7     /* core force sums, core kick                      */
#define MDN_PROF_N 8

/* kernel modes */
#define MDN_MODE_STEP 0       /* advance n_steps                                   */
#define MDN_MODE_FORCES 1     /* recompute forces/energies, no motion               */
#define MDN_MODE_MAKE_PAIR 2  /* MD::make_pair now                                  */
#define MDN_MODE_RELIST 3     /* pair lists from the current centres, no classification */

typedef struct RepParams {
  /* sizes */
  int n_ion, a_g, a_v, n_gas, n_vap, n_types;
  unsigned interactions, quirks;
  int gas_kind, force_mode;
  int n_ion_bonds, n_ion_angles, n_ion_dih, n_ion_rigid, n_ion_colors;
  int n_gas_bonds, n_gas_rigid;
  int n_vap_bonds, n_vap_angles, n_vap_dih, n_vap_rigid, n_vap_colors;
  int excl_words;
  int slab_cap, vcap, near_cap, gil_cap, gvl_cap;
  /* offsets inside the int blob */
  int o_ion_type, o_ion_bmh, o_ion_bonds, o_ion_angles, o_ion_dih, o_ion_rigid, o_ion_color, o_excl;
  int o_gas_type, o_gas_bonds, o_gas_rigid;
  int o_vap_type, o_vap_bonds, o_vap_angles, o_vap_dih, o_vap_rigid, o_vap_color;
  int o_dih_multi;
  /* SHAKE constraints in groups of coupled ones (sharing atoms), at most 3
   * per group, solved together (shake_group); 0 groups = colour sweeps */
  int n_ion_groups, o_ion_grp, o_ion_gstart;
  int n_vap_groups, o_vap_grp, o_vap_gstart;
  /* offsets inside the double blob */
  int d_bond, d_angle, d_dih, d_ljA, d_ljB, d_mass, d_c2;
  int d_ion_q, d_gas_x, d_gas_q, d_vap_x, d_vap_q;
  int d_ion_cons, d_gas_cons, d_vap_cons; /* per SHAKE constraint: d^2, 1/m_i, 1/m_j */
  int ggl_cap;                   /* gas-gas list entries (both directions), 0 without gg */
  /* run parameters */
  double dt, box, ml2, ri2, RI2, rcenter, overlap, margin;
  double coeff;                  /* 0.5*dt*4.184e-4 (src/verlet.cpp:49) */
  double gas_com_mass, vap_com_mass, gas_sigma, vap_sigma, ion_msum;
  double qqrd2e, kb_real, real_to_kcalmol;
  double efield[3];
  unsigned key0, key1;
  /* pool offsets (elements) */
  long long ion_off, mol_off, slab_off, vslab_off, near_off, gil_off, gvl_off, ggl_off;
  long long slab_moff, vslab_moff; /* molecule offsets of the two slabs */
  long long iblob_off, dblob_off;
  double work;                   /* cost estimate for the job order */
} RepParams;

typedef struct RepDyn {
  int loop_pair, loop_update, n_rebuilds, n_gas_in;
  int n_vap_in, parity, status, n_near;
  int gi_count, gv_count, nvt_mode, gg_count; /* gg_count: unordered gas-gas pairs */
  long long step;
  double zeta, margin_length, nvt_T, pad2;
  double ion_com[6];
} RepDyn;

/* one vapor in/out event (MD::Ovin / MD::Ovout) */
typedef struct DevEvent {
  int replica, molecule, kind, pad;
  long long step;
  double dx[3], dv[3];
} DevEvent;

typedef struct KArgs {
  const RepParams* P;
  RepDyn* D;
  const int* iblob;
  const double* dblob;
  double *ion_x, *ion_v, *ion_f;
  double *mol_x, *mol_v;
  unsigned char* region;
  int* slot;
  double *slab_x, *slab_v, *slab_f;
  int* slab_mol;
  double *vslab_x, *vslab_v, *vslab_f;
  float* vslab_w;
  int* vslab_mol;
  int* near_list;          /* slab slots of near molecules, ascending          */
  int* near_gi;            /* [slab slot] start of its gi entries (-1 = none)  */
  int* near_gv;            /* [slab slot] start of its gv entries              */
  unsigned short *gil_n, *gvl_n; /* [slab slot] entry counts                   */
  unsigned short *gil, *gvl;
  /* gas-gas (gg LJ, corrected form): for every slab molecule the slab slots
   * of its partners in both directions, CSR by slab slot; the gas-gas force
   * of each atom; the rebuild number that inserted the molecule (its taper
   * weights are 0 on the step of that rebuild); all NULL without gg */
  int *ggl_start, *ggl_n, *ggl;
  double* slab_fgg;
  int* slab_ins;
  long long* energy;       /* 8 per replica, fixed point                       */
  DevEvent* events;
  int* n_events;
  int ev_cap;
  int* status;             /* [n_replicas] MDN_ST_* bits, only ever OR-ed      */
  const int* ctl_mode;     /* [n_replicas] thermostat mode (MDN_NVT_*)         */
  const double* ctl_T;     /* [n_replicas] thermostat target (K)               */
  const int* job_order;
  int n_jobs;
  int* job_counter;
  long long n_steps;
  int energy_mode, mode;
  int keep_com;            /* MAKE_PAIR: classify against the stored ion centre */
  unsigned term_mask;
  long long* prof;         /* NULL, or [n_replicas][MDN_PROF_N] SM cycles per phase */
  int nc_cap;              /* core atoms the shared memory holds               */
  int nt_cap;              /* atom types the shared memory holds               */
  int excl_cap;            /* exclusion words the shared memory holds          */
  int colors_cap;
} KArgs;

/* A handle's device arrays that the snapshot kernels read (filled by
 * engine.cu for the allocation-free snapshot); stream is a cudaStream_t. */
typedef struct {
  const RepParams* P;
  const RepDyn* D;
  const int* iblob;
  int R;
  int dev;
  const double *ion_x, *ion_v, *slab_x, *slab_v, *vslab_x, *vslab_v;
  const long long* energy;
  void* stream;
} SnapshotArgs;

#endif
