/*
 * mdn.h -- C ABI of the B200 (sm_100a) engine for the per-step hot path of
 * MD_nucleation: effective-domain molecular dynamics of vapor nucleation
 * around an ion (the "seed"), many independent replicas per GPU.
 *
 * The reference program drives one replica through `class MD`
 * (src/md.hpp:9-114).  Its per-step work is `MD::verlet` (src/verlet.cpp:20-39)
 * plus the pair-list rebuild `MD::make_pair` (src/pairList/pairlist.cpp:16-49)
 * and the force plugins derived from `class Potential`
 * (src/potential/basePotential.hpp:5-17), registered by `MD::setPotential`
 * (src/initialization/setPotential.cpp:7-111).  This library replaces that
 * step for a batch of replicas: a host keeps parsing, initial placement and
 * output, hands the state over once through mdn_create / mdn_upload_state,
 * and advances it with mdn_step.
 *
 * Conventions: every function returns an int status (MDN_OK = 0, negative =
 * error) and never aborts; mdn_last_error() gives the message of the last
 * failure on the calling thread.  Units are the reference's "real" units:
 * Angstrom, fs, g/mol, kcal/mol, e.  All arrays are plain host pointers;
 * nothing in this header depends on CUDA or torch types.  A handle is not
 * re-entrant: one host thread drives one handle.
 */
#ifndef MDN_H
#define MDN_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDN_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define MDN_OK             0
#define MDN_ERR_ARG       -1  /* bad argument or descriptor */
#define MDN_ERR_CUDA      -2  /* a CUDA call failed */
#define MDN_ERR_NO_DEVICE -3  /* no CUDA device (or the library was built without one) */
#define MDN_ERR_CAPACITY  -4  /* a descriptor exceeds a compiled limit */
#define MDN_ERR_REPLICA   -5  /* one or more replicas raised a status bit, see mdn_get_status */

/* ---- per-replica status bits (mdn_get_status) ---------------------------- */
#define MDN_ST_SLAB_OVERFLOW   0x0001 /* more in-domain gas molecules than the slab holds */
#define MDN_ST_CORE_OVERFLOW   0x0002 /* more in-domain vapor atoms than the core holds */
#define MDN_ST_LIST_OVERFLOW   0x0004 /* gas-ion / gas-vapor / gas-gas pair list full
                                         (at most 64,511 gas molecules with list entries) */
#define MDN_ST_SHAKE_NOCONV    0x0008 /* SHAKE hit its iteration cap */
#define MDN_ST_NONFINITE       0x0010 /* a non-finite force, position or velocity */
#define MDN_ST_FIXED_OVERFLOW  0x0020 /* a force left the 64-bit fixed-point range */
#define MDN_ST_EVENT_OVERFLOW  0x0040 /* vapor in/out event log full (events dropped) */
/* Fatal bits freeze the replica (later steps skip it) and make mdn_step
 * return MDN_ERR_REPLICA; the others are warnings the replica runs on with:
 * a molecule entering the domain is placed without an overlap test
 * (src/pairList/updateGasIn.cpp:51-98), as in the reference, so an entry on
 * top of another atom produces a huge force -- the reference carries on with
 * it, the engine carries on with its force terms saturated at 2^21
 * kcal/mol/A (each gas pair term; for the core's own pairs, the sum of each
 * 32 x 32 tile on an atom). */
#define MDN_ST_FATAL (MDN_ST_SLAB_OVERFLOW | MDN_ST_CORE_OVERFLOW | MDN_ST_LIST_OVERFLOW | MDN_ST_NONFINITE)

/* ---- Interactions keywords (src/initialization/setCondition.cpp:186-228) - */
#define MDN_I_GI           0x0001 /* gi LJ                     (PotentialGasIon)     */
#define MDN_I_VI           0x0002 /* vi LJcoul                 (PotentialVaporIon)   */
#define MDN_I_VV           0x0004 /* vv LJcoul                 (PotentialVaporVapor) */
#define MDN_I_GV           0x0008 /* gv LJ                     (PotentialVaporGas)   */
#define MDN_I_GG           0x0010 /* gg LJ, corrected form     (PotentialGasGas)     */
#define MDN_I_AMBER        0x0020 /* ion AMBER                 (PotentialAMBER)      */
#define MDN_I_BMH          0x0040 /* ion Born-Mayer-Huggins-NaCl (PotentialBorn)     */
#define MDN_I_GAS_INTRA    0x0080 /* gas bonds                 (PotentialGasIntra)   */
#define MDN_I_VAPOR_INTRA  0x0100 /* vapor bonds/angles/dihedrals (PotentialVaporIntra) */
#define MDN_I_EFIELD       0x0200 /* uniform field on ion charges (PotentialEfield)  */
#define MDN_I_SHAKE        0x1000 /* "SHAKE H": X-H bonds are constraints */

/* ---- reference behaviours reproduced on request (mdn_options.quirks) ------
 * Each bit reproduces one behaviour of the reference that a corrected
 * implementation would change.  MDN_Q_ALL is the default, so that results
 * match the reference; clearing a bit selects the corrected behaviour.     */
#define MDN_Q_GV_GAS_COUNT   0x01 /* gv inner loop runs over the gas atom count
                                     (src/potential/VaporGas.cpp:15)          */
#define MDN_Q_GAS_ROT_ZY     0x02 /* gas insertion rotates (x, y, y), not (x, y, z)
                                     (src/pairList/updateGasIn.cpp:85,92)     */
#define MDN_Q_N2_ROT_VYVZ    0x04 /* N2 insertion spin puts v_rot on both y and z
                                     (src/pairList/updateGasIn.cpp:69-78)     */
#define MDN_Q_ENERGY_BUCKETS 0x08 /* vapor bond/angle energy -> Ugas, vapor dihedral
                                     -> Uion (src/potential/compute_intra.cpp:82,124,194) */
#define MDN_Q_SHAKE_NO_VCORR 0x10 /* SHAKE moves positions only, no velocity
                                     correction (src/shake.cpp:6-92)          */
#define MDN_Q_BLIND_INSERT   0x20 /* a molecule entering the domain is placed with one
                                     random rotation and no overlap test
                                     (src/pairList/updateGasIn.cpp:51-98,
                                     updateVaporIn.cpp:55-82).  Cleared: the rotation is
                                     re-drawn (up to 4 draws) until no atom lies within
                                     2 A of an ion or in-domain vapor atom (and, for an
                                     entering vapor molecule, of an in-domain gas atom),
                                     else the entry waits for the next rebuild.  At the
                                     gas densities of 20,000 in-domain atoms the blind
                                     form places atoms <0.5 A apart every few hundred
                                     steps. */
#define MDN_Q_ALL            0x2F /* MDN_Q_SHAKE_NO_VCORR is opt-in: the reference never
                                     calls its SHAKE (src/verlet.cpp:24), and the
                                     position-only form heats the system */
#define MDN_INSERT_MIN_DIST 2.0  /* A, the overlap test of the checked insertion */
#define MDN_INSERT_TRIES    4
#define MDN_INSERT_MAX_VAPOR 256 /* vapor entries tested per rebuild; later ones wait
                                    for the next rebuild */

/* energy buckets, the order of `struct Potentials` (src/struct.hpp:29-38) */
#define MDN_U_ION 0
#define MDN_U_GAS 1
#define MDN_U_VAP 2
#define MDN_U_GI  3
#define MDN_U_GG  4
#define MDN_U_VG  5
#define MDN_U_VI  6
#define MDN_U_VV  7
#define MDN_N_ENERGY 8

/* gas kinds, MD::gastype after readCondFile (src/initialization/setCondition.cpp:48-113) */
#define MDN_GAS_HE     1
#define MDN_GAS_N2     2
#define MDN_GAS_N2MONO 3
#define MDN_GAS_AR     4

/* thermostat modes for the relaxation phase (src/nvt.cpp) */
#define MDN_NVT_OFF   0   /* MD::setNVE */
#define MDN_NVT_SCALE 1   /* MD::velocity_scaling (target 300 K) */
#define MDN_NVT_NH    2   /* MD::nosehoover_zeta / nosehoover_ion */

/* One molecule kind: the ion, or the template of a gas or vapor molecule.
 * Indices are 0-based; types index the replica's type tables.             */
typedef struct mdn_topology {
  int           n_atoms;
  const int*    type;       /* [n_atoms] atom type                                  */
  const double* charge;     /* [n_atoms] partial charge (e)                         */
  const double* x;          /* [3*n_atoms] ion: coordinates; gas/vapor: template   */
  int n_bonds;     const int* bonds;      /* [3*n] i, j, bond type               */
  int n_rigid;     const int* rigid;      /* [3*n] i, j, bond type (SHAKE pairs) */
  int n_angles;    const int* angles;     /* [4*n] i, j, k, angle type           */
  int n_dihedrals; const int* dihedrals;  /* [5*n] i, j, k, l, dihedral type     */
} mdn_topology;

/* Everything one replica needs: the content of `Variables` after
 * MD::MD (src/initialization/md.cpp:8-40), in flat arrays.               */
typedef struct mdn_replica_desc {
  /* type tables (Variables::atypes/btypes/ctypes/dtypes, src/variables.hpp:98-101) */
  int n_atom_types;  const double* atom_mass; const double* atom_eps; const double* atom_sigma;
  int n_bond_types;  const double* bond_coeff;     /* [2*n] K (kcal/mol/A^2), r0 (A)         */
  int n_angle_types; const double* angle_coeff;    /* [2*n] K (kcal/mol/rad^2), theta0 (rad) */
  int n_dihedral_types; const int* dihedral_multi; /* [n] terms per type (<= 3)              */
  const double* dihedral_coeff;                    /* [15*n] per term: K, n, d(deg), cos d, sin d */
  /* the ion (seed) */
  mdn_topology  ion;
  const double* ion_v;          /* [3*ion.n_atoms] initial velocities (A/fs)             */
  const int*    ion_bmh_type;   /* [ion.n_atoms] Born-Mayer-Huggins row: 0 = Na, 1 = Cl  */
  /* gas species */
  mdn_topology  gas;
  int           gas_kind;       /* MDN_GAS_*                                             */
  double        gas_com_mass;   /* molecule mass dividing the centre of mass (vars->mass) */
  double        gas_mb_mass;    /* kg per molecule for Maxwell-Boltzmann draws (pp->mgas) */
  /* vapor species */
  mdn_topology  vapor;
  double        vapor_com_mass;
  double        vapor_mb_mass;
  /* molecules (centres of mass, reference order: gas 0..n_gas-1, then vapor) */
  int n_gas;   const double* gas_x;   const double* gas_v;   /* [3*n_gas]   */
  int n_vapor; const double* vapor_x; const double* vapor_v; /* [3*n_vapor] */
  /* run parameters */
  double dt;          /* fs                                          */
  double temperature; /* K                                           */
  double box;         /* cubic box edge d_size (A)                   */
  double cutoff;      /* CUTOFF (A); lists use (CUTOFF+MARGIN)^2     */
  double margin;      /* MARGIN (A)                                  */
  double r_inter;     /* effective-domain radius Rinter (A), 100     */
  double overlap;     /* taper shell width Overlap (A), 10           */
  unsigned int interactions;        /* MDN_I_* bits */
  int    nvt_mode;                  /* MDN_NVT_*    */
  double nvt_temperature;           /* Nose-Hoover target (pp->Tnh_ion) */
  double efield[3];                 /* Ecoeff for MDN_I_EFIELD */
  unsigned long long seed;          /* counter-based RNG key of this replica */
  /* optional LJ parameters per type pair, [n_atom_types^2] row-major and
   * symmetric, used instead of the Lorentz-Berthelot mixing of
   * Variables::setCrossPotentials (src/initialization/setCrossPotential.cpp:4-23);
   * NULL = mixing.  The parameters of the gradient harness (mdn_adjoint). */
  const double* pair_eps;
  const double* pair_sigma;
} mdn_replica_desc;

typedef struct mdn_options {
  unsigned int quirks;       /* MDN_Q_* bits to reproduce (default MDN_Q_ALL)          */
  int force_mode;            /* 0: FP32 pair math, int64 fixed-point sums (default);
                                1: FP64 pair math, int64 fixed-point sums            */
  int cluster_size;          /* CTAs cooperating on one replica (1..8); 0 = automatic   */
  int threads;               /* threads per CTA (32..512, multiple of 32); 0 = 512      */
  int steps_per_launch;      /* steps advanced per kernel launch; 0 = whole mdn_step    */
  int use_graph;             /* ignored: one launch already advances every step of an
                                mdn_step call                                          */
  double capacity_factor;    /* slab / list headroom over the expected counts (>= 1)   */
  int device;                /* CUDA device ordinal                                     */
} mdn_options;

typedef struct mdn_handle mdn_handle;

/* Sizes and counters of one replica. */
typedef struct mdn_replica_info {
  int n_ion, gas_atoms, vapor_atoms;   /* atoms in the ion / a gas / a vapor molecule */
  int n_gas, n_vapor;                  /* molecules                                  */
  int n_gas_in, n_vapor_in;            /* molecules inside the effective domain      */
  int loop_pair, loop_update;          /* MD::loopPair, MD::loop_update              */
  int n_rebuilds;
  long long step;                      /* steps advanced since creation              */
  int status;                          /* MDN_ST_* bits                              */
  int gi_pairs, gv_pairs, gg_pairs;    /* current pair-list sizes                    */
} mdn_replica_info;

/* Full state of one replica in the reference's layout (Variables, src/variables.hpp).
 * Molecule index 0 is the ion, 1..n_gas the gas, then the vapor (group[0..2]).
 * Atom rows of molecules outside the effective domain are not used: download
 * leaves them untouched and upload ignores them.                           */
typedef struct mdn_state {
  double* ion_x;   double* ion_v;   double* ion_f;     /* [3*n_ion]              */
  double* mol_x;   double* mol_v;                      /* [3*(1+n_gas+n_vapor)]  */
  unsigned char* region;                               /* [1+n_gas+n_vapor]      */
  double* gas_ax;  double* gas_av;  double* gas_af;    /* [3*gas_atoms*n_gas]    */
  double* vap_ax;  double* vap_av;  double* vap_af;    /* [3*vapor_atoms*n_vapor]*/
  double* vap_w;                                       /* [vapor_atoms*n_vapor] taper weights */
  int    loop_pair, loop_update;
  double zeta;
  double margin_length;
} mdn_state;

/* A vapor molecule that stayed in (kind 1) or left (kind 2) the domain at a
 * rebuild: the rows MD::Ovin / MD::Ovout append (src/output/output.cpp:44-65). */
typedef struct mdn_event {
  int replica, molecule, kind, pad;
  long long step;
  double dx[3], dv[3];   /* relative to the ion centre of mass */
} mdn_event;

/* ---- lifecycle ------------------------------------------------------------ */
int  mdn_abi_version(void);
void mdn_default_options(mdn_options* opt);
const char* mdn_last_error(void);
int  mdn_device_count(int* n);

/* Allocates device memory for n replicas, uploads them and performs the
 * initial MD::make_pair (src/initialization/md.cpp:34): every molecule starts
 * outside the domain, those within the sphere are inserted.                */
int  mdn_create(const mdn_replica_desc* descs, int n_replicas, const mdn_options* opt,
                mdn_handle** out);
void mdn_destroy(mdn_handle* h);

/* ---- stepping ------------------------------------------------------------- */
/* Advances every replica by n_steps calls of MD::verlet, rebuilding the
 * effective domain on the device whenever MD::check_pairlist would.
 * energy_mode: 0 = no energies, 1 = energies of the last step (eflag on the
 * last step, as MD::run sets it), 2 = energies summed over every step.   */
int  mdn_step(mdn_handle* h, long long n_steps, int energy_mode);
/* MD::make_pair for every replica now, classifying against the ion centre
 * of the current positions. */
int  mdn_make_pair(mdn_handle* h);
/* Re-centres every replica on its ion (src/run.cpp:42-53).  compat = 1 keeps
 * the reference's effect (only the ion centre entry is zeroed); compat = 0
 * shifts every position.  Then performs the MD::make_pair that MD::run calls
 * next (src/run.cpp:54), against the centre entry as the shift left it, so
 * no mdn_make_pair follows it.                                              */
int  mdn_recenter(mdn_handle* h, int compat);
/* Thermostat of one replica (replica < 0: all); MDN_NVT_OFF is MD::setNVE. */
int  mdn_set_nvt(mdn_handle* h, int replica, int mode, double temperature);
/* Thermostat modes and targets of every replica from host arrays
 * ([n_replicas] each; page-locked buffers make the copy asynchronous). */
int  mdn_set_nvt_batch(mdn_handle* h, const int* mode, const double* temperature);
/* Recomputes forces (and energies) on the current positions without moving
 * anything; term_mask selects MDN_I_* terms (0 = all enabled terms).      */
int  mdn_compute_forces(mdn_handle* h, unsigned int term_mask);

/* ---- results -------------------------------------------------------------- */
int  mdn_energies(mdn_handle* h, double* U);          /* [8*n_replicas], MDN_U_* order */
int  mdn_get_status(mdn_handle* h, int* status);      /* [n_replicas] MDN_ST_* bits    */
int  mdn_clear_status(mdn_handle* h);
int  mdn_replica_info_get(mdn_handle* h, int replica, mdn_replica_info* info);
int  mdn_download_state(mdn_handle* h, int replica, mdn_state* s);
int  mdn_upload_state(mdn_handle* h, int replica, const mdn_state* s);
/* Pair lists as (molecule, partner) rows: kind 0 = gas-ion (partner = ion
 * atom), 1 = gas-vapor (partner = vapor molecule index), 2 = gas-gas.
 * Molecule indices are 0-based within the gas / vapor groups.             */
int  mdn_pair_list(mdn_handle* h, int replica, int kind, int* pairs, int capacity, int* count);
/* In-domain atoms for the OVITO dump (MD::export_dump_close,
 * src/output/output.cpp:133-170), molecule order, ion first.            */
int  mdn_in_domain(mdn_handle* h, int replica, int capacity, int* count,
                   int* type, double* x, double* v);
/* Every replica's in-domain atoms plus the energies of the last mdn_step, in
 * one batched copy (device-side compaction, then one copy per array): the
 * feed of the OVITO dump and the energy logs of MD::display
 * (src/output/output.cpp:68-170) for the whole batch.  offset[r]..offset[r+1]
 * are the rows of replica r (ion atoms, then gas atoms of in-domain molecules
 * in ascending molecule order, then vapor atoms); type/x/v hold `capacity`
 * rows (x, v: 3 doubles per row); U: [8*n_replicas] or NULL.  Host buffers
 * from mdn_host_alloc make the copies asynchronous.  Returns
 * MDN_ERR_CAPACITY, with offset filled, when capacity is too small.        */
int  mdn_snapshot(mdn_handle* h, long long* offset, long long capacity, int* type, double* x, double* v,
                  double* U);
/* mdn_snapshot without any device allocation.  No counterpart in the
 * reference (its dump loop reads host memory).  mdn_snapshot allocates its
 * device staging on its first call, sized for every replica's largest
 * possible domain (hundreds of MB for a large batch).  A program that has
 * handed all free device memory to its own pool, or that runs under a fixed
 * device-memory budget, cannot let a dump taken late in a run allocate, or
 * fail for lack of memory.  This call stages the rows in a fixed array that
 * the library holds on each device until the process exits:
 * MDN_NOALLOC_MAX_ROWS rows (52 bytes each) and MDN_NOALLOC_MAX_REPLICAS
 * replicas, 3.4 MB in all.  A larger snapshot, or a larger batch, returns
 * MDN_ERR_CAPACITY and says so in mdn_last_error (offset filled when the
 * replica count fits); use mdn_snapshot for those.  The first mdn_create on
 * a device is where the array is loaded (and its 3.4 MB allocated) and
 * looked up, together with the snapshot kernels, once per device per
 * process; this call itself then loads nothing.  Every call in the process
 * shares the one array per device: calls that overlap in time on the same
 * device, from different threads or handles, race and may return each
 * other's rows.  Nothing in the array has to start at zero: each call writes
 * every offset and every row it copies back.  Arguments and results as
 * mdn_snapshot. */
#define MDN_NOALLOC_MAX_ROWS     65536
#define MDN_NOALLOC_MAX_REPLICAS 1024
int  mdn_snapshot_noalloc(mdn_handle* h, long long* offset, long long capacity, int* type, double* x,
                          double* v, double* U);
/* ---- gradient harness (no counterpart in the reference) -------------------
 * Sensitivities of an ion-vapor objective over a window of MD steps of one
 * replica to the gas-ion and vapor-ion LJ parameters and to a scale of the
 * ion's charges.  The objective is
 *   J = (1/n) sum_{t=1..n} [ w_energy * U_vi(x_t) + w_count * sum_m S(|c_m - c_ion|) ]
 * with U_vi the ion-vapor LJ + Coulomb energy (PotentialVaporIon's Uvi,
 * src/potential/VaporIon.cpp:5-43), c_m the centre of in-domain vapor
 * molecule m, c_ion the ion centre and S(r) = 1 / (1 + exp((r - R0) / W))
 * a smooth count of molecules within R0.  The parameters, in the order of
 * mdn_adjoint_params: (eps, sigma) of every (gas type, ion type) pair of the
 * replica, then of every (vapor type, ion type) pair, then the charge scale s
 * (ion charges q -> s q, derivative taken at s = 1).
 * The engine runs the window forward (FP32 pair terms) and keeps the
 * replica state every `checkpoint_every` steps; the adjoint then walks the
 * segments backwards, recomputing each one in FP64 from its checkpoint and
 * running reverse velocity Verlet through it: transposed force Jacobians of
 * the pair terms (with the taper weights and their dependence on the ion
 * centre), Jacobian-vector products of the bonded terms, and the adjoint of
 * the converged SHAKE projection with its velocity correction.  The window
 * must hold no effective-domain rebuild (the molecule set is fixed): a
 * window that would cross one is an error (raise Margin or shorten it).
 * Needs a handle with one replica and the thermostat off.  The recompute
 * runs every segment at once; each reverse sweep runs on a cluster of up
 * to 8 CTAs and sums with FP64 atomics, so two calls agree to FP64
 * rounding of those sums, not bit for bit.                              */
typedef struct mdn_adjoint_spec {
  long long n_steps;        /* window length                                  */
  int checkpoint_every;     /* K: steps per recomputed segment                */
  double count_radius;      /* R0 (A)                                         */
  double count_width;       /* W (A)                                          */
  double w_energy;          /* weight of U_vi                                 */
  double w_count;           /* weight of the smooth count                     */
} mdn_adjoint_spec;
/* Parameter rows of mdn_adjoint's gradient: rows[3*k] = 0 (gas-ion) / 1
 * (vapor-ion) / 2 (charge scale), rows[3*k+1..2] = the two types; parameter
 * 2k is the pair's eps, 2k+1 its sigma, the last one the charge scale.
 * *n_params receives the count; rows may be NULL.                          */
int  mdn_adjoint_params(const mdn_replica_desc* d, int* n_params, int* rows, int capacity);
/* Runs the window from the replica's current state (it advances by n_steps)
 * and returns J and dJ/dtheta (grad: n_params doubles).  d must be the
 * descriptor the handle was created with.  ms (may be NULL) receives the
 * device time of the forward window and of the adjoint (ms[0], ms[1]).     */
int  mdn_adjoint(mdn_handle* h, const mdn_replica_desc* d, const mdn_adjoint_spec* spec, double* J,
                 double* grad, double* ms);

/* Page-locked host memory for mdn_snapshot / mdn_upload_state buffers. */
int  mdn_host_alloc(size_t bytes, void** ptr);
int  mdn_host_free(void* ptr);

/* Drains the vapor in/out event log of every replica. */
int  mdn_events(mdn_handle* h, mdn_event* ev, int capacity, int* count);
/* Kinetic energies (MD Observer::computeProps, src/output/observer.cpp:5-36):
 * out[4*r + 0..3] = Kion, Kgas, Kvap (kcal/mol) and Tion (K).             */
int  mdn_kinetic(mdn_handle* h, double* out);

/* ---- initial placement ---------------------------------------------------- */
/* Initial centres and velocities of the gas and vapor molecules on the GPU,
 * replacing MD::initialization_gas / MD::initialization_vapor
 * (src/initialization/initializationGas.cpp:24-100,
 * src/initialization/initializationVapor.cpp:14-76).
 *
 * The reference draws centres uniformly in the cube and keeps one when every
 * row of its atom table is farther than min_dist (10 A), minimum image.  The
 * rows are the ion's atoms and, for each molecule already placed, its atoms
 * at the origin.  So a centre is kept when it is farther than min_dist from
 * every ion atom and, once any molecule is placed, from the origin.  Gas is
 * placed first, then vapor.
 *
 * The candidates come from a counter-based stream (Philox4x32-10, Salmon et
 * al., SC'11), so candidate k is tested independently of the others; the
 * molecules are the first n_gas (n_vapor) kept candidates in stream order.
 * Positions do not depend on the launch shape.  Centre velocities are
 * Maxwell-Boltzmann: sigma * N(0,1) * 1e-5 A/fs per component, the normal
 * deviates by Box-Muller from the same stream.
 *
 * ion_x, gas_x, gas_v, vapor_x, vapor_v are host arrays ([3*n]).
 * MDN_ERR_ARG when more than 1000 * (n + 10) candidates are drawn for a
 * species (the reference would loop for ever); MDN_ERR_NO_DEVICE without a
 * GPU.  Allocates device memory for the call and frees it before return. */
typedef struct mdn_place_desc {
  double box;                   /* cube edge (A); centres in [-box/2, box/2]   */
  double min_dist;              /* 10 A in the reference                      */
  int n_ion;                    /* ion atoms (after the ion's rotation)       */
  const double* ion_x;          /* [3*n_ion]                                  */
  int n_gas, n_vapor;
  double gas_sigma;             /* sqrt(kB T / m_gas) (m/s), m per molecule   */
  double vapor_sigma;           /* sqrt(kB T / m_vapor) (m/s)                 */
  unsigned long long seed;      /* keys the stream                            */
} mdn_place_desc;
int  mdn_place(int device, const mdn_place_desc* d, double* gas_x, double* gas_v, double* vapor_x,
               double* vapor_v);

/* ---- timing / tuning ------------------------------------------------------ */
/* Device time (ms) of the last mdn_step, measured with CUDA events on the
 * stream the kernels were launched on; kernel_launches = kernels issued.  */
int  mdn_last_timing(mdn_handle* h, double* ms, long long* kernel_launches);
int  mdn_set_launch(mdn_handle* h, int cluster_size, int threads, int steps_per_launch);
/* The launch shape mdn_step uses: cluster size (the automatic choice when
 * mdn_options.cluster_size is 0), threads per CTA, steps per launch. */
int  mdn_get_launch(mdn_handle* h, int* cluster_size, int* threads, int* steps_per_launch);
/* Launch-shape tuner: advances every replica by n_steps at each cluster size
 * 1, 2, 4 and 8, timing each block with CUDA events, and keeps the fastest
 * size for later mdn_step calls.  It then measures one block with the
 * cycle accounting (mdn_profile) and orders the replicas by their measured
 * cycles, slowest first, times one block in that order, and tries the split
 * launch below (up to 8 more blocks); *best (may be NULL) receives the
 * cluster size.  The steps are ordinary steps of the run: results do not
 * depend on the launch shape or the order.  A replica that fails during
 * tuning is reported as mdn_step reports it.  */
int  mdn_tune_launch(mdn_handle* h, long long n_steps, int* best);
/* Split step launch: the n_largest replicas at the head of the job order
 * (most estimated work, or most measured cycles once mdn_tune_launch has
 * ordered them) run in a second launch, concurrent with the first on its own stream, on
 * clusters of cluster_size CTAs (one cluster each), and the other replicas
 * on the SMs left at the ordinary cluster size.  The launch of a batch is
 * as long as its largest replica on its cluster, so giving the few largest
 * more SMs shortens it.  n_largest = 0 turns it off.  mdn_tune_launch, when
 * no split is set, also times n_largest = 2, 4, 8, 16 at two and four times
 * the best cluster size (at most 8 CTAs; n_steps each) and keeps a split
 * that beats the best single launch.
 * Results do not depend on the split.                                      */
int  mdn_set_split(mdn_handle* h, int n_largest, int cluster_size);
int  mdn_get_split(mdn_handle* h, int* n_largest, int* cluster_size);
/* Per-replica SM-cycle accounting of the step kernel: enable = 1 starts
 * accumulating (from zero), 0 stops.  out: [8*n_replicas] cycles per phase:
 * total, core integration, gas integration, rebuild, near gas molecules,
 * core bonded terms, core pair terms, core force sums and kick.  The gas
 * molecules are integrated beside the core's constraints, so their time is
 * counted under core integration; the gas slot holds the step's list
 * bookkeeping only. */
int  mdn_profile(mdn_handle* h, int enable, long long* out);

#ifdef __cplusplus
}
#endif
#endif /* MDN_H */
