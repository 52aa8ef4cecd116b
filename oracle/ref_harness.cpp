/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * Drives the reference program's own per-step routines on injected states.
 * oracle/Makefile compiles every reference source under src/ (where it lies,
 * read-only) except src/main.cpp and src/initialization/md.cpp, and links them
 * with this file into oracle/_ref/libref_harness.so.  This file supplies the
 * two members md.cpp would have defined (MD::MD, MD::~MD) so that a replica is
 * built from an mdn_replica_desc instead of the O(N^2) random placement of
 * MD::MD (src/initialization/md.cpp:8-40); every routine called afterwards
 * (MD::verlet, MD::make_pair, Potential::compute/makePair, MD::shake, ...) is
 * the reference's code, unmodified.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load
 * this library, and only as the checker / the timed reference arm.
 *
 * Two reference defects are avoided by construction, not by patching:
 *  - Born-Mayer-Huggins indexes bornCoeff[type][type] (2x2) with global type
 *    indices (src/potential/BMHFT/compute_born.cpp:24-33).  The harness orders
 *    the type table so that the ion's Na/Cl types are rows 0/1.
 *  - He/Ar/N2monoatomic never fill massGas (src/initialization/
 *    setCondition.cpp:48-113); the harness fills the gas template from the
 *    descriptor, so no gas kind runs with an empty mass vector.
 */
#include "md.hpp"
#include "mdn.h"

#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <typeinfo>

/* ---- the two members of src/initialization/md.cpp this harness replaces ---- */
MD::MD(char* /*condfile*/, int calcNumber) {
  startTime = omp_get_wtime();
  calculation_number = calcNumber;
  vars = new Variables();
  obs = new Observer();
  pp = new Physical();
  flags = new FLAG();
  mbdist = new MBdist();
  mbdistV = new MBdist();
  setDefaultVariables();
  loopPair = 0;
  loop_update = 0;
  margin_length = 0;
  zeta = 0;
}

MD::~MD(void) {
  delete vars;
  delete obs;
  delete pp;
  delete flags;
}

namespace {

struct Harness {
  MD* md;
  int n_ion, a_g, a_v, n_gas, n_vap;
  std::vector<int> perm;  /* descriptor type -> reference type row */
};

unsigned term_of(Potential* p) {
  if (dynamic_cast<PotentialGasIon*>(p)) return MDN_I_GI;
  if (dynamic_cast<PotentialVaporIon*>(p)) return MDN_I_VI;
  if (dynamic_cast<PotentialVaporVapor*>(p)) return MDN_I_VV;
  if (dynamic_cast<PotentialVaporGas*>(p)) return MDN_I_GV;
  if (dynamic_cast<PotentialGasGas*>(p)) return MDN_I_GG;
  if (dynamic_cast<PotentialAMBER*>(p)) return MDN_I_AMBER;
  if (dynamic_cast<PotentialBorn*>(p)) return MDN_I_BMH;
  if (dynamic_cast<PotentialGasIntra*>(p)) return MDN_I_GAS_INTRA;
  if (dynamic_cast<PotentialVaporIntra*>(p)) return MDN_I_VAPOR_INTRA;
  if (dynamic_cast<PotentialEfield*>(p)) return MDN_I_EFIELD;
  return 0;
}

std::array<double, 3> a3(const double* p) { return {p[0], p[1], p[2]}; }

}  // namespace

extern "C" {

/* Builds a replica.  do_make_pair = 1 performs the initial MD::make_pair of
 * MD::MD; 0 leaves every molecule outside the domain. */
void* ref_create(const mdn_replica_desc* d, int do_make_pair) {
  /* the reference mixes LJ parameters itself (Variables::setCrossPotentials) */
  if (d->pair_eps || d->pair_sigma) {
    fprintf(stderr, "ref_create: per-pair LJ parameters have no counterpart in the reference\n");
    return nullptr;
  }
  Harness* h = new Harness();
  MD* md = new MD(nullptr, 0);
  h->md = md;
  Variables* v = md->vars;
  h->n_ion = d->ion.n_atoms;
  h->a_g = d->gas.n_atoms;
  h->a_v = d->vapor.n_atoms;
  h->n_gas = d->n_gas;
  h->n_vap = d->n_vapor;

  /* run parameters (src/initialization/setCondition.cpp:119-146,247-250) */
  md->dt = d->dt;
  md->T = d->temperature;
  md->CUTOFF = d->cutoff;
  md->MARGIN = d->margin;
  md->d_size = d->box;
  md->V = d->box * d->box * d->box;
  md->CL2 = d->cutoff * d->cutoff;
  md->ML2 = (d->cutoff + d->margin) * (d->cutoff + d->margin);
  md->gastype = d->gas_kind;
  md->Nof_around_gas = d->n_gas;
  md->Nof_around_vapor = d->n_vapor;
  md->Ecoeff[0] = d->efield[0];
  md->Ecoeff[1] = d->efield[1];
  md->Ecoeff[2] = d->efield[2];

  FLAG* f = md->flags;
  unsigned I = d->interactions;
  f->force_lj = (I & MDN_I_GI) ? 1 : 0;
  f->inter_vi = (I & MDN_I_VI) ? 1 : 0;
  f->inter_vv = (I & MDN_I_VV) ? 1 : 0;
  f->inter_vg = (I & MDN_I_GV) ? 1 : 0;
  f->inter_gg = (I & MDN_I_GG) ? 1 : 0;
  f->intra_AMBER = (I & MDN_I_AMBER) ? 1 : 0;
  f->force_born = (I & MDN_I_BMH) ? 1 : 0;
  f->gas_intra = (I & MDN_I_GAS_INTRA) ? 1 : 0;
  f->vapor_intra = (I & MDN_I_VAPOR_INTRA) ? 1 : 0;
  f->efield = (I & MDN_I_EFIELD) ? 1 : 0;
  f->shakeH = (I & MDN_I_SHAKE) ? true : false;
  f->velocity_scaling = (d->nvt_mode == MDN_NVT_SCALE) ? 1 : 0;
  f->nose_hoover_ion = (d->nvt_mode == MDN_NVT_NH) ? 1 : 0;
  v->flags = f;
  md->pp->Tnh_ion = d->nvt_temperature;
  md->pp->mgas = d->gas_mb_mass;
  md->pp->mvapor = d->vapor_mb_mass;
  md->pp->Mgas = d->gas_com_mass;
  md->pp->Mvapor = d->vapor_com_mass;

  /* type table order: ion types first, Na/Cl on rows 0/1 when BMH is on */
  int nt = d->n_atom_types;
  h->perm.assign(nt, -1);
  int next = 0;
  if (I & MDN_I_BMH) {
    for (int row = 0; row < 2; row++)
      for (int i = 0; i < d->ion.n_atoms; i++)
        if (d->ion_bmh_type[i] == row && h->perm[d->ion.type[i]] < 0) h->perm[d->ion.type[i]] = next++;
  }
  for (int i = 0; i < d->ion.n_atoms; i++)
    if (h->perm[d->ion.type[i]] < 0) h->perm[d->ion.type[i]] = next++;
  for (int t = 0; t < nt; t++)
    if (h->perm[t] < 0) h->perm[t] = next++;
  v->atypes.resize(nt);
  for (int t = 0; t < nt; t++) {
    Atom_type& at = v->atypes[h->perm[t]];
    at.mass = d->atom_mass[t];
    at.coeff1 = d->atom_eps[t];
    at.coeff2 = d->atom_sigma[t];
    char nm[16];
    snprintf(nm, sizeof nm, "T%d", t);
    at.name = nm;
  }
  for (int t = 0; t < d->n_bond_types; t++) {
    Bond_type bt;
    bt.coeff[0] = d->bond_coeff[2 * t];
    bt.coeff[1] = d->bond_coeff[2 * t + 1];
    v->btypes.push_back(bt);
  }
  for (int t = 0; t < d->n_angle_types; t++) {
    Angle_type ct;
    ct.coeff[0] = d->angle_coeff[2 * t];
    ct.coeff[1] = d->angle_coeff[2 * t + 1];
    v->ctypes.push_back(ct);
  }
  for (int t = 0; t < d->n_dihedral_types; t++) {
    Dihedral_type dt;
    dt.multi = d->dihedral_multi[t];
    for (int k = 0; k < 15; k++) dt.coeff[k] = d->dihedral_coeff[15 * t + k];
    v->dtypes.push_back(dt);
  }

  auto bonds3 = [](const int* p, int n) {
    std::vector<std::array<double, 3>> o;
    for (int i = 0; i < n; i++) o.push_back({double(p[3 * i]), double(p[3 * i + 1]), double(p[3 * i + 2])});
    return o;
  };
  auto angles4 = [](const int* p, int n) {
    std::vector<std::array<double, 4>> o;
    for (int i = 0; i < n; i++)
      o.push_back({double(p[4 * i]), double(p[4 * i + 1]), double(p[4 * i + 2]), double(p[4 * i + 3])});
    return o;
  };
  auto dihed5 = [](const int* p, int n) {
    std::vector<std::array<double, 5>> o;
    for (int i = 0; i < n; i++)
      o.push_back({double(p[5 * i]), double(p[5 * i + 1]), double(p[5 * i + 2]), double(p[5 * i + 3]),
                   double(p[5 * i + 4])});
    return o;
  };

  /* the ion: molecule 0 (Variables::readIonFile, src/initialization/readIonFile.cpp:155-179) */
  {
    std::vector<std::array<double, 3>> xs, vs, fs;
    std::vector<double> ms, ps, ws;
    std::vector<int> ts;
    double tot = 0;
    for (int i = 0; i < d->ion.n_atoms; i++) {
      xs.push_back(a3(d->ion.x + 3 * i));
      vs.push_back(a3(d->ion_v + 3 * i));
      fs.push_back({0, 0, 0});
      ms.push_back(d->atom_mass[d->ion.type[i]]);
      tot += d->atom_mass[d->ion.type[i]];
      ps.push_back(d->ion.charge[i]);
      ts.push_back(h->perm[d->ion.type[i]]);
      ws.push_back(1);
    }
    v->positionAtom.push_back(xs);
    v->velocityAtom.push_back(vs);
    v->forceAtom.push_back(fs);
    v->massAtom.push_back(ms);
    v->chargeAtom.push_back(ps);
    v->weight.push_back(ws);
    v->typeAtom.push_back(ts);
    v->bonds.push_back(bonds3(d->ion.bonds, d->ion.n_bonds));
    v->angles.push_back(angles4(d->ion.angles, d->ion.n_angles));
    v->dihedrals.push_back(dihed5(d->ion.dihedrals, d->ion.n_dihedrals));
    v->rigid_pairs.push_back(bonds3(d->ion.rigid, d->ion.n_rigid));
    v->position.push_back({0, 0, 0});
    v->velocity.push_back({0, 0, 0});
    v->force.push_back({0, 0, 0});
    v->type.push_back(0);
    v->mass.push_back(tot);
    v->region.push_back(true);
    v->group[0].push_back(0);
  }
  /* gas template and molecules (src/initialization/initializationGas.cpp:24-90) */
  for (int i = 0; i < d->gas.n_atoms; i++) {
    v->positionGas.push_back(a3(d->gas.x + 3 * i));
    v->massGas.push_back(d->atom_mass[d->gas.type[i]]);
    v->typeGas.push_back(h->perm[d->gas.type[i]]);
    v->chargeGas.push_back(d->gas.charge[i]);
  }
  v->bondsGas = bonds3(d->gas.bonds, d->gas.n_bonds);
  v->bondsGasRigid = bonds3(d->gas.rigid, d->gas.n_rigid);
  for (int m = 0; m < d->n_gas; m++) {
    v->position.push_back(a3(d->gas_x + 3 * m));
    v->velocity.push_back(a3(d->gas_v + 3 * m));
    v->force.push_back({0, 0, 0});
    v->mass.push_back(d->gas_com_mass);
    v->type.push_back(0);
    v->region.push_back(false);
    v->group[1].push_back((int)v->mass.size() - 1);
    std::vector<std::array<double, 3>> z(d->gas.n_atoms, {0, 0, 0});
    v->positionAtom.push_back(z);
    v->velocityAtom.push_back(z);
    v->forceAtom.push_back(z);
    v->massAtom.push_back(v->massGas);
    v->typeAtom.push_back(v->typeGas);
    v->chargeAtom.push_back(v->chargeGas);
    v->bonds.push_back(v->bondsGas);
    v->angles.push_back({});
    v->dihedrals.push_back({});
    v->rigid_pairs.push_back(v->bondsGasRigid);
    v->weight.push_back(std::vector<double>(d->gas.n_atoms, 0.0));
  }
  /* vapor template and molecules (src/initialization/initializationVapor.cpp:14-77) */
  for (int i = 0; i < d->vapor.n_atoms; i++) {
    v->positionVapor.push_back(a3(d->vapor.x + 3 * i));
    v->massVapor.push_back(d->atom_mass[d->vapor.type[i]]);
    v->typeVapor.push_back(h->perm[d->vapor.type[i]]);
    v->chargeVapor.push_back(d->vapor.charge[i]);
  }
  v->bondsVapor = bonds3(d->vapor.bonds, d->vapor.n_bonds);
  v->bondsVaporRigid = bonds3(d->vapor.rigid, d->vapor.n_rigid);
  v->anglesVapor = angles4(d->vapor.angles, d->vapor.n_angles);
  v->dihedralsVapor = dihed5(d->vapor.dihedrals, d->vapor.n_dihedrals);
  for (int m = 0; m < d->n_vapor; m++) {
    v->position.push_back(a3(d->vapor_x + 3 * m));
    v->velocity.push_back(a3(d->vapor_v + 3 * m));
    v->force.push_back({0, 0, 0});
    v->mass.push_back(d->vapor_com_mass);
    v->type.push_back(0);
    v->region.push_back(false);
    v->group[2].push_back((int)v->mass.size() - 1);
    std::vector<std::array<double, 3>> z(d->vapor.n_atoms, {0, 0, 0});
    v->positionAtom.push_back(z);
    v->velocityAtom.push_back(z);
    v->forceAtom.push_back(z);
    v->massAtom.push_back(v->massVapor);
    v->typeAtom.push_back(v->typeVapor);
    v->chargeAtom.push_back(v->chargeVapor);
    v->bonds.push_back(v->bondsVapor);
    v->angles.push_back(v->anglesVapor);
    v->dihedrals.push_back(v->dihedralsVapor);
    v->rigid_pairs.push_back(v->bondsVaporRigid);
    v->weight.push_back(std::vector<double>(d->vapor.n_atoms, 0.0));
  }
  v->time = 0;
  v->zeta_ion = 0;
  v->Uzero();
  v->tzero();
  v->setCrossPotentials();
  md->setPotential(f, 1);
  md->margin_length = md->MARGIN;
  md->loopPair = 0;
  if (do_make_pair) md->make_pair();
  return h;
}

void ref_destroy(void* hp) {
  Harness* h = (Harness*)hp;
  delete h->md;
  delete h;
}

/* Seconds the reference's own placement takes: MD::initialization_gas and
 * MD::initialization_vapor (src/initialization/initializationGas.cpp:24-100,
 * src/initialization/initializationVapor.cpp:14-76) run as MD::MD calls them
 * (src/initialization/md.cpp:27-29), placing n_gas and n_vapor molecules
 * around the descriptor's ion in its box, on a replica built with none. */
double ref_time_placement(const mdn_replica_desc* d, int n_gas, int n_vapor) {
  mdn_replica_desc e = *d;
  e.n_gas = 0;
  e.n_vapor = 0;
  Harness* h = (Harness*)ref_create(&e, 0);
  if (!h) return -1.0;
  MD* md = h->md;
  md->Nof_around_gas = n_gas;
  md->Nof_around_vapor = n_vapor;
  const auto t0 = std::chrono::steady_clock::now();
  md->initialization_gas();
  md->initialization_vapor();
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ref_destroy(h);
  return s;
}

/* out: n_gas_in, n_vapor_in, loopPair, loop_update, gi pairs, gv pairs, vv pairs, gg pairs */
void ref_info(void* hp, int* out) {
  Harness* h = (Harness*)hp;
  MD* md = h->md;
  out[0] = (int)md->vars->gas_in.size();
  out[1] = (int)md->vars->vapor_in.size();
  out[2] = md->loopPair;
  out[3] = md->loop_update;
  out[4] = out[5] = out[6] = out[7] = 0;
  for (auto p : md->InterInter) {
    unsigned t = term_of(p);
    if (t == MDN_I_GI) out[4] = (int)p->pairList.size();
    if (t == MDN_I_GV) out[5] = (int)p->pairList.size();
    if (t == MDN_I_VV) out[6] = (int)p->pairList.size();
    if (t == MDN_I_GG) out[7] = (int)p->pairList.size();
  }
}

void ref_get_state(void* hp, mdn_state* s) {
  Harness* h = (Harness*)hp;
  Variables* v = h->md->vars;
  for (int i = 0; i < h->n_ion; i++)
    for (int k = 0; k < 3; k++) {
      if (s->ion_x) s->ion_x[3 * i + k] = v->positionAtom[0][i][k];
      if (s->ion_v) s->ion_v[3 * i + k] = v->velocityAtom[0][i][k];
      if (s->ion_f) s->ion_f[3 * i + k] = v->forceAtom[0][i][k];
    }
  int nm = 1 + h->n_gas + h->n_vap;
  for (int m = 0; m < nm; m++) {
    for (int k = 0; k < 3; k++) {
      if (s->mol_x) s->mol_x[3 * m + k] = v->position[m][k];
      if (s->mol_v) s->mol_v[3 * m + k] = v->velocity[m][k];
    }
    if (s->region) s->region[m] = v->region[m] ? 1 : 0;
  }
  for (int g = 0; g < h->n_gas; g++)
    for (int a = 0; a < h->a_g; a++)
      for (int k = 0; k < 3; k++) {
        size_t o = 3 * ((size_t)g * h->a_g + a) + k;
        if (s->gas_ax) s->gas_ax[o] = v->positionAtom[1 + g][a][k];
        if (s->gas_av) s->gas_av[o] = v->velocityAtom[1 + g][a][k];
        if (s->gas_af) s->gas_af[o] = v->forceAtom[1 + g][a][k];
      }
  for (int q = 0; q < h->n_vap; q++)
    for (int a = 0; a < h->a_v; a++) {
      int m = 1 + h->n_gas + q;
      for (int k = 0; k < 3; k++) {
        size_t o = 3 * ((size_t)q * h->a_v + a) + k;
        if (s->vap_ax) s->vap_ax[o] = v->positionAtom[m][a][k];
        if (s->vap_av) s->vap_av[o] = v->velocityAtom[m][a][k];
        if (s->vap_af) s->vap_af[o] = v->forceAtom[m][a][k];
      }
      if (s->vap_w) s->vap_w[(size_t)q * h->a_v + a] = v->weight[m][a];
    }
  s->loop_pair = h->md->loopPair;
  s->loop_update = h->md->loop_update;
  s->zeta = v->zeta_ion;
  s->margin_length = h->md->margin_length;
}

/* Writes a state; rebuilds gas_in / vapor_in from the region flags and calls
 * makePair of every pair potential on the given centres (no classification). */
void ref_set_state(void* hp, const mdn_state* s) {
  Harness* h = (Harness*)hp;
  MD* md = h->md;
  Variables* v = md->vars;
  for (int i = 0; i < h->n_ion; i++)
    for (int k = 0; k < 3; k++) {
      if (s->ion_x) v->positionAtom[0][i][k] = s->ion_x[3 * i + k];
      if (s->ion_v) v->velocityAtom[0][i][k] = s->ion_v[3 * i + k];
      if (s->ion_f) v->forceAtom[0][i][k] = s->ion_f[3 * i + k];
    }
  int nm = 1 + h->n_gas + h->n_vap;
  for (int m = 0; m < nm; m++) {
    for (int k = 0; k < 3; k++) {
      if (s->mol_x) v->position[m][k] = s->mol_x[3 * m + k];
      if (s->mol_v) v->velocity[m][k] = s->mol_v[3 * m + k];
    }
    if (s->region && m > 0) v->region[m] = s->region[m] != 0;
  }
  for (int g = 0; g < h->n_gas; g++)
    for (int a = 0; a < h->a_g; a++)
      for (int k = 0; k < 3; k++) {
        size_t o = 3 * ((size_t)g * h->a_g + a) + k;
        if (s->gas_ax) v->positionAtom[1 + g][a][k] = s->gas_ax[o];
        if (s->gas_av) v->velocityAtom[1 + g][a][k] = s->gas_av[o];
        if (s->gas_af) v->forceAtom[1 + g][a][k] = s->gas_af[o];
      }
  for (int q = 0; q < h->n_vap; q++)
    for (int a = 0; a < h->a_v; a++) {
      int m = 1 + h->n_gas + q;
      for (int k = 0; k < 3; k++) {
        size_t o = 3 * ((size_t)q * h->a_v + a) + k;
        if (s->vap_ax) v->positionAtom[m][a][k] = s->vap_ax[o];
        if (s->vap_av) v->velocityAtom[m][a][k] = s->vap_av[o];
        if (s->vap_af) v->forceAtom[m][a][k] = s->vap_af[o];
      }
      if (s->vap_w) v->weight[m][a] = s->vap_w[(size_t)q * h->a_v + a];
    }
  v->gas_in.clear();
  v->gas_out.clear();
  v->vapor_in.clear();
  v->vapor_out.clear();
  for (auto i : v->group[1]) (v->region[i] ? v->gas_in : v->gas_out).push_back(i);
  for (auto i : v->group[2]) (v->region[i] ? v->vapor_in : v->vapor_out).push_back(i);
  for (auto p : md->InterInter) p->makePair(v);
  md->loopPair = s->loop_pair;
  md->loop_update = s->loop_update;
  v->zeta_ion = s->zeta;
  if (s->margin_length > 0) md->margin_length = s->margin_length;
}

/* n calls of the reference's own MD::verlet (src/verlet.cpp:20-39).
 * energy_mode as mdn_step: 1 = eflag on the last step, 2 = on every step. */
void ref_verlet(void* hp, long long n, int energy_mode, double* U) {
  Harness* h = (Harness*)hp;
  MD* md = h->md;
  md->vars->Uzero();
  for (long long s = 0; s < n; s++) {
    if (energy_mode == 2 || (energy_mode == 1 && s == n - 1)) md->flags->eflag = 1;
    md->verlet();
  }
  if (U) {
    Potentials& u = md->vars->Utotal;
    U[0] = u.Uion; U[1] = u.Ugas; U[2] = u.Uvap; U[3] = u.Ugi;
    U[4] = u.Ugg;  U[5] = u.Uvg;  U[6] = u.Uvi;  U[7] = u.Uvv;
  }
}

/* Zeroes the forces of in-domain atoms (as MD::update_position does,
 * src/verlet.cpp:86) and calls compute() of the selected potentials in
 * registration order (src/verlet.cpp:31-32); term_mask 0 = all. */
void ref_compute_forces(void* hp, unsigned term_mask, double* U) {
  Harness* h = (Harness*)hp;
  MD* md = h->md;
  Variables* v = md->vars;
  int nm = (int)v->mass.size();
  for (int i = 0; i < nm; i++)
    if (v->region[i])
      for (auto& f : v->forceAtom[i]) f[0] = f[1] = f[2] = 0;
  v->Uzero();
  md->flags->eflag = 1;
  for (auto p : md->InterInter)
    if (!term_mask || (term_of(p) & term_mask)) p->compute(v, md->flags);
  for (auto p : md->IntraInter)
    if (!term_mask || (term_of(p) & term_mask)) p->compute(v, md->flags);
  md->flags->eflag = 0;
  if (U) {
    Potentials& u = v->Utotal;
    U[0] = u.Uion; U[1] = u.Ugas; U[2] = u.Uvap; U[3] = u.Ugi;
    U[4] = u.Ugg;  U[5] = u.Uvg;  U[6] = u.Uvi;  U[7] = u.Uvv;
  }
}

void ref_make_pair(void* hp) { ((Harness*)hp)->md->make_pair(); }
void ref_update_in_centers(void* hp) { ((Harness*)hp)->md->updateInCenters(); }
void ref_velocity_calculation(void* hp) { ((Harness*)hp)->md->velocity_calculation(); }
void ref_update_position(void* hp) { ((Harness*)hp)->md->update_position(); }
void ref_update_position_shake(void* hp) { ((Harness*)hp)->md->updatePositionSHAKE(); }
void ref_velocity_scaling(void* hp) { ((Harness*)hp)->md->velocity_scaling(); }
void ref_nosehoover_zeta(void* hp) { ((Harness*)hp)->md->nosehoover_zeta(); }
void ref_nosehoover_ion(void* hp) { ((Harness*)hp)->md->nosehoover_ion(); }
void ref_set_nve(void* hp) { ((Harness*)hp)->md->setNVE(); }

/* MD::shake on one molecule after the caller has set its positions; the
 * "old" positions are those passed in old_x (the reference records them in
 * MD::updatePositionSHAKE before drifting, src/shake.cpp:11-19).  mol is the
 * reference molecule index (0 = ion). */
void ref_shake(void* hp, int mol, const double* old_x) {
  Harness* h = (Harness*)hp;
  Variables* v = h->md->vars;
  v->oldPosition.clear();
  int n = (int)v->positionAtom[mol].size();
  for (int i = 0; i < n; i++) v->oldPosition.push_back(a3(old_x + 3 * i));
  h->md->shake(mol);
}

/* Variables::ROTATION (src/variables.hpp:94-98) */
void ref_rotation(double A, double B, double C, double x, double y, double z, double* out) {
  Variables v;
  v.ROTATION(out[0], out[1], out[2], A, B, C, x, y, z);
}

/* Observer::computeProps (src/output/observer.cpp:5-36): Kion, Kgas, Kvap, Tion, Tgas, Tvap */
void ref_kinetic(void* hp, double* out) {
  Harness* h = (Harness*)hp;
  Observer* o = h->md->obs;
  o->computeProps(h->md->vars);
  out[0] = o->Kion; out[1] = o->K_g; out[2] = o->K_v;
  out[3] = o->Tion; out[4] = o->T_g; out[5] = o->T_v;
}

/* Pair lists of the pair potentials as (molecule, partner) rows in the
 * numbering of mdn_pair_list: kind 0 gas-ion, 1 gas-vapor, 2 gas-gas.
 * Returns the number of rows (rows beyond capacity are counted, not written). */
int ref_pair_list(void* hp, int kind, int* pairs, int capacity) {
  Harness* h = (Harness*)hp;
  MD* md = h->md;
  unsigned want = kind == 0 ? MDN_I_GI : kind == 1 ? MDN_I_GV : MDN_I_GG;
  int n = 0;
  for (auto p : md->InterInter) {
    if (term_of(p) != want) continue;
    for (auto& pr : p->pairList) {
      int a = pr.i - 1, b = pr.j;
      if (kind == 1) b = pr.j - 1 - h->n_gas;
      if (kind == 2) { a = pr.i; b = pr.j; }
      if (n < capacity) { pairs[2 * n] = a; pairs[2 * n + 1] = b; }
      n++;
    }
  }
  return n;
}

/* Sequence of the reference's routines for one step with SHAKE enabled:
 * MD::verlet with MD::updatePositionSHAKE in place of MD::update_position
 * (the call the reference leaves commented out, src/verlet.cpp:24), followed
 * by the ion centre and taper weights that update_position would compute.
 * The centre/weight part restates src/verlet.cpp:90-134. */
void ref_verlet_shake(void* hp, long long n, int energy_mode, double* U) {
  Harness* h = (Harness*)hp;
  MD* md = h->md;
  Variables* v = md->vars;
  v->Uzero();
  for (long long s = 0; s < n; s++) {
    if (energy_mode == 2 || (energy_mode == 1 && s == n - 1)) md->flags->eflag = 1;
    md->velocity_calculation();
    if (md->flags->velocity_scaling == 1) md->velocity_scaling();
    md->updatePositionSHAKE();
    {
      int is = (int)v->positionAtom[0].size();
      std::array<double, 3>& x = v->position[0];
      std::array<double, 3>& vv = v->velocity[0];
      x = {0, 0, 0};
      vv = {0, 0, 0};
      for (int ii = 0; ii < is; ii++)
        for (int k = 0; k < 3; k++) {
          x[k] += v->positionAtom[0][ii][k] * v->massAtom[0][ii];
          vv[k] += v->velocityAtom[0][ii][k] * v->massAtom[0][ii];
        }
      double mInv = 1 / v->mass[0];
      for (int k = 0; k < 3; k++) { x[k] *= mInv; vv[k] *= mInv; }
      for (int I = 1; I < 3; I++)
        for (auto i : v->group[I]) {
          if (!v->region[i]) continue;
          for (size_t ii = 0; ii < v->positionAtom[i].size(); ii++) {
            double dx = v->positionAtom[i][ii][0] - x[0];
            double dy = v->positionAtom[i][ii][1] - x[1];
            double dz = v->positionAtom[i][ii][2] - x[2];
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < Ri2) v->weight[i][ii] = 1;
            else if (r2 > RI2) v->weight[i][ii] = 0;
            else {
              double dr = (sqrt(r2) - Rcenter);
              double C = cos(M_PI / Overlap * 0.5 * dr);
              v->weight[i][ii] = C * C;
            }
          }
        }
    }
    if (md->flags->nose_hoover_ion == 1) md->nosehoover_zeta();
    md->check_pairlist();
    v->totalVirial = 0;
    for (auto& a : md->InterInter) a->compute(v, md->flags);
    for (auto& a : md->IntraInter) a->compute(v, md->flags);
    md->velocity_calculation();
    if (md->flags->nose_hoover_ion == 1) md->nosehoover_ion();
    md->flags->eflag = 0;
  }
  if (U) {
    Potentials& u = v->Utotal;
    U[0] = u.Uion; U[1] = u.Ugas; U[2] = u.Uvap; U[3] = u.Ugi;
    U[4] = u.Ugg;  U[5] = u.Uvg;  U[6] = u.Uvi;  U[7] = u.Uvv;
  }
}

/* In-domain atoms counted the way MD::export_dump_close does (src/output/output.cpp:136-143). */
int ref_in_domain_atoms(void* hp) {
  Harness* h = (Harness*)hp;
  Variables* v = h->md->vars;
  int n = 0;
  for (size_t i = 0; i < v->mass.size(); i++)
    if (v->region[i]) n += (int)v->massAtom[i].size();
  return n;
}

/* MD::export_dump_close into `path` (the reference appends to pp->dump_path). */
void ref_export_dump(void* hp, const char* path, double time_fs) {
  Harness* h = (Harness*)hp;
  MD* md = h->md;
  static std::string keep;
  keep = path;
  md->pp->dump_path = (char*)keep.c_str();
  md->vars->time = time_fs;
  md->export_dump_close();
}

}  // extern "C"

namespace {

/* minimal JSON writer for ref_read_inputs */
struct Json {
  std::string s;
  void num(double v) {
    char b[64];
    snprintf(b, sizeof b, "%.17g", v);
    s += b;
  }
  void str(const std::string& v) {
    s += '"';
    for (char c : v) {
      if (c == '"' || c == '\\') s += '\\';
      s += c;
    }
    s += '"';
  }
  void key(const char* k) {
    if (!s.empty() && s.back() != '{' && s.back() != '[') s += ',';
    str(k);
    s += ':';
  }
  template <class V>
  void arr(const V& v) {
    s += '[';
    bool first = true;
    for (const auto& e : v) {
      if (!first) s += ',';
      first = false;
      num((double)e);
    }
    s += ']';
  }
  template <class V>
  void rows(const V& v) {
    s += '[';
    bool first = true;
    for (const auto& r : v) {
      if (!first) s += ',';
      first = false;
      arr(r);
    }
    s += ']';
  }
};

}  // namespace

extern "C" {
/* Runs the reference's own readers on a condition file and the files it
 * names -- MD::readCondFile (src/initialization/setCondition.cpp:4-254),
 * Variables::readIonFile (src/initialization/readIonFile.cpp:3-179) and
 * Variables::readVaporFile (src/initialization/readVaporFile.cpp:3-131), in
 * MD::MD's order -- and writes what they stored as JSON into buf.  Returns
 * the length, or -1 when buf is too small. */
int ref_read_inputs(const char* cond, int calc, char* buf, int cap) {
  MD* md = new MD(nullptr, calc);
  md->readCondFile((char*)cond);
  Variables* v = md->vars;
  v->readIonFile(md->atomFile);
  v->readVaporFile(md->vaporFile);
  FLAG* f = md->flags;
  Json j;
  j.s = "{";
  j.key("T"); j.num(md->T);
  j.key("p"); j.num(md->p);
  j.key("dt"); j.num(md->dt);
  j.key("cutoff"); j.num(md->CUTOFF);
  j.key("margin"); j.num(md->MARGIN);
  j.key("box"); j.num(md->d_size);
  j.key("total"); j.num((double)md->Noftimestep);
  j.key("relax"); j.num((double)md->step_relax);
  j.key("observe"); j.num(md->OBSERVE);
  j.key("gastype"); j.num(md->gastype);
  j.key("n_gas"); j.num(md->Nof_around_gas);
  j.key("n_vapor"); j.num(md->Nof_around_vapor);
  j.key("dump_path"); j.str(md->pp->dump_path ? md->pp->dump_path : "");
  j.key("Tnh_ion"); j.num(md->pp->Tnh_ion);
  j.key("Ecoeff"); j.arr(std::vector<double>{md->Ecoeff[0], md->Ecoeff[1], md->Ecoeff[2]});
  j.key("flags"); j.s += "{";
  j.key("force_lj"); j.num(f->force_lj);
  j.key("inter_vi"); j.num(f->inter_vi);
  j.key("inter_vv"); j.num(f->inter_vv);
  j.key("inter_vg"); j.num(f->inter_vg);
  j.key("inter_gg"); j.num(f->inter_gg);
  j.key("intra_AMBER"); j.num(f->intra_AMBER);
  j.key("force_born"); j.num(f->force_born);
  j.key("efield"); j.num(f->efield);
  j.key("gas_intra"); j.num(f->gas_intra);
  j.key("vapor_intra"); j.num(f->vapor_intra);
  j.key("shakeH"); j.num(f->shakeH ? 1 : 0);
  j.key("nose_hoover_ion"); j.num(f->nose_hoover_ion);
  j.key("velocity_scaling"); j.num(f->velocity_scaling);
  j.s += "}";
  j.key("atypes"); j.s += "[";
  for (size_t t = 0; t < v->atypes.size(); t++) {
    if (t) j.s += ",";
    j.s += "[";
    j.str(v->atypes[t].name);
    j.s += ",";
    j.num(v->atypes[t].mass);
    j.s += ",";
    j.num(v->atypes[t].coeff1);
    j.s += ",";
    j.num(v->atypes[t].coeff2);
    j.s += "]";
  }
  j.s += "]";
  std::vector<std::vector<double>> bt, ct, dt;
  for (auto& b : v->btypes) bt.push_back({b.coeff[0], b.coeff[1]});
  for (auto& c : v->ctypes) ct.push_back({c.coeff[0], c.coeff[1]});
  for (auto& d : v->dtypes) {
    std::vector<double> r{(double)d.multi};
    for (int k = 0; k < 15; k++) r.push_back(d.coeff[k]);
    dt.push_back(r);
  }
  j.key("btypes"); j.rows(bt);
  j.key("ctypes"); j.rows(ct);
  j.key("dtypes"); j.rows(dt);
  j.key("ion"); j.s += "{";
  j.key("type"); j.arr(v->typeAtom[0]);
  j.key("charge"); j.arr(v->chargeAtom[0]);
  j.key("x"); j.rows(v->positionAtom[0]);
  j.key("bonds"); j.rows(v->bonds[0]);
  j.key("rigid"); j.rows(v->rigid_pairs[0]);
  j.key("angles"); j.rows(v->angles[0]);
  j.key("dihedrals"); j.rows(v->dihedrals[0]);
  j.s += "}";
  j.key("vapor"); j.s += "{";
  j.key("type"); j.arr(v->typeVapor);
  j.key("charge"); j.arr(v->chargeVapor);
  j.key("x"); j.rows(v->positionVapor);
  j.key("bonds"); j.rows(v->bondsVapor);
  j.key("rigid"); j.rows(v->bondsVaporRigid);
  j.key("angles"); j.rows(v->anglesVapor);
  j.key("dihedrals"); j.rows(v->dihedralsVapor);
  j.s += "}";
  j.key("gas"); j.s += "{";
  j.key("type"); j.arr(v->typeGas);
  j.key("charge"); j.arr(v->chargeGas);
  j.key("x"); j.rows(v->positionGas);
  j.key("bonds"); j.rows(v->bondsGas);
  j.s += "}";
  j.s += "}";
  delete md;
  if ((int)j.s.size() + 1 > cap) return -1;
  memcpy(buf, j.s.c_str(), j.s.size() + 1);
  return (int)j.s.size();
}

/* The reference's replica model (src/main.cpp:22-29): one replica per OpenMP
 * thread, each running MD::verlet n times.  threads <= 0: all threads.
 * MD::verlet never calls the reference's SHAKE (src/verlet.cpp:24); its
 * iteration has no iteration limit, so it is not run here on replicas that
 * the reference's insertion may have blown up. */
void ref_verlet_many(void** hs, int n, long long steps, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; i++) {
    MD* md = ((Harness*)hs[i])->md;
    for (long long s = 0; s < steps; s++) md->verlet();
  }
}
}
