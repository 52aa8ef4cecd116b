/*
 * mdn_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the FP64 CPU restatement of the
 * per-step hot path, used as the checker of the CUDA engine and as the
 * "port" CPU baseline.  Nothing in the product links or loads it.
 *
 * It restates, in FP64 and in the reference's evaluation order (compiled with
 * -ffp-contract=off so no multiply-add is fused), the routines of one
 * replica step:
 *   MD::verlet                      src/verlet.cpp:20-39
 *   MD::velocity_calculation        src/verlet.cpp:47-65
 *   MD::update_position             src/verlet.cpp:73-136
 *   MD::check_pairlist / make_pair  src/pairList/pairlist.cpp:16-63
 *   MD::updateInCenters             src/pairList/updateCenters.cpp:6-58
 *   MD::update_gas_in (+insertion)  src/pairList/updateGasIn.cpp:10-99
 *   MD::update_vapor_in (+insertion) src/pairList/updateVaporIn.cpp:10-82
 *   Potential{GasIon,VaporIon,VaporGas,VaporVapor}::compute/makePair
 *                                   src/potential/{GasIon,VaporIon,VaporGas,VaporVapor}.cpp
 *   PotentialGasGas (corrected form) src/potential/GasGas.cpp:4-62
 *   PotentialAMBER                  src/potential/compute_AMBER.cpp:10-298
 *   PotentialBorn                   src/potential/BMHFT/compute_born.cpp:10-56
 *   PotentialGasIntra/VaporIntra    src/potential/compute_intra.cpp:14-245
 *   PotentialEfield                 src/potential/electricField.cpp:54-64
 *   MD::shake (restated, see below) src/shake.cpp:44-92
 *   MD::velocity_scaling / nosehoover_* src/nvt.cpp:5-42
 *   Observer::computeProps          src/output/observer.cpp:5-36
 * On deterministic paths (forces, kicks, drift, centres, weights, lists) it
 * is checked bit-for-bit against the reference routines themselves through
 * oracle/ref_harness.cpp.
 *
 * Where the reference draws from std::random_device (unseeded), this file
 * and the engine draw from Philox4x32-10 with this layout:
 *   key     = (seed & 0xffffffff, seed >> 32) of the replica
 *   counter = (molecule, rebuild number, purpose, word)
 *     molecule: 1 + gas index, or 1 + n_gas + vapor index
 *     rebuild number: make_pair calls so far on this replica (0 = the first)
 *     purpose 0, word 0: Maxwell-Boltzmann velocity of a molecule found
 *       outside the domain: Box-Muller on (w0, w1) gives vx, vy, on (w2, w3)
 *       gives vz (the second normal is unused)
 *     purpose 1, word 0: insertion angles a, b, c = 2 pi u01(w0..w2)
 *     purpose 1, word 1: N2 spin normals (vy_rot, vz_rot) from (w0, w1)
 *     purpose 1, word 1 + t (t = 1..3): insertion angles of the t-th re-draw
 *       of the checked insertion (MDN_Q_BLIND_INSERT cleared)
 *
 * SHAKE: the reference's iteration (src/shake.cpp:44-92) scales each
 * correction by (1/mi + 1/mj)^2 relative to the textbook multiplier
 * g = (d^2 - s^2) / (2 (1/mi + 1/mj) r.s) and has no iteration cap.  Both
 * converge to the same constrained positions (the correction direction and
 * the stopping test (s^2 - d^2)^2 <= 1e-20 are the same); this file and the
 * engine use the textbook multiplier, sweep the constraints in colour order
 * (constraints of one colour share no atom), test convergence after a whole
 * sweep (so the returned positions satisfy the tolerance, which the
 * reference's per-constraint test does not guarantee) and stop after 1000
 * sweeps with a status bit.  Unless MDN_Q_SHAKE_NO_VCORR is set, the half-step velocity
 * receives the constraint displacement divided by dt.
 */
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "mdn.h"
#include "philox.h"
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using V3 = std::array<double, 3>;

/* src/constants.hpp:28-53, same expressions */
const double Nw = 6.02e23;
const double kb = 1.38e-23;
const double kb_real = kb * Nw / 4184.0;
const double e0 = 8.85e-12;
const double e = 1.602e-19;
const double qqrd2e = e * e / 4.0 / M_PI / e0 * Nw * 1e10 / 4184.0;
const double real_to_kcalmol = 10000 / 4.184;
const double kb_real_inv = 1 / kb_real;

/* Tosi-Fumi NaCl table (src/potential/BMHFT/potentialBMHFT.hpp:21-39):
 * [row][col][0..4] = A/rho, 6C, 8D, sigma, 1/rho */
struct Born {
  double c[2][2][5];
  Born() {
    c[0][0][0] = 25.4435 * 3.1546 / 4.184;
    c[0][1][0] = c[1][0][0] = 20.3548 * 3.1546 / 4.184;
    c[1][1][0] = 15.2661 * 3.1546 / 4.184;
    c[0][0][1] = 6 * 101.1719 / 4.184;
    c[0][1][1] = c[1][0][1] = 6 * 674.4793 / 4.184;
    c[1][1][1] = 6 * 6985.6786 / 4.184;
    c[0][0][2] = 8 * 48.1771 / 4.184;
    c[0][1][2] = c[1][0][2] = 8 * 837.077 / 4.184;
    c[1][1][2] = 8 * 14031.5785 / 4.184;
    c[0][0][3] = 2.340;
    c[0][1][3] = c[1][0][3] = 2.755;
    c[1][1][3] = 3.170;
    c[0][0][4] = c[0][1][4] = c[1][0][4] = c[1][1][4] = 3.1546;
  }
};
const Born born;

struct Top {
  int n = 0;
  std::vector<int> type;
  std::vector<double> q, mass;
  std::vector<V3> x;
  std::vector<std::array<int, 3>> bonds, rigid;
  std::vector<std::array<int, 4>> angles;
  std::vector<std::array<int, 5>> dih;
  std::vector<int> rigid_color;  /* colour of each rigid pair */
  int n_colors = 0;
  double msum = 0;
};

/* Greedy colouring of constraints: in list order, each pair takes the lowest
 * colour not used by an earlier pair sharing an atom. */
void color_rigid(Top& t) {
  t.rigid_color.assign(t.rigid.size(), 0);
  t.n_colors = 0;
  for (size_t k = 0; k < t.rigid.size(); k++) {
    int c = 0;
    for (;;) {
      bool clash = false;
      for (size_t p = 0; p < k; p++)
        if (t.rigid_color[p] == c &&
            (t.rigid[p][0] == t.rigid[k][0] || t.rigid[p][0] == t.rigid[k][1] ||
             t.rigid[p][1] == t.rigid[k][0] || t.rigid[p][1] == t.rigid[k][1])) {
          clash = true;
          break;
        }
      if (!clash) break;
      c++;
    }
    t.rigid_color[k] = c;
    t.n_colors = std::max(t.n_colors, c + 1);
  }
}

Top load_top(const mdn_topology& s, const double* atom_mass) {
  Top t;
  t.n = s.n_atoms;
  for (int i = 0; i < s.n_atoms; i++) {
    t.type.push_back(s.type[i]);
    t.q.push_back(s.charge[i]);
    t.mass.push_back(atom_mass[s.type[i]]);
    t.x.push_back({s.x[3 * i], s.x[3 * i + 1], s.x[3 * i + 2]});
    t.msum += atom_mass[s.type[i]];
  }
  for (int i = 0; i < s.n_bonds; i++) t.bonds.push_back({s.bonds[3 * i], s.bonds[3 * i + 1], s.bonds[3 * i + 2]});
  for (int i = 0; i < s.n_rigid; i++) t.rigid.push_back({s.rigid[3 * i], s.rigid[3 * i + 1], s.rigid[3 * i + 2]});
  for (int i = 0; i < s.n_angles; i++)
    t.angles.push_back({s.angles[4 * i], s.angles[4 * i + 1], s.angles[4 * i + 2], s.angles[4 * i + 3]});
  for (int i = 0; i < s.n_dihedrals; i++)
    t.dih.push_back({s.dihedrals[5 * i], s.dihedrals[5 * i + 1], s.dihedrals[5 * i + 2],
                     s.dihedrals[5 * i + 3], s.dihedrals[5 * i + 4]});
  color_rigid(t);
  return t;
}

/* Variables::ROTATION (src/variables.hpp:94-98), same expression order */
inline void rotation(double& X, double& Y, double& Z, double A, double B, double C, double x, double y,
                     double z) {
  X = cos(C) * (x * cos(B) + y * sin(A) * sin(B) - z * cos(A) * sin(B)) + sin(C) * (y * cos(A) + z * sin(A));
  Y = -sin(C) * (x * cos(B) + y * sin(A) * sin(B) - z * cos(A) * sin(B)) + cos(C) * (y * cos(A) + z * sin(A));
  Z = x * sin(B) - y * sin(A) * cos(B) + z * cos(A) * cos(B);
}

struct Oracle {
  /* parameters */
  unsigned quirks = MDN_Q_ALL;
  int force_mode = 0;
  unsigned I = 0;
  int nt = 0;
  std::vector<double> ljA, ljB;  /* pair_coeff[ti][tj][0/1] */
  std::vector<std::array<double, 2>> bond_c, angle_c;
  std::vector<int> dih_multi;
  std::vector<std::array<double, 15>> dih_c;
  Top ion, gas, vap;
  std::vector<int> bmh;
  int gas_kind = 0;
  double gas_com_mass = 0, vap_com_mass = 0, gas_sigma = 0, vap_sigma = 0;
  int n_gas = 0, n_vap = 0, a_g = 0, a_v = 0;
  double dt = 1, T = 300, box = 0, ML2 = 0, Ri2 = 0, RI2 = 0, Rcenter = 0, Overlap = 10, margin = 10;
  int nvt_mode = 0;
  double nvt_T = 300;
  double Ef[3] = {0, 0, 0};
  uint32_t key0 = 0, key1 = 0;
  std::vector<char> excl;  /* AMBER exclusions, n_ion x n_ion */

  /* state */
  std::vector<V3> ion_x, ion_v, ion_f;
  std::vector<V3> mol_x, mol_v;  /* 0 = ion centre, 1.. gas, then vapor */
  std::vector<unsigned char> region;
  std::vector<V3> gx, gv, gf;  /* gas atoms, all molecules [n_gas*a_g] */
  std::vector<V3> vx, vv, vf;  /* vapor atoms [n_vap*a_v] */
  std::vector<double> gw, vw;
  std::vector<int> gas_in, vap_in;
  std::vector<std::array<int, 2>> gi_list, gv_list, gg_list;
  int loop_pair = 0, loop_update = 0, n_rebuilds = 0;
  double margin_length = 10, zeta = 0;
  long long step = 0;
  double U[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int status = 0;
  int eflag = 0;
  unsigned term_mask = 0;

  bool on(unsigned bit) const { return (I & bit) && (!term_mask || (term_mask & bit)); }
  double A(int ti, int tj) const { return ljA[ti * nt + tj]; }
  double B(int ti, int tj) const { return ljB[ti * nt + tj]; }

  /* ---------------------------------------------------------------------- */
  void velocity_calculation() {
    double const Coeff = 0.5 * dt * 4.184e-4;
    for (int i = 0; i < ion.n; i++) {
      double Coeff2 = Coeff / ion.mass[i];
      for (int k = 0; k < 3; k++) ion_v[i][k] += ion_f[i][k] * Coeff2;
    }
    for (int m : gas_in)
      for (int a = 0; a < a_g; a++) {
        double Coeff2 = Coeff / gas.mass[a];
        V3& v = gv[(size_t)m * a_g + a];
        const V3& f = gf[(size_t)m * a_g + a];
        for (int k = 0; k < 3; k++) v[k] += f[k] * Coeff2;
      }
    for (int m : vap_in)
      for (int a = 0; a < a_v; a++) {
        double Coeff2 = Coeff / vap.mass[a];
        V3& v = vv[(size_t)m * a_v + a];
        const V3& f = vf[(size_t)m * a_v + a];
        for (int k = 0; k < 3; k++) v[k] += f[k] * Coeff2;
      }
  }

  /* SHAKE of one molecule: x = drifted positions, r = positions before drift.
   * Sweeps in colour order; converged when every constraint satisfies
   * (s^2 - d^2)^2 <= 1e-20 after a full sweep. */
  void shake_mol(const Top& t, V3* x, V3* v, const V3* r) {
    if (t.rigid.empty()) return;
    std::vector<V3> x0(x, x + t.n);
    auto resid = [&](size_t k) {
      int i = t.rigid[k][0], j = t.rigid[k][1];
      double dk = bond_c[t.rigid[k][2]][1];
      double sx = x[i][0] - x[j][0], sy = x[i][1] - x[j][1], sz = x[i][2] - x[j][2];
      double dr = sx * sx + sy * sy + sz * sz - dk * dk;
      return dr * dr;
    };
    bool converge = false;
    for (int sweep = 0; sweep < 1000 && !converge; sweep++) {
      for (int c = 0; c < t.n_colors; c++)
        for (size_t k = 0; k < t.rigid.size(); k++) {
          if (t.rigid_color[k] != c) continue;
          int i = t.rigid[k][0], j = t.rigid[k][1];
          double dk = bond_c[t.rigid[k][2]][1];
          double rx = r[i][0] - r[j][0], ry = r[i][1] - r[j][1], rz = r[i][2] - r[j][2];
          double sx = x[i][0] - x[j][0], sy = x[i][1] - x[j][1], sz = x[i][2] - x[j][2];
          double s2 = sx * sx + sy * sy + sz * sz;
          double dot = rx * sx + ry * sy + rz * sz;
          double minv = 1 / t.mass[i] + 1 / t.mass[j];
          if (dot < 1e-10) dot = 1e-10;
          double g = (dk * dk - s2) / (2 * minv * dot);
          double ci = g / t.mass[i], cj = g / t.mass[j];
          x[i][0] += rx * ci; x[i][1] += ry * ci; x[i][2] += rz * ci;
          x[j][0] -= rx * cj; x[j][1] -= ry * cj; x[j][2] -= rz * cj;
        }
      converge = true;
      for (size_t k = 0; k < t.rigid.size(); k++)
        if (resid(k) > 1e-20) converge = false;
    }
    if (!converge) status |= MDN_ST_SHAKE_NOCONV;
    if (!(quirks & MDN_Q_SHAKE_NO_VCORR))
      for (int a = 0; a < t.n; a++)
        for (int k = 0; k < 3; k++) v[a][k] += (x[a][k] - x0[a][k]) / dt;
  }

  double weight_of(const V3& xa) const {
    const V3& x0 = mol_x[0];
    double dx = xa[0] - x0[0];
    double dy = xa[1] - x0[1];
    double dz = xa[2] - x0[2];
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < Ri2) return 1;
    if (r2 > RI2) return 0;
    double dr = (sqrt(r2) - Rcenter);
    double C = cos(M_PI / Overlap * 0.5 * dr);
    return C * C;
  }

  void update_position() {
    bool sh = (I & MDN_I_SHAKE) != 0;
    std::vector<V3> old;
    auto drift = [&](V3* x, V3* v, V3* f, int n) {
      for (int a = 0; a < n; a++) {
        x[a][0] += v[a][0] * dt;
        x[a][1] += v[a][1] * dt;
        x[a][2] += v[a][2] * dt;
        f[a][0] = f[a][1] = f[a][2] = 0.0;
      }
    };
    auto one = [&](const Top& t, V3* x, V3* v, V3* f) {
      if (sh && !t.rigid.empty()) {
        old.assign(x, x + t.n);
        drift(x, v, f, t.n);
        shake_mol(t, x, v, old.data());
      } else {
        drift(x, v, f, t.n);
      }
    };
    one(ion, ion_x.data(), ion_v.data(), ion_f.data());
    for (int m : gas_in) one(gas, &gx[(size_t)m * a_g], &gv[(size_t)m * a_g], &gf[(size_t)m * a_g]);
    for (int m : vap_in) one(vap, &vx[(size_t)m * a_v], &vv[(size_t)m * a_v], &vf[(size_t)m * a_v]);
    /* ion centre (src/verlet.cpp:90-107) */
    V3& x = mol_x[0];
    V3& v = mol_v[0];
    x = {0, 0, 0};
    v = {0, 0, 0};
    for (int ii = 0; ii < ion.n; ii++)
      for (int k = 0; k < 3; k++) {
        x[k] += ion_x[ii][k] * ion.mass[ii];
        v[k] += ion_v[ii][k] * ion.mass[ii];
      }
    double mInv = 1 / ion.msum;
    for (int k = 0; k < 3; k++) x[k] *= mInv;
    for (int k = 0; k < 3; k++) v[k] *= mInv;
    /* taper weights (src/verlet.cpp:109-134) */
    for (int m : gas_in)
      for (int a = 0; a < a_g; a++) gw[(size_t)m * a_g + a] = weight_of(gx[(size_t)m * a_g + a]);
    for (int m : vap_in)
      for (int a = 0; a < a_v; a++) vw[(size_t)m * a_v + a] = weight_of(vx[(size_t)m * a_v + a]);
  }

  /* Observer::computeProps, ion part */
  double ion_temperature() const {
    double Kion = 0;
    for (int i = 0; i < ion.n; i++) {
      Kion += ion_v[i][0] * ion_v[i][0] * ion.mass[i];
      Kion += ion_v[i][1] * ion_v[i][1] * ion.mass[i];
      Kion += ion_v[i][2] * ion_v[i][2] * ion.mass[i];
    }
    Kion *= 0.5 * real_to_kcalmol;
    return Kion / double(ion.n) * (kb_real_inv / 1.5);
  }

  void velocity_scaling() {
    double Tp = 300;
    double ratio = sqrt(Tp / ion_temperature());
    for (auto& a : ion_v) { a[0] *= ratio; a[1] *= ratio; a[2] *= ratio; }
  }
  void nosehoover_zeta() {
    int g = ion.n * 3;
    double Q_inv = 0.0001;
    zeta += (ion_temperature() - nvt_T) * g * kb_real * Q_inv * dt;
  }
  void nosehoover_ion() {
    double Coeff = exp(-zeta * 0.5 * dt);
    for (auto& a : ion_v) { a[0] *= Coeff; a[1] *= Coeff; a[2] *= Coeff; }
  }

  /* ---------------------------------------------------------------------- */
  /* effective domain                                                        */
  orc::U4 draw(int mol, int purpose, int word) const {
    orc::U4 c = {{(uint32_t)mol, (uint32_t)n_rebuilds, (uint32_t)purpose, (uint32_t)word}};
    return orc::philox4x32_10(c, key0, key1);
  }

  void update_in_centers() {
    auto com = [&](int mi, const V3* x, const V3* v, const Top& t, double mass) {
      V3& mx = mol_x[mi];
      V3& mv = mol_v[mi];
      mx = {0, 0, 0};
      mv = {0, 0, 0};
      for (int a = 0; a < t.n; a++)
        for (int k = 0; k < 3; k++) {
          mx[k] += x[a][k] * t.mass[a];
          mv[k] += v[a][k] * t.mass[a];
        }
      double massInv = 1 / mass;
      for (int k = 0; k < 3; k++) mx[k] *= massInv;
      for (int k = 0; k < 3; k++) mv[k] *= massInv;
    };
    for (int m : gas_in) com(1 + m, &gx[(size_t)m * a_g], &gv[(size_t)m * a_g], gas, gas_com_mass);
    for (int m : vap_in) com(1 + n_gas + m, &vx[(size_t)m * a_v], &vv[(size_t)m * a_v], vap, vap_com_mass);
  }

  /* Philox word of insertion draw t (word 1 is the N2 spin) */
  static int insert_word(int t) { return t == 0 ? 0 : 1 + t; }

  /* atoms in the domain before this rebuild: the core (ion + vapor) and the
   * gas; atoms of vapor molecules whose entry this rebuild accepted */
  std::vector<V3> core_before, gas_before, new_vapor;
  int n_vapor_candidates = 0;

  /* no atom of X within MDN_INSERT_MIN_DIST of the core and, for an entering
   * vapor molecule, of the in-domain gas (for an entering gas molecule, of
   * the vapor molecules accepted in this rebuild) */
  bool insert_clear(const V3* X, int n, bool vapor) const {
    const double d2min = MDN_INSERT_MIN_DIST * MDN_INSERT_MIN_DIST;
    for (const V3& c : core_before)
      for (int a = 0; a < n; a++) {
        double dx = X[a][0] - c[0], dy = X[a][1] - c[1], dz = X[a][2] - c[2];
        if (dx * dx + dy * dy + dz * dz < d2min) return false;
      }
    const std::vector<V3>& extra = vapor ? gas_before : new_vapor;
    for (const V3& c : extra)
      for (int a = 0; a < n; a++) {
        double dx = X[a][0] - c[0], dy = X[a][1] - c[1], dz = X[a][2] - c[2];
        if (dx * dx + dy * dy + dz * dz < d2min) return false;
      }
    /* with the gas-gas term on, an entering gas molecule is also tested
     * against the gas in the domain before this rebuild */
    if (!vapor && (I & MDN_I_GG))
      for (const V3& c : gas_before)
        for (int a = 0; a < n; a++) {
          double dx = X[a][0] - c[0], dy = X[a][1] - c[1], dz = X[a][2] - c[2];
          if (dx * dx + dy * dy + dz * dz < d2min) return false;
        }
    return true;
  }

  void insert_gas(int m, int t = 0) {
    int mi = 1 + m;
    V3* x = &gx[(size_t)m * a_g];
    V3* v = &gv[(size_t)m * a_g];
    for (int a = 0; a < a_g; a++) { x[a] = gas.x[a]; v[a] = {0, 0, 0}; }
    if (gas_kind == MDN_GAS_N2 && a_g == 2) {
      orc::U4 s = draw(mi, 1, 1);
      double vy_rot, vz_rot;
      orc::box_muller(s.v[0], s.v[1], &vy_rot, &vz_rot);
      vy_rot *= gas_sigma;
      vz_rot *= gas_sigma;
      double vz_use = (quirks & MDN_Q_N2_ROT_VYVZ) ? vy_rot : vz_rot;
      v[0] = {0, vy_rot, vz_use};
      v[1] = {0, -vy_rot, -vz_use};
    }
    orc::U4 s = draw(mi, 1, insert_word(t));
    double a = orc::u01(s.v[0]) * 2 * M_PI;
    double b = orc::u01(s.v[1]) * 2 * M_PI;
    double c = orc::u01(s.v[2]) * 2 * M_PI;
    bool zy = (quirks & MDN_Q_GAS_ROT_ZY) != 0;
    for (int k = 0; k < a_g; k++) {
      V3& ag = x[k];
      rotation(ag[0], ag[1], ag[2], a, b, c, ag[0], ag[1], zy ? ag[1] : ag[2]);
      ag[0] += mol_x[mi][0];
      ag[1] += mol_x[mi][1];
      ag[2] += mol_x[mi][2];
    }
    for (int k = 0; k < a_g; k++) {
      V3& ag = v[k];
      rotation(ag[0], ag[1], ag[2], a, b, c, ag[0], ag[1], zy ? ag[1] : ag[2]);
      ag[0] += mol_v[mi][0];
      ag[1] += mol_v[mi][1];
      ag[2] += mol_v[mi][2];
    }
    for (int k = 0; k < a_g; k++) gf[(size_t)m * a_g + k] = {0, 0, 0};
    /* as for vapor (insert_vapor): MD::update_position ran before this
     * rebuild, so the entering molecule's taper weights, which only the
     * gas-gas term reads, are 0 on this step */
    for (int k = 0; k < a_g; k++) gw[(size_t)m * a_g + k] = 0;
  }

  void insert_vapor(int m, int t = 0) {
    int mi = 1 + n_gas + m;
    V3* x = &vx[(size_t)m * a_v];
    V3* v = &vv[(size_t)m * a_v];
    V3* f = &vf[(size_t)m * a_v];
    for (int a = 0; a < a_v; a++) { x[a] = vap.x[a]; v[a] = {0, 0, 0}; f[a] = {0, 0, 0}; }
    /* MD::update_position ran before this rebuild, while the molecule was
     * outside, so its weights are not set for the current step: a first entry
     * has 0 (initializationVapor.cpp:70-71); a re-entry would carry the weights
     * of its previous visit, which this restatement (and the engine) also
     * sets to 0 */
    for (int a = 0; a < a_v; a++) vw[(size_t)m * a_v + a] = 0;
    orc::U4 s = draw(mi, 1, insert_word(t));
    double a = orc::u01(s.v[0]) * 2 * M_PI;
    double b = orc::u01(s.v[1]) * 2 * M_PI;
    double c = orc::u01(s.v[2]) * 2 * M_PI;
    for (int k = 0; k < a_v; k++) {
      V3& ag = x[k];
      rotation(ag[0], ag[1], ag[2], a, b, c, ag[0], ag[1], ag[2]);
      ag[0] += mol_x[mi][0];
      ag[1] += mol_x[mi][1];
      ag[2] += mol_x[mi][2];
    }
    for (int k = 0; k < a_v; k++) {
      V3& ag = v[k];
      rotation(ag[0], ag[1], ag[2], a, b, c, ag[0], ag[1], ag[2]);
      ag[0] += mol_v[mi][0];
      ag[1] += mol_v[mi][1];
      ag[2] += mol_v[mi][2];
    }
  }

  void resample(int mi, double sigma) {
    orc::U4 s = draw(mi, 0, 0);
    double z0, z1, z2, z3;
    orc::box_muller(s.v[0], s.v[1], &z0, &z1);
    orc::box_muller(s.v[2], s.v[3], &z2, &z3);
    mol_v[mi] = {z0 * sigma, z1 * sigma, z2 * sigma};
  }

  void classify(int first, int count, std::vector<int>& in_list, bool vapor) {
    in_list.clear();
    double HL = box * 0.5;
    const V3& x0 = mol_x[0];
    for (int q = 0; q < count; q++) {
      int i = first + q;
      V3& x = mol_x[i];
      double dx = x[0] - x0[0];
      double dy = x[1] - x0[1];
      double dz = x[2] - x0[2];
      double r2 = (dx * dx + dy * dy + dz * dz);
      if (r2 < RI2) {
        if (!region[i]) {
          if (quirks & MDN_Q_BLIND_INSERT) {
            if (vapor) insert_vapor(q); else insert_gas(q);
          } else {
            /* re-draw the rotation until no atom overlaps; all draws failing
             * leaves the molecule outside until the next rebuild; at most MDN_INSERT_MAX_VAPOR
             * vapor entries are tested per rebuild, later ones wait */
            if (vapor && n_vapor_candidates++ >= MDN_INSERT_MAX_VAPOR) {
              region[i] = 0;
              continue;
            }
            int t = 0;
            for (; t < MDN_INSERT_TRIES; t++) {
              if (vapor) insert_vapor(q, t); else insert_gas(q, t);
              const V3* X = vapor ? &vx[(size_t)q * a_v] : &gx[(size_t)q * a_g];
              if (insert_clear(X, vapor ? a_v : a_g, vapor)) break;
            }
            if (t == MDN_INSERT_TRIES) {
              region[i] = 0;
              continue;
            }
            if (vapor)
              for (int a = 0; a < a_v; a++) new_vapor.push_back(vx[(size_t)q * a_v + a]);
          }
        }
        in_list.push_back(q);
        region[i] = 1;
      } else {
        region[i] = 0;
        if (dx < -HL) x[0] += box;
        if (dy < -HL) x[1] += box;
        if (dz < -HL) x[2] += box;
        if (dx > HL) x[0] -= box;
        if (dy > HL) x[1] -= box;
        if (dz > HL) x[2] -= box;
        resample(i, vapor ? vap_sigma : gas_sigma);
      }
    }
  }

  double d2(const V3& a, const V3& b) const {
    double dx = a[0] - b[0];
    double dy = a[1] - b[1];
    double dz = a[2] - b[2];
    return (dx * dx + dy * dy + dz * dz);
  }

  void make_lists() {
    gi_list.clear();
    gv_list.clear();
    gg_list.clear();
    if (I & MDN_I_GI)
      for (int m : gas_in)
        for (int j = 0; j < ion.n; j++)
          if (d2(mol_x[1 + m], ion_x[j]) < ML2) gi_list.push_back({m, j});
    if (I & MDN_I_GG)
      for (size_t a = 0; a < gas_in.size(); a++)
        for (size_t b = a + 1; b < gas_in.size(); b++)
          if (d2(mol_x[1 + gas_in[a]], mol_x[1 + gas_in[b]]) < ML2) gg_list.push_back({gas_in[a], gas_in[b]});
    if (I & MDN_I_GV)
      for (int m : gas_in)
        for (int q : vap_in)
          if (d2(mol_x[1 + m], mol_x[1 + n_gas + q]) < ML2) gv_list.push_back({m, q});
  }

  void make_pair() {
    for (int q = 0; q < n_gas; q++) {
      int i = 1 + q;
      if (region[i]) continue;
      for (int k = 0; k < 3; k++) mol_x[i][k] += mol_v[i][k] * dt * loop_pair;
    }
    for (int q = 0; q < n_vap; q++) {
      int i = 1 + n_gas + q;
      if (region[i]) continue;
      for (int k = 0; k < 3; k++) mol_x[i][k] += mol_v[i][k] * dt * loop_pair;
    }
    update_in_centers();
    core_before.assign(ion_x.begin(), ion_x.end());
    for (int q : vap_in)
      for (int a = 0; a < a_v; a++) core_before.push_back(vx[(size_t)q * a_v + a]);
    gas_before.clear();
    if (!(quirks & MDN_Q_BLIND_INSERT))
      for (int m : gas_in)
        for (int a = 0; a < a_g; a++) gas_before.push_back(gx[(size_t)m * a_g + a]);
    /* vapor entries are decided first so that gas entries are tested against
     * them (each molecule's draws are independent of this order) */
    new_vapor.clear();
    n_vapor_candidates = 0;
    classify(1 + n_gas, n_vap, vap_in, true);
    classify(1, n_gas, gas_in, false);
    make_lists();
    double vmax2 = 0.0;
    for (auto& v : mol_v) {
      double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      if (vmax2 < v2) vmax2 = v2;
    }
    double vmax = sqrt(vmax2);
    double lu = margin_length / (vmax * dt);
    loop_update = lu >= 2147483647.0 ? 2147483647 : (int)lu;
    loop_pair = 0;
    n_rebuilds++;
  }

  void check_pairlist() {
    loop_pair++;
    if (loop_pair > loop_update) make_pair();
  }

  /* ---------------------------------------------------------------------- */
  /* forces                                                                  */
  void lj_pair(V3& fi, V3& fj, const V3& xi, const V3& xj, int ti, int tj, double wij, int bucket,
               bool coul, double qi, double qj, bool weighted) {
    double dx = xi[0] - xj[0];
    double dy = xi[1] - xj[1];
    double dz = xi[2] - xj[2];
    double rsq = (dx * dx + dy * dy + dz * dz);
    double r2inv = 1 / rsq;
    double r6inv = r2inv * r2inv * r2inv;
    double force_pair;
    if (!coul && !weighted) {
      force_pair = r6inv * (A(ti, tj) * r6inv - B(ti, tj)) * r2inv;
    } else {
      double force_lj = r6inv * (A(ti, tj) * r6inv - B(ti, tj));
      double force_coul = coul ? qqrd2e * qi * qj * sqrt(r2inv) : 0.0;
      force_pair = coul ? (force_lj + force_coul) * r2inv : (force_lj) * r2inv;
      if (weighted) force_pair = force_pair * wij;
      if (eflag && coul) {
        U[bucket] += r6inv * (A(ti, tj) / 12.0 * r6inv - B(ti, tj) / 6.0);
        U[bucket] += force_coul;
      }
    }
    fi[0] += force_pair * dx;
    fi[1] += force_pair * dy;
    fi[2] += force_pair * dz;
    fj[0] -= force_pair * dx;
    fj[1] -= force_pair * dy;
    fj[2] -= force_pair * dz;
    if (eflag && !coul) U[bucket] += r6inv * (A(ti, tj) / 12.0 * r6inv - B(ti, tj) / 6.0);
  }

  void bond_term(V3* x, V3* f, int i, int j, int type, int bucket) {
    double dx = x[i][0] - x[j][0];
    double dy = x[i][1] - x[j][1];
    double dz = x[i][2] - x[j][2];
    double rsq = (dx * dx + dy * dy + dz * dz);
    double r = sqrt(rsq);
    double dr = (r - bond_c[type][1]);
    double rk = bond_c[type][0] * dr;
    double force_bond_harmonic = -2.0 * rk / r;
    f[i][0] += force_bond_harmonic * dx;
    f[i][1] += force_bond_harmonic * dy;
    f[i][2] += force_bond_harmonic * dz;
    f[j][0] -= force_bond_harmonic * dx;
    f[j][1] -= force_bond_harmonic * dy;
    f[j][2] -= force_bond_harmonic * dz;
    if (eflag) U[bucket] += rk * dr;
  }

  void angle_term(V3* x, V3* f, int i, int j, int k, int type, int bucket) {
    double f1[3], f3[3];
    double dx1 = x[i][0] - x[j][0];
    double dy1 = x[i][1] - x[j][1];
    double dz1 = x[i][2] - x[j][2];
    double rsq1 = (dx1 * dx1 + dy1 * dy1 + dz1 * dz1);
    double r1 = sqrt(rsq1);
    double dx2 = x[k][0] - x[j][0];
    double dy2 = x[k][1] - x[j][1];
    double dz2 = x[k][2] - x[j][2];
    double rsq2 = (dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
    double r2 = sqrt(rsq2);
    double C = dx1 * dx2 + dy1 * dy2 + dz1 * dz2;
    C /= r1 * r2;
    double Cs = 1 / (sqrt(1.0 - C * C));
    double dtheta = acos(C) - angle_c[type][1];
    double tk = angle_c[type][0] * dtheta;
    double a = -2.0 * tk * Cs;
    double a11 = a * C / rsq1;
    double a12 = -a / (r1 * r2);
    double a22 = a * C / rsq2;
    f1[0] = a11 * dx1 + a12 * dx2;
    f1[1] = a11 * dy1 + a12 * dy2;
    f1[2] = a11 * dz1 + a12 * dz2;
    f3[0] = a22 * dx2 + a12 * dx1;
    f3[1] = a22 * dy2 + a12 * dy1;
    f3[2] = a22 * dz2 + a12 * dz1;
    f[i][0] += f1[0];
    f[i][1] += f1[1];
    f[i][2] += f1[2];
    f[j][0] -= f1[0] + f3[0];
    f[j][1] -= f1[1] + f3[1];
    f[j][2] -= f1[2] + f3[2];
    f[k][0] += f3[0];
    f[k][1] += f3[1];
    f[k][2] += f3[2];
    if (eflag) U[bucket] += tk * dtheta;
  }

  void dihedral_term(V3* x, V3* f, int i, int j, int k, int l, int type, int bucket) {
    double vb1x = x[i][0] - x[j][0];
    double vb1y = x[i][1] - x[j][1];
    double vb1z = x[i][2] - x[j][2];
    double vb2x = x[k][0] - x[j][0];
    double vb2y = x[k][1] - x[j][1];
    double vb2z = x[k][2] - x[j][2];
    double vb2xm = -vb2x;
    double vb2ym = -vb2y;
    double vb2zm = -vb2z;
    double vb3x = x[l][0] - x[k][0];
    double vb3y = x[l][1] - x[k][1];
    double vb3z = x[l][2] - x[k][2];
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
    double df = 0.0;
    const double* co = dih_c[type].data();
    for (int JJ = 0; JJ < dih_multi[type]; JJ++) {
      int JJ5 = JJ * 5;
      double p_ = 1.0, df1 = 0.0, ddf1 = 0.0;
      for (int loop = 0; loop < co[JJ5 + 1]; loop++) {
        ddf1 = p_ * c - df1 * s;
        df1 = p_ * s + df1 * c;
        p_ = ddf1;
      }
      p_ = p_ * co[JJ5 + 3] + df1 * co[JJ5 + 4];
      df1 = df1 * co[JJ5 + 3] - ddf1 * co[JJ5 + 4];
      df1 *= -co[JJ5 + 1];
      p_ += 1.0;
      if (co[1] == 0) {  /* tests term 0's periodicity for every term (compute_AMBER.cpp:199) */
        p_ = 1.0 + co[JJ5 + 3];
        df1 = 0.0;
      }
      df += (-co[JJ5] * df1);
      if (eflag) U[bucket] += co[JJ5] * p_;
    }
    double fg = vb1x * vb2xm + vb1y * vb2ym + vb1z * vb2zm;
    double hg = vb3x * vb2xm + vb3y * vb2ym + vb3z * vb2zm;
    double fga = fg * ra2inv * rginv;
    double hgb = hg * rb2inv * rginv;
    double gaa = -ra2inv * rg;
    double gbb = rb2inv * rg;
    double dtfx = gaa * ax, dtfy = gaa * ay, dtfz = gaa * az;
    double dtgx = fga * ax - hgb * bx, dtgy = fga * ay - hgb * by, dtgz = fga * az - hgb * bz;
    double dthx = gbb * bx, dthy = gbb * by, dthz = gbb * bz;
    double sx2 = df * dtgx, sy2 = df * dtgy, sz2 = df * dtgz;
    double ff1[3] = {df * dtfx, df * dtfy, df * dtfz};
    double ff2[3] = {sx2 - ff1[0], sy2 - ff1[1], sz2 - ff1[2]};
    double ff4[3] = {df * dthx, df * dthy, df * dthz};
    double ff3[3] = {-sx2 - ff4[0], -sy2 - ff4[1], -sz2 - ff4[2]};
    for (int q = 0; q < 3; q++) {
      f[i][q] += ff1[q];
      f[j][q] += ff2[q];
      f[k][q] += ff3[q];
      f[l][q] += ff4[q];
    }
  }

  void forces() {
    /* InterInter, registration order (src/initialization/setPotential.cpp:198-270) */
    if (on(MDN_I_GI))
      for (auto& p : gi_list) {
        int m = p[0], j = p[1];
        for (int a = 0; a < a_g; a++)
          lj_pair(gf[(size_t)m * a_g + a], ion_f[j], gx[(size_t)m * a_g + a], ion_x[j], gas.type[a],
                  ion.type[j], 1.0, MDN_U_GI, false, 0, 0, false);
      }
    if (on(MDN_I_VI))
      for (int q : vap_in)
        for (int a = 0; a < a_v; a++)
          for (int j = 0; j < ion.n; j++) {
            size_t o = (size_t)q * a_v + a;
            lj_pair(vf[o], ion_f[j], vx[o], ion_x[j], vap.type[a], ion.type[j], vw[o] * 1.0, MDN_U_VI,
                    true, vap.q[a], ion.q[j], true);
          }
    if (on(MDN_I_GG))
      for (auto& p : gg_list)
        for (int a = 0; a < a_g; a++)
          for (int b = 0; b < a_g; b++) {
            size_t oi = (size_t)p[0] * a_g + a, oj = (size_t)p[1] * a_g + b;
            lj_pair(gf[oi], gf[oj], gx[oi], gx[oj], gas.type[a], gas.type[b], gw[oi] * gw[oj], MDN_U_GG,
                    false, 0, 0, true);
          }
    if (on(MDN_I_GV)) {
      int nj = (quirks & MDN_Q_GV_GAS_COUNT) ? std::min(a_g, a_v) : a_v;
      for (auto& p : gv_list)
        for (int a = 0; a < a_g; a++)
          for (int b = 0; b < nj; b++) {
            size_t oi = (size_t)p[0] * a_g + a, oj = (size_t)p[1] * a_v + b;
            lj_pair(gf[oi], vf[oj], gx[oi], vx[oj], gas.type[a], vap.type[b], 1.0, MDN_U_VG, false, 0, 0,
                    false);
          }
    }
    if (on(MDN_I_VV))
      for (size_t i1 = 0; i1 + 1 < vap_in.size(); i1++)
        for (size_t i2 = i1 + 1; i2 < vap_in.size(); i2++)
          for (int a = 0; a < a_v; a++)
            for (int b = 0; b < a_v; b++) {
              size_t oi = (size_t)vap_in[i1] * a_v + a, oj = (size_t)vap_in[i2] * a_v + b;
              lj_pair(vf[oi], vf[oj], vx[oi], vx[oj], vap.type[a], vap.type[b], vw[oi] * vw[oj], MDN_U_VV,
                      true, vap.q[a], vap.q[b], true);
            }
    if (on(MDN_I_EFIELD))
      for (int i = 0; i < ion.n; i++) {
        double coeff = 5.55e-5 * ion.q[i];
        ion_f[i][0] += coeff * Ef[0];
        ion_f[i][1] += coeff * Ef[1];
        ion_f[i][2] += coeff * Ef[2];
      }
    /* IntraInter */
    if (on(MDN_I_AMBER)) {
      for (int i = 0; i < ion.n - 1; i++)
        for (int j = i + 1; j < ion.n; j++)
          if (!excl[(size_t)i * ion.n + j])
            lj_pair(ion_f[i], ion_f[j], ion_x[i], ion_x[j], ion.type[i], ion.type[j], 1.0, MDN_U_ION, true,
                    ion.q[i], ion.q[j], false);
      for (auto& b : ion.bonds) bond_term(ion_x.data(), ion_f.data(), b[0], b[1], b[2], MDN_U_ION);
      for (auto& a : ion.angles) angle_term(ion_x.data(), ion_f.data(), a[0], a[1], a[2], a[3], MDN_U_ION);
      for (auto& d : ion.dih) dihedral_term(ion_x.data(), ion_f.data(), d[0], d[1], d[2], d[3], d[4], MDN_U_ION);
    }
    if (on(MDN_I_BMH))
      for (int i = 0; i < ion.n - 1; i++)
        for (int j = i + 1; j < ion.n; j++) {
          const double* c = born.c[bmh[i]][bmh[j]];
          double dx = ion_x[i][0] - ion_x[j][0];
          double dy = ion_x[i][1] - ion_x[j][1];
          double dz = ion_x[i][2] - ion_x[j][2];
          double rsq = (dx * dx + dy * dy + dz * dz);
          double r2inv = 1 / rsq;
          double r6inv = r2inv * r2inv * r2inv;
          double r = sqrt(rsq);
          double rexp = exp(c[4] * (c[3] - r));
          double force1 = c[4] * c[0] * r * rexp;
          double force2 = -c[1] * r6inv;
          double force3 = -c[2] * r6inv * r2inv;
          double force_coul = qqrd2e * ion.q[i] * ion.q[j] * sqrt(r2inv);
          double force_pair = (force1 + force2 + force3 + force_coul) * r2inv;
          ion_f[i][0] += force_pair * dx;
          ion_f[i][1] += force_pair * dy;
          ion_f[i][2] += force_pair * dz;
          ion_f[j][0] -= force_pair * dx;
          ion_f[j][1] -= force_pair * dy;
          ion_f[j][2] -= force_pair * dz;
          if (eflag) {
            U[MDN_U_ION] += force_coul;
            U[MDN_U_ION] += rexp * c[0];
            U[MDN_U_ION] -= c[1] / 6.0 * r6inv;
            U[MDN_U_ION] -= c[2] / 8.0 * r6inv * r2inv;
          }
        }
    if (on(MDN_I_VAPOR_INTRA)) {
      bool qb = (quirks & MDN_Q_ENERGY_BUCKETS) != 0;
      for (int q : vap_in) {
        V3* x = &vx[(size_t)q * a_v];
        V3* f = &vf[(size_t)q * a_v];
        for (auto& b : vap.bonds) bond_term(x, f, b[0], b[1], b[2], qb ? MDN_U_GAS : MDN_U_VAP);
        for (auto& a : vap.angles) angle_term(x, f, a[0], a[1], a[2], a[3], qb ? MDN_U_GAS : MDN_U_VAP);
        for (auto& d : vap.dih) dihedral_term(x, f, d[0], d[1], d[2], d[3], d[4], qb ? MDN_U_ION : MDN_U_VAP);
      }
    }
    if (on(MDN_I_GAS_INTRA))
      for (int m : gas_in)
        for (auto& b : gas.bonds)
          bond_term(&gx[(size_t)m * a_g], &gf[(size_t)m * a_g], b[0], b[1], b[2], MDN_U_GAS);
  }

  /* ---------------------------------------------------------------------- */
  void verlet() {
    velocity_calculation();
    if (nvt_mode == MDN_NVT_SCALE) velocity_scaling();
    update_position();
    if (nvt_mode == MDN_NVT_NH) nosehoover_zeta();
    check_pairlist();
    forces();
    velocity_calculation();
    if (nvt_mode == MDN_NVT_NH) nosehoover_ion();
    step++;
  }

  /* The gradient harness's objective at the current state:
   *   w_energy * U_vi + w_count * sum_m 1 / (1 + exp((|c_m - c_ion| - R0) / W))
   * U_vi as PotentialVaporIon accumulates it (src/potential/VaporIon.cpp:5-43,
   * unweighted), c_m the mass centre of in-domain vapor molecule m, c_ion the
   * ion's mass centre of its atom positions. */
  double objective(double R0, double W, double we, double wc) const {
    double U = 0;
    for (int q : vap_in)
      for (int a = 0; a < a_v; a++) {
        const V3& xa = vx[(size_t)q * a_v + a];
        for (int j = 0; j < ion.n; j++) {
          double dx = xa[0] - ion_x[j][0], dy = xa[1] - ion_x[j][1], dz = xa[2] - ion_x[j][2];
          double r2 = dx * dx + dy * dy + dz * dz;
          double r2inv = 1 / r2;
          double r6inv = r2inv * r2inv * r2inv;
          int ta = vap.type[a], tj = ion.type[j];
          U += r6inv * (A(ta, tj) / 12.0 * r6inv - B(ta, tj) / 6.0) + qqrd2e * vap.q[a] * ion.q[j] * sqrt(r2inv);
        }
      }
    V3 c = {0, 0, 0};
    for (int j = 0; j < ion.n; j++)
      for (int k = 0; k < 3; k++) c[k] += ion_x[j][k] * ion.mass[j];
    for (int k = 0; k < 3; k++) c[k] /= ion.msum;
    double S = 0;
    for (int q : vap_in) {
      V3 cm = {0, 0, 0};
      for (int a = 0; a < a_v; a++)
        for (int k = 0; k < 3; k++) cm[k] += vx[(size_t)q * a_v + a][k] * vap.mass[a];
      double d2 = 0;
      for (int k = 0; k < 3; k++) {
        double dk = cm[k] / vap.msum - c[k];
        d2 += dk * dk;
      }
      S += 1.0 / (1.0 + exp((sqrt(d2) - R0) / W));
    }
    return we * U + wc * S;
  }

  void build_exclusions() {
    excl.assign((size_t)ion.n * ion.n, 0);
    auto mark = [&](int i, int j) {
      excl[(size_t)i * ion.n + j] = 1;
      excl[(size_t)j * ion.n + i] = 1;
    };
    for (auto& b : ion.bonds) mark(b[0], b[1]);
    for (auto& b : ion.rigid) mark(b[0], b[1]);
    for (auto& a : ion.angles) mark(a[0], a[2]);
    for (auto& d : ion.dih) mark(d[0], d[3]);
  }
};

Oracle* create(const mdn_replica_desc* d, unsigned quirks, int force_mode) {
  Oracle* o = new Oracle();
  o->quirks = quirks;
  o->force_mode = force_mode;
  o->I = d->interactions;
  o->nt = d->n_atom_types;
  o->ljA.resize((size_t)o->nt * o->nt);
  o->ljB.resize((size_t)o->nt * o->nt);
  for (int i = 0; i < o->nt; i++)
    for (int j = 0; j < o->nt; j++) {
      double epu = d->pair_eps ? d->pair_eps[(size_t)i * o->nt + j] : sqrt(d->atom_eps[i] * d->atom_eps[j]);
      double sigma = d->pair_sigma ? d->pair_sigma[(size_t)i * o->nt + j] : (d->atom_sigma[i] + d->atom_sigma[j]) * 0.5;
      o->ljA[(size_t)i * o->nt + j] = 48 * epu * pow(sigma, 12.0);
      o->ljB[(size_t)i * o->nt + j] = 24 * epu * pow(sigma, 6.0);
    }
  for (int t = 0; t < d->n_bond_types; t++) o->bond_c.push_back({d->bond_coeff[2 * t], d->bond_coeff[2 * t + 1]});
  for (int t = 0; t < d->n_angle_types; t++) o->angle_c.push_back({d->angle_coeff[2 * t], d->angle_coeff[2 * t + 1]});
  for (int t = 0; t < d->n_dihedral_types; t++) {
    o->dih_multi.push_back(d->dihedral_multi[t]);
    std::array<double, 15> c;
    for (int k = 0; k < 15; k++) c[k] = d->dihedral_coeff[15 * t + k];
    o->dih_c.push_back(c);
  }
  o->ion = load_top(d->ion, d->atom_mass);
  o->gas = load_top(d->gas, d->atom_mass);
  o->vap = load_top(d->vapor, d->atom_mass);
  for (int i = 0; i < d->ion.n_atoms; i++) o->bmh.push_back(d->ion_bmh_type ? d->ion_bmh_type[i] : 0);
  o->gas_kind = d->gas_kind;
  o->gas_com_mass = d->gas_com_mass;
  o->vap_com_mass = d->vapor_com_mass;
  o->gas_sigma = sqrt(kb * d->temperature / d->gas_mb_mass) * 1e-5;
  o->vap_sigma = d->vapor_mb_mass > 0 ? sqrt(kb * d->temperature / d->vapor_mb_mass) * 1e-5 : 0;
  o->n_gas = d->n_gas;
  o->n_vap = d->n_vapor;
  o->a_g = d->gas.n_atoms;
  o->a_v = d->vapor.n_atoms;
  o->dt = d->dt;
  o->T = d->temperature;
  o->box = d->box;
  o->ML2 = (d->cutoff + d->margin) * (d->cutoff + d->margin);
  o->Ri2 = d->r_inter * d->r_inter;
  o->RI2 = (d->r_inter + d->overlap) * (d->r_inter + d->overlap);
  o->Rcenter = d->r_inter - d->overlap * 0.5;
  o->Overlap = d->overlap;
  o->margin = d->margin;
  o->margin_length = d->margin;
  o->nvt_mode = d->nvt_mode;
  o->nvt_T = d->nvt_temperature;
  for (int k = 0; k < 3; k++) o->Ef[k] = d->efield[k];
  o->key0 = (uint32_t)(d->seed & 0xffffffffull);
  o->key1 = (uint32_t)(d->seed >> 32);
  o->build_exclusions();
  /* state */
  o->ion_x = o->ion.x;
  for (int i = 0; i < o->ion.n; i++) {
    o->ion_v.push_back({d->ion_v[3 * i], d->ion_v[3 * i + 1], d->ion_v[3 * i + 2]});
    o->ion_f.push_back({0, 0, 0});
  }
  int nm = 1 + o->n_gas + o->n_vap;
  o->mol_x.assign(nm, {0, 0, 0});
  o->mol_v.assign(nm, {0, 0, 0});
  o->region.assign(nm, 0);
  o->region[0] = 1;
  for (int q = 0; q < o->n_gas; q++)
    for (int k = 0; k < 3; k++) {
      o->mol_x[1 + q][k] = d->gas_x[3 * q + k];
      o->mol_v[1 + q][k] = d->gas_v[3 * q + k];
    }
  for (int q = 0; q < o->n_vap; q++)
    for (int k = 0; k < 3; k++) {
      o->mol_x[1 + o->n_gas + q][k] = d->vapor_x[3 * q + k];
      o->mol_v[1 + o->n_gas + q][k] = d->vapor_v[3 * q + k];
    }
  o->gx.assign((size_t)o->n_gas * o->a_g, {0, 0, 0});
  o->gv = o->gx;
  o->gf = o->gx;
  o->gw.assign((size_t)o->n_gas * o->a_g, 0);
  o->vx.assign((size_t)o->n_vap * o->a_v, {0, 0, 0});
  o->vv = o->vx;
  o->vf = o->vx;
  o->vw.assign((size_t)o->n_vap * o->a_v, 0);
  o->loop_pair = 0;
  o->make_pair();  /* MD::MD's initial make_pair; loopPair = 0, so no free flight */
  return o;
}

/* the FP64 CPU adjoint of the gradient harness (reverse-mode differentiation
 * of the window's steps) */
#include "adjoint_ad.h"

}  // namespace

extern "C" {

void* orc_create(const mdn_replica_desc* d, unsigned quirks, int force_mode) {
  return create(d, quirks, force_mode);
}
void orc_destroy(void* h) { delete (Oracle*)h; }

void orc_step(void* h, long long n, int energy_mode) {
  Oracle* o = (Oracle*)h;
  for (int k = 0; k < 8; k++) o->U[k] = 0;
  for (long long s = 0; s < n; s++) {
    o->eflag = (energy_mode == 2 || (energy_mode == 1 && s == n - 1)) ? 1 : 0;
    o->verlet();
    o->eflag = 0;
  }
}

void orc_step_many(void** hs, int n, long long steps, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; i++) orc_step(hs[i], steps, 0);
}

void orc_make_pair(void* h) { ((Oracle*)h)->make_pair(); }

void orc_recenter(void* h, int compat) {
  Oracle* o = (Oracle*)h;
  if (compat) {
    /* src/run.cpp:42-53 subtracts position[0] from every entry while that
     * entry is itself being zeroed: only the ion centre moves. */
    o->mol_x[0] = {0, 0, 0};
  } else {
    V3 c = o->mol_x[0];
    for (auto& x : o->mol_x) for (int k = 0; k < 3; k++) x[k] -= c[k];
    for (auto& x : o->ion_x) for (int k = 0; k < 3; k++) x[k] -= c[k];
    for (auto& x : o->gx) for (int k = 0; k < 3; k++) x[k] -= c[k];
    for (auto& x : o->vx) for (int k = 0; k < 3; k++) x[k] -= c[k];
  }
  o->make_pair();
}

void orc_set_nvt(void* h, int mode, double T) {
  Oracle* o = (Oracle*)h;
  o->nvt_mode = mode;
  o->nvt_T = T;
}

void orc_compute_forces(void* h, unsigned term_mask) {
  Oracle* o = (Oracle*)h;
  for (auto& f : o->ion_f) f = {0, 0, 0};
  for (int m : o->gas_in) for (int a = 0; a < o->a_g; a++) o->gf[(size_t)m * o->a_g + a] = {0, 0, 0};
  for (int m : o->vap_in) for (int a = 0; a < o->a_v; a++) o->vf[(size_t)m * o->a_v + a] = {0, 0, 0};
  for (int k = 0; k < 8; k++) o->U[k] = 0;
  o->eflag = 1;
  o->term_mask = term_mask;
  o->forces();
  o->term_mask = 0;
  o->eflag = 0;
}

void orc_energies(void* h, double* U) {
  for (int k = 0; k < 8; k++) U[k] = ((Oracle*)h)->U[k];
}

int orc_status(void* h) { return ((Oracle*)h)->status; }

void orc_info(void* h, mdn_replica_info* i) {
  Oracle* o = (Oracle*)h;
  memset(i, 0, sizeof *i);
  i->n_ion = o->ion.n;
  i->gas_atoms = o->a_g;
  i->vapor_atoms = o->a_v;
  i->n_gas = o->n_gas;
  i->n_vapor = o->n_vap;
  i->n_gas_in = (int)o->gas_in.size();
  i->n_vapor_in = (int)o->vap_in.size();
  i->loop_pair = o->loop_pair;
  i->loop_update = o->loop_update;
  i->n_rebuilds = o->n_rebuilds;
  i->step = o->step;
  i->status = o->status;
  i->gi_pairs = (int)o->gi_list.size();
  i->gv_pairs = (int)o->gv_list.size();
  i->gg_pairs = (int)o->gg_list.size();
}

void orc_get_state(void* h, mdn_state* s) {
  Oracle* o = (Oracle*)h;
  auto put = [](double* dst, const std::vector<V3>& src) {
    if (!dst) return;
    for (size_t i = 0; i < src.size(); i++) for (int k = 0; k < 3; k++) dst[3 * i + k] = src[i][k];
  };
  put(s->ion_x, o->ion_x);
  put(s->ion_v, o->ion_v);
  put(s->ion_f, o->ion_f);
  put(s->mol_x, o->mol_x);
  put(s->mol_v, o->mol_v);
  if (s->region) for (size_t i = 0; i < o->region.size(); i++) s->region[i] = o->region[i];
  put(s->gas_ax, o->gx);
  put(s->gas_av, o->gv);
  put(s->gas_af, o->gf);
  put(s->vap_ax, o->vx);
  put(s->vap_av, o->vv);
  put(s->vap_af, o->vf);
  if (s->vap_w) for (size_t i = 0; i < o->vw.size(); i++) s->vap_w[i] = o->vw[i];
  s->loop_pair = o->loop_pair;
  s->loop_update = o->loop_update;
  s->zeta = o->zeta;
  s->margin_length = o->margin_length;
}

void orc_set_state(void* h, const mdn_state* s) {
  Oracle* o = (Oracle*)h;
  auto get = [](std::vector<V3>& dst, const double* src) {
    if (!src) return;
    for (size_t i = 0; i < dst.size(); i++) for (int k = 0; k < 3; k++) dst[i][k] = src[3 * i + k];
  };
  get(o->ion_x, s->ion_x);
  get(o->ion_v, s->ion_v);
  get(o->ion_f, s->ion_f);
  get(o->mol_x, s->mol_x);
  get(o->mol_v, s->mol_v);
  if (s->region) for (size_t i = 1; i < o->region.size(); i++) o->region[i] = s->region[i] ? 1 : 0;
  get(o->gx, s->gas_ax);
  get(o->gv, s->gas_av);
  get(o->gf, s->gas_af);
  get(o->vx, s->vap_ax);
  get(o->vv, s->vap_av);
  get(o->vf, s->vap_af);
  if (s->vap_w) for (size_t i = 0; i < o->vw.size(); i++) o->vw[i] = s->vap_w[i];
  o->gas_in.clear();
  o->vap_in.clear();
  for (int q = 0; q < o->n_gas; q++) if (o->region[1 + q]) o->gas_in.push_back(q);
  for (int q = 0; q < o->n_vap; q++) if (o->region[1 + o->n_gas + q]) o->vap_in.push_back(q);
  o->make_lists();
  o->loop_pair = s->loop_pair;
  o->loop_update = s->loop_update;
  o->zeta = s->zeta;
  if (s->margin_length > 0) o->margin_length = s->margin_length;
}

int orc_pair_list(void* h, int kind, int* pairs, int capacity) {
  Oracle* o = (Oracle*)h;
  const auto& L = kind == 0 ? o->gi_list : kind == 1 ? o->gv_list : o->gg_list;
  int n = (int)L.size();
  for (int i = 0; i < n && i < capacity; i++) {
    pairs[2 * i] = L[i][0];
    pairs[2 * i + 1] = L[i][1];
  }
  return n;
}

/* Kion, Kgas, Kvap, Tion (Observer::computeProps) */
/* The gradient harness's objective at the current state (Oracle::objective). */
double orc_objective(void* h, double R0, double W, double we, double wc) {
  return ((Oracle*)h)->objective(R0, W, we, wc);
}

/* Advances n steps and returns the window average of the objective after
 * each step: the quantity mdn_adjoint differentiates. */
/* The window objective over the next n steps and its gradient by the FP64
 * CPU adjoint (adjoint_ad.h); theta / rows as mdn_adjoint_params (nrows rows,
 * 2 (nrows - 1) + 1 parameters, the values the replica was built with).
 * Returns 0, -1 for a window mdn_adjoint refuses too, -2 when SHAKE did not
 * converge.  The replica is not advanced. */
int orc_adjoint(void* h, long long n, double R0, double W, double we, double wc, const double* theta,
                const int* rows, int nrows, double* J, double* grad) {
  return adj::window_adjoint(*(Oracle*)h, n, R0, W, we, wc, theta, rows, nrows, J, grad);
}

double orc_window(void* h, long long n, double R0, double W, double we, double wc) {
  Oracle* o = (Oracle*)h;
  double s = 0;
  for (int k = 0; k < 8; k++) o->U[k] = 0;
  for (long long t = 0; t < n; t++) {
    o->eflag = 0;
    o->verlet();
    s += o->objective(R0, W, we, wc);
  }
  return n > 0 ? s / (double)n : 0.0;
}

void orc_kinetic(void* h, double* out) {
  Oracle* o = (Oracle*)h;
  double Kg = 0, Kv = 0;
  for (int q = 0; q < o->n_gas; q++) {
    const V3& v = o->mol_v[1 + q];
    Kg += v[0] * v[0] * o->gas_com_mass;
    Kg += v[1] * v[1] * o->gas_com_mass;
    Kg += v[2] * v[2] * o->gas_com_mass;
  }
  Kg *= (0.5 * real_to_kcalmol);
  for (int q = 0; q < o->n_vap; q++) {
    const V3& v = o->mol_v[1 + o->n_gas + q];
    Kv += v[0] * v[0] * o->vap_com_mass;
    Kv += v[1] * v[1] * o->vap_com_mass;
    Kv += v[2] * v[2] * o->vap_com_mass;
  }
  Kv *= 0.5 * real_to_kcalmol;
  double Tion = o->ion_temperature();
  out[0] = Tion * double(o->ion.n) / (kb_real_inv / 1.5);
  out[1] = Kg;
  out[2] = Kv;
  out[3] = Tion;
}

void orc_rotate(double a, double b, double c, double x, double y, double z, int zy, double* out) {
  rotation(out[0], out[1], out[2], a, b, c, x, y, zy ? y : z);
}

void orc_philox(unsigned long long key, const unsigned* ctr, unsigned* out) {
  orc::U4 c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
  orc::U4 r = orc::philox4x32_10(c, (uint32_t)(key & 0xffffffffull), (uint32_t)(key >> 32));
  for (int k = 0; k < 4; k++) out[k] = r.v[k];
}

/* Initial placement, MD::initialization_gas / initialization_vapor
 * (src/initialization/initializationGas.cpp:24-100,
 * src/initialization/initializationVapor.cpp:14-76), one candidate at a time
 * as the reference loops: the candidate's minimum image distance to every
 * row of the atom table (the ion's atoms, then one row at the origin per
 * molecule already placed) starts at 10000 and keeps the smallest; the
 * candidate is kept when it exceeds min_dist.  The candidates and the
 * velocities come from the stream that mdn_place (include/mdn.h) names:
 * key (seed lo, seed hi); counter (k lo, k hi, purpose, 0x706c6163) with
 * purpose 0 / 1 the gas / vapor centres (x, y, z = (u01(w0..w2) - 0.5) *
 * box), 2 / 3 the gas / vapor velocities of molecule k (Box-Muller on
 * (w0, w1) -> vx, vy and on (w2, w3) -> vz; times sigma, then 1e-5).
 * Returns 0, or -1 when a species needs more than 1000 * (n + 10) draws. */
int orc_place(const mdn_place_desc* p, double* gas_x, double* gas_v, double* vap_x, double* vap_v) {
  const uint32_t k0 = (uint32_t)(p->seed & 0xffffffffull), k1 = (uint32_t)(p->seed >> 32);
  const double L = p->box, LH = 0.5 * L;
  long long placed_rows = 0; /* molecules in the table, all at the origin */
  for (int sp = 0; sp < 2; sp++) {
    const long long n = sp == 0 ? p->n_gas : p->n_vapor;
    double* X = sp == 0 ? gas_x : vap_x;
    double* V = sp == 0 ? gas_v : vap_v;
    const double sigma = sp == 0 ? p->gas_sigma : p->vapor_sigma;
    const long long cap = 1000LL * (n + 10);
    long long i = 0, k = 0;
    while (i < n) {
      if (k >= cap) return -1;
      orc::U4 c = {{(uint32_t)k, (uint32_t)((unsigned long long)k >> 32), (uint32_t)sp, 0x706c6163u}};
      orc::U4 w = orc::philox4x32_10(c, k0, k1);
      k++;
      double Xc[3];
      for (int d = 0; d < 3; d++) Xc[d] = (orc::u01(w.v[d]) - 0.5) * L;
      double min_dis = 10000.0;
      auto row = [&](double ax, double ay, double az) {
        double dx = ax - Xc[0], dy = ay - Xc[1], dz = az - Xc[2];
        if (dx < -LH) dx += L;
        if (dx > LH) dx -= L;
        if (dy < -LH) dy += L;
        if (dy > LH) dy -= L;
        if (dz < -LH) dz += L;
        if (dz > LH) dz -= L;
        double dd = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (dd < min_dis) min_dis = dd;
      };
      for (int a = 0; a < p->n_ion; a++) row(p->ion_x[3 * a], p->ion_x[3 * a + 1], p->ion_x[3 * a + 2]);
      if (placed_rows > 0) row(0.0, 0.0, 0.0);
      if (!(min_dis > p->min_dist)) continue;
      for (int d = 0; d < 3; d++) X[3 * i + d] = Xc[d];
      orc::U4 cv = {{(uint32_t)i, (uint32_t)((unsigned long long)i >> 32), (uint32_t)(2 + sp), 0x706c6163u}};
      orc::U4 wv = orc::philox4x32_10(cv, k0, k1);
      double z[4];
      orc::box_muller(wv.v[0], wv.v[1], &z[0], &z[1]);
      orc::box_muller(wv.v[2], wv.v[3], &z[2], &z[3]);
      for (int d = 0; d < 3; d++) V[3 * i + d] = sigma * z[d] * 1e-5;
      i++;
      placed_rows++;
    }
  }
  return 0;
}

}  // extern "C"
