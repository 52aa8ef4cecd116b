/*
 * mdn_host.cpp -- the C++ host: condition file, molecule files, initial
 * placement, descriptor, run cadence and output files (see mdn_host.h).
 *
 * File formats and behaviours follow the reference:
 *   condition file      MD::readCondFile      src/initialization/setCondition.cpp:4-254
 *   ion / vapor files   Variables::readIonFile / readVaporFile
 *                       src/initialization/readIonFile.cpp:3-179, readVaporFile.cpp:3-131
 *   gas species table   src/initialization/setCondition.cpp:43-118
 *   ion orientation and velocities   Variables::ionInitial, src/initialization/variables.cpp:12-30
 *   gas / vapor placement  MD::initialization_gas / initialization_vapor
 *                       src/initialization/initializationGas.cpp:23-90, initializationVapor.cpp:13-77
 *   run cadence         MD::run, src/run.cpp:17-74
 *   output files        src/output/output.cpp:9-170
 */
#include "mdn_host.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

/* constants of src/constants.hpp:28-53, same expressions */
const double Nw = 6.02e23;
const double kb = 1.38e-23;
const double kb_real = kb * Nw / 4184.0;
const double real_to_kcalmol = 10000 / 4.184;
const double MN2 = 28.0, MHe = 4.0026, MAr = 39.948;
const double R_INTER = 100.0; /* Rinter, src/constants.hpp:44 */
const double OVERLAP = 10.0;  /* Overlap, src/constants.hpp:45 */
const unsigned long long SEED_BASE = 0x4D444E55ULL;

/* splits like std::getline(stream, token, delim): empty fields are kept */
std::vector<std::string> split(const std::string& s, char delim) {
  std::vector<std::string> out;
  std::istringstream in(s);
  std::string tok;
  while (std::getline(in, tok, delim)) out.push_back(tok);
  return out;
}

bool to_double(const std::string& s, double* v) {
  char* end = nullptr;
  *v = strtod(s.c_str(), &end);
  return end != s.c_str();
}

bool to_int(const std::string& s, long long* v) {
  char* end = nullptr;
  *v = strtoll(s.c_str(), &end, 10);
  return end != s.c_str();
}

/* atom-type names of Variables::readIonFile (suffix "") and readVaporFile
 * (suffix "(v)"); the vapor reader names phosphorus "P" without the suffix
 * (src/initialization/readVaporFile.cpp:47-48) */
std::string type_name(const std::string& code, bool vapor) {
  static const char* C[] = {"#c", "#cs", "#c1", "#c2", "#c3", "#ca", "#cp", "#cq", "#cc", "#cd",
                            "#ce", "#cf", "#cg", "#ch", "#cx", "#cy", "#cu", "#cv", "#cz"};
  static const char* H[] = {"#h1", "#h2", "#h3", "#h4", "#h5", "#ha", "#hc",
                            "#hn", "#ho", "#hp", "#hs", "#hw", "#hx"};
  static const char* N[] = {"#n",  "#n1", "#n2", "#n3", "#n4", "#na", "#nb", "#nc", "#nd",
                            "#ne", "#nf", "#nh", "#no", "#ns", "#nt", "#nx", "#ny", "#nz",
                            "#n+", "#nu", "#nv", "#n7", "#n8", "#n9"};
  static const char* O[] = {"#o", "#oh", "#os", "#ow"};
  static const char* P[] = {"#p2", "#p3", "#p4", "#p5", "#pb", "#pc", "#pd", "#pe", "#pf", "#px", "#py"};
  static const char* S[] = {"#s", "#s2", "#s4", "#s6", "#sh", "#ss", "#sx", "#sy"};
  auto in = [&](const char* const* list, size_t n) {
    for (size_t i = 0; i < n; i++)
      if (code == list[i]) return true;
    return false;
  };
  const std::string sfx = vapor ? "(v)" : "";
  if (in(C, sizeof C / sizeof *C)) return "C" + sfx;
  if (in(H, sizeof H / sizeof *H)) return "H" + sfx;
  if (code == "f") return "F" + sfx;
  if (code == "cl") return "Cl" + sfx;
  if (code == "br") return "Br" + sfx;
  if (code == "i") return "I" + sfx;
  if (in(N, sizeof N / sizeof *N)) return "N" + sfx;
  if (in(O, sizeof O / sizeof *O)) return "O" + sfx;
  if (in(P, sizeof P / sizeof *P)) return "P";
  if (in(S, sizeof S / sizeof *S)) return "S" + sfx;
  return code;
}

/* one molecule kind as read from a file, indices global to the replica */
struct Molecule {
  std::vector<int> type;
  std::vector<double> charge, x, v;  /* x, v: 3 per atom */
  std::vector<int> bonds, rigid;     /* 3 per row: i, j, type */
  std::vector<int> angles;           /* 4 per row */
  std::vector<int> dihedrals;        /* 5 per row */
  bool has_velocity = false;
};

}  // namespace

struct mdnh_system {
  mdnh_settings set{};
  std::string cond_path, ion_file, vapor_file, dump_path, gas_name;
  double T = 300, p = 1e5, dt = 0.5, cutoff = 20.0, margin = 10.0;
  double efield[3] = {0, 0, 0};
  bool shake_h = false;
  int nvt_gas = 0;
  unsigned long long seed = 0;
  /* type tables, in the reference's order: gas, ion, vapor */
  std::vector<std::string> names;
  std::vector<double> mass, eps, sigma;
  std::vector<double> bond_coeff, angle_coeff, dihedral_coeff;
  std::vector<int> dihedral_multi;
  Molecule ion, gas, vap;
  std::vector<int> ion_bmh;
  std::vector<double> gas_x, gas_v, vap_x, vap_v;
  double gas_com_mass = 0, gas_mb_mass = 0, vap_com_mass = 0, vap_mb_mass = 0;
  mdn_replica_desc desc{};
};

namespace {

/* ---- the condition file ---------------------------------------------------- */
int read_condition(mdnh_system* s, const char* path, int calc) {
  std::ifstream in(path);
  if (!in) return fail(MDN_ERR_ARG, "cannot open condition file %s", path);
  s->cond_path = path;
  unsigned I = MDN_I_GAS_INTRA | MDN_I_VAPOR_INTRA; /* FLAG::FLAG, src/flags.cpp:39-41 */
  bool have_gas = false;
  int observe = 10000000; /* MD::setDefaultVariables, src/initialization/defaultVariables.cpp:9 */
  long long total = 0, relax = 0;
  int n_gas = 1, n_vap = 1;
  int nvt = MDN_NVT_OFF;
  double nvt_T = 0;
  std::string line;
  int lineno = 0;
  while (std::getline(in, line)) {
    lineno++;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty()) continue;
    std::vector<std::string> r = split(line, ' ');
    if (r.empty()) continue;
    const std::string& k = r[0];
    auto need = [&](size_t n) {
      if (r.size() < n) {
        fail(MDN_ERR_ARG, "%s:%d: '%s' needs %zu fields", path, lineno, k.c_str(), n - 1);
        return false;
      }
      return true;
    };
    double d;
    long long ll;
    if (k == "Input") {
      if (!need(2)) return MDN_ERR_ARG;
      s->ion_file = r[1];
    } else if (k == "Vapor") {
      if (!need(3) || !to_int(r[2], &ll)) return fail(MDN_ERR_ARG, "%s:%d: Vapor <file> <count>", path, lineno);
      s->vapor_file = r[1];
      n_vap = (int)ll;
    } else if (k == "VaporStickPositions") {
      /* the stick-position log of the reference is not produced */
    } else if (k == "Gas") {
      if (!need(3) || !to_int(r[2], &ll)) return fail(MDN_ERR_ARG, "%s:%d: Gas <kind> <count>", path, lineno);
      s->gas_name = r[1];
      n_gas = (int)ll;
      have_gas = true;
    } else if (k == "Temperature") {
      if (!need(2) || !to_double(r[1], &s->T)) return fail(MDN_ERR_ARG, "%s:%d: Temperature <K>", path, lineno);
    } else if (k == "Pressure") {
      if (!need(2) || !to_double(r[1], &s->p)) return fail(MDN_ERR_ARG, "%s:%d: Pressure <Pa>", path, lineno);
    } else if (k == "dt") {
      if (!need(2) || !to_double(r[1], &s->dt)) return fail(MDN_ERR_ARG, "%s:%d: dt <fs>", path, lineno);
    } else if (k == "TotalSteps") {
      if (!need(2) || !to_double(r[1], &d)) return fail(MDN_ERR_ARG, "%s:%d: TotalSteps <n>", path, lineno);
      total = (long long)d;
    } else if (k == "RelaxSteps") {
      if (!need(2) || !to_double(r[1], &d)) return fail(MDN_ERR_ARG, "%s:%d: RelaxSteps <n>", path, lineno);
      relax = (long long)d;
    } else if (k == "CutOff") {
      if (!need(2) || !to_double(r[1], &s->cutoff)) return fail(MDN_ERR_ARG, "%s:%d: CutOff <A>", path, lineno);
    } else if (k == "Margin") {
      if (!need(2) || !to_double(r[1], &s->margin)) return fail(MDN_ERR_ARG, "%s:%d: Margin <A>", path, lineno);
    } else if (k == "Output") {
      if (!need(3) || !to_int(r[2], &ll) || ll <= 0)
        return fail(MDN_ERR_ARG, "%s:%d: Output <prefix> <steps>", path, lineno);
      s->dump_path = r[1] + "_" + std::to_string(calc) + ".dump";
      observe = (int)ll;
      FILE* f = fopen(s->dump_path.c_str(), "w");
      if (!f) return fail(MDN_ERR_ARG, "cannot create %s", s->dump_path.c_str());
      fclose(f);
    } else if (k == "NVTion") {
      if (!need(2)) return MDN_ERR_ARG;
      if (r[1] == "OFF") nvt = MDN_NVT_OFF;
      else if (r[1] == "scale") nvt = MDN_NVT_SCALE;
      else if (to_double(r[1], &nvt_T)) nvt = MDN_NVT_NH;
      else return fail(MDN_ERR_ARG, "%s:%d: NVTion OFF | scale | <K>", path, lineno);
    } else if (k == "NVTgas") {
      /* FLAG::nose_hoover_gas is set by the reference but read nowhere */
      if (need(2) && r[1] != "OFF") s->nvt_gas = 1;
    } else if (k == "Gyration") {
      /* the reference creates the file (src/initialization/setCondition.cpp:229-239) and never writes it */
      if (need(2)) {
        std::string g = r[1] + "_" + std::to_string(calc) + ".dat";
        FILE* f = fopen(g.c_str(), "w");
        if (f) fclose(f);
      }
    } else if (k == "SHAKE") {
      if (need(2) && r[1] == "H") s->shake_h = true;
    }
    /* the Interactions block: the reference tests the second field of every
     * line (src/initialization/setCondition.cpp:186-228) */
    if (k == "Interactions" || r.size() < 3) continue;
    const std::string& w = r[1];
    const std::string& v = r[2];
    if (w == "gg") {
      if (v == "LJ") I |= MDN_I_GG;
      else if (v == "OFF") I &= ~MDN_I_GG;
      else return fail(MDN_ERR_ARG, "%s:%d: unknown gas-gas parameter %s", path, lineno, v.c_str());
    } else if (w == "gi" || w == "ig") {
      if (v == "LJ") I |= MDN_I_GI;
      else if (v == "OFF") I &= ~MDN_I_GI;
      else return fail(MDN_ERR_ARG, "%s:%d: unsupported gas-ion parameter %s", path, lineno, v.c_str());
    } else if (w == "ion") {
      if (v == "AMBER") I |= MDN_I_AMBER;
      else if (v == "Born-Mayer-Huggins-NaCl") I |= MDN_I_BMH;
      else return fail(MDN_ERR_ARG, "%s:%d: unsupported ion potential %s", path, lineno, v.c_str());
    } else if (w == "vi" || w == "iv") {
      if (v == "LJcoul") I |= MDN_I_VI;
      else if (v == "OFF") I &= ~MDN_I_VI;
      else return fail(MDN_ERR_ARG, "%s:%d: unknown vapor-ion parameter %s", path, lineno, v.c_str());
    } else if (w == "vv") {
      if (v == "LJcoul") I |= MDN_I_VV;
      else if (v == "OFF") I &= ~MDN_I_VV;
      else return fail(MDN_ERR_ARG, "%s:%d: unknown vapor-vapor parameter %s", path, lineno, v.c_str());
    } else if (w == "gv" || w == "vg") {
      if (v == "LJ") I |= MDN_I_GV;
      else if (v == "OFF") I &= ~MDN_I_GV;
      else return fail(MDN_ERR_ARG, "%s:%d: unknown gas-vapor parameter %s", path, lineno, v.c_str());
    } else if (w == "Efield") {
      if (r.size() < 5 || !to_double(r[2], &s->efield[0]) || !to_double(r[3], &s->efield[1]) ||
          !to_double(r[4], &s->efield[2]))
        return fail(MDN_ERR_ARG, "%s:%d: Efield <ex> <ey> <ez>", path, lineno);
      I |= MDN_I_EFIELD;
    }
  }
  if (!have_gas) return fail(MDN_ERR_ARG, "%s: no Gas line", path);
  if (s->ion_file.empty()) return fail(MDN_ERR_ARG, "%s: no Input line", path);
  if (s->vapor_file.empty()) return fail(MDN_ERR_ARG, "%s: no Vapor line", path);
  if (s->shake_h) I |= MDN_I_SHAKE;
  mdnh_settings& st = s->set;
  st.total_steps = total;
  st.relax_steps = relax;
  st.observe = observe;
  st.calc_number = calc;
  st.pressure = s->p;
  st.n_gas = n_gas;
  st.n_vapor = n_vap;
  st.interactions = I;
  st.nvt_mode = nvt;
  st.nvt_temperature = nvt_T;
  st.box = pow(n_gas * kb * s->T / s->p, 1 / 3.0) * 1e10; /* src/initialization/setCondition.cpp:247 */
  return MDN_OK;
}

/* ---- the gas table, src/initialization/setCondition.cpp:43-118 ---------- */
int add_gas(mdnh_system* s, int reference_masses) {
  const std::string& g = s->gas_name;
  double m, e, sg, Mref;
  std::string nm;
  std::vector<double> x;
  int kind;
  if (g == "He") {
    kind = MDN_GAS_HE; m = 4.027; nm = "He(g)"; e = 0.0203; sg = 2.556; x = {0, 0, 0}; Mref = MHe;
  } else if (g == "N2") {
    kind = MDN_GAS_N2; m = 14.01; nm = "N(g)"; e = 0.1098; sg = 3.27351824993; x = {-0.549, 0, 0, 0.549, 0, 0};
    Mref = MN2;
  } else if (g == "N2monoatomic") {
    kind = MDN_GAS_N2MONO; m = 28.02; nm = "N2(g)"; e = 0.14397; sg = 3.798; x = {0, 0, 0}; Mref = MN2;
  } else if (g == "Ar") {
    kind = MDN_GAS_AR; m = 28.02; nm = "Ar(g)"; e = 0.14397; sg = 3.798; x = {0, 0, 0}; Mref = MAr;
  } else {
    return fail(MDN_ERR_ARG, "unknown gas %s (He, N2, N2monoatomic, Ar)", g.c_str());
  }
  s->set.gas_kind = kind;
  s->names.push_back(nm);
  s->mass.push_back(m);
  s->eps.push_back(e);
  s->sigma.push_back(sg);
  const int na = (int)x.size() / 3;
  s->gas.x = x;
  s->gas.type.assign(na, 0);
  s->gas.charge.assign(na, 0.0);
  if (kind == MDN_GAS_N2) {
    s->bond_coeff.push_back(1221.7);
    s->bond_coeff.push_back(1.098);
    s->gas.bonds = {0, 1, 0};
  }
  const double sum = m * na;
  s->gas_com_mass = reference_masses ? Mref : sum;
  s->gas_mb_mass = s->gas_com_mass / Nw / 1000.0; /* Physical::setPhysicalProp, src/initialization/PhysicalProp.cpp:26 */
  return MDN_OK;
}

/* ---- ion / vapor files ---------------------------------------------------- */
int read_molecule(mdnh_system* s, const std::string& path, bool vapor, Molecule* mol) {
  std::ifstream in(path);
  if (!in) return fail(MDN_ERR_ARG, "cannot open %s", path.c_str());
  /* the file's 1-based type numbers follow the entries already in the tables */
  const int t_off = (int)s->names.size() - 1;
  const int b_off = (int)(s->bond_coeff.size() / 2) - 1;
  const int c_off = (int)(s->angle_coeff.size() / 2) - 1;
  const int d_off = (int)s->dihedral_multi.size() - 1;
  int flag = 0, lineno = 0;
  std::vector<int> raw_bonds;
  std::string line;
  while (std::getline(in, line)) {
    lineno++;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty()) continue;
    if (line == "atom type") { flag = 1; continue; }
    if (line == "bond type") { flag = 2; continue; }
    if (line == "angle type") { flag = 3; continue; }
    if (line == "dihedral type") { flag = 4; continue; }
    if (line == "atoms") { flag = 5; continue; }
    if (line == "bonds") { flag = 6; continue; }
    if (line == "angles") { flag = 7; continue; }
    if (line == "dihedrals") { flag = 8; continue; }
    std::vector<std::string> r = split(line, '\t');
    std::vector<double> f(r.size(), 0.0);
    for (size_t i = 0; i < r.size(); i++) to_double(r[i], &f[i]);
    auto need = [&](size_t n) {
      if (r.size() < n) {
        fail(MDN_ERR_ARG, "%s:%d: %zu tab-separated fields expected", path.c_str(), lineno, n);
        return false;
      }
      return true;
    };
    switch (flag) {
      case 1:
        if (!need(5)) return MDN_ERR_ARG;
        s->names.push_back(type_name(r[1], vapor));
        s->mass.push_back(f[2]);
        s->eps.push_back(f[3]);
        s->sigma.push_back(f[4]);
        break;
      case 2:
        if (!need(4)) return MDN_ERR_ARG;
        s->bond_coeff.push_back(f[2]);
        s->bond_coeff.push_back(f[3]);
        break;
      case 3:
        if (!need(4)) return MDN_ERR_ARG;
        s->angle_coeff.push_back(f[2]);
        s->angle_coeff.push_back(f[3] / 180.0 * M_PI);
        break;
      case 4: {
        if (!need(12)) return MDN_ERR_ARG;
        s->dihedral_multi.push_back((int)f[2]);
        for (int t = 0; t < 3; t++) {
          const double K = f[3 + 3 * t], n = f[4 + 3 * t], dd = f[5 + 3 * t];
          s->dihedral_coeff.push_back(K);
          s->dihedral_coeff.push_back(n);
          s->dihedral_coeff.push_back(dd);
          s->dihedral_coeff.push_back(cos(dd / 180.0 * M_PI));
          s->dihedral_coeff.push_back(sin(dd / 180.0 * M_PI));
        }
        break;
      }
      case 5: {
        if (!need(6)) return MDN_ERR_ARG;
        const int ty = (int)f[1] + t_off;
        if (ty < 0 || ty >= (int)s->names.size())
          return fail(MDN_ERR_ARG, "%s:%d: atom type %s out of range", path.c_str(), lineno, r[1].c_str());
        mol->type.push_back(ty);
        mol->charge.push_back(f[2]);
        for (int k = 0; k < 3; k++) mol->x.push_back(f[3 + k]);
        if (r.size() > 8) {
          mol->has_velocity = true;
          for (int k = 0; k < 3; k++) mol->v.push_back(f[6 + k]);
        } else {
          for (int k = 0; k < 3; k++) mol->v.push_back(0.0);
        }
        break;
      }
      case 6:
        if (!need(3)) return MDN_ERR_ARG;
        raw_bonds.push_back((int)f[0] - 1);
        raw_bonds.push_back((int)f[1] - 1);
        raw_bonds.push_back((int)f[2] + b_off);
        break;
      case 7:
        if (!need(4)) return MDN_ERR_ARG;
        for (int k = 0; k < 3; k++) mol->angles.push_back((int)f[k] - 1);
        mol->angles.push_back((int)f[3] + c_off);
        break;
      case 8:
        if (!need(5)) return MDN_ERR_ARG;
        for (int k = 0; k < 4; k++) mol->dihedrals.push_back((int)f[k] - 1);
        mol->dihedrals.push_back((int)f[4] + d_off);
        break;
      default:
        break;
    }
  }
  const int na = (int)mol->type.size();
  if (na == 0) return fail(MDN_ERR_ARG, "%s: no atoms", path.c_str());
  /* SHAKE H: bonds with a hydrogen become constraints (readIonFile.cpp:131-136,
   * readVaporFile.cpp:105-110) */
  const std::string h = vapor ? "H(v)" : "H";
  for (size_t b = 0; b + 2 < raw_bonds.size(); b += 3) {
    const int i = raw_bonds[b], j = raw_bonds[b + 1];
    if (i < 0 || j < 0 || i >= na || j >= na) return fail(MDN_ERR_ARG, "%s: bond atom out of range", path.c_str());
    const bool rigid = s->shake_h && (s->names[mol->type[i]] == h || s->names[mol->type[j]] == h);
    std::vector<int>& dst = rigid ? mol->rigid : mol->bonds;
    dst.insert(dst.end(), {i, j, raw_bonds[b + 2]});
  }
  return MDN_OK;
}

/* ---- placement, MD::initialization_gas / _vapor and Variables::ionInitial - */
void rotation(double a, double b, double c, double* v) {
  /* uniform Euler rotation z(a) y(b) z(c) of one vector */
  const double ca = cos(a), sa = sin(a), cb = cos(b), sb = sin(b), cc = cos(c), sc = sin(c);
  const double x = v[0], y = v[1], z = v[2];
  const double x1 = cc * x - sc * y, y1 = sc * x + cc * y, z1 = z;
  const double x2 = cb * x1 + sb * z1, y2 = y1, z2 = -sb * x1 + cb * z1;
  v[0] = ca * x2 - sa * y2;
  v[1] = sa * x2 + ca * y2;
  v[2] = z2;
}

int place(mdnh_system* s, std::mt19937_64& rng, int place_device) {
  const double L = s->set.box, half = 0.5 * L, dis = 10.0;
  const int ni = (int)s->ion.type.size();
  /* orientation of the ion about the origin, uniform on SO(3) */
  {
    std::uniform_real_distribution<double> u(0.0, 1.0);
    const double a = 2 * M_PI * u(rng), c = 2 * M_PI * u(rng), b = acos(1 - 2 * u(rng));
    for (int i = 0; i < ni; i++) rotation(a, b, c, &s->ion.x[3 * i]);
    for (int i = 0; i < ni; i++) {
      const double matom = s->mass[s->ion.type[i]] * 1e-3 / Nw;
      std::normal_distribution<double> n(0.0, sqrt(kb * s->T / matom));
      for (int k = 0; k < 3; k++) s->ion.v[3 * i + k] = n(rng) * 1e-5;
    }
  }
  const int ng = s->set.n_gas, nv = s->set.n_vapor;
  const double gsig = sqrt(kb * s->T / s->gas_mb_mass), vsig = sqrt(kb * s->T / s->vap_mb_mass);
  if (place_device >= 0) {
    mdn_place_desc d;
    memset(&d, 0, sizeof d);
    d.box = L;
    d.min_dist = dis;
    d.n_ion = ni;
    d.ion_x = s->ion.x.data();
    d.n_gas = ng;
    d.n_vapor = nv;
    d.gas_sigma = gsig;
    d.vapor_sigma = vsig;
    d.seed = s->seed;
    s->gas_x.assign(3 * (size_t)ng, 0.0);
    s->gas_v.assign(3 * (size_t)ng, 0.0);
    s->vap_x.assign(3 * (size_t)nv, 0.0);
    s->vap_v.assign(3 * (size_t)nv, 0.0);
    int rc = mdn_place(place_device, &d, s->gas_x.data(), s->gas_v.data(), s->vap_x.data(), s->vap_v.data());
    if (rc) return fail(rc, "placement on device %d: %s", place_device, mdn_last_error());
    return MDN_OK;
  }
  /* a centre is kept when it is farther than 10 A (minimum image) from every
   * row of the reference's atom table: the ion atoms and, once a molecule
   * is placed, the origin, where the not yet inserted molecules' atoms sit */
  long long placed = 0;
  auto ok = [&](const double* X) {
    auto d2 = [&](const double* a) {
      double d[3];
      for (int k = 0; k < 3; k++) {
        d[k] = a[k] - X[k];
        if (d[k] < -half) d[k] += L;
        if (d[k] > half) d[k] -= L;
      }
      return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    };
    const double o[3] = {0, 0, 0};
    if (placed > 0 && sqrt(d2(o)) <= dis) return false;
    for (int i = 0; i < ni; i++)
      if (sqrt(d2(&s->ion.x[3 * i])) <= dis) return false;
    return true;
  };
  std::uniform_real_distribution<double> r(-half, half);
  auto fill = [&](int n, double sigma, std::vector<double>& xs, std::vector<double>& vs, const char* what) {
    std::normal_distribution<double> dist(0.0, sigma);
    xs.clear();
    vs.clear();
    long long tries = 0;
    const long long cap = 1000LL * (n + 10);
    while ((int)xs.size() / 3 < n) {
      if (++tries > cap) return fail(MDN_ERR_ARG, "%s placement did not converge (box %.1f A)", what, L);
      double X[3] = {r(rng), r(rng), r(rng)};
      if (!ok(X)) continue;
      xs.insert(xs.end(), X, X + 3);
      for (int k = 0; k < 3; k++) vs.push_back(dist(rng) * 1e-5);
      placed++;
    }
    return MDN_OK;
  };
  int rc = fill(ng, gsig, s->gas_x, s->gas_v, "gas");
  if (rc) return rc;
  return fill(nv, vsig, s->vap_x, s->vap_v, "vapor");
}

void topo(mdn_topology* t, const Molecule& m) {
  t->n_atoms = (int)m.type.size();
  t->type = m.type.data();
  t->charge = m.charge.data();
  t->x = m.x.data();
  t->n_bonds = (int)m.bonds.size() / 3;
  t->bonds = m.bonds.data();
  t->n_rigid = (int)m.rigid.size() / 3;
  t->rigid = m.rigid.data();
  t->n_angles = (int)m.angles.size() / 4;
  t->angles = m.angles.data();
  t->n_dihedrals = (int)m.dihedrals.size() / 5;
  t->dihedrals = m.dihedrals.data();
}

void build_desc(mdnh_system* s) {
  mdn_replica_desc& d = s->desc;
  memset(&d, 0, sizeof d);
  d.n_atom_types = (int)s->names.size();
  d.atom_mass = s->mass.data();
  d.atom_eps = s->eps.data();
  d.atom_sigma = s->sigma.data();
  d.n_bond_types = (int)s->bond_coeff.size() / 2;
  d.bond_coeff = s->bond_coeff.data();
  d.n_angle_types = (int)s->angle_coeff.size() / 2;
  d.angle_coeff = s->angle_coeff.data();
  d.n_dihedral_types = (int)s->dihedral_multi.size();
  d.dihedral_multi = s->dihedral_multi.data();
  d.dihedral_coeff = s->dihedral_coeff.data();
  topo(&d.ion, s->ion);
  d.ion_v = s->ion.v.data();
  d.ion_bmh_type = s->ion_bmh.data();
  topo(&d.gas, s->gas);
  d.gas_kind = s->set.gas_kind;
  d.gas_com_mass = s->gas_com_mass;
  d.gas_mb_mass = s->gas_mb_mass;
  topo(&d.vapor, s->vap);
  d.vapor_com_mass = s->vap_com_mass;
  d.vapor_mb_mass = s->vap_mb_mass;
  d.n_gas = s->set.n_gas;
  d.gas_x = s->gas_x.data();
  d.gas_v = s->gas_v.data();
  d.n_vapor = s->set.n_vapor;
  d.vapor_x = s->vap_x.data();
  d.vapor_v = s->vap_v.data();
  d.dt = s->dt;
  d.temperature = s->T;
  d.box = s->set.box;
  d.cutoff = s->cutoff;
  d.margin = s->margin;
  d.r_inter = R_INTER;
  d.overlap = OVERLAP;
  d.interactions = s->set.interactions;
  d.nvt_mode = s->set.nvt_mode;
  d.nvt_temperature = s->set.nvt_temperature;
  for (int k = 0; k < 3; k++) d.efield[k] = s->efield[k];
  d.seed = s->seed;
}

/* ---- output files --------------------------------------------------------- */
void append(const std::string& path, const char* fmt, ...) {
  FILE* f = fopen(path.c_str(), "a");
  if (!f) return;
  va_list ap;
  va_start(ap, fmt);
  vfprintf(f, fmt, ap);
  va_end(ap);
  fclose(f);
}

std::string out_name(const char* fmt, int a, int b = 0) {
  char buf[256];
  snprintf(buf, sizeof buf, fmt, a, b);
  return buf;
}

}  // namespace

/* ========================================================================== */
extern "C" {

const char* mdnh_last_error(void) { return g_err.c_str(); }

int mdnh_load(const char* condition_file, int calc_number, unsigned long long seed, int reference_masses,
              mdnh_system** out) {
  return mdnh_load_ex(condition_file, calc_number, seed, reference_masses, -1, out);
}

int mdnh_load_ex(const char* condition_file, int calc_number, unsigned long long seed, int reference_masses,
                 int place_device, mdnh_system** out) {
  if (!condition_file || !out) return fail(MDN_ERR_ARG, "null argument");
  *out = nullptr;
  mdnh_system* s = new mdnh_system();
  s->seed = seed ? seed : SEED_BASE + (unsigned long long)calc_number;
  int rc = read_condition(s, condition_file, calc_number);
  if (!rc) rc = add_gas(s, reference_masses);
  if (!rc) rc = read_molecule(s, s->ion_file, false, &s->ion);
  if (!rc) rc = read_molecule(s, s->vapor_file, true, &s->vap);
  if (rc) {
    delete s;
    return rc;
  }
  /* ion rows of the Born-Mayer-Huggins table: 0 = Na, 1 = Cl */
  const int ni = (int)s->ion.type.size();
  s->ion_bmh.assign(ni, 0);
  if (s->set.interactions & MDN_I_BMH)
    for (int i = 0; i < ni; i++) {
      const std::string& nm = s->names[s->ion.type[i]];
      if (nm == "Na") s->ion_bmh[i] = 0;
      else if (nm == "Cl") s->ion_bmh[i] = 1;
      else {
        delete s;
        return fail(MDN_ERR_ARG, "Born-Mayer-Huggins-NaCl needs Na and Cl ion atoms, found %s", nm.c_str());
      }
    }
  /* vapor molecular mass, Physical::readVaporProp (src/initialization/PhysicalProp.cpp:75-100) */
  double mv = 0;
  for (int t : s->vap.type) mv += s->mass[t];
  s->vap_com_mass = mv;
  s->vap_mb_mass = mv / Nw / 1000.0;
  std::mt19937_64 rng(s->seed);
  rc = place(s, rng, place_device);
  if (rc) {
    delete s;
    return rc;
  }
  build_desc(s);
  *out = s;
  return MDN_OK;
}

void mdnh_free(mdnh_system* s) { delete s; }

const mdn_replica_desc* mdnh_desc(const mdnh_system* s) { return s ? &s->desc : nullptr; }

int mdnh_get_settings(const mdnh_system* s, mdnh_settings* out) {
  if (!s || !out) return fail(MDN_ERR_ARG, "null argument");
  *out = s->set;
  return MDN_OK;
}

const char* mdnh_type_name(const mdnh_system* s, int type) {
  if (!s || type < 0 || type >= (int)s->names.size()) return "";
  return s->names[type].c_str();
}

const char* mdnh_dump_path(const mdnh_system* s) { return s ? s->dump_path.c_str() : ""; }

int mdnh_write_dump_frame(const mdnh_system* s, const char* path, int timestep, int n_rows, const int* type,
                          const double* x, const double* v, const double* shift) {
  if (!s || !path || n_rows < 0 || (n_rows > 0 && (!type || !x || !v))) return fail(MDN_ERR_ARG, "bad arguments");
  FILE* f = fopen(path, "a");
  if (!f) return fail(MDN_ERR_ARG, "cannot append to %s", path);
  const double h = s->set.box * 0.5;
  fprintf(f,
          "ITEM: TIMESTEP\n%d\nITEM: NUMBER OF ATOMS\n%d\nITEM: BOX BOUNDS pp pp pp\n%e %e\n%e %e\n%e %e\n"
          "ITEM: ATOMS id type x y z vx vy vz\n",
          timestep, n_rows, -h, h, -h, h, -h, h);
  const double X = shift ? shift[0] : 0, Y = shift ? shift[1] : 0, Z = shift ? shift[2] : 0;
  for (int i = 0; i < n_rows; i++)
    fprintf(f, "%d %s %f %f %f %f %f %f\n", i, mdnh_type_name(s, type[i]), x[3 * i] - X, x[3 * i + 1] - Y,
            x[3 * i + 2] - Z, v[3 * i], v[3 * i + 1], v[3 * i + 2]);
  fclose(f);
  return MDN_OK;
}

int mdnh_run(mdnh_system* const* systems, int n, const mdn_options* opt, int verbose) {
  if (!systems || n <= 0) return fail(MDN_ERR_ARG, "no systems");
  const mdnh_settings& s0 = systems[0]->set;
  for (int r = 1; r < n; r++) {
    const mdnh_settings& sr = systems[r]->set;
    if (sr.total_steps != s0.total_steps || sr.relax_steps != s0.relax_steps || sr.observe != s0.observe ||
        systems[r]->dt != systems[0]->dt)
      return fail(MDN_ERR_ARG, "a batch needs the same step counts, Output cadence and dt in every system");
  }
  std::vector<mdn_replica_desc> descs(n);
  for (int r = 0; r < n; r++) descs[r] = systems[r]->desc;
  mdn_handle* h = nullptr;
  int rc = mdn_create(descs.data(), n, opt, &h);
  if (rc) return fail(rc, "mdn_create: %s", mdn_last_error());
  const double dt = systems[0]->dt;
  const int OBSERVE = s0.observe;
  const long long logger = 10000; /* src/run.cpp:19 */

  /* output names, src/output/output.cpp:9-29 */
  std::vector<std::string> f_ion(n), f_vin(n), f_vout(n), f_K(n), f_U(n);
  for (int r = 0; r < n; r++) {
    const mdnh_system* s = systems[r];
    const int c = s->set.calc_number;
    f_ion[r] = out_name("ion_%d_%d.dat", (int)s->T, c);
    f_vin[r] = out_name("vapor_in_%d.dat", c);
    f_vout[r] = out_name("vapor_out_%d.dat", c);
    f_K[r] = out_name("K_%d.dat", c);
    f_U[r] = out_name("U_%d.dat", c);
    const std::string coll = out_name("vapor_collision_%d.dat", c);
    for (const std::string* p : {(const std::string*)&f_ion[r], (const std::string*)&f_vin[r],
                                 (const std::string*)&f_vout[r], (const std::string*)&f_K[r],
                                 (const std::string*)&f_U[r], &coll}) {
      FILE* f = fopen(p->c_str(), "w");
      if (f) fclose(f);
    }
  }
  /* snapshot buffers: every replica's in-domain atoms */
  long long cap = 0;
  for (int r = 0; r < n; r++) {
    const mdn_replica_desc& d = descs[r];
    cap += d.ion.n_atoms + (long long)d.n_gas * d.gas.n_atoms + (long long)d.n_vapor * d.vapor.n_atoms;
  }
  std::vector<long long> off(n + 1);
  std::vector<int> type(cap);
  std::vector<double> x(3 * cap), v(3 * cap), U(8 * n), K(4 * n);
  std::vector<mdn_event> ev(65536);
  double time = 0;          /* vars->time */
  long long phase_base = 0; /* engine steps before the current phase */

  auto ion_centre = [&](int r, double* c, double* cv) {
    const mdnh_system* s = systems[r];
    const int ni = (int)s->ion.type.size();
    double m = 0;
    for (int k = 0; k < 3; k++) c[k] = cv[k] = 0;
    for (int i = 0; i < ni; i++) {
      const long long row = off[r] + i;
      const double mi = s->mass[type[row]];
      m += mi;
      for (int k = 0; k < 3; k++) {
        c[k] += x[3 * row + k] * mi;
        cv[k] += v[3 * row + k] * mi;
      }
    }
    for (int k = 0; k < 3; k++) {
      c[k] /= m;
      cv[k] /= m;
    }
  };
  auto snapshot = [&]() -> int {
    int e = mdn_snapshot(h, off.data(), cap, type.data(), x.data(), v.data(), U.data());
    if (e) return fail(e, "mdn_snapshot: %s", mdn_last_error());
    return MDN_OK;
  };
  auto drain_events = [&]() -> int {
    int cnt = 0;
    int e = mdn_events(h, ev.data(), (int)ev.size(), &cnt);
    if (e) return fail(e, "mdn_events: %s", mdn_last_error());
    for (int i = 0; i < std::min(cnt, (int)ev.size()); i++) {
      const mdn_event& q = ev[i];
      const mdnh_system* s = systems[q.replica];
      const int mol = 1 + s->set.n_gas + q.molecule;
      const double t = (double)(q.step - phase_base) * dt;
      append(q.kind == 1 ? f_vin[q.replica] : f_vout[q.replica], "%d %e %e %e %e %e %e %e\n", mol, t, q.dx[0],
             q.dx[1], q.dx[2], q.dv[0], q.dv[1], q.dv[2]);
    }
    return MDN_OK;
  };
  /* MD::display (src/output/output.cpp:67-100) and MD::export_dump_close */
  auto observe = [&](int relax) -> int {
    int e = snapshot();
    if (e) return e;
    if ((e = mdn_kinetic(h, K.data()))) return fail(e, "mdn_kinetic: %s", mdn_last_error());
    for (int r = 0; r < n; r++) {
      const mdnh_system* s = systems[r];
      const double Kion = K[4 * r], Kg = K[4 * r + 1], Kv = K[4 * r + 2];
      const double coeff = 1.0 / kb_real / 1.5;
      const double Tg = s->set.n_gas ? Kg / s->set.n_gas * coeff : 0, Tv = s->set.n_vapor ? Kv / s->set.n_vapor * coeff : 0;
      const double* u = &U[8 * r];
      append(f_K[r], "%e %e %e %e %e\n", time, Kion, Kg, Kv, Kion + Kg + Kv);
      append(f_U[r], "%e %e %e %e %e %e %e %e %e\n", time, u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7]);
      if (verbose && r == 0) {
        printf("----------------------TIME = %g ps------------------------- (%s)\n", time / 1000.0,
               relax ? "relaxation" : "main run");
        printf("  Kion = %1.2e  Kgas = %1.2e  Kvap = %1.2e\n  Tion = %1.2f  Tgas = %1.2f  Tvap = %1.2f\n", Kion, Kg,
               Kv, K[4 * r + 3], Tg, Tv);
        printf("Uion = %1.2e  Ugas = %1.2e  Uvap = %1.2e\n  Ugi = %1.2e  Ugg = %1.2e  Uvi = %1.2e\n  Uvg = %1.2e  Uvv = %1.2e\n",
               u[0], u[1], u[2], u[3], u[4], u[6], u[5], u[7]);
      }
      double c[3], cv[3];
      ion_centre(r, c, cv);
      const long long rows = off[r + 1] - off[r];
      if (!s->dump_path.empty() &&
          (e = mdnh_write_dump_frame(s, s->dump_path.c_str(), (int)time, (int)rows, &type[off[r]], &x[3 * off[r]],
                                     &v[3 * off[r]], c)))
        return e;
    }
    return MDN_OK;
  };
  auto step = [&](long long k, int energy) -> int {
    int e = mdn_step(h, k, energy);
    if (e && e != MDN_ERR_REPLICA) return fail(e, "mdn_step: %s", mdn_last_error());
    if (e == MDN_ERR_REPLICA && verbose) fprintf(stderr, "mdn_step: %s\n", mdn_last_error());
    return drain_events();
  };

  /* ---- thermal relaxation, src/run.cpp:22-30 ---- */
  for (long long it = 0; it < s0.relax_steps;) {
    if (it % OBSERVE == 0) {
      if ((rc = observe(1))) goto done;
      time = it * dt;
    }
    const long long next = std::min(s0.relax_steps, (it / OBSERVE + 1) * (long long)OBSERVE);
    if ((rc = step(next - it, 0))) goto done;
    it = next;
  }
  /* ---- re-initialisation, src/run.cpp:40-56 ---- */
  time = 0;
  phase_base = s0.relax_steps;
  /* the shift and the make_pair that follows it (src/run.cpp:42-54) */
  if ((rc = mdn_recenter(h, 1)) && rc != MDN_ERR_REPLICA) {
    rc = fail(rc, "mdn_recenter: %s", mdn_last_error());
    goto done;
  }
  if ((rc = drain_events())) goto done;
  if ((rc = mdn_set_nvt(h, -1, MDN_NVT_OFF, 0.0))) { rc = fail(rc, "mdn_set_nvt: %s", mdn_last_error()); goto done; }
  /* ---- main run, src/run.cpp:59-73 ---- */
  for (long long it = 0; it < s0.total_steps;) {
    if (it % logger == 0) {
      if ((rc = snapshot())) goto done;
      for (int r = 0; r < n; r++) {
        double c[3], cv[3];
        ion_centre(r, c, cv);
        append(f_ion[r], "%e %e %e %e %e %e %e\n", time / 1e6, c[0], c[1], c[2], cv[0], cv[1], cv[2]);
      }
      time += logger * dt;
    }
    if (it % OBSERVE == 0 && (rc = observe(0))) goto done;
    long long next = std::min(s0.total_steps, (it / OBSERVE + 1) * (long long)OBSERVE);
    next = std::min(next, (it / logger + 1) * logger);
    /* eflag on the step before each OBSERVE boundary */
    if ((rc = step(next - it, next % OBSERVE == 0 ? 1 : 0))) goto done;
    it = next;
  }
  rc = MDN_OK;
done:
  mdn_destroy(h);
  return rc;
}

}  // extern "C"
