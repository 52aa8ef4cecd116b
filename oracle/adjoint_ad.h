/*
 * adjoint_ad.h -- TEST INFRASTRUCTURE ONLY, included by mdn_oracle.cpp: the
 * FP64 CPU adjoint of the gradient harness's window objective.
 *
 * The engine's mdn_adjoint differentiates the step by hand (analytic
 * transposes of the pair forces, dual numbers for the bonded terms, the
 * adjoint of the converged SHAKE projection).  This file gets the same
 * derivative a different way, as the check of it: the step of the window
 * (kick, drift, SHAKE with the velocity correction, forces, kick, the
 * objective) is written once for a generic scalar, run in plain FP64 for the
 * forward window, then step by step, last first, on a tape of elementary
 * operations (reverse-mode automatic differentiation) whose backward sweep
 * carries the adjoints of (x, v, F) to the previous step and accumulates
 * dJ/dtheta.  SHAKE is differentiated through the iterations it ran.
 *
 * The expressions and their order are those of the Oracle's routines, which
 * tests/test_oracle_pins.py holds bit for bit to the reference's own
 * Potential::compute (the src/potential/ sources), MD::update_position
 * (src/verlet.cpp:73-136) and MD::velocity_calculation (src/verlet.cpp:47-65),
 * so the forward window here equals orc_window's.
 *
 * Scope (that of mdn_adjoint): a window with a fixed molecule set (no
 * effective-domain rebuild), thermostat off, no gas-gas term.  Parameters:
 * (eps, sigma) of every gas-ion and vapor-ion type pair, then a scale s of
 * the ion charges (rows as mdn_adjoint_params).
 */

namespace adj {

/* ---- reverse-mode differentiation ----------------------------------------- */
struct Tape {
  std::vector<int> pa, pb;
  std::vector<double> da, db;
  void clear() {
    pa.clear();
    pb.clear();
    da.clear();
    db.clear();
  }
  int node(int a, double x, int b, double y) {
    pa.push_back(a);
    da.push_back(x);
    pb.push_back(b);
    db.push_back(y);
    return (int)pa.size() - 1;
  }
};

inline Tape& tape() {
  static thread_local Tape t;
  return t;
}

/* a value and its node on the tape (-1: a constant) */
struct D {
  double v;
  int i;
  D(double x = 0.0) : v(x), i(-1) {}
  D(double x, int k) : v(x), i(k) {}
};

inline D leaf(double v) { return D(v, tape().node(-1, 0.0, -1, 0.0)); }

/* a result with the partial derivatives x = d out / d a, y = d out / d b */
inline D mk(double v, int a, double x, int b, double y) {
  if (a < 0 && b < 0) return D(v);
  return D(v, tape().node(a, x, b, y));
}

inline D operator+(const D& a, const D& b) { return mk(a.v + b.v, a.i, 1.0, b.i, 1.0); }
inline D operator-(const D& a, const D& b) { return mk(a.v - b.v, a.i, 1.0, b.i, -1.0); }
inline D operator*(const D& a, const D& b) { return mk(a.v * b.v, a.i, b.v, b.i, a.v); }
inline D operator/(const D& a, const D& b) {
  const double q = a.v / b.v;
  return mk(q, a.i, 1.0 / b.v, b.i, -q / b.v);
}
inline D operator-(const D& a) { return mk(-a.v, a.i, -1.0, -1, 0.0); }
inline D& operator+=(D& a, const D& b) { return a = a + b; }
inline D& operator-=(D& a, const D& b) { return a = a - b; }
inline D& operator*=(D& a, const D& b) { return a = a * b; }
inline D sqrt(const D& a) {
  const double s = std::sqrt(a.v);
  return mk(s, a.i, 0.5 / s, -1, 0.0);
}
inline D exp(const D& a) {
  const double e = std::exp(a.v);
  return mk(e, a.i, e, -1, 0.0);
}
inline D cos(const D& a) { return mk(std::cos(a.v), a.i, -std::sin(a.v), -1, 0.0); }
inline D acos(const D& a) { return mk(std::acos(a.v), a.i, -1.0 / std::sqrt(1.0 - a.v * a.v), -1, 0.0); }

/* backward sweep: adj holds the seeds on entry, every node's adjoint on exit */
inline void backprop(std::vector<double>& adj) {
  Tape& t = tape();
  adj.resize(t.pa.size(), 0.0);
  for (int k = (int)t.pa.size() - 1; k >= 0; k--) {
    const double g = adj[k];
    if (g == 0.0) continue;
    if (t.pa[k] >= 0) adj[t.pa[k]] += t.da[k] * g;
    if (t.pb[k] >= 0) adj[t.pb[k]] += t.db[k] * g;
  }
}

inline double val(double x) { return x; }
inline double val(const D& x) { return x.v; }
using std::sqrt;
using std::exp;
using std::cos;
using std::acos;

/* a value with its partial derivatives by two other values (for the LJ
 * coefficients, whose values stay those of the Oracle's tables) */
inline double with2(double v, double, double, double, double) { return v; }
inline D with2(double v, const D& a, double x, const D& b, double y) { return mk(v, a.i, x, b.i, y); }

template <class S>
using V = std::vector<std::array<S, 3>>;

/* ---- the window's dense system ----------------------------------------------- */
/* ion atoms, then the atoms of the in-domain gas molecules (gas_in order),
 * then those of the in-domain vapor molecules (vap_in order) */
struct Dense {
  int ni = 0, G = 0, Vn = 0, ag = 0, av = 0, n = 0;
  std::vector<int> gk, vk;  /* gas / vapor molecule -> its place, -1 outside */
  std::vector<double> coef; /* 0.5 dt 4.184e-4 / m per dense atom */
  int gas0() const { return ni; }
  int vap0() const { return ni + G * ag; }
};

inline Dense dense_of(const Oracle& o) {
  Dense d;
  d.ni = o.ion.n;
  d.G = (int)o.gas_in.size();
  d.Vn = (int)o.vap_in.size();
  d.ag = o.a_g;
  d.av = o.a_v;
  d.n = d.ni + d.G * d.ag + d.Vn * d.av;
  d.gk.assign(o.n_gas, -1);
  d.vk.assign(o.n_vap, -1);
  for (int k = 0; k < d.G; k++) d.gk[o.gas_in[k]] = k;
  for (int k = 0; k < d.Vn; k++) d.vk[o.vap_in[k]] = k;
  double const Coeff = 0.5 * o.dt * 4.184e-4;
  for (int i = 0; i < d.ni; i++) d.coef.push_back(Coeff / o.ion.mass[i]);
  for (int k = 0; k < d.G; k++)
    for (int a = 0; a < d.ag; a++) d.coef.push_back(Coeff / o.gas.mass[a]);
  for (int k = 0; k < d.Vn; k++)
    for (int a = 0; a < d.av; a++) d.coef.push_back(Coeff / o.vap.mass[a]);
  return d;
}

/* ---- parameters ------------------------------------------------------------- */
template <class S>
struct Par {
  int nt = 0;
  std::vector<S> A, B;
  S s = 1.0;
};

template <class S>
Par<S> make_par(const Oracle& o, const std::vector<S>& th, const int* rows, int nrows) {
  Par<S> p;
  p.nt = o.nt;
  for (double a : o.ljA) p.A.push_back(S(a));
  for (double b : o.ljB) p.B.push_back(S(b));
  for (int k = 0; k < nrows - 1; k++) {
    const int a = rows[3 * k + 1], b = rows[3 * k + 2];
    const S& eps = th[2 * k];
    const S& sig = th[2 * k + 1];
    /* A = 48 eps sigma^12, B = 24 eps sigma^6 (setCrossPotential.cpp:15-19) */
    const double Av = o.A(a, b), Bv = o.B(a, b);
    const S A = with2(Av, eps, Av / val(eps), sig, 12.0 * Av / val(sig));
    const S B = with2(Bv, eps, Bv / val(eps), sig, 6.0 * Bv / val(sig));
    p.A[(size_t)a * o.nt + b] = A;
    p.A[(size_t)b * o.nt + a] = A;
    p.B[(size_t)a * o.nt + b] = B;
    p.B[(size_t)b * o.nt + a] = B;
  }
  p.s = th[2 * (nrows - 1)];
  return p;
}

/* ---- the Oracle's force routines for a generic scalar ----------------------- */
template <class S>
struct Terms {
  const Oracle& o;
  const Dense& d;
  const Par<S>& p;
  S A(int ti, int tj) const { return p.A[(size_t)ti * p.nt + tj]; }
  S B(int ti, int tj) const { return p.B[(size_t)ti * p.nt + tj]; }
  S qion(int i) const { return p.s * o.ion.q[i]; }

  void lj_pair(std::array<S, 3>& fi, std::array<S, 3>& fj, const std::array<S, 3>& xi, const std::array<S, 3>& xj,
               int ti, int tj, const S& wij, bool coul, const S& qi, const S& qj, bool weighted) const {
    S dx = xi[0] - xj[0];
    S dy = xi[1] - xj[1];
    S dz = xi[2] - xj[2];
    S rsq = (dx * dx + dy * dy + dz * dz);
    S r2inv = 1 / rsq;
    S r6inv = r2inv * r2inv * r2inv;
    S force_pair;
    if (!coul && !weighted) {
      force_pair = r6inv * (A(ti, tj) * r6inv - B(ti, tj)) * r2inv;
    } else {
      S force_lj = r6inv * (A(ti, tj) * r6inv - B(ti, tj));
      S force_coul = coul ? qqrd2e * qi * qj * sqrt(r2inv) : S(0.0);
      force_pair = coul ? (force_lj + force_coul) * r2inv : (force_lj) * r2inv;
      if (weighted) force_pair = force_pair * wij;
    }
    fi[0] += force_pair * dx;
    fi[1] += force_pair * dy;
    fi[2] += force_pair * dz;
    fj[0] -= force_pair * dx;
    fj[1] -= force_pair * dy;
    fj[2] -= force_pair * dz;
  }

  void bond_term(const std::array<S, 3>* x, std::array<S, 3>* f, int i, int j, int type) const {
    S dx = x[i][0] - x[j][0];
    S dy = x[i][1] - x[j][1];
    S dz = x[i][2] - x[j][2];
    S rsq = (dx * dx + dy * dy + dz * dz);
    S r = sqrt(rsq);
    S dr = (r - o.bond_c[type][1]);
    S rk = o.bond_c[type][0] * dr;
    S fb = -2.0 * rk / r;
    f[i][0] += fb * dx;
    f[i][1] += fb * dy;
    f[i][2] += fb * dz;
    f[j][0] -= fb * dx;
    f[j][1] -= fb * dy;
    f[j][2] -= fb * dz;
  }

  void angle_term(const std::array<S, 3>* x, std::array<S, 3>* f, int i, int j, int k, int type) const {
    S f1[3], f3[3];
    S dx1 = x[i][0] - x[j][0];
    S dy1 = x[i][1] - x[j][1];
    S dz1 = x[i][2] - x[j][2];
    S rsq1 = (dx1 * dx1 + dy1 * dy1 + dz1 * dz1);
    S r1 = sqrt(rsq1);
    S dx2 = x[k][0] - x[j][0];
    S dy2 = x[k][1] - x[j][1];
    S dz2 = x[k][2] - x[j][2];
    S rsq2 = (dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
    S r2 = sqrt(rsq2);
    S C = dx1 * dx2 + dy1 * dy2 + dz1 * dz2;
    C = C / (r1 * r2);
    S Cs = 1 / (sqrt(1.0 - C * C));
    S dtheta = acos(C) - o.angle_c[type][1];
    S tk = o.angle_c[type][0] * dtheta;
    S a = -2.0 * tk * Cs;
    S a11 = a * C / rsq1;
    S a12 = -a / (r1 * r2);
    S a22 = a * C / rsq2;
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
  }

  void dihedral_term(const std::array<S, 3>* x, std::array<S, 3>* f, int i, int j, int k, int l, int type) const {
    S vb1x = x[i][0] - x[j][0];
    S vb1y = x[i][1] - x[j][1];
    S vb1z = x[i][2] - x[j][2];
    S vb2x = x[k][0] - x[j][0];
    S vb2y = x[k][1] - x[j][1];
    S vb2z = x[k][2] - x[j][2];
    S vb2xm = -vb2x;
    S vb2ym = -vb2y;
    S vb2zm = -vb2z;
    S vb3x = x[l][0] - x[k][0];
    S vb3y = x[l][1] - x[k][1];
    S vb3z = x[l][2] - x[k][2];
    S ax = vb1y * vb2zm - vb1z * vb2ym;
    S ay = vb1z * vb2xm - vb1x * vb2zm;
    S az = vb1x * vb2ym - vb1y * vb2xm;
    S bx = vb3y * vb2zm - vb3z * vb2ym;
    S by = vb3z * vb2xm - vb3x * vb2zm;
    S bz = vb3x * vb2ym - vb3y * vb2xm;
    S rasq = ax * ax + ay * ay + az * az;
    S rbsq = bx * bx + by * by + bz * bz;
    S rgsq = vb2xm * vb2xm + vb2ym * vb2ym + vb2zm * vb2zm;
    S rg = sqrt(rgsq);
    S rginv = 0.0, ra2inv = 0.0, rb2inv = 0.0;
    if (val(rg) > 0) rginv = 1.0 / rg;
    if (val(rasq) > 0) ra2inv = 1.0 / rasq;
    if (val(rbsq) > 0) rb2inv = 1.0 / rbsq;
    S rabinv = sqrt(ra2inv * rb2inv);
    S c = (ax * bx + ay * by + az * bz) * rabinv;
    S s = rg * rabinv * (ax * vb3x + ay * vb3y + az * vb3z);
    S df = 0.0;
    const double* co = o.dih_c[type].data();
    for (int JJ = 0; JJ < o.dih_multi[type]; JJ++) {
      int JJ5 = JJ * 5;
      S p_ = 1.0, df1 = 0.0, ddf1 = 0.0;
      for (int loop = 0; loop < co[JJ5 + 1]; loop++) {
        ddf1 = p_ * c - df1 * s;
        df1 = p_ * s + df1 * c;
        p_ = ddf1;
      }
      p_ = p_ * co[JJ5 + 3] + df1 * co[JJ5 + 4];
      df1 = df1 * co[JJ5 + 3] - ddf1 * co[JJ5 + 4];
      df1 = df1 * -co[JJ5 + 1];
      p_ += 1.0;
      if (co[1] == 0) {
        p_ = 1.0 + co[JJ5 + 3];
        df1 = 0.0;
      }
      df += (-co[JJ5] * df1);
    }
    S fg = vb1x * vb2xm + vb1y * vb2ym + vb1z * vb2zm;
    S hg = vb3x * vb2xm + vb3y * vb2ym + vb3z * vb2zm;
    S fga = fg * ra2inv * rginv;
    S hgb = hg * rb2inv * rginv;
    S gaa = -ra2inv * rg;
    S gbb = rb2inv * rg;
    S dtfx = gaa * ax, dtfy = gaa * ay, dtfz = gaa * az;
    S dtgx = fga * ax - hgb * bx, dtgy = fga * ay - hgb * by, dtgz = fga * az - hgb * bz;
    S dthx = gbb * bx, dthy = gbb * by, dthz = gbb * bz;
    S sx2 = df * dtgx, sy2 = df * dtgy, sz2 = df * dtgz;
    S ff1[3] = {df * dtfx, df * dtfy, df * dtfz};
    S ff2[3] = {sx2 - ff1[0], sy2 - ff1[1], sz2 - ff1[2]};
    S ff4[3] = {df * dthx, df * dthy, df * dthz};
    S ff3[3] = {-sx2 - ff4[0], -sy2 - ff4[1], -sz2 - ff4[2]};
    for (int q = 0; q < 3; q++) {
      f[i][q] += ff1[q];
      f[j][q] += ff2[q];
      f[k][q] += ff3[q];
      f[l][q] += ff4[q];
    }
  }

  /* Oracle::forces on the dense system; vw = taper weights of the vapor atoms */
  void forces(const V<S>& x, V<S>& f, const std::vector<S>& vw) const {
    const int ni = d.ni, ag = d.ag, av = d.av, g0 = d.gas0(), v0 = d.vap0();
    for (auto& q : f) q = {S(0.0), S(0.0), S(0.0)};
    if (o.on(MDN_I_GI))
      for (auto& pr : o.gi_list) {
        const int m = d.gk[pr[0]], j = pr[1];
        for (int a = 0; a < ag; a++)
          lj_pair(f[g0 + m * ag + a], f[j], x[g0 + m * ag + a], x[j], o.gas.type[a], o.ion.type[j], S(1.0), false,
                  S(0.0), S(0.0), false);
      }
    if (o.on(MDN_I_VI))
      for (int q = 0; q < d.Vn; q++)
        for (int a = 0; a < av; a++)
          for (int j = 0; j < ni; j++) {
            const int oa = v0 + q * av + a;
            lj_pair(f[oa], f[j], x[oa], x[j], o.vap.type[a], o.ion.type[j], vw[q * av + a] * 1.0, true,
                    S(o.vap.q[a]), qion(j), true);
          }
    if (o.on(MDN_I_GV)) {
      const int nj = (o.quirks & MDN_Q_GV_GAS_COUNT) ? std::min(ag, av) : av;
      for (auto& pr : o.gv_list) {
        const int m = d.gk[pr[0]], q = d.vk[pr[1]];
        for (int a = 0; a < ag; a++)
          for (int b = 0; b < nj; b++)
            lj_pair(f[g0 + m * ag + a], f[v0 + q * av + b], x[g0 + m * ag + a], x[v0 + q * av + b], o.gas.type[a],
                    o.vap.type[b], S(1.0), false, S(0.0), S(0.0), false);
      }
    }
    if (o.on(MDN_I_VV))
      for (int i1 = 0; i1 + 1 < d.Vn; i1++)
        for (int i2 = i1 + 1; i2 < d.Vn; i2++)
          for (int a = 0; a < av; a++)
            for (int b = 0; b < av; b++) {
              const int oi = v0 + i1 * av + a, oj = v0 + i2 * av + b;
              lj_pair(f[oi], f[oj], x[oi], x[oj], o.vap.type[a], o.vap.type[b], vw[i1 * av + a] * vw[i2 * av + b],
                      true, S(o.vap.q[a]), S(o.vap.q[b]), true);
            }
    if (o.on(MDN_I_EFIELD))
      for (int i = 0; i < ni; i++) {
        S coeff = 5.55e-5 * qion(i);
        f[i][0] += coeff * o.Ef[0];
        f[i][1] += coeff * o.Ef[1];
        f[i][2] += coeff * o.Ef[2];
      }
    if (o.on(MDN_I_AMBER)) {
      for (int i = 0; i < ni - 1; i++)
        for (int j = i + 1; j < ni; j++)
          if (!o.excl[(size_t)i * ni + j])
            lj_pair(f[i], f[j], x[i], x[j], o.ion.type[i], o.ion.type[j], S(1.0), true, qion(i), qion(j), false);
      for (auto& b : o.ion.bonds) bond_term(x.data(), f.data(), b[0], b[1], b[2]);
      for (auto& a : o.ion.angles) angle_term(x.data(), f.data(), a[0], a[1], a[2], a[3]);
      for (auto& dd : o.ion.dih) dihedral_term(x.data(), f.data(), dd[0], dd[1], dd[2], dd[3], dd[4]);
    }
    if (o.on(MDN_I_BMH))
      for (int i = 0; i < ni - 1; i++)
        for (int j = i + 1; j < ni; j++) {
          const double* c = born.c[o.bmh[i]][o.bmh[j]];
          S dx = x[i][0] - x[j][0];
          S dy = x[i][1] - x[j][1];
          S dz = x[i][2] - x[j][2];
          S rsq = (dx * dx + dy * dy + dz * dz);
          S r2inv = 1 / rsq;
          S r6inv = r2inv * r2inv * r2inv;
          S r = sqrt(rsq);
          S rexp = exp(c[4] * (c[3] - r));
          S force1 = c[4] * c[0] * r * rexp;
          S force2 = -c[1] * r6inv;
          S force3 = -c[2] * r6inv * r2inv;
          S force_coul = qqrd2e * qion(i) * qion(j) * sqrt(r2inv);
          S force_pair = (force1 + force2 + force3 + force_coul) * r2inv;
          f[i][0] += force_pair * dx;
          f[i][1] += force_pair * dy;
          f[i][2] += force_pair * dz;
          f[j][0] -= force_pair * dx;
          f[j][1] -= force_pair * dy;
          f[j][2] -= force_pair * dz;
        }
    if (o.on(MDN_I_VAPOR_INTRA))
      for (int q = 0; q < d.Vn; q++) {
        const std::array<S, 3>* xm = x.data() + v0 + q * av;
        std::array<S, 3>* fm = f.data() + v0 + q * av;
        for (auto& b : o.vap.bonds) bond_term(xm, fm, b[0], b[1], b[2]);
        for (auto& a : o.vap.angles) angle_term(xm, fm, a[0], a[1], a[2], a[3]);
        for (auto& dd : o.vap.dih) dihedral_term(xm, fm, dd[0], dd[1], dd[2], dd[3], dd[4]);
      }
    if (o.on(MDN_I_GAS_INTRA))
      for (int m = 0; m < d.G; m++)
        for (auto& b : o.gas.bonds) bond_term(x.data() + g0 + m * ag, f.data() + g0 + m * ag, b[0], b[1], b[2]);
  }

  /* the ion centre as MD::update_position forms it (src/verlet.cpp:90-107) */
  std::array<S, 3> ion_centre(const V<S>& x) const {
    std::array<S, 3> c = {S(0.0), S(0.0), S(0.0)};
    for (int ii = 0; ii < d.ni; ii++)
      for (int k = 0; k < 3; k++) c[k] += x[ii][k] * o.ion.mass[ii];
    double mInv = 1 / o.ion.msum;
    for (int k = 0; k < 3; k++) c[k] = c[k] * mInv;
    return c;
  }

  /* Oracle::weight_of (src/verlet.cpp:109-134) */
  S weight_of(const std::array<S, 3>& xa, const std::array<S, 3>& x0) const {
    S dx = xa[0] - x0[0];
    S dy = xa[1] - x0[1];
    S dz = xa[2] - x0[2];
    S r2 = dx * dx + dy * dy + dz * dz;
    if (val(r2) < o.Ri2) return S(1.0);
    if (val(r2) > o.RI2) return S(0.0);
    S dr = (sqrt(r2) - o.Rcenter);
    S C = cos(M_PI / o.Overlap * 0.5 * dr);
    return C * C;
  }

  /* Oracle::objective */
  S objective(const V<S>& x, double R0, double W, double we, double wc) const {
    const int av = d.av, v0 = d.vap0();
    S U = 0.0;
    for (int q = 0; q < d.Vn; q++)
      for (int a = 0; a < av; a++) {
        const std::array<S, 3>& xa = x[v0 + q * av + a];
        for (int j = 0; j < d.ni; j++) {
          S dx = xa[0] - x[j][0], dy = xa[1] - x[j][1], dz = xa[2] - x[j][2];
          S r2 = dx * dx + dy * dy + dz * dz;
          S r2inv = 1 / r2;
          S r6inv = r2inv * r2inv * r2inv;
          int ta = o.vap.type[a], tj = o.ion.type[j];
          U += r6inv * (A(ta, tj) / 12.0 * r6inv - B(ta, tj) / 6.0) + qqrd2e * o.vap.q[a] * qion(j) * sqrt(r2inv);
        }
      }
    std::array<S, 3> c = {S(0.0), S(0.0), S(0.0)};
    for (int j = 0; j < d.ni; j++)
      for (int k = 0; k < 3; k++) c[k] += x[j][k] * o.ion.mass[j];
    for (int k = 0; k < 3; k++) c[k] = c[k] / o.ion.msum;
    S Sm = 0.0;
    for (int q = 0; q < d.Vn; q++) {
      std::array<S, 3> cm = {S(0.0), S(0.0), S(0.0)};
      for (int a = 0; a < av; a++)
        for (int k = 0; k < 3; k++) cm[k] += x[v0 + q * av + a][k] * o.vap.mass[a];
      S d2 = 0.0;
      for (int k = 0; k < 3; k++) {
        S dk = cm[k] / o.vap.msum - c[k];
        d2 += dk * dk;
      }
      Sm += 1.0 / (1.0 + exp((sqrt(d2) - R0) / W));
    }
    return we * U + wc * Sm;
  }

  /* Oracle::shake_mol on one molecule (x: drifted positions, r: before the
   * drift), with the velocity correction */
  void shake_mol(const Top& t, std::array<S, 3>* x, std::array<S, 3>* v, const std::array<S, 3>* r,
                 int* status) const {
    if (t.rigid.empty()) return;
    std::vector<std::array<S, 3>> x0(x, x + t.n);
    auto resid = [&](size_t k) {
      int i = t.rigid[k][0], j = t.rigid[k][1];
      double dk = o.bond_c[t.rigid[k][2]][1];
      double sx = val(x[i][0]) - val(x[j][0]), sy = val(x[i][1]) - val(x[j][1]), sz = val(x[i][2]) - val(x[j][2]);
      double dr = sx * sx + sy * sy + sz * sz - dk * dk;
      return dr * dr;
    };
    bool converge = false;
    for (int sweep = 0; sweep < 1000 && !converge; sweep++) {
      for (int c = 0; c < t.n_colors; c++)
        for (size_t k = 0; k < t.rigid.size(); k++) {
          if (t.rigid_color[k] != c) continue;
          int i = t.rigid[k][0], j = t.rigid[k][1];
          double dk = o.bond_c[t.rigid[k][2]][1];
          S rx = r[i][0] - r[j][0], ry = r[i][1] - r[j][1], rz = r[i][2] - r[j][2];
          S sx = x[i][0] - x[j][0], sy = x[i][1] - x[j][1], sz = x[i][2] - x[j][2];
          S s2 = sx * sx + sy * sy + sz * sz;
          S dot = rx * sx + ry * sy + rz * sz;
          double minv = 1 / t.mass[i] + 1 / t.mass[j];
          if (val(dot) < 1e-10) dot = S(1e-10);
          S g = (dk * dk - s2) / (2 * minv * dot);
          S ci = g / t.mass[i], cj = g / t.mass[j];
          x[i][0] += rx * ci; x[i][1] += ry * ci; x[i][2] += rz * ci;
          x[j][0] -= rx * cj; x[j][1] -= ry * cj; x[j][2] -= rz * cj;
        }
      converge = true;
      for (size_t k = 0; k < t.rigid.size(); k++)
        if (!(resid(k) <= 1e-20)) converge = false;
    }
    if (!converge) *status |= MDN_ST_SHAKE_NOCONV;
    if (!(o.quirks & MDN_Q_SHAKE_NO_VCORR))
      for (int a = 0; a < t.n; a++)
        for (int k = 0; k < 3; k++) v[a][k] += (x[a][k] - x0[a][k]) / o.dt;
  }

  /* one MD::verlet of the window (thermostat off, no rebuild): returns the
   * objective at the new positions */
  S step(const V<S>& x, const V<S>& v, const V<S>& f, V<S>& x1, V<S>& v1, V<S>& f1, double R0, double W,
         double we, double wc, int* status) const {
    const int n = d.n;
    V<S> va(n), r(n);
    for (int a = 0; a < n; a++)
      for (int k = 0; k < 3; k++) va[a][k] = v[a][k] + f[a][k] * d.coef[a];
    x1.assign(n, {S(0.0), S(0.0), S(0.0)});
    for (int a = 0; a < n; a++)
      for (int k = 0; k < 3; k++) {
        r[a][k] = x[a][k];
        x1[a][k] = x[a][k] + va[a][k] * o.dt;
      }
    if (o.I & MDN_I_SHAKE) {
      shake_mol(o.ion, x1.data(), va.data(), r.data(), status);
      for (int m = 0; m < d.G; m++) {
        const int b = d.gas0() + m * d.ag;
        shake_mol(o.gas, x1.data() + b, va.data() + b, r.data() + b, status);
      }
      for (int q = 0; q < d.Vn; q++) {
        const int b = d.vap0() + q * d.av;
        shake_mol(o.vap, x1.data() + b, va.data() + b, r.data() + b, status);
      }
    }
    const std::array<S, 3> c = ion_centre(x1);
    std::vector<S> vw((size_t)d.Vn * d.av);
    for (int q = 0; q < d.Vn; q++)
      for (int a = 0; a < d.av; a++) vw[q * d.av + a] = weight_of(x1[d.vap0() + q * d.av + a], c);
    f1.assign(n, {S(0.0), S(0.0), S(0.0)});
    forces(x1, f1, vw);
    v1.assign(n, {S(0.0), S(0.0), S(0.0)});
    for (int a = 0; a < n; a++)
      for (int k = 0; k < 3; k++) v1[a][k] = va[a][k] + f1[a][k] * d.coef[a];
    return objective(x1, R0, W, we, wc);
  }

  /* the forces at x with the weights of x (a force evaluation at the start) */
  void forces_at(const V<S>& x, V<S>& f) const {
    const std::array<S, 3> c = ion_centre(x);
    std::vector<S> vw((size_t)d.Vn * d.av);
    for (int q = 0; q < d.Vn; q++)
      for (int a = 0; a < d.av; a++) vw[q * d.av + a] = weight_of(x[d.vap0() + q * d.av + a], c);
    f.assign(d.n, {S(0.0), S(0.0), S(0.0)});
    forces(x, f, vw);
  }
};

/* the dense state of the Oracle */
inline void dense_state(const Oracle& o, const Dense& d, V<double>& x, V<double>& v, V<double>& f) {
  x.clear();
  v.clear();
  f.clear();
  for (int i = 0; i < d.ni; i++) {
    x.push_back(o.ion_x[i]);
    v.push_back(o.ion_v[i]);
    f.push_back(o.ion_f[i]);
  }
  for (int m : o.gas_in)
    for (int a = 0; a < d.ag; a++) {
      x.push_back(o.gx[(size_t)m * d.ag + a]);
      v.push_back(o.gv[(size_t)m * d.ag + a]);
      f.push_back(o.gf[(size_t)m * d.ag + a]);
    }
  for (int m : o.vap_in)
    for (int a = 0; a < d.av; a++) {
      x.push_back(o.vx[(size_t)m * d.av + a]);
      v.push_back(o.vv[(size_t)m * d.av + a]);
      f.push_back(o.vf[(size_t)m * d.av + a]);
    }
}

inline V<D> leaves(const V<double>& a) {
  V<D> out(a.size());
  for (size_t i = 0; i < a.size(); i++)
    for (int k = 0; k < 3; k++) out[i][k] = leaf(a[i][k]);
  return out;
}

/* J over n steps from the Oracle's state and dJ/dtheta; returns 0, or -1
 * when the window would cross a rebuild, a thermostat is on or gg is on,
 * -2 when SHAKE did not converge.  The Oracle is not advanced. */
inline int window_adjoint(const Oracle& o, long long n, double R0, double W, double we, double wc,
                          const double* theta, const int* rows, int nrows, double* J, double* grad) {
  if (n <= 0 || o.loop_pair + n > o.loop_update || o.nvt_mode != MDN_NVT_OFF || (o.I & MDN_I_GG)) return -1;
  const Dense d = dense_of(o);
  const int np = 2 * (nrows - 1) + 1;
  std::vector<double> th(theta, theta + np);
  const Par<double> pd = make_par<double>(o, th, rows, nrows);
  const Terms<double> td{o, d, pd};
  int status = 0;
  /* forward window, every step's state kept */
  std::vector<V<double>> X(n + 1), Vv(n + 1), F(n + 1);
  dense_state(o, d, X[0], Vv[0], F[0]);
  double js = 0;
  for (long long t = 0; t < n; t++) js += td.step(X[t], Vv[t], F[t], X[t + 1], Vv[t + 1], F[t + 1], R0, W, we, wc, &status);
  *J = js / (double)n;
  if (status & MDN_ST_SHAKE_NOCONV) return -2;
  /* backward, one step at a time, last first */
  const int N = d.n;
  V<double> lx(N, {0, 0, 0}), lv(N, {0, 0, 0}), lf(N, {0, 0, 0});
  std::vector<double> g(np, 0.0), adjv;
  for (long long t = n - 1; t >= 0; t--) {
    tape().clear();
    V<D> x = leaves(X[t]), v = leaves(Vv[t]), f = leaves(F[t]);
    std::vector<D> thd(np);
    for (int k = 0; k < np; k++) thd[k] = leaf(th[k]);
    const Par<D> p = make_par<D>(o, thd, rows, nrows);
    const Terms<D> tdd{o, d, p};
    V<D> x1, v1, f1;
    int st = 0;
    D jt = tdd.step(x, v, f, x1, v1, f1, R0, W, we, wc, &st);
    adjv.assign(tape().pa.size(), 0.0);
    auto seed = [&](const D& q, double s) {
      if (q.i >= 0) adjv[q.i] += s;
    };
    for (int a = 0; a < N; a++)
      for (int k = 0; k < 3; k++) {
        seed(x1[a][k], lx[a][k]);
        seed(v1[a][k], lv[a][k]);
        seed(f1[a][k], lf[a][k]);
      }
    seed(jt, 1.0 / (double)n);
    backprop(adjv);
    for (int a = 0; a < N; a++)
      for (int k = 0; k < 3; k++) {
        lx[a][k] = x[a][k].i >= 0 ? adjv[x[a][k].i] : 0.0;
        lv[a][k] = v[a][k].i >= 0 ? adjv[v[a][k].i] : 0.0;
        lf[a][k] = f[a][k].i >= 0 ? adjv[f[a][k].i] : 0.0;
      }
    for (int k = 0; k < np; k++) g[k] += adjv[thd[k].i];
  }
  /* the start forces: F(x_0; theta) once the replica has been stepped
   * (a replica never stepped holds zero forces, which no parameter moves) */
  if (o.step > 0) {
    tape().clear();
    V<D> x = leaves(X[0]);
    std::vector<D> thd(np);
    for (int k = 0; k < np; k++) thd[k] = leaf(th[k]);
    const Par<D> p = make_par<D>(o, thd, rows, nrows);
    const Terms<D> tdd{o, d, p};
    V<D> f0;
    tdd.forces_at(x, f0);
    adjv.assign(tape().pa.size(), 0.0);
    for (int a = 0; a < N; a++)
      for (int k = 0; k < 3; k++)
        if (f0[a][k].i >= 0) adjv[f0[a][k].i] += lf[a][k];
    backprop(adjv);
    for (int k = 0; k < np; k++) g[k] += adjv[thd[k].i];
  }
  tape().clear();
  for (int k = 0; k < np; k++) grad[k] = g[k];
  return 0;
}

}  // namespace adj
