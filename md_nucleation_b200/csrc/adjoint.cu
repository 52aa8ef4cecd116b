/*
 * adjoint.cu -- the gradient harness (no counterpart in the reference):
 * dJ/dtheta of an ion-vapor objective over a window of MD steps of one
 * replica, by the discrete adjoint of the engine's velocity Verlet step.
 *
 * Forward: the engine advances the window (FP32 pair terms, FP64
 * integration) and the replica's in-domain atoms are gathered every K steps
 * (checkpoints).  Backward: one CTA per segment, last segment first,
 * recomputes the segment in FP64 from its checkpoint, keeping x_t, v_t, F_t
 * and the SHAKE multipliers of each step, then runs the adjoint of
 *   (1) v_a = v + c F          (2) y = x + dt v_a          (3) x' = SHAKE(y; x)
 *   (4) v_b = v_a + (x' - y)/dt (5) F' = F(x'; theta)      (6) v' = v_b + c F'
 * (MD::verlet, src/verlet.cpp:20-39, with the SHAKE step of src/shake.cpp:6-92
 * and the velocity correction the engine applies) backwards through it:
 *   - (5): the transposed force Jacobian applied to the force adjoint:
 *     analytic for the pair terms (LJ, LJ + Coulomb, Born-Mayer-Huggins), the
 *     taper weights w(|x - c_ion|) of the vapor atoms included with their
 *     dependence on the ion centre; forward-mode (dual number) products for
 *     the bonded terms, whose force Jacobians are symmetric (F = -grad U);
 *   - (3): the adjoint of the converged projection x' = y + sum_k g_k D_k r_k
 *     (r_k the constraint vector at the step's start): G^T mu = rho solved by
 *     colour-ordered Gauss-Seidel sweeps, lambda_y = lambda - sum_k mu_k B_k^T,
 *     plus the g_k D_k dr_k terms into the previous positions.
 * Parameter derivatives accumulate in FP64 in shared memory; atomics make
 * sums independent of the launch shape up to FP64 rounding order.
 */
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <set>
#include <vector>

#include "mdn.h"
#include "mdn_types.h"

__attribute__((visibility("hidden"))) int mdn_error(int code, const char* msg);
__attribute__((visibility("hidden"))) unsigned mdn_internal_quirks(const mdn_handle* h);
int mdn_snapshot_device(const RepParams* dP, const RepDyn* dD, const int* d_iblob, int R, const double* ion_x,
                        const double* ion_v, const double* slab_x, const double* slab_v, const double* vslab_x,
                        const double* vslab_v, long long* d_offset, int* d_type, double* d_x, double* d_v,
                        long long d_capacity, cudaStream_t stream);
__attribute__((visibility("hidden"))) void mdn_snapshot_args(const mdn_handle* h, SnapshotArgs* s);

namespace {

constexpr int ADJ_THREADS = 512;
constexpr int ADJ_CLUSTER = 8; /* CTAs of a reverse sweep (16 measured no faster) */
constexpr int MAX_PARAMS = 512;
constexpr int SHAKE_SWEEPS = 1000;

enum PairKind : unsigned char { PK_GI = 0, PK_GV, PK_VI, PK_VV, PK_ION_LJC, PK_ION_BMH };

/* ------------------------------------------------------------------------- */
/* dual numbers: value and one tangent                                         */
/* ------------------------------------------------------------------------- */
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual mk(double v, double d = 0.0) { return {v, d}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)};
}
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator/(double a, Dual b) { return {a / b.v, -a * b.d / (b.v * b.v)}; }
__device__ __forceinline__ Dual dsqrt(Dual a) {
  double s = sqrt(a.v);
  return {s, a.d / (2.0 * s)};
}
__device__ __forceinline__ Dual dacos(Dual a) { return {acos(a.v), -a.d / sqrt(1.0 - a.v * a.v)}; }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double dacos(double a) { return acos(a); }
__device__ __forceinline__ bool gt0(Dual a) { return a.v > 0; }
__device__ __forceinline__ bool gt0(double a) { return a > 0; }

/* bonded forces, the engine's / reference's expressions
 * (src/potential/compute_AMBER.cpp:52-253), on atoms in fixed slots */
template <class T>
__device__ void bond_t(const T (*X)[3], const double* co, T (*f)[3]) {
  T dx = X[0][0] - X[1][0], dy = X[0][1] - X[1][1], dz = X[0][2] - X[1][2];
  T rsq = dx * dx + dy * dy + dz * dz;
  T r = dsqrt(rsq);
  T dr = r - T{co[1]};
  T rk = co[0] * dr;
  T fb = -2.0 * rk / r;
  f[0][0] = fb * dx; f[0][1] = fb * dy; f[0][2] = fb * dz;
  f[1][0] = -(fb * dx); f[1][1] = -(fb * dy); f[1][2] = -(fb * dz);
}

template <class T>
__device__ void angle_t(const T (*X)[3], const double* co, T (*f)[3]) {
  T dx1 = X[0][0] - X[1][0], dy1 = X[0][1] - X[1][1], dz1 = X[0][2] - X[1][2];
  T rsq1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1;
  T r1 = dsqrt(rsq1);
  T dx2 = X[2][0] - X[1][0], dy2 = X[2][1] - X[1][1], dz2 = X[2][2] - X[1][2];
  T rsq2 = dx2 * dx2 + dy2 * dy2 + dz2 * dz2;
  T r2 = dsqrt(rsq2);
  T C = dx1 * dx2 + dy1 * dy2 + dz1 * dz2;
  C = C / (r1 * r2);
  T Cs = 1.0 / dsqrt(1.0 - C * C);
  T dtheta = dacos(C) - T{co[1]};
  T tk = co[0] * dtheta;
  T a = -2.0 * tk * Cs;
  T a11 = a * C / rsq1;
  T a12 = -a / (r1 * r2);
  T a22 = a * C / rsq2;
  T f1[3] = {a11 * dx1 + a12 * dx2, a11 * dy1 + a12 * dy2, a11 * dz1 + a12 * dz2};
  T f3[3] = {a22 * dx2 + a12 * dx1, a22 * dy2 + a12 * dy1, a22 * dz2 + a12 * dz1};
  for (int q = 0; q < 3; q++) {
    f[0][q] = f1[q];
    f[1][q] = -(f1[q] + f3[q]);
    f[2][q] = f3[q];
  }
}

template <class T>
__device__ void dihedral_t(const T (*X)[3], const double* co, int multi, T (*f)[3]) {
  T vb1x = X[0][0] - X[1][0], vb1y = X[0][1] - X[1][1], vb1z = X[0][2] - X[1][2];
  T vb2x = X[2][0] - X[1][0], vb2y = X[2][1] - X[1][1], vb2z = X[2][2] - X[1][2];
  T vb2xm = -vb2x, vb2ym = -vb2y, vb2zm = -vb2z;
  T vb3x = X[3][0] - X[2][0], vb3y = X[3][1] - X[2][1], vb3z = X[3][2] - X[2][2];
  T ax = vb1y * vb2zm - vb1z * vb2ym;
  T ay = vb1z * vb2xm - vb1x * vb2zm;
  T az = vb1x * vb2ym - vb1y * vb2xm;
  T bx = vb3y * vb2zm - vb3z * vb2ym;
  T by = vb3z * vb2xm - vb3x * vb2zm;
  T bz = vb3x * vb2ym - vb3y * vb2xm;
  T rasq = ax * ax + ay * ay + az * az;
  T rbsq = bx * bx + by * by + bz * bz;
  T rgsq = vb2xm * vb2xm + vb2ym * vb2ym + vb2zm * vb2zm;
  T rg = dsqrt(rgsq);
  T rginv{0.0}, ra2inv{0.0}, rb2inv{0.0};
  if (gt0(rg)) rginv = 1.0 / rg;
  if (gt0(rasq)) ra2inv = 1.0 / rasq;
  if (gt0(rbsq)) rb2inv = 1.0 / rbsq;
  T rabinv = dsqrt(ra2inv * rb2inv);
  T c = (ax * bx + ay * by + az * bz) * rabinv;
  T s = rg * rabinv * (ax * vb3x + ay * vb3y + az * vb3z);
  T df{0.0};
  for (int JJ = 0; JJ < multi; JJ++) {
    const int J5 = JJ * 5;
    T p_{1.0}, df1{0.0}, ddf1{0.0};
    for (int loop = 0; loop < co[J5 + 1]; loop++) {
      ddf1 = p_ * c - df1 * s;
      df1 = p_ * s + df1 * c;
      p_ = ddf1;
    }
    p_ = p_ * co[J5 + 3] + df1 * co[J5 + 4];
    df1 = df1 * co[J5 + 3] - ddf1 * co[J5 + 4];
    df1 = df1 * (-co[J5 + 1]);
    if (co[1] == 0) df1 = T{0.0}; /* term 0's periodicity tested for every term (compute_AMBER.cpp:199) */
    df = df + (-co[J5]) * df1;
  }
  T fg = vb1x * vb2xm + vb1y * vb2ym + vb1z * vb2zm;
  T hg = vb3x * vb2xm + vb3y * vb2ym + vb3z * vb2zm;
  T fga = fg * ra2inv * rginv;
  T hgb = hg * rb2inv * rginv;
  T gaa = -ra2inv * rg;
  T gbb = rb2inv * rg;
  T dtf[3] = {gaa * ax, gaa * ay, gaa * az};
  T dtg[3] = {fga * ax - hgb * bx, fga * ay - hgb * by, fga * az - hgb * bz};
  T dth[3] = {gbb * bx, gbb * by, gbb * bz};
  for (int q = 0; q < 3; q++) {
    T s2 = df * dtg[q];
    T f1 = df * dtf[q];
    T f4 = df * dth[q];
    f[0][q] = f1;
    f[1][q] = s2 - f1;
    f[2][q] = -s2 - f4;
    f[3][q] = f4;
  }
}

/* Born-Mayer-Huggins (Tosi-Fumi NaCl, src/potential/BMHFT/potentialBMHFT.hpp:21-39):
 * c0 = A b, c1 = 6 C, c2 = 8 D (kcal/mol units), c3 = sigma, c4 = 1/rho */
__constant__ double kBornD[2][2][5] = {
    {{25.4435 * 3.1546 / 4.184, 6. * 101.1719 / 4.184, 8. * 48.1771 / 4.184, 2.340, 3.1546},
     {20.3548 * 3.1546 / 4.184, 6. * 674.4793 / 4.184, 8. * 837.077 / 4.184, 2.755, 3.1546}},
    {{20.3548 * 3.1546 / 4.184, 6. * 674.4793 / 4.184, 8. * 837.077 / 4.184, 2.755, 3.1546},
     {15.2661 * 3.1546 / 4.184, 6. * 6985.6786 / 4.184, 8. * 14031.5785 / 4.184, 3.170, 3.1546}}};

/* ------------------------------------------------------------------------- */
/* the dense system of the window                                              */
/* ------------------------------------------------------------------------- */
struct Sys {
  int N, n_ion, nt;
  const int* type;       /* [N] */
  const double* q;       /* [N] charges at s = 1 */
  const double* mass;    /* [N] */
  const double* c;       /* [N] kick coefficient 0.5 dt 4.184e-4 / m */
  const unsigned char* vapor; /* [N] 1 for vapor atoms (taper weights) */
  int n_pairs;
  const int* pi;
  const int* pj;
  const unsigned char* pk;
  const double* A;       /* [nt*nt] */
  const double* B;
  const double* eps;     /* [nt*nt] pair eps / sigma (for the derivatives) */
  const double* sig;
  const int* pidx;       /* [nt*nt] parameter base index (eps; sigma = +1), -1 */
  const int* bmh;        /* [N] Born-Mayer-Huggins row of ion atoms */
  int n_bonds, n_angles, n_dih;
  const int* bonds;      /* [3*n] i, j, type */
  const int* angles;     /* [4*n] */
  const int* dih;        /* [5*n] */
  const double* bond_c;  /* [2*types] */
  const double* angle_c;
  const double* dih_c;   /* [15*types] */
  const int* dih_multi;
  int n_cons, n_colors;
  const int* cons;       /* [3*n] i, j, bond type (length = bond_c[2*type+1]) */
  const int* cons_color;
  const int* cons_nb_off; /* CSR: constraints sharing an atom with constraint k */
  const int* cons_nb;
  int n_cons_nb;          /* entries of cons_nb */
  double ri2, RI2, rcenter, overlap;
  double ion_msum, qqrd2e, dt;
  double efield[3];
  int efield_on, vcorr;
  int n_vmol, a_v, vmol_first; /* in-domain vapor molecules: atoms vmol_first + m*a_v + a */
  double vmol_mass;
  double R0, W, w_energy, w_count, inv_n;
  int n_params;           /* the last one is the charge scale */
};

struct Buf {
  double* X;     /* [(K+1)*3N] positions of the segment */
  double* V;     /* [(K+1)*3N] */
  double* F;     /* [(K+1)*3N] */
  double* gam;   /* [K*n_cons] converged SHAKE multipliers of each step */
  double* lx;    /* [3N] adjoint of x, carried across segments */
  double* lv;    /* [3N] adjoint of v */
  double* lf;    /* [3N] adjoint of F */
  double* tmp;   /* [3N] */
  double* xb;    /* [3N] accumulates the adjoint of the previous positions */
  double* w;     /* [N] taper weights at the current positions */
  double* dw;    /* [3N] their gradients */
  double* om;    /* [N] weight adjoints of the current pass */
  double* mu;    /* [n_cons] */
  double* grad;  /* [n_params] */
  double* J;     /* [1] */
  int* flag;     /* [2] SHAKE convergence scratch, status */
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) red[32] = s;
  }
  __syncthreads();
  s = red[32];
  __syncthreads();
  return s;
}

/* The reverse sweep runs on a cluster of CTAs: its loops are split over all
 * the cluster's threads, its phases are separated by cluster barriers, and
 * global data that other CTAs wrote in the same launch are read from L2
 * (__ldcg), since the L1 caches are not coherent.  A kernel launched without
 * a cluster is a cluster of one CTA (the recompute). */
namespace cg = cooperative_groups;
__device__ __forceinline__ int ctid() { return (int)(cg::this_cluster().block_rank() * blockDim.x + threadIdx.x); }
__device__ __forceinline__ int cnthr() { return (int)(cg::this_cluster().num_blocks() * blockDim.x); }
__device__ __forceinline__ void csync() {
  cg::cluster_group cl = cg::this_cluster();
  if (cl.num_blocks() > 1) {
    __threadfence();
    cl.sync();
  } else {
    __syncthreads();
  }
}

/* three sums over the cluster at once, the same in every CTA (the CTAs'
 * sums added in rank order; two cluster barriers) */
/* three sums over the block, the same in every thread; red >= 67 doubles */
__device__ void block_sum3(double* v, double* red) {
#pragma unroll
  for (int k = 0; k < 3; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0)
    for (int k = 0; k < 3; k++) red[4 * w + k] = v[k];
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0;
    for (int q = 0; q < nw; q++) t += red[4 * q + threadIdx.x];
    red[64 + threadIdx.x] = t;
  }
  __syncthreads();
  for (int k = 0; k < 3; k++) v[k] = red[64 + k];
  __syncthreads();
}

__device__ void cluster_sum3(double* v, double* red) {
  cg::cluster_group cl = cg::this_cluster();
#pragma unroll
  for (int k = 0; k < 3; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0)
    for (int k = 0; k < 3; k++) red[4 * w + k] = v[k]; /* red holds >= 4 * 16 + 3 doubles */
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0;
    for (int q = 0; q < nw; q++) t += red[4 * q + threadIdx.x];
    red[64 + threadIdx.x] = t;
  }
  if (cl.num_blocks() > 1) {
    cl.sync();
    for (int k = 0; k < 3; k++) {
      double t = 0;
      for (unsigned r = 0; r < cl.num_blocks(); r++) t += *cl.map_shared_rank(&red[64 + k], r);
      v[k] = t;
    }
    cl.sync();
  } else {
    __syncthreads();
    for (int k = 0; k < 3; k++) v[k] = red[64 + k];
    __syncthreads();
  }
}

/* ion centre of x (mass-weighted) into cent[0..2] */
__device__ void ion_centre(const Sys& S, const double* x, double* cent, double* red) {
  double sx = 0, sy = 0, sz = 0;
  for (int i = threadIdx.x; i < S.n_ion; i += blockDim.x) {
    sx += x[3 * i] * S.mass[i];
    sy += x[3 * i + 1] * S.mass[i];
    sz += x[3 * i + 2] * S.mass[i];
  }
  sx = block_sum(sx, red);
  sy = block_sum(sy, red);
  sz = block_sum(sz, red);
  if (threadIdx.x == 0) {
    cent[0] = sx / S.ion_msum;
    cent[1] = sy / S.ion_msum;
    cent[2] = sz / S.ion_msum;
  }
  __syncthreads();
}

/* taper weights and their gradients (src/verlet.cpp:109-134) */
__device__ void weights(const Sys& S, const Buf& B, const double* x, const double* cent) {
  const double a = 3.141592653589793 / S.overlap * 0.5;
  for (int i = ctid(); i < S.N; i += cnthr()) {
    double w = 1, g0 = 0, g1 = 0, g2 = 0;
    if (S.vapor[i]) {
      double dx = x[3 * i] - cent[0], dy = x[3 * i + 1] - cent[1], dz = x[3 * i + 2] - cent[2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < S.ri2) w = 1;
      else if (r2 > S.RI2) w = 0;
      else {
        double r = sqrt(r2);
        double C = cos(a * (r - S.rcenter));
        w = C * C;
        double dwdr = -2.0 * C * sin(a * (r - S.rcenter)) * a;
        g0 = dwdr * dx / r;
        g1 = dwdr * dy / r;
        g2 = dwdr * dz / r;
      }
    }
    B.w[i] = w;
    B.dw[3 * i] = g0;
    B.dw[3 * i + 1] = g1;
    B.dw[3 * i + 2] = g2;
  }
  /* no barrier: the callers' next barrier comes before any read */
}

/* force factor f(u) and df/du of one pair (u = r^2), parameter derivatives
 * of f (d eps, d sigma, d s at s = 1), and the pair's weight */
struct PairEval {
  double f, fp, fe, fs_sig, fq, W;
  int p;  /* parameter base, -1 */
  bool ljp;
};

__device__ __forceinline__ PairEval eval_pair(const Sys& S, const Buf& B, int i, int j, int kind, double u) {
  PairEval o;
  o.p = -1;
  o.ljp = false;
  o.fe = o.fs_sig = o.fq = 0;
  o.W = 1;
  const int ti = S.type[i], tj = S.type[j];
  const int tt = ti * S.nt + tj;
  double f = 0, fp = 0;
  if (kind == PK_ION_BMH) {
    const double* cB = kBornD[S.bmh[i]][S.bmh[j]];
    double r = sqrt(u);
    double e = exp(cB[4] * (cB[3] - r));
    double qq = S.qqrd2e * S.q[i] * S.q[j];
    double g = cB[4] * cB[0] * r * e - cB[1] * pow(r, -6.0) - cB[2] * pow(r, -8.0) + qq / r;
    double gp = cB[4] * cB[0] * e * (1.0 - cB[4] * r) + 6.0 * cB[1] * pow(r, -7.0) + 8.0 * cB[2] * pow(r, -9.0) - qq / u;
    f = g / u;
    double dfdr = gp / u - 2.0 * g / (u * r);
    fp = dfdr / (2.0 * r);
    o.fq = 2.0 * qq / (r * u); /* Coulomb scales as s^2 */
  } else {
    const double Aij = S.A[tt], Bij = S.B[tt];
    const double u2 = u * u, u4 = u2 * u2, u3 = u2 * u, u7 = u4 * u3, u8 = u4 * u4;
    f = Aij / u7 - Bij / u4;
    fp = -7.0 * Aij / u8 + 4.0 * Bij / (u4 * u);
    if (kind == PK_GI || kind == PK_VI) {
      o.p = S.pidx[tt];
      if (o.p >= 0) {
        o.ljp = true;
        o.fe = f / S.eps[tt];
        o.fs_sig = (12.0 * Aij / u7 - 6.0 * Bij / u4) / S.sig[tt];
      }
    }
    if (kind == PK_VI || kind == PK_VV || kind == PK_ION_LJC) {
      double qq = S.qqrd2e * S.q[i] * S.q[j];
      double r = sqrt(u);
      double fc = qq / (u * r);
      f += fc;
      fp += -1.5 * fc / u;
      if (kind == PK_VI) o.fq = fc;
      else if (kind == PK_ION_LJC) o.fq = 2.0 * fc;
    }
    if (kind == PK_VI || kind == PK_VV) o.W = __ldcg(B.w + i) * __ldcg(B.w + j);
  }
  o.f = f;
  o.fp = fp;
  return o;
}

/* F(x): all terms, FP64 */
__device__ void forces(const Sys& S, const Buf& B, const double* x, double* F) {
  for (int q = threadIdx.x; q < 3 * S.N; q += blockDim.x) F[q] = 0;
  __syncthreads();
  for (int p = threadIdx.x; p < S.n_pairs; p += blockDim.x) {
    const int i = S.pi[p], j = S.pj[p], k = S.pk[p];
    double d0 = x[3 * i] - x[3 * j], d1 = x[3 * i + 1] - x[3 * j + 1], d2 = x[3 * i + 2] - x[3 * j + 2];
    double u = d0 * d0 + d1 * d1 + d2 * d2;
    PairEval e = eval_pair(S, B, i, j, k, u);
    double g = e.W * e.f;
    atomicAdd(&F[3 * i], g * d0);
    atomicAdd(&F[3 * i + 1], g * d1);
    atomicAdd(&F[3 * i + 2], g * d2);
    atomicAdd(&F[3 * j], -g * d0);
    atomicAdd(&F[3 * j + 1], -g * d1);
    atomicAdd(&F[3 * j + 2], -g * d2);
  }
  const int nb = S.n_bonds, na = S.n_angles, nd = S.n_dih;
  for (int t = threadIdx.x; t < nb + na + nd; t += blockDim.x) {
    int at[4], n;
    double X[4][3], f[4][3];
    if (t < nb) {
      const int* r = S.bonds + 3 * t;
      at[0] = r[0]; at[1] = r[1]; n = 2;
      for (int a = 0; a < n; a++)
        for (int k = 0; k < 3; k++) X[a][k] = x[3 * at[a] + k];
      bond_t<double>(X, S.bond_c + 2 * r[2], f);
    } else if (t < nb + na) {
      const int* r = S.angles + 4 * (t - nb);
      at[0] = r[0]; at[1] = r[1]; at[2] = r[2]; n = 3;
      for (int a = 0; a < n; a++)
        for (int k = 0; k < 3; k++) X[a][k] = x[3 * at[a] + k];
      angle_t<double>(X, S.angle_c + 2 * r[3], f);
    } else {
      const int* r = S.dih + 5 * (t - nb - na);
      at[0] = r[0]; at[1] = r[1]; at[2] = r[2]; at[3] = r[3]; n = 4;
      for (int a = 0; a < n; a++)
        for (int k = 0; k < 3; k++) X[a][k] = x[3 * at[a] + k];
      dihedral_t<double>(X, S.dih_c + 15 * r[4], S.dih_multi[r[4]], f);
    }
    for (int a = 0; a < n; a++)
      for (int k = 0; k < 3; k++) atomicAdd(&F[3 * at[a] + k], f[a][k]);
  }
  if (S.efield_on)
    for (int i = threadIdx.x; i < S.n_ion; i += blockDim.x) {
      double co = 5.55e-5 * S.q[i];
      for (int k = 0; k < 3; k++) atomicAdd(&F[3 * i + k], co * S.efield[k]);
    }
  __syncthreads();
}

/* The parameter derivatives of the pair loops, summed in registers: the
 * pairs are sorted by kind and type pair, so a thread's run of pairs keeps
 * one (eps, sigma) row for many pairs and adds its sums to the shared
 * gradient when the row changes; the charge scale, which every charged pair
 * touches, is summed over the warp first.  (Adding every pair's terms to the
 * few shared rows directly serialised the pair loops on those addresses.) */
__device__ __forceinline__ double warp_sum_dd(double v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}

struct ParamSums {
  int p = -1;
  double e = 0, s = 0, q = 0;
  __device__ __forceinline__ void add_lj(double* sgrad, int row, double de, double ds) {
    if (row != p) {
      flush_lj(sgrad);
      p = row;
    }
    e += de;
    s += ds;
  }
  __device__ __forceinline__ void flush_lj(double* sgrad) {
    if (p >= 0) {
      atomicAdd(&sgrad[p], e);
      atomicAdd(&sgrad[p + 1], s);
    }
    p = -1;
    e = s = 0;
  }
  /* all threads of the block */
  __device__ __forceinline__ void finish(double* sgrad, int n_params) {
    flush_lj(sgrad);
    const double t = warp_sum_dd(q);
    if ((threadIdx.x & 31) == 0 && t != 0) atomicAdd(&sgrad[n_params - 1], t);
    q = 0;
  }
};

/* out += J_F(x)^T lam; grad += (dF/dtheta)^T lam.  Weights must be current. */
__device__ void force_vjp(const Sys& S, const Buf& B, const double* x, const double* lam, double* out,
                          double* sgrad, const double* cent, double* red) {
  /* B.om was zeroed before the caller's last cluster barrier */
  ParamSums ps;
  for (int p = ctid(); p < S.n_pairs; p += cnthr()) {
    const int i = S.pi[p], j = S.pj[p], k = S.pk[p];
    double d[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
    double u = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    PairEval e = eval_pair(S, B, i, j, k, u);
    double m[3] = {__ldcg(lam + 3 * i) - __ldcg(lam + 3 * j), __ldcg(lam + 3 * i + 1) - __ldcg(lam + 3 * j + 1),
                   __ldcg(lam + 3 * i + 2) - __ldcg(lam + 3 * j + 2)};
    double dm = d[0] * m[0] + d[1] * m[1] + d[2] * m[2];
    for (int q = 0; q < 3; q++) {
      double g = e.W * (e.f * m[q] + 2.0 * e.fp * dm * d[q]);
      atomicAdd(&out[3 * i + q], g);
      atomicAdd(&out[3 * j + q], -g);
    }
    if (k == PK_VI || k == PK_VV) {
      double t = e.f * dm;
      if (S.vapor[i]) atomicAdd(&B.om[i], __ldcg(B.w + j) * t);
      if (S.vapor[j]) atomicAdd(&B.om[j], __ldcg(B.w + i) * t);
    }
    if (e.ljp) ps.add_lj(sgrad, e.p, e.W * e.fe * dm, e.W * e.fs_sig * dm);
    if (e.fq != 0) ps.q += e.W * e.fq * dm;
  }
  ps.finish(sgrad, S.n_params);
  csync();
  /* weights: x_i directly, and the ion centre c they are measured from */
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = ctid(); i < S.N; i += cnthr()) {
    if (!S.vapor[i]) continue;
    double o = __ldcg(B.om + i);
    double g0 = o * __ldcg(B.dw + 3 * i), g1 = o * __ldcg(B.dw + 3 * i + 1), g2 = o * __ldcg(B.dw + 3 * i + 2);
    atomicAdd(out + 3 * i, g0);
    atomicAdd(out + 3 * i + 1, g1);
    atomicAdd(out + 3 * i + 2, g2);
    s0 += g0;
    s1 += g1;
    s2 += g2;
  }
  {
    double sv[3] = {s0, s1, s2};
    cluster_sum3(sv, red);
    s0 = sv[0];
    s1 = sv[1];
    s2 = sv[2];
  }
  for (int a = ctid(); a < S.n_ion; a += cnthr()) {
    double fr = S.mass[a] / S.ion_msum;
    atomicAdd(out + 3 * a, -fr * s0);
    atomicAdd(out + 3 * a + 1, -fr * s1);
    atomicAdd(out + 3 * a + 2, -fr * s2);
  }
  /* bonded terms: J lam by forward-mode products (symmetric Jacobians) */
  const int nb = S.n_bonds, na = S.n_angles, nd = S.n_dih;
  for (int t = ctid(); t < nb + na + nd; t += cnthr()) {
    int at[4], n;
    Dual X[4][3], f[4][3];
    const int* r;
    if (t < nb) { r = S.bonds + 3 * t; n = 2; }
    else if (t < nb + na) { r = S.angles + 4 * (t - nb); n = 3; }
    else { r = S.dih + 5 * (t - nb - na); n = 4; }
    for (int a = 0; a < n; a++) {
      at[a] = r[a];
      for (int k = 0; k < 3; k++) X[a][k] = mk(x[3 * at[a] + k], __ldcg(lam + 3 * at[a] + k));
    }
    if (n == 2) bond_t<Dual>(X, S.bond_c + 2 * r[2], f);
    else if (n == 3) angle_t<Dual>(X, S.angle_c + 2 * r[3], f);
    else dihedral_t<Dual>(X, S.dih_c + 15 * r[4], S.dih_multi[r[4]], f);
    for (int a = 0; a < n; a++)
      for (int k = 0; k < 3; k++) atomicAdd(&out[3 * at[a] + k], f[a][k].d);
  }
  if (S.efield_on) {
    double sq = 0;
    for (int i = ctid(); i < S.n_ion; i += cnthr())
      sq += 5.55e-5 * S.q[i] *
            (S.efield[0] * __ldcg(lam + 3 * i) + S.efield[1] * __ldcg(lam + 3 * i + 1) +
             S.efield[2] * __ldcg(lam + 3 * i + 2));
    /* this CTA's share; the CTAs' gradients are summed at the end */
    sq = block_sum(sq, red);
    if (threadIdx.x == 0) sgrad[S.n_params - 1] += sq;
  }
  csync();
}

/* objective at x: value (returned by thread partial), gradient into out
 * (scaled by inv_n) and parameter derivatives into sgrad */
__device__ double objective(const Sys& S, const double* x, double* out, double* sgrad, const double* cent,
                            bool grad, double* red) {
  double jp = 0;
  ParamSums ps;
  if (S.w_energy != 0)
    for (int p = ctid(); p < S.n_pairs; p += cnthr()) {
      if (S.pk[p] != PK_VI) continue;
      const int i = S.pi[p], j = S.pj[p];
      const int tt = S.type[i] * S.nt + S.type[j];
      double d[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
      double u = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      double r = sqrt(u), u3 = u * u * u;
      double qq = S.qqrd2e * S.q[i] * S.q[j];
      double Ulj = S.A[tt] / 12.0 / (u3 * u3) - S.B[tt] / 6.0 / u3;
      jp += S.w_energy * (Ulj + qq / r);
      if (!grad) continue;
      double dUdu = -S.A[tt] / 2.0 / (u3 * u3 * u) + S.B[tt] / 2.0 / (u3 * u) - 0.5 * qq / (u * r);
      double c = 2.0 * dUdu * S.w_energy * S.inv_n;
      for (int q = 0; q < 3; q++) {
        atomicAdd(&out[3 * i + q], c * d[q]);
        atomicAdd(&out[3 * j + q], -c * d[q]);
      }
      const int pb = S.pidx[tt];
      if (pb >= 0)
        ps.add_lj(sgrad, pb, S.w_energy * S.inv_n * Ulj / S.eps[tt],
                  S.w_energy * S.inv_n * (S.A[tt] / (u3 * u3) - S.B[tt] / u3) / S.sig[tt]);
      ps.q += S.w_energy * S.inv_n * qq / r;
    }
  if (grad) ps.finish(sgrad, S.n_params);
  if (S.w_count != 0) {
    /* every CTA takes every molecule (a handful); the first CTA adds the
     * value and the vapor atoms' terms, and the ion atoms' shares of the
     * centre's derivative are summed over the molecules first and then added
     * once per ion atom, split over the cluster */
    const bool lead = cg::this_cluster().block_rank() == 0;
    double C[3] = {0, 0, 0};
    for (int m = threadIdx.x; m < S.n_vmol; m += blockDim.x) {
      const int a0 = S.vmol_first + m * S.a_v;
      double cm[3] = {0, 0, 0};
      for (int a = 0; a < S.a_v; a++)
        for (int q = 0; q < 3; q++) cm[q] += x[3 * (a0 + a) + q] * S.mass[a0 + a];
      for (int q = 0; q < 3; q++) cm[q] /= S.vmol_mass;
      double dv[3] = {cm[0] - cent[0], cm[1] - cent[1], cm[2] - cent[2]};
      double rho = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
      double sgm = 1.0 / (1.0 + exp((rho - S.R0) / S.W));
      if (lead) jp += S.w_count * sgm;
      if (!grad) continue;
      double dSdrho = -sgm * (1.0 - sgm) / S.W * S.w_count * S.inv_n;
      if (lead)
        for (int a = 0; a < S.a_v; a++) {
          double fr = S.mass[a0 + a] / S.vmol_mass;
          for (int q = 0; q < 3; q++) atomicAdd(&out[3 * (a0 + a) + q], dSdrho * fr * dv[q] / rho);
        }
      for (int q = 0; q < 3; q++) C[q] += dSdrho * dv[q] / rho;
    }
    if (grad) {
      block_sum3(C, red);
      for (int b = ctid(); b < S.n_ion; b += cnthr()) {
        double fr = S.mass[b] / S.ion_msum;
        for (int q = 0; q < 3; q++) atomicAdd(&out[3 * b + q], -fr * C[q]);
      }
    }
  }
  /* no barrier: out is read only after the callers' next one */
  return jp;
}

/* SHAKE of every constraint of y against the reference positions xr,
 * colour by colour; gam receives the accumulated multipliers */
__device__ void shake(const Sys& S, const Buf& B, double* y, const double* xr, double* gam) {
  for (int k = threadIdx.x; k < S.n_cons; k += blockDim.x) gam[k] = 0;
  __syncthreads();
  for (int sweep = 0; sweep < SHAKE_SWEEPS; sweep++) {
    for (int col = 0; col < S.n_colors; col++) {
      for (int k = threadIdx.x; k < S.n_cons; k += blockDim.x) {
        if (S.cons_color[k] != col) continue;
        const int i = S.cons[3 * k], j = S.cons[3 * k + 1];
        const double dk = S.bond_c[2 * S.cons[3 * k + 2] + 1];
        const double mi = S.mass[i], mj = S.mass[j];
        double r[3], s[3];
        for (int q = 0; q < 3; q++) {
          r[q] = xr[3 * i + q] - xr[3 * j + q];
          s[q] = y[3 * i + q] - y[3 * j + q];
        }
        double s2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
        double dot = r[0] * s[0] + r[1] * s[1] + r[2] * s[2];
        double minv = 1 / mi + 1 / mj;
        if (dot < 1e-10) dot = 1e-10;
        double g = (dk * dk - s2) / (2 * minv * dot);
        gam[k] += g;
        for (int q = 0; q < 3; q++) {
          y[3 * i + q] += r[q] * g / mi;
          y[3 * j + q] -= r[q] * g / mj;
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) B.flag[0] = 1;
    __syncthreads();
    for (int k = threadIdx.x; k < S.n_cons; k += blockDim.x) {
      const int i = S.cons[3 * k], j = S.cons[3 * k + 1];
      const double dk = S.bond_c[2 * S.cons[3 * k + 2] + 1];
      double s2 = 0;
      for (int q = 0; q < 3; q++) {
        double d = y[3 * i + q] - y[3 * j + q];
        s2 += d * d;
      }
      double dr = s2 - dk * dk;
      if (!(dr * dr <= 1e-20)) B.flag[0] = 0;
    }
    __syncthreads();
    const int conv = B.flag[0];
    __syncthreads();
    if (conv) return;
  }
  if (threadIdx.x == 0) B.flag[1] |= MDN_ST_SHAKE_NOCONV;
  __syncthreads();
}

/* adjoint of the converged projection x = y + sum_k g_k D_k r_k:
 * lam (adjoint of x) -> lam_y written into lam, and the g_k D_k dr_k terms
 * added into xb (adjoint of the reference positions xr) */
__device__ void shake_adjoint(const Sys& S, const Buf& B, const double* x, const double* xr, const double* gam,
                              double* lam, double* xb, double* sc) {
  /* the constraints are few: the first CTA of the cluster solves them with
   * block barriers (x-bar, which the other CTAs added to, read from L2), the
   * others wait at the cluster barrier below */
  if (S.n_cons > 0 && cg::this_cluster().block_rank() == 0) {
    /* G_{kl} = s_k . r_l * coef(k, l); G^T mu = rho, rho_l = r_l . (lam_i/m_i - lam_j/m_j) */
    for (int k = (int)threadIdx.x; k < S.n_cons; k += (int)blockDim.x) B.mu[k] = 0;
    __syncthreads();
    auto G = [&](int k, int l) {
      const int ik = S.cons[3 * k], jk = S.cons[3 * k + 1], il = S.cons[3 * l], jl = S.cons[3 * l + 1];
      double coef = 0;
      if (il == ik) coef += 1.0 / S.mass[il];
      if (jl == ik) coef -= 1.0 / S.mass[jl];
      if (il == jk) coef -= 1.0 / S.mass[il];
      if (jl == jk) coef += 1.0 / S.mass[jl];
      if (coef == 0) return 0.0;
      double sr = 0;
      for (int q = 0; q < 3; q++)
        sr += (x[3 * ik + q] - x[3 * jk + q]) * (xr[3 * il + q] - xr[3 * jl + q]);
      return sr * coef;
    };
    /* what the sweeps reuse, once per step into shared memory (sc): rho_l,
     * G_ll and G_kl of each neighbour entry */
    double* const srho = sc;
    double* const sdiag = sc + S.n_cons;
    double* const snb = sc + 2 * S.n_cons;
    for (int l = (int)threadIdx.x; l < S.n_cons; l += (int)blockDim.x) {
      const int il = S.cons[3 * l], jl = S.cons[3 * l + 1];
      double rho = 0;
      for (int q = 0; q < 3; q++) {
        double rl = xr[3 * il + q] - xr[3 * jl + q];
        rho += rl * (__ldcg(lam + 3 * il + q) / S.mass[il] - __ldcg(lam + 3 * jl + q) / S.mass[jl]);
      }
      srho[l] = rho;
      sdiag[l] = G(l, l);
      for (int e = S.cons_nb_off[l]; e < S.cons_nb_off[l + 1]; e++) snb[e] = G(S.cons_nb[e], l);
    }
    __syncthreads();
    for (int sweep = 0; sweep < SHAKE_SWEEPS; sweep++) {
      if ((int)threadIdx.x == 0) B.flag[0] = 1;
      __syncthreads();
      for (int col = 0; col < S.n_colors; col++) {
        for (int l = (int)threadIdx.x; l < S.n_cons; l += (int)blockDim.x) {
          if (S.cons_color[l] != col) continue;
          double acc = srho[l];
          for (int e = S.cons_nb_off[l]; e < S.cons_nb_off[l + 1]; e++) acc -= snb[e] * B.mu[S.cons_nb[e]];
          double nm = acc / sdiag[l];
          if (fabs(nm - B.mu[l]) > 1e-13 * (fabs(nm) + 1e-300)) B.flag[0] = 0;
          B.mu[l] = nm;
        }
        __syncthreads();
      }
      const int conv = B.flag[0];
      __syncthreads();
      if (conv) break;
    }
    /* lam_y = lam - sum_k mu_k B_k^T (B_k: +s_k at i_k, -s_k at j_k) */
    for (int k = (int)threadIdx.x; k < S.n_cons; k += (int)blockDim.x) {
      const int i = S.cons[3 * k], j = S.cons[3 * k + 1];
      const double mk_ = B.mu[k];
      for (int q = 0; q < 3; q++) {
        double sk = x[3 * i + q] - x[3 * j + q];
        atomicAdd(&lam[3 * i + q], -mk_ * sk);
        atomicAdd(&lam[3 * j + q], mk_ * sk);
      }
    }
    __syncthreads();
    /* g_l D_l dr_l: r_l = xr_i - xr_j */
    for (int l = (int)threadIdx.x; l < S.n_cons; l += (int)blockDim.x) {
      const int i = S.cons[3 * l], j = S.cons[3 * l + 1];
      for (int q = 0; q < 3; q++) {
        double t = gam[l] * (__ldcg(lam + 3 * i + q) / S.mass[i] - __ldcg(lam + 3 * j + q) / S.mass[j]);
        atomicAdd(&xb[3 * i + q], t);
        atomicAdd(&xb[3 * j + q], -t);
      }
    }
    __syncthreads();
  }
  csync();
}

/* The FP64 recompute of one segment: K steps from (X[0], V[0]), keeping x,
 * v, F and the converged SHAKE multipliers of every step; returns the
 * segment's sum of the objective.  first = 1 for the window's first segment,
 * whose start forces are the ones the state holds (f0; zero on a replica
 * that was never stepped, since the reference evaluates no force before the
 * first kick); other segments evaluate F(x_0). */
__device__ double recompute(const Sys& S, const Buf& B, int K, int first, const double* f0, double* red,
                            double* cent) {
  const int n3 = 3 * S.N;
  if (first) {
    for (int q = threadIdx.x; q < n3; q += blockDim.x) B.F[q] = f0[q];
    __syncthreads();
  } else {
    ion_centre(S, B.X, cent, red);
    weights(S, B, B.X, cent);
    forces(S, B, B.X, B.F);
  }
  double jacc = 0;
  for (int t = 1; t <= K; t++) {
    const double* x0 = B.X + (size_t)(t - 1) * n3;
    const double* v0 = B.V + (size_t)(t - 1) * n3;
    const double* f0t = B.F + (size_t)(t - 1) * n3;
    double* x1 = B.X + (size_t)t * n3;
    double* v1 = B.V + (size_t)t * n3;
    double* f1 = B.F + (size_t)t * n3;
    for (int q = threadIdx.x; q < n3; q += blockDim.x) {
      const int i = q / 3;
      double va = v0[q] + S.c[i] * f0t[q];
      v1[q] = va;
      x1[q] = x0[q] + S.dt * va;
    }
    __syncthreads();
    if (S.n_cons > 0) {
      shake(S, B, x1, x0, B.gam + (size_t)(t - 1) * S.n_cons);
      if (S.vcorr)
        for (int q = threadIdx.x; q < n3; q += blockDim.x) {
          double y = x0[q] + S.dt * v1[q];
          v1[q] += (x1[q] - y) / S.dt;
        }
      __syncthreads();
    }
    ion_centre(S, x1, cent, red);
    weights(S, B, x1, cent);
    forces(S, B, x1, f1);
    for (int q = threadIdx.x; q < n3; q += blockDim.x) v1[q] += S.c[q / 3] * f1[q];
    __syncthreads();
    jacc += objective(S, x1, nullptr, nullptr, cent, false, red);
  }
  return block_sum(jacc, red);
}

/* Every segment's recompute at once, one CTA each: CTA s starts from
 * checkpoint s (cpx, cpv) and writes its segment's trajectory at
 * B.X/V/F/gam + s * stride; its scratch (weights, SHAKE flags) at its own
 * offsets; Jseg[s] = the segment's objective sum, flags[2 s + 1] its
 * SHAKE status. */
__global__ void __launch_bounds__(ADJ_THREADS, 1) adjoint_recompute(Sys S, Buf B, int K, long long n_steps,
                                                                    const double* cpx, const double* cpv,
                                                                    const double* f0, double* Jseg) {
  __shared__ double red[40];
  __shared__ double cent[3];
  const int s = blockIdx.x;
  const int n3 = 3 * S.N;
  const int Ks = (int)min((long long)K, n_steps - (long long)s * K);
  Buf b = B;
  const size_t xs = (size_t)(K + 1) * n3;
  b.X += s * xs;
  b.V += s * xs;
  b.F += s * xs;
  b.gam += (size_t)s * K * max(S.n_cons, 1);
  b.w += (size_t)s * S.N;
  b.dw += (size_t)s * n3;
  b.flag += 2 * s;
  for (int q = threadIdx.x; q < n3; q += blockDim.x) {
    b.X[q] = cpx[(size_t)s * n3 + q];
    b.V[q] = cpv[(size_t)s * n3 + q];
  }
  if (threadIdx.x == 0) b.flag[1] = 0;
  __syncthreads();
  const double j = recompute(S, b, Ks, s == 0 ? 1 : 0, f0, red, cent);
  if (threadIdx.x == 0) Jseg[s] = j;
}

/* The reverse sweep of one segment over its recomputed trajectory (B
 * pointing at it), last step first; the adjoints of x, v, F carry over from
 * the segment after it.  f0_theta = 1 on the first segment when its start
 * forces came from a force evaluation at x_0, whose parameter dependence
 * then enters the gradient. */
__global__ void __launch_bounds__(ADJ_THREADS, 1) adjoint_segment(Sys S, Buf B, int K, int first,
                                                                  int f0_theta) {
  __shared__ double sgrad[MAX_PARAMS];
  __shared__ double red[72];
  __shared__ double cent[3];
  extern __shared__ double csh[]; /* 2 n_cons + n_cons_nb doubles for the SHAKE adjoint */
  const int n3 = 3 * S.N;
  for (int p = threadIdx.x; p < S.n_params; p += blockDim.x) sgrad[p] = 0;
  for (int i = ctid(); i < S.N; i += cnthr()) B.om[i] = 0;
  __syncthreads();
  for (int t = K; t >= 1; t--) {
    const double* x0 = B.X + (size_t)(t - 1) * n3;
    const double* x1 = B.X + (size_t)t * n3;
    /* every CTA its own copy of the centre */
    ion_centre(S, x1, cent, red);
    weights(S, B, x1, cent);
    /* objective at x_t */
    objective(S, x1, B.lx, sgrad, cent, true, red);
    /* (6): F-bar += c V-bar (each thread its own elements throughout) */
    for (int q = ctid(); q < n3; q += cnthr()) B.lf[q] += S.c[q / 3] * B.lv[q];
    csync();
    /* (5): x-bar += J^T F-bar */
    force_vjp(S, B, x1, B.lf, B.lx, sgrad, cent, red);
    /* (4): v_b = v_a + (x_t - y)/dt */
    const bool vc = S.n_cons > 0 && S.vcorr;
    for (int q = ctid(); q < n3; q += cnthr()) {
      if (vc) B.lx[q] = __ldcg(B.lx + q) + B.lv[q] / S.dt;
      B.xb[q] = 0;
    }
    csync();
    /* (3): SHAKE adjoint: lx becomes the adjoint of y; xb gets the r-terms */
    if (S.n_cons > 0) shake_adjoint(S, B, x1, x0, B.gam + (size_t)(t - 1) * S.n_cons, B.lx, B.xb, csh);
    /* (2) y = x + dt v_a; (1) v_a = v + c F */
    for (int q = ctid(); q < n3; q += cnthr()) {
      double ly = __ldcg(B.lx + q);
      if (vc) ly -= B.lv[q] / S.dt;
      const double lva = B.lv[q] + S.dt * ly;
      B.lx[q] = ly + __ldcg(B.xb + q);
      B.lv[q] = lva;
      B.lf[q] = S.c[q / 3] * lva;
    }
    /* the weight adjoints of the next force product start at zero */
    for (int i = ctid(); i < S.N; i += cnthr()) B.om[i] = 0;
    csync();
  }
  if (first && f0_theta) {
    /* F(x_0): its parameter dependence */
    ion_centre(S, B.X, cent, red);
    weights(S, B, B.X, cent);
    force_vjp(S, B, B.X, B.lf, B.tmp, sgrad, cent, red);
  }
  __syncthreads();
  /* the CTAs' shares of the gradient */
  for (int p = threadIdx.x; p < S.n_params; p += blockDim.x)
    if (sgrad[p] != 0) atomicAdd(B.grad + p, sgrad[p]);
}

/* ------------------------------------------------------------------------- */
/* host side                                                                   */
/* ------------------------------------------------------------------------- */
int err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return mdn_error(code, buf);
}

struct ParamRow {
  int kind, ta, tb;
};

/* the parameter rows of a descriptor, in the documented order */
std::vector<ParamRow> param_rows(const mdn_replica_desc* d) {
  std::set<int> gt, it, vt;
  for (int i = 0; i < d->gas.n_atoms; i++) gt.insert(d->gas.type[i]);
  for (int i = 0; i < d->ion.n_atoms; i++) it.insert(d->ion.type[i]);
  for (int i = 0; i < d->vapor.n_atoms; i++) vt.insert(d->vapor.type[i]);
  std::vector<ParamRow> rows;
  if (d->interactions & MDN_I_GI)
    for (int g : gt)
      for (int i : it) rows.push_back({0, g, i});
  if (d->interactions & MDN_I_VI)
    for (int v : vt)
      for (int i : it) rows.push_back({1, v, i});
  rows.push_back({2, 0, 0});
  return rows;
}

template <class T>
T* dput(const std::vector<T>& v, std::vector<void*>& owned) {
  T* p = nullptr;
  if (cudaMalloc((void**)&p, sizeof(T) * std::max<size_t>(v.size(), 1)) != cudaSuccess) return nullptr;
  owned.push_back(p);
  if (!v.empty()) cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
  return p;
}

template <class T>
T* dzero(size_t n, std::vector<void*>& owned) {
  T* p = nullptr;
  if (cudaMalloc((void**)&p, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess) return nullptr;
  owned.push_back(p);
  cudaMemset(p, 0, sizeof(T) * std::max<size_t>(n, 1));
  return p;
}

}  // namespace

extern "C" int mdn_adjoint_params(const mdn_replica_desc* d, int* n_params, int* rows, int capacity) {
  if (!d || !n_params) return err(MDN_ERR_ARG, "mdn_adjoint_params: null argument");
  std::vector<ParamRow> r = param_rows(d);
  *n_params = 2 * (int)(r.size() - 1) + 1;
  if (rows)
    for (int k = 0; k < (int)r.size() && k < capacity; k++) {
      rows[3 * k] = r[k].kind;
      rows[3 * k + 1] = r[k].ta;
      rows[3 * k + 2] = r[k].tb;
    }
  return MDN_OK;
}

extern "C" int mdn_adjoint(mdn_handle* h, const mdn_replica_desc* d, const mdn_adjoint_spec* spec, double* J,
                           double* grad, double* ms) {
  if (!h || !d || !spec || !J || !grad) return err(MDN_ERR_ARG, "mdn_adjoint: null argument");
  SnapshotArgs sa;
  mdn_snapshot_args(h, &sa);
  if (sa.R != 1) return err(MDN_ERR_ARG, "mdn_adjoint needs a handle with one replica (it has %d)", sa.R);
  if (spec->n_steps <= 0 || spec->checkpoint_every <= 0)
    return err(MDN_ERR_ARG, "mdn_adjoint: n_steps and checkpoint_every must be positive");
  if (d->nvt_mode != MDN_NVT_OFF) return err(MDN_ERR_ARG, "mdn_adjoint: the thermostat must be off");
  if (d->interactions & MDN_I_GG) return err(MDN_ERR_ARG, "mdn_adjoint: gg is not available");
  if (spec->count_width <= 0) return err(MDN_ERR_ARG, "mdn_adjoint: count_width must be positive");
  cudaSetDevice(sa.dev);
  const unsigned quirks = mdn_internal_quirks(h);
  mdn_replica_info info;
  int rc = mdn_replica_info_get(h, 0, &info);
  if (rc) return rc;
  if ((long long)info.loop_pair + spec->n_steps > info.loop_update)
    return err(MDN_ERR_ARG,
               "mdn_adjoint: the window of %lld steps crosses the rebuild after %d more steps; shorten it or "
               "raise the margin",
               spec->n_steps, info.loop_update - info.loop_pair);
  /* ---- the state at the window start and the dense atom order (the order
   * of the snapshot gather: ion, in-domain gas molecules, in-domain vapor) */
  const int ni = info.n_ion, ag = info.gas_atoms, av = info.vapor_atoms, ng = info.n_gas, nv = info.n_vapor;
  const size_t nm = 1 + (size_t)ng + nv;
  std::vector<double> ion_x(3 * ni), ion_v(3 * ni), ion_f(3 * ni), mol_x(3 * nm), mol_v(3 * nm);
  std::vector<unsigned char> region(nm);
  std::vector<double> gx(3 * (size_t)ng * ag), gvv(gx.size()), gf(gx.size());
  std::vector<double> vx(3 * (size_t)nv * av), vvv(vx.size()), vf(vx.size()), vw((size_t)nv * av);
  mdn_state st;
  memset(&st, 0, sizeof st);
  st.ion_x = ion_x.data(); st.ion_v = ion_v.data(); st.ion_f = ion_f.data();
  st.mol_x = mol_x.data(); st.mol_v = mol_v.data(); st.region = region.data();
  st.gas_ax = gx.data(); st.gas_av = gvv.data(); st.gas_af = gf.data();
  st.vap_ax = vx.data(); st.vap_av = vvv.data(); st.vap_af = vf.data(); st.vap_w = vw.data();
  if ((rc = mdn_download_state(h, 0, &st))) return rc;
  std::vector<int> gin, vin;
  for (int q = 0; q < ng; q++)
    if (region[1 + q]) gin.push_back(q);
  for (int q = 0; q < nv; q++)
    if (region[1 + ng + q]) vin.push_back(q);
  const int N = ni + (int)gin.size() * ag + (int)vin.size() * av;
  const int gas0 = ni, vap0 = ni + (int)gin.size() * ag;
  std::vector<int> gslot(ng, -1), vslot(nv, -1);
  for (size_t k = 0; k < gin.size(); k++) gslot[gin[k]] = (int)k;
  for (size_t k = 0; k < vin.size(); k++) vslot[vin[k]] = (int)k;
  std::vector<double> x0(3 * (size_t)N), v0(3 * (size_t)N);
  std::vector<int> type(N);
  std::vector<double> q(N), mass(N), cc(N);
  std::vector<unsigned char> isvap(N, 0);
  std::vector<int> bmh(N, 0);
  auto put = [&](int a, const double* xs, const double* vs, int t, double qa) {
    for (int k = 0; k < 3; k++) {
      x0[3 * a + k] = xs[k];
      v0[3 * a + k] = vs[k];
    }
    type[a] = t;
    q[a] = qa;
    mass[a] = d->atom_mass[t];
    cc[a] = 0.5 * d->dt * 4.184e-4 / d->atom_mass[t];
  };
  for (int i = 0; i < ni; i++) {
    put(i, &ion_x[3 * i], &ion_v[3 * i], d->ion.type[i], d->ion.charge[i]);
    bmh[i] = d->ion_bmh_type ? d->ion_bmh_type[i] : 0;
  }
  for (size_t k = 0; k < gin.size(); k++)
    for (int a = 0; a < ag; a++) {
      size_t src = 3 * ((size_t)gin[k] * ag + a);
      put(gas0 + (int)k * ag + a, &gx[src], &gvv[src], d->gas.type[a], d->gas.charge[a]);
    }
  for (size_t k = 0; k < vin.size(); k++)
    for (int a = 0; a < av; a++) {
      size_t src = 3 * ((size_t)vin[k] * av + a);
      const int at = vap0 + (int)k * av + a;
      put(at, &vx[src], &vvv[src], d->vapor.type[a], d->vapor.charge[a]);
      isvap[at] = 1;
    }
  /* ---- pairs ---- */
  const unsigned I = d->interactions;
  std::vector<int> pi, pj;
  std::vector<unsigned char> pk;
  auto addp = [&](int i, int j, int k) {
    pi.push_back(i);
    pj.push_back(j);
    pk.push_back((unsigned char)k);
  };
  if (I & MDN_I_GI) {
    int cnt = 0;
    if ((rc = mdn_pair_list(h, 0, 0, nullptr, 0, &cnt))) return rc;
    std::vector<int> pl(2 * (size_t)std::max(cnt, 1));
    if ((rc = mdn_pair_list(h, 0, 0, pl.data(), cnt, &cnt))) return rc;
    for (int e = 0; e < cnt; e++) {
      const int g = pl[2 * e], j = pl[2 * e + 1];
      if (gslot[g] < 0) return err(MDN_ERR_ARG, "mdn_adjoint: gas-ion list names molecule %d outside the domain", g);
      for (int a = 0; a < ag; a++) addp(gas0 + gslot[g] * ag + a, j, PK_GI);
    }
  }
  if (I & MDN_I_GV) {
    int cnt = 0;
    if ((rc = mdn_pair_list(h, 0, 1, nullptr, 0, &cnt))) return rc;
    std::vector<int> pl(2 * (size_t)std::max(cnt, 1));
    if ((rc = mdn_pair_list(h, 0, 1, pl.data(), cnt, &cnt))) return rc;
    const int nj = (quirks & MDN_Q_GV_GAS_COUNT) ? std::min(ag, av) : av;
    for (int e = 0; e < cnt; e++) {
      const int g = pl[2 * e], m = pl[2 * e + 1];
      if (gslot[g] < 0 || vslot[m] < 0) return err(MDN_ERR_ARG, "mdn_adjoint: gas-vapor list outside the domain");
      for (int a = 0; a < ag; a++)
        for (int b = 0; b < nj; b++) addp(gas0 + gslot[g] * ag + a, vap0 + vslot[m] * av + b, PK_GV);
    }
  }
  const int nvin = (int)vin.size();
  if (I & MDN_I_VI)
    for (int k = 0; k < nvin; k++)
      for (int a = 0; a < av; a++)
        for (int j = 0; j < ni; j++) addp(vap0 + k * av + a, j, PK_VI);
  if (I & MDN_I_VV)
    for (int k = 0; k < nvin; k++)
      for (int l = k + 1; l < nvin; l++)
        for (int a = 0; a < av; a++)
          for (int b = 0; b < av; b++) addp(vap0 + k * av + a, vap0 + l * av + b, PK_VV);
  if (I & MDN_I_AMBER) {
    std::vector<char> ex((size_t)ni * ni, 0);
    auto mark = [&](int a, int b) { ex[(size_t)a * ni + b] = ex[(size_t)b * ni + a] = 1; };
    for (int k = 0; k < d->ion.n_bonds; k++) mark(d->ion.bonds[3 * k], d->ion.bonds[3 * k + 1]);
    for (int k = 0; k < d->ion.n_rigid; k++) mark(d->ion.rigid[3 * k], d->ion.rigid[3 * k + 1]);
    for (int k = 0; k < d->ion.n_angles; k++) mark(d->ion.angles[4 * k], d->ion.angles[4 * k + 2]);
    for (int k = 0; k < d->ion.n_dihedrals; k++) mark(d->ion.dihedrals[5 * k], d->ion.dihedrals[5 * k + 3]);
    for (int i = 0; i < ni; i++)
      for (int j = i + 1; j < ni; j++)
        if (!ex[(size_t)i * ni + j]) addp(i, j, PK_ION_LJC);
  }
  if (I & MDN_I_BMH)
    for (int i = 0; i < ni; i++)
      for (int j = i + 1; j < ni; j++) addp(i, j, PK_ION_BMH);
  /* ---- bonded terms and constraints ---- */
  std::vector<int> bonds, angles, dih, cons;
  auto add_top = [&](const mdn_topology& t, int base, bool bonded) {
    if (bonded) {
      for (int k = 0; k < t.n_bonds; k++)
        bonds.insert(bonds.end(), {base + t.bonds[3 * k], base + t.bonds[3 * k + 1], t.bonds[3 * k + 2]});
      for (int k = 0; k < t.n_angles; k++)
        angles.insert(angles.end(), {base + t.angles[4 * k], base + t.angles[4 * k + 1], base + t.angles[4 * k + 2],
                                     t.angles[4 * k + 3]});
      for (int k = 0; k < t.n_dihedrals; k++)
        dih.insert(dih.end(), {base + t.dihedrals[5 * k], base + t.dihedrals[5 * k + 1], base + t.dihedrals[5 * k + 2],
                               base + t.dihedrals[5 * k + 3], t.dihedrals[5 * k + 4]});
    }
    if (I & MDN_I_SHAKE)
      for (int k = 0; k < t.n_rigid; k++)
        cons.insert(cons.end(), {base + t.rigid[3 * k], base + t.rigid[3 * k + 1], t.rigid[3 * k + 2]});
  };
  add_top(d->ion, 0, (I & MDN_I_AMBER) != 0);
  for (size_t k = 0; k < gin.size(); k++) add_top(d->gas, gas0 + (int)k * ag, (I & MDN_I_GAS_INTRA) != 0);
  for (size_t k = 0; k < vin.size(); k++) add_top(d->vapor, vap0 + (int)k * av, (I & MDN_I_VAPOR_INTRA) != 0);
  const int ncons = (int)cons.size() / 3;
  std::vector<int> color(ncons, 0);
  int ncolors = ncons ? 1 : 0;
  std::vector<std::vector<int>> by_atom(N);
  for (int k = 0; k < ncons; k++) {
    by_atom[cons[3 * k]].push_back(k);
    by_atom[cons[3 * k + 1]].push_back(k);
  }
  for (int k = 0; k < ncons; k++) {
    std::set<int> used;
    for (int a : {cons[3 * k], cons[3 * k + 1]})
      for (int l : by_atom[a])
        if (l < k) used.insert(color[l]);
    int c = 0;
    while (used.count(c)) c++;
    color[k] = c;
    ncolors = std::max(ncolors, c + 1);
  }
  std::vector<int> nboff(ncons + 1, 0), nb;
  for (int k = 0; k < ncons; k++) {
    std::set<int> s;
    for (int a : {cons[3 * k], cons[3 * k + 1]})
      for (int l : by_atom[a])
        if (l != k) s.insert(l);
    nb.insert(nb.end(), s.begin(), s.end());
    nboff[k + 1] = (int)nb.size();
  }
  /* ---- parameters ---- */
  const int nt = d->n_atom_types;
  std::vector<double> A((size_t)nt * nt), Bt((size_t)nt * nt), E((size_t)nt * nt), Sg((size_t)nt * nt);
  for (int i = 0; i < nt; i++)
    for (int j = 0; j < nt; j++) {
      const size_t t = (size_t)i * nt + j;
      E[t] = d->pair_eps ? d->pair_eps[t] : sqrt(d->atom_eps[i] * d->atom_eps[j]);
      Sg[t] = d->pair_sigma ? d->pair_sigma[t] : (d->atom_sigma[i] + d->atom_sigma[j]) * 0.5;
      A[t] = 48 * E[t] * pow(Sg[t], 12.0);
      Bt[t] = 24 * E[t] * pow(Sg[t], 6.0);
    }
  std::vector<ParamRow> rows = param_rows(d);
  const int n_params = 2 * (int)(rows.size() - 1) + 1;
  if (n_params > MAX_PARAMS) return err(MDN_ERR_CAPACITY, "mdn_adjoint: %d parameters, at most %d", n_params, MAX_PARAMS);
  std::vector<int> pidx((size_t)nt * nt, -1);
  for (size_t k = 0; k + 1 < rows.size(); k++) {
    const int a = rows[k].ta, b = rows[k].tb;
    if (pidx[(size_t)a * nt + b] >= 0) return err(MDN_ERR_ARG, "mdn_adjoint: type pair (%d, %d) is both gas-ion and vapor-ion", a, b);
    pidx[(size_t)a * nt + b] = pidx[(size_t)b * nt + a] = 2 * (int)k;
  }
  /* ---- device buffers ---- */
  const int K = spec->checkpoint_every;
  const long long nseg = (spec->n_steps + K - 1) / K;
  std::vector<void*> owned;
  auto cleanup = [&]() {
    for (void* p : owned) cudaFree(p);
  };
  Sys S;
  memset(&S, 0, sizeof S);
  S.N = N;
  S.n_ion = ni;
  S.nt = nt;
  S.type = dput(type, owned);
  S.q = dput(q, owned);
  S.mass = dput(mass, owned);
  S.c = dput(cc, owned);
  S.vapor = dput(isvap, owned);
  /* pairs grouped by kind and type pair, so that a thread's strided run of
   * pairs stays on one parameter row (ParamSums) */
  {
    std::vector<size_t> ord(pi.size());
    for (size_t k = 0; k < ord.size(); k++) ord[k] = k;
    auto key = [&](size_t k) { return ((long long)pk[k] * nt + type[pi[k]]) * nt + type[pj[k]]; };
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return key(a) < key(b); });
    std::vector<int> pi2(pi.size()), pj2(pi.size());
    std::vector<unsigned char> pk2(pi.size());
    for (size_t k = 0; k < ord.size(); k++) {
      pi2[k] = pi[ord[k]];
      pj2[k] = pj[ord[k]];
      pk2[k] = pk[ord[k]];
    }
    pi.swap(pi2);
    pj.swap(pj2);
    pk.swap(pk2);
  }
  S.n_pairs = (int)pi.size();
  S.pi = dput(pi, owned);
  S.pj = dput(pj, owned);
  S.pk = dput(pk, owned);
  S.A = dput(A, owned);
  S.B = dput(Bt, owned);
  S.eps = dput(E, owned);
  S.sig = dput(Sg, owned);
  S.pidx = dput(pidx, owned);
  S.bmh = dput(bmh, owned);
  S.n_bonds = (int)bonds.size() / 3;
  S.n_angles = (int)angles.size() / 4;
  S.n_dih = (int)dih.size() / 5;
  S.bonds = dput(bonds, owned);
  S.angles = dput(angles, owned);
  S.dih = dput(dih, owned);
  S.bond_c = dput(std::vector<double>(d->bond_coeff, d->bond_coeff + 2 * d->n_bond_types), owned);
  S.angle_c = dput(std::vector<double>(d->angle_coeff, d->angle_coeff + 2 * d->n_angle_types), owned);
  S.dih_c = dput(std::vector<double>(d->dihedral_coeff, d->dihedral_coeff + 15 * d->n_dihedral_types), owned);
  S.dih_multi = dput(std::vector<int>(d->dihedral_multi, d->dihedral_multi + d->n_dihedral_types), owned);
  S.n_cons = ncons;
  S.n_colors = ncolors;
  S.cons = dput(cons, owned);
  S.cons_color = dput(color, owned);
  S.cons_nb_off = dput(nboff, owned);
  S.cons_nb = dput(nb, owned);
  S.n_cons_nb = (int)nb.size();
  S.ri2 = d->r_inter * d->r_inter;
  S.RI2 = (d->r_inter + d->overlap) * (d->r_inter + d->overlap);
  S.rcenter = d->r_inter - d->overlap * 0.5;
  S.overlap = d->overlap;
  double msum = 0;
  for (int i = 0; i < ni; i++) msum += mass[i];
  S.ion_msum = msum;
  S.qqrd2e = 1.602e-19 * 1.602e-19 / 4.0 / M_PI / 8.85e-12 * 6.02e23 * 1e10 / 4184.0; /* src/constants.hpp */
  S.dt = d->dt;
  for (int k = 0; k < 3; k++) S.efield[k] = d->efield[k];
  S.efield_on = (I & MDN_I_EFIELD) != 0;
  S.vcorr = !(quirks & MDN_Q_SHAKE_NO_VCORR);
  S.n_vmol = nvin;
  S.a_v = av;
  S.vmol_first = vap0;
  double vm = 0;
  for (int a = 0; a < av; a++) vm += d->atom_mass[d->vapor.type[a]];
  S.vmol_mass = vm;
  S.R0 = spec->count_radius;
  S.W = spec->count_width;
  S.w_energy = spec->w_energy;
  S.w_count = spec->w_count;
  S.inv_n = 1.0 / (double)spec->n_steps;
  S.n_params = n_params;
  const size_t n3 = 3 * (size_t)N;
  Buf Bf;
  memset(&Bf, 0, sizeof Bf);
  /* every segment's recomputed trajectory (the recomputes run at once) */
  Bf.X = dzero<double>((size_t)nseg * (K + 1) * n3, owned);
  Bf.V = dzero<double>((size_t)nseg * (K + 1) * n3, owned);
  Bf.F = dzero<double>((size_t)nseg * (K + 1) * n3, owned);
  Bf.gam = dzero<double>((size_t)nseg * K * std::max(ncons, 1), owned);
  Bf.lx = dzero<double>(n3, owned);
  Bf.lv = dzero<double>(n3, owned);
  Bf.lf = dzero<double>(n3, owned);
  Bf.tmp = dzero<double>(n3, owned);
  Bf.xb = dzero<double>(n3, owned);
  Bf.w = dzero<double>((size_t)nseg * N, owned);
  Bf.dw = dzero<double>((size_t)nseg * n3, owned);
  Bf.om = dzero<double>(N, owned);
  Bf.mu = dzero<double>(std::max(ncons, 1), owned);
  Bf.grad = dzero<double>(n_params, owned);
  Bf.J = dzero<double>(1, owned);
  Bf.flag = dzero<int>(2 * (size_t)nseg, owned);
  double* d_jseg = dzero<double>(nseg, owned);
  /* the forces the state holds at the window start */
  std::vector<double> f0(3 * (size_t)N, 0.0);
  for (int i = 0; i < ni; i++)
    for (int k = 0; k < 3; k++) f0[3 * i + k] = ion_f[3 * i + k];
  for (size_t kq = 0; kq < gin.size(); kq++)
    for (int a = 0; a < ag; a++)
      for (int k = 0; k < 3; k++) f0[3 * (gas0 + kq * ag + a) + k] = gf[3 * ((size_t)gin[kq] * ag + a) + k];
  for (size_t kq = 0; kq < vin.size(); kq++)
    for (int a = 0; a < av; a++)
      for (int k = 0; k < 3; k++) f0[3 * (vap0 + kq * av + a) + k] = vf[3 * ((size_t)vin[kq] * av + a) + k];
  double* d_f0 = dput(f0, owned);
  const int f0_theta = info.step > 0 ? 1 : 0;
  /* checkpoints: x, v of every segment start, gathered on the device */
  double* cpx = dzero<double>((size_t)nseg * n3, owned);
  double* cpv = dzero<double>((size_t)nseg * n3, owned);
  long long* cpo = dzero<long long>(2, owned);
  int* cpt = dzero<int>(N, owned);
  for (void* p : owned)
    if (!p) {
      cleanup();
      return err(MDN_ERR_CUDA, "mdn_adjoint: device allocation failed");
    }
  if (!Bf.X || !cpx) {
    cleanup();
    return err(MDN_ERR_CUDA, "mdn_adjoint: device allocation failed");
  }
  /* ---- forward window on the engine, checkpoint at each segment start ---- */
  cudaStream_t stream = (cudaStream_t)sa.stream;
  float fwd_ms = 0;
  {
    std::vector<double> chk(n3);
    for (long long s = 0; s < nseg; s++) {
      if (mdn_snapshot_device(sa.P, sa.D, sa.iblob, 1, sa.ion_x, sa.ion_v, sa.slab_x, sa.slab_v, sa.vslab_x,
                              sa.vslab_v, cpo, cpt, cpx + s * n3, cpv + s * n3, N, stream)) {
        cleanup();
        return err(MDN_ERR_CUDA, "mdn_adjoint: checkpoint gather failed");
      }
      if (s == 0) {
        /* the gather's row order must be the dense order */
        cudaStreamSynchronize(stream);
        cudaMemcpy(chk.data(), cpx, sizeof(double) * n3, cudaMemcpyDeviceToHost);
        if (memcmp(chk.data(), x0.data(), sizeof(double) * n3) != 0) {
          cleanup();
          return err(MDN_ERR_ARG, "mdn_adjoint: the engine's slab order differs from ascending molecule order");
        }
      }
      const long long n = std::min<long long>(K, spec->n_steps - s * K);
      rc = mdn_step(h, n, 0);
      if (rc) {
        cleanup();
        return rc;
      }
      double step_ms = 0;
      long long nl = 0;
      mdn_last_timing(h, &step_ms, &nl);
      fwd_ms += (float)step_ms;
    }
  }
  /* ---- backward, one segment per launch, last first ---- */
  const size_t cbytes = sizeof(double) * (2 * (size_t)ncons + (size_t)S.n_cons_nb);
  if (cbytes > 200 * 1024) {
    cleanup();
    return err(MDN_ERR_CAPACITY, "mdn_adjoint: %d constraints in the domain, too many for the reverse sweep", ncons);
  }
  if (cbytes > 48 * 1024 &&
      cudaFuncSetAttribute(adjoint_segment, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cbytes) != cudaSuccess) {
    cleanup();
    return err(MDN_ERR_CUDA, "mdn_adjoint: reverse sweep shared memory");
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, stream);
  adjoint_recompute<<<(unsigned)nseg, ADJ_THREADS, 0, stream>>>(S, Bf, K, spec->n_steps, cpx, cpv, d_f0, d_jseg);
  for (long long s = nseg - 1; s >= 0; s--) {
    const int n = (int)std::min<long long>(K, spec->n_steps - s * K);
    Buf b = Bf;
    b.X += s * (K + 1) * n3;
    b.V += s * (K + 1) * n3;
    b.F += s * (K + 1) * n3;
    b.gam += (size_t)s * K * std::max(ncons, 1);
    /* one cluster of ADJ_CLUSTER CTAs per segment (fewer if the GPU cannot
     * place that many) */
    cudaError_t le = cudaErrorUnknown;
    if (ADJ_CLUSTER > 8) {
      cudaFuncSetAttribute(adjoint_segment, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      cudaGetLastError();
    }
    for (int C = ADJ_CLUSTER; C >= 1; C /= 2) {
      cudaLaunchConfig_t cfg;
      memset(&cfg, 0, sizeof cfg);
      cfg.gridDim = dim3(C);
      cfg.blockDim = dim3(ADJ_THREADS);
      cfg.dynamicSmemBytes = cbytes;
      cfg.stream = stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = C;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      le = cudaLaunchKernelEx(&cfg, adjoint_segment, S, b, n, s == 0 ? 1 : 0, f0_theta);
      if (le == cudaSuccess) break;
      cudaGetLastError();
    }
    if (le != cudaSuccess) {
      cleanup();
      return err(MDN_ERR_CUDA, "mdn_adjoint: reverse sweep launch: %s", cudaGetErrorString(le));
    }
  }
  cudaEventRecord(e1, stream);
  cudaError_t ce = cudaStreamSynchronize(stream);
  float adj_ms = 0;
  cudaEventElapsedTime(&adj_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ce != cudaSuccess || (ce = cudaGetLastError()) != cudaSuccess) {
    cleanup();
    return err(MDN_ERR_CUDA, "mdn_adjoint: %s", cudaGetErrorString(ce));
  }
  std::vector<int> fl(2 * (size_t)nseg, 0);
  cudaMemcpy(fl.data(), Bf.flag, sizeof(int) * fl.size(), cudaMemcpyDeviceToHost);
  int flags[2] = {0, 0};
  for (long long s = 0; s < nseg; s++) flags[1] |= fl[2 * s + 1];
  /* J: the segments' objective sums, last first (the order the sequential
   * form added them in) */
  std::vector<double> js((size_t)nseg, 0.0);
  cudaMemcpy(js.data(), d_jseg, sizeof(double) * nseg, cudaMemcpyDeviceToHost);
  double jsum = 0.0;
  for (long long s = nseg - 1; s >= 0; s--) jsum += js[s] * S.inv_n;
  *J = jsum;
  cudaMemcpy(grad, Bf.grad, sizeof(double) * n_params, cudaMemcpyDeviceToHost);
  if (ms) {
    ms[0] = fwd_ms;
    ms[1] = adj_ms;
  }
  cleanup();
  if (flags[1] & MDN_ST_SHAKE_NOCONV) return err(MDN_ERR_REPLICA, "mdn_adjoint: SHAKE did not converge in the recomputation");
  return MDN_OK;
}
