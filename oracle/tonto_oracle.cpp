// ============================================================================
// CPU ORACLE — test infrastructure only.
//
// A plain C++ restatement of Tonto's restricted direct J/K build, used by the
// tests, the smoke check and the CPU-baseline leg of bench.py as the checker.
// Nothing in the product (tonto_b200/, include/) links, loads or calls this.
//
// Reference algorithm followed (file:line inside the Tonto project):
//   make_r_JK_direct            foofiles/molecule.fock.foo:1235-1363  (spherical)
//   make_r_JK_engine outer loop foofiles/molecule.fock.foo:1365-1505  (Cartesian;
//        restated with the same integrals and digestion as the direct build —
//        the J-engine is an algebraic rearrangement of the same sums)
//   Schwarz_inequality_test     foofiles/molecule.fock.foo:3454-3495
//   make_max_density_elements   foofiles/molecule.fock.foo:3601-3633
//   make_max_abab_integrals     foofiles/molecule.fock.foo:3712-3752
//   weight_diagonal_blocks, blockwise_symmetric_fold
//                               foofiles/molecule.fock.foo:4181-4263
//   symmetric_reflect           foofiles/mat{intrinsic}.foo:4672-4700
//   SHELL1PAIR precompute       foofiles/shell1pair.foo:100-154
//   set_ab_new / set_cd_new     foofiles/shell1quartet.foo:131-420
//   make_ERI / make_ERI_c       foofiles/shell1quartet.foo:433-503
//   make_esfs_XX, form_esfs     foofiles/shell1quartet.foo:7418-7649
//   transfer_cd / transfer_ab   foofiles/shell1quartet.foo:8310-11134 (HRR)
//   change_to_spherical         foofiles/shell1quartet.foo:505-563
//   set_gaussian_indices        foofiles/gaussian_data.foo:295-479
//   make_xyz_to_solid_harmonics foofiles/gaussian_data.foo:1143-1290
// Rys nodes and weights come from the same generated piecewise tables the
// product uses (tonto_b200/csrc/rys_tables.inc, data only); the tables are
// pinned independently against 50-digit values in tests/golden.
//
// One-electron integrals (overlap, kinetic, nuclear attraction) for the SCF
// checker follow molecule.ints.foo:34-420 in meaning (Obara-Saika overlap and
// kinetic, Rys nuclear attraction).
// ============================================================================

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <array>
#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TF_RYS_CONST static const
#include "rys_tables.inc"
static const int tf_rys_xmax[] = TF_RYS_XMAX_INIT;
static const int tf_rys_offset[] = TF_RYS_OFFSET_INIT;
static const int tf_rys_hoffset[] = TF_RYS_HOFFSET_INIT;

namespace {

const double PI = 3.14159265358979323846;
const double TWOPI5ON2 = 34.9868366552497256925;   // 2 pi^(5/2)
const double SKIP_P = 1.0e-20;                       // TOL(20)

// ---------------------------------------------------------------------------
// Cartesian component tables in Tonto's lexical order (gaussian_data.foo:295-479)
// ---------------------------------------------------------------------------
struct Comp { int x, y, z; };
const int LTAB = 12;
std::vector<Comp> g_comp;          // all components l = 0..LTAB, concatenated
int g_first[LTAB + 2];             // index of the first component of l
int g_index_of[LTAB + 1][LTAB + 1][LTAB + 1];

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

void build_components() {
  if (!g_comp.empty()) return;
  for (int L = 0; L <= LTAB; ++L) {
    g_first[L] = (int)g_comp.size();
    for (int a = L; a >= (int)std::floor((L + 2) / 3.0); --a) {
      for (int b = std::min(L - a, a); b >= (int)std::floor((L - a + 1) * 0.5); --b) {
        int c = L - a - b;
        if (a == b && b == c) {
          g_comp.push_back({a, a, a});
        } else if (a > b && b == c) {
          g_comp.push_back({a, b, b}); g_comp.push_back({b, a, b}); g_comp.push_back({b, b, a});
        } else if (a == b && b > c) {
          g_comp.push_back({a, a, c}); g_comp.push_back({a, c, a}); g_comp.push_back({c, a, a});
        } else {
          g_comp.push_back({a, b, c}); g_comp.push_back({a, c, b}); g_comp.push_back({b, a, c});
          g_comp.push_back({c, a, b}); g_comp.push_back({b, c, a}); g_comp.push_back({c, b, a});
        }
      }
    }
  }
  g_first[LTAB + 1] = (int)g_comp.size();
  for (int i = 0; i < (int)g_comp.size(); ++i) {
    const Comp& c = g_comp[i];
    int L = c.x + c.y + c.z;
    g_index_of[c.x][c.y][c.z] = i - g_first[L];
  }
}

// ---------------------------------------------------------------------------
// Real solid harmonics (Helgaker, Jorgensen & Olsen eqs. 6.4.70-6.4.73), the
// recurrence Tonto uses (gaussian_data.foo:1143-1290).  sph[l] is
// ncart(l) x (2l+1), row = Cartesian component (Tonto order), column order
// m = 0, +1, -1, +2, -2, ... (into_std_S_order, gaussian_data.foo:1292-1350).
// ---------------------------------------------------------------------------
std::vector<std::vector<double>> g_sph;   // g_sph[l][i*(2l+1)+col]
inline int col_of_m(int m) { return m == 0 ? 0 : (m > 0 ? 2 * m - 1 : -2 * m); }

void build_spherical() {
  if (!g_sph.empty()) return;
  build_components();
  const int LS = 6;
  g_sph.resize(LS + 1);
  for (int l = 0; l <= LS; ++l) g_sph[l].assign(ncart(l) * (2 * l + 1), 0.0);
  g_sph[0][0] = 1.0;
  for (int L = 0; L < LS; ++L) {
    const int nsL = 2 * L + 1, nsP = 2 * L + 3;
    double top = 2 * L + 1;
    double fac = std::sqrt((L == 0 ? 2.0 : 1.0) * top / (top + 1));
    double del = (L == 0) ? 0.0 : 1.0;
    for (int i = 0; i < ncart(L); ++i) {
      const Comp& c = g_comp[g_first[L] + i];
      int ix = g_index_of[c.x + 1][c.y][c.z];
      int iy = g_index_of[c.x][c.y + 1][c.z];
      int iz = g_index_of[c.x][c.y][c.z + 1];
      double sLL = g_sph[L][i * nsL + col_of_m(L)];
      double sLmL = g_sph[L][i * nsL + col_of_m(-L)];
      double valp = fac * sLL, valm = fac * sLmL * del;
      g_sph[L + 1][ix * nsP + col_of_m(L + 1)] += valp;
      g_sph[L + 1][iy * nsP + col_of_m(L + 1)] -= valm;
      g_sph[L + 1][ix * nsP + col_of_m(-L - 1)] += valm;
      g_sph[L + 1][iy * nsP + col_of_m(-L - 1)] += valp;
      for (int M = -L; M <= L; ++M) {
        double bot = (double)(L + M + 1) * (L - M + 1);
        g_sph[L + 1][iz * nsP + col_of_m(M)] += (top / std::sqrt(bot)) * g_sph[L][i * nsL + col_of_m(M)];
      }
    }
    if (L >= 1) {
      const int nsM = 2 * L - 1;
      for (int i = 0; i < ncart(L - 1); ++i) {
        const Comp& c = g_comp[g_first[L - 1] + i];
        int ix = g_index_of[c.x + 2][c.y][c.z];
        int iy = g_index_of[c.x][c.y + 2][c.z];
        int iz = g_index_of[c.x][c.y][c.z + 2];
        for (int M = -L + 1; M <= L - 1; ++M) {
          double bot = (double)(L + M + 1) * (L - M + 1);
          double val = std::sqrt((double)(L + M) * (L - M) / bot) * g_sph[L - 1][i * nsM + col_of_m(M)];
          g_sph[L + 1][ix * nsP + col_of_m(M)] -= val;
          g_sph[L + 1][iy * nsP + col_of_m(M)] -= val;
          g_sph[L + 1][iz * nsP + col_of_m(M)] -= val;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FLOP counter: every floating-point +, -, *, /, sqrt and exp the code below
// executes for a shell quartet is tallied (one each) by category, per thread;
// jk_impl files the tally of each quartet under its (la lb|lc ld) class.
// ---------------------------------------------------------------------------
enum FlopCat {
  F_SETUP = 0,   // positioned ket primitive pairs of the quartet (set_cd_new)
  F_PAIR,        // per primitive quartet: rho, P-Q, x, prefactor (make_esfs_XX)
  F_ROOTS,       // Rys nodes and weights (get_weights)
  F_VRR,         // per root: recurrence coefficients, the 2D recurrences, weight
  F_FORM,        // (e0|f0) sums over roots and primitive quartets (form_esfs)
  F_HRR,         // horizontal transfers (transfer_cd, transfer_ab)
  F_SPH,         // Cartesian -> spherical of the integral block (change_to_spherical)
  F_DIGEST,      // J, K digestion (molecule.fock.foo:1322-1338)
  F_NCAT
};
// (the hot loops count into locals and add here once per call)
thread_local double tl_flops[F_NCAT];
inline void add_flops(int cat, double n) { tl_flops[cat] += n; }

// ---------------------------------------------------------------------------
// Rys nodes (t^2) and weights from the generated tables (rys.foo:89-134 role)
// ---------------------------------------------------------------------------
// Returns the FLOPs spent.
inline int rys_roots(int n, double x, double* u, double* w) {
  if (x < tf_rys_xmax[n]) {
    int j = (int)x;
    double s = x - j;
    const double* c = tf_rys_coef + tf_rys_offset[n] + (size_t)j * 2 * n * TF_RYS_NCOEF;
    for (int f = 0; f < 2 * n; ++f) {
      const double* cf = c + f * TF_RYS_NCOEF;
      double v = cf[TF_RYS_DEG];
      for (int k = TF_RYS_DEG - 1; k >= 0; --k) v = v * s + cf[k];
      if (f < n) u[f] = v; else w[f - n] = v;
    }
    return 1 + 2 * n * TF_RYS_DEG * 2;
  } else {
    double ix = 1.0 / x, isx = std::sqrt(ix);
    for (int i = 0; i < n; ++i) {
      u[i] = tf_rys_hroot2[tf_rys_hoffset[n] + i] * ix;
      w[i] = tf_rys_hweight[tf_rys_hoffset[n] + i] * isx;
    }
    return 2 + 2 * n;
  }
}

// ---------------------------------------------------------------------------
// Basis description handed in through the C ABI
// ---------------------------------------------------------------------------
struct Basis {
  int n_atom;
  const double* xyz;           // (n_atom,3) bohr
  int n_shell;
  const int* shell_atom;
  const int* shell_l;
  const int* shell_nprim;
  const int* shell_first_bf;   // Tonto first basis function (0-based)
  std::vector<int> prim_off;
  const double* exps;
  const double* coefs;         // Tonto "unnormalised" contraction coefficients
  int spherical;
  int n_bf;
  int nbf_of(int l) const { return (spherical && l >= 2) ? 2 * l + 1 : ncart(l); }
};

// Position-free shell-pair data (shell1pair.foo:100-154).  Primitive pairs in
// the order b outer, a inner.
struct PairData {
  int a, b;                    // shell indices (a >= b in Tonto pair order)
  int la, lb, l_max, l_min, l_sum;
  std::vector<double> zeta, zinv, cc;      // exponent sum, inverse, c_a c_b zeta^(-3/2)
  std::vector<double> ea, eb;               // the two exponents
};

void make_pair(const Basis& B, int a, int b, PairData& p) {
  p.a = a; p.b = b;
  p.la = B.shell_l[a]; p.lb = B.shell_l[b];
  p.l_max = std::max(p.la, p.lb); p.l_min = std::min(p.la, p.lb); p.l_sum = p.la + p.lb;
  int na = B.shell_nprim[a], nb = B.shell_nprim[b];
  p.zeta.clear(); p.zinv.clear(); p.cc.clear(); p.ea.clear(); p.eb.clear();
  for (int jb = 0; jb < nb; ++jb) {
    double eb = B.exps[B.prim_off[b] + jb], cb = B.coefs[B.prim_off[b] + jb];
    for (int ja = 0; ja < na; ++ja) {
      double ea = B.exps[B.prim_off[a] + ja], ca = B.coefs[B.prim_off[a] + ja];
      double s = ea + eb, inv = 1.0 / s;
      p.zeta.push_back(s); p.zinv.push_back(inv);
      p.cc.push_back(cb * ca * inv * std::sqrt(inv));
      p.ea.push_back(ea); p.eb.push_back(eb);
    }
  }
}

// Positioned primitive pairs of one side of a quartet (set_ab_new :131-275).
struct Side {
  int la, lb, l_max, l_sum;
  bool same_center;
  bool hi_is_first;                          // VRR centre is shell "a" (else "b")
  double R[3];                               // (hi centre) - (lo centre)
  std::vector<double> zeta, zinv, cc, P, PA; // P, PA: 3 per primitive pair
  int n() const { return (int)zeta.size(); }
};

void set_side(const Basis& B, const PairData& pr, bool skip, double pair_cutoff, Side& s) {
  const double* A = B.xyz + 3 * B.shell_atom[pr.a];
  const double* Bp = B.xyz + 3 * B.shell_atom[pr.b];
  s.la = pr.la; s.lb = pr.lb; s.l_max = pr.l_max; s.l_sum = pr.l_sum;
  s.same_center = (B.shell_atom[pr.a] == B.shell_atom[pr.b]);
  s.hi_is_first = (pr.la > pr.lb);           // "if (.a.l > .b.l) At = pos_a else pos_b"
  const double* At = s.hi_is_first ? A : Bp;
  const double* Lo = s.hi_is_first ? Bp : A;
  for (int k = 0; k < 3; ++k) s.R[k] = At[k] - Lo[k];
  s.zeta.clear(); s.zinv.clear(); s.cc.clear(); s.P.clear(); s.PA.clear();
  double AB[3] = {A[0] - Bp[0], A[1] - Bp[1], A[2] - Bp[2]};
  double r2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  double fl_setup = 8.0;
  int np = (int)pr.zeta.size();
  for (int i = 0; i < np; ++i) {
    if (s.same_center && !skip) {
      s.zeta.push_back(pr.zeta[i]); s.zinv.push_back(pr.zinv[i]); s.cc.push_back(pr.cc[i]);
      for (int k = 0; k < 3; ++k) { s.P.push_back(A[k]); s.PA.push_back(0.0); }
      continue;
    }
    double a = pr.ea[i], b = pr.eb[i];
    double inv = pr.zinv[i];
    double b_r2 = b * r2;
    double prefac = std::exp(-a * b_r2 * inv);
    fl_setup += 5.0;                          // b r2, -a, * b_r2, * inv, exp
    if (skip && prefac < pair_cutoff) continue;
    fl_setup += 1.0 + 3.0 * 5.0;              // prefactor; per axis (b B + a A) inv, P - At
    s.zeta.push_back(pr.zeta[i]); s.zinv.push_back(inv); s.cc.push_back(prefac * pr.cc[i]);
    for (int k = 0; k < 3; ++k) {
      double P = (b * Bp[k] + a * A[k]) * inv;
      s.P.push_back(P); s.PA.push_back(P - At[k]);
    }
  }
  add_flops(F_SETUP, fl_setup);
}

// ---------------------------------------------------------------------------
// Instrumented counters (per (l_a l_b | l_c l_d) class, canonical ordering)
// ---------------------------------------------------------------------------
struct ClassCount {
  double quartets = 0, prim_quartets = 0;
  double flops[F_NCAT] = {};
};

// ---------------------------------------------------------------------------
// (e0|f0) by Rys quadrature (make_esfs_XX + form_esfs)
// ---------------------------------------------------------------------------
struct Work {
  std::vector<double> Ix, Iy, Iz, esfs, tmp1, tmp2, cart, out;
  std::vector<double> u, w;
};

// esfs(e,f): e over components with l in [l_max_ab, l_sum_ab] (Tonto lexical
// order), f likewise for cd.  Returns the number of primitive quartets.
long make_esfs(const Side& ab, const Side& cd, Work& W) {
  const int dim1 = ab.l_sum + 1, dim2 = cd.l_sum + 1;
  const int n_roots = (dim1 + dim2) / 2;
  const int nab = ab.n(), ncd = cd.n();
  const int n_sum = n_roots * nab * ncd;
  const int d12 = dim1 * dim2;
  W.Ix.assign((size_t)n_sum * d12, 0.0);
  W.Iy.assign((size_t)n_sum * d12, 0.0);
  W.Iz.assign((size_t)n_sum * d12, 0.0);
  W.u.resize(n_roots); W.w.resize(n_roots);
  int i = 0;
  // recurrence work of one root, one axis (the loops below, counted once)
  double vrr_axis = 4.0 + 4.0 * std::max(0, dim1 - 2);
  for (int f = 0; f + 1 < dim2; ++f)
    for (int e = 0; e < dim1; ++e) vrr_axis += 1.0 + (f > 0 ? 3.0 : 0.0) + (e > 0 ? 3.0 : 0.0);
  const double vrr_root = 8.0 + 3.0 * vrr_axis + d12;
  double fl_pair = 0.0, fl_roots = 0.0;
  for (int k = 0; k < nab; ++k) {
    double ab_cc = ab.cc[k] * TWOPI5ON2, zeta = ab.zeta[k], zinv = ab.zinv[k], half_zinv = 0.5 * zinv;
    fl_pair += 2.0;
    const double* P = &ab.P[3 * k]; const double* PA = &ab.PA[3 * k];
    for (int j = 0; j < ncd; ++j) {
      double cd_cc = cd.cc[j], eta = cd.zeta[j], einv = cd.zinv[j];
      const double* Q = &cd.P[3 * j]; const double* QC = &cd.PA[3 * j];
      double rho = zeta * eta / (zeta + eta);
      double rho_zinv = rho * zinv, rho_einv = rho * einv, half_einv = 0.5 * einv;
      double QP[3] = {Q[0] - P[0], Q[1] - P[1], Q[2] - P[2]};
      double xx = rho * (QP[0] * QP[0] + QP[1] * QP[1] + QP[2] * QP[2]);
      fl_roots += rys_roots(n_roots, xx, W.u.data(), W.w.data());
      double scale = ab_cc * cd_cc * std::sqrt(rho);
      fl_pair += 18.0;                        // rho (3), rho/zeta, rho/eta, 1/(2 eta), Q-P (3), x (6), scale (3)
      for (int n = 0; n < n_roots; ++n, ++i) {
        double t2 = W.u[n];
        double wt = W.w[n] * scale;
        double t2_rz = t2 * rho_zinv, t2_re = t2 * rho_einv;
        double ce = (1.0 - t2_rz) * half_zinv;   // B10
        double cf = (1.0 - t2_re) * half_einv;   // B01
        double bb = t2_rz * half_einv;           // B00
        double* I3[3] = {&W.Ix[(size_t)i * d12], &W.Iy[(size_t)i * d12], &W.Iz[(size_t)i * d12]};
        for (int dir = 0; dir < 3; ++dir) {
          double* I = I3[dir];                   // I[e*dim2+f]
          double c00 = PA[dir] + t2_rz * QP[dir];
          double d00 = QC[dir] - t2_re * QP[dir];
          I[0] = 1.0;
          if (dim1 > 1) I[dim2] = c00;
          for (int e = 1; e + 1 < dim1; ++e) I[(e + 1) * dim2] = c00 * I[e * dim2] + e * ce * I[(e - 1) * dim2];
          for (int f = 0; f + 1 < dim2; ++f) {
            for (int e = 0; e < dim1; ++e) {
              double v = d00 * I[e * dim2 + f];
              if (f > 0) v += f * cf * I[e * dim2 + f - 1];
              if (e > 0) v += e * bb * I[(e - 1) * dim2 + f];
              I[e * dim2 + f + 1] = v;
            }
          }
          if (dir == 2) for (int q = 0; q < d12; ++q) I[q] *= wt;
        }
      }
    }
  }
  // form_esfs (:7615-7649)
  const int fe = g_first[ab.l_max], le = g_first[ab.l_sum + 1];
  const int ff = g_first[cd.l_max], lf = g_first[cd.l_sum + 1];
  const int ne = le - fe, nf = lf - ff;
  W.esfs.assign((size_t)ne * nf, 0.0);
  add_flops(F_PAIR, fl_pair);
  add_flops(F_ROOTS, fl_roots);
  add_flops(F_VRR, (double)n_sum * vrr_root);
  add_flops(F_FORM, 3.0 * ne * nf * (double)n_sum);
  for (int f = 0; f < nf; ++f) {
    const Comp& cf_ = g_comp[ff + f];
    for (int e = 0; e < ne; ++e) {
      const Comp& ce_ = g_comp[fe + e];
      int ox = ce_.x * dim2 + cf_.x, oy = ce_.y * dim2 + cf_.y, oz = ce_.z * dim2 + cf_.z;
      double s = 0.0;
      for (int q = 0; q < n_sum; ++q)
        s += W.Ix[(size_t)q * d12 + ox] * W.Iy[(size_t)q * d12 + oy] * W.Iz[(size_t)q * d12 + oz];
      W.esfs[(size_t)e * nf + f] = s;
    }
  }
  return (long)nab * ncd;
}

// HRR on one side: table G[x][rest] with x over components l in
// [l_hi, l_hi+l_lo] (lexical) -> T[xhi][ylo][rest], xhi in comps(l_hi),
// ylo in comps(l_lo): (x, y+1_i) = (x+1_i, y) + R_i (x, y) with R = hi - lo.
void hrr(int l_hi, int l_lo, const double* R, const double* G, int nrest, std::vector<double>& out,
         std::vector<double>& t1, std::vector<double>& t2) {
  // level-k tables: x over l in [l_hi, l_hi+l_lo-k] (offset from g_first[l_hi]),
  // y over comps(k)
  int nx0 = g_first[l_hi + l_lo + 1] - g_first[l_hi];
  t1.assign(G, G + (size_t)nx0 * nrest);    // k = 0, y = s
  int ny = 1;
  for (int k = 0; k < l_lo; ++k) {
    int nx_new = g_first[l_hi + l_lo - k] - g_first[l_hi];
    int ny_new = ncart(k + 1);
    t2.assign((size_t)nx_new * ny_new * nrest, 0.0);
    for (int y1 = 0; y1 < ny_new; ++y1) {
      const Comp& cy = g_comp[g_first[k + 1] + y1];
      int dir = (cy.x > 0) ? 0 : (cy.y > 0 ? 1 : 2);
      Comp cy0 = cy; if (dir == 0) cy0.x--; else if (dir == 1) cy0.y--; else cy0.z--;
      int y0 = g_index_of[cy0.x][cy0.y][cy0.z];
      for (int x = 0; x < nx_new; ++x) {
        const Comp& cx = g_comp[g_first[l_hi] + x];
        Comp cxp = cx; if (dir == 0) cxp.x++; else if (dir == 1) cxp.y++; else cxp.z++;
        int lxp = cxp.x + cxp.y + cxp.z;
        int xp = g_first[lxp] + g_index_of[cxp.x][cxp.y][cxp.z] - g_first[l_hi];
        const double* a = &t1[((size_t)xp * ny + y0) * nrest];
        const double* b = &t1[((size_t)x * ny + y0) * nrest];
        double* o = &t2[((size_t)x * ny_new + y1) * nrest];
        for (int r = 0; r < nrest; ++r) o[r] = a[r] + R[dir] * b[r];
      }
    }
    add_flops(F_HRR, 2.0 * nrest * (double)nx_new * ny_new);
    t1.swap(t2);
    ny = ny_new;
  }
  // keep only x in comps(l_hi)
  int nxh = ncart(l_hi);
  out.assign(t1.begin(), t1.begin() + (size_t)nxh * ny * nrest);
}

// Cartesian (ab|cd), a fastest: out[((d*nc + c)*nb + b)*na + a]
void make_cart_eri(const Side& ab, const Side& cd, Work& W) {
  make_esfs(ab, cd, W);
  const int ne = g_first[ab.l_sum + 1] - g_first[ab.l_max];
  const int nf = g_first[cd.l_sum + 1] - g_first[cd.l_max];
  const int l_hi_ab = ab.l_max, l_lo_ab = ab.l_sum - ab.l_max;
  const int l_hi_cd = cd.l_max, l_lo_cd = cd.l_sum - cd.l_max;
  // ket HRR: esfs[e][f] -> need f first: transpose to [f][e]
  std::vector<double> Gt((size_t)nf * ne);
  for (int e = 0; e < ne; ++e) for (int f = 0; f < nf; ++f) Gt[(size_t)f * ne + e] = W.esfs[(size_t)e * nf + f];
  std::vector<double> K;   // [chi][dlo][e]
  hrr(l_hi_cd, l_lo_cd, cd.R, Gt.data(), ne, K, W.tmp1, W.tmp2);
  const int nch = ncart(l_hi_cd), ncl = ncart(l_lo_cd);
  // bra HRR: need [e][chi][dlo]
  std::vector<double> G2((size_t)ne * nch * ncl);
  for (int c = 0; c < nch * ncl; ++c) for (int e = 0; e < ne; ++e) G2[(size_t)e * nch * ncl + c] = K[(size_t)c * ne + e];
  std::vector<double> Bra;  // [ahi][blo][chi][dlo]
  hrr(l_hi_ab, l_lo_ab, ab.R, G2.data(), nch * ncl, Bra, W.tmp1, W.tmp2);
  const int nah = ncart(l_hi_ab), nal = ncart(l_lo_ab);
  const int na = ncart(ab.la), nb = ncart(ab.lb), nc = ncart(cd.la), nd = ncart(cd.lb);
  W.cart.assign((size_t)na * nb * nc * nd, 0.0);
  for (int ih = 0; ih < nah; ++ih) for (int il = 0; il < nal; ++il)
    for (int jh = 0; jh < nch; ++jh) for (int jl = 0; jl < ncl; ++jl) {
      int a = ab.hi_is_first ? ih : il, b = ab.hi_is_first ? il : ih;
      int c = cd.hi_is_first ? jh : jl, d = cd.hi_is_first ? jl : jh;
      W.cart[(((size_t)d * nc + c) * nb + b) * na + a] = Bra[(((size_t)ih * nal + il) * nch + jh) * ncl + jl];
    }
}

// change_to_spherical (:505-563): transform each index with l >= 2
void to_spherical(int la, int lb, int lc, int ld, const std::vector<double>& C, std::vector<double>& S,
                  std::vector<double>& tmp) {
  int l4[4] = {la, lb, lc, ld};
  int dims[4] = {ncart(la), ncart(lb), ncart(lc), ncart(ld)};
  S = C;
  double fl_sph = 0.0;
  for (int idx = 0; idx < 4; ++idx) {
    int l = l4[idx];
    if (l < 2) continue;
    int nsph = 2 * l + 1, ncar = ncart(l);
    int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
    nd[idx] = nsph;
    tmp.assign((size_t)nd[0] * nd[1] * nd[2] * nd[3], 0.0);
    const std::vector<double>& U = g_sph[l];
    for (int d = 0; d < dims[3]; ++d) for (int c = 0; c < dims[2]; ++c)
      for (int b = 0; b < dims[1]; ++b) for (int a = 0; a < dims[0]; ++a) {
        int id[4] = {a, b, c, d};
        double v = S[(((size_t)d * dims[2] + c) * dims[1] + b) * dims[0] + a];
        if (v == 0.0) continue;
        int i = id[idx];
        fl_sph += 2.0 * nsph;
        for (int m = 0; m < nsph; ++m) {
          int o[4] = {a, b, c, d}; o[idx] = m;
          tmp[(((size_t)o[3] * nd[2] + o[2]) * nd[1] + o[1]) * nd[0] + o[0]] += U[i * nsph + m] * v;
        }
      }
    (void)ncar;
    S.swap(tmp);
    dims[idx] = nsph;
  }
  add_flops(F_SPH, fl_sph);
}

// make_ERI (:433-457): basis-function block, a fastest
void make_eri(const Basis& B, const Side& ab, const Side& cd, Work& W) {
  make_cart_eri(ab, cd, W);
  if (B.spherical && std::max(ab.l_max, cd.l_max) >= 2) to_spherical(ab.la, ab.lb, cd.la, cd.lb, W.cart, W.out, W.tmp1);
  else W.out = W.cart;
}

inline int pair_index(int a, int b) { return a * (a + 1) / 2 + b; }   // 0-based, a >= b

struct Ctx {
  Basis B;
  std::vector<PairData> pairs;        // Tonto pair order: ab = a(a+1)/2 + b
  std::vector<double> max_I;
  std::vector<ClassCount> counts;     // 5^4 classes (l <= 4)
  double schwarz_cutoff = 1e-12, pair_cutoff = 1e-6;
  // wall times of the last jk call: the shell-quartet loop alone, and the whole call
  // (density maxima, per-thread accumulators, their sum, fold and reflect included)
  double t_loop = 0.0, t_total = 0.0;
};

int class_id(int la, int lb, int lc, int ld) { return ((la * 5 + lb) * 5 + lc) * 5 + ld; }

void init_ctx(Ctx& C) {
  build_components();
  build_spherical();
  const Basis& B = C.B;
  int ns = B.n_shell;
  C.pairs.resize((size_t)ns * (ns + 1) / 2);
  for (int a = 0; a < ns; ++a) for (int b = 0; b <= a; ++b) make_pair(B, a, b, C.pairs[pair_index(a, b)]);
  // make_max_abab_integrals (:3712-3752)
  C.max_I.assign(C.pairs.size(), 0.0);
#pragma omp parallel
  {
    Work W; Side s;
#pragma omp for schedule(dynamic, 16)
    for (long ab = 0; ab < (long)C.pairs.size(); ++ab) {
      const PairData& pr = C.pairs[ab];
      set_side(B, pr, false, C.pair_cutoff, s);
      make_eri(B, s, s, W);
      int na = B.nbf_of(pr.la), nb = B.nbf_of(pr.lb);
      double m = 0.0;
      for (int a = 0; a < na; ++a) for (int b = 0; b < nb; ++b)
        m = std::max(m, std::fabs(W.out[(((size_t)b * na + a) * nb + b) * na + a]));
      C.max_I[ab] = std::sqrt(m);
    }
  }
}

// max |P(a,b)| over each shell pair (:3601-3633); P column-major n_bf x n_bf
void max_density(const Ctx& C, const double* P, std::vector<double>& Pm) {
  const Basis& B = C.B;
  Pm.assign(C.pairs.size(), 0.0);
  for (size_t ab = 0; ab < C.pairs.size(); ++ab) {
    const PairData& pr = C.pairs[ab];
    int fa = B.shell_first_bf[pr.a], fb = B.shell_first_bf[pr.b];
    int na = B.nbf_of(pr.la), nb = B.nbf_of(pr.lb);
    double m = 0.0;
    for (int a = fa; a < fa + na; ++a) for (int b = fb; b < fb + nb; ++b) m = std::max(m, std::fabs(P[(size_t)b * B.n_bf + a]));
    Pm[ab] = m;
  }
}

}  // namespace

// ===========================================================================
// C ABI of the oracle (used through ctypes by tests and bench.py only)
// ===========================================================================
extern "C" {

struct OracleCtx;

OracleCtx* oracle_create(int n_atom, const double* xyz, int n_shell, const int* shell_atom, const int* shell_l,
                         const int* shell_nprim, const int* shell_first_bf, const double* exps, const double* coefs,
                         int spherical, double schwarz_cutoff, double pair_cutoff) {
  Ctx* C = new Ctx();
  Basis& B = C->B;
  B.n_atom = n_atom; B.xyz = xyz; B.n_shell = n_shell; B.shell_atom = shell_atom; B.shell_l = shell_l;
  B.shell_nprim = shell_nprim; B.shell_first_bf = shell_first_bf; B.exps = exps; B.coefs = coefs;
  B.spherical = spherical;
  B.prim_off.resize(n_shell + 1);
  int off = 0;
  B.n_bf = 0;
  for (int s = 0; s < n_shell; ++s) { B.prim_off[s] = off; off += shell_nprim[s]; B.n_bf += B.nbf_of(shell_l[s]); }
  B.prim_off[n_shell] = off;
  C->schwarz_cutoff = schwarz_cutoff;
  C->pair_cutoff = pair_cutoff;
  C->counts.assign(625, ClassCount());
  init_ctx(*C);
  return reinterpret_cast<OracleCtx*>(C);
}

void oracle_destroy(OracleCtx* c) { delete reinterpret_cast<Ctx*>(c); }

void oracle_max_I(OracleCtx* c, double* out) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  std::copy(C->max_I.begin(), C->max_I.end(), out);
}

// One contracted shell quartet (a b|c d) (0-based shell indices, any order),
// Tonto basis-function block with a fastest; skip selects the pair-skip rule.
int oracle_shell_quartet(OracleCtx* c, int a, int b, int cc, int d, int skip, double* out) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  PairData p1, p2;
  make_pair(C->B, a, b, p1);
  make_pair(C->B, cc, d, p2);
  Side s1, s2;
  set_side(C->B, p1, skip != 0, C->pair_cutoff, s1);
  set_side(C->B, p2, skip != 0, C->pair_cutoff, s2);
  Work W;
  make_eri(C->B, s1, s2, W);
  std::copy(W.out.begin(), W.out.end(), out);
  return (int)W.out.size();
}

// make_r_JK_direct (:1235-1363).  P, J, K: column-major n_bf x n_bf.
// max_ab_pairs < 0: all bra pairs; otherwise only the first max_ab_pairs bra
// shell pairs (a bounded sample for CPU timing).  n_threads <= 0: all.
void oracle_jk_sample(OracleCtx* c, const double* P, double* J, double* K, long max_ab_pairs, int n_threads,
                      long ab_stride, long ab_offset);

void oracle_jk(OracleCtx* c, const double* P, double* J, double* K, long max_ab_pairs, int n_threads) {
  oracle_jk_sample(c, P, J, K, max_ab_pairs, n_threads, 1, 0);
}

// One shell quartet (ab|cd) of make_r_JK_direct's loop (molecule.fock.foo:1286-1338):
// Schwarz_inequality_test (:3454-3495), the coincidence factors, the integrals with
// the primitive-pair cutoff where no two atoms coincide, and the digestion into the
// accumulators Jl[sp], Kl[sp] of each density.  ab and cd are Tonto pair indices in
// either order; sides[0] / sides[1] are the bra's positioned primitive pairs without
// and with the cutoff.  The quartet's class counts and FLOPs go to cnt.
static void jk_quartet(const Ctx* C, long ab, long cd, const std::vector<double>& Pm, const Side* const* sides,
                       Side& s_cd, Work& W, int nd, const double* const* Ps, double* const* Jl, double* const* Kl,
                       std::vector<ClassCount>& cnt) {
  const Basis& B = C->B;
  const int n = B.n_bf;
  const double cutoff = C->schwarz_cutoff;
  const PairData& pab = C->pairs[ab];
  const int aa = pab.a, bb = pab.b;
  const int atom_a = B.shell_atom[aa], atom_b = B.shell_atom[bb];
  const bool ab_same = atom_a == atom_b;
  const PairData& pcd = C->pairs[cd];
  const int cc = pcd.a, dd = pcd.b;
  const int atom_c = B.shell_atom[cc], atom_d = B.shell_atom[dd];
  const bool cd_same = atom_c == atom_d;
  {
    const long ac = pair_index(std::max(aa, cc), std::min(aa, cc)), ad = pair_index(std::max(aa, dd), std::min(aa, dd));
    const long bc = pair_index(std::max(bb, cc), std::min(bb, cc)), bd = pair_index(std::max(bb, dd), std::min(bb, dd));
    const double pm = std::max({Pm[ab], Pm[cd], Pm[ac], Pm[ad], Pm[bc], Pm[bd]});
    bool skip;
    if (pm < SKIP_P) skip = true;
    else skip = !(pm * C->max_I[ab] * C->max_I[cd] > cutoff);
    if (skip) return;
  }
  double factor = 1.0;
  if (aa == bb) factor = 0.5;
  if (cc == dd) factor *= 0.5;
  if (ab == cd) factor *= 0.5;
  const bool any_same = ab_same || cd_same || atom_a == atom_c || atom_a == atom_d || atom_b == atom_c ||
                        atom_b == atom_d;
  for (int q = 0; q < F_NCAT; ++q) tl_flops[q] = 0.0;     // this quartet's tally
  set_side(B, pcd, !any_same, C->pair_cutoff, s_cd);
  const Side& s_ab = any_same ? *sides[0] : *sides[1];
  make_eri(B, s_ab, s_cd, W);
  const int fa = B.shell_first_bf[aa], fb = B.shell_first_bf[bb];
  const int na = B.nbf_of(pab.la), nb = B.nbf_of(pab.lb);
  const int fc = B.shell_first_bf[cc], fd = B.shell_first_bf[dd];
  const int nc = B.nbf_of(pcd.la), ndd = B.nbf_of(pcd.lb);
  const double* I = W.out.data();
  add_flops(F_DIGEST, 13.0 * nd * (double)na * nb * nc * ndd);   // factor I, six (+= I P) per density
  {
    // canonical class id: larger pair class first, each pair larger l first
    const int la = pab.la, lb = pab.lb, lc = pcd.la, ld = pcd.lb;
    int p1a = std::max(la, lb), p1b = std::min(la, lb), p2a = std::max(lc, ld), p2b = std::min(lc, ld);
    if (p1a * 5 + p1b < p2a * 5 + p2b) { std::swap(p1a, p2a); std::swap(p1b, p2b); }
    ClassCount& cf = cnt[class_id(p1a, p1b, p2a, p2b)];
    cf.quartets += 1;
    cf.prim_quartets += (double)s_ab.n() * s_cd.n();
    for (int q = 0; q < F_NCAT; ++q) cf.flops[q] += tl_flops[q];
  }
  for (int sp = 0; sp < nd; ++sp) {
    const double* P = Ps[sp];
    double* J = Jl[sp];
    double* K = Kl[sp];
    size_t abcd = 0;
    for (int d = fd; d < fd + ndd; ++d)
      for (int c2 = fc; c2 < fc + nc; ++c2)
        for (int b = fb; b < fb + nb; ++b)
          for (int a = fa; a < fa + na; ++a) {
            double Iv = factor * I[abcd++];
            J[(size_t)b * n + a] += Iv * P[(size_t)c2 * n + d];
            J[(size_t)d * n + c2] += Iv * P[(size_t)a * n + b];
            K[(size_t)c2 * n + a] += Iv * P[(size_t)b * n + d];
            K[(size_t)d * n + a] += Iv * P[(size_t)b * n + c2];
            K[(size_t)c2 * n + b] += Iv * P[(size_t)a * n + d];
            K[(size_t)d * n + b] += Iv * P[(size_t)a * n + c2];
          }
  }
}

// weight_diagonal_blocks(J, 2), blockwise_symmetric_fold(K), J = 2J and the reflection
// of the lower triangles (molecule.fock.foo:1351-1361, 4181-4263) on summed J, K.
static void finish_jk(const Basis& B, double* J, double* K) {
  const int n = B.n_bf;
  // weight_diagonal_blocks(J,2); blockwise_symmetric_fold(K); J = 2J; reflect
  for (int s = 0; s < B.n_shell; ++s) {
    int f = B.shell_first_bf[s], m = B.nbf_of(B.shell_l[s]);
    for (int j = f; j < f + m; ++j) for (int i = f; i < f + m; ++i) J[(size_t)j * n + i] *= 2.0;
  }
  for (int a = 0; a < B.n_shell; ++a) for (int b = 0; b <= a; ++b) {
    int fa = B.shell_first_bf[a], na = B.nbf_of(B.shell_l[a]);
    int fb = B.shell_first_bf[b], nb = B.nbf_of(B.shell_l[b]);
    if (a == b) {
      std::vector<double> blk((size_t)na * na);
      for (int j = 0; j < na; ++j) for (int i = 0; i < na; ++i) blk[(size_t)j * na + i] = K[(size_t)(fa + j) * n + fa + i];
      for (int j = 0; j < na; ++j) for (int i = 0; i < na; ++i)
        K[(size_t)(fa + j) * n + fa + i] = blk[(size_t)j * na + i] + blk[(size_t)i * na + j];
    } else {
      for (int j = 0; j < nb; ++j) for (int i = 0; i < na; ++i)
        K[(size_t)(fb + j) * n + fa + i] += K[(size_t)(fa + i) * n + fb + j];
    }
  }
  for (size_t q = 0; q < (size_t)n * n; ++q) J[q] *= 2.0;
  for (int i = 0; i < n; ++i) for (int j = 0; j < i; ++j) {
    J[(size_t)i * n + j] = J[(size_t)j * n + i];
    K[(size_t)i * n + j] = K[(size_t)j * n + i];
  }
}

// J, K of nd densities Ps[0..nd) (nd = 1: make_r_JK_direct, molecule.fock.foo:1235-1363;
// nd = 2: make_u_JK_direct, molecule.fock.foo:2360-2504, alpha and beta), screened
// with the maxima of Pscreen.  The outer shell-pair loop is restricted to
// ab = ab_offset, ab_offset + ab_stride, ... (one "rank" of Tonto's round-robin
// parallel do); used to time a bounded sample.
static void jk_impl(Ctx* C, const double* Pscreen, int nd, const double* const* Ps, double* const* Js,
                    double* const* Ks, long max_ab_pairs, int n_threads, long ab_stride, long ab_offset) {
  const Basis& B = C->B;
  const int n = B.n_bf;
  const double cutoff = C->schwarz_cutoff;
  using clk = std::chrono::steady_clock;
  const auto t_start = clk::now();
  std::vector<double> Pm;
  max_density(*C, Pscreen, Pm);
  double P_max = 0.0, I_max_all = 0.0;
  for (double v : Pm) P_max = std::max(P_max, v);
  for (double v : C->max_I) I_max_all = std::max(I_max_all, v);
  const double IP_max = I_max_all * P_max;
  long npairs = (long)C->pairs.size();
  long nab = (max_ab_pairs < 0) ? npairs : std::min(npairs, max_ab_pairs);
#ifdef _OPENMP
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#else
  int nt = 1;
#endif
  std::vector<std::vector<double>> Jt(nt * nd, std::vector<double>((size_t)n * n, 0.0));
  std::vector<std::vector<double>> Kt(nt * nd, std::vector<double>((size_t)n * n, 0.0));
  std::vector<std::vector<ClassCount>> cnt(nt, std::vector<ClassCount>(625));
  const auto t_loop0 = clk::now();
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
    int tid = omp_get_thread_num();
#else
    int tid = 0;
#endif
    Work W;
    Side s_ab_skip, s_ab_full, s_cd;
    // round-robin over ab, as Tonto's parallel do (FooToFortran.java:2762-2783); the
    // threads take the bra pairs from the last (most kets, cd <= ab) down, so that the
    // dynamic schedule ends on the cheapest pairs (the sums do not depend on the order
    // beyond rounding)
    const long n_mine = ab_offset < nab ? (nab - 1 - ab_offset) / ab_stride + 1 : 0;
#pragma omp for schedule(dynamic, 1)
    for (long it = 0; it < n_mine; ++it) {
      const long ab = ab_offset + (n_mine - 1 - it) * ab_stride;
      if (C->max_I[ab] * IP_max < cutoff) continue;
      const PairData& pab = C->pairs[ab];
      int aa = pab.a, bb = pab.b;
      int atom_a = B.shell_atom[aa], atom_b = B.shell_atom[bb];
      bool ab_same = atom_a == atom_b;
      if (!ab_same) set_side(B, pab, true, C->pair_cutoff, s_ab_skip);
      set_side(B, pab, false, C->pair_cutoff, s_ab_full);
      for (long cd = 0; cd <= ab; ++cd) {
        if (C->max_I[ab] * C->max_I[cd] * P_max < cutoff) continue;
        const Side* sides[2] = {&s_ab_full, ab_same ? &s_ab_full : &s_ab_skip};
        double* Jl[2] = {Jt[tid * nd].data(), nd > 1 ? Jt[tid * nd + 1].data() : nullptr};
        double* Kl[2] = {Kt[tid * nd].data(), nd > 1 ? Kt[tid * nd + 1].data() : nullptr};
        jk_quartet(C, ab, cd, Pm, sides, s_cd, W, nd, Ps, Jl, Kl, cnt[tid]);
      }
    }
  }
  const auto t_loop1 = clk::now();
  for (int sp = 0; sp < nd; ++sp) {
    double* J = Js[sp];
    double* K = Ks[sp];
    for (size_t q = 0; q < (size_t)n * n; ++q) {
      double sj = 0, sk = 0;
      for (int t = 0; t < nt; ++t) { sj += Jt[t * nd + sp][q]; sk += Kt[t * nd + sp][q]; }
      J[q] = sj; K[q] = sk;
    }
    finish_jk(B, J, K);
  }
  for (int t = 0; t < nt; ++t)
    for (int q = 0; q < 625; ++q) {
      C->counts[q].quartets += cnt[t][q].quartets;
      C->counts[q].prim_quartets += cnt[t][q].prim_quartets;
      for (int k = 0; k < F_NCAT; ++k) C->counts[q].flops[k] += cnt[t][q].flops[k];
    }
  C->t_loop = std::chrono::duration<double>(t_loop1 - t_loop0).count();
  C->t_total = std::chrono::duration<double>(clk::now() - t_start).count();
}

void oracle_jk_sample(OracleCtx* c, const double* P, double* J, double* K, long max_ab_pairs, int n_threads,
                      long ab_stride, long ab_offset) {
  const double* Ps[1] = {P};
  double* Js[1] = {J};
  double* Ks[1] = {K};
  jk_impl(reinterpret_cast<Ctx*>(c), P, 1, Ps, Js, Ks, max_ab_pairs, n_threads, ab_stride, ab_offset);
}

// J, K of an explicit set of shell quartets: quartet i is (bra[i] | ket[i]), Tonto
// pair indices in either order, with make_r_JK_direct's screening, factors,
// digestion and final fold (the same quartet body as jk_impl).  The J, K of
// disjoint quartet sets sum to those of their union, so the shares of a shard plan
// sum to the full build when the plan covers every quartet once.
void oracle_jk_quartets(OracleCtx* c, const double* P, double* J, double* K, long n_quartets, const int* bra,
                        const int* ket, int n_threads) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  const Basis& B = C->B;
  const int n = B.n_bf;
  std::vector<double> Pm;
  max_density(*C, P, Pm);
#ifdef _OPENMP
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#else
  int nt = 1;
#endif
  std::vector<std::vector<double>> Jt(nt, std::vector<double>((size_t)n * n, 0.0));
  std::vector<std::vector<double>> Kt(nt, std::vector<double>((size_t)n * n, 0.0));
  std::vector<std::vector<ClassCount>> cnt(nt, std::vector<ClassCount>(625));
  const double* Ps[1] = {P};
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
    int tid = omp_get_thread_num();
#else
    int tid = 0;
#endif
    Work W;
    Side s_ab_skip, s_ab_full, s_cd;
#pragma omp for schedule(dynamic, 64)
    for (long i = 0; i < n_quartets; ++i) {
      const long ab = bra[i], cd = ket[i];
      const PairData& pab = C->pairs[ab];
      const bool ab_same = B.shell_atom[pab.a] == B.shell_atom[pab.b];
      if (!ab_same) set_side(B, pab, true, C->pair_cutoff, s_ab_skip);
      set_side(B, pab, false, C->pair_cutoff, s_ab_full);
      const Side* sides[2] = {&s_ab_full, ab_same ? &s_ab_full : &s_ab_skip};
      double* Jl[1] = {Jt[tid].data()};
      double* Kl[1] = {Kt[tid].data()};
      jk_quartet(C, ab, cd, Pm, sides, s_cd, W, 1, Ps, Jl, Kl, cnt[tid]);
    }
  }
  for (size_t q = 0; q < (size_t)n * n; ++q) {
    double sj = 0, sk = 0;
    for (int t = 0; t < nt; ++t) { sj += Jt[t][q]; sk += Kt[t][q]; }
    J[q] = sj; K[q] = sk;
  }
  finish_jk(B, J, K);
}

// The error budget of a mixed-precision build: over the quartets that pass
// Tonto's screen and whose bound pm I_max(ab) I_max(cd) is below fp32_cut (the
// quartets a mixed build evaluates in FP32), each J or K element's sum of the
// bounds of the terms it receives: a digestion target element sums
// (number of terms) x factor x bound over those quartets (J(ab): nc nd terms,
// J(cd): na nb, K(ac): nb nd, K(ad): nb nc, K(bc): na nd, K(bd): na nc), then the
// fold and reflection of the build.  Since |(ab|cd) P| <= bound for every term, an
// FP32 evaluation with relative error delta changes an element by at most
// delta x Jb (or Kb).  Returns the number of such quartets.
long oracle_fp32_bound(OracleCtx* c, const double* P, double fp32_cut, double* Jb, double* Kb) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  const Basis& B = C->B;
  const int n = B.n_bf;
  const double cutoff = C->schwarz_cutoff;
  std::vector<double> Pm;
  max_density(*C, P, Pm);
  std::vector<double> J((size_t)n * n, 0.0), K((size_t)n * n, 0.0);
  long n_fp32 = 0;
  const long npairs = (long)C->pairs.size();
  for (long ab = 0; ab < npairs; ++ab) {
    const PairData& pab = C->pairs[ab];
    const int aa = pab.a, bb = pab.b;
    const int fa = B.shell_first_bf[aa], fb = B.shell_first_bf[bb];
    const int na = B.nbf_of(pab.la), nb = B.nbf_of(pab.lb);
    for (long cd = 0; cd <= ab; ++cd) {
      const PairData& pcd = C->pairs[cd];
      const int cc = pcd.a, dd = pcd.b;
      const long ac = pair_index(std::max(aa, cc), std::min(aa, cc)), ad = pair_index(std::max(aa, dd), std::min(aa, dd));
      const long bc = pair_index(std::max(bb, cc), std::min(bb, cc)), bd = pair_index(std::max(bb, dd), std::min(bb, dd));
      const double pm = std::max({Pm[ab], Pm[cd], Pm[ac], Pm[ad], Pm[bc], Pm[bd]});
      if (pm < SKIP_P) continue;
      const double bound = pm * C->max_I[ab] * C->max_I[cd];
      if (!(bound > cutoff) || !(bound < fp32_cut)) continue;
      ++n_fp32;
      double factor = 1.0;
      if (aa == bb) factor = 0.5;
      if (cc == dd) factor *= 0.5;
      if (ab == cd) factor *= 0.5;
      const double fb_ = factor * bound;
      const int fc = B.shell_first_bf[cc], fd = B.shell_first_bf[dd];
      const int nc = B.nbf_of(pcd.la), ndd = B.nbf_of(pcd.lb);
      auto add = [&](std::vector<double>& X, int r0, int nr, int c0, int ncl, double v) {
        for (int j = c0; j < c0 + ncl; ++j)
          for (int i = r0; i < r0 + nr; ++i) X[(size_t)j * n + i] += v;
      };
      add(J, fa, na, fb, nb, fb_ * nc * ndd);      // J(ab)
      add(J, fc, nc, fd, ndd, fb_ * na * nb);      // J(cd)
      add(K, fa, na, fc, nc, fb_ * nb * ndd);      // K(ac)
      add(K, fa, na, fd, ndd, fb_ * nb * nc);      // K(ad)
      add(K, fb, nb, fc, nc, fb_ * na * ndd);      // K(bc)
      add(K, fb, nb, fd, ndd, fb_ * na * nc);      // K(bd)
    }
  }
  // the fold moves contributions between triangles: bound both placements
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) {
      const double sj = J[(size_t)j * n + i] + J[(size_t)i * n + j], sk = K[(size_t)j * n + i] + K[(size_t)i * n + j];
      J[(size_t)j * n + i] = J[(size_t)i * n + j] = sj;
      K[(size_t)j * n + i] = K[(size_t)i * n + j] = sk;
    }
  for (size_t q = 0; q < (size_t)n * n; ++q) { Jb[q] = 4.0 * J[q]; Kb[q] = 2.0 * K[q]; }
  return n_fp32;
}

// make_u_JK_direct (molecule.fock.foo:2360-2504): screening on the maxima of
// Pa + Pb (:2397-2400), then alpha and beta J, K from each ERI.
void oracle_jk_uhf(OracleCtx* c, const double* Pa, const double* Pb, double* Ja, double* Jb, double* Ka, double* Kb,
                   int n_threads) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  const size_t nn = (size_t)C->B.n_bf * C->B.n_bf;
  std::vector<double> PP(nn);
  for (size_t q = 0; q < nn; ++q) PP[q] = Pa[q] + Pb[q];
  const double* Ps[2] = {Pa, Pb};
  double* Js[2] = {Ja, Jb};
  double* Ks[2] = {Ka, Kb};
  jk_impl(C, PP.data(), 2, Ps, Js, Ks, -1, n_threads, 1, 0);
}

// Counters accumulated over oracle_jk calls: out[class*2 + {0,1}] =
// (contracted quartets, primitive quartets) for the 625 (la lb|lc ld) classes.
void oracle_counts(OracleCtx* c, double* out, int reset) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  for (int q = 0; q < 625; ++q) { out[2 * q] = C->counts[q].quartets; out[2 * q + 1] = C->counts[q].prim_quartets; }
  if (reset) C->counts.assign(625, ClassCount());
}

// Counted FLOPs accumulated over oracle_jk calls: out[class * 8 + category] for the
// 625 (la lb|lc ld) classes and the eight categories of FlopCat (set-up, pair terms,
// roots, recurrences, (e0|f0) sums, transfers, spherical transform, digestion).
void oracle_flops(OracleCtx* c, double* out, int reset) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  for (int q = 0; q < 625; ++q)
    for (int k = 0; k < F_NCAT; ++k) out[q * F_NCAT + k] = C->counts[q].flops[k];
  if (reset) C->counts.assign(625, ClassCount());
}

// Wall times (seconds) of the last J/K call: out[0] the shell-quartet loop, out[1]
// the whole call.
void oracle_last_times(OracleCtx* c, double* out) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  out[0] = C->t_loop;
  out[1] = C->t_total;
}

// Cartesian-to-spherical matrix for l (ncart(l) x (2l+1), row-major)
int oracle_spherical_matrix(int l, double* out) {
  build_spherical();
  std::copy(g_sph[l].begin(), g_sph[l].end(), out);
  return (int)g_sph[l].size();
}

// Tonto Cartesian component order for l: 3 ints per component
int oracle_components(int l, int* out) {
  build_components();
  int n = ncart(l);
  for (int i = 0; i < n; ++i) {
    const Comp& cc = g_comp[g_first[l] + i];
    out[3 * i] = cc.x; out[3 * i + 1] = cc.y; out[3 * i + 2] = cc.z;
  }
  return n;
}

void oracle_rys(int n, double x, double* u, double* w) { rys_roots(n, x, u, w); }

}  // extern "C"

// ===========================================================================
// One-electron integrals (overlap, kinetic, nuclear attraction) for the SCF
// checker.  Cartesian x^l-normalised components as the two-electron part; the
// spherical transform uses the same matrices.
// ===========================================================================
namespace {

// 1-D overlap table s[i][j], i<=imax, j<=jmax, with PA, PB, 1/(2 zeta)
void overlap_1d(int imax, int jmax, double PA, double PB, double oo2z, double* s, int ld) {
  s[0] = 1.0;
  for (int i = 0; i <= imax; ++i) {
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      double v;
      if (i > 0) {
        v = PA * s[(i - 1) * ld + j];
        if (i > 1) v += (i - 1) * oo2z * s[(i - 2) * ld + j];
        if (j > 0) v += j * oo2z * s[(i - 1) * ld + j - 1];
      } else {
        v = PB * s[i * ld + j - 1];
        if (j > 1) v += (j - 1) * oo2z * s[i * ld + j - 2];
      }
      s[i * ld + j] = v;
    }
  }
}

}  // namespace

extern "C" {

// S, T, V (column-major n_bf x n_bf in the Tonto basis order).  Z: nuclear charges.
void oracle_one_electron(OracleCtx* c, const double* Z, double* S, double* T, double* V) {
  Ctx* C = reinterpret_cast<Ctx*>(c);
  const Basis& B = C->B;
  const int n = B.n_bf;
  std::fill(S, S + (size_t)n * n, 0.0);
  std::fill(T, T + (size_t)n * n, 0.0);
  std::fill(V, V + (size_t)n * n, 0.0);
  for (int sa = 0; sa < B.n_shell; ++sa) for (int sb = 0; sb <= sa; ++sb) {
    int la = B.shell_l[sa], lb = B.shell_l[sb];
    int nca = ncart(la), ncb = ncart(lb);
    const double* A = B.xyz + 3 * B.shell_atom[sa];
    const double* Bp = B.xyz + 3 * B.shell_atom[sb];
    double AB[3] = {A[0] - Bp[0], A[1] - Bp[1], A[2] - Bp[2]};
    double r2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    std::vector<double> s_c((size_t)nca * ncb, 0.0), t_c((size_t)nca * ncb, 0.0), v_c((size_t)nca * ncb, 0.0);
    const int ld = lb + 3;
    std::vector<double> sx((la + 2) * ld), sy((la + 2) * ld), sz((la + 2) * ld);
    int nroot = (la + lb) / 2 + 1;
    std::vector<double> ru(nroot), rw(nroot);
    for (int ia = 0; ia < B.shell_nprim[sa]; ++ia) for (int ib = 0; ib < B.shell_nprim[sb]; ++ib) {
      double a = B.exps[B.prim_off[sa] + ia], ca = B.coefs[B.prim_off[sa] + ia];
      double b = B.exps[B.prim_off[sb] + ib], cb = B.coefs[B.prim_off[sb] + ib];
      double z = a + b, oo2z = 0.5 / z;
      double Kab = std::exp(-a * b * r2 / z) * ca * cb;
      double P[3], PA[3], PB[3];
      for (int k = 0; k < 3; ++k) { P[k] = (a * A[k] + b * Bp[k]) / z; PA[k] = P[k] - A[k]; PB[k] = P[k] - Bp[k]; }
      overlap_1d(la + 1, lb + 2, PA[0], PB[0], oo2z, sx.data(), ld);
      overlap_1d(la + 1, lb + 2, PA[1], PB[1], oo2z, sy.data(), ld);
      overlap_1d(la + 1, lb + 2, PA[2], PB[2], oo2z, sz.data(), ld);
      double pre = Kab * std::pow(PI / z, 1.5);
      for (int i = 0; i < nca; ++i) {
        const Comp& ci = g_comp[g_first[la] + i];
        for (int j = 0; j < ncb; ++j) {
          const Comp& cj = g_comp[g_first[lb] + j];
          double Sx = sx[ci.x * ld + cj.x], Sy = sy[ci.y * ld + cj.y], Sz = sz[ci.z * ld + cj.z];
          auto kin = [&](const double* s1, int i1, int j1) {
            double v = -2.0 * b * b * s1[i1 * ld + j1 + 2] + b * (2 * j1 + 1) * s1[i1 * ld + j1];
            if (j1 >= 2) v += -0.5 * j1 * (j1 - 1) * s1[i1 * ld + j1 - 2];
            return v;
          };
          double Tx = kin(sx.data(), ci.x, cj.x), Ty = kin(sy.data(), ci.y, cj.y), Tz = kin(sz.data(), ci.z, cj.z);
          s_c[(size_t)j * nca + i] += pre * Sx * Sy * Sz;
          t_c[(size_t)j * nca + i] += pre * (Tx * Sy * Sz + Sx * Ty * Sz + Sx * Sy * Tz);
        }
      }
      // nuclear attraction by Rys quadrature: (a|1/r_C|b) = 2 pi / z * K * sum_i w_i Ix Iy Iz
      for (int iat = 0; iat < B.n_atom; ++iat) {
        const double* Cc = B.xyz + 3 * iat;
        double PC[3] = {P[0] - Cc[0], P[1] - Cc[1], P[2] - Cc[2]};
        double x = z * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        rys_roots(nroot, x, ru.data(), rw.data());
        double pv = -Z[iat] * 2.0 * PI / z * Kab;
        for (int r = 0; r < nroot; ++r) {
          double u = ru[r];
          // 1-D: I(i,0) recurrence then HRR to j
          double tab[3][8][8];
          for (int dir = 0; dir < 3; ++dir) {
            double c0 = PA[dir] - u * PC[dir];
            double bb = (1.0 - u) * oo2z;
            double g[16];
            g[0] = 1.0;
            int L = la + lb;
            if (L >= 1) g[1] = c0;
            for (int e = 1; e < L; ++e) g[e + 1] = c0 * g[e] + e * bb * g[e - 1];
            // HRR: I(i,j+1) = I(i+1,j) + AB I(i,j)
            double h[16][8];
            for (int e = 0; e <= L; ++e) h[e][0] = g[e];
            for (int j = 1; j <= lb; ++j)
              for (int e = 0; e <= L - j; ++e) h[e][j] = h[e + 1][j - 1] + AB[dir] * h[e][j - 1];
            for (int i2 = 0; i2 <= la; ++i2) for (int j = 0; j <= lb; ++j) tab[dir][i2][j] = h[i2][j];
          }
          double wv = pv * rw[r];
          for (int i = 0; i < nca; ++i) {
            const Comp& ci = g_comp[g_first[la] + i];
            for (int j = 0; j < ncb; ++j) {
              const Comp& cj = g_comp[g_first[lb] + j];
              v_c[(size_t)j * nca + i] += wv * tab[0][ci.x][cj.x] * tab[1][ci.y][cj.y] * tab[2][ci.z][cj.z];
            }
          }
        }
      }
    }
    // to the Tonto basis (spherical for l >= 2)
    int nfa = B.nbf_of(la), nfb = B.nbf_of(lb);
    auto transform = [&](const std::vector<double>& X, std::vector<double>& Y) {
      std::vector<double> tmp((size_t)nfa * ncb, 0.0);
      if (B.spherical && la >= 2) {
        for (int j = 0; j < ncb; ++j) for (int m = 0; m < nfa; ++m) {
          double s = 0; for (int i = 0; i < nca; ++i) s += g_sph[la][i * nfa + m] * X[(size_t)j * nca + i];
          tmp[(size_t)j * nfa + m] = s;
        }
      } else tmp = X;
      Y.assign((size_t)nfa * nfb, 0.0);
      if (B.spherical && lb >= 2) {
        for (int m2 = 0; m2 < nfb; ++m2) for (int m = 0; m < nfa; ++m) {
          double s = 0; for (int j = 0; j < ncb; ++j) s += g_sph[lb][j * nfb + m2] * tmp[(size_t)j * nfa + m];
          Y[(size_t)m2 * nfa + m] = s;
        }
      } else Y = tmp;
    };
    std::vector<double> So, To, Vo;
    transform(s_c, So); transform(t_c, To); transform(v_c, Vo);
    int fa = B.shell_first_bf[sa], fb = B.shell_first_bf[sb];
    for (int j = 0; j < nfb; ++j) for (int i = 0; i < nfa; ++i) {
      size_t p = (size_t)(fb + j) * n + fa + i, q = (size_t)(fa + i) * n + fb + j;
      S[p] = S[q] = So[(size_t)j * nfa + i];
      T[p] = T[q] = To[(size_t)j * nfa + i];
      V[p] = V[q] = Vo[(size_t)j * nfa + i];
    }
  }
}

}  // extern "C"
