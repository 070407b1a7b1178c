// tf_device.cuh — device-side building blocks of the B200 Rys J/K builder.
//
// Everything that depends on angular momentum is resolved at compile time:
// Cartesian component tables (Tonto's lexical order, gaussian_data.foo:295-479)
// are constexpr, loops over components are unrolled with static_for, and the
// integral arrays therefore live in registers.  One thread computes one
// contracted shell quartet:
//   primitive quartets -> Rys nodes/weights (piecewise tables, FP64)
//   -> 2D recurrences on the higher-l centre of each pair (make_esfs_XX,
//      shell1quartet.foo:7418-7609) -> (e0|f0) accumulation (form_esfs :7615)
//   -> horizontal transfer ket then bra (transfer_cd / transfer_ab :8310-11134)
//   -> digestion into J and K with Tonto's coincidence factors
//      (molecule.fock.foo:1296-1338).
// The spherical transform of make_ERI (:433-563) is not applied per quartet:
// the density is taken to the Cartesian basis once per build and J, K are taken
// back once (the transforms commute with the contraction).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>
#include <type_traits>

#define TF_RYS_CONST __device__ const
// the asymptotic-rule tables in the constant bank: read at compile-time indices,
// they become immediate operands instead of global loads
#define TF_RYS_SMALL_CONST __constant__ const
#include "rys_tables.inc"
#include "boys_table.inc"
#include "boys2_table.inc"

namespace tf {

// ---------------------------------------------------------------------------
// Reciprocal and reciprocal square root by Newton-Raphson iteration, seeded by
// the PTX approximate instructions rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64
// (about 20 correct bits).  Each step squares the relative error:
//   1/x:       y <- y + y (1 - x y)
//   1/sqrt(x): y <- y + y (1/2 - (x/2) y^2)
// so two steps reach the double-precision rounding level (a few ulp; checked
// against IEEE division and square root by tests/fast_math_check.cu).  Used for
// the exponent sums, rho, the Boys-function ratio and 1/x of the asymptotic
// rules: positive normal numbers far from the overflow range.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double h = 0.5 * x;
  double e = fma(-h * y, y, 0.5);
  y = fma(y, e, y);
  e = fma(-h * y, y, 0.5);
  return fma(y, e, y);
}

// ---------------------------------------------------------------------------
// Fock accumulation.  FX = false: an FP64 atomic add.  Deterministic builds
// (FX = true, a kernel instantiation of its own so that the default kernels carry
// none of this code): the contribution v is split into two 64-bit fixed-point words,
// hi = round(v 2^32) and lo = round((v - hi 2^-32) 2^60), added with integer
// atomics to the element's hi word (the accumulator itself, read as an integer)
// and to its lo word, fx_lo elements further on.  v - hi 2^-32 is exact (the two
// are within a factor of two of each other, or hi = 0), so each contribution is
// kept to 2^-61; integer sums are exact and wrap modulo 2^64, so the totals do
// not depend on the order of the additions, and k_finalize reads them as
// hi 2^-32 + lo 2^-60.  Contributions and totals below 2^31 in magnitude.
// ---------------------------------------------------------------------------
template <bool FX>
__device__ __forceinline__ void fock_add(double* addr, double v, long long fx_lo) {
  if constexpr (!FX) {
    atomicAdd(addr, v);
  } else {
    const double h = rint(v * 0x1p32);
    const long long hi = (long long)h;
    const long long lo = __double2ll_rn((v - h * 0x1p-32) * 0x1p60);
    atomicAdd(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)hi);
    atomicAdd(reinterpret_cast<unsigned long long*>(addr + fx_lo), (unsigned long long)lo);
  }
}

// The value of a Fock accumulator element (see fock_add).
__device__ __forceinline__ double fock_value(const double* m, size_t i, long long fx_lo) {
  if (fx_lo == 0) return m[i];
  const long long* q = reinterpret_cast<const long long*>(m);
  return (double)q[i] * 0x1p-32 + (double)q[i + fx_lo] * 0x1p-60;
}

// ---------------------------------------------------------------------------
// compile-time helpers
// ---------------------------------------------------------------------------
template <int... Is, class F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, F&& f) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int ncart_upto(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }

constexpr int LCOMP = 8;                         // components tabulated up to l = 8
constexpr int NCOMP_ALL = ncart_upto(LCOMP);     // 165

struct CompTable {
  int x[NCOMP_ALL], y[NCOMP_ALL], z[NCOMP_ALL];
  int first[LCOMP + 2];
  int idx[LCOMP + 1][LCOMP + 1][LCOMP + 1];      // position within its own l
};

__host__ __device__ constexpr void comp_push(CompTable& t, int& i, int X, int Y, int Z) {
  t.x[i] = X; t.y[i] = Y; t.z[i] = Z; ++i;
}

// Tonto's lexical Cartesian order: for L, the highest power a descends, then the
// second b, each pattern expanded in a fixed permutation order.
__host__ __device__ constexpr CompTable make_comp_table() {
  CompTable t{};
  int i = 0;
  for (int L = 0; L <= LCOMP; ++L) {
    t.first[L] = i;
    for (int a = L; a >= (L + 2) / 3; --a) {
      for (int b = (L - a < a ? L - a : a); b >= (L - a + 1) / 2; --b) {
        int c = L - a - b;
        if (a == b && b == c) {
          comp_push(t, i, a, a, a);
        } else if (a > b && b == c) {
          comp_push(t, i, a, b, b); comp_push(t, i, b, a, b); comp_push(t, i, b, b, a);
        } else if (a == b && b > c) {
          comp_push(t, i, a, a, c); comp_push(t, i, a, c, a); comp_push(t, i, c, a, a);
        } else {
          comp_push(t, i, a, b, c); comp_push(t, i, a, c, b); comp_push(t, i, b, a, c);
          comp_push(t, i, c, a, b); comp_push(t, i, b, c, a); comp_push(t, i, c, b, a);
        }
      }
    }
  }
  t.first[LCOMP + 1] = i;
  for (int k = 0; k < NCOMP_ALL; ++k) {
    int L = t.x[k] + t.y[k] + t.z[k];
    t.idx[t.x[k]][t.y[k]][t.z[k]] = k - t.first[L];
  }
  return t;
}

constexpr CompTable CT = make_comp_table();
static_assert(CT.first[LCOMP + 1] == NCOMP_ALL, "component table size");

__host__ __device__ constexpr int cx(int l, int i) { return CT.x[CT.first[l] + i]; }
__host__ __device__ constexpr int cy(int l, int i) { return CT.y[CT.first[l] + i]; }
__host__ __device__ constexpr int cz(int l, int i) { return CT.z[CT.first[l] + i]; }
// global lexical index -> powers
__host__ __device__ constexpr int gx(int g) { return CT.x[g]; }
__host__ __device__ constexpr int gy(int g) { return CT.y[g]; }
__host__ __device__ constexpr int gz(int g) { return CT.z[g]; }
__host__ __device__ constexpr int gidx(int x, int y, int z) { return CT.first[x + y + z] + CT.idx[x][y][z]; }

// ---------------------------------------------------------------------------
// data layouts shared with the host code
// ---------------------------------------------------------------------------
// One primitive pair (Gaussian product), positioned.  cc holds
// c_a c_b zeta^(-1) exp(-a b |AB|^2 / zeta): the prefactor c_a c_b zeta^(-3/2) exp(...)
// times sqrt(zeta), so that a primitive quartet's
// 2 pi^(5/2) cc_ab zeta^(-3/2) cc_cd eta^(-3/2) sqrt(rho), rho = zeta eta / (zeta + eta),
// becomes 2 pi^(5/2) cc_ab cc_cd / sqrt(zeta + eta): one reciprocal square root of
// zeta + eta gives both it and 1/(zeta + eta) (its square).
struct __align__(16) PrimPair {
  double Px, Py, Pz, zeta;
  double cc, half_zinv;              // prefactor, 1/(2 zeta)
  double PAx, PAy, PAz, pad;         // P - (centre of the higher-l shell)
};

// One shell pair, oriented so that shell "hi" has the higher l (ties: the
// shell with the larger index, as Tonto's pair (a >= b) orientation).
struct __align__(16) PairRec {
  int sh_hi, sh_lo;          // shell indices (Tonto order)
  int atom_hi, atom_lo;
  int cart_hi, cart_lo;      // first Cartesian function of each shell
  int full_off, n_full;      // primitive pairs without the pair cutoff
  int skip_off, n_skip;      // primitive pairs with the pair cutoff (atoms differ)
  int mol, tonto_ab;         // molecule (batched contexts), Tonto pair index a(a+1)/2+b within it
  double Rx, Ry, Rz;         // hi centre - lo centre
  double imax;               // Schwarz bound sqrt(max |(ab|ab)|)
};

// What the ERI kernels read of a shell pair, packed: rec[2 id] = {cart_hi, cart_lo,
// full_off, skip_off}, rec[2 id + 1] = {atom_hi, atom_lo, n_full | n_skip << 16,
// mol | (shell hi == shell lo) << 31} (32 bytes, one sector), and pairR[id] = (A - B, 0)
// read only by classes whose transfers need it.
struct PairJK {
  int cart_hi, cart_lo, full_off, skip_off;
  int atom_hi, atom_lo, n_full, n_skip, mol;
  bool same;                 // both shells the same (coincidence factor 1/2)
  double Rx, Ry, Rz;
};

__device__ __forceinline__ PairJK load_pair_jk(const int4* __restrict__ rec, const double2* __restrict__ pairR,
                                               int id) {
  const int4 x = __ldg(rec + 2 * id), y = __ldg(rec + 2 * id + 1);
  PairJK p;
  p.cart_hi = x.x; p.cart_lo = x.y; p.full_off = x.z; p.skip_off = x.w;
  p.atom_hi = y.x; p.atom_lo = y.y;
  p.n_full = y.z & 0xffff; p.n_skip = (int)((unsigned)y.z >> 16);
  p.mol = y.w & 0x7fffffff; p.same = y.w < 0;
  const double2 r0 = __ldg(pairR + 2 * id), r1 = __ldg(pairR + 2 * id + 1);
  p.Rx = r0.x; p.Ry = r0.y; p.Rz = r1.x;
  return p;
}

// Quartet range of a launch in a graph-captured build: list[range[0] - base,
// range[1] - base), read on the device and clamped to the list capacity.
__device__ __forceinline__ void resolve_range(const long long* range, long long base, long long cap,
                                              const int2*& q, long long& n) {
  if (range) {
    const long long s0 = range[0], s1 = min(range[1], base + cap);
    q += s0 - base;
    n = s1 > s0 ? s1 - s0 : 0;
  }
}

// One molecule of a (possibly batched) context: its shells are a contiguous
// global range; its matrices sit at fixed offsets in the concatenated buffers.
struct __align__(16) MolInfo {
  int shell0, n_shell;       // global shell range
  int cart0, bf0;            // first global Cartesian / basis function
  int n_cart, n_bf;
  int atom0, n_atom;         // global atom range
  long long cmat;            // offset of its n_cart x n_cart Cartesian block
  long long bmat;            // offset of its n_bf x n_bf Tonto-basis block
  long long pmax;            // offset of its n_shell x n_shell pair-maximum block
};

// molecule owning element t of a concatenated buffer with offsets off[0..n_mol]
__device__ __forceinline__ int find_mol(const long long* __restrict__ off, int n_mol, long long t) {
  int lo = 0, hi = n_mol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

constexpr double TWOPI5ON2 = 34.9868366552497256925;   // 2 pi^(5/2)

// ---------------------------------------------------------------------------
// Rys nodes and weights (FP64 always)
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int rys_xmax(int n) { const int t[] = TF_RYS_XMAX_INIT; return t[n]; }
__host__ __device__ constexpr int rys_offset(int n) { const int t[] = TF_RYS_OFFSET_INIT; return t[n]; }
__host__ __device__ constexpr int rys_hoffset(int n) { const int t[] = TF_RYS_HOFFSET_INIT; return t[n]; }

template <int N>
__device__ __forceinline__ void rys_eval(double x, double (&u)[N], double (&w)[N]) {
  constexpr int XMAX = rys_xmax(N), OFF = rys_offset(N), HOFF = rys_hoffset(N);
  if (x < (double)XMAX) {
    const int j = (int)x;
    const double s = x - (double)j;
    const double* c = tf_rys_coef + OFF + j * (2 * N * TF_RYS_NCOEF);
#pragma unroll
    for (int f = 0; f < 2 * N; ++f) {
      const double* cf = c + f * TF_RYS_NCOEF;
      double v = __ldg(cf + TF_RYS_DEG);
#pragma unroll
      for (int k = TF_RYS_DEG - 1; k >= 0; --k) v = fma(v, s, __ldg(cf + k));
      if (f < N) u[f] = v; else w[f - N] = v;
    }
  } else {
    const double ix = rcp_nr(x);
    const double isx = rsqrt_nr(x);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      u[i] = tf_rys_hroot2[HOFF + i] * ix;
      w[i] = tf_rys_hweight[HOFF + i] * isx;
    }
  }
}

// The same tables staged in shared memory, transposed to [coef][function][interval]
// so that lanes evaluating different intervals hit different banks.
template <int N>
struct RysSmem {
  static constexpr int NI = rys_xmax(N);              // intervals
  static constexpr int SIZE = TF_RYS_NCOEF * 2 * N * NI;
  // layout [k][j][i] with the pairs (u_i, w_i) adjacent: one 16-byte load per
  // (coefficient, root)
  static __device__ __forceinline__ void load(double* t) {
    constexpr int OFF = rys_offset(N);
    for (int q = threadIdx.x; q < SIZE; q += blockDim.x) {
      // q = ((k * NI + j) * N + i) * 2 + (0: node, 1: weight)
      const int uw = q & 1, i = (q >> 1) % N, kj = (q >> 1) / N, j = kj % NI, k = kj / NI;
      const int f = uw ? N + i : i;
      t[q] = tf_rys_coef[OFF + j * (2 * N * TF_RYS_NCOEF) + f * TF_RYS_NCOEF + k];
    }
  }
  static __device__ __forceinline__ void eval(const double* __restrict__ t, double x, double (&u)[N], double (&w)[N]) {
    if (x < (double)NI) {
      const int j = (int)x;
      const double s = x - (double)j;
      const double2* c = reinterpret_cast<const double2*>(t) + j * N;
      constexpr int KS = NI * N;                     // stride between coefficients (double2)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const double2 v = c[TF_RYS_DEG * KS + i];
        u[i] = v.x;
        w[i] = v.y;
      }
#pragma unroll
      for (int k = TF_RYS_DEG - 1; k >= 0; --k)
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const double2 v = c[k * KS + i];
          u[i] = fma(u[i], s, v.x);
          w[i] = fma(w[i], s, v.y);
        }
    } else {
      constexpr int HOFF = rys_hoffset(N);
      const double ix = rcp_nr(x);
      const double isx = rsqrt_nr(x);
#pragma unroll
      for (int i = 0; i < N; ++i) {
        u[i] = tf_rys_hroot2[HOFF + i] * ix;
        w[i] = tf_rys_hweight[HOFF + i] * isx;
      }
    }
  }
};

// One root: the rule is exact for f linear in t^2, so w = F0(x) and u = F1(x)/F0(x).
// F0 and F1 come from an 8-term Taylor step about the nearest point k/8 of a grid
// of F_0..F_8 (gen_boys_table.py; dF_m/dx = -F_{m+1}): five 16-byte table loads
// per evaluation instead of one per polynomial coefficient.
template <>
struct RysSmem<1> {
  static constexpr int SIZE = TF_BOYS_NPTS * TF_BOYS_NM;
  static __device__ __forceinline__ void load(double* t) {
    for (int q = threadIdx.x; q < SIZE; q += blockDim.x) t[q] = tf_boys_grid[q];
  }
  static __device__ __forceinline__ void eval(const double* __restrict__ t, double x, double (&u)[1], double (&w)[1]) {
    static_assert(TF_BOYS_NTERM == 8 && TF_BOYS_NM == 10, "Taylor step written for 8 terms");
    if (x < (double)TF_BOYS_XMAX) {
      const int k = (int)(x * (double)TF_BOYS_H_INV + 0.5);
      const double d = (double)k * (1.0 / TF_BOYS_H_INV) - x;
      const double2* g = reinterpret_cast<const double2*>(t + k * TF_BOYS_NM);
      const double2 f01 = g[0], f23 = g[1], f45 = g[2], f67 = g[3], f89 = g[4];
      const double d2 = d * 0.5, d3 = d * (1.0 / 3.0), d4 = d * 0.25, d5 = d * 0.2, d6 = d * (1.0 / 6.0),
                   d7 = d * (1.0 / 7.0);
      double a = fma(d7, f67.y, f67.x);      // F0 = f0 + d (f1 + d/2 (f2 + ... + d/7 f7))
      double b = fma(d7, f89.x, f67.y);      // F1 = f1 + d (f2 + d/2 (f3 + ... + d/7 f8))
      a = fma(d6, a, f45.y);
      b = fma(d6, b, f67.x);
      a = fma(d5, a, f45.x);
      b = fma(d5, b, f45.y);
      a = fma(d4, a, f23.y);
      b = fma(d4, b, f45.x);
      a = fma(d3, a, f23.x);
      b = fma(d3, b, f23.y);
      a = fma(d2, a, f01.y);
      b = fma(d2, b, f23.x);
      a = fma(d, a, f01.x);
      b = fma(d, b, f01.y);
      w[0] = a;
      u[0] = b * rcp_nr(a);
    } else {
      constexpr int HOFF = rys_hoffset(1);
      u[0] = tf_rys_hroot2[HOFF] * rcp_nr(x);
      w[0] = tf_rys_hweight[HOFF] * rsqrt_nr(x);
    }
  }
};

#ifndef TF_RYS2_MOMENTS
#define TF_RYS2_MOMENTS 1
#endif
#if TF_RYS2_MOMENTS
// Two roots: the Gauss rule of the moments F_0..F_3 (gen_boys_table.py): u_1, u_2
// are the roots of u^2 + a u + b, the monic polynomial orthogonal to 1 and u,
//   a = (F0 F3 - F1 F2) / (F1^2 - F0 F2),  b = (F2^2 - F1 F3) / (F1^2 - F0 F2),
// taken as q = (sqrt(a^2 - 4b) - a) / 2 (a < 0: no cancellation), u_1 = q,
// u_2 = b / q; w_1 = (F0 u_2 - F1) / (u_2 - u_1), w_2 = F0 - w_1.  F0..F3 by the
// 8-term Taylor step from a 1/8 grid of F_0..F_10: six 16-byte loads instead of 24.
template <>
struct RysSmem<2> {
  static constexpr int SIZE = TF_BOYS2_NPTS * TF_BOYS2_NM;
  static __device__ __forceinline__ void load(double* t) {
    for (int q = threadIdx.x; q < SIZE; q += blockDim.x) t[q] = tf_boys2_grid[q];
  }
  static __device__ __forceinline__ void eval(const double* __restrict__ t, double x, double (&u)[2], double (&w)[2]) {
    static_assert(TF_BOYS_NTERM == 8 && TF_BOYS2_NM == 12 && TF_BOYS2_XMAX == 50, "grid for the two-point rule");
    if (x < (double)TF_BOYS2_XMAX) {
      const int k = (int)(x * (double)TF_BOYS_H_INV + 0.5);
      const double d = (double)k * (1.0 / TF_BOYS_H_INV) - x;
      const double2* g = reinterpret_cast<const double2*>(t + k * TF_BOYS2_NM);
      double f[12];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const double2 v = g[q];
        f[2 * q] = v.x;
        f[2 * q + 1] = v.y;
      }
      const double dj[8] = {0.0, d, d * 0.5, d * (1.0 / 3.0), d * 0.25, d * 0.2, d * (1.0 / 6.0), d * (1.0 / 7.0)};
      double m[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {              // F_r = f_r + d (f_{r+1} + d/2 (... + d/7 f_{r+7}))
        double v = f[r + 7];
#pragma unroll
        for (int j = 7; j >= 1; --j) v = fma(dj[j], v, f[r + j - 1]);
        m[r] = v;
      }
      const double r = rcp_nr(m[1] * m[1] - m[0] * m[2]);
      const double a = (m[0] * m[3] - m[1] * m[2]) * r;
      const double b = (m[2] * m[2] - m[1] * m[3]) * r;
      const double disc = fma(a, a, -4.0 * b);
      const double q = 0.5 * (disc * rsqrt_nr(disc) - a);
      u[0] = q;
      u[1] = b * rcp_nr(q);
      const double w0 = (m[0] * u[1] - m[1]) * rcp_nr(u[1] - u[0]);
      w[0] = w0;
      w[1] = m[0] - w0;
    } else {
      constexpr int HOFF = rys_hoffset(2);
      const double ix = rcp_nr(x);
      const double isx = rsqrt_nr(x);
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        u[i] = tf_rys_hroot2[HOFF + i] * ix;
        w[i] = tf_rys_hweight[HOFF + i] * isx;
      }
    }
  }
};
#endif

// ---------------------------------------------------------------------------
// One contracted shell quartet (LA LB | LC LD), LA >= LB, LC >= LD, in
// arithmetic type T for the 2D recurrences and (e0|f0) sums (double, or float
// for the mixed-precision path); nodes/weights and the final integrals FP64.
// ---------------------------------------------------------------------------
template <int LA, int LB, int LC, int LD>
struct Quartet {
  static constexpr int LAB = LA + LB, LCD = LC + LD;
  static constexpr int NROOT = (LAB + LCD) / 2 + 1;
  static constexpr int FE = CT.first[LA], NE = CT.first[LAB + 1] - CT.first[LA];   // e: l in [LA, LA+LB]
  static constexpr int FF = CT.first[LC], NF = CT.first[LCD + 1] - CT.first[LC];
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NINT = NA * NB * NC * ND;
};

// read-only loads of a primitive-pair record: half 0 = (Px, Py, Pz, zeta),
// half 1 = (PAx, PAy, PAz, 1/(2 zeta))
__device__ __forceinline__ double4 ld4(const PrimPair* p, int half) {
  const double2* q = reinterpret_cast<const double2*>(p);
  if (half == 0) {
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
  }
  const double2 c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4);
  return make_double4(d.x, d.y, e.x, c.y);
}

// (e0|f0) accumulation over all primitive quartets of a contracted quartet.
#ifndef TF_PRIM_UNROLL
#define TF_PRIM_UNROLL 1
#endif

constexpr int kPrimUnroll = TF_PRIM_UNROLL;
constexpr int PPS = sizeof(PrimPair) / sizeof(double2);         // 5 16-byte loads per record

// The loaded part of a primitive-pair record: (Px, Py), (Pz, zeta), (cc, 1/(2 zeta)),
// and (PAx, PAy), (PAz, -) only where the recurrences need P - A.
struct PrimRegs {
  double2 P, Z, C, A0, A1;
};

template <bool NEED_PA>
__device__ __forceinline__ PrimRegs load_prim(const double2* __restrict__ q, int i) {
  PrimRegs r;
  r.P = __ldg(q + i * PPS);
  r.Z = __ldg(q + i * PPS + 1);
  r.C = __ldg(q + i * PPS + 2);
  if constexpr (NEED_PA) {
    r.A0 = __ldg(q + i * PPS + 3);
    r.A1 = __ldg(q + i * PPS + 4);
  } else {
    r.A0 = r.A1 = make_double2(0.0, 0.0);
  }
  return r;
}

// 1/x and 1/sqrt(x) in FP32 (the PTX approximate instructions, about 23 correct
// bits: the rounding level of the FP32 arithmetic they feed).
__device__ __forceinline__ float rcp_f32(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_f32(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// One primitive quartet in the mixed-precision path: the Boys-function argument
// and everything after the Rys nodes and weights in FP32 (exponent sums, rho, the
// prefactor, the recurrence coefficients, the 2D recurrences and the (e0|f0)
// products); P - Q in FP64 (a difference of positions), then the nodes and weights
// themselves in FP64 from the FP64 tables, as for the FP64 path.
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void prim_quartet_f32(const PrimRegs& B, const PrimRegs& K, double wmask,
                                                 float (&esfs)[Quartet<LA, LB, LC, LD>::NE][Quartet<LA, LB, LC, LD>::NF],
                                                 const double* __restrict__ rys_smem) {
  using Q = Quartet<LA, LB, LC, LD>;
  constexpr int D1 = Q::LAB + 1, D2 = Q::LCD + 1, NR = Q::NROOT;
  const float zeta = (float)B.Z.y, eta = (float)K.Z.y;
  const float half_zinv = (float)B.C.y, half_einv = (float)K.C.y;
  const float sq = rsqrt_f32(zeta + eta);
  const float inv = sq * sq;
  const float rho = zeta * eta * inv;
  const float QP[3] = {(float)(K.P.x - B.P.x), (float)(K.P.y - B.P.y), (float)(K.Z.x - B.Z.x)};
  const float xx = rho * (QP[0] * QP[0] + QP[1] * QP[1] + QP[2] * QP[2]);
  double u[NR], w[NR];
  if (rys_smem) RysSmem<NR>::eval(rys_smem, (double)xx, u, w);
  else rys_eval<NR>((double)xx, u, w);
  const float scale = (float)(B.C.x * K.C.x * (TWOPI5ON2 * wmask)) * sq;
  const float r_z = eta * inv;     // rho / zeta
  const float r_e = zeta * inv;    // rho / eta
  const float PA[3] = {(float)B.A0.x, (float)B.A0.y, (float)B.A1.x};
  const float QC[3] = {(float)K.A0.x, (float)K.A0.y, (float)K.A1.x};
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const float t2 = (float)u[r];
    const float t2_rz = t2 * r_z, t2_re = t2 * r_e;
    const float B10 = (1.0f - t2_rz) * half_zinv;
    const float B01 = (1.0f - t2_re) * half_einv;
    const float B00 = 0.5f * t2 * inv;
    const float wt = (float)w[r] * scale;
    float I[3][D1][D2];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float c00 = fmaf(t2_rz, QP[d], PA[d]);
      const float d00 = fmaf(-t2_re, QP[d], QC[d]);
      I[d][0][0] = (d == 2) ? wt : 1.0f;
      if (D1 > 1) I[d][1][0] = c00 * I[d][0][0];
#pragma unroll
      for (int e = 1; e + 1 < D1; ++e) I[d][e + 1][0] = c00 * I[d][e][0] + float(e) * B10 * I[d][e - 1][0];
#pragma unroll
      for (int f = 0; f + 1 < D2; ++f) {
#pragma unroll
        for (int e = 0; e < D1; ++e) {
          float v = d00 * I[d][e][f];
          if (f > 0) v += float(f) * B01 * I[d][e][f - 1];
          if (e > 0) v += float(e) * B00 * I[d][e - 1][f];
          I[d][e][f + 1] = v;
        }
      }
    }
    static_for<Q::NE>([&](auto e) {
      constexpr int ge = Q::FE + decltype(e)::value;
      static_for<Q::NF>([&](auto f) {
        constexpr int gf = Q::FF + decltype(f)::value;
        esfs[decltype(e)::value][decltype(f)::value] +=
            I[0][gx(ge)][gx(gf)] * I[1][gy(ge)][gy(gf)] * I[2][gz(ge)][gz(gf)];
      });
    });
  }
}

// One primitive quartet: Rys nodes and weights, the 2D recurrences and the
// (e0|f0) products, added to esfs with weight `wmask`.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void prim_quartet(const PrimRegs& B, const PrimRegs& K, double wmask,
                                             T (&esfs)[Quartet<LA, LB, LC, LD>::NE][Quartet<LA, LB, LC, LD>::NF],
                                             const double* __restrict__ rys_smem) {
  if constexpr (std::is_same<T, float>::value) {
    prim_quartet_f32<LA, LB, LC, LD>(B, K, wmask, esfs, rys_smem);
    return;
  }
  using Q = Quartet<LA, LB, LC, LD>;
  constexpr int D1 = Q::LAB + 1, D2 = Q::LCD + 1, NR = Q::NROOT;
  const double bcc = B.C.x * TWOPI5ON2, kcc = K.C.x;
  const double zeta = B.Z.y, half_zinv = B.C.y;
  const double eta = K.Z.y, half_einv = K.C.y;
  const double sq = rsqrt_nr(zeta + eta);     // 1/sqrt(zeta + eta)
  const double inv = sq * sq;
  const double rho = zeta * eta * inv;
  const double QPx = K.P.x - B.P.x, QPy = K.P.y - B.P.y, QPz = K.Z.x - B.Z.x;
  const double xx = rho * (QPx * QPx + QPy * QPy + QPz * QPz);
  double u[NR], w[NR];
  if (rys_smem) RysSmem<NR>::eval(rys_smem, xx, u, w);
  else rys_eval<NR>(xx, u, w);
  const double scale = bcc * kcc * sq * wmask;
  const double r_z = eta * inv;     // rho / zeta
  const double r_e = zeta * inv;    // rho / eta
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const double t2 = u[r];
    const double t2_rz = t2 * r_z, t2_re = t2 * r_e;
    const T B10 = T((1.0 - t2_rz) * half_zinv);
    const T B01 = T((1.0 - t2_re) * half_einv);
    const T B00 = T(0.5 * t2 * inv);
    const T wt = T(w[r] * scale);
    T I[3][D1][D2];
    const double PA[3] = {B.A0.x, B.A0.y, B.A1.x};
    const double QC[3] = {K.A0.x, K.A0.y, K.A1.x};
    const double QP[3] = {QPx, QPy, QPz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T c00 = T(PA[d] + t2_rz * QP[d]);
      const T d00 = T(QC[d] - t2_re * QP[d]);
      I[d][0][0] = (d == 2) ? wt : T(1);
      if (D1 > 1) I[d][1][0] = c00 * I[d][0][0];
#pragma unroll
      for (int e = 1; e + 1 < D1; ++e) I[d][e + 1][0] = c00 * I[d][e][0] + T(e) * B10 * I[d][e - 1][0];
#pragma unroll
      for (int f = 0; f + 1 < D2; ++f) {
#pragma unroll
        for (int e = 0; e < D1; ++e) {
          T v = d00 * I[d][e][f];
          if (f > 0) v += T(f) * B01 * I[d][e][f - 1];
          if (e > 0) v += T(e) * B00 * I[d][e - 1][f];
          I[d][e][f + 1] = v;
        }
      }
    }
    static_for<Q::NE>([&](auto e) {
      constexpr int ge = Q::FE + decltype(e)::value;
      static_for<Q::NF>([&](auto f) {
        constexpr int gf = Q::FF + decltype(f)::value;
        esfs[decltype(e)::value][decltype(f)::value] +=
            I[0][gx(ge)][gx(gf)] * I[1][gy(ge)][gy(gf)] * I[2][gz(ge)][gz(gf)];
      });
    });
  }
}

// One flat loop over the nbp x nkp primitive quartets: lanes with the same count but
// different (nbp, nkp) splits stay converged.  Kets are the outer index and bras the
// inner one: the lanes of a warp share the bra pair (bra-major lists), so the
// per-iteration bra loads are warp-wide broadcasts and each lane's ket record is
// read once per ket primitive, one iteration ahead.  (Two primitive quartets per
// iteration as independent chains measured no faster on (H2O)32.)
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void accumulate_esfs(const PrimPair* __restrict__ bp, int nbp,
                                                const PrimPair* __restrict__ kp, int nkp,
                                                T (&esfs)[Quartet<LA, LB, LC, LD>::NE][Quartet<LA, LB, LC, LD>::NF],
                                                const double* __restrict__ rys_smem = nullptr) {
  using Q = Quartet<LA, LB, LC, LD>;
  constexpr bool BPA = Q::LAB > 0, KPA = Q::LCD > 0;
#pragma unroll
  for (int e = 0; e < Q::NE; ++e)
#pragma unroll
    for (int f = 0; f < Q::NF; ++f) esfs[e][f] = T(0);
  const int npq = nbp * nkp;
  if (npq <= 0) return;
  const double2* bq = reinterpret_cast<const double2*>(bp);
  const double2* kq = reinterpret_cast<const double2*>(kp);
  int ib = 0, ik = 0;
  PrimRegs kc = load_prim<KPA>(kq, 0);
#pragma unroll(kPrimUnroll)
  for (int p = 0; p < npq; ++p) {
    const PrimRegs b = load_prim<BPA>(bq, ib);
    const PrimRegs k = kc;
    if (++ib == nbp) {
      ib = 0;
      ++ik;
      if (ik < nkp) kc = load_prim<KPA>(kq, ik);
    }
    prim_quartet<LA, LB, LC, LD, T>(b, k, 1.0, esfs, rys_smem);
  }
}

// Horizontal transfer on the ket: esfs[e][f] (f over l in [LC, LC+LD]) ->
// out[e][c][d], (c, d+1_i) = (c+1_i, d) + R_i (c, d), R = C - D.
// Level k holds d over comps(k) and c over l in [LC, LC+LD-k].
template <int LC, int LD, int NE, typename T>
__device__ __forceinline__ void hrr_ket(const T (&G)[NE][CT.first[LC + LD + 1] - CT.first[LC]], const double* R,
                                        T (&out)[NE][ncart(LC)][ncart(LD)]) {
  if constexpr (LD == 0) {
#pragma unroll
    for (int e = 0; e < NE; ++e)
#pragma unroll
      for (int c = 0; c < ncart(LC); ++c) out[e][c][0] = G[e][c];
  } else {
    // level tables: lev[k][c_global_offset][d], c over l in [LC, LC+LD-k]
    constexpr int NCR = CT.first[LC + LD + 1] - CT.first[LC];
    T cur[NE][NCR][ncart(LD)];
#pragma unroll
    for (int e = 0; e < NE; ++e)
#pragma unroll
      for (int c = 0; c < NCR; ++c) cur[e][c][0] = G[e][c];
    static_for<LD>([&](auto kk) {
      constexpr int k = decltype(kk)::value;           // building d level k+1
      constexpr int NCN = CT.first[LC + LD - k] - CT.first[LC];
      T nxt[NE][NCN > 0 ? NCN : 1][ncart(k + 1)];
      static_for<ncart(k + 1)>([&](auto dd) {
        constexpr int d1 = decltype(dd)::value;
        constexpr int px = cx(k + 1, d1), py = cy(k + 1, d1), pz = cz(k + 1, d1);
        constexpr int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
        constexpr int d0 = CT.idx[px - (dir == 0)][py - (dir == 1)][pz - (dir == 2)];
        static_for<NCN>([&](auto ci) {
          constexpr int c = decltype(ci)::value;
          constexpr int g = CT.first[LC] + c;
          constexpr int gp = gidx(gx(g) + (dir == 0), gy(g) + (dir == 1), gz(g) + (dir == 2)) - CT.first[LC];
#pragma unroll
          for (int e = 0; e < NE; ++e) nxt[e][c][d1] = cur[e][gp][d0] + T(R[dir]) * cur[e][c][d0];
        });
      });
#pragma unroll
      for (int e = 0; e < NE; ++e)
#pragma unroll
        for (int c = 0; c < NCN; ++c)
#pragma unroll
          for (int d = 0; d < ncart(k + 1); ++d) cur[e][c][d] = nxt[e][c][d];
    });
#pragma unroll
    for (int e = 0; e < NE; ++e)
#pragma unroll
      for (int c = 0; c < ncart(LC); ++c)
#pragma unroll
        for (int d = 0; d < ncart(LD); ++d) out[e][c][d] = cur[e][c][d];
  }
}

// Horizontal transfer on the bra: G[e][r] (e over l in [LA, LA+LB]) ->
// out[a][b][r] with R = A - B.
template <int LA, int LB, int NR, typename T>
__device__ __forceinline__ void hrr_bra(const T (&G)[CT.first[LA + LB + 1] - CT.first[LA]][NR], const double* R,
                                        T (&out)[ncart(LA)][ncart(LB)][NR]) {
  if constexpr (LB == 0) {
#pragma unroll
    for (int a = 0; a < ncart(LA); ++a)
#pragma unroll
      for (int r = 0; r < NR; ++r) out[a][0][r] = G[a][r];
  } else {
    constexpr int NAR = CT.first[LA + LB + 1] - CT.first[LA];
    T cur[NAR][ncart(LB)][NR];
#pragma unroll
    for (int a = 0; a < NAR; ++a)
#pragma unroll
      for (int r = 0; r < NR; ++r) cur[a][0][r] = G[a][r];
    static_for<LB>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      constexpr int NAN_ = CT.first[LA + LB - k] - CT.first[LA];
      T nxt[NAN_ > 0 ? NAN_ : 1][ncart(k + 1)][NR];
      static_for<ncart(k + 1)>([&](auto bb) {
        constexpr int b1 = decltype(bb)::value;
        constexpr int px = cx(k + 1, b1), py = cy(k + 1, b1), pz = cz(k + 1, b1);
        constexpr int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
        constexpr int b0 = CT.idx[px - (dir == 0)][py - (dir == 1)][pz - (dir == 2)];
        static_for<NAN_>([&](auto ai) {
          constexpr int a = decltype(ai)::value;
          constexpr int g = CT.first[LA] + a;
          constexpr int gp = gidx(gx(g) + (dir == 0), gy(g) + (dir == 1), gz(g) + (dir == 2)) - CT.first[LA];
#pragma unroll
          for (int r = 0; r < NR; ++r) nxt[a][b1][r] = cur[gp][b0][r] + T(R[dir]) * cur[a][b0][r];
        });
      });
#pragma unroll
      for (int a = 0; a < NAN_; ++a)
#pragma unroll
        for (int b = 0; b < ncart(k + 1); ++b)
#pragma unroll
          for (int r = 0; r < NR; ++r) cur[a][b][r] = nxt[a][b][r];
    });
#pragma unroll
    for (int a = 0; a < ncart(LA); ++a)
#pragma unroll
      for (int b = 0; b < ncart(LB); ++b)
#pragma unroll
        for (int r = 0; r < NR; ++r) out[a][b][r] = cur[a][b][r];
  }
}

// (e0|f0) of a bra family: the primitive loop runs once over the positioned
// primitive pairs the members share (bp, the first member's), each primitive
// quartet evaluated with a unit bra coefficient and added into every member's block
// with that member's coefficient product (bm[m][ib].cc; bm[m] null: no member m).
template <int LA, int LB, int LC, int LD, typename T, int MB>
__device__ __forceinline__ void accumulate_esfs_fam(const PrimPair* __restrict__ bp, int nbp,
                                                    const PrimPair* __restrict__ kp, int nkp,
                                                    const PrimPair* const (&bm)[MB],
                                                    T (&esfs)[MB][Quartet<LA, LB, LC, LD>::NE][Quartet<LA, LB, LC, LD>::NF],
                                                    const double* __restrict__ rys_smem) {
  using Q = Quartet<LA, LB, LC, LD>;
  constexpr bool BPA = Q::LAB > 0, KPA = Q::LCD > 0;
#pragma unroll
  for (int m = 0; m < MB; ++m)
#pragma unroll
    for (int e = 0; e < Q::NE; ++e)
#pragma unroll
      for (int f = 0; f < Q::NF; ++f) esfs[m][e][f] = T(0);
  const int npq = nbp * nkp;
  if (npq <= 0) return;
  const double2* bq = reinterpret_cast<const double2*>(bp);
  const double2* kq = reinterpret_cast<const double2*>(kp);
  int ib = 0, ik = 0;
  PrimRegs kc = load_prim<KPA>(kq, 0);
  for (int p = 0; p < npq; ++p) {
    PrimRegs b = load_prim<BPA>(bq, ib);
    double cb[MB];
#pragma unroll
    for (int m = 0; m < MB; ++m) cb[m] = bm[m] ? __ldg(&bm[m][ib].cc) : 0.0;
    b.C.x = 1.0;
    const PrimRegs k = kc;
    if (++ib == nbp) {
      ib = 0;
      ++ik;
      if (ik < nkp) kc = load_prim<KPA>(kq, ik);
    }
    T one[Q::NE][Q::NF];
#pragma unroll
    for (int e = 0; e < Q::NE; ++e)
#pragma unroll
      for (int f = 0; f < Q::NF; ++f) one[e][f] = T(0);
    prim_quartet<LA, LB, LC, LD, T>(b, k, 1.0, one, rys_smem);
#pragma unroll
    for (int m = 0; m < MB; ++m) {
      const T w = T(cb[m]);
#pragma unroll
      for (int e = 0; e < Q::NE; ++e)
#pragma unroll
        for (int f = 0; f < Q::NF; ++f) esfs[m][e][f] += w * one[e][f];
    }
  }
}

// Horizontal transfers of one (e0|f0) block to the Cartesian (ab|cd), as double.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void hrr_quartet(const T (&esfs)[Quartet<LA, LB, LC, LD>::NE][Quartet<LA, LB, LC, LD>::NF],
                                            const double* Rab, const double* Rcd,
                                            double (&abcd)[ncart(LA)][ncart(LB)][ncart(LC) * ncart(LD)]) {
  using Q = Quartet<LA, LB, LC, LD>;
  double ed[Q::NE][Q::NF];
#pragma unroll
  for (int e = 0; e < Q::NE; ++e)
#pragma unroll
    for (int f = 0; f < Q::NF; ++f) ed[e][f] = (double)esfs[e][f];
  double ket[Q::NE][Q::NC][Q::ND];
  hrr_ket<LC, LD, Q::NE, double>(ed, Rcd, ket);
  double flat[Q::NE][Q::NC * Q::ND];
#pragma unroll
  for (int e = 0; e < Q::NE; ++e)
#pragma unroll
    for (int c = 0; c < Q::NC; ++c)
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) flat[e][c * Q::ND + d] = ket[e][c][d];
  hrr_bra<LA, LB, Q::NC * Q::ND, double>(flat, Rab, abcd);
}

// Contracted Cartesian integrals (ab|cd) of one quartet, as double.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void quartet_integrals(const PrimPair* bp, int nbp, const PrimPair* kp, int nkp,
                                                  const double* Rab, const double* Rcd,
                                                  double (&abcd)[ncart(LA)][ncart(LB)][ncart(LC) * ncart(LD)],
                                                  const double* __restrict__ rys_smem = nullptr) {
  using Q = Quartet<LA, LB, LC, LD>;
  T esfs[Q::NE][Q::NF];
  accumulate_esfs<LA, LB, LC, LD, T>(bp, nbp, kp, nkp, esfs, rys_smem);
  double ed[Q::NE][Q::NF];
#pragma unroll
  for (int e = 0; e < Q::NE; ++e)
#pragma unroll
    for (int f = 0; f < Q::NF; ++f) ed[e][f] = (double)esfs[e][f];
  double ket[Q::NE][Q::NC][Q::ND];
  hrr_ket<LC, LD, Q::NE, double>(ed, Rcd, ket);
  double flat[Q::NE][Q::NC * Q::ND];
#pragma unroll
  for (int e = 0; e < Q::NE; ++e)
#pragma unroll
    for (int c = 0; c < Q::NC; ++c)
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) flat[e][c * Q::ND + d] = ket[e][c][d];
  hrr_bra<LA, LB, Q::NC * Q::ND, double>(flat, Rab, abcd);
}

}  // namespace tf
