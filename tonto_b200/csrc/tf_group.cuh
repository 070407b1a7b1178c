// tf_group.cuh — lane-group quartets for the classes whose (e0|f0) block is too
// large for one thread (pp|pp), (dp|pp), (dp|ds), (dp|dp), (dd|ps), (dd|pp),
// (dd|ds), (dd|dp), (dd|dd).
//
// A group of G = NF lanes computes one contracted quartet; a warp holds
// QPW = 32 / G groups.  Per primitive quartet:
//   * each lane evaluates the Rys nodes/weights (uniform within the group);
//   * the group's lanes build the 3 x NROOT 2D recurrence tables in shared
//     memory (make_esfs_XX, shell1quartet.foo:7418-7609);
//   * lane f reads the f-columns of the tables and accumulates (e0|f0) for all e
//     in registers (compile-time unrolled over e: form_esfs :7615-7649).
// After the primitive loop the block goes to shared memory for the horizontal
// transfers (transfer_cd / transfer_ab :8310-11134) and the digestion into J, K.
#pragma once
#include "tf_device.cuh"

namespace tf {

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int LA, int LB, int LC, int LD>
struct GroupCfg {
  using Q = Quartet<LA, LB, LC, LD>;
  static constexpr int G = Q::NF;
  static constexpr int QPW = 32 / G;
  static constexpr int NR = Q::NROOT, D1 = Q::LAB + 1, D2 = Q::LCD + 1;
  static constexpr int TS = (D1 * D2) | 1;     // one 2D table, odd stride (fewer bank conflicts)
  static constexpr int T2D = 3 * NR * TS;
  static constexpr int ket_level(int k) {   // size after building d level k+1
    return Q::NE * (ncart_upto(LC + LD - k - 1) - ncart_upto(LC - 1)) * ncart(k + 1);
  }
  static constexpr int bra_level(int k) {
    return (ncart_upto(LA + LB - k - 1) - ncart_upto(LA - 1)) * ncart(k + 1) * Q::NC * Q::ND;
  }
  static constexpr int buf() {
    int m = Q::NE * Q::NF;
    for (int k = 0; k < LD; ++k) m = cmax(m, ket_level(k));
    for (int k = 0; k < LB; ++k) m = cmax(m, bra_level(k));
    return cmax(m, Q::NE * Q::NC * Q::ND);
  }
  static constexpr int BUF = buf();
  static constexpr int PER_GROUP = T2D + 2 * BUF;
  static constexpr int PER_WARP = QPW * PER_GROUP;
};

// component tables copied to shared memory once per block
struct SmemComp {
  unsigned char x[NCOMP_ALL], y[NCOMP_ALL], z[NCOMP_ALL];
  unsigned char idx[(LCOMP + 1) * (LCOMP + 1) * (LCOMP + 1)];
};

__device__ __forceinline__ int sc_idx(const SmemComp& s, int x, int y, int z) {
  return s.idx[(x * (LCOMP + 1) + y) * (LCOMP + 1) + z];
}

// Index plan of the horizontal transfers of one class, built at compile time from
// the component tables: for every produced element of every level (ket levels
// first, then bra levels) the two source positions and the direction, packed as
// s1 | s2 << 13 | dir << 26, so that a lane does one table load per element
// instead of the component-table lookups.
template <int LA, int LB, int LC, int LD>
struct HrrPlan {
  using Q = Quartet<LA, LB, LC, LD>;
  static constexpr int ket_tot(int k) {
    return Q::NE * (ncart_upto(LC + LD - k - 1) - ncart_upto(LC - 1)) * ncart(k + 1);
  }
  static constexpr int bra_tot(int k) {
    return (ncart_upto(LA + LB - k - 1) - ncart_upto(LA - 1)) * ncart(k + 1) * Q::NC * Q::ND;
  }
  static constexpr int ket_off(int k) { int o = 0; for (int i = 0; i < k; ++i) o += ket_tot(i); return o; }
  static constexpr int bra_off(int k) {
    int o = ket_off(LD);
    for (int i = 0; i < k; ++i) o += bra_tot(i);
    return o;
  }
  static constexpr int N = bra_off(LB) > 0 ? bra_off(LB) : 1;
  int code[N];
};

template <int LA, int LB, int LC, int LD>
constexpr HrrPlan<LA, LB, LC, LD> make_hrr_plan() {
  using P = HrrPlan<LA, LB, LC, LD>;
  using Q = Quartet<LA, LB, LC, LD>;
  P p{};
  const int FF = ncart_upto(LC - 1), FE = ncart_upto(LA - 1);
  for (int k = 0; k < LD; ++k) {
    const int NCR = ncart_upto(LC + LD - k) - FF, NY = ncart(k);
    const int NCN = ncart_upto(LC + LD - k - 1) - FF, NYN = ncart(k + 1);
    for (int t = 0; t < P::ket_tot(k); ++t) {
      const int e = t / (NCN * NYN), rem = t - e * (NCN * NYN), c = rem / NYN, y1 = rem - c * NYN;
      const int gy = ncart_upto(k) + y1;           // global index of the level-(k+1) component
      const int px = CT.x[gy], py = CT.y[gy], pz = CT.z[gy];
      const int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
      const int y0 = CT.idx[px - (dir == 0)][py - (dir == 1)][pz - (dir == 2)];
      const int g = FF + c;
      const int ax = CT.x[g] + (dir == 0), ay = CT.y[g] + (dir == 1), az = CT.z[g] + (dir == 2);
      const int gp = ncart_upto(ax + ay + az - 1) + CT.idx[ax][ay][az] - FF;
      const int s1 = (e * NCR + gp) * NY + y0, s2 = (e * NCR + c) * NY + y0;
      p.code[P::ket_off(k) + t] = s1 | (s2 << 13) | (dir << 26);
    }
  }
  const int NCD = Q::NC * Q::ND;
  for (int k = 0; k < LB; ++k) {
    const int NBY = ncart(k), NAN_ = ncart_upto(LA + LB - k - 1) - FE, NBN = ncart(k + 1);
    for (int t = 0; t < P::bra_tot(k); ++t) {
      const int a = t / (NBN * NCD), rem = t - a * (NBN * NCD), b1 = rem / NCD, r = rem - b1 * NCD;
      const int gb = ncart_upto(k) + b1;
      const int px = CT.x[gb], py = CT.y[gb], pz = CT.z[gb];
      const int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
      const int b0 = CT.idx[px - (dir == 0)][py - (dir == 1)][pz - (dir == 2)];
      const int g = FE + a;
      const int ax = CT.x[g] + (dir == 0), ay = CT.y[g] + (dir == 1), az = CT.z[g] + (dir == 2);
      const int gp = ncart_upto(ax + ay + az - 1) + CT.idx[ax][ay][az] - FE;
      const int s1 = (gp * NBY + b0) * NCD + r, s2 = (a * NBY + b0) * NCD + r;
      p.code[P::bra_off(k) + t] = s1 | (s2 << 13) | (dir << 26);
    }
  }
  return p;
}

template <int LA, int LB, int LC, int LD>
__device__ const HrrPlan<LA, LB, LC, LD> g_hrr_plan = make_hrr_plan<LA, LB, LC, LD>();

// Horizontal transfers of one group's block in shared memory, from the index plan.
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ double* group_hrr_plan(double* src, double* dst, const double* Rab, const double* Rcd,
                                                  int gl) {
  using P = HrrPlan<LA, LB, LC, LD>;
  constexpr int G = GroupCfg<LA, LB, LC, LD>::G;
  const int* code = g_hrr_plan<LA, LB, LC, LD>.code;
  static_for<LD>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    constexpr int TOT = P::ket_tot(k), OFF = P::ket_off(k);
    for (int t = gl; t < TOT; t += G) {
      const int cd = __ldg(code + OFF + t);
      const int dir = cd >> 26;
      const double R = dir == 0 ? Rcd[0] : (dir == 1 ? Rcd[1] : Rcd[2]);
      dst[t] = src[cd & 0x1fff] + R * src[(cd >> 13) & 0x1fff];
    }
    __syncwarp();
    double* tmp = src; src = dst; dst = tmp;
  });
  static_for<LB>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    constexpr int TOT = P::bra_tot(k), OFF = P::bra_off(k);
    for (int t = gl; t < TOT; t += G) {
      const int cd = __ldg(code + OFF + t);
      const int dir = cd >> 26;
      const double R = dir == 0 ? Rab[0] : (dir == 1 ? Rab[1] : Rab[2]);
      dst[t] = src[cd & 0x1fff] + R * src[(cd >> 13) & 0x1fff];
    }
    __syncwarp();
    double* tmp = src; src = dst; dst = tmp;
  });
  return src;
}

// Horizontal transfers of one group's block in shared memory.  On entry `src`
// holds es[e][f]; on exit the returned pointer holds (ab|cd) as
// [a][b][c*ND + d].  `gl` is the lane within the group, `G` the group size.
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ double* group_hrr(double* src, double* dst, const SmemComp& sc, const double* Rab,
                                             const double* Rcd, int gl) {
  using Q = Quartet<LA, LB, LC, LD>;
  constexpr int G = GroupCfg<LA, LB, LC, LD>::G;
  constexpr int FF = ncart_upto(LC - 1), FE = ncart_upto(LA - 1);
  // ket: es[e][c][y] with c over l in [LC, LC+LD-k], y over comps(k)
  static_for<LD>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    constexpr int NCR = ncart_upto(LC + LD - k) - FF;        // c range at level k
    constexpr int NY = ncart(k);
    constexpr int NCN = ncart_upto(LC + LD - k - 1) - FF;
    constexpr int NYN = ncart(k + 1);
    constexpr int TOT = Q::NE * NCN * NYN;
    for (int t = gl; t < TOT; t += G) {
      const int e = t / (NCN * NYN), rem = t - e * (NCN * NYN), c = rem / NYN, y1 = rem - c * NYN;
      const int gy = ncart_upto(k) + y1;
      const int px = sc.x[gy], py = sc.y[gy], pz = sc.z[gy];
      const int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
      const int y0 = sc_idx(sc, px - (dir == 0), py - (dir == 1), pz - (dir == 2));
      const int g = FF + c;
      const int ax = sc.x[g] + (dir == 0), ay = sc.y[g] + (dir == 1), az = sc.z[g] + (dir == 2);
      const int gp = ncart_upto(ax + ay + az - 1) + sc_idx(sc, ax, ay, az) - FF;
      dst[t] = src[(e * NCR + gp) * NY + y0] + Rcd[dir] * src[(e * NCR + c) * NY + y0];
    }
    __syncwarp();
    double* tmp = src; src = dst; dst = tmp;
  });
  // now src = [e][c (ncart(LC))][d (ncart(LD))] = [e][cd]
  constexpr int NCD = Q::NC * Q::ND;
  static_for<LB>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    constexpr int NBY = ncart(k);
    constexpr int NAN_ = ncart_upto(LA + LB - k - 1) - FE;
    constexpr int NBN = ncart(k + 1);
    constexpr int TOT = NAN_ * NBN * NCD;
    for (int t = gl; t < TOT; t += G) {
      const int a = t / (NBN * NCD), rem = t - a * (NBN * NCD), b1 = rem / NCD, r = rem - b1 * NCD;
      const int gb = ncart_upto(k) + b1;
      const int px = sc.x[gb], py = sc.y[gb], pz = sc.z[gb];
      const int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
      const int b0 = sc_idx(sc, px - (dir == 0), py - (dir == 1), pz - (dir == 2));
      const int g = FE + a;
      const int ax = sc.x[g] + (dir == 0), ay = sc.y[g] + (dir == 1), az = sc.z[g] + (dir == 2);
      const int gp = ncart_upto(ax + ay + az - 1) + sc_idx(sc, ax, ay, az) - FE;
      dst[t] = src[(gp * NBY + b0) * NCD + r] + Rab[dir] * src[(a * NBY + b0) * NCD + r];
    }
    __syncwarp();
    double* tmp = src; src = dst; dst = tmp;
  });
  return src;
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
struct GroupArgs {
  const int2* quartets;
  long long n;
  const PairRec* pairs;
  const PrimPair* prim_full;
  const PrimPair* prim_skip;
  const double* P;
  double* J;
  double* K;
  const MolInfo* mols;
  unsigned long long* prim_count;
  const long long* range;       // graph builds: see resolve_range
  long long base, cap;
  const int4* jkrec;            // packed pair records (load_pair_jk)
  const double2* pairR;
  const double* P2;             // unrestricted: beta density and its J, K (else null)
  double* J2;
  double* K2;
  int want;                     // bit 0 J, bit 1 K
  unsigned long long* qcount;   // quartets counted per class (the launch's FP64 or FP32 half), or null
  long long fx_lo;              // deterministic builds: offset of the lo words (fock_add), else 0
};

// Rys nodes and weights of a lane group's primitive quartet: the 2 N polynomial
// pieces (u_1..u_N, w_1..w_N at the interval of x) are spread over the group's
// G lanes, each evaluated once, then exchanged with shuffles, instead of every
// lane of the group evaluating all of them.  x is uniform within a group; every
// lane of the warp takes part.  gbase: the group's first lane.
template <int N, int G>
__device__ __forceinline__ void group_rys(double x, int gl, int gbase, double (&u)[N], double (&w)[N]) {
  constexpr int NF2 = 2 * N, PER = (NF2 + G - 1) / G;
  constexpr int XMAX = rys_xmax(N), OFF = rys_offset(N), HOFF = rys_hoffset(N);
  const bool tab = x < (double)XMAX;
  const int j = tab ? (int)x : 0;
  const double s = x - (double)j;
  double val[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int f = gl + q * G;
    double v = 0.0;
    if (tab && f < NF2) {
      const double* cf = tf_rys_coef + OFF + j * (NF2 * TF_RYS_NCOEF) + f * TF_RYS_NCOEF;
      v = __ldg(cf + TF_RYS_DEG);
#pragma unroll
      for (int k = TF_RYS_DEG - 1; k >= 0; --k) v = fma(v, s, __ldg(cf + k));
    }
    val[q] = v;
  }
#pragma unroll
  for (int f = 0; f < NF2; ++f) {
    const double v = __shfl_sync(0xffffffffu, val[f / G], gbase + f % G);
    if (f < N) u[f] = v;
    else w[f - N] = v;
  }
  if (!tab) {
    const double ix = rcp_nr(x), isx = rsqrt_nr(x);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      u[i] = tf_rys_hroot2[HOFF + i] * ix;
      w[i] = tf_rys_hweight[HOFF + i] * isx;
    }
  }
}

__constant__ unsigned char c_gcomp[3][NCOMP_ALL];
__constant__ unsigned char c_gidx[(LCOMP + 1) * (LCOMP + 1) * (LCOMP + 1)];

template <int LA, int LB, int LC, int LD, bool FX>
__global__ void __launch_bounds__(128) k_jk_group(GroupArgs a) {
  using C = GroupCfg<LA, LB, LC, LD>;
  using Q = typename C::Q;
  constexpr int G = C::G, QPW = C::QPW, NR = C::NR, D1 = C::D1, D2 = C::D2, TS = C::TS;
  extern __shared__ double smem[];
  __shared__ SmemComp sc;
  for (int i = threadIdx.x; i < NCOMP_ALL; i += blockDim.x) {
    sc.x[i] = c_gcomp[0][i]; sc.y[i] = c_gcomp[1][i]; sc.z[i] = c_gcomp[2][i];
  }
  for (int i = threadIdx.x; i < (LCOMP + 1) * (LCOMP + 1) * (LCOMP + 1); i += blockDim.x) sc.idx[i] = c_gidx[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int g = lane / G;
  const bool in_group = g < QPW;
  const int gl = in_group ? lane - g * G : G;          // G: no element loop iterations
  double* gbase = smem + (size_t)(warp * QPW + (in_group ? g : 0)) * C::PER_GROUP;
  double* T2 = gbase;
  double* B0 = gbase + C::T2D;
  double* B1 = B0 + C::BUF;
  const int gf = Q::FF + (in_group ? gl : 0);
  const int fx = sc.x[gf], fy = sc.y[gf], fz = sc.z[gf];
  const long long nwarps = (long long)gridDim.x * wpb;
  unsigned long long nprim = 0, nquart = 0;
  const int2* quartets = a.quartets;
  long long nq = a.n;
  resolve_range(a.range, a.base, a.cap, quartets, nq);
  for (long long base = ((long long)blockIdx.x * wpb + warp) * QPW; base < nq; base += nwarps * QPW) {
    const long long t = base + (in_group ? g : 0);
    const bool act = in_group && t < nq;
    const int2 qd = act ? quartets[t] : make_int2(0, 0);
    const PairJK b = load_pair_jk(a.jkrec, a.pairR, qd.x);
    const PairJK k = load_pair_jk(a.jkrec, a.pairR, qd.y);
    const bool any_same = b.atom_hi == b.atom_lo || k.atom_hi == k.atom_lo || b.atom_hi == k.atom_hi ||
                          b.atom_hi == k.atom_lo || b.atom_lo == k.atom_hi || b.atom_lo == k.atom_lo;
    const PrimPair* bp = any_same ? a.prim_full + b.full_off : a.prim_skip + b.skip_off;
    const PrimPair* kp = any_same ? a.prim_full + k.full_off : a.prim_skip + k.skip_off;
    const int nbp = any_same ? b.n_full : b.n_skip;
    const int nkp = any_same ? k.n_full : k.n_skip;
    const int npq = act ? nbp * nkp : 0;
    if (act && gl == 0) { nprim += (unsigned long long)npq; nquart += 1; }
    const int maxnpq = __reduce_max_sync(0xffffffffu, npq);
    double es[Q::NE];
#pragma unroll
    for (int e = 0; e < Q::NE; ++e) es[e] = 0.0;
    int ib = 0, ik = 0;
    for (int p = 0; p < maxnpq; ++p) {
      const bool v = p < npq;
      double u[NR], w[NR];
      double4 b0 = make_double4(0, 0, 0, 1), b1 = make_double4(0, 0, 0, 0), k0 = make_double4(0, 0, 0, 1),
              k1 = make_double4(0, 0, 0, 0);
      double inv = 0.0, r_z = 0.0, r_e = 0.0, scale = 0.0, xx = 0.0;
      if (v) {
        b0 = ld4(bp + ib, 0); b1 = ld4(bp + ib, 1);
        k0 = ld4(kp + ik, 0); k1 = ld4(kp + ik, 1);
        const double bcc = __ldg(&bp[ib].cc) * TWOPI5ON2, kcc = __ldg(&kp[ik].cc);
        const double sq = rsqrt_nr(b0.w + k0.w);
        inv = sq * sq;
        const double rho = b0.w * k0.w * inv;
        const double QPx = k0.x - b0.x, QPy = k0.y - b0.y, QPz = k0.z - b0.z;
        xx = rho * (QPx * QPx + QPy * QPy + QPz * QPz);
        scale = bcc * kcc * sq;                  // (cc holds the pair's sqrt(zeta))
        r_z = k0.w * inv;
        r_e = b0.w * inv;
      }
      group_rys<NR, G>(xx, gl, lane - (in_group ? gl : 0), u, w);
      __syncwarp();
      if (v) {
        for (int task = gl; task < 3 * NR; task += G) {
          const int d = task / NR, r = task - d * NR;
          double t2 = 0.0, wr = 0.0;
#pragma unroll
          for (int i = 0; i < NR; ++i)
            if (i == r) { t2 = u[i]; wr = w[i]; }
          const double QPd = d == 0 ? k0.x - b0.x : (d == 1 ? k0.y - b0.y : k0.z - b0.z);
          const double PA = d == 0 ? b1.x : (d == 1 ? b1.y : b1.z);
          const double QC = d == 0 ? k1.x : (d == 1 ? k1.y : k1.z);
          const double t2_rz = t2 * r_z, t2_re = t2 * r_e;
          const double B10 = (1.0 - t2_rz) * b1.w, B01 = (1.0 - t2_re) * k1.w, B00 = 0.5 * t2 * inv;
          const double c00 = PA + t2_rz * QPd, d00 = QC - t2_re * QPd;
          double I[D1][D2];
          I[0][0] = d == 2 ? wr * scale : 1.0;
          if (D1 > 1) I[1][0] = c00 * I[0][0];
#pragma unroll
          for (int e = 1; e + 1 < D1; ++e) I[e + 1][0] = c00 * I[e][0] + e * B10 * I[e - 1][0];
#pragma unroll
          for (int f = 0; f + 1 < D2; ++f)
#pragma unroll
            for (int e = 0; e < D1; ++e) {
              double vv = d00 * I[e][f];
              if (f > 0) vv += f * B01 * I[e][f - 1];
              if (e > 0) vv += e * B00 * I[e - 1][f];
              I[e][f + 1] = vv;
            }
          double* out = T2 + (d * NR + r) * TS;
#pragma unroll
          for (int e = 0; e < D1; ++e)
#pragma unroll
            for (int f = 0; f < D2; ++f) out[e * D2 + f] = I[e][f];
        }
      }
      __syncwarp();
      if (v && gl < G) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          double cxv[D1], cyv[D1], czv[D1];
#pragma unroll
          for (int e = 0; e < D1; ++e) {
            cxv[e] = T2[(0 * NR + r) * TS + e * D2 + fx];
            cyv[e] = T2[(1 * NR + r) * TS + e * D2 + fy];
            czv[e] = T2[(2 * NR + r) * TS + e * D2 + fz];
          }
          static_for<Q::NE>([&](auto ee) {
            constexpr int e = decltype(ee)::value;
            constexpr int ge = Q::FE + e;
            es[e] += cxv[gx(ge)] * cyv[gy(ge)] * czv[gz(ge)];
          });
        }
      }
      if (++ik == nkp) { ik = 0; ++ib; }
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int e = 0; e < Q::NE; ++e) B0[e * Q::NF + gl] = es[e];
    }
    __syncwarp();
    const double Rab[3] = {b.Rx, b.Ry, b.Rz};
    const double Rcd[3] = {k.Rx, k.Ry, k.Rz};
    // lanes outside every group start beyond all element loops (they only keep the warp in step)
    const double* I = group_hrr_plan<LA, LB, LC, LD>(B0, B1, Rab, Rcd, in_group ? gl : 0x40000000);
    if (act) {
      const MolInfo mi = a.mols[b.mol];
      const int n = mi.n_cart;
      double f = 1.0;
      if (b.same) f *= 0.5;
      if (k.same) f *= 0.5;
      if (qd.x == qd.y) f *= 0.5;
      constexpr int NA = Q::NA, NB = Q::NB, NC = Q::NC, ND = Q::ND, NCD = NC * ND;
      const int oa = b.cart_hi, ob = b.cart_lo, oc = k.cart_hi, od = k.cart_lo;
      auto digest_j = [&](const double* __restrict__ P, double* __restrict__ Jm) {
        for (int e = gl; e < NA * NB; e += G) {            // J(ab) = sum_cd I P(cd)
          const int ia = e / NB, ibb = e - ia * NB;
          double s = 0.0;
#pragma unroll
          for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) s += I[e * NCD + c * ND + d] * __ldg(P + (size_t)(oc + c) * n + od + d);
          fock_add<FX>(Jm + (size_t)(oa + ia) * n + ob + ibb, f * s, a.fx_lo);
        }
        for (int e = gl; e < NCD; e += G) {                // J(cd) = sum_ab I P(ab)
          const int c = e / ND, d = e - c * ND;
          double s = 0.0;
#pragma unroll
          for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ibb = 0; ibb < NB; ++ibb)
              s += I[(ia * NB + ibb) * NCD + e] * __ldg(P + (size_t)(oa + ia) * n + ob + ibb);
          fock_add<FX>(Jm + (size_t)(oc + c) * n + od + d, f * s, a.fx_lo);
        }
      };
      if (a.want & 1) {
        digest_j(a.P + mi.cmat, a.J + mi.cmat);
        if (a.P2) digest_j(a.P2 + mi.cmat, a.J2 + mi.cmat);
      }
      auto digest_k = [&](const double* __restrict__ P, double* __restrict__ Km) {
        for (int e = gl; e < NA * NC; e += G) {            // K(ac) = sum_bd I P(bd)
          const int ia = e / NC, c = e - ia * NC;
          double s = 0.0;
#pragma unroll
          for (int ibb = 0; ibb < NB; ++ibb)
#pragma unroll
            for (int d = 0; d < ND; ++d)
              s += I[(ia * NB + ibb) * NCD + c * ND + d] * __ldg(P + (size_t)(ob + ibb) * n + od + d);
          fock_add<FX>(Km + (size_t)(oa + ia) * n + oc + c, f * s, a.fx_lo);
        }
        for (int e = gl; e < NA * ND; e += G) {            // K(ad) = sum_bc I P(bc)
          const int ia = e / ND, d = e - ia * ND;
          double s = 0.0;
#pragma unroll
          for (int ibb = 0; ibb < NB; ++ibb)
#pragma unroll
            for (int c = 0; c < NC; ++c)
              s += I[(ia * NB + ibb) * NCD + c * ND + d] * __ldg(P + (size_t)(ob + ibb) * n + oc + c);
          fock_add<FX>(Km + (size_t)(oa + ia) * n + od + d, f * s, a.fx_lo);
        }
        for (int e = gl; e < NB * NC; e += G) {            // K(bc) = sum_ad I P(ad)
          const int ibb = e / NC, c = e - ibb * NC;
          double s = 0.0;
#pragma unroll
          for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int d = 0; d < ND; ++d)
              s += I[(ia * NB + ibb) * NCD + c * ND + d] * __ldg(P + (size_t)(oa + ia) * n + od + d);
          fock_add<FX>(Km + (size_t)(ob + ibb) * n + oc + c, f * s, a.fx_lo);
        }
        for (int e = gl; e < NB * ND; e += G) {            // K(bd) = sum_ac I P(ac)
          const int ibb = e / ND, d = e - ibb * ND;
          double s = 0.0;
#pragma unroll
          for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int c = 0; c < NC; ++c)
              s += I[(ia * NB + ibb) * NCD + c * ND + d] * __ldg(P + (size_t)(oa + ia) * n + oc + c);
          fock_add<FX>(Km + (size_t)(ob + ibb) * n + od + d, f * s, a.fx_lo);
        }
      };
      if (a.want & 2) {
        digest_k(a.P + mi.cmat, a.K + mi.cmat);
        if (a.P2) digest_k(a.P2 + mi.cmat, a.K2 + mi.cmat);
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nprim += __shfl_xor_sync(0xffffffffu, nprim, o);
    nquart += __shfl_xor_sync(0xffffffffu, nquart, o);
  }
  if (lane == 0 && nprim) atomicAdd(a.prim_count + (((LA * 5 + LB) * 5 + LC) * 5 + LD), nprim);
  if (lane == 0 && nquart && a.qcount) atomicAdd(a.qcount + (((LA * 5 + LB) * 5 + LC) * 5 + LD), nquart);
}

template <int LA, int LB, int LC, int LD>
constexpr size_t group_smem_bytes(int warps_per_block) {
  return (size_t)warps_per_block * GroupCfg<LA, LB, LC, LD>::PER_WARP * sizeof(double);
}

}  // namespace tf
