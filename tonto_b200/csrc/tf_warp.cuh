// tf_warp.cuh — warp-cooperative shell quartets with runtime angular momenta, used
// for the Schwarz diagonal (ab|ab) of the pair classes above the thread kernels
// (the (e0|f0) block, up to 31 x 31 for (dd|dd), does not fit one thread's
// registers; the J/K builds of those classes use the lane-group kernels of
// tf_group.cuh), and for everything with an f shell: its Schwarz bounds and its
// J/K quartets (k_jk_warp), in a per-warp scratch area of global memory (up to
// 248 KB for (ff|ff)).  One warp computes one contracted quartet:
//   * every lane evaluates the Rys nodes/weights of the primitive quartet
//     (warp-uniform table reads);
//   * lanes (direction, root) build the 2D recurrence tables in shared memory;
//   * lanes own (e, f) elements of the (e0|f0) block and accumulate them in
//     shared memory across primitive quartets;
//   * the horizontal transfers and the digestion run with lanes over elements.
// Angular momenta are runtime values here (compiled once), so one kernel serves
// every pair class.
#pragma once
#include "tf_device.cuh"

namespace tf {

constexpr int cmax_w(int a, int b) { return a > b ? a : b; }

constexpr int WL_MAX = 3;                       // highest l in the warp path (f)
constexpr int WNR_MAX = 2 * WL_MAX + 1;         // roots for (ff|ff)

// Doubles one warp needs for a class of shells up to l = L: the 2D tables (3 axes x
// roots x D1 x D2), and two buffers each holding the largest of the (e0|f0) block,
// the ket transfer levels, the compacted [e][cd] block and the bra transfer levels.
constexpr int w_i2d_need(int L) { return 3 * (2 * L + 1) * (2 * L + 1) * (2 * L + 1); }
constexpr int w_buf_need(int L) {
  int m = 0;
  for (int la = 0; la <= L; ++la)
    for (int lb = 0; lb <= la; ++lb)
      for (int lc = 0; lc <= L; ++lc)
        for (int ld = 0; ld <= lc; ++ld) {
          const int fe = ncart_upto(la - 1), ne = ncart_upto(la + lb) - fe;
          const int ff = ncart_upto(lc - 1), nf = ncart_upto(lc + ld) - ff;
          const int ncd = ncart(lc) * ncart(ld);
          m = cmax_w(m, ne * nf);
          for (int k = 0; k < ld; ++k) m = cmax_w(m, ne * (ncart_upto(lc + ld - k - 1) - ff) * ncart(k + 1));
          m = cmax_w(m, ne * ncd);
          for (int k = 0; k < lb; ++k) m = cmax_w(m, (ncart_upto(la + lb - k - 1) - fe) * ncart(k + 1) * ncd);
        }
  return m;
}
// s, p, d (the Schwarz bounds of the d pair classes, in shared memory)
constexpr int W_I2D = w_i2d_need(2);            // 375
constexpr int W_BUF = w_buf_need(2);
constexpr int W_SMEM = W_I2D + 2 * W_BUF;
// up to f (quartets with an f shell, in global scratch)
constexpr int WF_I2D = w_i2d_need(3);           // 1029
constexpr int WF_BUF = w_buf_need(3);
constexpr int WF_SCRATCH = WF_I2D + 2 * WF_BUF;

struct WarpQuartet {
  int la, lb, lc, ld;
  int d1, d2, nr, ne, nf, fe, ff;
};

__device__ __forceinline__ WarpQuartet wq_make(int la, int lb, int lc, int ld) {
  WarpQuartet q;
  q.la = la; q.lb = lb; q.lc = lc; q.ld = ld;
  q.d1 = la + lb + 1; q.d2 = lc + ld + 1;
  q.nr = (la + lb + lc + ld) / 2 + 1;
  q.fe = ncart_upto(la - 1); q.ne = ncart_upto(la + lb) - q.fe;
  q.ff = ncart_upto(lc - 1); q.nf = ncart_upto(lc + ld) - q.ff;
  return q;
}

// component lookup (runtime index into the constexpr table, via a switch-free
// arithmetic decode held in a small __constant__ copy)
__constant__ unsigned char c_comp[3][NCOMP_ALL];
__constant__ unsigned char c_cidx[LCOMP + 1][LCOMP + 1][LCOMP + 1];

// Cartesian (ab|cd) of one quartet into out[((a*nb + b)*nc + c)*nd + d].
// sm: this warp's scratch, i2d + 2 buf doubles (W_SMEM for s, p, d in shared memory,
// WF_SCRATCH up to f).  Returns the number of primitive quartets.
__device__ int warp_quartet(const WarpQuartet& q, const PrimPair* __restrict__ bp, int nbp,
                            const PrimPair* __restrict__ kp, int nkp, const double* Rab, const double* Rcd,
                            double* __restrict__ sm, double*& out, int i2d = W_I2D, int buf = W_BUF) {
  const int lane = threadIdx.x & 31;
  double* I2 = sm;                     // [3][nr][d1][d2]
  double* es = sm + i2d;               // esfs [ne][nf]
  double* tb = es + buf;               // scratch
  const int nef = q.ne * q.nf;
  for (int k = lane; k < nef; k += 32) es[k] = 0.0;
  const int tsz = q.d1 * q.d2;
  for (int ib = 0; ib < nbp; ++ib) {
    const double4 b0 = ld4(bp + ib, 0);
    const double4 b1 = ld4(bp + ib, 1);
    const double bcc = __ldg(&bp[ib].cc) * TWOPI5ON2;
    for (int ik = 0; ik < nkp; ++ik) {
      const double4 k0 = ld4(kp + ik, 0);
      const double4 k1 = ld4(kp + ik, 1);
      const double kcc = __ldg(&kp[ik].cc);
      const double zeta = b0.w, eta = k0.w;
      const double sq = rsqrt_nr(zeta + eta);
      const double inv = sq * sq;
      const double rho = zeta * eta * inv;
      const double QP[3] = {k0.x - b0.x, k0.y - b0.y, k0.z - b0.z};
      const double xx = rho * (QP[0] * QP[0] + QP[1] * QP[1] + QP[2] * QP[2]);
      double u[WNR_MAX], w[WNR_MAX];
      switch (q.nr) {
        case 1: { double uu[1], ww[1]; rys_eval<1>(xx, uu, ww); u[0] = uu[0]; w[0] = ww[0]; } break;
        case 2: { double uu[2], ww[2]; rys_eval<2>(xx, uu, ww); for (int i = 0; i < 2; ++i) { u[i] = uu[i]; w[i] = ww[i]; } } break;
        case 3: { double uu[3], ww[3]; rys_eval<3>(xx, uu, ww); for (int i = 0; i < 3; ++i) { u[i] = uu[i]; w[i] = ww[i]; } } break;
        case 4: { double uu[4], ww[4]; rys_eval<4>(xx, uu, ww); for (int i = 0; i < 4; ++i) { u[i] = uu[i]; w[i] = ww[i]; } } break;
        case 5: { double uu[5], ww[5]; rys_eval<5>(xx, uu, ww); for (int i = 0; i < 5; ++i) { u[i] = uu[i]; w[i] = ww[i]; } } break;
        case 6: { double uu[6], ww[6]; rys_eval<6>(xx, uu, ww); for (int i = 0; i < 6; ++i) { u[i] = uu[i]; w[i] = ww[i]; } } break;
        default: { double uu[7], ww[7]; rys_eval<7>(xx, uu, ww); for (int i = 0; i < 7; ++i) { u[i] = uu[i]; w[i] = ww[i]; } } break;
      }
      const double scale = bcc * kcc * sq;      // (cc holds the pair's sqrt(zeta))
      const double r_z = eta * inv, r_e = zeta * inv;
      __syncwarp();
      // 2D tables: lane -> (direction, root)
      if (lane < 3 * q.nr) {
        const int d = lane / q.nr, r = lane % q.nr;
        double t2 = 0.0, wr = 0.0;
#pragma unroll
        for (int i = 0; i < WNR_MAX; ++i)
          if (i == r) { t2 = u[i]; wr = w[i]; }
        const double t2_rz = t2 * r_z, t2_re = t2 * r_e;
        const double B10 = (1.0 - t2_rz) * b1.w, B01 = (1.0 - t2_re) * k1.w, B00 = 0.5 * t2 * inv;
        const double PA = d == 0 ? b1.x : (d == 1 ? b1.y : b1.z);
        const double QC = d == 0 ? k1.x : (d == 1 ? k1.y : k1.z);
        const double c00 = PA + t2_rz * QP[d], d00 = QC - t2_re * QP[d];
        double* I = I2 + (d * q.nr + r) * tsz;
        I[0] = (d == 2) ? wr * scale : 1.0;
        if (q.d1 > 1) I[q.d2] = c00 * I[0];
        for (int e = 1; e + 1 < q.d1; ++e) I[(e + 1) * q.d2] = c00 * I[e * q.d2] + e * B10 * I[(e - 1) * q.d2];
        for (int f = 0; f + 1 < q.d2; ++f)
          for (int e = 0; e < q.d1; ++e) {
            double v = d00 * I[e * q.d2 + f];
            if (f > 0) v += f * B01 * I[e * q.d2 + f - 1];
            if (e > 0) v += e * B00 * I[(e - 1) * q.d2 + f];
            I[e * q.d2 + f + 1] = v;
          }
      }
      __syncwarp();
      for (int k = lane; k < nef; k += 32) {
        const int e = k / q.nf, f = k % q.nf;
        const int ge = q.fe + e, gf = q.ff + f;
        const int ox = c_comp[0][ge] * q.d2 + c_comp[0][gf];
        const int oy = c_comp[1][ge] * q.d2 + c_comp[1][gf];
        const int oz = c_comp[2][ge] * q.d2 + c_comp[2][gf];
        double s = 0.0;
        for (int r = 0; r < q.nr; ++r)
          s += I2[(0 * q.nr + r) * tsz + ox] * I2[(1 * q.nr + r) * tsz + oy] * I2[(2 * q.nr + r) * tsz + oz];
        es[k] += s;
      }
    }
  }
  __syncwarp();
  // ket HRR: es[e][f] -> [e][c][d] (levels in tb / es ping-pong)
  double* src = es;
  double* dst = tb;
  {
    const int ncr0 = q.nf;   // c over l in [lc, lc+ld]
    int ny = 1;              // d comps at current level
    int ncr = ncr0;
    // src layout: [e][c][y] with c over current range, y over comps(level)
    for (int k = 0; k < q.ld; ++k) {
      const int ncn = ncart_upto(q.lc + q.ld - k - 1) - q.ff;
      const int nyn = ncart(k + 1);
      const int tot = q.ne * ncn * nyn;
      for (int t = lane; t < tot; t += 32) {
        const int e = t / (ncn * nyn), rem = t % (ncn * nyn), c = rem / nyn, y1 = rem % nyn;
        const int gy = ncart_upto(k) + y1;
        const int px = c_comp[0][gy], py = c_comp[1][gy], pz = c_comp[2][gy];
        const int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
        const int y0 = c_cidx[px - (dir == 0)][py - (dir == 1)][pz - (dir == 2)];
        const int g = q.ff + c;
        const int cx2 = c_comp[0][g] + (dir == 0), cy2 = c_comp[1][g] + (dir == 1), cz2 = c_comp[2][g] + (dir == 2);
        const int gp = ncart_upto(cx2 + cy2 + cz2 - 1) + c_cidx[cx2][cy2][cz2] - q.ff;
        dst[t] = src[(e * ncr + gp) * ny + y0] + Rcd[dir] * src[(e * ncr + c) * ny + y0];
      }
      __syncwarp();
      double* tmp = src; src = dst; dst = tmp;
      ncr = ncn;
      ny = nyn;
    }
    // src: [e][c(ncr)][d(ny)], keep c < ncart(lc)
  }
  const int nc = ncart(q.lc), nd = ncart(q.ld), ncr_fin = q.ld > 0 ? ncart(q.lc) : q.nf;
  // bra HRR on [e][cd]: rest = nc*nd (entries with c < ncart(lc))
  const int ncd = nc * nd;
  // compact to [e][cd]
  {
    const int tot = q.ne * ncd;
    for (int t = lane; t < tot; t += 32) {
      const int e = t / ncd, cd = t % ncd;
      dst[t] = src[(e * ncr_fin) * nd + cd];
    }
    __syncwarp();
    double* tmp = src; src = dst; dst = tmp;
  }
  {
    int nar = q.ne, nb = 1;
    for (int k = 0; k < q.lb; ++k) {
      const int nan_ = ncart_upto(q.la + q.lb - k - 1) - q.fe;
      const int nbn = ncart(k + 1);
      const int tot = nan_ * nbn * ncd;
      for (int t = lane; t < tot; t += 32) {
        const int a = t / (nbn * ncd), rem = t % (nbn * ncd), b1 = rem / ncd, r = rem % ncd;
        const int gb = ncart_upto(k) + b1;
        const int px = c_comp[0][gb], py = c_comp[1][gb], pz = c_comp[2][gb];
        const int dir = px > 0 ? 0 : (py > 0 ? 1 : 2);
        const int b0 = c_cidx[px - (dir == 0)][py - (dir == 1)][pz - (dir == 2)];
        const int g = q.fe + a;
        const int ax = c_comp[0][g] + (dir == 0), ay = c_comp[1][g] + (dir == 1), az = c_comp[2][g] + (dir == 2);
        const int gp = ncart_upto(ax + ay + az - 1) + c_cidx[ax][ay][az] - q.fe;
        dst[t] = src[(gp * nb + b0) * ncd + r] + Rab[dir] * src[(a * nb + b0) * ncd + r];
      }
      __syncwarp();
      double* tmp = src; src = dst; dst = tmp;
      nar = nan_;
      nb = nbn;
    }
    (void)nar;
  }
  // src: [a][b][c][d] with a over the first ncart(la) entries
  out = src;
  return nbp * nkp;
}

}  // namespace tf
