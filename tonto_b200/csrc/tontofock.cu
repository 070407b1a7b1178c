// tontofock.cu — kernels and C ABI of the B200 direct-SCF J/K builder.
//
// Per context (one molecule, one device):
//   k_pair_prep      positioned primitive pairs of every shell pair, with and
//                    without the primitive-pair cutoff (set_ab_new,
//                    shell1quartet.foo:131-275); one thread per shell pair
//   k_schwarz<LA,LB> I_max(ab) = sqrt(max |(ab|ab)|) in the Tonto basis
//                    (make_max_abab_integrals, molecule.fock.foo:3712-3752)
// Per build:
//   k_density_to_cart  P (Tonto basis) -> P in the Cartesian basis
//   k_pmax             max |P| per shell pair, global max (molecule.fock.foo:3601)
//   k_count / k_write  Schwarz-screened quartet lists per class pair, bra-major,
//                      deterministic order (Schwarz_inequality_test :3454-3495)
//   k_jk<LA,LB,LC,LD>  one thread per quartet: Rys ERIs + digestion into J, K
//   k_finalize         J = 2(J + J^T), K = K + K^T (weight_diagonal_blocks,
//                      blockwise_symmetric_fold, symmetric_reflect :4181-4263),
//                      back to the Tonto basis
#include "tf_device.cuh"
#include "tf_warp.cuh"
#include "tf_group.cuh"
#include "../../include/tontofock.h"

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>
#include <atomic>
#include <mutex>
#include <map>

namespace tf {

constexpr int LMAX_SUPPORTED = 3;                 // s, p, d, f shells (f: the warp path)
constexpr int NPAIRCLS = (LMAX_SUPPORTED + 1) * (LMAX_SUPPORTED + 2) / 2;
constexpr int NQCLS = 625;                        // (la lb lc ld) counter slots, l <= 4
// Counters of a build, zeroed with it and read back after it: primitive quartets per
// class [0, NQCLS), the non-finite-density flag [NQCLS], contracted quartets per class
// of the FP64 buckets [NQCLS + 1, 2 NQCLS + 1) and of the FP32 buckets after them.
constexpr int BUILD_COUNTERS = 3 * NQCLS + 1;
__host__ __device__ constexpr int pair_class(int lh, int ll) { return lh * (lh + 1) / 2 + ll; }
__host__ __device__ constexpr int qclass_id(int la, int lb, int lc, int ld) { return ((la * 5 + lb) * 5 + lc) * 5 + ld; }
// Bra-family members the thread kernel of a class holds at once (accumulator
// capacity), for the classes where evaluating a bra family's primitive quartets once
// measured faster on (H2O)32 cc-pVDZ: (ss|ss) 9.36 -> 8.36 ms, (ds|ss) 3.87 -> 3.63 ms.
// (ps|ss), (ps|ps) and (ds|ps) measured slower with it (13.33 -> 13.45, 8.55 -> 8.90
// and 4.29 -> 5.63 ms: the extra accumulators cost registers and the coefficient
// loads and products every primitive quartet, and few of their bras are families),
// so they, like every other class, take one member per list entry (capacity 1).
__host__ __device__ constexpr int fam_cap_l(int la, int lb, int lc, int ld) {
  return (la == 0 && lb == 0 && lc == 0 && ld == 0) ? 4 : (la == 2 && lb == 0 && lc == 0 && ld == 0) ? 2 : 1;
}

__constant__ double c_U[4][10 * 7];               // Cartesian -> spherical, l = 0..3, [cart][m]

// ---------------------------------------------------------------------------
// error helpers
// ---------------------------------------------------------------------------
#define TF_CUDA(call)                                                     \
  do {                                                                    \
    cudaError_t e__ = (call);                                             \
    if (e__ != cudaSuccess) {                                             \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e__));     \
      return e__ == cudaErrorMemoryAllocation ? TF_ENOMEM : TF_ECUDA;     \
    }                                                                     \
  } while (0)

// Returns from the calling function with the status of a call that failed.
#define TF_TRY_RC(call)              \
  do {                               \
    const int rc__ = (call);         \
    if (rc__ != TF_OK) return rc__;  \
  } while (0)

thread_local std::string g_last_error;
void set_error(const std::string& s) { g_last_error = s; }

// Allocation-failure injection for the failure tests (tf_debug_fail_alloc): when
// positive, the countdown-th later device allocation of any context fails as if the
// device were out of memory.  0: off.
static std::atomic<int> g_fail_alloc{0};
static bool inject_alloc_failure() {
  int v = g_fail_alloc.load();
  while (v > 0) {
    if (g_fail_alloc.compare_exchange_weak(v, v - 1)) return v == 1;
  }
  return false;
}

// ---------------------------------------------------------------------------
// kernels: shell pairs
// ---------------------------------------------------------------------------
__global__ void k_pair_prep(int n_pairs, PairRec* __restrict__ pairs, const double* __restrict__ xyz,
                            const int* __restrict__ shell_nprim, const int* __restrict__ shell_poff,
                            const double* __restrict__ exps, const double* __restrict__ coefs,
                            PrimPair* __restrict__ prim_full, PrimPair* __restrict__ prim_skip, double pair_cutoff) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_pairs) return;
  PairRec pr = pairs[p];
  const double* A = xyz + 3 * pr.atom_hi;
  const double* B = xyz + 3 * pr.atom_lo;
  pr.Rx = A[0] - B[0]; pr.Ry = A[1] - B[1]; pr.Rz = A[2] - B[2];
  const double r2 = pr.Rx * pr.Rx + pr.Ry * pr.Ry + pr.Rz * pr.Rz;
  const bool same = pr.atom_hi == pr.atom_lo;
  // Tonto's pair (a >= b by shell index) decides the operand order of the skip test
  const bool hi_is_a = pr.sh_hi >= pr.sh_lo;
  const int nh = shell_nprim[pr.sh_hi], nl = shell_nprim[pr.sh_lo];
  int k = 0, i = 0;
  for (int ih = 0; ih < nh; ++ih) {
    const double eh = exps[shell_poff[pr.sh_hi] + ih], ch = coefs[shell_poff[pr.sh_hi] + ih];
    for (int il = 0; il < nl; ++il, ++i) {
      const double el = exps[shell_poff[pr.sh_lo] + il], cl = coefs[shell_poff[pr.sh_lo] + il];
      const double zeta = eh + el, inv = 1.0 / zeta;
      const double ea = hi_is_a ? eh : el, eb = hi_is_a ? el : eh;
      const double prefac = same ? 1.0 : exp(-ea * (eb * r2) * inv);
      PrimPair q;
      q.Px = (eh * A[0] + el * B[0]) * inv;
      q.Py = (eh * A[1] + el * B[1]) * inv;
      q.Pz = (eh * A[2] + el * B[2]) * inv;
      q.zeta = zeta;
      q.PAx = q.Px - A[0]; q.PAy = q.Py - A[1]; q.PAz = q.Pz - A[2];
      q.half_zinv = 0.5 * inv;
      q.cc = ch * cl * inv * prefac;      // c_a c_b / zeta x prefactor: see PrimPair
      q.pad = 0.0;
      static_assert(sizeof(PrimPair) == 80, "primitive-pair record layout");
      prim_full[pr.full_off + i] = q;
      if (!same && !(prefac < pair_cutoff)) prim_skip[pr.skip_off + k++] = q;
    }
  }
  pr.n_skip = same ? 0 : k;
  pairs[p] = pr;
}

template <int LA, int LB>
__global__ void k_schwarz(const int* __restrict__ ids, int n, PairRec* __restrict__ pairs,
                          const PrimPair* __restrict__ prim_full, int spherical) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int p = ids[t];
  const PairRec pr = pairs[p];
  const double R[3] = {pr.Rx, pr.Ry, pr.Rz};
  constexpr int NA = ncart(LA), NB = ncart(LB);
  double I[NA][NB][NA * NB];
  quartet_integrals<LA, LB, LA, LB, double>(prim_full + pr.full_off, pr.n_full, prim_full + pr.full_off,
                                            pr.n_full, R, R, I);
  double m = 0.0;
  const bool sa = spherical && LA >= 2, sb = spherical && LB >= 2;
  const int MA = sa ? 2 * LA + 1 : NA, MB = sb ? 2 * LB + 1 : NB;
  for (int ma = 0; ma < MA; ++ma)
    for (int mb = 0; mb < MB; ++mb) {
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        const double ua = sa ? c_U[LA][a * (2 * LA + 1) + ma] : (a == ma ? 1.0 : 0.0);
        if (ua == 0.0) continue;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const double ub = sb ? c_U[LB][b * (2 * LB + 1) + mb] : (b == mb ? 1.0 : 0.0);
          if (ub == 0.0) continue;
#pragma unroll
          for (int c = 0; c < NA; ++c) {
            const double uc = sa ? c_U[LA][c * (2 * LA + 1) + ma] : (c == ma ? 1.0 : 0.0);
            if (uc == 0.0) continue;
#pragma unroll
            for (int d = 0; d < NB; ++d) {
              const double ud = sb ? c_U[LB][d * (2 * LB + 1) + mb] : (d == mb ? 1.0 : 0.0);
              s += ua * ub * uc * ud * I[a][b][c * NB + d];
            }
          }
        }
      }
      m = fmax(m, fabs(s));
    }
  pairs[p].imax = sqrt(m);
}

// ---------------------------------------------------------------------------
// kernels: per-build density preparation
// ---------------------------------------------------------------------------
struct BatchArgs {
  const MolInfo* mols;
  int n_mol;
  const long long* cmat_off;    // n_mol + 1 prefix offsets of the Cartesian blocks
  const long long* bmat_off;    // ... of the Tonto-basis blocks
  const long long* pmax_off;    // ... of the pair-maximum blocks
  const int* cart_shell;        // global Cartesian function -> global shell
  const int* cart_local;        // ... -> component within the shell
  const int* bf_shell;          // global basis function -> global shell
  const int* bf_local;
  const int* shell_l;
  const int* shell_first_bf;    // within the molecule
  const int* shell_cart;        // within the molecule
  const int* shell_nbf;
  int spherical;
};

// P_cart[p][q] = sum U_A[p][m] P[m][m'] U_B[q][m'] over the shell blocks, for every
// molecule of the batch (P, Pc: concatenated per-molecule blocks).
__global__ void k_density_to_cart(BatchArgs b, const double* __restrict__ P, const double* __restrict__ P2,
                                  double* __restrict__ Pc) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.cmat_off[b.n_mol]) return;
  const int m = find_mol(b.cmat_off, b.n_mol, t);
  const MolInfo mi = b.mols[m];
  const long long r = t - mi.cmat;
  const int p = (int)(r / mi.n_cart), q = (int)(r % mi.n_cart);
  const int sp = b.cart_shell[mi.cart0 + p], sq = b.cart_shell[mi.cart0 + q];
  const int ip = b.cart_local[mi.cart0 + p], iq = b.cart_local[mi.cart0 + q];
  const int lp = b.shell_l[sp], lq = b.shell_l[sq];
  const int fp = b.shell_first_bf[sp], fq = b.shell_first_bf[sq];
  const bool tp = b.spherical && lp >= 2, tq = b.spherical && lq >= 2;
  const double* Pm = P + mi.bmat;
  const double* Pm2 = P2 ? P2 + mi.bmat : nullptr;      // second density: the sum is transformed
  const int n_bf = mi.n_bf;
  double s = 0.0;
  if (!tp && !tq) {
    const size_t at = (size_t)(fq + iq) * n_bf + fp + ip;
    s = Pm[at] + (Pm2 ? Pm2[at] : 0.0);
  } else {
    const int mp = tp ? 2 * lp + 1 : 1, mq = tq ? 2 * lq + 1 : 1;
    for (int a = 0; a < mp; ++a) {
      const double ua = tp ? c_U[lp][ip * mp + a] : 1.0;
      const int ia = tp ? fp + a : fp + ip;
      if (ua == 0.0) continue;
      for (int bb = 0; bb < mq; ++bb) {
        const double ub = tq ? c_U[lq][iq * mq + bb] : 1.0;
        const int ib = tq ? fq + bb : fq + iq;
        const size_t at = (size_t)ib * n_bf + ia;
        s += ua * ub * (Pm[at] + (Pm2 ? Pm2[at] : 0.0));
      }
    }
  }
  Pc[t] = s;
}

// max |P(a,b)| over each shell pair block (Tonto basis) and, per molecule, the
// maximum over all pairs (an upper bound: the high word is rounded up).  A
// non-finite density element is left out of the maxima and raises *bad; the list
// passes then write no quartets and the host reports the density as invalid.
__global__ void k_pmax(BatchArgs b, const double* __restrict__ P, const double* __restrict__ P2,
                       double* __restrict__ pmax, unsigned long long* __restrict__ pglob,
                       unsigned long long* __restrict__ bad) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = b.pmax_off[b.n_mol];
  double mx = 0.0;
  int m = 0;
  bool nonfinite = false;
  if (t < total) {
    m = find_mol(b.pmax_off, b.n_mol, t);
    const MolInfo mi = b.mols[m];
    const long long r = t - mi.pmax;
    const int sa = mi.shell0 + (int)(r / mi.n_shell), sb = mi.shell0 + (int)(r % mi.n_shell);
    const int fa = b.shell_first_bf[sa], fb = b.shell_first_bf[sb], na = b.shell_nbf[sa], nb = b.shell_nbf[sb];
    const double* Pm = P + mi.bmat;
    const double* Pm2 = P2 ? P2 + mi.bmat : nullptr;    // unrestricted: of P_alpha + P_beta, as the reference
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < na; ++i) {
        const size_t at = (size_t)(fb + j) * mi.n_bf + fa + i;
        const double v = fabs(Pm[at] + (Pm2 ? Pm2[at] : 0.0));
        if (v <= 1.7976931348623157e308) mx = fmax(mx, v);
        else nonfinite = true;                           // NaN or infinity
      }
    pmax[t] = mx;
  }
  if (__any_sync(0xffffffffu, nonfinite) && (threadIdx.x & 31) == 0) atomicOr(bad, 1ull);
  // nonnegative doubles order like their bit patterns; reduce the high words
  // among the lanes of the same molecule, then one atomic per molecule and warp
  const unsigned hi = (unsigned)((unsigned long long)__double_as_longlong(mx) >> 32);
  const unsigned grp = __match_any_sync(0xffffffffu, t < total ? m : -1);
  const unsigned mhi = __reduce_max_sync(grp, hi);
  if (t < total && (threadIdx.x & 31) == __ffs(grp) - 1 && mhi)
    atomicMax(pglob + m, ((unsigned long long)mhi << 32) | 0xffffffffull);
}

// ---------------------------------------------------------------------------
// kernels: quartet lists
// ---------------------------------------------------------------------------
// Cost buckets of the primitive-quartet count npq: npq itself below 8, then quarter
// octaves (counts within a factor 1.19 share a bucket), so that the lanes of a warp
// loop over nearly the same number of primitive quartets.
constexpr int NCOST = 47;
constexpr int NBUCKET = 2 * NCOST;         // FP64 buckets, then FP32 buckets
static_assert(NBUCKET < 0xff, "bucket ids are recorded as bytes, 0xff = screened out");

// One (class pair, molecule) unit of the list builder.  Units of the same class
// pair are consecutive and form a group; the quartets of a group are one launch.
struct CPUnit {
  int p1, p2;                   // bra and ket pair classes
  int bra_off, ket_off;         // offsets of the molecule's class lists: the bra list in `csorted`
                                // (family units) or `sorted`, the ket list in `sorted`
  int n_ket, mol;
  int fam;                      // 1: the bra tasks are shell-pair families (see make_pair_families)
  int bra_xoff;                 // offset of the bra class's list in `sorted` (family units)
};

// Shell-pair families of a context (built on the host, see make_pair_families).
struct PairFamilies {
  std::vector<int> rep;                    // first member of each pair's family (pair ids)
  std::vector<int> index;                  // position of each pair in its family
  std::vector<int4> members;               // the family's member pair ids, -1 padded
  std::vector<int> n;                      // members of the pair's family
};

// Class lists of a context (built on the host, see make_class_lists).
struct ClassLists {
  std::vector<int> sorted;                 // pair ids by (molecule, class), band order, families contiguous
  std::vector<double> simax, sbmax;        // I_max of each position; largest family I_max of its band
  std::vector<int> cls_n, cls_off;         // [mol * NPAIRCLS + class]
  // the same lists with each shell-pair family collapsed to its first member
  std::vector<int> csorted;                // first member's pair id
  std::vector<double> cimax;               // the family's largest I_max
  std::vector<int> cxstart, cn;            // position of the first member in the class's `sorted` list; members
  std::vector<int> cls_cn, cls_coff;       // [mol * NPAIRCLS + class]
  std::vector<int> cls_maxm;               // largest family of the (molecule, class) list
};

struct ListArgs {
  const int2* tasks;            // (unit, bra position)
  long long t_base;             // tasks [t_base, n_tasks) are processed
  long long n_tasks;
  const CPUnit* units;
  const int* unit_group;        // unit -> group (class pair)
  const int* group_task0;       // first task of each group
  const int* sorted;            // pair ids, grouped by (molecule, class), in I_max bands (see setup_pairs)
  const double* sorted_imax;
  const double* sorted_bmax;    // largest I_max of the position's band (non-increasing)
  const int4* srec;             // screening record of each sorted position (see ScreenRec)
  const PairRec* pairs;
  const MolInfo* mols;
  const double* pmax;           // per-molecule n_shell x n_shell blocks
  const unsigned long long* pglob;   // per molecule
  double cutoff;
  const double* mol_cut;        // per-molecule cutoffs in place of `cutoff` (tf_set_molecule_cutoffs), or null
  double fp32_cut;              // 0: no FP32 quartets
  long long out_base;           // list index of out[0] (chunked list writes)
  long long out_cap;            // entries of out (writes beyond are dropped; the host sees the count)
  // screening record (optional): the counting pass stores one byte per candidate
  // ket (its bucket, or 0xff when screened out) at cand[cand_off[t] + j] and the
  // number of candidates it examined in task_len[t]; the writing pass then only
  // compacts, without screening again
  unsigned char* cand;
  const long long* cand_off;
  int* task_len;
  // captured builds: the list length (written by the scan); a list longer than
  // out_base + out_cap is not written at all (that build is redone), else null
  const long long* list_total;
  // raised by k_pmax when the density has a non-finite element: no quartets listed
  const unsigned long long* bad;
  // family units (CPUnit::fam): the collapsed bra lists, and per list entry the mask of
  // the bra family's members whose quartet with the ket passes the screen
  const int* csorted;
  const double* cimax;
  const int* cxstart;
  const int* cn;
  unsigned char* qmask;
  // the family tasks (ascending task indices) and, with the screening record, where
  // each one's member masks start in cmask (one byte per candidate ket)
  const int* fam_tasks;
  const long long* fam_coff;
  unsigned char* cmask;
};

// Screening record of a sorted pair position, 16 bytes read in list order (coalesced):
// x = local shell hi | local shell lo << 16, y = local atom hi | local atom lo << 16,
// z = primitive pairs without | with the pair cutoff << 16, w = pair id.
__device__ __forceinline__ int lo16(int v) { return v & 0xffff; }
__device__ __forceinline__ int hi16(int v) { return (int)((unsigned)v >> 16); }

__device__ __forceinline__ double quartet_bound(const ListArgs& a, const MolInfo& mi, const int4 b, const int4 k,
                                                double Ib, double Ik) {
  const double* pm = a.pmax + mi.pmax;
  const int ns = mi.n_shell;
  const int sa = lo16(b.x), sb = hi16(b.x), sc = lo16(k.x), sd = hi16(k.x);
  double m = fmax(pm[sa * ns + sb], pm[sc * ns + sd]);
  m = fmax(m, fmax(pm[sa * ns + sc], pm[sa * ns + sd]));
  m = fmax(m, fmax(pm[sb * ns + sc], pm[sb * ns + sd]));
  if (m < 1.0e-20) return -1.0;                 // TOL(20): skipped
  return m * Ib * Ik;
}

__device__ __forceinline__ int cost_bucket(const int4 b, const int4 k) {
  const int bh = lo16(b.y), bl = hi16(b.y), kh = lo16(k.y), kl = hi16(k.y);
  const bool any_same = bh == bl || kh == kl || bh == kh || bh == kl || bl == kh || bl == kl;
  const int npq = any_same ? lo16(b.z) * lo16(k.z) : hi16(b.z) * hi16(k.z);
  if (npq < 8) return npq > 0 ? npq - 1 : 0;
  const int lg = 31 - __clz(npq);                          // >= 3
  const int bucket = 7 + (lg - 3) * 4 + ((npq >> (lg - 2)) & 3);
  return bucket < NCOST ? bucket : NCOST - 1;
}

// Index of (task, bucket) in the count/offset arrays: group (class pair), then
// bucket, then task (molecule by molecule) -> each class pair's list is bucket-
// sorted across the whole batch, with all FP32 buckets after the FP64 ones.
__device__ __forceinline__ long long slot(const ListArgs& a, long long t, int g, int bucket) {
  const long long t0 = a.group_task0[g], nt = a.group_task0[g + 1] - t0;
  return t0 * NBUCKET + (long long)bucket * nt + (t - t0);
}

// Bra-family members a family task can hold (the largest fam_cap_l); the member
// mask of a list entry is one byte.
constexpr int FAM_LIST_MAX = 4;
static_assert(fam_cap_l(0, 0, 0, 0) <= FAM_LIST_MAX && fam_cap_l(2, 0, 0, 0) <= FAM_LIST_MAX,
              "family capacity beyond the list pass");

// One warp per bra task.  MODE 0: screen every candidate ket and count the
// survivors per bucket (and record the screening when a.cand is set); MODE 1:
// screen again and write the survivors; MODE 2: write the survivors from the
// recorded screening.  Lanes are grouped by bucket with one warp match per 32
// candidates; per-warp bucket counters live in shared memory.  FAM = false takes
// the tasks [t_base, n_tasks) and skips family tasks; FAM = true takes the family
// tasks a.fam_tasks[t_base .. n_tasks) (a bra family: every surviving ket carries
// the mask of the members whose quartet with it passes the screen, recorded in
// MODE 0 beside the bucket at cmask[fam_coff[w] + j]).
constexpr int LIST_THREADS = 256;

// (six resident blocks per SM: the pass waits on dependent L1 loads, so warps in
// flight matter more than registers; measured 0.5 ms faster per (H2O)32 build
// than four blocks, eight spill.  The family instantiation holds its members'
// screening data in registers and runs four: 0.45 ms faster than six, which
// spill.  Loading the next 32 candidates' records one chunk ahead measured
// 0.2 ms slower.)
template <int MODE, bool FAM>
__global__ void __launch_bounds__(LIST_THREADS, FAM ? 4 : 6) k_quartets(ListArgs a, long long* __restrict__ counts,
                                                           const long long* __restrict__ offsets,
                                                           int2* __restrict__ out) {
  __shared__ int scnt[LIST_THREADS / 32][NBUCKET];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long w = a.t_base + (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (w >= a.n_tasks) return;                    // uniform over the warp
  if (MODE != 0 && a.list_total && *a.list_total - a.out_base > a.out_cap) return;
  const long long t = FAM ? (long long)a.fam_tasks[w] : w;
  const int2 task = a.tasks[t];
  const CPUnit cp = a.units[task.x];
  if (!FAM && cp.fam) return;                    // the family instantiation's task
  for (int k = lane; k < NBUCKET; k += 32) scnt[warp][k] = 0;
  __syncwarp();
  const int g = a.unit_group[task.x];
  const int i = task.y;
  // a family task: the family's first member stands for the bra; its members sit at
  // xs .. xs + nm - 1 of the bra class's list
  const int bra = FAM ? a.csorted[cp.bra_off + i] : a.sorted[cp.bra_off + i];
  const int xs = FAM ? a.cxstart[cp.bra_off + i] : 0;
  const int nm = FAM ? a.cn[cp.bra_off + i] : 1;
  const int jend = (a.bad && *a.bad) ? 0 : ((cp.p1 == cp.p2) ? (FAM ? xs + nm : i + 1) : cp.n_ket);
  const long long coff = a.cand ? a.cand_off[t] : 0;
  const long long foff = FAM && a.cand ? a.fam_coff[w] : 0;
  const int len = MODE == 2 ? a.task_len[t] : jend;
  double Ib = 0.0, pg = 0.0, cut = a.cutoff;
  int4 b = make_int4(0, 0, 0, 0);
  MolInfo mi{};
  if (MODE != 2) {
    Ib = FAM ? a.cimax[cp.bra_off + i] : a.sorted_imax[cp.bra_off + i];
    b = FAM ? a.srec[cp.bra_xoff + xs] : a.srec[cp.bra_off + i];
    mi = a.mols[cp.mol];
    pg = __longlong_as_double((long long)a.pglob[cp.mol]);
    if (a.mol_cut) cut = a.mol_cut[cp.mol];
  }
  // the members' shells, Schwarz factors and bra density maxima, read once per task
  int mshell[FAM_LIST_MAX];
  double mib[FAM_LIST_MAX], mpab[FAM_LIST_MAX];
  if (FAM && MODE != 2) {
    const double* pm = a.pmax + mi.pmax;
#pragma unroll
    for (int m = 0; m < FAM_LIST_MAX; ++m) {
      mshell[m] = 0; mib[m] = 0.0; mpab[m] = 0.0;
      if (m < nm) {
        mshell[m] = a.srec[cp.bra_xoff + xs + m].x;
        mib[m] = a.sorted_imax[cp.bra_xoff + xs + m];
        mpab[m] = pm[lo16(mshell[m]) * mi.n_shell + hi16(mshell[m])];
      }
    }
  }
  // members of the bra family whose quartet with ket position j passes the screen
  // (inside the family's own block, p1 == p2, only members at or after the ket):
  // quartet_bound member by member, the ket's own density maximum read once
  auto family_mask = [&](int j, const int4 k, double Ik, double& maxb) {
    const double* pm = a.pmax + mi.pmax;
    const int ns = mi.n_shell;
    const int sc = lo16(k.x), sd = hi16(k.x);
    const double pcd = pm[sc * ns + sd];
    unsigned m_ok = 0;
    maxb = 0.0;
#pragma unroll
    for (int m = 0; m < FAM_LIST_MAX; ++m) {
      if (m >= nm || (cp.p1 == cp.p2 && j - xs > m)) continue;
      const int sa = lo16(mshell[m]), sb = hi16(mshell[m]);
      double p = fmax(mpab[m], pcd);
      p = fmax(p, fmax(pm[sa * ns + sc], pm[sa * ns + sd]));
      p = fmax(p, fmax(pm[sb * ns + sc], pm[sb * ns + sd]));
      if (p < 1.0e-20) continue;                  // TOL(20): skipped
      const double bound = p * mib[m] * Ik;
      if (bound > cut) { m_ok |= 1u << m; maxb = fmax(maxb, bound); }
    }
    return m_ok;
  };
  int scanned = 0;
  for (int j0 = 0; j0 < len; j0 += 32) {
    const int j = j0 + lane;
    bool beyond = false;
    int ket = 0, bucket = -1;
    unsigned fmask = 1;
    if (MODE == 2) {
      if (j < len) {
        const unsigned char cb = a.cand[coff + j];
        if (cb != 0xff) {
          bucket = cb;
          ket = a.sorted[cp.ket_off + j];
          if (FAM) fmask = a.cmask[foff + j];
        }
      }
    } else if (j < jend) {
      const double Ik = a.sorted_imax[cp.ket_off + j];
      const int4 k = a.srec[cp.ket_off + j];
      if (!(Ib * a.sorted_bmax[cp.ket_off + j] * pg > cut)) {
        beyond = true;                           // bands are in decreasing I_max: nothing further survives
      } else if (Ib * Ik * pg > cut) {
        ket = k.w;
        if (FAM) {
          double maxb;
          fmask = family_mask(j, k, Ik, maxb);
          if (fmask) bucket = cost_bucket(b, k) + (maxb < a.fp32_cut ? NCOST : 0);
        } else {
          const double bound = quartet_bound(a, mi, b, k, Ib, Ik);
          if (bound > cut) bucket = cost_bucket(b, k) + (bound < a.fp32_cut ? NCOST : 0);
        }
      }
      if (MODE == 0 && a.cand) {
        a.cand[coff + j] = bucket >= 0 ? (unsigned char)bucket : (unsigned char)0xff;
        if (FAM && bucket >= 0) a.cmask[foff + j] = (unsigned char)fmask;
      }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, bucket);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const int base = bucket >= 0 ? scnt[warp][bucket] : 0;
    __syncwarp();
    if (bucket >= 0 && rank == 0) scnt[warp][bucket] = base + __popc(peers);
    __syncwarp();
    if (MODE != 0 && bucket >= 0) {
      const long long pos = offsets[slot(a, t, g, bucket)] - a.out_base + base + rank;
      if (pos < a.out_cap) {
        out[pos] = make_int2(bra, ket);
        if (FAM) a.qmask[pos] = (unsigned char)fmask;
      }
    }
    scanned = j0 + 32;
    if (MODE != 2 && __any_sync(0xffffffffu, beyond)) break;
  }
  if (MODE == 0) {
    for (int k = lane; k < NBUCKET; k += 32) counts[slot(a, t, g, k)] = scnt[warp][k];
    if (a.cand && lane == 0) a.task_len[t] = min(scanned, jend);
  }
}

// ---------------------------------------------------------------------------
// kernel: ERIs + digestion (one thread per contracted quartet)
// ---------------------------------------------------------------------------
struct JKArgs {
  const int2* quartets;
  long long n;
  const PairRec* pairs;
  const PrimPair* prim_full;
  const PrimPair* prim_skip;
  const double* P;              // Cartesian density (per-molecule blocks)
  double* J;                    // Cartesian accumulators
  double* K;
  const MolInfo* mols;
  unsigned long long* prim_count;   // per quartet class
  // graph builds: the launch's quartets are list[range[0] - base, range[1] - base),
  // range read on the device and clamped to base + cap (quartets = list start)
  const long long* range;
  long long base, cap;
  const int4* jkrec;            // packed pair records (load_pair_jk)
  const double2* pairR;
  // unrestricted builds: the beta density and its J, K (else null); P, J, K above
  // are then the alpha ones.  want: bit 0 J, bit 1 K.
  const double* P2;
  double* J2;
  double* K2;
  int want;
  // classes with an f shell (k_jk_warp): per-warp global scratch and its warp count
  double* wscratch;
  long long wscratch_warps;
  // bra families (family groups): per list entry the members' mask, per pair its
  // family members; member quartets counted per class, FP64 buckets then FP32
  const unsigned char* qmask;
  const int4* fam_mem;
  unsigned long long* qcount;
  int fam;                      // bra-family capacity of the launch's kernel (1: none)
  int bucket32;                 // 1: the launch covers the FP32 buckets
  long long fx_lo;              // deterministic builds: offset of the lo words (fock_add), else 0
};


#ifndef TF_JK_MINB_N1
#define TF_JK_MINB_N1 5
#endif
#ifndef TF_JK_MINB
#define TF_JK_MINB 1
#endif
// Resident warps per SM, in units of four (bounds the registers per thread).
// Variant 0 leaves the registers to the compiler (one-root classes: 20 warps);
// variant 1 asks for more resident warps (24 for one root, 16 otherwise), at the
// price of fewer registers.  The autotuner times the variants per class.
template <int LA, int LB, int LC, int LD, int V>
constexpr int jk_min_blocks() {
  return Quartet<LA, LB, LC, LD>::NROOT == 1 ? ((V & 1) ? 6 : TF_JK_MINB_N1) : ((V & 1) ? 4 : TF_JK_MINB);
}
// Variant bits: 1 = more resident warps (see above); 2 = K atomics of lanes that hit
// the same element summed first (segmented warp sums over lanes of one bra); 4 =
// deterministic accumulation (fock_add), set by the context, not by the autotuner.
constexpr int JK_VARIANTS = 4;
// Threads per block: the resident warps of an SM form one block, so the SM holds
// one copy of the shared Rys/Boys grid and leaves the rest of its shared storage to
// the L1 cache, which serves the bra primitive records every iteration re-reads
// (measured on (H2O)32, (ps|ss): L1 hit rate 42% -> 62%, 14.8 -> 13.7 ms against
// five blocks of 128 threads).  A variant with no register bound uses up to 255
// registers: 256 threads per SM.
template <int LA, int LB, int LC, int LD, int V>
constexpr int jk_threads() {
  return jk_min_blocks<LA, LB, LC, LD, V>() == 1 ? 256 : 128 * jk_min_blocks<LA, LB, LC, LD, V>();
}

// Digestion of one quartet's Cartesian integrals I into J and K with the coincidence
// factor f (f = 0: the lane adds nothing but still takes part in the warp sums):
// bid is the bra pair (lanes of one bra are summed together), ob/oa the bra's and
// oc/od the ket's first Cartesian functions.
//   J(ab) += f sum_cd I P(cd);  J(cd) += f sum_ab I P(ab)  (per spin when unrestricted)
//   K(ac) += f sum_bd I P(bd);  K(ad) += f sum_bc I P(bc)
//   K(bc) += f sum_ad I P(ad);  K(bd) += f sum_ac I P(ac)
// The lists are bra-major, so the lanes of a warp usually share the bra pair: then
// J(ab) is summed over the warp and added once, and P(ab) is a broadcast.  Otherwise
// the lanes of one bra are neighbours (a bra's kets of one cost bucket are
// consecutive) and J(ab) is summed over each run of equal bras by a segmented warp
// scan, then added by the run's last lane.  Variant bit 2: the K rows a and b are the
// same for all lanes of one bra, and lanes whose kets share the c (or d) shell add to
// the same K elements; such lanes are neighbours (pair-id order), so each run of
// equal (bra, shell) keys is summed with a segmented warp scan and added once, by its
// last lane.  K(bc), K(bd) are summed over a's components in registers first.
template <int LA, int LB, int LC, int LD, int V>
__device__ __forceinline__ void digest_jk(const JKArgs& a, const MolInfo& mi,
                                          const double (&I)[ncart(LA)][ncart(LB)][ncart(LC) * ncart(LD)], double f,
                                          int bid, int oa, int ob, int oc, int od) {
  using Q = Quartet<LA, LB, LC, LD>;
  constexpr bool FX = (V & 4) != 0;
  const int lane = threadIdx.x & 31;
  const bool live = f != 0.0;
  const int n = mi.n_cart;
  const bool uni = __all_sync(0xffffffffu, bid == __shfl_sync(0xffffffffu, bid, 0));
  const unsigned lt_mask = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
  // (every lane executes the shuffle: none may be skipped by a short-circuit)
  const int upx = __shfl_up_sync(0xffffffffu, bid, 1);
  const bool headx = lane == 0 || bid != upx;
  const unsigned heada = __ballot_sync(0xffffffffu, headx);
  const int sega = 31 - __clz(heada & lt_mask);
  const bool taila = lane == 31 || ((heada >> (lane + 1)) & 1u);
  auto digest_j = [&](const double* __restrict__ P, double* __restrict__ Jm) {
    double Pcd[Q::NC][Q::ND];
#pragma unroll
    for (int c = 0; c < Q::NC; ++c)
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) Pcd[c][d] = __ldg(P + (size_t)(oc + c) * n + od + d);
#pragma unroll
    for (int ia = 0; ia < Q::NA; ++ia)
#pragma unroll
      for (int ib = 0; ib < Q::NB; ++ib) {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < Q::NC; ++c)
#pragma unroll
          for (int d = 0; d < Q::ND; ++d) s += I[ia][ib][c * Q::ND + d] * Pcd[c][d];
        s *= f;
        if (uni) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (lane == 0 && s != 0.0) fock_add<FX>(Jm + (size_t)(oa + ia) * n + ob + ib, s, a.fx_lo);
        } else {                       // idle lanes join the last run with s = 0
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane - o >= sega) s += t;
          }
          if (taila && s != 0.0) fock_add<FX>(Jm + (size_t)(oa + ia) * n + ob + ib, s, a.fx_lo);
        }
      }
    if (live) {
      double Pab[Q::NA][Q::NB];
#pragma unroll
      for (int ia = 0; ia < Q::NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < Q::NB; ++ib) Pab[ia][ib] = __ldg(P + (size_t)(oa + ia) * n + ob + ib);
#pragma unroll
      for (int c = 0; c < Q::NC; ++c)
#pragma unroll
        for (int d = 0; d < Q::ND; ++d) {
          double s = 0.0;
#pragma unroll
          for (int ia = 0; ia < Q::NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < Q::NB; ++ib) s += I[ia][ib][c * Q::ND + d] * Pab[ia][ib];
          fock_add<FX>(Jm + (size_t)(oc + c) * n + od + d, f * s, a.fx_lo);
        }
    }
  };
  if (a.want & 1) {                    // uniform over the warp (the J(ab) sums shuffle)
    digest_j(a.P + mi.cmat, a.J + mi.cmat);
    if (a.P2) digest_j(a.P2 + mi.cmat, a.J2 + mi.cmat);
  }
  constexpr bool SEG = (V & 2) != 0;
  int segc = lane, segd = lane;
  bool tailc = true, taild = true;
  if constexpr (SEG) {
    // (every lane executes both shuffles: none may be skipped by a short-circuit)
    const int upc = __shfl_up_sync(0xffffffffu, oc, 1), upd = __shfl_up_sync(0xffffffffu, od, 1);
    const unsigned headc = __ballot_sync(0xffffffffu, headx || oc != upc);
    const unsigned headd = __ballot_sync(0xffffffffu, headx || od != upd);
    segc = 31 - __clz(headc & lt_mask);
    segd = 31 - __clz(headd & lt_mask);
    tailc = lane == 31 || ((headc >> (lane + 1)) & 1u);
    taild = lane == 31 || ((headd >> (lane + 1)) & 1u);
  }
  auto kadd = [&](double* addr, double v, int seg, bool tail) {
    if constexpr (SEG) {
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane - o >= seg) v += t;
      }
      if (tail && v != 0.0) fock_add<FX>(addr, v, a.fx_lo);
    } else {
      fock_add<FX>(addr, v, a.fx_lo);
    }
  };
#define TF_KADD_C(addr, v) kadd((addr), (v), segc, tailc)
#define TF_KADD_D(addr, v) kadd((addr), (v), segd, taild)
  auto digest_k = [&](const double* __restrict__ P, double* __restrict__ Km) {
    double Pbd[Q::NB][Q::ND], Pbc[Q::NB][Q::NC];
    double Kbc[Q::NB][Q::NC], Kbd[Q::NB][Q::ND];
#pragma unroll
    for (int ib = 0; ib < Q::NB; ++ib) {
#pragma unroll
      for (int c = 0; c < Q::NC; ++c) Kbc[ib][c] = 0.0;
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) Kbd[ib][d] = 0.0;
    }
#pragma unroll
    for (int ib = 0; ib < Q::NB; ++ib) {
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) Pbd[ib][d] = __ldg(P + (size_t)(ob + ib) * n + od + d);
#pragma unroll
      for (int c = 0; c < Q::NC; ++c) Pbc[ib][c] = __ldg(P + (size_t)(ob + ib) * n + oc + c);
    }
#pragma unroll
    for (int ia = 0; ia < Q::NA; ++ia) {
      double Pad[Q::ND], Pac[Q::NC];
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) Pad[d] = __ldg(P + (size_t)(oa + ia) * n + od + d);
#pragma unroll
      for (int c = 0; c < Q::NC; ++c) Pac[c] = __ldg(P + (size_t)(oa + ia) * n + oc + c);
#pragma unroll
      for (int c = 0; c < Q::NC; ++c) {
        double s = 0.0;
#pragma unroll
        for (int ib = 0; ib < Q::NB; ++ib)
#pragma unroll
          for (int d = 0; d < Q::ND; ++d) s += I[ia][ib][c * Q::ND + d] * Pbd[ib][d];
        TF_KADD_C(Km + (size_t)(oa + ia) * n + oc + c, f * s);
      }
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) {
        double s = 0.0;
#pragma unroll
        for (int ib = 0; ib < Q::NB; ++ib)
#pragma unroll
          for (int c = 0; c < Q::NC; ++c) s += I[ia][ib][c * Q::ND + d] * Pbc[ib][c];
        TF_KADD_D(Km + (size_t)(oa + ia) * n + od + d, f * s);
      }
#pragma unroll
      for (int ib = 0; ib < Q::NB; ++ib) {
#pragma unroll
        for (int c = 0; c < Q::NC; ++c)
#pragma unroll
          for (int d = 0; d < Q::ND; ++d) Kbc[ib][c] += I[ia][ib][c * Q::ND + d] * Pad[d];
#pragma unroll
        for (int d = 0; d < Q::ND; ++d)
#pragma unroll
          for (int c = 0; c < Q::NC; ++c) Kbd[ib][d] += I[ia][ib][c * Q::ND + d] * Pac[c];
      }
    }
    // K(bc), K(bd): summed over the a components first, one atomic per element
#pragma unroll
    for (int ib = 0; ib < Q::NB; ++ib) {
#pragma unroll
      for (int c = 0; c < Q::NC; ++c) TF_KADD_C(Km + (size_t)(ob + ib) * n + oc + c, f * Kbc[ib][c]);
#pragma unroll
      for (int d = 0; d < Q::ND; ++d) TF_KADD_D(Km + (size_t)(ob + ib) * n + od + d, f * Kbd[ib][d]);
    }
  };
  // with segmented sums every lane takes part (idle lanes add f = 0)
  if ((SEG || live) && (a.want & 2)) {
    digest_k(a.P + mi.cmat, a.K + mi.cmat);
    if (a.P2) digest_k(a.P2 + mi.cmat, a.K2 + mi.cmat);
  }
#undef TF_KADD_C
#undef TF_KADD_D
}

// Per-class counters of a launch, summed over the warp: primitive quartets, and
// contracted (member) quartets of the FP64 or the FP32 buckets.
__device__ __forceinline__ void count_quartets(const JKArgs& a, int cls, unsigned long long nprim,
                                               unsigned long long nq) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nprim += __shfl_xor_sync(0xffffffffu, nprim, o);
    nq += __shfl_xor_sync(0xffffffffu, nq, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (nprim) atomicAdd(a.prim_count + cls, nprim);
    if (nq) atomicAdd(a.qcount + (a.bucket32 ? NQCLS : 0) + cls, nq);
  }
}

// One thread per contracted quartet.  MB = 1: a list entry is one quartet.  MB > 1
// (family groups): a list entry is a bra family (its first member's pair id) with a
// ket, and the mask of the members whose quartet passed the screen; the primitive
// loop runs once for all members (accumulate_esfs_fam), then each member quartet of
// the mask is transferred and digested with its own Cartesian offsets and
// coincidence factors (molecule.fock.foo:1296-1300).
template <int LA, int LB, int LC, int LD, typename T, int V, int MB>
__global__ void __launch_bounds__(jk_threads<LA, LB, LC, LD, V>(), 1) k_jk(JKArgs a) {
  using Q = Quartet<LA, LB, LC, LD>;
  using RS = RysSmem<Q::NROOT>;
  extern __shared__ double rys_tab[];
  RS::load(rys_tab);
  __syncthreads();
  unsigned long long nprim = 0, nquart = 0;
  const int2* quartets = a.quartets;
  long long nq = a.n;
  long long qoff = 0;
  resolve_range(a.range, a.base, a.cap, quartets, nq);
  qoff = quartets - a.quartets;                      // offset of this launch's entries in the mask array
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long n_pad = (nq + 31) / 32 * 32;      // whole warps stay in the loop together
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_pad; t += stride) {
    // lanes past the end repeat the last quartet with weight 0, so that whole warps
    // take part in the warp reductions below
    const bool active = t < nq;
    const long long te = active ? t : nq - 1;
    const int2 qd = quartets[te];
    const PairJK b = load_pair_jk(a.jkrec, a.pairR, qd.x);
    const PairJK k = load_pair_jk(a.jkrec, a.pairR, qd.y);
    const bool any_same = b.atom_hi == b.atom_lo || k.atom_hi == k.atom_lo || b.atom_hi == k.atom_hi ||
                          b.atom_hi == k.atom_lo || b.atom_lo == k.atom_hi || b.atom_lo == k.atom_lo;
    const PrimPair* bp = any_same ? a.prim_full + b.full_off : a.prim_skip + b.skip_off;
    const PrimPair* kp = any_same ? a.prim_full + k.full_off : a.prim_skip + k.skip_off;
    const int nbp = any_same ? b.n_full : b.n_skip;
    const int nkp = any_same ? k.n_full : k.n_skip;
    const double Rab[3] = {b.Rx, b.Ry, b.Rz};
    const double Rcd[3] = {k.Rx, k.Ry, k.Rz};
    const MolInfo mi = a.mols[b.mol];
    double fk = 1.0;
    if (k.same) fk *= 0.5;
    if constexpr (MB == 1) {
      if (active) { nprim += (unsigned long long)nbp * nkp; nquart += 1; }
      double f = active ? fk : 0.0;
      if (b.same) f *= 0.5;
      if (qd.x == qd.y) f *= 0.5;
      double I[Q::NA][Q::NB][Q::NC * Q::ND];
      quartet_integrals<LA, LB, LC, LD, T>(bp, nbp, kp, nkp, Rab, Rcd, I, rys_tab);
      digest_jk<LA, LB, LC, LD, V>(a, mi, I, f, qd.x, b.cart_hi, b.cart_lo, k.cart_hi, k.cart_lo);
    } else {
      const unsigned mask = active ? a.qmask[qoff + te] : 0u;
      nprim += (unsigned long long)nbp * nkp * __popc(mask);
      nquart += __popc(mask);
      const int4 mv = a.fam_mem[qd.x];
      const int mid[4] = {mv.x, mv.y, mv.z, mv.w};
      PairJK bm[MB];
      const PrimPair* bmp[MB];
#pragma unroll
      for (int m = 0; m < MB; ++m) {
        bm[m] = load_pair_jk(a.jkrec, a.pairR, mid[m] >= 0 ? mid[m] : qd.x);
        bmp[m] = mid[m] < 0 ? nullptr : (any_same ? a.prim_full + bm[m].full_off : a.prim_skip + bm[m].skip_off);
      }
      T esfs[MB][Q::NE][Q::NF];
      accumulate_esfs_fam<LA, LB, LC, LD, T, MB>(bp, nbp, kp, nkp, bmp, esfs, rys_tab);
#pragma unroll
      for (int m = 0; m < MB; ++m) {
        if (!__any_sync(0xffffffffu, (mask >> m) & 1u)) continue;      // uniform over the warp
        double f = ((mask >> m) & 1u) ? fk : 0.0;
        if (bm[m].same) f *= 0.5;
        if (mid[m] == qd.y) f *= 0.5;
        double I[Q::NA][Q::NB][Q::NC * Q::ND];
        hrr_quartet<LA, LB, LC, LD, T>(esfs[m], Rab, Rcd, I);
        digest_jk<LA, LB, LC, LD, V>(a, mi, I, f, mid[m] >= 0 ? mid[m] : qd.x, bm[m].cart_hi, bm[m].cart_lo,
                                     k.cart_hi, k.cart_lo);
      }
    }
  }
  count_quartets(a, qclass_id(LA, LB, LC, LD), nprim, nquart);
}

// ---------------------------------------------------------------------------
// kernel: Schwarz bounds of the classes above the thread kernels (one warp per pair)
// ---------------------------------------------------------------------------
constexpr int WARPS_PER_BLOCK = 2;

// Schwarz bound of any pair class with the warp path (one warp per pair).  gscr:
// per-warp scratch of WF_SCRATCH doubles in global memory (pair classes with an f
// shell), else null (shared memory, W_SMEM doubles per warp).
__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK) k_schwarz_warp(const int* __restrict__ ids, int n,
                                                                      PairRec* __restrict__ pairs,
                                                                      const PrimPair* __restrict__ prim_full,
                                                                      int spherical, int la, int lb,
                                                                      double* __restrict__ gscr) {
  extern __shared__ double smem_all[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* sm = gscr ? gscr + (size_t)(blockIdx.x * WARPS_PER_BLOCK + wib) * WF_SCRATCH : smem_all + wib * W_SMEM;
  const int i2d = gscr ? WF_I2D : W_I2D, wbuf = gscr ? WF_BUF : W_BUF;
  const WarpQuartet q = wq_make(la, lb, la, lb);
  const int na = ncart(la), nb = ncart(lb);
  const bool sa = spherical && la >= 2, sb = spherical && lb >= 2;
  const int MA = sa ? 2 * la + 1 : na, MB = sb ? 2 * lb + 1 : nb;
  const long long nwarps = (long long)gridDim.x * WARPS_PER_BLOCK;
  for (long long t = (long long)blockIdx.x * WARPS_PER_BLOCK + wib; t < n; t += nwarps) {
    const int p = ids[t];
    const PairRec pr = pairs[p];
    const double R[3] = {pr.Rx, pr.Ry, pr.Rz};
    double* I = nullptr;
    warp_quartet(q, prim_full + pr.full_off, pr.n_full, prim_full + pr.full_off, pr.n_full, R, R, sm, I, i2d, wbuf);
    double m = 0.0;
    for (int e = lane; e < MA * MB; e += 32) {
      const int ma = e / MB, mb = e % MB;
      double s = 0.0;
      for (int ia = 0; ia < na; ++ia) {
        const double ua = sa ? c_U[la][ia * (2 * la + 1) + ma] : (ia == ma ? 1.0 : 0.0);
        if (ua == 0.0) continue;
        for (int ib = 0; ib < nb; ++ib) {
          const double ub = sb ? c_U[lb][ib * (2 * lb + 1) + mb] : (ib == mb ? 1.0 : 0.0);
          if (ub == 0.0) continue;
          for (int ic = 0; ic < na; ++ic) {
            const double uc = sa ? c_U[la][ic * (2 * la + 1) + ma] : (ic == ma ? 1.0 : 0.0);
            if (uc == 0.0) continue;
            for (int id = 0; id < nb; ++id) {
              const double ud = sb ? c_U[lb][id * (2 * lb + 1) + mb] : (id == mb ? 1.0 : 0.0);
              s += ua * ub * uc * ud * I[((ia * nb + ib) * na + ic) * nb + id];
            }
          }
        }
      }
      m = fmax(m, fabs(s));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) pairs[p].imax = sqrt(m);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// kernel: J/K of the classes with an f shell, one warp per quartet with runtime
// angular momenta (the warp path above; shell1quartet.foo's generic make_esfs_XX,
// transfer_cd/transfer_ab, and the digestion of molecule.fock.foo:1322-1338).
// gscr: WF_SCRATCH doubles of global memory per warp of the grid.  Used for the
// FP64 and the FP32 buckets alike (f classes are always evaluated in FP64).
// ---------------------------------------------------------------------------
template <bool FX>
__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK) k_jk_warp(JKArgs a, int la, int lb, int lc, int ld,
                                                                 double* __restrict__ gscr) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const long long gw = (long long)blockIdx.x * WARPS_PER_BLOCK + wib;
  const long long nwarps = (long long)gridDim.x * WARPS_PER_BLOCK;
  double* sm = gscr + (size_t)gw * WF_SCRATCH;
  const WarpQuartet q = wq_make(la, lb, lc, ld);
  const int2* quartets = a.quartets;
  long long nq = a.n;
  resolve_range(a.range, a.base, a.cap, quartets, nq);
  const int NA = ncart(la), NB = ncart(lb), NC = ncart(lc), ND = ncart(ld), NCD = NC * ND;
  unsigned long long nprim = 0, nquart = 0;
  for (long long t = gw; t < nq; t += nwarps) {
    const int2 qd = quartets[t];
    const PairJK b = load_pair_jk(a.jkrec, a.pairR, qd.x);
    const PairJK k = load_pair_jk(a.jkrec, a.pairR, qd.y);
    const bool any_same = b.atom_hi == b.atom_lo || k.atom_hi == k.atom_lo || b.atom_hi == k.atom_hi ||
                          b.atom_hi == k.atom_lo || b.atom_lo == k.atom_hi || b.atom_lo == k.atom_lo;
    const PrimPair* bp = any_same ? a.prim_full + b.full_off : a.prim_skip + b.skip_off;
    const PrimPair* kp = any_same ? a.prim_full + k.full_off : a.prim_skip + k.skip_off;
    const int nbp = any_same ? b.n_full : b.n_skip;
    const int nkp = any_same ? k.n_full : k.n_skip;
    const double Rab[3] = {b.Rx, b.Ry, b.Rz};
    const double Rcd[3] = {k.Rx, k.Ry, k.Rz};
    double* I = nullptr;
    const int npq = warp_quartet(q, bp, nbp, kp, nkp, Rab, Rcd, sm, I, WF_I2D, WF_BUF);
    nprim += (unsigned long long)npq;
    double f = 1.0;
    if (b.same) f *= 0.5;
    if (k.same) f *= 0.5;
    if (qd.x == qd.y) f *= 0.5;
    const MolInfo mi = a.mols[b.mol];
    const int n = mi.n_cart;
    const int oa = b.cart_hi, ob = b.cart_lo, oc = k.cart_hi, od = k.cart_lo;
    auto digest = [&](const double* __restrict__ P, double* __restrict__ Jm, double* __restrict__ Km) {
      if (a.want & 1) {
        for (int e = lane; e < NA * NB; e += 32) {             // J(ab) = sum_cd I P(cd)
          const int ia = e / NB, ib = e - ia * NB;
          double s = 0.0;
          for (int c = 0; c < NC; ++c)
            for (int d = 0; d < ND; ++d) s += I[e * NCD + c * ND + d] * __ldg(P + (size_t)(oc + c) * n + od + d);
          fock_add<FX>(Jm + (size_t)(oa + ia) * n + ob + ib, f * s, a.fx_lo);
        }
        for (int e = lane; e < NCD; e += 32) {                 // J(cd) = sum_ab I P(ab)
          const int c = e / ND, d = e - c * ND;
          double s = 0.0;
          for (int ia = 0; ia < NA; ++ia)
            for (int ib = 0; ib < NB; ++ib) s += I[(ia * NB + ib) * NCD + e] * __ldg(P + (size_t)(oa + ia) * n + ob + ib);
          fock_add<FX>(Jm + (size_t)(oc + c) * n + od + d, f * s, a.fx_lo);
        }
      }
      if (a.want & 2) {
        for (int e = lane; e < NA * NC; e += 32) {             // K(ac) = sum_bd I P(bd)
          const int ia = e / NC, c = e - ia * NC;
          double s = 0.0;
          for (int ib = 0; ib < NB; ++ib)
            for (int d = 0; d < ND; ++d)
              s += I[(ia * NB + ib) * NCD + c * ND + d] * __ldg(P + (size_t)(ob + ib) * n + od + d);
          fock_add<FX>(Km + (size_t)(oa + ia) * n + oc + c, f * s, a.fx_lo);
        }
        for (int e = lane; e < NA * ND; e += 32) {             // K(ad) = sum_bc I P(bc)
          const int ia = e / ND, d = e - ia * ND;
          double s = 0.0;
          for (int ib = 0; ib < NB; ++ib)
            for (int c = 0; c < NC; ++c)
              s += I[(ia * NB + ib) * NCD + c * ND + d] * __ldg(P + (size_t)(ob + ib) * n + oc + c);
          fock_add<FX>(Km + (size_t)(oa + ia) * n + od + d, f * s, a.fx_lo);
        }
        for (int e = lane; e < NB * NC; e += 32) {             // K(bc) = sum_ad I P(ad)
          const int ib = e / NC, c = e - ib * NC;
          double s = 0.0;
          for (int ia = 0; ia < NA; ++ia)
            for (int d = 0; d < ND; ++d)
              s += I[(ia * NB + ib) * NCD + c * ND + d] * __ldg(P + (size_t)(oa + ia) * n + od + d);
          fock_add<FX>(Km + (size_t)(ob + ib) * n + oc + c, f * s, a.fx_lo);
        }
        for (int e = lane; e < NB * ND; e += 32) {             // K(bd) = sum_ac I P(ac)
          const int ib = e / ND, d = e - ib * ND;
          double s = 0.0;
          for (int ia = 0; ia < NA; ++ia)
            for (int c = 0; c < NC; ++c)
              s += I[(ia * NB + ib) * NCD + c * ND + d] * __ldg(P + (size_t)(oa + ia) * n + oc + c);
          fock_add<FX>(Km + (size_t)(ob + ib) * n + od + d, f * s, a.fx_lo);
        }
      }
    };
    digest(a.P + mi.cmat, a.J + mi.cmat, a.K + mi.cmat);
    if (a.P2) digest(a.P2 + mi.cmat, a.J2 + mi.cmat, a.K2 + mi.cmat);
    nquart += 1;
    __syncwarp();                        // the next quartet reuses the scratch
  }
  if (lane == 0) {
    if (nprim) atomicAdd(a.prim_count + qclass_id(la, lb, lc, ld), nprim);
    if (nquart) atomicAdd(a.qcount + (a.bucket32 ? NQCLS : 0) + qclass_id(la, lb, lc, ld), nquart);
  }
}

// ---------------------------------------------------------------------------
// kernel: fold, reflect and return to the Tonto basis
// ---------------------------------------------------------------------------
// J = 2 (J + J^T), K = K + K^T in the Cartesian basis, then to the Tonto basis
// (column-major), for every molecule of the batch.
__global__ void k_finalize(BatchArgs bt, const double* __restrict__ Jc, const double* __restrict__ Kc,
                           double* __restrict__ J, double* __restrict__ K, long long fx_lo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= bt.bmat_off[bt.n_mol]) return;
  const int m = find_mol(bt.bmat_off, bt.n_mol, t);
  const MolInfo mi = bt.mols[m];
  const long long r = t - mi.bmat;
  const int j = (int)(r / mi.n_bf), i = (int)(r % mi.n_bf);
  const int si = bt.bf_shell[mi.bf0 + i], sj = bt.bf_shell[mi.bf0 + j];
  const int mi_ = bt.bf_local[mi.bf0 + i], mj = bt.bf_local[mi.bf0 + j];
  const int li = bt.shell_l[si], lj = bt.shell_l[sj];
  const int ci = bt.shell_cart[si], cj = bt.shell_cart[sj];
  const bool ti = bt.spherical && li >= 2, tj = bt.spherical && lj >= 2;
  const double* Jm = Jc + mi.cmat;
  const double* Km = Kc + mi.cmat;
  const int nc = mi.n_cart;
  double sJ = 0.0, sK = 0.0;
  const int ni = ti ? ncart(li) : 1, nj = tj ? ncart(lj) : 1;
  for (int p = 0; p < ni; ++p) {
    const double up = ti ? c_U[li][p * (2 * li + 1) + mi_] : 1.0;
    if (up == 0.0) continue;
    const int cp = ti ? ci + p : ci + mi_;
    for (int q = 0; q < nj; ++q) {
      const double uq = tj ? c_U[lj][q * (2 * lj + 1) + mj] : 1.0;
      if (uq == 0.0) continue;
      const int cq = tj ? cj + q : cj + mj;
      const double w = up * uq;
      sJ += w * (fock_value(Jm, (size_t)cp * nc + cq, fx_lo) + fock_value(Jm, (size_t)cq * nc + cp, fx_lo));
      sK += w * (fock_value(Km, (size_t)cp * nc + cq, fx_lo) + fock_value(Km, (size_t)cq * nc + cp, fx_lo));
    }
  }
  J[t] = 2.0 * sJ;
  K[t] = sK;
}

__global__ void k_fock(long long n, const double* __restrict__ H, const double* __restrict__ J,
                       const double* __restrict__ K, double* __restrict__ F) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) F[t] = H[t] + J[t] - 0.5 * K[t];
}

// ---------------------------------------------------------------------------
// kernel: one-electron integrals S, T, V (Cartesian blocks), one thread per
// shell pair a >= b.  Overlap and kinetic by the Obara-Saika 1D recurrences,
// nuclear attraction by Rys quadrature (molecule.ints.foo:34-420 in meaning).
// ---------------------------------------------------------------------------
template <int N>
__device__ __forceinline__ void rys_eval_n(double x, double* u, double* w) {
  double uu[N], ww[N];
  rys_eval<N>(x, uu, ww);
#pragma unroll
  for (int i = 0; i < N; ++i) { u[i] = uu[i]; w[i] = ww[i]; }
}

// One thread per shell pair record (pairs of one molecule only); the Cartesian
// blocks go into the molecule's n_cart x n_cart slices of S, T, V.
__global__ void k_one_electron(long long n_pairs, const PairRec* __restrict__ pairs, const MolInfo* __restrict__ mols,
                               const double* __restrict__ xyz, const double* __restrict__ Z,
                               const int* __restrict__ shell_atom, const int* __restrict__ shell_l,
                               const int* __restrict__ shell_nprim, const int* __restrict__ shell_poff,
                               const int* __restrict__ shell_cart, const double* __restrict__ exps,
                               const double* __restrict__ coefs, double* __restrict__ S,
                               double* __restrict__ T, double* __restrict__ V) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_pairs) return;
  const PairRec pr = pairs[t];
  const MolInfo mi = mols[pr.mol];
  const int sa = pr.sh_hi, sb = pr.sh_lo;
  const int n_cart = mi.n_cart;
  S += mi.cmat;
  T += mi.cmat;
  V += mi.cmat;
  const int la = shell_l[sa], lb = shell_l[sb];
  const int na = ncart(la), nb = ncart(lb);
  const double* A = xyz + 3 * shell_atom[sa];
  const double* B = xyz + 3 * shell_atom[sb];
  const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double r2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  double s_c[100], t_c[100], v_c[100];     // na x nb, l <= 3
  for (int i = 0; i < na * nb; ++i) { s_c[i] = 0.0; t_c[i] = 0.0; v_c[i] = 0.0; }
  constexpr int LD = 6;                    // 1D table edge (l <= 3: i <= 4, j <= 5)
  const int nroot = (la + lb) / 2 + 1;
  for (int ia = 0; ia < shell_nprim[sa]; ++ia)
    for (int ib = 0; ib < shell_nprim[sb]; ++ib) {
      const double a = exps[shell_poff[sa] + ia], ca = coefs[shell_poff[sa] + ia];
      const double b = exps[shell_poff[sb] + ib], cb = coefs[shell_poff[sb] + ib];
      const double z = a + b, oo2z = 0.5 / z;
      const double Kab = exp(-a * b * r2 / z) * ca * cb;
      double P[3], PA[3], PB[3];
      for (int k = 0; k < 3; ++k) { P[k] = (a * A[k] + b * B[k]) / z; PA[k] = P[k] - A[k]; PB[k] = P[k] - B[k]; }
      double s1[3][LD][LD];
      for (int d = 0; d < 3; ++d) {
        s1[d][0][0] = 1.0;
        for (int i = 0; i <= la + 1; ++i)
          for (int j = 0; j <= lb + 2; ++j) {
            if (i == 0 && j == 0) continue;
            double v;
            if (i > 0) {
              v = PA[d] * s1[d][i - 1][j];
              if (i > 1) v += (i - 1) * oo2z * s1[d][i - 2][j];
              if (j > 0) v += j * oo2z * s1[d][i - 1][j - 1];
            } else {
              v = PB[d] * s1[d][0][j - 1];
              if (j > 1) v += (j - 1) * oo2z * s1[d][0][j - 2];
            }
            s1[d][i][j] = v;
          }
      }
      const double pre = Kab * pow(M_PI / z, 1.5);
      for (int i = 0; i < na; ++i) {
        const int g = ncart_upto(la - 1) + i;
        const int ix = c_comp[0][g], iy = c_comp[1][g], iz = c_comp[2][g];
        for (int j = 0; j < nb; ++j) {
          const int h = ncart_upto(lb - 1) + j;
          const int jx = c_comp[0][h], jy = c_comp[1][h], jz = c_comp[2][h];
          const double Sx = s1[0][ix][jx], Sy = s1[1][iy][jy], Sz = s1[2][iz][jz];
          auto kin = [&](int d, int i1, int j1) {
            double v = -2.0 * b * b * s1[d][i1][j1 + 2] + b * (2 * j1 + 1) * s1[d][i1][j1];
            if (j1 >= 2) v += -0.5 * j1 * (j1 - 1) * s1[d][i1][j1 - 2];
            return v;
          };
          s_c[i * nb + j] += pre * Sx * Sy * Sz;
          t_c[i * nb + j] += pre * (kin(0, ix, jx) * Sy * Sz + Sx * kin(1, iy, jy) * Sz + Sx * Sy * kin(2, iz, jz));
        }
      }
      for (int at = mi.atom0; at < mi.atom0 + mi.n_atom; ++at) {
        const double* C = xyz + 3 * at;
        const double PC[3] = {P[0] - C[0], P[1] - C[1], P[2] - C[2]};
        const double x = z * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        double u[4], w[4];
        if (nroot == 1) rys_eval_n<1>(x, u, w);
        else if (nroot == 2) rys_eval_n<2>(x, u, w);
        else if (nroot == 3) rys_eval_n<3>(x, u, w);
        else rys_eval_n<4>(x, u, w);
        const double pv = -Z[at] * 2.0 * M_PI / z * Kab;
        for (int r = 0; r < nroot; ++r) {
          double tab[3][4][4];
          for (int d = 0; d < 3; ++d) {
            const double c0 = PA[d] - u[r] * PC[d], bb = (1.0 - u[r]) * oo2z;
            double g[7], h[7][4];
            g[0] = 1.0;
            const int L = la + lb;
            if (L >= 1) g[1] = c0;
            for (int e = 1; e < L; ++e) g[e + 1] = c0 * g[e] + e * bb * g[e - 1];
            for (int e = 0; e <= L; ++e) h[e][0] = g[e];
            for (int j = 1; j <= lb; ++j)
              for (int e = 0; e <= L - j; ++e) h[e][j] = h[e + 1][j - 1] + AB[d] * h[e][j - 1];
            for (int i = 0; i <= la; ++i)
              for (int j = 0; j <= lb; ++j) tab[d][i][j] = h[i][j];
          }
          const double wv = pv * w[r];
          for (int i = 0; i < na; ++i) {
            const int g2 = ncart_upto(la - 1) + i;
            for (int j = 0; j < nb; ++j) {
              const int h2 = ncart_upto(lb - 1) + j;
              v_c[i * nb + j] += wv * tab[0][c_comp[0][g2]][c_comp[0][h2]] * tab[1][c_comp[1][g2]][c_comp[1][h2]] * tab[2][c_comp[2][g2]][c_comp[2][h2]];
            }
          }
        }
      }
    }
  const int oa = shell_cart[sa], ob = shell_cart[sb];
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      const size_t p = (size_t)(oa + i) * n_cart + ob + j, q = (size_t)(ob + j) * n_cart + oa + i;
      S[p] = S[q] = s_c[i * nb + j];
      T[p] = T[q] = t_c[i * nb + j];
      V[p] = V[q] = v_c[i * nb + j];
    }
}

// Cartesian symmetric matrices -> Tonto basis (column-major), no folding, for
// every molecule of the batch.
__global__ void k_cart_to_basis(BatchArgs bt, const double* __restrict__ Xc, double* __restrict__ X) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= bt.bmat_off[bt.n_mol]) return;
  const int m = find_mol(bt.bmat_off, bt.n_mol, t);
  const MolInfo mi = bt.mols[m];
  const long long r = t - mi.bmat;
  const int j = (int)(r / mi.n_bf), i = (int)(r % mi.n_bf);
  const int si = bt.bf_shell[mi.bf0 + i], sj = bt.bf_shell[mi.bf0 + j];
  const int mi_ = bt.bf_local[mi.bf0 + i], mj = bt.bf_local[mi.bf0 + j];
  const int li = bt.shell_l[si], lj = bt.shell_l[sj], ci = bt.shell_cart[si], cj = bt.shell_cart[sj];
  const bool ti = bt.spherical && li >= 2, tj = bt.spherical && lj >= 2;
  const int ni = ti ? ncart(li) : 1, nj = tj ? ncart(lj) : 1;
  const double* Xm = Xc + mi.cmat;
  double s = 0.0;
  for (int p = 0; p < ni; ++p) {
    const double up = ti ? c_U[li][p * (2 * li + 1) + mi_] : 1.0;
    if (up == 0.0) continue;
    const int cp = ti ? ci + p : ci + mi_;
    for (int q = 0; q < nj; ++q) {
      const double uq = tj ? c_U[lj][q * (2 * lj + 1) + mj] : 1.0;
      if (uq == 0.0) continue;
      s += up * uq * Xm[(size_t)cp * mi.n_cart + (tj ? cj + q : cj + mj)];
    }
  }
  X[t] = s;
}

// Single-molecule forms (shell pairs from the triangular index, one Cartesian
// block) used by the no-allocation entry point.
__global__ void k_one_electron_single(int n_shell, int n_atom, const double* __restrict__ xyz, const double* __restrict__ Z,
                               const int* __restrict__ shell_atom, const int* __restrict__ shell_l,
                               const int* __restrict__ shell_nprim, const int* __restrict__ shell_poff,
                               const int* __restrict__ shell_cart, const double* __restrict__ exps,
                               const double* __restrict__ coefs, int n_cart, double* __restrict__ S,
                               double* __restrict__ T, double* __restrict__ V) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n_shell * (n_shell + 1) / 2) return;
  int sa = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((long long)sa * (sa + 1) / 2 > t) --sa;
  while ((long long)(sa + 1) * (sa + 2) / 2 <= t) ++sa;
  const int sb = (int)(t - (long long)sa * (sa + 1) / 2);
  const int la = shell_l[sa], lb = shell_l[sb];
  const int na = ncart(la), nb = ncart(lb);
  const double* A = xyz + 3 * shell_atom[sa];
  const double* B = xyz + 3 * shell_atom[sb];
  const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double r2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  double s_c[100], t_c[100], v_c[100];     // na x nb, l <= 3
  for (int i = 0; i < na * nb; ++i) { s_c[i] = 0.0; t_c[i] = 0.0; v_c[i] = 0.0; }
  constexpr int LD = 6;                    // 1D table edge (l <= 3: i <= 4, j <= 5)
  const int nroot = (la + lb) / 2 + 1;
  for (int ia = 0; ia < shell_nprim[sa]; ++ia)
    for (int ib = 0; ib < shell_nprim[sb]; ++ib) {
      const double a = exps[shell_poff[sa] + ia], ca = coefs[shell_poff[sa] + ia];
      const double b = exps[shell_poff[sb] + ib], cb = coefs[shell_poff[sb] + ib];
      const double z = a + b, oo2z = 0.5 / z;
      const double Kab = exp(-a * b * r2 / z) * ca * cb;
      double P[3], PA[3], PB[3];
      for (int k = 0; k < 3; ++k) { P[k] = (a * A[k] + b * B[k]) / z; PA[k] = P[k] - A[k]; PB[k] = P[k] - B[k]; }
      double s1[3][LD][LD];
      for (int d = 0; d < 3; ++d) {
        s1[d][0][0] = 1.0;
        for (int i = 0; i <= la + 1; ++i)
          for (int j = 0; j <= lb + 2; ++j) {
            if (i == 0 && j == 0) continue;
            double v;
            if (i > 0) {
              v = PA[d] * s1[d][i - 1][j];
              if (i > 1) v += (i - 1) * oo2z * s1[d][i - 2][j];
              if (j > 0) v += j * oo2z * s1[d][i - 1][j - 1];
            } else {
              v = PB[d] * s1[d][0][j - 1];
              if (j > 1) v += (j - 1) * oo2z * s1[d][0][j - 2];
            }
            s1[d][i][j] = v;
          }
      }
      const double pre = Kab * pow(M_PI / z, 1.5);
      for (int i = 0; i < na; ++i) {
        const int g = ncart_upto(la - 1) + i;
        const int ix = c_comp[0][g], iy = c_comp[1][g], iz = c_comp[2][g];
        for (int j = 0; j < nb; ++j) {
          const int h = ncart_upto(lb - 1) + j;
          const int jx = c_comp[0][h], jy = c_comp[1][h], jz = c_comp[2][h];
          const double Sx = s1[0][ix][jx], Sy = s1[1][iy][jy], Sz = s1[2][iz][jz];
          auto kin = [&](int d, int i1, int j1) {
            double v = -2.0 * b * b * s1[d][i1][j1 + 2] + b * (2 * j1 + 1) * s1[d][i1][j1];
            if (j1 >= 2) v += -0.5 * j1 * (j1 - 1) * s1[d][i1][j1 - 2];
            return v;
          };
          s_c[i * nb + j] += pre * Sx * Sy * Sz;
          t_c[i * nb + j] += pre * (kin(0, ix, jx) * Sy * Sz + Sx * kin(1, iy, jy) * Sz + Sx * Sy * kin(2, iz, jz));
        }
      }
      for (int at = 0; at < n_atom; ++at) {
        const double* C = xyz + 3 * at;
        const double PC[3] = {P[0] - C[0], P[1] - C[1], P[2] - C[2]};
        const double x = z * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        double u[4], w[4];
        if (nroot == 1) rys_eval_n<1>(x, u, w);
        else if (nroot == 2) rys_eval_n<2>(x, u, w);
        else if (nroot == 3) rys_eval_n<3>(x, u, w);
        else rys_eval_n<4>(x, u, w);
        const double pv = -Z[at] * 2.0 * M_PI / z * Kab;
        for (int r = 0; r < nroot; ++r) {
          double tab[3][4][4];
          for (int d = 0; d < 3; ++d) {
            const double c0 = PA[d] - u[r] * PC[d], bb = (1.0 - u[r]) * oo2z;
            double g[7], h[7][4];
            g[0] = 1.0;
            const int L = la + lb;
            if (L >= 1) g[1] = c0;
            for (int e = 1; e < L; ++e) g[e + 1] = c0 * g[e] + e * bb * g[e - 1];
            for (int e = 0; e <= L; ++e) h[e][0] = g[e];
            for (int j = 1; j <= lb; ++j)
              for (int e = 0; e <= L - j; ++e) h[e][j] = h[e + 1][j - 1] + AB[d] * h[e][j - 1];
            for (int i = 0; i <= la; ++i)
              for (int j = 0; j <= lb; ++j) tab[d][i][j] = h[i][j];
          }
          const double wv = pv * w[r];
          for (int i = 0; i < na; ++i) {
            const int g2 = ncart_upto(la - 1) + i;
            for (int j = 0; j < nb; ++j) {
              const int h2 = ncart_upto(lb - 1) + j;
              v_c[i * nb + j] += wv * tab[0][c_comp[0][g2]][c_comp[0][h2]] * tab[1][c_comp[1][g2]][c_comp[1][h2]] * tab[2][c_comp[2][g2]][c_comp[2][h2]];
            }
          }
        }
      }
    }
  const int oa = shell_cart[sa], ob = shell_cart[sb];
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      const size_t p = (size_t)(oa + i) * n_cart + ob + j, q = (size_t)(ob + j) * n_cart + oa + i;
      S[p] = S[q] = s_c[i * nb + j];
      T[p] = T[q] = t_c[i * nb + j];
      V[p] = V[q] = v_c[i * nb + j];
    }
}

// Cartesian symmetric matrix -> Tonto basis (column-major), no folding.
__global__ void k_cart_to_basis_single(int n_bf, int n_cart, const double* __restrict__ Xc, const int* __restrict__ bf_shell,
                                const int* __restrict__ bf_local, const int* __restrict__ shell_l,
                                const int* __restrict__ shell_cart, int spherical, double* __restrict__ X) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n_bf * n_bf) return;
  const int j = (int)(t / n_bf), i = (int)(t % n_bf);
  const int si = bf_shell[i], sj = bf_shell[j], mi = bf_local[i], mj = bf_local[j];
  const int li = shell_l[si], lj = shell_l[sj], ci = shell_cart[si], cj = shell_cart[sj];
  const bool ti = spherical && li >= 2, tj = spherical && lj >= 2;
  const int ni = ti ? ncart(li) : 1, nj = tj ? ncart(lj) : 1;
  double s = 0.0;
  for (int p = 0; p < ni; ++p) {
    const double up = ti ? c_U[li][p * (2 * li + 1) + mi] : 1.0;
    if (up == 0.0) continue;
    const int cp = ti ? ci + p : ci + mi;
    for (int q = 0; q < nj; ++q) {
      const double uq = tj ? c_U[lj][q * (2 * lj + 1) + mj] : 1.0;
      if (uq == 0.0) continue;
      s += up * uq * Xc[(size_t)cp * n_cart + (tj ? cj + q : cj + mj)];
    }
  }
  X[(size_t)j * n_bf + i] = s;
}

// ---------------------------------------------------------------------------
// host: spherical matrices (Helgaker-Jorgensen-Olsen real solid harmonics,
// the recurrence of gaussian_data.foo:1143-1290; columns m = 0,+1,-1,+2,...)
// ---------------------------------------------------------------------------
std::vector<double> spherical_matrix(int l) {
  auto col = [](int m) { return m == 0 ? 0 : (m > 0 ? 2 * m - 1 : -2 * m); };
  std::vector<std::vector<double>> S(l + 1);
  S[0] = {1.0};
  for (int L = 0; L < l; ++L) {
    const int nsL = 2 * L + 1, nsP = 2 * L + 3;
    std::vector<double> nx((size_t)ncart(L + 1) * nsP, 0.0);
    const double top = 2 * L + 1;
    const double fac = std::sqrt((L == 0 ? 2.0 : 1.0) * top / (top + 1));
    const double del = L == 0 ? 0.0 : 1.0;
    for (int i = 0; i < ncart(L); ++i) {
      const int X = CT.x[CT.first[L] + i], Y = CT.y[CT.first[L] + i], Z = CT.z[CT.first[L] + i];
      const int ix = CT.idx[X + 1][Y][Z], iy = CT.idx[X][Y + 1][Z], iz = CT.idx[X][Y][Z + 1];
      const double vp = fac * S[L][i * nsL + col(L)], vm = fac * S[L][i * nsL + col(-L)] * del;
      nx[ix * nsP + col(L + 1)] += vp;
      nx[iy * nsP + col(L + 1)] -= vm;
      nx[ix * nsP + col(-L - 1)] += vm;
      nx[iy * nsP + col(-L - 1)] += vp;
      for (int M = -L; M <= L; ++M)
        nx[iz * nsP + col(M)] += top / std::sqrt((double)(L + M + 1) * (L - M + 1)) * S[L][i * nsL + col(M)];
    }
    if (L >= 1) {
      const int nsM = 2 * L - 1;
      for (int i = 0; i < ncart(L - 1); ++i) {
        const int X = CT.x[CT.first[L - 1] + i], Y = CT.y[CT.first[L - 1] + i], Z = CT.z[CT.first[L - 1] + i];
        const int ix = CT.idx[X + 2][Y][Z], iy = CT.idx[X][Y + 2][Z], iz = CT.idx[X][Y][Z + 2];
        for (int M = -L + 1; M <= L - 1; ++M) {
          const double v = std::sqrt((double)(L + M) * (L - M) / ((double)(L + M + 1) * (L - M + 1))) *
                           S[L - 1][i * nsM + col(M)];
          nx[ix * nsP + col(M)] -= v;
          nx[iy * nsP + col(M)] -= v;
          nx[iz * nsP + col(M)] -= v;
        }
      }
    }
    S[L + 1] = nx;
  }
  return S[l];
}

// Host copies of the constant tables, built once when the library is loaded.
struct HostTables {
  double U[4][70];
  unsigned char comp[3][NCOMP_ALL];
  unsigned char cidx[LCOMP + 1][LCOMP + 1][LCOMP + 1];
  HostTables() {
    std::memset(U, 0, sizeof(U));
    for (int l = 0; l <= 3; ++l) {
      std::vector<double> m = spherical_matrix(l);
      std::copy(m.begin(), m.end(), U[l]);
    }
    std::memset(cidx, 0, sizeof(cidx));
    for (int g = 0; g < NCOMP_ALL; ++g) {
      comp[0][g] = (unsigned char)CT.x[g]; comp[1][g] = (unsigned char)CT.y[g]; comp[2][g] = (unsigned char)CT.z[g];
      cidx[CT.x[g]][CT.y[g]][CT.z[g]] = (unsigned char)CT.idx[CT.x[g]][CT.y[g]][CT.z[g]];
    }
  }
};
static const HostTables g_tables;

// ---------------------------------------------------------------------------
// host: device buffer
// ---------------------------------------------------------------------------
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DBuf() { if (p) cudaFree(p); }
  cudaError_t reserve(size_t m) {
    if (m <= n && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (inject_alloc_failure()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(m, 1) * sizeof(T));
    if (e == cudaSuccess) n = std::max<size_t>(m, 1);
    return e;
  }
};

// Per-context host staging in pinned memory (group offsets and primitive counts
// read back after a build; pinned so that a captured graph can copy into them).
struct PinnedStage {
  long long* goff = nullptr;                 // 3 per group, then the list length
  unsigned long long* pc = nullptr;          // tf::BUILD_COUNTERS (see there)
  size_t n_goff = 0;
  ~PinnedStage() {
    if (goff) cudaFreeHost(goff);
    if (pc) cudaFreeHost(pc);
  }
  cudaError_t reserve(size_t ng3) {
    if (!pc) {
      cudaError_t e = cudaMallocHost(&pc, tf::BUILD_COUNTERS * sizeof(unsigned long long));
      if (e != cudaSuccess) return e;
    }
    if (ng3 <= n_goff && goff) return cudaSuccess;
    if (goff) cudaFreeHost(goff);
    goff = nullptr;
    n_goff = 0;
    cudaError_t e = cudaMallocHost(&goff, std::max<size_t>(ng3, 1) * sizeof(long long));
    if (e == cudaSuccess) n_goff = std::max<size_t>(ng3, 1);
    return e;
  }
};

}  // namespace tf

// ===========================================================================
// context
// ===========================================================================
struct tf_ctx {
  tf_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  cudaEvent_t order_ev = nullptr;                        // orders the context stream with a caller's stream
  // molecules (a single-molecule context is a batch of one)
  int n_mol = 0, spherical = 0;
  std::vector<tf::MolInfo> mols;
  std::vector<long long> cmat_off, bmat_off, pmax_off;   // n_mol + 1 prefix offsets
  std::vector<long long> mol_pair0;                      // first pair of each molecule (n_mol + 1)
  int n_atom = 0, n_shell = 0, n_cart = 0, n_bf = 0;     // totals
  std::vector<double> xyz;
  std::vector<int> shell_atom, shell_l, shell_nprim, shell_first_bf, shell_poff, shell_cart, shell_nbf;
  std::vector<double> exps, coefs;
  // pairs and list units
  long long n_pairs = 0;
  std::vector<tf::PairRec> pairs_h;
  std::vector<int> pair_cls;
  std::vector<int> cls_n, cls_off;                       // [mol * NPAIRCLS + class]
  tf::ClassLists lists;                                  // host copy of the sorted class lists
  std::vector<double> shard_cost;                        // estimated FLOPs of every shard (tf_set_shard)
  std::vector<tf::CPUnit> units;
  std::vector<int> unit_group, group_task0;
  std::vector<int2> group_cls;                           // (bra class, ket class) of each group
  std::vector<int> group_fam;                            // bra-family capacity of each group's kernel (1: none)
  tf::PairFamilies fams;                                 // shell-pair families (host)
  long long n_tasks = 0;
  std::vector<int> fam_tasks;                            // family tasks, ascending
  long long list_budget = 1LL << 30;                     // quartets per list chunk (8 B each)
  // screening record: one byte per candidate (bra task, ket) pair, when it fits
  bool use_cand = false;
  long long cand_budget = 12LL << 30;                    // bytes
  int shard_index = 0, shard_count = 1;                  // round-robin share of the bra tasks
  bool geometry_ready = false;
  // device
  tf::DBuf<tf::MolInfo> d_mols;
  tf::DBuf<long long> d_cmat_off, d_bmat_off, d_pmax_off;
  tf::DBuf<double> d_xyz, d_exps, d_coefs, d_P, d_Pc, d_Jc, d_Kc, d_J, d_K, d_H, d_pmax, d_sorted_imax, d_sorted_bmax;
  tf::DBuf<double> d_PcB, d_JcB, d_KcB, d_Pb, d_Jb, d_Kb;  // unrestricted builds (allocated on first use)
  tf::DBuf<double> d_wscratch;                             // f shells: per-warp scratch of the warp path
  tf::DBuf<int> d_csorted, d_cxstart, d_cn;                // collapsed (family) class lists
  tf::DBuf<double> d_cimax;
  tf::DBuf<int4> d_fam_mem;                                // family members of every pair
  tf::DBuf<unsigned char> d_qmask;                         // per list entry: the bra members it holds
  tf::DBuf<unsigned long long> d_qcount;                   // member quartets per class, FP64 then FP32
  long long wscratch_warps = 0;
  tf::DBuf<int> d_shell_atom, d_shell_nprim, d_shell_poff, d_shell_l, d_shell_first_bf, d_shell_nbf, d_shell_cart;
  tf::DBuf<int> d_cart_shell, d_cart_local, d_bf_shell, d_bf_local, d_sorted, d_schwarz_ids;
  tf::DBuf<tf::PairRec> d_pairs;
  tf::DBuf<tf::PrimPair> d_prim_full, d_prim_skip;
  tf::DBuf<int2> d_tasks, d_quartets;
  tf::DBuf<tf::CPUnit> d_units;
  tf::DBuf<int> d_unit_group, d_group_task0, d_task_len;
  tf::DBuf<unsigned char> d_cand;
  tf::DBuf<int> d_fam_tasks;                             // family tasks (k_quartets<.., true>)
  tf::DBuf<long long> d_fam_coff;                        // their member masks in d_cmask
  tf::DBuf<unsigned char> d_cmask;                       // recorded member mask per candidate ket
  tf::DBuf<int4> d_srec, d_jkrec;
  tf::DBuf<double2> d_pairR;
  tf::DBuf<long long> d_task_cand_off;
  tf::DBuf<long long> d_counts, d_offsets, d_group_offsets;
  tf::DBuf<double> d_mol_cut;                            // per-molecule cutoffs (tf_set_molecule_cutoffs)
  bool use_mol_cut = false;
  tf::DBuf<unsigned long long> d_pglob, d_prim_count;
  tf::DBuf<unsigned char> d_scan_tmp;
  std::vector<cudaEvent_t> cls_ev;                       // start and end of each group's launches
  std::vector<tf_class_stats> cls_stats;
  std::vector<double> max_I_tonto;                       // per molecule, Tonto pair order
  tf_stats stats{};
  // graph builds
  bool use_graph = true;
  long long graph_cap = 0;                               // list entries a captured build may use
  cudaGraphExec_t graph_exec = nullptr;
  const double* graph_key_P = nullptr;
  double* graph_key_J = nullptr;
  double* graph_key_K = nullptr;
  bool graph_key_mixed = false;
  int graph_key_want = 3;
  double graph_key_cutoff = 0.0;
  bool graph_key_mol_cut = false;             // the captured list passes read per-molecule cutoffs
  int graph_kernels = 0;
  // class schedule (autotuned): graph branches and the branch of each class pair
  int sched_streams = 1;
  std::vector<int> sched_stream_of;
  std::vector<int> cls_variant;                          // launch-bound variant of each class pair's kernel
  std::vector<cudaStream_t> side;                        // branch streams besides the context stream
  cudaEvent_t fork_ev = nullptr;
  std::vector<cudaEvent_t> join_ev;
  cudaEvent_t list_fork_ev = nullptr, list_join_ev = nullptr;   // family list pass on side[0]
  tf_tune tune{};                                        // last autotuner result
  tf::PinnedStage pin_obj;
  tf::PinnedStage* pin = &pin_obj;
};

namespace tf {

static void drop_graph(tf_ctx* c) {
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  c->graph_exec = nullptr;
  c->graph_key_P = nullptr;
}

static int set_device(tf_ctx* c) {
  TF_CUDA(cudaSetDevice(c->device));
  return TF_OK;
}

static BatchArgs batch_args(tf_ctx* c) {
  return BatchArgs{c->d_mols.p,       c->n_mol,          c->d_cmat_off.p,     c->d_bmat_off.p,
                   c->d_pmax_off.p,   c->d_cart_shell.p, c->d_cart_local.p,   c->d_bf_shell.p,
                   c->d_bf_local.p,   c->d_shell_l.p,    c->d_shell_first_bf.p, c->d_shell_cart.p,
                   c->d_shell_nbf.p,  c->spherical};
}

// gather (start, FP32 start, end) of every group's quartet range, and the list
// length at out[3 n_groups].  A list longer than cap (the buffer of a captured
// build) gets empty ranges: that build's class launches do nothing, and the host,
// seeing the length, redoes the build with a larger buffer.
__global__ void k_group_offsets(int n_groups, const int* __restrict__ group_task0, const long long* __restrict__ offs,
                                long long cap, long long* __restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_groups) return;
  const long long total = offs[(long long)group_task0[n_groups] * NBUCKET];
  if (g == 0) out[3 * n_groups] = total;
  if (total > cap) {
    out[3 * g] = out[3 * g + 1] = out[3 * g + 2] = 0;
    return;
  }
  const long long t0 = group_task0[g], t1 = group_task0[g + 1];
  out[3 * g] = offs[t0 * NBUCKET];
  out[3 * g + 1] = offs[t0 * NBUCKET + (long long)NCOST * (t1 - t0)];
  out[3 * g + 2] = offs[t1 * NBUCKET];
}

// Kernel variant of each class pair chosen by the last tf_autotune on a device; new
// contexts on that device start from it (class pairs are enumerated alike in every
// context).
static std::mutex g_variant_mutex;
static std::map<int, std::vector<int>> g_variant_cache;

// ---------------------------------------------------------------------------
// host planning, no device calls: shell-pair records, the class lists in I_max
// bands and the bra tasks with their shard assignment.  Shared by the contexts
// and by tf_plan_shards.
// ---------------------------------------------------------------------------
double class_flops(int la, int lb, int lc, int ld, double nq, double npq);

// Pair records of one molecule (Tonto pair order ab = a(a+1)/2 + b, a >= b), the
// higher-l shell first; shell arrays global over the context, shells of molecule m
// at [shell0, shell0 + n_shell).  Primitive-pair offsets continue from *full_tot.
static void append_pair_records(int m, int shell0, int n_shell, const int* shell_l, const int* shell_atom,
                                const int* shell_cart, const int* shell_nprim, long long* full_tot,
                                std::vector<PairRec>& pairs, std::vector<int>& pair_cls) {
  for (int la = 0; la < n_shell; ++la)
    for (int lb = 0; lb <= la; ++lb) {
      const int a = shell0 + la, b = shell0 + lb;
      PairRec p{};
      const bool a_hi = shell_l[a] >= shell_l[b];
      p.sh_hi = a_hi ? a : b;
      p.sh_lo = a_hi ? b : a;
      p.atom_hi = shell_atom[p.sh_hi];
      p.atom_lo = shell_atom[p.sh_lo];
      p.cart_hi = shell_cart[p.sh_hi];
      p.cart_lo = shell_cart[p.sh_lo];
      p.n_full = shell_nprim[a] * shell_nprim[b];
      p.full_off = (int)*full_tot;
      p.skip_off = (int)*full_tot;
      *full_tot += p.n_full;
      p.mol = m;
      p.tonto_ab = la * (la + 1) / 2 + lb;
      pairs.push_back(p);
      pair_cls.push_back(pair_class(shell_l[p.sh_hi], shell_l[p.sh_lo]));
    }
}

// Shell-pair families.  Two shells of one atom with the same l and the same
// primitive exponents (cc-pVDZ's oxygen 1s and 2s: eight exponents, two
// contractions; Tonto stores them as two segmented shells) form a shell family.
// The pairs (a', b') with a' in the family of a and b' in that of b then have the
// same positioned primitive pairs, up to the contraction coefficients, so a kernel
// can evaluate each primitive quartet once for all of them and weight it with
// each member's coefficients.  Families have at most two shells (consecutive
// members of a larger group pair up), a pair family at most four members.

// shell_* arrays global over the context; prim_off[s]: first primitive of shell s in exps.
static void make_pair_families(const std::vector<PairRec>& pairs, int n_mol, const std::vector<long long>& mol_pair0,
                               const int* mol_shell0, const int* mol_nshell, const int* shell_l, const int* shell_atom,
                               const int* shell_nprim, const int* prim_off, const double* exps, PairFamilies& F) {
  const size_t np = pairs.size();
  F.rep.resize(np);
  F.index.assign(np, 0);
  F.members.assign(np, make_int4(-1, -1, -1, -1));
  F.n.assign(np, 1);
  for (size_t p = 0; p < np; ++p) { F.rep[p] = (int)p; F.members[p].x = (int)p; }
  auto same_exps = [&](int s, int t) {
    if (shell_l[s] != shell_l[t] || shell_atom[s] != shell_atom[t] || shell_nprim[s] != shell_nprim[t]) return false;
    for (int k = 0; k < shell_nprim[s]; ++k)
      if (exps[prim_off[s] + k] != exps[prim_off[t] + k]) return false;
    return true;
  };
  for (int m = 0; m < n_mol; ++m) {
    const int s0 = mol_shell0[m], ns = mol_nshell[m];
    std::vector<int> partner(ns, -1), done(ns, 0);
    for (int u = 0; u < ns; ++u) {
      if (done[u]) continue;
      std::vector<int> grp{u};
      for (int v = u + 1; v < ns; ++v)
        if (!done[v] && same_exps(s0 + u, s0 + v)) grp.push_back(v);
      for (int v : grp) done[v] = 1;
      for (size_t k = 0; k + 1 < grp.size(); k += 2) { partner[grp[k]] = grp[k + 1]; partner[grp[k + 1]] = grp[k]; }
    }
    const long long base = mol_pair0[m];
    auto pid = [&](int x, int y) { const int hi = std::max(x, y), lo = std::min(x, y); return base + (long long)hi * (hi + 1) / 2 + lo; };
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b <= a; ++b) {
        const long long p = pid(a, b);
        if (partner[a] < 0 && partner[b] < 0) continue;
        std::vector<long long> mem;
        for (int x : {a, partner[a]})
          for (int y : {b, partner[b]})
            if (x >= 0 && y >= 0) mem.push_back(pid(x, y));
        std::sort(mem.begin(), mem.end());
        mem.erase(std::unique(mem.begin(), mem.end()), mem.end());
        if (mem.size() < 2 || mem.size() > 4) continue;
        // members must share the positioned primitive pairs: the same atoms, angular
        // momenta and exponents of the higher-l shell and of the other shell
        const PairRec& r0 = pairs[mem[0]];
        bool ok = true;
        for (long long q : mem) {
          const PairRec& rq = pairs[q];
          if (rq.atom_hi != r0.atom_hi || rq.atom_lo != r0.atom_lo || !same_exps(rq.sh_hi, r0.sh_hi) ||
              !same_exps(rq.sh_lo, r0.sh_lo) || rq.n_full != r0.n_full)
            ok = false;
        }
        if (!ok) continue;
        int4 mv = make_int4(-1, -1, -1, -1);
        int* mp = &mv.x;
        for (size_t k = 0; k < mem.size(); ++k) mp[k] = (int)mem[k];
        for (size_t k = 0; k < mem.size(); ++k) {
          F.rep[mem[k]] = (int)mem[0];
          F.index[mem[k]] = (int)k;
          F.members[mem[k]] = mv;
          F.n[mem[k]] = (int)mem.size();
        }
      }
  }
}

// Each (molecule, class) list in I_max bands (half decades, largest first) and by
// pair id inside a band, the members of a family next to each other (the family
// placed by its largest I_max).  The list kernels stop a bra's ket scan at the first
// band whose largest I_max fails the screen, and the pair-id order inside a band
// puts neighbouring shells on neighbouring lanes, so the ERI kernels' pair,
// primitive, density and Fock accesses of a warp fall on few cache lines.  The
// collapsed lists hold one entry per family.
static void make_class_lists(const std::vector<PairRec>& pairs, const std::vector<int>& pair_cls, int n_mol,
                             const PairFamilies& F, ClassLists& L) {
  const long long n_pairs = (long long)pairs.size();
  L = ClassLists{};
  L.cls_n.assign((size_t)n_mol * NPAIRCLS, 0);
  L.cls_off.assign((size_t)n_mol * NPAIRCLS, 0);
  L.cls_cn.assign((size_t)n_mol * NPAIRCLS, 0);
  L.cls_coff.assign((size_t)n_mol * NPAIRCLS, 0);
  L.cls_maxm.assign((size_t)n_mol * NPAIRCLS, 1);
  std::vector<std::vector<int>> lists((size_t)n_mol * NPAIRCLS);
  for (long long p = 0; p < n_pairs; ++p)
    if (F.rep[p] == p) lists[(size_t)pairs[p].mol * NPAIRCLS + pair_cls[p]].push_back((int)p);
  std::vector<double> fmax(n_pairs, 0.0);             // largest I_max of each family (at its first member)
  std::vector<int> band_of(n_pairs);                  // half-decade band of each family
  for (long long p = 0; p < n_pairs; ++p) {
    const int r = F.rep[p];
    fmax[r] = std::max(fmax[r], pairs[p].imax);
  }
  for (long long p = 0; p < n_pairs; ++p) {
    const double v = fmax[p];
    band_of[p] = v > 0.0 ? (int)std::floor(2.0 * std::log10(v)) : -1000000;
  }
  L.sorted.reserve(n_pairs);
  L.simax.reserve(n_pairs);
  L.sbmax.reserve(n_pairs);
  L.csorted.reserve(n_pairs);
  L.cimax.reserve(n_pairs);
  L.cxstart.reserve(n_pairs);
  L.cn.reserve(n_pairs);
  std::vector<int> cnt, tmp;
  for (size_t q = 0; q < lists.size(); ++q) {
    auto& v = lists[q];
    // bands in decreasing order, pair ids increasing inside a band: the lists were
    // filled in increasing pair id, so a stable counting sort over the few bands of
    // the list gives that order (families without a bound, band -1000000, last)
    if (v.size() > 1) {
      int bhi = -1000000, blo = 1000000;
      for (int x : v)
        if (band_of[x] != -1000000) { bhi = std::max(bhi, band_of[x]); blo = std::min(blo, band_of[x]); }
      const int nb = bhi >= blo ? bhi - blo + 2 : 1;      // the last slot holds the unbounded ones
      auto slot = [&](int x) { return band_of[x] == -1000000 ? nb - 1 : bhi - band_of[x]; };
      cnt.assign(nb + 1, 0);
      for (int x : v) ++cnt[slot(x) + 1];
      for (int k = 0; k < nb; ++k) cnt[k + 1] += cnt[k];
      tmp.resize(v.size());
      for (int x : v) tmp[cnt[slot(x)]++] = x;
      v.swap(tmp);
    }
    L.cls_off[q] = (int)L.sorted.size();
    L.cls_coff[q] = (int)L.csorted.size();
    L.cls_cn[q] = (int)v.size();
    for (size_t i = 0; i < v.size();) {
      size_t e = i;
      double bm = 0.0;
      while (e < v.size() && band_of[v[e]] == band_of[v[i]]) bm = std::max(bm, fmax[v[e++]]);
      for (; i < e; ++i) {
        const int r = v[i];
        L.csorted.push_back(r);
        L.cimax.push_back(fmax[r]);
        L.cxstart.push_back((int)L.sorted.size() - L.cls_off[q]);
        L.cn.push_back(F.n[r]);
        L.cls_maxm[q] = std::max(L.cls_maxm[q], F.n[r]);
        const int* mp = &F.members[r].x;
        for (int k = 0; k < F.n[r]; ++k) {
          L.sorted.push_back(mp[k]);
          L.simax.push_back(pairs[mp[k]].imax);
          L.sbmax.push_back(bm);
        }
      }
    }
    L.cls_n[q] = (int)L.sorted.size() - L.cls_off[q];
  }
}

// Members a kernel of the class pair (bra class p1, ket class p2) can evaluate at once
// from one bra family (its accumulator capacity): the thread-kernel classes whose
// bra has an s shell; 1 elsewhere (family quartets are then listed member by member).
static int family_capacity(int p1, int p2) {
  int lh1 = 0; while ((lh1 + 1) * (lh1 + 2) / 2 <= p1) ++lh1;
  const int ll1 = p1 - lh1 * (lh1 + 1) / 2;
  int lh2 = 0; while ((lh2 + 1) * (lh2 + 2) / 2 <= p2) ++lh2;
  const int ll2 = p2 - lh2 * (lh2 + 1) / 2;
  return fam_cap_l(lh1, ll1, lh2, ll2);
}

// Bra tasks: groups (class pairs p1 >= p2) of units (one per molecule having both
// classes); a task is (unit, bra position) and covers the kets of class p2 (for
// p1 == p2 those at positions up to the bra's own).  In a family group (the class
// pair's kernel takes bra families, family_capacity, and some bra family has several
// members) the bra positions are those of the collapsed list: one task per bra
// family, whose kets are those of its members (for p1 == p2 up to the end of the
// family's own block, the ket members of that block paired with the bra members at or
// after them).  With n_shards > 1 every task gets an estimated cost and the tasks
// are dealt to the shards largest first, each to the least-loaded shard
// (longest-processing-time rule), so that the shards' FLOPs, not their task counts,
// come out even.  The estimate: the kets of the task's bands that pass the Schwarz
// bound I_max(bra) I_max(ket) > cutoff at a unit density maximum, times the
// primitive quartets and the per-class FLOP model.
struct TaskPlan {
  std::vector<CPUnit> units;
  std::vector<int> unit_group;
  std::vector<int2> group_cls;             // (bra class, ket class) of each group
  std::vector<int> group_fam;              // bra-family capacity of each group's kernel (1: none)
  std::vector<int2> tasks;                 // every task, group by group
  std::vector<int> task_group;
  std::vector<double> cost;                // estimated FLOPs (n_shards > 1)
  std::vector<int> shard;                  // shard of each task
  std::vector<double> shard_cost;
};

static void make_task_plan(const ClassLists& L, const std::vector<PairRec>& pairs, int n_mol, double cutoff,
                           int n_shards, TaskPlan& T) {
  T = TaskPlan{};
  for (int p1 = 0; p1 < NPAIRCLS; ++p1)
    for (int p2 = 0; p2 <= p1; ++p2) {
      const int g = (int)T.group_cls.size();
      T.group_cls.push_back(make_int2(p1, p2));
      // a family group when the kernel takes bra families and some bra family has
      // several members, none more than the kernel holds
      const int cap = family_capacity(p1, p2);
      int maxm = 1;
      for (int m = 0; m < n_mol; ++m)
        if (L.cls_n[m * NPAIRCLS + p2] > 0) maxm = std::max(maxm, L.cls_maxm[m * NPAIRCLS + p1]);
      const bool fam = cap >= 2 && maxm >= 2 && maxm <= cap;
      T.group_fam.push_back(fam ? cap : 1);
      for (int m = 0; m < n_mol; ++m) {
        const int q1 = m * NPAIRCLS + p1, q2 = m * NPAIRCLS + p2;
        const int n1 = fam ? L.cls_cn[q1] : L.cls_n[q1], n2 = L.cls_n[q2];
        if (n1 == 0 || n2 == 0) continue;
        const int u = (int)T.units.size();
        T.units.push_back(CPUnit{p1, p2, fam ? L.cls_coff[q1] : L.cls_off[q1], L.cls_off[q2], n2, m, fam ? 1 : 0,
                                 L.cls_off[q1]});
        T.unit_group.push_back(g);
        for (int i = 0; i < n1; ++i) {
          T.tasks.push_back(make_int2(u, i));
          T.task_group.push_back(g);
        }
      }
    }
  const size_t nt = T.tasks.size();
  T.shard.assign(nt, 0);
  T.shard_cost.assign(std::max(1, n_shards), 0.0);
  if (n_shards <= 1) return;
  // prefix sums of primitive pairs over the sorted positions
  std::vector<double> pref(L.sorted.size() + 1, 0.0);
  for (size_t q = 0; q < L.sorted.size(); ++q) pref[q + 1] = pref[q] + pairs[L.sorted[q]].n_full;
  T.cost.assign(nt, 0.0);
  for (size_t t = 0; t < nt; ++t) {
    const CPUnit& u = T.units[T.tasks[t].x];
    const int i = T.tasks[t].y;
    int lh1, ll1, lh2, ll2;
    lh1 = 0; while ((lh1 + 1) * (lh1 + 2) / 2 <= u.p1) ++lh1; ll1 = u.p1 - lh1 * (lh1 + 1) / 2;
    lh2 = 0; while ((lh2 + 1) * (lh2 + 2) / 2 <= u.p2) ++lh2; ll2 = u.p2 - lh2 * (lh2 + 1) / 2;
    const double Ib = u.fam ? L.cimax[u.bra_off + i] : L.simax[u.bra_off + i];
    const int bra = u.fam ? L.csorted[u.bra_off + i] : L.sorted[u.bra_off + i];
    const int jend = (u.p1 == u.p2) ? (u.fam ? L.cxstart[u.bra_off + i] + L.cn[u.bra_off + i] : i + 1) : u.n_ket;
    // band maxima are non-increasing along the list: the passing kets are a prefix
    int lo = 0, hi = jend;
    while (lo < hi) {
      const int mid = (lo + hi) / 2;
      if (Ib * L.sbmax[u.ket_off + mid] > cutoff) lo = mid + 1; else hi = mid;
    }
    const double nprim_kets = pref[u.ket_off + lo] - pref[u.ket_off];
    const double nb = pairs[bra].n_full;
    T.cost[t] = class_flops(lh1, ll1, lh2, ll2, (double)lo, nb * nprim_kets) + 1.0;
  }
  std::vector<size_t> order(nt);
  for (size_t t = 0; t < nt; ++t) order[t] = t;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return T.cost[x] > T.cost[y]; });
  for (size_t t : order) {
    int best = 0;
    for (int r = 1; r < n_shards; ++r)
      if (T.shard_cost[r] < T.shard_cost[best]) best = r;
    T.shard[t] = best;
    T.shard_cost[best] += T.cost[t];
  }
}

// Groups (class pairs p1 >= p2) of units (one per molecule having both classes);
// tasks are (unit, bra position); with sharding this context keeps the tasks that
// make_task_plan deals to its shard (Tonto's parallel do shares the bra pairs
// round-robin, molecule.fock.foo:1274; here they are shared by estimated cost).
static int build_tasks(tf_ctx* c) {
  drop_graph(c);                       // captured launches hold the old task arrays and grid sizes
  TaskPlan T;
  make_task_plan(c->lists, c->pairs_h, c->n_mol, c->opt.eri_schwarz_cutoff, c->shard_count, T);
  c->units = T.units;
  c->unit_group = T.unit_group;
  c->group_cls = T.group_cls;
  c->group_fam = T.group_fam;
  c->group_task0.clear();
  c->shard_cost = T.shard_cost;
  std::vector<int2> tasks;
  size_t t = 0;
  for (int g = 0; g < (int)c->group_cls.size(); ++g) {
    c->group_task0.push_back((int)tasks.size());
    for (; t < T.tasks.size() && T.task_group[t] == g; ++t)
      if (T.shard[t] == c->shard_index) tasks.push_back(T.tasks[t]);
  }
  c->group_task0.push_back((int)tasks.size());
  c->n_tasks = (long long)tasks.size();
  c->cls_variant.assign(c->group_cls.size(), 0);
  {                                    // start from the last autotuned choice on this device
    std::lock_guard<std::mutex> lock(g_variant_mutex);
    const auto it = g_variant_cache.find(c->device);
    if (it != g_variant_cache.end() && it->second.size() == c->cls_variant.size()) c->cls_variant = it->second;
  }
  // candidate kets per task (all that a task may examine), for the screening record
  std::vector<long long> cand_off(tasks.size() + 1, 0);
  for (size_t t = 0; t < tasks.size(); ++t) {
    const CPUnit& u = c->units[tasks[t].x];
    const int i = tasks[t].y;
    const long long nk = u.p1 != u.p2 ? u.n_ket
                         : u.fam ? c->lists.cxstart[u.bra_off + i] + c->lists.cn[u.bra_off + i] : i + 1;
    cand_off[t + 1] = cand_off[t] + nk;
  }
  // family tasks, and where their member masks start in the screening record
  c->fam_tasks.clear();
  std::vector<long long> fam_coff(1, 0);
  for (size_t t = 0; t < tasks.size(); ++t)
    if (c->units[tasks[t].x].fam) {
      c->fam_tasks.push_back((int)t);
      fam_coff.push_back(fam_coff.back() + (cand_off[t + 1] - cand_off[t]));
    }
  TF_CUDA(c->d_fam_tasks.reserve(std::max<size_t>(c->fam_tasks.size(), 1)));
  if (!c->fam_tasks.empty())
    TF_CUDA(cudaMemcpyAsync(c->d_fam_tasks.p, c->fam_tasks.data(), c->fam_tasks.size() * sizeof(int),
                            cudaMemcpyHostToDevice, c->stream));
  c->use_cand = false;
  if (cand_off.back() + fam_coff.back() <= c->cand_budget &&
      c->d_cand.reserve(std::max<long long>(cand_off.back(), 1)) == cudaSuccess &&
      c->d_cmask.reserve(std::max<long long>(fam_coff.back(), 1)) == cudaSuccess &&
      c->d_fam_coff.reserve(fam_coff.size()) == cudaSuccess &&
      c->d_task_cand_off.reserve(cand_off.size()) == cudaSuccess &&
      c->d_task_len.reserve(std::max<size_t>(tasks.size(), 1)) == cudaSuccess) {
    TF_CUDA(cudaMemcpyAsync(c->d_task_cand_off.p, cand_off.data(), cand_off.size() * sizeof(long long),
                            cudaMemcpyHostToDevice, c->stream));
    TF_CUDA(cudaMemcpyAsync(c->d_fam_coff.p, fam_coff.data(), fam_coff.size() * sizeof(long long),
                            cudaMemcpyHostToDevice, c->stream));
    c->use_cand = true;
  }
  cudaGetLastError();
  const size_t ng = c->group_cls.size();
  TF_CUDA(c->d_units.reserve(std::max<size_t>(c->units.size(), 1)));
  TF_CUDA(c->d_unit_group.reserve(std::max<size_t>(c->unit_group.size(), 1)));
  TF_CUDA(c->d_group_task0.reserve(ng + 1));
  TF_CUDA(c->d_group_offsets.reserve(3 * ng + 1));
  TF_CUDA(c->d_tasks.reserve(std::max<size_t>(tasks.size(), 1)));
  if ((long long)tasks.size() * NBUCKET + 1 > 0x7fffffffLL) {    // the count scan indexes with int
    set_error("too many bra tasks for the quartet-list counts");
    return TF_EUNSUPPORTED;
  }
  TF_CUDA(c->d_counts.reserve(tasks.size() * NBUCKET + 1));
  TF_CUDA(c->d_offsets.reserve(tasks.size() * NBUCKET + 1));
  if (!c->units.empty()) {
    TF_CUDA(cudaMemcpyAsync(c->d_units.p, c->units.data(), c->units.size() * sizeof(CPUnit), cudaMemcpyHostToDevice,
                            c->stream));
    TF_CUDA(cudaMemcpyAsync(c->d_unit_group.p, c->unit_group.data(), c->unit_group.size() * sizeof(int),
                            cudaMemcpyHostToDevice, c->stream));
  }
  TF_CUDA(cudaMemcpyAsync(c->d_group_task0.p, c->group_task0.data(), (ng + 1) * sizeof(int), cudaMemcpyHostToDevice,
                          c->stream));
  if (!tasks.empty())
    TF_CUDA(cudaMemcpyAsync(c->d_tasks.p, tasks.data(), tasks.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  TF_CUDA(cudaStreamSynchronize(c->stream));
  return TF_OK;
}

// Build pair records, run pair prep + Schwarz, sort each molecule's pairs per class.
static int setup_pairs(tf_ctx* c) {
  drop_graph(c);
  c->pairs_h.clear();
  c->pair_cls.clear();
  c->mol_pair0.assign(c->n_mol + 1, 0);
  long long full_tot = 0;
  {
    long long np_all = 0;
    for (int m = 0; m < c->n_mol; ++m) np_all += (long long)c->mols[m].n_shell * (c->mols[m].n_shell + 1) / 2;
    c->pairs_h.reserve(np_all);
    c->pair_cls.reserve(np_all);
  }
  for (int m = 0; m < c->n_mol; ++m) {
    const MolInfo& mi = c->mols[m];
    c->mol_pair0[m] = (long long)c->pairs_h.size();
    append_pair_records(m, mi.shell0, mi.n_shell, c->shell_l.data(), c->shell_atom.data(), c->shell_cart.data(),
                        c->shell_nprim.data(), &full_tot, c->pairs_h, c->pair_cls);
  }
  c->mol_pair0[c->n_mol] = (long long)c->pairs_h.size();
  c->n_pairs = (long long)c->pairs_h.size();
  if (full_tot > 0x7fffffffLL) { set_error("too many primitive pairs"); return TF_EUNSUPPORTED; }
  TF_CUDA(c->d_pairs.reserve(c->n_pairs));
  TF_CUDA(c->d_prim_full.reserve(full_tot));
  TF_CUDA(c->d_prim_skip.reserve(full_tot));
  TF_CUDA(cudaMemcpyAsync(c->d_pairs.p, c->pairs_h.data(), c->n_pairs * sizeof(PairRec), cudaMemcpyHostToDevice,
                          c->stream));
  const int thr = 128;
  k_pair_prep<<<(unsigned)((c->n_pairs + thr - 1) / thr), thr, 0, c->stream>>>(
      (int)c->n_pairs, c->d_pairs.p, c->d_xyz.p, c->d_shell_nprim.p, c->d_shell_poff.p, c->d_exps.p, c->d_coefs.p,
      c->d_prim_full.p, c->d_prim_skip.p, c->opt.eri_primitive_pair_cutoff);
  TF_CUDA(cudaGetLastError());
  // Schwarz bounds per pair class
  std::vector<std::vector<int>> by_cls(NPAIRCLS);
  for (long long p = 0; p < c->n_pairs; ++p) by_cls[c->pair_cls[p]].push_back((int)p);
  std::vector<int> ids;
  std::vector<int> cls_start(NPAIRCLS + 1, 0);
  for (int k = 0; k < NPAIRCLS; ++k) {
    cls_start[k] = (int)ids.size();
    ids.insert(ids.end(), by_cls[k].begin(), by_cls[k].end());
  }
  cls_start[NPAIRCLS] = (int)ids.size();
  TF_CUDA(c->d_schwarz_ids.reserve(std::max<size_t>(ids.size(), 1)));
  TF_CUDA(cudaMemcpyAsync(c->d_schwarz_ids.p, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice,
                          c->stream));
#define TF_SCHWARZ(LH, LL)                                                                                 \
  {                                                                                                        \
    const int k = pair_class(LH, LL);                                                                      \
    const int nk = cls_start[k + 1] - cls_start[k];                                                        \
    if (nk > 0)                                                                                            \
      k_schwarz<LH, LL><<<(nk + 63) / 64, 64, 0, c->stream>>>(c->d_schwarz_ids.p + cls_start[k], nk,       \
                                                              c->d_pairs.p, c->d_prim_full.p, c->spherical); \
  }
  TF_SCHWARZ(0, 0) TF_SCHWARZ(1, 0) TF_SCHWARZ(1, 1) TF_SCHWARZ(2, 0)
#undef TF_SCHWARZ
  for (int lh = 2; lh <= 2; ++lh)
    for (int ll = 1; ll <= lh; ++ll) {
      const int k = pair_class(lh, ll);
      const int nk = cls_start[k + 1] - cls_start[k];
      if (nk > 0)
        k_schwarz_warp<<<std::min(4096, (nk + WARPS_PER_BLOCK - 1) / WARPS_PER_BLOCK), 32 * WARPS_PER_BLOCK,
                         WARPS_PER_BLOCK * W_SMEM * sizeof(double), c->stream>>>(
            c->d_schwarz_ids.p + cls_start[k], nk, c->d_pairs.p, c->d_prim_full.p, c->spherical, lh, ll, nullptr);
    }
  // pair classes with an f shell: the warp path in global scratch, which the f-class
  // J/K kernels use too (two blocks of WARPS_PER_BLOCK warps per SM)
  if (cls_start[NPAIRCLS] > cls_start[pair_class(3, 0)]) {
    int dev = 0, nsm = 148;
    TF_CUDA(cudaGetDevice(&dev));
    TF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const long long warps = (long long)nsm * 2 * WARPS_PER_BLOCK;
    TF_CUDA(c->d_wscratch.reserve((size_t)warps * WF_SCRATCH));
    c->wscratch_warps = warps;
    for (int ll = 0; ll <= 3; ++ll) {
      const int k = pair_class(3, ll);
      const int nk = cls_start[k + 1] - cls_start[k];
      if (nk > 0)
        k_schwarz_warp<<<(unsigned)std::min<long long>(warps / WARPS_PER_BLOCK, (nk + WARPS_PER_BLOCK - 1) / WARPS_PER_BLOCK),
                         32 * WARPS_PER_BLOCK, 0, c->stream>>>(c->d_schwarz_ids.p + cls_start[k], nk, c->d_pairs.p,
                                                              c->d_prim_full.p, c->spherical, 3, ll, c->d_wscratch.p);
    }
  }
  TF_CUDA(cudaGetLastError());
  TF_CUDA(cudaMemcpyAsync(c->pairs_h.data(), c->d_pairs.p, c->n_pairs * sizeof(PairRec), cudaMemcpyDeviceToHost,
                          c->stream));
  TF_CUDA(cudaStreamSynchronize(c->stream));
  c->max_I_tonto.assign(c->n_pairs, 0.0);
  for (long long p = 0; p < c->n_pairs; ++p) {
    const PairRec& pr = c->pairs_h[p];
    c->max_I_tonto[c->mol_pair0[pr.mol] + pr.tonto_ab] = pr.imax;
  }
  {
    std::vector<int> shell0(c->n_mol), nshell(c->n_mol);
    for (int m = 0; m < c->n_mol; ++m) { shell0[m] = c->mols[m].shell0; nshell[m] = c->mols[m].n_shell; }
    make_pair_families(c->pairs_h, c->n_mol, c->mol_pair0, shell0.data(), nshell.data(), c->shell_l.data(),
                       c->shell_atom.data(), c->shell_nprim.data(), c->shell_poff.data(), c->exps.data(), c->fams);
  }
  make_class_lists(c->pairs_h, c->pair_cls, c->n_mol, c->fams, c->lists);
  c->cls_n = c->lists.cls_n;
  c->cls_off = c->lists.cls_off;
  const std::vector<int>& sorted = c->lists.sorted;
  const std::vector<double>& simax = c->lists.simax;
  const std::vector<double>& sbmax = c->lists.sbmax;
  // packed pair records of the ERI kernels (load_pair_jk)
  {
    std::vector<int4> jr(2 * c->n_pairs);
    std::vector<double2> pr2(2 * c->n_pairs);
    for (long long p = 0; p < c->n_pairs; ++p) {
      const PairRec& q = c->pairs_h[p];
      if (q.n_full > 0xffff || q.n_skip > 0xffff) { set_error("too many primitive pairs in one shell pair"); return TF_EUNSUPPORTED; }
      jr[2 * p] = make_int4(q.cart_hi, q.cart_lo, q.full_off, q.skip_off);
      jr[2 * p + 1] = make_int4(q.atom_hi, q.atom_lo, q.n_full | (q.n_skip << 16),
                                (int)((unsigned)q.mol | (q.sh_hi == q.sh_lo ? 0x80000000u : 0u)));
      pr2[2 * p] = make_double2(q.Rx, q.Ry);
      pr2[2 * p + 1] = make_double2(q.Rz, 0.0);
    }
    TF_CUDA(c->d_jkrec.reserve(std::max<size_t>(jr.size(), 1)));
    TF_CUDA(c->d_pairR.reserve(std::max<size_t>(pr2.size(), 1)));
    TF_CUDA(cudaMemcpy(c->d_jkrec.p, jr.data(), jr.size() * sizeof(int4), cudaMemcpyHostToDevice));
    TF_CUDA(cudaMemcpy(c->d_pairR.p, pr2.data(), pr2.size() * sizeof(double2), cudaMemcpyHostToDevice));
  }
  std::vector<int4> srec(sorted.size());
  for (size_t q = 0; q < sorted.size(); ++q) {
    const PairRec& pr = c->pairs_h[sorted[q]];
    const MolInfo& mi = c->mols[pr.mol];
    const int sh = pr.sh_hi - mi.shell0, sl = pr.sh_lo - mi.shell0;
    const int ah = pr.atom_hi - mi.atom0, al = pr.atom_lo - mi.atom0;
    if (sh > 0xffff || sl > 0xffff || ah > 0xffff || al > 0xffff || pr.n_full > 0xffff || pr.n_skip > 0xffff) {
      set_error("molecule too large for the screening records (65535 shells, atoms or primitive pairs)");
      return TF_EUNSUPPORTED;
    }
    srec[q] = make_int4(sh | (sl << 16), ah | (al << 16), pr.n_full | (pr.n_skip << 16), sorted[q]);
  }
  {                                    // collapsed (family) lists and family members
    const ClassLists& L = c->lists;
    TF_CUDA(c->d_csorted.reserve(std::max<size_t>(L.csorted.size(), 1)));
    TF_CUDA(c->d_cimax.reserve(std::max<size_t>(L.cimax.size(), 1)));
    TF_CUDA(c->d_cxstart.reserve(std::max<size_t>(L.cxstart.size(), 1)));
    TF_CUDA(c->d_cn.reserve(std::max<size_t>(L.cn.size(), 1)));
    TF_CUDA(c->d_fam_mem.reserve(std::max<size_t>(c->fams.members.size(), 1)));
    if (!L.csorted.empty()) {
      TF_CUDA(cudaMemcpy(c->d_csorted.p, L.csorted.data(), L.csorted.size() * sizeof(int), cudaMemcpyHostToDevice));
      TF_CUDA(cudaMemcpy(c->d_cimax.p, L.cimax.data(), L.cimax.size() * sizeof(double), cudaMemcpyHostToDevice));
      TF_CUDA(cudaMemcpy(c->d_cxstart.p, L.cxstart.data(), L.cxstart.size() * sizeof(int), cudaMemcpyHostToDevice));
      TF_CUDA(cudaMemcpy(c->d_cn.p, L.cn.data(), L.cn.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (!c->fams.members.empty())
      TF_CUDA(cudaMemcpy(c->d_fam_mem.p, c->fams.members.data(), c->fams.members.size() * sizeof(int4),
                         cudaMemcpyHostToDevice));
  }
  TF_CUDA(c->d_srec.reserve(std::max<size_t>(srec.size(), 1)));
  TF_CUDA(cudaMemcpyAsync(c->d_srec.p, srec.data(), srec.size() * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
  TF_CUDA(c->d_sorted.reserve(std::max<size_t>(sorted.size(), 1)));
  TF_CUDA(c->d_sorted_imax.reserve(std::max<size_t>(simax.size(), 1)));
  TF_CUDA(c->d_sorted_bmax.reserve(std::max<size_t>(sbmax.size(), 1)));
  TF_CUDA(cudaMemcpyAsync(c->d_sorted.p, sorted.data(), sorted.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  TF_CUDA(cudaMemcpyAsync(c->d_sorted_imax.p, simax.data(), simax.size() * sizeof(double), cudaMemcpyHostToDevice,
                          c->stream));
  TF_CUDA(cudaMemcpyAsync(c->d_sorted_bmax.p, sbmax.data(), sbmax.size() * sizeof(double), cudaMemcpyHostToDevice,
                          c->stream));
  TF_CUDA(cudaStreamSynchronize(c->stream));
  int rc = build_tasks(c);
  if (rc) return rc;
  c->geometry_ready = true;
  return TF_OK;
}

// pair class id -> (lh, ll)
static void class_l(int k, int& lh, int& ll) {
  lh = 0;
  while ((lh + 1) * (lh + 2) / 2 <= k) ++lh;
  ll = k - lh * (lh + 1) / 2;
}

// Launch set-up (shared-memory attribute, resident blocks per SM), done once per
// kernel and before any graph capture: a zero-sized, range-less JKArgs only sets up.
template <int LA, int LB, int LC, int LD, typename T, int V, int MB>
static void launch_jk_t(const JKArgs& a, cudaStream_t s) {
  constexpr int thr = jk_threads<LA, LB, LC, LD, V>();
  constexpr size_t smem = RysSmem<Quartet<LA, LB, LC, LD>::NROOT>::SIZE * sizeof(double);
  static int blocks_per_sm = -1;
  if (blocks_per_sm < 0) {
    cudaFuncSetAttribute(k_jk<LA, LB, LC, LD, T, V, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    {                                  // shared storage for one block, the rest to L1
      int dev = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
      const int pct = per_sm > 0 ? std::min(100, (int)((smem + 2048) * 100 / per_sm) + 1) : 100;
      cudaFuncSetAttribute(k_jk<LA, LB, LC, LD, T, V, MB>, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_jk<LA, LB, LC, LD, T, V, MB>, thr, smem);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  if (a.n <= 0 && !a.range) return;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long full = (long long)nsm * blocks_per_sm;
  const long long blocks = a.range ? full : std::min<long long>((a.n + thr - 1) / thr, full);
  k_jk<LA, LB, LC, LD, T, V, MB><<<(unsigned)blocks, thr, smem, s>>>(a);
}

template <int LA, int LB, int LC, int LD, int V, int MB>
static void launch_jk_v(const JKArgs& a, cudaStream_t s, bool fp32) {
  if (fp32) launch_jk_t<LA, LB, LC, LD, float, V, MB>(a, s);
  else launch_jk_t<LA, LB, LC, LD, double, V, MB>(a, s);
}

template <int LA, int LB, int LC, int LD, int MB>
static void launch_jk_m(const JKArgs& a, cudaStream_t s, bool fp32, int variant) {
  switch (variant & 7) {
    case 1: launch_jk_v<LA, LB, LC, LD, 1, MB>(a, s, fp32); break;
    case 2: launch_jk_v<LA, LB, LC, LD, 2, MB>(a, s, fp32); break;
    case 3: launch_jk_v<LA, LB, LC, LD, 3, MB>(a, s, fp32); break;
    case 4: case 6: launch_jk_v<LA, LB, LC, LD, 6, MB>(a, s, fp32); break;   // deterministic: always bit 2
    case 5: case 7: launch_jk_v<LA, LB, LC, LD, 7, MB>(a, s, fp32); break;
    default: launch_jk_v<LA, LB, LC, LD, 0, MB>(a, s, fp32); break;
  }
}

// The bra-family kernel of the class (family_capacity) when the launch is a family group.
template <int LA, int LB, int LC, int LD>
static void launch_jk(const JKArgs& a, cudaStream_t s, bool fp32, int variant) {
  constexpr int CAP = fam_cap_l(LA, LB, LC, LD);
  if constexpr (CAP > 1) {
    if (a.fam > 1) {
      launch_jk_m<LA, LB, LC, LD, CAP>(a, s, fp32, variant);
      return;
    }
  }
  launch_jk_m<LA, LB, LC, LD, 1>(a, s, fp32, variant);
}

constexpr int GROUP_WPB = 4;
// Warps per block of a lane-group kernel: four, or one where a warp's several groups
// need more than 16 KB of shared memory ((dd|ps), (dd|pp), (dd|ds), (dd|dp): 25-31 KB per
// warp), so that an SM holds as many warps as its shared memory fits (seven) instead of
// one four-warp block.  Measured on (H2O)32: (dd|ps) 2.09 -> 1.65 ms, (dd|ds) 0.86 -> 0.69,
// (dd|dp) 1.07 -> 1.02; (dd|dd), one group per warp, ran 13 % slower and keeps four.
template <int LA, int LB, int LC, int LD>
constexpr int group_wpb() {
  using C = GroupCfg<LA, LB, LC, LD>;
  return C::PER_WARP * sizeof(double) > 16384 && C::QPW > 1 ? 1 : GROUP_WPB;
}

template <int LA, int LB, int LC, int LD>
static int launch_group(const JKArgs& a, cudaStream_t s) {
  constexpr int WPB = group_wpb<LA, LB, LC, LD>();
  constexpr size_t smem = group_smem_bytes<LA, LB, LC, LD>(WPB);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_jk_group<LA, LB, LC, LD, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(k_jk_group<LA, LB, LC, LD, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess) {
      set_error("shared memory attribute");
      return TF_ECUDA;
    }
    attr = true;
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  constexpr int QPB = GroupCfg<LA, LB, LC, LD>::QPW * WPB;
  static int group_blocks_per_sm = -1;
  if (group_blocks_per_sm < 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&group_blocks_per_sm, k_jk_group<LA, LB, LC, LD, false>,
                                                  32 * WPB, smem);
    if (group_blocks_per_sm < 1) group_blocks_per_sm = 1;
  }
  if (a.n <= 0 && !a.range) return TF_OK;
  const long long full = (long long)nsm * group_blocks_per_sm;
  const long long blocks = a.range ? full : std::min<long long>((a.n + QPB - 1) / QPB, (long long)nsm * 32);
  GroupArgs g{a.quartets, a.n, a.pairs, a.prim_full, a.prim_skip, a.P, a.J, a.K, a.mols, a.prim_count,
              a.range, a.base, a.cap, a.jkrec, a.pairR, a.P2, a.J2, a.K2, a.want,
              a.qcount ? a.qcount + (a.bucket32 ? NQCLS : 0) : nullptr, a.fx_lo};
  if (a.fx_lo) k_jk_group<LA, LB, LC, LD, true><<<(unsigned)blocks, 32 * WPB, smem, s>>>(g);
  else k_jk_group<LA, LB, LC, LD, false><<<(unsigned)blocks, 32 * WPB, smem, s>>>(g);
  return TF_OK;
}

// Classes with an f shell: one warp per quartet (k_jk_warp), a persistent grid of
// as many warps as the scratch holds.
static int launch_warp_jk(const JKArgs& a, cudaStream_t s, int la, int lb, int lc, int ld) {
  if (a.n <= 0 && !a.range) return TF_OK;
  if (!a.wscratch || a.wscratch_warps < WARPS_PER_BLOCK) { set_error("no scratch for the f-shell kernel"); return TF_ESTATE; }
  const long long full = a.wscratch_warps / WARPS_PER_BLOCK;
  const long long blocks = a.range ? full : std::min<long long>((a.n + WARPS_PER_BLOCK - 1) / WARPS_PER_BLOCK, full);
  if (a.fx_lo) k_jk_warp<true><<<(unsigned)blocks, 32 * WARPS_PER_BLOCK, 0, s>>>(a, la, lb, lc, ld, a.wscratch);
  else k_jk_warp<false><<<(unsigned)blocks, 32 * WARPS_PER_BLOCK, 0, s>>>(a, la, lb, lc, ld, a.wscratch);
  return TF_OK;
}

// fp32: evaluate the 2D recurrences and (e0|f0) sums in FP32 (thread-per-quartet
// classes); roots, weights, transfers and the Fock accumulation stay FP64.
static int dispatch_jk(int la, int lb, int lc, int ld, const JKArgs& a, cudaStream_t s, bool fp32, int variant = 0) {
  if (la > 2 || lb > 2 || lc > 2 || ld > 2) return launch_warp_jk(a, s, la, lb, lc, ld);
  const int key = ((la * 3 + lb) * 3 + lc) * 3 + ld;
  switch (key) {
#define TF_CASE(A, B, C, D) \
  case ((A * 3 + B) * 3 + C) * 3 + D: launch_jk<A, B, C, D>(a, s, fp32, variant); return TF_OK;
    TF_CASE(0, 0, 0, 0)
    TF_CASE(1, 0, 0, 0) TF_CASE(1, 0, 1, 0)
    TF_CASE(1, 1, 0, 0) TF_CASE(1, 1, 1, 0)
    TF_CASE(2, 0, 0, 0) TF_CASE(2, 0, 1, 0) TF_CASE(2, 0, 1, 1) TF_CASE(2, 0, 2, 0)
    TF_CASE(2, 1, 0, 0) TF_CASE(2, 1, 1, 0)
    TF_CASE(2, 2, 0, 0)
#undef TF_CASE
#define TF_GCASE(A, B, C, D) \
  case ((A * 3 + B) * 3 + C) * 3 + D: return launch_group<A, B, C, D>(a, s);
    TF_GCASE(1, 1, 1, 1)
    TF_GCASE(2, 1, 1, 1) TF_GCASE(2, 1, 2, 0) TF_GCASE(2, 1, 2, 1)
    TF_GCASE(2, 2, 1, 0) TF_GCASE(2, 2, 1, 1) TF_GCASE(2, 2, 2, 0) TF_GCASE(2, 2, 2, 1) TF_GCASE(2, 2, 2, 2)
#undef TF_GCASE
    default:
      set_error("quartet class not built");
      return TF_EUNSUPPORTED;
  }
}

// Algorithmic FLOP model (per primitive quartet and per contracted quartet).
double class_flops(int la, int lb, int lc, int ld, double nq, double npq) {
  const int L = la + lb + lc + ld, nr = L / 2 + 1;
  const int d1 = la + lb + 1, d2 = lc + ld + 1;
  const int ne = ncart_upto(la + lb) - ncart_upto(la - 1), nf = ncart_upto(lc + ld) - ncart_upto(lc - 1);
  const double per_prim = 20.0 + 4.0 * nr * TF_RYS_DEG + nr * (10.0 + 3.0 * (4.0 + 6.0 * d1 * d2) + d1 * d2 +
                                                              3.0 * ne * nf);
  const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
  const double nint = (double)na * nb * nc * nd;
  double hrr = 0.0;
  for (int k = 1; k <= ld; ++k) hrr += 2.0 * ne * (ncart_upto(lc + ld - k) - ncart_upto(lc - 1)) * ncart(k);
  for (int k = 1; k <= lb; ++k) hrr += 2.0 * nc * nd * (ncart_upto(la + lb - k) - ncart_upto(la - 1)) * ncart(k);
  const double per_q = hrr + 12.0 * nint;
  return npq * per_prim + nq * per_q;
}

// Deterministic builds (tf_options.deterministic): the Fock accumulators hold two
// fixed-point words per element (fock_add), the lo words after all the hi words,
// and the kernels are their deterministic instantiations (variant bit 4, fock_add)
// with the K contributions of neighbouring lanes that hit the same element always
// summed in FP64 first (bit 2, whatever the autotuner chose): which lanes are
// summed, and in which order, follows from an entry's position in its class pair's
// list (lane = position mod 32), which neither the launch shape, the graph nor the
// list chunking changes, so every path adds the same values.  (Each contribution
// costs two integer atomics here, so the merged ones pay twice.)
static long long fx_offset(const tf_ctx* c) { return c->opt.deterministic ? c->cmat_off[c->n_mol] : 0; }
static long long acc_elems(const tf_ctx* c) { return (c->opt.deterministic ? 2 : 1) * c->cmat_off[c->n_mol]; }
static int jk_variant(const tf_ctx* c, int g) {
  return c->opt.deterministic ? (c->cls_variant[g] | 6) : c->cls_variant[g];
}

// The list pass MODE over tasks [t0, t1): the plain tasks, then the family tasks
// among them (their own instantiation, over the family task list).  The two passes
// touch disjoint tasks (their counts, records and list positions), so when the
// context has a branch stream (tf_autotune creates them) the family pass runs on it,
// beside the plain pass, and the context stream waits for both.
template <int MODE>
static int launch_list(tf_ctx* c, ListArgs a, long long t0, long long t1, long long* counts,
                       const long long* offsets, int2* out, cudaStream_t s, int& kernels) {
  const long long thr = LIST_THREADS;
  const auto& ft = c->fam_tasks;
  const long long f0 = std::lower_bound(ft.begin(), ft.end(), (int)t0) - ft.begin();
  const long long f1 = std::lower_bound(ft.begin(), ft.end(), (int)t1) - ft.begin();
  const bool side = f1 > f0 && !c->side.empty() && c->list_fork_ev && c->list_join_ev;
  if (f1 > f0) {
    cudaStream_t sf = s;
    if (side) {
      TF_CUDA(cudaEventRecord(c->list_fork_ev, s));
      TF_CUDA(cudaStreamWaitEvent(c->side[0], c->list_fork_ev, 0));
      sf = c->side[0];
    }
    ListArgs af = a;
    af.t_base = f0;
    af.n_tasks = f1;
    k_quartets<MODE, true><<<(unsigned)(((f1 - f0) * 32 + thr - 1) / thr), (unsigned)thr, 0, sf>>>(af, counts, offsets,
                                                                                                   out);
    kernels++;
    if (side) TF_CUDA(cudaEventRecord(c->list_join_ev, sf));
  }
  a.t_base = t0;
  a.n_tasks = t1;
  k_quartets<MODE, false><<<(unsigned)std::max<long long>(1, ((t1 - t0) * 32 + thr - 1) / thr), (unsigned)thr, 0, s>>>(
      a, counts, offsets, out);
  kernels++;
  if (side) TF_CUDA(cudaStreamWaitEvent(s, c->list_join_ev, 0));
  return TF_OK;
}

// Density transform, pair maxima, quartet counts, their scan and the per-group
// (start, FP32 start, end) offsets on the device: the part of a build shared by
// the dynamic and the graph paths.
static int enqueue_counts(tf_ctx* c, const double* dP, const double* dPb, bool mixed, long long cap, ListArgs& la,
                          int& kernels) {
  cudaStream_t s = c->stream;
  const BatchArgs bt = batch_args(c);
  const long long nc2 = c->cmat_off[c->n_mol], ns2 = c->pmax_off[c->n_mol];
  const unsigned gc = (unsigned)std::max<long long>(1, (nc2 + 255) / 256);
  k_density_to_cart<<<gc, 256, 0, s>>>(bt, dP, nullptr, c->d_Pc.p);
  kernels++;
  if (dPb) {                                   // unrestricted: the beta density too
    k_density_to_cart<<<gc, 256, 0, s>>>(bt, dPb, nullptr, c->d_PcB.p);
    kernels++;
  }
  TF_CUDA(cudaMemsetAsync(c->d_pglob.p, 0, c->n_mol * sizeof(unsigned long long), s));
  // per-class primitive counters and, after them, the non-finite-density flag
  TF_CUDA(cudaMemsetAsync(c->d_prim_count.p, 0, BUILD_COUNTERS * sizeof(unsigned long long), s));
  k_pmax<<<(unsigned)std::max<long long>(1, (ns2 + 255) / 256), 256, 0, s>>>(bt, dP, dPb, c->d_pmax.p, c->d_pglob.p,
                                                                             c->d_prim_count.p + NQCLS);
  kernels++;
  la = ListArgs{c->d_tasks.p,    0,           c->n_tasks,    c->d_units.p, c->d_unit_group.p, c->d_group_task0.p,
                c->d_sorted.p,   c->d_sorted_imax.p, c->d_sorted_bmax.p, c->d_srec.p, c->d_pairs.p,  c->d_mols.p,
                c->d_pmax.p,
                c->d_pglob.p,    c->opt.eri_schwarz_cutoff, c->use_mol_cut ? c->d_mol_cut.p : nullptr,
                mixed ? c->opt.mixed_fp32_cut : 0.0, 0, LLONG_MAX,
                c->use_cand ? c->d_cand.p : nullptr, c->d_task_cand_off.p, c->d_task_len.p};
  la.bad = c->d_prim_count.p + NQCLS;
  la.csorted = c->d_csorted.p;
  la.cimax = c->d_cimax.p;
  la.cxstart = c->d_cxstart.p;
  la.cn = c->d_cn.p;
  la.qmask = c->d_qmask.p;
  la.fam_tasks = c->d_fam_tasks.p;
  la.fam_coff = c->d_fam_coff.p;
  la.cmask = c->d_cmask.p;
  const long long nslots = c->n_tasks * NBUCKET;
  TF_TRY_RC(launch_list<0>(c, la, 0, c->n_tasks, c->d_counts.p, nullptr, nullptr, s, kernels));
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, c->d_counts.p, c->d_offsets.p, (int)(nslots + 1), s);
  if (tmp_bytes > c->d_scan_tmp.n) { set_error("scan scratch not sized"); return TF_ESTATE; }
  TF_CUDA(cudaMemsetAsync(c->d_counts.p + nslots, 0, sizeof(long long), s));
  TF_CUDA(cub::DeviceScan::ExclusiveSum(c->d_scan_tmp.p, tmp_bytes, c->d_counts.p, c->d_offsets.p, (int)(nslots + 1),
                                        s));
  const int ng = (int)c->group_cls.size();
  k_group_offsets<<<(ng + 63) / 64, 64, 0, s>>>(ng, c->d_group_task0.p, c->d_offsets.p, cap, c->d_group_offsets.p);
  kernels += 3;
  const long long nacc = acc_elems(c);
  TF_CUDA(cudaMemsetAsync(c->d_Jc.p, 0, nacc * sizeof(double), s));
  TF_CUDA(cudaMemsetAsync(c->d_Kc.p, 0, nacc * sizeof(double), s));
  if (dPb) {
    TF_CUDA(cudaMemsetAsync(c->d_JcB.p, 0, nacc * sizeof(double), s));
    TF_CUDA(cudaMemsetAsync(c->d_KcB.p, 0, nacc * sizeof(double), s));
  }
  return TF_OK;
}

static int enqueue_finalize(tf_ctx* c, double* dJ, double* dK, double* dJb, double* dKb, int& kernels) {
  cudaStream_t s = c->stream;
  const BatchArgs bt = batch_args(c);
  const long long nb2 = c->bmat_off[c->n_mol];
  const unsigned gb = (unsigned)std::max<long long>(1, (nb2 + 255) / 256);
  k_finalize<<<gb, 256, 0, s>>>(bt, c->d_Jc.p, c->d_Kc.p, dJ, dK, fx_offset(c));
  kernels++;
  if (dKb) {                                   // unrestricted: the beta J and K
    k_finalize<<<gb, 256, 0, s>>>(bt, c->d_JcB.p, c->d_KcB.p, dJb, dKb, fx_offset(c));
    kernels++;
  }
  TF_CUDA(cudaGetLastError());
  const int ng = (int)c->group_cls.size();
  TF_CUDA(cudaMemcpyAsync(c->pin->goff, c->d_group_offsets.p, (3 * ng + 1) * sizeof(long long), cudaMemcpyDeviceToHost,
                          s));
  TF_CUDA(cudaMemcpyAsync(c->pin->pc, c->d_prim_count.p, BUILD_COUNTERS * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, s));
  return TF_OK;
}

// Graph path: every class launch reads its quartet range from the device
// (persistent grids of fixed size), so the whole build is one captured graph
// with no host round trip inside.  The list buffer holds list_cap quartets; a
// build whose list is longer is detected on the host after the graph (the
// ranges are clamped, so nothing is written out of bounds) and re-run on the
// dynamic path with a larger buffer.
static int enqueue_graph_body(tf_ctx* c, const double* dP, double* dJ, double* dK, bool mixed, int want,
                              int& kernels) {
  cudaStream_t s = c->stream;
  ListArgs la;
  int rc = enqueue_counts(c, dP, nullptr, mixed, c->graph_cap, la, kernels);
  if (rc) return rc;
  ListArgs lw = la;
  lw.out_cap = c->graph_cap;
  lw.list_total = c->d_offsets.p + c->n_tasks * NBUCKET;     // an overflowing list is not written
  if (c->use_cand) TF_TRY_RC(launch_list<2>(c, lw, 0, c->n_tasks, nullptr, c->d_offsets.p, c->d_quartets.p, s, kernels));
  else TF_TRY_RC(launch_list<1>(c, lw, 0, c->n_tasks, nullptr, c->d_offsets.p, c->d_quartets.p, s, kernels));
  const int ng = (int)c->group_cls.size();
  // class schedule: the class launches are spread over sched_streams branches of
  // the graph (the autotuner's choice), so that one class's tail overlaps another
  // class's start; J and K are summed with atomics, so the order is free
  const int ns = std::max(1, std::min(c->sched_streams, 1 + (int)c->side.size()));
  if (ns > 1) {
    TF_CUDA(cudaEventRecord(c->fork_ev, s));
    for (int i = 0; i + 1 < ns; ++i) TF_CUDA(cudaStreamWaitEvent(c->side[i], c->fork_ev, 0));
  }
  for (int g = 0; g < ng; ++g) {
    if (c->group_task0[g + 1] == c->group_task0[g]) continue;   // no molecule has this class pair
    int l1h, l1l, l2h, l2l;
    class_l(c->group_cls[g].x, l1h, l1l);
    class_l(c->group_cls[g].y, l2h, l2l);
    const int si = ns > 1 && g < (int)c->sched_stream_of.size() ? c->sched_stream_of[g] % ns : 0;
    cudaStream_t sg = si == 0 ? s : c->side[si - 1];
    JKArgs a{c->d_quartets.p, 0, c->d_pairs.p, c->d_prim_full.p, c->d_prim_skip.p, c->d_Pc.p, c->d_Jc.p,
             c->d_Kc.p, c->d_mols.p, c->d_prim_count.p, c->d_group_offsets.p + 3 * g, 0, c->graph_cap,
             c->d_jkrec.p, c->d_pairR.p, nullptr, nullptr, nullptr, want};
    a.wscratch = c->d_wscratch.p;
    a.wscratch_warps = c->wscratch_warps;
    a.qmask = c->d_qmask.p;
    a.fam_mem = c->d_fam_mem.p;
    a.qcount = c->d_prim_count.p + NQCLS + 1;
    a.fam = c->group_fam[g];
    a.bucket32 = 0;
    a.fx_lo = fx_offset(c);
    JKArgs a32 = a;
    a32.range = c->d_group_offsets.p + 3 * g + 1;
    a32.bucket32 = 1;
    rc = dispatch_jk(l1h, l1l, l2h, l2l, a, sg, false, jk_variant(c, g));
    if (rc != TF_OK) return rc;
    kernels++;
    if (mixed) {
      rc = dispatch_jk(l1h, l1l, l2h, l2l, a32, sg, true, jk_variant(c, g));
      if (rc != TF_OK) return rc;
      kernels++;
    }
  }
  if (ns > 1)
    for (int i = 0; i + 1 < ns; ++i) {
      TF_CUDA(cudaEventRecord(c->join_ev[i], c->side[i]));
      TF_CUDA(cudaStreamWaitEvent(s, c->join_ev[i], 0));
    }
  return enqueue_finalize(c, dJ, dK, nullptr, nullptr, kernels);
}

// Statistics of the finished build from the pinned read-backs and the events.
static int finish_stats(tf_ctx* c, int kernels, bool graph) {
  const int ng = (int)c->group_cls.size();
  const long long* goff = c->pin->goff;
  const unsigned long long* pc = c->pin->pc;
  if (pc[NQCLS]) {                      // k_pmax saw NaN or infinity: nothing was listed
    set_error("the density has non-finite elements (NaN or infinity)");
    return TF_EINVAL;
  }
  float ms_all = 0.f, ms_eri = 0.f;
  TF_CUDA(cudaEventElapsedTime(&ms_all, c->ev0, c->ev2));
  double npq = 0.0, flops = 0.0, n_all = 0.0, n_fp32 = 0.0;
  c->cls_stats.clear();
  const unsigned long long* q64 = pc + NQCLS + 1;        // contracted (member) quartets per class
  const unsigned long long* q32 = q64 + NQCLS;
  for (int g = 0; g < ng; ++g) {
    if (goff[3 * g + 2] == goff[3 * g]) continue;       // no list entries
    int l1h, l1l, l2h, l2l;
    class_l(c->group_cls[g].x, l1h, l1l);
    class_l(c->group_cls[g].y, l2h, l2l);
    const int cid = qclass_id(l1h, l1l, l2h, l2l);
    const double nq = (double)q64[cid] + (double)q32[cid];
    n_all += nq;
    n_fp32 += (double)q32[cid];
    const double p = (double)pc[cid];
    npq += p;
    const double fl = class_flops(l1h, l1l, l2h, l2l, (double)nq, p);
    flops += fl;
    float ms = 0.f;                       // per-class device time: direct builds only
    if (!graph) {
      TF_CUDA(cudaEventElapsedTime(&ms, c->cls_ev[2 * g], c->cls_ev[2 * g + 1]));
      ms_eri += ms;
    }
    tf_class_stats cs;
    cs.l[0] = l1h; cs.l[1] = l1l; cs.l[2] = l2h; cs.l[3] = l2l;
    cs.quartets = (double)nq;
    cs.prim_quartets = p;
    cs.flops = fl;
    cs.ms = ms;
    c->cls_stats.push_back(cs);
  }
  c->stats.build_ms = ms_all;
  c->stats.eri_ms = graph ? ms_all : ms_eri;
  c->stats.quartets = n_all;
  c->stats.quartets_fp32 = n_fp32;
  c->stats.prim_quartets = npq;
  c->stats.flops = flops;
  c->stats.kernels = kernels;
  c->stats.graph = graph ? 1 : 0;
  return TF_OK;
}

// One J/K build for every molecule of the context: dP, dJ, dK are the
// concatenated per-molecule n_bf x n_bf (column-major) device blocks.
static int build_jk_device(tf_ctx* c, const double* dP, double* dJ, double* dK, int flags,
                           const double* dPb = nullptr, double* dJb = nullptr, double* dKb = nullptr) {
  if (!c->geometry_ready) { set_error("no geometry"); return TF_ESTATE; }
  if (flags & ~(TF_JK_MIXED | TF_JK_DELTA | TF_JK_NO_COPYBACK | TF_JK_J_ONLY | TF_JK_K_ONLY)) {
    set_error("unknown flags"); return TF_EINVAL;
  }
  if ((flags & TF_JK_J_ONLY) && (flags & TF_JK_K_ONLY)) { set_error("J-only and K-only together"); return TF_EINVAL; }
  const int want = (flags & TF_JK_J_ONLY) ? 1 : (flags & TF_JK_K_ONLY) ? 2 : 3;
  cudaStream_t s = c->stream;
  const bool mixed = (flags & TF_JK_MIXED) != 0;
  if (dPb) {                                    // unrestricted: per-spin Cartesian densities and exchange
    const long long nc = c->cmat_off[c->n_mol];
    if (!dJb || !dKb || c->d_PcB.reserve(nc) != cudaSuccess || c->d_JcB.reserve(acc_elems(c)) != cudaSuccess ||
        c->d_KcB.reserve(acc_elems(c)) != cudaSuccess) {
      cudaGetLastError();
      set_error("device allocation");
      return TF_ENOMEM;
    }
  }
  const int ng = (int)c->group_cls.size();
  while ((int)c->cls_ev.size() < 2 * ng) {
    cudaEvent_t e;
    TF_CUDA(cudaEventCreate(&e));
    c->cls_ev.push_back(e);
  }
  TF_CUDA(c->pin->reserve(3 * (size_t)ng + 1));
  {
    size_t tmp_bytes = 0;
    const long long nslots = c->n_tasks * NBUCKET;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, c->d_counts.p, c->d_offsets.p, (int)(nslots + 1), s);
    if (tmp_bytes > c->d_scan_tmp.n || !c->d_scan_tmp.p) {
      drop_graph(c);                     // a captured build holds the scan scratch it was given
      if (c->d_scan_tmp.reserve(tmp_bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("scan scratch does not fit in device memory");
        return TF_ENOMEM;
      }
    }
  }
  // graph path: once a dynamic build has sized the list buffer and set up every
  // launch, later builds with the same arrays replay one captured graph
  if (c->use_graph && c->graph_cap > 0 && !dPb) {
    const bool same = c->graph_exec && c->graph_key_P == dP && c->graph_key_J == dJ && c->graph_key_K == dK &&
                      c->graph_key_mixed == mixed && c->graph_key_cutoff == c->opt.eri_schwarz_cutoff &&
                      c->graph_key_want == want && c->graph_key_mol_cut == c->use_mol_cut;
    if (!same) {
      drop_graph(c);
      for (int g = 0; g < ng; ++g) {         // launch set-up of every class, outside the capture
        int l1h, l1l, l2h, l2l;
        class_l(c->group_cls[g].x, l1h, l1l);
        class_l(c->group_cls[g].y, l2h, l2l);
        JKArgs none{};
        none.fam = c->group_fam[g];
        for (int fp32 = 0; fp32 < 2; ++fp32) {
          const int rc = dispatch_jk(l1h, l1l, l2h, l2l, none, s, fp32 != 0, jk_variant(c, g));
          if (rc != TF_OK) return rc;
        }
      }
      int kernels = 0;
      cudaGraph_t graph = nullptr;
      TF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue_graph_body(c, dP, dJ, dK, mixed, want, kernels);
      cudaError_t ce = cudaStreamEndCapture(s, &graph);
      if (rc != TF_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
      if (ce != cudaSuccess) { set_error(cudaGetErrorString(ce)); return TF_ECUDA; }
      ce = cudaGraphInstantiate(&c->graph_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) { c->graph_exec = nullptr; set_error(cudaGetErrorString(ce)); return TF_ECUDA; }
      c->graph_key_P = dP; c->graph_key_J = dJ; c->graph_key_K = dK;
      c->graph_key_mixed = mixed;
      c->graph_key_cutoff = c->opt.eri_schwarz_cutoff;
      c->graph_key_want = want;
      c->graph_key_mol_cut = c->use_mol_cut;
      c->graph_kernels = kernels;
    }
    TF_CUDA(cudaEventRecord(c->ev0, s));
    TF_CUDA(cudaGraphLaunch(c->graph_exec, s));
    TF_CUDA(cudaEventRecord(c->ev2, s));
    TF_CUDA(cudaStreamSynchronize(s));
    const long long total = c->pin->goff[3 * ng];
    if (total <= c->graph_cap) return finish_stats(c, c->graph_kernels, true);
    drop_graph(c);                          // list outgrew the buffer: redo this build dynamically
  }
  int kernels = 0;
  TF_CUDA(cudaEventRecord(c->ev0, s));
  ListArgs la;
  int rc = enqueue_counts(c, dP, dPb, mixed, LLONG_MAX, la, kernels);
  if (rc) return rc;
  std::vector<long long> goff(3 * ng + 1);
  TF_CUDA(cudaMemcpyAsync(goff.data(), c->d_group_offsets.p, (3 * ng + 1) * sizeof(long long), cudaMemcpyDeviceToHost,
                          s));
  TF_CUDA(cudaStreamSynchronize(s));
  TF_CUDA(cudaEventRecord(c->ev1, s));
  const long long nq_total = ng > 0 ? goff[3 * (ng - 1) + 2] : 0;
  // The lists are written and consumed in chunks of whole class pairs, each at
  // most list_budget quartets (a single larger class pair is one chunk), so a
  // large batch needs one chunk-sized list buffer rather than the whole list.
  std::vector<int> chunk{0};
  long long chunk_max = 1;
  while (chunk.back() < ng) {
    const int g0 = chunk.back();
    int g1 = g0 + 1;
    while (g1 < ng && goff[3 * g1 + 2] - goff[3 * g0] <= c->list_budget) ++g1;
    chunk_max = std::max(chunk_max, goff[3 * (g1 - 1) + 2] - goff[3 * g0]);
    chunk.push_back(g1);
  }
  // a single chunk whose list fits leaves a buffer that later graph builds reuse
  const bool one_chunk = chunk.size() == 2;
  const long long list_n = one_chunk ? std::max<long long>(chunk_max + chunk_max / 4, c->d_quartets.n) : chunk_max;
  if (c->d_quartets.reserve(list_n) != cudaSuccess) {
    cudaGetLastError();
    drop_graph(c);                       // a captured build may hold the freed buffer
    c->graph_cap = 0;
    if (c->d_quartets.reserve(chunk_max) != cudaSuccess) {
      cudaGetLastError();
      set_error("quartet list chunk does not fit in device memory");
      return TF_ENOMEM;
    }
  }
  // family groups: one member mask per list entry
  if (std::any_of(c->group_fam.begin(), c->group_fam.end(), [](int v) { return v > 1; }) &&
      c->d_qmask.n < c->d_quartets.n) {
    drop_graph(c);                       // a captured build holds the old mask buffer
    if (c->d_qmask.reserve(c->d_quartets.n) != cudaSuccess) {
      cudaGetLastError();
      c->graph_cap = 0;
      set_error("quartet list masks do not fit in device memory");
      return TF_ENOMEM;
    }
  }
  if (one_chunk && c->graph_cap != (long long)c->d_quartets.n) {
    drop_graph(c);
    c->graph_cap = (long long)c->d_quartets.n;
  } else if (!one_chunk) {
    drop_graph(c);
    c->graph_cap = 0;
  }
  for (size_t ci = 0; ci + 1 < chunk.size(); ++ci) {
    const int g0 = chunk[ci], g1 = chunk[ci + 1];
    const long long base = goff[3 * g0], nq = goff[3 * (g1 - 1) + 2] - base;
    if (nq > 0) {
      ListArgs lw = la;
      lw.out_base = base;
      lw.qmask = c->d_qmask.p;
      if (c->use_cand)
        rc = launch_list<2>(c, lw, c->group_task0[g0], c->group_task0[g1], nullptr, c->d_offsets.p,
                            c->d_quartets.p, s, kernels);
      else
        rc = launch_list<1>(c, lw, c->group_task0[g0], c->group_task0[g1], nullptr, c->d_offsets.p,
                            c->d_quartets.p, s, kernels);
      if (rc) return rc;
    }
    for (int g = g0; g < g1; ++g) {
      int l1h, l1l, l2h, l2l;
      class_l(c->group_cls[g].x, l1h, l1l);
      class_l(c->group_cls[g].y, l2h, l2l);
      TF_CUDA(cudaEventRecord(c->cls_ev[2 * g], s));
      JKArgs a{c->d_quartets.p + (goff[3 * g] - base), goff[3 * g + 1] - goff[3 * g], c->d_pairs.p,
               c->d_prim_full.p, c->d_prim_skip.p, c->d_Pc.p, c->d_Jc.p, c->d_Kc.p, c->d_mols.p,
               c->d_prim_count.p, nullptr, 0, LLONG_MAX, c->d_jkrec.p, c->d_pairR.p,
               dPb ? c->d_PcB.p : nullptr, dPb ? c->d_JcB.p : nullptr, dPb ? c->d_KcB.p : nullptr, want};
      a.wscratch = c->d_wscratch.p;
      a.wscratch_warps = c->wscratch_warps;
      a.qmask = c->d_qmask.p + (goff[3 * g] - base);
      a.fam_mem = c->d_fam_mem.p;
      a.qcount = c->d_prim_count.p + NQCLS + 1;
      a.fam = c->group_fam[g];
      a.bucket32 = 0;
      a.fx_lo = fx_offset(c);
      JKArgs a32 = a;
      a32.quartets = c->d_quartets.p + (goff[3 * g + 1] - base);
      a32.qmask = c->d_qmask.p + (goff[3 * g + 1] - base);
      a32.n = goff[3 * g + 2] - goff[3 * g + 1];
      a32.bucket32 = 1;
      if (a.n > 0) {
        rc = dispatch_jk(l1h, l1l, l2h, l2l, a, s, false, jk_variant(c, g));
        if (rc != TF_OK) return rc;
        kernels++;
      }
      if (a32.n > 0) {
        rc = dispatch_jk(l1h, l1l, l2h, l2l, a32, s, true, jk_variant(c, g));
        if (rc != TF_OK) return rc;
        kernels++;
      }
      TF_CUDA(cudaEventRecord(c->cls_ev[2 * g + 1], s));
    }
  }
  (void)nq_total;
  rc = enqueue_finalize(c, dJ, dK, dJb, dKb, kernels);
  if (rc) return rc;
  TF_CUDA(cudaEventRecord(c->ev2, s));
  TF_CUDA(cudaStreamSynchronize(s));
  return finish_stats(c, kernels, false);
}

// Checks of one molecule's basis description, made before any device call: every
// array present, shells on existing atoms with l in range and at least one
// primitive, contiguous first basis functions, finite positions, exponents
// positive and finite, coefficients finite.
static int validate_basis(const tf_basis* B) {
  if (B->n_atom <= 0 || B->n_shell <= 0 || !B->xyz || !B->shell_atom || !B->shell_l || !B->shell_nprim ||
      !B->shell_first_bf || !B->exponents || !B->coefficients) {
    set_error("incomplete basis description");
    return TF_EINVAL;
  }
  for (int i = 0; i < 3 * B->n_atom; ++i)
    if (!std::isfinite(B->xyz[i])) { set_error("non-finite atom position"); return TF_EINVAL; }
  long long np = 0, nb = 0;
  for (int s = 0; s < B->n_shell; ++s) {
    const int l = B->shell_l[s];
    if (l < 0) { set_error("negative angular momentum"); return TF_EINVAL; }
    if (l > LMAX_SUPPORTED) { set_error("angular momentum beyond the built kernels"); return TF_EUNSUPPORTED; }
    if (B->shell_atom[s] < 0 || B->shell_atom[s] >= B->n_atom || B->shell_nprim[s] <= 0) {
      set_error("bad shell record"); return TF_EINVAL;
    }
    if (B->shell_first_bf[s] != nb) { set_error("shell_first_bf not contiguous"); return TF_EINVAL; }
    for (int k = 0; k < B->shell_nprim[s]; ++k) {
      const double e = B->exponents[np + k], cf = B->coefficients[np + k];
      if (!(e > 0.0) || !std::isfinite(e) || !std::isfinite(cf)) {
        set_error("exponents must be positive and finite, coefficients finite");
        return TF_EINVAL;
      }
    }
    np += B->shell_nprim[s];
    nb += (B->is_spherical && l >= 2) ? 2 * l + 1 : ncart(l);
  }
  return TF_OK;
}

static int create_impl(const tf_basis* bases, int n_mol, const tf_options* opt, tf_ctx** out) {
  if (!bases || !out || n_mol <= 0) { set_error("null argument"); return TF_EINVAL; }
  *out = nullptr;
  for (int m = 0; m < n_mol; ++m) {
    const int rc = validate_basis(bases + m);
    if (rc) return rc;
    if ((bases[m].is_spherical ? 1 : 0) != (bases[0].is_spherical ? 1 : 0)) {
      set_error("all molecules of a batch must use the same basis kind"); return TF_EINVAL;
    }
  }
  if (opt && (!(opt->eri_schwarz_cutoff > 0.0) || !(opt->eri_primitive_pair_cutoff >= 0.0) ||
              !(opt->mixed_fp32_cut >= 0.0) || opt->device < 0 ||
              (opt->deterministic != 0 && opt->deterministic != 1))) {
    set_error("bad options"); return TF_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) { set_error("no CUDA device"); return TF_ENODEVICE; }
  tf_ctx* c = new tf_ctx();
  if (opt) c->opt = *opt; else tf_default_options(&c->opt);
  c->device = c->opt.device;
  if (c->device < 0 || c->device >= ndev) { delete c; set_error("bad device ordinal"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) { delete c; return rc; }
  c->n_mol = n_mol;
  c->spherical = bases[0].is_spherical ? 1 : 0;
  std::vector<int> cart_shell, cart_local, bf_shell, bf_local;
  c->cmat_off.assign(n_mol + 1, 0);
  c->bmat_off.assign(n_mol + 1, 0);
  c->pmax_off.assign(n_mol + 1, 0);
  for (int m = 0; m < n_mol; ++m) {
    const tf_basis* B = bases + m;
    if (B->n_atom <= 0 || B->n_shell <= 0 || !B->xyz || !B->shell_atom || !B->shell_l || !B->shell_nprim ||
        !B->shell_first_bf || !B->exponents || !B->coefficients) {
      delete c; set_error("incomplete basis description"); return TF_EINVAL;
    }
    if ((B->is_spherical ? 1 : 0) != c->spherical) {
      delete c; set_error("all molecules of a batch must use the same basis kind"); return TF_EINVAL;
    }
    MolInfo mi{};
    mi.shell0 = c->n_shell;
    mi.n_shell = B->n_shell;
    mi.cart0 = c->n_cart;
    mi.bf0 = c->n_bf;
    mi.atom0 = c->n_atom;
    mi.n_atom = B->n_atom;
    int np = 0, nc = 0, nb = 0;
    for (int s = 0; s < B->n_shell; ++s) {
      const int l = B->shell_l[s];
      if (l < 0 || l > LMAX_SUPPORTED) { delete c; set_error("angular momentum beyond the built kernels"); return TF_EUNSUPPORTED; }
      if (B->shell_atom[s] < 0 || B->shell_atom[s] >= B->n_atom || B->shell_nprim[s] <= 0) {
        delete c; set_error("bad shell record"); return TF_EINVAL;
      }
      if (B->shell_first_bf[s] != nb) { delete c; set_error("shell_first_bf not contiguous"); return TF_EINVAL; }
      c->shell_atom.push_back(mi.atom0 + B->shell_atom[s]);
      c->shell_l.push_back(l);
      c->shell_nprim.push_back(B->shell_nprim[s]);
      c->shell_first_bf.push_back(nb);
      c->shell_poff.push_back((int)c->exps.size() + np);
      c->shell_cart.push_back(nc);
      const int nbf_s = (c->spherical && l >= 2) ? 2 * l + 1 : ncart(l);
      c->shell_nbf.push_back(nbf_s);
      for (int i = 0; i < ncart(l); ++i) { cart_shell.push_back(mi.shell0 + s); cart_local.push_back(i); }
      for (int i = 0; i < nbf_s; ++i) { bf_shell.push_back(mi.shell0 + s); bf_local.push_back(i); }
      np += B->shell_nprim[s];
      nc += ncart(l);
      nb += nbf_s;
    }
    c->exps.insert(c->exps.end(), B->exponents, B->exponents + np);
    c->coefs.insert(c->coefs.end(), B->coefficients, B->coefficients + np);
    c->xyz.insert(c->xyz.end(), B->xyz, B->xyz + 3 * B->n_atom);
    mi.n_cart = nc;
    mi.n_bf = nb;
    mi.cmat = c->cmat_off[m];
    mi.bmat = c->bmat_off[m];
    mi.pmax = c->pmax_off[m];
    c->cmat_off[m + 1] = c->cmat_off[m] + (long long)nc * nc;
    c->bmat_off[m + 1] = c->bmat_off[m] + (long long)nb * nb;
    c->pmax_off[m + 1] = c->pmax_off[m] + (long long)B->n_shell * B->n_shell;
    c->mols.push_back(mi);
    c->n_shell += B->n_shell;
    c->n_cart += nc;
    c->n_bf += nb;
    c->n_atom += B->n_atom;
  }
  if (c->cmat_off[n_mol] > (1LL << 36)) { delete c; set_error("batch too large"); return TF_EUNSUPPORTED; }
  {
    if (cudaMemcpyToSymbol(c_U, g_tables.U, sizeof(g_tables.U)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_comp, g_tables.comp, sizeof(g_tables.comp)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_cidx, g_tables.cidx, sizeof(g_tables.cidx)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_gcomp, g_tables.comp, sizeof(g_tables.comp)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_gidx, g_tables.cidx, sizeof(g_tables.cidx)) != cudaSuccess ||
        cudaFuncSetAttribute(k_schwarz_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             WARPS_PER_BLOCK * W_SMEM * (int)sizeof(double)) != cudaSuccess) {
      delete c; set_error("constant upload"); return TF_ECUDA;
    }
  }
#define TF_TRY(x)                               \
  do {                                          \
    int r__ = (x);                              \
    if (r__) { tf_ctx_destroy(c); return r__; } \
  } while (0)
  auto up = [&](auto& buf, const auto& v) -> int {
    if (buf.reserve(std::max<size_t>(v.size(), 1)) != cudaSuccess) { set_error("device allocation"); return TF_ENOMEM; }
    if (!v.empty() && cudaMemcpy(buf.p, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("upload"); return TF_ECUDA;
    }
    return TF_OK;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaEventCreate(&c->ev2) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->order_ev, cudaEventDisableTiming) != cudaSuccess) {
    tf_ctx_destroy(c); set_error("stream/event creation"); return TF_ECUDA;
  }
  TF_TRY(up(c->d_mols, c->mols));
  TF_TRY(up(c->d_cmat_off, c->cmat_off));
  TF_TRY(up(c->d_bmat_off, c->bmat_off));
  TF_TRY(up(c->d_pmax_off, c->pmax_off));
  TF_TRY(up(c->d_xyz, c->xyz));
  TF_TRY(up(c->d_exps, c->exps));
  TF_TRY(up(c->d_coefs, c->coefs));
  TF_TRY(up(c->d_shell_atom, c->shell_atom));
  TF_TRY(up(c->d_shell_nprim, c->shell_nprim));
  TF_TRY(up(c->d_shell_poff, c->shell_poff));
  TF_TRY(up(c->d_shell_l, c->shell_l));
  TF_TRY(up(c->d_shell_first_bf, c->shell_first_bf));
  TF_TRY(up(c->d_shell_nbf, c->shell_nbf));
  TF_TRY(up(c->d_shell_cart, c->shell_cart));
  TF_TRY(up(c->d_cart_shell, cart_shell));
  TF_TRY(up(c->d_cart_local, cart_local));
  TF_TRY(up(c->d_bf_shell, bf_shell));
  TF_TRY(up(c->d_bf_local, bf_local));
  const size_t nb2 = (size_t)c->bmat_off[n_mol], nc2 = (size_t)c->cmat_off[n_mol];
  if (c->d_P.reserve(nb2) || c->d_J.reserve(nb2) || c->d_K.reserve(nb2) || c->d_H.reserve(nb2) ||
      c->d_Pc.reserve(nc2) || c->d_Jc.reserve(c->opt.deterministic ? 2 * nc2 : nc2) ||
      c->d_Kc.reserve(c->opt.deterministic ? 2 * nc2 : nc2) ||
      c->d_pmax.reserve((size_t)c->pmax_off[n_mol]) || c->d_pglob.reserve(n_mol) ||
      c->d_prim_count.reserve(BUILD_COUNTERS)) {
    tf_ctx_destroy(c); set_error("device allocation"); return TF_ENOMEM;
  }
  TF_TRY(setup_pairs(c));
#undef TF_TRY
  *out = c;
  return TF_OK;
}

}  // namespace tf

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int tf_default_options(tf_options* opt) {
  if (!opt) return TF_EINVAL;
  opt->eri_schwarz_cutoff = 1.0e-9;
  opt->eri_primitive_pair_cutoff = 1.0e-6;
  opt->mixed_fp32_cut = 1.0e-6;
  opt->device = 0;
  opt->deterministic = 0;
  return TF_OK;
}

int tf_ctx_create(const tf_basis* B, const tf_options* opt, tf_ctx** out) {
  return tf::create_impl(B, 1, opt, out);
}

int tf_ctx_create_batch(const tf_basis* bases, int n, const tf_options* opt, tf_ctx** out) {
  return tf::create_impl(bases, n, opt, out);
}

int tf_batch_info(const tf_ctx* c, int* n_bf_per_mol) {
  if (!c) return TF_EINVAL;
  if (n_bf_per_mol)
    for (int m = 0; m < c->n_mol; ++m) n_bf_per_mol[m] = c->mols[m].n_bf;
  return c->n_mol;
}

int tf_set_geometry(tf_ctx* c, const double* xyz) {
  using namespace tf;
  if (!c || !xyz) return TF_EINVAL;
  int rc = set_device(c);
  if (rc) return rc;
  c->xyz.assign(xyz, xyz + 3 * c->n_atom);
  TF_CUDA(cudaMemcpy(c->d_xyz.p, c->xyz.data(), c->xyz.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->geometry_ready = false;
  return setup_pairs(c);
}

int tf_set_schwarz_cutoff(tf_ctx* c, double cutoff) {
  if (!c || !(cutoff > 0.0)) { tf::set_error("bad cutoff"); return TF_EINVAL; }
  c->opt.eri_schwarz_cutoff = cutoff;
  return TF_OK;
}

int tf_set_molecule_cutoffs(tf_ctx* c, const double* cutoffs) {
  using namespace tf;
  if (!c) { set_error("null context"); return TF_EINVAL; }
  if (!cutoffs) {
    c->use_mol_cut = false;
    return TF_OK;
  }
  for (int m = 0; m < c->n_mol; ++m)
    if (!(cutoffs[m] > 0.0) || !std::isfinite(cutoffs[m])) { set_error("bad molecule cutoff"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  if (c->d_mol_cut.reserve(c->n_mol) != cudaSuccess) { cudaGetLastError(); set_error("device allocation"); return TF_ENOMEM; }
  // builds are synchronous, so no captured or running build reads the array now; a
  // captured graph reads the new values at its next replay
  TF_CUDA(cudaMemcpy(c->d_mol_cut.p, cutoffs, c->n_mol * sizeof(double), cudaMemcpyHostToDevice));
  c->use_mol_cut = true;
  return TF_OK;
}

int tf_set_list_budget(tf_ctx* c, long long quartets) {
  if (!c || quartets <= 0) { tf::set_error("bad list budget"); return TF_EINVAL; }
  c->list_budget = quartets;
  return TF_OK;
}

int tf_set_screen_record_budget(tf_ctx* c, long long bytes) {
  if (!c || bytes < 0) { tf::set_error("bad screening-record budget"); return TF_EINVAL; }
  int rc = tf::set_device(c);
  if (rc) return rc;
  c->cand_budget = bytes;
  const std::vector<int> keep = c->cls_variant;
  rc = tf::build_tasks(c);             // decides whether the record is used
  if (rc == TF_OK && keep.size() == c->cls_variant.size()) c->cls_variant = keep;
  return rc;
}

int tf_set_kernel_variant(tf_ctx* c, int variant) {
  if (!c || variant < 0 || variant >= tf::JK_VARIANTS) { tf::set_error("bad kernel variant"); return TF_EINVAL; }
  std::fill(c->cls_variant.begin(), c->cls_variant.end(), variant);
  tf::drop_graph(c);                   // captured launches hold the old kernels
  return TF_OK;
}

int tf_set_graph(tf_ctx* c, int on) {
  if (!c) { tf::set_error("null argument"); return TF_EINVAL; }
  int rc = tf::set_device(c);
  if (rc) return rc;
  c->use_graph = on != 0;
  tf::drop_graph(c);
  return TF_OK;
}

int tf_autotune(tf_ctx* c, const double* dP, double* dJ, double* dK, int flags, int max_streams, tf_tune* out) {
  using namespace tf;
  if (!c || !dP || !dJ || !dK || max_streams < 1 || max_streams > 8) { set_error("bad argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  TF_CUDA(cudaDeviceSynchronize());    // dP may still be being written on any of the caller's streams
  while ((int)c->side.size() < max_streams - 1) {
    cudaStream_t x;
    cudaEvent_t e;
    TF_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    c->side.push_back(x);
    TF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->join_ev.push_back(e);
  }
  if (!c->fork_ev) TF_CUDA(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
  if (!c->list_fork_ev) TF_CUDA(cudaEventCreateWithFlags(&c->list_fork_ev, cudaEventDisableTiming));
  if (!c->list_join_ev) TF_CUDA(cudaEventCreateWithFlags(&c->list_join_ev, cudaEventDisableTiming));
  const bool use_graph = c->use_graph;
  tf_tune res{};
  const int ng = (int)c->group_cls.size();
  // launch-bound variant of each class pair's kernel: class-by-class builds with
  // every class on one variant (the first of two warms the kernels up), then per
  // class the faster variant
  c->use_graph = false;
  drop_graph(c);
  std::vector<std::vector<double>> tv(JK_VARIANTS, std::vector<double>(ng, 0.0));
  for (int v = 0; v < JK_VARIANTS; ++v) {
    std::fill(c->cls_variant.begin(), c->cls_variant.end(), v);
    for (int rep = 0; rep < 2; ++rep) {
      rc = build_jk_device(c, dP, dJ, dK, flags);
      if (rc) { c->use_graph = use_graph; return rc; }
    }
    for (int g = 0; g < ng; ++g) {
      float ms = 0.f;
      TF_CUDA(cudaEventElapsedTime(&ms, c->cls_ev[2 * g], c->cls_ev[2 * g + 1]));
      tv[v][g] = ms;
    }
  }
  for (int g = 0; g < ng; ++g) {
    int best_v = 0;
    for (int v = 1; v < JK_VARIANTS; ++v)
      if (tv[v][g] < tv[best_v][g] * 0.98) best_v = v;
    c->cls_variant[g] = best_v;
    if (best_v) res.variant_classes++;
  }
  {                                    // later contexts on this device start from this choice
    std::lock_guard<std::mutex> lock(g_variant_mutex);
    g_variant_cache[c->device] = c->cls_variant;
  }
  // class-pair times from a class-by-class build with the chosen variants
  rc = build_jk_device(c, dP, dJ, dK, flags);
  c->use_graph = use_graph;
  if (rc) return rc;
  res.direct_ms = c->stats.build_ms;
  std::vector<double> t(ng, 0.0);
  for (int g = 0; g < ng; ++g) {
    float ms = 0.f;
    TF_CUDA(cudaEventElapsedTime(&ms, c->cls_ev[2 * g], c->cls_ev[2 * g + 1]));
    t[g] = ms;
  }
  std::vector<int> order(ng);
  for (int g = 0; g < ng; ++g) order[g] = g;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return t[x] > t[y]; });
  int best = 1;
  double best_ms = 1e300;
  std::vector<int> best_of(ng, 0);
  if (c->graph_cap > 0) {
    const bool saved = c->use_graph;
    c->use_graph = true;
    for (int ns = 1; ns <= max_streams; ++ns) {
      std::vector<double> load(ns, 0.0);
      std::vector<int> of(ng, 0);
      for (int g : order) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        of[g] = k;
        load[k] += t[g];
      }
      c->sched_streams = ns;
      c->sched_stream_of = of;
      drop_graph(c);
      double ms = 1e300;
      for (int rep = 0; rep < 4; ++rep) {
        rc = build_jk_device(c, dP, dJ, dK, flags);
        if (rc) { c->use_graph = saved; return rc; }
        if (rep > 0 && c->stats.graph) ms = std::min(ms, c->stats.build_ms);
      }
      res.ms[ns - 1] = ms;
      res.candidates = ns;
      if (ms < best_ms * 0.99) { best_ms = ms; best = ns; best_of = of; }
    }
    c->use_graph = saved;
  }
  c->sched_streams = best;
  c->sched_stream_of = best_of;
  drop_graph(c);
  res.streams = best;
  c->tune = res;
  if (out) *out = res;
  return TF_OK;
}

int tf_set_shard(tf_ctx* c, int index, int count) {
  using namespace tf;
  if (!c || count < 1 || index < 0 || index >= count) { set_error("bad shard"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  c->shard_index = index;
  c->shard_count = count;
  return c->geometry_ready ? build_tasks(c) : TF_OK;
}

int tf_plan_shards(const tf_basis* basis, const double* max_I, double schwarz_cutoff, int n_shards,
                   long long* n_rows, int* row_bra, int* row_ket_class, int* row_ket_limit, int* row_shard,
                   int* pair_position, double* shard_cost) {
  using namespace tf;
  if (!basis || !max_I || !n_rows || n_shards < 1 || !(schwarz_cutoff > 0.0)) {
    set_error("bad argument"); return TF_EINVAL;
  }
  int rc = validate_basis(basis);
  if (rc) return rc;
  const int ns = basis->n_shell;
  std::vector<int> shell_cart(ns), prim_off(ns);
  for (int s = 0, nc = 0, np = 0; s < ns; ++s) {
    shell_cart[s] = nc; nc += ncart(basis->shell_l[s]);
    prim_off[s] = np; np += basis->shell_nprim[s];
  }
  std::vector<PairRec> pairs;
  std::vector<int> pcls;
  long long full_tot = 0;
  append_pair_records(0, 0, ns, basis->shell_l, basis->shell_atom, shell_cart.data(), basis->shell_nprim,
                      &full_tot, pairs, pcls);
  for (PairRec& pr : pairs) pr.imax = max_I[pr.tonto_ab];
  PairFamilies F;
  const std::vector<long long> mol_pair0{0, (long long)pairs.size()};
  const int shell0 = 0;
  make_pair_families(pairs, 1, mol_pair0, &shell0, &ns, basis->shell_l, basis->shell_atom, basis->shell_nprim,
                     prim_off.data(), basis->exponents, F);
  ClassLists L;
  make_class_lists(pairs, pcls, 1, F, L);
  TaskPlan T;
  make_task_plan(L, pairs, 1, schwarz_cutoff, n_shards, T);
  long long r = 0;
  for (size_t t = 0; t < T.tasks.size(); ++t) {
    const CPUnit& u = T.units[T.tasks[t].x];
    const int i = T.tasks[t].y;
    const int nmem = u.fam ? L.cn[u.bra_off + i] : 1;
    for (int k = 0; k < nmem; ++k, ++r) {
      const int bra = u.fam ? L.sorted[u.bra_xoff + L.cxstart[u.bra_off + i] + k] : L.sorted[u.bra_off + i];
      const int lim = u.p1 == u.p2 ? (u.fam ? L.cxstart[u.bra_off + i] + k : i) : u.n_ket - 1;
      if (row_bra) row_bra[r] = pairs[bra].tonto_ab;
      if (row_ket_class) row_ket_class[r] = u.p2;
      if (row_ket_limit) row_ket_limit[r] = lim;
      if (row_shard) row_shard[r] = T.shard[t];
    }
  }
  *n_rows = r;
  if (pair_position)
    for (int q = 0; q < NPAIRCLS; ++q)
      for (int i = 0; i < L.cls_n[q]; ++i) pair_position[pairs[L.sorted[L.cls_off[q] + i]].tonto_ab] = i;
  if (shard_cost)
    for (int k = 0; k < n_shards; ++k) shard_cost[k] = T.shard_cost[k];
  return TF_OK;
}

int tf_build_jk_device(tf_ctx* c, const double* dP, double* dJ, double* dK, int flags, void* stream) {
  using namespace tf;
  if (!c || !dP || !dJ || !dK) { set_error("null argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  // NULL is the legacy default stream, which the context's non-blocking stream does
  // not synchronise with: it is ordered explicitly like any other caller stream
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  if (user != c->stream) {
    // order the context stream after the caller's work, and the caller's after ours
    // (one event per context, recorded again each time: a wait takes the state of
    // the event at the time of the wait call)
    TF_CUDA(cudaEventRecord(c->order_ev, user));
    TF_CUDA(cudaStreamWaitEvent(c->stream, c->order_ev, 0));
    rc = build_jk_device(c, dP, dJ, dK, flags);
    TF_CUDA(cudaEventRecord(c->order_ev, c->stream));
    TF_CUDA(cudaStreamWaitEvent(user, c->order_ev, 0));
    return rc;
  }
  return build_jk_device(c, dP, dJ, dK, flags);
}

int tf_build_jk(tf_ctx* c, const double* P, double* J, double* K, int flags) {
  using namespace tf;
  if (!c || !P || !J || !K) { set_error("null argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  const size_t bytes = (size_t)c->bmat_off[c->n_mol] * sizeof(double);
  TF_CUDA(cudaMemcpyAsync(c->d_P.p, P, bytes, cudaMemcpyHostToDevice, c->stream));
  rc = build_jk_device(c, c->d_P.p, c->d_J.p, c->d_K.p, flags);
  if (rc) return rc;
  TF_CUDA(cudaMemcpyAsync(J, c->d_J.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TF_CUDA(cudaMemcpyAsync(K, c->d_K.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TF_CUDA(cudaStreamSynchronize(c->stream));
  c->stats.h2d_bytes = (long long)bytes;
  c->stats.d2h_bytes = 2 * (long long)bytes;
  return TF_OK;
}

int tf_build_jk_uhf_device(tf_ctx* c, const double* dPa, const double* dPb, double* dJa, double* dJb, double* dKa,
                           double* dKb, int flags, void* stream) {
  using namespace tf;
  if (!c || !dPa || !dPb || !dJa || !dJb || !dKa || !dKb) { set_error("null argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t user = static_cast<cudaStream_t>(stream);   // NULL: the legacy default stream
  if (user != c->stream) {
    TF_CUDA(cudaEventRecord(c->order_ev, user));
    TF_CUDA(cudaStreamWaitEvent(c->stream, c->order_ev, 0));
    rc = build_jk_device(c, dPa, dJa, dKa, flags, dPb, dJb, dKb);
    TF_CUDA(cudaEventRecord(c->order_ev, c->stream));
    TF_CUDA(cudaStreamWaitEvent(user, c->order_ev, 0));
    return rc;
  }
  return build_jk_device(c, dPa, dJa, dKa, flags, dPb, dJb, dKb);
}

int tf_build_jk_uhf(tf_ctx* c, const double* Pa, const double* Pb, double* Ja, double* Jb, double* Ka, double* Kb,
                    int flags) {
  using namespace tf;
  if (!c || !Pa || !Pb || !Ja || !Jb || !Ka || !Kb) { set_error("null argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  const long long nb = c->bmat_off[c->n_mol];
  const size_t bytes = (size_t)nb * sizeof(double);
  if (c->d_Pb.reserve(nb) != cudaSuccess || c->d_Jb.reserve(nb) != cudaSuccess || c->d_Kb.reserve(nb) != cudaSuccess) {
    cudaGetLastError();
    set_error("device allocation");
    return TF_ENOMEM;
  }
  TF_CUDA(cudaMemcpyAsync(c->d_P.p, Pa, bytes, cudaMemcpyHostToDevice, c->stream));
  TF_CUDA(cudaMemcpyAsync(c->d_Pb.p, Pb, bytes, cudaMemcpyHostToDevice, c->stream));
  rc = build_jk_device(c, c->d_P.p, c->d_J.p, c->d_K.p, flags, c->d_Pb.p, c->d_Jb.p, c->d_Kb.p);
  if (rc) return rc;
  TF_CUDA(cudaMemcpyAsync(Ja, c->d_J.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TF_CUDA(cudaMemcpyAsync(Jb, c->d_Jb.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TF_CUDA(cudaMemcpyAsync(Ka, c->d_K.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TF_CUDA(cudaMemcpyAsync(Kb, c->d_Kb.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TF_CUDA(cudaStreamSynchronize(c->stream));
  c->stats.h2d_bytes = 2 * (long long)bytes;
  c->stats.d2h_bytes = 4 * (long long)bytes;
  return TF_OK;
}

int tf_build_jk_batched(tf_ctx* c, const double* const* P, double* const* J, double* const* K, int flags) {
  using namespace tf;
  if (!c || !P || !J || !K) { set_error("null argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  long long bytes = 0;
  for (int m = 0; m < c->n_mol; ++m) {
    if (!P[m] || !J[m] || !K[m]) { set_error("null molecule array"); return TF_EINVAL; }
    const size_t b = (size_t)c->mols[m].n_bf * c->mols[m].n_bf * sizeof(double);
    TF_CUDA(cudaMemcpyAsync(c->d_P.p + c->bmat_off[m], P[m], b, cudaMemcpyHostToDevice, c->stream));
    bytes += (long long)b;
  }
  rc = build_jk_device(c, c->d_P.p, c->d_J.p, c->d_K.p, flags);
  if (rc) return rc;
  for (int m = 0; m < c->n_mol; ++m) {
    const size_t b = (size_t)c->mols[m].n_bf * c->mols[m].n_bf * sizeof(double);
    TF_CUDA(cudaMemcpyAsync(J[m], c->d_J.p + c->bmat_off[m], b, cudaMemcpyDeviceToHost, c->stream));
    TF_CUDA(cudaMemcpyAsync(K[m], c->d_K.p + c->bmat_off[m], b, cudaMemcpyDeviceToHost, c->stream));
  }
  TF_CUDA(cudaStreamSynchronize(c->stream));
  c->stats.h2d_bytes = bytes;
  c->stats.d2h_bytes = 2 * bytes;
  return TF_OK;
}

int tf_build_fock(tf_ctx* c, const double* P, const double* H, double* F) {
  using namespace tf;
  if (!c || !P || !H || !F) { set_error("null argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  const size_t n2 = (size_t)c->bmat_off[c->n_mol], bytes = n2 * sizeof(double);
  TF_CUDA(cudaMemcpyAsync(c->d_P.p, P, bytes, cudaMemcpyHostToDevice, c->stream));
  TF_CUDA(cudaMemcpyAsync(c->d_H.p, H, bytes, cudaMemcpyHostToDevice, c->stream));
  rc = build_jk_device(c, c->d_P.p, c->d_J.p, c->d_K.p, 0);
  if (rc) return rc;
  k_fock<<<(unsigned)((n2 + 255) / 256), 256, 0, c->stream>>>((long long)n2, c->d_H.p, c->d_J.p, c->d_K.p, c->d_J.p);
  TF_CUDA(cudaGetLastError());
  TF_CUDA(cudaMemcpyAsync(F, c->d_J.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TF_CUDA(cudaStreamSynchronize(c->stream));
  c->stats.h2d_bytes = 2 * (long long)bytes;
  c->stats.d2h_bytes = (long long)bytes;
  return TF_OK;
}

void tf_build_jk_f(tf_ctx* c, const double* P, double* J, double* K, int flags, int* status) {
  const int rc = tf_build_jk(c, P, J, K, flags);
  if (status) *status = rc;
}

void tf_build_fock_f(tf_ctx* c, const double* P, const double* H, double* F, int* status) {
  const int rc = tf_build_fock(c, P, H, F);
  if (status) *status = rc;
}

void tf_build_jk_uhf_f(tf_ctx* c, const double* Pa, const double* Pb, double* Ja, double* Jb, double* Ka,
                       double* Kb, int flags, int* status) {
  const int rc = tf_build_jk_uhf(c, Pa, Pb, Ja, Jb, Ka, Kb, flags);
  if (status) *status = rc;
}

int tf_debug_fail_alloc(int countdown) {
  if (countdown < 0) { tf::set_error("negative countdown"); return TF_EINVAL; }
  tf::g_fail_alloc.store(countdown);
  return TF_OK;
}

int tf_build_jk_batch(tf_ctx** ctx, int n, const double* const* P, double* const* J, double* const* K, int flags) {
  if (!ctx || n < 0 || (n > 0 && (!P || !J || !K))) return TF_EINVAL;
  for (int i = 0; i < n; ++i) {
    int rc = tf_build_jk(ctx[i], P[i], J[i], K[i], flags);
    if (rc) return rc;
  }
  return TF_OK;
}

int tf_one_electron(tf_ctx* c, const double* Z, double* S, double* T, double* V) {
  using namespace tf;
  if (!c || !Z || !S || !T || !V) { set_error("null argument"); return TF_EINVAL; }
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t s = c->stream;
  DBuf<double> dZ;
  TF_CUDA(dZ.reserve(c->n_atom));
  TF_CUDA(cudaMemcpyAsync(dZ.p, Z, c->n_atom * sizeof(double), cudaMemcpyHostToDevice, s));
  // Cartesian blocks into the (reused) Cartesian accumulators, then to the basis
  double* Sc = c->d_Jc.p;
  double* Tc = c->d_Kc.p;
  double* Vc = c->d_Pc.p;
  k_one_electron<<<(unsigned)((c->n_pairs + 127) / 128), 128, 0, s>>>(
      c->n_pairs, c->d_pairs.p, c->d_mols.p, c->d_xyz.p, dZ.p, c->d_shell_atom.p, c->d_shell_l.p,
      c->d_shell_nprim.p, c->d_shell_poff.p, c->d_shell_cart.p, c->d_exps.p, c->d_coefs.p, Sc, Tc, Vc);
  TF_CUDA(cudaGetLastError());
  const long long n2 = c->bmat_off[c->n_mol];
  const BatchArgs bt = batch_args(c);
  double* outs[3] = {S, T, V};
  double* ins[3] = {Sc, Tc, Vc};
  for (int k = 0; k < 3; ++k) {
    k_cart_to_basis<<<(unsigned)((n2 + 255) / 256), 256, 0, s>>>(bt, ins[k], c->d_J.p);
    TF_CUDA(cudaMemcpyAsync(outs[k], c->d_J.p, n2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    TF_CUDA(cudaStreamSynchronize(s));
  }
  TF_CUDA(cudaGetLastError());
  return TF_OK;
}

}  // extern "C"

// ===========================================================================
// One-electron integrals with no device allocation.
//
// For callers that cannot call cudaMalloc at the point where they need the
// integrals — code running inside a host framework that owns the device
// allocator (an MPI rank driven by a Fortran program that pre-reserves the GPU
// memory), or a context where allocation is forbidden or would serialize the
// device.  The caller passes the basis (host arrays, as tf_basis) and three
// device output arrays; everything else — the staged basis, the derived index
// tables and the Cartesian S, T, V blocks — lives in one file-scope __device__
// array of fixed size, held by every GPU that loads this library until exit.
// ===========================================================================
namespace tf {

constexpr int NOALLOC_MAX_ATOM = 256;
constexpr int NOALLOC_MAX_SHELL = 512;
constexpr int NOALLOC_MAX_PRIM = 4096;
constexpr int NOALLOC_MAX_CART = 512;      // also bounds n_bf
constexpr int NOALLOC_MAX_DEVICES = 64;

// The caller's inputs as the kernels read them: copied into this layout on the host
// first (a static, pageable array), then sent in one copy into the scratch array.
struct NoAllocInputs {
  double xyz[3 * NOALLOC_MAX_ATOM];
  double Z[NOALLOC_MAX_ATOM];
  double exps[NOALLOC_MAX_PRIM];
  double coefs[NOALLOC_MAX_PRIM];
  int shell_atom[NOALLOC_MAX_SHELL];
  int shell_l[NOALLOC_MAX_SHELL];
  int shell_nprim[NOALLOC_MAX_SHELL];
};

struct NoAllocScratch {
  double S[NOALLOC_MAX_CART * NOALLOC_MAX_CART];
  double T[NOALLOC_MAX_CART * NOALLOC_MAX_CART];
  double V[NOALLOC_MAX_CART * NOALLOC_MAX_CART];
  NoAllocInputs in;
  int shell_poff[NOALLOC_MAX_SHELL];
  int shell_cart[NOALLOC_MAX_SHELL];
  int bf_shell[NOALLOC_MAX_CART];
  int bf_local[NOALLOC_MAX_CART];
};

// The scratch array: about 6.4 MB, shared by every call on a device.
static __device__ __align__(256) unsigned char tf_noalloc_scratch[sizeof(NoAllocScratch)];

// Device addresses of the array, one per device, looked up on the first call on
// that device (host code cannot use the symbol's host-side name as an address);
// the look-up and the constant-table upload run under this lock.
static NoAllocScratch* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
static std::mutex g_noalloc_setup_mutex;

// Host staging of the inputs.  It is ordinary pageable memory, so a copy from it
// has read it completely when cudaMemcpyAsync returns; the caller's arrays (pinned
// or not) are therefore free again when the entry point returns.  One staging area
// for all threads, held under its lock from the fill to the end of the copy call.
static NoAllocInputs g_noalloc_stage;
static std::mutex g_noalloc_stage_mutex;

// Derived index tables (first primitive, first Cartesian function per shell,
// basis function -> shell and position) from shell_l / shell_nprim.
__global__ void k_noalloc_index(int n_shell, int spherical, NoAllocScratch* sc) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int np = 0, nc = 0, nb = 0;
  for (int s = 0; s < n_shell; ++s) {
    const int l = sc->in.shell_l[s];
    sc->shell_poff[s] = np;
    sc->shell_cart[s] = nc;
    np += sc->in.shell_nprim[s];
    nc += ncart(l);
    const int m = (spherical && l >= 2) ? 2 * l + 1 : ncart(l);
    for (int i = 0; i < m; ++i) { sc->bf_shell[nb + i] = s; sc->bf_local[nb + i] = i; }
    nb += m;
  }
}

static int noalloc_setup(int dev, NoAllocScratch** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) { set_error("device ordinal beyond the no-allocation table"); return TF_EINVAL; }
  std::lock_guard<std::mutex> lock(g_noalloc_setup_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    TF_CUDA(cudaGetSymbolAddress(&ptr, tf_noalloc_scratch));
    // constant tables (component order, spherical matrices) for this device
    TF_CUDA(cudaMemcpyToSymbol(c_U, g_tables.U, sizeof(g_tables.U)));
    TF_CUDA(cudaMemcpyToSymbol(c_comp, g_tables.comp, sizeof(g_tables.comp)));
    g_noalloc_ptr[dev] = static_cast<NoAllocScratch*>(ptr);
  }
  *out = g_noalloc_ptr[dev];
  return TF_OK;
}

// An output array must be device (or managed) memory of the current device.
static bool device_array_on(const void* p, int dev) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == dev;
}

}  // namespace tf

extern "C" {

int tf_one_electron_noalloc(const tf_basis* B, const double* Z, double* dS, double* dT, double* dV, void* stream) {
  using namespace tf;
  if (!B || !Z || !dS || !dT || !dV || !B->xyz || !B->shell_atom || !B->shell_l || !B->shell_nprim ||
      !B->shell_first_bf || !B->exponents || !B->coefficients) {
    set_error("null argument");
    return TF_EINVAL;
  }
  if (B->n_atom <= 0 || B->n_atom > NOALLOC_MAX_ATOM || B->n_shell <= 0 || B->n_shell > NOALLOC_MAX_SHELL) {
    set_error("tf_one_electron_noalloc: at most 256 atoms and 512 shells");
    return TF_EUNSUPPORTED;
  }
  int np = 0, nc = 0, nb = 0;
  for (int s = 0; s < B->n_shell; ++s) {
    const int l = B->shell_l[s];
    if (l < 0 || l > LMAX_SUPPORTED || B->shell_nprim[s] <= 0 || B->shell_atom[s] < 0 ||
        B->shell_atom[s] >= B->n_atom || B->shell_first_bf[s] != nb) {
      set_error("tf_one_electron_noalloc: bad shell record");
      return TF_EINVAL;
    }
    np += B->shell_nprim[s];
    nc += ncart(l);
    nb += (B->is_spherical && l >= 2) ? 2 * l + 1 : ncart(l);
    if (np > NOALLOC_MAX_PRIM || nc > NOALLOC_MAX_CART) break;
  }
  if (np > NOALLOC_MAX_PRIM || nc > NOALLOC_MAX_CART) {
    set_error("tf_one_electron_noalloc: at most 4096 primitives and 512 Cartesian functions");
    return TF_EUNSUPPORTED;
  }
  int dev = 0;
  TF_CUDA(cudaGetDevice(&dev));
  if (!device_array_on(dS, dev) || !device_array_on(dT, dev) || !device_array_on(dV, dev)) {
    set_error("tf_one_electron_noalloc: dS, dT, dV must be device memory of the current device");
    return TF_EINVAL;
  }
  NoAllocScratch* sc = nullptr;
  int rc = noalloc_setup(dev, &sc);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  {
    // stage the inputs on the host, then one copy from pageable memory: the caller
    // may overwrite or free its arrays as soon as this call returns
    std::lock_guard<std::mutex> lock(g_noalloc_stage_mutex);
    NoAllocInputs& h = g_noalloc_stage;
    std::memcpy(h.xyz, B->xyz, 3 * B->n_atom * sizeof(double));
    std::memcpy(h.Z, Z, B->n_atom * sizeof(double));
    std::memcpy(h.exps, B->exponents, np * sizeof(double));
    std::memcpy(h.coefs, B->coefficients, np * sizeof(double));
    std::memcpy(h.shell_atom, B->shell_atom, B->n_shell * sizeof(int));
    std::memcpy(h.shell_l, B->shell_l, B->n_shell * sizeof(int));
    std::memcpy(h.shell_nprim, B->shell_nprim, B->n_shell * sizeof(int));
    TF_CUDA(cudaMemcpyAsync(&sc->in, &h, sizeof(NoAllocInputs), cudaMemcpyHostToDevice, s));
  }
  k_noalloc_index<<<1, 1, 0, s>>>(B->n_shell, B->is_spherical ? 1 : 0, sc);
  // every Cartesian element of S, T, V is written by the pair kernel (both
  // triangles of every shell-pair block), so nothing needs clearing first
  const long long npair = (long long)B->n_shell * (B->n_shell + 1) / 2;
  k_one_electron_single<<<(unsigned)((npair + 127) / 128), 128, 0, s>>>(
      B->n_shell, B->n_atom, sc->in.xyz, sc->in.Z, sc->in.shell_atom, sc->in.shell_l, sc->in.shell_nprim,
      sc->shell_poff, sc->shell_cart, sc->in.exps, sc->in.coefs, nc, sc->S, sc->T, sc->V);
  const long long n2 = (long long)nb * nb;
  double* outs[3] = {dS, dT, dV};
  double* ins[3] = {sc->S, sc->T, sc->V};
  for (int k = 0; k < 3; ++k)
    k_cart_to_basis_single<<<(unsigned)((n2 + 255) / 256), 256, 0, s>>>(nb, nc, ins[k], sc->bf_shell, sc->bf_local,
                                                                 sc->in.shell_l, sc->shell_cart,
                                                                 B->is_spherical ? 1 : 0, outs[k]);
  TF_CUDA(cudaGetLastError());
  return TF_OK;
}

int tf_last_stats(const tf_ctx* c, tf_stats* s) {
  if (!c || !s) return TF_EINVAL;
  *s = c->stats;
  return TF_OK;
}

int tf_last_class_stats(const tf_ctx* c, tf_class_stats* out, int max) {
  if (!c || (!out && max > 0)) return TF_EINVAL;
  const int n = (int)c->cls_stats.size();
  for (int i = 0; i < n && i < max; ++i) out[i] = c->cls_stats[i];
  return n;
}

int tf_n_bf(const tf_ctx* c) { return c ? c->n_bf : TF_EINVAL; }

int tf_schwarz(const tf_ctx* c, double* max_I) {
  if (!c || !max_I) return TF_EINVAL;
  std::copy(c->max_I_tonto.begin(), c->max_I_tonto.end(), max_I);
  return TF_OK;
}

void tf_ctx_destroy(tf_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  tf::drop_graph(c);
  for (cudaStream_t x : c->side) cudaStreamDestroy(x);
  for (cudaEvent_t x : c->join_ev) cudaEventDestroy(x);
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->list_fork_ev) cudaEventDestroy(c->list_fork_ev);
  if (c->list_join_ev) cudaEventDestroy(c->list_join_ev);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev2) cudaEventDestroy(c->ev2);
  if (c->order_ev) cudaEventDestroy(c->order_ev);
  for (cudaEvent_t e : c->cls_ev) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* tf_error_string(int code) {
  switch (code) {
    case TF_OK: return "ok";
    case TF_EINVAL: return "invalid argument";
    case TF_ECUDA: return tf::g_last_error.empty() ? "CUDA error" : tf::g_last_error.c_str();
    case TF_ENOMEM: return "out of memory";
    case TF_EUNSUPPORTED: return "unsupported (angular momentum or size)";
    case TF_ETIMEOUT: return "bounded device wait ran out";
    case TF_ENODEVICE: return "no usable CUDA device";
    case TF_ESTATE: return "call out of order";
    default: return "unknown error";
  }
}

const char* tf_version(void) { return "tontofock 0.1 (sm_100a)"; }

}  // extern "C"
