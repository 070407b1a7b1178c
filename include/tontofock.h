/*
 * tontofock.h — C ABI of the B200 direct-SCF J/K (Fock) builder.
 *
 * Drop-in for the two-electron part of Tonto's restricted Fock build.  The entry
 * points replace these reference interfaces (paths inside the Tonto project):
 *
 *   tf_ctx_create / tf_set_geometry
 *       MOLECULE:update_shell_info           foofiles/molecule.set.foo:2687-2737
 *       SHELL1PAIR:make_precalculated_data   foofiles/shell1pair.foo:100-154
 *       MOLECULE.FOCK:initialize_max_I       foofiles/molecule.fock.foo:3705-3752
 *   tf_build_jk
 *       MOLECULE.FOCK:make_r_JK_direct(J,K,P)   foofiles/molecule.fock.foo:1235-1363
 *                     (spherical basis, use_spherical_basis= TRUE)
 *       MOLECULE.FOCK:make_r_JK_engine(J,K,P)   foofiles/molecule.fock.foo:1365-1505
 *                     (Cartesian basis)
 *   tf_build_fock
 *       MOLECULE.FOCK:make_r_Fock_mx(F,P)       foofiles/molecule.fock.foo:88-155
 *                     (F = core + J - K/2, the ee_adiabatic_constant = 1 case)
 *   tf_build_jk_batch
 *       no single reference routine: many independent make_r_JK_direct calls
 *       (one per molecule) issued as one launch sequence.
 *
 * Conventions (identical to Tonto's):
 *   - P, J, K, H, F are n_bf x n_bf doubles, column-major (Fortran order), in the
 *     Tonto basis-function order (atoms in order, shells in basis-library order,
 *     Cartesian components in Tonto order, or real solid harmonics ordered
 *     m = 0,+1,-1,+2,-2,... for l >= 2 in a spherical basis).
 *   - Shell contraction coefficients are Tonto's "unnormalised" ones (after
 *     SHELL:unnormalize, foofiles/shell.foo:492-505).
 *   - All indices are 0-based.  Coordinates are in bohr.
 *   - J and K are fully overwritten (reference: J = ZERO, K = ZERO at :1259-1260).
 *
 * Errors: every int-returning call returns TF_OK (0) or a negative TF_E* code;
 * tf_error_string() gives a message.  No exception or exit crosses the ABI.
 * The library's kernels never wait on one another (no device-side spin waits);
 * TF_ETIMEOUT is reserved for a bounded wait and not returned by this version.
 *
 * Threading: one caller thread per context.  Contexts are independent; each is
 * bound to the CUDA device given in tf_options.device.
 */
#ifndef TONTOFOCK_H
#define TONTOFOCK_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TF_OK            0
#define TF_EINVAL      (-1)   /* bad argument */
#define TF_ECUDA       (-2)   /* CUDA runtime error */
#define TF_ENOMEM      (-3)   /* device or host allocation failed */
#define TF_EUNSUPPORTED (-4)  /* angular momentum or size beyond what was built */
#define TF_ETIMEOUT    (-5)   /* a bounded device wait ran out */
#define TF_ENODEVICE   (-6)   /* no CUDA device / extension not usable */
#define TF_ESTATE      (-7)   /* call out of order (e.g. no geometry) */

/* tf_build_jk flags */
#define TF_JK_FULL        0x0   /* full FP64 build */
#define TF_JK_MIXED       0x1   /* quartets with Schwarz x density bound < mixed_cut in FP32 (FP64 roots, accumulation) */
#define TF_JK_DELTA       0x2   /* incremental: P is a density difference; J, K are increments */
#define TF_JK_NO_COPYBACK 0x4   /* (device entry points only) leave results on the device */
#define TF_JK_J_ONLY      0x8   /* Coulomb only: K is returned as zero (screening as for J and K) */
#define TF_JK_K_ONLY      0x10  /* exchange only: J is returned as zero */

/* Precision of a context's default build */
#define TF_PRECISION_FP64  0
#define TF_PRECISION_MIXED 1

typedef struct tf_basis {
  int n_atom;
  const double* xyz;            /* [n_atom][3], bohr */
  int n_shell;
  const int* shell_atom;        /* [n_shell] atom of each shell */
  const int* shell_l;           /* [n_shell] angular momentum (s, p, d, f: 0..3; higher l is
                                   refused with TF_EUNSUPPORTED) */
  const int* shell_nprim;       /* [n_shell] primitives per shell */
  const int* shell_first_bf;    /* [n_shell] first basis function (Tonto order) */
  const double* exponents;      /* [sum nprim] primitive exponents, shell after shell */
  const double* coefficients;   /* [sum nprim] Tonto unnormalised contraction coefficients */
  int is_spherical;             /* Tonto use_spherical_basis */
} tf_basis;

typedef struct tf_options {
  double eri_schwarz_cutoff;         /* SCF_DATA ERI_Schwarz_cutoff (Tonto default 1e-9, types.foo:6097) */
  double eri_primitive_pair_cutoff;  /* SHELL1QUARTET pair_cutoff (Tonto default 1e-6, macros.in:695) */
  double mixed_fp32_cut;             /* TF_JK_MIXED: Schwarz x density bound below which FP32 is used */
  int device;                        /* CUDA device ordinal */
  int deterministic;                 /* 0: J and K accumulate with FP64 atomics (reproducible to
                                        rounding, not bitwise).  1: bitwise-reproducible builds:
                                        every contribution is added as two 64-bit fixed-point
                                        words (2^-32 and 2^-60 units) with integer atomics, whose
                                        sums do not depend on the order of the additions, so a
                                        build gives the same bits whatever the launch schedule,
                                        graph or not, kernel variants and list chunking (for a
                                        fixed shard plan); elements and contributions must stay
                                        below 2^31 in magnitude.  Costs twice the accumulator
                                        memory and about one more atomic per contribution */
} tf_options;

typedef struct tf_stats {
  double build_ms;                   /* device time of the last build (CUDA events) */
  double eri_ms;                     /* device time of the ERI + digestion kernels (graph builds:
                                        the whole graph) */
  double quartets;                   /* contracted shell quartets computed */
  double quartets_fp32;              /* of which in FP32 */
  double prim_quartets;              /* primitive quartets computed */
  double flops;                      /* algorithmic FLOP count of the last build (per-class model) */
  long long h2d_bytes, d2h_bytes;    /* host<->device bytes of the last call */
  int kernels;                       /* kernel launches issued by the last build */
  int graph;                         /* 1: the build replayed a captured CUDA graph */
} tf_stats;

/* Per quartet-class figures of the last build (one entry per (la lb|lc ld) launch). */
typedef struct tf_class_stats {
  int l[4];                          /* la >= lb, lc >= ld, pair class (la lb) >= (lc ld) */
  double quartets, prim_quartets;    /* contracted and primitive quartets computed */
  double flops;                      /* algorithmic FLOPs */
  double ms;                         /* device time of the launch (CUDA events; 0 for graph builds) */
} tf_class_stats;

typedef struct tf_ctx tf_ctx;

/* Fill *opt with Tonto's defaults (Schwarz 1e-9, pair 1e-6, device 0). */
int tf_default_options(tf_options* opt);

/* Create a context: copies the basis, builds shell-pair data and Schwarz bounds
 * on the device (replaces update_shell_info + initialize_max_I). */
int tf_ctx_create(const tf_basis* basis, const tf_options* opt, tf_ctx** ctx);

/* A context holding n independent molecules (same basis kind).  Every build then
 * computes J and K of all of them with one launch per (la lb|lc ld) class: the
 * many separate make_r_JK_direct calls of a set of SCFs, batched.  Device arrays
 * for such a context are the molecules' n_bf x n_bf blocks concatenated in
 * order; tf_batch_info gives the sizes. */
int tf_ctx_create_batch(const tf_basis* bases, int n, const tf_options* opt, tf_ctx** ctx);

/* Number of molecules of the context; fills n_bf_per_mol[n] if not NULL. */
int tf_batch_info(const tf_ctx* ctx, int* n_bf_per_mol);

/* Unrestricted J and K: MOLECULE.FOCK:make_u_JK_direct (molecule.fock.foo:2360-2504).
 * Ja, Ka from the alpha density Pa and Jb, Kb from the beta density Pb, with the
 * shell quartets screened on max |Pa + Pb| as the reference does and each ERI
 * evaluated once for both spins.  Host arrays, n_bf x n_bf column-major; the
 * Fock matrices are F_a = H + Ja + Jb - Ka, F_b = H + Ja + Jb - Kb.  flags as
 * tf_build_jk (TF_JK_MIXED, TF_JK_DELTA, TF_JK_J_ONLY, TF_JK_K_ONLY). */
int tf_build_jk_uhf(tf_ctx* ctx, const double* Pa, const double* Pb, double* Ja, double* Jb, double* Ka,
                    double* Kb, int flags);

/* The same on device arrays (the context's concatenated molecule blocks), ordered
 * after the caller's earlier work on `stream` and before its later work, as
 * tf_build_jk_device. */
int tf_build_jk_uhf_device(tf_ctx* ctx, const double* dPa, const double* dPb, double* dJa, double* dJb,
                           double* dKa, double* dKb, int flags, void* stream);

/* J, K of every molecule of a batched context (host arrays per molecule). */
int tf_build_jk_batched(tf_ctx* ctx, const double* const* P, double* const* J, double* const* K, int flags);

/* New atom positions ([n_atom][3] bohr): rebuilds pair data and Schwarz bounds. */
int tf_set_geometry(tf_ctx* ctx, const double* xyz);

/* Schwarz x density cutoff for subsequent builds (SCF_DATA ERI_Schwarz_cutoff).
 * The pair data are unchanged; only which quartets are computed.  An SCF may
 * use a looser cutoff while far from convergence and tighten it as it converges
 * (the reference keeps it fixed). */
int tf_set_schwarz_cutoff(tf_ctx* ctx, double cutoff);

/* Per-molecule Schwarz x density cutoffs of a batched context: the quartets of
 * molecule m are screened against cutoffs[m] (host array of one value per molecule,
 * each > 0) in place of the context's cutoff, so that the molecules of one batched
 * build can be at different stages of their SCFs (a loose cutoff for early cycles,
 * the tight one for the final full builds).  NULL returns every molecule to the
 * context's cutoff.  No reference counterpart (the reference builds one molecule
 * at a time with one cutoff). */
int tf_set_molecule_cutoffs(tf_ctx* ctx, const double* cutoffs);

/* Device memory for the screened quartet lists: a build writes and consumes them
 * in chunks of whole (la lb|lc ld) class pairs of at most `quartets` entries
 * (8 bytes each; default 2^30, 8 GiB).  A class pair larger than the budget is
 * one chunk of its own.  Results do not depend on it beyond summation order.
 * No reference counterpart (the reference keeps no quartet lists). */
int tf_set_list_budget(tf_ctx* ctx, long long quartets);

/* Device memory for the screening record (one byte per candidate bra-ket pair,
 * default 12 GiB): when the candidates fit, the counting pass records its
 * screening and the list write only compacts the record; otherwise the list write
 * screens again.  bytes = 0 always screens twice.  Results do not depend on it.
 * No reference counterpart. */
int tf_set_screen_record_budget(tf_ctx* ctx, long long bytes);

/* CUDA-graph builds (default on).  After a first build has sized the quartet
 * list, each build is one captured graph (density transform, screening, list,
 * every class launch with its quartet range read on the device, Fock
 * accumulation) with no host round trip inside; it is re-captured when the
 * density/J/K arrays, the precision flag or the cutoff change, and a build whose
 * list outgrows the buffer is redone on the direct path.  on = 0: every build
 * launches class by class after reading the list sizes back.  No reference
 * counterpart. */
int tf_set_graph(tf_ctx* ctx, int on);

/* Result of tf_autotune. */
typedef struct tf_tune {
  int streams;                       /* graph branches chosen for the class launches */
  int candidates;                    /* schedules timed (1 .. max_streams branches) */
  double ms[8];                      /* best graph build time of each candidate */
  double direct_ms;                  /* the class-by-class build used for the class times */
  int variant_classes;               /* class pairs whose kernel runs a variant other than the default */
} tf_tune;

/* Autotuner for the kernels and the class schedule of graph builds.  It first waits
 * for all earlier work on the device; then class-by-class
 * builds of the density dP (device arrays as tf_build_jk_device) time each class
 * pair's kernel in its variants (registers left to the compiler or more resident
 * warps; exchange atomics per lane or summed first over lanes that hit the same
 * element) and keep the fastest per class pair; a further build gives
 * each class pair's device time; then for 1 .. max_streams (<= 8) graph branches the class pairs
 * are assigned longest first to the least-loaded branch, each schedule is
 * captured and timed over three builds, and the fastest is kept for this
 * context's later graph builds.  Contexts created later on the same device start
 * from the kernel variants chosen here.  Fills *out if not NULL.  Results do not depend
 * on the schedule beyond summation order.  No reference counterpart. */
int tf_autotune(tf_ctx* ctx, const double* dP, double* dJ, double* dK, int flags, int max_streams, tf_tune* out);

/* Run every class pair's thread kernel in one variant (0 .. 3, as tf_autotune
 * numbers them: bit 0 more resident warps, bit 1 exchange atomics summed over lanes
 * first) until the next tf_autotune or tf_set_kernel_variant.  A deterministic
 * context always sums over lanes first (bit 1), whatever the variant.
 * Results do not depend on it beyond summation order (deterministic contexts: not at
 * all).  No reference counterpart. */
int tf_set_kernel_variant(tf_ctx* ctx, int variant);

/* Restrict this context's builds to shard `index` of `count`: the bra shell-pair
 * tasks tf_plan_shards deals to that shard (by estimated cost; Tonto's MPI ranks
 * share the bra pairs round-robin, FooToFortran.java:2762-2783,
 * molecule.fock.foo:1274).  The shards' J and K sum to the full J and K (the caller
 * reduces them, e.g. one NCCL all-reduce, as PARALLEL_SYMMETRIC_SUM does at
 * molecule.fock.foo:1355-1357). */
int tf_set_shard(tf_ctx* ctx, int index, int count);

/* The shard plan of one molecule's build, on the host (no device calls, runs without
 * a GPU): the bra tasks tf_set_shard deals out, and the shard of each, written as
 * rows of (bra shell pair, ket pair class, ket limit, shard).  A row covers the ket
 * pairs of its class at class-list positions up to its limit; the class list orders a
 * class's pairs by half-decade I_max band (largest first; a shell-pair family, see
 * tf_ctx_create, placed by its largest I_max with its members together), then by
 * pair index.  A task whose bra is a family gives one row per member.  Together the
 * rows hold every unordered pair of shell pairs once, as Tonto's outer loop ab with
 * cd <= ab does (molecule.fock.foo:1274-1286).  Tasks are dealt largest estimated
 * cost first to the least-loaded shard (the estimate: the kets passing
 * I_max(ab) I_max(cd) > cutoff at a unit density maximum, times primitive quartets
 * and a per-class FLOP model); Tonto's parallel do deals them round-robin
 * (FooToFortran.java:2762-2783), which leaves the shards' work uneven.
 *   max_I: Schwarz bounds in Tonto pair order ab = a(a+1)/2 + b (tf_schwarz);
 *   *n_rows: the number of rows; the arrays, if not NULL, receive per row the bra's
 *   Tonto pair index, the ket pair class (l_hi(l_hi+1)/2 + l_lo), the ket limit and
 *   the shard; pair_position[n_pairs]: each pair's position in its class list;
 *   shard_cost[n_shards]: the estimated FLOPs of every shard. */
int tf_plan_shards(const tf_basis* basis, const double* max_I, double schwarz_cutoff, int n_shards,
                   long long* n_rows, int* row_bra, int* row_ket_class, int* row_ket_limit, int* row_shard,
                   int* pair_position, double* shard_cost);

/* J and K from the symmetric density P (host arrays, column-major n_bf x n_bf).
 * Replaces make_r_JK_direct / make_r_JK_engine.  flags: TF_JK_*.  A density with a
 * NaN or infinite element is refused with TF_EINVAL (J and K are then undefined);
 * the check is made on the device during the build, at no extra pass. */
int tf_build_jk(tf_ctx* ctx, const double* P, double* J, double* K, int flags);

/* Same, on device arrays (n_bf*n_bf doubles each).  `stream` is the caller's
 * cudaStream_t (NULL is CUDA's legacy default stream): the build runs on the
 * context's own stream, ordered after the caller's earlier work on `stream` (so
 * dP may still be being written there) and before its later work; the call
 * returns when the build has finished. */
int tf_build_jk_device(tf_ctx* ctx, const double* dP, double* dJ, double* dK, int flags, void* stream);

/* F = Hcore + J - K/2 from P (host arrays).  Replaces make_r_Fock_mx. */
int tf_build_fock(tf_ctx* ctx, const double* P, const double* Hcore, double* F);

/* The three host builds with the status returned through the last argument instead
 * of the function value, for Fortran callers that must bind them as PURE
 * subroutines: make_r_JK_direct / make_r_JK_engine (molecule.fock.foo:1235,1365),
 * make_r_Fock_mx (:88) and make_u_JK_direct (:2360) are PURE, a PURE procedure may
 * only call PURE procedures, and a PURE function may not have INTENT(OUT)
 * arguments, so the binding is a PURE subroutine over these.
 * *status receives what tf_build_jk / tf_build_fock / tf_build_jk_uhf return. */
void tf_build_jk_f(tf_ctx* ctx, const double* P, double* J, double* K, int flags, int* status);
void tf_build_fock_f(tf_ctx* ctx, const double* P, const double* Hcore, double* F, int* status);
void tf_build_jk_uhf_f(tf_ctx* ctx, const double* Pa, const double* Pb, double* Ja, double* Jb, double* Ka,
                       double* Kb, int flags, int* status);

/* Many independent molecules in one launch sequence: P[i], J[i], K[i] are host
 * arrays of ctx[i]'s size.  All contexts must be on the same device. */
int tf_build_jk_batch(tf_ctx** ctx, int n, const double* const* P, double* const* J, double* const* K, int flags);

/* One-electron integrals in the Tonto basis (column-major n_bf x n_bf): overlap S,
 * kinetic T and nuclear attraction V for nuclear charges Z[n_atom].  Replaces
 * MOLECULE.INTS:make_overlap_mx, make_kinetic_energy_mx, make_nuclear_attraction_mx
 * (foofiles/molecule.ints.foo:34-420); H_core = T + V. */
int tf_one_electron(tf_ctx* ctx, const double* Z, double* S, double* T, double* V);

/* One-electron integrals (S, T, V as tf_one_electron) without any device
 * allocation, for callers that cannot call cudaMalloc where they need them: a
 * program whose host framework owns the GPU memory, or code running where
 * allocating would be forbidden or would stall the device.  No counterpart in
 * the reference (Tonto allocates freely on the host); this is an addition.
 *   basis: host arrays as for tf_ctx_create; Z: host nuclear charges.  They are
 *          copied before the call returns (through a pageable staging area), so
 *          the caller may overwrite or free them, pinned or not, on return;
 *   dS, dT, dV: caller-owned DEVICE arrays of n_bf*n_bf doubles (column-major) on
 *          the current device (anything else: TF_EINVAL);
 *   stream: cudaStream_t or NULL; the kernels are asynchronous on that stream.
 * Limits: 256 atoms, 512 shells, 4096 primitives, 512 Cartesian functions
 * (hence n_bf <= 512); larger inputs return TF_EUNSUPPORTED.  All scratch lives
 * in one fixed array of about 6.4 MB in device memory, held by every GPU that
 * loads this library until the process exits.  The first call on a device looks
 * up that array's device address and uploads constant tables (under a lock, so
 * threads may race to it); make that first call before any stream capture.
 * Every call on a device reuses the same array, so calls whose work overlaps on
 * the GPU (different streams, no ordering) race; calls in order on one stream
 * do not. */
int tf_one_electron_noalloc(const tf_basis* basis, const double* Z, double* dS, double* dT, double* dV,
                            void* stream);

/* Failure injection for tests: the countdown-th device allocation made after this
 * call (by any context) fails as an out-of-memory would, so every allocation path's
 * error return (TF_ENOMEM, context left usable or cleanly destroyed) can be tested
 * without exhausting a shared GPU.  0 turns it off.  No reference counterpart. */
int tf_debug_fail_alloc(int countdown);

/* Statistics of the last build on this context. */
int tf_last_stats(const tf_ctx* ctx, tf_stats* stats);

/* Copies up to max per-class entries of the last build into out; returns the
 * number of entries available (no reference counterpart: instrumentation). */
int tf_last_class_stats(const tf_ctx* ctx, tf_class_stats* out, int max);

/* Number of basis functions of the context (Tonto n_bf; the sum over molecules
 * for a batched context). */
int tf_n_bf(const tf_ctx* ctx);

/* Schwarz bounds sqrt(max |(ab|ab)|) per Tonto shell pair ab = a(a+1)/2 + b (a >= b);
 * for a batched context, molecule after molecule. */
int tf_schwarz(const tf_ctx* ctx, double* max_I);

void tf_ctx_destroy(tf_ctx* ctx);

const char* tf_error_string(int code);

/* Library version string. */
const char* tf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TONTOFOCK_H */
