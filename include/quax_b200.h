/*
 * quax_b200.h -- C ABI of the B200-native two-electron integral library
 * (libquax_b200.so).
 *
 * This replaces the ERI subset of the reference's pybind11 module
 * `libint_interface` (quax/integrals/libint_interface.cc:2784-2807).  The reference
 * keeps global state between initialize() and finalize(); here the same state lives
 * in an opaque handle, so several molecules can coexist.  All arguments are plain
 * pointers and sizes; no torch, pybind11 or JAX types cross this boundary.
 *
 * Conventions
 *   - Coordinates are in bohr.  (The reference's initialize() reads an Angstrom
 *     xyz file through Libint; the Python layer of this package does that parse.)
 *   - Shells are Cartesian (Libint "standard" component order xx,xy,xz,yy,yz,zz,...)
 *     with Libint normalisation; coefficients are passed raw, as tabulated, and
 *     normalised by the library (the reference's BasisSet does the same).
 *   - Dense outputs use the reference layout: ERI row-major i*n^3+j*n^2+k*n+l
 *     (libint_interface.cc:571-585); first-derivative tensor (3N, n, n, n, n)
 *     (libint_interface.cc:2626-2627, reshaped at quax/integrals/tei.py:33).
 *   - Every entry point returns QX_OK (0) or a negative QX_E_* code; the message is
 *     available from qx_last_error() on the calling thread.  Kernels never trap: a
 *     failure inside a kernel sets a device error word that the entry point reads.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Work on device buffers is stream-ordered and asynchronous unless stated.
 *   - `out_on_device` = 1: the pointer is device memory of the handle's device and
 *     the call is asynchronous on `stream`.  0: the pointer is host memory; the
 *     library stages through device memory and returns after the copy completes.
 */
#ifndef QUAX_B200_H
#define QUAX_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define QX_OK 0
#define QX_E_INVALID (-1)     /* bad argument (sizes, NaN coordinates, exponents...) */
#define QX_E_CUDA (-2)        /* CUDA runtime error */
#define QX_E_UNSUPPORTED (-3) /* angular momentum / derivative order not compiled */
#define QX_E_NOMEM (-4)       /* device allocation failed */
#define QX_E_DEVICE (-5)      /* a kernel reported an error through the error word */

/* Highest angular momentum per shell the library is compiled for (f shells). */
#define QX_MAX_L 3

typedef struct qx_handle qx_handle;

/* Thread-local message of the last failing call (never NULL). */
const char *qx_last_error(void);

/* Library build information: highest shell AM and derivative order compiled.
 * Replaces the module attribute LIBINT2_MAX_DERIV_ORDER
 * (libint_interface.cc:2806). */
int qx_max_deriv_order(void);
int qx_max_l(void);

/* Replaces initialize(xyz, basis1..4, ints_tol) (libint_interface.cc:38-95) for
 * the case bs1 == bs2 == bs3 == bs4 that the ERI path uses (quax/methods/ints.py:20).
 *   natom, coords[3*natom]        geometry in bohr
 *   nshell, shell_l[], shell_nprim[], shell_atom[]
 *   exps[], coefs[]               primitives of all shells concatenated (shell order)
 *   pure                          0 = Cartesian (the reference); 1 is reserved
 *   ints_tol                      the reference's `threshold` (Schwarz tolerance)
 * The handle is bound to the CUDA device current at the call; it computes the
 * Schwarz table (libint_interface.cc:158-229) and the screened, class-sorted list of
 * unique shell quartets on that device. */
int qx_initialize(int natom, const double *coords, int nshell, const int *shell_l, const int *shell_nprim,
                  const int *shell_atom, const double *exps, const double *coefs, int pure, double ints_tol,
                  qx_handle **out);

/* Replaces finalize() (libint_interface.cc:97-99). */
int qx_finalize(qx_handle *h);

/* Sizes of the handle: number of basis functions, atoms and shells. */
int qx_nbf(const qx_handle *h);
int qx_natom(const qx_handle *h);
int qx_nshell(const qx_handle *h);

/* Number of screened 8-fold-unique shell quartets (the throughput unit) and the
 * number of doubles qx_eri_unique writes. */
long long qx_unique_quartets(const qx_handle *h);
long long qx_unique_size(const qx_handle *h);

/* Schwarz table as the reference computes it (libint_interface.cc:158-229):
 * K[s1*nshell+s2] = max |(f1 f2|f1 f2)| (not square-rooted), symmetric, host
 * memory of nshell*nshell doubles; *kmax receives max K. Synchronous. */
int qx_schwarz(qx_handle *h, double *K, double *kmax);

/* Replaces compute_2e_int("eri", 0.) (libint_interface.cc:486-647): the dense
 * Cartesian ERI tensor, n^4 doubles, with the reference's screening; elements of
 * screened-out quartets are zero. */
int qx_compute_2e_int(qx_handle *h, double *out, int out_on_device, void *stream);

/* Every screened unique quartet's contracted Cartesian block, written class by
 * class (canonical shell order within a quartet: higher AM first), element-major
 * within a class.  No counterpart in the reference (it only produces the dense
 * tensor); this is the throughput path.  Device memory only. */
int qx_eri_unique(qx_handle *h, double *out_dev, void *stream);

/* Replaces eri_deriv_core(order) (libint_interface.cc:2582-2779): the full
 * derivative tensor of order 1 to 4.  Order 1: 3N*n^4 doubles, layout
 * (3N, n, n, n, n), nuclear index 3*atom + xyz.  Order k: C(M+k-1, k) * n^4
 * doubles (M = 3N), one slice per sorted nuclear multi-index nu1 <= ... <= nuk in
 * the reference's combinations-with-repetition order (utils.h:158-172; order 2:
 * rank = nu1*M - nu1(nu1-1)/2 + nu2 - nu1), each the sum over the shells on the
 * atoms of nu (the reference's cartesian product of shell choices,
 * libint_interface.cc:1200-1226).  Quartets whose four shells sit on one atom are
 * skipped (zero), as in the reference. */
int qx_eri_deriv_core(qx_handle *h, int order, double *out, int out_on_device, void *stream);

/* Replaces compute_2e_deriv("eri", 0., deriv_vec) (libint_interface.cc:1097-1335):
 * one n^4 derivative slice selected by deriv_vec[3*natom] (non-negative counts;
 * total order 1 to 4). */
int qx_compute_2e_deriv(qx_handle *h, const int *deriv_vec, int len, double *out, int out_on_device,
                        void *stream);

/* Adjoint (contracted) gradient, no counterpart in the reference, which obtains it
 * by jacfwd through the 3N x n^4 tensor (quax/methods/hartree_fock.py:79-80 with
 * quax/integrals/tei.py:336-340):
 *     grad[3*atom + xyz] = sum_ijkl Gamma_ijkl d(ij|kl)/dR_{atom,xyz},
 *     Gamma_ijkl = cj * D_ij D_kl + ck * D_ik D_jl   (D symmetric, n x n, row-major).
 * For the RHF energy of the reference (E_2e = 2 sum Gamma G with cj = 1,
 * ck = -1/2) pass cj = 2, ck = -1.  grad (3*natom doubles) is overwritten.  D and
 * grad are device pointers when on_device = 1, host pointers otherwise. */
int qx_grad_adjoint(qx_handle *h, const double *D, double cj, double ck, double *grad, int on_device,
                    void *stream);

/* Direct Coulomb and exchange matrices, replacing the dense jk_build contractions
 * of quax/methods/hartree_fock.py:26-28,79-80,92-93 (J = jk_build(G, D),
 * K = jk_build(G.transpose(0,2,1,3), D)) without forming G:
 *     J_ij = sum_kl (ij|kl) D_kl,   K_ij = sum_kl (ik|jl) D_kl      (n x n, row-major)
 * over the screened unique quartets, for a symmetric D (the densities of an SCF;
 * the images of each integral are folded with D_kl = D_lk).  J and K are
 * overwritten; D, J, K are device pointers when on_device = 1, host pointers
 * otherwise. */
int qx_jk(qx_handle *h, const double *D, double *J, double *K, int on_device, void *stream);

/* Angular-momentum classes (canonical (la lb|lc ld), la>=lb, lc>=ld, bra class >=
 * ket class) and per-class work of a handle: screened unique quartets, primitive
 * quartets, and algorithmic FP64 FLOPs of the plain and first-derivative programs
 * (counting rule in quax_b200/csrc/gen_eri.py).  No counterpart in the reference;
 * used for roofline accounting and per-class timing. */
int qx_num_classes(void);
int qx_class_info(const qx_handle *h, int cls, int *l4, long long *nquartets, long long *nprim_quartets,
                  double *flops, double *flops_deriv);

/* Hessian-vector product of the adjoint, no counterpart in the reference (which
 * forms Hessians by jacfwd through eri_deriv_jvp, tei.py:342-346, over the order-2
 * tensor): Hv = sum_nu2 v_nu2 sum_ijkl Gamma_ijkl d2(ij|kl)/dR_nu1 dR_nu2 with
 * Gamma fixed (as in qx_grad_adjoint), one Hessian column per call for a unit v,
 * without the 3N(3N+1)/2 * n^4 tensor.  v and Hv hold 3N doubles.  Every shell
 * up to f. */
int qx_grad_adjoint_jvp(qx_handle *h, const double *D, double cj, double ck, const double *v, double *Hv,
                        int on_device, void *stream);

/* Direct J/K with density screening, no counterpart in the reference: like
 * qx_jk (device pointers only) but a quartet is skipped when
 * sqrt(K_ab) sqrt(K_cd) max|D| over its six shell-pair blocks < thr, which bounds
 * every J/K contribution it could make (Schwarz inequality).  With the density
 * change of an SCF iteration as D (incremental Fock builds) most quartets drop
 * out as the SCF converges.  The first call uploads per-pair bounds
 * (synchronises); later calls allocate nothing. */
int qx_jk_screened(qx_handle *h, const double *D, double *J, double *K, double thr, void *stream);

/* One-electron integrals (the reference's compute_1e_int("overlap"|"kinetic"|
 * "potential"), libint_interface.cc:232-483, and oei_deriv_core(1), :2403-2579),
 * on the device, Cartesian, same conventions as the two-electron integrals.
 * qx_set_charges gives the nuclear charges (natom doubles; the reference reads
 * them from the xyz file) and must precede them.  qx_oei writes any of S, T, V
 * (n x n, device, NULL to skip); qx_oei_deriv_core writes the three (3N, n, n)
 * first-derivative tensors, nuclear index 3*atom + xyz. */
int qx_set_charges(qx_handle *h, const double *Z);
int qx_oei(qx_handle *h, double *S, double *T, double *V, void *stream);
int qx_oei_deriv_core(qx_handle *h, int order, double *dS, double *dT, double *dV, void *stream);

/* qx_eri_unique restricted to one class (same output positions). */
int qx_eri_unique_class(qx_handle *h, int cls, double *out_dev, void *stream);

/* qx_grad_adjoint restricted to one class: adds that class's contribution into
 * grad_dev (3N doubles, device memory; not zeroed here).  D_dev is n x n on the
 * device.  For per-class timing and engine tuning. */
int qx_grad_adjoint_class(qx_handle *h, int cls, const double *D_dev, double cj, double ck, double *grad_dev,
                          void *stream);

/* Multi-GPU sharding, no counterpart in the reference (which runs on one host).
 * qx_set_shard restricts the handle to rank `rank` of `nranks`: each class keeps a
 * cost-balanced contiguous range of its screened quartets, so per-rank results
 * (dense and derivative tensors, J, K, adjoint gradients) sum over the ranks to
 * the full result -- one all-reduce.  The unique layout and qx_unique_quartets
 * then describe this rank's quartets.  Synchronises the device; call it before
 * qx_autotune.  nranks = 1 restores the full lists.
 * qx_partition_costs is the host-only cut it uses: items with costs cost[0..n)
 * split into nranks contiguous ranges bounds[r]..bounds[r+1] of near-equal cost. */
int qx_set_shard(qx_handle *h, int rank, int nranks);
int qx_partition_costs(const double *cost, long long n, int nranks, long long *bounds);

/* Mixed precision, no counterpart in the reference (Libint is FP64 throughout).
 * Quartets whose Schwarz bound sqrt(K_ab K_cd) is below `bound` run their
 * Obara-Saika recurrences in FP32 on the warp and split engines, in classes
 * whose HRR has at most two transfer steps (lb + ld <= 2: the HRR amplifies the
 * FP32 error about tenfold per step, so the others stay FP64); the primitive
 * set-up, the Boys function, the sums over primitives, the HRR, the epilogues and
 * every accumulation into J, K, gradients and tensors stay FP64.  Each class's
 * list is reordered with its FP64 quartets first, which reorders the unique
 * layout.  bound <= 0 (the default) keeps everything FP64.  Synchronises the
 * device; call qx_autotune afterwards.  qx_precision_split returns how many of a
 * class's quartets (in this rank's view) stay FP64. */
int qx_set_precision(qx_handle *h, double bound);
long long qx_precision_split(const qx_handle *h, int cls);

/* Autotuner, no counterpart in the reference.  Times, on this handle's own
 * quartet lists, every engine configuration each class can run and keeps the
 * fastest: straight-line kernels with 1..32 lanes per quartet, warp kernels with
 * 1 or 4 warps per quartet, the warp-VRR + cooperative-HRR pair, the cooperative
 * engines.  what: bit 0 = plain ERI (timed in unique mode), bit 1 = first
 * derivatives (timed in adjoint-gradient mode).  Synchronises `stream`;
 * allocates and frees its own scratch. */
int qx_autotune(qx_handle *h, int what, void *stream);

/* Engine configuration of one class: cfg[0] plain engine (0 straight-line,
 * 1 warp, 2 cooperative, 4 warp VRR into global accumulators + warp HRR),
 * cfg[1] its parameter (log2 lanes per quartet, or warps per quartet), cfg[2]
 * derivative engine (1 warp, 2 cooperative, 3 warp VRR into
 * global accumulators + cooperative HRR, 5 warp VRR into global accumulators +
 * warp HRR), cfg[3] its warps per quartet. */
int qx_engine_config(const qx_handle *h, int cls, int *cfg);

/* Engine of one class chosen by the caller, no counterpart in the reference: the
 * autotuner's choice made by hand, for tests and measurements.  plain / deriv are
 * engine ids as qx_engine_config reports them (6 = Rys quadrature, available for
 * every class), -1 keeps the current choice; pparam / dparam as in
 * qx_engine_config.  QX_E_UNSUPPORTED when the class lacks the engine.
 * Synchronises the device. */
int qx_set_engine(qx_handle *h, int cls, int plain, int pparam, int deriv, int dparam);

/* Bounded waits, no counterpart in the reference: the split-mode kernels stage
 * primitive pairs into shared memory with bulk copies and wait for them at most
 * `polls` mbarrier polls (default 4M).  A wait that runs out sets the handle's
 * error word (after a further bounded wait for the copies to land), which the
 * host-synchronising calls (host outputs) report as QX_E_DEVICE and clear.  A
 * limit of 0 makes every such wait run out: a way to exercise the failure path
 * without faulting the GPU. */
int qx_set_wait_limit(qx_handle *h, int polls);

/* Frees the first-derivative accumulators of the split-mode classes that a
 * handle keeps after its first derivative call (up to 512 MiB per class; the
 * next derivative call allocates them again).  No counterpart in the reference;
 * for callers that hold many handles on one device (batched SCF).  Synchronises
 * the device. */
int qx_release_scratch(qx_handle *h);

/* The canonical shell indices (s1, s2, s3, s4) of one class's screened unique
 * quartets, in the order of the unique layout (shells[4*qi + i], host memory of
 * 4 * nquartets ints).  No counterpart in the reference; lets a caller map the
 * unique layout of qx_eri_unique back to shell quartets. */
int qx_class_quartets(const qx_handle *h, int cls, int *shells);

/* The plain (materialise-then-contract) derivative path, tile by tile, no
 * counterpart as an entry point in the reference, whose gradient contracts the
 * dense (3N, n^4) tensor of eri_deriv_core (libint_interface.cc:2582-2779) with
 * Gamma under jacfwd (quax/methods/hartree_fock.py:79-80):
 * qx_deriv_tile writes the first-derivative integrals of quartets [q0, q1) of a
 * class (its unique-layout order) into B, a (3N, E) row-major device buffer the
 * caller zeroes: row = nuclear index 3*atom + xyz, column = (q - q0) * ncomp +
 * component (images = 0), or that index * 8 + image for each distinct image of
 * the integral -- (ij|kl), (ji|kl), (ij|lk), (ji|lk), (kl|ij), (lk|ij), (kl|ji),
 * (lk|ji) -- which are the reference tensor's elements (images = 1).
 * qx_gamma_tile writes Gamma (cj D_ij D_kl + ck D_ik D_jl) for the same columns
 * (summed over the distinct images when images = 0), so B @ gam summed over the
 * tiles is the adjoint gradient.  Device pointers; asynchronous on `stream`. */
int qx_deriv_tile(qx_handle *h, int cls, long long q0, long long q1, int images, double *B, long long E,
                  void *stream);
int qx_gamma_tile(qx_handle *h, int cls, long long q0, long long q1, int images, const double *D, double cj,
                  double ck, double *gam, void *stream);

/* Spherical blocks of one class of the unique layout.  No counterpart in the
 * reference, whose Libint path is Cartesian (libint_interface.cc:47-73); it
 * serves spherical bases on top of the Cartesian kernels.  in_dev holds the
 * class's Cartesian unique blocks (ncart(la) ncart(lb) ncart(lc) ncart(ld) planes
 * of nq doubles, as qx_eri_unique writes them), out_dev receives
 * (2la+1)(2lb+1)(2lc+1)(2ld+1) planes of nq doubles in the same order.  T_host
 * (host memory): the solid-harmonic matrices T_l, (2l+1) x ncart(l) row-major,
 * for l = 0..QX_MAX_L, concatenated (110 doubles).  Allocates nothing;
 * asynchronous on `stream`. */
int qx_cart2sph_block(const double *in_dev, double *out_dev, const int *l4, long long nq, const double *T_host,
                      void *stream);

/* Size of the fixed device array qx_compute_2e_int_noalloc works in. */
#define QX_NOALLOC_SCRATCH_BYTES (16u << 20)

/* Dense ERI tensor for callers that cannot allocate device memory.  No counterpart
 * in the reference: it exists for hosts where the library must not call cudaMalloc,
 * such as an XLA/JAX custom call (the runtime owns and pre-reserves the device
 * memory), real-time hosts that forbid allocation after start-up, and code that
 * accounts for every device byte in its own pool.  It computes what
 * qx_initialize + qx_compute_2e_int + qx_finalize compute (same arguments as
 * qx_initialize, Cartesian shells, out_dev = n^4 doubles of caller-owned device
 * memory) but keeps every internal table in one static device array of
 * QX_NOALLOC_SCRATCH_BYTES, held on every device that uses it until the process
 * exits.  It calls no cudaMalloc/cudaFree, creates no streams, runs on `stream` and
 * returns when the tensor is complete.  A basis whose tables do not fit (about
 * 1.5 million screened unique quartets) is rejected with QX_E_INVALID.  All calls
 * share the array, which keeps the previous call's contents, so calls that overlap
 * on the GPU race and must be serialised by the caller.  Every call blocks the host
 * (it reads the Schwarz values back and returns when the tensor is complete), so it
 * cannot be recorded into a CUDA graph: on a stream that is capturing it returns
 * QX_E_INVALID.  The first call on a device looks up the array's address and
 * uploads a constant table synchronously.  Shells up to d (l <= 2).  Errors are
 * reported through qx_last_error(). */
int qx_compute_2e_int_noalloc(int natom, const double *coords, int nshell, const int *shell_l,
                              const int *shell_nprim, const int *shell_atom, const double *exps,
                              const double *coefs, double ints_tol, double *out_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QUAX_B200_H */
