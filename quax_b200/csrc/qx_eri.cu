// qx_eri.cu -- host side of libquax_b200.so and the ERI quartet kernels.
//
// Host responsibilities (what the reference's libint_interface.cc does around
// Libint):
//   * validate and normalise the shells (Libint convention);
//   * build shell-pair / primitive-pair records and upload them;
//   * Schwarz screening with the reference's semantics
//     (quax/integrals/libint_interface.cc:158-229), evaluated on the GPU;
//   * enumerate the screened 8-fold-unique quartets, bucket them by
//     angular-momentum class and sort each bucket by primitive counts;
//   * launch one kernel per class.
// Device work: one thread per contracted shell quartet; the generated per-class
// VRR runs once per primitive quartet into FP64 accumulators and the generated
// HRR runs once per contracted quartet, followed by the output epilogue.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <memory>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "quax_b200.h"
#include "qx_warp.cuh"
#include "qx_rys.cuh"
#include "qx_setup.h"
#include "gen/warp_index.cuh"
#include "gen/rys_index.cuh"

using namespace qx;

// ------------------------------------------------------------------ errors ----
static thread_local std::string g_err = "no error";

static int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define QX_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(QX_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                        \
    } while (0)

extern "C" const char* qx_last_error(void) { return g_err.c_str(); }
void qx_set_last_error(const char* msg) { g_err = msg; }
extern "C" int qx_max_l(void) { return QX_RYS_LMAX; }
extern "C" int qx_max_deriv_order(void) { return 4; }

static constexpr int pair_class(int l1, int l2) { return l1 * (l1 + 1) / 2 + l2; }
static constexpr int quartet_class(int pb, int pk) { return pb * (pb + 1) / 2 + pk; }

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Per-class launch table: straight-line kernels where generated, the
// warp-cooperative engine for the large classes.
static EriLaunch g_eri_launch[QX_NCLS_ALL];
static long long g_class_scratch[QX_NCLS_ALL];
static int g_class_nout[QX_NCLS_ALL];
static const int g_class_coop[QX_NCLS_ALL] = QX_CLASS_COOP;
static const long long g_class_vrr_flops[QX_NCLS_ALL] = QX_CLASS_VRR_FLOPS;
static const long long g_class_hrr_flops[QX_NCLS_ALL] = QX_CLASS_HRR_FLOPS;
static const long long g_class_dvrr_flops[QX_NCLS_ALL] = QX_CLASS_DVRR_FLOPS;
static const long long g_class_dhrr_flops[QX_NCLS_ALL] = QX_CLASS_DHRR_FLOPS;
static const int g_class_l[QX_NCLS_ALL][4] = {
#define QX_L_ENTRY(id, a, b, c, d) {a, b, c, d},
    QX_FOR_EACH_CLASS_ALL(QX_L_ENTRY)
#undef QX_L_ENTRY
};
// Rys-engine launchers, one per class (gen/k_rys_<id>.cu): 0 = launched, 1 = this
// kind is not compiled for the class or its tables exceed shared memory.
typedef int (*RysLaunch)(const qx::RysArgs&, int kind, int mode, long long nwork, cudaStream_t);
#define QX_DECL_RYS(id, a, b, c, d) int qx_launch_rys_##id(const qx::RysArgs&, int, int, long long, cudaStream_t);
QX_FOR_EACH_CLASS_ALL(QX_DECL_RYS)
#undef QX_DECL_RYS
static RysLaunch g_rys_launch[QX_NCLS_ALL];
const double* qx_rys_table();
static int g_coop_idx[QX_NCLS_ALL];
static int g_der_idx[QX_NCLS_ALL];
static const int g_class_nacc[QX_NCLS_ALL] = QX_CLASS_NACC;
static const int g_has_warp_plain[QX_NCLS_ALL] = QX_CLASS_WARP_PLAIN;
static const int g_has_warp_deriv[QX_NCLS_ALL] = QX_CLASS_WARP_DERIV;
static const int g_has_wvrr[QX_NCLS_ALL] = QX_CLASS_WVRR;
static const int g_has_pvrr[QX_NCLS_ALL] = QX_CLASS_PVRR;
static const int g_has_dsplit[QX_NCLS_ALL] = QX_CLASS_DSPLIT;
static WarpLaunch g_warp_plain[QX_NCLS_ALL];
static WarpLaunch g_warp_deriv[QX_NCLS_ALL];
static WarpLaunch g_warp_deriv2[QX_NCLS_ALL];  // second derivatives (classes with l <= 1)
static WvrrLaunch g_wvrr[QX_NCLS_ALL];          // derivative VRR into global accumulators
static WvrrLaunch g_pvrr[QX_NCLS_ALL];          // plain VRR into global accumulators
static WvrrLaunch g_dsplit[QX_NCLS_ALL];        // derivative VRR into item-order accumulators
#define QX_DECL_WP(id) void qx_launch_warp_p##id(const qx::WarpArgs&, int, cudaStream_t);
QX_FOR_EACH_WARP_PLAIN(QX_DECL_WP)
#define QX_DECL_WD(id) void qx_launch_warp_d##id(const qx::WarpArgs&, int, cudaStream_t);
QX_FOR_EACH_WARP_DERIV(QX_DECL_WD)
#define QX_DECL_WH(id) void qx_launch_warp_h##id(const qx::WarpArgs&, int, cudaStream_t);
QX_FOR_EACH_WARP_DERIV2(QX_DECL_WH)
#define QX_DECL_WV(id) \
    void qx_launch_wvrr_d##id(const qx::EriArgs&, const int2*, long long, int, double*, int, cudaStream_t);
QX_FOR_EACH_WVRR(QX_DECL_WV)
#define QX_DECL_PV(id) \
    void qx_launch_pvrr_p##id(const qx::EriArgs&, const int2*, long long, int, double*, int, cudaStream_t);
QX_FOR_EACH_PVRR(QX_DECL_PV)
#define QX_DECL_DS(id) \
    void qx_launch_dsplit_d##id(const qx::EriArgs&, const int2*, long long, int, double*, int, cudaStream_t);
QX_FOR_EACH_DSPLIT(QX_DECL_DS)
// Engines per class.  Plain ERI: straight-line per-thread kernels (small classes),
// warp-per-quartet kernels (lanes = primitive quartets), or the cooperative engine
// (classes whose VRR does not fit a lane's registers).  Derivatives: warp kernels
// where they fit, else the cooperative derivative engine.
// ENG_WVRR (derivatives): warp-program VRR into global accumulators + the
// cooperative HRR; ENG_WSPLIT (plain): the same VRR split + the warp HRR.
// ENG_DSPLIT (derivatives): the split VRR into item-order accumulators + the warp
// kernel's own HRR and epilogue.
// ENG_RYS (plain and derivatives): the Rys-quadrature engine (qx_rys.cuh), the only
// engine of the classes with an f shell.
enum { ENG_SL = 0, ENG_WARP = 1, ENG_COOP = 2, ENG_WVRR = 3, ENG_WSPLIT = 4, ENG_DSPLIT = 5, ENG_RYS = 6 };
int qx_der_index(int cls);
void qx_launch_der_split(int der_idx, const qx::EriArgs& a, int mode, const double* D, double cj, double ck,
                         double* grad, int slice, const int2* tasks, long long ntask, double* scratch, cudaStream_t s);
long long qx_der_nacc(int der_idx);
int qx_der_chunk();
void qx_launch_der_hrr(int der_idx, const qx::EriArgs& a, int mode, const double* D, double cj, double ck,
                       double* grad, int slice, const double* acc, cudaStream_t s);
void qx_launch_der(int der_idx, const qx::EriArgs& a, int mode, const double* D, double cj, double ck, double* grad,
                   int slice, cudaStream_t s);
enum { QX_MODE_DER_DENSE = 10, QX_MODE_DER_SLICE = 11, QX_MODE_GRAD = 12, QX_MODE_DER2_DENSE = 13,
       QX_MODE_DER2_SLICE = 14, QX_MODE_HVP = 15 };
static bool has_os(int c) { return c < QX_NUM_CLASSES; }  // generated Obara-Saika programs (l <= 2)
static bool init_class_tables() {
    static const int nout_os[QX_NUM_CLASSES] = QX_CLASS_NOUT;
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        g_eri_launch[c] = nullptr;
        g_class_scratch[c] = 0;
        g_coop_idx[c] = has_os(c) && g_class_coop[c] ? qx_coop_index(c) : -1;
        g_der_idx[c] = has_os(c) ? qx_der_index(c) : -1;
        int nout = 1;
        for (int i = 0; i < 4; ++i) nout *= (g_class_l[c][i] + 1) * (g_class_l[c][i] + 2) / 2;
        g_class_nout[c] = nout;
        if (has_os(c) && nout_os[c] != nout) return false;
        g_warp_plain[c] = nullptr;
        g_warp_deriv[c] = nullptr;
        g_warp_deriv2[c] = nullptr;
        g_wvrr[c] = nullptr;
        g_pvrr[c] = nullptr;
        g_dsplit[c] = nullptr;
    }
#define QX_SET_WP(id) g_warp_plain[1##id - 100] = &qx_launch_warp_p##id;
    QX_FOR_EACH_WARP_PLAIN(QX_SET_WP)
#define QX_SET_WD(id) g_warp_deriv[1##id - 100] = &qx_launch_warp_d##id;
    QX_FOR_EACH_WARP_DERIV(QX_SET_WD)
#define QX_SET_WH(id) g_warp_deriv2[1##id - 100] = &qx_launch_warp_h##id;
    QX_FOR_EACH_WARP_DERIV2(QX_SET_WH)
#define QX_SET_WV(id) g_wvrr[1##id - 100] = &qx_launch_wvrr_d##id;
    QX_FOR_EACH_WVRR(QX_SET_WV)
#define QX_SET_PV(id) g_pvrr[1##id - 100] = &qx_launch_pvrr_p##id;
    QX_FOR_EACH_PVRR(QX_SET_PV)
#define QX_SET_DS(id) g_dsplit[1##id - 100] = &qx_launch_dsplit_d##id;
    QX_FOR_EACH_DSPLIT(QX_SET_DS)
#define QX_RYS_ENTRY(id, a, b, c, d) g_rys_launch[1##id - 100] = &qx_launch_rys_##id;
    QX_FOR_EACH_CLASS_ALL(QX_RYS_ENTRY)
#undef QX_RYS_ENTRY
#define QX_SL_ENTRY(id, a, b, c, d)                            \
    g_eri_launch[id] = &qx_launch_eri_##id;                    \
    g_class_scratch[id] = qx::scratch_per_quartet<a, b, c, d>();
    QX_FOR_EACH_SL_CLASS(QX_SL_ENTRY)
    return true;
}
static const bool g_tables_ready = init_class_tables();

// ------------------------------------------------------------------ handle ----
struct ClassWork {
    long long nq = 0;
    int2* d_q = nullptr;       // this rank's quartets: a view into d_q_full
    int2* d_q_full = nullptr;  // the class's full screened list (owned)
    long long nq_full = 0;
    long long unique_base = 0;
    long long prims = 0;       // primitive quartets of the class
    int log2g = 0;             // lanes per quartet = 2^log2g
    double* scratch = nullptr; // global accumulators (ACC_GLOBAL classes), owned
    // derivative split mode (largest classes): primitive-chunk tasks and the
    // per-quartet accumulator sums
    int2* d_dtasks = nullptr;
    long long ndtask = 0;
    double* d_dacc = nullptr;
    // the quartet list is cut into slices whose accumulators fit the split-mode
    // buffers; task quartet indices are relative to their slice
    std::vector<long long> slice_q, slice_t;  // quartet / task boundaries, nslice + 1 each
    double* d_pacc = nullptr;  // plain split-mode accumulators (one slice)
    // mixed precision: the full list holds its FP64 quartets first; n64_full of
    // them, nq64 in this rank's view
    long long n64_full = 0x7fffffffffffffffLL, nq64 = 0x7fffffffffffffffLL;
};

// Bytes of accumulator buffer the split modes may use per class.
static constexpr long long QX_SPLIT_ACC_BYTES = 512LL << 20;

static constexpr int QX_NSTREAMS = 8;

// Lanes per quartet: split a quartet's primitive loop over up to 32 lanes while
// the class has too few quartets to fill the GPU and each lane keeps >= 8
// primitive quartets of work.
static int choose_log2g(long long nq, long long prims) {
    int lg = 0;
    const double avg = nq ? (double)prims / nq : 0.0;
    while (lg < 5 && (nq << lg) < 150000 && avg / (1 << (lg + 1)) >= 8.0) ++lg;
    return lg;
}

static long long launch_threads(long long nq, int log2g) { return (((nq << log2g) + 127) / 128) * 128; }

struct qx_handle {
    int device = 0;
    int natom = 0, nshell = 0, nbf = 0, pure = 0;
    double tol = 0.0;
    std::vector<int> l, nprim, atom, poff, bf;
    std::vector<double> coords, centers, alpha, coef;
    // all shell pairs s1 >= s2 (reference order), canonical records
    std::vector<PairInfo> pairs;
    std::vector<int> pcls;
    PrimPair* d_prims = nullptr;
    PairInfo* d_pairs = nullptr;
    double* d_boys = nullptr;
    const double* d_rys = nullptr;  // Rys node/weight table (module data, not owned)
    int* d_err = nullptr;
    double* d_scratch = nullptr;  // accumulators of classes too large for shared memory
    long long scratch_len = 0;
    std::vector<double> K;  // nshell^2
    double kmax = 0.0;
    ClassWork work[QX_NCLS_ALL];
    long long nunique = 0, unique_size = 0;
    cudaStream_t streams[QX_NSTREAMS] = {};
    cudaEvent_t done[QX_NSTREAMS] = {};
    cudaEvent_t start = nullptr;
    int order[QX_NCLS_ALL];  // classes by decreasing primitive work
    int plain_eng[QX_NCLS_ALL];
    int deriv_eng[QX_NCLS_ALL];
    int wpq[QX_NCLS_ALL];        // warps per quartet, plain warp kernels
    int wpq_deriv[QX_NCLS_ALL];  // warps per quartet, derivative warp kernels
    int rys_lp[QX_NCLS_ALL];     // Rys adjoint gradient: 1 = level-parallel table build (RK_GRADL)
    int shard_rank = 0, shard_n = 1;
    int prim_stage = 0;  // split-mode VRR: primitive pairs staged per warp (2 x largest pair), 0 = off
    int wait_limit = 1 << 22;  // polls of the bounded waits on those staging copies
    // J/K density screening: sqrt(K) and max |D| per pair record, threshold of the
    // call in progress (0 = off)
    double* d_kpair = nullptr;
    double* d_dmax = nullptr;
    double jk_thr = 0.0;
    // one-electron integrals: nuclear charges and positions on the device
    double* d_Z = nullptr;
    double* d_xyz = nullptr;
    double f32_bound = 0.0;  // mixed precision: FP32 recurrences below this Schwarz bound
};

// Primitive-chunk tasks (quartet, first primitive quartet) of the split modes,
// built at set-up for the classes that use them by default and otherwise at the
// first call that needs them; the derivative accumulator buffer is allocated at
// the first derivative call (need_dacc).  The quartets are cut into slices of at
// most QX_SPLIT_ACC_BYTES of derivative accumulators; each slice runs as its own
// VRR + HRR pair.  `list` is the class's current view when the caller has it on
// the host (set-up), else it is copied back from the device.
// Runs f(0..nt-1) on nt host threads (f(0) on the caller's).
template <class F>
static void host_parallel(int nt, F&& f) {
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back([&f, t] { f(t); });
    f(0);
    for (auto& th : pool) th.join();
}

static int ensure_split_tasks(qx_handle* h, int c, bool need_dacc = false, const int2* list = nullptr,
                              bool sync = true) {
    ClassWork& w = h->work[c];
    if (!w.nq) return QX_OK;
    const long long nacc = qx_der_nacc(g_der_idx[c]);
    const long long cap_q = std::max(1LL, QX_SPLIT_ACC_BYTES / (8 * nacc));
    if (!w.d_dtasks) {
        std::vector<int2> L;
        if (!list) {
            L.resize((size_t)w.nq);
            QX_CUDA(cudaMemcpy(L.data(), w.d_q, sizeof(int2) * w.nq, cudaMemcpyDeviceToHost));
            list = L.data();
        }
        // tasks (slice-relative quartet, first primitive quartet), ch primitive
        // quartets each; slices of cap_q quartets.  Built over host threads: each
        // counts the tasks of a contiguous quartet range, then writes them after an
        // exclusive scan, recording the task offset of the slice starts in its range.
        const int ch = qx_der_chunk();
        const long long nslice = (w.nq + cap_q - 1) / cap_q;
        const int nt = (int)std::max(1LL, std::min<long long>(std::max(1u, std::thread::hardware_concurrency()),
                                                              w.nq / 65536));
        std::vector<long long> tcount(nt + 1, 0);
        auto q_lo = [&](int t) { return w.nq * t / nt; };
        auto ntask = [&](long long qi) {
            const int np_q = h->pairs[list[qi].x].nprim * h->pairs[list[qi].y].nprim;
            return (long long)((np_q + ch - 1) / ch);
        };
        host_parallel(nt, [&](int t) {
            long long n = 0;
            for (long long qi = q_lo(t); qi < q_lo(t + 1); ++qi) n += ntask(qi);
            tcount[t + 1] = n;
        });
        for (int t = 0; t < nt; ++t) tcount[t + 1] += tcount[t];
        const long long ntot = tcount[nt];
        std::unique_ptr<int2[]> tasks(new int2[(size_t)std::max(1LL, ntot)]);
        w.slice_q.assign((size_t)nslice + 1, 0);
        w.slice_t.assign((size_t)nslice + 1, 0);
        for (long long k = 0; k <= nslice; ++k) w.slice_q[k] = std::min(w.nq, k * cap_q);
        w.slice_t[nslice] = ntot;
        host_parallel(nt, [&](int t) {
            long long pos = tcount[t];
            for (long long qi = q_lo(t); qi < q_lo(t + 1); ++qi) {
                if (qi % cap_q == 0) w.slice_t[qi / cap_q] = pos;
                const int rel = (int)(qi % cap_q);
                const int np_q = h->pairs[list[qi].x].nprim * h->pairs[list[qi].y].nprim;
                for (int t0 = 0; t0 < np_q; t0 += ch) tasks[pos++] = make_int2(rel, t0);
            }
        });
        if (cudaMalloc((void**)&w.d_dtasks, sizeof(int2) * std::max(1LL, ntot)) != cudaSuccess) {
            cudaGetLastError();
            w.d_dtasks = nullptr;
            return fail(QX_E_NOMEM, "split-mode tasks for class %d", c);
        }
        w.ndtask = ntot;
        QX_CUDA(cudaMemcpy(w.d_dtasks, tasks.get(), sizeof(int2) * ntot, cudaMemcpyHostToDevice));
        // a pageable host-to-device copy may still be in flight when cudaMemcpy
        // returns, and the kernels that read the tasks run on non-blocking streams
        // (set-up synchronises once at its end instead)
        if (sync) QX_CUDA(cudaDeviceSynchronize());
    }
    if (need_dacc && !w.d_dacc &&
        cudaMalloc((void**)&w.d_dacc, sizeof(double) * std::min(w.nq, cap_q) * ((nacc + 15) / 16 * 16)) !=
            cudaSuccess) {
        cudaGetLastError();
        w.d_dacc = nullptr;
        return fail(QX_E_NOMEM, "split-mode derivative accumulators for class %d", c);
    }
    return QX_OK;
}

// Plain items per quartet of the warp programs (the accumulator targets, padded
// to the 16-item staging groups).
static long long plain_items(int c) { return (g_class_nacc[c] + 15) / 16 * 16; }

// Warps per quartet: classes with few quartets but long primitive loops let four
// warps share a quartet so the GPU fills up.
static int choose_wpq(long long nq, long long prims) {
    const double avg = nq ? (double)prims / nq : 0.0;
    return (nq < 20000 && avg >= 4 * 32) ? 4 : 1;
}

// Default engine choice, overridable with QX_PLAIN_ENGINE=sl|warp|coop|wsplit and
// QX_DERIV_ENGINE=coop|wvrr|dsplit (for measuring alternatives); an override that a class
// cannot honour falls back to the default.
static void choose_engines(qx_handle* h) {
    const char* pe = std::getenv("QX_PLAIN_ENGINE");
    const char* de = std::getenv("QX_DERIV_ENGINE");
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        if (!has_os(c)) {  // f shells: the Rys engine only
            h->plain_eng[c] = h->deriv_eng[c] = ENG_RYS;
            continue;
        }
        int p;
        if (g_has_pvrr[c]) p = ENG_WSPLIT;  // measured fastest for these classes
        else if (g_has_warp_plain[c] && g_class_nacc[c] > 48) p = ENG_WARP;
        else if (!g_class_coop[c]) p = ENG_SL;
        else p = g_has_warp_plain[c] ? ENG_WARP : ENG_COOP;
        if (pe) {
            if (!std::strcmp(pe, "sl") && !g_class_coop[c]) p = ENG_SL;
            if (!std::strcmp(pe, "warp") && g_has_warp_plain[c]) p = ENG_WARP;
            if (!std::strcmp(pe, "coop") && g_class_coop[c]) p = ENG_COOP;
            if (!std::strcmp(pe, "wsplit") && g_has_pvrr[c]) p = ENG_WSPLIT;
        }
        // split VRR with the warp HRR where the class has it, else the split VRR with
        // the cooperative HRR for L >= 6 (measured on the 10-atom workload); the
        // autotuner settles each class per molecule
        const int L = g_class_l[c][0] + g_class_l[c][1] + g_class_l[c][2] + g_class_l[c][3];
        int d = g_has_dsplit[c] ? ENG_DSPLIT
                : (g_has_wvrr[c] && (L >= 6 || !g_has_warp_deriv[c])) ? ENG_WVRR
                : (g_has_warp_deriv[c] ? ENG_WARP : ENG_COOP);
        if (de && !std::strcmp(de, "coop")) d = ENG_COOP;
        if (de && !std::strcmp(de, "wvrr") && g_has_wvrr[c]) d = ENG_WVRR;
        if (de && !std::strcmp(de, "dsplit") && g_has_dsplit[c]) d = ENG_DSPLIT;
        h->plain_eng[c] = p;
        h->deriv_eng[c] = d;
    }
}

static int pair_index(int s1, int s2) { return s1 * (s1 + 1) / 2 + s2; }  // s1 >= s2

static void free_handle(qx_handle* h) {
    if (!h) return;
    cudaFree(h->d_prims);
    cudaFree(h->d_pairs);
    cudaFree(h->d_boys);
    cudaFree(h->d_err);
    cudaFree(h->d_scratch);
    for (auto& w : h->work) {
        cudaFree(w.d_q_full);
        cudaFree(w.scratch);
        cudaFree(w.d_dtasks);
        cudaFree(w.d_dacc);
        cudaFree(w.d_pacc);
    }
    for (int i = 0; i < QX_NSTREAMS; ++i) {
        if (h->streams[i]) cudaStreamDestroy(h->streams[i]);
        if (h->done[i]) cudaEventDestroy(h->done[i]);
    }
    if (h->start) cudaEventDestroy(h->start);
    cudaFree(h->d_Z);
    cudaFree(h->d_xyz);
    cudaFree(h->d_kpair);
    cudaFree(h->d_dmax);
    delete h;
}

static int run_class(qx_handle* h, int cls, int mode, const int2* d_q, long long nq, double* out, long long n,
                     long long base, cudaStream_t s, int log2g = 0, double* scratch = nullptr, double* out2 = nullptr,
                     const double* dens = nullptr) {
    const int eng = h->plain_eng[cls];
    EriArgs a;
    a.quartets = d_q;
    a.nq = nq;
    a.pairs = h->d_pairs;
    a.prims = h->d_prims;
    a.boys = h->d_boys;
    a.out = out;
    a.n = n;
    a.base = base;
    a.scratch = scratch ? scratch : h->d_scratch;
    a.out2 = out2;
    a.dens = dens;
    a.log2g = eng == ENG_SL ? log2g : 0;
    a.err = h->d_err;
    if (d_q == h->work[cls].d_q) a.nq64 = h->work[cls].nq64;
    if (mode == MODE_JK && h->jk_thr > 0.0) {
        a.jk_thr = h->jk_thr;
        a.jk_kpair = h->d_kpair;
        a.jk_dmax = h->d_dmax;
    }
    if (eng == ENG_RYS) {
        RysArgs ra;
        ra.e = a;
        ra.rys = h->d_rys;
        if (g_rys_launch[cls](ra, RK_PLAIN, mode, nq, s))
            return fail(QX_E_UNSUPPORTED, "class (%d%d|%d%d): no Rys program", g_class_l[cls][0], g_class_l[cls][1],
                        g_class_l[cls][2], g_class_l[cls][3]);
    } else if (eng == ENG_COOP) {
        qx_launch_coop(g_coop_idx[cls], a, mode, s);
    } else if (eng == ENG_WARP || eng == ENG_WSPLIT) {
        WarpArgs wa;
        wa.e = a;
        wa.wpq = h->wpq[cls];
        wa.D = nullptr;
        wa.cj = wa.ck = 0.0;
        wa.grad = nullptr;
        wa.slice = -1;
        ClassWork& w = h->work[cls];
        if (eng == ENG_WSPLIT && d_q == w.d_q && !ensure_split_tasks(h, cls) && w.slice_q.size() == 2) {
            // VRR by (quartet, primitive chunk) tasks into global accumulators, then
            // the warp HRR + epilogue from them (one quartet per warp).  A class too
            // large for one accumulator slice runs the plain warp kernel instead.
            const long long np = plain_items(cls);
            if (!w.d_pacc && cudaMalloc((void**)&w.d_pacc, sizeof(double) * w.nq * np) != cudaSuccess) {
                cudaGetLastError();
                w.d_pacc = nullptr;
                return fail(QX_E_NOMEM, "plain split-mode accumulators for class %d", cls);
            }
            QX_CUDA(cudaMemsetAsync(w.d_pacc, 0, sizeof(double) * w.nq * np, s));
            EriArgs av = a;
            av.prim_stage = h->prim_stage;
            av.wait_limit = h->wait_limit;
            g_pvrr[cls](av, w.d_dtasks, w.ndtask, qx_der_chunk(), w.d_pacc, (int)np, s);
            wa.wpq = 1;
            wa.acc_in = w.d_pacc;
        }
        g_warp_plain[cls](wa, mode, s);
    } else {
        g_eri_launch[cls](a, mode, s);
    }
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

// QX_TRACE_INIT=1 prints the set-up phases' wall times to stderr (diagnostics).
namespace {
struct InitTrace {
    bool on = std::getenv("QX_TRACE_INIT") != nullptr;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    void mark(const char* what) {
        if (!on) return;
        const auto t1 = std::chrono::steady_clock::now();
        std::fprintf(stderr, "qx_initialize: %-28s %8.3f ms\n", what,
                     std::chrono::duration<double, std::milli>(t1 - t0).count());
        t0 = t1;
    }
};
}  // namespace

extern "C" int qx_initialize(int natom, const double* coords, int nshell, const int* shell_l, const int* shell_nprim,
                             const int* shell_atom, const double* exps, const double* coefs, int pure,
                             double ints_tol, qx_handle** out) {
    if (!out) return fail(QX_E_INVALID, "qx_initialize: out is NULL");
    *out = nullptr;
    if (natom <= 0 || nshell <= 0 || !coords || !shell_l || !shell_nprim || !shell_atom || !exps || !coefs)
        return fail(QX_E_INVALID, "qx_initialize: empty geometry or shell list");
    if (pure != 0) return fail(QX_E_UNSUPPORTED, "qx_initialize: only Cartesian shells (pure=0) are supported");
    if (!(ints_tol > 0.0) || !std::isfinite(ints_tol)) return fail(QX_E_INVALID, "qx_initialize: ints_tol must be > 0");
    for (int i = 0; i < 3 * natom; ++i)
        if (!std::isfinite(coords[i])) return fail(QX_E_INVALID, "qx_initialize: non-finite coordinate %d", i);
    InitTrace trace;
    qx_handle* h = new qx_handle();
    cudaGetDevice(&h->device);
    choose_engines(h);
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        h->wpq[c] = h->wpq_deriv[c] = 1;
        h->rys_lp[c] = 0;
    }
    h->natom = natom;
    h->nshell = nshell;
    h->pure = pure;
    h->tol = ints_tol;
    h->coords.assign(coords, coords + 3 * natom);
    ShellTables shells;
    {
        std::string err;
        const int rc = normalize_shells("qx_initialize", natom, nshell, shell_l, shell_nprim, shell_atom, exps, coefs,
                                        QX_RYS_LMAX, shells, err);
        if (rc) {
            free_handle(h);
            return fail(rc, "%s", err.c_str());
        }
    }
    h->l = shells.l;
    h->nprim = shells.nprim;
    h->atom = shells.atom;
    h->poff = shells.poff;
    h->bf = shells.bf;
    h->alpha = shells.alpha;
    h->coef = shells.coef;
    h->nbf = shells.nbf;
    for (int s = 0; s < nshell; ++s)
        for (int c = 0; c < 3; ++c) h->centers.push_back(coords[3 * shells.atom[s] + c]);
    trace.mark("shells");
    // pair records
    std::vector<PrimPair> prims;
    build_pairs(shells, coords, prims, h->pairs, h->pcls);
    const std::vector<double>& boys = boys_table();
    const int np = (int)h->pairs.size();
    {
        // bulk-copy staging of the primitive pairs in the split-mode VRR kernels:
        // room for one bra and one ket pair, up to 64 primitive pairs each (10 KB
        // per warp); QX_NO_STAGE=1 reads them from global memory instead
        int mx = 0;
        for (const auto& pi : h->pairs) mx = std::max(mx, pi.nprim);
        h->prim_stage = (mx <= 64 && !std::getenv("QX_NO_STAGE")) ? 2 * mx : 0;
    }
#define QX_ALLOC(ptr, bytes)                                                          \
    do {                                                                              \
        if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) {                     \
            cudaGetLastError();                                                       \
            free_handle(h);                                                           \
            return fail(QX_E_NOMEM, "qx_initialize: cudaMalloc of %zu bytes failed", \
                        (size_t)(bytes));                                             \
        }                                                                             \
    } while (0)
    h->d_rys = qx_rys_table();
    if (!h->d_rys) {
        free_handle(h);
        return fail(QX_E_CUDA, "qx_initialize: Rys table not found on device %d", h->device);
    }
    QX_ALLOC(h->d_prims, sizeof(PrimPair) * prims.size());
    QX_ALLOC(h->d_pairs, sizeof(PairInfo) * np);
    QX_ALLOC(h->d_boys, sizeof(double) * boys.size());
    QX_ALLOC(h->d_err, sizeof(int));
    cudaMemcpy(h->d_prims, prims.data(), sizeof(PrimPair) * prims.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_pairs, h->pairs.data(), sizeof(PairInfo) * np, cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_boys, boys.data(), sizeof(double) * boys.size(), cudaMemcpyHostToDevice);
    cudaMemset(h->d_err, 0, sizeof(int));
    // global accumulator scratch, sized for the largest launch that needs it
    {
        long long need = 0;
        for (int c = 0; c < QX_NCLS_ALL; ++c) need = std::max(need, g_class_scratch[c] * launch_threads(np, 0));
        if (need) {
            QX_ALLOC(h->d_scratch, sizeof(double) * need);
            h->scratch_len = need;
        }
    }
    // Schwarz: diagonal quartets (P|P) of every pair
    {
        std::vector<std::vector<int2>> diag(QX_NPCLS_ALL);
        for (int p = 0; p < np; ++p) diag[h->pcls[p]].push_back(make_int2(p, p));
        double* d_kp = nullptr;
        int2* d_dq = nullptr;
        QX_ALLOC(d_kp, sizeof(double) * np);
        QX_ALLOC(d_dq, sizeof(int2) * np);
        long long o = 0;
        for (int pc = 0; pc < QX_NPCLS_ALL; ++pc) {
            if (diag[pc].empty()) continue;
            cudaMemcpy(d_dq + o, diag[pc].data(), sizeof(int2) * diag[pc].size(), cudaMemcpyHostToDevice);
            // few quartets with long primitive loops: 32 lanes (straight-line kernels
            // without global accumulators) or 4 warps (warp kernels) per quartet
            const int cls = quartet_class(pc, pc);
            const int keep_wpq = h->wpq[cls];
            h->wpq[cls] = 4;
            int rc = run_class(h, cls, MODE_SCHWARZ, d_dq + o, (long long)diag[pc].size(), d_kp, 0, 0, 0,
                               g_class_scratch[cls] ? 0 : 5);
            h->wpq[cls] = keep_wpq;
            if (rc) { cudaFree(d_kp); cudaFree(d_dq); free_handle(h); return rc; }
            o += diag[pc].size();
        }
        std::vector<double> kp(np);
        cudaError_t e = cudaMemcpy(kp.data(), d_kp, sizeof(double) * np, cudaMemcpyDeviceToHost);
        cudaFree(d_kp);
        cudaFree(d_dq);
        if (e != cudaSuccess) {
            free_handle(h);
            return fail(QX_E_CUDA, "qx_initialize: Schwarz kernels failed: %s", cudaGetErrorString(e));
        }
        h->K.assign((size_t)nshell * nshell, 0.0);
        for (int p = 0; p < np; ++p) {
            const int s1 = h->pairs[p].s1, s2 = h->pairs[p].s2;
            h->K[(size_t)s1 * nshell + s2] = h->K[(size_t)s2 * nshell + s1] = kp[p];
            h->kmax = std::max(h->kmax, kp[p]);
        }
    }
    trace.mark("pairs, uploads, Schwarz");
    // screened pair list (reference order s1 >= s2) and unique quartets
    const double thr2 = ints_tol * ints_tol;
    const double cut = thr2 / h->kmax;
    std::vector<int> kept;
    std::vector<double> kk;
    for (int s1 = 0; s1 < nshell; ++s1)
        for (int s2 = 0; s2 <= s1; ++s2)
            if (h->K[(size_t)s1 * nshell + s2] >= cut) {
                kept.push_back(pair_index(s1, s2));
                kk.push_back(h->K[(size_t)s1 * nshell + s2]);
            }
    // Pair-pair enumeration and the per-class counting sort by (bra nprim, ket
    // nprim), largest first (equal trip counts within a warp, the cheap quartets in
    // the tail of a launch), as a two-pass stable counting sort over host threads:
    // thread t takes a contiguous range of i of about equal work (~i^2 / 2), counts
    // its quartets per (class, key), and after an exclusive scan in (key, thread)
    // order writes them straight to their sorted positions -- the same lists as a
    // serial enumeration followed by a stable sort.
    constexpr int NKEY = 64 * 64;
    const size_t nk = kept.size();
    const int nt = (int)std::max<size_t>(
        1, std::min<size_t>(std::min(32u, std::max(1u, std::thread::hardware_concurrency())),
                            std::max<size_t>(1, nk / 256)));  // <= 32: the count tables grow with the thread count
    std::vector<size_t> cut_i(nt + 1, nk);
    cut_i[0] = 0;
    for (int t = 1; t < nt; ++t) cut_i[t] = (size_t)(nk * std::sqrt((double)t / nt));
    auto key = [&](int pb, int pk) {
        return NKEY - 1 - std::min((h->pairs[pb].nprim - 1) * 64 + (h->pairs[pk].nprim - 1), NKEY - 1);
    };
    auto visit = [&](int t, auto&& fn) {
        for (size_t i = cut_i[t]; i < cut_i[t + 1]; ++i)
            for (size_t j = 0; j <= i; ++j) {
                if (kk[i] * kk[j] < thr2) continue;
                int pb = kept[i], pk = kept[j];
                if (h->pcls[pb] < h->pcls[pk]) std::swap(pb, pk);
                fn(quartet_class(h->pcls[pb], h->pcls[pk]), key(pb, pk), pb, pk);
            }
    };
    std::vector<long long> cnt((size_t)nt * QX_NCLS_ALL * NKEY, 0);
    std::vector<long long> tprims((size_t)nt * QX_NCLS_ALL, 0);
    host_parallel(nt, [&](int t) {
        long long* C = cnt.data() + (size_t)t * QX_NCLS_ALL * NKEY;
        long long* P = tprims.data() + (size_t)t * QX_NCLS_ALL;
        visit(t, [&](int c, int k, int pb, int pk) {
            C[(size_t)c * NKEY + k]++;
            P[c] += (long long)h->pairs[pb].nprim * h->pairs[pk].nprim;
        });
    });
    std::vector<long long> nq_c(QX_NCLS_ALL, 0), prims_c(QX_NCLS_ALL, 0);
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        long long run = 0;
        for (int k = 0; k < NKEY; ++k)
            for (int t = 0; t < nt; ++t) {
                long long& x = cnt[((size_t)t * QX_NCLS_ALL + c) * NKEY + k];
                const long long v = x;
                x = run;
                run += v;
            }
        nq_c[c] = run;
        for (int t = 0; t < nt; ++t) prims_c[c] += tprims[(size_t)t * QX_NCLS_ALL + c];
    }
    std::vector<std::unique_ptr<int2[]>> sorted(QX_NCLS_ALL);
    for (int c = 0; c < QX_NCLS_ALL; ++c)
        if (nq_c[c]) sorted[c].reset(new int2[(size_t)nq_c[c]]);
    host_parallel(nt, [&](int t) {
        long long* C = cnt.data() + (size_t)t * QX_NCLS_ALL * NKEY;
        visit(t, [&](int c, int k, int pb, int pk) { sorted[c][C[(size_t)c * NKEY + k]++] = make_int2(pb, pk); });
    });
    std::vector<long long>().swap(cnt);
    trace.mark("quartet enumeration, sort");
    long long base = 0;
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        ClassWork& w = h->work[c];
        w.nq = nq_c[c];
        w.prims = prims_c[c];
        w.log2g = h->plain_eng[c] == ENG_SL ? choose_log2g(w.nq, w.prims) : 0;
        h->wpq[c] = h->wpq_deriv[c] = choose_wpq(w.nq, w.prims);
        w.unique_base = base;
        base += w.nq * g_class_nout[c];
        h->nunique += w.nq;
        if (w.nq) {
            QX_ALLOC(w.d_q, sizeof(int2) * w.nq);
            cudaMemcpy(w.d_q, sorted[c].get(), sizeof(int2) * w.nq, cudaMemcpyHostToDevice);
            w.d_q_full = w.d_q;
            w.nq_full = w.nq;
            if (h->plain_eng[c] == ENG_WSPLIT) {
                int rc = ensure_split_tasks(h, c, false, sorted[c].get(), false);
                if (rc) {
                    free_handle(h);
                    return rc;
                }
            }
            if (g_class_scratch[c] && h->plain_eng[c] == ENG_SL)
                QX_ALLOC(w.scratch, sizeof(double) * g_class_scratch[c] * launch_threads(w.nq, w.log2g));
            sorted[c].reset();
        }
    }
    h->unique_size = base;
    trace.mark("list uploads, split tasks");
    for (int c = 0; c < QX_NCLS_ALL; ++c) h->order[c] = c;
    std::sort(h->order, h->order + QX_NCLS_ALL,
              [&](int x, int y) { return h->work[x].prims * g_class_nout[x] > h->work[y].prims * g_class_nout[y]; });
    for (int i = 0; i < QX_NSTREAMS; ++i) {
        if (cudaStreamCreateWithFlags(&h->streams[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->done[i], cudaEventDisableTiming) != cudaSuccess) {
            free_handle(h);
            return fail(QX_E_CUDA, "qx_initialize: stream creation failed");
        }
    }
    if (cudaEventCreateWithFlags(&h->start, cudaEventDisableTiming) != cudaSuccess) {
        free_handle(h);
        return fail(QX_E_CUDA, "qx_initialize: event creation failed");
    }
#undef QX_ALLOC
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        free_handle(h);
        return fail(QX_E_CUDA, "qx_initialize: %s", cudaGetErrorString(e));
    }
    trace.mark("streams, final sync");
    *out = h;
    return QX_OK;
}

// ------------------------------------------------------------------ shards ----
// Cost-balanced contiguous cut of a list: item i (cost c_i, prefix C_i, total T)
// goes to rank floor(nranks (C_i + c_i / 2) / T), which is monotone in i, so each
// rank gets one contiguous range; bounds[r] .. bounds[r+1] is rank r's.
extern "C" int qx_partition_costs(const double* cost, long long n, int nranks, long long* bounds) {
    if (!bounds || nranks < 1 || n < 0 || (n > 0 && !cost)) return fail(QX_E_INVALID, "qx_partition_costs: bad argument");
    double T = 0.0;
    for (long long i = 0; i < n; ++i) {
        if (!(cost[i] >= 0.0) || !std::isfinite(cost[i])) return fail(QX_E_INVALID, "qx_partition_costs: bad cost");
        T += cost[i];
    }
    for (int r = 0; r <= nranks; ++r) bounds[r] = r == 0 ? 0 : n;
    if (n == 0) return QX_OK;
    double C = 0.0;
    int cur = 0;
    for (long long i = 0; i < n; ++i) {
        int r = T > 0.0 ? (int)std::floor(nranks * (C + 0.5 * cost[i]) / T) : (int)(i * nranks / n);
        r = std::min(std::max(r, cur), nranks - 1);
        while (cur < r) bounds[++cur] = i;
        C += cost[i];
    }
    while (cur < nranks - 1) bounds[++cur] = n;
    bounds[nranks] = n;
    return QX_OK;
}

// Recompute every class's view (this rank's contiguous range of the full list,
// with its FP64/FP32 boundary) and the unique layout; split-mode buffers belong to
// the old view and are dropped.
static int rebuild_views(qx_handle* h) {
    QX_CUDA(cudaDeviceSynchronize());
    const int rank = h->shard_rank, nranks = h->shard_n;
    long long base = 0;
    h->nunique = 0;
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        ClassWork& w = h->work[c];
        cudaFree(w.d_dtasks);
        cudaFree(w.d_dacc);
        cudaFree(w.d_pacc);
        w.d_dtasks = nullptr;
        w.d_dacc = w.d_pacc = nullptr;
        w.ndtask = 0;
        w.slice_q.clear();
        w.slice_t.clear();
        long long lo = 0, hi = w.nq_full;
        long long prims = 0;
        if (w.nq_full) {
            std::vector<int2> L((size_t)w.nq_full);
            QX_CUDA(cudaMemcpy(L.data(), w.d_q_full, sizeof(int2) * w.nq_full, cudaMemcpyDeviceToHost));
            std::vector<double> cost((size_t)w.nq_full);
            for (long long i = 0; i < w.nq_full; ++i)
                cost[i] = (double)h->pairs[L[i].x].nprim * h->pairs[L[i].y].nprim;
            std::vector<long long> b(nranks + 1);
            int rc = qx_partition_costs(cost.data(), w.nq_full, nranks, b.data());
            if (rc) return rc;
            lo = b[rank];
            hi = b[rank + 1];
            for (long long i = lo; i < hi; ++i) prims += (long long)cost[i];
        }
        w.d_q = w.d_q_full + lo;
        w.nq = hi - lo;
        w.prims = prims;
        w.nq64 = w.n64_full >= hi ? 0x7fffffffffffffffLL : std::max(0LL, w.n64_full - lo);
        w.unique_base = base;
        base += w.nq * g_class_nout[c];
        h->nunique += w.nq;
    }
    h->unique_size = base;
    return QX_OK;
}

// Restrict the handle to rank `rank` of `nranks`: every class keeps a
// cost-balanced contiguous range of its screened quartets (cost = primitive
// quartets), so the ranks' results (dense tensors, derivative tensors, J, K,
// gradients) sum to the full one.  The unique layout then holds this rank's
// quartets only.  nranks = 1 restores the full lists.
extern "C" int qx_set_shard(qx_handle* h, int rank, int nranks) {
    if (!h || nranks < 1 || rank < 0 || rank >= nranks) return fail(QX_E_INVALID, "qx_set_shard: bad rank/nranks");
    DeviceGuard g(h->device);
    h->shard_rank = rank;
    h->shard_n = nranks;
    return rebuild_views(h);
}

// Mixed precision: quartets whose Schwarz bound sqrt(K_ab K_cd) is below `bound`
// run their recurrences in FP32 (warp and split engines; set-up, Boys function,
// accumulation over primitives, HRR and epilogues stay FP64).  Each class's list
// is reordered to hold its FP64 quartets first (both parts keep the
// largest-primitive-count-first order), which also reorders the unique layout.
// bound <= 0 makes every quartet FP64 again.
extern "C" int qx_set_precision(qx_handle* h, double bound) {
    if (!h || !std::isfinite(bound)) return fail(QX_E_INVALID, "qx_set_precision: bad argument");
    DeviceGuard g(h->device);
    QX_CUDA(cudaDeviceSynchronize());
    h->f32_bound = bound > 0.0 ? bound : 0.0;
    const double b2 = h->f32_bound * h->f32_bound;
    const int ns = h->nshell;
    auto kpair = [&](const PairInfo& p) { return h->K[(size_t)p.s1 * ns + p.s2]; };
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        ClassWork& w = h->work[c];
        if (!w.nq_full) continue;
        std::vector<int2> L((size_t)w.nq_full);
        QX_CUDA(cudaMemcpy(L.data(), w.d_q_full, sizeof(int2) * w.nq_full, cudaMemcpyDeviceToHost));
        // restore the set-up order (bra nprim, then ket nprim, largest first), then
        // split by the bound
        auto key = [&](const int2& q) { return h->pairs[q.x].nprim * 64 + h->pairs[q.y].nprim; };
        std::stable_sort(L.begin(), L.end(), [&](const int2& x, const int2& y) { return key(x) > key(y); });
        // FP32 recurrence errors are amplified by the HRR's cancellations, about
        // tenfold per transfer step (measured relative error of the FP32 path:
        // <= 4e-5 with lb + ld <= 1, ~2e-3 with 2, 1e-1 with 3, above 1 with 4), so
        // classes with more than two transfer steps stay FP64
        const bool eligible = has_os(c) && g_class_l[c][1] + g_class_l[c][3] <= 2;
        auto is64 = [&](const int2& q) {
            return !eligible || b2 <= 0.0 || kpair(h->pairs[q.x]) * kpair(h->pairs[q.y]) >= b2;
        };
        auto mid = std::stable_partition(L.begin(), L.end(), is64);
        const long long n64 = (long long)(mid - L.begin());
        w.n64_full = n64 == w.nq_full ? 0x7fffffffffffffffLL : n64;
        QX_CUDA(cudaMemcpy(w.d_q_full, L.data(), sizeof(int2) * w.nq_full, cudaMemcpyHostToDevice));
    }
    return rebuild_views(h);
}

extern "C" long long qx_precision_split(const qx_handle* h, int cls) {
    if (!h || cls < 0 || cls >= QX_NCLS_ALL) return fail(QX_E_INVALID, "qx_precision_split: bad argument");
    const ClassWork& w = h->work[cls];
    return w.nq64 >= w.nq ? w.nq : w.nq64;
}

extern "C" int qx_finalize(qx_handle* h) {
    if (!h) return fail(QX_E_INVALID, "qx_finalize: NULL handle");
    DeviceGuard g(h->device);
    free_handle(h);
    return QX_OK;
}

extern "C" int qx_nbf(const qx_handle* h) { return h ? h->nbf : fail(QX_E_INVALID, "NULL handle"); }
extern "C" int qx_natom(const qx_handle* h) { return h ? h->natom : fail(QX_E_INVALID, "NULL handle"); }
extern "C" int qx_nshell(const qx_handle* h) { return h ? h->nshell : fail(QX_E_INVALID, "NULL handle"); }
extern "C" long long qx_unique_quartets(const qx_handle* h) { return h ? h->nunique : -1; }
extern "C" long long qx_unique_size(const qx_handle* h) { return h ? h->unique_size : -1; }

extern "C" int qx_schwarz(qx_handle* h, double* K, double* kmax) {
    if (!h || !K) return fail(QX_E_INVALID, "qx_schwarz: NULL argument");
    std::memcpy(K, h->K.data(), sizeof(double) * h->K.size());
    if (kmax) *kmax = h->kmax;
    return QX_OK;
}

static int check_err_word(qx_handle* h, cudaStream_t s) {
    int e = 0;
    QX_CUDA(cudaMemcpyAsync(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    QX_CUDA(cudaStreamSynchronize(s));
    if (e) {
        cudaMemsetAsync(h->d_err, 0, sizeof(int), s);
        return fail(QX_E_DEVICE, "kernel error word 0x%x", e);
    }
    return QX_OK;
}

// Launch every class on the handle's internal streams (largest work first,
// round-robin), ordered after the caller's stream and joined back into it.
static int run_all_classes(qx_handle* h, int mode, double* out, long long n, cudaStream_t s, double* out2 = nullptr,
                           const double* dens = nullptr) {
    QX_CUDA(cudaEventRecord(h->start, s));
    for (int i = 0; i < QX_NSTREAMS; ++i) QX_CUDA(cudaStreamWaitEvent(h->streams[i], h->start, 0));
    int k = 0;
    for (int oi = 0; oi < QX_NCLS_ALL; ++oi) {
        const int c = h->order[oi];
        const ClassWork& w = h->work[c];
        if (!w.nq) continue;
        cudaStream_t cs = h->streams[k++ % QX_NSTREAMS];
        int rc = run_class(h, c, mode, w.d_q, w.nq, out, n, w.unique_base, cs, w.log2g, w.scratch, out2, dens);
        if (rc) return rc;
    }
    for (int i = 0; i < QX_NSTREAMS; ++i) {
        QX_CUDA(cudaEventRecord(h->done[i], h->streams[i]));
        QX_CUDA(cudaStreamWaitEvent(s, h->done[i], 0));
    }
    return QX_OK;
}

// Device staging of host outputs: one buffer per device, grown on demand and kept
// for the life of the process, so a host-output call allocates nothing once the
// buffer is large enough (the dense tensors are GBs: a cudaMalloc/cudaFree pair
// per call cost up to a few hundred ms).  Calls that stage on the same device are
// serialised by the device's lock, held until their copy-out completes.
namespace {
struct Staging {
    std::mutex mu;
    double* p = nullptr;
    size_t cap = 0;  // doubles
};
constexpr int kStagingDevices = 64;
Staging g_staging[kStagingDevices];
}  // namespace

// Returns the device's staging buffer with room for `count` doubles (lk must lock
// the device's mutex), or nullptr when the device cannot provide it.
static double* staging_get(int dev, size_t count, std::unique_lock<std::mutex>& lk) {
    if (dev < 0 || dev >= kStagingDevices) return nullptr;
    Staging& st = g_staging[dev];
    lk = std::unique_lock<std::mutex>(st.mu);
    if (st.cap < count) {
        cudaFree(st.p);
        st.p = nullptr;
        st.cap = 0;
        if (cudaMalloc((void**)&st.p, sizeof(double) * count) != cudaSuccess) {
            cudaGetLastError();
            st.p = nullptr;
            return nullptr;
        }
        st.cap = count;
    }
    return st.p;
}

// Stages a host output buffer through the device when out_on_device == 0.
template <class F>
static int with_output(qx_handle* h, double* out, size_t count, int out_on_device, cudaStream_t s, F&& body) {
    if (out_on_device) return body(out);
    std::unique_lock<std::mutex> lk;
    double* d = staging_get(h->device, count, lk);
    if (!d) return fail(QX_E_NOMEM, "cannot stage %zu bytes on the device", sizeof(double) * count);
    int rc = body(d);
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(out, d, sizeof(double) * count, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(QX_E_CUDA, "copy-out failed: %s", cudaGetErrorString(e));
    }
    if (!rc) rc = check_err_word(h, s);
    return rc;
}

static int eri_dense_dev(qx_handle* h, double* out, cudaStream_t s) {
    const long long n = h->nbf;
    QX_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * n * n * n * n, s));
    return run_all_classes(h, MODE_DENSE, out, n, s);
}

extern "C" int qx_compute_2e_int(qx_handle* h, double* out, int out_on_device, void* stream) {
    if (!h || !out) return fail(QX_E_INVALID, "qx_compute_2e_int: NULL argument");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = h->nbf;
    return with_output(h, out, (size_t)(n * n * n * n), out_on_device, s, [&](double* d) { return eri_dense_dev(h, d, s); });
}

extern "C" int qx_eri_unique(qx_handle* h, double* out_dev, void* stream) {
    if (!h || !out_dev) return fail(QX_E_INVALID, "qx_eri_unique: NULL argument");
    DeviceGuard g(h->device);
    return run_all_classes(h, MODE_UNIQUE, out_dev, 0, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- derivatives --
static EriArgs class_args(qx_handle* h, int c, double* out) {
    const ClassWork& w = h->work[c];
    EriArgs a;
    a.quartets = w.d_q;
    a.nq = w.nq;
    a.pairs = h->d_pairs;
    a.prims = h->d_prims;
    a.boys = h->d_boys;
    a.out = out;
    a.n = h->nbf;
    a.base = 0;
    a.scratch = nullptr;
    a.log2g = 0;
    a.err = h->d_err;
    a.out2 = nullptr;
    a.dens = nullptr;
    a.nq64 = w.nq64;
    return a;
}

static long long binom_ll(int n, int k) {
    long long r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

static int rys_unsupported(int c, const char* what) {
    return fail(QX_E_UNSUPPORTED, "class (%d%d|%d%d): the Rys %s program does not fit shared memory or is not compiled",
                g_class_l[c][0], g_class_l[c][1], g_class_l[c][2], g_class_l[c][3], what);
}

// Derivative tensor of order k (1..4) of one class through the Rys engine:
// dense (nu == nullptr; slot = the reference's rank of the sorted nuclear indices
// over M = 3N) or the one slice of the sorted nuclear indices nu[0..k).
static int run_rys_derk(qx_handle* h, int c, int k, double* out, const int* nu, cudaStream_t cs) {
    const ClassWork& w = h->work[c];
    if (!w.nq) return QX_OK;
    RysArgs ra;
    ra.e = class_args(h, c, out);
    ra.rys = h->d_rys;
    ra.M = 3 * h->natom;
    const int nm = (int)binom_ll(11 + k, k);  // multisets of k of the 12 centre-directions
    ra.chunk = std::min(nm, RYS_CHMAX);
    ra.nchunk = (nm + ra.chunk - 1) / ra.chunk;
    if (nu) {
        ra.slice_k = k;
        for (int i = 0; i < k; ++i) ra.slice_nu[i] = nu[i];
    }
    if (g_rys_launch[c](ra, RK_DER1 + k - 1, 0, w.nq * ra.nchunk, cs)) return rys_unsupported(c, "derivative");
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

// Adjoint gradient (kind RK_GRAD) or Hessian-vector product (RK_HVP) of one
// class through the Rys engine.
static int run_rys_contract(qx_handle* h, int c, int kind, const double* D, double cj, double ck, double* grad,
                            const double* dir, cudaStream_t cs) {
    const ClassWork& w = h->work[c];
    if (!w.nq) return QX_OK;
    RysArgs ra;
    ra.e = class_args(h, c, nullptr);
    ra.rys = h->d_rys;
    ra.D = D;
    ra.cj = cj;
    ra.ck = ck;
    ra.grad = grad;
    ra.dir = dir;
    ra.M = 3 * h->natom;
    if (kind == RK_GRAD && h->rys_lp[c]) kind = RK_GRADL;
    if (g_rys_launch[c](ra, kind, 0, w.nq, cs)) return rys_unsupported(c, kind == RK_HVP ? "Hessian" : "gradient");
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

// One class through its first-derivative engine on stream `cs`.
static int run_deriv_class(qx_handle* h, int c, int mode, double* out, const double* D, double cj, double ck,
                           double* grad, int slice, cudaStream_t cs) {
    if (h->deriv_eng[c] == ENG_RYS) {
        if (mode == QX_MODE_GRAD) return run_rys_contract(h, c, RK_GRAD, D, cj, ck, grad, nullptr, cs);
        if (mode == QX_MODE_DER_DENSE) return run_rys_derk(h, c, 1, out, nullptr, cs);
        return run_rys_derk(h, c, 1, out, &slice, cs);
    }
    if (h->deriv_eng[c] == ENG_WARP) {
        WarpArgs wa;
        wa.e = class_args(h, c, out);
        wa.wpq = h->wpq_deriv[c];
        wa.D = D;
        wa.cj = cj;
        wa.ck = ck;
        wa.grad = grad;
        wa.slice = slice;
        g_warp_deriv[c](wa, mode, cs);
    } else {
        // split modes, slice by slice: warp-program VRR into global accumulators
        // (ENG_WVRR) or the cooperative VRR, then the cooperative HRR pass
        if (g_der_idx[c] < 0) return fail(QX_E_UNSUPPORTED, "no derivative program for class %d", c);
        int rc = ensure_split_tasks(h, c, true);
        if (rc) return rc;
        const ClassWork& w = h->work[c];
        const long long nacc = qx_der_nacc(g_der_idx[c]);
        for (size_t sl = 0; sl + 1 < w.slice_q.size(); ++sl) {
            EriArgs a = class_args(h, c, out);
            a.quartets = w.d_q + w.slice_q[sl];
            a.nq = w.slice_q[sl + 1] - w.slice_q[sl];
            a.nq64 = w.nq64 - w.slice_q[sl];
            const int2* tk = w.d_dtasks + w.slice_t[sl];
            const long long nt = w.slice_t[sl + 1] - w.slice_t[sl];
            if (h->deriv_eng[c] == ENG_WVRR) {
                QX_CUDA(cudaMemsetAsync(w.d_dacc, 0, sizeof(double) * a.nq * nacc, cs));
                EriArgs av = a;
                av.prim_stage = h->prim_stage;
            av.wait_limit = h->wait_limit;
                g_wvrr[c](av, tk, nt, qx_der_chunk(), w.d_dacc, (int)nacc, cs);
                qx_launch_der_hrr(g_der_idx[c], a, mode, D, cj, ck, grad, slice, w.d_dacc, cs);
            } else if (h->deriv_eng[c] == ENG_DSPLIT) {
                const long long npad = (nacc + 15) / 16 * 16;  // the warp program's NITEM_PAD
                QX_CUDA(cudaMemsetAsync(w.d_dacc, 0, sizeof(double) * a.nq * npad, cs));
                EriArgs av = a;
                av.prim_stage = h->prim_stage;
            av.wait_limit = h->wait_limit;
                g_dsplit[c](av, tk, nt, qx_der_chunk(), w.d_dacc, (int)npad, cs);
                WarpArgs wa;
                wa.e = a;
                wa.wpq = 1;
                wa.D = D;
                wa.cj = cj;
                wa.ck = ck;
                wa.grad = grad;
                wa.slice = slice;
                wa.acc_in = w.d_dacc;
                g_warp_deriv[c](wa, mode, cs);
            } else {
                qx_launch_der_split(g_der_idx[c], a, mode, D, cj, ck, grad, slice, tk, nt, w.d_dacc, cs);
            }
        }
    }
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

// Every class through the derivative engine on the internal streams, joined
// back into `s`.
static int run_all_deriv(qx_handle* h, int mode, double* out, const double* D, double cj, double ck, double* grad,
                         int slice, cudaStream_t s) {
    QX_CUDA(cudaEventRecord(h->start, s));
    for (int i = 0; i < QX_NSTREAMS; ++i) QX_CUDA(cudaStreamWaitEvent(h->streams[i], h->start, 0));
    int k = 0;
    for (int oi = 0; oi < QX_NCLS_ALL; ++oi) {
        const int c = h->order[oi];
        if (!h->work[c].nq) continue;
        int rc = run_deriv_class(h, c, mode, out, D, cj, ck, grad, slice, h->streams[k++ % QX_NSTREAMS]);
        if (rc) return rc;
    }
    for (int i = 0; i < QX_NSTREAMS; ++i) {
        QX_CUDA(cudaEventRecord(h->done[i], h->streams[i]));
        QX_CUDA(cudaStreamWaitEvent(s, h->done[i], 0));
    }
    return QX_OK;
}

// Second derivatives: every class through its warp order-2 program.  `slice` is
// 3N for the dense tensor, or the packed nuclear pair nu1 | nu2 << 16 (nu1 <= nu2).
static int run_all_deriv2(qx_handle* h, int mode, double* out, int slice, cudaStream_t s, const double* D = nullptr,
                          double cj = 0.0, double ck = 0.0, double* hv = nullptr, const double* dir = nullptr) {
    QX_CUDA(cudaEventRecord(h->start, s));
    for (int i = 0; i < QX_NSTREAMS; ++i) QX_CUDA(cudaStreamWaitEvent(h->streams[i], h->start, 0));
    int k = 0;
    for (int oi = 0; oi < QX_NCLS_ALL; ++oi) {
        const int c = h->order[oi];
        if (!h->work[c].nq) continue;
        cudaStream_t cs = h->streams[k++ % QX_NSTREAMS];
        if (!g_warp_deriv2[c]) {  // classes with d or f shells: the Rys engine
            int rc;
            if (mode == QX_MODE_HVP) {
                rc = run_rys_contract(h, c, RK_HVP, D, cj, ck, hv, dir, cs);
            } else if (mode == QX_MODE_DER2_DENSE) {
                rc = run_rys_derk(h, c, 2, out, nullptr, cs);
            } else {
                const int nu[2] = {slice & 0xffff, slice >> 16};
                rc = run_rys_derk(h, c, 2, out, nu, cs);
            }
            if (rc) return rc;
            continue;
        }
        WarpArgs wa;
        wa.e = class_args(h, c, out);
        wa.wpq = h->wpq_deriv[c];
        wa.D = D;
        wa.cj = cj;
        wa.ck = ck;
        wa.grad = hv;
        wa.slice = slice;
        wa.dir = dir;
        g_warp_deriv2[c](wa, mode, cs);
        QX_CUDA(cudaGetLastError());
    }
    for (int i = 0; i < QX_NSTREAMS; ++i) {
        QX_CUDA(cudaEventRecord(h->done[i], h->streams[i]));
        QX_CUDA(cudaStreamWaitEvent(s, h->done[i], 0));
    }
    return QX_OK;
}

// Derivative tensors of order 3 or 4: every class through the Rys engine on the
// internal streams (dense when nu == nullptr, else the slice nu[0..k)).
static int run_all_derk(qx_handle* h, int k, double* out, const int* nu, cudaStream_t s) {
    QX_CUDA(cudaEventRecord(h->start, s));
    for (int i = 0; i < QX_NSTREAMS; ++i) QX_CUDA(cudaStreamWaitEvent(h->streams[i], h->start, 0));
    int j = 0;
    for (int oi = 0; oi < QX_NCLS_ALL; ++oi) {
        const int c = h->order[oi];
        if (!h->work[c].nq) continue;
        int rc = run_rys_derk(h, c, k, out, nu, h->streams[j++ % QX_NSTREAMS]);
        if (rc) return rc;
    }
    for (int i = 0; i < QX_NSTREAMS; ++i) {
        QX_CUDA(cudaEventRecord(h->done[i], h->streams[i]));
        QX_CUDA(cudaStreamWaitEvent(s, h->done[i], 0));
    }
    return QX_OK;
}

extern "C" int qx_eri_deriv_core(qx_handle* h, int order, double* out, int out_on_device, void* stream) {
    if (!h || !out) return fail(QX_E_INVALID, "qx_eri_deriv_core: NULL argument");
    if (order < 1 || order > 4)
        return fail(QX_E_UNSUPPORTED, "qx_eri_deriv_core: derivative order %d (this library: 1 to 4)", order);
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = h->nbf, n4 = n * n * n * n;
    const long long M = 3LL * h->natom;
    const size_t count = (size_t)binom_ll((int)M + order - 1, order) * (size_t)n4;
    return with_output(h, out, count, out_on_device, s, [&](double* d) {
        QX_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * count, s));
        if (order >= 3) return run_all_derk(h, order, d, nullptr, s);
        if (order == 2) return run_all_deriv2(h, QX_MODE_DER2_DENSE, d, (int)M, s);
        return run_all_deriv(h, QX_MODE_DER_DENSE, d, nullptr, 0.0, 0.0, nullptr, -1, s);
    });
}

extern "C" int qx_compute_2e_deriv(qx_handle* h, const int* deriv_vec, int len, double* out, int out_on_device,
                                   void* stream) {
    if (!h || !out || !deriv_vec) return fail(QX_E_INVALID, "qx_compute_2e_deriv: NULL argument");
    if (len != 3 * h->natom)
        return fail(QX_E_INVALID, "qx_compute_2e_deriv: deriv_vec has %d entries, expected 3*natom = %d", len,
                    3 * h->natom);
    int order = 0, nu[4] = {-1, -1, -1, -1};
    for (int i = 0; i < len; ++i) {
        if (deriv_vec[i] < 0) return fail(QX_E_INVALID, "qx_compute_2e_deriv: negative entry in deriv_vec");
        if (deriv_vec[i] > 4) return fail(QX_E_UNSUPPORTED, "qx_compute_2e_deriv: derivative order above 4");
        for (int r = 0; r < deriv_vec[i] && order + r < 4; ++r) nu[order + r] = i;
        order += deriv_vec[i];
    }
    if (order < 1 || order > 4)
        return fail(QX_E_UNSUPPORTED, "qx_compute_2e_deriv: derivative order %d (this library: 1 to 4)", order);
    if (order == 2 && len > 0xffff) return fail(QX_E_INVALID, "qx_compute_2e_deriv: too many atoms for order 2");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = h->nbf, n4 = n * n * n * n;
    return with_output(h, out, (size_t)n4, out_on_device, s, [&](double* d) {
        QX_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n4, s));
        if (order >= 3) return run_all_derk(h, order, d, nu, s);
        if (order == 2) return run_all_deriv2(h, QX_MODE_DER2_SLICE, d, nu[0] | nu[1] << 16, s);
        return run_all_deriv(h, QX_MODE_DER_SLICE, d, nullptr, 0.0, 0.0, nullptr, nu[0], s);
    });
}

extern "C" int qx_grad_adjoint(qx_handle* h, const double* D, double cj, double ck, double* grad, int on_device,
                               void* stream) {
    if (!h || !D || !grad) return fail(QX_E_INVALID, "qx_grad_adjoint: NULL argument");
    if (!std::isfinite(cj) || !std::isfinite(ck)) return fail(QX_E_INVALID, "qx_grad_adjoint: non-finite coefficient");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = h->nbf;
    const int N3 = 3 * h->natom;
    if (on_device) {
        QX_CUDA(cudaMemsetAsync(grad, 0, sizeof(double) * N3, s));
        return run_all_deriv(h, QX_MODE_GRAD, nullptr, D, cj, ck, grad, -1, s);
    }
    double *dD = nullptr, *dg = nullptr;
    if (cudaMalloc((void**)&dD, sizeof(double) * n * n) != cudaSuccess ||
        cudaMalloc((void**)&dg, sizeof(double) * N3) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(dD);
        return fail(QX_E_NOMEM, "qx_grad_adjoint: staging allocation failed");
    }
    int rc = QX_OK;
    cudaError_t e = cudaMemcpyAsync(dD, D, sizeof(double) * n * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dg, 0, sizeof(double) * N3, s);
    if (e != cudaSuccess) rc = fail(QX_E_CUDA, "qx_grad_adjoint: %s", cudaGetErrorString(e));
    if (!rc) rc = run_all_deriv(h, QX_MODE_GRAD, nullptr, dD, cj, ck, dg, -1, s);
    if (!rc) {
        e = cudaMemcpyAsync(grad, dg, sizeof(double) * N3, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(QX_E_CUDA, "qx_grad_adjoint: %s", cudaGetErrorString(e));
    }
    cudaFree(dD);
    cudaFree(dg);
    if (!rc) rc = check_err_word(h, s);
    return rc;
}

extern "C" int qx_grad_adjoint_jvp(qx_handle* h, const double* D, double cj, double ck, const double* v, double* Hv,
                                   int on_device, void* stream) {
    if (!h || !D || !v || !Hv) return fail(QX_E_INVALID, "qx_grad_adjoint_jvp: NULL argument");
    if (!std::isfinite(cj) || !std::isfinite(ck))
        return fail(QX_E_INVALID, "qx_grad_adjoint_jvp: non-finite coefficient");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = h->nbf;
    const int N3 = 3 * h->natom;
    if (on_device) {
        QX_CUDA(cudaMemsetAsync(Hv, 0, sizeof(double) * N3, s));
        return run_all_deriv2(h, QX_MODE_HVP, nullptr, -1, s, D, cj, ck, Hv, v);
    }
    double *dD = nullptr, *dv = nullptr, *dh = nullptr;
    if (cudaMalloc((void**)&dD, sizeof(double) * n * n) != cudaSuccess ||
        cudaMalloc((void**)&dv, sizeof(double) * N3) != cudaSuccess ||
        cudaMalloc((void**)&dh, sizeof(double) * N3) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(dD);
        cudaFree(dv);
        return fail(QX_E_NOMEM, "qx_grad_adjoint_jvp: staging allocation failed");
    }
    int rc = QX_OK;
    cudaError_t e = cudaMemcpyAsync(dD, D, sizeof(double) * n * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dv, v, sizeof(double) * N3, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dh, 0, sizeof(double) * N3, s);
    if (e != cudaSuccess) rc = fail(QX_E_CUDA, "qx_grad_adjoint_jvp: %s", cudaGetErrorString(e));
    if (!rc) rc = run_all_deriv2(h, QX_MODE_HVP, nullptr, -1, s, dD, cj, ck, dh, dv);
    if (!rc) {
        e = cudaMemcpyAsync(Hv, dh, sizeof(double) * N3, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(QX_E_CUDA, "qx_grad_adjoint_jvp: %s", cudaGetErrorString(e));
    }
    cudaFree(dD);
    cudaFree(dv);
    cudaFree(dh);
    if (!rc) rc = check_err_word(h, s);
    return rc;
}

// ------------------------------------------------------ one-electron integrals --
void qx_launch_oei(const qx::PairInfo* pairs, int npair, const qx::PrimPair* prims, const double* boys,
                   const double* xyz, const double* Z, int natom, long long n, double* S, double* T, double* V,
                   double* dS, double* dT, double* dV, cudaStream_t s);

extern "C" int qx_set_charges(qx_handle* h, const double* Z) {
    if (!h || !Z) return fail(QX_E_INVALID, "qx_set_charges: NULL argument");
    for (int i = 0; i < h->natom; ++i)
        if (!std::isfinite(Z[i])) return fail(QX_E_INVALID, "qx_set_charges: non-finite charge %d", i);
    DeviceGuard g(h->device);
    if (!h->d_Z && (cudaMalloc((void**)&h->d_Z, sizeof(double) * h->natom) != cudaSuccess ||
                    cudaMalloc((void**)&h->d_xyz, sizeof(double) * 3 * h->natom) != cudaSuccess)) {
        cudaGetLastError();
        cudaFree(h->d_Z);
        h->d_Z = nullptr;
        return fail(QX_E_NOMEM, "qx_set_charges: allocation failed");
    }
    QX_CUDA(cudaMemcpy(h->d_Z, Z, sizeof(double) * h->natom, cudaMemcpyHostToDevice));
    QX_CUDA(cudaMemcpy(h->d_xyz, h->coords.data(), sizeof(double) * 3 * h->natom, cudaMemcpyHostToDevice));
    QX_CUDA(cudaDeviceSynchronize());  // the copies complete before any stream reads them
    return QX_OK;
}

extern "C" int qx_oei(qx_handle* h, double* S, double* T, double* V, void* stream) {
    if (!h) return fail(QX_E_INVALID, "qx_oei: NULL handle");
    if (!h->d_Z) return fail(QX_E_INVALID, "qx_oei: nuclear charges not set (qx_set_charges)");
    DeviceGuard g(h->device);
    qx_launch_oei(h->d_pairs, (int)h->pairs.size(), h->d_prims, h->d_boys, h->d_xyz, h->d_Z, h->natom, h->nbf, S, T,
                  V, nullptr, nullptr, nullptr, (cudaStream_t)stream);
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

extern "C" int qx_oei_deriv_core(qx_handle* h, int order, double* dS, double* dT, double* dV, void* stream) {
    if (!h || !dS || !dT || !dV) return fail(QX_E_INVALID, "qx_oei_deriv_core: NULL argument");
    if (order != 1) return fail(QX_E_UNSUPPORTED, "qx_oei_deriv_core: derivative order %d (this library: 1)", order);
    if (!h->d_Z) return fail(QX_E_INVALID, "qx_oei_deriv_core: nuclear charges not set (qx_set_charges)");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = sizeof(double) * 3 * h->natom * (size_t)h->nbf * h->nbf;
    QX_CUDA(cudaMemsetAsync(dS, 0, bytes, s));
    QX_CUDA(cudaMemsetAsync(dT, 0, bytes, s));
    QX_CUDA(cudaMemsetAsync(dV, 0, bytes, s));
    qx_launch_oei(h->d_pairs, (int)h->pairs.size(), h->d_prims, h->d_boys, h->d_xyz, h->d_Z, h->natom, h->nbf,
                  nullptr, nullptr, nullptr, dS, dT, dV, s);
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

// ---------------------------------------------------------------- class info ---
// Algorithmic FP64 FLOPs of one primitive quartet of the Rys programs (plain:
// deriv = 0; adjoint gradient: deriv = 1), counted per step of qx_rys.cuh: the
// 2n Chebyshev series (13 Clenshaw steps, 4 flops each), the 3n two-dimensional
// tables (5 flops per entry), the transfer levels (2 per entry), the gradient's
// four derivative tables (3 per entry) and the products (plain: 3 per component
// and root; gradient: 22).
static double rys_prim_flops(const int* l, int deriv) {
    const int L = l[0] + l[1] + l[2] + l[3];
    const int A1 = l[0] + 1 + deriv, B1 = l[1] + 1 + deriv, C1 = l[2] + 1 + deriv, D1 = l[3] + 1;
    const int NI = A1 + B1 - 1, NK = C1 + D1 - 1, NR = (L + deriv) / 2 + 1;
    double ncomp = 1.0, sz0 = 1.0;
    for (int i = 0; i < 4; ++i) {
        ncomp *= (l[i] + 1) * (l[i] + 2) / 2;
        sz0 *= l[i] + 1;
    }
    double f = 2.0 * NR * 52.0 + 3.0 * NR * NI * NK * 5.0;
    for (int b = 1; b < B1; ++b) f += 3.0 * NR * (NI - b) * NK * 2.0;
    for (int d = 1; d < D1; ++d) f += 3.0 * NR * A1 * B1 * (NK - d) * 2.0;
    if (deriv) f += 3.0 * NR * 4.0 * sz0 * 3.0 + ncomp * NR * 22.0;
    else f += ncomp * NR * 3.0;
    return f;
}

extern "C" int qx_num_classes(void) { return QX_NCLS_ALL; }

extern "C" int qx_class_info(const qx_handle* h, int cls, int* l4, long long* nquartets, long long* nprim_quartets,
                             double* flops, double* flops_deriv) {
    if (!h || cls < 0 || cls >= QX_NCLS_ALL) return fail(QX_E_INVALID, "qx_class_info: bad handle or class");
    const ClassWork& w = h->work[cls];
    if (l4)
        for (int i = 0; i < 4; ++i) l4[i] = g_class_l[cls][i];
    if (nquartets) *nquartets = w.nq;
    if (nprim_quartets) *nprim_quartets = w.prims;
    if (!has_os(cls)) {
        if (flops) *flops = (double)w.prims * rys_prim_flops(g_class_l[cls], 0);
        if (flops_deriv) *flops_deriv = (double)w.prims * rys_prim_flops(g_class_l[cls], 1);
        return QX_OK;
    }
    if (flops) *flops = (double)w.prims * g_class_vrr_flops[cls] + (double)w.nq * g_class_hrr_flops[cls];
    if (flops_deriv) *flops_deriv = (double)w.prims * g_class_dvrr_flops[cls] + (double)w.nq * g_class_dhrr_flops[cls];
    return QX_OK;
}

extern "C" int qx_eri_unique_class(qx_handle* h, int cls, double* out_dev, void* stream) {
    if (!h || !out_dev || cls < 0 || cls >= QX_NCLS_ALL) return fail(QX_E_INVALID, "qx_eri_unique_class: bad argument");
    DeviceGuard g(h->device);
    const ClassWork& w = h->work[cls];
    if (!w.nq) return QX_OK;
    return run_class(h, cls, MODE_UNIQUE, w.d_q, w.nq, out_dev, 0, w.unique_base, (cudaStream_t)stream, w.log2g,
                     w.scratch);
}

extern "C" int qx_grad_adjoint_class(qx_handle* h, int cls, const double* D_dev, double cj, double ck,
                                     double* grad_dev, void* stream) {
    if (!h || !D_dev || !grad_dev || cls < 0 || cls >= QX_NCLS_ALL)
        return fail(QX_E_INVALID, "qx_grad_adjoint_class: bad argument");
    DeviceGuard g(h->device);
    if (!h->work[cls].nq) return QX_OK;
    return run_deriv_class(h, cls, QX_MODE_GRAD, nullptr, D_dev, cj, ck, grad_dev, -1, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- autotuner ----
// Times every engine configuration a class can run (straight-line with 1..32
// lanes per quartet, warp kernels with 1 or 4 warps per quartet, the warp-VRR +
// cooperative-HRR pair, the cooperative engines) on this handle's own quartet
// lists and keeps the fastest.  Plain configurations are timed in unique-ERI
// mode, derivative ones in adjoint-gradient mode.  All engines compute the same
// sums, in different orders, so the choice changes results only by rounding.
namespace {
struct TuneCfg {
    int eng, param;  // param: log2g (straight-line) or warps per quartet (warp)
};
}  // namespace

static int time_config(cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, float* best_ms,
                       const std::function<int()>& launch) {
    int rc = launch();  // warm-up (lazy allocations, kernel attributes)
    if (rc) return rc;
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        QX_CUDA(cudaEventRecord(e0, s));
        rc = launch();
        if (rc) return rc;
        QX_CUDA(cudaEventRecord(e1, s));
        QX_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        QX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    *best_ms = best;
    return QX_OK;
}

extern "C" int qx_autotune(qx_handle* h, int what, void* stream) {
    if (!h || (what & ~3) || !what) return fail(QX_E_INVALID, "qx_autotune: bad argument");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    long long max_out = 0;
    for (int c = 0; c < QX_NCLS_ALL; ++c) max_out = std::max(max_out, h->work[c].nq * (long long)g_class_nout[c]);
    const long long n = h->nbf;
    double *d_out = nullptr, *d_D = nullptr, *d_g = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = QX_OK;
    if (cudaMalloc((void**)&d_out, sizeof(double) * std::max(1LL, max_out)) != cudaSuccess ||
        cudaMalloc((void**)&d_D, sizeof(double) * n * n) != cudaSuccess ||
        cudaMalloc((void**)&d_g, sizeof(double) * 3 * h->natom) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(QX_E_NOMEM, "qx_autotune: scratch allocation failed");
    }
    if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = fail(QX_E_CUDA, "qx_autotune: event creation failed");
    // a positive density (every byte 0x3f: 4.8e-4 in each entry)
    if (!rc && cudaMemsetAsync(d_D, 0x3f, sizeof(double) * n * n, s) != cudaSuccess)
        rc = fail(QX_E_CUDA, "qx_autotune: memset failed");
    if (!rc && cudaMemsetAsync(d_g, 0, sizeof(double) * 3 * h->natom, s) != cudaSuccess)
        rc = fail(QX_E_CUDA, "qx_autotune: memset failed");
    for (int c = 0; c < QX_NCLS_ALL && !rc; ++c) {
        ClassWork& w = h->work[c];
        if (!w.nq) continue;
        if ((what & 1) && has_os(c)) {  // the f classes have one plain engine
            std::vector<TuneCfg> cand;
            if (!g_class_coop[c] && !g_class_scratch[c])
                for (int lg = 0; lg <= 5; ++lg) cand.push_back({ENG_SL, lg});
            if (g_has_warp_plain[c]) {
                cand.push_back({ENG_WARP, 1});
                cand.push_back({ENG_WARP, 4});
            }
            if (g_class_coop[c]) cand.push_back({ENG_COOP, 0});
            if (g_has_pvrr[c] && g_has_warp_plain[c] && !ensure_split_tasks(h, c) && w.slice_q.size() == 2)
                cand.push_back({ENG_WSPLIT, 1});
            cand.push_back({ENG_RYS, 0});
            const int keep_wpq = h->wpq[c], keep_lg = w.log2g;
            float best = 1e30f;
            TuneCfg bc{h->plain_eng[c], h->plain_eng[c] == ENG_SL ? keep_lg : keep_wpq};
            for (const TuneCfg& t : cand) {
                h->plain_eng[c] = t.eng;
                if (t.eng == ENG_WARP || t.eng == ENG_WSPLIT) h->wpq[c] = t.param;
                const int lg = t.eng == ENG_SL ? t.param : 0;
                float ms = 0.f;
                rc = time_config(s, e0, e1, &ms, [&] {
                    return run_class(h, c, MODE_UNIQUE, w.d_q, w.nq, d_out, 0, 0, s, lg, w.scratch);
                });
                if (rc) break;
                if (ms < best) {
                    best = ms;
                    bc = t;
                }
            }
            h->plain_eng[c] = bc.eng;
            h->wpq[c] = (bc.eng == ENG_WARP || bc.eng == ENG_WSPLIT) ? bc.param : keep_wpq;
            w.log2g = bc.eng == ENG_SL ? bc.param : keep_lg;
        }
        if ((what & 2) && !rc) {
            std::vector<TuneCfg> cand;
            if (g_has_warp_deriv[c]) {
                cand.push_back({ENG_WARP, 1});
                cand.push_back({ENG_WARP, 4});
            }
            if (g_has_wvrr[c]) cand.push_back({ENG_WVRR, 0});
            if (g_has_dsplit[c]) cand.push_back({ENG_DSPLIT, 0});
            if (g_der_idx[c] >= 0) cand.push_back({ENG_COOP, 0});
            cand.push_back({ENG_RYS, 0});  // Rys, per-unit table build for small units
            cand.push_back({ENG_RYS, 1});  // Rys, level-parallel table build
            float best = 1e30f;
            TuneCfg bc{h->deriv_eng[c], h->deriv_eng[c] == ENG_RYS ? h->rys_lp[c] : h->wpq_deriv[c]};
            for (const TuneCfg& t : cand) {
                h->deriv_eng[c] = t.eng;
                if (t.eng == ENG_WARP) h->wpq_deriv[c] = t.param;
                if (t.eng == ENG_RYS) h->rys_lp[c] = t.param;
                float ms = 0.f;
                rc = time_config(s, e0, e1, &ms, [&] {
                    return run_deriv_class(h, c, QX_MODE_GRAD, nullptr, d_D, 1.0, -0.5, d_g, -1, s);
                });
                if (rc) break;
                if (ms < best) {
                    best = ms;
                    bc = t;
                }
            }
            h->deriv_eng[c] = bc.eng;
            if (bc.eng == ENG_WARP) h->wpq_deriv[c] = bc.param;
            h->rys_lp[c] = bc.eng == ENG_RYS ? bc.param : 0;
        }
    }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(QX_E_CUDA, "qx_autotune: %s", cudaGetErrorString(e));
    }
    if (!rc) rc = check_err_word(h, s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_out);
    cudaFree(d_D);
    cudaFree(d_g);
    return rc;
}

// Engine of one class chosen by the caller (tests, measurements): the autotuner's
// choice made by hand.  plain / deriv: engine ids as qx_engine_config reports
// them, -1 keeps the current one; pparam / dparam: log2 lanes per quartet
// (straight-line) or warps per quartet (warp kernels); for the Rys derivative
// engine dparam 0 or 1 picks the adjoint gradient's table build (per-unit for
// small units, or level-parallel); ignored otherwise.
extern "C" int qx_set_engine(qx_handle* h, int cls, int plain, int pparam, int deriv, int dparam) {
    if (!h || cls < 0 || cls >= QX_NCLS_ALL) return fail(QX_E_INVALID, "qx_set_engine: bad handle or class");
    DeviceGuard g(h->device);
    ClassWork& w = h->work[cls];
    const int* L = g_class_l[cls];
    auto no = [&](const char* what, int e) {
        return fail(QX_E_UNSUPPORTED, "qx_set_engine: class (%d%d|%d%d) has no %s engine %d", L[0], L[1], L[2], L[3],
                    what, e);
    };
    if (plain >= 0) {
        bool ok = false;
        if (plain == ENG_SL) ok = has_os(cls) && !g_class_coop[cls] && pparam >= 0 && pparam <= 5;
        if (plain == ENG_WARP) ok = has_os(cls) && g_has_warp_plain[cls] && (pparam == 1 || pparam == 4);
        if (plain == ENG_COOP) ok = has_os(cls) && g_class_coop[cls];
        if (plain == ENG_WSPLIT) ok = has_os(cls) && g_has_pvrr[cls] && g_has_warp_plain[cls];
        if (plain == ENG_RYS) ok = true;
        if (!ok) return no("plain", plain);
        QX_CUDA(cudaDeviceSynchronize());
        if (plain == ENG_SL && g_class_scratch[cls] && w.nq) {  // global accumulators for this lane count
            cudaFree(w.scratch);
            w.scratch = nullptr;
            if (cudaMalloc((void**)&w.scratch, sizeof(double) * g_class_scratch[cls] * launch_threads(w.nq, pparam)) !=
                cudaSuccess) {
                cudaGetLastError();
                w.scratch = nullptr;
                return fail(QX_E_NOMEM, "qx_set_engine: accumulators for class %d", cls);
            }
        }
        if (plain == ENG_WSPLIT) {
            int rc = ensure_split_tasks(h, cls);
            if (rc) return rc;
        }
        h->plain_eng[cls] = plain;
        if (plain == ENG_SL) w.log2g = pparam;
        if (plain == ENG_WARP) h->wpq[cls] = pparam;
        if (plain == ENG_WSPLIT) h->wpq[cls] = 1;
    }
    if (deriv >= 0) {
        bool ok = false;
        if (deriv == ENG_WARP) ok = has_os(cls) && g_has_warp_deriv[cls] && (dparam == 1 || dparam == 4);
        if (deriv == ENG_WVRR) ok = has_os(cls) && g_has_wvrr[cls];
        if (deriv == ENG_DSPLIT) ok = has_os(cls) && g_has_dsplit[cls];
        if (deriv == ENG_COOP) ok = g_der_idx[cls] >= 0;
        if (deriv == ENG_RYS) ok = dparam == 0 || dparam == 1;
        if (!ok) return no("derivative", deriv);
        h->deriv_eng[cls] = deriv;
        if (deriv == ENG_WARP) h->wpq_deriv[cls] = dparam;
        if (deriv == ENG_RYS) h->rys_lp[cls] = dparam;
    }
    return QX_OK;
}

// Frees the first-derivative split-mode accumulators the handle keeps between
// calls (the next derivative call of the class allocates them again), for
// callers that hold many handles on one device.
extern "C" int qx_release_scratch(qx_handle* h) {
    if (!h) return fail(QX_E_INVALID, "qx_release_scratch: bad handle");
    DeviceGuard g(h->device);
    QX_CUDA(cudaDeviceSynchronize());  // no kernel of the handle still uses them
    for (int c = 0; c < QX_NCLS_ALL; ++c) {
        cudaFree(h->work[c].d_dacc);
        h->work[c].d_dacc = nullptr;
    }
    return QX_OK;
}

// Polls of the bounded waits on the split-mode staging copies (default 4M); a
// wait that runs out sets the error word, which host-synchronising calls report
// as QX_E_DEVICE.  A limit of 0 makes every such wait run out (failure-path tests).
extern "C" int qx_set_wait_limit(qx_handle* h, int polls) {
    if (!h || polls < 0) return fail(QX_E_INVALID, "qx_set_wait_limit: bad argument");
    h->wait_limit = polls;
    return QX_OK;
}

// The canonical shells of a class's quartets in this handle's list order (the
// order of the unique layout): shells[4 * qi + 0..3] = (s1 s2|s3 s4).
extern "C" int qx_class_quartets(const qx_handle* h, int cls, int* shells) {
    if (!h || !shells || cls < 0 || cls >= QX_NCLS_ALL) return fail(QX_E_INVALID, "qx_class_quartets: bad argument");
    DeviceGuard g(h->device);
    const ClassWork& w = h->work[cls];
    if (!w.nq) return QX_OK;
    std::vector<int2> L((size_t)w.nq);
    QX_CUDA(cudaMemcpy(L.data(), w.d_q, sizeof(int2) * w.nq, cudaMemcpyDeviceToHost));
    for (long long i = 0; i < w.nq; ++i) {
        const PairInfo& P = h->pairs[L[i].x];
        const PairInfo& Q = h->pairs[L[i].y];
        shells[4 * i + 0] = P.s1;
        shells[4 * i + 1] = P.s2;
        shells[4 * i + 2] = Q.s1;
        shells[4 * i + 3] = Q.s2;
    }
    return QX_OK;
}

extern "C" int qx_engine_config(const qx_handle* h, int cls, int* cfg) {
    if (!h || !cfg || cls < 0 || cls >= QX_NCLS_ALL) return fail(QX_E_INVALID, "qx_engine_config: bad argument");
    cfg[0] = h->plain_eng[cls];
    cfg[1] = h->plain_eng[cls] == ENG_SL ? h->work[cls].log2g : (h->plain_eng[cls] == ENG_WARP ? h->wpq[cls] : 0);
    cfg[2] = h->deriv_eng[cls];
    cfg[3] = h->deriv_eng[cls] == ENG_WARP ? h->wpq_deriv[cls] : (h->deriv_eng[cls] == ENG_RYS ? h->rys_lp[cls] : 0);
    return QX_OK;
}

// ------------------------------------------------- derivative tiles (plain path) --
// Gamma of a tile of one class's unique quartets, in the layout of the derivative
// tiles: per element (quartet-local qi, component o) the sum of Gamma over the
// integral's distinct images (images = 0), or Gamma of each image in its slot of 8
// (images = 1; absent images 0).  Gamma_ijkl = cj D_ij D_kl + ck D_ik D_jl.
__global__ void __launch_bounds__(128) k_gamma_tile(const int2* __restrict__ quartets, long long nq,
                                                    const PairInfo* __restrict__ pairs, int nb, int nc, int nd,
                                                    int nout, const double* __restrict__ D, long long n, double cj,
                                                    double ck, int images, double* __restrict__ gam) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq * nout) return;
    const long long qi = t / nout;
    const int o = (int)(t - qi * nout);
    const int2 pq = quartets[qi];
    const PairInfo P = pairs[pq.x], Q = pairs[pq.y];
    const int id = o % nd, ic = (o / nd) % nc, ib = (o / (nd * nc)) % nb, ia = o / (nd * nc * nb);
    const long long i = P.bf1 + ia, j = P.bf2 + ib, k = Q.bf1 + ic, l = Q.bf2 + id;
    const bool s12 = P.s1 != P.s2, s34 = Q.s1 != Q.s2, sPQ = pq.x != pq.y;
    auto G = [&](long long p, long long q, long long r, long long s) {
        return cj * __ldg(D + p * n + q) * __ldg(D + r * n + s) + ck * __ldg(D + p * n + r) * __ldg(D + q * n + s);
    };
    const double g[8] = {G(i, j, k, l), s12 ? G(j, i, k, l) : 0.0, s34 ? G(i, j, l, k) : 0.0,
                         (s12 && s34) ? G(j, i, l, k) : 0.0, sPQ ? G(k, l, i, j) : 0.0,
                         (sPQ && s34) ? G(l, k, i, j) : 0.0, (sPQ && s12) ? G(k, l, j, i) : 0.0,
                         (sPQ && s12 && s34) ? G(l, k, j, i) : 0.0};
    if (images) {
        for (int m = 0; m < 8; ++m) gam[t * 8 + m] = g[m];
    } else {
        double s = 0.0;
        for (int m = 0; m < 8; ++m) s += g[m];
        gam[t] = s;
    }
}

static int tile_check(qx_handle* h, int cls, long long q0, long long q1) {
    if (!h || cls < 0 || cls >= QX_NCLS_ALL) return fail(QX_E_INVALID, "derivative tile: bad handle or class");
    const ClassWork& w = h->work[cls];
    if (q0 < 0 || q1 < q0 || q1 > w.nq) return fail(QX_E_INVALID, "derivative tile: quartet range %lld..%lld of %lld", q0, q1, w.nq);
    return QX_OK;
}

extern "C" int qx_deriv_tile(qx_handle* h, int cls, long long q0, long long q1, int images, double* B, long long E,
                             void* stream) {
    int rc = tile_check(h, cls, q0, q1);
    if (rc) return rc;
    if (!B) return fail(QX_E_INVALID, "qx_deriv_tile: NULL buffer");
    const long long need = (q1 - q0) * g_class_nout[cls] * (images ? 8 : 1);
    if (E < need) return fail(QX_E_INVALID, "qx_deriv_tile: row length %lld < %lld elements", E, need);
    if (q1 == q0) return QX_OK;
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const ClassWork& w = h->work[cls];
    EriArgs a = class_args(h, cls, B);
    a.quartets = w.d_q + q0;
    a.nq = q1 - q0;
    a.nq64 = w.nq64 >= q1 ? a.nq : std::max(0LL, w.nq64 - q0);
    if (h->deriv_eng[cls] == ENG_WARP) {
        WarpArgs wa;
        wa.e = a;
        wa.wpq = h->wpq_deriv[cls];
        wa.D = nullptr;
        wa.cj = wa.ck = 0.0;
        wa.grad = nullptr;
        wa.slice = -1;
        wa.tile_E = E;
        wa.tile_images = images;
        g_warp_deriv[cls](wa, WMODE_DER_TILE, s);
    } else {  // the Rys engine serves every class (the split-mode engines have no tile epilogue)
        RysArgs ra;
        ra.e = a;
        ra.rys = h->d_rys;
        ra.M = 3 * h->natom;
        ra.tile_E = E;
        ra.tile_images = images;
        if (g_rys_launch[cls](ra, RK_GRADT, 0, a.nq, s)) return rys_unsupported(cls, "derivative-tile");
    }
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

extern "C" int qx_gamma_tile(qx_handle* h, int cls, long long q0, long long q1, int images, const double* D,
                             double cj, double ck, double* gam, void* stream) {
    int rc = tile_check(h, cls, q0, q1);
    if (rc) return rc;
    if (!D || !gam) return fail(QX_E_INVALID, "qx_gamma_tile: NULL argument");
    if (q1 == q0) return QX_OK;
    DeviceGuard g(h->device);
    const ClassWork& w = h->work[cls];
    const int* L = g_class_l[cls];
    const int nb = (L[1] + 1) * (L[1] + 2) / 2, nc = (L[2] + 1) * (L[2] + 2) / 2, nd = (L[3] + 1) * (L[3] + 2) / 2;
    const long long tot = (q1 - q0) * g_class_nout[cls];
    k_gamma_tile<<<(unsigned)((tot + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        w.d_q + q0, q1 - q0, h->d_pairs, nb, nc, nd, g_class_nout[cls], D, h->nbf, cj, ck, images, gam);
    QX_CUDA(cudaGetLastError());
    return QX_OK;
}

// ---------------------------------------------------------------- direct J/K ---
// max |D| over each pair record's block (one warp per pair record)
__global__ void __launch_bounds__(128) k_pair_dmax(const PairInfo* __restrict__ pairs, int npair,
                                                   const double* __restrict__ D, long long n, double* __restrict__ out) {
    const int p = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (p >= npair) return;
    const PairInfo P = pairs[p];
    const int na = (P.l1 + 1) * (P.l1 + 2) / 2, nb = (P.l2 + 1) * (P.l2 + 2) / 2;
    double m = 0.0;
    for (int e = lane; e < na * nb; e += 32) {
        const long long i = P.bf1 + e / nb, j = P.bf2 + e % nb;
        m = fmax(m, fmax(fabs(D[i * n + j]), fabs(D[j * n + i])));
    }
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0) out[p] = m;
}

extern "C" int qx_jk_screened(qx_handle* h, const double* D, double* J, double* K, double thr, void* stream) {
    if (!h || !D || !J || !K) return fail(QX_E_INVALID, "qx_jk_screened: NULL argument");
    if (!(thr >= 0.0) || !std::isfinite(thr)) return fail(QX_E_INVALID, "qx_jk_screened: bad threshold");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const int np = (int)h->pairs.size();
    if (!h->d_kpair) {  // first call: per-pair sqrt(K) (host data) and the max |D| buffer
        std::vector<double> kp(np);
        for (int p = 0; p < np; ++p)
            kp[p] = std::sqrt(h->K[(size_t)h->pairs[p].s1 * h->nshell + h->pairs[p].s2]);
        if (cudaMalloc((void**)&h->d_kpair, sizeof(double) * np) != cudaSuccess ||
            cudaMalloc((void**)&h->d_dmax, sizeof(double) * np) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(h->d_kpair);
            h->d_kpair = nullptr;
            return fail(QX_E_NOMEM, "qx_jk_screened: allocation failed");
        }
        QX_CUDA(cudaMemcpy(h->d_kpair, kp.data(), sizeof(double) * np, cudaMemcpyHostToDevice));
        QX_CUDA(cudaDeviceSynchronize());  // the copy completes before any stream reads it
    }
    const long long n = h->nbf;
    QX_CUDA(cudaMemsetAsync(J, 0, sizeof(double) * n * n, s));
    QX_CUDA(cudaMemsetAsync(K, 0, sizeof(double) * n * n, s));
    k_pair_dmax<<<(np + 3) / 4, 128, 0, s>>>(h->d_pairs, np, D, n, h->d_dmax);
    QX_CUDA(cudaGetLastError());
    h->jk_thr = thr;
    int rc = run_all_classes(h, MODE_JK, J, n, s, K, D);
    h->jk_thr = 0.0;
    return rc;
}

extern "C" int qx_jk(qx_handle* h, const double* D, double* J, double* K, int on_device, void* stream) {
    if (!h || !D || !J || !K) return fail(QX_E_INVALID, "qx_jk: NULL argument");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = h->nbf;
    const size_t bytes = sizeof(double) * n * n;
    if (on_device) {
        QX_CUDA(cudaMemsetAsync(J, 0, bytes, s));
        QX_CUDA(cudaMemsetAsync(K, 0, bytes, s));
        return run_all_classes(h, MODE_JK, J, n, s, K, D);
    }
    double* d = nullptr;
    if (cudaMalloc((void**)&d, 3 * bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(QX_E_NOMEM, "qx_jk: staging allocation failed");
    }
    int rc = QX_OK;
    cudaError_t e = cudaMemcpyAsync(d, D, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d + n * n, 0, 2 * bytes, s);
    if (e != cudaSuccess) rc = fail(QX_E_CUDA, "qx_jk: %s", cudaGetErrorString(e));
    if (!rc) rc = run_all_classes(h, MODE_JK, d + n * n, n, s, d + 2 * n * n, d);
    if (!rc) {
        e = cudaMemcpyAsync(J, d + n * n, bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(K, d + 2 * n * n, bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(QX_E_CUDA, "qx_jk: %s", cudaGetErrorString(e));
    }
    cudaFree(d);
    if (!rc) rc = check_err_word(h, s);
    return rc;
}
