// qx_noalloc.cu -- dense ERI tensor without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: an XLA/JAX custom call runs
// inside a runtime that owns (and usually pre-reserves) the device memory, so an
// allocation from inside the handler can fail or fragment that pool; real-time or
// embedded hosts forbid allocation after start-up; and code running under a
// caller-managed memory pool wants every byte accounted for by the caller.  For
// them, qx_compute_2e_int_noalloc computes the same dense ERI tensor as
// qx_initialize + qx_compute_2e_int + qx_finalize, but the only device memory it
// touches besides the caller's output is the fixed array below: the Boys table,
// the primitive-pair and shell-pair records, the Schwarz values and the screened
// quartet lists are all placed there.  It calls no cudaMalloc/cudaFree, creates no
// streams or events, and launches everything on the caller's stream.
//
// Limits and sharing rules (also stated in include/quax_b200.h):
//   * the array holds QX_NOALLOC_SCRATCH_BYTES (16 MiB) per device, kept from the
//     library's load until process exit on every device that uses it;
//   * a basis whose tables do not fit is rejected with QX_E_INVALID before any
//     device work (roughly: up to ~1.5 million screened unique quartets);
//   * every call reuses the same array and it keeps the last call's contents;
//     calls that overlap on the GPU (other streams, other host threads) race on
//     it and must be serialised by the caller;
//   * every call blocks the host: it reads the Schwarz values back to build the
//     screened lists and returns once the tensor is complete, so no call can be
//     recorded into a CUDA graph; a call on a stream that is capturing is refused
//     with QX_E_INVALID (an XLA handler must be registered as not capturable);
//   * the first call on a device looks up the array's device address and uploads
//     the Boys table, synchronously.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "quax_b200.h"
#include "qx_kernels.cuh"
#include "qx_setup.h"

using namespace qx;

// QX_NOALLOC_SCRATCH_BYTES (16 MiB) is defined in quax_b200.h.
void qx_set_last_error(const char* msg);  // defined with the other error state

// The scratch itself.  In host code this name is only a stand-in for the symbol:
// host code must use the address returned by cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[QX_NOALLOC_SCRATCH_BYTES];

namespace {

int nofail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    qx_set_last_error(buf);  // reported by qx_last_error()
    return code;
}

constexpr int quartet_cls(int pb, int pk) { return pb * (pb + 1) / 2 + pk; }
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kBoysBytes = sizeof(double) * BOYS_NG * BOYS_NM;

const int k_class_coop[QX_NUM_CLASSES] = QX_CLASS_COOP;
// classes whose straight-line kernel keeps its accumulators in global memory
// (none with the current class split; such a class would be refused here)
const std::vector<long long> k_class_scratch = [] {
    std::vector<long long> v(QX_NUM_CLASSES, 0);
#define QX_NA_SCR(id, a, b, c, d) v[id] = qx::scratch_per_quartet<a, b, c, d>();
    QX_FOR_EACH_SL_CLASS(QX_NA_SCR)
#undef QX_NA_SCR
    return v;
}();

struct DeviceState {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_noalloc_scratch
};
std::mutex g_mtx;
DeviceState g_state[256];

// One-time set-up per device, with that device current.
int setup_device(int dev) {
    std::lock_guard<std::mutex> lk(g_mtx);
    if (dev < 0 || dev >= 256) return nofail(QX_E_INVALID, "qx_compute_2e_int_noalloc: device %d out of range", dev);
    DeviceState& st = g_state[dev];
    if (st.ready) return QX_OK;
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
        return nofail(QX_E_CUDA, "qx_compute_2e_int_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    const auto& tab = boys_table();
    e = cudaMemcpy(ptr, tab.data(), kBoysBytes, cudaMemcpyHostToDevice);
    // a pageable host-to-device copy can still be in flight when cudaMemcpy returns;
    // the caller's stream may not order after it, so wait here (set-up only)
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
        return nofail(QX_E_CUDA, "qx_compute_2e_int_noalloc: Boys table upload failed: %s", cudaGetErrorString(e));
    st.base = (unsigned char*)ptr;
    st.ready = true;
    return QX_OK;
}

int choose_lg(long long nq, long long prims) {
    int lg = 0;
    const double avg = nq ? (double)prims / nq : 0.0;
    while (lg < 5 && (nq << lg) < 150000 && avg / (1 << (lg + 1)) >= 8.0) ++lg;
    return lg;
}

void launch_class(int cls, const EriArgs& a, int mode, cudaStream_t s) {
    if (k_class_coop[cls]) {
        qx_launch_coop(qx_coop_index(cls), a, mode, s);
        return;
    }
    switch (cls) {
#define QX_NA_CASE(id, a_, b_, c_, d_) \
    case id: qx_launch_eri_##id(a, mode, s); break;
        QX_FOR_EACH_SL_CLASS(QX_NA_CASE)
        default: break;
    }
}

}  // namespace

extern "C" int qx_compute_2e_int_noalloc(int natom, const double* coords, int nshell, const int* shell_l,
                                         const int* shell_nprim, const int* shell_atom, const double* exps,
                                         const double* coefs, double ints_tol, double* out_dev, void* stream) {
    if (natom <= 0 || nshell <= 0 || !coords || !shell_l || !shell_nprim || !shell_atom || !exps || !coefs || !out_dev)
        return nofail(QX_E_INVALID, "qx_compute_2e_int_noalloc: empty geometry, shell list or output");
    if (!(ints_tol > 0.0) || !std::isfinite(ints_tol))
        return nofail(QX_E_INVALID, "qx_compute_2e_int_noalloc: ints_tol must be > 0");
    for (int i = 0; i < 3 * natom; ++i)
        if (!std::isfinite(coords[i])) return nofail(QX_E_INVALID, "qx_compute_2e_int_noalloc: non-finite coordinate");
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing((cudaStream_t)stream, &cs) != cudaSuccess) {
            cudaGetLastError();
            return nofail(QX_E_INVALID, "qx_compute_2e_int_noalloc: cannot query the stream's capture state");
        }
        if (cs != cudaStreamCaptureStatusNone)
            return nofail(QX_E_INVALID,
                          "qx_compute_2e_int_noalloc: the stream is capturing; this call synchronises and cannot be "
                          "recorded into a CUDA graph");
    }
    // --- host tables (shared with qx_initialize) ---
    ShellTables shells;
    {
        std::string err;
        const int rc = normalize_shells("qx_compute_2e_int_noalloc", natom, nshell, shell_l, shell_nprim, shell_atom,
                                        exps, coefs, QX_GEN_LMAX, shells, err);
        if (rc) return nofail(rc, "%s", err.c_str());
    }
    const int nbf = shells.nbf;
    std::vector<PrimPair> prims;
    std::vector<PairInfo> pairs;
    std::vector<int> pcls;
    build_pairs(shells, coords, prims, pairs, pcls);
    const int np = (int)pairs.size();
    // --- scratch layout part 1: Boys | prims | pairs | K per pair | diagonal lists ---
    const size_t o_prims = align256(kBoysBytes);
    const size_t o_pairs = align256(o_prims + sizeof(PrimPair) * prims.size());
    const size_t o_kp = align256(o_pairs + sizeof(PairInfo) * np);
    const size_t o_diag = align256(o_kp + sizeof(double) * np);
    const size_t o_lists = align256(o_diag + sizeof(int2) * np);
    if (o_lists > QX_NOALLOC_SCRATCH_BYTES)
        return nofail(QX_E_INVALID,
                      "qx_compute_2e_int_noalloc: basis needs more than the %u-byte scratch (%zu bytes of pair tables)",
                      QX_NOALLOC_SCRATCH_BYTES, o_lists);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return nofail(QX_E_CUDA, "qx_compute_2e_int_noalloc: %s", cudaGetErrorString(e));
    int rc = setup_device(dev);
    if (rc) return rc;
    unsigned char* base = g_state[dev].base;
    cudaStream_t s = (cudaStream_t)stream;
#define NA_CUDA(call)                                                                                          \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) return nofail(QX_E_CUDA, "qx_compute_2e_int_noalloc: %s: %s", #call,            \
                                             cudaGetErrorString(e_));                                          \
    } while (0)
    PrimPair* d_prims = (PrimPair*)(base + o_prims);
    PairInfo* d_pairs = (PairInfo*)(base + o_pairs);
    double* d_kp = (double*)(base + o_kp);
    int2* d_diag = (int2*)(base + o_diag);
    const double* d_boys = (const double*)base;
    NA_CUDA(cudaMemcpyAsync(d_prims, prims.data(), sizeof(PrimPair) * prims.size(), cudaMemcpyHostToDevice, s));
    NA_CUDA(cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(PairInfo) * np, cudaMemcpyHostToDevice, s));
    // Schwarz: diagonal quartets (P|P) of every pair, grouped by pair class
    std::vector<int2> diag;
    std::vector<std::pair<int, int>> diag_rng;  // (start, count) per pair class
    for (int pc = 0; pc < QX_NUM_PAIR_CLASSES; ++pc) {
        const int st = (int)diag.size();
        for (int p = 0; p < np; ++p)
            if (pcls[p] == pc) diag.push_back(make_int2(p, p));
        diag_rng.push_back({st, (int)diag.size() - st});
    }
    NA_CUDA(cudaMemcpyAsync(d_diag, diag.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, s));
    auto args = [&](const int2* q, long long nq, double* out, long long n, int lg) {
        EriArgs a;
        a.quartets = q;
        a.nq = nq;
        a.pairs = d_pairs;
        a.prims = d_prims;
        a.boys = d_boys;
        a.out = out;
        a.n = n;
        a.base = 0;
        a.scratch = nullptr;
        a.log2g = lg;
        a.err = nullptr;
        return a;
    };
    for (int pc = 0; pc < QX_NUM_PAIR_CLASSES; ++pc) {
        if (!diag_rng[pc].second) continue;
        const int cls = quartet_cls(pc, pc);
        if (!k_class_coop[cls] && k_class_scratch[cls])
            return nofail(QX_E_UNSUPPORTED, "qx_compute_2e_int_noalloc: class %d needs global accumulators", cls);
        launch_class(cls, args(d_diag + diag_rng[pc].first, diag_rng[pc].second, d_kp, 0, 0), MODE_SCHWARZ, s);
        NA_CUDA(cudaGetLastError());
    }
    std::vector<double> kp(np);
    NA_CUDA(cudaMemcpyAsync(kp.data(), d_kp, sizeof(double) * np, cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
    // screening with the reference's semantics, unique quartets per class
    double kmax = 0.0;
    for (double v : kp) kmax = std::max(kmax, v);
    const double thr2 = ints_tol * ints_tol, cut = thr2 / kmax;
    std::vector<int> kept;
    for (int s1 = 0; s1 < nshell; ++s1)
        for (int s2 = 0; s2 <= s1; ++s2) {
            const int p = s1 * (s1 + 1) / 2 + s2;
            if (kp[p] >= cut) kept.push_back(p);
        }
    std::vector<std::vector<int2>> lists(QX_NUM_CLASSES);
    for (size_t i = 0; i < kept.size(); ++i)
        for (size_t j = 0; j <= i; ++j) {
            if (kp[kept[i]] * kp[kept[j]] < thr2) continue;
            int pb = kept[i], pk = kept[j];
            if (pcls[pb] < pcls[pk]) std::swap(pb, pk);
            lists[quartet_cls(pcls[pb], pcls[pk])].push_back(make_int2(pb, pk));
        }
    // --- scratch layout part 2: the class lists, sorted by primitive counts ---
    size_t o = o_lists;
    std::vector<size_t> loff(QX_NUM_CLASSES);
    std::vector<long long> prim_work(QX_NUM_CLASSES, 0);
    for (int c = 0; c < QX_NUM_CLASSES; ++c) {
        auto& L = lists[c];
        std::stable_sort(L.begin(), L.end(), [&](const int2& x, const int2& y) {
            const int kx = pairs[x.x].nprim * 64 + pairs[x.y].nprim, ky = pairs[y.x].nprim * 64 + pairs[y.y].nprim;
            return kx > ky;
        });
        for (auto& q : L) prim_work[c] += (long long)pairs[q.x].nprim * pairs[q.y].nprim;
        if (!L.empty() && !k_class_coop[c] && k_class_scratch[c])
            return nofail(QX_E_UNSUPPORTED, "qx_compute_2e_int_noalloc: class %d needs global accumulators", c);
        loff[c] = o;
        o = align256(o + sizeof(int2) * L.size());
    }
    if (o > QX_NOALLOC_SCRATCH_BYTES)
        return nofail(QX_E_INVALID,
                      "qx_compute_2e_int_noalloc: %zu bytes of tables exceed the %u-byte scratch; use the handle API",
                      o, QX_NOALLOC_SCRATCH_BYTES);
    for (int c = 0; c < QX_NUM_CLASSES; ++c)
        if (!lists[c].empty())
            NA_CUDA(cudaMemcpyAsync(base + loff[c], lists[c].data(), sizeof(int2) * lists[c].size(),
                                    cudaMemcpyHostToDevice, s));
    const long long n = nbf;
    NA_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double) * n * n * n * n, s));
    for (int c = 0; c < QX_NUM_CLASSES; ++c) {
        if (lists[c].empty()) continue;
        const long long nq = (long long)lists[c].size();
        const int lg = k_class_coop[c] ? 0 : choose_lg(nq, prim_work[c]);
        launch_class(c, args((const int2*)(base + loff[c]), nq, out_dev, n, lg), MODE_DENSE, s);
        NA_CUDA(cudaGetLastError());
    }
    // returns once the tensor is complete (the host tables above are freed on return)
    NA_CUDA(cudaStreamSynchronize(s));
#undef NA_CUDA
    return QX_OK;
}
