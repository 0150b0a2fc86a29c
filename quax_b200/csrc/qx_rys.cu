// qx_rys.cu -- the Rys quadrature table on the device.
//
// The node/weight table (qx_rys_table.inc, ~345 KB) is a statically initialised
// __device__ array: it is loaded with the module, so no allocation or copy is
// needed.  Host code reaches it through qx_rys_table(), which looks up the
// array's device address once per device (cudaGetSymbolAddress) -- the symbol
// itself is only a host-side stand-in.
#include <cuda_runtime.h>

#include <mutex>

#include "qx_rys.cuh"

__device__ const double g_qx_rys_table[qx::RYS_TABLE_DOUBLES] = {QX_RYS_TAB_DATA QX_RYS_ASYM_Y_DATA,
                                                                 QX_RYS_ASYM_W_DATA};

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
const double* g_addr[kMaxDevices] = {};
}  // namespace

// Device address of the table on the current device (nullptr on failure).
const double* qx_rys_table() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_qx_rys_table) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_addr[dev] = static_cast<const double*>(p);
    }
    return g_addr[dev];
}
