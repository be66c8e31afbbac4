// Workspace sizing, version and tuning entry points of libtsecuda.so.
#include <atomic>

#include "tse_common.cuh"

namespace tse {
namespace {
std::atomic<int> g_exact_sweep{1};
std::atomic<int> g_batch_loop{1};
}  // namespace
int exact_sweep_mode() { return g_exact_sweep.load(std::memory_order_relaxed); }
int batch_loop_mode() { return g_batch_loop.load(std::memory_order_relaxed); }
size_t pressure_ws_bytes(const Layout& L, long long* Ncal_out);
size_t transport_ws_bytes(const Layout& L, long long* Ncal_out);
size_t reduce_ws_bytes();
size_t dc_extra_bytes(const Layout& L);
}  // namespace tse

using namespace tse;

extern "C" size_t tse_workspace_bytes(const TseGrid* grid, int32_t kind) {
    if (!grid || grid->nx < 1 || grid->ny < 1 || grid->nz < 1) return 0;
    Layout L = make_layout(grid->nx, grid->ny, grid->nz);
    switch (kind) {
        case TSE_WS_PRESSURE: return pressure_ws_bytes(L, nullptr);
        case TSE_WS_TRANSPORT: return transport_ws_bytes(L, nullptr);
        case TSE_WS_REDUCE: return reduce_ws_bytes();
        case TSE_WS_PRESSURE_DC: return pressure_ws_bytes(L, nullptr) + dc_extra_bytes(L);
        case TSE_WS_TRANSPORT_DC: return transport_ws_bytes(L, nullptr) + dc_extra_bytes(L);
        default: return 0;
    }
}

extern "C" int32_t tse_set_exact_sweep(int32_t mode) {
    if (mode != 0 && mode != 1) return TSE_ERR_ARG;
    return g_exact_sweep.exchange(mode);
}

extern "C" int32_t tse_set_batch_loop(int32_t mode) {
    if (mode != 0 && mode != 1) return TSE_ERR_ARG;
    return g_batch_loop.exchange(mode);
}

extern "C" const char* tse_version(void) { return "transportse_b200 libtsecuda 0.1 (sm_100a)"; }
