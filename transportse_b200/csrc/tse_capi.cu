// Workspace sizing and version entry points of libtsecuda.so.
#include "tse_common.cuh"

namespace tse {
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

extern "C" const char* tse_version(void) { return "transportse_b200 libtsecuda 0.1 (sm_100a)"; }
