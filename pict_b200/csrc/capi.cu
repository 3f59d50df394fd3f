// capi.cu -- library-level entry points: version, error reporting, launch helpers.
#include <cstdio>
#include <cstring>
#include <mutex>
#include "launch.h"

namespace pict {

static thread_local char g_last_error[512] = "";

pict_status_t set_error(pict_status_t code, const char* msg) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg ? msg : "");
    return code;
}

pict_status_t check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
        return set_error(PICT_ERR_CUDA, buf);
    }
    return PICT_OK;
}

int device_sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

int cell_grid(int n, int threads) {
    int g = (n + threads - 1) / threads;
    const int cap = device_sm_count() * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return g;
}

int domain_grid(const pict_domain_t* dom, int threads) {
    if (!dom->tiles || dom->num_tiles <= 0 || dom->tile_cells <= 0) return cell_grid(dom->num_cells, threads);
    const long long total = (long long)dom->num_tiles * ((dom->tile_cells + threads - 1) / threads);
    const long long cap = (long long)device_sm_count() * 16;
    return (int)(total < cap ? (total < 1 ? 1 : total) : cap);
}

}  // namespace pict

extern "C" {

const char* pict_version(void) { return "pict_b200 0.1 (sm_100a)"; }
const char* pict_last_error(void) { return pict::g_last_error; }
int32_t pict_sizeof_block(void) { return (int32_t)sizeof(pict_block_t); }
int32_t pict_sizeof_domain(void) { return (int32_t)sizeof(pict_domain_t); }

}  // extern "C"
