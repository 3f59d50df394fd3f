// refine.cu -- FP64 iterative refinement around the FP32 pressure solve (mixed precision).
//
// The reference solves the pressure Poisson system once per corrector in the domain dtype
// (cgSolveGPU, extensions/cg_solver_kernel.cu:114-456, tolerance on the RMS residual).  In FP32 the
// attainable accuracy of that solve bounds the error of the whole step.  Mixed precision keeps the
// stencil coefficients and Krylov vectors in FP32 and adds an outer loop in FP64:
//
//   x64 = x32 (first FP32 solve);  r = b - P x64  (FP64 arithmetic, stored in the solve dtype)
//   P d = r   (FP32 solve of the correction);  x64 += d;  ... ;  x = x64 - mean(x64)
//
// The residual uses the same stencil rows as the Krylov kernels (neighbours through the domain's
// neighbour table, fixed faces contributing nothing).
#include <cstdio>
#include "common.cuh"
#include "launch.h"

namespace pict {

// r = b - P x in FP64; x is x0 (solve dtype) when given, else x64.  With x0, x64 is initialised to it.
template <typename T, int D>
__global__ void k_refine_residual(pict_domain_t dom, const T* coef, const T* b, const T* x0, double* x64, T* r) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const double xi = x0 ? (double)x0[i] : x64[i];
        double acc = (double)coef[i] * xi;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int j = dom.nbr[(size_t)f * N + i];
            if (j >= 0) acc += (double)coef[(size_t)(f + 1) * N + i] * (x0 ? (double)x0[j] : x64[j]);
        }
        r[i] = (T)((double)b[i] - acc);
        if (x0) x64[i] = xi;
    }
}

template <typename T>
__global__ void k_refine_update(int N, double* x64, const T* d) {
    PICT_CELL_LOOP(i, N) x64[i] += (double)d[i];
}

__device__ __forceinline__ double cta_sum(double v, double* s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

// per-tile sums of x64 (one CTA per Krylov work tile)
__global__ void k_refine_partials(pict_domain_t dom, const double* x64, double* partial) {
    __shared__ double s_red[32];
    const int t = blockIdx.x;
    const int s0 = dom.tiles[4 * t + 2], cnt = dom.tiles[4 * t + 3];
    double acc = 0.0;
    for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) acc += x64[i];
    acc = cta_sum(acc, s_red);
    if (threadIdx.x == 0) partial[t] = acc;
}

// x = x64 - mean of its system (mean from the tile partials in a fixed order), optionally also into
// the blocks' pressure; one CTA per tile
template <typename T>
__global__ void k_refine_finish(pict_domain_t dom, const double* x64, const double* partial, T* x, int subtract_mean,
                                int write_bp) {
    __shared__ double s_red[32];
    __shared__ double s_mean;
    const int t = blockIdx.x;
    const int sim = dom.tiles[4 * t], s0 = dom.tiles[4 * t + 2], cnt = dom.tiles[4 * t + 3];
    if (subtract_mean) {
        double acc = 0.0;
        for (int k = dom.sim_tiles[sim] + threadIdx.x; k < dom.sim_tiles[sim + 1]; k += blockDim.x) acc += partial[k];
        acc = cta_sum(acc, s_red);
        if (threadIdx.x == 0) s_mean = acc / (double)(dom.sim_cells[sim + 1] - dom.sim_cells[sim]);
    } else if (threadIdx.x == 0) {
        s_mean = 0.0;
    }
    __syncthreads();
    const double m = s_mean;
    const pict_block_t& B = dom.blocks[dom.tiles[4 * t + 1]];
    T* pb = reinterpret_cast<T*>(B.pressure);
    for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) {
        const T v = (T)(x64[i] - m);
        x[i] = v;
        if (write_bp) pb[i - B.offset] = v;
    }
}

// per-tile sums of a vector in the solve dtype
template <typename T>
__global__ void k_tile_partials(pict_domain_t dom, const T* v, double* partial) {
    __shared__ double s_red[32];
    const int t = blockIdx.x;
    const int s0 = dom.tiles[4 * t + 2], cnt = dom.tiles[4 * t + 3];
    double acc = 0.0;
    for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) acc += (double)v[i];
    acc = cta_sum(acc, s_red);
    if (threadIdx.x == 0) partial[t] = acc;
}

// v -= mean of its system (from the tile partials, fixed order); one CTA per tile
template <typename T>
__global__ void k_tile_subtract_mean(pict_domain_t dom, T* v, const double* partial) {
    __shared__ double s_red[32];
    __shared__ double s_mean;
    const int t = blockIdx.x;
    const int sim = dom.tiles[4 * t], s0 = dom.tiles[4 * t + 2], cnt = dom.tiles[4 * t + 3];
    double acc = 0.0;
    for (int k = dom.sim_tiles[sim] + threadIdx.x; k < dom.sim_tiles[sim + 1]; k += blockDim.x) acc += partial[k];
    acc = cta_sum(acc, s_red);
    if (threadIdx.x == 0) s_mean = acc / (double)(dom.sim_cells[sim + 1] - dom.sim_cells[sim]);
    __syncthreads();
    const T m = (T)s_mean;
    for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) v[i] -= m;
}

// out = alpha x + beta y over n values
template <typename T>
__global__ void k_vector_axpby(int n, T alpha, const T* x, T beta, const T* y, T* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x)
        out[i] = alpha * x[i] + beta * y[i];
}

}  // namespace pict

using namespace pict;

extern "C" {

pict_status_t pict_vector_axpby(int32_t n, int32_t dtype, double alpha, const void* x, double beta, const void* y,
                                void* out, void* stream) {
    if (n < 0 || !x || !y || !out) return set_error(PICT_ERR_ARG, "vector_axpby: invalid argument");
    if (n == 0) return PICT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(n, 256);
    if (dtype == PICT_F64)
        k_vector_axpby<double><<<grid, 256, 0, st>>>(n, alpha, (const double*)x, beta, (const double*)y, (double*)out);
    else
        k_vector_axpby<float><<<grid, 256, 0, st>>>(n, (float)alpha, (const float*)x, (float)beta, (const float*)y,
                                                   (float*)out);
    return check_launch("vector_axpby");
}

pict_status_t pict_refine_residual(const pict_domain_t* dom, const void* coef, const void* rhs, const void* x_init,
                                   double* x64, void* residual, int32_t project_mean, double* tile_scratch,
                                   void* stream) {
    if (!dom || !coef || !rhs || !x64 || !residual || dom->num_cells <= 0 || !dom->nbr)
        return set_error(PICT_ERR_ARG, "refine_residual: NULL argument or unprepared domain");
    if (project_mean && (!tile_scratch || !dom->tiles || !dom->sim_tiles || dom->num_tiles <= 0))
        return set_error(PICT_ERR_ARG, "refine_residual: projection needs the tile table and tile_scratch");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_refine_residual<float, 2><<<grid, 256, 0, st>>>(*dom, (const float*)coef, (const float*)rhs, (const float*)x_init, x64, (float*)residual);
        else k_refine_residual<float, 3><<<grid, 256, 0, st>>>(*dom, (const float*)coef, (const float*)rhs, (const float*)x_init, x64, (float*)residual);
    } else {
        if (dom->dims == 2) k_refine_residual<double, 2><<<grid, 256, 0, st>>>(*dom, (const double*)coef, (const double*)rhs, (const double*)x_init, x64, (double*)residual);
        else k_refine_residual<double, 3><<<grid, 256, 0, st>>>(*dom, (const double*)coef, (const double*)rhs, (const double*)x_init, x64, (double*)residual);
    }
    pict_status_t s = check_launch("refine_residual");
    if (s || !project_mean) return s;
    // the constant mode of a singular (pure Neumann / periodic) system cannot be solved for: drop it
    if (dom->dtype == PICT_F32) {
        k_tile_partials<float><<<dom->num_tiles, 256, 0, st>>>(*dom, (const float*)residual, tile_scratch);
        k_tile_subtract_mean<float><<<dom->num_tiles, 256, 0, st>>>(*dom, (float*)residual, tile_scratch);
    } else {
        k_tile_partials<double><<<dom->num_tiles, 256, 0, st>>>(*dom, (const double*)residual, tile_scratch);
        k_tile_subtract_mean<double><<<dom->num_tiles, 256, 0, st>>>(*dom, (double*)residual, tile_scratch);
    }
    return check_launch("refine_residual projection");
}

pict_status_t pict_refine_update(const pict_domain_t* dom, double* x64, const void* correction, void* stream) {
    if (!dom || !x64 || !correction) return set_error(PICT_ERR_ARG, "refine_update: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) k_refine_update<float><<<grid, 256, 0, st>>>(dom->num_cells, x64, (const float*)correction);
    else k_refine_update<double><<<grid, 256, 0, st>>>(dom->num_cells, x64, (const double*)correction);
    return check_launch("refine_update");
}

pict_status_t pict_refine_finish(const pict_domain_t* dom, const double* x64, void* x, int32_t subtract_mean,
                                 int32_t write_block_pressure, double* tile_scratch, void* stream) {
    if (!dom || !x64 || !x || !dom->sim_cells || !dom->tiles || !dom->sim_tiles || dom->num_tiles <= 0 ||
        (subtract_mean && !tile_scratch))
        return set_error(PICT_ERR_ARG, "refine_finish: NULL argument or missing tile table");
    cudaStream_t st = (cudaStream_t)stream;
    if (subtract_mean) {
        k_refine_partials<<<dom->num_tiles, 256, 0, st>>>(*dom, x64, tile_scratch);
        pict_status_t s = check_launch("refine_partials");
        if (s) return s;
    }
    if (dom->dtype == PICT_F32)
        k_refine_finish<float><<<dom->num_tiles, 256, 0, st>>>(*dom, x64, tile_scratch, (float*)x, subtract_mean, write_block_pressure);
    else
        k_refine_finish<double><<<dom->num_tiles, 256, 0, st>>>(*dom, x64, tile_scratch, (double*)x, subtract_mean, write_block_pressure);
    return check_launch("refine_finish");
}

}  // extern "C"
