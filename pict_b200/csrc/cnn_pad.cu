// cnn_pad.cu -- the padding of the multi-block convolution (MultiblockConv, the reference's
// lib/modules/multiblock_cnn.py:92-369): every block's field surrounded by `padding` cells taken from the
// blocks it is connected to (and zeros at fixed faces), as one gather over all blocks, and its gradient as
// one gather-sum over the inverse map.
//
// Fields are [batch][channels][cells] per block (the NC(D)HW tensors flattened), addressed through the blocks'
// pointers passed by value in the kernel parameters (up to MB_MAX blocks), so the blocks are read in place
// (no concatenated copy) and a call needs no host-to-device copy.  The map is built once
// on the host: for every padded cell (output block, position) its source (block, cell) or -1 (zero); the
// inverse lists, for every source cell, the padded cells that read it (CSR), so the gradient of each
// source cell is the sum of its readers' gradients in a fixed order (deterministic, no atomics).
#include "common.cuh"
#include "launch.h"

namespace pict {

constexpr int PAD_THREADS = 256;
constexpr int MB_MAX = 64;  // blocks per call (the pointer tables travel in the kernel parameters)

template <typename T>
struct MbTable {
    T* p[MB_MAX];
    int64_t n[MB_MAX];  // cells per block (unpadded for the sources, padded for the outputs)
};

// out[ob][bc][pos] = src[sb][bc][loc] (0 where sb < 0) for padded cell j = (ob, pos) <- (sb, loc)
template <typename T>
__global__ void k_mb_pad_gather(int n, int bc, const int32_t* __restrict__ ob, const int32_t* __restrict__ pos,
                                const int32_t* __restrict__ sb, const int32_t* __restrict__ loc, const MbTable<T> src,
                                const MbTable<T> out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int o = ob[j], p = pos[j], s = sb[j], l = loc[j];
    T* dst = out.p[o] + p;
    const int64_t os = out.n[o];
    if (s < 0) {
        for (int c = blockIdx.y; c < bc; c += gridDim.y) dst[(size_t)c * os] = T(0);
        return;
    }
    const T* from = src.p[s] + l;
    const int64_t ss = src.n[s];
    for (int c = blockIdx.y; c < bc; c += gridDim.y) dst[(size_t)c * os] = from[(size_t)c * ss];
}

// gsrc[sb][bc][loc] = sum over the readers k of source cell g = (sb, loc) of gout[ob_k][bc][pos_k]
template <typename T>
__global__ void k_mb_pad_scatter_sum(int n, int bc, const int32_t* __restrict__ sb, const int32_t* __restrict__ loc,
                                     const int32_t* __restrict__ ptr, const int32_t* __restrict__ rob,
                                     const int32_t* __restrict__ rpos, const MbTable<T> gout, const MbTable<T> gsrc) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int s = sb[g], l = loc[g], k0 = ptr[g], k1 = ptr[g + 1];
    T* dst = gsrc.p[s] + l;
    const int64_t ss = gsrc.n[s];
    for (int c = blockIdx.y; c < bc; c += gridDim.y) {
        T acc = T(0);
        for (int k = k0; k < k1; ++k) acc += gout.p[rob[k]][(size_t)c * gout.n[rob[k]] + rpos[k]];
        dst[(size_t)c * ss] = acc;
    }
}

template <typename T>
static bool mb_table(int nb, const void* const* ptrs, const int64_t* cells, MbTable<T>& t) {
    if (nb < 1 || nb > MB_MAX) return false;
    for (int b = 0; b < MB_MAX; ++b) {
        t.p[b] = b < nb ? (T*)ptrs[b] : nullptr;
        t.n[b] = b < nb ? cells[b] : 0;
    }
    return true;
}

static dim3 pad_grid(int n, int bc) {
    const int gx = (n + PAD_THREADS - 1) / PAD_THREADS;
    // enough CTAs to fill the device; each CTA of the y dimension covers a stride of channels
    int gy = bc < 1 ? 1 : bc;
    const long long want = 8ll * device_sm_count();
    while (gy > 1 && (long long)gx * gy > 4 * want) gy = (gy + 1) / 2;
    if (gy > 65535) gy = 65535;
    return dim3(gx < 1 ? 1 : gx, gy);
}

}  // namespace pict

using namespace pict;

extern "C" {

pict_status_t pict_mb_pad_gather(int32_t n, int32_t batch_channels, int32_t dtype, int32_t num_blocks,
                                 const int32_t* out_block, const int32_t* out_pos, const int32_t* src_block,
                                 const int32_t* src_loc, const void* const* src_ptrs, const int64_t* src_cells,
                                 void* const* out_ptrs, const int64_t* out_cells, void* stream) {
    if (n < 0 || batch_channels < 0 || (n > 0 && (!out_block || !out_pos || !src_block || !src_loc || !src_ptrs ||
                                                  !src_cells || !out_ptrs || !out_cells)))
        return set_error(PICT_ERR_ARG, "mb_pad_gather: invalid argument");
    if (n == 0 || batch_channels == 0) return PICT_OK;
    const dim3 grid = pad_grid(n, batch_channels);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == PICT_F64) {
        MbTable<double> src, out;
        if (!mb_table(num_blocks, src_ptrs, src_cells, src) || !mb_table(num_blocks, (const void* const*)out_ptrs, out_cells, out))
            return set_error(PICT_ERR_ARG, "mb_pad_gather: 1 to 64 blocks");
        k_mb_pad_gather<double><<<grid, PAD_THREADS, 0, st>>>(n, batch_channels, out_block, out_pos, src_block, src_loc,
                                                               src, out);
    } else {
        MbTable<float> src, out;
        if (!mb_table(num_blocks, src_ptrs, src_cells, src) || !mb_table(num_blocks, (const void* const*)out_ptrs, out_cells, out))
            return set_error(PICT_ERR_ARG, "mb_pad_gather: 1 to 64 blocks");
        k_mb_pad_gather<float><<<grid, PAD_THREADS, 0, st>>>(n, batch_channels, out_block, out_pos, src_block, src_loc,
                                                              src, out);
    }
    return check_launch("mb_pad_gather");
}

pict_status_t pict_mb_pad_scatter_sum(int32_t n, int32_t batch_channels, int32_t dtype, int32_t num_blocks,
                                      const int32_t* src_block, const int32_t* src_loc, const int32_t* reader_ptr,
                                      const int32_t* reader_block, const int32_t* reader_pos,
                                      const void* const* gout_ptrs, const int64_t* out_cells, void* const* gsrc_ptrs,
                                      const int64_t* src_cells, void* stream) {
    if (n < 0 || batch_channels < 0 || (n > 0 && (!src_block || !src_loc || !reader_ptr || !reader_block ||
                                                  !reader_pos || !gout_ptrs || !out_cells || !gsrc_ptrs ||
                                                  !src_cells)))
        return set_error(PICT_ERR_ARG, "mb_pad_scatter_sum: invalid argument");
    if (n == 0 || batch_channels == 0) return PICT_OK;
    const dim3 grid = pad_grid(n, batch_channels);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == PICT_F64) {
        MbTable<double> gout, gsrc;
        if (!mb_table(num_blocks, gout_ptrs, out_cells, gout) || !mb_table(num_blocks, (const void* const*)gsrc_ptrs, src_cells, gsrc))
            return set_error(PICT_ERR_ARG, "mb_pad_scatter_sum: 1 to 64 blocks");
        k_mb_pad_scatter_sum<double><<<grid, PAD_THREADS, 0, st>>>(n, batch_channels, src_block, src_loc, reader_ptr,
                                                                    reader_block, reader_pos, gout, gsrc);
    } else {
        MbTable<float> gout, gsrc;
        if (!mb_table(num_blocks, gout_ptrs, out_cells, gout) || !mb_table(num_blocks, (const void* const*)gsrc_ptrs, src_cells, gsrc))
            return set_error(PICT_ERR_ARG, "mb_pad_scatter_sum: 1 to 64 blocks");
        k_mb_pad_scatter_sum<float><<<grid, PAD_THREADS, 0, st>>>(n, batch_channels, src_block, src_loc, reader_ptr,
                                                                   reader_block, reader_pos, gout, gsrc);
    }
    return check_launch("mb_pad_scatter_sum");
}

}  // extern "C"
