// common.cuh -- device-side helpers shared by the PISO kernels.
//
// The reference resolves neighbours per thread through a switch over boundary
// types (resolveNeighborCell / computeConnectedPos, extensions/PISO_multiblock_cuda_kernel.cu:326-345,
// 432-477).  Here the topology is precomputed once per domain into a
// neighbour table nbr[2D][N] (pict_build_topology); kernels only need the
// face type to tell connected faces apart (their neighbour lives in another
// block, possibly with permuted axes).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "pict_b200.h"

namespace pict {

template <int D> struct TS { static constexpr int value = 2 * D * D + 1; };  // transform stride

struct CellPos {
    int b;       // block index
    int l;       // local (block) flat index
    int p[3];    // x, y, z
};

__device__ __forceinline__ void unflatten(int l, const int32_t* size, int* p) {
    const int sx = size[0], sy = size[1];
    p[0] = l % sx;
    const int t = l / sx;
    p[1] = t % sy;
    p[2] = t / sy;
}

__device__ __forceinline__ bool at_face(const int* p, const int32_t* size, int f) {
    const int a = f >> 1;
    return (f & 1) ? (p[a] == size[a] - 1) : (p[a] == 0);
}

// Flat index into the face arrays of a fixed boundary: position with the face axis set to 0,
// flattened with the boundary's own size (block size with 1 along the face axis),
// like getFixedBoundaryData (extensions/PISO_multiblock_cuda_kernel.cu:2420-2428).
__device__ __forceinline__ int boundary_flat(const int* p, const int32_t* size, int f) {
    const int a = f >> 1;
    int bs[3] = {size[0], size[1], size[2]};
    bs[a] = 1;
    int q[3] = {p[0], p[1], p[2]};
    q[a] = 0;
    return q[0] + bs[0] * (q[1] + bs[1] * q[2]);
}

__device__ __forceinline__ int face_cells(const int32_t* size, int f) {
    const int a = f >> 1;
    int n = 1;
    for (int k = 0; k < 3; ++k) n *= (k == a) ? 1 : size[k];
    return n;
}

template <typename T, int D>
__device__ __forceinline__ T tr_det(const T* tr) { return tr ? tr[2 * D * D] : T(1); }

// Minv[r][c]
template <typename T, int D>
__device__ __forceinline__ T tr_minv(const T* tr, int r, int c) { return tr[D * D + r * D + c]; }

// Contravariant component c of vector u: det * Minv[c] . u (VelocityToContravariantComponent, extensions/PISO_multiblock_cuda_kernel.cu:479-494).
template <typename T, int D>
__device__ __forceinline__ T contravariant(const T* tr, int c, const T* u) {
    if (!tr) return u[c];
    T s = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) s += tr_minv<T, D>(tr, c, k) * u[k];
    return tr_det<T, D>(tr) * s;
}

// Orthogonal Laplace coefficient det * |Minv[c]|^2 (getLaplaceCoefficientOrthogonal, extensions/PISO_multiblock_cuda_kernel.cu:1209-1224).
template <typename T, int D>
__device__ __forceinline__ T laplace_coef(const T* tr, int c) {
    if (!tr) return T(1);
    T s = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const T m = tr_minv<T, D>(tr, c, k);
        s += m * m;
    }
    return tr_det<T, D>(tr) * s;
}

template <typename T, int D>
__device__ __forceinline__ const T* cell_transform(const pict_block_t& B, int l) {
    return B.transform ? reinterpret_cast<const T*>(B.transform) + (size_t)l * TS<D>::value : nullptr;
}

template <typename T>
__device__ __forceinline__ int block_cells(const pict_block_t& B) { return B.size[0] * B.size[1] * B.size[2]; }

// Viscosity at a cell of a block (getViscosityBlock, extensions/PISO_multiblock_cuda_kernel.cu:1801-1822).
template <typename T>
__device__ __forceinline__ T cell_viscosity(const pict_domain_t& dom, const pict_block_t& B, int l) {
    if (B.viscosity) {
        const T* v = reinterpret_cast<const T*>(B.viscosity);
        return B.viscosity_static ? v[0] : v[l];
    }
    return reinterpret_cast<const T*>(dom.sim_viscosity)[B.sim];
}

// Velocity source component c (getBlockVelocitySource, extensions/PISO_multiblock_cuda_kernel.cu:2241-2251).
template <typename T>
__device__ __forceinline__ T cell_source(const pict_block_t& B, int l, int c, int ncells) {
    if (!B.source) return T(0);
    const T* s = reinterpret_cast<const T*>(B.source);
    return B.source_static ? s[c] : s[(size_t)c * ncells + l];
}

template <typename T>
__device__ __forceinline__ T sim_time_step(const pict_domain_t& dom, int sim, double dt) {
    return dom.sim_dt ? reinterpret_cast<const T*>(dom.sim_dt)[sim] : T(dt);
}

// Neighbour across face f of a cell: block, local index, the component of the neighbour that is
// aligned with this face's axis, and the flux sign across the connection (computeFluxesNDLoop,
// extensions/PISO_multiblock_cuda_kernel.cu:1589-1606; computeConnectedPosWithChannel extensions/PISO_multiblock_cuda_kernel.cu:349-360).
struct Nbr {
    int j;      // global index, -1 on fixed faces
    int b;      // block
    int l;      // local index in block b
    int comp;   // neighbour component aligned with this face's axis
    int flip;   // -1 if the connection joins two lower or two upper faces
    int back;   // face of the neighbour pointing back to this cell
};

// A cell that is not on face f of its block has its neighbour inside the block at l +- stride of
// the face's axis (the table holds the same index there), so the table is read on block faces only.
__device__ __forceinline__ Nbr neighbour(const pict_domain_t& dom, const pict_block_t& B, int b, const int* p,
                                         int i, int f) {
    Nbr n;
    n.b = b;
    n.comp = f >> 1;
    n.flip = 1;
    n.back = f ^ 1;
    if (!at_face(p, B.size, f)) {
        const int a = f >> 1;
        const int stride = a == 0 ? 1 : (a == 1 ? B.size[0] : B.size[0] * B.size[1]);
        const int s = (f & 1) ? stride : -stride;
        n.j = i + s;
        n.l = i - B.offset + s;
        return n;
    }
    n.j = dom.nbr[(size_t)f * dom.num_cells + i];
    if (n.j >= 0 && B.face[f].type == PICT_FACE_CONNECTED) {
        const pict_face_t& F = B.face[f];
        n.b = F.conn_block;
        n.comp = F.conn_axes[0] >> 1;
        n.flip = ((F.conn_axes[0] & 1) == (f & 1)) ? -1 : 1;
        n.back = F.conn_axes[0];
    }
    n.l = (n.j >= 0) ? n.j - dom.blocks[n.b].offset : -1;
    return n;
}

// Boundary data of a fixed face: velocity vector, contravariant flux along the face axis and the
// boundary Laplace coefficient (getFixedBoundaryData extensions/PISO_multiblock_cuda_kernel.cu:2374-2433,
// getContravariantComponentBoundaryFixed extensions/PISO_multiblock_cuda_kernel.cu:728-748, extensions/PISO_multiblock_cuda_kernel.cu:1434-1447).
template <typename T, int D>
struct FixedFace {
    T vel[D];
    T contra;
    T alpha;
};

template <typename T, int D>
__device__ __forceinline__ FixedFace<T, D> fixed_face(const pict_block_t& B, const int* p, int f) {
    FixedFace<T, D> r;
    const pict_face_t& F = B.face[f];
    const int a = f >> 1;
    const int bf = boundary_flat(p, B.size, f);
    const T* v = reinterpret_cast<const T*>(F.velocity);
    if (F.vel_static) {
#pragma unroll
        for (int c = 0; c < D; ++c) r.vel[c] = v[c];
    } else {
        const int nf = face_cells(B.size, f);
#pragma unroll
        for (int c = 0; c < D; ++c) r.vel[c] = v[(size_t)c * nf + bf];
    }
    const T* tr = F.transform ? reinterpret_cast<const T*>(F.transform) + (size_t)bf * TS<D>::value : nullptr;
    r.contra = contravariant<T, D>(tr, a, r.vel);
    r.alpha = laplace_coef<T, D>(tr, a);
    return r;
}

template <typename T, int D>
__device__ __forceinline__ void load_block_vec(const pict_block_t& B, const void* base, int l, T* u) {
    const T* v = reinterpret_cast<const T*>(base);
    const int n = B.size[0] * B.size[1] * B.size[2];
#pragma unroll
    for (int c = 0; c < D; ++c) u[c] = v[(size_t)c * n + l];
}

template <typename T, int D>
__device__ __forceinline__ void load_global_vec(const T* v, int N, int j, T* u) {
#pragma unroll
    for (int c = 0; c < D; ++c) u[c] = v[(size_t)c * N + j];
}

// grid-stride loop helper
#define PICT_CELL_LOOP(i, N) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (N); i += blockDim.x * gridDim.x)

// Per-cell loop over a domain, f(i, b) with i the global cell and b its block.  With the domain's work
// tiles (runs of at most tile_cells cells of one block, covering every cell once) the grid strides over
// (tile, chunk of blockDim cells) pairs, so a CTA's block index is one uniform load of the tile instead
// of a per-cell read of cell_block that every other load of the cell waits for; without tiles, a
// grid-stride loop over the cells.  The host sizes the grid with domain_grid().
template <typename F>
__device__ __forceinline__ void for_each_cell(const pict_domain_t& dom, F&& f) {
    if (dom.tiles != nullptr && dom.num_tiles > 0 && dom.tile_cells > 0) {
        const int4* tl = reinterpret_cast<const int4*>(dom.tiles);
        const int per = (dom.tile_cells + blockDim.x - 1) / blockDim.x;
        const int total = dom.num_tiles * per;
        for (int v = blockIdx.x; v < total; v += gridDim.x) {
            const int t = v / per;
            const int4 d = tl[t];  // system, block, first cell, cell count
            const int k = (v - t * per) * blockDim.x + threadIdx.x;
            if (k < d.w) f(d.z + k, d.y);
        }
    } else {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < dom.num_cells; i += blockDim.x * gridDim.x)
            f(i, dom.cell_block[i]);
    }
}

}  // namespace pict
