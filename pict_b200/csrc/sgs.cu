// sgs.cu -- Smagorinsky sub-grid-scale viscosity (SGSviscosityIncompressibleSmagorinsky,
// extensions/PISO_multiblock_cuda_kernel.cu:6896-7019).
//
// Per cell: the velocity gradient by differences of the two neighbours along each computational axis
// (getBlockDataGradient, extensions/PISO_multiblock_cuda_kernel.cu:2987-3031: across a fixed face the
// boundary velocity at half a cell, across a connection the same component of the connected block's
// adjacent cell, periodic faces wrap), times Minv; the strain-rate norm |S| = sqrt(2 S:S); and
// nu_sgs = coefficient * delta * |S| with delta the largest squared column length of the cell's
// transform M (1 without a transform), as the reference computes it.
#include "common.cuh"
#include "launch.h"

namespace pict {

template <typename T, int D>
__global__ void k_sgs_smagorinsky(pict_domain_t dom, T coefficient, T* out) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        T g[D][D];  // g[c][k] = d u_c / d xi_k (computational axes)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            T dist = T(2);
            T v[2][D];
#pragma unroll
            for (int up = 0; up < 2; ++up) {
                const int f = 2 * k + up;
                const Nbr n = neighbour(dom, B, b, p, i, f);
                if (n.j >= 0) {
                    const pict_block_t& Bn = dom.blocks[n.b];
                    const int ncn = Bn.size[0] * Bn.size[1] * Bn.size[2];
                    const T* un = reinterpret_cast<const T*>(Bn.velocity);
#pragma unroll
                    for (int c = 0; c < D; ++c) v[up][c] = un[(size_t)c * ncn + n.l];
                } else {
                    const FixedFace<T, D> ff = fixed_face<T, D>(B, p, f);
#pragma unroll
                    for (int c = 0; c < D; ++c) v[up][c] = ff.vel[c];
                    dist -= T(0.5);
                }
            }
#pragma unroll
            for (int c = 0; c < D; ++c) g[c][k] = (v[1][c] - v[0][c]) / dist;
        }
        T G[D][D];  // G[c][j] = sum_k g[c][k] Minv[k][j]
#pragma unroll
        for (int c = 0; c < D; ++c)
#pragma unroll
            for (int j = 0; j < D; ++j) {
                if (tr) {
                    T s = T(0);
#pragma unroll
                    for (int k = 0; k < D; ++k) s += g[c][k] * tr_minv<T, D>(tr, k, j);
                    G[c][j] = s;
                } else {
                    G[c][j] = g[c][j];
                }
            }
        T ss = T(0);
#pragma unroll
        for (int a = 0; a < D; ++a)
#pragma unroll
            for (int c = a; c < D; ++c) {
                T s = T(0.5) * (G[a][c] + G[c][a]);
                s *= s;
                ss += (a != c) ? T(2) * s : s;
            }
        const T norm = sqrt(T(2) * ss);
        T delta = T(1);
        if (tr) {
            delta = T(0);
#pragma unroll
            for (int col = 0; col < D; ++col) {
                T m = T(0);
#pragma unroll
                for (int row = 0; row < D; ++row) m += tr[row * D + col] * tr[row * D + col];
                delta = m > delta ? m : delta;
            }
        }
        out[i] = coefficient * delta * norm;
    }
}

}  // namespace pict

using namespace pict;

extern "C" pict_status_t pict_sgs_smagorinsky(const pict_domain_t* dom, double coefficient, void* out, void* stream) {
    if (!dom || !out || !dom->blocks || !dom->nbr || !dom->cell_block) return set_error(PICT_ERR_ARG, "sgs_smagorinsky: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_sgs_smagorinsky<float, 2><<<grid, 256, 0, st>>>(*dom, (float)coefficient, (float*)out);
        else if (dom->dims == 3) k_sgs_smagorinsky<float, 3><<<grid, 256, 0, st>>>(*dom, (float)coefficient, (float*)out);
        else return set_error(PICT_ERR_UNSUPPORTED, "sgs_smagorinsky: unsupported dims");
    } else if (dom->dtype == PICT_F64) {
        if (dom->dims == 2) k_sgs_smagorinsky<double, 2><<<grid, 256, 0, st>>>(*dom, coefficient, (double*)out);
        else if (dom->dims == 3) k_sgs_smagorinsky<double, 3><<<grid, 256, 0, st>>>(*dom, coefficient, (double*)out);
        else return set_error(PICT_ERR_UNSUPPORTED, "sgs_smagorinsky: unsupported dims");
    } else {
        return set_error(PICT_ERR_UNSUPPORTED, "sgs_smagorinsky: unsupported dtype");
    }
    return check_launch("sgs_smagorinsky");
}
