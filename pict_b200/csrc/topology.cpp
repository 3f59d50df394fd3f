// topology.cpp -- host-side neighbour tables for structured multi-block domains.
//
// Restates the neighbour resolution the reference performs per thread inside
// every kernel (resolveNeighborCell extensions/PISO_multiblock_cuda_kernel.cu:432-477, computeConnectedPos
// extensions/PISO_multiblock_cuda_kernel.cu:326-345) as a one-off table build, plus the connection checks of
// Domain::PrepareSolve (extensions/domain_structs.cpp:2554-2676).
#include <cstdio>
#include <cstring>
#include <string>
#include "pict_b200.h"

namespace pict {
pict_status_t set_error(pict_status_t code, const char* msg);
}

extern "C" pict_status_t pict_build_topology(const pict_block_t* blocks, int32_t num_blocks, int32_t dims,
                                             int32_t num_cells, int32_t* nbr, int32_t* cell_block) {
    using pict::set_error;
    if (!blocks || !nbr || !cell_block || num_blocks <= 0) return set_error(PICT_ERR_ARG, "topology: NULL argument");
    if (dims < 1 || dims > 3) return set_error(PICT_ERR_ARG, "topology: dims must be 1..3");
    char msg[256];
    // offsets and sizes
    int64_t off = 0;
    for (int b = 0; b < num_blocks; ++b) {
        const pict_block_t& B = blocks[b];
        for (int a = 0; a < 3; ++a) {
            if (B.size[a] < 1 || (a >= dims && B.size[a] != 1)) {
                std::snprintf(msg, sizeof(msg), "topology: block %d has invalid size", b);
                return set_error(PICT_ERR_ARG, msg);
            }
        }
        if (B.offset != off) {
            std::snprintf(msg, sizeof(msg), "topology: block %d offset %d, expected %lld", b, B.offset, (long long)off);
            return set_error(PICT_ERR_ARG, msg);
        }
        off += (int64_t)B.size[0] * B.size[1] * B.size[2];
    }
    if (off != num_cells) return set_error(PICT_ERR_ARG, "topology: num_cells does not match the blocks");
    // connection checks (extensions/domain_structs.cpp:2575-2650)
    for (int b = 0; b < num_blocks; ++b) {
        const pict_block_t& B = blocks[b];
        for (int f = 0; f < 2 * dims; ++f) {
            const pict_face_t& F = B.face[f];
            if (F.type == PICT_FACE_PERIODIC) {
                if (B.face[f ^ 1].type != PICT_FACE_PERIODIC) {
                    std::snprintf(msg, sizeof(msg), "topology: block %d face %d periodic but the opposite face is not", b, f);
                    return set_error(PICT_ERR_ARG, msg);
                }
            } else if (F.type == PICT_FACE_CONNECTED) {
                const int o = F.conn_block;
                if (o < 0 || o >= num_blocks) return set_error(PICT_ERR_ARG, "topology: connected block out of range");
                const int of = F.conn_axes[0];
                if (of < 0 || of >= 2 * dims) return set_error(PICT_ERR_ARG, "topology: connected face out of range");
                const pict_face_t& G = blocks[o].face[of];
                if (G.type != PICT_FACE_CONNECTED || G.conn_block != b || G.conn_axes[0] != f) {
                    std::snprintf(msg, sizeof(msg), "topology: block %d face %d: connection is not mutual", b, f);
                    return set_error(PICT_ERR_ARG, msg);
                }
                if (blocks[o].sim != B.sim) return set_error(PICT_ERR_ARG, "topology: blocks of different systems are connected");
                // tangential sizes must match
                for (int k = 1; k < dims; ++k) {
                    const int ax = ((f >> 1) + k) % dims;
                    const int oax = F.conn_axes[k] >> 1;
                    if (B.size[ax] != blocks[o].size[oax]) {
                        std::snprintf(msg, sizeof(msg), "topology: block %d face %d: connection axis %d size mismatch", b, f, k);
                        return set_error(PICT_ERR_ARG, msg);
                    }
                }
            } else if (F.type != PICT_FACE_FIXED) {
                return set_error(PICT_ERR_ARG, "topology: unknown face type");
            }
        }
    }
    // tables
    const int64_t N = num_cells;
    for (int b = 0; b < num_blocks; ++b) {
        const pict_block_t& B = blocks[b];
        const int sx = B.size[0], sy = B.size[1], sz = B.size[2];
        const int stride[3] = {1, sx, sx * sy};
        const int n = sx * sy * sz;
        for (int l = 0; l < n; ++l) {
            const int i = B.offset + l;
            cell_block[i] = b;
            const int p[3] = {l % sx, (l / sx) % sy, l / (sx * sy)};
            for (int f = 0; f < 2 * dims; ++f) {
                const int a = f >> 1;
                const int up = f & 1;
                const bool at = up ? (p[a] == B.size[a] - 1) : (p[a] == 0);
                int j;
                if (!at) {
                    j = i + (up ? stride[a] : -stride[a]);
                } else {
                    const pict_face_t& F = B.face[f];
                    if (F.type == PICT_FACE_FIXED) {
                        j = -1;
                    } else if (F.type == PICT_FACE_PERIODIC) {
                        int q[3] = {p[0], p[1], p[2]};
                        q[a] = up ? 0 : B.size[a] - 1;
                        j = B.offset + q[0] + stride[1] * q[1] + stride[2] * q[2];
                    } else {
                        const pict_block_t& O = blocks[F.conn_block];
                        int q[3] = {p[0], p[1], p[2]};
                        const int ca = F.conn_axes[0] >> 1;
                        q[ca] = (F.conn_axes[0] & 1) ? O.size[ca] - 1 : 0;
                        for (int k = 1; k < dims; ++k) {
                            const int ax = (a + k) % dims;
                            const int cak = F.conn_axes[k] >> 1;
                            q[cak] = (F.conn_axes[k] & 1) ? O.size[cak] - 1 - p[ax] : p[ax];
                        }
                        j = O.offset + q[0] + O.size[0] * (q[1] + O.size[1] * q[2]);
                    }
                }
                nbr[(int64_t)f * N + i] = j;
            }
        }
    }
    return PICT_OK;
}

extern "C" pict_status_t pict_build_tiles(const pict_block_t* blocks, int32_t num_blocks, int32_t num_sims,
                                          int32_t tile_cells, int32_t* tiles, int32_t max_tiles, int32_t* sim_tiles,
                                          int32_t* num_tiles_out) {
    using pict::set_error;
    if (!blocks || !sim_tiles || !num_tiles_out || num_blocks <= 0 || num_sims <= 0 || tile_cells <= 0)
        return set_error(PICT_ERR_ARG, "tiles: invalid argument");
    int32_t n = 0;
    int32_t sim = 0;
    sim_tiles[0] = 0;
    for (int b = 0; b < num_blocks; ++b) {
        const pict_block_t& B = blocks[b];
        if (B.sim < sim || B.sim >= num_sims) return set_error(PICT_ERR_ARG, "tiles: blocks must be ordered by system");
        while (sim < B.sim) sim_tiles[++sim] = n;
        const int cells = B.size[0] * B.size[1] * B.size[2];
        for (int c = 0; c < cells; c += tile_cells) {
            if (tiles && n < max_tiles) {
                tiles[4 * n + 0] = B.sim;
                tiles[4 * n + 1] = b;
                tiles[4 * n + 2] = B.offset + c;
                tiles[4 * n + 3] = (cells - c) < tile_cells ? (cells - c) : tile_cells;
            }
            ++n;
        }
    }
    while (sim < num_sims) sim_tiles[++sim] = n;
    *num_tiles_out = n;
    if (!tiles || n > max_tiles) return set_error(PICT_ERR_ARG, "tiles: output buffer too small");
    return PICT_OK;
}
