// krylov.cu -- persistent, tiled CG and BiCGStab on structured stencil matrices.
//
// Replaces the reference's host-driven Krylov loops (cgSolveGPU,
// extensions/cg_solver_kernel.cu:114-456; bicgstabSolveGPU,
// extensions/bicgstab_solver_kernel.cu:47-395), which issue one cuSPARSE SpMV
// plus several cuBLAS calls with host round trips per iteration, by one
// persistent launch per solve that advances every system of a (batched) domain
// in lock step:
//
//  * the cells of all systems are cut into tiles (contiguous runs of at most
//    tile_cells cells inside one block, pict_build_tiles); each CTA owns a fixed
//    set of tiles (round robin) and, per phase, sweeps its tiles of the systems
//    that are still iterating, so uneven systems share the SMs and converged
//    systems cost nothing;
//  * one bounded grid barrier per phase (two per CG iteration, four per
//    BiCGStab iteration); every wait has an iteration limit after which the
//    kernel records an error and returns;
//  * inner products are accumulated in FP64, reduced per tile inside the CTA
//    and then per system over the tile partials in a fixed order, so results do
//    not depend on the number of CTAs and are bitwise reproducible;
//  * the stencil SpMV reads structured neighbours directly (i +- stride) and
//    uses the precomputed neighbour table only on block faces; the search
//    direction is formed on the fly for the neighbours (double buffered), so
//    vector updates need no extra pass;
//  * BiCGStab advances all right-hand sides of a system (the D velocity
//    components) together, sharing the matrix loads, each with its own scalars
//    and convergence state.
//
// Iteration semantics, stopping rule and reported iteration counts follow the
// reference: CG extensions/cg_solver_kernel.cu:236-427, BiCGStab extensions/bicgstab_solver_kernel.cu:240-360, convergence criterion
// NORM2 / NORM2_NORMALIZED extensions/cg_solver_kernel.cu:77-110.  As in the Python wrapper
// (PISOtorch_diff.py:245-293), an all-zero right-hand side yields x = 0.
#include <cmath>
#include <cstdio>
#include <mutex>
#include <cooperative_groups.h>
#include "common.cuh"
#include "launch.h"

namespace cgrp = cooperative_groups;

#ifndef PICT_SPIN_LIMIT
#define PICT_SPIN_LIMIT (1ll << 26)
#endif

namespace pict {

constexpr int KR_NV = 8;         // values per tile partial
constexpr int KR_SLOTS = 32;     // tiles per CTA (lane j of warp 0 holds the scalars of slot j)
constexpr int KR_THREADS = 512;  // threads per CTA
constexpr int KR_CPT = 4;        // cells per thread per tile: tile_cells <= KR_CPT * KR_THREADS
constexpr int KR_MAX_TILE = KR_CPT * KR_THREADS;
constexpr int KR_U = 2;          // cells per thread and pass of the phase sweeps (loads of both in flight)
constexpr int KR_PASS = KR_U * KR_THREADS;

// ctrl words in the workspace header (cleared before every launch)
// CTRL_BAR_COUNT counts barrier arrivals (monotonic).  CTRL_DONE counts finished systems (classic CG /
// BiCGStab: increments and reads are always separated by a grid barrier).  The single-reduction CG
// has one barrier per iteration, so completions of iteration i go to CTRL_DONE_PAR + (i & 1) and are
// read only after the barrier of iteration i+1.
enum { CTRL_ERR = 0, CTRL_DONE = 1, CTRL_BAR_COUNT = 2, CTRL_DONE_PAR = 4, CTRL_SCHED = 8 };

template <typename T>
struct KArgs {
    pict_domain_t dom;
    const T* coef;
    const T* b;
    T* x;
    T* r;
    T* rw;
    T* p0;
    T* p1;
    T* v0;
    T* v1;
    T* t;
    T* r1;  // two-barrier BiCGStab: second residual buffer
    int* ctrl;
    double* partials;  // [2][num_tiles][KR_NV]
    pict_solve_info_t* info;
    int maxit;
    double tol;
    int normalized;
    int nrhs;  // stride of the info records per system
    int x_zero;
    int sub_mean;
    int write_bp;
    int reset;  // CG: restart period (0: none)
    int best;   // CG: keep and return the best iterate
    T* xbest;
    int abs_crit;  // classic CG: 0 NORM2 criteria, else PICT_CONV_ABS_SUM / _MEAN / _MAX
    int rankdef;   // classic CG: operator A + s |.|_1 e (matrixRankDeficient)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Bounded barrier over all CTAs of the launch.  The arrival counter is monotonic: barrier number
// `epoch` (1, 2, ...) is complete once it reaches epoch * gridDim.x, so each CTA issues one atomic and
// nothing is reset.  After the wait thread 0 also reads the completion counters into s_ctrl
// ([CTRL_DONE, CTRL_DONE_PAR, CTRL_DONE_PAR + 1]); they stay valid until the next barrier.
__device__ bool grid_barrier(int* ctrl, unsigned& epoch, int* s_ctrl) {
    __shared__ int s_ok;
    __syncthreads();
    ++epoch;
    if (threadIdx.x == 0) {
        int ok = 1;
        if (gridDim.x > 1) {
            unsigned* count = reinterpret_cast<unsigned*>(ctrl + CTRL_BAR_COUNT);
            const unsigned target = epoch * gridDim.x;
            __threadfence();
            atomicAdd(count, 1u);
            long long spins = 0;
            while ((int)(*(volatile unsigned*)count - target) < 0) {
                if (++spins > PICT_SPIN_LIMIT) { ok = 0; atomicExch(ctrl + CTRL_ERR, 1); break; }
                if ((spins & 63) == 0 && *(volatile int*)(ctrl + CTRL_ERR)) { ok = 0; break; }
                __nanosleep(16);
            }
            __threadfence();
        }
        const int err = *(volatile int*)(ctrl + CTRL_ERR);
        s_ctrl[0] = *(volatile int*)(ctrl + CTRL_DONE);
        s_ctrl[1] = *(volatile int*)(ctrl + CTRL_DONE_PAR);
        s_ctrl[2] = *(volatile int*)(ctrl + CTRL_DONE_PAR + 1);
        s_ok = ok && err == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

// Block-wide sum of NV values; the result is returned to every thread.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
    __shared__ double s_red[KR_THREADS / 32][KR_NV];
    __shared__ double s_out[KR_NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const double w = warp_sum(v[k]);
        if (lane == 0) s_red[warp][k] = w;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double w = lane < nwarps ? s_red[lane][k] : 0.0;
            w = warp_sum(w);
            if (lane == 0) s_out[k] = w;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = s_out[k];
    __syncthreads();
}

// Per-phase tile partials: every tile's values are reduced within each warp (shuffles, no block
// synchronisation) into s_warp[slot][warp][k]; after all tiles of the phase, flush_partials() sums
// over the warps in a fixed order and writes the tile partials (one __syncthreads per phase).
struct PhaseRed {
    double v[KR_SLOTS][KR_THREADS / 32][KR_NV];
};

// Components whose bit is set in MAXMASK are combined by maximum instead of sum (ABS_MAX criterion).
template <int NV, unsigned MAXMASK = 0u>
__device__ __forceinline__ void warp_partial(PhaseRed& R, int slot, const double (&acc)[NV]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const double w = ((MAXMASK >> k) & 1u) ? warp_max(acc[k]) : warp_sum(acc[k]);
        if (lane == 0) R.v[slot][warp][k] = w;
    }
}

// Per-CTA tile bookkeeping in shared memory.
struct TileSlots {
    int n;                       // slots used by this CTA
    int tile[KR_SLOTS];
    int sim[KR_SLOTS];
    int block[KR_SLOTS];
    int start[KR_SLOTS];
    int count[KR_SLOTS];
    int t0[KR_SLOTS];            // tile range of the slot's system
    int t1[KR_SLOTS];
    int owner[KR_SLOTS];         // 1 if this slot holds the first tile of its system
    int ncell[KR_SLOTS];         // cells of the slot's system
};

__device__ void load_slots(const pict_domain_t& dom, TileSlots& S) {
    const int nt = dom.num_tiles;
    if (threadIdx.x == 0) S.n = (int)blockIdx.x < nt ? (nt - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
    __syncthreads();
    if ((int)threadIdx.x < S.n) {
        const int j = threadIdx.x;
        const int t = blockIdx.x + j * gridDim.x;
        const int* tt = dom.tiles + 4 * t;
        S.tile[j] = t;
        S.sim[j] = tt[0];
        S.block[j] = tt[1];
        S.start[j] = tt[2];
        S.count[j] = tt[3];
        S.t0[j] = dom.sim_tiles[tt[0]];
        S.t1[j] = dom.sim_tiles[tt[0] + 1];
        S.owner[j] = (t == S.t0[j]);
        S.ncell[j] = dom.sim_cells[tt[0] + 1] - dom.sim_cells[tt[0]];
    }
    __syncthreads();
}

// Sum the tile partials of each slot's system (one warp per slot, fixed order) into out[slot][k].
// Only slots whose bit is set in `mask` are reduced.
template <int NV, unsigned MAXMASK = 0u>
__device__ void system_sums(const double* partials, const TileSlots& S, unsigned mask, double (*out)[KR_NV]) {
    const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int j = threadIdx.x >> 5; j < S.n; j += nwarps) {
        if (!(mask & (1u << j))) continue;
        double acc[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] = 0.0;
        for (int t = S.t0[j] + lane; t < S.t1[j]; t += 32) {
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const double v = __ldcg(partials + (size_t)t * KR_NV + k);
                acc[k] = ((MAXMASK >> k) & 1u) ? fmax(acc[k], v) : acc[k] + v;
            }
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const double s = ((MAXMASK >> k) & 1u) ? warp_max(acc[k]) : warp_sum(acc[k]);
            if (lane == 0) out[j][k] = s;
        }
    }
    __syncthreads();
}

// Sum the warp partials of the slots in `mask` and write the tile partials (fixed order).
template <int NV, unsigned MAXMASK = 0u>
__device__ __forceinline__ void flush_partials(PhaseRed& R, const TileSlots& S, unsigned mask, double* partials) {
    __syncthreads();
    const int nwarps = blockDim.x >> 5;
    const int j = threadIdx.x / NV, k = threadIdx.x % NV;
    if (j < S.n && ((mask >> j) & 1u)) {
        double s = 0.0;
        for (int w = 0; w < nwarps; ++w) s = ((MAXMASK >> k) & 1u) ? fmax(s, R.v[j][w][k]) : s + R.v[j][w][k];
        partials[(size_t)S.tile[j] * KR_NV + k] = s;
    }
}

// One stencil row applied to a vector given by `load(j)`; TRANS applies the transposed matrix
// (the coefficient of row j pointing back to i).  Branch-free gathers: inside a block the neighbour is
// i +- stride, on a block face it comes from the neighbour table; where there is none (-1) the cell
// itself is loaded and the term is masked, so all loads of a row (and of the rows a thread handles in
// one pass) are unconditional and can be in flight together.
template <typename T, int D, bool TRANS, typename F>
__device__ __forceinline__ T spmv_row(const pict_domain_t& dom, const T* __restrict__ coef, int N, int i,
                                      const pict_block_t& B, const int* p, F load) {
    T acc = coef[i] * load(i);
    const int stride[3] = {1, B.size[0], B.size[0] * B.size[1]};
#pragma unroll
    for (int f = 0; f < 2 * D; ++f) {
        const int a = f >> 1;
        const bool up = f & 1;
        const bool at = up ? (p[a] == B.size[a] - 1) : (p[a] == 0);
        int j = i + (up ? stride[a] : -stride[a]);
        int back = f ^ 1;
        if (at) {
            j = dom.nbr[(size_t)f * N + i];
            if (B.face[f].type == PICT_FACE_CONNECTED) back = B.face[f].conn_axes[0];
        }
        const bool ok = j >= 0;
        const int jj = ok ? j : i;
        const T c = TRANS ? coef[(size_t)(back + 1) * N + jj] : coef[(size_t)(f + 1) * N + i];
        const T v = load(jj);
        acc += ok ? c * v : T(0);
    }
    return acc;
}

__device__ __forceinline__ double conv_crit(double sq, int normalized, int n) {
    const double nrm = sqrt(sq);
    return normalized ? nrm / sqrt((double)n) : nrm;
}

// ComputeConvergenceCriterion (extensions/cg_solver_kernel.cu:77-110): abs = sum |r| (ABS_SUM, ABS_MEAN) or
// max |r| (ABS_MAX); sq = r.r for the NORM2 criteria.
__device__ __forceinline__ double conv_crit_any(double sq, double abs, int abs_crit, int normalized, int n) {
    if (abs_crit == PICT_CONV_ABS_MEAN) return abs / (double)n;
    if (abs_crit == PICT_CONV_ABS_SUM || abs_crit == PICT_CONV_ABS_MAX) return abs;
    return conv_crit(sq, normalized, n);
}

// One residual entry into the criterion partial: v^2 (NORM2 criteria), |v| (ABS_SUM / ABS_MEAN) or max |v| (ABS_MAX).
__device__ __forceinline__ void crit_acc(double& acc, double v, int abs_crit) {
    if (abs_crit == PICT_CONV_ABS_MAX) acc = fmax(acc, fabs(v));
    else if (abs_crit) acc += fabs(v);
    else acc += v * v;
}

__device__ __forceinline__ pict_solve_info_t fresh_info() {
    pict_solve_info_t inf;
    inf.final_residual = 0.0;
    inf.used_iterations = -1;
    inf.converged = 0;
    inf.finite = 1;
    inf.status = 0;
    return inf;
}

// ---------------------------------------------------------------------------------------------
// CG (extensions/cg_solver_kernel.cu:236-427)
// ---------------------------------------------------------------------------------------------
template <typename T, int D, bool TRANS>
__global__ void __launch_bounds__(KR_THREADS, 2) k_cg(KArgs<T> a) {
    const pict_domain_t& dom = a.dom;
    const int N = dom.num_cells;
    __shared__ TileSlots S;
    __shared__ PhaseRed R;
    __shared__ double s_sum[KR_SLOTS][KR_NV];
    __shared__ double s_rho[KR_SLOTS], s_beta[KR_SLOTS], s_alpha[KR_SLOTS];
    __shared__ unsigned s_active;  // bit per slot
    __shared__ pict_solve_info_t s_info[KR_SLOTS];
    __shared__ double s_best[KR_SLOTS], s_last[KR_SLOTS];
    __shared__ int s_best_it[KR_SLOTS], s_rising[KR_SLOTS];
    __shared__ unsigned s_save, s_restore;
    __shared__ double s_rds[KR_SLOTS], s_rdc[KR_SLOTS];  // rank-deficient scale s and constant s |v|_1
    load_slots(dom, S);
    __shared__ int s_ctrl[3];
    unsigned epoch = 0;
    const T* __restrict__ coef = a.coef;
    const T* __restrict__ bv = a.b;
    T* __restrict__ x = a.x;
    T* __restrict__ r = a.r;
    T* __restrict__ q = a.t;
    T* pc = a.p0;
    T* pn = a.p1;
    int phase = 0;
    double* part = a.partials;
    const size_t pstride = (size_t)dom.num_tiles * KR_NV;

    // ---- matrixRankDeficient (extensions/cg_solver_kernel.cu:240-253): s = sum |diag| / n^3 per system and
    // the constant s |x|_1 that the reference adds to b - A x
    if (a.rankdef) {
        for (int j = 0; j < S.n; ++j) {
            double acc[2] = {0.0, 0.0};
            for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
                acc[0] += fabs((double)coef[i]);
                if (!a.x_zero) acc[1] += fabs((double)x[i]);
            }
            warp_partial<2>(R, j, acc);
        }
        flush_partials<2>(R, S, 0xffffffffu, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        system_sums<2>(part + phase * pstride, S, 0xffffffffu, s_sum);
        phase ^= 1;
        if ((int)threadIdx.x < S.n) {
            const double n = (double)S.ncell[threadIdx.x];
            s_rds[threadIdx.x] = s_sum[threadIdx.x][0] / n / n / n;
            s_rdc[threadIdx.x] = s_rds[threadIdx.x] * s_sum[threadIdx.x][1];
        }
        __syncthreads();
    }
    // ---- initial residual r = b - A x, |r|^2, |b|^2 per tile
    for (int j = 0; j < S.n; ++j) {
        const pict_block_t& B = dom.blocks[S.block[j]];
        double acc[2] = {0.0, 0.0};
        const int s0 = S.start[j], s1 = s0 + S.count[j];
        const T rdc = a.rankdef ? (T)s_rdc[j] : T(0);
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            int p[3];
            unflatten(i - B.offset, B.size, p);
            const T bi = bv[i];
            T ri = bi;
            if (!a.x_zero) ri -= spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int jj) { return x[jj]; });
            if (a.rankdef) ri += rdc;
            r[i] = ri;
            pc[i] = T(0);
            acc[0] += (double)ri * (double)ri;
            acc[1] += (double)bi * (double)bi;
        }
        warp_partial<2>(R, j, acc);
    }
    flush_partials<2>(R, S, 0xffffffffu, part + phase * pstride);
    if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
    system_sums<2>(part + phase * pstride, S, 0xffffffffu, s_sum);
    phase ^= 1;
    if (threadIdx.x < 32) {  // lane j: slot j
        const int j = threadIdx.x;
        bool act = false;
        if (j < S.n) {
            pict_solve_info_t inf = fresh_info();
            s_rho[j] = s_sum[j][0];
            s_beta[j] = 0.0;
            if (s_sum[j][1] == 0.0) {
                inf.converged = 1;
                inf.used_iterations = 0;
                if (S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE, 1);
            } else {
                act = true;
            }
            s_info[j] = inf;
        }
        const unsigned m = __ballot_sync(0xffffffffu, act);
        if (j == 0) s_active = m;
    }
    __syncthreads();
    // x = 0 where the iteration starts from zero or the right-hand side vanishes
    for (int j = 0; j < S.n; ++j) {
        if (!a.x_zero && ((s_active >> j) & 1u)) continue;
        for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) x[i] = T(0);
    }

    for (int it = 0; it < a.maxit; ++it) {
        // restart (residualResetSteps, extensions/cg_solver_kernel.cu:266-286): r = b - A x, p = r, rho = r.r
        if (a.reset > 0 && (it + 1) % a.reset == 0) {
            if (a.rankdef) {  // s |x|_1 for the restarted residual
                for (int j = 0; j < S.n; ++j) {
                    if (!((s_active >> j) & 1u)) continue;
                    double acc[1] = {0.0};
                    for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x)
                        acc[0] += fabs((double)x[i]);
                    warp_partial<1>(R, j, acc);
                }
                flush_partials<1>(R, S, s_active, part + phase * pstride);
                if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
                system_sums<1>(part + phase * pstride, S, s_active, s_sum);
                phase ^= 1;
                if ((int)threadIdx.x < S.n) s_rdc[threadIdx.x] = s_rds[threadIdx.x] * s_sum[threadIdx.x][0];
                __syncthreads();
            }
            for (int j = 0; j < S.n; ++j) {
                if (!((s_active >> j) & 1u)) continue;
                const pict_block_t& B = dom.blocks[S.block[j]];
                double acc[1] = {0.0};
                const T rdc = a.rankdef ? (T)s_rdc[j] : T(0);
                for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
                    int p[3];
                    unflatten(i - B.offset, B.size, p);
                    const T ri = bv[i] - spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int jj) { return x[jj]; }) + rdc;
                    r[i] = ri;
                    acc[0] += (double)ri * (double)ri;
                }
                warp_partial<1>(R, j, acc);
            }
            flush_partials<1>(R, S, s_active, part + phase * pstride);
            if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
            system_sums<1>(part + phase * pstride, S, s_active, s_sum);
            phase ^= 1;
            if ((int)threadIdx.x < S.n && ((s_active >> threadIdx.x) & 1u)) {
                s_rho[threadIdx.x] = s_sum[threadIdx.x][0];
                s_beta[threadIdx.x] = 0.0;
            }
            __syncthreads();
        }
        // phase 1: p <- r + beta p (on the fly for neighbours), q = A p, p.q
        for (int j = 0; j < S.n; ++j) {
            if (!((s_active >> j) & 1u)) continue;
            const pict_block_t& B = dom.blocks[S.block[j]];
            const T bt = (T)s_beta[j];
            double acc[3] = {0.0, 0.0, 0.0};
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T pi[KR_U], qi[KR_U];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                    const int i = s0 + l;
                    int p[3];
                    unflatten(i - B.offset, B.size, p);
                    pi[k] = r[i] + bt * pc[i];
                    qi[k] = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int jj) { return r[jj] + bt * pc[jj]; });
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l < cnt) {
                        pn[s0 + l] = pi[k];
                        q[s0 + l] = qi[k];
                        acc[0] += (double)pi[k] * (double)qi[k];
                        if (a.rankdef) {
                            acc[1] += fabs((double)pi[k]);
                            acc[2] += (double)pi[k];
                        }
                    }
                }
            }
            if (a.rankdef) warp_partial<3>(R, j, acc);
            else warp_partial<1>(R, j, reinterpret_cast<const double(&)[1]>(acc));
        }
        if (a.rankdef) flush_partials<3>(R, S, s_active, part + phase * pstride);
        else flush_partials<1>(R, S, s_active, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        if (s_ctrl[0] == dom.num_sims) break;
        if (a.rankdef) system_sums<3>(part + phase * pstride, S, s_active, s_sum);
        else system_sums<1>(part + phase * pstride, S, s_active, s_sum);
        phase ^= 1;
        if ((int)threadIdx.x < S.n && ((s_active >> threadIdx.x) & 1u)) {
            const int j = threadIdx.x;
            double pq = s_sum[j][0];
            if (a.rankdef) {  // q = A p + s |p|_1 e (extensions/cg_solver_kernel.cu:293-298): p.q gains s |p|_1 sum(p)
                s_rdc[j] = s_rds[j] * s_sum[j][1];
                pq += s_rdc[j] * s_sum[j][2];
            }
            s_alpha[j] = s_rho[j] / pq;
        }
        __syncthreads();
        // phase 2: x += alpha p, r -= alpha q, r.r
        for (int j = 0; j < S.n; ++j) {
            if (!((s_active >> j) & 1u)) continue;
            const T al = (T)s_alpha[j];
            const T rdc = a.rankdef ? (T)s_rdc[j] : T(0);
            double acc[2] = {0.0, 0.0};
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T xi[KR_U], ri[KR_U];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                    xi[k] = x[i] + al * pn[i];
                    ri[k] = a.rankdef ? r[i] - al * (q[i] + rdc) : r[i] - al * q[i];
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l < cnt) {
                        x[s0 + l] = xi[k];
                        r[s0 + l] = ri[k];
                        acc[0] += (double)ri[k] * (double)ri[k];
                        if (a.abs_crit) {
                            const double v = fabs((double)ri[k]);
                            acc[1] = a.abs_crit == PICT_CONV_ABS_MAX ? fmax(acc[1], v) : acc[1] + v;
                        }
                    }
                }
            }
            if (a.abs_crit == PICT_CONV_ABS_MAX) warp_partial<2, 2u>(R, j, acc);
            else if (a.abs_crit) warp_partial<2>(R, j, acc);
            else warp_partial<1>(R, j, reinterpret_cast<const double(&)[1]>(acc));
        }
        if (a.abs_crit == PICT_CONV_ABS_MAX) flush_partials<2, 2u>(R, S, s_active, part + phase * pstride);
        else if (a.abs_crit) flush_partials<2>(R, S, s_active, part + phase * pstride);
        else flush_partials<1>(R, S, s_active, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        if (a.abs_crit == PICT_CONV_ABS_MAX) system_sums<2, 2u>(part + phase * pstride, S, s_active, s_sum);
        else if (a.abs_crit) system_sums<2>(part + phase * pstride, S, s_active, s_sum);
        else system_sums<1>(part + phase * pstride, S, s_active, s_sum);
        phase ^= 1;
        if (threadIdx.x < 32) {
            const int j = threadIdx.x;
            bool act = j < S.n && ((s_active >> j) & 1u);
            bool save = false, restore = false;
            if (act) {
                const double rr = s_sum[j][0];
                const double crit = conv_crit_any(rr, s_sum[j][1], a.abs_crit, a.normalized, S.ncell[j]);
                s_info[j].used_iterations = it;
                s_info[j].final_residual = crit;
                bool fin = false;
                if (!isfinite(crit)) { s_info[j].finite = 0; fin = true; }
                else {
                    if (a.best) {  // extensions/cg_solver_kernel.cu:330-346
                        if (it == 0 || crit < s_best[j]) {
                            s_best[j] = crit;
                            s_best_it[j] = it;
                            save = true;
                        }
                        s_rising[j] = (it > 0 && crit >= s_last[j]) ? s_rising[j] + 1 : 0;
                        s_last[j] = crit;
                    }
                    if (crit < a.tol) { s_info[j].converged = 1; fin = true; }
                    else if (a.best && (it == a.maxit - 1 || s_rising[j] >= 100)) {  // :399-413
                        restore = true;
                        s_info[j].used_iterations = s_best_it[j];
                        s_info[j].final_residual = s_best[j];
                        fin = true;
                    } else {
                        s_beta[j] = rr / s_rho[j];
                        s_rho[j] = rr;
                    }
                }
                if (fin) {
                    act = false;
                    if (S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE, 1);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, act);
            const unsigned ms = __ballot_sync(0xffffffffu, save);
            const unsigned mr = __ballot_sync(0xffffffffu, restore);
            if (j == 0) {
                s_active = m;
                s_save = ms;
                s_restore = mr;
            }
        }
        __syncthreads();
        if (a.best && (s_save | s_restore)) {
            // this CTA's tiles of the system: keep x as the best iterate / put the best iterate back
            for (int j = 0; j < S.n; ++j) {
                const bool sv = (s_save >> j) & 1u, rs = (s_restore >> j) & 1u;
                if (!sv && !rs) continue;
                for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
                    if (sv) a.xbest[i] = x[i];
                    if (rs) x[i] = a.xbest[i];
                }
            }
        }
        T* tmp = pc; pc = pn; pn = tmp;
    }
    // ---- mean removal (PISOtorch_simulation.py:1243-1244) and copy into the blocks' pressure
    if (a.sub_mean || a.write_bp) {
        if (a.sub_mean) {
            for (int j = 0; j < S.n; ++j) {
                double acc[1] = {0.0};
                for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) acc[0] += (double)x[i];
                warp_partial<1>(R, j, acc);
            }
            flush_partials<1>(R, S, 0xffffffffu, part + phase * pstride);
            if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
            system_sums<1>(part + phase * pstride, S, 0xffffffffu, s_sum);
            phase ^= 1;
        }
        for (int j = 0; j < S.n; ++j) {
            const pict_block_t& B = dom.blocks[S.block[j]];
            const int n = S.ncell[j];
            const T mean = a.sub_mean ? (T)(s_sum[j][0] / (double)n) : T(0);
            T* pb = reinterpret_cast<T*>(B.pressure);
            for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
                const T v = x[i] - mean;
                x[i] = v;
                if (a.write_bp) pb[i - B.offset] = v;
            }
        }
    }
    if ((int)threadIdx.x < S.n && S.owner[threadIdx.x]) a.info[S.sim[threadIdx.x]] = s_info[threadIdx.x];
}

// ---------------------------------------------------------------------------------------------
// CG, single-reduction recurrence (Chronopoulos & Gear 1989): with w = A r, s = A p,
//   p_i = r_i + b_i p_{i-1},  s_i = w_i + b_i s_{i-1},  x += a_i p_i,  r_{i+1} = r_i - a_i s_i,
//   w_{i+1} = A r_{i+1},  g_{i+1} = (r_{i+1}, r_{i+1}),  d_{i+1} = (w_{i+1}, r_{i+1}),
//   b_{i+1} = g_{i+1} / g_i,  a_{i+1} = g_{i+1} / (d_{i+1} - b_{i+1} g_{i+1} / a_i).
// The same iterates as classic CG in exact arithmetic; one fused sweep (r_{i+1} of the neighbours
// formed on the fly) and one grid-wide reduction per iteration.  Stopping rule and reported
// iteration counts as extensions/cg_solver_kernel.cu:303-397.
// ---------------------------------------------------------------------------------------------
template <typename T, int D, bool TRANS>
__global__ void __launch_bounds__(KR_THREADS, 2) k_cg1(KArgs<T> a) {
    const pict_domain_t& dom = a.dom;
    const int N = dom.num_cells;
    __shared__ TileSlots S;
    __shared__ PhaseRed R;
    __shared__ double s_sum[KR_SLOTS][KR_NV];
    __shared__ double s_g[KR_SLOTS], s_alpha[KR_SLOTS], s_beta[KR_SLOTS];
    __shared__ unsigned s_active;
    __shared__ pict_solve_info_t s_info[KR_SLOTS];
    load_slots(dom, S);
    __shared__ int s_ctrl[3];
    unsigned epoch = 0;
    const T* __restrict__ coef = a.coef;
    const T* __restrict__ bv = a.b;
    T* __restrict__ x = a.x;
    T* __restrict__ p = a.t;
    T* rc = a.r;   // r_i
    T* rn = a.rw;  // r_{i+1}
    T* wc = a.p0;
    T* wn = a.p1;
    T* sc = a.v0;
    T* sn = a.v1;
    int phase = 0;
    double* part = a.partials;
    const size_t pstride = (size_t)dom.num_tiles * KR_NV;

    // ---- init: r0 = b - A x0 (when x0 != 0: extra sweep), w0 = A r0, g0, d0, |b|^2
    if (!a.x_zero) {
        for (int j = 0; j < S.n; ++j) {
            const pict_block_t& B = dom.blocks[S.block[j]];
            for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
                int q[3];
                unflatten(i - B.offset, B.size, q);
                rc[i] = bv[i] - spmv_row<T, D, TRANS>(dom, coef, N, i, B, q, [&](int jj) { return x[jj]; });
            }
        }
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
    }
    const T* r0 = a.x_zero ? bv : rc;
    for (int j = 0; j < S.n; ++j) {
        const pict_block_t& B = dom.blocks[S.block[j]];
        double acc[3] = {0.0, 0.0, 0.0};
        for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
            int q[3];
            unflatten(i - B.offset, B.size, q);
            const T ri = r0[i];
            const T wi = spmv_row<T, D, TRANS>(dom, coef, N, i, B, q, [&](int jj) { return r0[jj]; });
            if (a.x_zero) { rc[i] = ri; x[i] = T(0); }
            wc[i] = wi;
            sc[i] = T(0);
            p[i] = T(0);
            const T bi = bv[i];
            acc[0] += (double)ri * (double)ri;
            acc[1] += (double)wi * (double)ri;
            acc[2] += (double)bi * (double)bi;
        }
        warp_partial<3>(R, j, acc);
    }
    flush_partials<3>(R, S, 0xffffffffu, part + phase * pstride);
    if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
    system_sums<3>(part + phase * pstride, S, 0xffffffffu, s_sum);
    phase ^= 1;
    if (threadIdx.x < 32) {  // lane j: slot j
        const int j = threadIdx.x;
        bool act = false;
        if (j < S.n) {
            pict_solve_info_t inf = fresh_info();
            s_g[j] = s_sum[j][0];
            s_alpha[j] = s_sum[j][0] / s_sum[j][1];
            s_beta[j] = 0.0;
            if (s_sum[j][2] == 0.0) {
                inf.converged = 1;
                inf.used_iterations = 0;
                if (S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE_PAR + 1, 1);  // iteration -1
            } else {
                act = true;
            }
            s_info[j] = inf;
        }
        const unsigned m = __ballot_sync(0xffffffffu, act);
        if (j == 0) s_active = m;
    }
    __syncthreads();
    for (int j = 0; j < S.n; ++j) {
        if ((s_active >> j) & 1u) continue;
        for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) x[i] = T(0);
    }

    int cum[2] = {0, 0};  // completions per iteration parity, as read by this CTA
    for (int it = 0; it < a.maxit; ++it) {
        for (int j = 0; j < S.n; ++j) {
            if (!((s_active >> j) & 1u)) continue;
            const pict_block_t& B = dom.blocks[S.block[j]];
            const T al = (T)s_alpha[j], bt = (T)s_beta[j];
            double acc[2] = {0.0, 0.0};
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T rni[KR_U], wni[KR_U], pi[KR_U], si[KR_U], xi[KR_U];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                    int q[3];
                    unflatten(i - B.offset, B.size, q);
                    pi[k] = rc[i] + bt * p[i];
                    si[k] = wc[i] + bt * sc[i];
                    rni[k] = rc[i] - al * si[k];
                    xi[k] = x[i] + al * pi[k];
                    wni[k] = spmv_row<T, D, TRANS>(dom, coef, N, i, B, q,
                                                   [&](int jj) { return rc[jj] - al * (wc[jj] + bt * sc[jj]); });
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l < cnt) {
                        const int i = s0 + l;
                        x[i] = xi[k];
                        p[i] = pi[k];
                        sn[i] = si[k];
                        rn[i] = rni[k];
                        wn[i] = wni[k];
                        acc[0] += (double)rni[k] * (double)rni[k];
                        acc[1] += (double)wni[k] * (double)rni[k];
                    }
                }
            }
            warp_partial<2>(R, j, acc);
        }
        flush_partials<2>(R, S, s_active, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        // completions of iteration it-1 are complete and stable here (see CTRL_DONE_PAR)
        cum[(it - 1) & 1] = s_ctrl[1 + ((it - 1) & 1)];
        if (cum[0] + cum[1] == dom.num_sims) break;
        system_sums<2>(part + phase * pstride, S, s_active, s_sum);
        phase ^= 1;
        if (threadIdx.x < 32) {
            const int j = threadIdx.x;
            bool act = j < S.n && ((s_active >> j) & 1u);
            if (act) {
                const double g = s_sum[j][0], d = s_sum[j][1];
                const double crit = conv_crit(g, a.normalized, S.ncell[j]);
                s_info[j].used_iterations = it;
                s_info[j].final_residual = crit;
                bool fin = false;
                if (!isfinite(crit)) { s_info[j].finite = 0; fin = true; }
                else if (crit < a.tol) { s_info[j].converged = 1; fin = true; }
                else {
                    const double bnew = g / s_g[j];
                    s_alpha[j] = g / (d - bnew * g / s_alpha[j]);
                    s_beta[j] = bnew;
                    s_g[j] = g;
                }
                if (fin) {
                    act = false;
                    if (S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE_PAR + (it & 1), 1);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, act);
            if (j == 0) s_active = m;
        }
        __syncthreads();
        T* t0 = rc; rc = rn; rn = t0;
        T* t1 = wc; wc = wn; wn = t1;
        T* t2 = sc; sc = sn; sn = t2;
    }
    if (a.sub_mean || a.write_bp) {
        if (a.sub_mean) {
            for (int j = 0; j < S.n; ++j) {
                double acc[1] = {0.0};
                for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) acc[0] += (double)x[i];
                warp_partial<1>(R, j, acc);
            }
            flush_partials<1>(R, S, 0xffffffffu, part + phase * pstride);
            if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
            system_sums<1>(part + phase * pstride, S, 0xffffffffu, s_sum);
            phase ^= 1;
        }
        for (int j = 0; j < S.n; ++j) {
            const pict_block_t& B = dom.blocks[S.block[j]];
            const int n = S.ncell[j];
            const T mean = a.sub_mean ? (T)(s_sum[j][0] / (double)n) : T(0);
            T* pb = reinterpret_cast<T*>(B.pressure);
            for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
                const T v = x[i] - mean;
                x[i] = v;
                if (a.write_bp) pb[i - B.offset] = v;
            }
        }
    }
    if ((int)threadIdx.x < S.n && S.owner[threadIdx.x]) a.info[S.sim[threadIdx.x]] = s_info[threadIdx.x];
}

// ---------------------------------------------------------------------------------------------
// BiCGStab without preconditioner (extensions/bicgstab_solver_kernel.cu:240-360), NR right-hand sides sharing the matrix
// ---------------------------------------------------------------------------------------------
template <typename T, int D, int NR, bool TRANS>
__global__ void __launch_bounds__(KR_THREADS, 2) k_bicgstab(KArgs<T> a) {
    const pict_domain_t& dom = a.dom;
    const int N = dom.num_cells;
    const size_t NS = (size_t)N;
    __shared__ TileSlots S;
    __shared__ PhaseRed R;
    __shared__ double s_sum[KR_SLOTS][KR_NV];
    __shared__ double s_rho[KR_SLOTS][NR], s_alpha[KR_SLOTS][NR], s_omega[KR_SLOTS][NR], s_beta[KR_SLOTS][NR],
        s_rwr[KR_SLOTS][NR];
    __shared__ unsigned s_act[KR_SLOTS];  // bit per component
    __shared__ unsigned s_any;            // bit per slot with an active component
    __shared__ pict_solve_info_t s_info[KR_SLOTS][NR];
    load_slots(dom, S);
    __shared__ int s_ctrl[3];
    unsigned epoch = 0;
    const T* __restrict__ coef = a.coef;
    T* __restrict__ x = a.x;
    T* __restrict__ r = a.r;
    const T* __restrict__ rw = a.rw;
    T* __restrict__ tv = a.t;
    T* pc = a.p0;
    T* pn = a.p1;
    T* vc = a.v0;
    T* vn = a.v1;
    int phase = 0;
    double* part = a.partials;
    const size_t pstride = (size_t)dom.num_tiles * KR_NV;
    const int total = dom.num_sims * NR;

    // ---- init: r = b - A x, rw = r, p = v = 0
    for (int j = 0; j < S.n; ++j) {
        const pict_block_t& B = dom.blocks[S.block[j]];
        double acc[3 * NR];  // r.r, b.b, and the ABS criterion partial of r
#pragma unroll
        for (int k = 0; k < 3 * NR; ++k) acc[k] = 0.0;
        for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
            int p[3];
            unflatten(i - B.offset, B.size, p);
#pragma unroll
            for (int c = 0; c < NR; ++c) {
                const T* xc = x + c * NS;
                const T bi = a.b[c * NS + i];
                T ri = bi;
                if (!a.x_zero) ri -= spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int jj) { return xc[jj]; });
                r[c * NS + i] = ri;
                a.rw[c * NS + i] = ri;
                pc[c * NS + i] = T(0);
                vc[c * NS + i] = T(0);
                acc[c] += (double)ri * (double)ri;
                acc[NR + c] += (double)bi * (double)bi;
                if (a.abs_crit) crit_acc(acc[2 * NR + c], (double)ri, a.abs_crit);
            }
        }
        // the ABS criteria take a third group of partials; the host launches them with NR <= 2 (3 NR <= KR_NV)
        constexpr unsigned kAbsMax = ((1u << NR) - 1u) << (2 * NR);
        const double(&acc2)[2 * NR] = reinterpret_cast<const double(&)[2 * NR]>(acc);
        if constexpr (3 * NR <= KR_NV) {
            if (a.abs_crit == PICT_CONV_ABS_MAX) warp_partial<3 * NR, kAbsMax>(R, j, acc);
            else if (a.abs_crit) warp_partial<3 * NR>(R, j, acc);
            else warp_partial<2 * NR>(R, j, acc2);
        } else {
            warp_partial<2 * NR>(R, j, acc2);
        }
    }
    if constexpr (3 * NR <= KR_NV) {
        if (a.abs_crit == PICT_CONV_ABS_MAX) flush_partials<3 * NR, ((1u << NR) - 1u) << (2 * NR)>(R, S, 0xffffffffu, part + phase * pstride);
        else if (a.abs_crit) flush_partials<3 * NR>(R, S, 0xffffffffu, part + phase * pstride);
        else flush_partials<2 * NR>(R, S, 0xffffffffu, part + phase * pstride);
    } else {
        flush_partials<2 * NR>(R, S, 0xffffffffu, part + phase * pstride);
    }
    if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
    if constexpr (3 * NR <= KR_NV) {
        if (a.abs_crit == PICT_CONV_ABS_MAX) system_sums<3 * NR, ((1u << NR) - 1u) << (2 * NR)>(part + phase * pstride, S, 0xffffffffu, s_sum);
        else if (a.abs_crit) system_sums<3 * NR>(part + phase * pstride, S, 0xffffffffu, s_sum);
        else system_sums<2 * NR>(part + phase * pstride, S, 0xffffffffu, s_sum);
    } else {
        system_sums<2 * NR>(part + phase * pstride, S, 0xffffffffu, s_sum);
    }
    phase ^= 1;
    if (threadIdx.x < 32) {  // lane j: slot j
        const int j = threadIdx.x;
        unsigned act = 0;
        if (j < S.n) {
            const int n = S.ncell[j];
            for (int c = 0; c < NR; ++c) {
                pict_solve_info_t inf = fresh_info();
                s_rho[j][c] = 0.0; s_alpha[j][c] = 0.0; s_omega[j][c] = 0.0; s_beta[j][c] = 0.0;
                s_rwr[j][c] = s_sum[j][c];
                bool fin = false;
                if (s_sum[j][NR + c] == 0.0) {
                    inf.converged = 1;
                    inf.used_iterations = 0;
                    fin = true;
                } else {
                    const double nrmr0 = conv_crit_any(s_sum[j][c], a.abs_crit ? s_sum[j][2 * NR + c] : 0.0, a.abs_crit,
                                                       a.normalized, n);
                    if (nrmr0 < a.tol) {
                        inf.converged = 1;
                        inf.used_iterations = -1;
                        inf.final_residual = nrmr0;
                        fin = true;
                    } else {
                        act |= 1u << c;
                    }
                }
                if (fin && S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE, 1);
                s_info[j][c] = inf;
            }
            s_act[j] = act;
        }
        const unsigned m = __ballot_sync(0xffffffffu, act != 0);
        if (j == 0) s_any = m;
    }
    __syncthreads();
    // x = 0 where the iteration starts from zero or the right-hand side vanishes
    for (int j = 0; j < S.n; ++j) {
        for (int c = 0; c < NR; ++c) {
            const bool zero_rhs = s_info[j][c].converged && s_info[j][c].used_iterations == 0;
            if (a.x_zero || zero_rhs)
                for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) x[c * NS + i] = T(0);
        }
    }

    for (int it = 0; it < a.maxit; ++it) {
        if ((int)threadIdx.x < S.n) {
            const int j = threadIdx.x;
            for (int c = 0; c < NR; ++c) {
                if (!((s_act[j] >> c) & 1u)) continue;
                const double rhop = s_rho[j][c];
                s_rho[j][c] = s_rwr[j][c];
                s_beta[j][c] = it > 0 ? (s_rho[j][c] / rhop) * (s_alpha[j][c] / s_omega[j][c]) : 0.0;
            }
        }
        __syncthreads();
        // phase A: p = r + beta (p - omega v) on the fly, v = A p, rw.v
        for (int j = 0; j < S.n; ++j) {
            if (!((s_any >> j) & 1u)) continue;
            const unsigned act = s_act[j];
            const pict_block_t& B = dom.blocks[S.block[j]];
            double acc[NR];
#pragma unroll
            for (int c = 0; c < NR; ++c) acc[c] = 0.0;
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T pv[KR_U][NR], vv[KR_U][NR], wv[KR_U][NR];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                    int p[3];
                    unflatten(i - B.offset, B.size, p);
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        pv[k][c] = vv[k][c] = wv[k][c] = T(0);
                        if (!((act >> c) & 1u)) continue;
                        const T bt = (T)s_beta[j][c], om = (T)s_omega[j][c];
                        const T* rc = r + c * NS;
                        const T* pcc = pc + c * NS;
                        const T* vcc = vc + c * NS;
                        pv[k][c] = rc[i] + bt * (pcc[i] - om * vcc[i]);
                        vv[k][c] = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p,
                                                         [&](int jj) { return rc[jj] + bt * (pcc[jj] - om * vcc[jj]); });
                        wv[k][c] = rw[c * NS + i];
                    }
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l >= cnt) continue;
                    const int i = s0 + l;
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        if (!((act >> c) & 1u)) continue;
                        pn[c * NS + i] = pv[k][c];
                        vn[c * NS + i] = vv[k][c];
                        acc[c] += (double)wv[k][c] * (double)vv[k][c];
                    }
                }
            }
            warp_partial<NR>(R, j, acc);
        }
        flush_partials<NR>(R, S, s_any, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        if (s_ctrl[0] == total) break;
        system_sums<NR>(part + phase * pstride, S, s_any, s_sum);
        phase ^= 1;
        if ((int)threadIdx.x < S.n) {
            const int j = threadIdx.x;
            for (int c = 0; c < NR; ++c)
                if ((s_act[j] >> c) & 1u) s_alpha[j][c] = s_rho[j][c] / s_sum[j][c];
        }
        __syncthreads();
        // phase B: s = r - alpha v (in r), x += alpha p, |s|^2
        for (int j = 0; j < S.n; ++j) {
            if (!((s_any >> j) & 1u)) continue;
            const unsigned act = s_act[j];
            double acc[NR];
#pragma unroll
            for (int c = 0; c < NR; ++c) acc[c] = 0.0;
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T sv[KR_U][NR], xv[KR_U][NR];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        sv[k][c] = xv[k][c] = T(0);
                        if (!((act >> c) & 1u)) continue;
                        const T al = (T)s_alpha[j][c];
                        sv[k][c] = r[c * NS + i] - al * vn[c * NS + i];
                        xv[k][c] = x[c * NS + i] + al * pn[c * NS + i];
                    }
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l >= cnt) continue;
                    const int i = s0 + l;
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        if (!((act >> c) & 1u)) continue;
                        r[c * NS + i] = sv[k][c];
                        x[c * NS + i] = xv[k][c];
                        crit_acc(acc[c], (double)sv[k][c], a.abs_crit);
                    }
                }
            }
            if (a.abs_crit == PICT_CONV_ABS_MAX) warp_partial<NR, (1u << NR) - 1u>(R, j, acc);
            else warp_partial<NR>(R, j, acc);
        }
        if (a.abs_crit == PICT_CONV_ABS_MAX) flush_partials<NR, (1u << NR) - 1u>(R, S, s_any, part + phase * pstride);
        else flush_partials<NR>(R, S, s_any, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        if (a.abs_crit == PICT_CONV_ABS_MAX) system_sums<NR, (1u << NR) - 1u>(part + phase * pstride, S, s_any, s_sum);
        else system_sums<NR>(part + phase * pstride, S, s_any, s_sum);
        phase ^= 1;
        if (threadIdx.x < 32) {
            const int j = threadIdx.x;
            unsigned act = j < S.n ? s_act[j] : 0u;
            if (act) {
                const int n = S.ncell[j];
                for (int c = 0; c < NR; ++c) {
                    if (!((act >> c) & 1u)) continue;
                    const double nr = conv_crit_any(s_sum[j][c], s_sum[j][c], a.abs_crit, a.normalized, n);
                    s_info[j][c].used_iterations = it;
                    s_info[j][c].final_residual = nr;
                    bool fin = false;
                    if (!isfinite(nr)) { s_info[j][c].finite = 0; fin = true; }
                    else if (nr < a.tol) { s_info[j][c].converged = 1; fin = true; }
                    if (fin) {
                        act &= ~(1u << c);
                        if (S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE, 1);
                    }
                }
                s_act[j] = act;
            }
            const unsigned m = __ballot_sync(0xffffffffu, act != 0);
            if (j == 0) s_any = m;
        }
        __syncthreads();
        // phase C: t = A s, t.s, t.t
        for (int j = 0; j < S.n; ++j) {
            if (!((s_any >> j) & 1u)) continue;
            const unsigned act = s_act[j];
            const pict_block_t& B = dom.blocks[S.block[j]];
            double acc[2 * NR];
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) acc[k] = 0.0;
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T tv2[KR_U][NR], sv[KR_U][NR];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                    int p[3];
                    unflatten(i - B.offset, B.size, p);
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        tv2[k][c] = sv[k][c] = T(0);
                        if (!((act >> c) & 1u)) continue;
                        const T* scc = r + c * NS;
                        tv2[k][c] = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int jj) { return scc[jj]; });
                        sv[k][c] = scc[i];
                    }
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l >= cnt) continue;
                    const int i = s0 + l;
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        if (!((act >> c) & 1u)) continue;
                        tv[c * NS + i] = tv2[k][c];
                        acc[2 * c] += (double)tv2[k][c] * (double)sv[k][c];
                        acc[2 * c + 1] += (double)tv2[k][c] * (double)tv2[k][c];
                    }
                }
            }
            warp_partial<2 * NR>(R, j, acc);
        }
        flush_partials<2 * NR>(R, S, s_any, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        system_sums<2 * NR>(part + phase * pstride, S, s_any, s_sum);
        phase ^= 1;
        if ((int)threadIdx.x < S.n) {
            const int j = threadIdx.x;
            for (int c = 0; c < NR; ++c)
                if ((s_act[j] >> c) & 1u) s_omega[j][c] = s_sum[j][2 * c] / s_sum[j][2 * c + 1];
        }
        __syncthreads();
        // phase D: x += omega s, r = s - omega t, r.r, rw.r
        for (int j = 0; j < S.n; ++j) {
            if (!((s_any >> j) & 1u)) continue;
            const unsigned act = s_act[j];
            double acc[2 * NR];
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) acc[k] = 0.0;
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T xv[KR_U][NR], rv[KR_U][NR], wv[KR_U][NR];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        xv[k][c] = rv[k][c] = wv[k][c] = T(0);
                        if (!((act >> c) & 1u)) continue;
                        const T om = (T)s_omega[j][c];
                        const T si = r[c * NS + i];
                        xv[k][c] = x[c * NS + i] + om * si;
                        rv[k][c] = si - om * tv[c * NS + i];
                        wv[k][c] = rw[c * NS + i];
                    }
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l >= cnt) continue;
                    const int i = s0 + l;
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        if (!((act >> c) & 1u)) continue;
                        x[c * NS + i] = xv[k][c];
                        r[c * NS + i] = rv[k][c];
                        crit_acc(acc[2 * c], (double)rv[k][c], a.abs_crit);
                        acc[2 * c + 1] += (double)wv[k][c] * (double)rv[k][c];
                    }
                }
            }
            if (a.abs_crit == PICT_CONV_ABS_MAX) warp_partial<2 * NR, 0x15u>(R, j, acc);
            else warp_partial<2 * NR>(R, j, acc);
        }
        if (a.abs_crit == PICT_CONV_ABS_MAX) flush_partials<2 * NR, 0x15u>(R, S, s_any, part + phase * pstride);
        else flush_partials<2 * NR>(R, S, s_any, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        if (a.abs_crit == PICT_CONV_ABS_MAX) system_sums<2 * NR, 0x15u>(part + phase * pstride, S, s_any, s_sum);
        else system_sums<2 * NR>(part + phase * pstride, S, s_any, s_sum);
        phase ^= 1;
        if (threadIdx.x < 32) {
            const int j = threadIdx.x;
            unsigned act = j < S.n ? s_act[j] : 0u;
            if (act) {
                const int n = S.ncell[j];
                for (int c = 0; c < NR; ++c) {
                    if (!((act >> c) & 1u)) continue;
                    s_rwr[j][c] = s_sum[j][2 * c + 1];
                    const double nr = conv_crit_any(s_sum[j][2 * c], s_sum[j][2 * c], a.abs_crit, a.normalized, n);
                    s_info[j][c].final_residual = nr;
                    if (nr < a.tol) {
                        s_info[j][c].converged = 1;
                        s_info[j][c].used_iterations = it + 1;
                        act &= ~(1u << c);
                        if (S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE, 1);
                    }
                }
                s_act[j] = act;
            }
            const unsigned m = __ballot_sync(0xffffffffu, act != 0);
            if (j == 0) s_any = m;
        }
        __syncthreads();
        T* tp = pc; pc = pn; pn = tp;
        T* tq = vc; vc = vn; vn = tq;
    }
    if ((int)threadIdx.x < S.n && S.owner[threadIdx.x]) {
        const int j = threadIdx.x;
        for (int c = 0; c < NR; ++c) a.info[S.sim[j] * a.nrhs + c] = s_info[j][c];
    }
}

// ---------------------------------------------------------------------------------------------
// BiCGStab with two grid barriers per iteration (NORM2 criteria, up to two right-hand sides per launch).
//
// Same iterates, stopping rule and reports as k_bicgstab, in two sweeps per iteration:
//  * half step: s = r - alpha v formed on the fly (also for the neighbours), t = A s, and the inner
//    products s.s, t.s, t.t, rw.t; after the barrier the half-step convergence test on |s|, then
//    omega = t.s / t.t and rho' = rw.r' by the recurrence rw.r - alpha rw.v - omega rw.t, which gives
//    beta = (rho' / rho)(alpha / omega) before r' exists;
//  * full step merged with the next search direction: x += alpha p + omega s, r' = s - omega t (into
//    the other residual buffer: the neighbours still read r), p' = r' + beta (p - omega v) formed on the
//    fly from r, v, t and p of the neighbours, v' = A p', and the exact |r'|^2, rw.r', rw.v'.  After the
//    barrier the full-step convergence test on the exact |r'|, and the next alpha uses the exact rho'.
// The four-barrier kernel stores s and r' between its phases: per iteration and right-hand side this one
// moves 14 instead of 20 vectors (plus the two stencil passes) and waits at half the barriers.  Systems
// that converge at the full step spend the search direction of one iteration they do not take.
// Completions are counted only after the full-step barrier and read at the half-step barrier (a barrier
// separates every increment from every read, so all CTAs take the same exit).
// ---------------------------------------------------------------------------------------------
template <typename T, int D, int NR, bool TRANS, int MINB>
__global__ void __launch_bounds__(KR_THREADS, MINB) k_bicgstab2(KArgs<T> a) {
    static_assert(4 * NR <= KR_NV, "two-barrier BiCGStab: at most two right-hand sides per launch");
    const pict_domain_t& dom = a.dom;
    const int N = dom.num_cells;
    const size_t NS = (size_t)N;
    __shared__ TileSlots S;
    __shared__ PhaseRed R;
    __shared__ double s_sum[KR_SLOTS][KR_NV];
    __shared__ double s_rho[KR_SLOTS][NR], s_rwv[KR_SLOTS][NR], s_alpha[KR_SLOTS][NR], s_omega[KR_SLOTS][NR],
        s_beta[KR_SLOTS][NR];
    __shared__ unsigned s_act[KR_SLOTS];   // bit per component still iterating
    __shared__ unsigned s_half[KR_SLOTS];  // bit per component that stopped at this iteration's half step
    __shared__ unsigned s_any;             // bit per slot with an iterating or half-step component
    __shared__ pict_solve_info_t s_info[KR_SLOTS][NR];
    load_slots(dom, S);
    __shared__ int s_ctrl[3];
    unsigned epoch = 0;
    const T* __restrict__ coef = a.coef;
    T* __restrict__ x = a.x;
    const T* __restrict__ rw = a.rw;
    T* __restrict__ tv = a.t;
    T* rc = a.r;
    T* rn = a.r1;
    T* pc = a.p0;
    T* pn = a.p1;
    T* vc = a.v0;
    T* vn = a.v1;
    int phase = 0;
    double* part = a.partials;
    const size_t pstride = (size_t)dom.num_tiles * KR_NV;
    const int total = dom.num_sims * NR;

    // ---- init: r = b - A x, rw = r, p = v = 0; r.r and b.b
    for (int j = 0; j < S.n; ++j) {
        const pict_block_t& B = dom.blocks[S.block[j]];
        double acc[2 * NR];
#pragma unroll
        for (int k = 0; k < 2 * NR; ++k) acc[k] = 0.0;
        for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) {
            int p[3];
            unflatten(i - B.offset, B.size, p);
#pragma unroll
            for (int c = 0; c < NR; ++c) {
                const T* xc = x + c * NS;
                const T bi = a.b[c * NS + i];
                T ri = bi;
                if (!a.x_zero) ri -= spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int jj) { return xc[jj]; });
                rc[c * NS + i] = ri;
                a.rw[c * NS + i] = ri;
                pc[c * NS + i] = T(0);
                vc[c * NS + i] = T(0);
                acc[c] += (double)ri * (double)ri;
                acc[NR + c] += (double)bi * (double)bi;
            }
        }
        warp_partial<2 * NR>(R, j, acc);
    }
    flush_partials<2 * NR>(R, S, 0xffffffffu, part + phase * pstride);
    if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
    system_sums<2 * NR>(part + phase * pstride, S, 0xffffffffu, s_sum);
    phase ^= 1;
    if (threadIdx.x < 32) {  // lane j: slot j
        const int j = threadIdx.x;
        unsigned act = 0;
        if (j < S.n) {
            const int n = S.ncell[j];
            for (int c = 0; c < NR; ++c) {
                pict_solve_info_t inf = fresh_info();
                s_rho[j][c] = s_sum[j][c];
                s_rwv[j][c] = 0.0; s_alpha[j][c] = 0.0; s_omega[j][c] = 0.0; s_beta[j][c] = 0.0;
                bool fin = false;
                if (s_sum[j][NR + c] == 0.0) {
                    inf.converged = 1;
                    inf.used_iterations = 0;
                    fin = true;
                } else {
                    const double nrmr0 = conv_crit(s_sum[j][c], a.normalized, n);
                    if (nrmr0 < a.tol) {
                        inf.converged = 1;
                        inf.used_iterations = -1;
                        inf.final_residual = nrmr0;
                        fin = true;
                    } else {
                        act |= 1u << c;
                    }
                }
                if (fin && S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE, 1);
                s_info[j][c] = inf;
            }
            s_act[j] = act;
            s_half[j] = 0u;
        }
        const unsigned m = __ballot_sync(0xffffffffu, act != 0);
        if (j == 0) s_any = m;
    }
    __syncthreads();
    for (int j = 0; j < S.n; ++j) {
        for (int c = 0; c < NR; ++c) {
            const bool zero_rhs = s_info[j][c].converged && s_info[j][c].used_iterations == 0;
            if (a.x_zero || zero_rhs)
                for (int i = S.start[j] + threadIdx.x; i < S.start[j] + S.count[j]; i += blockDim.x) x[c * NS + i] = T(0);
        }
    }

    // ---- first search direction: p = r, v = A r, rw.v
    for (int j = 0; j < S.n; ++j) {
        if (!((s_any >> j) & 1u)) continue;
        const unsigned act = s_act[j];
        const pict_block_t& B = dom.blocks[S.block[j]];
        double acc[NR];
#pragma unroll
        for (int c = 0; c < NR; ++c) acc[c] = 0.0;
        const int s0 = S.start[j], cnt = S.count[j];
        for (int base = 0; base < cnt; base += KR_PASS) {
            T pv[KR_U][NR], vv[KR_U][NR], wv[KR_U][NR];
#pragma unroll
            for (int k = 0; k < KR_U; ++k) {
                const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                int p[3];
                unflatten(i - B.offset, B.size, p);
#pragma unroll
                for (int c = 0; c < NR; ++c) {
                    pv[k][c] = vv[k][c] = wv[k][c] = T(0);
                    if (!((act >> c) & 1u)) continue;
                    const T* rcc = rc + c * NS;
                    pv[k][c] = rcc[i];
                    vv[k][c] = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int jj) { return rcc[jj]; });
                    wv[k][c] = rw[c * NS + i];
                }
            }
#pragma unroll
            for (int k = 0; k < KR_U; ++k) {
                const int l = base + (int)threadIdx.x + k * KR_THREADS;
                if (l >= cnt) continue;
                const int i = s0 + l;
#pragma unroll
                for (int c = 0; c < NR; ++c) {
                    if (!((act >> c) & 1u)) continue;
                    pc[c * NS + i] = pv[k][c];
                    vc[c * NS + i] = vv[k][c];
                    acc[c] += (double)wv[k][c] * (double)vv[k][c];
                }
            }
        }
        warp_partial<NR>(R, j, acc);
    }
    flush_partials<NR>(R, S, s_any, part + phase * pstride);
    if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
    system_sums<NR>(part + phase * pstride, S, s_any, s_sum);
    phase ^= 1;
    if ((int)threadIdx.x < S.n) {
        const int j = threadIdx.x;
        for (int c = 0; c < NR; ++c)
            if ((s_act[j] >> c) & 1u) s_rwv[j][c] = s_sum[j][c];
    }
    __syncthreads();
    if (s_ctrl[0] == total) goto done;

    for (int it = 0; it < a.maxit; ++it) {
        if ((int)threadIdx.x < S.n) {
            const int j = threadIdx.x;
            for (int c = 0; c < NR; ++c)
                if ((s_act[j] >> c) & 1u) s_alpha[j][c] = s_rho[j][c] / s_rwv[j][c];
        }
        __syncthreads();
        // half step: s = r - alpha v on the fly, t = A s; s.s, t.s, t.t, rw.t
        for (int j = 0; j < S.n; ++j) {
            if (!((s_any >> j) & 1u)) continue;
            const unsigned act = s_act[j];
            const pict_block_t& B = dom.blocks[S.block[j]];
            double acc[4 * NR];
#pragma unroll
            for (int k = 0; k < 4 * NR; ++k) acc[k] = 0.0;
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                T sv[KR_U][NR], tt[KR_U][NR], wv[KR_U][NR];
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                    int p[3];
                    unflatten(i - B.offset, B.size, p);
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        sv[k][c] = tt[k][c] = wv[k][c] = T(0);
                        if (!((act >> c) & 1u)) continue;
                        const T al = (T)s_alpha[j][c];
                        const T* rcc = rc + c * NS;
                        const T* vcc = vc + c * NS;
                        sv[k][c] = rcc[i] - al * vcc[i];
                        tt[k][c] = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p,
                                                         [&](int jj) { return rcc[jj] - al * vcc[jj]; });
                        wv[k][c] = rw[c * NS + i];
                    }
                }
#pragma unroll
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    if (l >= cnt) continue;
                    const int i = s0 + l;
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        if (!((act >> c) & 1u)) continue;
                        tv[c * NS + i] = tt[k][c];
                        const double sd = (double)sv[k][c], td = (double)tt[k][c];
                        acc[4 * c] += sd * sd;
                        acc[4 * c + 1] += td * sd;
                        acc[4 * c + 2] += td * td;
                        acc[4 * c + 3] += (double)wv[k][c] * td;
                    }
                }
            }
            warp_partial<4 * NR>(R, j, acc);
        }
        flush_partials<4 * NR>(R, S, s_any, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        if (s_ctrl[0] == total) break;
        system_sums<4 * NR>(part + phase * pstride, S, s_any, s_sum);
        phase ^= 1;
        if (threadIdx.x < 32) {
            const int j = threadIdx.x;
            unsigned act = j < S.n ? s_act[j] : 0u;
            unsigned half = 0u;
            if (act) {
                const int n = S.ncell[j];
                for (int c = 0; c < NR; ++c) {
                    if (!((act >> c) & 1u)) continue;
                    const double ss = s_sum[j][4 * c], ts = s_sum[j][4 * c + 1], tt = s_sum[j][4 * c + 2],
                                 wt = s_sum[j][4 * c + 3];
                    const double nr = conv_crit(ss, a.normalized, n);
                    s_info[j][c].used_iterations = it;
                    s_info[j][c].final_residual = nr;
                    bool stop = false;
                    if (!isfinite(nr)) { s_info[j][c].finite = 0; stop = true; }
                    else if (nr < a.tol) { s_info[j][c].converged = 1; stop = true; }
                    if (stop) {
                        half |= 1u << c;
                        act &= ~(1u << c);
                        continue;
                    }
                    const double om = ts / tt;
                    const double rho_next = s_rho[j][c] - s_alpha[j][c] * s_rwv[j][c] - om * wt;
                    s_omega[j][c] = om;
                    s_beta[j][c] = (rho_next / s_rho[j][c]) * (s_alpha[j][c] / om);
                }
                s_act[j] = act;
                s_half[j] = half;
            }
            const unsigned m = __ballot_sync(0xffffffffu, (act | half) != 0);
            if (j == 0) s_any = m;
        }
        __syncthreads();
        // full step and next direction: x += alpha p + omega s, r' = s - omega t, p' = r' + beta (p - omega v),
        // v' = A p'; |r'|^2, rw.r', rw.v'.  Components that stopped at the half step take x += alpha p only.
        for (int j = 0; j < S.n; ++j) {
            if (!((s_any >> j) & 1u)) continue;
            const unsigned act = s_act[j], half = s_half[j];
            const pict_block_t& B = dom.blocks[S.block[j]];
            double acc[3 * NR];
#pragma unroll
            for (int k = 0; k < 3 * NR; ++k) acc[k] = 0.0;
            const int s0 = S.start[j], cnt = S.count[j];
            for (int base = 0; base < cnt; base += KR_PASS) {
                // own-cell results are stored as they are formed (x, r' and p' are not read at neighbours in
                // this sweep; r' and p' go to the other buffers), which keeps the register footprint small
#pragma unroll 1
                for (int k = 0; k < KR_U; ++k) {
                    const int l = base + (int)threadIdx.x + k * KR_THREADS;
                    const bool valid = l < cnt;
                    const int i = s0 + min(l, cnt - 1);
                    int p[3];
                    unflatten(i - B.offset, B.size, p);
#pragma unroll
                    for (int c = 0; c < NR; ++c) {
                        const bool on = (act >> c) & 1u, hf = (half >> c) & 1u;
                        if (!on && !hf) continue;
                        const T al = (T)s_alpha[j][c];
                        const T* rcc = rc + c * NS;
                        const T* vcc = vc + c * NS;
                        const T* pcc = pc + c * NS;
                        T xi = x[c * NS + i] + al * pcc[i];
                        if (!on) {
                            if (valid) x[c * NS + i] = xi;
                            continue;
                        }
                        const T om = (T)s_omega[j][c], bt = (T)s_beta[j][c];
                        const T* tcc = tv + c * NS;
                        const T si = rcc[i] - al * vcc[i];
                        xi = xi + om * si;
                        auto rnew = [&](int jj) { return (rcc[jj] - al * vcc[jj]) - om * tcc[jj]; };
                        auto pnew = [&](int jj) { return rnew(jj) + bt * (pcc[jj] - om * vcc[jj]); };
                        const T ri = rnew(i);
                        const T pi = pnew(i);
                        const T vi = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, pnew);
                        if (!valid) continue;
                        x[c * NS + i] = xi;
                        rn[c * NS + i] = ri;
                        pn[c * NS + i] = pi;
                        vn[c * NS + i] = vi;
                        const double rd = (double)ri, wd = (double)rw[c * NS + i];
                        acc[3 * c] += rd * rd;
                        acc[3 * c + 1] += wd * rd;
                        acc[3 * c + 2] += wd * (double)vi;
                    }
                }
            }
            warp_partial<3 * NR>(R, j, acc);
        }
        flush_partials<3 * NR>(R, S, s_any, part + phase * pstride);
        if (!grid_barrier(a.ctrl, epoch, s_ctrl)) return;
        system_sums<3 * NR>(part + phase * pstride, S, s_any, s_sum);
        phase ^= 1;
        if (threadIdx.x < 32) {
            const int j = threadIdx.x;
            unsigned act = j < S.n ? s_act[j] : 0u;
            unsigned fin = j < S.n ? s_half[j] : 0u;
            if (act) {
                const int n = S.ncell[j];
                for (int c = 0; c < NR; ++c) {
                    if (!((act >> c) & 1u)) continue;
                    const double nr = conv_crit(s_sum[j][3 * c], a.normalized, n);
                    s_info[j][c].final_residual = nr;
                    if (nr < a.tol) {
                        s_info[j][c].converged = 1;
                        s_info[j][c].used_iterations = it + 1;
                        act &= ~(1u << c);
                        fin |= 1u << c;
                    } else {
                        s_rho[j][c] = s_sum[j][3 * c + 1];
                        s_rwv[j][c] = s_sum[j][3 * c + 2];
                    }
                }
                s_act[j] = act;
            }
            if (j < S.n) {
                s_half[j] = 0u;
                if (fin && S.owner[j]) atomicAdd(a.ctrl + CTRL_DONE, __popc(fin));
            }
            const unsigned m = __ballot_sync(0xffffffffu, act != 0);
            if (j == 0) s_any = m;
        }
        __syncthreads();
        T* tr = rc; rc = rn; rn = tr;
        T* tp = pc; pc = pn; pn = tp;
        T* tq = vc; vc = vn; vn = tq;
    }
done:
    if ((int)threadIdx.x < S.n && S.owner[threadIdx.x]) {
        const int j = threadIdx.x;
        for (int c = 0; c < NR; ++c) a.info[S.sim[j] * a.nrhs + c] = s_info[j][c];
    }
}

// ---------------------------------------------------------------------------------------------
// Cluster CG: the single-reduction recurrence of k_cg1, one thread-block cluster per system.
//
// The cluster's first CTA takes the next system from a counter in the workspace (systems are ordered
// largest first) and hands it to every CTA of the cluster through distributed shared memory; the CTAs
// sweep that system's tiles round robin (rank, rank + CL, ...) and reduce the iteration's inner
// products through distributed shared memory: every CTA writes its partials into the first CTA's shared
// memory, one cluster barrier (hardware, release / acquire at cluster scope, which also orders the
// vectors written to global memory by the other CTAs of the cluster), then every CTA sums the partials
// in rank order, so all CTAs take the same decisions from the same numbers.  No grid-wide barrier:
// systems advance independently and a cluster that finishes one takes the next.
// ---------------------------------------------------------------------------------------------
constexpr int KC_MAX_CL = 16;
constexpr int KC_NV = 4;  // values per CTA partial (one layout for every reduction: the two buffers never overlap)

struct ClusterRed {
    double part[2][KC_MAX_CL][KC_NV];
};

// sum of NV <= KC_NV values over the cluster (block sum, then partials through distributed shared memory,
// alternating between two buffers: a CTA writes buffer e & 1 only after every CTA passed the barrier of
// reduction e - 1, i.e. finished reading buffer (e - 2) & 1)
template <int NV>
__device__ __forceinline__ void cluster_sum(cgrp::cluster_group& cl, ClusterRed& red, int& epoch,
                                            double (&v)[NV]) {
    static_assert(NV <= KC_NV, "cluster_sum: too many values");
    __shared__ double s_tot[NV];
    block_sum<NV>(v);
    const int par = epoch & 1;
    ++epoch;
    if (threadIdx.x == 0) {
        ClusterRed* r0 = cl.map_shared_rank(&red, 0);
#pragma unroll
        for (int k = 0; k < NV; ++k) r0->part[par][cl.block_rank()][k] = v[k];
    }
    cl.sync();
    if (threadIdx.x < 32) {  // half-warp h sums value k = h, h + 2, ...: lane r loads rank r's partial, then a
        // fixed butterfly over the 16 lanes (one remote load per lane, all in flight together)
        const ClusterRed* r0 = cl.map_shared_rank(&red, 0);
        const unsigned r = threadIdx.x & 15, h = threadIdx.x >> 4;
#pragma unroll
        for (int k0 = 0; k0 < NV; k0 += 2) {
            const int k = k0 + (int)h;
            double t = (r < cl.num_blocks() && k < NV) ? r0->part[par][r][k < NV ? k : 0] : 0.0;
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (r == 0 && k < NV) s_tot[k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = s_tot[k];
    __syncthreads();
}

template <typename T, int D, bool TRANS>
__global__ void __launch_bounds__(KR_THREADS, 2) k_cg1_cluster(KArgs<T> a) {
    cgrp::cluster_group cl = cgrp::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int rank = (int)cl.block_rank();
    const pict_domain_t& dom = a.dom;
    const int N = dom.num_cells;
    __shared__ ClusterRed red;
    __shared__ int s_sys;
    int epoch = 0;
    const T* __restrict__ coef = a.coef;
    const T* __restrict__ bv = a.b;
    T* __restrict__ x = a.x;
    T* __restrict__ p = a.t;
    cl.sync();  // every CTA of the cluster runs before any distributed shared memory access

    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            const int sys = atomicAdd(a.ctrl + CTRL_SCHED, 1);
            for (int r = 0; r < CL; ++r) *cl.map_shared_rank(&s_sys, r) = sys;
        }
        cl.sync();
        const int sys = s_sys;
        if (sys >= dom.num_sims) break;
        const int t0 = dom.sim_tiles[sys], t1 = dom.sim_tiles[sys + 1];
        const int n = dom.sim_cells[sys + 1] - dom.sim_cells[sys];
        T* rc = a.r;   // r_i
        T* rn = a.rw;  // r_{i+1}
        T* wc = a.p0;
        T* wn = a.p1;
        T* sc = a.v0;
        T* sn = a.v1;
        // the tiles of this CTA: t0 + rank, t0 + rank + CL, ...
#define KC_TILES(t, blk, s0, cnt)                                                                   \
    for (int t = t0 + rank; t < t1; t += CL)                                                        \
        for (int blk = dom.tiles[4 * t + 1], s0 = dom.tiles[4 * t + 2], cnt = dom.tiles[4 * t + 3]; \
             cnt > 0; cnt = 0)

        // ---- init: r0 = b - A x0 (when x0 != 0), w0 = A r0, g0, d0, |b|^2
        if (!a.x_zero) {
            KC_TILES(t, blk, s0, cnt) {
                const pict_block_t& B = dom.blocks[blk];
                for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) {
                    int q[3];
                    unflatten(i - B.offset, B.size, q);
                    rc[i] = bv[i] - spmv_row<T, D, TRANS>(dom, coef, N, i, B, q, [&](int jj) { return x[jj]; });
                }
            }
            cl.sync();
        }
        const T* r0 = a.x_zero ? bv : rc;
        double acc3[3] = {0.0, 0.0, 0.0};
        KC_TILES(t, blk, s0, cnt) {
            const pict_block_t& B = dom.blocks[blk];
            for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) {
                int q[3];
                unflatten(i - B.offset, B.size, q);
                const T ri = r0[i];
                const T wi = spmv_row<T, D, TRANS>(dom, coef, N, i, B, q, [&](int jj) { return r0[jj]; });
                wc[i] = wi;
                sc[i] = T(0);
                p[i] = T(0);
                const T bi = bv[i];
                acc3[0] += (double)ri * (double)ri;
                acc3[1] += (double)wi * (double)ri;
                acc3[2] += (double)bi * (double)bi;
            }
        }
        cluster_sum<3>(cl, red, epoch, acc3);
        if (a.x_zero) {
            KC_TILES(t, blk, s0, cnt) {
                for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) {
                    rc[i] = bv[i];
                    x[i] = T(0);
                }
            }
        }
        pict_solve_info_t inf = fresh_info();
        double g = acc3[0], alpha = acc3[0] / acc3[1], beta = 0.0;
        bool active = true;
        if (acc3[2] == 0.0) {
            inf.converged = 1;
            inf.used_iterations = 0;
            active = false;
            KC_TILES(t, blk, s0, cnt) {
                for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) x[i] = T(0);
            }
        }
        if (active) cl.sync();  // rc / x of the x_zero start visible before the first sweep reads neighbours
        for (int it = 0; active && it < a.maxit; ++it) {
            const T al = (T)alpha, bt = (T)beta;
            double acc[2] = {0.0, 0.0};
            KC_TILES(t, blk, s0, cnt) {
                const pict_block_t& B = dom.blocks[blk];
                for (int base = 0; base < cnt; base += KR_PASS) {
                    T rni[KR_U], wni[KR_U], pi[KR_U], si[KR_U], xi[KR_U];
#pragma unroll
                    for (int k = 0; k < KR_U; ++k) {
                        const int i = s0 + min(base + (int)threadIdx.x + k * KR_THREADS, cnt - 1);
                        int q[3];
                        unflatten(i - B.offset, B.size, q);
                        pi[k] = rc[i] + bt * p[i];
                        si[k] = wc[i] + bt * sc[i];
                        rni[k] = rc[i] - al * si[k];
                        xi[k] = x[i] + al * pi[k];
                        wni[k] = spmv_row<T, D, TRANS>(dom, coef, N, i, B, q,
                                                       [&](int jj) { return rc[jj] - al * (wc[jj] + bt * sc[jj]); });
                    }
#pragma unroll
                    for (int k = 0; k < KR_U; ++k) {
                        const int l = base + (int)threadIdx.x + k * KR_THREADS;
                        if (l < cnt) {
                            const int i = s0 + l;
                            x[i] = xi[k];
                            p[i] = pi[k];
                            sn[i] = si[k];
                            rn[i] = rni[k];
                            wn[i] = wni[k];
                            acc[0] += (double)rni[k] * (double)rni[k];
                            acc[1] += (double)wni[k] * (double)rni[k];
                        }
                    }
                }
            }
            cluster_sum<2>(cl, red, epoch, acc);
            const double gn = acc[0], d = acc[1];
            const double crit = conv_crit(gn, a.normalized, n);
            inf.used_iterations = it;
            inf.final_residual = crit;
            if (!isfinite(crit)) { inf.finite = 0; active = false; }
            else if (crit < a.tol) { inf.converged = 1; active = false; }
            else {
                const double bnew = gn / g;
                alpha = gn / (d - bnew * gn / alpha);
                beta = bnew;
                g = gn;
            }
            T* t0p = rc; rc = rn; rn = t0p;
            T* t1p = wc; wc = wn; wn = t1p;
            T* t2p = sc; sc = sn; sn = t2p;
        }
        if (a.sub_mean || a.write_bp) {
            double m[1] = {0.0};
            if (a.sub_mean) {
                KC_TILES(t, blk, s0, cnt) {
                    for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) m[0] += (double)x[i];
                }
                cluster_sum<1>(cl, red, epoch, m);
            }
            const T mean = a.sub_mean ? (T)(m[0] / (double)n) : T(0);
            KC_TILES(t, blk, s0, cnt) {
                const pict_block_t& B = dom.blocks[blk];
                T* pb = reinterpret_cast<T*>(B.pressure);
                for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) {
                    const T v = x[i] - mean;
                    x[i] = v;
                    if (a.write_bp) pb[i - B.offset] = v;
                }
            }
        }
#undef KC_TILES
        if (rank == 0 && threadIdx.x == 0) a.info[sys] = inf;
        cl.sync();  // every CTA is done with s_sys and the vectors of this system
    }
}

__global__ void k_init_info(pict_solve_info_t* info, int n) {
    PICT_CELL_LOOP(i, n) {
        info[i].final_residual = 0.0;
        info[i].used_iterations = -1;
        info[i].converged = 0;
        info[i].finite = 1;
        info[i].status = 2;
    }
}

// status 1 for every system if any barrier timed out
__global__ void k_finish_info(pict_solve_info_t* info, int n, const int* ctrl) {
    if (ctrl[CTRL_ERR] == 0) return;
    PICT_CELL_LOOP(i, n) { info[i].status = 1; info[i].converged = 0; }
}

// ---------------------------------------------------------------------------------------------
// host side: launch plan and workspace
// ---------------------------------------------------------------------------------------------

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// workspace: ctrl (256 B) | partials [2][num_tiles][KR_NV] doubles | vectors
static size_t header_bytes(const pict_domain_t* dom) {
    return align256(256) + align256(sizeof(double) * 2 * (size_t)dom->num_tiles * KR_NV);
}

static int nrhs_per_launch(const pict_solve_params_t* prm) {
    // BiCGStab with an ABS criterion keeps a third group of initial partials: at most 2 components per launch
    const int cap = prm->convergence >= PICT_CONV_ABS_SUM ? 2 : 3;
    return prm->use_bicg ? (prm->nrhs > cap ? cap : prm->nrhs) : 1;
}

static size_t vec_bytes(const pict_domain_t* dom, const pict_solve_params_t* prm) {
    const size_t esz = dom->dtype == PICT_F64 ? 8 : 4;
    return align256(esz * (size_t)dom->num_cells * nrhs_per_launch(prm));
}

// BiCGStab kernel choice (pict_krylov_set_bicgstab_variant), see below
static int g_bicgstab_variant = 0;

// bicg: 7 vectors (8 for the two-barrier kernel: two residual buffers); cg1: 7; cg: r p0 p1 q (+ the best iterate)
static int workspace_vectors(const pict_solve_params_t* prm) {
    if (prm->use_bicg) return g_bicgstab_variant != 0 ? 8 : 7;
    return prm->variant == 1 ? 7 : (prm->return_best_result ? 5 : 4);
}

static size_t workspace_total(const pict_domain_t* dom, const pict_solve_params_t* prm) {
    return header_bytes(dom) + vec_bytes(dom, prm) * workspace_vectors(prm);
}

// 0: persistent grid only; 1: clusters where they apply (default); 2: clusters whenever possible
static int g_cluster_mode = 1;
// BiCGStab kernel: 0 (default) the four-barrier form for every solve; 1 the two-barrier form (NORM2
// criteria, up to two right-hand sides per launch) with one 512-thread CTA per SM and 128 registers per
// thread, 2 the same with two CTAs per SM (64 registers, some spilled).  Measured on the batch of 256
// cavities (mixed-precision step): 8.22 ms per step with 0, 9.04 with 1, 8.63 with 2 -- the merged sweep
// gathers r, v, t and p at every neighbour, which costs more than the two barriers it saves; on single
// small domains (cylinder street, 64^2 cavity) 1 is 1-3% faster.  The workspace size depends on the choice
// (pict_solve_workspace_bytes): switch before sizing the workspace.

// Launch k_cg1_cluster with clusters of `cl` CTAs, as many clusters as fit on the device at once (at most
// one per system).  Returns PICT_ERR_UNSUPPORTED (nothing launched) if no cluster of that size fits.
template <typename T, int D, bool TRANS>
static pict_status_t launch_cg1_cluster(KArgs<T>& a, int cl, cudaStream_t st) {
    auto kern = k_cg1_cluster<T, D, TRANS>;
    if (cl > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return PICT_ERR_UNSUPPORTED;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(KR_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(cl);
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) != cudaSuccess || ncl < 1) {
        cudaGetLastError();
        return PICT_ERR_UNSUPPORTED;
    }
    if (ncl > a.dom.num_sims) ncl = a.dom.num_sims;
    cfg.gridDim = dim3(ncl * cl);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a);
    if (e != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof(buf), "cluster CG launch (%d clusters of %d): %s", ncl, cl, cudaGetErrorString(e));
        cudaGetLastError();
        return set_error(PICT_ERR_CUDA, buf);
    }
    return PICT_OK;
}

template <typename KernelT>
static int max_coresident(KernelT kernel) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, KR_THREADS, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * device_sm_count();
}

template <typename T>
static pict_status_t launch_kernel(void (*kernel)(KArgs<T>), int grid, KArgs<T>& args, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(KR_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = grid > 1 ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, args);
    if (e != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof(buf), "krylov launch (grid %d x %d threads): %s", grid, KR_THREADS, cudaGetErrorString(e));
        cudaGetLastError();
        return set_error(PICT_ERR_CUDA, buf);
    }
    return PICT_OK;
}

template <typename T, int D, bool TRANS>
static pict_status_t run_solve(const pict_domain_t* dom, const void* coef, const void* rhs, void* x,
                               const pict_solve_params_t* prm, void* info_out, void* ws, int64_t ws_bytes,
                               cudaStream_t st) {
    if ((int64_t)workspace_total(dom, prm) > ws_bytes) return set_error(PICT_ERR_ARG, "solve: workspace too small");
    if (dom->tile_cells > KR_MAX_TILE || dom->tile_cells <= 0 || !dom->tiles || !dom->sim_tiles || dom->num_tiles <= 0)
        return set_error(PICT_ERR_ARG, "solve: invalid tile table (tile_cells must be in [1, 2048])");
    char* base = reinterpret_cast<char*>(ws);
    int* ctrl = reinterpret_cast<int*>(base);
    double* partials = reinterpret_cast<double*>(base + align256(256));
    const size_t off = header_bytes(dom);
    const size_t vb = vec_bytes(dom, prm);
    const int nvec = workspace_vectors(prm);
    T* vec[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int k = 0; k < nvec; ++k) vec[k] = reinterpret_cast<T*>(base + off + vb * k);

    const int nrhs_total = prm->nrhs;
    pict_solve_info_t* info = reinterpret_cast<pict_solve_info_t*>(info_out);
    const int ninfo = dom->num_sims * nrhs_total;
    k_init_info<<<cell_grid(ninfo, 128), 128, 0, st>>>(info, ninfo);
    pict_status_t s = check_launch("init_info");
    if (s) return s;
    const size_t NS = (size_t)dom->num_cells;
    const int per = nrhs_per_launch(prm);
    for (int c0 = 0; c0 < nrhs_total; c0 += per) {
        const int nr = (nrhs_total - c0) < per ? (nrhs_total - c0) : per;
        if (cudaMemsetAsync(ctrl, 0, 256, st) != cudaSuccess) return check_launch("workspace memset");
        KArgs<T> a;
        a.dom = *dom;
        a.coef = reinterpret_cast<const T*>(coef);
        a.b = reinterpret_cast<const T*>(rhs) + c0 * NS;
        a.x = reinterpret_cast<T*>(x) + c0 * NS;
        a.ctrl = ctrl;
        a.partials = partials;
        a.maxit = prm->max_iterations;
        a.tol = prm->tolerance;
        a.normalized = prm->convergence == PICT_CONV_NORM2_NORMALIZED;
        a.x_zero = prm->x_is_zero;
        a.sub_mean = prm->subtract_mean;
        a.write_bp = prm->write_block_pressure;
        a.reset = prm->use_bicg ? 0 : (prm->residual_reset_steps > 0 ? prm->residual_reset_steps : 0);
        a.best = prm->use_bicg ? 0 : (prm->return_best_result ? 1 : 0);
        a.xbest = nullptr;
        a.abs_crit = prm->convergence >= PICT_CONV_ABS_SUM ? prm->convergence : 0;
        a.rankdef = prm->use_bicg ? 0 : (prm->rank_deficient ? 1 : 0);
        a.info = info + c0;
        a.r1 = nullptr;
        a.nrhs = nrhs_total;
        void (*kern)(KArgs<T>) = nullptr;
        if (prm->use_bicg) {
            a.r = vec[0]; a.rw = vec[1]; a.p0 = vec[2]; a.p1 = vec[3]; a.v0 = vec[4]; a.v1 = vec[5]; a.t = vec[6];
            a.r1 = vec[7];  // null with the four-barrier kernel (7 vectors)
            if (g_bicgstab_variant == 1 && a.abs_crit == 0 && nr <= 2)
                kern = nr == 1 ? k_bicgstab2<T, D, 1, TRANS, 1> : k_bicgstab2<T, D, 2, TRANS, 1>;
            else if (g_bicgstab_variant == 2 && a.abs_crit == 0 && nr <= 2)
                kern = nr == 1 ? k_bicgstab2<T, D, 1, TRANS, 2> : k_bicgstab2<T, D, 2, TRANS, 2>;
            else
                kern = nr == 1 ? k_bicgstab<T, D, 1, TRANS> : (nr == 2 ? k_bicgstab<T, D, 2, TRANS> : k_bicgstab<T, D, 3, TRANS>);
        } else if (prm->variant == 1 && a.reset == 0 && a.best == 0 && a.abs_crit == 0 && a.rankdef == 0) {
            a.r = vec[0]; a.rw = vec[1]; a.p0 = vec[2]; a.p1 = vec[3]; a.v0 = vec[4]; a.v1 = vec[5]; a.t = vec[6];
            kern = k_cg1<T, D, TRANS>;
            // one thread-block cluster per system where systems are small enough for one cluster's SMs to
            // stream: latency-bound small systems, or many systems that fill the device between them
            // few systems: with many, the lockstep grid amortises one barrier per iteration over all of
            // them while each cluster would pay its own per system
            const bool few_small = dom->num_sims <= 8 && dom->max_sim_cells <= 262144;
            if (g_cluster_mode == 2 || (g_cluster_mode == 1 && few_small)) {
                s = launch_cg1_cluster<T, D, TRANS>(a, 16, st);
                if (s == PICT_ERR_UNSUPPORTED) s = launch_cg1_cluster<T, D, TRANS>(a, 8, st);
                if (s == PICT_OK) {
                    k_finish_info<<<1, 128, 0, st>>>(info, ninfo, ctrl);
                    s = check_launch("finish_info");
                    if (s) return s;
                    continue;
                }
                if (s != PICT_ERR_UNSUPPORTED) return s;
            }
        } else {
            a.r = vec[0]; a.p0 = vec[1]; a.p1 = vec[2]; a.t = vec[3];
            a.rw = nullptr; a.v0 = nullptr; a.v1 = nullptr;
            if (a.best) a.xbest = vec[4];
            if (a.best && !a.xbest) return set_error(PICT_ERR_ARG, "solve: no workspace vector for the best iterate");
            kern = k_cg<T, D, TRANS>;
        }
        // grid: every CTA owns at most KR_SLOTS tiles; all CTAs must be co-resident
        const int cores = max_coresident(kern);
        int grid = dom->num_tiles < cores ? dom->num_tiles : cores;
        if (prm->group_size > 0 && grid > prm->group_size) grid = prm->group_size;
        const int min_grid = (dom->num_tiles + KR_SLOTS - 1) / KR_SLOTS;
        if (grid < min_grid) grid = min_grid;
        if (grid > cores) return set_error(PICT_ERR_ARG, "solve: too many tiles for one persistent launch (raise tile_cells)");
        s = launch_kernel<T>(kern, grid, a, st);
        if (s) return s;
        k_finish_info<<<1, 128, 0, st>>>(info, ninfo, ctrl);
        s = check_launch("finish_info");
        if (s) return s;
    }
    return PICT_OK;
}

// ---------------------------------------------------------------------------------------------
// Fixed scratch for pict_solve_static: callers that hold no device allocator (a plain C or ctypes
// binding without torch, or a loop that must not call cudaMalloc, which synchronises the device)
// solve small systems with the workspace placed in this module's own device memory.
// ---------------------------------------------------------------------------------------------
// 8 MiB.  Which solves fit depends on the solver's vector count: 4 vectors of N values for CG, 5 with
// returnBestResult, 7 for the single-reduction CG (variant 1), and 7 x (right-hand sides per launch)
// for BiCGStab, plus a small header; e.g. FP32 CG fits ~520k cells, single-reduction CG ~290k,
// a 2D BiCGStab velocity solve (2 components) ~150k.  Every device that loads the library holds
// this array for the life of the process, whether or not pict_solve_static is ever called.
constexpr size_t KR_STATIC_SCRATCH_BYTES = size_t(8) << 20;
static __device__ __align__(256) unsigned char kr_static_scratch[KR_STATIC_SCRATCH_BYTES];

// Device address of kr_static_scratch in the current context.  Looked up on every call: the
// address belongs to the context the module is loaded in (a context re-created after
// cudaDeviceReset, or another context made current through the driver API, can place the module
// elsewhere), and the lookup allocates nothing.  The first call in a context loads the module.
static pict_status_t static_scratch(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, kr_static_scratch);
    if (e != cudaSuccess || !p) {
        char buf[256];
        snprintf(buf, sizeof(buf), "solve_static: cudaGetSymbolAddress of the scratch failed: %s", cudaGetErrorString(e));
        cudaGetLastError();
        return set_error(e == cudaErrorNoDevice ? PICT_ERR_NO_DEVICE : PICT_ERR_CUDA, buf);
    }
    *out = p;
    return PICT_OK;
}

}  // namespace pict

using namespace pict;

extern "C" {

int64_t pict_solve_static_scratch_bytes(void) { return (int64_t)KR_STATIC_SCRATCH_BYTES; }

void pict_krylov_set_cluster_mode(int32_t mode) { g_cluster_mode = mode < 0 ? 0 : (mode > 2 ? 2 : mode); }
void pict_krylov_set_bicgstab_variant(int32_t variant) { g_bicgstab_variant = variant < 0 ? 0 : (variant > 2 ? 2 : variant); }

pict_status_t pict_solve_static(const pict_domain_t* dom, const void* coef, const void* rhs, void* x,
                                const pict_solve_params_t* prm, void* info_out, void* stream) {
    if (!dom || !prm) return set_error(PICT_ERR_ARG, "solve_static: NULL argument");
    const int64_t need = pict_solve_workspace_bytes(dom, prm);
    if (need < 0 || need > (int64_t)KR_STATIC_SCRATCH_BYTES) {
        char buf[256];
        snprintf(buf, sizeof(buf),
                 "solve_static: the solve needs %lld bytes of workspace, more than the %lld bytes of static scratch; "
                 "use pict_solve with a caller-provided workspace",
                 (long long)need, (long long)KR_STATIC_SCRATCH_BYTES);
        return set_error(PICT_ERR_ARG, buf);
    }
    void* ws = nullptr;
    const pict_status_t s = static_scratch(&ws);
    if (s) return s;
    return pict_solve(dom, coef, rhs, x, prm, info_out, ws, (int64_t)KR_STATIC_SCRATCH_BYTES, stream);
}

int64_t pict_solve_workspace_bytes(const pict_domain_t* dom, const pict_solve_params_t* prm) {
    if (!dom || !prm) return -1;
    return (int64_t)workspace_total(dom, prm);
}

pict_status_t pict_solve(const pict_domain_t* dom, const void* coef, const void* rhs, void* x,
                         const pict_solve_params_t* prm, void* info_out, void* ws, int64_t ws_bytes, void* stream) {
    if (!dom || !prm || !coef || !rhs || !x || !info_out || !ws) return set_error(PICT_ERR_ARG, "solve: NULL argument");
    if (dom->num_cells <= 0 || !dom->blocks || !dom->nbr || !dom->sim_cells || !dom->sim_blocks)
        return set_error(PICT_ERR_ARG, "solve: domain is not prepared");
    if (prm->nrhs < 1) return set_error(PICT_ERR_ARG, "solve: nrhs must be >= 1");
    if (prm->max_iterations < 0) return set_error(PICT_ERR_ARG, "solve: max_iterations must be >= 0");
    if (prm->convergence < PICT_CONV_NORM2 || prm->convergence > PICT_CONV_ABS_MAX)
        return set_error(PICT_ERR_ARG, "solve: unknown convergence criterion");
    if (prm->use_bicg && prm->rank_deficient)
        return set_error(PICT_ERR_UNSUPPORTED, "solve: rank_deficient applies to CG only");
    if (prm->variant != 0 && (prm->use_bicg || prm->variant != 1))
        return set_error(PICT_ERR_ARG, "solve: variant 1 (single-reduction) applies to CG only");
    if (!prm->use_bicg && prm->nrhs != 1)
        return set_error(PICT_ERR_UNSUPPORTED, "solve: CG takes one right-hand side per call");
    cudaStream_t st = (cudaStream_t)stream;
    const bool tr = prm->transpose != 0;
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) return tr ? run_solve<float, 2, true>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st)
                                      : run_solve<float, 2, false>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st);
        if (dom->dims == 3) return tr ? run_solve<float, 3, true>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st)
                                      : run_solve<float, 3, false>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st);
    } else if (dom->dtype == PICT_F64) {
        if (dom->dims == 2) return tr ? run_solve<double, 2, true>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st)
                                      : run_solve<double, 2, false>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st);
        if (dom->dims == 3) return tr ? run_solve<double, 3, true>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st)
                                      : run_solve<double, 3, false>(dom, coef, rhs, x, prm, info_out, ws, ws_bytes, st);
    }
    return set_error(PICT_ERR_UNSUPPORTED, "solve: unsupported dtype/dims");
}

}  // extern "C"
