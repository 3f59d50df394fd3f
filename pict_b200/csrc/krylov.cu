// krylov.cu -- persistent CG and BiCGStab on structured stencil matrices.
//
// Replaces the reference's host-driven Krylov loops (cgSolveGPU,
// extensions/cg_solver_kernel.cu:114-456; bicgstabSolveGPU,
// extensions/bicgstab_solver_kernel.cu:47-395), which issue one cuSPARSE SpMV
// plus several cuBLAS calls with host round trips per iteration, by one
// persistent launch per solve:
//
//  * a group of G cooperating CTAs owns one system (simulation) at a time and
//    pulls the next system from a device work queue, so a batch of uneven
//    systems is solved in a single launch;
//  * the stencil SpMV reads structured neighbours directly (i +- stride) and
//    falls back to the precomputed neighbour table only on block faces;
//  * vector updates are fused into the SpMV sweeps (the search direction is
//    formed on the fly for the neighbours, double-buffered), leaving two
//    group-wide reductions per CG iteration and four per BiCGStab iteration;
//  * inner products and norms are accumulated in FP64 with a fixed reduction
//    order (deterministic), for FP32 and FP64 vectors alike;
//  * BiCGStab advances all D velocity components at once (shared matrix
//    loads), each with its own scalars and convergence state;
//  * every inter-CTA wait is bounded: on timeout the kernel records an error
//    and returns (the host reports it through pict_solve_info_t.status).
//
// Iteration semantics, stopping rule and reported iteration counts follow the
// reference: CG cg.cu:236-427, BiCGStab bicg.cu:240-360, convergence criterion
// NORM2 / NORM2_NORMALIZED cg.cu:77-110.  As in the Python wrapper
// (PISOtorch_diff.py:245-293), an all-zero right-hand side yields x = 0.
#include <cmath>
#include <cstdio>
#include "common.cuh"
#include "launch.h"

#ifndef PICT_SPIN_LIMIT
#define PICT_SPIN_LIMIT (1ll << 26)
#endif

namespace pict {

constexpr int KR_NV = 8;      // partial-sum slots per reduction
constexpr int KR_MAX_WARPS = 16;

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
    int* queue;
    int* err;
    int* group_sys;
    unsigned* sync;       // [ngroups][32]
    double* partials;     // [ngroups][2][G][KR_NV]
    pict_solve_info_t* info;
    int maxit;
    double tol;
    int normalized;
    int nrhs;
    int G;
    int x_zero;
    int sub_mean;
    int write_bp;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Bounded barrier of the G CTAs of one group (sense by generation counter).
__device__ bool group_barrier(unsigned* sync, int G, int* err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* vgen = sync + 1;
        const unsigned g0 = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(sync, 1u);
        if (arrived == (unsigned)(G - 1)) {
            atomicExch(sync, 0u);
            __threadfence();
            atomicAdd(sync + 1, 1u);
        } else {
            long long spins = 0;
            while (*vgen == g0) {
                if (++spins > PICT_SPIN_LIMIT) { ok = 0; atomicExch(err, 1); break; }
                if (*(volatile int*)err) { ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Sum NV doubles over the CTA, then over the G CTAs of the group (fixed order).
template <int NV, typename T>
__device__ bool reduce(double (&v)[NV], const KArgs<T>& a, int grp, int rank, int& phase) {
    __shared__ double s_red[KR_MAX_WARPS][KR_NV];
    __shared__ double s_out[KR_NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
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
    if (a.G > 1) {
        double* part = a.partials + ((size_t)(grp * 2 + phase) * a.G) * KR_NV;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) part[rank * KR_NV + k] = s_out[k];
        }
        if (!group_barrier(a.sync + grp * 32, a.G, a.err)) return false;
        if (threadIdx.x < NV) {
            double s = 0;
            for (int r = 0; r < a.G; ++r) s += __ldcg(part + r * KR_NV + threadIdx.x);
            s_out[threadIdx.x] = s;
        }
        phase ^= 1;
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = s_out[k];
    __syncthreads();
    return true;
}

// Fetch the next system for this group from the work queue (-1: none left, -2: aborted).
template <typename T>
__device__ int next_system(const KArgs<T>& a, int grp, int rank) {
    __shared__ int s_sys;
    if (a.G == 1) {
        if (threadIdx.x == 0) s_sys = atomicAdd(a.queue, 1);
        __syncthreads();
    } else {
        if (rank == 0 && threadIdx.x == 0) {
            const int s = atomicAdd(a.queue, 1);
            *(volatile int*)(a.group_sys + grp) = s;
        }
        if (!group_barrier(a.sync + grp * 32, a.G, a.err)) return -2;
        if (threadIdx.x == 0) s_sys = *(volatile int*)(a.group_sys + grp);
        __syncthreads();
    }
    const int s = s_sys;
    __syncthreads();
    return s < a.dom.num_sims ? s : -1;
}

// Iterate the cells [lo,hi) of the system's blocks [b0,b1) owned by this CTA.
#define KR_FOR_CELLS(...)                                                                  \
    for (int bb = b0; bb < b1; ++bb) {                                                     \
        const pict_block_t& B = dom.blocks[bb];                                            \
        const int bo = B.offset;                                                           \
        const int bn = B.size[0] * B.size[1] * B.size[2];                                  \
        const int cs = max(bo, lo), ce = min(bo + bn, hi);                                 \
        for (int i = cs + (int)threadIdx.x; i < ce; i += blockDim.x) {                     \
            const int l = i - bo;                                                          \
            int p[3];                                                                      \
            unflatten(l, B.size, p);                                                       \
            __VA_ARGS__                                                                    \
        }                                                                                  \
    }

// One stencil row applied to a vector given by `load(j)`; TRANS applies the transposed matrix
// (the coefficient of row j pointing back to i).
template <typename T, int D, bool TRANS, typename F>
__device__ __forceinline__ T spmv_row(const pict_domain_t& dom, const T* coef, int N, int i, const pict_block_t& B,
                                      const int* p, F load) {
    T acc = coef[i] * load(i);
    const int stride[3] = {1, B.size[0], B.size[0] * B.size[1]};
#pragma unroll
    for (int f = 0; f < 2 * D; ++f) {
        const int a = f >> 1;
        const bool up = f & 1;
        const bool at = up ? (p[a] == B.size[a] - 1) : (p[a] == 0);
        int j, back = f ^ 1;
        if (!at) {
            j = i + (up ? stride[a] : -stride[a]);
        } else {
            j = dom.nbr[(size_t)f * N + i];
            if (j >= 0 && B.face[f].type == PICT_FACE_CONNECTED) back = B.face[f].conn_axes[0];
        }
        if (j >= 0) {
            const T c = TRANS ? coef[(size_t)(back + 1) * N + j] : coef[(size_t)(f + 1) * N + i];
            acc += c * load(j);
        }
    }
    return acc;
}

__device__ __forceinline__ double conv_crit(double sq, int normalized, int n) {
    const double nrm = sqrt(sq);
    return normalized ? nrm / sqrt((double)n) : nrm;
}

// ---------------------------------------------------------------------------------------------
// CG (cg.cu:236-427)
// ---------------------------------------------------------------------------------------------
template <typename T, int D, bool TRANS>
__global__ void __launch_bounds__(512) k_cg(KArgs<T> a) {
    const pict_domain_t& dom = a.dom;
    const int N = dom.num_cells;
    const int G = a.G;
    const int grp = blockIdx.x / G, rank = blockIdx.x % G;
    int phase = 0;
    for (;;) {
        const int s = next_system(a, grp, rank);
        if (s < 0) return;
        const int c0 = dom.sim_cells[s], c1 = dom.sim_cells[s + 1];
        const int b0 = dom.sim_blocks[s], b1 = dom.sim_blocks[s + 1];
        const int n = c1 - c0;
        const int chunk = (n + G - 1) / G;
        const int lo = c0 + rank * chunk, hi = min(c1, lo + chunk);
        const T* coef = a.coef;
        const T* bv = a.b;
        T* x = a.x;
        T* r = a.r;
        T* q = a.t;
        T* pc = a.p0;
        T* pn = a.p1;
        // initial residual r = b - A x
        double acc[2] = {0.0, 0.0};
        KR_FOR_CELLS({
            const T bi = bv[i];
            T ri = bi;
            if (!a.x_zero) ri -= spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int j) { return x[j]; });
            r[i] = ri;
            pc[i] = T(0);
            if (a.x_zero) x[i] = T(0);
            acc[0] += (double)ri * (double)ri;
            acc[1] += (double)bi * (double)bi;
        })
        if (!reduce<2>(acc, a, grp, rank, phase)) return;
        pict_solve_info_t info;
        info.final_residual = 0.0;
        info.used_iterations = -1;
        info.converged = 0;
        info.finite = 1;
        info.status = 0;
        if (acc[1] == 0.0) {
            KR_FOR_CELLS({ x[i] = T(0); })
            info.converged = 1;
            info.used_iterations = 0;
        } else {
            double rho = acc[0];
            double beta = 0.0;
            for (int it = 0; it < a.maxit; ++it) {
                // p <- r + beta p (on the fly for neighbours), q = A p
                double pq[1] = {0.0};
                const T bt = (T)beta;
                KR_FOR_CELLS({
                    const T pi = r[i] + bt * pc[i];
                    const T qi = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int j) { return r[j] + bt * pc[j]; });
                    pn[i] = pi;
                    q[i] = qi;
                    pq[0] += (double)pi * (double)qi;
                })
                if (!reduce<1>(pq, a, grp, rank, phase)) return;
                const double alpha = rho / pq[0];
                const T at = (T)alpha;
                double rr[1] = {0.0};
                KR_FOR_CELLS({
                    x[i] += at * pn[i];
                    const T ri = r[i] - at * q[i];
                    r[i] = ri;
                    rr[0] += (double)ri * (double)ri;
                })
                if (!reduce<1>(rr, a, grp, rank, phase)) return;
                const double crit = conv_crit(rr[0], a.normalized, n);
                info.used_iterations = it;
                info.final_residual = crit;
                if (!isfinite(crit)) { info.finite = 0; break; }
                if (crit < a.tol) { info.converged = 1; break; }
                beta = rr[0] / rho;
                rho = rr[0];
                T* tmp = pc; pc = pn; pn = tmp;
            }
        }
        if (a.sub_mean || a.write_bp) {
            double sm[1] = {0.0};
            if (a.sub_mean) {
                KR_FOR_CELLS({ sm[0] += (double)x[i]; })
                if (!reduce<1>(sm, a, grp, rank, phase)) return;
            }
            const T mean = a.sub_mean ? (T)(sm[0] / (double)n) : T(0);
            KR_FOR_CELLS({
                const T v = x[i] - mean;
                x[i] = v;
                if (a.write_bp) reinterpret_cast<T*>(B.pressure)[l] = v;
            })
        }
        if (rank == 0 && threadIdx.x == 0) a.info[s] = info;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// BiCGStab without preconditioner (bicg.cu:240-360), NR right-hand sides sharing the matrix
// ---------------------------------------------------------------------------------------------
template <typename T, int D, int NR, bool TRANS>
__global__ void __launch_bounds__(512) k_bicgstab(KArgs<T> a) {
    const pict_domain_t& dom = a.dom;
    const int N = dom.num_cells;
    const int G = a.G;
    const int grp = blockIdx.x / G, rank = blockIdx.x % G;
    int phase = 0;
    for (;;) {
        const int s = next_system(a, grp, rank);
        if (s < 0) return;
        const int c0 = dom.sim_cells[s], c1 = dom.sim_cells[s + 1];
        const int b0 = dom.sim_blocks[s], b1 = dom.sim_blocks[s + 1];
        const int n = c1 - c0;
        const int chunk = (n + G - 1) / G;
        const int lo = c0 + rank * chunk, hi = min(c1, lo + chunk);
        const T* coef = a.coef;
        const size_t NS = (size_t)N;
        T* pc = a.p0; T* pn = a.p1;
        T* vc = a.v0; T* vn = a.v1;
        // init: r = b - A x, rw = r, p = v = 0
        double acc[2 * NR];
#pragma unroll
        for (int k = 0; k < 2 * NR; ++k) acc[k] = 0.0;
        KR_FOR_CELLS({
#pragma unroll
            for (int c = 0; c < NR; ++c) {
                const T* xc = a.x + c * NS;
                const T bi = a.b[c * NS + i];
                T ri = bi;
                if (!a.x_zero) ri -= spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int j) { return xc[j]; });
                if (a.x_zero) a.x[c * NS + i] = T(0);
                a.r[c * NS + i] = ri;
                a.rw[c * NS + i] = ri;
                pc[c * NS + i] = T(0);
                vc[c * NS + i] = T(0);
                acc[c] += (double)ri * (double)ri;
                acc[NR + c] += (double)bi * (double)bi;
            }
        })
        if (!reduce<2 * NR>(acc, a, grp, rank, phase)) return;
        pict_solve_info_t info[NR];
        double rho[NR], alpha[NR], omega[NR], beta[NR], rwr[NR];
        int active = 0, zero = 0;
#pragma unroll
        for (int c = 0; c < NR; ++c) {
            info[c].final_residual = 0.0;
            info[c].used_iterations = -1;
            info[c].converged = 0;
            info[c].finite = 1;
            info[c].status = 0;
            rho[c] = 0.0; alpha[c] = 0.0; omega[c] = 0.0; beta[c] = 0.0;
            rwr[c] = acc[c];
            if (acc[NR + c] == 0.0) {
                zero |= 1 << c;
                info[c].converged = 1;
                info[c].used_iterations = 0;
            } else {
                const double nrmr0 = conv_crit(acc[c], a.normalized, n);
                if (nrmr0 < a.tol) {
                    info[c].converged = 1;
                    info[c].used_iterations = -1;
                    info[c].final_residual = nrmr0;
                } else {
                    active |= 1 << c;
                }
            }
        }
        if (zero) {
            KR_FOR_CELLS({
#pragma unroll
                for (int c = 0; c < NR; ++c)
                    if (zero & (1 << c)) a.x[c * NS + i] = T(0);
            })
        }
        for (int it = 0; it < a.maxit && active; ++it) {
#pragma unroll
            for (int c = 0; c < NR; ++c) {
                if (!(active & (1 << c))) continue;
                const double rhop = rho[c];
                rho[c] = rwr[c];
                beta[c] = it > 0 ? (rho[c] / rhop) * (alpha[c] / omega[c]) : 0.0;
            }
            // phase A: p = r + beta (p - omega v) on the fly, v = A p, rw.v
            double rwv[NR];
#pragma unroll
            for (int c = 0; c < NR; ++c) rwv[c] = 0.0;
            KR_FOR_CELLS({
#pragma unroll
                for (int c = 0; c < NR; ++c) {
                    if (!(active & (1 << c))) continue;
                    const T bt = (T)beta[c], om = (T)omega[c];
                    const T* rc = a.r + c * NS;
                    const T* pcc = pc + c * NS;
                    const T* vcc = vc + c * NS;
                    const T pi = rc[i] + bt * (pcc[i] - om * vcc[i]);
                    const T vi = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p,
                                                       [&](int j) { return rc[j] + bt * (pcc[j] - om * vcc[j]); });
                    pn[c * NS + i] = pi;
                    vn[c * NS + i] = vi;
                    rwv[c] += (double)a.rw[c * NS + i] * (double)vi;
                }
            })
            if (!reduce<NR>(rwv, a, grp, rank, phase)) return;
#pragma unroll
            for (int c = 0; c < NR; ++c)
                if (active & (1 << c)) alpha[c] = rho[c] / rwv[c];
            // phase B: s = r - alpha v (in r), x += alpha p, |s|^2
            double ss[NR];
#pragma unroll
            for (int c = 0; c < NR; ++c) ss[c] = 0.0;
            KR_FOR_CELLS({
#pragma unroll
                for (int c = 0; c < NR; ++c) {
                    if (!(active & (1 << c))) continue;
                    const T al = (T)alpha[c];
                    const T si = a.r[c * NS + i] - al * vn[c * NS + i];
                    a.r[c * NS + i] = si;
                    a.x[c * NS + i] += al * pn[c * NS + i];
                    ss[c] += (double)si * (double)si;
                }
            })
            if (!reduce<NR>(ss, a, grp, rank, phase)) return;
#pragma unroll
            for (int c = 0; c < NR; ++c) {
                if (!(active & (1 << c))) continue;
                const double nr = conv_crit(ss[c], a.normalized, n);
                info[c].used_iterations = it;
                info[c].final_residual = nr;
                if (!isfinite(nr)) { info[c].finite = 0; active &= ~(1 << c); }
                else if (nr < a.tol) { info[c].converged = 1; active &= ~(1 << c); }
            }
            if (!active) break;
            // phase C: t = A s, t.s, t.t
            double ts[2 * NR];
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) ts[k] = 0.0;
            KR_FOR_CELLS({
#pragma unroll
                for (int c = 0; c < NR; ++c) {
                    if (!(active & (1 << c))) continue;
                    const T* sc = a.r + c * NS;
                    const T ti = spmv_row<T, D, TRANS>(dom, coef, N, i, B, p, [&](int j) { return sc[j]; });
                    a.t[c * NS + i] = ti;
                    ts[2 * c] += (double)ti * (double)sc[i];
                    ts[2 * c + 1] += (double)ti * (double)ti;
                }
            })
            if (!reduce<2 * NR>(ts, a, grp, rank, phase)) return;
#pragma unroll
            for (int c = 0; c < NR; ++c)
                if (active & (1 << c)) omega[c] = ts[2 * c] / ts[2 * c + 1];
            // phase D: x += omega s, r = s - omega t, r.r, rw.r
            double rr[2 * NR];
#pragma unroll
            for (int k = 0; k < 2 * NR; ++k) rr[k] = 0.0;
            KR_FOR_CELLS({
#pragma unroll
                for (int c = 0; c < NR; ++c) {
                    if (!(active & (1 << c))) continue;
                    const T om = (T)omega[c];
                    const T si = a.r[c * NS + i];
                    a.x[c * NS + i] += om * si;
                    const T ri = si - om * a.t[c * NS + i];
                    a.r[c * NS + i] = ri;
                    rr[2 * c] += (double)ri * (double)ri;
                    rr[2 * c + 1] += (double)a.rw[c * NS + i] * (double)ri;
                }
            })
            if (!reduce<2 * NR>(rr, a, grp, rank, phase)) return;
#pragma unroll
            for (int c = 0; c < NR; ++c) {
                if (!(active & (1 << c))) continue;
                rwr[c] = rr[2 * c + 1];
                const double nr = conv_crit(rr[2 * c], a.normalized, n);
                info[c].final_residual = nr;
                if (nr < a.tol) {
                    info[c].converged = 1;
                    info[c].used_iterations = it + 1;
                    active &= ~(1 << c);
                }
            }
            T* tp = pc; pc = pn; pn = tp;
            T* tv = vc; vc = vn; vn = tv;
        }
        if (rank == 0 && threadIdx.x == 0) {
#pragma unroll
            for (int c = 0; c < NR; ++c) a.info[s * a.nrhs + c] = info[c];
        }
        __syncthreads();
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
__global__ void k_finish_info(pict_solve_info_t* info, int n, const int* err) {
    if (*err == 0) return;
    PICT_CELL_LOOP(i, n) { info[i].status = 1; info[i].converged = 0; }
}

// ---------------------------------------------------------------------------------------------
// host side: launch plan and workspace
// ---------------------------------------------------------------------------------------------

struct Plan {
    int threads;
    int G;
    int ngroups;
    bool coop;
    int nvec;
    int nrhs_launch;  // right-hand sides per launch
    size_t header_bytes;
    size_t vec_bytes;
    size_t total;
};

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Workspace header sized for the largest possible plan (32 CTAs per SM), so its layout does not
// depend on the occupancy-derived plan: [queue, err] | group_sys[NG] | sync[NG][32] | partials.
static int max_ctas() { return device_sm_count() * 32; }
static int max_groups(const pict_domain_t* dom) { return dom->num_sims < max_ctas() ? dom->num_sims : max_ctas(); }
static size_t off_group_sys() { return align256(256); }
static size_t off_sync(const pict_domain_t* dom) { return off_group_sys() + align256(sizeof(int) * max_groups(dom)); }
static size_t off_partials(const pict_domain_t* dom) { return off_sync(dom) + align256(sizeof(unsigned) * 32 * max_groups(dom)); }
static size_t header_bytes(const pict_domain_t* dom) {
    return off_partials(dom) + align256(sizeof(double) * 2 * (size_t)max_ctas() * KR_NV);
}

template <typename KernelT>
static int max_coresident(KernelT kernel, int threads) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    return per_sm * device_sm_count();
}

static Plan make_plan(const pict_domain_t* dom, const pict_solve_params_t* prm, int coresident) {
    Plan P;
    const size_t esz = dom->dtype == PICT_F64 ? 8 : 4;
    P.nrhs_launch = prm->use_bicg ? (prm->nrhs > 3 ? 3 : prm->nrhs) : 1;
    P.threads = prm->threads > 0 ? (prm->threads > 512 ? 512 : prm->threads) : 512;
    int G = prm->group_size;
    if (G <= 0) {
        const int target = P.threads * 8;
        G = (dom->max_sim_cells + target - 1) / target;
        if (dom->num_sims > 1) {
            const int share = coresident / dom->num_sims;
            if (G > share) G = share;
        }
    }
    if (G < 1) G = 1;
    if (G > coresident) G = coresident;
    P.G = G;
    if (G == 1) {
        P.ngroups = dom->num_sims < coresident ? dom->num_sims : coresident;
        P.coop = false;
    } else {
        int ng = coresident / G;
        if (ng > dom->num_sims) ng = dom->num_sims;
        if (ng < 1) ng = 1;
        P.ngroups = ng;
        P.coop = true;
    }
    if (P.ngroups < 1) P.ngroups = 1;
    P.nvec = prm->use_bicg ? 7 : 4;  // bicg: r rw p0 p1 v0 v1 t; cg: r p0 p1 q
    P.header_bytes = header_bytes(dom);
    P.vec_bytes = align256(esz * (size_t)dom->num_cells * P.nrhs_launch);
    P.total = P.header_bytes + P.vec_bytes * P.nvec;
    return P;
}

template <typename T, int D, bool TRANS>
static int coresident_for(const pict_solve_params_t* prm, int threads) {
    if (prm->use_bicg) {
        const int nr = prm->nrhs >= 3 ? 3 : prm->nrhs;
        if (nr == 1) return max_coresident(k_bicgstab<T, D, 1, TRANS>, threads);
        if (nr == 2) return max_coresident(k_bicgstab<T, D, 2, TRANS>, threads);
        return max_coresident(k_bicgstab<T, D, 3, TRANS>, threads);
    }
    return max_coresident(k_cg<T, D, TRANS>, threads);
}

template <typename T>
static pict_status_t launch_kernel(void (*kernel)(KArgs<T>), const Plan& P, KArgs<T>& args, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P.ngroups * P.G);
    cfg.blockDim = dim3(P.threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = P.coop ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, args);
    if (e != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof(buf), "krylov launch (grid %d x %d threads, coop %d): %s", P.ngroups * P.G, P.threads,
                 (int)P.coop, cudaGetErrorString(e));
        cudaGetLastError();
        return set_error(PICT_ERR_CUDA, buf);
    }
    return PICT_OK;
}

template <typename T, int D, bool TRANS>
static pict_status_t run_solve(const pict_domain_t* dom, const void* coef, const void* rhs, void* x,
                               const pict_solve_params_t* prm, void* info_out, void* ws, int64_t ws_bytes,
                               cudaStream_t st) {
    const int threads = prm->threads > 0 ? (prm->threads > 512 ? 512 : prm->threads) : 512;
    const int cores = coresident_for<T, D, TRANS>(prm, threads);
    const Plan P = make_plan(dom, prm, cores);
    if ((int64_t)P.total > ws_bytes) return set_error(PICT_ERR_ARG, "solve: workspace too small");
    char* base = reinterpret_cast<char*>(ws);
    int* queue = reinterpret_cast<int*>(base);
    int* err = queue + 1;
    int* group_sys = reinterpret_cast<int*>(base + off_group_sys());
    unsigned* sync = reinterpret_cast<unsigned*>(base + off_sync(dom));
    double* partials = reinterpret_cast<double*>(base + off_partials(dom));
    const size_t off = P.header_bytes;
    T* vec[7];
    for (int k = 0; k < P.nvec; ++k) vec[k] = reinterpret_cast<T*>(base + off + P.vec_bytes * k);

    const int nrhs_total = prm->nrhs;
    pict_solve_info_t* info = reinterpret_cast<pict_solve_info_t*>(info_out);
    {
        const int ninfo = dom->num_sims * nrhs_total;
        k_init_info<<<cell_grid(ninfo, 128), 128, 0, st>>>(info, ninfo);
        pict_status_t s = check_launch("init_info");
        if (s) return s;
    }
    const size_t NS = (size_t)dom->num_cells;
    for (int c0 = 0; c0 < nrhs_total; c0 += P.nrhs_launch) {
        const int nr = (nrhs_total - c0) < P.nrhs_launch ? (nrhs_total - c0) : P.nrhs_launch;
        if (cudaMemsetAsync(base, 0, P.header_bytes, st) != cudaSuccess) return check_launch("workspace memset");
        KArgs<T> a;
        a.dom = *dom;
        a.coef = reinterpret_cast<const T*>(coef);
        a.b = reinterpret_cast<const T*>(rhs) + c0 * NS;
        a.x = reinterpret_cast<T*>(x) + c0 * NS;
        a.queue = queue;
        a.err = err;
        a.group_sys = group_sys;
        a.sync = sync;
        a.partials = partials;
        a.maxit = prm->max_iterations;
        a.tol = prm->tolerance;
        a.normalized = prm->convergence == PICT_CONV_NORM2_NORMALIZED;
        a.G = P.G;
        a.x_zero = prm->x_is_zero;
        a.sub_mean = prm->subtract_mean;
        a.write_bp = prm->write_block_pressure;
        pict_status_t s;
        if (prm->use_bicg) {
            a.r = vec[0]; a.rw = vec[1]; a.p0 = vec[2]; a.p1 = vec[3]; a.v0 = vec[4]; a.v1 = vec[5]; a.t = vec[6];
            // infos of this chunk: info[s*nrhs_total + c0 + c]; use a strided view via nrhs = nrhs_total
            a.info = info + c0;
            a.nrhs = nrhs_total;
            if (nr == 1) s = launch_kernel<T>(k_bicgstab<T, D, 1, TRANS>, P, a, st);
            else if (nr == 2) s = launch_kernel<T>(k_bicgstab<T, D, 2, TRANS>, P, a, st);
            else s = launch_kernel<T>(k_bicgstab<T, D, 3, TRANS>, P, a, st);
        } else {
            a.r = vec[0]; a.p0 = vec[1]; a.p1 = vec[2]; a.t = vec[3];
            a.rw = nullptr; a.v0 = nullptr; a.v1 = nullptr;
            a.info = info + c0;  // CG writes info[s] -> per-launch view; stride handled below
            a.nrhs = 1;
            if (nrhs_total == 1) {
                s = launch_kernel<T>(k_cg<T, D, TRANS>, P, a, st);
            } else {
                return set_error(PICT_ERR_UNSUPPORTED, "CG with several right-hand sides per system: split on the host");
            }
        }
        if (s) return s;
        k_finish_info<<<1, 128, 0, st>>>(info, dom->num_sims * nrhs_total, err);
        s = check_launch("finish_info");
        if (s) return s;
    }
    return PICT_OK;
}

}  // namespace pict

using namespace pict;

extern "C" {

int64_t pict_solve_workspace_bytes(const pict_domain_t* dom, const pict_solve_params_t* prm) {
    if (!dom || !prm) return -1;
    // vectors do not depend on the launch plan and the header is sized for the largest plan
    const Plan P = make_plan(dom, prm, max_ctas());
    const size_t t = P.total;
    return (int64_t)t;
}

pict_status_t pict_solve(const pict_domain_t* dom, const void* coef, const void* rhs, void* x,
                         const pict_solve_params_t* prm, void* info_out, void* ws, int64_t ws_bytes, void* stream) {
    if (!dom || !prm || !coef || !rhs || !x || !info_out || !ws) return set_error(PICT_ERR_ARG, "solve: NULL argument");
    if (dom->num_cells <= 0 || !dom->blocks || !dom->nbr || !dom->sim_cells || !dom->sim_blocks)
        return set_error(PICT_ERR_ARG, "solve: domain is not prepared");
    if (prm->nrhs < 1) return set_error(PICT_ERR_ARG, "solve: nrhs must be >= 1");
    if (prm->max_iterations < 0) return set_error(PICT_ERR_ARG, "solve: max_iterations must be >= 0");
    if (!(prm->convergence == PICT_CONV_NORM2 || prm->convergence == PICT_CONV_NORM2_NORMALIZED))
        return set_error(PICT_ERR_UNSUPPORTED, "solve: only NORM2 and NORM2_NORMALIZED convergence criteria are supported");
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
