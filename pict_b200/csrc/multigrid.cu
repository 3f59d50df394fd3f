// multigrid.cu -- multigrid-preconditioned CG for the pressure correction solve of the mixed precision
// step (no counterpart in the reference, whose pressure solve is unpreconditioned CG,
// extensions/cg_solver_kernel.cu:114-456).
//
// Scope: domains whose systems are single blocks with fixed or periodic faces (the batched cavities,
// the periodic channel and box).  Each level coarsens every block by 2 along the axes its coupling is
// strong in (semi-coarsening on stretched grids, full coarsening on isotropic ones; aggregates of up to
// 2^D cells, ceil(n/2) cells per coarsened axis); the coarse operator is the Galerkin product R A P with
// piecewise-constant prolongation P and R = P^T, computed on the device from the fine stencil.  The
// V-cycle uses one damped-Jacobi sweep before and after the coarse correction (symmetric), a fixed
// number of Jacobi sweeps on the coarsest level and a scaled prolongation (aggregation coarse
// operators are too stiff by about 2).  The constant mode of the singular (Neumann / periodic) block
// operators is removed on the coarsest level and from every preconditioned residual (folded into the
// inner products and into the search direction, which the SpMV forms on the fly).  The preconditioned CG runs a fixed number of iterations with
// per-system scalars; every inner product is reduced per work tile and then per system in a fixed
// order, so results do not depend on the launch shape.
#include <cmath>
#include <cstdio>
#include "common.cuh"
#include "launch.h"

namespace pict {

// block of a level: first cell, sizes, periodic flags, system, and the coarsening shifts (log2 of the
// factor, 0 or 1 per axis) from the next finer level
struct MgBlock {
    int off, sx, sy, sz, px, py, pz, sys, shx, shy, shz;
};

constexpr int MG_BT = 12;  // ints per block-table entry
constexpr int MG_SC = 6;   // per-system PCG scalars: rho, alpha, beta, |r|^2, mean(z), unused

__device__ __forceinline__ MgBlock mg_block(const pict_mg_level_t& L, int b) {
    const int* t = L.blocks + MG_BT * b;
    return MgBlock{t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], t[9], t[10]};
}

// neighbour across face f with its coordinates (q in: cell, out: neighbour); -1 at a fixed face
__device__ __forceinline__ int mg_nbr_q(const MgBlock& B, int* q, int f) {
    const int a = f >> 1;
    const int n[3] = {B.sx, B.sy, B.sz};
    const int per[3] = {B.px, B.py, B.pz};
    q[a] += (f & 1) ? 1 : -1;
    if (q[a] < 0 || q[a] >= n[a]) {
        if (!per[a]) return -1;
        q[a] = (q[a] + n[a]) % n[a];
    }
    return B.off + q[0] + B.sx * (q[1] + B.sy * q[2]);
}

// neighbour of local cell (x,y,z) across face f inside a block (periodic wrap, -1 at a fixed face)
__device__ __forceinline__ int mg_nbr(const MgBlock& B, int x, int y, int z, int f) {
    int q[3] = {x, y, z};
    return mg_nbr_q(B, q, f);
}

__device__ __forceinline__ void mg_unflatten(const MgBlock& B, int l, int& x, int& y, int& z) {
    x = l % B.sx;
    const int t = l / B.sx;
    y = t % B.sy;
    z = t / B.sy;
}

// y = A x on a level (stencil rows through the structured neighbours)
template <typename T, int D>
__device__ __forceinline__ T mg_apply(const pict_mg_level_t& L, const T* coef, const T* xv, int i, const MgBlock& B,
                                      int x, int y, int z) {
    const int N = L.num_cells;
    T acc = coef[i] * xv[i];
#pragma unroll
    for (int f = 0; f < 2 * D; ++f) {
        const int j = mg_nbr(B, x, y, z, f);
        if (j >= 0) acc += coef[(size_t)(f + 1) * N + i] * xv[j];
    }
    return acc;
}

// ---------------------------------------------------------------------------------------------
// Galerkin coarse operator: one thread per coarse cell, summing the couplings of its children
// ---------------------------------------------------------------------------------------------
template <typename T, int D>
__global__ void k_mg_galerkin(pict_mg_level_t F, pict_mg_level_t C) {
    const T* cf = reinterpret_cast<const T*>(F.coef);
    T* cc = reinterpret_cast<T*>(C.coef);
    const int Nc = C.num_cells, Nf = F.num_cells;
    PICT_CELL_LOOP(I, Nc) {
        const int b = C.cell_block[I];
        const MgBlock Bc = mg_block(C, b), Bf = mg_block(F, b);
        int X, Y, Z;
        mg_unflatten(Bc, I - Bc.off, X, Y, Z);
        T diag = 0, off[2 * D];
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) off[f] = 0;
        for (int dz = 0; dz < (1 << Bc.shz); ++dz)
            for (int dy = 0; dy < (1 << Bc.shy); ++dy)
                for (int dx = 0; dx < (1 << Bc.shx); ++dx) {
                    const int x = (X << Bc.shx) + dx, y = (Y << Bc.shy) + dy, z = (Z << Bc.shz) + dz;
                    if (x >= Bf.sx || y >= Bf.sy || z >= Bf.sz) continue;
                    const int i = Bf.off + x + Bf.sx * (y + Bf.sy * z);
                    diag += cf[i];
#pragma unroll
                    for (int f = 0; f < 2 * D; ++f) {
                        const int j = mg_nbr(Bf, x, y, z, f);
                        if (j < 0) continue;
                        int xj, yj, zj;
                        mg_unflatten(Bf, j - Bf.off, xj, yj, zj);
                        const int J = Bc.off + (xj >> Bc.shx) + Bc.sx * ((yj >> Bc.shy) + Bc.sy * (zj >> Bc.shz));
                        const T c = cf[(size_t)(f + 1) * Nf + i];
                        if (J == I) diag += c;
                        else off[f] += c;
                    }
                }
        cc[I] = diag;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) cc[(size_t)(f + 1) * Nc + I] = off[f];
    }
}

// x_out = x_in + w (b - A x_in) / diag   (x_in == nullptr: x_out = w b / diag)
template <typename T, int D>
__global__ void k_mg_jacobi(pict_mg_level_t L, const T* bv, const T* xin, T* xout, T w) {
    const T* coef = reinterpret_cast<const T*>(L.coef);
    PICT_CELL_LOOP(i, L.num_cells) {
        const T d = coef[i];
        const T rd = (d != T(0)) ? w / d : T(0);
        if (!xin) {
            xout[i] = rd * bv[i];
        } else {
            const MgBlock B = mg_block(L, L.cell_block[i]);
            int x, y, z;
            mg_unflatten(B, i - B.off, x, y, z);
            xout[i] = xin[i] + rd * (bv[i] - mg_apply<T, D>(L, coef, xin, i, B, x, y, z));
        }
    }
}

// b_c = R (b - A x) on the children of each coarse cell
template <typename T, int D>
__global__ void k_mg_residual_restrict(pict_mg_level_t F, pict_mg_level_t C, const T* bv, const T* xv, T* bc) {
    const T* cf = reinterpret_cast<const T*>(F.coef);
    PICT_CELL_LOOP(I, C.num_cells) {
        const int b = C.cell_block[I];
        const MgBlock Bc = mg_block(C, b), Bf = mg_block(F, b);
        int X, Y, Z;
        mg_unflatten(Bc, I - Bc.off, X, Y, Z);
        T acc = 0;
        for (int dz = 0; dz < (1 << Bc.shz); ++dz)
            for (int dy = 0; dy < (1 << Bc.shy); ++dy)
                for (int dx = 0; dx < (1 << Bc.shx); ++dx) {
                    const int x = (X << Bc.shx) + dx, y = (Y << Bc.shy) + dy, z = (Z << Bc.shz) + dz;
                    if (x >= Bf.sx || y >= Bf.sy || z >= Bf.sz) continue;
                    const int i = Bf.off + x + Bf.sx * (y + Bf.sy * z);
                    acc += bv[i] - mg_apply<T, D>(F, cf, xv, i, Bf, x, y, z);
                }
        bc[I] = acc;
    }
}

// prolongation fused into the post-smoothing sweep: with x' = x_f + s P e_c (formed on the fly for
// the neighbours), x_out = x' + w (b - A x') / diag
template <typename T, int D>
__global__ void k_mg_prolong_jacobi(pict_mg_level_t F, pict_mg_level_t C, const T* bv, const T* xf, const T* ec,
                                    T* xout, T s, T w) {
    const T* coef = reinterpret_cast<const T*>(F.coef);
    const int N = F.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = F.cell_block[i];
        const MgBlock Bf = mg_block(F, b), Bc = mg_block(C, b);
        int x, y, z;
        mg_unflatten(Bf, i - Bf.off, x, y, z);
        const T xi = xf[i] + s * ec[Bc.off + (x >> Bc.shx) + Bc.sx * ((y >> Bc.shy) + Bc.sy * (z >> Bc.shz))];
        const T d = coef[i];
        T acc = d * xi;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            int q[3] = {x, y, z};
            const int j = mg_nbr_q(Bf, q, f);
            if (j < 0) continue;
            const T xj = xf[j] + s * ec[Bc.off + (q[0] >> Bc.shx) + Bc.sx * ((q[1] >> Bc.shy) + Bc.sy * (q[2] >> Bc.shz))];
            acc += coef[(size_t)(f + 1) * N + i] * xj;
        }
        xout[i] = xi + ((d != T(0)) ? w * (bv[i] - acc) / d : T(0));
    }
}

// coarsest level: `sweeps` damped-Jacobi sweeps from zero and mean removal, one CTA per block with the
// iterate in shared memory (coarsest blocks hold at most MG_COARSE_MAX cells)
constexpr int MG_COARSE_MAX = 256;

template <typename T, int D>
__global__ void k_mg_coarse_solve(pict_mg_level_t L, const T* bv, T* xout, T w, int sweeps) {
    __shared__ T s_x[2][MG_COARSE_MAX];
    __shared__ double s_red[32];
    __shared__ double s_mean;
    const T* coef = reinterpret_cast<const T*>(L.coef);
    const int N = L.num_cells;
    const MgBlock B = mg_block(L, blockIdx.x);
    const int n = B.sx * B.sy * B.sz;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const T d = coef[B.off + k];
        s_x[0][k] = (d != T(0)) ? w * bv[B.off + k] / d : T(0);
    }
    __syncthreads();
    int cur = 0;
    for (int it = 1; it < sweeps; ++it) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const int i = B.off + k;
            int x, y, z;
            mg_unflatten(B, k, x, y, z);
            T acc = coef[i] * s_x[cur][k];
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                const int j = mg_nbr(B, x, y, z, f);
                if (j >= 0) acc += coef[(size_t)(f + 1) * N + i] * s_x[cur][j - B.off];
            }
            const T d = coef[i];
            s_x[cur ^ 1][k] = s_x[cur][k] + ((d != T(0)) ? w * (bv[i] - acc) / d : T(0));
        }
        __syncthreads();
        cur ^= 1;
    }
    double acc = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) acc += (double)s_x[cur][k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) v += s_red[wv];
        s_mean = v / (double)n;
    }
    __syncthreads();
    const T m = (T)s_mean;
    for (int k = threadIdx.x; k < n; k += blockDim.x) xout[B.off + k] = s_x[cur][k] - m;
}

// ---------------------------------------------------------------------------------------------
// PCG vector kernels on the finest level; per-system scalars in FP64
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double mg_cta_sum(double v, double* s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    return r;
}

// p_new = (z - m) + beta p_old formed on the fly (also for the neighbours), q = A p_new, and the tile
// partial of p_new.q (one CTA per work tile of the domain); m, beta per system from sc
template <typename T, int D>
__global__ void k_pcg_spmv_dot(pict_domain_t dom, pict_mg_level_t L, const T* z, const T* pold, T* pnew, T* q,
                               const double* sc, double* part) {
    __shared__ double s_red[32];
    const T* coef = reinterpret_cast<const T*>(L.coef);
    const int N = L.num_cells;
    const int t = blockIdx.x;
    const int sys = dom.tiles[4 * t], s0 = dom.tiles[4 * t + 2], cnt = dom.tiles[4 * t + 3];
    const MgBlock B = mg_block(L, dom.tiles[4 * t + 1]);
    const T m = (T)sc[MG_SC * sys + 4], bt = (T)sc[MG_SC * sys + 2];
    double acc = 0.0;
    for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) {
        int x, y, z3;
        mg_unflatten(B, i - B.off, x, y, z3);
        const T pi = (z[i] - m) + bt * pold[i];
        T qi = coef[i] * pi;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int j = mg_nbr(B, x, y, z3, f);
            if (j >= 0) qi += coef[(size_t)(f + 1) * N + i] * ((z[j] - m) + bt * pold[j]);
        }
        pnew[i] = pi;
        q[i] = qi;
        acc += (double)pi * (double)qi;
    }
    acc = mg_cta_sum(acc, s_red);
    if (threadIdx.x == 0) part[t] = acc;
}

// tile partials of r.z, r.r, sum(z), sum(r)
template <typename T>
__global__ void k_pcg_dot4(pict_domain_t dom, const T* r, const T* z, double* part) {
    __shared__ double s_red[32];
    const int t = blockIdx.x;
    const int s0 = dom.tiles[4 * t + 2], cnt = dom.tiles[4 * t + 3];
    double a = 0.0, c = 0.0, sz = 0.0, sr = 0.0;
    for (int i = s0 + threadIdx.x; i < s0 + cnt; i += blockDim.x) {
        const double ri = (double)r[i], zi = (double)z[i];
        a += ri * zi;
        c += ri * ri;
        sz += zi;
        sr += ri;
    }
    a = mg_cta_sum(a, s_red);
    c = mg_cta_sum(c, s_red);
    sz = mg_cta_sum(sz, s_red);
    sr = mg_cta_sum(sr, s_red);
    if (threadIdx.x == 0) {
        part[4 * t] = a;
        part[4 * t + 1] = c;
        part[4 * t + 2] = sz;
        part[4 * t + 3] = sr;
    }
}

// per-system scalars (one warp per system, tiles summed lane-strided in a fixed order):
// stage 0: rho = r.(z - m), |r|^2, m = mean(z);  stage 1: alpha = rho / p.q;
// stage 2: rho' = r.(z - m), beta = rho'/rho, rho = rho', |r|^2, m
// The preconditioned residual z is used mean-free (z - m): the constant mode of a singular system is
// undetermined.  sc[s*MG_SC + {0: rho, 1: alpha, 2: beta, 3: |r|^2, 4: m}]

__global__ void k_pcg_scalars(pict_domain_t dom, const double* part, int stride, int stage, double* sc) {
    const int lane = threadIdx.x & 31;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= dom.num_sims) return;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = dom.sim_tiles[s] + lane; t < dom.sim_tiles[s + 1]; t += 32)
        for (int k = 0; k < stride; ++k) v[k] += part[(size_t)stride * t + k];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane != 0) return;
    double* S = sc + MG_SC * s;
    if (stage == 1) {
        const double a = v[0];
        S[1] = (a != 0.0 && S[0] != 0.0 && isfinite(a)) ? S[0] / a : 0.0;
        return;
    }
    const int n = dom.sim_cells[s + 1] - dom.sim_cells[s];
    const double m = v[2] / (double)n;
    const double rho = v[0] - m * v[3];
    if (stage == 0) {
        S[2] = 0.0;
    } else {
        S[2] = (S[0] != 0.0 && isfinite(rho)) ? rho / S[0] : 0.0;
    }
    S[0] = rho;
    S[3] = v[1];
    S[4] = m;
}

template <typename T>
__device__ __forceinline__ int cell_sys(const pict_domain_t& dom, int i) { return dom.blocks[dom.cell_block[i]].sim; }

// x += alpha p, r -= alpha q, and the first pre-smoothing sweep of the next V-cycle on the finest
// level: x0 = w r / diag
template <typename T>
__global__ void k_pcg_update_xr(pict_domain_t dom, pict_mg_level_t L, T* x, T* r, const T* p, const T* q,
                                const double* sc, T* x0, T w) {
    const T* coef = reinterpret_cast<const T*>(L.coef);
    PICT_CELL_LOOP(i, dom.num_cells) {
        const T al = (T)sc[MG_SC * cell_sys<T>(dom, i) + 1];
        x[i] += al * p[i];
        const T ri = r[i] - al * q[i];
        r[i] = ri;
        const T d = coef[i];
        x0[i] = (d != T(0)) ? w * ri / d : T(0);
    }
}

// r = b, x = 0, search directions 0
template <typename T>
__global__ void k_pcg_init(int N, const T* b, T* r, T* x, T* p0, T* p1) {
    PICT_CELL_LOOP(i, N) {
        r[i] = b[i];
        x[i] = T(0);
        p0[i] = T(0);
        p1[i] = T(0);
    }
}

__global__ void k_pcg_report(pict_domain_t dom, const double* sc, pict_solve_info_t* info, int iterations, double tol,
                             int normalized) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= dom.num_sims) return;
    const int n = dom.sim_cells[s + 1] - dom.sim_cells[s];
    const double nrm = sqrt(sc[MG_SC * s + 3]);
    const double crit = normalized ? nrm / sqrt((double)n) : nrm;
    pict_solve_info_t inf;
    inf.final_residual = crit;
    inf.used_iterations = iterations;
    inf.finite = isfinite(crit) ? 1 : 0;
    inf.converged = (inf.finite && crit < tol) ? 1 : 0;
    inf.status = 0;
    info[s] = inf;
}

template <typename T>
static size_t vbytes(int n) { return ((size_t)n * sizeof(T) + 255) & ~(size_t)255; }

// workspace: per level x0, x1, b (levels >= 1; level 0: x0, x1) | r, z, p, q | partials | scalars
template <typename T, int D>
static pict_status_t run_pcg_mg(const pict_domain_t* dom, const pict_mg_level_t* levels, int nl, const T* rhs, T* xout,
                                int iterations, double tol, int normalized, pict_solve_info_t* info, char* ws,
                                int64_t ws_bytes, double omega, double scale, int coarse_sweeps, cudaStream_t st) {
    const int N = dom->num_cells;
    // carve the workspace
    char* w = ws;
    T* lx0[16];
    T* lx1[16];
    T* lb[16];
    for (int l = 0; l < nl; ++l) {
        const int n = levels[l].num_cells;
        lx0[l] = reinterpret_cast<T*>(w); w += vbytes<T>(n);
        lx1[l] = reinterpret_cast<T*>(w); w += vbytes<T>(n);
        lb[l] = reinterpret_cast<T*>(w); w += vbytes<T>(n);
    }
    T* r = reinterpret_cast<T*>(w); w += vbytes<T>(N);
    T* z = reinterpret_cast<T*>(w); w += vbytes<T>(N);
    T* p = reinterpret_cast<T*>(w); w += vbytes<T>(N);
    T* q = reinterpret_cast<T*>(w); w += vbytes<T>(N);
    double* part = reinterpret_cast<double*>(w); w += ((size_t)4 * dom->num_tiles * 8 + 255) & ~(size_t)255;
    double* sc = reinterpret_cast<double*>(w); w += ((size_t)MG_SC * dom->num_sims * 8 + 255) & ~(size_t)255;
    if ((int64_t)(w - ws) > ws_bytes) return set_error(PICT_ERR_ARG, "pcg_mg: workspace too small");

    auto grid_of = [](int n) { return cell_grid(n, 256); };
    const T wj = (T)omega, sp = (T)scale;
    // z = M r (V-cycle); r is the finest right-hand side.  presmoothed: the first finest sweep
    // (lx0[0] = w r / diag) was already written by the x/r update.  Every level's corrected iterate
    // ends in lx1 (lx0 on the coarsest), so the prolongation reads it without copies.
    auto vcycle = [&](const T* rhs0, T* z0, bool presmoothed) -> pict_status_t {
        const T* b = rhs0;
        for (int l = 0; l < nl; ++l) {
            const pict_mg_level_t& L = levels[l];
            if (l > 0) b = lb[l];
            if (l == nl - 1) {
                // coarsest: Jacobi sweeps from zero and mean removal in one launch, result in lx0
                k_mg_coarse_solve<T, D><<<L.num_blocks, 64, 0, st>>>(L, b, lx0[l], wj, coarse_sweeps);
                break;
            }
            if (l > 0 || !presmoothed) k_mg_jacobi<T, D><<<grid_of(L.num_cells), 256, 0, st>>>(L, b, nullptr, lx0[l], wj);
            k_mg_residual_restrict<T, D><<<grid_of(levels[l + 1].num_cells), 256, 0, st>>>(L, levels[l + 1], b, lx0[l], lb[l + 1]);
        }
        const T* ec = lx0[nl - 1];
        for (int l = nl - 2; l >= 0; --l) {
            const pict_mg_level_t& L = levels[l];
            const T* bl = (l == 0) ? rhs0 : lb[l];
            T* dst = (l == 0) ? z0 : lx1[l];
            k_mg_prolong_jacobi<T, D><<<grid_of(L.num_cells), 256, 0, st>>>(L, levels[l + 1], bl, lx0[l], ec, dst, sp, wj);
            ec = dst;
        }
        if (nl == 1) cudaMemcpyAsync(z0, lx0[0], sizeof(T) * N, cudaMemcpyDeviceToDevice, st);
        return check_launch("pcg_mg vcycle");
    };

    // search directions alternate between p and pb; each is formed from z inside the SpMV
    T* pb = lx1[0];
    const int nt = dom->num_tiles;
    const int sg = (dom->num_sims + 127) / 128;
    const int swg = (dom->num_sims * 32 + 127) / 128;  // one warp per system
    k_pcg_init<T><<<grid_of(N), 256, 0, st>>>(N, rhs, r, xout, p, pb);
    pict_status_t s = vcycle(r, z, false);
    if (s) return s;
    k_pcg_dot4<T><<<nt, 256, 0, st>>>(*dom, r, z, part);
    k_pcg_scalars<<<swg, 128, 0, st>>>(*dom, part, 4, 0, sc);
    for (int it = 0; it < iterations; ++it) {
        k_pcg_spmv_dot<T, D><<<nt, 256, 0, st>>>(*dom, levels[0], z, p, pb, q, sc, part);
        k_pcg_scalars<<<swg, 128, 0, st>>>(*dom, part, 1, 1, sc);
        k_pcg_update_xr<T><<<grid_of(N), 256, 0, st>>>(*dom, levels[0], xout, r, pb, q, sc, lx0[0], wj);
        const bool last = it + 1 == iterations;
        if (!last) {
            s = vcycle(r, z, true);
            if (s) return s;
        }
        // on the last iteration only |r|^2 is used (r.z and sum(z) of the stale z are ignored)
        k_pcg_dot4<T><<<nt, 256, 0, st>>>(*dom, r, z, part);
        k_pcg_scalars<<<swg, 128, 0, st>>>(*dom, part, 4, 2, sc);
        T* tmp = p; p = pb; pb = tmp;
    }
    k_pcg_report<<<sg, 128, 0, st>>>(*dom, sc, info, iterations, tol, normalized);
    return check_launch("pcg_mg");
}

}  // namespace pict

using namespace pict;

extern "C" {

pict_status_t pict_mg_galerkin(const pict_mg_level_t* fine, const pict_mg_level_t* coarse, void* stream) {
    if (!fine || !coarse || !fine->coef || !coarse->coef || !fine->blocks || !coarse->blocks || !coarse->cell_block)
        return set_error(PICT_ERR_ARG, "mg_galerkin: NULL argument");
    if (fine->num_blocks != coarse->num_blocks || fine->dims != coarse->dims || fine->dtype != coarse->dtype)
        return set_error(PICT_ERR_ARG, "mg_galerkin: level mismatch");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(coarse->num_cells, 256);
    if (fine->dtype == PICT_F32) {
        if (fine->dims == 2) k_mg_galerkin<float, 2><<<grid, 256, 0, st>>>(*fine, *coarse);
        else k_mg_galerkin<float, 3><<<grid, 256, 0, st>>>(*fine, *coarse);
    } else {
        if (fine->dims == 2) k_mg_galerkin<double, 2><<<grid, 256, 0, st>>>(*fine, *coarse);
        else k_mg_galerkin<double, 3><<<grid, 256, 0, st>>>(*fine, *coarse);
    }
    return check_launch("mg_galerkin");
}

int64_t pict_pcg_mg_workspace_bytes(const pict_domain_t* dom, const pict_mg_level_t* levels, int32_t num_levels) {
    if (!dom || !levels || num_levels < 1 || num_levels > 16) return -1;
    const size_t esz = dom->dtype == PICT_F64 ? 8 : 4;
    auto vb = [&](int n) { return ((size_t)n * esz + 255) & ~(size_t)255; };
    size_t b = 0;
    for (int l = 0; l < num_levels; ++l) b += 3 * vb(levels[l].num_cells);
    b += 4 * vb(dom->num_cells);
    b += ((size_t)4 * dom->num_tiles * 8 + 255) & ~(size_t)255;
    b += ((size_t)MG_SC * dom->num_sims * 8 + 255) & ~(size_t)255;
    return (int64_t)b;
}

pict_status_t pict_pcg_mg(const pict_domain_t* dom, const pict_mg_level_t* levels, int32_t num_levels, const void* rhs,
                          void* x, int32_t iterations, double tolerance, int32_t convergence, void* info_out,
                          void* workspace, int64_t workspace_bytes, double omega, double prolong_scale,
                          int32_t coarse_sweeps, void* stream) {
    if (!dom || !levels || !rhs || !x || !info_out || !workspace) return set_error(PICT_ERR_ARG, "pcg_mg: NULL argument");
    if (num_levels < 1 || num_levels > 16 || iterations < 0 || coarse_sweeps < 1)
        return set_error(PICT_ERR_ARG, "pcg_mg: bad level count / iterations / sweeps");
    if (levels[0].num_cells != dom->num_cells || levels[0].num_blocks != dom->num_blocks || !dom->tiles ||
        dom->num_tiles <= 0)
        return set_error(PICT_ERR_ARG, "pcg_mg: level 0 must describe the domain (and tiles are needed)");
    cudaStream_t st = (cudaStream_t)stream;
    const int norm = convergence == PICT_CONV_NORM2_NORMALIZED;
    char* ws = reinterpret_cast<char*>(workspace);
    pict_solve_info_t* info = reinterpret_cast<pict_solve_info_t*>(info_out);
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2)
            return run_pcg_mg<float, 2>(dom, levels, num_levels, (const float*)rhs, (float*)x, iterations, tolerance, norm,
                                        info, ws, workspace_bytes, omega, prolong_scale, coarse_sweeps, st);
        return run_pcg_mg<float, 3>(dom, levels, num_levels, (const float*)rhs, (float*)x, iterations, tolerance, norm,
                                    info, ws, workspace_bytes, omega, prolong_scale, coarse_sweeps, st);
    }
    if (dom->dims == 2)
        return run_pcg_mg<double, 2>(dom, levels, num_levels, (const double*)rhs, (double*)x, iterations, tolerance, norm,
                                     info, ws, workspace_bytes, omega, prolong_scale, coarse_sweeps, st);
    return run_pcg_mg<double, 3>(dom, levels, num_levels, (const double*)rhs, (double*)x, iterations, tolerance, norm,
                                 info, ws, workspace_bytes, omega, prolong_scale, coarse_sweeps, st);
}

}  // extern "C"
