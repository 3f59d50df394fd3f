// multigrid.cu -- multigrid-preconditioned CG for the pressure correction solve of the mixed precision
// step (no counterpart in the reference, whose pressure solve is unpreconditioned CG,
// extensions/cg_solver_kernel.cu:114-456).
//
// Scope: domains whose systems are single blocks with fixed or periodic faces (the batched cavities,
// the periodic channel and box).  Each level coarsens every block by 2 along the axes its coupling is
// strong in (semi-coarsening on stretched grids, full coarsening on isotropic ones; aggregates of up to
// 2^D cells, ceil(n/2) cells per coarsened axis); the coarse operator is the Galerkin product R A P with
// piecewise-constant prolongation P and R = P^T, computed on the device from the fine stencil.  The
// V-cycle uses two damped-Jacobi sweeps before and after the coarse correction (one on levels whose tiles
// cannot stage the halo rows of two; the same number before and after, so the preconditioner stays
// symmetric), a fixed number of Jacobi sweeps on the coarsest level and a scaled prolongation
// (aggregation coarse operators are too stiff by about 2).  The constant mode of the singular (Neumann / periodic) block
// operators is removed on the coarsest level and from every preconditioned residual (folded into the
// inner products and into the search direction, which the SpMV forms on the fly).  The preconditioned
// CG runs a fixed number of iterations with per-system scalars; every inner product is reduced per warp
// of a work tile and then per system in a fixed order, so results do not depend on the launch shape.
//
// Launch structure of one PCG iteration: SpMV (+ direction update, p.q partials); scalars; the finest
// restriction with the x/r update fused in; the restrictions of the next levels; the V-cycle below a
// size cutoff in one CTA per block (shared memory); the prolongations up to level 1; the finest
// prolongation with the r.z partials fused in; scalars.  The pre-smoothing sweep from zero is never
// stored: x0 = w b / diag is formed where it is read.
#include <cmath>
#include <cstdio>
#include "bulk.cuh"
#include "common.cuh"
#include "launch.h"

namespace pict {

// 1: 2D PCG SpMV with bulk-copy staging where it applies (default); 0: the gather kernel only
static int g_mg_bulk = 1;
// cap on the damped-Jacobi sweeps of each smoothing step: 2 (default) where a level allows it, 1 everywhere
static int g_mg_sweeps = 2;
// 1 (default): under stream capture the PCG iterations after the first become a conditional WHILE node of the
// graph that stops once every system has converged; 0: the fixed launch sequence of `iterations` iterations
static int g_mg_graph_loop = 1;
// per device: the stream the loop body is captured on (created outside capture, on the first solve)
static cudaStream_t g_mg_body_stream[64];
// 1 (default): the PCG loop's kernels are launched with programmatic stream serialization (each waits for its
// predecessor in mg_pdl_entry); 0: plain launches
static int g_mg_pdl = 1;

template <typename... KArgs, typename... Args>
static void mg_launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
    if (!g_mg_pdl) {
        k<<<grid, block, smem, st>>>(args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, args...);
}

// block of a level: first cell, sizes, periodic flags, system, and the coarsening shifts (log2 of the
// factor, 0 or 1 per axis) from the next finer level
struct MgBlock {
    int off, sx, sy, sz, px, py, pz, sys, shx, shy, shz;
};

constexpr int MG_BT = 12;  // ints per block-table entry
constexpr int MG_SC = 7;   // per-system PCG scalars: rho, alpha, beta, |r|^2, mean(z), done, update pending

// A system is done once its residual met the tolerance: sc[5] = iterations at that point + 1 (0 while
// iterating).  The kernels of later iterations skip the tiles / blocks of done systems, so their iterate
// and report stay those of the converged iteration.
__device__ __forceinline__ bool mg_done(const double* sc, int sys) { return sc && sc[MG_SC * sys + 5] != 0.0; }

// A system whose new residual |r - alpha q| met the tolerance at this iteration's scalar stage (before its
// V-cycle) is done with its update x += alpha p, r -= alpha q still to apply: the finest restriction (or the
// update kernel) applies it and skips the rest; the end-of-iteration scalar stage clears the flag.
__device__ __forceinline__ bool mg_pending(const double* sc, int sys) { return sc && sc[MG_SC * sys + 6] != 0.0; }

// First statement of every kernel of the PCG loop: wait for the previous kernel of the stream (its writes are
// visible after the wait), then let the next one launch (programmatic dependent launch: its CTAs are
// scheduled while this kernel's last CTAs run, and wait here in turn).  Without the launch attribute both are
// no-ops.
__device__ __forceinline__ void mg_pdl_entry() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

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

// ---------------------------------------------------------------------------------------------
// Tile kernels.  One CTA per work tile of a level ([system, block, first cell, count]); each thread
// handles MG_CPT cells of a pass with branch-free, independent loads.
// ---------------------------------------------------------------------------------------------
constexpr int MG_TPB = 256;
constexpr int MG_CPT = 2;
constexpr int MG_PASS = MG_TPB * MG_CPT;  // cells of one pass of a tile CTA
constexpr int MG_STAGE = 4096;            // cells of the shared-memory stage of the 2D tile kernels
constexpr int MG_NW = MG_TPB / 32;        // warps of a tile CTA (partial sums are written per warp)

struct MgTile {
    int sys, blk, s0, cnt;
};

__device__ __forceinline__ MgTile mg_tile(const int32_t* tiles, int t) {
    const int32_t* p = tiles + 4 * t;
    return MgTile{p[0], p[1], p[2], p[3]};
}

template <typename T>
__device__ __forceinline__ T mg_div(T a, T b);
template <>
__device__ __forceinline__ float mg_div<float>(float a, float b) { return __fdividef(a, b); }
template <>
__device__ __forceinline__ double mg_div<double>(double a, double b) { return a / b; }

// the pre-smoothing sweep from zero at a cell: x0 = w b / diag
template <typename T>
__device__ __forceinline__ T mg_x0(T d, T b, T w) {
    return (d != T(0)) ? mg_div(w * b, d) : T(0);
}

// The neighbours of a cell across its 2D faces, branch-free: where a fixed face has no neighbour the
// index is the cell itself and ok is false (its term is masked), so every gather load is unconditional
// and the loads of several cells can be in flight together.
template <int D>
struct MgNbrs {
    int j[2 * D];
    int c[2 * D][3];
    bool ok[2 * D];
};

template <int D>
__device__ __forceinline__ void mg_nbrs(const MgBlock& B, int x, int y, int z, MgNbrs<D>& nb) {
    const int p[3] = {x, y, z};
    const int n[3] = {B.sx, B.sy, B.sz};
    const int per[3] = {B.px, B.py, B.pz};
#pragma unroll
    for (int f = 0; f < 2 * D; ++f) {
        const int a = f >> 1;
        const int c = p[a];
        int v;
        bool ok;
        if (f & 1) {
            ok = c + 1 < n[a] || per[a];
            v = c + 1 < n[a] ? c + 1 : (per[a] ? 0 : c);
        } else {
            ok = c > 0 || per[a];
            v = c > 0 ? c - 1 : (per[a] ? n[a] - 1 : c);
        }
        int q[3] = {x, y, z};
        q[a] = v;
        nb.c[f][0] = q[0];
        nb.c[f][1] = q[1];
        nb.c[f][2] = q[2];
        nb.ok[f] = ok;
        nb.j[f] = B.off + q[0] + B.sx * (q[1] + B.sy * q[2]);
    }
}

// right-hand side of the finest V-cycle at a cell: r, or r - alpha q when the PCG update is fused
template <typename T, bool UPD>
struct MgRhs {
    const T* __restrict__ r;
    const T* __restrict__ q;
    T al;
    __device__ __forceinline__ T operator()(int j) const { return UPD ? r[j] - al * q[j] : r[j]; }
};

__device__ __forceinline__ int mg_coarse_index(const MgBlock& Bc, int x, int y, int z) {
    return Bc.off + (x >> Bc.shx) + Bc.sx * ((y >> Bc.shy) + Bc.sy * (z >> Bc.shz));
}

__device__ __forceinline__ double mg_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// this warp's slot of the partial sums: part[(tile * MG_NW + warp) * stride ..]
__device__ __forceinline__ double* mg_warp_part(double* part, int stride) {
    return part + ((size_t)blockIdx.x * MG_NW + (threadIdx.x >> 5)) * stride;
}

// b_c = R (b - A x_s) over the children of each coarse cell, x_s the pre-smoothed iterate: x0 (nu = 1) or
// x1 = x0 + w (b - A x0) / diag (nu = 2), both from zero.  UPD (finest level): b = r - alpha q is formed on
// the fly and stored to rn, and x += alpha p (x = alpha p when first) for the children.
//
// 2D tiles whose fine rows (children rows plus nu halo rows on each side) fit the stage (cap cells) take
// the staged path: b and diag of those rows go to shared memory once, x_s is formed there, then each coarse
// cell sums its children's residuals from there (a y-periodic wrap, nu = 1 only, forms x0 of that
// neighbour from global).  nu = 2 is taken only where every tile of the level fits the stage.
template <typename T, int D, bool UPD>
__global__ void __launch_bounds__(MG_TPB, 4) k_mg_restrict(pict_mg_level_t F, pict_mg_level_t C,
                                                           const T* __restrict__ r, const T* __restrict__ q,
                                                           T* __restrict__ rn, T* __restrict__ x,
                                                           const T* __restrict__ p, const double* __restrict__ sc,
                                                           int first, T* __restrict__ bc, T w, int cap,
                                                           const double* __restrict__ dn, int nu) {
    mg_pdl_entry();
    extern __shared__ __align__(16) unsigned char mg_stage_raw[];
    const MgTile tl = mg_tile(C.tiles, blockIdx.x);
    const bool pend = UPD && mg_pending(sc, tl.sys);
    if (mg_done(dn, tl.sys) && !pend) return;
    const MgBlock Bc = mg_block(C, tl.blk), Bf = mg_block(F, tl.blk);
    const T* __restrict__ cf = reinterpret_cast<const T*>(F.coef);
    const int Nf = F.num_cells;
    const T al = UPD ? (T)sc[MG_SC * tl.sys + 1] : T(0);
    if (UPD && pend) {  // converged at this iteration: the update of the children, no restriction
        for (int k = threadIdx.x; k < tl.cnt; k += MG_TPB) {
            int X, Y, Z;
            mg_unflatten(Bc, tl.s0 + k - Bc.off, X, Y, Z);
#pragma unroll
            for (int c = 0; c < (1 << D); ++c) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
                const int xs = (X << Bc.shx) + dx, ys = (Y << Bc.shy) + dy, zs = (Z << Bc.shz) + dz;
                if ((dx && !Bc.shx) || (dy && !Bc.shy) || (dz && !Bc.shz) || xs >= Bf.sx || ys >= Bf.sy || zs >= Bf.sz)
                    continue;
                const int i = Bf.off + xs + Bf.sx * (ys + Bf.sy * zs);
                rn[i] = r[i] - al * q[i];
                x[i] = first ? al * p[i] : x[i] + al * p[i];
            }
        }
        return;
    }
    const MgRhs<T, UPD> rhs{r, q, al};
    const int sx = Bf.sx;
    int ylo = 0, yhi = -1;
    if (D == 2) {
        const int lc0 = tl.s0 - Bc.off, lc1 = lc0 + tl.cnt - 1;
        ylo = max(0, ((lc0 / Bc.sx) << Bc.shy) - nu);
        yhi = min(Bf.sy - 1, ((lc1 / Bc.sx + 1) << Bc.shy) - 1 + nu);
    }
    if (D == 2 && (yhi - ylo + 1) * sx <= cap) {
        T* s_x0 = reinterpret_cast<T*>(mg_stage_raw);  // x_s: x0 (nu = 1) or x1 (nu = 2)
        T* s_b = s_x0 + cap;
        T* s_d = s_b + cap;
        const int lo = Bf.off + ylo * sx, nh = (yhi - ylo + 1) * sx;
        const int lc0 = tl.s0 - Bc.off, lc1 = lc0 + tl.cnt - 1;
        const int dq = MG_TPB / sx, dr = MG_TPB - dq * sx;
        int yy = (int)threadIdx.x / sx, xx = (int)threadIdx.x - yy * sx;
        yy += ylo;
        for (int e = threadIdx.x; e < nh; e += MG_TPB) {
            const int i = lo + e;
            const T bi = rhs(i), di = cf[i];
            if (nu == 1) {
                s_x0[e] = mg_x0(di, bi, w);
                s_d[e] = di;
            } else {
                s_d[e] = (di != T(0)) ? mg_div(w, di) : T(0);  // w / diag
            }
            s_b[e] = bi;
            if (UPD) {
                const int par = (xx >> Bc.shx) + Bc.sx * (yy >> Bc.shy);
                if (par >= lc0 && par <= lc1) {
                    rn[i] = bi;
                    x[i] = first ? al * p[i] : x[i] + al * p[i];
                }
            }
            xx += dr;
            yy += dq;
            if (xx >= sx) {
                xx -= sx;
                ++yy;
            }
        }
        __syncthreads();
        if (nu == 2) {
            // x1 = x0 + w (b - A x0) / diag on the stage, x0 = (w / diag) b formed from the staged b and w / diag.
            // Rows of the stage's edge whose outer neighbour row lies outside the stage get a value that no
            // child reads (children rows are at least one row inside); the block's own edges are fixed faces.
            auto x0s = [&](int c) { return s_d[c] * s_b[c]; };
            int ey = (int)threadIdx.x / sx, ex = (int)threadIdx.x - ey * sx;
            for (int e = threadIdx.x; e < nh; e += MG_TPB) {
                const int i = lo + e, yg = ylo + ey;
                const T di = cf[i], xi = x0s(e);
                const T xm = ex > 0 ? x0s(e - 1) : x0s(e + sx - 1);
                const T xp = ex + 1 < sx ? x0s(e + 1) : x0s(e - sx + 1);
                const bool hm = ey > 0, hp = ey + 1 < nh / sx;
                const T ym = hm ? x0s(e - sx) : T(0), yp = hp ? x0s(e + sx) : T(0);
                T ax = di * xi;
                ax += (ex > 0 || Bf.px) ? cf[(size_t)Nf + i] * xm : T(0);
                ax += (ex + 1 < sx || Bf.px) ? cf[(size_t)2 * Nf + i] * xp : T(0);
                ax += (yg > 0 && hm) ? cf[(size_t)3 * Nf + i] * ym : T(0);
                ax += (yg + 1 < Bf.sy && hp) ? cf[(size_t)4 * Nf + i] * yp : T(0);
                s_x0[e] = xi + s_d[e] * (s_b[e] - ax);
                ex += dr;
                ey += dq;
                if (ex >= sx) {
                    ex -= sx;
                    ++ey;
                }
            }
            __syncthreads();
        }
        auto far = [&](int xq, int yq) -> T {
            const int j = Bf.off + xq + sx * yq;
            return mg_x0(cf[j], rhs(j), w);
        };
        const int dqc = MG_TPB / Bc.sx, drc = MG_TPB - dqc * Bc.sx;
        const int l = lc0 + (int)threadIdx.x;
        int Y = l / Bc.sx, X = l - Y * Bc.sx;
        for (int k = threadIdx.x; k < tl.cnt; k += MG_TPB) {
            T acc = T(0);
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) {
                const int dx = ch & 1, dy = ch >> 1;
                const int xs = (X << Bc.shx) + dx, ys = (Y << Bc.shy) + dy;
                const bool valid = !((dx && !Bc.shx) || (dy && !Bc.shy)) && xs < sx && ys < Bf.sy;
                if (!valid) continue;
                const int i = Bf.off + xs + sx * ys, c = (ys - ylo) * sx + xs;
                const T xi = s_x0[c];
                const T xm = xs > 0 ? s_x0[c - 1] : s_x0[c + sx - 1];
                const T xp = xs + 1 < sx ? s_x0[c + 1] : s_x0[c - sx + 1];
                const T ym = ys > 0 ? s_x0[c - sx] : (Bf.py ? far(xs, Bf.sy - 1) : T(0));
                const T yp = ys + 1 < Bf.sy ? s_x0[c + sx] : (Bf.py ? far(xs, 0) : T(0));
                T ax = (nu == 2 ? cf[i] : s_d[c]) * xi;
                ax += (xs > 0 || Bf.px) ? cf[(size_t)Nf + i] * xm : T(0);
                ax += (xs + 1 < sx || Bf.px) ? cf[(size_t)2 * Nf + i] * xp : T(0);
                ax += (ys > 0 || Bf.py) ? cf[(size_t)3 * Nf + i] * ym : T(0);
                ax += (ys + 1 < Bf.sy || Bf.py) ? cf[(size_t)4 * Nf + i] * yp : T(0);
                acc += s_b[c] - ax;
            }
            bc[tl.s0 + k] = acc;
            X += drc;
            Y += dqc;
            if (X >= Bc.sx) {
                X -= Bc.sx;
                ++Y;
            }
        }
        return;
    }
    for (int base = 0; base < tl.cnt; base += MG_PASS) {
        T acc[MG_CPT];
#pragma unroll
        for (int k = 0; k < MG_CPT; ++k) {
            const int l0 = base + k * MG_TPB + (int)threadIdx.x;
            const bool live = l0 < tl.cnt;
            const int l = live ? l0 : tl.cnt - 1;
            int X, Y, Z;
            mg_unflatten(Bc, tl.s0 + l - Bc.off, X, Y, Z);
            acc[k] = T(0);
#pragma unroll
            for (int c = 0; c < (1 << D); ++c) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
                int xs = (X << Bc.shx) + dx, ys = (Y << Bc.shy) + dy, zs = (Z << Bc.shz) + dz;
                const bool valid = !((dx && !Bc.shx) || (dy && !Bc.shy) || (dz && !Bc.shz)) && xs < Bf.sx &&
                                   ys < Bf.sy && zs < Bf.sz;
                if (!valid) {  // the first child always exists
                    xs = X << Bc.shx;
                    ys = Y << Bc.shy;
                    zs = Z << Bc.shz;
                }
                const int i = Bf.off + xs + Bf.sx * (ys + Bf.sy * zs);
                MgNbrs<D> nb;
                mg_nbrs<D>(Bf, xs, ys, zs, nb);
                const T bi = rhs(i);
                const T di = cf[i];
                T ax = di * mg_x0(di, bi, w);
#pragma unroll
                for (int f = 0; f < 2 * D; ++f) {
                    const T cj = cf[(size_t)(f + 1) * Nf + i];
                    const T xj = mg_x0(cf[nb.j[f]], rhs(nb.j[f]), w);
                    ax += nb.ok[f] ? cj * xj : T(0);
                }
                if (UPD && valid && live) {
                    rn[i] = bi;
                    x[i] = first ? al * p[i] : x[i] + al * p[i];
                }
                acc[k] += valid ? bi - ax : T(0);
            }
        }
#pragma unroll
        for (int k = 0; k < MG_CPT; ++k) {
            const int l = base + k * MG_TPB + (int)threadIdx.x;
            if (l < tl.cnt) bc[tl.s0 + l] = acc[k];
        }
    }
}

// post-smoothing with the coarse correction: x' = x_s + s P e_c (formed on the fly, also for the
// neighbours), then nu damped-Jacobi sweeps x <- x + w (b - A x) / diag.  x_s is the pre-smoothed iterate
// of the restriction, recomputed here: x0 = w b / diag (nu = 1) or x1 = x0 + w (b - A x0) / diag (nu = 2).
// DOT (finest level): per-warp partials of b.out, b.b, sum(out), sum(b).
//
// 2D tiles take a staged path where their rows plus the halo rows fit the stage.
// nu = 1 (cap cells per array): x' of every cell of [first - sx, last + sx] is formed once into shared memory (with b and diag),
// then the stencil reads its neighbours there; a y-periodic wrap reaches outside the stage and forms x'
// of that neighbour from global memory.  nu = 2: b and diag of [first - 3 sx, last + 3 sx] are staged,
// x1 (the pre-smoothed iterate) of [first - 2 sx, last + 2 sx], then the first post sweep of
// [first - sx, last + sx] (x' formed from x1 and e_c on the fly), then the second sweep of the tile's
// cells, in four arrays of 3 cap / 4 cells; taken only where every tile of the level fits (no y-periodic
// wrap).
template <typename T, int D, bool DOT>
__global__ void __launch_bounds__(MG_TPB, 4) k_mg_prolong(pict_mg_level_t F, pict_mg_level_t C, const int32_t* tiles,
                                                          const T* __restrict__ bv, const T* __restrict__ ec,
                                                          T* __restrict__ out, T s, T w, double* __restrict__ part,
                                                          int cap, const double* __restrict__ dn, int nu) {
    mg_pdl_entry();
    extern __shared__ __align__(16) unsigned char mg_stage_raw[];
    const MgTile tl = mg_tile(tiles, blockIdx.x);
    if (mg_done(dn, tl.sys)) return;
    const MgBlock Bf = mg_block(F, tl.blk), Bc = mg_block(C, tl.blk);
    const T* __restrict__ cf = reinterpret_cast<const T*>(F.coef);
    const int N = F.num_cells;
    double a = 0.0, c2 = 0.0, sz = 0.0, sr = 0.0;
    const int sx = Bf.sx;
    const int cap4 = (3 * cap) / 4;  // four arrays in the shared memory of three of `cap` cells
    if (D == 2 && nu == 2 && tl.cnt + 6 * sx <= cap4) {
        T* s_x = reinterpret_cast<T*>(mg_stage_raw);  // x0, then the first post sweep
        T* s_b = s_x + cap4;
        T* s_r = s_b + cap4;                           // w / diag
        T* s_y = s_r + cap4;                           // x1, then x' = x1 + s P e_c
        const int nf = sx * Bf.sy;
        const int lo = max(Bf.off, tl.s0 - 3 * sx), hi = min(Bf.off + nf, tl.s0 + tl.cnt + 3 * sx);
        for (int e = threadIdx.x; e < hi - lo; e += MG_TPB) {
            const T d = cf[lo + e], bb = bv[lo + e];
            const T r = (d != T(0)) ? mg_div(w, d) : T(0);
            s_b[e] = bb;
            s_r[e] = r;
            s_x[e] = r * bb;
        }
        __syncthreads();
        // one damped-Jacobi sweep over the global cells [g0, g1): dst = src + (w / diag) (b - A src), src and dst
        // on the stage; neighbours outside the block are fixed faces (no y-periodic wrap on this path)
        auto sweep = [&](int g0, int g1, const T* src, T* dst) {
            const int dq = MG_TPB / sx, dr = MG_TPB - dq * sx;
            int l = g0 - Bf.off + (int)threadIdx.x;
            int y = l / sx, x = l - y * sx;
            for (int i = g0 + (int)threadIdx.x; i < g1; i += MG_TPB) {
                const int c = i - lo;
                const T xi = src[c];
                const T xm = x > 0 ? src[c - 1] : src[c + sx - 1];
                const T xp = x + 1 < sx ? src[c + 1] : src[c - sx + 1];
                const T ym = y > 0 ? src[c - sx] : T(0);
                const T yp = y + 1 < Bf.sy ? src[c + sx] : T(0);
                T acc = cf[i] * xi;
                acc += (x > 0 || Bf.px) ? cf[(size_t)N + i] * xm : T(0);
                acc += (x + 1 < sx || Bf.px) ? cf[(size_t)2 * N + i] * xp : T(0);
                acc += y > 0 ? cf[(size_t)3 * N + i] * ym : T(0);
                acc += y + 1 < Bf.sy ? cf[(size_t)4 * N + i] * yp : T(0);
                dst[c] = xi + s_r[c] * (s_b[c] - acc);
                x += dr;
                y += dq;
                if (x >= sx) {
                    x -= sx;
                    ++y;
                }
            }
        };
        const int a1 = max(Bf.off, tl.s0 - 2 * sx), b1 = min(Bf.off + nf, tl.s0 + tl.cnt + 2 * sx);
        const int a2 = max(Bf.off, tl.s0 - sx), b2 = min(Bf.off + nf, tl.s0 + tl.cnt + sx);
        sweep(a1, b1, s_x, s_y);  // x1: the pre-smoothed iterate of the restriction
        __syncthreads();
        {  // x' = x1 + s P e_c
            const int dq = MG_TPB / sx, dr = MG_TPB - dq * sx;
            int l = a1 - Bf.off + (int)threadIdx.x;
            int y = l / sx, x = l - y * sx;
            for (int i = a1 + (int)threadIdx.x; i < b1; i += MG_TPB) {
                s_y[i - lo] += s * ec[Bc.off + (x >> Bc.shx) + Bc.sx * (y >> Bc.shy)];
                x += dr;
                y += dq;
                if (x >= sx) {
                    x -= sx;
                    ++y;
                }
            }
        }
        __syncthreads();
        sweep(a2, b2, s_y, s_x);  // first post sweep
        __syncthreads();
        // second post sweep of the tile's cells
        const int dq = MG_TPB / sx, dr = MG_TPB - dq * sx;
        int l = tl.s0 - Bf.off + (int)threadIdx.x;
        int y = l / sx, x = l - y * sx;
        for (int k = threadIdx.x; k < tl.cnt; k += MG_TPB) {
            const int i = tl.s0 + k, c = i - lo;
            const T xi = s_x[c], bi = s_b[c];
            const T xm = x > 0 ? s_x[c - 1] : s_x[c + sx - 1];
            const T xp = x + 1 < sx ? s_x[c + 1] : s_x[c - sx + 1];
            const T ym = y > 0 ? s_x[c - sx] : T(0);
            const T yp = y + 1 < Bf.sy ? s_x[c + sx] : T(0);
            T acc = cf[i] * xi;
            acc += (x > 0 || Bf.px) ? cf[(size_t)N + i] * xm : T(0);
            acc += (x + 1 < sx || Bf.px) ? cf[(size_t)2 * N + i] * xp : T(0);
            acc += y > 0 ? cf[(size_t)3 * N + i] * ym : T(0);
            acc += y + 1 < Bf.sy ? cf[(size_t)4 * N + i] * yp : T(0);
            const T zi = xi + s_r[c] * (bi - acc);
            out[i] = zi;
            if (DOT) {
                a += (double)bi * (double)zi;
                c2 += (double)bi * (double)bi;
                sz += (double)zi;
                sr += (double)bi;
            }
            x += dr;
            y += dq;
            if (x >= sx) {
                x -= sx;
                ++y;
            }
        }
    } else if (D == 2 && tl.cnt + 2 * sx <= cap) {
        T* s_x = reinterpret_cast<T*>(mg_stage_raw);
        T* s_b = s_x + cap;
        T* s_d = s_b + cap;
        const int nf = sx * Bf.sy;
        const int lo = max(Bf.off, tl.s0 - sx), hi = min(Bf.off + nf, tl.s0 + tl.cnt + sx);
        const int dq = MG_TPB / sx, dr = MG_TPB - dq * sx;
        int l = lo - Bf.off + (int)threadIdx.x;
        int y = l / sx, x = l - y * sx;
        for (int e = threadIdx.x; e < hi - lo; e += MG_TPB) {
            const int i = lo + e;
            const T d = cf[i], b = bv[i];
            s_x[e] = mg_x0(d, b, w) + s * ec[Bc.off + (x >> Bc.shx) + Bc.sx * (y >> Bc.shy)];
            s_b[e] = b;
            s_d[e] = d;
            x += dr;
            y += dq;
            if (x >= sx) {
                x -= sx;
                ++y;
            }
        }
        __syncthreads();
        // x' of a neighbour across the y-periodic wrap (outside the stage)
        auto far = [&](int xq, int yq) -> T {
            const int j = Bf.off + xq + sx * yq;
            return mg_x0(cf[j], bv[j], w) + s * ec[Bc.off + (xq >> Bc.shx) + Bc.sx * (yq >> Bc.shy)];
        };
        l = tl.s0 - Bf.off + (int)threadIdx.x;
        y = l / sx;
        x = l - y * sx;
        for (int k = threadIdx.x; k < tl.cnt; k += MG_TPB) {
            const int i = tl.s0 + k, c = i - lo;
            const T xi = s_x[c], di = s_d[c], bi = s_b[c];
            const T xm = x > 0 ? s_x[c - 1] : s_x[c + sx - 1];
            const T xp = x + 1 < sx ? s_x[c + 1] : s_x[c - sx + 1];
            const bool okm = x > 0 || Bf.px, okp = x + 1 < sx || Bf.px;
            const T ym = y > 0 ? s_x[c - sx] : (Bf.py ? far(x, Bf.sy - 1) : T(0));
            const T yp = y + 1 < Bf.sy ? s_x[c + sx] : (Bf.py ? far(x, 0) : T(0));
            T acc = di * xi;
            acc += okm ? cf[(size_t)N + i] * xm : T(0);
            acc += okp ? cf[(size_t)2 * N + i] * xp : T(0);
            acc += (y > 0 || Bf.py) ? cf[(size_t)3 * N + i] * ym : T(0);
            acc += (y + 1 < Bf.sy || Bf.py) ? cf[(size_t)4 * N + i] * yp : T(0);
            const T zi = xi + ((di != T(0)) ? mg_div(w * (bi - acc), di) : T(0));
            out[i] = zi;
            if (DOT) {
                a += (double)bi * (double)zi;
                c2 += (double)bi * (double)bi;
                sz += (double)zi;
                sr += (double)bi;
            }
            x += dr;
            y += dq;
            if (x >= sx) {
                x -= sx;
                ++y;
            }
        }
    } else {
        for (int base = 0; base < tl.cnt; base += MG_PASS) {
            T zv[MG_CPT], bvk[MG_CPT];
#pragma unroll
            for (int k = 0; k < MG_CPT; ++k) {
                const int l0 = base + k * MG_TPB + (int)threadIdx.x;
                const int l = l0 < tl.cnt ? l0 : tl.cnt - 1;
                const int i = tl.s0 + l;
                int x, y, z;
                mg_unflatten(Bf, i - Bf.off, x, y, z);
                MgNbrs<D> nb;
                mg_nbrs<D>(Bf, x, y, z, nb);
                const T di = cf[i], bi = bv[i];
                const T xi = mg_x0(di, bi, w) + s * ec[mg_coarse_index(Bc, x, y, z)];
                T acc = di * xi;
#pragma unroll
                for (int f = 0; f < 2 * D; ++f) {
                    const int j = nb.j[f];
                    const T cj = cf[(size_t)(f + 1) * N + i];
                    const T xj =
                        mg_x0(cf[j], bv[j], w) + s * ec[mg_coarse_index(Bc, nb.c[f][0], nb.c[f][1], nb.c[f][2])];
                    acc += nb.ok[f] ? cj * xj : T(0);
                }
                zv[k] = xi + ((di != T(0)) ? mg_div(w * (bi - acc), di) : T(0));
                bvk[k] = bi;
            }
#pragma unroll
            for (int k = 0; k < MG_CPT; ++k) {
                const int l = base + k * MG_TPB + (int)threadIdx.x;
                if (l >= tl.cnt) continue;
                out[tl.s0 + l] = zv[k];
                if (DOT) {
                    const double ri = (double)bvk[k], zi = (double)zv[k];
                    a += ri * zi;
                    c2 += ri * ri;
                    sz += zi;
                    sr += ri;
                }
            }
        }
    }
    if (DOT) {
        a = mg_warp_sum(a);
        c2 = mg_warp_sum(c2);
        sz = mg_warp_sum(sz);
        sr = mg_warp_sum(sr);
        if ((threadIdx.x & 31) == 0) {
            double* P = mg_warp_part(part, 4);
            P[0] = a;
            P[1] = c2;
            P[2] = sz;
            P[3] = sr;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// The V-cycle below a size cutoff in one launch: one CTA per block runs the levels lv[0..n-1] of its
// block (nu pre-smoothing sweeps from zero and restriction down to the coarsest, `sweeps` damped-Jacobi
// sweeps from zero and mean removal on the coarsest, prolongation and nu post-smoothing sweeps up) with every level's right-hand side, iterate and
// stencil in shared memory (the stencils are loaded once, at the start).  bin: right-hand side of lv[0]
// (global), xout: its iterate.
// ---------------------------------------------------------------------------------------------
constexpr int MG_SUB_LEVELS = 16;
constexpr int MG_SUB_THREADS = 512;
constexpr int MG_SUB_MAX = 2048;            // the cycle moves into one CTA per block from the first level
constexpr size_t MG_SUB_SMEM = 160 * 1024;  // whose blocks have at most this many cells and whose
                                            // sub-cycle fits this much shared memory

struct MgSub {
    pict_mg_level_t lv[MG_SUB_LEVELS];
    int n;
};

// shared memory of the sub-cycle: b, x and the 2D+1 stencil rows of every level (this block's cells)
// and one scratch vector
static size_t mg_sub_smem(const pict_mg_level_t* lv, int n, size_t esz) {
    const size_t K = 2 * (size_t)lv[0].dims + 1;
    size_t c = (size_t)lv[0].max_block_cells;
    for (int k = 0; k < n; ++k) c += (2 + K) * (size_t)lv[k].max_block_cells;
    return c * esz;
}

// one damped-Jacobi sweep of a sub-cycle level in shared memory: xd = xs + w (b - A xs) / diag
template <typename T, int D>
__device__ __forceinline__ void mg_sub_sweep(const MgBlock& B, int n, const T* sc, const T* sb, const T* xs, T* xd,
                                             T w) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        int x, y, z;
        mg_unflatten(B, e, x, y, z);
        T acc = sc[e] * xs[e];
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int j = mg_nbr(B, x, y, z, f);
            if (j >= 0) acc += sc[(f + 1) * n + e] * xs[j - B.off];
        }
        const T d = sc[e];
        xd[e] = xs[e] + ((d != T(0)) ? mg_div(w * (sb[e] - acc), d) : T(0));
    }
}

template <typename T, int D>
__global__ void __launch_bounds__(MG_SUB_THREADS) k_mg_subcycle(MgSub S, const T* __restrict__ bin,
                                                                T* __restrict__ xout, T w, T sp, int sweeps,
                                                                const double* __restrict__ dn, int nu) {
    mg_pdl_entry();
    constexpr int K = 2 * D + 1;
    extern __shared__ __align__(16) unsigned char mg_sub_raw[];
    T* sm = reinterpret_cast<T*>(mg_sub_raw);
    __shared__ int s_off[MG_SUB_LEVELS + 1];
    __shared__ double s_red[32];
    __shared__ double s_mean;
    const int b = blockIdx.x;
    if (mg_done(dn, mg_block(S.lv[0], b).sys)) return;
    if (threadIdx.x == 0) {
        int o = 0;
        for (int k = 0; k < S.n; ++k) {
            const MgBlock B = mg_block(S.lv[k], b);
            s_off[k] = o;
            o += (2 + K) * B.sx * B.sy * B.sz;
        }
        s_off[S.n] = o;
    }
    __syncthreads();
    T* scr = sm + s_off[S.n];
    // level k of this block: b at sm + s_off[k], x after it, then the stencil rows
    for (int k = 0; k < S.n; ++k) {
        const pict_mg_level_t& L = S.lv[k];
        const MgBlock B = mg_block(L, b);
        const int n = B.sx * B.sy * B.sz;
        const T* __restrict__ cf = reinterpret_cast<const T*>(L.coef);
        T* sc = sm + s_off[k] + 2 * n;
        for (int f = 0; f < K; ++f)
            for (int e = threadIdx.x; e < n; e += blockDim.x) sc[f * n + e] = cf[(size_t)f * L.num_cells + B.off + e];
        if (k == 0)
            for (int e = threadIdx.x; e < n; e += blockDim.x) sm[s_off[0] + e] = bin[B.off + e];
    }
    __syncthreads();
    // down: x0 = w b / diag (kept in the level's x), b_c = R (b - A x0)
    for (int k = 0; k + 1 < S.n; ++k) {
        const MgBlock Bf = mg_block(S.lv[k], b), Bc = mg_block(S.lv[k + 1], b);
        const int nf = Bf.sx * Bf.sy * Bf.sz, nc = Bc.sx * Bc.sy * Bc.sz;
        T* sb = sm + s_off[k];
        T* sx = sb + nf;
        const T* sc = sx + nf;
        T* sbc = sm + s_off[k + 1];
        for (int e = threadIdx.x; e < nf; e += blockDim.x) sx[e] = mg_x0(sc[e], sb[e], w);
        __syncthreads();
        if (nu == 2) {  // second pre-smoothing sweep (through the scratch vector)
            mg_sub_sweep<T, D>(Bf, nf, sc, sb, sx, scr, w);
            __syncthreads();
            for (int e = threadIdx.x; e < nf; e += blockDim.x) sx[e] = scr[e];
            __syncthreads();
        }
        for (int E = threadIdx.x; E < nc; E += blockDim.x) {
            int X, Y, Z;
            mg_unflatten(Bc, E, X, Y, Z);
            T acc = T(0);
            for (int c = 0; c < (1 << D); ++c) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
                if ((dx && !Bc.shx) || (dy && !Bc.shy) || (dz && !Bc.shz)) continue;
                const int xs = (X << Bc.shx) + dx, ys = (Y << Bc.shy) + dy, zs = (Z << Bc.shz) + dz;
                if (xs >= Bf.sx || ys >= Bf.sy || zs >= Bf.sz) continue;
                const int il = xs + Bf.sx * (ys + Bf.sy * zs);
                T ax = sc[il] * sx[il];
#pragma unroll
                for (int f = 0; f < 2 * D; ++f) {
                    const int j = mg_nbr(Bf, xs, ys, zs, f);
                    if (j >= 0) ax += sc[(f + 1) * nf + il] * sx[j - Bf.off];
                }
                acc += sb[il] - ax;
            }
            sbc[E] = acc;
        }
        __syncthreads();
    }
    // coarsest: sweeps from zero (ping-pong between x and the scratch vector), then mean removal
    {
        const MgBlock B = mg_block(S.lv[S.n - 1], b);
        const int n = B.sx * B.sy * B.sz;
        T* sb = sm + s_off[S.n - 1];
        T* const xa = sb + n;
        const T* sc = xa + n;
        for (int e = threadIdx.x; e < n; e += blockDim.x) xa[e] = mg_x0(sc[e], sb[e], w);
        __syncthreads();
        int cur = 0;
        for (int it = 1; it < sweeps; ++it) {
            const T* xs = cur ? scr : xa;
            T* xd = cur ? xa : scr;
            for (int e = threadIdx.x; e < n; e += blockDim.x) {
                int x, y, z;
                mg_unflatten(B, e, x, y, z);
                T acc = sc[e] * xs[e];
#pragma unroll
                for (int f = 0; f < 2 * D; ++f) {
                    const int j = mg_nbr(B, x, y, z, f);
                    if (j >= 0) acc += sc[(f + 1) * n + e] * xs[j - B.off];
                }
                const T d = sc[e];
                xd[e] = xs[e] + ((d != T(0)) ? mg_div(w * (sb[e] - acc), d) : T(0));
            }
            __syncthreads();
            cur ^= 1;
        }
        const T* xr = cur ? scr : xa;
        double acc = 0.0;
        for (int e = threadIdx.x; e < n; e += blockDim.x) acc += (double)xr[e];
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
        for (int e = threadIdx.x; e < n; e += blockDim.x) xa[e] = xr[e] - m;
        __syncthreads();
    }
    // up: x' = x0 + sp P x_c (scratch), x = x' + w (b - A x') / diag
    for (int k = S.n - 2; k >= 0; --k) {
        const MgBlock Bf = mg_block(S.lv[k], b), Bc = mg_block(S.lv[k + 1], b);
        const int nf = Bf.sx * Bf.sy * Bf.sz, nc = Bc.sx * Bc.sy * Bc.sz;
        T* sb = sm + s_off[k];
        T* sx = sb + nf;
        const T* sc = sx + nf;
        const T* sxc = sm + s_off[k + 1] + nc;
        for (int e = threadIdx.x; e < nf; e += blockDim.x) {
            int x, y, z;
            mg_unflatten(Bf, e, x, y, z);
            scr[e] = sx[e] + sp * sxc[(x >> Bc.shx) + Bc.sx * ((y >> Bc.shy) + Bc.sy * (z >> Bc.shz))];
        }
        __syncthreads();
        mg_sub_sweep<T, D>(Bf, nf, sc, sb, scr, sx, w);
        __syncthreads();
        if (nu == 2) {  // second post-smoothing sweep
            mg_sub_sweep<T, D>(Bf, nf, sc, sb, sx, scr, w);
            __syncthreads();
            for (int e = threadIdx.x; e < nf; e += blockDim.x) sx[e] = scr[e];
            __syncthreads();
        }
    }
    {
        const MgBlock B = mg_block(S.lv[0], b);
        const int n = B.sx * B.sy * B.sz;
        const T* sx = sm + s_off[0] + n;
        for (int e = threadIdx.x; e < n; e += blockDim.x) xout[B.off + e] = sx[e];
    }
}

// ---------------------------------------------------------------------------------------------
// PCG vector kernels on the finest level; per-system scalars in FP64
// ---------------------------------------------------------------------------------------------

// p_new = (z - m) + beta p_old formed on the fly (also for the neighbours; the first direction passes
// p_old = z with beta = 0), q = A p_new, and the per-warp partials of p_new.q (one CTA per work tile of
// the domain); m, beta per system from sc
template <typename T, int D>
__global__ void __launch_bounds__(MG_TPB) k_pcg_spmv_dot(pict_domain_t dom, pict_mg_level_t L, const T* __restrict__ z,
                                                         const T* __restrict__ pold, T* __restrict__ pnew,
                                                         T* __restrict__ q, const double* __restrict__ sc, int first,
                                                         double* __restrict__ part, const T* __restrict__ r) {
    mg_pdl_entry();
    const T* __restrict__ coef = reinterpret_cast<const T*>(L.coef);
    const int N = L.num_cells;
    const MgTile tl = mg_tile(dom.tiles, blockIdx.x);
    if (mg_done(sc, tl.sys)) return;
    const MgBlock B = mg_block(L, tl.blk);
    const T m = (T)sc[MG_SC * tl.sys + 4];
    const T bt = first ? T(0) : (T)sc[MG_SC * tl.sys + 2];
    double acc = 0.0, arq = 0.0, aqq = 0.0;
    for (int base = 0; base < tl.cnt; base += MG_PASS) {
        T pv[MG_CPT], qv[MG_CPT];
#pragma unroll
        for (int k = 0; k < MG_CPT; ++k) {
            const int l0 = base + k * MG_TPB + (int)threadIdx.x;
            const int l = l0 < tl.cnt ? l0 : tl.cnt - 1;
            const int i = tl.s0 + l;
            int x, y, z3;
            mg_unflatten(B, i - B.off, x, y, z3);
            MgNbrs<D> nb;
            mg_nbrs<D>(B, x, y, z3, nb);
            const T pi = (z[i] - m) + bt * pold[i];
            T qi = coef[i] * pi;
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                const int j = nb.j[f];
                const T cj = coef[(size_t)(f + 1) * N + i];
                const T pj = (z[j] - m) + bt * pold[j];
                qi += nb.ok[f] ? cj * pj : T(0);
            }
            pv[k] = pi;
            qv[k] = qi;
        }
#pragma unroll
        for (int k = 0; k < MG_CPT; ++k) {
            const int l = base + k * MG_TPB + (int)threadIdx.x;
            if (l >= tl.cnt) continue;
            pnew[tl.s0 + l] = pv[k];
            q[tl.s0 + l] = qv[k];
            const double qd = (double)qv[k];
            acc += (double)pv[k] * qd;
            arq += (double)r[tl.s0 + l] * qd;
            aqq += qd * qd;
        }
    }
    acc = mg_warp_sum(acc);
    arq = mg_warp_sum(arq);
    aqq = mg_warp_sum(aqq);
    if ((threadIdx.x & 31) == 0) {
        double* P = mg_warp_part(part, 3);
        P[0] = acc;
        P[1] = arq;
        P[2] = aqq;
    }
}

// k_pcg_spmv_dot for 2D tiles with its operands staged by asynchronous bulk copies: a persistent grid
// in which every CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...; per tile one thread issues
// bulk copies of z and p_old over the tile plus one block row on each side and of the K coefficient
// rows of the tile, completing on the mbarrier of one of two stage buffers, so the next tile's copies
// are in flight while the current tile is computed from shared memory.  A neighbour across a y-periodic
// wrap lies outside the stage and is read from global memory.  Cells, arithmetic and per-warp partials
// are those of k_pcg_spmv_dot.  A stage buffer holds z and p_old ([cap_h] each) and the coefficient rows
// ([K][cap_t]); err is set if a wait gives up.
constexpr long long MG_WAIT_LIMIT = 1ll << 22;
constexpr int MG_BULK_MAX_TILES = 64;  // tiles per CTA of the persistent grid (descriptors kept in shared memory)

template <typename T>
__global__ void __launch_bounds__(MG_TPB) k_pcg_spmv_dot_bulk(pict_domain_t dom, pict_mg_level_t L,
                                                              const T* __restrict__ z, const T* __restrict__ pold,
                                                              T* __restrict__ pnew, T* __restrict__ q,
                                                              const double* __restrict__ sc, int first,
                                                              double* __restrict__ part, int cap_h, int cap_t,
                                                              int* __restrict__ err, const T* __restrict__ r) {
    mg_pdl_entry();
    constexpr int K = 5;
    extern __shared__ __align__(128) unsigned char mg_bulk_raw[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ MgTile s_tl[MG_BULK_MAX_TILES];
    __shared__ MgBlock s_bk[MG_BULK_MAX_TILES];
    __shared__ int s_tix[MG_BULK_MAX_TILES];  // tile index of each live (not yet converged) tile
    __shared__ int s_nlive;
    const T* __restrict__ coef = reinterpret_cast<const T*>(L.coef);
    const int N = L.num_cells;
    const int nt = dom.num_tiles;
    const int per_buf = 2 * cap_h + K * cap_t;
    T* const stage = reinterpret_cast<T*>(mg_bulk_raw);
    const T* const pv_src = first ? z : pold;  // the first direction starts from p_old = z (beta = 0)
    // this CTA's tiles blockIdx.x + j gridDim.x and their blocks, loaded once (the host guarantees at most
    // MG_BULK_MAX_TILES per CTA)
    const int all_tiles = (int)blockIdx.x < nt ? (nt - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    if (threadIdx.x == 0) {  // the live tiles, in order (tiles of converged systems are skipped)
        int n = 0;
        for (int j = 0; j < all_tiles; ++j) {
            const int t = blockIdx.x + j * gridDim.x;
            const MgTile tl = mg_tile(dom.tiles, t);
            if (mg_done(sc, tl.sys)) continue;
            s_tl[n] = tl;
            s_bk[n] = mg_block(L, tl.blk);
            s_tix[n] = t;
            ++n;
        }
        s_nlive = n;
    }

    struct Runs {
        BulkRun<T> z, p, c[K];
        int lo;
    };
    auto runs_of = [&](const MgTile& tl, const MgBlock& B) {
        Runs R;
        R.lo = max(B.off, tl.s0 - B.sx);
        const int hi = min(B.off + B.sx * B.sy, tl.s0 + tl.cnt + B.sx);
        R.z = bulk_run(z, R.lo, hi - R.lo);
        R.p = bulk_run(pv_src, R.lo, hi - R.lo);
#pragma unroll
        for (int f = 0; f < K; ++f) R.c[f] = bulk_run(coef, (long long)f * N + tl.s0, tl.cnt);
        return R;
    };
    auto issue = [&](int j, int b) {  // one thread: tile j of this CTA into stage buffer b
        const Runs R = runs_of(s_tl[j], s_bk[j]);
        T* buf = stage + (size_t)b * per_buf;
        uint32_t bytes = R.z.bytes + (first ? 0u : R.p.bytes);
#pragma unroll
        for (int f = 0; f < K; ++f) bytes += R.c[f].bytes;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[b], bytes);
        bulk_issue(R.z, buf, &bar[b]);
        if (!first) bulk_issue(R.p, buf + cap_h, &bar[b]);
#pragma unroll
        for (int f = 0; f < K; ++f) bulk_issue(R.c[f], buf + 2 * cap_h + f * cap_t, &bar[b]);
    };

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    const int my_tiles = s_nlive;
    if (threadIdx.x == 0 && my_tiles > 0) issue(0, 0);
    for (int k = 0; k < my_tiles; ++k) {
        const int b = k & 1;
        if (threadIdx.x == 0 && k + 1 < my_tiles) issue(k + 1, b ^ 1);
        const MgTile tl = s_tl[k];
        const MgBlock B = s_bk[k];
        const int t = s_tix[k];
        const Runs R = runs_of(tl, B);
        T* const buf = stage + (size_t)b * per_buf;
        T* const zs = buf;
        T* const ps = first ? buf : buf + cap_h;
        bulk_tail(R.z, zs);
        if (!first) bulk_tail(R.p, ps);
#pragma unroll
        for (int f = 0; f < K; ++f) bulk_tail(R.c[f], buf + 2 * cap_h + f * cap_t);
        const bool ok = mbar_wait(&bar[b], (k >> 1) & 1, MG_WAIT_LIMIT);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(err, 1);
                // the other buffer's copies may still be in flight: wait for them before the CTA ends
                if (k + 1 < my_tiles) mbar_wait(&bar[b ^ 1], ((k + 1) >> 1) & 1, MG_WAIT_LIMIT);
            }
            __syncthreads();
            return;
        }
        const T m = (T)sc[MG_SC * tl.sys + 4];
        const T bt = first ? T(0) : (T)sc[MG_SC * tl.sys + 2];
        const int hz = R.z.lead - R.lo, hp = R.p.lead - R.lo;  // stage index of global cell j: j + hz / j + hp
        const T* const c0 = buf + 2 * cap_h + R.c[0].lead;
        const T* const c1 = buf + 2 * cap_h + 1 * cap_t + R.c[1].lead;
        const T* const c2 = buf + 2 * cap_h + 2 * cap_t + R.c[2].lead;
        const T* const c3 = buf + 2 * cap_h + 3 * cap_t + R.c[3].lead;
        const T* const c4 = buf + 2 * cap_h + 4 * cap_t + R.c[4].lead;
        double acc = 0.0, arq = 0.0, aqq = 0.0;
        for (int base = 0; base < tl.cnt; base += MG_PASS) {
            T pvk[MG_CPT], qvk[MG_CPT];
#pragma unroll
            for (int kk = 0; kk < MG_CPT; ++kk) {
                const int l0 = base + kk * MG_TPB + (int)threadIdx.x;
                const int l = l0 < tl.cnt ? l0 : tl.cnt - 1;
                const int i = tl.s0 + l;
                const int li = i - B.off;
                const int y = li / B.sx, x = li - y * B.sx;
                const T pi = (zs[i + hz] - m) + bt * ps[i + hp];
                T qi = c0[l] * pi;
                // -x, +x: in the stage (a periodic wrap stays in the row)
                {
                    const bool okm = x > 0 || B.px;
                    const int jm = x > 0 ? i - 1 : (B.px ? i + B.sx - 1 : i);
                    const T pj = (zs[jm + hz] - m) + bt * ps[jm + hp];
                    qi += okm ? c1[l] * pj : T(0);
                }
                {
                    const bool okp = x + 1 < B.sx || B.px;
                    const int jp = x + 1 < B.sx ? i + 1 : (B.px ? i - B.sx + 1 : i);
                    const T pj = (zs[jp + hz] - m) + bt * ps[jp + hp];
                    qi += okp ? c2[l] * pj : T(0);
                }
                // -y, +y: in the stage, except across a periodic wrap
                {
                    const bool okm = y > 0 || B.py;
                    T pj;
                    if (y > 0) {
                        pj = (zs[i - B.sx + hz] - m) + bt * ps[i - B.sx + hp];
                    } else {
                        const int j = B.py ? B.off + x + B.sx * (B.sy - 1) : i;
                        pj = B.py ? (z[j] - m) + bt * pv_src[j] : pi;
                    }
                    qi += okm ? c3[l] * pj : T(0);
                }
                {
                    const bool okp = y + 1 < B.sy || B.py;
                    T pj;
                    if (y + 1 < B.sy) {
                        pj = (zs[i + B.sx + hz] - m) + bt * ps[i + B.sx + hp];
                    } else {
                        const int j = B.py ? B.off + x : i;
                        pj = B.py ? (z[j] - m) + bt * pv_src[j] : pi;
                    }
                    qi += okp ? c4[l] * pj : T(0);
                }
                pvk[kk] = pi;
                qvk[kk] = qi;
            }
#pragma unroll
            for (int kk = 0; kk < MG_CPT; ++kk) {
                const int l = base + kk * MG_TPB + (int)threadIdx.x;
                if (l >= tl.cnt) continue;
                pnew[tl.s0 + l] = pvk[kk];
                q[tl.s0 + l] = qvk[kk];
                const double qd = (double)qvk[kk];
                acc += (double)pvk[kk] * qd;
                arq += (double)r[tl.s0 + l] * qd;
                aqq += qd * qd;
            }
        }
        acc = mg_warp_sum(acc);
        arq = mg_warp_sum(arq);
        aqq = mg_warp_sum(aqq);
        if ((threadIdx.x & 31) == 0) {
            double* P = part + ((size_t)t * MG_NW + (threadIdx.x >> 5)) * 3;
            P[0] = acc;
            P[1] = arq;
            P[2] = aqq;
        }
        __syncthreads();  // stage buffer b is free for the tile after next
    }
}

// per-warp partials of r.z, r.r, sum(z), sum(r) (one CTA per work tile)
template <typename T>
__global__ void __launch_bounds__(MG_TPB) k_pcg_dot4(pict_domain_t dom, const T* r, const T* z, double* part,
                                                     const double* __restrict__ dn) {
    mg_pdl_entry();
    const MgTile tl = mg_tile(dom.tiles, blockIdx.x);
    if (mg_done(dn, tl.sys)) return;
    double a = 0.0, c = 0.0, sz = 0.0, sr = 0.0;
    for (int i = tl.s0 + threadIdx.x; i < tl.s0 + tl.cnt; i += MG_TPB) {
        const double ri = (double)r[i], zi = (double)z[i];
        a += ri * zi;
        c += ri * ri;
        sz += zi;
        sr += ri;
    }
    a = mg_warp_sum(a);
    c = mg_warp_sum(c);
    sz = mg_warp_sum(sz);
    sr = mg_warp_sum(sr);
    if ((threadIdx.x & 31) == 0) {
        double* P = mg_warp_part(part, 4);
        P[0] = a;
        P[1] = c;
        P[2] = sz;
        P[3] = sr;
    }
}

// per-system scalars (one warp per system; the per-warp partials of its tiles summed lane-strided in
// a fixed order):
// stage 0: rho = r.(z - m), |r|^2, m = mean(z);  stage 1: alpha = rho / p.q;
// stage 2: rho' = r.(z - m), beta = rho'/rho, rho = rho', |r|^2, m
// The preconditioned residual z is used mean-free (z - m): the constant mode of a singular system is
// undetermined.  sc[s*MG_SC + {0: rho, 1: alpha, 2: beta, 3: |r|^2, 4: m}]
// it: the PCG iteration; inside a graph's conditional loop it is an offset to the device counter ctr
template <int STRIDE>
__global__ void k_pcg_scalars(pict_domain_t dom, const double* __restrict__ part, int stage, double* sc, int it,
                              double tol, int normalized, const int* __restrict__ ctr) {
    mg_pdl_entry();
    if (ctr) it += *ctr;
    const int lane = threadIdx.x & 31;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= dom.num_sims) return;
    if (stage != 0 && sc[MG_SC * s + 5] != 0.0) {  // converged earlier: keep its scalars
        if (stage == 2 && lane == 0) sc[MG_SC * s + 6] = 0.0;  // its last update has been applied
        return;
    }
    double v[4] = {0.0, 0.0, 0.0, 0.0}, u[STRIDE];
#pragma unroll
    for (int k = 0; k < STRIDE; ++k) u[k] = 0.0;
    // two interleaved accumulators per lane (independent loads in flight), combined in a fixed order
    const int t1 = dom.sim_tiles[s + 1] * MG_NW;
    int t = dom.sim_tiles[s] * MG_NW + lane;
    for (; t + 32 < t1; t += 64) {
#pragma unroll
        for (int k = 0; k < STRIDE; ++k) {
            v[k] += part[(size_t)STRIDE * t + k];
            u[k] += part[(size_t)STRIDE * (t + 32) + k];
        }
    }
    if (t < t1) {
#pragma unroll
        for (int k = 0; k < STRIDE; ++k) v[k] += part[(size_t)STRIDE * t + k];
    }
#pragma unroll
    for (int k = 0; k < STRIDE; ++k) v[k] += u[k];
#pragma unroll
    for (int k = 0; k < STRIDE; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane != 0) return;
    double* S = sc + MG_SC * s;
    const int n = dom.sim_cells[s + 1] - dom.sim_cells[s];
    if (stage == 1) {
        // alpha from p.q; with STRIDE 3 also |r - alpha q|^2 = |r|^2 - 2 alpha r.q + alpha^2 q.q: a system that
        // meets the tolerance here is done after this iteration's update (its V-cycle is skipped)
        const double a = v[0];
        const double al = (a != 0.0 && S[0] != 0.0 && isfinite(a)) ? S[0] / a : 0.0;
        S[1] = al;
        if (STRIDE >= 3) {
            const double r2 = fmax(S[3] - 2.0 * al * v[1] + al * al * v[2], 0.0);
            const double crit1 = normalized ? sqrt(r2) / sqrt((double)n) : sqrt(r2);
            if (crit1 < tol) {
                S[3] = r2;
                S[5] = (double)(it + 2);
                S[6] = 1.0;
            }
        }
        return;
    }
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
    // converged: iterations done so far (0 after the initial cycle, it + 1 after iteration it) plus one
    const double crit = normalized ? sqrt(v[1]) / sqrt((double)n) : sqrt(v[1]);
    S[5] = (crit < tol) ? (stage == 0 ? 1.0 : (double)(it + 2)) : 0.0;
}

// rn = r - alpha q, x += alpha p (x = alpha p when first), and the per-warp partials of
// (0, rn.rn, 0, sum(rn)) (the PCG update where no V-cycle follows: the last iteration, or a
// single-level hierarchy)
template <typename T>
__global__ void __launch_bounds__(MG_TPB) k_pcg_update(pict_domain_t dom, const T* __restrict__ r,
                                                       const T* __restrict__ q, T* __restrict__ rn, T* __restrict__ x,
                                                       const T* __restrict__ p, const double* __restrict__ sc, int first,
                                                       double* __restrict__ part) {
    mg_pdl_entry();
    const MgTile tl = mg_tile(dom.tiles, blockIdx.x);
    if (mg_done(sc, tl.sys) && !mg_pending(sc, tl.sys)) return;
    const T al = (T)sc[MG_SC * tl.sys + 1];
    double c2 = 0.0, sr = 0.0;
    for (int l = threadIdx.x; l < tl.cnt; l += MG_TPB) {
        const int i = tl.s0 + l;
        const T ri = r[i] - al * q[i];
        rn[i] = ri;
        x[i] = first ? al * p[i] : x[i] + al * p[i];
        c2 += (double)ri * (double)ri;
        sr += (double)ri;
    }
    c2 = mg_warp_sum(c2);
    sr = mg_warp_sum(sr);
    if ((threadIdx.x & 31) == 0) {
        double* P = mg_warp_part(part, 4);
        P[0] = 0.0;
        P[1] = c2;
        P[2] = 0.0;
        P[3] = sr;
    }
}

__global__ void k_pcg_report(pict_domain_t dom, const double* sc, pict_solve_info_t* info, int iterations, double tol,
                             int normalized, const int* err) {
    mg_pdl_entry();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= dom.num_sims) return;
    const int n = dom.sim_cells[s + 1] - dom.sim_cells[s];
    const double nrm = sqrt(sc[MG_SC * s + 3]);
    const double crit = normalized ? nrm / sqrt((double)n) : nrm;
    pict_solve_info_t inf;
    inf.final_residual = crit;
    inf.used_iterations = sc[MG_SC * s + 5] != 0.0 ? (int)sc[MG_SC * s + 5] - 1 : iterations;
    inf.finite = isfinite(crit) ? 1 : 0;
    inf.converged = (inf.finite && crit < tol) ? 1 : 0;
    inf.status = 0;
    if (*err) {  // a stage wait gave up: report like a barrier timeout
        inf.status = 1;
        inf.converged = 0;
    }
    info[s] = inf;
}

// Condition of the graph's PCG loop (one CTA): ctr = init (init > 0) or ctr += step, then keep looping
// while a system is still iterating and the next two iterations (ctr, ctr + 1) are within the cap.
__global__ void k_pcg_loop_cond(pict_domain_t dom, const double* __restrict__ sc, int* ctr, int init, int step,
                                int limit, cudaGraphConditionalHandle h) {
    mg_pdl_entry();
    __shared__ int s_any;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    int any = 0;
    for (int s = threadIdx.x; s < dom.num_sims; s += blockDim.x) any |= sc[MG_SC * s + 5] == 0.0;
    if (__syncthreads_or(any) && threadIdx.x == 0) s_any = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        const int c = init > 0 ? init : *ctr + step;
        *ctr = c;
        cudaGraphSetConditional(h, (s_any && c + 2 <= limit) ? 1u : 0u);
    }
}

// workspace: levels >= 1: b, x | finest: r (two, alternating), z, p (two, alternating), q | per-warp
// partials | scalars.  Returns the bytes; fills the pointers when ws != nullptr.
struct MgWork {
    char* lb[16];
    char* lx[16];
    char* r[2];
    char* z;
    char* p[2];
    char* q;
    double* part;
    double* sc;
    int* err;
};

static size_t mg_carve(const pict_domain_t* dom, const pict_mg_level_t* levels, int nl, size_t esz, char* ws,
                       MgWork* w) {
    auto vb = [&](int n) { return ((size_t)n * esz + 255) & ~(size_t)255; };
    size_t o = 0;
    auto take = [&](size_t bytes) {
        char* ptr = ws ? ws + o : nullptr;
        o += bytes;
        return ptr;
    };
    for (int l = 1; l < nl; ++l) {
        w->lb[l] = take(vb(levels[l].num_cells));
        w->lx[l] = take(vb(levels[l].num_cells));
    }
    const int N = dom->num_cells;
    w->r[0] = take(vb(N));
    w->r[1] = take(vb(N));
    w->z = take(vb(N));
    w->p[0] = take(vb(N));
    w->p[1] = take(vb(N));
    w->q = take(vb(N));
    w->part = reinterpret_cast<double*>(take(((size_t)4 * MG_NW * dom->num_tiles * 8 + 255) & ~(size_t)255));
    w->sc = reinterpret_cast<double*>(take(((size_t)MG_SC * dom->num_sims * 8 + 255) & ~(size_t)255));
    w->err = reinterpret_cast<int*>(take(256));  // [0] stage-wait error, [1] iteration counter of the graph loop
    return o;
}

template <typename T, int D>
static pict_status_t run_pcg_mg(const pict_domain_t* dom, const pict_mg_level_t* levels, int nl, const T* rhs, T* xout,
                                int iterations, double tol, int normalized, pict_solve_info_t* info, char* ws,
                                int64_t ws_bytes, double omega, double scale, int coarse_sweeps, cudaStream_t st) {
    const int N = dom->num_cells;
    MgWork W;
    if ((int64_t)mg_carve(dom, levels, nl, sizeof(T), ws, &W) > ws_bytes)
        return set_error(PICT_ERR_ARG, "pcg_mg: workspace too small");
    for (int l = 1; l < nl; ++l)
        if (levels[l].num_tiles <= 0 || !levels[l].tiles) return set_error(PICT_ERR_ARG, "pcg_mg: level without tiles");
    T* lb[16];
    T* lx[16];
    for (int l = 1; l < nl; ++l) {
        lb[l] = reinterpret_cast<T*>(W.lb[l]);
        lx[l] = reinterpret_cast<T*>(W.lx[l]);
    }
    T* rbuf[2] = {reinterpret_cast<T*>(W.r[0]), reinterpret_cast<T*>(W.r[1])};
    T* z = reinterpret_cast<T*>(W.z);
    T* pbuf[2] = {reinterpret_cast<T*>(W.p[0]), reinterpret_cast<T*>(W.p[1])};
    T* q = reinterpret_cast<T*>(W.q);
    double* part = W.part;
    double* sc = W.sc;
    int* err = W.err;

    const T wj = (T)omega, sp = (T)scale;
    const int nt = dom->num_tiles;
    const int sg = (dom->num_sims + 127) / 128;
    const int swg = (dom->num_sims * 32 + 127) / 128;  // one warp per system

    // the cycle runs in one CTA per block from level lc on (lc = 0 only for a single-level hierarchy)
    int lc = nl - 1;
    for (int l = 1; l < nl; ++l)
        if (levels[l].max_block_cells <= MG_SUB_MAX && mg_sub_smem(levels + l, nl - l, sizeof(T)) <= MG_SUB_SMEM) {
            lc = l;
            break;
        }
    if (nl == 1) lc = 0;
    MgSub sub;
    sub.n = nl - lc;
    for (int k = 0; k < sub.n; ++k) sub.lv[k] = levels[lc + k];
    const size_t sub_smem = mg_sub_smem(sub.lv, sub.n, sizeof(T));
    if (sub_smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_mg_subcycle<T, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sub_smem);
        if (e != cudaSuccess) return set_error(PICT_ERR_CUDA, "pcg_mg: sub-cycle shared memory");
    }
    // shared-memory stages of the 2D restriction / prolongation: x or x0, b, diag
    const int cap = D == 2 ? MG_STAGE : 0;
    const size_t stage3 = D == 2 ? 3 * (size_t)MG_STAGE * sizeof(T) : 0;
    if (D == 2) {
        cudaError_t e = cudaFuncSetAttribute(k_mg_restrict<T, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)stage3);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_mg_restrict<T, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)stage3);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_mg_prolong<T, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)stage3);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_mg_prolong<T, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)stage3);
        if (e != cudaSuccess) return set_error(PICT_ERR_CUDA, "pcg_mg: stage shared memory");
    }

    // smoothing sweeps per level of the tile kernels: the level's own choice (every tile's stage holds the
    // halo rows of two sweeps) capped by the process-wide setting; level 0 also needs the domain's tiles to
    // fit the four-array stage of the two-sweep prolongation.  The one-launch sub-cycle takes the setting.
    int nu[16];
    for (int l = 0; l < nl; ++l) nu[l] = (D == 2 && g_mg_sweeps >= 2 && levels[l].sweeps >= 2) ? 2 : 1;
    if (nu[0] == 2 && dom->tile_cells + 6 * levels[0].max_block_sx > (3 * cap) / 4) nu[0] = 1;
    const int nu_sub = g_mg_sweeps >= 2 ? 2 : 1;

    // z = M r_new (V-cycle) and the per-warp partials of r_new.z, |r_new|^2, sum(z), sum(r_new).  upd:
    // the finest restriction first forms r_new = r - alpha q (stored to rn) and x += alpha p.
    auto vcycle = [&](const T* r, bool upd, T* rn, const T* p, int first, cudaStream_t st) -> pict_status_t {
        const T* rnew = upd ? rn : r;
        if (lc == 0) {
            if (upd) mg_launch(k_pcg_update<T>, nt, MG_TPB, 0, st, *dom, r, q, rn, xout, p, sc, first, part);
            mg_launch(k_mg_subcycle<T, D>, levels[0].num_blocks, MG_SUB_THREADS, sub_smem, st, sub, rnew, z, wj, sp,
                                                                                     coarse_sweeps, sc, nu_sub);
            mg_launch(k_pcg_dot4<T>, nt, MG_TPB, 0, st, *dom, rnew, z, part, sc);
            return check_launch("pcg_mg vcycle");
        }
        for (int l = 0; l < lc; ++l) {
            const pict_mg_level_t& F = levels[l];
            const pict_mg_level_t& C = levels[l + 1];
            if (l == 0 && upd)
                mg_launch(k_mg_restrict<T, D, true>, C.num_tiles, MG_TPB, stage3, st, F, C, r, q, rn, xout, p, sc, first,
                                                                                lb[1], wj, cap, sc, nu[0]);
            else
                mg_launch(k_mg_restrict<T, D, false>, C.num_tiles, MG_TPB, stage3, st, 
                    F, C, l == 0 ? r : lb[l], nullptr, nullptr, nullptr, nullptr, nullptr, 0, lb[l + 1], wj, cap, sc,
                    nu[l]);
        }
        // levels lc.. in one launch (one CTA per block)
        mg_launch(k_mg_subcycle<T, D>, levels[lc].num_blocks, MG_SUB_THREADS, sub_smem, st, sub, lb[lc], lx[lc], wj, sp,
                                                                                  coarse_sweeps, sc, nu_sub);
        for (int l = lc - 1; l >= 1; --l)
            mg_launch(k_mg_prolong<T, D, false>, levels[l].num_tiles, MG_TPB, stage3, st, 
                levels[l], levels[l + 1], levels[l].tiles, lb[l], lx[l + 1], lx[l], sp, wj, nullptr, cap, sc, nu[l]);
        mg_launch(k_mg_prolong<T, D, true>, nt, MG_TPB, stage3, st, levels[0], levels[1], dom->tiles, rnew, lx[1], z, sp, wj,
                                                             part, cap, sc, nu[0]);
        return check_launch("pcg_mg vcycle");
    };

    // bulk-staged SpMV (2D): stage buffers sized by the domain's tile size and longest block row; every
    // operand's base must be 16-byte aligned (bulk copies start on 16-byte boundaries)
    auto al16 = [](const void* ptr) { return ((uintptr_t)ptr & 15) == 0; };
    const int cap_h = ((dom->tile_cells + 2 * levels[0].max_block_sx + 8 + 7) / 8) * 8;
    const int cap_t = ((dom->tile_cells + 8 + 7) / 8) * 8;
    const size_t bulk_smem = 2 * (size_t)(2 * cap_h + (2 * D + 1) * cap_t) * sizeof(T);
    int bulk_grid = 0;
    if (D == 2 && g_mg_bulk && levels[0].max_block_sx > 0 && bulk_smem <= 200 * 1024 && al16(levels[0].coef) &&
        al16(z) && al16(pbuf[0]) && al16(pbuf[1])) {
        cudaError_t e = cudaFuncSetAttribute(k_pcg_spmv_dot_bulk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)bulk_smem);
        int per_sm = 0;
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_spmv_dot_bulk<T>, MG_TPB, bulk_smem);
        if (e != cudaSuccess) {
            cudaGetLastError();
            per_sm = 0;
        }
        bulk_grid = per_sm * device_sm_count();
        if (bulk_grid > nt) bulk_grid = nt;
        if ((long long)bulk_grid * MG_BULK_MAX_TILES < nt) bulk_grid = 0;  // descriptors would not fit
    }
    // x from zero (a system that is done before its first update keeps x = 0); no system is done yet
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess || cudaMemsetAsync(xout, 0, sizeof(T) * N, st) != cudaSuccess ||
        cudaMemsetAsync(sc, 0, sizeof(double) * MG_SC * dom->num_sims, st) != cudaSuccess)
        return check_launch("pcg_mg initial state");
    pict_status_t s = vcycle(rhs, false, nullptr, nullptr, 0, st);
    if (s) return s;
    mg_launch(k_pcg_scalars<4>, swg, 128, 0, st, *dom, part, 0, sc, 0, tol, normalized, nullptr);
    // one PCG iteration; it >= 0: iteration `it` with its buffers and reports fixed at launch (the last one
    // only updates); it < 0: an iteration of the graph loop with buffer parity `par`, its number read from the
    // device counter plus `off`
    int* ctr = err + 1;
    auto iteration = [&](int it, int par, int off, cudaStream_t st) -> pict_status_t {
        const bool fixed = it >= 0;
        const int first = it == 0;
        T* pnew = pbuf[par];
        const T* pold = first ? z : pbuf[par ^ 1];
        T* rn = rbuf[par];
        const T* r = first ? rhs : rbuf[par ^ 1];
        const int* c = fixed ? nullptr : ctr;
        const int itv = fixed ? it : off;
        if (bulk_grid > 0)
            mg_launch(k_pcg_spmv_dot_bulk<T>, bulk_grid, MG_TPB, bulk_smem, st, *dom, levels[0], z, pold, pnew, q, sc, first,
                                                                         part, cap_h, cap_t, err, r);
        else
            mg_launch(k_pcg_spmv_dot<T, D>, nt, MG_TPB, 0, st, *dom, levels[0], z, pold, pnew, q, sc, first, part, r);
        mg_launch(k_pcg_scalars<3>, swg, 128, 0, st, *dom, part, 1, sc, itv, tol, normalized, c);
        if (!fixed || it + 1 < iterations) {
            pict_status_t e = vcycle(r, true, rn, pnew, first, st);
            if (e) return e;
        } else {
            // last iteration: only the update and |r|^2 (r.z and sum(z) are not used)
            mg_launch(k_pcg_update<T>, nt, MG_TPB, 0, st, *dom, r, q, rn, xout, pnew, sc, first, part);
        }
        mg_launch(k_pcg_scalars<4>, swg, 128, 0, st, *dom, part, 2, sc, itv, tol, normalized, c);
        return check_launch("pcg_mg iteration");
    };
    // under stream capture: iteration 0, then iterations (1, 2), (3, 4), ... as the body of a conditional
    // WHILE node that ends once every system has converged, then (cap even) the last iteration
    int dev = 0;
    cudaGetDevice(&dev);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return check_launch("pcg_mg capture status");
    if (cs == cudaStreamCaptureStatusNone && dev < 64 && !g_mg_body_stream[dev])
        if (cudaStreamCreateWithFlags(&g_mg_body_stream[dev], cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            g_mg_body_stream[dev] = nullptr;
        }
    const bool loop = g_mg_graph_loop && cs == cudaStreamCaptureStatusActive && iterations >= 3 && dev < 64 &&
                      g_mg_body_stream[dev];
    if (!loop) {
        for (int it = 0; it < iterations; ++it)
            if ((s = iteration(it, it & 1, 0, st))) return s;
    } else {
        if ((s = iteration(0, 0, 0, st))) return s;
        cudaGraph_t graph = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaGraphConditionalHandle h;
        if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps) != cudaSuccess ||
            cudaGraphConditionalHandleCreate(&h, graph, 0, 0) != cudaSuccess)
            return check_launch("pcg_mg conditional handle");
        mg_launch(k_pcg_loop_cond, 1, 256, 0, st, *dom, sc, ctr, 1, 0, iterations, h);
        if ((s = check_launch("pcg_mg loop condition"))) return s;
        if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps) != cudaSuccess)
            return check_launch("pcg_mg capture info");
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, graph, deps, ndeps, &cp) != cudaSuccess)
            return check_launch("pcg_mg conditional node");
        cudaStream_t bs = g_mg_body_stream[dev];
        if (cudaStreamBeginCaptureToGraph(bs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed) != cudaSuccess)
            return check_launch("pcg_mg loop body capture");
        pict_status_t sb = iteration(-1, 1, 0, bs);
        if (!sb) sb = iteration(-1, 0, 1, bs);
        if (!sb) {
            mg_launch(k_pcg_loop_cond, 1, 256, 0, bs, *dom, sc, ctr, 0, 2, iterations, h);
            sb = check_launch("pcg_mg loop condition");
        }
        cudaGraph_t body = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(bs, &body);
        if (sb) return sb;
        if (ee != cudaSuccess) return check_launch("pcg_mg loop body end capture");
        if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
            return check_launch("pcg_mg capture dependencies");
        if ((iterations - 1) % 2 == 1)
            if ((s = iteration(iterations - 1, (iterations - 1) & 1, 0, st))) return s;
    }
    mg_launch(k_pcg_report, sg, 128, 0, st, *dom, sc, info, iterations, tol, normalized, err);
    return check_launch("pcg_mg");
}

}  // namespace pict

using namespace pict;

extern "C" {

void pict_mg_set_bulk_staging(int32_t enable) { g_mg_bulk = enable ? 1 : 0; }
void pict_mg_set_smoothing_sweeps(int32_t sweeps) { g_mg_sweeps = sweeps >= 2 ? 2 : 1; }
void pict_mg_set_graph_loop(int32_t enable) { g_mg_graph_loop = enable ? 1 : 0; }
void pict_mg_set_dependent_launch(int32_t enable) { g_mg_pdl = enable ? 1 : 0; }

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
    MgWork w;
    return (int64_t)mg_carve(dom, levels, num_levels, dom->dtype == PICT_F64 ? 8 : 4, nullptr, &w);
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
    if (!(convergence == PICT_CONV_NORM2 || convergence == PICT_CONV_NORM2_NORMALIZED))
        return set_error(PICT_ERR_UNSUPPORTED, "pcg_mg: takes the NORM2 and NORM2_NORMALIZED criteria");
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
