// nonortho.cu -- non-orthogonal terms of the PISO operators (nonOrthoFlags != 0).
//
// On skewed grids the Laplacian of the viscous term and of the pressure equation has off-diagonal
// metric coefficients alpha_at = det Minv[a].Minv[t]: the flux through a face of axis a has a part
// proportional to the tangential derivative along t, taken as the difference of the two corner values
// of the face, each the average of the cells around that corner.  The reference splits it into
// implicit matrix terms (the cell, the face neighbour and the tangential neighbour of a corner) and
// explicit right-hand-side terms (the diagonal cell, from the previous result).  Restated here:
//   getCornerValue                        extensions/PISO_multiblock_cuda_kernel.cu:2742-2860
//   interpolateNonOrthoLaplaceComponents  extensions/PISO_multiblock_cuda_kernel.cu:1911-1987
//   PISO_build_matrix (non-ortho part)    extensions/PISO_multiblock_cuda_kernel.cu:3736-3800
//   PISO_build_pressure_matrix (part)     extensions/PISO_multiblock_cuda_kernel.cu:4877-4934
//   getNonOrthoLaplaceRHS_v2              extensions/PISO_multiblock_cuda_kernel.cu:3033-3187
//   k_pressureRHSaddNonOrthoComponents    extensions/PISO_multiblock_cuda_kernel.cu:5423-5453
// including the reference's treatment of block connections (the corner walk and the neighbour reads
// of the right-hand side land on the second cell layer of the connected block, computeConnectedPos
// with borderOffset 1) and of cells next to a wall (the interpolated coefficient of both faces of
// that axis is zero).
//
// Each pass runs after the orthogonal kernel of the same operator (one thread per cell) and adds
// its terms: the orthogonal path is unchanged when the flags are 0.
#include "common.cuh"
#include "launch.h"

namespace pict {

constexpr int NO_DIRECT_MATRIX = 1;
constexpr int NO_DIRECT_RHS = 2;
constexpr int NO_DIAGONAL_RHS = 8;
constexpr int NO_CENTER_MATRIX = 16;

__device__ __forceinline__ bool face_fixed(const pict_block_t& B, int f) { return B.face[f].type == PICT_FACE_FIXED; }

__device__ __forceinline__ int flat3(const int32_t* size, const int* q) { return q[0] + size[0] * (q[1] + size[1] * q[2]); }

// computeConnectedPos (extensions/PISO_multiblock_cuda_kernel.cu:326-345): the cell `offset` layers into the
// block across the connection of face f
template <int D>
__device__ __forceinline__ int conn_pos(const pict_domain_t& dom, const pict_block_t& B, int f, const int* p,
                                        int offset, int* q) {
    const pict_face_t& F = B.face[f];
    const pict_block_t& O = dom.blocks[F.conn_block];
    const int a = f >> 1;
    q[0] = p[0];
    q[1] = p[1];
    q[2] = p[2];
    {
        const int ca = F.conn_axes[0] >> 1;
        q[ca] = (F.conn_axes[0] & 1) ? O.size[ca] - 1 - offset : offset;
    }
#pragma unroll
    for (int k = 1; k < D; ++k) {
        const int ax = (a + k) % D;
        const int ca = F.conn_axes[k] >> 1;
        q[ca] = (F.conn_axes[k] & 1) ? O.size[ca] - 1 - p[ax] : p[ax];
    }
    return F.conn_block;
}

// computeConnectedDir (extensions/PISO_multiblock_cuda_kernel.cu:314-323)
template <int D>
__device__ __forceinline__ int conn_dir(const pict_block_t& B, int f, int d) {
    const int rel = (((d >> 1) - (f >> 1)) % D + D) % D;
    return B.face[f].conn_axes[rel] ^ (d & 1);
}

// data kinds of the corner values: structure only (matrices), velocity result, pressure result, passive scalar result
enum { NK_FLAG = 0, NK_VEL = 1, NK_P = 2, NK_SC = 3 };

// passive scalar viscosity of channel c (getViscosity with forPassiveScalar, extensions/PISO_multiblock_cuda_kernel.cu:1788-1799):
// the domain's scalar viscosity, else the domain viscosity
template <typename T>
__device__ __forceinline__ T scalar_nu(const pict_domain_t& dom, const pict_block_t& B, int c) {
    if (dom.scalar_viscosity) {
        const T* v = reinterpret_cast<const T*>(dom.scalar_viscosity);
        return dom.scalar_viscosity_static ? v[0] : v[c];
    }
    return reinterpret_cast<const T*>(dom.sim_viscosity)[B.sim];
}

// boundary type of passive scalar channel c at a fixed face (getFixedBoundaryType, extensions/PISO_multiblock_cuda_kernel.cu:2353-2376)
__device__ __forceinline__ bool scalar_neumann(const pict_domain_t& dom, int b, int f, int c) {
    return (dom.blocks[b].face[f].scalar_neumann >> c) & 1u;
}

// fixed boundary data (getFixedBoundaryData, extensions/PISO_multiblock_cuda_kernel.cu:2379-2447): velocity
// component c; the fixed boundary pressure is a static zero; the structure kind reads 1
template <typename T, int D, int KIND>
__device__ __forceinline__ T fixed_data(const pict_block_t& B, int f, const int* q, int c) {
    if (KIND == NK_FLAG) return T(1);
    if (KIND == NK_P) return T(0);
    const pict_face_t& F = B.face[f];
    if (KIND == NK_SC) {
        const T* v = reinterpret_cast<const T*>(F.scalar);
        if (!v) return T(0);
        if (F.scalar_static) return v[c];
        return v[(size_t)c * face_cells(B.size, f) + boundary_flat(q, B.size, f)];
    }
    const T* v = reinterpret_cast<const T*>(F.velocity);
    if (F.vel_static) return v[c];
    return v[(size_t)c * face_cells(B.size, f) + boundary_flat(q, B.size, f)];
}

template <typename T, int KIND>
__device__ __forceinline__ T cell_data(const pict_domain_t& dom, int b, const int* q, const T* data) {
    if (KIND == NK_FLAG) return T(0);
    const pict_block_t& B = dom.blocks[b];
    return data[B.offset + flat3(B.size, q)];
}

template <typename T>
struct Corner {
    T value;
    int cells;     // 0: the value comes from a fixed boundary
    bool neumann;  // boundary type of that fixed boundary
};

// What a corner value reads, in the order of getCornerValue (extensions/PISO_multiblock_cuda_kernel.cu:2742-2860)
// without the centre cell, depth 2: the data cells summed (value = sum / cells), or, when the walk hits a
// fixed face (cells == 0), the one or two boundary entries averaged.
struct CornerWalk {
    int cells;
    int nvis;
    int vb[4];
    int vp[4][3];
    int fb, ff, nfp;
    int fp[2][3];
};

// walk around the corner between faces dir1 and dir2 in both directions until the walks meet
template <int D>
__device__ void corner_walk(const pict_domain_t& dom, int b0, const int* p0, int dir1, int dir2, bool incl1,
                            CornerWalk& w) {
    w.nvis = 0;
    int n = 1;
    int wd1[2] = {dir1, dir2}, wd2[2] = {dir2, dir1}, wb[2] = {b0, b0};
    int wp[2][3] = {{p0[0], p0[1], p0[2]}, {p0[0], p0[1], p0[2]}};
    for (int depth = 1; depth <= 2; ++depth) {
        for (int d = 0; d < 2; ++d) {
            const pict_block_t& B = dom.blocks[wb[d]];
            const int d1 = wd1[d], d2 = wd2[d];
            const int a = d1 >> 1;
            if (at_face(wp[d], B.size, d1)) {
                const pict_face_t& F = B.face[d1];
                if (F.type == PICT_FACE_FIXED) {
                    w.cells = 0;
                    w.fb = wb[d];
                    w.ff = d1;
                    w.fp[0][0] = wp[d][0];
                    w.fp[0][1] = wp[d][1];
                    w.fp[0][2] = wp[d][2];
                    if (at_face(wp[d], B.size, d2)) {
                        w.nfp = 1;
                    } else {
                        w.nfp = 2;
                        w.fp[1][0] = wp[d][0];
                        w.fp[1][1] = wp[d][1];
                        w.fp[1][2] = wp[d][2];
                        w.fp[1][d2 >> 1] += (d2 & 1) ? 1 : -1;
                    }
                    return;
                }
                if (F.type == PICT_FACE_CONNECTED) {
                    int q[3];
                    const int nb = conn_pos<D>(dom, B, d1, wp[d], 1, q);
                    wd1[d] = conn_dir<D>(B, d1, d2);
                    wd2[d] = conn_dir<D>(B, d1, d1) ^ 1;
                    wb[d] = nb;
                    wp[d][0] = q[0];
                    wp[d][1] = q[1];
                    wp[d][2] = q[2];
                } else {  // periodic
                    wp[d][a] = (d1 & 1) ? 0 : B.size[a] - 1;
                    wd1[d] = d2;
                    wd2[d] = d1 ^ 1;
                }
            } else {
                wp[d][a] += (d1 & 1) ? 1 : -1;
                wd1[d] = d2;
                wd2[d] = d1 ^ 1;
            }
            const int o = d ^ 1;
            if (wb[d] == wb[o] && wp[d][0] == wp[o][0] && wp[d][1] == wp[o][1] && wp[d][2] == wp[o][2]) {
                w.cells = n;
                return;
            }
            if (depth > 1 || incl1) {
                w.vb[w.nvis] = wb[d];
                w.vp[w.nvis][0] = wp[d][0];
                w.vp[w.nvis][1] = wp[d][1];
                w.vp[w.nvis][2] = wp[d][2];
                ++w.nvis;
            }
            ++n;
        }
    }
    w.cells = n;
}

template <typename T, int D, int KIND>
__device__ Corner<T> corner_value(const pict_domain_t& dom, int b0, const int* p0, int dir1, int dir2, bool incl1,
                                  int comp, const T* data) {
    CornerWalk w;
    corner_walk<D>(dom, b0, p0, dir1, dir2, incl1, w);
    Corner<T> r;
    r.cells = w.cells;
    if (w.cells == 0) {
        const pict_block_t& B = dom.blocks[w.fb];
        r.neumann = (KIND == NK_P) || (KIND == NK_SC && scalar_neumann(dom, w.fb, w.ff, comp));
        r.value = w.nfp == 1 ? fixed_data<T, D, KIND>(B, w.ff, w.fp[0], comp)
                             : (fixed_data<T, D, KIND>(B, w.ff, w.fp[0], comp) + fixed_data<T, D, KIND>(B, w.ff, w.fp[1], comp)) *
                                   T(0.5);
        return r;
    }
    T acc = T(0);
    for (int k = 0; k < w.nvis; ++k) acc += cell_data<T, KIND>(dom, w.vb[k], w.vp[k], data);
    r.value = acc / T(w.cells);
    r.neumann = false;
    return r;
}

// Full Laplace coefficients det Minv[c1].Minv[c2] (getLaplaceCoefficientsFull, extensions/PISO_multiblock_cuda_kernel.cu:1270-1295)
template <typename T, int D>
__device__ __forceinline__ T lap(const T* tr, int c1, int c2) {
    if (!tr) return c1 == c2 ? T(1) : T(0);
    T s = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) s += tr_minv<T, D>(tr, c1, k) * tr_minv<T, D>(tr, c2, k);
    return tr_det<T, D>(tr) * s;
}

// ---------------------------------------------------------------------------------------------
// matrix terms: WHICH 0 = advection (viscosity, divided by det, C and A), 1 = pressure (1/A, P),
// 2 = passive scalar channel ch (scalar viscosity, divided by det, C and A; corners on the channel's
// Neumann faces take the one-sided treatment)
// ---------------------------------------------------------------------------------------------
template <typename T, int D, int WHICH>
__global__ void k_nonortho_matrix(pict_domain_t dom, int flags, int ch) {
    constexpr int K = 2 * D + 1;
    const int N = dom.num_cells;
    T* M = reinterpret_cast<T*>(WHICH == 1 ? dom.P : dom.C);
    T* Ad = reinterpret_cast<T*>(dom.A);
    const bool incl_nb = flags & NO_DIRECT_MATRIX, incl_diag = flags & NO_CENTER_MATRIX;
    const T sgn = WHICH == 1 ? T(1) : T(-1);
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T raP = WHICH == 0 ? cell_viscosity<T>(dom, B, l) : WHICH == 1 ? T(1) / Ad[i] : scalar_nu<T>(dom, B, ch);
        T add[K];
#pragma unroll
        for (int k = 0; k < K; ++k) add[k] = T(0);
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const bool fixed = face_fixed(B, f);
            if (at_face(p, B.size, f) && fixed) continue;  // prescribed face
            // interpolateNonOrthoLaplaceComponents: a face counts unless the cell is strictly inside along
            // its axis or the face is not a prescribed type
            if (!((0 < p[a] && p[a] < B.size[a] - 1) || !fixed)) continue;
            int q[3] = {p[0], p[1], p[2]};
            int nb = b;
            if (at_face(p, B.size, f) && B.face[f].type == PICT_FACE_CONNECTED) {
                nb = conn_pos<D>(dom, B, f, p, 0, q);
            } else if (at_face(p, B.size, f)) {
                q[a] = (f & 1) ? 0 : B.size[a] - 1;
            } else {
                q[a] += (f & 1) ? 1 : -1;
            }
            const pict_block_t& Bn = dom.blocks[nb];
            const int ln = flat3(Bn.size, q);
            const T* trn = cell_transform<T, D>(Bn, ln);
            const T raN = WHICH == 0 ? cell_viscosity<T>(dom, Bn, ln) : WHICH == 1 ? T(1) / Ad[Bn.offset + ln] : raP;
            const T fs = (f & 1) ? T(1) : T(-1);
#pragma unroll
            for (int k = 1; k < D; ++k) {
                const int t = (a + k) % D;
                const T alpha = (lap<T, D>(tr, a, t) * raP + lap<T, D>(trn, t, a) * raN) * T(0.5);
                if (alpha == T(0)) continue;
#pragma unroll
                for (int tup = 0; tup < 2; ++tup) {
                    const int tf = 2 * t + tup;
                    const T ts = tup ? T(1) : T(-1);
                    CornerWalk cv;
                    corner_walk<D>(dom, b, p, f, tf, false, cv);
                    // fixed velocity faces are Dirichlet; pressure faces are Neumann; scalar faces per channel
                    const bool grad = WHICH == 0 ? false : WHICH == 1 ? true : (cv.cells < 1 && scalar_neumann(dom, cv.fb, cv.ff, ch));
                    if (cv.cells < 1) {
                        if (grad) {
                            const T v = fs * ts * alpha * T(0.25);
                            if (incl_diag) add[0] += sgn * T(3) * v;
                            if (incl_nb) {
                                add[f + 1] += sgn * T(3) * v;
                                add[(tf ^ 1) + 1] -= sgn * v;
                            }
                        }
                    } else {
                        const T v = fs * ts * alpha / T(cv.cells);
                        if (incl_diag) add[0] += sgn * v;
                        if (incl_nb) {
                            add[f + 1] += sgn * v;
                            add[tf + 1] += sgn * v;
                        }
                    }
                }
            }
        }
        const T scale = WHICH != 1 ? T(1) / tr_det<T, D>(tr) : T(1);
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (add[k] != T(0)) M[(size_t)k * N + i] += add[k] * scale;
        if (WHICH != 1) Ad[i] = M[i];
    }
}

// ---------------------------------------------------------------------------------------------
// right-hand-side terms (getNonOrthoLaplaceRHS_v2): KIND NK_VEL subtracts them from the velocity RHS
// (viscosity, divided by det), KIND NK_P adds them to the pressure RHS divergence (1/A)
// ---------------------------------------------------------------------------------------------

// getBlockDataNeighbor (extensions/PISO_multiblock_cuda_kernel.cu:2519-2560), second layer across connections
template <typename T, int D, int KIND>
__device__ T neighbor_data(const pict_domain_t& dom, int b, const int* p, int f, int comp, const T* data) {
    const pict_block_t& B = dom.blocks[b];
    const int a = f >> 1;
    int q[3] = {p[0], p[1], p[2]};
    int nb = b;
    if (at_face(p, B.size, f)) {
        if (B.face[f].type == PICT_FACE_FIXED) return fixed_data<T, D, KIND>(B, f, p, comp);
        if (B.face[f].type == PICT_FACE_CONNECTED) nb = conn_pos<D>(dom, B, f, p, 1, q);
        else q[a] = (f & 1) ? 0 : B.size[a] - 1;
    } else {
        q[a] += (f & 1) ? 1 : -1;
    }
    return cell_data<T, KIND>(dom, nb, q, data);
}

// getBlockDataNeighborDiagonal (extensions/PISO_multiblock_cuda_kernel.cu:2615-2660)
template <typename T, int D, int KIND>
__device__ T diagonal_data(const pict_domain_t& dom, int b, const int* p, int dir1, int dir2, int comp, const T* data) {
    const bool first_fixed = face_fixed(dom.blocks[b], dir1);
    const int dirs[2] = {first_fixed ? dir2 : dir1, first_fixed ? dir1 : dir2};
    int cb = b;
    int q[3] = {p[0], p[1], p[2]};
    for (int s = 0; s < 2; ++s) {
        const int f = dirs[s];
        const pict_block_t& B = dom.blocks[cb];
        const int a = f >> 1;
        if (at_face(q, B.size, f)) {
            if (B.face[f].type == PICT_FACE_FIXED) return fixed_data<T, D, KIND>(B, f, q, comp);
            if (B.face[f].type == PICT_FACE_CONNECTED) {
                int r[3];
                cb = conn_pos<D>(dom, B, f, q, 1, r);
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
            } else {
                q[a] = (f & 1) ? 0 : B.size[a] - 1;
            }
        } else {
            q[a] += (f & 1) ? 1 : -1;
        }
    }
    return cell_data<T, KIND>(dom, cb, q, data);
}

template <typename T, int D, int KIND>
__global__ void k_nonortho_rhs(pict_domain_t dom, int flags) {
    const int NC = KIND == NK_VEL ? D : KIND == NK_SC ? dom.scalar_channels : 1;
    const int N = dom.num_cells;
    const T* Ad = reinterpret_cast<const T*>(dom.A);
    const T* data = reinterpret_cast<const T*>(KIND == NK_VEL ? dom.velocity_result
                                               : KIND == NK_SC ? dom.scalar_result : dom.pressure_result);
    T* out = reinterpret_cast<T*>(KIND == NK_VEL ? dom.velocity_rhs : KIND == NK_SC ? dom.scalar_rhs : dom.pressure_rhs_div);
    const bool incl1 = flags & NO_DIRECT_RHS;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T raP0 = KIND == NK_VEL ? cell_viscosity<T>(dom, B, l) : KIND == NK_SC ? T(0) : T(1) / Ad[i];
#pragma unroll 1
        for (int c = 0; c < NC; ++c) {
            const T raP = KIND == NK_SC ? scalar_nu<T>(dom, B, c) : raP0;
            const T* dc = data + (size_t)c * N;
            T S = T(0);
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                const int a = f >> 1;
                const T fs = (f & 1) ? T(1) : T(-1);
                if (at_face(p, B.size, f) && face_fixed(B, f)) {
                    if (KIND == NK_P) continue;  // pressure: zero normal gradient at fixed faces
                    if (KIND == NK_SC && scalar_neumann(dom, b, f, c)) continue;
                    // velocity (Dirichlet): tangential gradient of the boundary data
                    const pict_face_t& F = B.face[f];
                    const int bf = boundary_flat(p, B.size, f);
                    const T* btr = F.transform ? reinterpret_cast<const T*>(F.transform) + (size_t)bf * TS<D>::value : nullptr;
#pragma unroll
                    for (int k = 1; k < D; ++k) {
                        const int t = (a + k) % D;
                        const bool tlo = p[t] == 0, thi = p[t] == B.size[t] - 1;
                        int lo[3] = {p[0], p[1], p[2]}, hi[3] = {p[0], p[1], p[2]};
                        if (!tlo) lo[t] -= 1;
                        if (!thi) hi[t] += 1;
                        const T df = (tlo || thi) ? T(1) : T(0.5);
                        const T tg = df * (fixed_data<T, D, KIND>(B, f, hi, c) - fixed_data<T, D, KIND>(B, f, lo, c));
                        S -= fs * lap<T, D>(btr, t, a) * tg * raP;
                    }
                    continue;
                }
                // the neighbour across f (resolveNeighborCell) with its axis mapping
                int q[3] = {p[0], p[1], p[2]};
                int nb = b;
                int map[3] = {0, 2, 4};
                if (at_face(p, B.size, f) && B.face[f].type == PICT_FACE_CONNECTED) {
                    nb = conn_pos<D>(dom, B, f, p, 0, q);
#pragma unroll
                    for (int k = 0; k < D; ++k) map[k] = conn_dir<D>(B, f, map[k]);
                } else if (at_face(p, B.size, f)) {
                    q[a] = (f & 1) ? 0 : B.size[a] - 1;
                } else {
                    q[a] += (f & 1) ? 1 : -1;
                }
                const pict_block_t& Bn = dom.blocks[nb];
                const int ln = flat3(Bn.size, q);
                const T* trn = cell_transform<T, D>(Bn, ln);
                const T raN = KIND == NK_VEL ? cell_viscosity<T>(dom, Bn, ln) : KIND == NK_SC ? raP : T(1) / Ad[Bn.offset + ln];
#pragma unroll
                for (int k = 1; k < D; ++k) {
                    const int t = (a + k) % D;
                    // getLaplaceCoefficientsSingleAxisNeighbor with the axis mapping of the connection
                    const T aN = lap<T, D>(trn, map[t] >> 1, map[a] >> 1);
                    const T fa = (lap<T, D>(tr, a, t) * raP + aN * raN) * T(0.5);
                    T tg = T(0);
#pragma unroll
                    for (int tup = 0; tup < 2; ++tup) {
                        const int tf = 2 * t + tup;
                        const T ts = tup ? T(1) : T(-1);
                        const Corner<T> cv = corner_value<T, D, KIND>(dom, b, p, f, tf, incl1, c, dc);
                        if (cv.cells == 0 && (cv.neumann || KIND == NK_P)) {
                            const int to = tf ^ 1;
                            if (flags & NO_DIRECT_RHS) {
                                tg += ts * neighbor_data<T, D, KIND>(dom, b, p, f, c, dc) * T(0.75);
                                tg -= ts * neighbor_data<T, D, KIND>(dom, b, p, to, c, dc) * T(0.25);
                            }
                            if (flags & NO_DIAGONAL_RHS) tg -= ts * diagonal_data<T, D, KIND>(dom, b, p, f, to, c, dc) * T(0.25);
                        } else {
                            tg += ts * cv.value;
                        }
                    }
                    S -= fs * fa * tg;
                }
            }
            if (KIND == NK_P) out[i] += S;
            else out[(size_t)c * N + i] -= S / tr_det<T, D>(tr);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// gradients (the non-orthogonal parts of the reference's *_GRAD kernels: scatterNonOrthoLaplaceComponents_GRAD
// extensions/PISO_multiblock_cuda_kernel.cu:1992-2098, scatterNonOrthoLaplaceRHS_v2_GRAD :3212-3392, and their
// callers in the matrix and RHS gradient kernels).  The terms are linear in the result fields and in
// the face coefficients alpha = (a_P r_P + a_N r_N) / 2 with r = viscosity (advection) or 1/A
// (pressure); each thread recomputes its cell's terms and scatters their adjoints with atomics to
// the cells they read (the reference scatters with atomics too).
// ---------------------------------------------------------------------------------------------

// location read by getBlockDataNeighbor: a data cell (true, block nb, position q) or a fixed face (false)
template <int D>
__device__ bool neighbor_loc(const pict_domain_t& dom, int b, const int* p, int f, int& nb, int* q) {
    const pict_block_t& B = dom.blocks[b];
    const int a = f >> 1;
    nb = b;
    q[0] = p[0];
    q[1] = p[1];
    q[2] = p[2];
    if (at_face(p, B.size, f)) {
        if (B.face[f].type == PICT_FACE_FIXED) return false;
        if (B.face[f].type == PICT_FACE_CONNECTED) nb = conn_pos<D>(dom, B, f, p, 1, q);
        else q[a] = (f & 1) ? 0 : B.size[a] - 1;
    } else {
        q[a] += (f & 1) ? 1 : -1;
    }
    return true;
}

// location read by getBlockDataNeighborDiagonal
template <int D>
__device__ bool diagonal_loc(const pict_domain_t& dom, int b, const int* p, int dir1, int dir2, int& cb, int* q) {
    const bool first_fixed = face_fixed(dom.blocks[b], dir1);
    const int dirs[2] = {first_fixed ? dir2 : dir1, first_fixed ? dir1 : dir2};
    cb = b;
    q[0] = p[0];
    q[1] = p[1];
    q[2] = p[2];
    for (int s = 0; s < 2; ++s) {
        const int f = dirs[s];
        const pict_block_t& B = dom.blocks[cb];
        const int a = f >> 1;
        if (at_face(q, B.size, f)) {
            if (B.face[f].type == PICT_FACE_FIXED) return false;
            if (B.face[f].type == PICT_FACE_CONNECTED) {
                int r[3];
                cb = conn_pos<D>(dom, B, f, q, 1, r);
                q[0] = r[0];
                q[1] = r[1];
                q[2] = r[2];
            } else {
                q[a] = (f & 1) ? 0 : B.size[a] - 1;
            }
        } else {
            q[a] += (f & 1) ? 1 : -1;
        }
    }
    return true;
}

template <typename T>
__device__ __forceinline__ void atomic_add(T* p, T v) {
    if (v != T(0)) atomicAdd(p, v);
}

// matrix terms: M_bar (C_grad / P_grad [K][N]) and, for the advection matrices, A_bar (A = C[0]) to the
// coefficient adjoint: viscosity (WHICH 0), A (WHICH 1) or the scalar viscosity of channel ch (WHICH 2),
// per cell
template <typename T, int D, int WHICH>
__global__ void k_nonortho_matrix_grad(pict_domain_t dom, int flags, const T* Mbar, const T* Abar, T* coef_bar, int ch) {
    constexpr int K = 2 * D + 1;
    const int N = dom.num_cells;
    const T* Ad = reinterpret_cast<const T*>(dom.A);
    const bool incl_nb = flags & NO_DIRECT_MATRIX, incl_diag = flags & NO_CENTER_MATRIX;
    const T sgn = WHICH == 1 ? T(1) : T(-1);
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T raP = WHICH == 0 ? cell_viscosity<T>(dom, B, l) : WHICH == 1 ? T(1) / Ad[i] : scalar_nu<T>(dom, B, ch);
        const T scale = WHICH != 1 ? T(1) / tr_det<T, D>(tr) : T(1);
        T mb[K];
#pragma unroll
        for (int k = 0; k < K; ++k) mb[k] = Mbar[(size_t)k * N + i] * scale;
        if (WHICH != 1 && Abar) mb[0] += Abar[i] * scale;
        T raP_bar = T(0);
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const bool fixed = face_fixed(B, f);
            if (at_face(p, B.size, f) && fixed) continue;
            if (!((0 < p[a] && p[a] < B.size[a] - 1) || !fixed)) continue;
            int q[3] = {p[0], p[1], p[2]};
            int nb = b;
            if (at_face(p, B.size, f) && B.face[f].type == PICT_FACE_CONNECTED) nb = conn_pos<D>(dom, B, f, p, 0, q);
            else if (at_face(p, B.size, f)) q[a] = (f & 1) ? 0 : B.size[a] - 1;
            else q[a] += (f & 1) ? 1 : -1;
            const pict_block_t& Bn = dom.blocks[nb];
            const int ln = flat3(Bn.size, q);
            const int gN = Bn.offset + ln;
            const T* trn = cell_transform<T, D>(Bn, ln);
            const T raN = WHICH == 0 ? cell_viscosity<T>(dom, Bn, ln) : WHICH == 1 ? T(1) / Ad[gN] : raP;
            const T fs = (f & 1) ? T(1) : T(-1);
#pragma unroll
            for (int k = 1; k < D; ++k) {
                const int t = (a + k) % D;
                const T aP = lap<T, D>(tr, a, t), aN = lap<T, D>(trn, t, a);
                // the reference's gradient tests the geometric coefficient, without viscosity or 1/A
                if ((aP + aN) * T(0.5) == T(0)) continue;
                T alpha_bar = T(0);  // d L / d alpha
#pragma unroll
                for (int tup = 0; tup < 2; ++tup) {
                    const int tf = 2 * t + tup;
                    const T ts = tup ? T(1) : T(-1);
                    CornerWalk w;
                    corner_walk<D>(dom, b, p, f, tf, false, w);
                    // fixed velocity faces are Dirichlet, pressure faces Neumann, scalar faces per channel
                    const bool grad = WHICH == 0 ? false : WHICH == 1 ? true : (w.cells < 1 && scalar_neumann(dom, w.fb, w.ff, ch));
                    if (w.cells < 1) {
                        if (grad) {
                            const T v = fs * ts * T(0.25);
                            if (incl_diag) alpha_bar += mb[0] * sgn * T(3) * v;
                            if (incl_nb) alpha_bar += mb[f + 1] * sgn * T(3) * v - mb[(tf ^ 1) + 1] * sgn * v;
                        }
                    } else {
                        const T v = fs * ts / T(w.cells);
                        if (incl_diag) alpha_bar += mb[0] * sgn * v;
                        if (incl_nb) alpha_bar += (mb[f + 1] + mb[tf + 1]) * sgn * v;
                    }
                }
                raP_bar += alpha_bar * aP * T(0.5);
                const T rN_bar = alpha_bar * aN * T(0.5);
                atomic_add(coef_bar + gN, WHICH != 1 ? rN_bar : rN_bar * (-raN * raN));
            }
        }
        atomic_add(coef_bar + i, WHICH != 1 ? raP_bar : raP_bar * (-raP * raP));
    }
}

// RHS terms: out_bar (velocityRHS_grad [D][N] or scalarRHS_grad [C][N], the term entering as -S/det; or
// pressureRHSdiv_grad [N], entering as +S) to the result field (data_bar), the coefficient adjoint
// (viscosity [N], A [N], scalar viscosity [C][N]) and the fixed boundary data (velocity or scalar,
// vb_bar [2D][D or C][N], per adjacent cell)
template <typename T, int D, int KIND>
__global__ void k_nonortho_rhs_grad(pict_domain_t dom, int flags, const T* out_bar, T* data_bar, T* coef_bar,
                                    T* vb_bar) {
    const int NC = KIND == NK_VEL ? D : KIND == NK_SC ? dom.scalar_channels : 1;
    const int N = dom.num_cells;
    const T* Ad = reinterpret_cast<const T*>(dom.A);
    const T* data = reinterpret_cast<const T*>(KIND == NK_VEL ? dom.velocity_result
                                               : KIND == NK_SC ? dom.scalar_result : dom.pressure_result);
    const bool incl1 = flags & NO_DIRECT_RHS;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T raP0 = KIND == NK_VEL ? cell_viscosity<T>(dom, B, l) : KIND == NK_SC ? T(0) : T(1) / Ad[i];
        T raP_bar = T(0);
#pragma unroll 1
        for (int c = 0; c < NC; ++c) {
            const T raP = KIND == NK_SC ? scalar_nu<T>(dom, B, c) : raP0;
            T* cb_c = coef_bar + (KIND == NK_SC ? (size_t)c * N : 0);
            if (KIND == NK_SC) raP_bar = T(0);
            const T sbar = KIND == NK_P ? out_bar[i] : -out_bar[(size_t)c * N + i] / tr_det<T, D>(tr);
            if (sbar == T(0)) continue;
            const T* dc = data + (size_t)c * N;
            T* dcb = data_bar + (size_t)c * N;
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                const int a = f >> 1;
                const T fs = (f & 1) ? T(1) : T(-1);
                if (at_face(p, B.size, f) && face_fixed(B, f)) {
                    if (KIND == NK_P) continue;
                    if (KIND == NK_SC && scalar_neumann(dom, b, f, c)) continue;
                    const pict_face_t& F = B.face[f];
                    const int bf = boundary_flat(p, B.size, f);
                    const T* btr = F.transform ? reinterpret_cast<const T*>(F.transform) + (size_t)bf * TS<D>::value : nullptr;
#pragma unroll
                    for (int k = 1; k < D; ++k) {
                        const int t = (a + k) % D;
                        const bool tlo = p[t] == 0, thi = p[t] == B.size[t] - 1;
                        int lo[3] = {p[0], p[1], p[2]}, hi[3] = {p[0], p[1], p[2]};
                        if (!tlo) lo[t] -= 1;
                        if (!thi) hi[t] += 1;
                        const T df = (tlo || thi) ? T(1) : T(0.5);
                        const T bal = lap<T, D>(btr, t, a);
                        const T tg = df * (fixed_data<T, D, KIND>(B, f, hi, c) - fixed_data<T, D, KIND>(B, f, lo, c));
                        raP_bar += sbar * (-fs * bal * tg);
                        const T wv = sbar * (-fs * bal * raP) * df;
                        atomic_add(vb_bar + ((size_t)f * NC + c) * N + B.offset + flat3(B.size, hi), wv);
                        atomic_add(vb_bar + ((size_t)f * NC + c) * N + B.offset + flat3(B.size, lo), -wv);
                    }
                    continue;
                }
                int q[3] = {p[0], p[1], p[2]};
                int nb = b;
                int map[3] = {0, 2, 4};
                if (at_face(p, B.size, f) && B.face[f].type == PICT_FACE_CONNECTED) {
                    nb = conn_pos<D>(dom, B, f, p, 0, q);
#pragma unroll
                    for (int k = 0; k < D; ++k) map[k] = conn_dir<D>(B, f, map[k]);
                } else if (at_face(p, B.size, f)) {
                    q[a] = (f & 1) ? 0 : B.size[a] - 1;
                } else {
                    q[a] += (f & 1) ? 1 : -1;
                }
                const pict_block_t& Bn = dom.blocks[nb];
                const int ln = flat3(Bn.size, q);
                const int gN = Bn.offset + ln;
                const T* trn = cell_transform<T, D>(Bn, ln);
                const T raN = KIND == NK_VEL ? cell_viscosity<T>(dom, Bn, ln) : KIND == NK_SC ? raP : T(1) / Ad[gN];
#pragma unroll
                for (int k = 1; k < D; ++k) {
                    const int t = (a + k) % D;
                    const T aN = lap<T, D>(trn, map[t] >> 1, map[a] >> 1);
                    const T aP = lap<T, D>(tr, a, t);
                    const T fa = (aP * raP + aN * raN) * T(0.5);
                    T tg = T(0);
                    const T tg_bar = sbar * (-fs * fa);
#pragma unroll
                    for (int tup = 0; tup < 2; ++tup) {
                        const int tf = 2 * t + tup;
                        const T ts = tup ? T(1) : T(-1);
                        CornerWalk w;
                        corner_walk<D>(dom, b, p, f, tf, incl1, w);
                        // fixed velocity faces are Dirichlet, pressure faces Neumann, scalar faces per channel
                        const bool grad_bound = (w.cells == 0) &&
                                                (KIND == NK_P || (KIND == NK_SC && scalar_neumann(dom, w.fb, w.ff, c)));
                        if (grad_bound) {
                            const int to = tf ^ 1;
                            int cb;
                            int r[3];
                            if (flags & NO_DIRECT_RHS) {
                                if (neighbor_loc<D>(dom, b, p, f, cb, r)) {
                                    const int j = dom.blocks[cb].offset + flat3(dom.blocks[cb].size, r);
                                    tg += ts * dc[j] * T(0.75);
                                    atomic_add(dcb + j, tg_bar * ts * T(0.75));
                                }
                                if (neighbor_loc<D>(dom, b, p, to, cb, r)) {
                                    const int j = dom.blocks[cb].offset + flat3(dom.blocks[cb].size, r);
                                    tg -= ts * dc[j] * T(0.25);
                                    atomic_add(dcb + j, -tg_bar * ts * T(0.25));
                                }
                            }
                            if ((flags & NO_DIAGONAL_RHS) && diagonal_loc<D>(dom, b, p, f, to, cb, r)) {
                                const int j = dom.blocks[cb].offset + flat3(dom.blocks[cb].size, r);
                                tg -= ts * dc[j] * T(0.25);
                                atomic_add(dcb + j, -tg_bar * ts * T(0.25));
                            }
                        } else if (w.cells == 0) {
                            const pict_block_t& Bf = dom.blocks[w.fb];
                            const T wgt = w.nfp == 1 ? T(1) : T(0.5);
                            for (int k2 = 0; k2 < w.nfp; ++k2) {
                                tg += ts * wgt * fixed_data<T, D, KIND>(Bf, w.ff, w.fp[k2], c);
                                atomic_add(vb_bar + ((size_t)w.ff * NC + c) * N + Bf.offset + flat3(Bf.size, w.fp[k2]),
                                           tg_bar * ts * wgt);
                            }
                        } else {
                            T acc = T(0);
                            for (int k2 = 0; k2 < w.nvis; ++k2) {
                                const int j = dom.blocks[w.vb[k2]].offset + flat3(dom.blocks[w.vb[k2]].size, w.vp[k2]);
                                acc += dc[j];
                                atomic_add(dcb + j, tg_bar * ts / T(w.cells));
                            }
                            tg += ts * (acc / T(w.cells));
                        }
                    }
                    const T fa_bar = sbar * (-fs * tg);
                    raP_bar += fa_bar * aP * T(0.5);
                    const T rN_bar = fa_bar * aN * T(0.5);
                    atomic_add(cb_c + gN, KIND == NK_P ? rN_bar * (-raN * raN) : rN_bar);
                }
            }
            if (KIND == NK_SC) atomic_add(cb_c + i, raP_bar);
        }
        if (KIND != NK_SC) atomic_add(coef_bar + i, KIND == NK_VEL ? raP_bar : raP_bar * (-raP0 * raP0));
    }
}

template <typename T, int D>
static pict_status_t launch_nonortho_grad(const pict_domain_t* dom, int flags, int what, int ch, const void* out_bar,
                                          const void* A_bar, void* data_bar, void* coef_bar, void* vb_bar,
                                          cudaStream_t st) {
    const int grid = cell_grid(dom->num_cells, 128);
    switch (what) {
        case 0:
            k_nonortho_matrix_grad<T, D, 0><<<grid, 128, 0, st>>>(*dom, flags, (const T*)out_bar, (const T*)A_bar,
                                                                  (T*)coef_bar, 0);
            break;
        case 4:
            k_nonortho_matrix_grad<T, D, 2><<<grid, 128, 0, st>>>(*dom, flags, (const T*)out_bar, (const T*)A_bar,
                                                                  (T*)coef_bar, ch);
            break;
        case 5:
            k_nonortho_rhs_grad<T, D, NK_SC><<<grid, 128, 0, st>>>(*dom, flags, (const T*)out_bar, (T*)data_bar,
                                                                   (T*)coef_bar, (T*)vb_bar);
            break;
        case 1:
            k_nonortho_rhs_grad<T, D, NK_VEL><<<grid, 128, 0, st>>>(*dom, flags, (const T*)out_bar, (T*)data_bar,
                                                                    (T*)coef_bar, (T*)vb_bar);
            break;
        case 2:
            k_nonortho_matrix_grad<T, D, 1><<<grid, 128, 0, st>>>(*dom, flags, (const T*)out_bar, nullptr, (T*)coef_bar, 0);
            break;
        default:
            k_nonortho_rhs_grad<T, D, NK_P><<<grid, 128, 0, st>>>(*dom, flags, (const T*)out_bar, (T*)data_bar,
                                                                  (T*)coef_bar, (T*)vb_bar);
            break;
    }
    return check_launch("nonortho_grad");
}

template <typename T, int D>
static pict_status_t launch_nonortho(const pict_domain_t* dom, int flags, int what, int ch, cudaStream_t st) {
    const int grid = cell_grid(dom->num_cells, 128);
    switch (what) {
        case 0: k_nonortho_matrix<T, D, 0><<<grid, 128, 0, st>>>(*dom, flags, 0); break;
        case 1: k_nonortho_rhs<T, D, NK_VEL><<<grid, 128, 0, st>>>(*dom, flags); break;
        case 2: k_nonortho_matrix<T, D, 1><<<grid, 128, 0, st>>>(*dom, flags, 0); break;
        case 4: k_nonortho_matrix<T, D, 2><<<grid, 128, 0, st>>>(*dom, flags, ch); break;
        case 5: k_nonortho_rhs<T, D, NK_SC><<<grid, 128, 0, st>>>(*dom, flags); break;
        default: k_nonortho_rhs<T, D, NK_P><<<grid, 128, 0, st>>>(*dom, flags); break;
    }
    return check_launch("nonortho");
}

pict_status_t nonortho_pass(const pict_domain_t* dom, int32_t flags, int32_t what, void* stream) {
    return nonortho_pass_ch(dom, flags, what, 0, stream);
}

pict_status_t nonortho_pass_ch(const pict_domain_t* dom, int32_t flags, int32_t what, int32_t ch, void* stream) {
    const bool matrix = (what == 0 || what == 2 || what == 4);
    if (matrix && !(flags & (NO_DIRECT_MATRIX | NO_CENTER_MATRIX))) return PICT_OK;
    if (!matrix && !(flags & (NO_DIRECT_RHS | NO_DIAGONAL_RHS))) return PICT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) return launch_nonortho<float, 2>(dom, flags, what, ch, st);
        if (dom->dims == 3) return launch_nonortho<float, 3>(dom, flags, what, ch, st);
    } else if (dom->dtype == PICT_F64) {
        if (dom->dims == 2) return launch_nonortho<double, 2>(dom, flags, what, ch, st);
        if (dom->dims == 3) return launch_nonortho<double, 3>(dom, flags, what, ch, st);
    }
    return set_error(PICT_ERR_UNSUPPORTED, "non-orthogonal terms: unsupported dtype/dims");
}

pict_status_t nonortho_grad_scalar(const pict_domain_t* dom, int32_t flags, int32_t what, int32_t ch, const void* out_bar,
                                   const void* A_bar, void* data_bar, void* coef_bar, void* sb_bar, void* stream) {
    const bool matrix = what == 4;
    if (matrix && !(flags & (NO_DIRECT_MATRIX | NO_CENTER_MATRIX))) return PICT_OK;
    if (!matrix && !(flags & (NO_DIRECT_RHS | NO_DIAGONAL_RHS))) return PICT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) return launch_nonortho_grad<float, 2>(dom, flags, what, ch, out_bar, A_bar, data_bar, coef_bar, sb_bar, st);
        if (dom->dims == 3) return launch_nonortho_grad<float, 3>(dom, flags, what, ch, out_bar, A_bar, data_bar, coef_bar, sb_bar, st);
    } else if (dom->dtype == PICT_F64) {
        if (dom->dims == 2) return launch_nonortho_grad<double, 2>(dom, flags, what, ch, out_bar, A_bar, data_bar, coef_bar, sb_bar, st);
        if (dom->dims == 3) return launch_nonortho_grad<double, 3>(dom, flags, what, ch, out_bar, A_bar, data_bar, coef_bar, sb_bar, st);
    }
    return set_error(PICT_ERR_UNSUPPORTED, "nonortho_grad: unsupported dtype/dims");
}

}  // namespace pict

using namespace pict;

extern "C" pict_status_t pict_nonortho_grad(const pict_domain_t* dom, int32_t flags, int32_t what, const void* out_bar,
                                            const void* A_bar, void* data_bar, void* coef_bar,
                                            void* boundary_velocity_grad, void* stream) {
    if (!dom || !out_bar || !coef_bar) return set_error(PICT_ERR_ARG, "nonortho_grad: NULL argument");
    if (what < 0 || what > 3) return set_error(PICT_ERR_ARG, "nonortho_grad: what must be 0..3");
    if ((what == 1 || what == 3) && !data_bar) return set_error(PICT_ERR_ARG, "nonortho_grad: data gradient missing");
    if (what == 1 && !boundary_velocity_grad) return set_error(PICT_ERR_ARG, "nonortho_grad: boundary gradient missing");
    const bool matrix = (what == 0 || what == 2);
    if (matrix && !(flags & (NO_DIRECT_MATRIX | NO_CENTER_MATRIX))) return PICT_OK;
    if (!matrix && !(flags & (NO_DIRECT_RHS | NO_DIAGONAL_RHS))) return PICT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2)
            return launch_nonortho_grad<float, 2>(dom, flags, what, 0, out_bar, A_bar, data_bar, coef_bar, boundary_velocity_grad, st);
        if (dom->dims == 3)
            return launch_nonortho_grad<float, 3>(dom, flags, what, 0, out_bar, A_bar, data_bar, coef_bar, boundary_velocity_grad, st);
    } else if (dom->dtype == PICT_F64) {
        if (dom->dims == 2)
            return launch_nonortho_grad<double, 2>(dom, flags, what, 0, out_bar, A_bar, data_bar, coef_bar, boundary_velocity_grad, st);
        if (dom->dims == 3)
            return launch_nonortho_grad<double, 3>(dom, flags, what, 0, out_bar, A_bar, data_bar, coef_bar, boundary_velocity_grad, st);
    }
    return set_error(PICT_ERR_UNSUPPORTED, "nonortho_grad: unsupported dtype/dims");
}
