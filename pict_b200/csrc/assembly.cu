// assembly.cu -- per-cell assembly kernels of the PISO step (forward).
//
// One thread per cell over the global cell range of a (possibly batched)
// domain.  Stencil coefficients are written as coef[K][N] (structure of
// arrays, coalesced) instead of the reference's sorted CSR rows.
//
// Reference kernels restated here (kernel.cu = extensions/PISO_multiblock_cuda_kernel.cu):
//   PISO_build_matrix            extensions/PISO_multiblock_cuda_kernel.cu:3601-3865
//   kPISO_build_advection_RHS    extensions/PISO_multiblock_cuda_kernel.cu:4281-4385
//   PISO_build_pressure_matrix   extensions/PISO_multiblock_cuda_kernel.cu:4797-4963
//   PISO_build_pressure_rhs      extensions/PISO_multiblock_cuda_kernel.cu:5121-5240
//   k_computePressureRHSdivergenceFromFlux extensions/PISO_multiblock_cuda_kernel.cu:5374-5419
//   PISO_update_velocity (FD)    extensions/PISO_multiblock_cuda_kernel.cu:5947-5980 with getPressureGradient extensions/PISO_multiblock_cuda_kernel.cu:801-834
//   k_computeVelocityDivergenceFromFlux    extensions/PISO_multiblock_cuda_kernel.cu:6333-6357
#include "common.cuh"
#include "launch.h"

namespace pict {

// ---------------------------------------------------------------------------------------------
// advection matrix + RHS
// ---------------------------------------------------------------------------------------------

// Pressure gradient by central differences, one-sided at fixed faces, times Minv^T
// (getPressureGradient extensions/PISO_multiblock_cuda_kernel.cu:801-834, getPressureAtWithBounds extensions/PISO_multiblock_cuda_kernel.cu:2160-2239).
template <typename T, int D>
__device__ __forceinline__ void pressure_grad_fd(const pict_domain_t& dom, const pict_block_t& B, int b,
                                                 const int* p, int i, int l, const T* tr, T* g) {
    const T* pb = reinterpret_cast<const T*>(B.pressure);
    const T pc = pb[l];
    T gl[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        T fac = T(0.5);
        T vN, vP;
        const Nbr nl = neighbour(dom, B, b, p, i, 2 * d);
        if (nl.j < 0) { vN = pc; fac = T(1); }
        else vN = reinterpret_cast<const T*>(dom.blocks[nl.b].pressure)[nl.l];
        const Nbr nh = neighbour(dom, B, b, p, i, 2 * d + 1);
        if (nh.j < 0) { vP = pc; fac = T(1); }
        else vP = reinterpret_cast<const T*>(dom.blocks[nh.b].pressure)[nh.l];
        gl[d] = (vP - vN) * fac;
    }
    if (tr) {
#pragma unroll
        for (int c = 0; c < D; ++c) {
            T s = 0;
#pragma unroll
            for (int k = 0; k < D; ++k) s += gl[k] * tr_minv<T, D>(tr, k, c);
            g[c] = s;
        }
    } else {
#pragma unroll
        for (int c = 0; c < D; ++c) g[c] = gl[c];
    }
}

template <typename T, int D, bool MATRIX, bool RHS>
__global__ void __launch_bounds__(256, 6) k_adv_setup(pict_domain_t dom, double dt_arg, int apply_pgrad) {
    constexpr int K = 2 * D + 1;
    const int N = dom.num_cells;
    T* C = reinterpret_cast<T*>(dom.C);
    T* A = reinterpret_cast<T*>(dom.A);
    T* vrhs = reinterpret_cast<T*>(dom.velocity_rhs);
    for_each_cell(dom, [&](const int i, const int b) {
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T det = tr_det<T, D>(tr);
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
        T u[D];
        load_block_vec<T, D>(B, B.velocity, l, u);
        const T nu = cell_viscosity<T>(dom, B, l);

        T diag = det / dt;
        T off[2 * D];
        T rhs[D];
#pragma unroll
        for (int c = 0; c < D; ++c) rhs[c] = det * u[c] / dt;
        T alpha_p[D], velC[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            alpha_p[d] = laplace_coef<T, D>(tr, d);
            velC[d] = contravariant<T, D>(tr, d, u);
        }
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const T sign = (f & 1) ? T(1) : T(-1);
            const Nbr n = neighbour(dom, B, b, p, i, f);
            off[f] = T(0);
            if (n.j < 0) {
                // prescribed (fixed Dirichlet) face: diffusion towards the wall value, no advective
                // term in the matrix (extensions/PISO_multiblock_cuda_kernel.cu:3801-3833); wall sources on the RHS (extensions/PISO_multiblock_cuda_kernel.cu:4307-4327)
                if (MATRIX) diag += T(2) * nu * alpha_p[a];
                if (RHS) {
                    const FixedFace<T, D> ff = fixed_face<T, D>(B, p, f);
                    const T flux = ff.contra * sign;
#pragma unroll
                    for (int c = 0; c < D; ++c) rhs[c] += -ff.vel[c] * flux + ff.vel[c] * nu * T(2) * ff.alpha;
                }
            } else if (MATRIX) {
                const pict_block_t& Bn = dom.blocks[n.b];
                const T* trn = cell_transform<T, D>(Bn, n.l);
                T un[D];
                load_block_vec<T, D>(Bn, Bn.velocity, n.l, un);
                const T velN = contravariant<T, D>(trn, n.comp, un) * T(n.flip);
                const T flux = (velN + velC[a]) * T(0.5);
                const T faceFlux = sign * T(0.5) * flux;
                const T alpha_n = laplace_coef<T, D>(trn, n.comp);
                const T nu_n = cell_viscosity<T>(dom, Bn, n.l);
                const T vc = (alpha_p[a] * nu + alpha_n * nu_n) * T(0.5);
                diag += faceFlux + vc;
                off[f] = faceFlux - vc;
            }
        }
        if (MATRIX) {
            const T rdet = T(1) / det;
            C[i] = diag / det;
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) C[(size_t)(f + 1) * N + i] = off[f] / det;
            A[i] = diag / det;
            (void)rdet;
        }
        if (RHS) {
            T g[D];
            if (apply_pgrad) pressure_grad_fd<T, D>(dom, B, b, p, i, l, tr, g);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                T r = rhs[c] / det + cell_source<T>(B, l, c, nc);
                if (apply_pgrad) r -= g[c] * dt;
                vrhs[(size_t)c * N + i] = r;
            }
        }
        (void)K;
    });
}

// ---------------------------------------------------------------------------------------------
// pressure matrix + H/A right-hand side
// ---------------------------------------------------------------------------------------------

template <typename T, int D, bool MATRIX, bool RHS>
__global__ void __launch_bounds__(256, 6) k_pressure_setup(pict_domain_t dom, double dt_arg) {
    const int N = dom.num_cells;
    const T* C = reinterpret_cast<const T*>(dom.C);
    const T* A = reinterpret_cast<const T*>(dom.A);
    T* P = reinterpret_cast<T*>(dom.P);
    const T* vres = reinterpret_cast<const T*>(dom.velocity_result);
    T* prhs = reinterpret_cast<T*>(dom.pressure_rhs);
    for_each_cell(dom, [&](const int i, const int b) {
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T raP = T(1) / A[i];
        Nbr nb[2 * D];
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) nb[f] = neighbour(dom, B, b, p, i, f);
        if (MATRIX) {
            T diag = 0;
            T off[2 * D];
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                off[f] = 0;
                if (nb[f].j >= 0) {
                    const int a = f >> 1;
                    const pict_block_t& Bn = dom.blocks[nb[f].b];
                    const T alphaN = laplace_coef<T, D>(cell_transform<T, D>(Bn, nb[f].l), nb[f].comp);
                    const T raN = T(1) / A[nb[f].j];
                    const T cf = T(0.5) * (laplace_coef<T, D>(tr, a) * raP + alphaN * raN);
                    diag -= cf;
                    off[f] = cf;
                }
            }
            P[i] = diag;
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) P[(size_t)(f + 1) * N + i] = off[f];
        }
        if (RHS) {
            const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
            const T det = tr_det<T, D>(tr);
            const T nu = cell_viscosity<T>(dom, B, l);
            T u[D];
            load_block_vec<T, D>(B, B.velocity, l, u);
            T S[D], H[D];
#pragma unroll
            for (int c = 0; c < D; ++c) { S[c] = 0; H[c] = 0; }
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                if (nb[f].j >= 0) {
                    if (nb[f].j != i) {
                        const T cf = C[(size_t)(f + 1) * N + i];
#pragma unroll
                        for (int c = 0; c < D; ++c) H[c] += cf * vres[(size_t)c * N + nb[f].j];
                    }
                } else {
                    const T sign = (f & 1) ? T(1) : T(-1);
                    const FixedFace<T, D> ff = fixed_face<T, D>(B, p, f);
                    const T flux = ff.contra * sign;
#pragma unroll
                    for (int c = 0; c < D; ++c) S[c] += -ff.vel[c] * flux + ff.vel[c] * nu * T(2) * ff.alpha;
                }
            }
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const T s = S[c] / det + cell_source<T>(B, l, c, nc);
                prhs[(size_t)c * N + i] = raP * (u[c] / dt - H[c] + s);
            }
        }
    });
}

// ---------------------------------------------------------------------------------------------
// divergence of a cell-centred vector field from central face fluxes
// ---------------------------------------------------------------------------------------------

// SRC_GLOBAL: the field is a global [D][N] vector (pressureRHS); otherwise the blocks' velocity.
template <typename T, int D, bool SRC_GLOBAL>
__global__ void k_flux_divergence(pict_domain_t dom, const T* field, T* out, double dt_arg, int time_step_norm) {
    const int N = dom.num_cells;
    for_each_cell(dom, [&](const int i, const int b) {
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        T u[D];
        if (SRC_GLOBAL) load_global_vec<T, D>(field, N, i, u);
        else load_block_vec<T, D>(B, B.velocity, l, u);
        T div = 0;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const Nbr n = neighbour(dom, B, b, p, i, f);
            T flux;
            if (n.j < 0) {
                flux = fixed_face<T, D>(B, p, f).contra;
            } else {
                const pict_block_t& Bn = dom.blocks[n.b];
                T un[D];
                if (SRC_GLOBAL) load_global_vec<T, D>(field, N, n.j, un);
                else load_block_vec<T, D>(Bn, Bn.velocity, n.l, un);
                const T velN = contravariant<T, D>(cell_transform<T, D>(Bn, n.l), n.comp, un) * T(n.flip);
                const T velC = contravariant<T, D>(tr, a, u);
                flux = (velN + velC) * T(0.5);
            }
            div += (f & 1) ? flux : -flux;
        }
        if (time_step_norm) div /= sim_time_step<T>(dom, B.sim, dt_arg);
        out[i] = div;
    });
}

// ---------------------------------------------------------------------------------------------
// velocity correction u = h - grad(p)/A
// ---------------------------------------------------------------------------------------------

// Row r of Minv, component c, of a transform that may be absent (identity).
template <typename T, int D>
__device__ __forceinline__ T minv_or_id(const T* tr, int r, int c) {
    return tr ? tr_minv<T, D>(tr, r, c) : (r == c ? T(1) : T(0));
}

// Finite-volume pressure gradient (getPressureGradientFVM, extensions/PISO_multiblock_cuda_kernel.cu:991-1123): the sum
// over faces of the face pressure times the face area vector (row of det Minv), divided by the cell's
// det.  INTERP 0 averages the two cells' fluxes det Minv[axis] p (with the connected neighbour's aligned
// axis and the sign flip of a connection joining two lower or two upper faces); INTERP 3 takes the
// staggered face transform times the mean pressure.  A prescribed face extrapolates the pressure from
// the opposite neighbour, half a cell with the boundary transform (INTERP 0), a full cell (INTERP 3).
// Blocks without a transform take the finite-difference gradient.  A missing boundary, neighbour or
// face transform counts as the identity.
template <typename T, int D, int INTERP>
__device__ __forceinline__ void pressure_grad_fvm(const pict_domain_t& dom, const pict_block_t& B, int b,
                                                  const int* p, int i, int l, const T* tr, T* g) {
    if (!tr) {
        pressure_grad_fd<T, D>(dom, B, b, p, i, l, tr, g);
        return;
    }
    const T* pb = reinterpret_cast<const T*>(B.pressure);
    const T pP = pb[l];
    const T dP = tr_det<T, D>(tr);
    T acc[D];
#pragma unroll
    for (int c = 0; c < D; ++c) acc[c] = T(0);
#pragma unroll
    for (int f = 0; f < 2 * D; ++f) {
        const int a = f >> 1;
        const int up = f & 1;
        const T fs = up ? T(1) : T(-1);
        T pn;
        const T* trn = tr;
        int an = a;
        T tsgn = T(1);
        if (at_face(p, B.size, f) && B.face[f].type == PICT_FACE_FIXED) {
            int q[3] = {p[0], p[1], p[2]};
            if (B.size[a] > 1) q[a] += up ? -1 : 1;
            const T p_in = pb[q[0] + B.size[0] * (q[1] + B.size[1] * q[2])];
            if (INTERP != 3) {
                const pict_face_t& F = B.face[f];
                const T* bt = F.transform
                                  ? reinterpret_cast<const T*>(F.transform) + (size_t)boundary_flat(p, B.size, f) * TS<D>::value
                                  : nullptr;
                const T v = tr_det<T, D>(bt) * (pP + (pP - p_in) * T(0.5)) * fs;
#pragma unroll
                for (int c = 0; c < D; ++c) acc[c] += minv_or_id<T, D>(bt, a, c) * v;
                continue;
            }
            pn = pP + (pP - p_in);
        } else {
            const Nbr n = neighbour(dom, B, b, p, i, f);
            const pict_block_t& Bn = dom.blocks[n.b];
            pn = reinterpret_cast<const T*>(Bn.pressure)[n.l];
            trn = cell_transform<T, D>(Bn, n.l);
            an = n.comp;
            tsgn = T(n.flip);
        }
        if (INTERP == 0) {
            const T vp = dP * pP, vn = tr_det<T, D>(trn) * pn * tsgn;
#pragma unroll
            for (int c = 0; c < D; ++c)
                acc[c] += (tr_minv<T, D>(tr, a, c) * vp + minv_or_id<T, D>(trn, an, c) * vn) * (T(0.5) * fs);
        } else {
            int fp[3] = {p[0], p[1], p[2]};
            fp[a] += up;
            const int fx = B.size[0] + 1, fy = D > 1 ? B.size[1] + 1 : 1, fz = D > 2 ? B.size[2] + 1 : 1;
            const T* ft = B.face_transform
                              ? reinterpret_cast<const T*>(B.face_transform) +
                                    ((((size_t)a * fz + fp[2]) * fy + fp[1]) * fx + fp[0]) * TS<D>::value
                              : nullptr;
            const T v = tr_det<T, D>(ft) * (pn + pP) * T(0.5) * fs;
#pragma unroll
            for (int c = 0; c < D; ++c) acc[c] += minv_or_id<T, D>(ft, a, c) * v;
        }
    }
#pragma unroll
    for (int c = 0; c < D; ++c) g[c] = acc[c] / dP;
}

// MODE -1: finite-difference gradient (versions 0/1); 0 / 3: finite-volume gradient (versions 5 / 6)
template <typename T, int D, int MODE>
__global__ void k_correct_velocity(pict_domain_t dom, double dt_arg, int time_step_norm, int write_block) {
    const int N = dom.num_cells;
    const T* A = reinterpret_cast<const T*>(dom.A);
    const T* prhs = reinterpret_cast<const T*>(dom.pressure_rhs);
    T* vres = reinterpret_cast<T*>(dom.velocity_result);
    for_each_cell(dom, [&](const int i, const int b) {
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        T g[D];
        if (MODE < 0) pressure_grad_fd<T, D>(dom, B, b, p, i, l, tr, g);
        else pressure_grad_fvm<T, D, MODE>(dom, B, b, p, i, l, tr, g);
        const T rA = T(1) / A[i];
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
        T* ub = reinterpret_cast<T*>(B.velocity);
#pragma unroll
        for (int c = 0; c < D; ++c) {
            T du = -rA * g[c];
            if (time_step_norm) du *= dt;
            const T v = du + prhs[(size_t)c * N + i];
            vres[(size_t)c * N + i] = v;
            if (write_block) ub[(size_t)c * nc + l] = v;
        }
    });
}

// Version 4 (PISO_update_velocity_v4_orthogonal, extensions/PISO_multiblock_cuda_kernel.cu:6053-6160): per axis the mean of
// the two face fluxes (cc h + cc_N h_N - (cc t / A + cc_N t_N / A_N) dp dt) / 4 with orthogonal metrics
// t and cc = det t, transformed back by 1 / (det t); a prescribed face contributes nothing.  The cell's
// own t is Minv[0][0] for every axis (the reference reads it at the cell position, channel 0), the
// neighbour's is Minv[d][d] (its component aligned with the face across a connection).
template <typename T, int D>
__global__ void k_correct_velocity_v4(pict_domain_t dom, double dt_arg, int write_block) {
    const int N = dom.num_cells;
    const T* A = reinterpret_cast<const T*>(dom.A);
    const T* prhs = reinterpret_cast<const T*>(dom.pressure_rhs);
    T* vres = reinterpret_cast<T*>(dom.velocity_result);
    for_each_cell(dom, [&](const int i, const int b) {
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T det = tr_det<T, D>(tr);
        const T ra = T(1) / A[i];
        const T pc = reinterpret_cast<const T*>(B.pressure)[l];
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
        T* ub = reinterpret_cast<T*>(B.velocity);
        const T t = minv_or_id<T, D>(tr, 0, 0);
        const T cc = det * t;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const T hb = prhs[(size_t)d * N + i];
            T v = T(0);
#pragma unroll
            for (int up = 0; up < 2; ++up) {
                const int f = 2 * d + up;
                if (at_face(p, B.size, f) && B.face[f].type == PICT_FACE_FIXED) continue;
                const Nbr n = neighbour(dom, B, b, p, i, f);
                const pict_block_t& Bn = dom.blocks[n.b];
                const T* trn = cell_transform<T, D>(Bn, n.l);
                const T tN = minv_or_id<T, D>(trn, n.comp, n.comp);
                const T ccN = tr_det<T, D>(trn) * tN;
                const T pN = reinterpret_cast<const T*>(Bn.pressure)[n.l];
                const T dp = up ? (pN - pc) : (pc - pN);
                v += (cc * hb + ccN * prhs[(size_t)n.comp * N + n.j] - (cc * t * ra + ccN * tN / A[n.j]) * dp * dt) *
                     T(0.25);
            }
            v /= det * t;
            vres[(size_t)d * N + i] = v;
            if (write_block) ub[(size_t)d * nc + l] = v;
        }
    });
}

// ---------------------------------------------------------------------------------------------
// copies between global result vectors and block fields (extensions/PISO_multiblock_cuda_kernel.cu:6543-6733)
// ---------------------------------------------------------------------------------------------

template <typename T, bool TO_BLOCKS, bool VECTOR>
__global__ void k_copy_result(pict_domain_t dom, int D) {
    const int N = dom.num_cells;
    T* g = reinterpret_cast<T*>(VECTOR ? dom.velocity_result : dom.pressure_result);
    for_each_cell(dom, [&](const int i, const int b) {
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        T* bf = reinterpret_cast<T*>(VECTOR ? B.velocity : B.pressure);
        const int ncomp = VECTOR ? D : 1;
        for (int c = 0; c < ncomp; ++c) {
            if (TO_BLOCKS) bf[(size_t)c * nc + l] = g[(size_t)c * N + i];
            else g[(size_t)c * N + i] = bf[(size_t)c * nc + l];
        }
    });
}

// Initial guess of the advection solve from the previous step's increment: velocityResult = u + incr
// (SUB = false), or after the solve incr = velocityResult - u (SUB = true), u the blocks' velocity
template <typename T, bool SUB>
__global__ void k_advection_increment(pict_domain_t dom, int D, T* __restrict__ incr) {
    const int N = dom.num_cells;
    T* g = reinterpret_cast<T*>(dom.velocity_result);
    for_each_cell(dom, [&](const int i, const int b) {
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        const T* bf = reinterpret_cast<const T*>(B.velocity);
        for (int c = 0; c < D; ++c) {
            const T u = bf[(size_t)c * nc + l];
            const size_t k = (size_t)c * N + i;
            if (SUB) incr[k] = g[k] - u;
            else g[k] = u + incr[k];
        }
    });
}

// ---------------------------------------------------------------------------------------------
// transforms from vertex coordinates (extensions/grid_gen.cu:284-339 and 383-466)
// ---------------------------------------------------------------------------------------------

template <typename T, int D>
__device__ __forceinline__ void write_transform(T* out, const T (&M)[D][D]) {
    T det, inv[D][D];
    if (D == 1) {
        det = M[0][0];
        inv[0][0] = T(1) / det;
    } else if (D == 2) {
        det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        const T r = T(1) / det;
        inv[0][0] = M[1][1] * r; inv[0][1] = -M[0][1] * r;
        inv[1][0] = -M[1][0] * r; inv[1][1] = M[0][0] * r;
    } else {
        // cofactor expansion
        const T c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
        const T c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
        const T c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
        det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
        const T r = T(1) / det;
        inv[0][0] = c00 * r;
        inv[1][0] = c01 * r;
        inv[2][0] = c02 * r;
        inv[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * r;
        inv[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * r;
        inv[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) * r;
        inv[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * r;
        inv[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) * r;
        inv[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * r;
    }
    int k = 0;
#pragma unroll
    for (int r0 = 0; r0 < D; ++r0)
#pragma unroll
        for (int c0 = 0; c0 < D; ++c0) out[k++] = M[r0][c0];
#pragma unroll
    for (int r0 = 0; r0 < D; ++r0)
#pragma unroll
        for (int c0 = 0; c0 < D; ++c0) out[k++] = inv[r0][c0];
    out[k] = det;
}

// coords [D][(Z)][Y][X] vertex grid with vsize = cells+1 per axis
template <typename T, int D>
__global__ void k_coords_to_transforms(const T* coords, int3 vsize, T* out) {
    const int cx = vsize.x - 1, cy = D > 1 ? vsize.y - 1 : 1, cz = D > 2 ? vsize.z - 1 : 1;
    const int n = cx * cy * cz;
    const int vn = vsize.x * (D > 1 ? vsize.y : 1) * (D > 2 ? vsize.z : 1);
    PICT_CELL_LOOP(i, n) {
        const int x = i % cx, y = (i / cx) % cy, z = i / (cx * cy);
        T face[2 * D][D];
#pragma unroll
        for (int f = 0; f < 2 * D; ++f)
#pragma unroll
            for (int c = 0; c < D; ++c) face[f][c] = 0;
        for (int v = 0; v < (1 << D); ++v) {
            const int vx = x + (v & 1), vy = y + ((v >> 1) & 1), vz = z + ((v >> 2) & 1);
            const int vf = vx + vsize.x * (vy + (D > 1 ? vsize.y : 1) * vz);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const T co = coords[(size_t)c * vn + vf];
#pragma unroll
                for (int k = 0; k < D; ++k) face[2 * k + ((v >> k) & 1)][c] += co;
            }
        }
        const T norm = T(1) / T(1 << (D - 1));
        T M[D][D];
#pragma unroll
        for (int c = 0; c < D; ++c)
#pragma unroll
            for (int k = 0; k < D; ++k) M[c][k] = (face[2 * k + 1][c] - face[2 * k][c]) * norm;
        write_transform<T, D>(out + (size_t)i * TS<D>::value, M);
    }
}

// face transforms on the staggered vertex grid: out [D][(Z)][Y][X][T]
template <typename T, int D>
__global__ void k_coords_to_face_transforms(const T* coords, int3 vsize, T* out) {
    const int sz[3] = {vsize.x, D > 1 ? vsize.y : 1, D > 2 ? vsize.z : 1};
    const int vn = sz[0] * sz[1] * sz[2];
    constexpr int NFV = 1 << (D - 1);
    constexpr int NEV = D >= 2 ? (1 << (D - 2)) : 1;
    PICT_CELL_LOOP(i, vn) {
        int pos[3] = {i % sz[0], (i / sz[0]) % sz[1], i / (sz[0] * sz[1])};
        auto vidx = [&](const int* q) { return q[0] + sz[0] * (q[1] + sz[1] * q[2]); };
        for (int dim = 0; dim < D; ++dim) {
            bool skip = false;
            for (int k = 1; k < D; ++k) {
                const int t = (dim + k) % D;
                if (pos[t] == sz[t] - 1) skip = true;
            }
            if (skip) continue;
            T M[D][D];
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) M[r][c] = 0;
            T normw = T(0.5);
            for (int up = 0; up < 2; ++up) {
                const int sign = up * 2 - 1;
                const bool atb = up ? (pos[dim] == sz[dim] - 1) : (pos[dim] == 0);
                int fpos[3] = {pos[0], pos[1], pos[2]};
                if (!atb) fpos[dim] += sign;
                else normw = T(1);
                for (int vi = 0; vi < NFV; ++vi) {
                    int vp[3] = {fpos[0], fpos[1], fpos[2]};
                    for (int k = 1; k < D; ++k) vp[(dim + k) % D] += (vi & k) != 0;
                    const int vf = vidx(vp);
#pragma unroll
                    for (int c = 0; c < D; ++c) M[c][dim] += coords[(size_t)c * vn + vf] * T(sign);
                }
            }
            normw /= T(NFV);
#pragma unroll
            for (int c = 0; c < D; ++c) M[c][dim] *= normw;
            for (int k = 1; k < D; ++k) {
                const int tdim = (dim + k) % D;
                for (int vi = 0; vi < NFV; ++vi) {
                    int vp[3] = {pos[0], pos[1], pos[2]};
                    for (int kk = 1; kk < D; ++kk) vp[(dim + kk) % D] += (vi & kk) != 0;
                    const T ts = (vi & k) ? T(1) : T(-1);
                    const int vf = vidx(vp);
#pragma unroll
                    for (int c = 0; c < D; ++c) M[c][tdim] += coords[(size_t)c * vn + vf] * ts;
                }
#pragma unroll
                for (int c = 0; c < D; ++c) M[c][tdim] *= T(1) / T(NEV);
            }
            write_transform<T, D>(out + ((size_t)dim * vn + i) * TS<D>::value, M);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// CSR export / import
// ---------------------------------------------------------------------------------------------

template <int D>
__global__ void k_csr_row_counts(pict_domain_t dom, int32_t* counts) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        int c = 1;
        for (int f = 0; f < 2 * D; ++f) c += dom.nbr[(size_t)f * N + i] >= 0;
        counts[i] = c;
    }
}

// single-CTA exclusive scan of counts[N] into row[N+1] (row[0] = 0)
__global__ void k_scan_rows(const int32_t* counts, int32_t* row, int N) {
    __shared__ int32_t s_part[1024];
    const int t = threadIdx.x;
    const int nt = blockDim.x;
    const int chunk = (N + nt - 1) / nt;
    const int lo = t * chunk, hi = min(N, lo + chunk);
    int32_t sum = 0;
    for (int k = lo; k < hi; ++k) sum += counts[k];
    s_part[t] = sum;
    __syncthreads();
    if (t == 0) {
        int32_t acc = 0;
        for (int k = 0; k < nt; ++k) {
            const int32_t v = s_part[k];
            s_part[k] = acc;
            acc += v;
        }
    }
    __syncthreads();
    int32_t acc = s_part[t];
    if (t == 0) row[0] = 0;
    for (int k = lo; k < hi; ++k) {
        acc += counts[k];
        row[k + 1] = acc;
    }
}

template <typename T, int D>
__global__ void k_stencil_to_csr(pict_domain_t dom, const T* coef, const int32_t* row, T* val, int32_t* idx) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        int cols[2 * D + 1];
        T vals[2 * D + 1];
        int n = 0;
        cols[n] = i; vals[n] = coef[i]; ++n;
        for (int f = 0; f < 2 * D; ++f) {
            const int j = dom.nbr[(size_t)f * N + i];
            if (j >= 0) { cols[n] = j; vals[n] = coef[(size_t)(f + 1) * N + i]; ++n; }
        }
        // insertion sort by column (stable), extensions/PISO_multiblock_cuda_kernel.cu:3846-3860 sorts rows by column index
        for (int a = 1; a < n; ++a) {
            const int c = cols[a];
            const T v = vals[a];
            int k = a - 1;
            while (k >= 0 && cols[k] > c) { cols[k + 1] = cols[k]; vals[k + 1] = vals[k]; --k; }
            cols[k + 1] = c; vals[k + 1] = v;
        }
        const int r0 = row[i];
        for (int k = 0; k < n; ++k) { idx[r0 + k] = cols[k]; val[r0 + k] = vals[k]; }
    }
}

template <typename T, int D>
__global__ void k_csr_to_stencil(pict_domain_t dom, const T* val, const int32_t* row, const int32_t* idx, T* coef) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        for (int f = 0; f <= 2 * D; ++f) coef[(size_t)f * N + i] = T(0);
        bool used[2 * D];
        for (int f = 0; f < 2 * D; ++f) used[f] = false;
        bool diag_used = false;
        for (int e = row[i]; e < row[i + 1]; ++e) {
            const int j = idx[e];
            if (j == i && !diag_used) { coef[i] += val[e]; diag_used = true; continue; }
            for (int f = 0; f < 2 * D; ++f) {
                if (!used[f] && dom.nbr[(size_t)f * N + i] == j) {
                    coef[(size_t)(f + 1) * N + i] = val[e];
                    used[f] = true;
                    break;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------------------------

template <typename T, int D>
static pict_status_t launch_adv(const pict_domain_t* dom, double dt, bool matrix, bool rhs, int pgrad, cudaStream_t st) {
    const int grid = domain_grid(dom, 256);
    if (matrix && rhs) k_adv_setup<T, D, true, true><<<grid, 256, 0, st>>>(*dom, dt, pgrad);
    else if (matrix) k_adv_setup<T, D, true, false><<<grid, 256, 0, st>>>(*dom, dt, pgrad);
    else k_adv_setup<T, D, false, true><<<grid, 256, 0, st>>>(*dom, dt, pgrad);
    return check_launch("adv_setup");
}

template <typename T, int D>
static pict_status_t launch_pressure(const pict_domain_t* dom, double dt, bool matrix, bool rhs, bool div,
                                     int tsn, cudaStream_t st) {
    const int grid = domain_grid(dom, 256);
    if (matrix && rhs) k_pressure_setup<T, D, true, true><<<grid, 256, 0, st>>>(*dom, dt);
    else if (matrix) k_pressure_setup<T, D, true, false><<<grid, 256, 0, st>>>(*dom, dt);
    else if (rhs) k_pressure_setup<T, D, false, true><<<grid, 256, 0, st>>>(*dom, dt);
    pict_status_t s = check_launch("pressure_setup");
    if (s != PICT_OK) return s;
    if (div) {
        k_flux_divergence<T, D, true><<<grid, 256, 0, st>>>(
            *dom, reinterpret_cast<const T*>(dom->pressure_rhs), reinterpret_cast<T*>(dom->pressure_rhs_div), dt, tsn);
        s = check_launch("pressure_rhs_div");
    }
    return s;
}

}  // namespace pict

using namespace pict;

#define PICT_DISPATCH(dom, FN, ...)                                                   \
    do {                                                                              \
        if ((dom)->dtype == PICT_F32) {                                               \
            if ((dom)->dims == 2) return FN<float, 2>(__VA_ARGS__);                   \
            if ((dom)->dims == 3) return FN<float, 3>(__VA_ARGS__);                   \
        } else if ((dom)->dtype == PICT_F64) {                                        \
            if ((dom)->dims == 2) return FN<double, 2>(__VA_ARGS__);                  \
            if ((dom)->dims == 3) return FN<double, 3>(__VA_ARGS__);                  \
        }                                                                             \
        return set_error(PICT_ERR_UNSUPPORTED, "unsupported dtype/dims");             \
    } while (0)

static pict_status_t check_dom(const pict_domain_t* dom) {
    if (!dom) return set_error(PICT_ERR_ARG, "domain is NULL");
    if (dom->dims < 2 || dom->dims > 3) return set_error(PICT_ERR_UNSUPPORTED, "only 2D and 3D domains are supported");
    if (dom->num_cells <= 0 || !dom->blocks || !dom->nbr || !dom->cell_block)
        return set_error(PICT_ERR_ARG, "domain is not prepared (missing block table or topology)");
    return PICT_OK;
}

extern "C" {

static pict_status_t adv_matrix(const pict_domain_t* dom, double dt, void* stream) {
    PICT_DISPATCH(dom, launch_adv, dom, dt, true, false, 0, (cudaStream_t)stream);
}

static pict_status_t adv_velocity(const pict_domain_t* dom, double dt, int32_t pgrad, void* stream) {
    PICT_DISPATCH(dom, launch_adv, dom, dt, false, true, pgrad, (cudaStream_t)stream);
}

static pict_status_t pressure_ops(const pict_domain_t* dom, double dt, bool matrix, bool rhs, bool div, int32_t tsn,
                                  void* stream) {
    PICT_DISPATCH(dom, launch_pressure, dom, dt, matrix, rhs, div, tsn, (cudaStream_t)stream);
}

pict_status_t pict_setup_advection_matrix(const pict_domain_t* dom, double dt, int32_t non_ortho_flags, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    s = adv_matrix(dom, dt, stream);
    if (s || !non_ortho_flags) return s;
    return nonortho_pass(dom, non_ortho_flags, 0, stream);
}

pict_status_t pict_setup_advection_velocity(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                            int32_t apply_pressure_gradient, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    s = adv_velocity(dom, dt, apply_pressure_gradient, stream);
    if (s || !non_ortho_flags) return s;
    return nonortho_pass(dom, non_ortho_flags, 1, stream);
}

pict_status_t pict_setup_advection(const pict_domain_t* dom, double dt, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    PICT_DISPATCH(dom, launch_adv, dom, dt, true, true, 0, (cudaStream_t)stream);
}

pict_status_t pict_setup_pressure_matrix(const pict_domain_t* dom, int32_t non_ortho_flags, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    s = pressure_ops(dom, 1.0, true, false, false, 0, stream);
    if (s || !non_ortho_flags) return s;
    return nonortho_pass(dom, non_ortho_flags, 2, stream);
}

pict_status_t pict_setup_pressure_rhs(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                      int32_t time_step_norm, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    s = pressure_ops(dom, dt, false, true, true, time_step_norm, stream);
    if (s || !non_ortho_flags) return s;
    return nonortho_pass(dom, non_ortho_flags, 3, stream);
}

pict_status_t pict_setup_pressure_rhs_div(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                          int32_t time_step_norm, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    s = pressure_ops(dom, dt, false, false, true, time_step_norm, stream);
    if (s || !non_ortho_flags) return s;
    return nonortho_pass(dom, non_ortho_flags, 3, stream);
}

pict_status_t pict_setup_pressure_correction(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                             int32_t time_step_norm, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    s = pressure_ops(dom, dt, true, true, true, time_step_norm, stream);
    if (s || !non_ortho_flags) return s;
    s = nonortho_pass(dom, non_ortho_flags, 2, stream);
    if (s) return s;
    return nonortho_pass(dom, non_ortho_flags, 3, stream);
}

}  // extern "C"

template <typename T, int D>
static pict_status_t launch_correct(const pict_domain_t* dom, double dt, int version, int tsn, int wb, cudaStream_t st) {
    const int grid = domain_grid(dom, 256);
    switch (version) {
        case 4: k_correct_velocity_v4<T, D><<<grid, 256, 0, st>>>(*dom, dt, wb); break;
        case 5: k_correct_velocity<T, D, 0><<<grid, 256, 0, st>>>(*dom, dt, tsn, wb); break;
        case 6: k_correct_velocity<T, D, 3><<<grid, 256, 0, st>>>(*dom, dt, tsn, wb); break;
        default: k_correct_velocity<T, D, -1><<<grid, 256, 0, st>>>(*dom, dt, tsn, wb); break;
    }
    return check_launch("correct_velocity");
}

template <typename T, int D>
static pict_status_t launch_increment(const pict_domain_t* dom, int sub, void* incr, cudaStream_t st) {
    const int grid = domain_grid(dom, 256);
    if (sub) k_advection_increment<T, true><<<grid, 256, 0, st>>>(*dom, D, reinterpret_cast<T*>(incr));
    else k_advection_increment<T, false><<<grid, 256, 0, st>>>(*dom, D, reinterpret_cast<T*>(incr));
    return check_launch("advection increment");
}

template <typename T, int D>
static pict_status_t launch_copy(const pict_domain_t* dom, int which, cudaStream_t st) {
    const int grid = domain_grid(dom, 256);
    switch (which) {
        case 0: k_copy_result<T, true, true><<<grid, 256, 0, st>>>(*dom, D); break;
        case 1: k_copy_result<T, false, true><<<grid, 256, 0, st>>>(*dom, D); break;
        case 2: k_copy_result<T, true, false><<<grid, 256, 0, st>>>(*dom, D); break;
        default: k_copy_result<T, false, false><<<grid, 256, 0, st>>>(*dom, D); break;
    }
    return check_launch("copy_result");
}

template <typename T, int D>
static pict_status_t launch_vel_div(const pict_domain_t* dom, void* out, cudaStream_t st) {
    k_flux_divergence<T, D, false><<<domain_grid(dom, 256), 256, 0, st>>>(*dom, nullptr,
                                                                                  reinterpret_cast<T*>(out), 1.0, 0);
    return check_launch("velocity_divergence");
}

template <typename T, int D>
static pict_status_t launch_csr_counts(const pict_domain_t* dom, int32_t* row, cudaStream_t st) {
    // counts are written into row[1..N] first, then scanned in place through a temporary view
    k_csr_row_counts<D><<<cell_grid(dom->num_cells, 256), 256, 0, st>>>(*dom, row + 1);
    pict_status_t s = check_launch("csr_row_counts");
    if (s) return s;
    k_scan_rows<<<1, 1024, 0, st>>>(row + 1, row, dom->num_cells);
    return check_launch("csr_scan");
}

template <typename T, int D>
static pict_status_t launch_s2c(const pict_domain_t* dom, const void* coef, const int32_t* row, void* val,
                                int32_t* idx, cudaStream_t st) {
    k_stencil_to_csr<T, D><<<cell_grid(dom->num_cells, 256), 256, 0, st>>>(
        *dom, reinterpret_cast<const T*>(coef), row, reinterpret_cast<T*>(val), idx);
    return check_launch("stencil_to_csr");
}

template <typename T, int D>
static pict_status_t launch_c2s(const pict_domain_t* dom, const void* val, const int32_t* row, const int32_t* idx,
                                void* coef, cudaStream_t st) {
    k_csr_to_stencil<T, D><<<cell_grid(dom->num_cells, 256), 256, 0, st>>>(
        *dom, reinterpret_cast<const T*>(val), row, idx, reinterpret_cast<T*>(coef));
    return check_launch("csr_to_stencil");
}

extern "C" {

pict_status_t pict_correct_velocity(const pict_domain_t* dom, double dt, int32_t version, int32_t time_step_norm,
                                    int32_t write_block_velocity, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    if (!(version == 0 || version == 1 || version == 4 || version == 5 || version == 6))
        return set_error(PICT_ERR_UNSUPPORTED, "velocity corrector versions 0/1 (FD), 4, 5 and 6 (FVM) are supported");
    PICT_DISPATCH(dom, launch_correct, dom, dt, version, time_step_norm, write_block_velocity, (cudaStream_t)stream);
}

pict_status_t pict_copy_velocity_result_to_blocks(const pict_domain_t* dom, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    PICT_DISPATCH(dom, launch_copy, dom, 0, (cudaStream_t)stream);
}
pict_status_t pict_advection_guess(const pict_domain_t* dom, void* increment, int32_t after_solve, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    if (!increment) return set_error(PICT_ERR_ARG, "advection_guess: NULL increment");
    PICT_DISPATCH(dom, launch_increment, dom, after_solve ? 1 : 0, increment, (cudaStream_t)stream);
}
pict_status_t pict_copy_velocity_result_from_blocks(const pict_domain_t* dom, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    PICT_DISPATCH(dom, launch_copy, dom, 1, (cudaStream_t)stream);
}
pict_status_t pict_copy_pressure_result_to_blocks(const pict_domain_t* dom, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    PICT_DISPATCH(dom, launch_copy, dom, 2, (cudaStream_t)stream);
}
pict_status_t pict_copy_pressure_result_from_blocks(const pict_domain_t* dom, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    PICT_DISPATCH(dom, launch_copy, dom, 3, (cudaStream_t)stream);
}

pict_status_t pict_velocity_divergence(const pict_domain_t* dom, void* out, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    if (!out) return set_error(PICT_ERR_ARG, "out is NULL");
    PICT_DISPATCH(dom, launch_vel_div, dom, out, (cudaStream_t)stream);
}

pict_status_t pict_csr_row_ptr(const pict_domain_t* dom, int32_t* row_out, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    if (!row_out) return set_error(PICT_ERR_ARG, "row_out is NULL");
    PICT_DISPATCH(dom, launch_csr_counts, dom, row_out, (cudaStream_t)stream);
}

pict_status_t pict_stencil_to_csr(const pict_domain_t* dom, const void* coef, const int32_t* row, void* value_out,
                                  int32_t* index_out, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    if (!coef || !row || !value_out || !index_out) return set_error(PICT_ERR_ARG, "NULL argument");
    PICT_DISPATCH(dom, launch_s2c, dom, coef, row, value_out, index_out, (cudaStream_t)stream);
}

pict_status_t pict_csr_to_stencil(const pict_domain_t* dom, const void* value, const int32_t* row, const int32_t* index,
                                  void* coef_out, void* stream) {
    pict_status_t s = check_dom(dom);
    if (s) return s;
    if (!value || !row || !index || !coef_out) return set_error(PICT_ERR_ARG, "NULL argument");
    PICT_DISPATCH(dom, launch_c2s, dom, value, row, index, coef_out, (cudaStream_t)stream);
}

pict_status_t pict_coords_to_transforms(const void* coords, int32_t dims, const int32_t* size_xyz, int32_t dtype,
                                        void* out, void* stream) {
    if (!coords || !out || !size_xyz) return set_error(PICT_ERR_ARG, "NULL argument");
    const int3 vs = make_int3(size_xyz[0] + 1, dims > 1 ? size_xyz[1] + 1 : 1, dims > 2 ? size_xyz[2] + 1 : 1);
    const int n = size_xyz[0] * (dims > 1 ? size_xyz[1] : 1) * (dims > 2 ? size_xyz[2] : 1);
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(n, 128);
    if (dtype == PICT_F32 && dims == 2) k_coords_to_transforms<float, 2><<<grid, 128, 0, st>>>((const float*)coords, vs, (float*)out);
    else if (dtype == PICT_F32 && dims == 3) k_coords_to_transforms<float, 3><<<grid, 128, 0, st>>>((const float*)coords, vs, (float*)out);
    else if (dtype == PICT_F64 && dims == 2) k_coords_to_transforms<double, 2><<<grid, 128, 0, st>>>((const double*)coords, vs, (double*)out);
    else if (dtype == PICT_F64 && dims == 3) k_coords_to_transforms<double, 3><<<grid, 128, 0, st>>>((const double*)coords, vs, (double*)out);
    else return set_error(PICT_ERR_UNSUPPORTED, "unsupported dtype/dims");
    return check_launch("coords_to_transforms");
}

pict_status_t pict_coords_to_face_transforms(const void* coords, int32_t dims, const int32_t* size_xyz, int32_t dtype,
                                             void* out, void* stream) {
    if (!coords || !out || !size_xyz) return set_error(PICT_ERR_ARG, "NULL argument");
    const int3 vs = make_int3(size_xyz[0] + 1, dims > 1 ? size_xyz[1] + 1 : 1, dims > 2 ? size_xyz[2] + 1 : 1);
    const int n = vs.x * vs.y * vs.z;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(n, 128);
    if (dtype == PICT_F32 && dims == 2) k_coords_to_face_transforms<float, 2><<<grid, 128, 0, st>>>((const float*)coords, vs, (float*)out);
    else if (dtype == PICT_F32 && dims == 3) k_coords_to_face_transforms<float, 3><<<grid, 128, 0, st>>>((const float*)coords, vs, (float*)out);
    else if (dtype == PICT_F64 && dims == 2) k_coords_to_face_transforms<double, 2><<<grid, 128, 0, st>>>((const double*)coords, vs, (double*)out);
    else if (dtype == PICT_F64 && dims == 3) k_coords_to_face_transforms<double, 3><<<grid, 128, 0, st>>>((const double*)coords, vs, (double*)out);
    else return set_error(PICT_ERR_UNSUPPORTED, "unsupported dtype/dims");
    return check_launch("coords_to_face_transforms");
}

}  // extern "C"
