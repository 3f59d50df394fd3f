// adjoint.cu -- reverse-mode kernels of the orthogonal PISO step.
//
// The reference differentiates the step operator by operator (PISOtorch_diff.py: SetupAdvectionMatrix
// :377-441, SetupAdvectionVelocity :531-613, SetupPressureCorrection :802-895, CorrectVelocity
// :1160-1236, linear_solve_GPU :295-375) with *_GRAD kernels scattering into the inputs with atomics
// (extensions/PISO_multiblock_cuda_kernel.cu:3869-4077, 4388-4478, 4967-5117, 5243-5371, 5423-5453,
// 6224-6293).  Here every adjoint is written in gather form: each thread owns one cell and collects
// the contributions of the stencil rows that reference it (through the same neighbour table and
// back-face relation as the forward), so there are no atomics and results are bitwise reproducible.
//
// Forward (per cell i, face f with axis a = f>>1, sign s_f = +-1, neighbour j, aligned neighbour
// axis a' and flip phi; cc_i(a, k) = d contra(tr_i, a, u) / d u[k] = det_i Minv_i[a][k]):
//   advection  C_f,i = (s_f/4 (phi contra_j(a', u_j) + contra_i(a, u_i)) - (al_i[a] nu_i + al_j[a'] nu_j)/2) / det_i
//              A_i = C_0,i = (det_i/dt + sum_f (faceFlux_f + visc_f) + sum_fixed 2 nu_i al_i[a]) / det_i
//              rhs_i = u_i/dt + sum_fixed (-vb s_f contra_b + vb nu_i 2 al_b)/det_i + src_i
//   H/A        h_i = (u_i/dt - sum_f C_f,i U_j + S_i/det_i + src_i) / A_i
//   divergence div_i = sum_f s_f flux_f,  flux = (phi contra_j(a', h_j) + contra_i(a, h_i))/2 or contra_b(vb)
//   pressure   P_f,i = (al_i[a]/A_i + al_j[a']/A_j)/2,  P_0,i = -sum_f P_f,i;  P p = div; p -= mean(p)
//   correction u_i = h_i - G_i(p)/A_i  (FD gradient, one-sided at fixed faces, times Minv)
//
// Accumulators are global vectors: un_bar [D][N] (velocity at the start of the step), nu_bar [N]
// (per-cell viscosity), src_bar [D][N], vb_bar [2D][D][N] (boundary velocity, per adjacent cell);
// pict_adjoint_to_blocks() maps them onto the blocks' and boundaries' gradient tensors.
#include <cstdio>
#include "common.cuh"
#include "launch.h"

namespace pict {

// d contra(tr, a, v) / d v[k]
template <typename T, int D>
__device__ __forceinline__ T cc(const T* tr, int a, int k) {
    if (!tr) return a == k ? T(1) : T(0);
    return tr_det<T, D>(tr) * tr_minv<T, D>(tr, a, k);
}

// Minv[d][c] (identity without transform): FD gradient g[c] = sum_d gl[d] Minv[d][c]
template <typename T, int D>
__device__ __forceinline__ T minv_or_id(const T* tr, int d, int c) {
    if (!tr) return d == c ? T(1) : T(0);
    return tr_minv<T, D>(tr, d, c);
}

__device__ __forceinline__ int face_sign(int f) { return (f & 1) ? 1 : -1; }

template <typename T, int D>
__device__ __forceinline__ const T* boundary_transform(const pict_block_t& B, const int* p, int f) {
    const pict_face_t& F = B.face[f];
    if (!F.transform) return nullptr;
    return reinterpret_cast<const T*>(F.transform) + (size_t)boundary_flat(p, B.size, f) * TS<D>::value;
}

// FD pressure-gradient factor along axis d of cell i: 1 if one side is a fixed face, else 1/2.
__device__ __forceinline__ float fd_factor(const pict_domain_t& dom, int i, int d) {
    const int N = dom.num_cells;
    return (dom.nbr[(size_t)(2 * d) * N + i] < 0 || dom.nbr[(size_t)(2 * d + 1) * N + i] < 0) ? 1.f : 0.5f;
}

// ---------------------------------------------------------------------------------------------
// velocity correction u = h - G(p)/A:  h_bar = u_bar, A_bar += u_bar.g/A^2, p_bar = -G^T (u_bar/A)
// ---------------------------------------------------------------------------------------------
template <typename T, int D>
__global__ void k_correct_velocity_grad(pict_domain_t dom, const T* A, const T* pv, const T* ubar, T* Abar,
                                        T* pbar, T* hbar) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T rA = T(1) / A[i];
        T ub[D];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            ub[c] = ubar[(size_t)c * N + i];
            hbar[(size_t)c * N + i] = ub[c];
        }
        // forward gradient g (for A_bar) and own one-sided contributions to p_bar
        T gl[D];
        T pb = 0;
        const T pc = pv[i];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const Nbr nl = neighbour(dom, B, b, p, i, 2 * d);
            const Nbr nh = neighbour(dom, B, b, p, i, 2 * d + 1);
            const T fac = (nl.j < 0 || nh.j < 0) ? T(1) : T(0.5);
            const T vN = nl.j < 0 ? pc : pv[nl.j];
            const T vP = nh.j < 0 ? pc : pv[nh.j];
            gl[d] = (vP - vN) * fac;
            T glb = 0;  // d L / d gl[d]
#pragma unroll
            for (int c = 0; c < D; ++c) glb += -ub[c] * rA * minv_or_id<T, D>(tr, d, c);
            if (nh.j < 0) pb += fac * glb;
            if (nl.j < 0) pb -= fac * glb;
        }
        T ag = 0;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            T g = 0;
#pragma unroll
            for (int d = 0; d < D; ++d) g += gl[d] * minv_or_id<T, D>(tr, d, c);
            ag += ub[c] * g;
        }
        Abar[i] += ag * rA * rA;
        // neighbours whose FD gradient reads p_i
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const Nbr n = neighbour(dom, B, b, p, i, f);
            if (n.j < 0) continue;
            const int fb = n.back;  // face of j pointing to i
            const int dj = fb >> 1;
            const pict_block_t& Bj = dom.blocks[n.b];
            const T* trj = cell_transform<T, D>(Bj, n.l);
            const T rAj = T(1) / A[n.j];
            T glb = 0;
#pragma unroll
            for (int c = 0; c < D; ++c) glb += -ubar[(size_t)c * N + n.j] * rAj * minv_or_id<T, D>(trj, dj, c);
            const T fac = (T)fd_factor(dom, n.j, dj);
            pb += (fb & 1) ? fac * glb : -fac * glb;
        }
        pbar[i] = pb;
    }
}

// ---------------------------------------------------------------------------------------------
// per-system mean removal x -= mean(x) (deterministic: one CTA per system, fixed reduction order)
// ---------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_sim_mean_project(pict_domain_t dom, T* x) {
    __shared__ double s_red[32];
    __shared__ double s_mean;
    const int s = blockIdx.x;
    const int c0 = dom.sim_cells[s], c1 = dom.sim_cells[s + 1];
    double acc = 0.0;
    for (int i = c0 + threadIdx.x; i < c1; i += blockDim.x) acc += (double)x[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) s_mean = v / (double)(c1 - c0);
    }
    __syncthreads();
    const T m = (T)s_mean;
    for (int i = c0 + threadIdx.x; i < c1; i += blockDim.x) x[i] -= m;
}

// ---------------------------------------------------------------------------------------------
// flux divergence: h_bar += Dv^T lambda, vb_bar += d div / d vb
// ---------------------------------------------------------------------------------------------
template <typename T, int D>
__global__ void k_divergence_grad(pict_domain_t dom, const T* lam, T* hbar, T* vbbar) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T li = lam[i];
        T hb[D];
#pragma unroll
        for (int c = 0; c < D; ++c) hb[c] = 0;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const T sf = (T)face_sign(f);
            const Nbr n = neighbour(dom, B, b, p, i, f);
            if (n.j < 0) {
                const T* trb = boundary_transform<T, D>(B, p, f);
#pragma unroll
                for (int c = 0; c < D; ++c) vbbar[((size_t)f * D + c) * N + i] += sf * li * cc<T, D>(trb, a, c);
                continue;
            }
            // own contravariant component in this cell's flux
#pragma unroll
            for (int k = 0; k < D; ++k) hb[k] += sf * li * T(0.5) * cc<T, D>(tr, a, k);
            // this cell's component in the neighbour's flux through its face n.back
            const T sb = (T)face_sign(n.back);
            const T lj = lam[n.j];
#pragma unroll
            for (int k = 0; k < D; ++k) hb[k] += sb * lj * T(0.5) * T(n.flip) * cc<T, D>(tr, a, k);
        }
#pragma unroll
        for (int c = 0; c < D; ++c) hbar[(size_t)c * N + i] += hb[c];
    }
}

// ---------------------------------------------------------------------------------------------
// H/A right-hand side and pressure matrix of one corrector
//   in:  h_bar, h, A, C, U (velocity used in H), lambda (P^-T p_bar), x (pressure solution)
//   out: A_bar +=, C_bar (off-diagonal) +=, U_bar =, un_bar +=, src_bar +=, nu_bar +=, vb_bar +=
// ---------------------------------------------------------------------------------------------
template <typename T, int D>
__global__ void k_pressure_rhs_grad(pict_domain_t dom, double dt_arg, const T* hbar, const T* h, const T* A,
                                    const T* C, const T* U, const T* lam, const T* xv, T* Abar, T* Cbar, T* Ubar,
                                    T* unbar, T* srcbar, T* nubar, T* vbbar) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T det = tr_det<T, D>(tr);
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
        const T nu = cell_viscosity<T>(dom, B, l);
        const T rA = T(1) / A[i];
        T rb[D];
        T ab = 0;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const T hb = hbar[(size_t)c * N + i];
            rb[c] = hb * rA;
            ab -= hb * h[(size_t)c * N + i] * rA;
            unbar[(size_t)c * N + i] += rb[c] / dt;
            if (srcbar) srcbar[(size_t)c * N + i] += rb[c];
        }
        T ub[D];
#pragma unroll
        for (int c = 0; c < D; ++c) ub[c] = 0;
        T nb_ = 0;
        T pm = 0;  // pressure-matrix term
        const T li = lam[i], xi = xv[i];
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const Nbr n = neighbour(dom, B, b, p, i, f);
            if (n.j < 0) {
                const T sf = (T)face_sign(f);
                const FixedFace<T, D> ff = fixed_face<T, D>(B, p, f);
                const T* trb = boundary_transform<T, D>(B, p, f);
                const T flux = ff.contra * sf;
                T q = 0;  // sum_c r_bar[c] vb[c]
#pragma unroll
                for (int c = 0; c < D; ++c) q += rb[c] * ff.vel[c];
#pragma unroll
                for (int c = 0; c < D; ++c)
                    vbbar[((size_t)f * D + c) * N + i] += (rb[c] * (-flux + nu * T(2) * ff.alpha) - q * sf * cc<T, D>(trb, a, c)) / det;
                nb_ += q * T(2) * ff.alpha / det;
                continue;
            }
            pm += laplace_coef<T, D>(tr, a) * (xv[n.j] - xi) * (lam[n.j] - li);
            if (n.j == i) continue;
            // C_bar of this row's off-diagonal entry
            T cb = 0;
#pragma unroll
            for (int c = 0; c < D; ++c) cb -= rb[c] * U[(size_t)c * N + n.j];
            Cbar[(size_t)(f + 1) * N + i] += cb;
            // rows of neighbours that use U_i: U_bar_i -= C_back,j r_bar_j
            const T cj = C[(size_t)(n.back + 1) * N + n.j];
            const T rAj = T(1) / A[n.j];
#pragma unroll
            for (int c = 0; c < D; ++c) ub[c] -= cj * hbar[(size_t)c * N + n.j] * rAj;
        }
        ab -= T(0.5) * rA * rA * pm;
        Abar[i] += ab;
        if (nubar) nubar[i] += nb_;
#pragma unroll
        for (int c = 0; c < D; ++c) Ubar[(size_t)c * N + i] = ub[c];
    }
}

// ---------------------------------------------------------------------------------------------
// advection matrix + RHS, including the outer product of the advection solve C u* = rhs:
//   D_bar_i = A_bar_i + C_bar_0,i - rhs_bar_i.u*_i,  O_bar_f,i = C_bar_f,i - rhs_bar_i.u*_j
//   out: un_bar +=, nu_bar +=, vb_bar +=, src_bar +=
// ---------------------------------------------------------------------------------------------
template <typename T, int D>
__device__ __forceinline__ T diag_bar(const T* Abar, const T* Cbar, const T* rhsbar, const T* us, int N, int i) {
    T d = Abar[i] + Cbar[i];
#pragma unroll
    for (int c = 0; c < D; ++c) d -= rhsbar[(size_t)c * N + i] * us[(size_t)c * N + i];
    return d;
}

template <typename T, int D>
__global__ void k_advection_grad(pict_domain_t dom, double dt_arg, const T* us, const T* rhsbar, const T* Cbar,
                                 const T* Abar, T* unbar, T* nubar, T* vbbar, T* srcbar) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T det = tr_det<T, D>(tr);
        const T rdet = T(1) / det;
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
        const T nu = cell_viscosity<T>(dom, B, l);
        const T Dbi = diag_bar<T, D>(Abar, Cbar, rhsbar, us, N, i);
        T q[D], usi[D];
        T ub[D];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            q[c] = rhsbar[(size_t)c * N + i] * rdet;
            usi[c] = us[(size_t)c * N + i];
            ub[c] = rhsbar[(size_t)c * N + i] / dt;
            if (srcbar) srcbar[(size_t)c * N + i] += rhsbar[(size_t)c * N + i];
        }
        T nb_ = 0;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const T sf = (T)face_sign(f);
            const T al = laplace_coef<T, D>(tr, a);
            const Nbr n = neighbour(dom, B, b, p, i, f);
            if (n.j < 0) {
                nb_ += Dbi * rdet * T(2) * al;
                const FixedFace<T, D> ff = fixed_face<T, D>(B, p, f);
                const T* trb = boundary_transform<T, D>(B, p, f);
                const T flux = ff.contra * sf;
                T qv = 0;
#pragma unroll
                for (int c = 0; c < D; ++c) qv += q[c] * ff.vel[c];
#pragma unroll
                for (int c = 0; c < D; ++c)
                    vbbar[((size_t)f * D + c) * N + i] += q[c] * (-flux + nu * T(2) * ff.alpha) - qv * sf * cc<T, D>(trb, a, c);
                nb_ += qv * T(2) * ff.alpha;
                continue;
            }
            // own row, face f
            T Ob = Cbar[(size_t)(f + 1) * N + i];
#pragma unroll
            for (int c = 0; c < D; ++c) Ob -= rhsbar[(size_t)c * N + i] * us[(size_t)c * N + n.j];
            const T Fb = (Dbi + Ob) * rdet, Vb = (Dbi - Ob) * rdet;
#pragma unroll
            for (int k = 0; k < D; ++k) ub[k] += sf * T(0.25) * Fb * cc<T, D>(tr, a, k);
            nb_ += Vb * al * T(0.5);
            // neighbour's row, its face n.back pointing here
            const int fb = n.back;
            const T sb = (T)face_sign(fb);
            const pict_block_t& Bj = dom.blocks[n.b];
            const T detj = tr_det<T, D>(cell_transform<T, D>(Bj, n.l));
            const T Dbj = diag_bar<T, D>(Abar, Cbar, rhsbar, us, N, n.j);
            T Obj = Cbar[(size_t)(fb + 1) * N + n.j];
#pragma unroll
            for (int c = 0; c < D; ++c) Obj -= rhsbar[(size_t)c * N + n.j] * usi[c];
            const T Fbj = (Dbj + Obj) / detj, Vbj = (Dbj - Obj) / detj;
#pragma unroll
            for (int k = 0; k < D; ++k) ub[k] += T(n.flip) * sb * T(0.25) * Fbj * cc<T, D>(tr, a, k);
            nb_ += Vbj * al * T(0.5);
        }
#pragma unroll
        for (int c = 0; c < D; ++c) unbar[(size_t)c * N + i] += ub[c];
        if (nubar) nubar[i] += nb_;
    }
}

// ---------------------------------------------------------------------------------------------
// accumulators -> gradient tensors of blocks and boundaries (one CTA per block, fixed order)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double block_reduce_sum(double v, double* s_red) {
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
    return r;  // valid in thread 0
}

template <typename T, int D>
__global__ void k_adjoint_to_blocks(pict_domain_t dom, const T* unbar, const T* nubar, const T* srcbar,
                                    const T* vbbar, double* block_nu) {
    __shared__ double s_red[32];
    const int N = dom.num_cells;
    const int bi = blockIdx.x;
    const pict_block_t& B = dom.blocks[bi];
    const int nc = B.size[0] * B.size[1] * B.size[2];
    const int off = B.offset;
    // velocity
    if (B.velocity_grad && unbar) {
        T* g = reinterpret_cast<T*>(B.velocity_grad);
        for (int l = threadIdx.x; l < nc; l += blockDim.x)
#pragma unroll
            for (int c = 0; c < D; ++c) g[(size_t)c * nc + l] += unbar[(size_t)c * N + off + l];
    }
    // viscosity: per-cell / static block viscosity, else a per-block partial of the system's viscosity
    if (nubar) {
        if (B.viscosity && !B.viscosity_static) {
            if (B.viscosity_grad) {
                T* g = reinterpret_cast<T*>(B.viscosity_grad);
                for (int l = threadIdx.x; l < nc; l += blockDim.x) g[l] += nubar[off + l];
            }
        } else {
            double acc = 0.0;
            for (int l = threadIdx.x; l < nc; l += blockDim.x) acc += (double)nubar[off + l];
            acc = block_reduce_sum(acc, s_red);
            if (threadIdx.x == 0) {
                if (B.viscosity) {
                    if (B.viscosity_grad) reinterpret_cast<T*>(B.viscosity_grad)[0] += (T)acc;
                    if (block_nu) block_nu[bi] = 0.0;
                } else if (block_nu) {
                    block_nu[bi] = acc;
                }
            }
        }
    }
    // velocity source
    if (srcbar && B.source && B.source_grad) {
        T* g = reinterpret_cast<T*>(B.source_grad);
        if (!B.source_static) {
            for (int l = threadIdx.x; l < nc; l += blockDim.x)
#pragma unroll
                for (int c = 0; c < D; ++c) g[(size_t)c * nc + l] += srcbar[(size_t)c * N + off + l];
        } else {
#pragma unroll
            for (int c = 0; c < D; ++c) {
                double acc = 0.0;
                for (int l = threadIdx.x; l < nc; l += blockDim.x) acc += (double)srcbar[(size_t)c * N + off + l];
                acc = block_reduce_sum(acc, s_red);
                if (threadIdx.x == 0) g[c] += (T)acc;
            }
        }
    }
    // boundary velocity of fixed faces
    if (vbbar) {
        for (int f = 0; f < 2 * D; ++f) {
            const pict_face_t& F = B.face[f];
            if (F.type != PICT_FACE_FIXED || !F.velocity_grad) continue;
            T* g = reinterpret_cast<T*>(F.velocity_grad);
            const int nf = face_cells(B.size, f);
            const int a = f >> 1;
            // face cell k -> adjacent cell of the block
            auto cell_of = [&](int k) {
                int q[3];
                int bs[3] = {B.size[0], B.size[1], B.size[2]};
                bs[a] = 1;
                q[0] = k % bs[0];
                q[1] = (k / bs[0]) % bs[1];
                q[2] = k / (bs[0] * bs[1]);
                q[a] = (f & 1) ? B.size[a] - 1 : 0;
                return q[0] + B.size[0] * (q[1] + B.size[1] * q[2]);
            };
            if (!F.vel_static) {
                for (int k = threadIdx.x; k < nf; k += blockDim.x) {
                    const int i = off + cell_of(k);
#pragma unroll
                    for (int c = 0; c < D; ++c) g[(size_t)c * nf + k] += vbbar[((size_t)f * D + c) * N + i];
                }
            } else {
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    double acc = 0.0;
                    for (int k = threadIdx.x; k < nf; k += blockDim.x) acc += (double)vbbar[((size_t)f * D + c) * N + off + cell_of(k)];
                    acc = block_reduce_sum(acc, s_red);
                    if (threadIdx.x == 0) g[c] += (T)acc;
                }
            }
        }
    }
}

// system viscosity gradient: sum of the per-block partials of each system (fixed order)
template <typename T>
__global__ void k_sim_viscosity_grad(pict_domain_t dom, const double* block_nu, T* sim_nu_bar) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= dom.num_sims) return;
    double acc = 0.0;
    for (int b = dom.sim_blocks[s]; b < dom.sim_blocks[s + 1]; ++b) acc += block_nu[b];
    sim_nu_bar[s] += (T)acc;
}

// generic copies between a global [ncomp][N] vector and a per-block field selected by `which`
enum { FIELD_VELOCITY = 0, FIELD_PRESSURE = 1, FIELD_SOURCE = 2, FIELD_VELOCITY_GRAD = 3, FIELD_PRESSURE_GRAD = 4,
       FIELD_SOURCE_GRAD = 5 };

template <typename T>
__global__ void k_copy_field(pict_domain_t dom, int which, int to_blocks, T* glob, int D, int accumulate) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const pict_block_t& B = dom.blocks[dom.cell_block[i]];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        void* ptr = nullptr;
        int ncomp = D;
        switch (which) {
            case FIELD_VELOCITY: ptr = B.velocity; break;
            case FIELD_PRESSURE: ptr = B.pressure; ncomp = 1; break;
            case FIELD_SOURCE: ptr = B.source_static ? nullptr : const_cast<void*>(B.source); break;
            case FIELD_VELOCITY_GRAD: ptr = B.velocity_grad; break;
            case FIELD_PRESSURE_GRAD: ptr = B.pressure_grad; ncomp = 1; break;
            case FIELD_SOURCE_GRAD: ptr = B.source_static ? nullptr : B.source_grad; break;
        }
        if (!ptr) continue;
        T* bf = reinterpret_cast<T*>(ptr);
        for (int c = 0; c < ncomp; ++c) {
            T& bv = bf[(size_t)c * nc + l];
            T& gv = glob[(size_t)c * N + i];
            if (to_blocks) bv = accumulate ? bv + gv : gv;
            else gv = accumulate ? gv + bv : bv;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// SparseOuterProduct on stencils (extensions/PISO_multiblock_cuda_kernel.cu via PISOtorch.cpp:564,
// used by the linear-solve gradient -b_grad x^T, PISOtorch_diff.py:352-371):
//   out[0][i] += s sum_c a_c[i] b_c[i],   out[f+1][i] += s sum_c a_c[i] b_c[j(f,i)]
// ---------------------------------------------------------------------------------------------
template <typename T, int D>
__global__ void k_stencil_outer(pict_domain_t dom, const T* a, const T* bv, int nrhs, T* out, T scale) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        T d = 0;
        for (int c = 0; c < nrhs; ++c) d += a[(size_t)c * N + i] * bv[(size_t)c * N + i];
        out[i] += scale * d;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int j = dom.nbr[(size_t)f * N + i];
            if (j < 0) continue;
            T o = 0;
            for (int c = 0; c < nrhs; ++c) o += a[(size_t)c * N + i] * bv[(size_t)c * N + j];
            out[(size_t)(f + 1) * N + i] += scale * o;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// SetupPressureMatrix gradient (PISOtorch_diff.py:897-965): P_f,i = (al_i[a]/A_i + al_j[a']/A_j)/2,
// P_0,i = -sum_f P_f,i  ->  A_bar_i += -al_i(f>>1)/(2 A_i^2) (P_bar_f,i - P_bar_0,i + P_bar_back,j - P_bar_0,j)
// ---------------------------------------------------------------------------------------------
template <typename T, int D>
__global__ void k_pressure_matrix_grad(pict_domain_t dom, const T* A, const T* Pbar, T* Abar) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T rA = T(1) / A[i];
        const T p0 = Pbar[i];
        T acc = 0;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const Nbr n = neighbour(dom, B, b, p, i, f);
            if (n.j < 0) continue;
            const T g = Pbar[(size_t)(f + 1) * N + i] - p0 + Pbar[(size_t)(n.back + 1) * N + n.j] - Pbar[n.j];
            acc += laplace_coef<T, D>(tr, f >> 1) * g;
        }
        Abar[i] += -T(0.5) * rA * rA * acc;
    }
}

#define PICT_ADJ_DISPATCH(NAME, ...)                                                                 \
    do {                                                                                              \
        if (dom->dtype == PICT_F32 && dom->dims == 2) { NAME<float, 2><<<grid, 256, 0, st>>>(__VA_ARGS__); } \
        else if (dom->dtype == PICT_F32 && dom->dims == 3) { NAME<float, 3><<<grid, 256, 0, st>>>(__VA_ARGS__); } \
        else if (dom->dtype == PICT_F64 && dom->dims == 2) { NAME<double, 2><<<grid, 256, 0, st>>>(__VA_ARGS__); } \
        else if (dom->dtype == PICT_F64 && dom->dims == 3) { NAME<double, 3><<<grid, 256, 0, st>>>(__VA_ARGS__); } \
        else return set_error(PICT_ERR_UNSUPPORTED, #NAME ": unsupported dtype/dims");              \
    } while (0)

static pict_status_t check_dom(const pict_domain_t* dom, const char* what) {
    if (!dom || dom->num_cells <= 0 || !dom->blocks || !dom->nbr || !dom->cell_block) {
        char buf[160];
        snprintf(buf, sizeof(buf), "%s: domain is not prepared", what);
        return set_error(PICT_ERR_ARG, buf);
    }
    return PICT_OK;
}

}  // namespace pict

using namespace pict;

extern "C" {

pict_status_t pict_correct_velocity_grad(const pict_domain_t* dom, const void* A, const void* pressure,
                                         const void* velocity_result_grad, void* A_grad, void* pressure_grad,
                                         void* pressure_rhs_grad, void* stream) {
    pict_status_t s = check_dom(dom, "correct_velocity_grad");
    if (s) return s;
    if (!A || !pressure || !velocity_result_grad || !A_grad || !pressure_grad || !pressure_rhs_grad)
        return set_error(PICT_ERR_ARG, "correct_velocity_grad: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_correct_velocity_grad<float, 2><<<grid, 256, 0, st>>>(*dom, (const float*)A, (const float*)pressure, (const float*)velocity_result_grad, (float*)A_grad, (float*)pressure_grad, (float*)pressure_rhs_grad);
        else k_correct_velocity_grad<float, 3><<<grid, 256, 0, st>>>(*dom, (const float*)A, (const float*)pressure, (const float*)velocity_result_grad, (float*)A_grad, (float*)pressure_grad, (float*)pressure_rhs_grad);
    } else {
        if (dom->dims == 2) k_correct_velocity_grad<double, 2><<<grid, 256, 0, st>>>(*dom, (const double*)A, (const double*)pressure, (const double*)velocity_result_grad, (double*)A_grad, (double*)pressure_grad, (double*)pressure_rhs_grad);
        else k_correct_velocity_grad<double, 3><<<grid, 256, 0, st>>>(*dom, (const double*)A, (const double*)pressure, (const double*)velocity_result_grad, (double*)A_grad, (double*)pressure_grad, (double*)pressure_rhs_grad);
    }
    return check_launch("correct_velocity_grad");
}

pict_status_t pict_sim_mean_project(const pict_domain_t* dom, void* x, void* stream) {
    pict_status_t s = check_dom(dom, "sim_mean_project");
    if (s) return s;
    if (!x || !dom->sim_cells) return set_error(PICT_ERR_ARG, "sim_mean_project: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (dom->dtype == PICT_F32) k_sim_mean_project<float><<<dom->num_sims, 1024, 0, st>>>(*dom, (float*)x);
    else k_sim_mean_project<double><<<dom->num_sims, 1024, 0, st>>>(*dom, (double*)x);
    return check_launch("sim_mean_project");
}

pict_status_t pict_divergence_grad(const pict_domain_t* dom, const void* div_grad, void* pressure_rhs_grad,
                                   void* boundary_velocity_grad, void* stream) {
    pict_status_t s = check_dom(dom, "divergence_grad");
    if (s) return s;
    if (!div_grad || !pressure_rhs_grad || !boundary_velocity_grad) return set_error(PICT_ERR_ARG, "divergence_grad: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_divergence_grad<float, 2><<<grid, 256, 0, st>>>(*dom, (const float*)div_grad, (float*)pressure_rhs_grad, (float*)boundary_velocity_grad);
        else k_divergence_grad<float, 3><<<grid, 256, 0, st>>>(*dom, (const float*)div_grad, (float*)pressure_rhs_grad, (float*)boundary_velocity_grad);
    } else {
        if (dom->dims == 2) k_divergence_grad<double, 2><<<grid, 256, 0, st>>>(*dom, (const double*)div_grad, (double*)pressure_rhs_grad, (double*)boundary_velocity_grad);
        else k_divergence_grad<double, 3><<<grid, 256, 0, st>>>(*dom, (const double*)div_grad, (double*)pressure_rhs_grad, (double*)boundary_velocity_grad);
    }
    return check_launch("divergence_grad");
}

pict_status_t pict_pressure_rhs_grad(const pict_domain_t* dom, double dt, const void* h_grad, const void* h,
                                     const void* A, const void* C, const void* U, const void* lambda,
                                     const void* pressure, void* A_grad, void* C_grad, void* U_grad,
                                     void* velocity_grad, void* source_grad, void* viscosity_grad,
                                     void* boundary_velocity_grad, void* stream) {
    pict_status_t s = check_dom(dom, "pressure_rhs_grad");
    if (s) return s;
    if (!h_grad || !h || !A || !C || !U || !lambda || !pressure || !A_grad || !C_grad || !U_grad || !velocity_grad ||
        !boundary_velocity_grad)
        return set_error(PICT_ERR_ARG, "pressure_rhs_grad: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
#define PRG_ARGS(T)                                                                                             \
    *dom, dt, (const T*)h_grad, (const T*)h, (const T*)A, (const T*)C, (const T*)U, (const T*)lambda,          \
        (const T*)pressure, (T*)A_grad, (T*)C_grad, (T*)U_grad, (T*)velocity_grad, (T*)source_grad, (T*)viscosity_grad, \
        (T*)boundary_velocity_grad
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_pressure_rhs_grad<float, 2><<<grid, 256, 0, st>>>(PRG_ARGS(float));
        else k_pressure_rhs_grad<float, 3><<<grid, 256, 0, st>>>(PRG_ARGS(float));
    } else {
        if (dom->dims == 2) k_pressure_rhs_grad<double, 2><<<grid, 256, 0, st>>>(PRG_ARGS(double));
        else k_pressure_rhs_grad<double, 3><<<grid, 256, 0, st>>>(PRG_ARGS(double));
    }
#undef PRG_ARGS
    return check_launch("pressure_rhs_grad");
}

pict_status_t pict_advection_grad(const pict_domain_t* dom, double dt, const void* velocity_result,
                                  const void* velocity_rhs_grad, const void* C_grad, const void* A_grad,
                                  void* velocity_grad, void* viscosity_grad, void* boundary_velocity_grad,
                                  void* source_grad, void* stream) {
    pict_status_t s = check_dom(dom, "advection_grad");
    if (s) return s;
    if (!velocity_result || !velocity_rhs_grad || !C_grad || !A_grad || !velocity_grad || !boundary_velocity_grad)
        return set_error(PICT_ERR_ARG, "advection_grad: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
#define AG_ARGS(T)                                                                                              \
    *dom, dt, (const T*)velocity_result, (const T*)velocity_rhs_grad, (const T*)C_grad, (const T*)A_grad,       \
        (T*)velocity_grad, (T*)viscosity_grad, (T*)boundary_velocity_grad, (T*)source_grad
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_advection_grad<float, 2><<<grid, 256, 0, st>>>(AG_ARGS(float));
        else k_advection_grad<float, 3><<<grid, 256, 0, st>>>(AG_ARGS(float));
    } else {
        if (dom->dims == 2) k_advection_grad<double, 2><<<grid, 256, 0, st>>>(AG_ARGS(double));
        else k_advection_grad<double, 3><<<grid, 256, 0, st>>>(AG_ARGS(double));
    }
#undef AG_ARGS
    return check_launch("advection_grad");
}

pict_status_t pict_adjoint_to_blocks(const pict_domain_t* dom, const void* velocity_grad, const void* viscosity_grad,
                                     const void* source_grad, const void* boundary_velocity_grad,
                                     void* sim_viscosity_grad, void* block_scratch, void* stream) {
    pict_status_t s = check_dom(dom, "adjoint_to_blocks");
    if (s) return s;
    if (viscosity_grad && (!sim_viscosity_grad || !block_scratch))
        return set_error(PICT_ERR_ARG, "adjoint_to_blocks: viscosity needs sim_viscosity_grad and block_scratch");
    cudaStream_t st = (cudaStream_t)stream;
    double* bn = reinterpret_cast<double*>(block_scratch);
    if (bn) cudaMemsetAsync(bn, 0, sizeof(double) * dom->num_blocks, st);
#define ATB(T, DD)                                                                                              \
    k_adjoint_to_blocks<T, DD><<<dom->num_blocks, 256, 0, st>>>(*dom, (const T*)velocity_grad, (const T*)viscosity_grad, \
                                                                (const T*)source_grad, (const T*)boundary_velocity_grad, bn)
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) ATB(float, 2); else ATB(float, 3);
    } else {
        if (dom->dims == 2) ATB(double, 2); else ATB(double, 3);
    }
#undef ATB
    s = check_launch("adjoint_to_blocks");
    if (s) return s;
    if (viscosity_grad) {
        const int g = (dom->num_sims + 127) / 128;
        if (dom->dtype == PICT_F32) k_sim_viscosity_grad<float><<<g, 128, 0, st>>>(*dom, bn, (float*)sim_viscosity_grad);
        else k_sim_viscosity_grad<double><<<g, 128, 0, st>>>(*dom, bn, (double*)sim_viscosity_grad);
        s = check_launch("sim_viscosity_grad");
    }
    return s;
}

pict_status_t pict_stencil_outer_product(const pict_domain_t* dom, const void* a, const void* b, int32_t nrhs,
                                        void* coef_out, double scale, void* stream) {
    pict_status_t s = check_dom(dom, "stencil_outer_product");
    if (s) return s;
    if (!a || !b || !coef_out || nrhs < 1) return set_error(PICT_ERR_ARG, "stencil_outer_product: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_stencil_outer<float, 2><<<grid, 256, 0, st>>>(*dom, (const float*)a, (const float*)b, nrhs, (float*)coef_out, (float)scale);
        else k_stencil_outer<float, 3><<<grid, 256, 0, st>>>(*dom, (const float*)a, (const float*)b, nrhs, (float*)coef_out, (float)scale);
    } else {
        if (dom->dims == 2) k_stencil_outer<double, 2><<<grid, 256, 0, st>>>(*dom, (const double*)a, (const double*)b, nrhs, (double*)coef_out, scale);
        else k_stencil_outer<double, 3><<<grid, 256, 0, st>>>(*dom, (const double*)a, (const double*)b, nrhs, (double*)coef_out, scale);
    }
    return check_launch("stencil_outer_product");
}

pict_status_t pict_pressure_matrix_grad(const pict_domain_t* dom, const void* A, const void* P_grad, void* A_grad,
                                        void* stream) {
    pict_status_t s = check_dom(dom, "pressure_matrix_grad");
    if (s) return s;
    if (!A || !P_grad || !A_grad) return set_error(PICT_ERR_ARG, "pressure_matrix_grad: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2) k_pressure_matrix_grad<float, 2><<<grid, 256, 0, st>>>(*dom, (const float*)A, (const float*)P_grad, (float*)A_grad);
        else k_pressure_matrix_grad<float, 3><<<grid, 256, 0, st>>>(*dom, (const float*)A, (const float*)P_grad, (float*)A_grad);
    } else {
        if (dom->dims == 2) k_pressure_matrix_grad<double, 2><<<grid, 256, 0, st>>>(*dom, (const double*)A, (const double*)P_grad, (double*)A_grad);
        else k_pressure_matrix_grad<double, 3><<<grid, 256, 0, st>>>(*dom, (const double*)A, (const double*)P_grad, (double*)A_grad);
    }
    return check_launch("pressure_matrix_grad");
}

pict_status_t pict_copy_field(const pict_domain_t* dom, int32_t which, int32_t to_blocks, void* global_vec,
                              int32_t accumulate, void* stream) {
    pict_status_t s = check_dom(dom, "copy_field");
    if (s) return s;
    if (!global_vec || which < 0 || which > FIELD_SOURCE_GRAD) return set_error(PICT_ERR_ARG, "copy_field: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) k_copy_field<float><<<grid, 256, 0, st>>>(*dom, which, to_blocks, (float*)global_vec, dom->dims, accumulate);
    else k_copy_field<double><<<grid, 256, 0, st>>>(*dom, which, to_blocks, (double*)global_vec, dom->dims, accumulate);
    return check_launch("copy_field");
}

}  // extern "C"
