// scalar.cu -- passive scalar transport operators.
//
// A passive scalar (C channels, Block::passiveScalar [1,C,...]) is advected with the velocity of the
// step and diffuses with the scalar viscosity (Domain scalarViscosity [1] or [C], else the domain
// viscosity; block viscosities do not apply).  Restated here:
//   PISO_build_matrix with forPassiveScalar      extensions/PISO_multiblock_cuda_kernel.cu:3601-3865
//   kPISO_build_scalar_advection_RHS             extensions/PISO_multiblock_cuda_kernel.cu:4079-4183
//   CopyScalarResult{To,From}Blocks              extensions/PISO_multiblock_cuda_kernel.cu:6543-6733
// Fixed faces carry a per-channel boundary type: Dirichlet faces diffuse towards the boundary value
// (2 nu alpha on the diagonal, 2 nu alpha s_b on the RHS), Neumann faces add nu s_b on the RHS (s_b
// is then the prescribed gradient) and nothing to the matrix; the advective flux through a fixed face
// moves s_b.  The non-orthogonal terms are added by the passes of nonortho.cu.
#include "common.cuh"
#include "launch.h"

namespace pict {

template <typename T>
__device__ __forceinline__ T scalar_viscosity(const pict_domain_t& dom, const pict_block_t& B, int c) {
    if (dom.scalar_viscosity) {
        const T* v = reinterpret_cast<const T*>(dom.scalar_viscosity);
        return dom.scalar_viscosity_static ? v[0] : v[c];
    }
    return reinterpret_cast<const T*>(dom.sim_viscosity)[B.sim];
}

// C and A of channel ch: the advection-diffusion matrix of the velocity operator with the scalar
// viscosity and no diffusion through the channel's Neumann faces.
template <typename T, int D>
__global__ void k_scalar_matrix(pict_domain_t dom, double dt_arg, int ch) {
    const int N = dom.num_cells;
    T* C = reinterpret_cast<T*>(dom.C);
    T* A = reinterpret_cast<T*>(dom.A);
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T det = tr_det<T, D>(tr);
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
        const T nu = scalar_viscosity<T>(dom, B, ch);
        T u[D];
        load_block_vec<T, D>(B, B.velocity, l, u);
        T diag = det / dt;
        T off[2 * D];
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const T sign = (f & 1) ? T(1) : T(-1);
            const T alpha_p = laplace_coef<T, D>(tr, a);
            const Nbr n = neighbour(dom, B, b, p, i, f);
            off[f] = T(0);
            if (n.j < 0) {
                if (!((B.face[f].scalar_neumann >> ch) & 1u)) diag += T(2) * nu * alpha_p;
            } else {
                const pict_block_t& Bn = dom.blocks[n.b];
                const T* trn = cell_transform<T, D>(Bn, n.l);
                T un[D];
                load_block_vec<T, D>(Bn, Bn.velocity, n.l, un);
                const T velN = contravariant<T, D>(trn, n.comp, un) * T(n.flip);
                const T faceFlux = sign * T(0.5) * (velN + contravariant<T, D>(tr, a, u)) * T(0.5);
                const T vc = (alpha_p + laplace_coef<T, D>(trn, n.comp)) * nu * T(0.5);
                diag += faceFlux + vc;
                off[f] = faceFlux - vc;
            }
        }
        C[i] = diag / det;
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) C[(size_t)(f + 1) * N + i] = off[f] / det;
        A[i] = diag / det;
    }
}

// scalar_rhs [C][N]: (det s / dt + fixed-face terms) / det for every channel.
template <typename T, int D>
__global__ void k_scalar_rhs(pict_domain_t dom, double dt_arg) {
    const int N = dom.num_cells;
    const int NC = dom.scalar_channels;
    T* out = reinterpret_cast<T*>(dom.scalar_rhs);
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T det = tr_det<T, D>(tr);
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
        const T* s = reinterpret_cast<const T*>(B.scalar);
#pragma unroll 1
        for (int c = 0; c < NC; ++c) {
            T r = det * (s ? s[(size_t)c * nc + l] : T(0)) / dt;
            const T nu = scalar_viscosity<T>(dom, B, c);
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                if (!at_face(p, B.size, f) || B.face[f].type != PICT_FACE_FIXED) continue;
                const pict_face_t& F = B.face[f];
                const int bf = boundary_flat(p, B.size, f);
                const T* sv = reinterpret_cast<const T*>(F.scalar);
                const T sb = sv ? (F.scalar_static ? sv[c] : sv[(size_t)c * face_cells(B.size, f) + bf]) : T(0);
                const FixedFace<T, D> ff = fixed_face<T, D>(B, p, f);
                r -= sb * ff.contra * ((f & 1) ? T(1) : T(-1));
                r += ((F.scalar_neumann >> c) & 1u) ? sb * nu : sb * nu * T(2) * ff.alpha;
            }
            out[(size_t)c * N + i] = r / det;
        }
    }
}

template <typename T, bool TO_BLOCKS>
__global__ void k_copy_scalar(pict_domain_t dom) {
    const int N = dom.num_cells;
    const int NC = dom.scalar_channels;
    T* g = reinterpret_cast<T*>(dom.scalar_result);
    PICT_CELL_LOOP(i, N) {
        const pict_block_t& B = dom.blocks[dom.cell_block[i]];
        T* s = reinterpret_cast<T*>(B.scalar);
        if (!s) continue;
        const int l = i - B.offset;
        const int nc = B.size[0] * B.size[1] * B.size[2];
        for (int c = 0; c < NC; ++c) {
            if (TO_BLOCKS) s[(size_t)c * nc + l] = g[(size_t)c * N + i];
            else g[(size_t)c * N + i] = s[(size_t)c * nc + l];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// gradients (PISO_build_matrix_GRAD with forPassiveScalar, extensions/PISO_multiblock_cuda_kernel.cu:3869-4077;
// kPISO_build_scalar_advection_RHS_GRAD :4185-4278)
// ---------------------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ void atomic_add_nz(T* p, T v) {
    if (v != T(0)) atomicAdd(p, v);
}

// C_bar [K][N], A_bar [N] of channel ch -> u_bar [D][N] (block velocity, through the face fluxes) and
// nu_bar [N] (the channel's scalar viscosity, per cell contribution)
template <typename T, int D>
__global__ void k_scalar_matrix_grad(pict_domain_t dom, int ch, const T* Cbar, const T* Abar, T* u_bar, T* nu_bar) {
    const int N = dom.num_cells;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T rdet = T(1) / tr_det<T, D>(tr);
        const T diag_bar = (Cbar[i] + (Abar ? Abar[i] : T(0))) * rdet;
        const T nu = scalar_viscosity<T>(dom, B, ch);
        T nub = T(0);
        T ub[D];
#pragma unroll
        for (int c = 0; c < D; ++c) ub[c] = T(0);
#pragma unroll
        for (int f = 0; f < 2 * D; ++f) {
            const int a = f >> 1;
            const T sign = (f & 1) ? T(1) : T(-1);
            const T alpha_p = laplace_coef<T, D>(tr, a);
            const Nbr n = neighbour(dom, B, b, p, i, f);
            if (n.j < 0) {
                if (!((B.face[f].scalar_neumann >> ch) & 1u)) nub += T(2) * alpha_p * diag_bar;
                continue;
            }
            const T off_bar = Cbar[(size_t)(f + 1) * N + i] * rdet;
            const pict_block_t& Bn = dom.blocks[n.b];
            const T* trn = cell_transform<T, D>(Bn, n.l);
            // faceFlux = sign/4 (contra(u) + flip contra_N(u_N)), entering diag and off with +
            const T flux_bar = sign * T(0.25) * (diag_bar + off_bar);
            const T dP = tr_det<T, D>(tr), dN = tr_det<T, D>(trn);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                ub[c] += flux_bar * dP * (tr ? tr_minv<T, D>(tr, a, c) : (a == c ? T(1) : T(0)));
                const T wn = flux_bar * T(n.flip) * dN * (trn ? tr_minv<T, D>(trn, n.comp, c) : (n.comp == c ? T(1) : T(0)));
                atomic_add_nz(u_bar + (size_t)c * N + n.j, wn);
            }
            // vc = (alpha_p + alpha_n) nu / 2 enters diag with + and off with -
            nub += (alpha_p + laplace_coef<T, D>(trn, n.comp)) * T(0.5) * (diag_bar - off_bar);
        }
#pragma unroll
        for (int c = 0; c < D; ++c) atomic_add_nz(u_bar + (size_t)c * N + i, ub[c]);
        atomic_add_nz(nu_bar + i, nub);
        (void)nu;
    }
}

// scalarRHS_bar [C][N] -> s_bar [C][N] (block scalar, assigned), sb_bar [2D][C][N] (boundary scalar, per
// adjacent cell), vb_bar [2D][D][N] (boundary velocity, through the boundary flux), nu_bar [C][N]
template <typename T, int D>
__global__ void k_scalar_rhs_grad(pict_domain_t dom, double dt_arg, const T* rhs_bar, T* s_bar, T* sb_bar, T* vb_bar,
                                  T* nu_bar) {
    const int N = dom.num_cells;
    const int NC = dom.scalar_channels;
    PICT_CELL_LOOP(i, N) {
        const int b = dom.cell_block[i];
        const pict_block_t& B = dom.blocks[b];
        const int l = i - B.offset;
        int p[3];
        unflatten(l, B.size, p);
        const T* tr = cell_transform<T, D>(B, l);
        const T rdet = T(1) / tr_det<T, D>(tr);
        const T dt = sim_time_step<T>(dom, B.sim, dt_arg);
#pragma unroll 1
        for (int c = 0; c < NC; ++c) {
            const T rb = rhs_bar[(size_t)c * N + i];
            s_bar[(size_t)c * N + i] = rb / dt;
            const T r = rb * rdet;
            const T nu = scalar_viscosity<T>(dom, B, c);
            T nub = T(0);
#pragma unroll
            for (int f = 0; f < 2 * D; ++f) {
                if (!at_face(p, B.size, f) || B.face[f].type != PICT_FACE_FIXED) continue;
                const pict_face_t& F = B.face[f];
                const int a = f >> 1;
                const T sign = (f & 1) ? T(1) : T(-1);
                const int bf = boundary_flat(p, B.size, f);
                const T* sv = reinterpret_cast<const T*>(F.scalar);
                const T sb = sv ? (F.scalar_static ? sv[c] : sv[(size_t)c * face_cells(B.size, f) + bf]) : T(0);
                const FixedFace<T, D> ff = fixed_face<T, D>(B, p, f);
                const bool neu = (F.scalar_neumann >> c) & 1u;
                T s_grad = -ff.contra * sign * r;
                if (neu) {
                    s_grad += nu * r;
                    nub += sb * r;
                } else {
                    s_grad += nu * T(2) * ff.alpha * r;
                    nub += sb * T(2) * ff.alpha * r;
                }
                atomic_add_nz(sb_bar + ((size_t)f * NC + c) * N + i, s_grad);
                // flux = contra(v_b) * sign: d/dv_b[k] = det_b Minv_b[a][k] sign
                const T* btr = F.transform ? reinterpret_cast<const T*>(F.transform) + (size_t)bf * TS<D>::value : nullptr;
                const T fg = -sb * r * sign * tr_det<T, D>(btr);
#pragma unroll
                for (int k = 0; k < D; ++k)
                    atomic_add_nz(vb_bar + ((size_t)f * D + k) * N + i, fg * (btr ? tr_minv<T, D>(btr, a, k) : (a == k ? T(1) : T(0))));
            }
            atomic_add_nz(nu_bar + (size_t)c * N + i, nub);
        }
    }
}

static pict_status_t check_scalar_dom(const pict_domain_t* dom, bool need_rhs) {
    if (!dom || !dom->blocks || !dom->cell_block || !dom->nbr) return set_error(PICT_ERR_ARG, "scalar: domain is not prepared");
    if (dom->scalar_channels < 1) return set_error(PICT_ERR_ARG, "scalar: the domain has no passive scalar channels");
    if (dom->scalar_channels > 32) return set_error(PICT_ERR_UNSUPPORTED, "scalar: at most 32 passive scalar channels");
    if (need_rhs && (!dom->scalar_rhs || !dom->scalar_result)) return set_error(PICT_ERR_ARG, "scalar: scalarRHS / scalarResult missing");
    if (!(dom->dims == 2 || dom->dims == 3) || !(dom->dtype == PICT_F32 || dom->dtype == PICT_F64))
        return set_error(PICT_ERR_UNSUPPORTED, "scalar: unsupported dtype/dims");
    return PICT_OK;
}

}  // namespace pict

using namespace pict;

#define PICT_SC_DISPATCH(KERNEL, ...)                                                                          \
    do {                                                                                                         \
        if (dom->dtype == PICT_F32) {                                                                            \
            if (dom->dims == 2) KERNEL<float, 2><<<grid, 256, 0, st>>>(__VA_ARGS__);                            \
            else KERNEL<float, 3><<<grid, 256, 0, st>>>(__VA_ARGS__);                                           \
        } else {                                                                                                 \
            if (dom->dims == 2) KERNEL<double, 2><<<grid, 256, 0, st>>>(__VA_ARGS__);                           \
            else KERNEL<double, 3><<<grid, 256, 0, st>>>(__VA_ARGS__);                                          \
        }                                                                                                        \
    } while (0)

extern "C" pict_status_t pict_setup_scalar_matrix(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                                  int32_t channel, void* stream) {
    pict_status_t s = check_scalar_dom(dom, false);
    if (s) return s;
    if (channel < 0 || channel >= dom->scalar_channels) return set_error(PICT_ERR_ARG, "scalar matrix: channel out of range");
    if (!dom->C || !dom->A) return set_error(PICT_ERR_ARG, "scalar matrix: C / A missing");
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    PICT_SC_DISPATCH(k_scalar_matrix, *dom, dt, channel);
    s = check_launch("scalar_matrix");
    if (s || !non_ortho_flags) return s;
    return nonortho_pass_ch(dom, non_ortho_flags, 4, channel, stream);
}

extern "C" pict_status_t pict_setup_scalar_rhs(const pict_domain_t* dom, double dt, int32_t non_ortho_flags, void* stream) {
    pict_status_t s = check_scalar_dom(dom, true);
    if (s) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    PICT_SC_DISPATCH(k_scalar_rhs, *dom, dt);
    s = check_launch("scalar_rhs");
    if (s || !non_ortho_flags) return s;
    return nonortho_pass_ch(dom, non_ortho_flags, 5, 0, stream);
}

extern "C" pict_status_t pict_copy_scalar_result(const pict_domain_t* dom, int32_t to_blocks, void* stream) {
    pict_status_t s = check_scalar_dom(dom, true);
    if (s) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = cell_grid(dom->num_cells, 256);
    if (dom->dtype == PICT_F32) {
        if (to_blocks) k_copy_scalar<float, true><<<grid, 256, 0, st>>>(*dom);
        else k_copy_scalar<float, false><<<grid, 256, 0, st>>>(*dom);
    } else {
        if (to_blocks) k_copy_scalar<double, true><<<grid, 256, 0, st>>>(*dom);
        else k_copy_scalar<double, false><<<grid, 256, 0, st>>>(*dom);
    }
    return check_launch("copy_scalar_result");
}

template <typename T, int D>
static pict_status_t launch_scalar_grad(const pict_domain_t* dom, double dt, int flags, int what, int ch, const void* in_bar,
                                        const void* A_bar, void* u_bar, void* s_bar, void* sres_bar, void* sb_bar,
                                        void* vb_bar, void* nu_bar, cudaStream_t st) {
    const int grid = cell_grid(dom->num_cells, 256);
    if (what == 0) {
        k_scalar_matrix_grad<T, D><<<grid, 256, 0, st>>>(*dom, ch, (const T*)in_bar, (const T*)A_bar, (T*)u_bar, (T*)nu_bar);
        pict_status_t s = check_launch("scalar_matrix_grad");
        if (s || !flags) return s;
        return nonortho_grad_scalar(dom, flags, 4, ch, in_bar, A_bar, nullptr, nu_bar, nullptr, st);
    }
    k_scalar_rhs_grad<T, D><<<grid, 256, 0, st>>>(*dom, dt, (const T*)in_bar, (T*)s_bar, (T*)sb_bar, (T*)vb_bar, (T*)nu_bar);
    pict_status_t s = check_launch("scalar_rhs_grad");
    if (s || !flags) return s;
    return nonortho_grad_scalar(dom, flags, 5, 0, in_bar, nullptr, sres_bar, nu_bar, sb_bar, st);
}

extern "C" pict_status_t pict_scalar_grad(const pict_domain_t* dom, double dt, int32_t non_ortho_flags, int32_t what,
                                          int32_t channel, const void* in_bar, const void* A_bar, void* u_bar,
                                          void* s_bar, void* s_result_bar, void* boundary_scalar_grad,
                                          void* boundary_velocity_grad, void* nu_bar, void* stream) {
    pict_status_t s = check_scalar_dom(dom, what == 1);
    if (s) return s;
    if (!in_bar || !nu_bar) return set_error(PICT_ERR_ARG, "scalar_grad: NULL argument");
    if (what == 0) {
        if (channel < 0 || channel >= dom->scalar_channels) return set_error(PICT_ERR_ARG, "scalar_grad: channel out of range");
        if (!u_bar) return set_error(PICT_ERR_ARG, "scalar_grad: velocity gradient missing");
    } else if (what == 1) {
        if (!s_bar || !s_result_bar || !boundary_scalar_grad || !boundary_velocity_grad)
            return set_error(PICT_ERR_ARG, "scalar_grad: gradient output missing");
    } else {
        return set_error(PICT_ERR_ARG, "scalar_grad: what must be 0 or 1");
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (dom->dtype == PICT_F32) {
        if (dom->dims == 2)
            return launch_scalar_grad<float, 2>(dom, dt, non_ortho_flags, what, channel, in_bar, A_bar, u_bar, s_bar, s_result_bar,
                                                boundary_scalar_grad, boundary_velocity_grad, nu_bar, st);
        return launch_scalar_grad<float, 3>(dom, dt, non_ortho_flags, what, channel, in_bar, A_bar, u_bar, s_bar, s_result_bar,
                                            boundary_scalar_grad, boundary_velocity_grad, nu_bar, st);
    }
    if (dom->dims == 2)
        return launch_scalar_grad<double, 2>(dom, dt, non_ortho_flags, what, channel, in_bar, A_bar, u_bar, s_bar, s_result_bar,
                                             boundary_scalar_grad, boundary_velocity_grad, nu_bar, st);
    return launch_scalar_grad<double, 3>(dom, dt, non_ortho_flags, what, channel, in_bar, A_bar, u_bar, s_bar, s_result_bar,
                                         boundary_scalar_grad, boundary_velocity_grad, nu_bar, st);
}
