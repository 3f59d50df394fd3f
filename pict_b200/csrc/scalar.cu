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
