// outflow.cu -- advective outflow boundaries on the device (update_advective_boundaries and
// balance_boundary_fluxes, PISOtorch_simulation.py:145-312), so that a step with outflow faces stays
// free of host round trips and can be captured in a CUDA graph.
//
// One CTA does the whole update, because the outflow faces of a domain hold a few hundred cells and
// the flux balance is a reduction over every fixed face followed by a rescale of the outflow faces:
//   1. each outflow face cell moves its boundary velocity towards the adjacent cell of the block,
//      u_b <- u_b - t (u_b - u_cell), t = 1 - 1/(1 + 2 dt c), c the face-normal component of the
//      characteristic velocity (row `axis` of the boundary transform's M^-1 times it, or its
//      component along the face axis without a transform);
//   2. the net outward flux det (M^-1 u_b)_axis of all fixed faces, summed in FP64, split into the
//      outflow faces' part and the rest (FixedBoundary::GetFluxes, extensions/domain_structs.cpp:527-542;
//      lower faces count negative);
//   3. unless |rest + outflow| is within the given tolerance of zero, the outflow faces' velocity is
//      scaled by -rest / outflow.
// The boundary velocity is updated in place: the block table keeps pointing at the same tensors.
#include "common.cuh"
#include "launch.h"

namespace pict {

constexpr int OF_THREADS = 512;

struct OutflowFaces {
    int n;
    int block[PICT_MAX_OUTFLOW_FACES];
    int face[PICT_MAX_OUTFLOW_FACES];
    double velm[3];
};

// position of face cell q of face f of a block (the cell layer next to the face)
__device__ __forceinline__ int face_cell_local(const int32_t* size, int f, int q) {
    const int a = f >> 1;
    int bs[3] = {size[0], size[1], size[2]};
    bs[a] = 1;
    int p[3];
    p[0] = q % bs[0];
    const int t = q / bs[0];
    p[1] = t % bs[1];
    p[2] = t / bs[1];
    p[a] = (f & 1) ? size[a] - 1 : 0;
    return p[0] + size[0] * (p[1] + size[1] * p[2]);
}

__device__ __forceinline__ bool is_outflow(const OutflowFaces& of, int b, int f) {
    for (int k = 0; k < of.n; ++k)
        if (of.block[k] == b && of.face[k] == f) return true;
    return false;
}

template <typename T, int D>
__global__ void __launch_bounds__(OF_THREADS) k_advective_outflow(pict_domain_t dom, OutflowFaces of, double dt,
                                                                  double atol) {
    __shared__ double red[2][OF_THREADS / 32];
    __shared__ double scale_s;
    const int tid = threadIdx.x;
    // 1. implicit upwind update of the outflow faces
    for (int k = 0; k < of.n; ++k) {
        const pict_block_t& B = dom.blocks[of.block[k]];
        const int f = of.face[k];
        const int a = f >> 1;
        const pict_face_t& F = B.face[f];
        T* vb = reinterpret_cast<T*>(const_cast<void*>(F.velocity));
        const T* vc = reinterpret_cast<const T*>(B.velocity);
        const int nf = face_cells(B.size, f);
        const int nc = B.size[0] * B.size[1] * B.size[2];
        const T dts = sim_time_step<T>(dom, B.sim, dt);
        for (int q = tid; q < nf; q += blockDim.x) {
            T c;
            if (F.transform) {
                const T* tr = reinterpret_cast<const T*>(F.transform) + (size_t)q * TS<D>::value;
                c = T(0);
#pragma unroll
                for (int j = 0; j < D; ++j) c += tr_minv<T, D>(tr, a, j) * T(of.velm[j]);
            } else {
                c = T(of.velm[a]);
            }
            const T alpha = dts * T(2) * c;
            const T t = T(1) - T(1) / (T(1) + alpha);
            const int l = face_cell_local(B.size, f, q);
#pragma unroll
            for (int comp = 0; comp < D; ++comp) {
                const T ub = vb[(size_t)comp * nf + q];
                vb[(size_t)comp * nf + q] = ub - t * (ub - vc[(size_t)comp * nc + l]);
            }
        }
    }
    __syncthreads();
    // 2. net outward flux of the fixed faces, FP64
    double s_rest = 0.0, s_out = 0.0;
    for (int b = 0; b < dom.num_blocks; ++b) {
        const pict_block_t& B = dom.blocks[b];
        for (int f = 0; f < 2 * D; ++f) {
            const pict_face_t& F = B.face[f];
            if (F.type != PICT_FACE_FIXED) continue;
            const int a = f >> 1;
            const int nf = face_cells(B.size, f);
            const T* v = reinterpret_cast<const T*>(F.velocity);
            const bool out = is_outflow(of, b, f);
            double s = 0.0;
            for (int q = tid; q < nf; q += blockDim.x) {
                T u[D];
#pragma unroll
                for (int comp = 0; comp < D; ++comp) u[comp] = F.vel_static ? v[comp] : v[(size_t)comp * nf + q];
                const T* tr = F.transform ? reinterpret_cast<const T*>(F.transform) + (size_t)q * TS<D>::value : nullptr;
                s += (double)contravariant<T, D>(tr, a, u);
            }
            if (!(f & 1)) s = -s;
            if (out) s_out += s; else s_rest += s;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s_rest += __shfl_xor_sync(0xffffffffu, s_rest, o);
        s_out += __shfl_xor_sync(0xffffffffu, s_out, o);
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = s_rest;
        red[1][tid >> 5] = s_out;
    }
    __syncthreads();
    if (tid == 0) {
        double r = 0.0, o = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {  // fixed order: result independent of timing
            r += red[0][w];
            o += red[1][w];
        }
        scale_s = (fabs(r + o) > atol && o != 0.0) ? -r / o : 1.0;
    }
    __syncthreads();
    // 3. rescale the outflow faces
    const double scale = scale_s;
    if (scale == 1.0) return;
    const T sc = T(scale);
    for (int k = 0; k < of.n; ++k) {
        const pict_block_t& B = dom.blocks[of.block[k]];
        const int f = of.face[k];
        T* vb = reinterpret_cast<T*>(const_cast<void*>(B.face[f].velocity));
        const int n = D * face_cells(B.size, f);
        for (int q = tid; q < n; q += blockDim.x) vb[q] = vb[q] * sc;
    }
}

}  // namespace pict

using namespace pict;

extern "C" pict_status_t pict_advective_outflow(const pict_domain_t* dom, const int32_t* faces, int32_t num_faces,
                                                const double* char_velocity, double dt, double atol, void* stream) {
    if (!dom || !faces || !char_velocity || !dom->blocks) return set_error(PICT_ERR_ARG, "advective_outflow: NULL argument");
    if (num_faces < 1 || num_faces > PICT_MAX_OUTFLOW_FACES)
        return set_error(PICT_ERR_ARG, "advective_outflow: between 1 and PICT_MAX_OUTFLOW_FACES outflow faces");
    if (dom->num_sims != 1)
        return set_error(PICT_ERR_UNSUPPORTED, "advective_outflow: the flux balance covers one simulation per domain");
    const int D = dom->dims;
    if (D < 1 || D > 3) return set_error(PICT_ERR_UNSUPPORTED, "advective_outflow: unsupported dims");
    OutflowFaces of = {};
    of.n = num_faces;
    for (int k = 0; k < num_faces; ++k) {
        of.block[k] = faces[2 * k];
        of.face[k] = faces[2 * k + 1];
        if (of.block[k] < 0 || of.block[k] >= dom->num_blocks || of.face[k] < 0 || of.face[k] >= 2 * D)
            return set_error(PICT_ERR_ARG, "advective_outflow: face index out of range");
    }
    for (int d = 0; d < 3; ++d) of.velm[d] = d < D ? char_velocity[d] : 0.0;
    cudaStream_t st = (cudaStream_t)stream;
    if (dom->dtype == PICT_F32) {
        if (D == 2) k_advective_outflow<float, 2><<<1, OF_THREADS, 0, st>>>(*dom, of, dt, atol);
        else if (D == 3) k_advective_outflow<float, 3><<<1, OF_THREADS, 0, st>>>(*dom, of, dt, atol);
        else return set_error(PICT_ERR_UNSUPPORTED, "advective_outflow: unsupported dims");
    } else if (dom->dtype == PICT_F64) {
        if (D == 2) k_advective_outflow<double, 2><<<1, OF_THREADS, 0, st>>>(*dom, of, dt, atol);
        else if (D == 3) k_advective_outflow<double, 3><<<1, OF_THREADS, 0, st>>>(*dom, of, dt, atol);
        else return set_error(PICT_ERR_UNSUPPORTED, "advective_outflow: unsupported dims");
    } else {
        return set_error(PICT_ERR_UNSUPPORTED, "advective_outflow: unsupported dtype");
    }
    return check_launch("advective_outflow");
}
