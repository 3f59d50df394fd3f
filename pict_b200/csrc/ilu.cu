// ilu.cu -- ILU(0)-preconditioned BiCGStab (SolveLinear with BiCGwithPreconditioner, bicgstabSolveGPU
// extensions/bicgstab_solver_kernel.cu:47-395), the fallback the reference's solve wrapper takes when an
// unpreconditioned BiCGStab solve fails (PISOtorch_diff.py:276-286).
//
// The matrix is the CSR form of the stencil (rows sorted by column, as the reference's).  ILU(0) keeps
// the pattern: for every row i, for every lower entry k (column c < i, in column order) l_ic = a_ic / u_cc
// and a_ij -= l_ic u_cj for the later entries j of the row whose column also occurs in row c (the
// IKJ order of csrilu02); L has a unit diagonal, U the computed one.  Rows depend on the rows of their
// lower entries, so the factorisation and the triangular solves run level by level: the levels of the
// forward dependencies (level(i) = 1 + max level of its lower entries) and of the backward ones come from
// the pattern alone, once per domain, on the host (pict_ilu_analyze); each level is one launch over its
// rows.  The stencil pattern is structurally symmetric, so the transposed solves read entry (j, i)
// through a map of transposed positions.
//
// The solve is the reference's right-preconditioned BiCGStab loop (residual checks after both half
// steps, the same reported iterations), driven from the host with the scalars read back per reduction.
// Two preconditioners:
//  * PICT_PRECOND_AS_REFERENCE: the operator the reference's build applies, M = T T with T the lower
//    triangle of A including its diagonal (the matrix values, not the factors), applied as two forward
//    sweeps T^-1 T^-1 (transposed: two backward sweeps T^-T T^-T).  This reproduces the reference's
//    preconditioned solves (iterations, residuals, solutions) on the recorded systems;
//  * PICT_PRECOND_ILU0: M = L U of the ILU(0) factors, applied as U^-1 L^-1 (transposed: M^T = U^T L^T,
//    applied as L^-T U^-T).
#include <cmath>
#include <cstdio>
#include <vector>
#include "common.cuh"
#include "launch.h"

namespace pict {

constexpr int ILU_THREADS = 256;
constexpr int ILU_RED_BLOCKS = 296;

template <typename T>
__global__ void k_ilu_level(const int* __restrict__ row, const int* __restrict__ index, const int* __restrict__ diag,
                            T* __restrict__ f, const int* __restrict__ order, int begin, int count) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int i = order[begin + t];
    const int e = row[i + 1];
    for (int k = row[i]; k < e; ++k) {
        const int c = index[k];
        if (c >= i) break;
        const T lic = f[k] / f[diag[c]];
        f[k] = lic;
        for (int j = k + 1; j < e; ++j) {
            const int cj = index[j];
            for (int m = row[c]; m < row[c + 1]; ++m)
                if (index[m] == cj) {
                    f[j] -= lic * f[m];
                    break;
                }
        }
    }
}

// One level of a triangular solve.  FWD: entries with column < i, else column > i.  UNIT: unit diagonal.
// TR: the transposed factor (entry (i, j) read at tpos of the stored (j, i)).
template <typename T, bool FWD, bool UNIT, bool TR>
__global__ void k_trsv_level(const int* __restrict__ row, const int* __restrict__ index, const int* __restrict__ diag,
                             const int* __restrict__ tpos, const T* __restrict__ f, const T* __restrict__ in,
                             T* __restrict__ out, const int* __restrict__ order, int begin, int count) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int i = order[begin + t];
    T acc = in[i];
    for (int k = row[i]; k < row[i + 1]; ++k) {
        const int j = index[k];
        if (FWD ? j < i : j > i) acc -= (TR ? f[tpos[k]] : f[k]) * out[j];
    }
    out[i] = UNIT ? acc : acc / f[diag[i]];
}

template <typename T, bool TR>
__global__ void k_csr_spmv(int n, const int* __restrict__ row, const int* __restrict__ index,
                           const int* __restrict__ tpos, const T* __restrict__ a, const T* __restrict__ x,
                           T* __restrict__ y) {
    PICT_CELL_LOOP(i, n) {
        T acc = T(0);
        for (int k = row[i]; k < row[i + 1]; ++k) acc += (TR ? a[tpos[k]] : a[k]) * x[index[k]];
        y[i] = acc;
    }
}

// y = a x + b y (and the variants the loop needs)
template <typename T>
__global__ void k_axpby(int n, T a, const T* __restrict__ x, T b, T* __restrict__ y) {
    PICT_CELL_LOOP(i, n) y[i] = a * x[i] + b * y[i];
}

// p = r + beta (p - omega v)
template <typename T>
__global__ void k_bicg_dir(int n, const T* __restrict__ r, T beta, T omega, const T* __restrict__ v, T* __restrict__ p) {
    PICT_CELL_LOOP(i, n) p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

// per-CTA FP64 partials of a.b (KIND 0), |a| (1), max |a| (2); fixed grid, then one CTA sums in order
template <typename T, int KIND>
__global__ void k_red_partial(int n, const T* __restrict__ a, const T* __restrict__ b, double* __restrict__ part) {
    __shared__ double s[ILU_THREADS / 32];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x) {
        const double v = (double)a[i];
        if (KIND == 0) acc += v * (double)b[i];
        else if (KIND == 1) acc += fabs(v);
        else acc = fmax(acc, fabs(v));
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, acc, o);
        acc = KIND == 2 ? fmax(acc, w) : acc + w;
    }
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = KIND == 2 ? fmax(t, s[w]) : t + s[w];
        part[blockIdx.x] = t;
    }
}

template <int KIND>
__global__ void k_red_final(const double* __restrict__ part, int m, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    for (int k = 0; k < m; ++k) t = KIND == 2 ? fmax(t, part[k]) : t + part[k];
    *out = t;
}

struct IluPlan {
    int n, nnz, nlf, nlb;
    const int *row, *index, *diag, *tpos, *order_f, *ptr_f_dev, *order_b, *ptr_b_dev;
    std::vector<int> ptr_f, ptr_b;  // level starts (host)
};

template <typename T>
struct IluSolver {
    const IluPlan& P;
    cudaStream_t st;
    double* part;
    double* scal;  // device scalar
    double host = 0.0;

    pict_status_t reduce(int kind, const T* a, const T* b, double* out) {
        if (kind == 0) k_red_partial<T, 0><<<ILU_RED_BLOCKS, ILU_THREADS, 0, st>>>(P.n, a, b, part);
        else if (kind == 1) k_red_partial<T, 1><<<ILU_RED_BLOCKS, ILU_THREADS, 0, st>>>(P.n, a, b, part);
        else k_red_partial<T, 2><<<ILU_RED_BLOCKS, ILU_THREADS, 0, st>>>(P.n, a, b, part);
        if (kind == 0) k_red_final<0><<<1, 32, 0, st>>>(part, ILU_RED_BLOCKS, scal);
        else if (kind == 1) k_red_final<1><<<1, 32, 0, st>>>(part, ILU_RED_BLOCKS, scal);
        else k_red_final<2><<<1, 32, 0, st>>>(part, ILU_RED_BLOCKS, scal);
        pict_status_t s = check_launch("ilu reduction");
        if (s) return s;
        if (cudaMemcpyAsync(&host, scal, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return check_launch("ilu reduction read-back");
        *out = host;
        return PICT_OK;
    }

    // ComputeConvergenceCriterion (extensions/cg_solver_kernel.cu:77-110); ABS_MAX is max |r|
    pict_status_t crit(const T* r, int conv, double* out) {
        double v = 0.0;
        pict_status_t s;
        if (conv == PICT_CONV_ABS_SUM || conv == PICT_CONV_ABS_MEAN) s = reduce(1, r, nullptr, &v);
        else if (conv == PICT_CONV_ABS_MAX) s = reduce(2, r, nullptr, &v);
        else s = reduce(0, r, r, &v);
        if (s) return s;
        if (conv == PICT_CONV_NORM2) v = sqrt(v);
        else if (conv == PICT_CONV_NORM2_NORMALIZED) v = sqrt(v) / sqrt((double)P.n);
        else if (conv == PICT_CONV_ABS_MEAN) v = v / (double)P.n;
        *out = v;
        return PICT_OK;
    }

    template <bool FWD, bool UNIT, bool TR>
    pict_status_t trsv(const T* f, const T* in, T* out) {
        const std::vector<int>& ptr = FWD ? P.ptr_f : P.ptr_b;
        const int* order = FWD ? P.order_f : P.order_b;
        const int nl = FWD ? P.nlf : P.nlb;
        for (int l = 0; l < nl; ++l) {
            const int b = ptr[l], c = ptr[l + 1] - ptr[l];
            k_trsv_level<T, FWD, UNIT, TR><<<(c + ILU_THREADS - 1) / ILU_THREADS, ILU_THREADS, 0, st>>>(
                P.row, P.index, P.diag, P.tpos, f, in, out, order, b, c);
        }
        return check_launch("ilu triangular solve");
    }

    // out = M^-1 in, or M^-T in; y: scratch.  ilu: M = L U of the factors f; else M = T T, T the lower
    // triangle (with diagonal) of the matrix values f
    pict_status_t apply(const T* f, const T* in, T* y, T* out, bool tr, bool ilu) {
        pict_status_t s;
        if (!ilu) {
            if (!tr) {
                s = trsv<true, false, false>(f, in, y);  // T y = in
                if (s) return s;
                return trsv<true, false, false>(f, y, out);  // T out = y
            }
            s = trsv<false, false, true>(f, in, y);  // T^T y = in
            if (s) return s;
            return trsv<false, false, true>(f, y, out);  // T^T out = y
        }
        if (!tr) {
            s = trsv<true, true, false>(f, in, y);  // L y = in
            if (s) return s;
            return trsv<false, false, false>(f, y, out);  // U out = y
        }
        s = trsv<true, false, true>(f, in, y);  // U^T y = in
        if (s) return s;
        return trsv<false, true, true>(f, y, out);  // L^T out = y
    }

    pict_status_t spmv(const T* a, const T* x, T* y, bool tr) {
        const int g = cell_grid(P.n, ILU_THREADS);
        if (tr) k_csr_spmv<T, true><<<g, ILU_THREADS, 0, st>>>(P.n, P.row, P.index, P.tpos, a, x, y);
        else k_csr_spmv<T, false><<<g, ILU_THREADS, 0, st>>>(P.n, P.row, P.index, P.tpos, a, x, y);
        return check_launch("ilu spmv");
    }
};

template <typename T>
static pict_status_t ilu_factor(const IluPlan& P, const T* a, T* f, cudaStream_t st) {
    if (cudaMemcpyAsync(f, a, sizeof(T) * P.nnz, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return check_launch("ilu copy");
    for (int l = 0; l < P.nlf; ++l) {
        const int b = P.ptr_f[l], c = P.ptr_f[l + 1] - P.ptr_f[l];
        k_ilu_level<T><<<(c + ILU_THREADS - 1) / ILU_THREADS, ILU_THREADS, 0, st>>>(P.row, P.index, P.diag, f,
                                                                                  P.order_f, b, c);
    }
    return check_launch("ilu factorisation");
}

template <typename T>
static pict_status_t run_bicgstab_ilu(const IluPlan& P, const T* aval, const T* rhs, T* x, int nrhs, int maxit,
                                      double tol, int conv, int x_zero, int tr, int kind,
                                      pict_solve_info_t* info_host, char* ws, cudaStream_t st) {
    const size_t vb = (((size_t)P.n * sizeof(T)) + 255) & ~(size_t)255;
    char* o = ws;
    T* f = reinterpret_cast<T*>(o);
    o += (((size_t)P.nnz * sizeof(T)) + 255) & ~(size_t)255;
    T *r = (T*)o, *rw = (T*)(o + vb), *p = (T*)(o + 2 * vb), *pw = (T*)(o + 3 * vb), *v = (T*)(o + 4 * vb),
      *s = (T*)(o + 5 * vb), *t = (T*)(o + 6 * vb), *y = (T*)(o + 7 * vb);
    o += 8 * vb;
    double* part = reinterpret_cast<double*>(o);
    double* scal = part + ILU_RED_BLOCKS;
    const bool ilu = kind == PICT_PRECOND_ILU0;
    pict_status_t st_ = PICT_OK;
    if (ilu) {
        if ((st_ = ilu_factor<T>(P, aval, f, st))) return st_;
    } else {
        f = const_cast<T*>(aval);  // the sweeps read the matrix values themselves
    }
    IluSolver<T> S{P, st, part, scal};
    const int n = P.n;
    const int g = cell_grid(n, ILU_THREADS);
    for (int c = 0; c < nrhs; ++c) {
        const T* b = rhs + (size_t)c * n;
        T* xc = x + (size_t)c * n;
        pict_solve_info_t inf;
        inf.final_residual = 0.0;
        inf.used_iterations = -1;
        inf.converged = 0;
        inf.finite = 1;
        inf.status = 0;
        if (x_zero) cudaMemsetAsync(xc, 0, sizeof(T) * n, st);
        cudaMemsetAsync(v, 0, sizeof(T) * n, st);
        // r = b - A x
        if ((st_ = S.spmv(aval, xc, r, tr))) return st_;
        k_axpby<T><<<g, ILU_THREADS, 0, st>>>(n, T(1), b, T(-1), r);
        cudaMemcpyAsync(rw, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(p, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
        double nrm = 0.0;
        if ((st_ = S.crit(r, conv, &nrm))) return st_;
        if (nrm < tol) {
            inf.converged = 1;
            inf.used_iterations = -1;
            inf.final_residual = nrm;
            info_host[c] = inf;
            continue;
        }
        double rho = 0.0, rhop, alpha = 0.0, omega = 0.0, tmp, tmp2;
        for (int i = 0; i < maxit; ++i) {
            rhop = rho;
            if ((st_ = S.reduce(0, rw, r, &rho))) return st_;
            if (i > 0) {
                const double beta = (rho / rhop) * (alpha / omega);
                k_bicg_dir<T><<<g, ILU_THREADS, 0, st>>>(n, r, (T)beta, (T)omega, v, p);
            }
            if ((st_ = S.apply(f, p, y, pw, tr, ilu))) return st_;
            if ((st_ = S.spmv(aval, pw, v, tr))) return st_;
            if ((st_ = S.reduce(0, rw, v, &tmp))) return st_;
            alpha = rho / tmp;
            k_axpby<T><<<g, ILU_THREADS, 0, st>>>(n, (T)(-alpha), v, T(1), r);
            k_axpby<T><<<g, ILU_THREADS, 0, st>>>(n, (T)alpha, pw, T(1), xc);
            if ((st_ = S.crit(r, conv, &nrm))) return st_;
            if (!std::isfinite(nrm)) {
                inf.converged = 0;
                inf.used_iterations = i;
                inf.final_residual = nrm;
                inf.finite = 0;
                break;
            }
            inf.used_iterations = i;
            inf.final_residual = nrm;
            if (nrm < tol) {
                inf.converged = 1;
                break;
            }
            if ((st_ = S.apply(f, r, y, s, tr, ilu))) return st_;
            if ((st_ = S.spmv(aval, s, t, tr))) return st_;
            if ((st_ = S.reduce(0, t, r, &tmp))) return st_;
            if ((st_ = S.reduce(0, t, t, &tmp2))) return st_;
            omega = tmp / tmp2;
            k_axpby<T><<<g, ILU_THREADS, 0, st>>>(n, (T)omega, s, T(1), xc);
            k_axpby<T><<<g, ILU_THREADS, 0, st>>>(n, (T)(-omega), t, T(1), r);
            if ((st_ = S.crit(r, conv, &nrm))) return st_;
            inf.final_residual = nrm;
            if (nrm < tol) {
                inf.converged = 1;
                inf.used_iterations = i + 1;
                break;
            }
        }
        info_host[c] = inf;
    }
    return check_launch("bicgstab ilu");
}

}  // namespace pict

using namespace pict;

extern "C" {

// Host analysis of a CSR pattern (rows sorted by column, structurally symmetric): diagonal positions,
// positions of the transposed entries, and the rows grouped by forward / backward dependency level.
// order_f / order_b [n]: rows by level; ptr_f / ptr_b [n + 1]: level starts.  Returns the level counts.
pict_status_t pict_ilu_analyze(int32_t n, const int32_t* row, const int32_t* index, int32_t* diag, int32_t* tpos,
                               int32_t* order_f, int32_t* ptr_f, int32_t* order_b, int32_t* ptr_b, int32_t* nlev_f,
                               int32_t* nlev_b) {
    if (n <= 0 || !row || !index || !diag || !tpos || !order_f || !ptr_f || !order_b || !ptr_b || !nlev_f || !nlev_b)
        return set_error(PICT_ERR_ARG, "ilu_analyze: invalid argument");
    std::vector<int> lf(n, 0), lb(n, 0);
    for (int i = 0; i < n; ++i) {
        diag[i] = -1;
        for (int k = row[i]; k < row[i + 1]; ++k) {
            const int j = index[k];
            if (j < 0 || j >= n) return set_error(PICT_ERR_ARG, "ilu_analyze: column out of range");
            if (k > row[i] && index[k - 1] >= j) return set_error(PICT_ERR_ARG, "ilu_analyze: rows must be sorted by column");
            if (j == i) diag[i] = k;
            // transposed entry (j, i)
            int tk = -1;
            for (int m = row[j]; m < row[j + 1]; ++m)
                if (index[m] == i) { tk = m; break; }
            if (tk < 0) return set_error(PICT_ERR_ARG, "ilu_analyze: pattern not structurally symmetric");
            tpos[k] = tk;
        }
        if (diag[i] < 0) return set_error(PICT_ERR_ARG, "ilu_analyze: missing diagonal entry");
    }
    int mf = 0, mb = 0;
    for (int i = 0; i < n; ++i) {
        int l = 0;
        for (int k = row[i]; k < row[i + 1] && index[k] < i; ++k) l = lf[index[k]] + 1 > l ? lf[index[k]] + 1 : l;
        lf[i] = l;
        mf = l + 1 > mf ? l + 1 : mf;
    }
    for (int i = n - 1; i >= 0; --i) {
        int l = 0;
        for (int k = row[i]; k < row[i + 1]; ++k)
            if (index[k] > i) l = lb[index[k]] + 1 > l ? lb[index[k]] + 1 : l;
        lb[i] = l;
        mb = l + 1 > mb ? l + 1 : mb;
    }
    auto group = [n](const std::vector<int>& lev, int m, int32_t* order, int32_t* ptr) {
        std::vector<int> cnt(m + 1, 0);
        for (int i = 0; i < n; ++i) ++cnt[lev[i] + 1];
        for (int l = 0; l < m; ++l) cnt[l + 1] += cnt[l];
        for (int l = 0; l <= m; ++l) ptr[l] = cnt[l];
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        for (int i = 0; i < n; ++i) order[pos[lev[i]]++] = i;
    };
    group(lf, mf, order_f, ptr_f);
    group(lb, mb, order_b, ptr_b);
    *nlev_f = mf;
    *nlev_b = mb;
    return PICT_OK;
}

int64_t pict_bicgstab_ilu_workspace_bytes(int32_t n, int32_t nnz, int32_t dtype) {
    const size_t esz = dtype == PICT_F64 ? 8 : 4;
    const size_t vb = ((size_t)n * esz + 255) & ~(size_t)255;
    return (int64_t)((((size_t)nnz * esz) + 255 & ~(size_t)255) + 8 * vb + 8 * (ILU_RED_BLOCKS + 8));
}

// ILU(0) factors of the CSR values `a` into `f` (same pattern), level by level.
pict_status_t pict_ilu0_factor(int32_t n, int32_t nnz, int32_t dtype, const int32_t* row, const int32_t* index,
                               const int32_t* diag, const int32_t* order_f, const int32_t* ptr_f_host, int32_t nlev_f,
                               const void* a, void* f, void* stream) {
    if (n <= 0 || !row || !index || !diag || !order_f || !ptr_f_host || !a || !f)
        return set_error(PICT_ERR_ARG, "ilu0_factor: invalid argument");
    IluPlan P;
    P.n = n;
    P.nnz = nnz;
    P.nlf = nlev_f;
    P.nlb = 0;
    P.row = row;
    P.index = index;
    P.diag = diag;
    P.tpos = nullptr;
    P.order_f = order_f;
    P.ptr_f.assign(ptr_f_host, ptr_f_host + nlev_f + 1);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == PICT_F64) return ilu_factor<double>(P, (const double*)a, (double*)f, st);
    return ilu_factor<float>(P, (const float*)a, (float*)f, st);
}

// BiCGStab with a right preconditioner (PICT_PRECOND_*) on the CSR matrix (row, index, aval) of a single-system
// domain; rhs, x: [nrhs][n] (device); info_host: [nrhs] (host).  Synchronises the stream per reduction.
pict_status_t pict_bicgstab_ilu(int32_t n, int32_t nnz, int32_t dtype, const int32_t* row, const int32_t* index,
                                const int32_t* diag, const int32_t* tpos, const int32_t* order_f,
                                const int32_t* ptr_f_host, int32_t nlev_f, const int32_t* order_b,
                                const int32_t* ptr_b_host, int32_t nlev_b, const void* aval, const void* rhs, void* x,
                                int32_t nrhs, int32_t max_iterations, double tolerance, int32_t convergence,
                                int32_t x_is_zero, int32_t transpose, int32_t preconditioner, void* info_host,
                                void* workspace, int64_t workspace_bytes, void* stream) {
    if (n <= 0 || !row || !index || !diag || !tpos || !order_f || !ptr_f_host || !order_b || !ptr_b_host || !aval ||
        !rhs || !x || !info_host || !workspace || nrhs < 1)
        return set_error(PICT_ERR_ARG, "bicgstab_ilu: invalid argument");
    if (workspace_bytes < pict_bicgstab_ilu_workspace_bytes(n, nnz, dtype))
        return set_error(PICT_ERR_ARG, "bicgstab_ilu: workspace too small");
    if (convergence < PICT_CONV_NORM2 || convergence > PICT_CONV_ABS_MAX)
        return set_error(PICT_ERR_ARG, "bicgstab_ilu: unknown convergence criterion");
    if (preconditioner != PICT_PRECOND_AS_REFERENCE && preconditioner != PICT_PRECOND_ILU0)
        return set_error(PICT_ERR_ARG, "bicgstab_ilu: unknown preconditioner");
    IluPlan P;
    P.n = n;
    P.nnz = nnz;
    P.nlf = nlev_f;
    P.nlb = nlev_b;
    P.row = row;
    P.index = index;
    P.diag = diag;
    P.tpos = tpos;
    P.order_f = order_f;
    P.order_b = order_b;
    P.ptr_f.assign(ptr_f_host, ptr_f_host + nlev_f + 1);
    P.ptr_b.assign(ptr_b_host, ptr_b_host + nlev_b + 1);
    cudaStream_t st = (cudaStream_t)stream;
    pict_solve_info_t* info = reinterpret_cast<pict_solve_info_t*>(info_host);
    char* ws = reinterpret_cast<char*>(workspace);
    if (dtype == PICT_F64)
        return run_bicgstab_ilu<double>(P, (const double*)aval, (const double*)rhs, (double*)x, nrhs, max_iterations,
                                        tolerance, convergence, x_is_zero, transpose, preconditioner, info, ws, st);
    return run_bicgstab_ilu<float>(P, (const float*)aval, (const float*)rhs, (float*)x, nrhs, max_iterations, tolerance,
                                   convergence, x_is_zero, transpose, preconditioner, info, ws, st);
}

}  // extern "C"
