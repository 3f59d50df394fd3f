// launch.h -- host-side launch helpers and error reporting for libpict_b200.
#pragma once

#include <cuda_runtime.h>
#include "pict_b200.h"

namespace pict {

// Records the last error message (thread local) and returns the code.
pict_status_t set_error(pict_status_t code, const char* msg);
// cudaGetLastError after a launch -> PICT_ERR_CUDA with the kernel name.
pict_status_t check_launch(const char* what);
// Number of SMs of the current device (cached per device).
int device_sm_count();
// grid for a grid-stride per-cell kernel: enough CTAs to cover N, capped at a few waves
int cell_grid(int n, int threads);
// grid for a kernel that walks a domain's cells with for_each_cell (common.cuh): one CTA per chunk of
// `threads` cells of a work tile when the domain carries tiles, capped like cell_grid
int domain_grid(const pict_domain_t* dom, int threads);
// Non-orthogonal terms (nonortho.cu), added after the orthogonal kernel of an operator:
// what 0 advection matrix (C, A), 1 velocity RHS, 2 pressure matrix, 3 pressure RHS divergence.
// Returns PICT_OK without launching when `flags` selects no term of that operator.
pict_status_t nonortho_pass(const pict_domain_t* dom, int32_t flags, int32_t what, void* stream);
// The same with a passive scalar channel: what 4 scalar matrix of channel `ch` (C, A), 5 scalar RHS
// (all channels).
pict_status_t nonortho_pass_ch(const pict_domain_t* dom, int32_t flags, int32_t what, int32_t ch, void* stream);
// Gradients of the non-orthogonal passive scalar terms: what 4 matrix of channel `ch` (out_bar = C_bar
// [K][N], A_bar [N] -> coef_bar += scalar viscosity adjoint per cell [N]), 5 RHS (out_bar = scalarRHS_bar
// [C][N] -> data_bar += scalarResult adjoint [C][N], coef_bar += [C][N], sb_bar += boundary scalar
// adjoint [2D][C][N] per adjacent cell).
pict_status_t nonortho_grad_scalar(const pict_domain_t* dom, int32_t flags, int32_t what, int32_t ch, const void* out_bar,
                                   const void* A_bar, void* data_bar, void* coef_bar, void* sb_bar, void* stream);

}  // namespace pict
