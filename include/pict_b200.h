/*
 * pict_b200.h -- C ABI of the B200-native PISO step (libpict_b200.so).
 *
 * This is the drop-in boundary of the build: plain C structs, raw device
 * pointers and sizes, no torch types.  The Python package ``pict_b200``
 * (module ``pict_b200.PISOtorch``) binds these entry points with ctypes and
 * mirrors the reference's pybind11 ``PISOtorch`` operator surface on top of
 * them.  Each entry point below cites the reference interface it replaces
 * (file:line, paths relative to the PICT repository).
 *
 * Conventions
 *  - Every compute entry point is stream-ordered on the given stream, performs
 *    no host synchronisation and no device allocation, and returns a
 *    pict_status_t (PICT_OK == 0).  The last error message is available from
 *    pict_last_error().
 *  - Scalars use the domain dtype (PICT_F32 or PICT_F64); the Krylov inner
 *    products, norms and convergence tests are always accumulated in FP64.
 *  - Faces are indexed [-x,+x,-y,+y,-z,+z] = 0..5; axis = face>>1,
 *    upper = face&1.  Cells are flattened x-fastest per block; global vectors
 *    concatenate the blocks; vector fields are component-major [D][N].
 *  - System matrices are structured stencils: coef[K][N], K = 2D+1, in the
 *    order [diag,-x,+x,-y,+y,-z,+z]; faces on fixed boundaries hold 0.
 *  - A "system" (sim) is an independent simulation inside a batched domain;
 *    blocks of one system are contiguous and systems never connect.
 */
#ifndef PICT_B200_H
#define PICT_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t pict_status_t;
#define PICT_OK 0
#define PICT_ERR_ARG 1        /* invalid argument or size */
#define PICT_ERR_CUDA 2       /* CUDA launch/runtime error */
#define PICT_ERR_UNSUPPORTED 3
#define PICT_ERR_NO_DEVICE 4

#define PICT_F32 0
#define PICT_F64 1

#define PICT_FACE_FIXED 0
#define PICT_FACE_PERIODIC 1
#define PICT_FACE_CONNECTED 2

#define PICT_MAX_BLOCK_FACES 6

/* One block face (BoundaryGPU, extensions/domain_structs_gpu.h:253-263). */
typedef struct pict_face {
    int32_t type;          /* PICT_FACE_* */
    int32_t conn_block;    /* connected: index of the other block */
    int32_t conn_axes[3];  /* connected: ConnectedBoundary::axes (extensions/domain_structs.h:329-338) */
    int32_t vel_static;    /* fixed: 1 if velocity is a static [D] vector */
    const void* velocity;  /* fixed: boundary velocity [D] or [D][face cells] (device) */
    const void* transform; /* fixed: boundary transform [face cells][2D^2+1] or NULL */
    void* velocity_grad;   /* fixed: gradient of velocity (adjoint), same layout, or NULL */
    int32_t scalar_static;   /* fixed: 1 if the passive scalar is a static [C] vector */
    uint32_t scalar_neumann; /* fixed: bit c set = passive scalar channel c is a Neumann (gradient) boundary */
    const void* scalar;      /* fixed: passive scalar [C] or [C][face cells], or NULL */
    void* scalar_grad;       /* fixed: gradient of the passive scalar, same layout, or NULL */
} pict_face_t;

/* One structured block (BlockGPU, extensions/domain_structs_gpu.h:266-305). */
typedef struct pict_block {
    int32_t size[3];          /* x, y, z cells (1 for unused axes) */
    int32_t offset;           /* first global cell index of this block */
    int32_t sim;              /* system index */
    int32_t viscosity_static; /* 1: viscosity is [1], 0: [cells] */
    int32_t source_static;    /* 1: source is [D], 0: [D][cells] */
    int32_t pad0;
    void* velocity;           /* [D][cells] block velocity u^n (device) */
    void* pressure;           /* [cells] block pressure (device) */
    const void* transform;    /* [cells][2D^2+1] (M, Minv, det) or NULL */
    const void* viscosity;    /* NULL (use system viscosity), [1] or [cells] */
    const void* source;       /* NULL, [D] or [D][cells] velocity source */
    void* velocity_grad;      /* adjoint of velocity or NULL */
    void* pressure_grad;      /* adjoint of pressure or NULL */
    void* viscosity_grad;     /* adjoint of block viscosity or NULL */
    void* source_grad;        /* adjoint of velocity source or NULL */
    pict_face_t face[PICT_MAX_BLOCK_FACES];
    const void* face_transform; /* [D][(z+1)][y+1][x+1][2D^2+1] staggered face transforms or NULL
                                   (Block::faceTransform; read by the FVM velocity corrector, version 6) */
    void* scalar;             /* [C][cells] passive scalar of the block, or NULL */
    void* scalar_grad;        /* adjoint of the passive scalar, or NULL */
} pict_block_t;

/* A (possibly batched) domain.  All pointers are device pointers unless noted.
 * Mirrors DomainGPU (extensions/domain_structs_gpu.h:307-370) with stencil storage. */
typedef struct pict_domain {
    int32_t dims;
    int32_t num_blocks;
    int32_t num_cells;        /* N, all systems */
    int32_t num_sims;
    int32_t dtype;            /* PICT_F32 / PICT_F64 */
    int32_t max_sim_cells;    /* host hint: largest system */
    const pict_block_t* blocks;    /* [num_blocks] block table (device copy) */
    const int32_t* nbr;            /* [2D][N] neighbour cell across each face, -1 on fixed faces */
    const int32_t* cell_block;     /* [N] block index of each cell */
    const int32_t* sim_cells;      /* [num_sims+1] cell range of each system */
    const int32_t* sim_blocks;     /* [num_sims+1] block range of each system */
    const int32_t* tiles;          /* [num_tiles][4] Krylov work tiles: system, block, first cell, cell count */
    const int32_t* sim_tiles;      /* [num_sims+1] tile range of each system */
    int32_t num_tiles;
    int32_t tile_cells;            /* upper bound of cells per tile */
    const void* sim_viscosity;     /* [num_sims] domain viscosity per system */
    const void* sim_dt;            /* [num_sims] time step per system, or NULL (use the scalar argument) */
    void* C;                  /* [K][N] advection matrix */
    void* A;                  /* [N] its diagonal */
    void* P;                  /* [K][N] pressure matrix */
    void* velocity_rhs;       /* [D][N] */
    void* velocity_result;    /* [D][N] */
    void* pressure_rhs;       /* [D][N] (H/A vector field) */
    void* pressure_rhs_div;   /* [N] */
    void* pressure_result;    /* [N] */
    int32_t scalar_channels;        /* passive scalar channels C (0: none) */
    int32_t scalar_viscosity_static; /* 1: scalar_viscosity is [1], 0: [C] */
    const void* scalar_viscosity;   /* NULL (use the domain viscosity), [1] or [C] */
    void* scalar_rhs;               /* [C][N] */
    void* scalar_result;            /* [C][N] */
} pict_domain_t;

/* Per right-hand-side solver report (LinearSolverResultInfo, extensions/bicgstab_solver.h:20-25). */
typedef struct pict_solve_info {
    double final_residual;
    int32_t used_iterations;
    int32_t converged;
    int32_t finite;
    int32_t status;           /* 0 ok, 1 barrier timeout, 2 not started */
} pict_solve_info_t;

#define PICT_CONV_NORM2 0
#define PICT_CONV_NORM2_NORMALIZED 1
#define PICT_CONV_ABS_SUM 2
#define PICT_CONV_ABS_MEAN 3
#define PICT_CONV_ABS_MAX 4

/* Parameters of a linear solve (PISOtorch.SolveLinear arguments, extensions/PISOtorch.cpp:559-563). */
typedef struct pict_solve_params {
    int32_t max_iterations;
    int32_t use_bicg;          /* 1: BiCGStab, 0: CG */
    int32_t nrhs;              /* right-hand sides per system sharing the matrix (BiCG: D components) */
    int32_t x_is_zero;         /* 1: skip the initial A*x (x must hold zeros) */
    int32_t transpose;         /* solve with A^T (adjoint solves) */
    int32_t convergence;       /* PICT_CONV_* (ComputeConvergenceCriterion, extensions/cg_solver_kernel.cu:77-110);
                                  the ABS criteria with CG only (classic order) */
    int32_t group_size;        /* upper bound of CTAs of the persistent launch (0: automatic) */
    int32_t threads;           /* threads per CTA (0: automatic) */
    int32_t subtract_mean;     /* 1: x -= mean(x) per system after the solve (PISOtorch_simulation.py:1243-1244) */
    int32_t write_block_pressure; /* 1: also copy x into the blocks' pressure (CopyPressureResultToBlocks) */
    int32_t variant;           /* CG only: 0 classic order (extensions/cg_solver_kernel.cu:236-427, two reductions per iteration),
                                  1 single-reduction recurrence (Chronopoulos-Gear): same iterates in exact
                                  arithmetic, one grid-wide reduction per iteration */
    int32_t residual_reset_steps; /* CG only: > 0 restarts the iteration (r = b - A x, p = r) before every
                                     iteration i with (i+1) % residual_reset_steps == 0, as residualResetSteps
                                     of extensions/cg_solver_kernel.cu:266-286; runs the classic order (variant 0) */
    int32_t return_best_result;   /* CG only: keep the iterate with the lowest criterion and return it when the
                                     solve stops unconverged (at max_iterations, or after 100 iterations of a
                                     non-falling criterion), reporting its iteration and criterion
                                     (returnBestResult, extensions/cg_solver_kernel.cu:330-413); classic order */
    int32_t rank_deficient;       /* CG only: iterate with the reference's rank-deficient operator A v + s |v|_1 e,
                                     s = sum |diag A| / n^3 per system, and initial residual b - A x + s |x|_1 e
                                     (matrixRankDeficient, extensions/cg_solver_kernel.cu:240-298); classic order */
    double tolerance;
} pict_solve_params_t;

/* ---------------- version / library ---------------- */
const char* pict_version(void);
const char* pict_last_error(void);
int32_t pict_sizeof_block(void);   /* sizeof(pict_block_t), for binding checks */
int32_t pict_sizeof_domain(void);  /* sizeof(pict_domain_t) */

/* ---------------- host-side topology (no GPU needed) ----------------
 * Replaces the per-thread neighbour resolution of the reference
 * (resolveNeighborCell / computeConnectedPos, extensions/PISO_multiblock_cuda_kernel.cu:326-345, 432-477) and
 * the connection checks of Domain::PrepareSolve (extensions/domain_structs.cpp:2554-2676)
 * with a precomputed table.  host_blocks is a HOST array.
 * nbr_out: [2*dims][num_cells], cell_block_out: [num_cells] (host buffers). */
pict_status_t pict_build_topology(const pict_block_t* host_blocks, int32_t num_blocks, int32_t dims,
                                  int32_t num_cells, int32_t* nbr_out, int32_t* cell_block_out);

/* Work tiles for the Krylov kernels: every block is cut into contiguous runs of at most
 * tile_cells cells; tiles of one system are contiguous.  tiles_out: [max_tiles][4] (system, block,
 * first global cell, count), sim_tiles_out: [num_sims+1].  *num_tiles_out receives the count
 * (also when max_tiles is too small, then PICT_ERR_ARG is returned).  Host buffers. */
pict_status_t pict_build_tiles(const pict_block_t* host_blocks, int32_t num_blocks, int32_t num_sims,
                               int32_t tile_cells, int32_t* tiles_out, int32_t max_tiles, int32_t* sim_tiles_out,
                               int32_t* num_tiles_out);

/* ---------------- assembly (forward) ----------------
 * non_ortho_flags: the reference's nonOrthoFlags bits (extensions/PISO_multiblock_cuda.h:9-13): 1 direct
 * matrix terms, 2 direct RHS terms, 8 diagonal RHS terms, 16 centre matrix terms (4 has no effect, as in
 * the reference).  The matrix bits add the tangential-flux terms to C / A and P, the RHS bits add the
 * explicit terms of the current velocityResult to the velocity RHS and of the current pressureResult
 * to the pressure RHS divergence (extensions/PISO_multiblock_cuda_kernel.cu:1911-1987, 2742-2860, 3033-3187). */
/* SetupAdvectionMatrix (extensions/PISOtorch.cpp:531-533 -> extensions/PISO_multiblock_cuda_kernel.cu:4510 PISO_build_matrix):
 * writes C and A from the blocks' velocity. */
pict_status_t pict_setup_advection_matrix(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                          void* stream);
/* SetupAdvectionVelocity (extensions/PISOtorch.cpp:537-539 -> extensions/PISO_multiblock_cuda_kernel.cu:4677 kPISO_build_advection_RHS). */
pict_status_t pict_setup_advection_velocity(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                            int32_t apply_pressure_gradient, void* stream);
/* Fused SetupAdvectionMatrix + SetupAdvectionVelocity in one pass over the cells. */
pict_status_t pict_setup_advection(const pict_domain_t* dom, double dt, void* stream);
/* SetupPressureMatrix (extensions/PISOtorch.cpp:544-546 -> extensions/PISO_multiblock_cuda_kernel.cu:4797 PISO_build_pressure_matrix). */
pict_status_t pict_setup_pressure_matrix(const pict_domain_t* dom, int32_t non_ortho_flags, void* stream);
/* SetupPressureRHS (extensions/PISOtorch.cpp:547-549 -> extensions/PISO_multiblock_cuda_kernel.cu:5121 PISO_build_pressure_rhs
 * + extensions/PISO_multiblock_cuda_kernel.cu:5374 k_computePressureRHSdivergenceFromFlux). */
pict_status_t pict_setup_pressure_rhs(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                      int32_t time_step_norm, void* stream);
/* SetupPressureRHSdiv (extensions/PISOtorch.cpp:550-552 -> extensions/PISO_multiblock_cuda_kernel.cu:5374). */
pict_status_t pict_setup_pressure_rhs_div(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                          int32_t time_step_norm, void* stream);
/* SetupPressureCorrection (extensions/PISOtorch.cpp:541-543): matrix + RHS + div, matrix and RHS fused. */
pict_status_t pict_setup_pressure_correction(const pict_domain_t* dom, double dt, int32_t non_ortho_flags,
                                             int32_t time_step_norm, void* stream);
/* CorrectVelocity (extensions/PISOtorch.cpp:553-555 -> extensions/PISO_multiblock_cuda_kernel.cu:6163-6201): version 0/1
 * finite-difference pressure gradient (PISO_update_velocity :5947-5980), 4 mean of the two face fluxes with
 * orthogonal metrics (PISO_update_velocity_v4_orthogonal :6053-6160), 5 / 6 finite-volume pressure gradient
 * with interpolated cell fluxes / staggered face transforms (PISO_update_velocity_PressureFVM :6013-6050,
 * getPressureGradientFVM :991-1123).  write_block_velocity=1 additionally stores the result in the
 * blocks' velocity (CopyVelocityResultToBlocks fused). */
pict_status_t pict_correct_velocity(const pict_domain_t* dom, double dt, int32_t version,
                                    int32_t time_step_norm, int32_t write_block_velocity, void* stream);
/* Copy{Velocity,Pressure}Result{To,From}Blocks (extensions/PISOtorch.cpp:561-566 -> extensions/PISO_multiblock_cuda_kernel.cu:6543-6733). */
pict_status_t pict_copy_velocity_result_to_blocks(const pict_domain_t* dom, void* stream);
pict_status_t pict_copy_velocity_result_from_blocks(const pict_domain_t* dom, void* stream);
/* Initial guess of the advection solve (no counterpart in the reference, whose driver can start the solve from
 * the previous result, PISOtorch_simulation.py advect_use_prev_result): after_solve = 0 sets
 * velocityResult = block velocity + increment; after_solve = 1 stores increment = velocityResult - block
 * velocity (the step's advection increment, the next step's guess).  increment: [D][N], zero on the first step. */
pict_status_t pict_advection_guess(const pict_domain_t* dom, void* increment, int32_t after_solve, void* stream);
pict_status_t pict_copy_pressure_result_to_blocks(const pict_domain_t* dom, void* stream);
pict_status_t pict_copy_pressure_result_from_blocks(const pict_domain_t* dom, void* stream);
/* ComputeVelocityDivergence (extensions/PISOtorch.cpp:556 -> extensions/PISO_multiblock_cuda_kernel.cu:6333): div of the blocks' velocity, out [N]. */
pict_status_t pict_velocity_divergence(const pict_domain_t* dom, void* out, void* stream);

/* ---------------- linear solves ---------------- */
/* Bytes of scratch memory a solve needs (vectors, reduction partials, barriers). */
int64_t pict_solve_workspace_bytes(const pict_domain_t* dom, const pict_solve_params_t* params);
/* SolveLinear (extensions/PISOtorch.cpp:559-563 -> extensions/PISO_multiblock_cuda_kernel.cu:7070 -> cgSolveGPU extensions/cg_solver_kernel.cu:114 / bicgstabSolveGPU extensions/bicgstab_solver_kernel.cu:47)
 * on a stencil matrix coef [K][N] of the domain's topology.  rhs, x: [nrhs][N].
 * info_out: device array [num_sims][nrhs] of pict_solve_info_t.  workspace: device memory of
 * pict_solve_workspace_bytes() bytes. */
pict_status_t pict_solve(const pict_domain_t* dom, const void* coef, const void* rhs, void* x,
                         const pict_solve_params_t* params, void* info_out, void* workspace,
                         int64_t workspace_bytes, void* stream);

/* Process-wide choice of the launch form of the single-reduction CG (variant 1; no counterpart in the
 * reference): 1 (default) solves each system with one thread-block cluster (16 CTAs, else 8) when a
 * domain holds few systems (at most 8) of at most 262,144 cells, reducing the inner products through
 * distributed shared memory with one cluster barrier per iteration and no grid-wide barrier; 0 always
 * uses the persistent grid; 2 uses clusters whenever they fit. */
void pict_krylov_set_cluster_mode(int32_t mode);
/* BiCGStab kernel (no counterpart in the reference): 0 (default) four grid barriers per iteration for every
 * solve; 1 two barriers per iteration (NORM2 / NORM2_NORMALIZED criteria, up to two right-hand sides per launch;
 * the half step forms s on the fly, the full step forms the next search direction on the fly with rho' from the
 * recurrence rw.r - alpha rw.v - omega rw.t) with one CTA per SM, 2 the same with two CTAs per SM.  All follow
 * bicgstabSolveGPU's iteration and reports.  Variants 1 and 2 take one more workspace vector per right-hand side
 * (pict_solve_workspace_bytes follows the current choice). */
void pict_krylov_set_bicgstab_variant(int32_t variant);

/* pict_solve without a caller-provided workspace (no counterpart in the reference).  For callers
 * that hold no device allocator (a plain C or ctypes binding without torch, or a loop that must not
 * call cudaMalloc, which synchronises the device).  The workspace is a fixed scratch array of
 * pict_solve_static_scratch_bytes() bytes (8 MiB) in the library's own device memory; the call
 * allocates nothing.  Solves whose pict_solve_workspace_bytes() exceeds it are rejected with
 * PICT_ERR_ARG; compare the two functions to know beforehand.  The workspace holds 4 vectors of the
 * system size for CG (5 with return_best_result), 7 for the single-reduction CG (variant 1) and 7
 * per right-hand side of a launch for BiCGStab: in FP32 about 520k, 290k and, for a 2D velocity
 * solve, 150k cells.  Every call looks up the scratch address in the current CUDA context (the
 * address is per context); the first call in a context loads the library's device code, so make
 * it before any stream capture.  All calls on a device share the one scratch: calls that overlap
 * in time (two streams, two host threads) race and must be serialised by the caller.  Nothing in
 * the scratch has to start at zero; the barrier words are cleared by every call.  The array is
 * part of the library's device code: every device that loads the library holds its 8 MiB until
 * the process exits, whether or not this function is called. */
int64_t pict_solve_static_scratch_bytes(void);
pict_status_t pict_solve_static(const pict_domain_t* dom, const void* coef, const void* rhs, void* x,
                                const pict_solve_params_t* params, void* info_out, void* stream);

/* ---------------- mixed precision: FP64 iterative refinement of a solve ----------------
 * No counterpart in the reference, which solves once in the domain dtype (cgSolveGPU,
 * extensions/cg_solver_kernel.cu:114-456).  x64: FP64 accumulator [N] of the solution.
 * pict_refine_residual: residual = rhs - coef*x in FP64 arithmetic (stored in the domain dtype); x is
 *   x_init when non-NULL (and x64 is set to it), else x64.  project_mean=1 removes the per-system mean
 *   of the residual (the unsolvable constant mode of a singular pressure system; needs tile_scratch of
 *   num_tiles doubles).
 * pict_refine_update: x64 += correction.
 * pict_refine_finish: x = x64 (minus its per-system mean), optionally also into the blocks' pressure;
 *   tile_scratch: num_tiles doubles (needed with subtract_mean). */
pict_status_t pict_refine_residual(const pict_domain_t* dom, const void* coef, const void* rhs, const void* x_init,
                                   double* x64, void* residual, int32_t project_mean, double* tile_scratch,
                                   void* stream);
pict_status_t pict_refine_update(const pict_domain_t* dom, double* x64, const void* correction, void* stream);
/* out = alpha x + beta y over n values of `dtype` (out may alias x or y); the step's warm starts combine vectors
 * with it (no counterpart in the reference). */
pict_status_t pict_vector_axpby(int32_t n, int32_t dtype, double alpha, const void* x, double beta, const void* y,
                                void* out, void* stream);
pict_status_t pict_refine_finish(const pict_domain_t* dom, const double* x64, void* x, int32_t subtract_mean,
                                 int32_t write_block_pressure, double* tile_scratch, void* stream);

/* ---------------- multigrid-preconditioned CG (mixed-precision correction solves) ----------------
 * No counterpart in the reference.  For domains whose systems are single blocks with fixed or
 * periodic faces.  A level describes the cells of every block at one coarsening depth. */
typedef struct pict_mg_level {
    int32_t num_cells;
    int32_t num_blocks;
    int32_t dims;
    int32_t dtype;
    const int32_t* blocks;     /* [num_blocks][12]: first cell, size x, y, z, periodic x, y, z, system, coarsening
                                  shift x, y, z from the next finer level (0: kept, 1: halved), unused (device) */
    const int32_t* cell_block; /* [num_cells] block of each cell (device) */
    void* coef;                /* [2D+1][num_cells] stencil of the level (device) */
    int32_t num_tiles;         /* work tiles of the level (levels >= 1; level 0 runs on the domain's tiles) */
    int32_t max_block_cells;   /* cells of the largest block of the level */
    const int32_t* tiles;      /* [num_tiles][4]: system, block, first cell, cell count (device) */
    int32_t max_block_sx;      /* largest x size (cells per row) of a block of the level */
    int32_t sweeps;            /* damped-Jacobi sweeps of each smoothing step at this level when the restriction
                                  and prolongation tile kernels handle it: 2 where every tile's shared-memory
                                  stage holds two halo rows (2D, not y-periodic), else 1 (0 reads as 1) */
} pict_mg_level_t;

/* Process-wide choice of the 2D PCG SpMV kernel (no counterpart in the reference): 1 (default) stages
 * each work tile's operands in shared memory with asynchronous bulk copies (cp.async.bulk on an mbarrier,
 * double-buffered across the tiles of a persistent grid) wherever the operands are 16-byte aligned and
 * the stage fits; 0 runs the gather kernel only.  Both give the same per-warp partial sums. */
void pict_mg_set_bulk_staging(int32_t enable);
/* Process-wide cap on the smoothing sweeps of the V-cycle (no counterpart in the reference): 2 (default) two
 * damped-Jacobi sweeps before and after the coarse correction where a level allows it (pict_mg_level_t.sweeps)
 * and always inside the one-launch sub-cycle; 1 one sweep everywhere. */
void pict_mg_set_smoothing_sweeps(int32_t sweeps);
/* Process-wide choice (no counterpart in the reference): 1 (default) when pict_pcg_mg is called on a stream
 * under capture, the PCG iterations after the first are captured as the body (two iterations) of a conditional
 * WHILE node that ends once every system has met the tolerance or the cap is reached, so a replay launches only
 * the iterations the systems need; 0 captures the fixed sequence of `iterations` iterations. */
void pict_mg_set_graph_loop(int32_t enable);
/* Process-wide choice (no counterpart in the reference): 1 (default) the kernels of pict_pcg_mg are launched with
 * programmatic stream serialization (each one waits for its predecessor's writes at its first instruction and lets
 * the next one launch at once, so launch latency overlaps the predecessor's last CTAs); 0 plain launches. */
void pict_mg_set_dependent_launch(int32_t enable);
/* Galerkin coarse operator R A P of `fine` into coarse->coef (aggregates of 2^D cells). */
pict_status_t pict_mg_galerkin(const pict_mg_level_t* fine, const pict_mg_level_t* coarse, void* stream);
int64_t pict_pcg_mg_workspace_bytes(const pict_domain_t* dom, const pict_mg_level_t* levels, int32_t num_levels);
/* `iterations` preconditioned CG iterations on levels[0].coef x = rhs from x = 0, V-cycle with one or two
 * damped-Jacobi sweeps (omega) before and after the coarse correction, prolongation scaled by prolong_scale,
 * coarse_sweeps Jacobi sweeps on the coarsest
 * level; per-system report (final RMS / 2-norm residual of the recursion) in info_out[num_sims]. */
pict_status_t pict_pcg_mg(const pict_domain_t* dom, const pict_mg_level_t* levels, int32_t num_levels, const void* rhs,
                          void* x, int32_t iterations, double tolerance, int32_t convergence, void* info_out,
                          void* workspace, int64_t workspace_bytes, double omega, double prolong_scale,
                          int32_t coarse_sweeps, void* stream);

/* ---------------- adjoint (reverse mode) of the orthogonal step ----------------
 * Gather-form adjoints of the forward operators (no atomics, deterministic).  They read the forward
 * quantities from explicit global vectors (a per-step tape) and accumulate into global vectors:
 * velocity_grad [D][N] (velocity at the start of the step), viscosity_grad [N] (per cell),
 * source_grad [D][N] (NULL: not needed), boundary_velocity_grad [2D][D][N] (per fixed face and
 * adjacent cell).  pict_adjoint_to_blocks() maps them onto the blocks' gradient tensors.
 * Replace the *_GRAD kernels behind PISOtorch_diff (extensions/PISO_multiblock_cuda_kernel.cu:3869-4077,
 * 4388-4478, 4967-5117, 5243-5371, 5423-5453, 6224-6293). */

/* CorrectVelocityGrad (PISOtorch_diff.py:1160-1236, FD version): h_grad = u_grad,
 * A_grad += u_grad.g/A^2, pressure_grad = -G^T(u_grad/A) (pressure: [N], the corrector's solution). */
pict_status_t pict_correct_velocity_grad(const pict_domain_t* dom, const void* A, const void* pressure,
                                         const void* velocity_result_grad, void* A_grad, void* pressure_grad,
                                         void* pressure_rhs_grad, void* stream);
/* x -= mean(x) per system (adjoint of the pressure mean removal, PISOtorch_simulation.py:1286-1287). */
pict_status_t pict_sim_mean_project(const pict_domain_t* dom, void* x, void* stream);
/* SetupPressureRHSdiv gradient (PISOtorch_diff.py:1067-1158): pressure_rhs_grad += Dv^T div_grad,
 * boundary_velocity_grad += d div / d boundary velocity. */
pict_status_t pict_divergence_grad(const pict_domain_t* dom, const void* div_grad, void* pressure_rhs_grad,
                                   void* boundary_velocity_grad, void* stream);
/* SetupPressureRHS + SetupPressureMatrix gradients of one corrector (PISOtorch_diff.py:897-1065) with the
 * pressure solve's matrix gradient -lambda x^T folded in (lambda = P^-T x_grad, x = the solution):
 * A_grad +=, C_grad (off-diagonal rows) +=, U_grad = (gradient of the velocity used in H/A),
 * velocity_grad / source_grad / viscosity_grad / boundary_velocity_grad +=. */
pict_status_t pict_pressure_rhs_grad(const pict_domain_t* dom, double dt, const void* h_grad, const void* h,
                                     const void* A, const void* C, const void* U, const void* lambda,
                                     const void* pressure, void* A_grad, void* C_grad, void* U_grad,
                                     void* velocity_grad, void* source_grad, void* viscosity_grad,
                                     void* boundary_velocity_grad, void* stream);
/* SetupAdvectionMatrix + SetupAdvectionVelocity gradients (PISOtorch_diff.py:377-441, 531-613) with the
 * advection solve's matrix gradient -rhs_grad u*^T folded in (velocity_result: the solution u*). */
pict_status_t pict_advection_grad(const pict_domain_t* dom, double dt, const void* velocity_result,
                                  const void* velocity_rhs_grad, const void* C_grad, const void* A_grad,
                                  void* velocity_grad, void* viscosity_grad, void* boundary_velocity_grad,
                                  void* source_grad, void* stream);
/* Accumulators -> gradient tensors of the block table (velocity_grad, viscosity_grad, source_grad, faces'
 * velocity_grad; static tensors receive the sum) and sim_viscosity_grad [num_sims] for blocks that use
 * the system viscosity.  block_scratch: device memory of num_blocks doubles. */
pict_status_t pict_adjoint_to_blocks(const pict_domain_t* dom, const void* velocity_grad, const void* viscosity_grad,
                                     const void* source_grad, const void* boundary_velocity_grad,
                                     void* sim_viscosity_grad, void* block_scratch, void* stream);
/* SparseOuterProduct (extensions/PISOtorch.cpp:564) on the stencil pattern, summed over nrhs stacked
 * vectors: coef_out[0][i] += scale sum_c a_c[i] b_c[i], coef_out[f+1][i] += scale sum_c a_c[i] b_c[nbr(f,i)]
 * (the matrix gradient of a linear solve is -b_grad x^T, PISOtorch_diff.py:352-371). */
pict_status_t pict_stencil_outer_product(const pict_domain_t* dom, const void* a, const void* b, int32_t nrhs,
                                        void* coef_out, double scale, void* stream);
/* SetupPressureMatrixGrad (PISOtorch_diff.py:897-965): A_grad += d(P : P_grad)/dA. */
pict_status_t pict_pressure_matrix_grad(const pict_domain_t* dom, const void* A, const void* P_grad, void* A_grad,
                                        void* stream);
/* Passive scalars (extensions/PISO_multiblock_cuda_kernel.cu:3601-3865 with forPassiveScalar, 4079-4183; driver
 * PISOtorch_simulation.py:1085-1167).  SetupAdvectionMatrix(forPassiveScalar=True, passiveScalarChannel=channel):
 * C and A of channel `channel`, with the scalar viscosity and the channel's boundary types (no diffusion
 * through Neumann faces), plus the non-orthogonal matrix terms of `non_ortho_flags`. */
pict_status_t pict_setup_scalar_matrix(const pict_domain_t* dom, double dt, int32_t non_ortho_flags, int32_t channel,
                                       void* stream);
/* SetupAdvectionScalar: scalar_rhs [C][N] = (det s / dt + boundary advection and diffusion terms - the explicit
 * non-orthogonal terms of scalar_result) / det. */
pict_status_t pict_setup_scalar_rhs(const pict_domain_t* dom, double dt, int32_t non_ortho_flags, void* stream);
/* CopyScalarResultToBlocks (to_blocks=1) / CopyScalarResultFromBlocks (0). */
pict_status_t pict_copy_scalar_result(const pict_domain_t* dom, int32_t to_blocks, void* stream);
/* Gradients of the passive scalar operators (SetupAdvectionMatrixGrad with forPassiveScalar,
 * extensions/PISO_multiblock_cuda_kernel.cu:3869-4077; SetupAdvectionScalarGrad :4185-4278), including the
 * non-orthogonal terms of `non_ortho_flags`.  what 0: in_bar = C_grad [K][N] and A_bar = A_grad [N] of
 * `channel` -> u_bar [D][N] += (block velocity), nu_bar [N] += (the channel's scalar viscosity, per cell).
 * what 1: in_bar = scalarRHS_grad [C][N] -> s_bar [C][N] = (block scalar), s_result_bar [C][N] +=
 * (scalarResult, explicit terms), boundary_scalar_grad [2D][C][N] += and boundary_velocity_grad
 * [2D][D][N] += (per adjacent cell), nu_bar [C][N] += (per cell). */
pict_status_t pict_scalar_grad(const pict_domain_t* dom, double dt, int32_t non_ortho_flags, int32_t what, int32_t channel,
                               const void* in_bar, const void* A_bar, void* u_bar, void* s_bar, void* s_result_bar,
                               void* boundary_scalar_grad, void* boundary_velocity_grad, void* nu_bar, void* stream);

/* SGSviscosityIncompressibleSmagorinsky (extensions/PISOtorch.cpp:540-542 -> extensions/PISO_multiblock_cuda_kernel.cu:6896-7019):
 * out [N] = coefficient * delta * |S| per cell from the blocks' velocity (delta: largest squared column
 * length of the cell transform M, 1 without one). */
pict_status_t pict_sgs_smagorinsky(const pict_domain_t* dom, double coefficient, void* out, void* stream);

/* ---------------- multi-block convolution padding (MultiblockConv, lib/modules/multiblock_cnn.py:92-369) --------
 * Fields are [batch][channels][cells] per block.  src_ptrs / out_ptrs / gout_ptrs / gsrc_ptrs: HOST arrays of the
 * num_blocks (1..64) blocks' device pointers, src_cells / out_cells: HOST arrays of their cells (unpadded /
 * padded); they travel in the kernel parameters.  batch_channels: batch x channels.
 * pict_mb_pad_gather: for the n padded cells j, out[out_block[j]][c][out_pos[j]] = src[src_block[j]][c][src_loc[j]],
 *   0 where src_block[j] < 0 (fixed faces, unreachable corners).
 * pict_mb_pad_scatter_sum: its gradient, for the n source cells g = (src_block[g], src_loc[g]):
 *   gsrc[..][c][..] = sum over k in [reader_ptr[g], reader_ptr[g + 1]) of gout[reader_block[k]][c][reader_pos[k]]
 *   (every source cell written; a fixed order: deterministic).  The index arrays are device arrays. */
pict_status_t pict_mb_pad_gather(int32_t n, int32_t batch_channels, int32_t dtype, int32_t num_blocks,
                                 const int32_t* out_block, const int32_t* out_pos, const int32_t* src_block,
                                 const int32_t* src_loc, const void* const* src_ptrs, const int64_t* src_cells,
                                 void* const* out_ptrs, const int64_t* out_cells, void* stream);
pict_status_t pict_mb_pad_scatter_sum(int32_t n, int32_t batch_channels, int32_t dtype, int32_t num_blocks,
                                      const int32_t* src_block, const int32_t* src_loc, const int32_t* reader_ptr,
                                      const int32_t* reader_block, const int32_t* reader_pos,
                                      const void* const* gout_ptrs, const int64_t* out_cells, void* const* gsrc_ptrs,
                                      const int64_t* src_cells, void* stream);

/* ---------------- preconditioned BiCGStab ----------------
 * SolveLinear with useBiCG and BiCGwithPreconditioner (bicgstabSolveGPU, extensions/bicgstab_solver_kernel.cu:47-395),
 * the fallback of the reference's solve wrapper (PISOtorch_diff.py:276-286), on the CSR form of a stencil matrix
 * (pict_csr_row_ptr / pict_stencil_to_csr; rows sorted by column) of a single-system domain.
 * Preconditioners: PICT_PRECOND_AS_REFERENCE, the operator the reference's build applies (M = T T, T the lower
 * triangle of the matrix including its diagonal: two forward sweeps per application; it sets up csrilu02 factors
 * at extensions/bicgstab_solver_kernel.cu:150-208 but its triangular solves do not apply them); PICT_PRECOND_ILU0,
 * M = L U of the zero-fill incomplete LU factors (what the reference's set-up intends).
 * pict_ilu_analyze (host arrays): diagonal and transposed-entry positions, rows grouped by forward / backward
 *   dependency level (order [n], level starts ptr [n + 1]); the pattern must be structurally symmetric.
 * pict_ilu0_factor: ILU(0) factors (IKJ order, unit lower factor) of the CSR values `a` into `f`, level by level.
 * pict_bicgstab_ilu: right-preconditioned BiCGStab (preconditioner: PICT_PRECOND_*; with transpose the operator and
 *   preconditioner are transposed) in the reference's loop order and reporting; rhs, x [nrhs][n] (device), info_host [nrhs]
 *   (host); synchronises the stream once per reduction; workspace of pict_bicgstab_ilu_workspace_bytes(). */
#define PICT_PRECOND_AS_REFERENCE 0
#define PICT_PRECOND_ILU0 1
pict_status_t pict_ilu_analyze(int32_t n, const int32_t* row, const int32_t* index, int32_t* diag, int32_t* tpos,
                               int32_t* order_f, int32_t* ptr_f, int32_t* order_b, int32_t* ptr_b, int32_t* nlev_f,
                               int32_t* nlev_b);
int64_t pict_bicgstab_ilu_workspace_bytes(int32_t n, int32_t nnz, int32_t dtype);
pict_status_t pict_ilu0_factor(int32_t n, int32_t nnz, int32_t dtype, const int32_t* row, const int32_t* index,
                               const int32_t* diag, const int32_t* order_f, const int32_t* ptr_f_host, int32_t nlev_f,
                               const void* a, void* f, void* stream);
pict_status_t pict_bicgstab_ilu(int32_t n, int32_t nnz, int32_t dtype, const int32_t* row, const int32_t* index,
                                const int32_t* diag, const int32_t* tpos, const int32_t* order_f,
                                const int32_t* ptr_f_host, int32_t nlev_f, const int32_t* order_b,
                                const int32_t* ptr_b_host, int32_t nlev_b, const void* aval, const void* rhs, void* x,
                                int32_t nrhs, int32_t max_iterations, double tolerance, int32_t convergence,
                                int32_t x_is_zero, int32_t transpose, int32_t preconditioner, void* info_host,
                                void* workspace, int64_t workspace_bytes, void* stream);

/* ---------------- advective outflow boundaries ----------------
 * update_advective_boundaries followed by balance_boundary_fluxes (PISOtorch_simulation.py:145-312, the
 * reference's host-side PyTorch code run through the driver's prep_fn before each step), on the device.
 * faces: host array [num_faces][2] of (block, face) pairs, 1 <= num_faces <= PICT_MAX_OUTFLOW_FACES,
 * each a fixed face whose boundary velocity is varying ([D][face cells]); char_velocity: host [D],
 * the static characteristic velocity.  Each outflow face cell moves its boundary velocity towards
 * the adjacent block cell by t = 1 - 1/(1 + 2 dt c), c the face-normal component of char_velocity
 * (row `axis` of the boundary transform's inverse times it, if the face has a transform); then,
 * unless the net outward flux of all fixed faces (FixedBoundary::GetFluxes, extensions/domain_structs.cpp:527-542,
 * summed in FP64) is within `atol` of zero, the outflow faces' velocity is scaled by -(flux of the
 * other fixed faces) / (flux of the outflow faces).  The reference's atol is 1% of the solver
 * tolerance (1e-7 in FP32, 1e-10 in FP64).  Boundary velocities are updated in place.  One
 * simulation per domain (num_sims == 1).  dt: the time step, or per system from dom->sim_dt. */
#define PICT_MAX_OUTFLOW_FACES 16
pict_status_t pict_advective_outflow(const pict_domain_t* dom, const int32_t* faces, int32_t num_faces,
                                     const double* char_velocity, double dt, double atol, void* stream);

/* Gradients of the non-orthogonal terms (nonOrthoFlags; the non-orthogonal parts of the reference's *_GRAD
 * kernels, extensions/PISO_multiblock_cuda_kernel.cu:1992-2098, 3212-3392).  what 0: advection matrix, out_bar =
 * C_grad [K][N] with A_bar = A_grad [N] -> coef_bar = viscosity gradient [N] (per cell); 1: velocity RHS,
 * out_bar = velocityRHS_grad [D][N] -> data_bar = velocityResult gradient [D][N], coef_bar = viscosity
 * gradient [N], boundary_velocity_grad [2D][D][N]; 2: pressure matrix, out_bar = P_grad [K][N] -> coef_bar
 * = A gradient [N]; 3: pressure RHS divergence, out_bar = pressureRHSdiv_grad [N] -> data_bar =
 * pressureResult gradient [N], coef_bar = A gradient [N].  Accumulates (atomics). */
pict_status_t pict_nonortho_grad(const pict_domain_t* dom, int32_t flags, int32_t what, const void* out_bar,
                                 const void* A_bar, void* data_bar, void* coef_bar, void* boundary_velocity_grad,
                                 void* stream);
/* Copy between a global [ncomp][N] vector and a per-block field (0 velocity, 1 pressure, 2 source,
 * 3 velocity_grad, 4 pressure_grad, 5 source_grad); accumulate=1 adds instead of overwriting. */
pict_status_t pict_copy_field(const pict_domain_t* dom, int32_t which, int32_t to_blocks, void* global_vec,
                              int32_t accumulate, void* stream);

/* ---------------- matrix export / utilities ---------------- */
/* CSR materialisation of a stencil matrix in the reference's row layout (rows sorted by
 * column, extensions/PISO_multiblock_cuda_kernel.cu:3846-3860).  row_out [N+1] must be computed first by pict_csr_row_ptr. */
pict_status_t pict_csr_row_ptr(const pict_domain_t* dom, int32_t* row_out, void* stream);
pict_status_t pict_stencil_to_csr(const pict_domain_t* dom, const void* coef, const int32_t* row,
                                  void* value_out, int32_t* index_out, void* stream);
pict_status_t pict_csr_to_stencil(const pict_domain_t* dom, const void* value, const int32_t* row,
                                  const int32_t* index, void* coef_out, void* stream);
/* CoordsToTransforms / CoordsToFaceTransforms (extensions/grid_gen.cu:341-375, 468-514). coords [D][(z+1)][y+1][x+1]. */
pict_status_t pict_coords_to_transforms(const void* coords, int32_t dims, const int32_t* size_xyz,
                                        int32_t dtype, void* out, void* stream);
pict_status_t pict_coords_to_face_transforms(const void* coords, int32_t dims, const int32_t* size_xyz,
                                             int32_t dtype, void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PICT_B200_H */
