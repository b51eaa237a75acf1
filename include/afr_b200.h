/*
 * afr_b200.h -- C-ABI of the B200 (sm_100a) FR residual-and-update library.
 *
 * The library replaces, behind one C-ABI, the reference solver's residual /
 * time-step seam for the explicit Flux-Reconstruction path of AutoFlowCFD.
 * Reference interfaces replaced (paths relative to the reference's
 * src/autoflowcfd):
 *
 *   afr_create              HighOrderMesh + FRSolver set-up consumed by the path:
 *                           core/fr_solver/solver.py:58-243 (ctor),
 *                           core/fr_operators/face_kernels.py:228-369 (FlatFaceGeometry),
 *                           boundary/fr_ghost_state.py:144-189 (ghost provider tables),
 *                           core/gpu/gpu_solver.py:51-157 (GPUFRSolver.__init__ upload)
 *   afr_inviscid_residual   FRSolver.compute_inviscid_residual, core/fr_solver/solver.py:351-400
 *                           (GPU form: core/gpu/gpu_inviscid.py:31 compute_inviscid_residual_fr_gpu)
 *   afr_viscous_residual    FRSolver.compute_viscous_residual, core/fr_solver/solver.py:402-432
 *                           (GPU form: core/gpu/gpu_viscous.py:36)
 *   afr_local_dt            FRSolver._compute_local_time_step, core/fr_solver/cfl.py:12-147
 *                           (GPU form: core/gpu/gpu_solver.py:251-293)
 *   afr_sst_update          FRSolver.compute_turbulence_source, core/fr_solver/turbulence.py:178-330
 *   afr_step                FRSolver.step, core/fr_solver/step.py:15-221
 *                           (GPU form: GPUFRSolver.step, core/gpu/gpu_solver.py:295-401)
 *   afr_cd_cl               compute_aerodynamic_coefficients_fr, postprocess/fr_coefficients.py:27-152
 *   afr_flux_point_jobs     build_face_flux_points (set-up), fr/face_flux_points_merge.py:51-434
 *   afr_prolong             interpolate_to_new_order (order continuation),
 *                           core/utils/order_continuation.py:62-124
 *   afr_destroy             GPUFRSolver.cleanup, core/gpu/gpu_solver_io.py:20-35
 *
 * Conventions: every call returns an int status (AFR_OK = 0).  Arrays passed
 * to afr_create are HOST pointers that are copied; arrays passed to the other
 * calls are DEVICE pointers owned by the caller (contiguous, row-major, the
 * reference's own layouts: U is (n_cells, n_sps, n_vars) float64, fields are
 * (n_cells, n_sps) float64).  The library never frees caller memory.  Calls
 * on one handle are not thread safe.  `stream` is a cudaStream_t (0 = the
 * legacy default stream).  afr_create range-checks every table index
 * (AFR_EINDEX) before any kernel runs.  Kernels never trap: non-finite values
 * and tensor-core wait time-outs are reported through a device status word
 * (AFR_ENONFINITE, AFR_ECUDA) that the calls read back (see afr_step and
 * afr_status).
 */
#ifndef AFR_B200_H
#define AFR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  AFR_OK = 0,
  AFR_EINVAL = 1,       /* bad argument / inconsistent tables */
  AFR_ENOMEM = 2,       /* device allocation failed */
  AFR_ECUDA = 3,        /* CUDA runtime error */
  AFR_ENONFINITE = 4,   /* non-finite value detected by a kernel */
  AFR_EUNSUPPORTED = 5, /* order / feature not built into this library */
  AFR_EINDEX = 6        /* a table index out of range */
};

enum { AFR_TURB_NONE = 0, AFR_TURB_SST = 1 };

/* Arithmetic form of the residual-and-update stage.  AFR_PREC_FP64 is FP64
 * throughout.  AFR_PREC_MIXED runs the operator contractions (c2f, the
 * folded f2c*D_fine divergence, the viscous D_3d divergence, the gradients
 * and the extrapolation to faces) on the tensor cores as BF16 hi+lo split
 * products with FP32 accumulation and the pointwise fluxes in FP32, keeping
 * FP64 for the state, geometry metrics, primitive recovery, residual sums,
 * RK update, norm and Cd/Cl.  Viscous terms are built up to P2 in the mixed
 * form (P3 mixed handles must be inviscid).  A contraction accumulated in FP32
 * carries about 2^-24 * (operator row l1 norm) * |x|, so afr_create refuses
 * the mixed form (AFR_EUNSUPPORTED) when a present cell type's operators have
 * row l1 norms above 1e6: the reference's collapsed-tet operators at P2 and P3
 * (row l1 norms ~2e11 and ~2e8); prisms at every order and tets at P1 pass. */
enum { AFR_PREC_FP64 = 0, AFR_PREC_MIXED = 1 };
enum { AFR_BC_WALL = 0, AFR_BC_FARFIELD = 1, AFR_BC_INLET = 2, AFR_BC_OUTLET = 3, AFR_BC_SYMMETRY = 4 };

typedef struct afr_handle afr_handle;

/* Mesh, operators and face tables, as flattened by the reference
 * (core/fr_operators/face_kernels.py:124-187).  All host pointers.
 * order 0 is the reference's finite-volume path (one point per cell,
 * core/fr_residual/inviscid_p0.py:18-85): n_sps = n_fine = n_fp = 1, the FP64
 * form, laminar, inviscid or SST (the SST closure and transport run the
 * generic one-point kernels, as the reference runs its FR transport there);
 * c2f, D_fine and f2c may be NULL there (the reference has none) and
 * true_area_weight is required (the face areas). */
typedef struct afr_mesh_desc {
  int32_t n_cells, n_prism, order, n_sps, n_fine, n_fp, n_faces;
  int32_t n_nb_src1, n_ow_src1; /* rows of the compact second-source tables */
  /* geometry */
  const double* det_jacs;       /* (N,S) */
  const double* inv_jacs;       /* (N,S,3,3) */
  const double* det_jacs_fine;  /* (N,Fn) */
  const double* inv_jacs_fine;  /* (N,Fn,3,3) */
  const double* cell_volumes;   /* (N) Gauss-Legendre volume (high_order_mesh.py:335-354) */
  const double* wall_distance;  /* (N,S) or NULL (required for SST) */
  /* operators, index 0 = prism, 1 = tet (may be NULL for an absent type) */
  const double* D_3d[2];        /* (S,S,3) */
  const double* c2f[2];         /* (Fn,S) */
  const double* D_fine[2];      /* (Fn,Fn,3) */
  const double* f2c[2];         /* (S,Fn) */
  const double* filter[2];      /* (S,S) */
  const double* boundary_extrap;/* (2,3,2,P,S) */
  const double* g_left;         /* (order+1) */
  const double* g_right;
  const int64_t* dist_fp_of_sp;         /* (3,S) */
  const int64_t* dist_axis_coord_of_sp; /* (3,S) */
  /* face records */
  const int64_t* owner_cell;    /* (F) */
  const int64_t* neighbor_cell; /* (F), -1 on boundary */
  const int64_t* owner_axis;
  const int64_t* neighbor_axis;
  const double* owner_side;
  const double* neighbor_side;
  const uint8_t* is_boundary;
  const uint8_t* owner_is_primary;
  const uint8_t* neighbor_is_primary;
  const double* true_normal;    /* (F,P,3) */
  const int64_t* nb_src0_cell; const double* nb_src0_mat; /* (F), (F,P,S) */
  const int64_t* nb_src1_idx;  const int64_t* nb_src1_cell; const double* nb_src1_mat;
  const int64_t* ow_src0_cell; const double* ow_src0_mat;
  const int64_t* ow_src1_idx;  const int64_t* ow_src1_cell; const double* ow_src1_mat;
  const int32_t* colors;        /* (F) greedy face color (core/utils/face_coloring.py:124-176) */
  /* boundary conditions: row bc_group[f] of the table for boundary face f */
  int32_t n_bc;
  const int32_t* bc_group;      /* (F) */
  const int32_t* bc_type;       /* (n_bc) AFR_BC_* */
  const int32_t* bc_noslip;     /* (n_bc) */
  const double* bc_wall_vel;    /* (n_bc,3) */
  const double* bc_Q;           /* (n_bc,5) free-stream / inlet primitive state */
  const double* bc_p_out;       /* (n_bc) */
  /* force integration (optional) */
  const uint8_t* cd_wall_face;      /* (F) or NULL */
  const double* true_area_weight;   /* (F,P); NULL allowed above order 0 without forces */
  /* optional indexed form of the interpolation matrices: when src_mat_table
   * is non-NULL the four *_mat arrays above are ignored and record f's
   * matrix is src_mat_table[*_mat_index[f]]; the library keeps the table on
   * the device and reads each record's rows through its index (dense inputs
   * are read through identity indices) */
  int32_t n_src_mats;
  const double* src_mat_table;      /* (n_src_mats,P,S) */
  const int32_t* nb_src0_mat_index; /* (F) */
  const int32_t* nb_src1_mat_index; /* (n_nb_src1) */
  const int32_t* ow_src0_mat_index; /* (F) */
  const int32_t* ow_src1_mat_index; /* (n_ow_src1) */
  /* optional fields of a solver whose order changed (order continuation,
   * core/utils/order_continuation.py:207-425), NULL otherwise:
   * fv_cell_volumes   (N) divisor of the order-0 finite-volume residual: the
   *                   mesh's cell_volumes attribute, computed once at the
   *                   order the mesh was loaded at (inviscid_p0.py:44-51),
   *                   while cell_volumes above is the current order's
   *                   (high_order_mesh.py:335-354, the local-dt length);
   * metric_flux_scale (N,S) geometric local-dt scale sum_m |adj(J)[m,:]|:
   *                   the reference caches it at its first evaluation and
   *                   reuses it, broadcast over the points, while the cell
   *                   count is unchanged (solver_geometry.py:18-32); NULL
   *                   forms it from this order's Jacobians */
  const double* fv_cell_volumes;
  const double* metric_flux_scale;
} afr_mesh_desc;

typedef struct afr_params {
  int32_t n_vars;           /* 5, or 7 with SST (columns 5:7 carried, zero residual) */
  int32_t turb;             /* AFR_TURB_* */
  int32_t inviscid_only;    /* 1: viscous residual is zero (Euler) */
  int32_t precision;        /* AFR_PREC_FP64 (plain form) or AFR_PREC_MIXED */
  double mu;                /* molecular viscosity of the mean flow (FRSolver mu_molecular) */
  double rho_inf, vel_inf, p_inf;
  double global_dt_factor;  /* >0: dt = factor * min(dt_local) everywhere (time-accurate runs) */
  /* 1: build the mixed form even for operators above the row-l1 bound (its
   * results then carry errors of about 2^-24 * row l1 * |x|); for measuring
   * that error only, the refusal (0) is the default */
  int32_t mixed_ignore_conditioning;
} afr_params;

int afr_create(const afr_mesh_desc* mesh, const afr_params* params, void* stream, afr_handle** out);
int afr_destroy(afr_handle* h);
/* Message of the last failure on h; with h == NULL, of the last failed
 * afr_create on the calling thread. */
const char* afr_last_error(const afr_handle* h);
const char* afr_status_string(int status);
int afr_version(void);

/* Residuals of the state U (device, (N,S,n_vars)), written to R (device, same
 * shape, turbulence columns zero).  nu_t (device (N,S) or NULL) is the
 * kinematic eddy viscosity; mu_t = max(rho,1e-10) * nu_t. */
int afr_inviscid_residual(afr_handle* h, const double* U, double* R, void* stream);
int afr_viscous_residual(afr_handle* h, const double* U, const double* nu_t, double* R, void* stream);

/* Local time step (device (N,S)). */
int afr_local_dt(afr_handle* h, const double* U, const double* nu_t, double* dt, void* stream);

/* SST source + transport + point-implicit update of k, omega (in place) and
 * nu_t (overwritten with the new eddy viscosity).  diag (device (N,S,4) or
 * NULL) receives Sk, S_omega, transport_k, transport_omega. */
int afr_sst_update(afr_handle* h, const double* U, const double* dt_local, double* k, double* omega,
                   double* nu_t, double* diag, void* stream);

/* One SSP-RK3 step in place on U (and k, omega, nu_t with SST; pass NULL
 * otherwise).  *norm_out (host) receives the RMS of dU/dt at stage 0; the call
 * then synchronises the stream and returns the device status (AFR_ENONFINITE
 * when any cell's dU/dt at stage 0 is not finite).  With norm_out == NULL the
 * call does not synchronise: it queues a copy of the status word to pinned
 * host memory, and the next afr_step on the handle returns the problem once
 * that copy has completed (inside a stream capture the copy is part of the
 * graph and afr_status reads the word).  The device status is sticky until
 * afr_status clears it. */
int afr_step(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* norm_out,
             void* stream);

/* One physical step of the dual-time scheme (DUAL_TIME,
 * core/fr_solver/step.py:167-185 and core/time_integration/dual.py:19-158):
 * the SST fields advance once with the physical step dt_physical; the mean
 * flow solves the BDF-implicit equation (BDF1 when has_prev == 0, BDF2 with
 * the previous level U_prev otherwise) by up to max_inner_iter pseudo-time
 * SSP-RK3 iterations with the local time step and the reference's adaptive
 * CFL factor (0.1 .. 10), stopping when the dual residual dropped 1e-6
 * relative, fell below tol (from the second iteration), or an update moved
 * the state by less than 1e-10 (L2).  Positivity and the modal filter follow
 * every stage and the pseudo step.  U (device) is advanced in place; U_prev
 * (device, same shape, caller-owned) receives the state at the start of the
 * step for the next call.  *norm_out (host, may be NULL) receives the RMS of
 * the spatial dU/dt at the start of the step.  Synchronises (the iteration's
 * control flow reads norms); not for stream capture. */
int afr_step_dual_time(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* U_prev,
                       int32_t has_prev, double dt_physical, int32_t max_inner_iter, double tol, double* norm_out,
                       void* stream);

/* One step of the IMEX Euler scheme (IMEX_EULER, core/fr_solver/step.py:186-193
 * and core/time_integration/imex.py:17-97): the inviscid residual at the start
 * of the step is explicit, the viscous residual implicit, solved by up to five
 * damped Picard iterations (damping 0.5, adapted between 0.1 and 1) with the
 * local time step and positivity; SST as in afr_step.  Synchronises. */
int afr_step_imex(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* norm_out, void* stream);

/* Device status of the handle after the work queued on stream (synchronises;
 * not inside a stream capture): AFR_OK, AFR_ENONFINITE, AFR_EINDEX or AFR_ECUDA
 * (a tensor-core wait ran out).  With nseg > 0, seg_status[i] receives the
 * status of cells [cell_ptr[i], cell_ptr[i+1]) -- AFR_ENONFINITE when any of
 * their stage-0 dU/dt values of the last step is not finite -- so that
 * independent cases concatenated into one handle fail one by one.  clear = 1
 * resets the device status afterwards.  Replaces the per-case status of the
 * batched driver (the reference has one case per solver and raises Python
 * exceptions, core/fr_solver/step.py:217-221). */
int afr_status(afr_handle* h, int32_t nseg, const int64_t* cell_ptr, int32_t* seg_status, int32_t clear,
               void* stream);

/* afr_step with a CUDA event after every launch group; ms_out[i] receives the
 * device time of group i: local dt, [SST point, SST face, SST update],
 * then per RK stage (gradient pre-pass, fused stage kernel), the norm
 * reduction.  *launches receives the kernel launches of the step. */
int afr_step_profile(afr_handle* h, double* U, double* k, double* omega, double* nu_t, double* ms_out, int n_ms,
                     int* launches, void* stream);

/* Wall force coefficients (Cd, Cl, Cs) of state U into out3 (host), in
 * FP64.  Mixed-precision handles keep no FP64 point fields between calls:
 * this call allocates them (N x S x 18 doubles) for its duration and
 * synchronises the stream. */
int afr_cd_cl(afr_handle* h, const double* U, const double* nu_t, double reference_area, double* out3,
              void* stream);

/* Host utility (no GPU): greedy face coloring in face order, the smallest
 * color not used by any earlier face sharing a cell (owner, and neighbour of
 * interior faces).  Restates core/utils/face_coloring.py:124-176. */
int afr_greedy_face_coloring(int64_t n_faces, int64_t n_cells, const int64_t* owner_cell,
                             const int64_t* neighbor_cell, const uint8_t* is_boundary, int32_t* colors_out);

/* RMS norm sqrt(sum(x^2) / n) of a device array x of n doubles, written to
 * the device double *out, without allocating any memory.  No counterpart in
 * the reference: it is the step's residual-norm reduction offered on its own
 * for callers that may not allocate at call time -- code running while a CUDA
 * graph is being captured (cudaMalloc is not a stream operation and breaks the
 * capture), real-time step loops where an allocation would synchronise the
 * device, and host applications that own all device memory through their own
 * pool.  Its scratch is a fixed 32 KiB file-scope device array (4096 block
 * partials); n may be at most 4096 * 65536 = 268,435,456, larger n returns
 * AFR_EINVAL.  The first call on each device looks up that array's device
 * address (cudaGetSymbolAddress, with the device current) and should come
 * before any stream capture.  Every call shares the array: calls that overlap
 * on the GPU (different streams, no ordering between them) race.  Each call
 * writes every partial it reads, so nothing needs clearing between calls.
 * The sum order is fixed for a given n, so results are bitwise repeatable. */
int afr_rms_norm_noalloc(const double* x, int64_t n, double* out, void* stream);

/* Launch-shape autotuner of the mixed form: times one residual evaluation of
 * the state U (nu_t for SST handles) for each candidate pre-pass CTAs per SM,
 * face-kernel block size (64/128/256) and update-kernel cells per CTA (half /
 * base / double), one parameter at a time, and keeps the fastest in the
 * handle.  U is not modified.  choice_out (3 ints, may be NULL) receives the
 * choices; plain-form handles keep their fixed shapes (choices -1).  No
 * counterpart in the reference (launch shapes have none there). */
int afr_autotune(afr_handle* h, const double* U, const double* nu_t, int32_t* choice_out, void* stream);

/* Current launch shapes of a handle (8 ints): pre-pass CTAs per SM, its
 * maximum (the CTAs that fit by registers, shared memory and threads, capped
 * by 512 tensor-memory columns per SM), the runtime occupancy query's value
 * for the pre-pass (one for any kernel that uses tensor memory), volume-kernel
 * CTAs per SM, the runtime query's value for it, face-kernel block,
 * update-kernel variant (0 half, 1 base, 2 double cells per CTA) and the
 * device's SM count.
 * Plain-form handles report -1 except the SM count.  No counterpart in the
 * reference. */
int afr_launch_shape(const afr_handle* h, int32_t* out);

/* Per-segment RMS residual norms of the last afr_step: segment i is cells
 * [cell_ptr[i], cell_ptr[i+1]) (host array of nseg+1).  which = 0: the norm
 * over all variables, sqrt(sum(dU/dt^2) / (cells * n_sps * n_vars)), as
 * FRState.get_residual_norm (state.py:99-108); which = 1: the density column
 * only, sqrt(sum((drho/dt)^2) / (cells * n_sps)).  Summed in a fixed order.
 * For several independent cases concatenated into one handle, and for the
 * density-residual stopping rule of a steady solve (nseg = 1).  Synchronises
 * the stream. */
int afr_segment_norms(afr_handle* h, int32_t nseg, const int64_t* cell_ptr, int32_t which, double* out,
                      void* stream);

/* Sums of squares of the last afr_step's stage-0 dU/dt into the caller's
 * device buffer out2: out2[0] over all variables, out2[1] over the density
 * column, each summed in the fixed order of the step norm (the RMS norms are
 * sqrt(out2[0] / (cells * n_sps * n_vars)) and sqrt(out2[1] / (cells *
 * n_sps))).  Kernel launches and a device-to-device copy only: no
 * synchronisation and no allocation, so a steady-solve driver can record it
 * in the CUDA graph of a slice of steps and poll the result.  Extends
 * FRState.get_residual_norm (core/fr_solver/state.py:99-108) to the
 * density-residual stopping rule of a steady solve. */
int afr_residual_sums(afr_handle* h, double* out2, void* stream);

/* Tensor-core self-check: D[128 x n] = A[128 x k] * B[n x k]^T on the
 * calling device with tcgen05.mma, A and B row-major BF16 bit patterns and D
 * row-major FP32, all device memory; 16 <= n, k <= 256, both multiples of 16.
 * It runs the shared-memory layout, descriptors and bounded waits of the
 * mixed-precision kernels on one CTA and synchronises the stream.  No
 * counterpart in the reference (diagnostic for the mixed-precision form). */
int afr_tc_check(int n, int k, const void* A, const void* B, float* D, void* stream);

/* Order continuation: prolong a field of the same mesh held at a lower order
 * (n_sps_old points per cell) to this handle's order,
 *   new[c, a, v] = sum_b W[a, b] * old[c, b, v]   (b ascending),
 * the np.einsum("ab,cbv->cav") of interpolate_to_new_order
 * (core/utils/order_continuation.py:62-124).  W is a HOST (n_sps x
 * n_sps_old) row-major matrix (the reference's trilinear interpolation
 * matrix between the two Gauss-Legendre tensor grids, formed by the caller);
 * old is (n_cells, n_sps_old, n_cols) and new (n_cells, n_sps, n_cols) on the
 * device, n_cols 1..8, not overlapping.  The first call allocates a small
 * matrix buffer on the handle; W is copied before the call returns. */
int afr_prolong(afr_handle* h, const double* old_field, int32_t n_sps_old, int32_t n_cols, const double* W,
                double* new_field, void* stream);

/* Flux-point construction (set-up; no handle).  Each job locates the flux
 * points of one face side on the other side's cell and forms that side's
 * cross-interpolation rows:
 *   job j: the order-`order` flux points of cube face src_code[j] of cell
 *   src_cell[j] are mapped to physical space, shifted by the face's periodic
 *   translation (sign[j] < 0: minus, owner -> neighbour; > 0: plus), located
 *   on cube face tgt_code[j] of cell tgt_cell[j] (closed form on tets, the
 *   reference's damped Newton iteration with backtracking on prisms, both
 *   with the face's sqrt(area) as length scale), and the rows
 *   V(located points) * v_inv of that cell type are written to mats[j]
 *   (n_fp x n_sps); mode[j] = 0 writes every row, 1 only the rows whose bit is
 *   set in mask[j], 2 only the others (the two halves of a split prism quad
 *   face), the remaining rows are zero.  coords[j] gets the located free
 *   coordinates (n_fp x 2), resid[j] the largest location residual.
 * Restates build_fp_newton_parallel (fr/face_flux_points_numba.py:30-251) and
 * build_ms_interp_parallel (fr/face_flux_points_ms_numba.py:31-317).  All
 * pointers are HOST memory; cells are prisms [0, n_prism) then tets; v_inv_*
 * is the (n_sps x n_sps) inverse modal Vandermonde matrix of that cell type
 * (NULL when the type is absent); sps_1d the order+1 Gauss-Legendre points.
 * Every index is range-checked before any kernel runs (AFR_EINDEX); the
 * device memory is allocated per call and released before it returns. */
int afr_flux_point_jobs(int32_t order, int32_t n_prism, int64_t n_tet, int64_t n_nodes, const double* nodes,
                        const int32_t* prism_conn, const int32_t* tet_conn, const double* v_inv_prism,
                        const double* v_inv_tet, const double* sps_1d, int64_t n_faces, const double* area,
                        const double* translation, int64_t n_jobs, const int32_t* face, const int32_t* src_cell,
                        const int32_t* src_code, const int32_t* tgt_cell, const int32_t* tgt_code,
                        const int32_t* sign, const int32_t* mode, const uint32_t* mask, double* mats, double* coords,
                        double* resid);

/* Bytes of device memory the handle owns (tables + scratch). */
int afr_device_bytes(const afr_handle* h, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif /* AFR_B200_H */
