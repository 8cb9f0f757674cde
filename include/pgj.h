/* libpgj — B200 (sm_100a) periodic HEX8 homogenization with the partial Green-Jacobi PCG.
 *
 * C ABI: plain pointers, sizes and status codes; no torch or C++ types. Every device buffer is
 * owned by the caller. The library allocates no device memory: a context is laid out inside a
 * caller-provided workspace whose size is queried once (pgj_workspace_bytes). Every entry point
 * takes an explicit CUDA stream (passed as void*, i.e. a cudaStream_t) and performs no host
 * synchronisation except where stated (the certified solve reads a few scalars per attempt).
 *
 * Conventions (shared with the reference, yufangjie1643/partial-green-jacobi):
 *   n          periodic grid edge; N = n^3 nodes = elements; unit cube, voxel h = 1/n
 *   DOF vector (L, 3N) float64, node-major, xyz interleaved, nodes in (z, y, x) order
 *   field      (n, n, n) float64 in (z, y, x) order; a = element stiffness multiplier
 *   macros     (L, 6) engineering Voigt strains (xx, yy, zz, yz, xz, xy), HOST memory
 *   medium     isotropic C0(lambda, mu); C(x) = a(x) C0
 *
 * Each declaration names the reference interface it replaces (file:line in the reference tree).
 */
#ifndef PGJ_H
#define PGJ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define PGJ_OK 0
#define PGJ_ERR_ARGUMENT 1       /* bad pointer, size, shape or value (TORCH_CHECK in the reference) */
#define PGJ_ERR_UNSUPPORTED 2    /* grid size outside the built FFT radices / limits */
#define PGJ_ERR_LAUNCH 3         /* CUDA launch or runtime error (C10_CUDA_KERNEL_LAUNCH_CHECK) */
#define PGJ_ERR_NONFINITE 4      /* non-finite input or non-positive curvature latch */
#define PGJ_ERR_ITERATION_CAP 5  /* the PCG loop ran into its body bound (iteration cap + 100) */
#define PGJ_ERR_CERTIFICATION 6  /* 'true residual certification failed' (resident.py:208) */
#define PGJ_ERR_TIMEOUT 7        /* a bounded device wait expired */
#define PGJ_ERR_WORKSPACE 8      /* workspace missing, too small or misaligned */

#define PGJ_FP64 0               /* all solver arithmetic in float64 */
#define PGJ_FP32 1               /* inner operator / Green / PCG vectors in float32 */

typedef struct pgj_ctx pgj_ctx;  /* opaque; host object over a caller-owned device workspace */

/* One record per load, the reference's info dict (exp/asg_gpu_resident_20261103/resident.py:206-207). */
typedef struct pgj_load_info {
  double rhs_norm;
  double absolute_residual;
  double threshold;
  double relative_residual;
  int32_t iterations;
  int32_t converged;
  int32_t restarts;
  int32_t bad;
} pgj_load_info;

int pgj_version(void);
const char* pgj_status_string(int status);
/* Last CUDA error code seen by the library in this thread (0 if none). */
int pgj_last_cuda_error(void);

/* ------------------------------------------------------------------ context / operator object
 * Replaces the operator construction Backend.build -> HybridFIOperator + enable_fi_reference +
 * native.attach (solver/experiments/adaptive_green_scaling/study.py:61-77,
 * solver/src/materials/hybrid_adapter.py:45-68, solver/src/reference_medium/formula_adapter.py:40-68,
 * solver/src/spectral/native_adapter.py:16-35). Holds the FI Green symbol (6 coefficients, 1/N
 * folded), the FFT tables, the scale field and the solver state for up to `loads` recurrences.
 * `precision` selects the inner arithmetic (PGJ_FP64 or PGJ_FP32). The workspace must be
 * 256-byte aligned and at least pgj_workspace_bytes(...) long; pgj_ctx_create clears it. */
int pgj_workspace_bytes(int n, int loads, int precision, size_t* bytes);
int pgj_ctx_create(int n, int loads, int precision, double lam, double mu,
                   void* workspace, size_t workspace_bytes, void* stream, pgj_ctx** out);
int pgj_ctx_destroy(pgj_ctx* ctx);
/* Batched context: `designs` independent designs of the same grid and medium, `loads` right-hand
 * sides each, solved as designs * loads recurrences by the same kernels (every launch carries all
 * designs). No reference counterpart: the reference batches only the loads of one design
 * (load_mode='parallel', exp/asg_gpu_resident_20261103/resident.py:72-73) and loops over designs on
 * the host (exp/asg_density_selector_20261105/run.py:105-119). Load l belongs to design l / loads;
 * macros, u and info of a solve are (designs * loads) records in that order. Restarts are decided per
 * design, and a design that took its last attempt is left untouched by the later attempts of the
 * others, so every design's result and iteration counts are those of a solve of that design alone
 * (same grid, precision and tile shapes). designs <= 16, loads <= 8. pgj_ctx_create is the one-design
 * case. */
int pgj_workspace_bytes_batch(int n, int designs, int loads, int precision, size_t* bytes);
int pgj_ctx_create_batch(int n, int designs, int loads, int precision, double lam, double mu,
                         void* workspace, size_t workspace_bytes, void* stream, pgj_ctx** out);
int pgj_ctx_designs(pgj_ctx* ctx);
/* Design d's material field (a copy of the device field a) and preconditioner exponent (its
 * D^-alpha/2 scale); pgj_set_material / pgj_set_alpha address design 0. */
int pgj_set_material_at(pgj_ctx* ctx, int design, const double* a, void* stream);
int pgj_set_alpha_at(pgj_ctx* ctx, int design, double alpha, void* stream);
/* Homogenized tensor of design d from its six Voigt solutions u (6, 3N), 36 float64 to device C. */
int pgj_effective_tensor_at(pgj_ctx* ctx, int design, const double* u, double* C, void* stream);

/* Device pointer to the context's (loads, 3N) float64 solution / warm-start block (the
 * reference's Resident.solutions, resident.py:79-82). */
double* pgj_ctx_solutions(pgj_ctx* ctx);
/* Device pointer to the context's (1, 3N) float64 scale field D^-alpha/2 (resident.py:88); a batched
 * context holds one per design, (designs, 3N). */
double* pgj_ctx_scale(pgj_ctx* ctx);
/* Device pointer to the context's (n, n, n) float64 material field a (op._material_field,
 * solver/experiments/adaptive_green_scaling/study.py:74); (designs, n, n, n) in a batched context. */
double* pgj_ctx_material(pgj_ctx* ctx);

/* Density multiplier a (n^3 float64, device) -> context material field; no N x 21 expansion
 * (replaces Resident.material, resident.py:152-154). The pointer is copied, not retained. */
int pgj_set_material(pgj_ctx* ctx, const double* a, void* stream);
/* scale = exp(-alpha/2 (log d - mean log d)), d = stiffness diagonal of K(a); alpha = 0 gives 1
 * (Resident.select / SelectorResident.build_scale, resident.py:156-174,
 * exp/asg_density_selector_20261105/run.py:69-77; element_diagonal,
 * solver/experiments/smooth_contrast/study.py:56-66). */
int pgj_set_alpha(pgj_ctx* ctx, double alpha, void* stream);

/* q = K(a) p for `loads` vectors (loads <= context loads); loads whose active[l] == 0 get q = 0.
 * active may be NULL (all active). Replaces scalar.apply (exp/asg_gpu_resident_20261103/scalar_fi.cu:14-36,
 * 46-54) and the certification operator hybrid.apply (solver/src/materials/hybrid_kernels.cu:26-48,117-127). */
int pgj_apply(pgj_ctx* ctx, int loads, const double* p, const int32_t* active, double* q, void* stream);
/* float32 variant of pgj_apply on float32 vectors (inner operator of the mixed solver). */
int pgj_apply_f32(pgj_ctx* ctx, int loads, const float* p, const int32_t* active, float* q, void* stream);
/* f = -V sum B_c^T (a C0) eps for each macro strain (hybrid rhs_kernel,
 * solver/src/materials/hybrid_kernels.cu:50-68,128-137). macros: HOST (loads, 6). */
int pgj_rhs(pgj_ctx* ctx, int loads, const double* macros, double* f, void* stream);
/* z = M_alpha^-1 r = P(s . G(s . P r)) with the context scale (Resident.B, resident.py:104-117;
 * op.apply_precond, solver/src/spectral/native_adapter.py:23-30). */
int pgj_precondition(pgj_ctx* ctx, int loads, const double* r, double* z, void* stream);
/* Build the dense FI Green symbol for (n, lambda, mu) into a caller buffer of 6 * n*n*(n/2+1)
 * float64 (fi_coeff_kernel solver/src/reference_medium/formula_kernels.cu:104-126 + dense
 * prepare_kernel solver/src/spectral/precision_kernels.cu:57-89). */
int pgj_green_symbol(int n, double lam, double mu, double* symbol, void* stream);

/* ------------------------------------------------------------------ certified solve
 * Masked multi-load PCG with true-residual certification and at most two restarts
 * (Resident._solve_batch, resident.py:186-209; PaperResident.solve, reproduction.py:144-151).
 * u: device (loads, 3N) float64, warm start in / certified solution out (may alias
 * pgj_ctx_solutions). macros: HOST (loads, 6). info: HOST array of `loads` records.
 * Returns PGJ_ERR_CERTIFICATION when the reference would raise. In PGJ_FP32 contexts the solve
 * is FP32 inner PCG (relative tolerance inner_rtol) inside FP64 iterative refinement; the
 * certificate and the stopping rule are the FP64 ones. */
int pgj_solve(pgj_ctx* ctx, int loads, const double* macros, double rtol, double* u,
              pgj_load_info* info, void* stream);
/* Enqueue the same certified solve on `stream` without any host synchronisation: the restarts of
 * resident.py:194-205 are decided on the device (a graph WHILE node), so the whole solve is one
 * graph launch. Several contexts on several streams therefore run concurrently. Complete it with
 * pgj_solve_wait, which synchronises `stream` once and fills `info`. Not available for mixed mode 1
 * (PGJ_ERR_UNSUPPORTED). */
int pgj_solve_async(pgj_ctx* ctx, int loads, const double* macros, double rtol, double* u, void* stream);
int pgj_solve_wait(pgj_ctx* ctx, pgj_load_info* info, void* stream);
/* Inner relative tolerance of the FP32 refinement sweeps (mode 1; default 1e-5). */
int pgj_set_inner_rtol(pgj_ctx* ctx, double inner_rtol);
/* Mixed-precision scheme of a PGJ_FP32 context (no reference counterpart: the reference is FP64 only).
 * mode 0 (default): one FP32 PCG recurrence per load with reliable updates; whenever the recurrence
 * residual falls below delta times its value at the last replacement (or the recurrence reports
 * convergence), the FP32 correction is added to the FP64 solution and the recurrence residual is
 * replaced by the FP64 true residual f - K u, on the device, without restarting the Krylov space
 * (delta in (0,1), default 0.1). mode 1: restarted refinement sweeps (FP32 solve to inner_rtol,
 * u += d, FP64 residual), at most 12 sweeps. */
int pgj_set_mixed_mode(pgj_ctx* ctx, int mode, double delta);
/* Per-load PCG iteration cap of the context's solves (default 4000, the reference's cap,
 * resident.py:120; 1 <= cap <= 16000). The FP64 drop-in keeps the default. No reference counterpart
 * for other values: the mixed scheme's FP32 recurrence takes more, cheaper iterations at high
 * contrast, and a larger cap lets it certify where the FP64 recurrence needs most of the 4000. */
int pgj_set_iteration_cap(pgj_ctx* ctx, int cap);
int pgj_iteration_cap(pgj_ctx* ctx);
/* Direction update of the FP32 recurrences of a PGJ_FP32 context (no reference counterpart; FP64
 * contexts keep the reference's beta = r.z / r_prev.z_prev): 1 selects the flexible (Polak-Ribiere)
 * form beta = r.(z - z_prev) / r_prev.z_prev, which keeps the new direction locally orthogonal when
 * the FP32 preconditioner apply is inexact (the slab-fused iteration stores z for the next
 * iteration; the step-by-step one reads it back from the last Green output). PGJ_ERR_UNSUPPORTED for
 * PGJ_FP64 contexts. Default 0. */
int pgj_set_flexible_beta(pgj_ctx* ctx, int on);
/* Arithmetic of the recurrence operator of a PGJ_FP32 context (no reference counterpart): 0 (default)
 * FP32; 1 FP64 element actions and node sums on the FP32 vectors, for high-contrast designs (weak
 * material ratios near 1e-9), where FP32 node sums of stiff and weak elements cancel. The Green
 * apply and the vectors stay FP32. PGJ_FP64 contexts accept 1 only. */
int pgj_set_mixed_operator(pgj_ctx* ctx, int fp64);
/* Refinement count of the last pgj_solve: 1 for PGJ_FP64; sweeps in mixed mode 1; 1 + true-residual
 * replacements in mixed mode 0. */
int pgj_last_refinements(pgj_ctx* ctx);

/* Kernel launches issued by the last pgj_solve (graph nodes included), for launch accounting. */
long long pgj_last_launches(pgj_ctx* ctx);
/* Measurement hook (no reference counterpart; the reference times stages with CUDA events,
 * exp/asg_gpu_resident_20261103/run.py:29-53): starts a zero-start solve of `loads` macros and
 * times each kernel of the PCG iteration separately with CUDA events on `stream`, over `reps`
 * back-to-back launches of that kernel (after two warm launches; the values drift, the work does
 * not). Writes PGJ_PROFILE_KERNELS mean durations (ms) and algorithmic bytes per launch
 * (HOST arrays) in the order: operator, update_ur, fft_x, fft_y, fft_z+symbol, ifft_y, ifft_x,
 * update_p. Leaves the context's iterate undefined (the next pgj_solve starts from its u). */
#define PGJ_PROFILE_KERNELS 8
int pgj_profile_iteration(pgj_ctx* ctx, int loads, const double* macros, int reps, double* ms, double* bytes,
                          void* stream);

/* Kernel set of the PCG iteration (no reference counterpart; both give the reference's recurrence).
 * 1: four kernels per iteration (operator; update + x/y transforms; z pass; inverse x/y + direction
 * update), used when a transform slab fits in shared memory; 0: the operator, the two vector updates
 * and the five Green passes as separate kernels. pgj_set_fused_iteration returns
 * PGJ_ERR_UNSUPPORTED for 1 when the slab does not fit. */
int pgj_fused_iteration(pgj_ctx* ctx);
int pgj_set_fused_iteration(pgj_ctx* ctx, int on);

/* Tile shapes the context's autotuners picked (no reference counterpart): out[0] operator rows per
 * block, out[1] operator z-planes per block, out[2] rows per x-pass block, out[3] / out[4] kx columns
 * per y / z-pass block, out[5] fused iteration flag. */
int pgj_tile_shapes(pgj_ctx* ctx, int* out);
/* The context's tile configuration as the tile table records it (no reference counterpart): out[0..3]
 * operator rows per block, z-planes per block, plane buffers, occupancy variant; out[4..6] requested FFT
 * rows per x block, y chunks, z chunks; out[7] fused iteration flag; out[8] where the shapes came from
 * (0 timed at creation, 1 the tile table built in, 2 environment override). */
int pgj_tile_config(pgj_ctx* ctx, int* out);

/* Failure-detection self-test (no reference counterpart): runs the bounded device wait used by the
 * kernels' TMA staging on an mbarrier that nothing completes, giving up after `tries` polls.
 * Returns PGJ_ERR_TIMEOUT when the wait expired and was reported (the expected outcome); the
 * context stays usable. Never faults or hangs: no copy is issued and the wait is bounded. */
int pgj_selftest_wait_timeout(pgj_ctx* ctx, int tries, void* stream);

/* ------------------------------------------------------------------ responses
 * Per-element energies e_l = v^T Ke(C0) v / h^3, v = u_l + A_l (affine macro field), for each of
 * `loads` (u, macros); e: (loads, N) device (energy.cu evaluate,
 * exp/asg_scenarios_20261105/energy.cu:7-35; Backend.affine, exp/asg_topopt_20261103/backend.py:153-162). */
int pgj_energies(pgj_ctx* ctx, int loads, const double* u, const double* macros, double* e, void* stream);
/* Homogenized tensor of six Voigt loads: C[i][j] = mean(a v_i^T Ke v_j)/h^3, written as 36
 * float64 to device `C` (PaperResident.effective_tensor, reproduction.py:166-176). */
int pgj_effective_tensor(pgj_ctx* ctx, const double* u, double* C, void* stream);

/* Homogenized tensor of six Voigt solutions without any device allocation (no counterpart in the
 * reference). For callers that cannot allocate device memory, such as a host application that owns
 * the device memory pool and forbids third-party allocations. The caller passes a (n^3), u (6, 3N)
 * and C (36 float64), all device; the scratch lives in a fixed file-scope device array of about
 * 0.69 MB per GPU, held until exit, and the unit Voigt strains in a statically initialised device
 * table. Accepts 2 <= n <= 256 (PGJ_ERR_ARGUMENT otherwise). The first call on a device (and the
 * first after its context is replaced, e.g. by cudaDeviceReset) looks up the array's device
 * address. All calls share the array: calls that overlap on the GPU race and must be ordered on one
 * stream. */
int pgj_effective_tensor_noalloc(int n, double lam, double mu, const double* a, const double* u, double* C,
                                 void* stream);

/* ------------------------------------------------------------------ design update (OC)
 * Study II (paper) chain: clipped cone filter, tanh(beta, eta) projection and damped OC with the
 * MATLAB bisection stop (PaperOuter, exp/asg_sctop_reproduction_20261105/reproduction.py:69-118,
 * outer.cu:8-39). Fields are (n, n, n) float64 device. */
int pgj_cone_filter(int n, const int32_t* offsets, const double* weights, int count,
                    const double* x, double* y, void* stream);
int pgj_paper_project(int n, const double* t, const double* hs, double beta, double eta, double emin,
                      double* ph, double* dp, double* a, void* stream);
/* Full OC update: inputs x, ph, dp, hs, local objective density `energy`; output `xnew` and
 * host `steps` (bisections taken) and `change` (max |xnew - x|), read back with one stream
 * synchronisation. With steps and change both NULL the update is only enqueued (no
 * synchronisation); the bisections taken and the change are then left at scratch[4 n^3 + 3] and
 * scratch[4 n^3 + 4]. scratch: 4 n^3 + 512 float64 device. */
int pgj_paper_oc(int n, const int32_t* offsets, const double* weights, int count, const double* x,
                 const double* ph, const double* dp, const double* hs, const double* energy,
                 double volume, double beta, double eta, double emin, double move, double exponent,
                 double floor_, double* xnew, double* scratch, int* steps, double* change, void* stream);
/* Study I chain: periodic separable Gaussian (sigma = 0.9 n/32), tanh projection at 1/2, SIMP
 * eta=1e-4 and 45-step OC (ResidentOuter, exp/asg_gpu_resident_20261103/outer.py:12-59, outer.cu:7-37). */
int pgj_gaussian_filter(int n, const double* weights, int radius, const double* x, double* y,
                        double* scratch, void* stream);
int pgj_study1_project(int n, const double* t, double beta, double* ph, double* dp, double* a, void* stream);
int pgj_study1_oc(int n, const double* weights, int radius, const double* x, const double* ph,
                  const double* dp, const double* energy, double beta, double volume, double move,
                  double* xnew, double* scratch, double* change, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PGJ_H */
