/* C ABI of libspgrid_gpu_solver.so — the B200 narrow-band SPGrid elasticity
 * solver.
 *
 * fem_solve() is the drop-in entry: same symbol, same arguments and same
 * ownership rules as the reference CPU solver library (libSPGridCPUSolver.so),
 * so a caller linked against that library can link against this one instead.
 * The sgs_* functions are additive: a session API that keeps the problem on the
 * GPU between calls, used by the Python layer, the tests and the benchmark.
 */
#ifndef SPGRID_FEM_H
#define SPGRID_FEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGS_API __attribute__((visibility("default")))

/* Error codes (FEMOutputs.error_code and sgs_* return values). */
#define SGS_OK 0
#define SGS_ERR_INPUT 1      /* invalid arguments or parameters */
#define SGS_ERR_UNSUPPORTED 2 /* mode the solver does not implement (use_density_only = false) */
#define SGS_ERR_MG_LEVEL 3   /* mg_level = 2 */
#define SGS_ERR_GRID 4       /* blocks outside the grid, unaligned blocks, non-finite values */
#define SGS_ERR_ACTIVATION 5 /* a material cell lacks its +1 neighbour blocks */
#define SGS_ERR_PADDING 6    /* blocks too close to the grid border for the hierarchy */
#define SGS_ERR_BREAKDOWN 8  /* CG breakdown (s.q <= 0), non-finite residual, singular bottom */
#define SGS_ERR_WIRE 9       /* malformed input blob */
#define SGS_ERR_CUDA 10      /* CUDA runtime failure */
#define SGS_ERR_INTERNAL 11

/* Replaces: extern "C" void fem_solve(void *input, void *output)
 *   (reference topo_opt/fem_interface.h:11, solver/SPGrid_CPU_Solver.cpp:26).
 * input : serialized FEMInputs blob; its first 8 bytes hold the total length
 *         (topo_opt/serialization.h:318-329).
 * output: really a void**; receives a serialized FEMOutputs blob allocated with
 *         new char[] that the caller releases with delete[] (or fem_solve_free)
 *         (fem_interface.h:414-441, 477).
 * Never aborts or throws: failures come back as success = 0 with error_code and
 * info set.  Extra knobs (all optional) in FEMInputs.extra_ints:
 *   "sgs_precision"  0 = reference arithmetic (float-rounded CG updates and
 *                        V-cycle casts, the default), 1 = FP64, 2 = FP32 V-cycle
 *                        with FP64 outer PCG;
 *   "sgs_honor_max_iterations"  1 = stop at krylov.max_iterations instead of 500;
 *   "sgs_tensor_cores"  1 = the FP32 V-cycle's level-0 residual on the tensor
 *                        cores (tcgen05), 0 = on the CUDA cores (default, faster
 *                        as measured);
 *   "sgs_dense_bottom_max"  largest bottom (unknowns) inverted densely (default
 *                        24576).  A larger bottom -- the reference driver's
 *                        default mg_bottom_size 64 gives 10^5-10^6 unknowns,
 *                        which the reference factors with PARDISO -- is solved
 *                        exactly (to round-off) by CG preconditioned with
 *                        V-cycles over further levels coarsened below it.
 *   "sgs_device_loop"  0 = test convergence on the host after every PCG
 *                        iteration (one graph launch per iteration) instead of
 *                        running the whole loop as one graph whose WHILE node
 *                        the test kernel drives (default 1; the output's
 *                        extra_ints "device_loop" says which ran);
 *   "sgs_loop_history"  residuals one launch of the device loop records before
 *                        it pauses for the host to take them out (2-1024,
 *                        default 1024; smaller values only add launches).
 *   "sgs_inner_smoothing", "sgs_inner_boundary_smoothing"  full and
 *                        boundary-band sweeps per level and direction of the
 *                        V-cycle inside the inner CG of a large bottom (default
 *                        3 and 0; the bottom is solved to round-off either way).
 * A solve that reaches the iteration cap returns success = 1 as the
 * reference's does, with extra_ints "converged" = 0. 
 * Warm starting as the reference's (SPGrid_CPU_Solver.cpp:56-73, 240-321,
 * 389-408): with extra_ints "keep_state" = 1 the output's extra_ints
 * "state_ptr_lower"/"state_ptr_higher" name a solver state (the last solution
 * per level-0 page and the first call's zero-guess residual); passed back in
 * the next input, the previous solution is the initial guess when
 * "forced_reuse" is set or it beats the zero guess, and the stopping rule stays
 * relative to the stored residual.  A call without keep_state releases the
 * state it was given. */
SGS_API void fem_solve(void* input, void* output);

/* Release an output blob from fem_solve (callers that cannot call delete[]). */
SGS_API void fem_solve_free(void* blob);

/* ---- session API ---------------------------------------------------------- */
typedef struct sgs_session sgs_session;

typedef struct {
  int32_t iterations;
  int32_t levels;
  double initial_residual; /* L-inf of the zero-guess residual */
  double final_residual;   /* L-inf of the last CG residual */
  double setup_seconds;
  double solve_seconds;    /* PCG only, host wall clock */
  int64_t launches_per_iteration;
  int64_t dof;             /* 3 * active level-0 nodes (the unknowns of the problem) */
  int64_t bottom_unknowns;
  double solve_device_seconds; /* PCG, CUDA events on the solver stream */
  int64_t kernel_launches;     /* kernels executed by the last solve */
  double h2d_bytes, d2h_bytes; /* host<->device bytes moved by the library so far */
} sgs_stats;

/* Build a session from an FEMInputs blob.  precision: 0 reference, 1 fp64, 2 mixed,
 * or SGS_HOST_SETUP_ONLY to build only the host-side hierarchy (no GPU needed;
 * the inspection calls below work, the solve calls return SGS_ERR_INPUT).
 * Returns 0 and *out, or an error code with a message in err. */
#define SGS_HOST_SETUP_ONLY 3
SGS_API int sgs_create(const void* input_blob, int precision, sgs_session** out, char* err, int errlen);
SGS_API void sgs_destroy(sgs_session* s);
SGS_API const char* sgs_last_error(sgs_session* s);

/* Run the PCG.  tolerance <= 0 keeps the blob's krylov.tolerance; max_iterations
 * <= 0 keeps 500.  Relative L-inf stopping rule (SPGrid_CPU_Solver.cpp:320-326). */
SGS_API int sgs_solve(sgs_session* s, double tolerance, int max_iterations, sgs_stats* stats);
SGS_API int sgs_residual_history(sgs_session* s, double* out, int cap);

/* Displacements per input block: out[nblocks][64][4] = (u_x, u_y, u_z, |r|_inf),
 * input block order and in-block index i*16 + j*4 + k (SPGrid_CPU_Solver.cpp:343-364). */
SGS_API int sgs_displacements(sgs_session* s, double* out);

/* SIMP compliance sensitivity after a solve (topo_opt/objective/minimal_compliance.cpp:86-146).
 * density: [nblocks][64] cell densities of the input blocks.  Writes
 * dc[nblocks][64] = p rho^(p-1) (1 - Emin) u_e^T K0 u_e and, when non-null,
 * element_energy[nblocks][64] = u_e^T K0 u_e (K0 with the material mu, lambda; no dx).
 * Returns the objective sum u_e^T K0 u_e (Emin + rho^p (1 - Emin)). */
SGS_API double sgs_sensitivity(sgs_session* s, const double* density, double* dc, double* element_energy);

/* Density-weighted sensitivity filter of the optimizer's driver, Opt::smooth_dc
 * (topo_opt/spgrid_topo_opt.cpp:527-579), on the input blocks of the session:
 * dc1 = sum_n w_n dc0_n rho_n / (sum_n w_n (rho + 1e-3)) over the cells n with
 * density > 0 inside the cube of half width floor(filter_size) (w = max(0,
 * filter_size - |offset|)); cells with density <= 0 get 0.  dc0 follows the
 * driver's sign (the gradient, -dc of sgs_sensitivity).  Host arrays [nblocks][64]. */
SGS_API int sgs_filter_sensitivity(sgs_session* s, const double* density, const double* dc0, double* dc1,
                                   double filter_size);

/* One optimality-criteria density update, OptimalityCriterion::optimize
 * (topo_opt/optimizer/optimality_criterion.cpp:19-145): bisection on the Lagrange
 * multiplier in [1e-20, 1e20] until lower*(1+1e-7) >= upper, new density
 * clamp(clamp(rho*sqrt(max(0, -dc0 - shift)/mid), rho -/+ step_limit),
 * minimum_density, 1) for cells with density > 0 (shift = min(0, min -dc0) when
 * smart_oc, else 0), fixed cells (fixed[i] != 0, may be NULL) set to fixed_density
 * and left out of the volume when exclude_fixed; the volume target is
 * volume_fraction x (container cells - counted fixed cells).  density
 * [nblocks][64] is updated in place; lagrange and max_change (may be NULL)
 * receive the multiplier and the largest density change. */
SGS_API int sgs_oc_update(sgs_session* s, double* density, const double* dc0, const uint8_t* fixed,
                          double volume_fraction, double step_limit, double minimum_density, double fixed_density,
                          int smart_oc, int exclude_fixed, double* lagrange, double* max_change);

/* The optimizer loop kept on the GPU.  The reference's driver runs one
 * Opt::iterate per step (topo_opt/spgrid_topo_opt.cpp:1289-1331): objective and
 * sensitivity, smooth_dc, the OC update, then the next fem_solve with the new
 * densities.  sgs_design_set uploads the design densities [nblocks][64] (and an
 * optional fixed-cell mask, which may be NULL); each sgs_design_step solves with
 * the current densities, computes the sensitivity, filters it, applies the OC
 * update (container cells kept at density >= DBL_MIN, as the driver's packing
 * does, spgrid_topo_opt.cpp:1122) and rebuilds the stiffness scales, coarse
 * operators and bottom inverse on the device; sgs_design_get copies the
 * densities back.  The material pattern of the session does not change. */
typedef struct sgs_design_params {
  double tolerance;        /* solve: relative L-inf residual */
  double volume_fraction;  /* OC volume target fraction */
  double step_limit;       /* OC move limit (0.2 in the driver) */
  double filter_size;      /* smooth_dc radius (1.5 in the driver) */
  double minimum_density;  /* OC lower bound */
  double fixed_density;    /* density of fixed cells */
  int32_t smart_oc;        /* shift by min(0, min -dc0) */
  int32_t exclude_fixed;   /* leave fixed cells out of the volume */
} sgs_design_params;

typedef struct sgs_design_result {
  double objective;             /* sum u_e^T K0 u_e (Emin + rho^p (1 - Emin)) before the update */
  double change;                /* largest density change of the OC update */
  double lagrange;              /* OC multiplier */
  int32_t cg_iterations;
  int32_t reserved;
  double solve_device_seconds;
  double solve_seconds;         /* host wall time of the solve */
  double step_seconds;          /* sensitivity, filter, OC and operator rebuild */
} sgs_design_result;

SGS_API int sgs_design_set(sgs_session* s, const double* density, const uint8_t* fixed);
SGS_API int sgs_design_step(sgs_session* s, const sgs_design_params* params, sgs_design_result* result);
SGS_API int sgs_design_get(sgs_session* s, double* density);

/* No counterpart in the reference.  Allocation-free variant of sgs_sensitivity
 * for callers that cannot allocate device memory while they run (frameworks
 * that own the allocator, code that must not call cudaMalloc/cudaFree once it
 * has started).  Like sgs_sensitivity it reads the displacements of the
 * session's last sgs_solve: call it after a solve (before one it reads zeros,
 * after a change of density it reads the previous solution).  All arrays are
 * caller-owned DEVICE buffers on the session's device, and that device must be
 * current (another current device returns SGS_ERR_INPUT):
 * density_dev[nblocks][64] in, dc_dev and element_energy_dev [nblocks][64] out,
 * objective_dev one double out.  The only scratch, the per-CTA partial sums of
 * the objective, lives in a static device array of
 * SGS_SENSITIVITY_STATIC_MAX_PARTIALS doubles that every GPU loading the
 * library holds until exit; problems with more than that many 256-cell CTAs
 * (nblocks * 64 > MAX * 256) are rejected with SGS_ERR_INPUT.  The session's
 * set-up (sgs_create) looks the array's device address up on its device, so
 * this call itself makes no lookup.  Every call reuses the same array: calls
 * that overlap on the GPU (other host threads, other sessions on the device)
 * race.  Synchronous; returns 0 or an error code (message in sgs_last_error). */
#define SGS_SENSITIVITY_STATIC_MAX_PARTIALS 16384
SGS_API int sgs_sensitivity_static(sgs_session* s, const double* density_dev, double* dc_dev,
                                   double* element_energy_dev, double* objective_dev);

/* Replace the densities of a resident problem ([nblocks][64], input block
 * order) keeping its material pattern (cells with density > 0): E, the Galerkin
 * operators and the bottom inverse are rebuilt, the hierarchy is kept.  Returns
 * SGS_ERR_INPUT when a cell's material status would change. */
SGS_API int sgs_set_density(sgs_session* s, const double* density);

/* ---- device-resident calls (the PyTorch layer) --------------------------- */
/* No counterpart in the reference (its driver owns host arrays only).  These
 * keep the differentiable compliance on the GPU: densities in, compliance and
 * gradient out, all as DEVICE buffers on the session's device, which must be
 * current.  caller_stream (a cudaStream_t, may be NULL for a device-wide
 * synchronization) is the stream that produced the inputs; the session's
 * stream waits for it, and each call returns when its results are complete.
 * Return 0 or an error code (message in sgs_last_error). */

/* Entries of the level-0 solution in the layout the gradient reads: 3 * nodes. */
SGS_API int64_t sgs_solution_size(sgs_session* s);
/* sgs_set_density from device memory ([nblocks][64], input block order): the
 * stiffness scales, Galerkin operators and bottom are rebuilt on the device;
 * SGS_ERR_INPUT when a cell's material status would change or a stiffness is
 * not finite (the session is then unchanged). */
SGS_API int sgs_set_density_device(sgs_session* s, const double* density_dev, void* caller_stream);
/* Copy the last solve's displacements (level-0 layout, sgs_solution_size entries). */
SGS_API int sgs_solution_device(sgs_session* s, double* u_dev, void* caller_stream);
/* out_dev[0] = f.u of the last solve: each loaded node once, with the force
 * the solve assembled for it (the last entry of a node, SPGrid_CPU_Solver.cpp:290-296). */
SGS_API int sgs_compliance_device(sgs_session* s, double* out_dev, void* caller_stream);
/* grad[nblocks][64] = factor * (*scale_dev) * p rho^(p-1) (1 - Emin) u_e^T K0 u_e
 * (topo_opt/objective/minimal_compliance.cpp:86-146), 0 for cells with rho <= 0;
 * u_dev is a saved solution (sgs_solution_device) or NULL for the last solve;
 * scale_dev may be NULL (1). */
SGS_API int sgs_sensitivity_device(sgs_session* s, const double* u_dev, const double* density_dev, double factor,
                                   const double* scale_dev, double* grad_dev, void* caller_stream);

/* ---- inspection and unit operators (tests) ------------------------------ */
SGS_API int sgs_level_count(sgs_session* s);
/* Active blocks of a level in SPGrid page order; coords may be null. */
SGS_API int sgs_level_blocks(sgs_session* s, int level, int32_t* coords);
SGS_API int sgs_level_flags(sgs_session* s, int level, uint32_t* flags);
SGS_API int sgs_boundary_blocks(sgs_session* s, int level, int32_t* ordinals);

/* Apply one operator to host arrays in the compact layout [3][nblocks*128]:
 *  0 level-0 K*u            1 level-0 residual b - K u
 *  2 one smoothing sweep    (arg bit0 forward, bit1 boundary band only)
 *  3 restriction level -> level+1     4 prolongation level+1 -> level (accumulate)
 *  5 stencil multiply       6 bottom solve (the V-cycle's last level, mg_level - 1)
 *  7 one V-cycle on level 0
 *  8 level-0 residual b - K u as the V-cycle computes it on its packed (u, E)
 *    iterate: in FP32 in mixed sessions (on the tensor cores with extra_ints
 *    "sgs_tensor_cores" = 1), FP64 otherwise; sessions whose V-cycle has more
 *    than one level */
SGS_API int sgs_apply(sgs_session* s, int op, int level, int arg, const double* in, const double* in2, double* out);

/* Galerkin stencils of a level as [nblocks*128][243] (row node, comp v; column
 * neighbour (i,j,k)-1, comp w at ((i*3+j)*3+k)*9 + v*3 + w) and spoke masks. */
SGS_API int sgs_level_stencils(sgs_session* s, int level, double* out, uint32_t* spokes);

/* Average device time (ms, CUDA events) of `reps` back-to-back runs of a level-0
 * operator on the session's resident data: 0 the PCG matvec q = K s (FP64, with
 * Project and the s.q partials), 1 residual, 2 one smoothing sweep (8 colours),
 * 3 one preconditioner application (V-cycle), 4 K u on the planar fields (on
 * the tensor cores when the session uses them), 5 the V-cycle's residual on
 * the tensor cores (mixed sessions).  Ops 1, 2, 4 and 5 run in the V-cycle's
 * precision (FP32 in mixed sessions). */
SGS_API int sgs_time_op(sgs_session* s, int op, int reps, double* ms);

/* Decode a blob and encode it again with this library's codec (which = 0 for
 * FEMInputs, 1 for FEMOutputs); *out receives a new[] blob for fem_solve_free.
 * Lets callers check byte compatibility without a GPU. */
SGS_API int sgs_codec_roundtrip(const void* blob, int which, void** out);

/* ---- narrow band: the optimizer driver's page maps ---------------------- */
/* The driver keeps its design on a grid of 4x4x4 blocks with four page maps
 * (topo_opt/spgrid_topo_opt.h:116-134): the container; the thin map, blocks that
 * still hold material; the fat map, whose cells the filter and the OC update
 * visit; the fatter map, the blocks packed into FEMInputs for fem_solve
 * (spgrid_topo_opt.cpp:1068-1160).  A band holds the container on the GPU
 * (blocks, per-cell flags and densities, FEMInputs density layout: cell
 * e = i*16 + j*4 + k of block b at b*64 + e) and the three maps as one byte per
 * block in the caller's block order.  Before the first update every map is the
 * whole container (spgrid_topo_opt.cpp:391-394). */
typedef struct sgs_band sgs_band;

/* Cell flag bits: TopOptFlags inside_container, has_force, fixed_density
 * (topo_opt/spgrid_topo_opt.h:30-42). */
#define SGS_CELL_INSIDE 1
#define SGS_CELL_FORCE 2
#define SGS_CELL_FIXED 4

typedef struct sgs_band_params {
  double minimum_density;         /* Opt::minimum_density */
  double active_threshold;        /* config "active_threshold" (driver default 1e-6) */
  double fraction_to_keep;        /* config "fraction_to_keep" (1.0: no selection) */
  int32_t fat_margin;             /* config "fat_margin" (default 1; 0..4 supported) */
  int32_t connectivity_filtering; /* config "connectivity_filtering" (default 1) */
} sgs_band_params;

typedef struct sgs_band_stats {
  int64_t container_blocks;
  int64_t thin_before_pruning; /* thin blocks before fraction_to_keep and the connectivity filter */
  int64_t thin_blocks, fat_blocks, fatter_blocks;
  int64_t components;          /* 6-connected components of the thin blocks (0 when not filtered) */
  int64_t active_voxels;       /* container cells of fatter blocks above active_threshold */
  double device_seconds;       /* the update on the GPU (CUDA events) */
  int64_t fat_changed;         /* blocks that entered or left the fat map (0: a session packed
                                  before the update still matches) */
} sgs_band_stats;

/* Replaces the driver's container set-up of the four maps
 * (spgrid_topo_opt.cpp:263-394): block_base[nblocks][3] are the container's
 * 4x4x4 block bases (multiples of 4 inside resolution), cell_flags and density
 * [nblocks][64].  Returns 0 and *out, or an error code with a message in err. */
SGS_API int sgs_band_create(const int32_t* block_base, int64_t nblocks, const int32_t resolution[3],
                            const uint8_t* cell_flags, const double* density, sgs_band** out, char* err,
                            int errlen);
SGS_API void sgs_band_destroy(sgs_band* b);
SGS_API const char* sgs_band_last_error(sgs_band* b);
SGS_API int sgs_band_set_density(sgs_band* b, const double* density);
SGS_API int sgs_band_get_density(sgs_band* b, double* density);
/* Replace the fat map the next update prunes from ([nblocks] bytes, 0/1). */
SGS_API int sgs_band_set_fat(sgs_band* b, const uint8_t* fat);

/* Replaces Opt::update_thin_page_map (spgrid_topo_opt.cpp:92-152), then, when
 * connectivity_filtering, Opt::filter_isolated_blocks (:1404-1510), then
 * Opt::update_fat_page_map (:154-241).  Where the reference stops (TC_ASSERT /
 * TC_ERROR: no thin block, not exactly one component above 30% of the thin
 * blocks, a fraction_to_keep selection beyond the fat list) this returns
 * SGS_ERR_INPUT with the maps unchanged.  stats may be NULL. */
SGS_API int sgs_band_update(sgs_band* b, const sgs_band_params* params, sgs_band_stats* stats);
/* Copy the maps out, one byte per container block; any pointer may be NULL. */
SGS_API int sgs_band_maps(sgs_band* b, uint8_t* thin, uint8_t* fat, uint8_t* fatter);
/* Copy the cell flags out ([nblocks][64]); the voxel filter and the kill change them. */
SGS_API int sgs_band_get_flags(sgs_band* b, uint8_t* cell_flags);

typedef struct sgs_band_voxel_stats {
  int64_t voxels;         /* container cells of the thin blocks (the search's total) */
  int64_t components;     /* their 6-connected components */
  int64_t kept, removed;  /* cells of the component kept / cells taken out of the container */
  double device_seconds;
} sgs_band_voxel_stats;

/* Replaces Opt::filter_isolated_voxels (spgrid_topo_opt.cpp:1512-1633), the
 * driver's "voxel_connectivity_filtering" action (:625-627): the 6-connected
 * components of the container cells of the thin blocks; with more than one,
 * the single component above 30% of those cells stays and every other cell
 * leaves the container with density 0.  The container voxel count behind the
 * volume target stays as it was, as in the reference.  No container cell in a
 * thin block, or not exactly one component above 30%, returns SGS_ERR_INPUT
 * with nothing changed.  stats may be NULL. */
SGS_API int sgs_band_filter_voxels(sgs_band* b, sgs_band_voxel_stats* stats);
/* The first loop of Opt::threshold_and_kill (spgrid_topo_opt.cpp:1333-1344):
 * every container cell with density below threshold leaves the container (its
 * density stays).  The reference's action then runs the voxel filter and a
 * page-map update without the block filter (:1341-1343); chain
 * sgs_band_filter_voxels and sgs_band_update for that.  killed may be NULL. */
SGS_API int sgs_band_kill_below(sgs_band* b, double threshold, int64_t* killed);
/* Replaces Opt::threshold_density (spgrid_topo_opt.cpp:1780-1797) and, with a
 * threshold >= 0, Opt::threshold_density_trail(threshold, true) (:1756-1778):
 * every cell of the fat blocks whose density is >= the threshold, or that has a
 * fixed density, becomes 1, every other cell of those blocks 0.  A negative
 * threshold asks for the reference's bisection on [0, 1] (until lo + 1e-8 >= hi)
 * against volume_fraction x the container voxel count; the threshold used and
 * the solid voxel count come back (either pointer may be NULL). */
SGS_API int sgs_band_threshold_density(sgs_band* b, double volume_fraction, double threshold,
                                       double* threshold_used, int64_t* solid_voxels);

/* The driver's iteration on a band.  A session holds the fatter blocks as the
 * driver packs them into FEMInputs (spgrid_topo_opt.cpp:1068-1160): its input
 * block i is container block container_block[i], its cells hold max(density,
 * DBL_MIN) in the container cells of fat blocks and 0 elsewhere.
 * sgs_band_attach checks that and binds the two; build a new session (and
 * attach it) whenever an update changes the fat map.
 * sgs_band_step then runs Opt::iterate after its page-map update
 * (spgrid_topo_opt.cpp:1301-1330): clear_gradients over the fat blocks, the
 * solve, the compliance sensitivity of the fat container cells
 * (minimal_compliance.cpp:74-146), smooth_dc over the fat blocks (:527-579,
 * neighbours read from the whole container, stale values included), the OC
 * update over the fat container cells with the volume target taken against all
 * container cells (optimality_criterion.cpp:19-145; fixed cells from
 * SGS_CELL_FIXED), and the session's new stiffness scales.  The densities stay
 * on the band (sgs_band_get_density). */
SGS_API int sgs_band_attach(sgs_band* b, sgs_session* s, const int64_t* container_block);
/* Pack and build that session from the band's current maps and densities and
 * attach it, in one call: template_blob is an FEMInputs blob whose settings,
 * forces and Dirichlet nodes are used as they are (its density grid is
 * ignored; an empty one keeps the blob small).  precision as for sgs_create. */
SGS_API int sgs_band_session(sgs_band* b, const void* template_blob, int precision, sgs_session** out, char* err,
                             int errlen);
SGS_API int sgs_band_step(sgs_band* b, sgs_session* s, const sgs_design_params* params, sgs_design_result* result);

/* ---- headless density renderer ------------------------------------------ */
/* The reference's visualiser (misc/volume_rendering_kernel.cu:340-437 with
 * misc/volume_renderer.cpp:410-480) without window, OpenGL buffer or texture
 * unit.  The cells with positive density span the volume (their bounding box,
 * one voxel per cell: 0 for density 0, else uchar(d * 254) + 1); camera rays
 * are traced per pixel and `frames` jittered frames are averaged.  mode 0:
 * surface, the first voxel above `threshold` shaded by three ambient-occlusion
 * rays under a two-colour sky; mode 1: volume, exp(-extinction *
 * max(0.01 * sum of 1025 jittered samples - threshold, 0)).  Random numbers
 * come from a counter-based hash of (pixel, frame, seed).  rgba[height][width]
 * receives (a << 24 | b << 16 | g << 8 | r), row 0 at the bottom as in the
 * reference's pixel buffer. */
typedef struct sgs_render_params {
  int32_t width, height;
  int32_t mode;            /* 0 surface, 1 volume */
  int32_t frames;          /* >= 1, the reference's progressive sample counter */
  float threshold;         /* surface: solid above; volume: subtracted from the integral */
  float extinction;        /* volume only */
  float slice;             /* cut along z: 0.99999 shows the whole volume */
  uint32_t seed;
  float camera[12];        /* 3x4 rows: camera-to-world rotation | eye position (c_invViewMatrix) */
  int32_t reverse_mapping; /* 1: densities are SIMP stiffness (penalty 0): d -> (d - 1e-6)^(1/3) (1 - 1e-6) */
  int32_t mirror;          /* bits 0-2: show the volume mirrored across its +x, +y, +z face (the viewer's
                              mirroring, volume_rendering_kernel.cu:133-143, volume_renderer.cpp set_mirroring) */
} sgs_render_params;

/* Host arrays in the FEMInputs density layout; volume_res (may be NULL)
 * receives the volume's size. */
SGS_API int sgs_render(const int32_t* block_base, int64_t nblocks, const double* density, const sgs_render_params* p,
                       uint32_t* rgba, int32_t* volume_res);
/* The same for a band's current densities, without a host round trip. */
SGS_API int sgs_band_render(sgs_band* b, const sgs_render_params* p, uint32_t* rgba, int32_t* volume_res);

#ifdef __cplusplus
}
#endif
#endif
