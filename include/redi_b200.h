/*
 * redi_b200.h — C-ABI of the B200-native Redi neutral-diffusion step.
 *
 * Drop-in boundary for the reference's `ocean_redi` module
 * (JorgeG94/more_benchmarks_dc_ocean, redi/ocean_redi.F90). Two layers:
 *
 *  1. A handle API that mirrors the Fortran public interface one to one:
 *       ocean_redi_t%init / %destroy       -> redi_b200_init / redi_b200_destroy
 *       redi_calc_coeffs(grid, metrics, eos, this, ms)
 *                                          -> redi_b200_calc_coeffs
 *       redi_apply_flux(grid, metrics, this, ms, dt, khtr_u_ext, khtr_v_ext, bc)
 *                                          -> redi_b200_apply_flux
 *     The structs mirror the derived types the Fortran passes (hgrid_t,
 *     ocean_metrics_t, ocean_eos_t, multilayer_cgrid_state_t, ocean_bc_state_t).
 *     Array arguments are DEVICE pointers (what `!$acc host_data use_device`
 *     or `c_loc` of a device array yields), column-major with the reference
 *     shapes. Calls are stream-ordered on `stream` (a cudaStream_t; NULL = the
 *     legacy default stream) and do not synchronise.
 *
 *  2. Exports with the exact signatures of the reference's CUDA launchers
 *     (redi/opt_kernel.cu:534-549 `redi_opt_launch`, redi/redi_kernel.cu:537-549
 *     `redi_cuda_launch_`), so the reference's bridge (redi/drivers/redi_bridge.F90)
 *     and RK2 harness (ideal_benchmark/wrap/rk2_redi.F90) link unchanged.
 *
 * Status codes: >= 0 success (REDI_B200_SKIPPED = a reference gate made the call
 * a no-op, exactly where the Fortran returns early), < 0 error; the message of
 * the last error on the calling thread is redi_b200_last_error().
 */
#ifndef REDI_B200_H
#define REDI_B200_H

#if defined(__GNUC__)
#define REDI_B200_API __attribute__((visibility("default")))
#else
#define REDI_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define REDI_B200_OK 0
#define REDI_B200_SKIPPED 1
#define REDI_B200_E_ARG (-1)
#define REDI_B200_E_STATE (-2)
#define REDI_B200_E_CUDA (-3)
#define REDI_B200_E_NOMEM (-4)
#define REDI_B200_E_UNSUPPORTED (-5)

/* Arithmetic of the step. FP64: bit-identical to the reference with FMA
 * contraction off. MIXED: FP32 reconstruction / flux arithmetic and compact
 * coefficient storage, FP64 density differences, slope denominators and
 * tracer accumulation. */
#define REDI_B200_FP64 0
#define REDI_B200_MIXED 1

#define REDI_B200_OBC_WALL 1 /* redi/ocean_boundary_types.F90:14 OBC_WALL */

/* hgrid_t (redi/grid.F90:17-25). */
typedef struct redi_b200_grid {
    int nx_total, ny_total; /* cells incl. ghosts: n_phys + 2*nghost */
    int nx_phys, ny_phys;
    int nghost;
    double dx, dy;
} redi_b200_grid;

/* ocean_metrics_t (redi/ocean_metrics.F90:14-22); device pointers. */
typedef struct redi_b200_metrics {
    const double* dy_cu; /* (nx+1, ny) */
    const double* dx_cv; /* (nx, ny+1) */
    const double* idxCu; /* (nx+1, ny) */
    const double* idyCv; /* (nx, ny+1) */
    const double* areaT; /* (nx, ny)   */
    const double* wet_u; /* (nx+1, ny) */
    const double* wet_v; /* (nx, ny+1) */
} redi_b200_metrics;

/* ocean_eos_t (redi/ocean_eos.F90:239-278). variant takes the reference's
 * codes (ocean_eos.F90:39-51): REDI_B200_EOS_LINEAR (0 is accepted as LINEAR,
 * a zero-initialised struct), REDI_B200_EOS_WRIGHT_97, REDI_B200_EOS_ROQUET_SPV;
 * 3 (TEOS-10) is reserved in the reference and rejected with E_UNSUPPORTED.
 * The linear coefficients are read by the LINEAR branch only; rho0 also sets
 * the hydrostatic interface pressure for every variant (ocean_redi.F90:643-646). */
#define REDI_B200_EOS_LINEAR 1
#define REDI_B200_EOS_WRIGHT_97 2
#define REDI_B200_EOS_ROQUET_SPV 4
typedef struct redi_b200_eos {
    int variant;
    double rho0, T_ref, S_ref, alpha_T, beta_S;
} redi_b200_eos;

/* multilayer_cgrid_state_t (redi/multilayer_cgrid_state.F90:18-28).
 * idx_temperature / idx_salinity are 1-based indices into hTr (0 = not
 * registered), as in the Fortran. hTr is a HOST array of ntracers DEVICE
 * pointers, each an (nx, ny, nz_ml) thickness-weighted tracer. */
typedef struct redi_b200_state {
    int nz_ml;
    int idx_temperature, idx_salinity;
    int ntracers;
    const double* h_layer; /* (nx, ny, nz_ml), k=1 the bed */
    double* const* hTr;
} redi_b200_state;

/* ocean_bc_state_t (redi/ocean_boundary_types.F90:20-24): bc_type per edge. */
typedef struct redi_b200_bc {
    int west, east, south, north;
} redi_b200_bc;

/* Device pointers of the Phase-A coefficient slots held by a handle
 * (ocean_redi_t%uPoL ... %vhEff, ocean_redi.F90:105-110), FP64 handles only. */
typedef struct redi_b200_coeffs {
    double *uPoL, *uPoR, *uhEff;
    int *uKoL, *uKoR;
    double *vPoL, *vPoR, *vhEff;
    int *vKoL, *vKoR;
    double *khtr_u, *khtr_v;
    int nsurf;
} redi_b200_coeffs;

typedef struct redi_b200 redi_b200; /* ocean_redi_t */

/* ocean_redi_init (ocean_redi.F90:466-507): allocate the coefficient slots for
 * grid%nx_total x grid%ny_total x nz_ml (nz_ml < 1 is taken as 1) and set them
 * to the inert state (Po = 0, Ko = 1, hEff = 0). Fails with E_UNSUPPORTED where
 * the reference's init `error stop`s (the column is longer than the kernels
 * support). The new handle has enable = 0 and khtr = 0, like the Fortran. */
REDI_B200_API int redi_b200_init(const redi_b200_grid* grid, int nz_ml, int precision, redi_b200** out);

/* ocean_redi_destroy (ocean_redi.F90:509-529). NULL is accepted. */
REDI_B200_API int redi_b200_destroy(redi_b200* self);

/* ocean_redi_t%enable, %khtr (ocean_redi.F90:78-87). */
REDI_B200_API int redi_b200_set_enable(redi_b200* self, int enable);
REDI_B200_API int redi_b200_set_khtr(redi_b200* self, double khtr);

/* redi_calc_coeffs (ocean_redi.F90:572-607). */
REDI_B200_API int redi_b200_calc_coeffs(const redi_b200_grid* grid, const redi_b200_metrics* metrics, const redi_b200_eos* eos,
                          redi_b200* self, const redi_b200_state* ms, void* stream);

/* redi_apply_flux (ocean_redi.F90:927-1002). khtr_u_ext / khtr_v_ext (device,
 * (nx+1,ny) / (nx,ny+1)) are optional: both non-NULL selects the per-face path,
 * otherwise the scalar khtr is broadcast. bc may be NULL (all edges WALL).
 * Every tracer of ms is updated, all in one fused pass. */
REDI_B200_API int redi_b200_apply_flux(const redi_b200_grid* grid, const redi_b200_metrics* metrics, redi_b200* self,
                         const redi_b200_state* ms, double dt, const double* khtr_u_ext, const double* khtr_v_ext,
                         const redi_b200_bc* bc, void* stream);

/* redi_b200_calc_coeffs followed by redi_b200_apply_flux on a model state held
 * in HOST memory (no counterpart in the reference, whose CPU build keeps its
 * state on the host and steps it there): ms->h_layer and ms->hTr[t] are host
 * pointers to the (nx, ny, nz) fields, read and updated in place; metrics and
 * khtr_u_ext/khtr_v_ext stay device pointers. The step is pipelined over
 * nbands bands of rows (1..64): rows are copied up on one stream, each band
 * is stepped as soon as its rows and the next row are on the device, and
 * finished rows are copied back on a third stream, so host<->device traffic
 * overlaps the kernels and itself. With nbands >= 3 and at least 4 rows per
 * band the last two bands are a half and a quarter of the others (the last
 * band's kernels and download start only when every row is up, so a short
 * last band shortens the step). Results equal the two device entry points
 * bit for bit. Stream-ordered on `stream`: the host arrays are in use until
 * the stream reaches this call's end; page-locked host memory is needed for
 * the copies to overlap. Each phase keeps its own gates; SKIPPED when both
 * are gated. The handle holds device copies of h and of every tracer (twice)
 * from the first call on. */
REDI_B200_API int redi_b200_step_host(const redi_b200_grid* grid, const redi_b200_metrics* metrics,
                                      const redi_b200_eos* eos, redi_b200* self, const redi_b200_state* ms,
                                      double dt, const double* khtr_u_ext, const double* khtr_v_ext,
                                      const redi_b200_bc* bc, int nbands, void* stream);

/* One whole step: redi_b200_calc_coeffs followed by redi_b200_apply_flux on
 * the same state, with the same arguments, gates, status and results (bit for
 * bit). No counterpart in the reference as one routine (its driver calls the
 * two in turn; its redi_opt_launch does both). Since nothing can change the
 * tracers between the phases, when tracers 1 and 2 are T and S (either order)
 * the column state of Phase A and the reconstruction of T and S for Phase B
 * are computed in one pass over the columns. Stream-ordered on `stream`. */
REDI_B200_API int redi_b200_step(const redi_b200_grid* grid, const redi_b200_metrics* metrics,
                                 const redi_b200_eos* eos, redi_b200* self, const redi_b200_state* ms, double dt,
                                 const double* khtr_u_ext, const double* khtr_v_ext, const redi_b200_bc* bc,
                                 void* stream);

/* Device pointers of the handle's coefficient slots (FP64 handles). The handle
 * keeps a record of the faces whose slots hold inert coefficients (dry faces:
 * redi_calc_coeffs does not rewrite them while they stay dry, and
 * redi_apply_flux does not walk them); since the caller may write into the
 * slots through these pointers, this call clears that record (and waits for
 * the device), so later steps give the reference's results for whatever the
 * slots then hold. */
REDI_B200_API int redi_b200_get_coeffs(const redi_b200* self, redi_b200_coeffs* out);

/* Bytes of device scratch the handle holds beside its coefficient slots. */
REDI_B200_API long long redi_b200_workspace_bytes(const redi_b200* self);

/* Number of coefficient sublayers the cell update found out of order (cell-side
 * Ko decreasing along a face, or outside 1..nz) since the last reset; always 0
 * for coefficients produced by redi_b200_calc_coeffs. Synchronises the device.
 * reset != 0 zeroes the count. (No counterpart in the reference.) */
REDI_B200_API int redi_b200_error_count(const redi_b200* self, int reset);

/* Message of the last error on the calling thread ("" if none). */
REDI_B200_API const char* redi_b200_last_error(void);

/* Library version: major*10000 + minor*100 + patch. */
REDI_B200_API int redi_b200_version(void);

/* Instrumentation (no counterpart in the reference). Kernel ids are
 * 0 column_state, 1 neutral_sweep, 2 tracer_recon, 3 cell_gather (the per-cell
 * update), 4 face_flux, 5 mixed_recon, 6 mixed_flux, 7 mixed_sweep,
 * 8 domain_persistent, 9 auxiliary, and the MEKE step's (meke_b200.h) 10 pass A,
 * 11 biharmonic Laplacian, 12 pass B, and the ALE remap step's (ale_b200.h) 13 column
 * tiles, 14 face tiles, then 15 flux_fold and 16 mixed_fold (the fused Phase-B
 * pass); redi_b200_kernel_count() is their number.
 * redi_b200_launch_count(k) counts launches of kernel k since load (k < 0:
 * all). Between profile_begin and profile_end every launch is bracketed by a
 * CUDA event pair on its own stream; profile_end waits for them and returns,
 * per kernel id, the summed device time (ms) and the number of launches. */
REDI_B200_API int redi_b200_kernel_count(void);

/* Launch shape of the Phase-B cell update, process-wide (no counterpart in the
 * reference): a bx x by tile of T-cell columns per block (bx*by a multiple of
 * 32, at most 128) and the vertical chunk of layers processed per face pass
 * (4, 8 or 16). Results do not depend on it; the autotuner picks it. */
REDI_B200_API int redi_b200_set_tuning(int bx, int by, int chunk);
REDI_B200_API int redi_b200_get_tuning(int* bx, int* by, int* chunk);

/* eos_density_point and eos_specvol_derivs (redi/ocean_eos.F90:450-546), the
 * reference's public point routines, at n points: T, S, p (Pa) and the outputs
 * rho, dSV/dT, dSV/dS are device arrays of n doubles. The values are exactly
 * those the column state uses at each interface. Stream-ordered. */
REDI_B200_API int redi_b200_eos_points(const redi_b200_eos* eos, int n, const double* T, const double* S,
                                       const double* p, double* rho, double* dsv_dt, double* dsv_ds, void* stream);

/* Largest number of tracers whose face fluxes one launch computes (1, 2, 4
 * or 8; default 8), process-wide (no counterpart in the reference). Larger
 * groups read the Phase-A coefficients fewer times per step, smaller ones run
 * at higher occupancy; results do not depend on it. */
REDI_B200_API int redi_b200_set_tracer_group(int max_group);
REDI_B200_API int redi_b200_get_tracer_group(void);

/* Tracers one cell-gather launch folds (2, 4 or 8; default 2) and where it
 * keeps a chunk's per-layer sums (smem = 1, the default: the thread's slots in
 * shared memory, one load-add-store per flux; 2: the same, fetching 8
 * sublayers per round trip instead of 3 or 4; 3: the same with batches of 4
 * software-pipelined, the next batch in flight while one is folded; 0:
 * registers, a select-add over the chunk), process-wide (no counterpart in the
 * reference). 4 tracers read
 * the cell-side Ko half as often as 2. 8 folds the fluxes of two face-flux
 * launches of 4 tracers in one walk; it applies with face-flux groups of 4,
 * shared-memory sums, 4-layer chunks and 128-thread tiles (else 4 is used).
 * Results do not depend on either choice.
 * get returns n and writes the smem choice if the pointer is non-NULL. */
REDI_B200_API int redi_b200_set_gather_tracers(int n, int smem);
REDI_B200_API int redi_b200_get_gather_tracers(int* smem);

/* Face flux form, process-wide (no counterpart in the reference): 0 loads each
 * sublayer's reconstruction values when needed; 1 copies the next sublayer's
 * into shared memory (cp.async) while the current one is evaluated (caps the
 * face-flux tracer group at 2); 2 reads each column's reconstruction through a
 * two-layer ring in shared memory, the layer below fetched when a side enters a
 * layer (caps the group at 4). Results do not depend on it. */
REDI_B200_API int redi_b200_set_flux_staged(int on);
REDI_B200_API int redi_b200_get_flux_staged(void);
/* Neutral sweep form, process-wide (no counterpart in the reference): 0 keeps
 * each column's three-interface window in registers with a shared-memory
 * look-ahead ring; 3, 4 (the default) or 5 keeps both windows in a per-thread
 * shared-memory ring of 3, 4 or 5 interfaces (none, one or two in flight), read
 * through one code path whichever column the step advances. Results do not
 * depend on it. */
REDI_B200_API int redi_b200_set_sweep_form(int form);
REDI_B200_API int redi_b200_get_sweep_form(void);
/* Phase B as one fused pass per tile of cells (no counterpart in the
 * reference), process-wide: every face's sublayer fluxes are computed once per
 * tile and added to the cells' tendencies in shared memory, so no flux buffer
 * crosses HBM and all tracers go through one launch. enable is a mask: bit 0
 * runs the FP64 form this way, bit 1 the mixed form, bit 2 makes the mixed form
 * add in the reference's order too. The FP64 form always adds in the
 * reference's order (results bit-identical to the face-flux + cell-gather pair
 * it replaces); the mixed form otherwise adds each term as soon as it is
 * computed (shared-memory atomics: the same terms, FP64 accumulation, in an
 * order that can differ from run to run by the last bits). rows: cell rows per
 * tile (1 or 2); tracers: tracers per pass (1, 2, 4, or 0 for the most that
 * keep two tiles per SM). Off by default (the pair runs; rows = 2).
 * redi_b200_fold_shape reports the (rows, tracers) a step of the given
 * precision, nz and tracer count runs with; tracers = 0 means the pair runs
 * (the fused pass is off for that form, or its shared memory would not fit:
 * very deep columns). Kernel ids 15 (FP64) and 16 (mixed) time it. */
REDI_B200_API int redi_b200_set_fold(int enable, int rows, int tracers);
REDI_B200_API int redi_b200_get_fold(int* enable, int* rows, int* tracers);
REDI_B200_API int redi_b200_fold_shape(int precision, int nz, int ntracers, int* rows, int* tracers);
REDI_B200_API unsigned long long redi_b200_launch_count(int kernel);
REDI_B200_API int redi_b200_profile_begin(void);
REDI_B200_API int redi_b200_profile_end(double* total_ms, unsigned long long* counts, int n);

/* Same signature, argument meaning and launch sequence as the reference's
 * optimized launcher (redi/opt_kernel.cu:534-574): Phase A into the caller's
 * u/v slots, khtr_u/v = khtr_*_ext, then Phase B for T (t_htr) and S (s_htr);
 * synchronises the device before returning. All arrays are device pointers,
 * all scalars by reference (Fortran default). tr_snap is accepted and not
 * written (the fused Phase B reads pre-step tracers from its own scratch).
 * Like the reference it returns nothing: argument errors are reported through
 * redi_b200_last_error() and stderr, and no kernel is launched. */
REDI_B200_API void redi_opt_launch(const int* nx, const int* ny, const int* nz, const int* ns, const double* dt,
                     const int* nghost, const int* nxp, const int* nyp, const int* ww, const int* we,
                     const int* wsz, const int* wn, const double* rho0, const double* T_ref, const double* S_ref,
                     const double* alpha_T, const double* beta_S, const double* h_layer, double* t_htr,
                     double* s_htr, const double* wet_u, const double* wet_v, double* uPoL, double* uPoR,
                     int* uKoL, int* uKoR, double* uhEff, double* vPoL, double* vPoR, int* vKoL, int* vKoR,
                     double* vhEff, const double* khtr_u_ext, const double* khtr_v_ext, double* khtr_u,
                     double* khtr_v, const double* dy_cu, const double* dx_cv, const double* idxCu,
                     const double* idyCv, const double* areaT, double* tr_snap);

/* The reference's faithful launcher name (redi/redi_kernel.cu:537-549); same
 * behaviour as redi_opt_launch (the two reference launchers are bit-identical). */
REDI_B200_API void redi_cuda_launch_(const int* nx, const int* ny, const int* nz, const int* ns, const double* dt,
                       const int* nghost, const int* nxp, const int* nyp, const int* ww, const int* we,
                       const int* wsz, const int* wn, const double* rho0, const double* T_ref, const double* S_ref,
                       const double* alpha_T, const double* beta_S, const double* h_layer, double* t_htr,
                       double* s_htr, const double* wet_u, const double* wet_v, double* uPoL, double* uPoR,
                       int* uKoL, int* uKoR, double* uhEff, double* vPoL, double* vPoR, int* vKoL, int* vKoR,
                       double* vhEff, const double* khtr_u_ext, const double* khtr_v_ext, double* khtr_u,
                       double* khtr_v, const double* dy_cu, const double* dx_cv, const double* idxCu,
                       const double* idyCv, const double* areaT, double* tr_snap);

/* The reference-compatible step without any device allocation. No counterpart
 * in the reference. For callers that must not call cudaMalloc/cudaFree while
 * stepping: those calls can synchronise the whole device, cannot run while a
 * stream is being captured, and some host models hand out all device memory
 * from their own pool. Arguments and results are those of redi_opt_launch (all
 * arrays device pointers, scalars by reference; tr_snap is not written), plus
 * the stream to run on (NULL: legacy default stream); the call is
 * stream-ordered and does not synchronise.
 * Scratch comes from one 64 MiB array inside the library, held on every GPU
 * that loads the library until exit, and shared by all calls: calls that
 * overlap on the GPU race on it, so issue them in stream order. Its device
 * address is resolved by the first call on each device: make that call before
 * any stream capture. A domain whose scratch exceeds 64 MiB (about 18 000
 * columns at nz = 25, 6 000 at nz = 75) is refused with
 * REDI_B200_E_UNSUPPORTED; the message (redi_b200_last_error) gives the
 * limit. The array pointers are checked as redi_opt_launch checks them
 * (doubles 8-byte, the int Ko slots 4-byte aligned). Its Phase B uses the
 * coefficients its own Phase A just made, which are never out of order, so no
 * out-of-order count is kept for it (redi_b200_error_count is per handle).
 * The device address of the array is cached per device index for the life of
 * the process: do not call it again on a device after cudaDeviceReset.
 * Returns REDI_B200_OK or a negative status. */
REDI_B200_API int redi_b200_opt_launch_noalloc(
    const int* nx, const int* ny, const int* nz, const int* ns, const double* dt, const int* nghost, const int* nxp,
    const int* nyp, const int* ww, const int* we, const int* wsz, const int* wn, const double* rho0,
    const double* T_ref, const double* S_ref, const double* alpha_T, const double* beta_S, const double* h_layer,
    double* t_htr, double* s_htr, const double* wet_u, const double* wet_v, double* uPoL, double* uPoR, int* uKoL,
    int* uKoR, double* uhEff, double* vPoL, double* vPoR, int* vKoL, int* vKoR, double* vhEff,
    const double* khtr_u_ext, const double* khtr_v_ext, double* khtr_u, double* khtr_v, const double* dy_cu,
    const double* dx_cv, const double* idxCu, const double* idyCv, const double* areaT, double* tr_snap,
    void* stream);

/* Halo packing for a domain split into tiles (no counterpart in the reference,
 * which steps one undivided domain): copies column `index` (axis 0) or row
 * `index` (axis 1) of each of the nfields (nx, ny, nz) fields (device
 * pointers; at most 65) into the device buffer buf (to_buf != 0), field after
 * field, nz x ny or nz x nx values each, layer-major; or from buf back into the
 * fields (to_buf == 0). One launch, stream-ordered. */
REDI_B200_API int redi_b200_halo_copy(double* const* fields, int nfields, int nx, int ny, int nz, int axis, int index,
                                      double* buf, int to_buf, void* stream);

/* ---------------------------------------------------------------------------
 * Many independent regional domains stepped by one persistent kernel (no
 * counterpart in the reference, whose driver steps one domain per call). The
 * step of every domain (redi_calc_coeffs then redi_apply_flux for all of its
 * tracers) is cut into tiles of columns, faces and cells; one grid of resident
 * blocks drains that work queue, largest domains first, each tile starting
 * once the previous stage of its own domain is complete. Per domain the
 * results equal those of redi_b200_calc_coeffs + redi_b200_apply_flux on a
 * handle of the same precision, bit for bit.
 * ------------------------------------------------------------------------- */
#define REDI_B200_STATUS_TIMEOUT 1 /* a tile waited longer than the wait limit */

/* One domain: what redi_b200_calc_coeffs and redi_b200_apply_flux take. The
 * per-face diffusivities are required (khtr_u_ext / khtr_v_ext non-NULL); ms
 * needs 2..64 tracers with T and S registered. All arrays stay owned by the
 * caller and must outlive the batch; their addresses are baked into it. */
typedef struct redi_b200_domain {
    redi_b200_grid grid;
    redi_b200_metrics metrics;
    redi_b200_eos eos;
    redi_b200_state ms;
    const double* khtr_u_ext;
    const double* khtr_v_ext;
    redi_b200_bc bc;
    double dt;
} redi_b200_domain;

typedef struct redi_b200_batch redi_b200_batch;

/* Builds the batch: Phase-A coefficient slots and scratch per domain, the work
 * queue, and the persistent grid (as many 128-thread blocks as are resident on
 * the current device). tile_bx x tile_by (= 128) is the cell tile of the
 * gather, chunk (4, 8, 16) its vertical chunk. use_graph != 0 captures the step
 * (counter reset + persistent kernel) in a CUDA graph on the first
 * redi_b200_batch_step and replays it afterwards. Synchronises the device. */
REDI_B200_API int redi_b200_batch_create(int ndomains, const redi_b200_domain* domains, int precision, int tile_bx,
                                         int tile_by, int chunk, int use_graph, redi_b200_batch** out);

/* One step of every domain, stream-ordered on stream; does not synchronise. */
REDI_B200_API int redi_b200_batch_step(redi_b200_batch* b, void* stream);

/* Outcome of the last step (synchronous read): status 0 or
 * REDI_B200_STATUS_TIMEOUT, with the domain and stage (0 column state,
 * 1 neutral sweep, 2 tracer reconstruction, 3 + 2g / 4 + 2g face flux / gather
 * of tracer pair g) of the first tile that gave up; bad = fluxes the gather
 * found out of order (0 for coefficients made in the step). Any out pointer
 * but status may be NULL. After a timeout the step's results are incomplete. */
REDI_B200_API int redi_b200_batch_status(const redi_b200_batch* b, int* status, int* domain, int* stage, int* bad);

/* Launch shape of an existing batch (tile and chunk as in
 * redi_b200_batch_create; occupancy = resident blocks per SM the kernel's
 * registers are budgeted for, 4, 5 or 6, 0 keeps the current one, 4 at
 * creation). Results do not depend on it. Rebuilds the work queue, keeps every
 * domain's memory; synchronises the device. get_tuning also returns the
 * persistent grid size (blocks). */
REDI_B200_API int redi_b200_batch_set_tuning(redi_b200_batch* b, int tile_bx, int tile_by, int chunk, int occupancy);
REDI_B200_API int redi_b200_batch_get_tuning(const redi_b200_batch* b, int* tile_bx, int* tile_by, int* chunk,
                                             int* occupancy, int* grid);

/* Per-stage accounting of the last step (off by default): with on != 0 the
 * kernel sums, per stage kind (0 column state, 1 neutral sweep, 2 tracer
 * reconstruction, 3 face flux, 4 gather), the time blocks waited for
 * predecessors and spent on tiles (ms, summed over blocks) and the tiles done.
 * stage_times synchronises the device; any out array may be NULL. */
REDI_B200_API int redi_b200_batch_set_accounting(redi_b200_batch* b, int on);
REDI_B200_API int redi_b200_batch_stage_times(const redi_b200_batch* b, double* wait_ms, double* busy_ms,
                                              long long* tiles);

/* Longest time a tile waits for its predecessors, in ns (default 2e9). */
REDI_B200_API int redi_b200_batch_set_wait_limit(redi_b200_batch* b, long long ns);

/* Fault injection for tests: hold != 0 keeps the domain's first stage waiting
 * on a release flag that nothing sets while the step runs, so the step ends
 * with REDI_B200_STATUS_TIMEOUT after the wait limit. */
REDI_B200_API int redi_b200_batch_hold(redi_b200_batch* b, int domain, int hold);

/* Tracer-cell updates per step (physical cells x layers x tracers, summed),
 * and the number of tiles in the work queue. */
REDI_B200_API long long redi_b200_batch_updates(const redi_b200_batch* b);
REDI_B200_API long long redi_b200_batch_items(const redi_b200_batch* b);

/* Frees the batch's device memory and graph. NULL is accepted. */
REDI_B200_API int redi_b200_batch_destroy(redi_b200_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* REDI_B200_H */
