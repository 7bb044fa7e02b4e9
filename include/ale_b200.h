/*
 * ale_b200.h — C-ABI of the B200-native ALE remap step (the vertical remap that
 * runs in the same RK2 stage as the Redi step).
 *
 * Drop-in boundary for the reference's `ale_remap_step` (JorgeG94/more_benchmarks_dc_ocean,
 * ale_remap/ale_remap.F90:76-188, production's `ocean_apply_ale_remap_step`):
 * zstar target thicknesses, conservative remap of every tracer (heat / salt
 * budgets for T and S), remap of the u / v face velocities (optional
 * KE-conserving rescale), mass budget, h commit and bt_eta. Two layers:
 *
 *  1. Exports with the exact signatures of the reference's CUDA launchers, so
 *     its native driver (ale_remap/drivers/cpp_main.cu) links unchanged:
 *       ale_remap_cuda(...)  ale_remap/ale_kernel.cu:453-482
 *       ale_remap_opt(...)   ale_remap/opt_kernel.cu:399-413
 *       cuda_sync()          ale_remap/ale_kernel.cu:37
 *     Like the reference's they are asynchronous on the legacy default stream
 *     (cuda_sync() waits). Argument errors are printed to stderr and kept for
 *     ale_b200_last_error(); nothing is launched then.
 *
 *  2. ale_b200_remap_step (no counterpart in the reference's C-ABI): the
 *     Fortran routine's full interface — any number of tracer slots, the
 *     remap method, the KE switch, optional face velocities — stream-ordered.
 *
 * Methods are the reference's codes (ale_remap/constants.F90:22-26): 1 PCM,
 * 2 PLM, 3 PPM (the default and the one its CUDA implements); 4 PPM_H4 and
 * 5 PQM are rejected (ALE_B200_E_UNSUPPORTED); any other code takes the
 * select-case default, PLM (kernel_remap.F90:54-67). The reference's CUDA
 * launchers ignore `method` and always run PPM; these exports honour it.
 *
 * Arrays are DEVICE pointers, Fortran column-major: cells (nx, ny), layers
 * (nx, ny, nz), u faces (nx+1, ny, nz), v faces (nx, ny+1, nz), dsig (nz).
 * nz is at most ALE_B200_NZ_MAX (the reference's NZ_STACK_MAX). All FP64.
 */
#ifndef ALE_B200_H
#define ALE_B200_H

#if defined(__GNUC__)
#define ALE_B200_API __attribute__((visibility("default")))
#else
#define ALE_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ALE_B200_OK 0
#define ALE_B200_E_ARG (-1)
#define ALE_B200_E_CUDA (-3)
#define ALE_B200_E_UNSUPPORTED (-5)

#define ALE_B200_NZ_MAX 128
#define ALE_B200_REMAP_PCM 1
#define ALE_B200_REMAP_PLM 2
#define ALE_B200_REMAP_PPM 3

/* ale_remap_step's state (ocean_vcoord_t + multilayer_cgrid_state_t fields,
 * ale_remap/remap_state.F90:28-58). tracers is a HOST array of ntracers device
 * pointers (NULL = an unallocated slot, skipped); idx_temperature /
 * idx_salinity are 0-based slots (-1 = none) whose remap adds to heat_budget /
 * salt_budget. u and v both non-NULL remap the face velocities. total_h and
 * h_ref may be NULL (not written). */
typedef struct ale_b200_step_args {
    int nx, ny, nz, method, conserve_ke, ntracers, idx_temperature, idx_salinity;
    double* h_layer;
    double* const* tracers;
    double *u, *v;
    double *mass_budget, *heat_budget, *salt_budget;
    double* bt_eta;
    const double *bt_H_ref, *dsig;
    double *total_h, *h_ref, *h_old, *target_h;
} ale_b200_step_args;

/* One ale_remap_step on `stream` (a cudaStream_t; NULL = legacy default);
 * does not synchronise. */
ALE_B200_API int ale_b200_remap_step(const ale_b200_step_args* args, void* stream);
ALE_B200_API const char* ale_b200_last_error(void);

/* --- exact exports of the reference's launchers ---------------------------- */
ALE_B200_API void ale_remap_cuda(int nx, int ny, int nz, int method, int fused, double* h_layer, double* h_old,
                                 double* target_h, double* total_h, double* h_ref, double* hTr_t, double* hTr_s,
                                 double* u, double* v, double* mass_b, double* heat_b, double* salt_b, double* eta,
                                 double* H_ref, double* dsig);
ALE_B200_API void ale_remap_opt(int nx, int ny, int nz, double* h_layer, double* h_old, double* target_h,
                                double* hTr_t, double* hTr_s, double* u, double* v, double* mass_b, double* heat_b,
                                double* salt_b, double* eta, double* H_ref, double* dsig);
ALE_B200_API void cuda_sync(void);

#ifdef __cplusplus
}
#endif

#endif /* ALE_B200_H */
