/*
 * meke_b200.h — C-ABI of the B200-native MEKE step (the eddy-kinetic-energy
 * producer of the diffusivities the Redi step consumes).
 *
 * Drop-in boundary for the reference's MEKE step (JorgeG94/more_benchmarks_dc_ocean,
 * meke/meke.F90:60-131 `meke_step_ext`, bit-identical to its fused form
 * `meke_step_ext_fused`, :158-315). Two layers:
 *
 *  1. Exports with the exact signatures of the reference's CUDA launchers, so
 *     its drivers (meke/drivers/cpp_main.cu, meke/drivers/meke_bridge.F90)
 *     link unchanged:
 *       meke_cuda_launch(args, mode)        meke/meke_args.h:56-61,
 *                                           meke/meke_kernel.cu:253-278
 *       meke_cuda_graph_reset()             meke/meke_kernel.cu:280-283
 *       meke_opt_launch(args, meke_scratch) meke/opt_kernel.cu:274-295
 *       meke_opt_launch_flat(...)           meke/opt_kernel.cu:302-344
 *     Each call is synchronous on return, as the reference's are. Errors are
 *     printed to stderr, as the reference prints CUDA errors, and kept for
 *     meke_b200_last_error().
 *
 *  2. A stream-ordered handle API (no counterpart in the reference):
 *     meke_b200_create / meke_b200_step / meke_b200_destroy. The handle owns
 *     the step's scratch (post-drag energy, the pre-step kh_diff, the
 *     biharmonic Laplacian), so a step allocates nothing.
 *
 * Semantics are those of meke_step_ext for every configuration: the lateral
 * step runs only when kh >= 0 or k4 >= 0 and the second drag half only then
 * (meke/meke.F90:107-123), and the biharmonic block of meke_lateral
 * (:674-729) runs when k4 >= 0. The reference's CUDA launchers run the
 * lateral step unconditionally and have no biharmonic block; the two agree for
 * kh >= 0 and k4 < 0, the configuration those launchers are written for.
 *
 * Arrays are DEVICE pointers, Fortran column-major with the reference shapes:
 * (nx, ny) cell fields, (nx+1, ny) u faces, (nx, ny+1) v faces, (nx, ny, nz)
 * layers (meke/meke_args.h:16-23). All arithmetic is FP64.
 */
#ifndef MEKE_B200_H
#define MEKE_B200_H

#if defined(__GNUC__)
#define MEKE_B200_API __attribute__((visibility("default")))
#else
#define MEKE_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MEKE_B200_OK 0
#define MEKE_B200_E_ARG (-1)
#define MEKE_B200_E_CUDA (-3)
#define MEKE_B200_E_NOMEM (-4)

/* The reference's argument block, field for field and in the same order
 * (meke/meke_args.h:38-52): its drivers and the Fortran bind(C) type
 * meke_args_t lay it out this way. kh_bg is ocean_meke_t%kh. */
struct MekeArgs {
    /* workspaces / prognostic */
    double *meke, *kh_diff, *le, *ku, *i_mass, *depth_tot, *bottom_fac2;
    double *barotr_fac2, *src, *uflux, *vflux, *mass_ws, *rd_ws;
    double *sn_u_ws, *sn_v_ws, *ke_diss_ws;
    /* read-only inputs */
    const double *u_bbl2, *f_centre, *gm_src, *ke_diss_ext;
    const double *h_layer, *rho_layer;
    const double *areaT, *iareaT, *idxT, *idyT, *dy_cu, *dx_cv, *idxCu, *idyCv;
    int nx, ny, nz;
    /* configuration scalars (ocean_meke_t, meke/meke_state.F90:52-80) */
    double dt, dtscale, cd_scale, cb, ct, min_gamma2, cdrag, uscale;
    double a_deform, a_rhines, a_eady, a_frict, a_grid;
    double bgsrc, gmcoeff, frcoeff, damping;
    double kh_bg, k4, khmeke_fac, khcoeff, visc_coeff_ku, rho0;
    int backscatter;
};

typedef struct meke_b200 meke_b200;

/* Scratch for steps of an nx x ny x nz domain on the current device. */
MEKE_B200_API int meke_b200_create(int nx, int ny, int nz, meke_b200** out);
MEKE_B200_API int meke_b200_destroy(meke_b200* self);

/* One meke_step_ext on `stream` (a cudaStream_t; NULL = the legacy default
 * stream); does not synchronise. `del2` is ocean_meke_t%del2 (nx*ny doubles):
 * with k4 >= 0 it receives the biharmonic tendency, as meke_lateral leaves it;
 * NULL uses the handle's own. uflux / vflux may be NULL (not written). */
MEKE_B200_API int meke_b200_step(meke_b200* self, const struct MekeArgs* args, double* del2, void* stream);

/* The handle's post-drag energy after the last step (pass-A output), for tests. */
MEKE_B200_API const double* meke_b200_scratch_energy(const meke_b200* self);

/* Message of the last error on the calling thread ("" if none). */
MEKE_B200_API const char* meke_b200_last_error(void);

/* --- exact exports of the reference's launchers -------------------------- */

/* mode 0, 1: the step on the legacy default stream, then cudaDeviceSynchronize.
 * mode 2: the step captured once into a CUDA graph on a private stream and
 * replayed (re-captured when the argument block changes), then that stream is
 * synchronised. All three give the same result. */
MEKE_B200_API void meke_cuda_launch(const struct MekeArgs* ap, int mode);
MEKE_B200_API void meke_cuda_graph_reset(void);

/* The step with the caller's nx*ny scratch for the post-drag energy (left
 * holding it, as the reference's pass A leaves it), then cudaDeviceSynchronize. */
MEKE_B200_API void meke_opt_launch(const struct MekeArgs* ap, double* meke_scratch);
MEKE_B200_API void meke_opt_launch_flat(
    double* meke, double* kh_diff, double* le, double* ku, double* i_mass, double* depth_tot, double* bottom_fac2,
    double* barotr_fac2, double* src, double* uflux, double* vflux, double* mass_ws, double* rd_ws, double* sn_u_ws,
    double* sn_v_ws, double* ke_diss_ws, const double* u_bbl2, const double* f_centre, const double* gm_src,
    const double* ke_diss_ext, const double* h_layer, const double* rho_layer, const double* areaT,
    const double* iareaT, const double* idxT, const double* idyT, const double* dy_cu, const double* dx_cv,
    const double* idxCu, const double* idyCv, int nx, int ny, int nz, double dt, double dtscale, double cd_scale,
    double cb, double ct, double min_gamma2, double cdrag, double uscale, double a_deform, double a_rhines,
    double a_eady, double a_frict, double a_grid, double bgsrc, double gmcoeff, double frcoeff, double damping,
    double kh_bg, double k4, double khmeke_fac, double khcoeff, double visc_coeff_ku, double rho0, int backscatter,
    double* meke_scratch);

#ifdef __cplusplus
}
#endif

#endif /* MEKE_B200_H */
