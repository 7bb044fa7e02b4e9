// TEST INFRASTRUCTURE ONLY — the CPU oracle for the MEKE step. Nothing in the
// product path links or calls this file; tests, smoke() and the CPU baseline of
// bench.py use it as the checker.
//
// A plain C++ restatement of `meke_step_ext` (meke/meke.F90:60-131), loop by
// loop, in the reference's order:
//   stage zeros (meke_zero_2d, :316-324)        rd_ws, sn_u_ws, sn_v_ws
//   meke_mass (:355-388)                        column mass, 1/mass, depth
//   meke_length_scales (:420-505) with meke_inv_lmix (:390-418)
//   meke_stage_rd of ke_diss (:326-335) and meke_source (:507-530)
//   meke_drag (:532-556), the first half step
//   meke_lateral (:645-751) when kh >= 0 or k4 >= 0, biharmonic block included
//   meke_drag again when kh >= 0 or k4 >= 0
//   meke_kh_closure (:575-595) and meke_ku_closure (:597-622)
// with the have_rho / have_ws / have_vm branches resolved as meke_step_ext
// resolves them (meke/meke.F90:29-34: rho_layer used, rd and SN zeroed).
//
// Arithmetic follows the Fortran expressions operand for operand (left to right,
// x**2 as x*x, x**p as pow) and is compiled with -ffp-contract=off, so every
// FP64 result is the IEEE sequence of the source. MAX is fmax, as in the
// reference's CUDA launchers (meke/meke_kernel.cu). Arrays are Fortran
// column-major, 1-based in the reference; here 0-based with the same strides.

#include <cmath>
#include <cstddef>

namespace {

constexpr double MASS_NEGLECT = 1.0e-30;  // meke/meke.F90:51
constexpr double H_VANISHED = 1.5e-4;     // meke/constants.F90:15

}  // namespace

// Field order mirrors `struct MekeArgs` (meke/meke_args.h:38-52) with host
// pointers, plus the biharmonic workspace `del2` that meke_lateral uses.
struct MekeOracleArgs {
    double *meke, *kh_diff, *le, *ku, *i_mass, *depth_tot, *bottom_fac2;
    double *barotr_fac2, *src, *uflux, *vflux, *mass_ws, *rd_ws;
    double *sn_u_ws, *sn_v_ws, *ke_diss_ws;
    const double *u_bbl2, *f_centre, *gm_src, *ke_diss_ext;
    const double *h_layer, *rho_layer;
    const double *areaT, *iareaT, *idxT, *idyT, *dy_cu, *dx_cv, *idxCu, *idyCv;
    int nx, ny, nz;
    double dt, dtscale, cd_scale, cb, ct, min_gamma2, cdrag, uscale;
    double a_deform, a_rhines, a_eady, a_frict, a_grid;
    double bgsrc, gmcoeff, frcoeff, damping;
    double kh_bg, k4, khmeke_fac, khcoeff, visc_coeff_ku, rho0;
    int backscatter;
    double *del2;
};

namespace {

struct Idx {
    int nx, ny;
    // (nx, ny) cell arrays, (nx+1, ny) u faces, (nx, ny+1) v faces; 1-based i, j
    size_t t(int i, int j) const { return (size_t)(i - 1) + (size_t)nx * (size_t)(j - 1); }
    size_t u(int i, int j) const { return (size_t)(i - 1) + (size_t)(nx + 1) * (size_t)(j - 1); }
    size_t v(int i, int j) const { return (size_t)(i - 1) + (size_t)nx * (size_t)(j - 1); }
    size_t c(int i, int j, int k) const {
        return (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1));
    }
};

// meke_inv_lmix (meke/meke.F90:390-418)
double inv_lmix(double ueddy, double sn, double beta, double area, double rd_over_dx, double depth, double cdrag,
                double a_deform, double a_rhines, double a_eady, double a_frict, double a_grid) {
    double lgrid = std::sqrt(std::fmax(area, 0.0));
    double ldeform = lgrid * rd_over_dx;
    double lfrict = 0.0;
    if (cdrag > 0.0) lfrict = depth / cdrag;
    double lrhines = 0.0;
    if (beta > 0.0) lrhines = std::sqrt(std::fmax(ueddy, 0.0) / beta);
    double leady = 0.0;
    if (sn > 1.0e-15) leady = ueddy / sn;
    double inv_l = 0.0;
    if (a_deform * ldeform > 0.0) inv_l = inv_l + 1.0 / (a_deform * ldeform);
    if (a_frict * lfrict > 0.0) inv_l = inv_l + 1.0 / (a_frict * lfrict);
    if (a_rhines * lrhines > 0.0) inv_l = inv_l + 1.0 / (a_rhines * lrhines);
    if (a_eady * leady > 0.0) inv_l = inv_l + 1.0 / (a_eady * leady);
    if (a_grid * lgrid > 0.0) inv_l = inv_l + 1.0 / (a_grid * lgrid);
    return inv_l;
}

// meke_drag (meke/meke.F90:532-556)
void drag(const MekeOracleArgs &a, const Idx &x, double sdt_damp) {
    const double cd2 = a.cdrag * a.cdrag;
#pragma omp parallel for
    for (int j = 1; j <= a.ny; ++j)
        for (int i = 1; i <= a.nx; ++i) {
            size_t t = x.t(i, j);
            double e = a.meke[t];
            double drag_rate = a.i_mass[t] * std::sqrt(cd2 * ((std::fmax(0.0, 2.0 * a.bottom_fac2[t] * e) +
                                                               a.u_bbl2[t]) + a.uscale * a.uscale));
            double damp_rate = a.damping + drag_rate * a.bottom_fac2[t];
            if (e < 0.0) damp_rate = 0.0;
            a.meke[t] = e / (1.0 + sdt_damp * damp_rate);
        }
}

// harmonic mean of two column masses (meke/meke.F90:700-701, 713-714)
inline double hmass(double m1, double m2) { return 2.0 * m1 * m2 / ((m1 + m2) + MASS_NEGLECT); }

// meke_lateral (meke/meke.F90:645-751)
void lateral(const MekeOracleArgs &a, const Idx &x, double sdt, bool kh_flux_enabled) {
    const int nx = a.nx, ny = a.ny;
    double *uflux = a.uflux, *vflux = a.vflux, *del2 = a.del2, *meke = a.meke;
    const double *mass = a.mass_ws;
    if (a.k4 >= 0.0) {
        // bare-gradient flux of E and its divergence del2
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx + 1; ++i) uflux[x.u(i, j)] = 0.0;
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 2; i <= nx; ++i)
                uflux[x.u(i, j)] = (a.dy_cu[x.u(i, j)] * a.idxCu[x.u(i, j)]) * (meke[x.t(i, j)] - meke[x.t(i - 1, j)]);
#pragma omp parallel for
        for (int j = 1; j <= ny + 1; ++j)
            for (int i = 1; i <= nx; ++i) vflux[x.v(i, j)] = 0.0;
#pragma omp parallel for
        for (int j = 2; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                vflux[x.v(i, j)] = (a.dx_cv[x.v(i, j)] * a.idyCv[x.v(i, j)]) * (meke[x.t(i, j)] - meke[x.t(i, j - 1)]);
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                del2[x.t(i, j)] = a.iareaT[x.t(i, j)] * ((uflux[x.u(i + 1, j)] - uflux[x.u(i, j)]) +
                                                         (vflux[x.v(i, j + 1)] - vflux[x.v(i, j)]));
        // harmonic-mass flux of del2 with K4, CFL cap 0.3
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx + 1; ++i) uflux[x.u(i, j)] = 0.0;
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 2; i <= nx; ++i) {
                double geo = a.dy_cu[x.u(i, j)] * a.idxCu[x.u(i, j)];
                double g = geo * std::fmax(a.iareaT[x.t(i - 1, j)], a.iareaT[x.t(i, j)]);
                double inv_max = 64.0 * sdt * (g * g);
                double k4_u = a.k4;
                if (k4_u * inv_max > 0.3) k4_u = 0.3 / inv_max;
                double hm = hmass(mass[x.t(i - 1, j)], mass[x.t(i, j)]);
                uflux[x.u(i, j)] = (k4_u * geo) * hm * (del2[x.t(i, j)] - del2[x.t(i - 1, j)]);
            }
#pragma omp parallel for
        for (int j = 1; j <= ny + 1; ++j)
            for (int i = 1; i <= nx; ++i) vflux[x.v(i, j)] = 0.0;
#pragma omp parallel for
        for (int j = 2; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double geo = a.dx_cv[x.v(i, j)] * a.idyCv[x.v(i, j)];
                double g = geo * std::fmax(a.iareaT[x.t(i, j - 1)], a.iareaT[x.t(i, j)]);
                double inv_max = 64.0 * sdt * (g * g);
                double k4_v = a.k4;
                if (k4_v * inv_max > 0.3) k4_v = 0.3 / inv_max;
                double hm = hmass(mass[x.t(i, j - 1)], mass[x.t(i, j)]);
                vflux[x.v(i, j)] = (k4_v * geo) * hm * (del2[x.t(i, j)] - del2[x.t(i, j - 1)]);
            }
        // the biharmonic tendency, stashed in del2
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                del2[x.t(i, j)] = sdt * (a.iareaT[x.t(i, j)] * a.i_mass[x.t(i, j)]) *
                                  ((uflux[x.u(i, j)] - uflux[x.u(i + 1, j)]) + (vflux[x.v(i, j)] - vflux[x.v(i, j + 1)]));
    }
    if (kh_flux_enabled) {
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx + 1; ++i) uflux[x.u(i, j)] = 0.0;
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 2; i <= nx; ++i) {
                double geo = a.dy_cu[x.u(i, j)] * a.idxCu[x.u(i, j)];
                double kh_u = std::fmax(0.0, a.kh_bg) +
                              a.khmeke_fac * 0.5 * (a.kh_diff[x.t(i - 1, j)] + a.kh_diff[x.t(i, j)]);
                double inv_max = 2.0 * sdt * (geo * std::fmax(a.iareaT[x.t(i - 1, j)], a.iareaT[x.t(i, j)]));
                if (kh_u * inv_max > 0.25) kh_u = 0.25 / inv_max;
                double hm = hmass(mass[x.t(i - 1, j)], mass[x.t(i, j)]);
                uflux[x.u(i, j)] = (kh_u * geo) * hm * (meke[x.t(i - 1, j)] - meke[x.t(i, j)]);
            }
#pragma omp parallel for
        for (int j = 1; j <= ny + 1; ++j)
            for (int i = 1; i <= nx; ++i) vflux[x.v(i, j)] = 0.0;
#pragma omp parallel for
        for (int j = 2; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double geo = a.dx_cv[x.v(i, j)] * a.idyCv[x.v(i, j)];
                double kh_v = std::fmax(0.0, a.kh_bg) +
                              a.khmeke_fac * 0.5 * (a.kh_diff[x.t(i, j - 1)] + a.kh_diff[x.t(i, j)]);
                double inv_max = 2.0 * sdt * (geo * std::fmax(a.iareaT[x.t(i, j - 1)], a.iareaT[x.t(i, j)]));
                if (kh_v * inv_max > 0.25) kh_v = 0.25 / inv_max;
                double hm = hmass(mass[x.t(i, j - 1)], mass[x.t(i, j)]);
                vflux[x.v(i, j)] = (kh_v * geo) * hm * (meke[x.t(i, j - 1)] - meke[x.t(i, j)]);
            }
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double mke = sdt * (a.iareaT[x.t(i, j)] * a.i_mass[x.t(i, j)]) *
                             ((uflux[x.u(i, j)] - uflux[x.u(i + 1, j)]) + (vflux[x.v(i, j)] - vflux[x.v(i, j + 1)]));
                meke[x.t(i, j)] = meke[x.t(i, j)] + mke;
            }
    }
    if (a.k4 >= 0.0) {
#pragma omp parallel for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) meke[x.t(i, j)] = meke[x.t(i, j)] + del2[x.t(i, j)];
    }
}

}  // namespace

extern "C" {

// One meke_step_ext (meke/meke.F90:60-131). `del2` may be null when k4 < 0.
// Returns 0, or -1 when k4 >= 0 and no del2 workspace was given.
int meke_oracle_step(const MekeOracleArgs *ap) {
    const MekeOracleArgs &a = *ap;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (a.k4 >= 0.0 && !a.del2) return -1;
    const Idx x{nx, ny};
    const double sdt = a.dt * a.dtscale;
    double damp_step = 1.0;
    if (a.kh_bg >= 0.0 || a.k4 >= 0.0) damp_step = 0.5;
    const double sdt_damp = sdt * damp_step;
    const bool kh_flux_enabled = a.kh_bg >= 0.0;

    // 0. stage optional inputs: no wave-speed or VarMix slot, so zero
    for (size_t t = 0; t < (size_t)nx * ny; ++t) a.rd_ws[t] = 0.0;
    for (size_t t = 0; t < (size_t)(nx + 1) * ny; ++t) a.sn_u_ws[t] = 0.0;
    for (size_t t = 0; t < (size_t)nx * (ny + 1); ++t) a.sn_v_ws[t] = 0.0;

    // 1. column mass (have_rho)
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double mass = 0.0, dsum = 0.0;
            for (int k = 1; k <= nz; ++k) {
                double hk = std::fmax(a.h_layer[x.c(i, j, k)], H_VANISHED);
                double rhok = a.rho_layer[x.c(i, j, k)];
                mass = mass + rhok * hk;
                dsum = dsum + a.h_layer[x.c(i, j, k)];
            }
            size_t t = x.t(i, j);
            a.depth_tot[t] = dsum;
            a.mass_ws[t] = mass;
            a.i_mass[t] = mass > 0.0 ? 1.0 / mass : 0.0;
        }

    // 2. structure factors and mixing length
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            size_t t = x.t(i, j);
            double rd = a.rd_ws[t];
            double lgrid = std::sqrt(std::fmax(a.areaT[t], 0.0));
            double ldeform = lgrid * rd;
            double lfrict = 0.0;
            if (a.cdrag > 0.0) lfrict = a.depth_tot[t] / a.cdrag;
            double bf2 = a.cd_scale * a.cd_scale;
            if (lfrict * a.cb > 0.0) {
                double ratio = ldeform / lfrict;
                bf2 = bf2 + 1.0 / std::pow(1.0 + a.cb * ratio, 0.8);
            }
            bf2 = std::fmax(bf2, a.min_gamma2);
            a.bottom_fac2[t] = bf2;
            double tf2 = 1.0;
            if (lfrict * a.ct > 0.0) {
                double ratio = ldeform / lfrict;
                tf2 = 1.0 / std::pow(1.0 + a.ct * ratio, 0.25);
            }
            tf2 = std::fmax(tf2, a.min_gamma2);
            a.barotr_fac2[t] = tf2;
            double ueddy = std::sqrt(2.0 * std::fmax(0.0, tf2 * a.meke[t]));
            double beta = 0.0;
            if (i > 1 && i < nx) {
                double d = 0.5 * (a.f_centre[x.t(i + 1, j)] - a.f_centre[x.t(i - 1, j)]) * a.idxT[t];
                beta = beta + d * d;
            }
            if (j > 1 && j < ny) {
                double d = 0.5 * (a.f_centre[x.t(i, j + 1)] - a.f_centre[x.t(i, j - 1)]) * a.idyT[t];
                beta = beta + d * d;
            }
            beta = std::sqrt(beta);
            double sn = 0.0;
            if (a.a_eady > 0.0)
                sn = 0.25 * ((a.sn_u_ws[x.u(i, j)] + a.sn_u_ws[x.u(i + 1, j)]) +
                             (a.sn_v_ws[x.v(i, j)] + a.sn_v_ws[x.v(i, j + 1)]));
            double il = inv_lmix(ueddy, sn, beta, a.areaT[t], rd, a.depth_tot[t], a.cdrag, a.a_deform, a.a_rhines,
                                 a.a_eady, a.a_frict, a.a_grid);
            a.le[t] = il > 0.0 ? 1.0 / il : 0.0;
        }

    // 3. stage ke_diss, then the source and the explicit bump
    for (size_t t = 0; t < (size_t)nx * ny; ++t) a.ke_diss_ws[t] = a.ke_diss_ext[t];
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            size_t t = x.t(i, j);
            double s = a.bgsrc;
            if (a.gmcoeff >= 0.0) s = s + a.gmcoeff * a.i_mass[t] * a.gm_src[t];
            if (a.frcoeff >= 0.0) s = s - a.frcoeff * a.i_mass[t] * a.ke_diss_ws[t];
            a.src[t] = s;
            a.meke[t] = a.meke[t] + sdt * s;
        }

    // 4. implicit drag, first half
    drag(a, x, sdt_damp);
    // 5. lateral diffusion
    if (kh_flux_enabled || a.k4 >= 0.0) lateral(a, x, sdt, kh_flux_enabled);
    // 6. implicit drag, second half
    if (a.kh_bg >= 0.0 || a.k4 >= 0.0) drag(a, x, sdt_damp);
    // 7. closures
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            size_t t = x.t(i, j);
            if (a.khcoeff > 0.0) {
                double ueddy = std::sqrt(2.0 * std::fmax(0.0, a.barotr_fac2[t] * a.meke[t]));
                a.kh_diff[t] = a.khcoeff * ueddy * a.le[t];
            } else {
                a.kh_diff[t] = 0.0;
            }
            if (a.backscatter && a.visc_coeff_ku != 0.0) {
                double ueddy = std::sqrt(2.0 * std::fmax(0.0, a.meke[t]));
                a.ku[t] = a.visc_coeff_ku * ueddy * a.le[t];
            } else {
                a.ku[t] = 0.0;
            }
        }
    return 0;
}

}  // extern "C"
