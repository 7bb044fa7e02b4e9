// TEST INFRASTRUCTURE ONLY — the CPU oracle for the Redi neutral-diffusion step.
//
// This file is the checker, never the product: only tests/, the smoke check and
// bench.py's CPU-baseline / reference arm load it. The CUDA product path never
// links or calls it and fails loudly if its own extension is missing.
//
// It restates, function by function, the reference's do-concurrent Fortran
// (redi/ocean_redi.F90, the "faithful" path that `make verify` / `DATA=none`
// runs on the CPU) and the point EOS of redi/ocean_eos.F90 (LINEAR here, the
// WRIGHT_97 and ROQUET_SPV branches in redi_eos_oracle.h). Every
// floating-point expression keeps the reference's operand order and
// association (Fortran evaluates a*b*c as (a*b)*c, as the reference's own CUDA
// transliteration redi/redi_kernel.cu does). Build with
// -O2 -ffp-contract=off -fno-fast-math so no FMA contraction or reassociation
// happens: the result is then the exact IEEE-754 sequence the reference
// specifies, and the sm_100a kernels built with FMA contraction off must match
// it bit for bit.
//
// Parity pin: tests/golden/ holds outputs of the reference's own CUDA
// launchers (redi/redi_kernel.cu `redi_cuda_launch_`, redi/opt_kernel.cu
// `redi_opt_launch`), compiled from the reference sources with nvcc
// (FMA contraction off) by oracle/ref_build.sh and run on a B200, and the
// oracle is checked against them.
//
// The scalar type is a template parameter: `double` for results, `OpCount`
// (a double that tallies every FP64 add/sub, mul, div, compare and int->fp
// conversion) for the exact FP64 operation counts used in the roofline.
//
// Loop structure differs from the Fortran only where the result cannot change:
// OpenMP parallelises the (j, i) loops exactly as `do concurrent` allows.

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>
#include <omp.h>

#include "redi_eos_oracle.h"

namespace {

constexpr double GRAVITY = 9.80665;     // redi/constants.F90:19
constexpr double H_DIV_EPS = 1.0e-20;   // redi/constants.F90:21
constexpr double H_NEGLECT = 1.0e-30;   // ocean_redi.F90:242 (interface_scalar default)

// ---------------------------------------------------------------------------
// Counting scalar: every arithmetic op on two FP64 values increments a
// per-thread counter. Used only to derive the FP64 op budget of the step.
// ---------------------------------------------------------------------------
struct OpTally {
    uint64_t add = 0, mul = 0, div = 0, cmp = 0, cvt = 0;
};
thread_local OpTally g_tally;

struct OpCount {
    double v;
    OpCount() : v(0.0) {}
    OpCount(double x) : v(x) {}  // NOLINT: implicit from literals
    explicit operator double() const { return v; }
};
inline OpCount operator+(OpCount a, OpCount b) { g_tally.add++; return OpCount(a.v + b.v); }
inline OpCount operator-(OpCount a, OpCount b) { g_tally.add++; return OpCount(a.v - b.v); }
inline OpCount operator*(OpCount a, OpCount b) { g_tally.mul++; return OpCount(a.v * b.v); }
inline OpCount operator/(OpCount a, OpCount b) { g_tally.div++; return OpCount(a.v / b.v); }
inline OpCount operator-(OpCount a) { return OpCount(-a.v); }
inline bool operator<(OpCount a, OpCount b) { g_tally.cmp++; return a.v < b.v; }
inline bool operator>(OpCount a, OpCount b) { g_tally.cmp++; return a.v > b.v; }
inline bool operator<=(OpCount a, OpCount b) { g_tally.cmp++; return a.v <= b.v; }
inline bool operator>=(OpCount a, OpCount b) { g_tally.cmp++; return a.v >= b.v; }
inline bool operator==(OpCount a, OpCount b) { g_tally.cmp++; return a.v == b.v; }
inline bool operator!=(OpCount a, OpCount b) { g_tally.cmp++; return a.v != b.v; }

inline double r_abs(double x) { return std::fabs(x); }
inline OpCount r_abs(OpCount x) { return OpCount(std::fabs(x.v)); }
inline double r_sign(double a, double x) { return std::copysign(a, x); }
inline OpCount r_sign(OpCount a, OpCount x) { return OpCount(std::copysign(a.v, x.v)); }
inline double r_min(double a, double b) { return std::fmin(a, b); }
inline OpCount r_min(OpCount a, OpCount b) { g_tally.cmp++; return OpCount(std::fmin(a.v, b.v)); }
inline double r_max(double a, double b) { return std::fmax(a, b); }
inline OpCount r_max(OpCount a, OpCount b) { g_tally.cmp++; return OpCount(std::fmax(a.v, b.v)); }
template <class R> inline R r_from_int(int k);
template <> inline double r_from_int<double>(int k) { return static_cast<double>(k); }
template <> inline OpCount r_from_int<OpCount>(int k) { g_tally.cvt++; return OpCount(static_cast<double>(k)); }

template <class R>
struct Eos {  // ocean_eos.F90:239-278 (the scalar members the point routines read)
    R rho0, T_ref, S_ref, alpha_T, beta_S;
    int variant;  // ocean_eos.F90:39-51: 1 (or 0) LINEAR, 2 WRIGHT_97, 4 ROQUET_SPV
};

// ---- ocean_eos.F90:543-545 eos_density_point, LINEAR -----------------------
template <class R>
inline R eos_density_point(const Eos<R>& e, R T, R S) {
    return e.rho0 + e.beta_S * (S - e.S_ref) - e.alpha_T * (T - e.T_ref);
}
// ---- ocean_eos.F90:510-513 eos_specvol_derivs, LINEAR ----------------------
template <class R>
inline void eos_specvol_derivs(const Eos<R>& e, R& dsv_dt, R& dsv_ds) {
    dsv_dt = e.alpha_T / (e.rho0 * e.rho0);
    dsv_ds = -e.beta_S / (e.rho0 * e.rho0);
}

// ---- ocean_redi.F90:135-150 redi_fv_diff -----------------------------------
template <class R>
inline R fv_diff(R hkm1, R hk, R hkp1, R skm1, R sk, R skp1) {
    R h_sum = (hkm1 + hkp1) + hk;
    if (h_sum != R(0.0)) h_sum = R(1.0) / h_sum;
    R hm = hkm1 + hk;
    if (hm != R(0.0)) hm = R(1.0) / hm;
    R hp = hkp1 + hk;
    if (hp != R(0.0)) hp = R(1.0) / hp;
    return (hk * h_sum) * ((R(2.0) * hkm1 + hk) * hp * (skp1 - sk) + (R(2.0) * hkp1 + hk) * hm * (sk - skm1));
}

// ---- ocean_redi.F90:153-160 redi_signum ------------------------------------
template <class R>
inline R signum(R a, R x) {
    R s = r_sign(a, x);
    if (x == R(0.0)) s = R(0.0);
    return s;
}

// ---- ocean_redi.F90:165-190 redi_plm_diff (1-based k in comments) ----------
template <class R>
void plm_diff(int nk, const R* h, const R* s, R* diff) {
    for (int k = 2; k <= nk - 1; ++k) {
        if ((h[k] + h[k - 1]) * (h[k - 2] + h[k - 1]) > R(0.0)) {
            R diff_c = fv_diff(h[k - 2], h[k - 1], h[k], s[k - 2], s[k - 1], s[k]);
            R diff_l = R(2.0) * (s[k - 1] - s[k - 2]);
            R diff_r = R(2.0) * (s[k] - s[k - 1]);
            if (signum(R(1.0), diff_l) * signum(R(1.0), diff_r) <= R(0.0)) {
                diff[k - 1] = R(0.0);
            } else {
                diff[k - 1] = r_sign(r_min(r_min(r_abs(diff_l), r_abs(diff_c)), r_abs(diff_r)), diff_c);
            }
        } else {
            diff[k - 1] = R(0.0);
        }
    }
    diff[0] = R(0.0);
    diff[nk - 1] = R(0.0);
}

// ---- ocean_redi.F90:194-225 redi_ppm_edge ----------------------------------
template <class R>
R ppm_edge(R hkm1, R hk, R hkp1, R hkp2, R ak, R akp1, R pk, R pkp1, R h_neglect) {
    R r_hk_hkp1 = hk + hkp1;
    if (r_hk_hkp1 <= R(0.0)) return R(0.5) * (ak + akp1);
    r_hk_hkp1 = R(1.0) / r_hk_hkp1;
    R e;
    if (hk < hkp1) e = ak + (hk * r_hk_hkp1) * (akp1 - ak);
    else           e = akp1 + (hkp1 * r_hk_hkp1) * (ak - akp1);
    R r_2hk_hkp1 = R(1.0) / ((R(2.0) * hk + hkp1) + h_neglect);
    R r_hk_2hkp1 = R(1.0) / ((hk + R(2.0) * hkp1) + h_neglect);
    R f1 = R(1.0) / ((hk + hkp1) + (hkm1 + hkp2));
    R f2 = R(2.0) * (hkp1 * hk) * r_hk_hkp1 * ((hkm1 + hk) * r_2hk_hkp1 - (hkp2 + hkp1) * r_hk_2hkp1);
    R f3 = hk * (hkm1 + hk) * r_2hk_hkp1;
    R f4 = hkp1 * (hkp1 + hkp2) * r_hk_2hkp1;
    return e + f1 * (f2 * (akp1 - ak) - (f3 * pkp1 - f4 * pk));
}

// ---- ocean_redi.F90:231-254 redi_interface_scalar --------------------------
template <class R>
void interface_scalar(int nk, const R* h, const R* tr, R* edge, R* diff /* scratch nk */) {
    plm_diff(nk, h, tr, diff);
    edge[0] = tr[0] - R(0.5) * diff[0];
    for (int k = 2; k <= nk; ++k) {
        int km2 = k - 2 > 1 ? k - 2 : 1;
        int kp1 = k + 1 < nk ? k + 1 : nk;
        edge[k - 1] = ppm_edge(h[km2 - 1], h[k - 2], h[k - 1], h[kp1 - 1],
                               tr[k - 2], tr[k - 1], diff[k - 2], diff[k - 1], R(H_NEGLECT));
    }
    edge[nk] = tr[nk - 1] + R(0.5) * diff[nk - 1];
}

// ---- ocean_redi.F90:260-285 redi_interpolate_position ----------------------
template <class R>
R interpolate_position(R dRhoNeg, R Pneg, R dRhoPos, R Ppos) {
    if ((Ppos > Pneg) && (dRhoPos - dRhoNeg >= R(0.0))) {
        if (dRhoPos - dRhoNeg > R(0.0)) return r_min(R(1.0), r_max(R(0.0), -dRhoNeg / (dRhoPos - dRhoNeg)));
        if (dRhoNeg > R(0.0)) return R(0.0);
        if (dRhoNeg < R(0.0)) return R(1.0);
        return R(0.5);
    } else if (Ppos == Pneg) {
        return R(0.5);
    }
    return R(0.5);
}

// ---- ocean_redi.F90:289-298 redi_absolute_position -------------------------
template <class R>
inline R absolute_position(const R* Pint, int Karr, R frac) {
    return Pint[Karr - 1] + frac * (Pint[Karr] - Pint[Karr - 1]);
}

// ---- ocean_redi.F90:307-464 redi_neutral_positions_continuous -------------
template <class R>
void neutral_positions_continuous(int nk, const R* Pl, const R* Tl, const R* Sl, const R* dRdTl, const R* dRdSl,
                                  const R* Pr, const R* Tr, const R* Sr, const R* dRdTr, const R* dRdSr,
                                  R* PoL, R* PoR, int* KoL, int* KoR, R* hEff) {
    const int ns = 2 * nk + 2;
    int kr = 1, kl = 1;
    R lastP_right = R(0.0), lastP_left = R(0.0);
    int lastK_right = 1, lastK_left = 1;
    bool reached_bottom = false, searching_left_column = false, searching_right_column = false;

    for (int k_surface = 1; k_surface <= ns; ++k_surface) {
        int klm1 = kl - 1 > 1 ? kl - 1 : 1;
        int krm1 = kr - 1 > 1 ? kr - 1 : 1;
        R dRho = R(0.5) * ((dRdTr[kr - 1] + dRdTl[kl - 1]) * (Tr[kr - 1] - Tl[kl - 1]) +
                           (dRdSr[kr - 1] + dRdSl[kl - 1]) * (Sr[kr - 1] - Sl[kl - 1]));
        if (!reached_bottom) {
            if (dRho < R(0.0)) {
                searching_left_column = true;
                searching_right_column = false;
            } else if (dRho > R(0.0)) {
                searching_right_column = true;
                searching_left_column = false;
            } else {
                if (kl + kr == 2) {
                    searching_left_column = true;
                    searching_right_column = false;
                } else {
                    searching_left_column = !searching_left_column;
                    searching_right_column = !searching_right_column;
                }
            }
        }
        const int s = k_surface - 1;
        if (searching_left_column) {
            R dRhoTop = R(0.5) * ((dRdTl[klm1 - 1] + dRdTr[kr - 1]) * (Tl[klm1 - 1] - Tr[kr - 1]) +
                                  (dRdSl[klm1 - 1] + dRdSr[kr - 1]) * (Sl[klm1 - 1] - Sr[kr - 1]));
            R dRhoBot = R(0.5) * ((dRdTl[klm1] + dRdTr[kr - 1]) * (Tl[klm1] - Tr[kr - 1]) +
                                  (dRdSl[klm1] + dRdSr[kr - 1]) * (Sl[klm1] - Sr[kr - 1]));
            if (dRhoTop > R(0.0) || kr + kl == 2) PoL[s] = R(0.0);
            else if (dRhoTop >= dRhoBot) PoL[s] = R(1.0);
            else PoL[s] = interpolate_position(dRhoTop, Pl[klm1 - 1], dRhoBot, Pl[klm1]);
            if (PoL[s] >= R(1.0) && klm1 < nk) {
                klm1 += 1;
                PoL[s] = PoL[s] - R(1.0);
            }
            if (r_from_int<R>(klm1 - lastK_left) + (PoL[s] - lastP_left) < R(0.0)) {
                PoL[s] = lastP_left;
                klm1 = lastK_left;
            }
            KoL[s] = klm1;
            if (kr <= nk) { PoR[s] = R(0.0); KoR[s] = kr; }
            else          { PoR[s] = R(1.0); KoR[s] = nk; }
            if (kr <= nk) kr += 1;
            else { reached_bottom = true; searching_right_column = true; searching_left_column = false; }
        } else if (searching_right_column) {
            R dRhoTop = R(0.5) * ((dRdTr[krm1 - 1] + dRdTl[kl - 1]) * (Tr[krm1 - 1] - Tl[kl - 1]) +
                                  (dRdSr[krm1 - 1] + dRdSl[kl - 1]) * (Sr[krm1 - 1] - Sl[kl - 1]));
            R dRhoBot = R(0.5) * ((dRdTr[krm1] + dRdTl[kl - 1]) * (Tr[krm1] - Tl[kl - 1]) +
                                  (dRdSr[krm1] + dRdSl[kl - 1]) * (Sr[krm1] - Sl[kl - 1]));
            if (dRhoTop >= R(0.0) || kr + kl == 2) PoR[s] = R(0.0);
            else if (dRhoTop >= dRhoBot) PoR[s] = R(1.0);
            else PoR[s] = interpolate_position(dRhoTop, Pr[krm1 - 1], dRhoBot, Pr[krm1]);
            if (PoR[s] >= R(1.0) && krm1 < nk) {
                krm1 += 1;
                PoR[s] = PoR[s] - R(1.0);
            }
            if (r_from_int<R>(krm1 - lastK_right) + (PoR[s] - lastP_right) < R(0.0)) {
                PoR[s] = lastP_right;
                krm1 = lastK_right;
            }
            KoR[s] = krm1;
            if (kl <= nk) { PoL[s] = R(0.0); KoL[s] = kl; }
            else          { PoL[s] = R(1.0); KoL[s] = nk; }
            if (kl <= nk) kl += 1;
            else { reached_bottom = true; searching_right_column = false; searching_left_column = true; }
        }
        lastK_left = KoL[s];
        lastP_left = PoL[s];
        lastK_right = KoR[s];
        lastP_right = PoR[s];
        if (k_surface > 1) {
            R hL = absolute_position(Pl, KoL[s], PoL[s]) - absolute_position(Pl, KoL[s - 1], PoL[s - 1]);
            R hR = absolute_position(Pr, KoR[s], PoR[s]) - absolute_position(Pr, KoR[s - 1], PoR[s - 1]);
            if (hL + hR > R(0.0)) hEff[s - 1] = R(2.0) * hL * hR / (hL + hR);
            else hEff[s - 1] = R(0.0);
        }
    }
}

// Per-thread column scratch, sized for one face (both columns).
template <class R>
struct ColumnScratch {
    std::vector<R> htd, ttd, std_, diff;
    std::vector<R> Pl, Tl, Sl, dTl, dSl, Pr, Tr, Sr, dTr, dSr;
    std::vector<R> hL, tL, sL, hR, tR, sR;
    std::vector<R> PoL, PoR, hEff;
    std::vector<int> KoL, KoR;
    explicit ColumnScratch(int nz) {
        for (auto* v : {&htd, &ttd, &std_, &diff, &hL, &tL, &sL, &hR, &tR, &sR}) v->assign(nz, R(0.0));
        for (auto* v : {&Pl, &Tl, &Sl, &dTl, &dSl, &Pr, &Tr, &Sr, &dTr, &dSr}) v->assign(nz + 1, R(0.0));
        const int ns = 2 * nz + 2;
        PoL.assign(ns, R(0.0));
        PoR.assign(ns, R(0.0));
        hEff.assign(ns - 1, R(0.0));
        KoL.assign(ns, 1);
        KoR.assign(ns, 1);
    }
};

// ---- ocean_redi.F90:609-654 redi_build_column ------------------------------
template <class R>
void build_column(int nz, const R* h_col, const R* thtr_col, const R* shtr_col, const Eos<R>& eos,
                  R* Pint, R* Tint, R* Sint, R* dRdT, R* dRdS, ColumnScratch<R>& w) {
    for (int k = 1; k <= nz; ++k) {
        int kf = nz + 1 - k;
        R he = r_max(h_col[k - 1], R(H_DIV_EPS));
        w.htd[kf - 1] = h_col[k - 1];
        w.ttd[kf - 1] = thtr_col[k - 1] / he;
        w.std_[kf - 1] = shtr_col[k - 1] / he;
    }
    interface_scalar(nz, w.htd.data(), w.ttd.data(), Tint, w.diff.data());
    interface_scalar(nz, w.htd.data(), w.std_.data(), Sint, w.diff.data());
    Pint[0] = R(0.0);
    for (int k = 1; k <= nz; ++k) Pint[k] = Pint[k - 1] + R(GRAVITY) * eos.rho0 * w.htd[k - 1];
    R dsv_dt, dsv_ds;
    for (int k = 1; k <= nz + 1; ++k) {
        R rho_i;
        if constexpr (std::is_same<R, double>::value) {
            if (eos.variant == 2 || eos.variant == 4) {  // WRIGHT_97 / ROQUET_SPV at the interface pressure
                eos_oracle::point(eos.variant, Tint[k - 1], Sint[k - 1], Pint[k - 1], rho_i, dsv_dt, dsv_ds);
            } else {
                rho_i = eos_density_point(eos, Tint[k - 1], Sint[k - 1]);
                eos_specvol_derivs(eos, dsv_dt, dsv_ds);
            }
        } else {  // operation counts: the LINEAR branch
            rho_i = eos_density_point(eos, Tint[k - 1], Sint[k - 1]);
            eos_specvol_derivs(eos, dsv_dt, dsv_ds);
        }
        dRdT[k - 1] = -(rho_i * rho_i) * dsv_dt;
        dRdS[k - 1] = -(rho_i * rho_i) * dsv_ds;
    }
}

// ---- ocean_redi.F90:656-692 redi_face_coeffs -------------------------------
template <class R>
void face_coeffs(int nz, int ns, const Eos<R>& eos, ColumnScratch<R>& w) {
    build_column(nz, w.hL.data(), w.tL.data(), w.sL.data(), eos, w.Pl.data(), w.Tl.data(), w.Sl.data(),
                 w.dTl.data(), w.dSl.data(), w);
    build_column(nz, w.hR.data(), w.tR.data(), w.sR.data(), eos, w.Pr.data(), w.Tr.data(), w.Sr.data(),
                 w.dTr.data(), w.dSr.data(), w);
    neutral_positions_continuous(nz, w.Pl.data(), w.Tl.data(), w.Sl.data(), w.dTl.data(), w.dSl.data(),
                                 w.Pr.data(), w.Tr.data(), w.Sr.data(), w.dTr.data(), w.dSr.data(),
                                 w.PoL.data(), w.PoR.data(), w.KoL.data(), w.KoR.data(), w.hEff.data());
    R pa_to_h = R(1.0) / (R(GRAVITY) * eos.rho0);
    for (int ks = 1; ks <= ns - 1; ++ks) w.hEff[ks - 1] = w.hEff[ks - 1] * pa_to_h;
}

// Column-major (Fortran) flat indices, 1-based arguments.
inline size_t I3(int i, int j, int k, int n1, int n2) {
    return ((size_t)(k - 1) * (size_t)n2 + (size_t)(j - 1)) * (size_t)n1 + (size_t)(i - 1);
}
inline size_t I2(int i, int j, int n1) { return (size_t)(j - 1) * (size_t)n1 + (size_t)(i - 1); }

// ---- ocean_redi.F90:694-753 / 755-812 redi_calc_coeffs_x / _y ---------------
// dir = 0: u-faces (i = 2..nx, all j; west column i-1, east column i).
// dir = 1: v-faces (j = 2..ny, all i; south column j-1, north column j).
template <class R>
void calc_coeffs_dir(int dir, int nx, int ny, int nz, int ns, const Eos<R>& eos,
                     const double* h, const double* th, const double* sh, const double* wet,
                     double* PoL, double* PoR, int* KoL, int* KoR, double* hEff, int nthreads) {
    const int nfa = dir == 0 ? nx + 1 : nx;
    const int nfb = dir == 0 ? ny : ny + 1;
    const int j0 = dir == 0 ? 1 : 2;
    const int i0 = dir == 0 ? 2 : 1;
    const int i1 = nx;
#pragma omp parallel num_threads(nthreads)
    {
        ColumnScratch<R> w(nz);
#pragma omp for schedule(dynamic, 1)
        for (int j = j0; j <= ny; ++j) {
            for (int i = i0; i <= i1; ++i) {
                for (int s = 1; s <= ns; ++s) {
                    size_t o = I3(i, j, s, nfa, nfb);
                    PoL[o] = 0.0; PoR[o] = 0.0; KoL[o] = 1; KoR[o] = 1;
                }
                for (int s = 1; s <= ns - 1; ++s) hEff[I3(i, j, s, nfa, nfb)] = 0.0;
                if (wet[I2(i, j, nfa)] > 0.0) {
                    const int iw = dir == 0 ? i - 1 : i, jw = dir == 0 ? j : j - 1;
                    for (int k = 1; k <= nz; ++k) {
                        w.hL[k - 1] = R(h[I3(iw, jw, k, nx, ny)]);
                        w.tL[k - 1] = R(th[I3(iw, jw, k, nx, ny)]);
                        w.sL[k - 1] = R(sh[I3(iw, jw, k, nx, ny)]);
                        w.hR[k - 1] = R(h[I3(i, j, k, nx, ny)]);
                        w.tR[k - 1] = R(th[I3(i, j, k, nx, ny)]);
                        w.sR[k - 1] = R(sh[I3(i, j, k, nx, ny)]);
                    }
                    face_coeffs(nz, ns, eos, w);
                    for (int s = 1; s <= ns; ++s) {
                        size_t o = I3(i, j, s, nfa, nfb);
                        PoL[o] = double(w.PoL[s - 1]);
                        PoR[o] = double(w.PoR[s - 1]);
                        KoL[o] = w.KoL[s - 1];
                        KoR[o] = w.KoR[s - 1];
                    }
                    for (int s = 1; s <= ns - 1; ++s) hEff[I3(i, j, s, nfa, nfb)] = double(w.hEff[s - 1]);
                }
            }
        }
    }
}

// ---- ocean_redi.F90:824-831 redi_signum1 -----------------------------------
template <class R>
inline R signum1(R x) {
    R s = r_sign(R(1.0), x);
    if (x == R(0.0)) s = R(0.0);
    return s;
}

// ---- ocean_redi.F90:833-850 redi_ppm_ave -----------------------------------
template <class R>
inline R ppm_ave(R xL, R xR, R aL, R aR, R aMean) {
    R dx = xR - xL;
    R xave = R(0.5) * (xR + xL);
    R a6o3 = R(2.0) * aMean - (aL + aR);
    R a6 = R(3.0) * a6o3;
    if (dx > R(0.0) && dx <= R(1.0)) return (aL + xave * ((aR - aL) + a6)) - a6o3 * (xR * xR + xR * xL + xL * xL);
    return aL + (aR - aL) * xR + a6 * xR * (R(1.0) - xR);
}

template <class R>
struct TracerColumn {
    std::vector<R> h, htr, htd, Tlay, Tint, tedge, aLe, aRe, diff;
    explicit TracerColumn(int nz) {
        for (auto* v : {&h, &htr, &htd, &Tlay, &aLe, &aRe, &diff}) v->assign(nz, R(0.0));
        Tint.assign(nz + 1, R(0.0));
        tedge.assign(nz + 1, R(0.0));
    }
};

// ---- ocean_redi.F90:852-891 redi_tracer_column -----------------------------
template <class R>
void tracer_column(int nz, TracerColumn<R>& c) {
    for (int k = 1; k <= nz; ++k) {
        int kf = nz + 1 - k;
        R he = r_max(c.h[k - 1], R(H_DIV_EPS));
        c.htd[kf - 1] = c.h[k - 1];
        c.Tlay[kf - 1] = c.htr[k - 1] / he;
    }
    interface_scalar(nz, c.htd.data(), c.Tlay.data(), c.tedge.data(), c.diff.data());
    for (int k = 1; k <= nz + 1; ++k) c.Tint[k - 1] = c.tedge[k - 1];
    for (int k = 1; k <= nz; ++k) {
        R alk = c.Tint[k - 1];
        R ark = c.Tint[k];
        R tlk = c.Tlay[k - 1];
        if (signum1(ark - tlk) * signum1(tlk - alk) <= R(0.0)) {
            alk = tlk;
            ark = tlk;
        } else if (r_sign(R(3.0), ark - alk) * ((tlk - alk) + (tlk - ark)) > r_abs(ark - alk)) {
            alk = tlk + R(2.0) * (tlk - ark);
        } else if (r_sign(R(3.0), ark - alk) * ((tlk - alk) + (tlk - ark)) < -r_abs(ark - alk)) {
            ark = tlk + R(2.0) * (tlk - alk);
        }
        c.aLe[k - 1] = alk;
        c.aRe[k - 1] = ark;
    }
}

// ---- ocean_redi.F90:893-925 redi_sublayer_dT -------------------------------
template <class R>
R sublayer_dT(int klt, int klb, int krt, int krb, R PoLt, R PoLb, R PoRt, R PoRb,
              const TracerColumn<R>& L, const TracerColumn<R>& Rc) {
    R tlt = (R(1.0) - PoLt) * L.Tint[klt - 1] + PoLt * L.Tint[klt];
    R tlb = (R(1.0) - PoLb) * L.Tint[klb - 1] + PoLb * L.Tint[klb];
    R trt = (R(1.0) - PoRt) * Rc.Tint[krt - 1] + PoRt * Rc.Tint[krt];
    R trb = (R(1.0) - PoRb) * Rc.Tint[krb - 1] + PoRb * Rc.Tint[krb];
    R tlay = ppm_ave(PoLt, PoLb + r_from_int<R>(klb - klt), L.aLe[klt - 1], L.aRe[klt - 1], L.Tlay[klt - 1]);
    R trlay = ppm_ave(PoRt, PoRb + r_from_int<R>(krb - krt), Rc.aLe[krt - 1], Rc.aRe[krt - 1], Rc.Tlay[krt - 1]);
    R dT_top = trt - tlt;
    R dT_bot = trb - tlb;
    R dT_ave = R(0.5) * (dT_top + dT_bot);
    R dT_layer = trlay - tlay;
    if (signum1(dT_top) * signum1(dT_bot) <= R(0.0) || signum1(dT_ave) * signum1(dT_layer) <= R(0.0))
        return R(0.0);
    return dT_layer;
}

struct FaceArrays {
    const double *PoL, *PoR, *hEff;
    const int *KoL, *KoR;
    int nfa, nfb;
};

// ---- ocean_redi.F90:1037-1092 redi_face_flux -------------------------------
template <class R>
void face_flux(int nz, int ns, int nxc, int nyc, const double* h, const double* hTr_in,
               int iL, int jL, int iR, int jR, int fa, int fb, const FaceArrays& F, R coef, bool is_left,
               R* dTr, TracerColumn<R>& L, TracerColumn<R>& Rc) {
    for (int k = 1; k <= nz; ++k) {
        L.h[k - 1] = R(h[I3(iL, jL, k, nxc, nyc)]);
        L.htr[k - 1] = R(hTr_in[I3(iL, jL, k, nxc, nyc)]);
        Rc.h[k - 1] = R(h[I3(iR, jR, k, nxc, nyc)]);
        Rc.htr[k - 1] = R(hTr_in[I3(iR, jR, k, nxc, nyc)]);
    }
    tracer_column(nz, L);
    tracer_column(nz, Rc);
    for (int ks = 1; ks <= ns - 1; ++ks) {
        const size_t o0 = I3(fa, fb, ks, F.nfa, F.nfb), o1 = I3(fa, fb, ks + 1, F.nfa, F.nfb);
        R he = R(F.hEff[o0]);
        if (he != R(0.0)) {
            R dtdiff = sublayer_dT(F.KoL[o0], F.KoL[o1], F.KoR[o0], F.KoR[o1], R(F.PoL[o0]), R(F.PoL[o1]),
                                   R(F.PoR[o0]), R(F.PoR[o1]), L, Rc);
            R flx = dtdiff * he * coef;
            if (is_left) {
                int knat = nz + 1 - F.KoL[o0];
                dTr[knat - 1] = dTr[knat - 1] + flx;
            } else {
                int knat = nz + 1 - F.KoR[o0];
                dTr[knat - 1] = dTr[knat - 1] - flx;
            }
        }
    }
}

// ---- ocean_redi.F90:1094-1181 redi_apply_flux_impl (one tracer) ------------
template <class R>
void apply_flux_impl(int nx, int ny, int nz, int ns, double dt, int nghost, int nxp, int nyp,
                     bool wall_w, bool wall_e, bool wall_s, bool wall_n,
                     const double* khtr_u, const double* khtr_v, const double* dy_cu, const double* dx_cv,
                     const double* idxCu, const double* idyCv, const double* areaT,
                     const double* h, const double* hTr_in, double* hTr,
                     const FaceArrays& U, const FaceArrays& V, int nthreads) {
    const int wuf_w = nghost + 1, wuf_e = nghost + nxp + 1;
    const int wvf_s = nghost + 1, wvf_n = nghost + nyp + 1;
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<R> dTr(nz);
        TracerColumn<R> L(nz), Rc(nz);
#pragma omp for schedule(dynamic, 1)
        for (int j = 1; j <= ny; ++j) {
            for (int i = 1; i <= nx; ++i) {
                for (int k = 1; k <= nz; ++k) dTr[k - 1] = R(0.0);
                if (i >= 2 && !((wall_w && i == wuf_w) || (wall_e && i == wuf_e)))
                    face_flux(nz, ns, nx, ny, h, hTr_in, i - 1, j, i, j, i, j, U,
                              R(dt) * R(khtr_u[I2(i, j, nx + 1)]) * R(dy_cu[I2(i, j, nx + 1)]) * R(idxCu[I2(i, j, nx + 1)]),
                              false, dTr.data(), L, Rc);
                if (i <= nx - 1 && !((wall_w && i + 1 == wuf_w) || (wall_e && i + 1 == wuf_e)))
                    face_flux(nz, ns, nx, ny, h, hTr_in, i, j, i + 1, j, i + 1, j, U,
                              R(dt) * R(khtr_u[I2(i + 1, j, nx + 1)]) * R(dy_cu[I2(i + 1, j, nx + 1)]) *
                                  R(idxCu[I2(i + 1, j, nx + 1)]),
                              true, dTr.data(), L, Rc);
                if (j >= 2 && !((wall_s && j == wvf_s) || (wall_n && j == wvf_n)))
                    face_flux(nz, ns, nx, ny, h, hTr_in, i, j - 1, i, j, i, j, V,
                              R(dt) * R(khtr_v[I2(i, j, nx)]) * R(dx_cv[I2(i, j, nx)]) * R(idyCv[I2(i, j, nx)]),
                              false, dTr.data(), L, Rc);
                if (j <= ny - 1 && !((wall_s && j + 1 == wvf_s) || (wall_n && j + 1 == wvf_n)))
                    face_flux(nz, ns, nx, ny, h, hTr_in, i, j, i, j + 1, i, j + 1, V,
                              R(dt) * R(khtr_v[I2(i, j + 1, nx)]) * R(dx_cv[I2(i, j + 1, nx)]) *
                                  R(idyCv[I2(i, j + 1, nx)]),
                              true, dTr.data(), L, Rc);
                R iaij = R(1.0) / R(areaT[I2(i, j, nx)]);
                for (int k = 1; k <= nz; ++k) {
                    size_t o = I3(i, j, k, nx, ny);
                    hTr[o] = double(R(hTr[o]) + dTr[k - 1] * iaij);
                }
            }
        }
    }
}

int resolve_threads(int n) {
    if (n > 0) return n;
    return omp_get_max_threads();
}

}  // namespace

extern "C" {

// Phase A: redi_calc_coeffs (ocean_redi.F90:572-607 gates excluded; the caller
// checks them). Arrays are column-major with the reference shapes:
// h/th/sh (nx,ny,nz); wet_u (nx+1,ny); wet_v (nx,ny+1); u* (nx+1,ny,ns|ns-1);
// v* (nx,ny+1,ns|ns-1). Faces the reference never touches (u: i=1, nx+1;
// v: j=1, ny+1) are left as the caller initialised them.
void redi_oracle_calc_coeffs(int nx, int ny, int nz, int ns, double rho0, double T_ref, double S_ref,
                             double alpha_T, double beta_S, const double* h, const double* th, const double* sh,
                             const double* wet_u, const double* wet_v, double* uPoL, double* uPoR, int* uKoL,
                             int* uKoR, double* uhEff, double* vPoL, double* vPoR, int* vKoL, int* vKoR,
                             double* vhEff, int nthreads, int eos_variant) {
    Eos<double> e{rho0, T_ref, S_ref, alpha_T, beta_S, eos_variant};
    nthreads = resolve_threads(nthreads);
    calc_coeffs_dir<double>(0, nx, ny, nz, ns, e, h, th, sh, wet_u, uPoL, uPoR, uKoL, uKoR, uhEff, nthreads);
    calc_coeffs_dir<double>(1, nx, ny, nz, ns, e, h, th, sh, wet_v, vPoL, vPoR, vKoL, vKoR, vhEff, nthreads);
}

// Phase B: redi_apply_flux (ocean_redi.F90:927-1002) for ntr tracers, each
// snapshotted then updated in place, in tracer order. khtr_u/khtr_v are the
// resolved per-face diffusivities (the use_ext copy or the scalar broadcast).
void redi_oracle_apply_flux(int nx, int ny, int nz, int ns, double dt, int nghost, int nxp, int nyp, int wall_w,
                            int wall_e, int wall_s, int wall_n, const double* khtr_u, const double* khtr_v,
                            const double* dy_cu, const double* dx_cv, const double* idxCu, const double* idyCv,
                            const double* areaT, const double* h, int ntr, double* const* htr,
                            const double* uPoL, const double* uPoR, const int* uKoL, const int* uKoR,
                            const double* uhEff, const double* vPoL, const double* vPoR, const int* vKoL,
                            const int* vKoR, const double* vhEff, int nthreads) {
    nthreads = resolve_threads(nthreads);
    FaceArrays U{uPoL, uPoR, uhEff, uKoL, uKoR, nx + 1, ny};
    FaceArrays V{vPoL, vPoR, vhEff, vKoL, vKoR, nx, ny + 1};
    const size_t ncell = (size_t)nx * ny * nz;
    std::vector<double> snap(ncell);
    for (int it = 0; it < ntr; ++it) {
        std::memcpy(snap.data(), htr[it], ncell * sizeof(double));  // redi_snapshot (:1004-1013)
        apply_flux_impl<double>(nx, ny, nz, ns, dt, nghost, nxp, nyp, wall_w != 0, wall_e != 0, wall_s != 0,
                                wall_n != 0, khtr_u, khtr_v, dy_cu, dx_cv, idxCu, idyCv, areaT, h, snap.data(),
                                htr[it], U, V, nthreads);
    }
}

// Exact FP64 operation counts of one step (Phase A over all faces + Phase B
// for `ntr` tracers), by running the same code on the counting scalar, single
// threaded. out[0..4] = add/sub, mul, div, compare, int->fp conversions.
// Inputs/outputs are as for the two calls above; htr is updated in place.
void redi_oracle_count_ops(int nx, int ny, int nz, int ns, double rho0, double T_ref, double S_ref,
                           double alpha_T, double beta_S, double dt, int nghost, int nxp, int nyp,
                           const double* h, int ntr, double* const* htr, const double* wet_u,
                           const double* wet_v, const double* khtr_u, const double* khtr_v, const double* dy_cu,
                           const double* dx_cv, const double* idxCu, const double* idyCv, const double* areaT,
                           double* uPoL, double* uPoR, int* uKoL, int* uKoR, double* uhEff, double* vPoL,
                           double* vPoR, int* vKoL, int* vKoR, double* vhEff, uint64_t* outA, uint64_t* outB) {
    Eos<OpCount> e{rho0, T_ref, S_ref, alpha_T, beta_S, 1};
    g_tally = OpTally{};
    calc_coeffs_dir<OpCount>(0, nx, ny, nz, ns, e, h, htr[0], htr[1], wet_u, uPoL, uPoR, uKoL, uKoR, uhEff, 1);
    calc_coeffs_dir<OpCount>(1, nx, ny, nz, ns, e, h, htr[0], htr[1], wet_v, vPoL, vPoR, vKoL, vKoR, vhEff, 1);
    outA[0] = g_tally.add; outA[1] = g_tally.mul; outA[2] = g_tally.div; outA[3] = g_tally.cmp; outA[4] = g_tally.cvt;
    g_tally = OpTally{};
    FaceArrays U{uPoL, uPoR, uhEff, uKoL, uKoR, nx + 1, ny};
    FaceArrays V{vPoL, vPoR, vhEff, vKoL, vKoR, nx, ny + 1};
    const size_t ncell = (size_t)nx * ny * nz;
    std::vector<double> snap(ncell);
    for (int it = 0; it < ntr; ++it) {
        std::memcpy(snap.data(), htr[it], ncell * sizeof(double));
        apply_flux_impl<OpCount>(nx, ny, nz, ns, dt, nghost, nxp, nyp, true, true, true, true, khtr_u, khtr_v,
                                 dy_cu, dx_cv, idxCu, idyCv, areaT, h, snap.data(), htr[it], U, V, 1);
    }
    outB[0] = g_tally.add; outB[1] = g_tally.mul; outB[2] = g_tally.div; outB[3] = g_tally.cmp; outB[4] = g_tally.cvt;
}

int redi_oracle_max_threads(void) { return omp_get_max_threads(); }

// One interface's density and specific-volume derivatives, as the column
// builder combines eos_density_point and eos_specvol_derivs
// (ocean_redi.F90:649-653), for every variant.
void redi_oracle_eos_point(int variant, double rho0, double T_ref, double S_ref, double alpha_T, double beta_S,
                           double T, double S, double p, double* rho, double* dsv_dt, double* dsv_ds) {
    Eos<double> e{rho0, T_ref, S_ref, alpha_T, beta_S, variant};
    if (variant == 2 || variant == 4) {
        eos_oracle::point(variant, T, S, p, *rho, *dsv_dt, *dsv_ds);
    } else {
        *rho = eos_density_point(e, T, S);
        eos_specvol_derivs(e, *dsv_dt, *dsv_ds);
    }
}

// Specific volume of the Roquet polynomial alone (roquet_spv_point's `sv`).
double redi_oracle_roquet_sv(double T, double S, double p) {
    double sv, a, b;
    eos_oracle::roquet_point(T, S, p, sv, a, b);
    return sv;
}

}  // extern "C"
