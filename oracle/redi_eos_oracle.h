// TEST INFRASTRUCTURE ONLY — CPU restatement of the non-linear branches of the
// reference's point EOS (redi/ocean_eos.F90), included by redi_oracle.cpp.
//
// Variants use the reference's codes (ocean_eos.F90:39-51): 1 LINEAR (also 0,
// a zero-initialised handle), 2 WRIGHT_97, 4 ROQUET_SPV; 3 (TEOS-10) is
// reserved there and not implemented.
//
// Every expression keeps the reference's association (Fortran evaluates
// a + b*c + d as (a + b*c) + d and honours parentheses). Coefficients that
// the Fortran folds at compile time (x*ROQ_I_TS**n, ...) are formed here as
// double products evaluated left to right, powers as repeated
// multiplication; a Fortran compiler that folds x**n with a single rounding
// can differ from these in the last bit of a few coefficients, so bit parity
// with the Fortran itself is unpinned (no Fortran compiler in this image).
// wright_dsv is pinned bit for bit against the reference's own CUDA
// transcriptions of eos_specvol_derivs (epbl/epbl_kernel.cu:112-137,
// kappa_shear/ks_kernel.cu:108-134; golden vectors
// tests/golden/eos_specvol_ref.npz, 2318 points, 0 ulp). wright_rho and the
// Roquet branch have no compiled counterpart in the reference and are pinned
// by (a) finite-difference consistency of dSV/dT and dSV/dS with SV (the check
// the reference's comments name, ocean_eos.F90:300-306), (b) plausible
// seawater densities, and (c) bit equality with the independently written
// device code.
#pragma once

#include <cmath>

namespace eos_oracle {

// ---- Wright (1997) Table A1, ocean_eos.F90:82-97 --------------------------------
constexpr double WA0 = 7.057924e-4, WA1 = 3.480336e-7, WA2 = -1.112733e-7;
constexpr double WB0 = 5.790749e8, WB1 = 3.516535e6, WB2 = -4.002714e4, WB3 = 2.084372e2, WB4 = 5.944068e5,
                 WB5 = -9.643486e3;
constexpr double WC0 = 1.704853e5, WC1 = 7.904722e2, WC2 = -7.984422e0, WC3 = 5.140652e-2, WC4 = -2.302158e2,
                 WC5 = -3.079464e0;

// eos_density_point, WRIGHT_97 branch (ocean_eos.F90:534-542).
inline double wright_rho(double T, double S, double p) {
    const double T_sq = T * T;
    const double alpha_0 = WA0 + WA1 * T + WA2 * S;
    const double p_0 = WB0 + WB1 * T + WB2 * T_sq + WB3 * T_sq * T + WB4 * S + WB5 * S * T;
    const double lambda = WC0 + WC1 * T + WC2 * T_sq + WC3 * T_sq * T + WC4 * S + WC5 * S * T;
    const double p_plus_p0 = p + p_0;
    return p_plus_p0 / (lambda + alpha_0 * p_plus_p0);
}

// eos_specvol_derivs, WRIGHT_97 branch (ocean_eos.F90:493-509).
inline void wright_dsv(double T, double S, double p, double& dsv_dt, double& dsv_ds) {
    const double T_sq = T * T;
    const double p_0 = WB0 + WB1 * T + WB2 * T_sq + WB3 * T_sq * T + WB4 * S + WB5 * S * T;
    const double lambda = WC0 + WC1 * T + WC2 * T_sq + WC3 * T_sq * T + WC4 * S + WC5 * S * T;
    const double dp0_dt = WB1 + 2.0 * WB2 * T + 3.0 * WB3 * T_sq + WB5 * S;
    const double dlam_dt = WC1 + 2.0 * WC2 * T + 3.0 * WC3 * T_sq + WC5 * S;
    const double dp0_ds = WB4 + WB5 * T;
    const double dlam_ds = WC4 + WC5 * T;
    const double big_p = p + p_0;
    const double inv_p = 1.0 / big_p;
    const double inv_p2 = inv_p * inv_p;
    dsv_dt = WA1 + dlam_dt * inv_p - lambda * dp0_dt * inv_p2;
    dsv_ds = WA2 + dlam_ds * inv_p - lambda * dp0_ds * inv_p2;
}

// ---- Roquet et al. (2015) SpV polynomial, ocean_eos.F90:114-237 -----------------
constexpr double PA2KB = 1.0e-8;
constexpr double RDELTAS = 24.0;
constexpr double R1_S0 = 0.875 / 35.16504;
constexpr double I_TS = 0.025;
constexpr double SR_FACTOR = 35.16504 / 35.0;
constexpr double CP0 = 3991.86795711963;
constexpr double CT_SFAC = 0.0248826675584615;

constexpr double PA2KB2 = PA2KB * PA2KB, PA2KB3 = PA2KB2 * PA2KB, PA2KB4 = PA2KB3 * PA2KB,
                 PA2KB5 = PA2KB4 * PA2KB, PA2KB6 = PA2KB5 * PA2KB;
constexpr double I_TS2 = I_TS * I_TS, I_TS3 = I_TS2 * I_TS, I_TS4 = I_TS3 * I_TS, I_TS5 = I_TS4 * I_TS,
                 I_TS6 = I_TS5 * I_TS;

constexpr double V00 = -4.4015007269e-05 * PA2KB;
constexpr double V01 = 6.9232335784e-06 * PA2KB2;
constexpr double V02 = -7.5004675975e-07 * PA2KB3;
constexpr double V03 = 1.7009109288e-08 * PA2KB4;
constexpr double V04 = -1.6884162004e-08 * PA2KB5;
constexpr double V05 = 1.9613503930e-09 * PA2KB6;

constexpr double S000 = 1.0772899069e-03, S100 = -3.1263658781e-04, S200 = 6.7615860683e-04,
                 S300 = -8.6127884515e-04, S400 = 5.9010812596e-04, S500 = -2.1503943538e-04,
                 S600 = 3.2678954455e-05;
constexpr double S010 = -1.4949652640e-05 * I_TS, S110 = 3.1866349188e-05 * I_TS, S210 = -3.8070687610e-05 * I_TS,
                 S310 = 2.9818473563e-05 * I_TS, S410 = -1.0011321965e-05 * I_TS, S510 = 1.0751931163e-06 * I_TS;
constexpr double S020 = 2.7546851539e-05 * I_TS2, S120 = -3.6597334199e-05 * I_TS2,
                 S220 = 3.4489154625e-05 * I_TS2, S320 = -1.7663254122e-05 * I_TS2,
                 S420 = 3.5965131935e-06 * I_TS2;
constexpr double S030 = -1.6506828994e-05 * I_TS3, S130 = 2.4412359055e-05 * I_TS3,
                 S230 = -1.4606740723e-05 * I_TS3, S330 = 2.3293406656e-06 * I_TS3;
constexpr double S040 = 6.7896174634e-06 * I_TS4, S140 = -8.7951832993e-06 * I_TS4,
                 S240 = 4.4249040774e-06 * I_TS4;
constexpr double S050 = -7.2535743349e-07 * I_TS5, S150 = -3.4680559205e-07 * I_TS5;
constexpr double S060 = 1.9041365570e-07 * I_TS6;
constexpr double S001 = -1.6889436589e-05 * PA2KB, S101 = 2.1106556158e-05 * PA2KB,
                 S201 = -2.1322804368e-05 * PA2KB, S301 = 1.7347655458e-05 * PA2KB,
                 S401 = -4.3209400767e-06 * PA2KB;
constexpr double S011 = 1.5355844621e-05 * (I_TS * PA2KB), S111 = 2.0914122241e-06 * (I_TS * PA2KB),
                 S211 = -5.7751479725e-06 * (I_TS * PA2KB), S311 = 1.0767234341e-06 * (I_TS * PA2KB);
constexpr double S021 = -9.6659393016e-06 * (I_TS2 * PA2KB), S121 = -7.0686982208e-07 * (I_TS2 * PA2KB),
                 S221 = 1.4488066593e-06 * (I_TS2 * PA2KB);
constexpr double S031 = 3.1134283336e-06 * (I_TS3 * PA2KB), S131 = 7.9562529879e-08 * (I_TS3 * PA2KB);
constexpr double S041 = -5.6590253863e-07 * (I_TS4 * PA2KB);
constexpr double S002 = 1.0500241168e-06 * PA2KB2, S102 = 1.9600661704e-06 * PA2KB2,
                 S202 = -2.1666693382e-06 * PA2KB2;
constexpr double S012 = -3.8541359685e-06 * (I_TS * PA2KB2), S112 = 1.0157632247e-06 * (I_TS * PA2KB2);
constexpr double S022 = 1.7178343158e-06 * (I_TS2 * PA2KB2);
constexpr double S003 = -4.1503454190e-07 * PA2KB3, S103 = 3.5627020989e-07 * PA2KB3;
constexpr double S013 = -1.1293871415e-07 * (I_TS * PA2KB3);

// dSV/dCT table: d/dzt of the SV table (zt-power b -> b * coefficient).
constexpr double A000 = S010, A100 = S110, A200 = S210, A300 = S310, A400 = S410, A500 = S510;
constexpr double A010 = 2.0 * S020, A110 = 2.0 * S120, A210 = 2.0 * S220, A310 = 2.0 * S320, A410 = 2.0 * S420;
constexpr double A020 = 3.0 * S030, A120 = 3.0 * S130, A220 = 3.0 * S230, A320 = 3.0 * S330;
constexpr double A030 = 4.0 * S040, A130 = 4.0 * S140, A230 = 4.0 * S240;
constexpr double A040 = 5.0 * S050, A140 = 5.0 * S150;
constexpr double A050 = 6.0 * S060;
constexpr double A001 = S011, A101 = S111, A201 = S211, A301 = S311;
constexpr double A011 = 2.0 * S021, A111 = 2.0 * S121, A211 = 2.0 * S221;
constexpr double A021 = 3.0 * S031, A121 = 3.0 * S131;
constexpr double A031 = 4.0 * S041;
constexpr double A002 = S012, A102 = S112;
constexpr double A012 = 2.0 * S022;
constexpr double A003 = S013;

// dSV/dSA table: d/dzs with the chain factor 0.5*R1_S0 folded per
// coefficient (zs-power a -> 0.5*a * coefficient * R1_S0); the remaining 1/zs
// is applied where the derivative is formed.
constexpr double B000 = 0.5 * S100 * R1_S0, B100 = S200 * R1_S0, B200 = 1.5 * S300 * R1_S0,
                 B300 = 2.0 * S400 * R1_S0, B400 = 2.5 * S500 * R1_S0, B500 = 3.0 * S600 * R1_S0;
constexpr double B010 = 0.5 * S110 * R1_S0, B110 = S210 * R1_S0, B210 = 1.5 * S310 * R1_S0,
                 B310 = 2.0 * S410 * R1_S0, B410 = 2.5 * S510 * R1_S0;
constexpr double B020 = 0.5 * S120 * R1_S0, B120 = S220 * R1_S0, B220 = 1.5 * S320 * R1_S0,
                 B320 = 2.0 * S420 * R1_S0;
constexpr double B030 = 0.5 * S130 * R1_S0, B130 = S230 * R1_S0, B230 = 1.5 * S330 * R1_S0;
constexpr double B040 = 0.5 * S140 * R1_S0, B140 = S240 * R1_S0;
constexpr double B050 = 0.5 * S150 * R1_S0;
constexpr double B001 = 0.5 * S101 * R1_S0, B101 = S201 * R1_S0, B201 = 1.5 * S301 * R1_S0,
                 B301 = 2.0 * S401 * R1_S0;
constexpr double B011 = 0.5 * S111 * R1_S0, B111 = S211 * R1_S0, B211 = 1.5 * S311 * R1_S0;
constexpr double B021 = 0.5 * S121 * R1_S0, B121 = S221 * R1_S0;
constexpr double B031 = 0.5 * S131 * R1_S0;
constexpr double B002 = 0.5 * S102 * R1_S0, B102 = S202 * R1_S0;
constexpr double B012 = 0.5 * S112 * R1_S0;
constexpr double B003 = 0.5 * S103 * R1_S0;

// roquet_spv_point (ocean_eos.F90:282-448): specific volume and its
// derivatives with respect to the model's potential temperature and practical
// salinity, via Reference Salinity SR = SP*35.16504/35 and the 7-term
// conservative-temperature polynomial CT(SR, PT) and its analytic
// derivatives.
inline void roquet_point(double T_pt, double S_sp, double p, double& sv, double& dsv_dt, double& dsv_ds) {
    const double SR = S_sp * SR_FACTOR;
    const double x2 = std::fmax(CT_SFAC * SR, 1.0e-20);
    const double xx = std::sqrt(x2);
    const double yy = T_pt * 0.025;
    const double c0 = 61.01362420681071 +
                      x2 * (268.5520265845071 + xx * (937.2099110620707 + xx * (-1687.914374187449 + xx * 246.9598888781377)));
    const double c1 = 168776.46138048015 +
                      x2 * (-12019.028203559312 + xx * (588.1802812170108 + xx * (936.3206544460336 + xx * 123.59576582457964)));
    const double c2 = -2735.2785605119625 +
                      x2 * (3734.858026725145 + xx * (248.39476522971285 + xx * (-942.7827304544439 + xx * (-48.5891069025409))));
    const double c3 = 2574.2164453821433 + x2 * (-2046.7671145057618 + xx * (-3.871557904936333 + xx * 369.4389437509002));
    const double c4 = -1536.6644434977543 + x2 * (465.28655623126450 + xx * (-2.6268019854268356 + xx * (-33.83664947895248)));
    const double c5 = 545.7340497931629 + x2 * (-0.6370820302831379 + xx * (-9.987880382780322));
    const double c6 = -50.91091728474331 + x2 * (-10.650848542359153);
    const double c7 = -18.30489878927802;
    const double d0 = xx * (2.0 * 268.5520265845071 +
                            xx * (3.0 * 937.2099110620707 + xx * (4.0 * (-1687.914374187449) + xx * 5.0 * 246.9598888781377)));
    const double d1 = xx * (2.0 * (-12019.028203559312) +
                            xx * (3.0 * 588.1802812170108 + xx * (4.0 * 936.3206544460336 + xx * 5.0 * 123.59576582457964)));
    const double d2 = xx * (2.0 * 3734.858026725145 +
                            xx * (3.0 * 248.39476522971285 + xx * (4.0 * (-942.7827304544439) + xx * 5.0 * (-48.5891069025409))));
    const double d3 = xx * (2.0 * (-2046.7671145057618) + xx * (3.0 * (-3.871557904936333) + xx * 4.0 * 369.4389437509002));
    const double d4 = xx * (2.0 * 465.28655623126450 + xx * (3.0 * (-2.6268019854268356) + xx * 4.0 * (-33.83664947895248)));
    const double d5 = xx * (2.0 * (-0.6370820302831379) + xx * 3.0 * (-9.987880382780322));
    const double d6 = xx * 2.0 * (-10.650848542359153);
    const double d7 = 0.0;
    const double hh = c0 + yy * (c1 + yy * (c2 + yy * (c3 + yy * (c4 + yy * (c5 + yy * (c6 + yy * c7))))));
    const double dh_dy =
        c1 + yy * (2.0 * c2 + yy * (3.0 * c3 + yy * (4.0 * c4 + yy * (5.0 * c5 + yy * (6.0 * c6 + yy * 7.0 * c7)))));
    const double dh_dx = d0 + yy * (d1 + yy * (d2 + yy * (d3 + yy * (d4 + yy * (d5 + yy * (d6 + yy * d7))))));
    const double CT = hh / CP0;
    const double dct_dpt = 0.025 * dh_dy / CP0;
    const double dct_dsr = dh_dx * (CT_SFAC / (2.0 * xx)) / CP0;

    const double zt = CT;
    const double zs = std::sqrt(std::fabs(S_sp * SR_FACTOR + RDELTAS) * R1_S0);
    const double zp = p;

    const double sv_ts3 = S003 + (zs * S103 + zt * S013);
    const double sv_ts2 = S002 + (zs * (S102 + zs * S202) + zt * (S012 + (zs * S112 + zt * S022)));
    const double sv_ts1 =
        S001 + (zs * (S101 + zs * (S201 + zs * (S301 + zs * S401))) +
                zt * (S011 + (zs * (S111 + zs * (S211 + zs * S311)) +
                              zt * (S021 + (zs * (S121 + zs * S221) + zt * (S031 + (zs * S131 + zt * S041)))))));
    const double sv_ts0 =
        zt * (S010 +
              (zs * (S110 + zs * (S210 + zs * (S310 + zs * (S410 + zs * S510)))) +
               zt * (S020 + (zs * (S120 + zs * (S220 + zs * (S320 + zs * S420))) +
                             zt * (S030 + (zs * (S130 + zs * (S230 + zs * S330)) +
                                           zt * (S040 + (zs * (S140 + zs * S240) +
                                                         zt * (S050 + (zs * S150 + zt * S060))))))))));
    const double sv_0s0 = S000 + zs * (S100 + zs * (S200 + zs * (S300 + zs * (S400 + zs * (S500 + zs * S600)))));
    const double sv_00p = zp * (V00 + zp * (V01 + zp * (V02 + zp * (V03 + zp * (V04 + zp * V05)))));
    sv = ((sv_ts0 + sv_0s0) + zp * (sv_ts1 + zp * (sv_ts2 + zp * sv_ts3))) + sv_00p;

    const double dvdzt3 = A003;
    const double dvdzt2 = A002 + (zs * A102 + zt * A012);
    const double dvdzt1 = A001 + (zs * (A101 + zs * (A201 + zs * A301)) +
                                  zt * (A011 + (zs * (A111 + zs * A211) + zt * (A021 + (zs * A121 + zt * A031)))));
    const double dvdzt0 =
        A000 + (zs * (A100 + zs * (A200 + zs * (A300 + zs * (A400 + zs * A500)))) +
                zt * (A010 + (zs * (A110 + zs * (A210 + zs * (A310 + zs * A410))) +
                              zt * (A020 + (zs * (A120 + zs * (A220 + zs * A320)) +
                                            zt * (A030 + (zt * (A040 + (zs * A140 + zt * A050)) +
                                                          zs * (A130 + zs * A230))))))));
    const double dsv_dct = dvdzt0 + zp * (dvdzt1 + zp * (dvdzt2 + zp * dvdzt3));

    const double dvdzs3 = B003;
    const double dvdzs2 = B002 + (zs * B102 + zt * B012);
    const double dvdzs1 = B001 + (zs * (B101 + zs * (B201 + zs * B301)) +
                                  zt * (B011 + (zs * (B111 + zs * B211) + zt * (B021 + (zs * B121 + zt * B031)))));
    const double dvdzs0 =
        B000 + (zs * (B100 + zs * (B200 + zs * (B300 + zs * (B400 + zs * B500)))) +
                zt * (B010 + (zs * (B110 + zs * (B210 + zs * (B310 + zs * B410))) +
                              zt * (B020 + (zs * (B120 + zs * (B220 + zs * B320)) +
                                            zt * (B030 + (zt * (B040 + (zs * B140 + zt * B050)) +
                                                          zs * (B130 + zs * B230))))))));
    const double dsv_dsa = (dvdzs0 + zp * (dvdzs1 + zp * (dvdzs2 + zp * dvdzs3))) / zs;

    dsv_dt = dsv_dct * dct_dpt;
    dsv_ds = (dsv_dsa + dsv_dct * dct_dsr) * SR_FACTOR;
}

// Density and specific-volume derivatives at one interface, as
// redi_build_column combines eos_density_point and eos_specvol_derivs
// (ocean_redi.F90:649-653), for the two non-linear variants.
inline void point(int variant, double T, double S, double p, double& rho, double& dsv_dt, double& dsv_ds) {
    if (variant == 4) {
        double sv;
        roquet_point(T, S, p, sv, dsv_dt, dsv_ds);
        rho = 1.0 / sv;
    } else {
        rho = wright_rho(T, S, p);
        wright_dsv(T, S, p, dsv_dt, dsv_ds);
    }
}

}  // namespace eos_oracle
