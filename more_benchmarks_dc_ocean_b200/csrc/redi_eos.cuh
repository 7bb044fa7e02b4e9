// Point equation of state at one interface: density and specific-volume
// derivatives as redi_build_column combines eos_density_point and
// eos_specvol_derivs (ocean_redi.F90:649-653; ocean_eos.F90:450-546).
//
// Variants carry the reference's codes (ocean_eos.F90:39-51): LINEAR 1 (0 is
// taken as LINEAR: a zero-initialised handle), WRIGHT_97 2, ROQUET_SPV 4.
// TEOS-10 (3) is reserved in the reference and rejected by the C-ABI.
//
// Every expression keeps the reference's association (Fortran evaluates
// a + b*c + d as (a + b*c) + d and honours parentheses). Coefficients that the
// Fortran folds at compile time are formed as double products evaluated left
// to right, integer powers as repeated multiplication. Compile with FMA
// contraction off. sqrt and division are the correctly rounded IEEE
// operations.
#pragma once

#include <cuda_runtime.h>

namespace redi {
namespace eos {

enum Variant : int { kLinear = 1, kWright97 = 2, kRoquetSpV = 4 };

// ---- Wright (1997), Table A1 (ocean_eos.F90:82-97) ------------------------------
constexpr double kWrightA0 = 7.057924e-4, kWrightA1 = 3.480336e-7, kWrightA2 = -1.112733e-7;
constexpr double kWrightB0 = 5.790749e8, kWrightB1 = 3.516535e6, kWrightB2 = -4.002714e4, kWrightB3 = 2.084372e2,
                 kWrightB4 = 5.944068e5, kWrightB5 = -9.643486e3;
constexpr double kWrightC0 = 1.704853e5, kWrightC1 = 7.904722e2, kWrightC2 = -7.984422e0, kWrightC3 = 5.140652e-2,
                 kWrightC4 = -2.302158e2, kWrightC5 = -3.079464e0;

// eos_density_point (:534-542) and eos_specvol_derivs (:493-509), WRIGHT_97.
__device__ __forceinline__ void wright97(double T, double S, double p, double& rho, double& dsv_dt, double& dsv_ds) {
    const double T_sq = T * T;
    const double alpha_0 = kWrightA0 + kWrightA1 * T + kWrightA2 * S;
    const double p_0 = kWrightB0 + kWrightB1 * T + kWrightB2 * T_sq + kWrightB3 * T_sq * T + kWrightB4 * S +
                       kWrightB5 * S * T;
    const double lambda = kWrightC0 + kWrightC1 * T + kWrightC2 * T_sq + kWrightC3 * T_sq * T + kWrightC4 * S +
                          kWrightC5 * S * T;
    const double p_plus_p0 = p + p_0;
    rho = p_plus_p0 / (lambda + alpha_0 * p_plus_p0);
    const double dp0_dt = kWrightB1 + 2.0 * kWrightB2 * T + 3.0 * kWrightB3 * T_sq + kWrightB5 * S;
    const double dlam_dt = kWrightC1 + 2.0 * kWrightC2 * T + 3.0 * kWrightC3 * T_sq + kWrightC5 * S;
    const double dp0_ds = kWrightB4 + kWrightB5 * T;
    const double dlam_ds = kWrightC4 + kWrightC5 * T;
    const double inv_p = 1.0 / p_plus_p0;  // big_p = p + p_0, the same value
    const double inv_p2 = inv_p * inv_p;
    dsv_dt = kWrightA1 + dlam_dt * inv_p - lambda * dp0_dt * inv_p2;
    dsv_ds = kWrightA2 + dlam_ds * inv_p - lambda * dp0_ds * inv_p2;
}

// ---- Roquet et al. (2015) specific-volume polynomial (ocean_eos.F90:114-237) ----
namespace roq {
constexpr double kPa2kb = 1.0e-8;
constexpr double kRDeltaS = 24.0;
constexpr double kR1S0 = 0.875 / 35.16504;
constexpr double kITs = 0.025;
constexpr double kSrFactor = 35.16504 / 35.0;
constexpr double kCp0 = 3991.86795711963;
constexpr double kCtSfac = 0.0248826675584615;
constexpr double P1 = kPa2kb, P2 = P1 * kPa2kb, P3 = P2 * kPa2kb, P4 = P3 * kPa2kb, P5 = P4 * kPa2kb,
                 P6 = P5 * kPa2kb;
constexpr double T1 = kITs, T2 = T1 * kITs, T3 = T2 * kITs, T4 = T3 * kITs, T5 = T4 * kITs, T6 = T5 * kITs;

// Reference profile SV00p (pressure only).
constexpr double V00 = -4.4015007269e-05 * P1, V01 = 6.9232335784e-06 * P2, V02 = -7.5004675975e-07 * P3,
                 V03 = 1.7009109288e-08 * P4, V04 = -1.6884162004e-08 * P5, V05 = 1.9613503930e-09 * P6;

// SV term coefficients, SPV_abc for zs^a zt^b zp^c.
constexpr double SPV000 = 1.0772899069e-03, SPV100 = -3.1263658781e-04, SPV200 = 6.7615860683e-04,
                 SPV300 = -8.6127884515e-04, SPV400 = 5.9010812596e-04, SPV500 = -2.1503943538e-04,
                 SPV600 = 3.2678954455e-05;
constexpr double SPV010 = -1.4949652640e-05 * T1, SPV110 = 3.1866349188e-05 * T1,
                 SPV210 = -3.8070687610e-05 * T1, SPV310 = 2.9818473563e-05 * T1,
                 SPV410 = -1.0011321965e-05 * T1, SPV510 = 1.0751931163e-06 * T1;
constexpr double SPV020 = 2.7546851539e-05 * T2, SPV120 = -3.6597334199e-05 * T2, SPV220 = 3.4489154625e-05 * T2,
                 SPV320 = -1.7663254122e-05 * T2, SPV420 = 3.5965131935e-06 * T2;
constexpr double SPV030 = -1.6506828994e-05 * T3, SPV130 = 2.4412359055e-05 * T3,
                 SPV230 = -1.4606740723e-05 * T3, SPV330 = 2.3293406656e-06 * T3;
constexpr double SPV040 = 6.7896174634e-06 * T4, SPV140 = -8.7951832993e-06 * T4, SPV240 = 4.4249040774e-06 * T4;
constexpr double SPV050 = -7.2535743349e-07 * T5, SPV150 = -3.4680559205e-07 * T5;
constexpr double SPV060 = 1.9041365570e-07 * T6;
constexpr double SPV001 = -1.6889436589e-05 * P1, SPV101 = 2.1106556158e-05 * P1, SPV201 = -2.1322804368e-05 * P1,
                 SPV301 = 1.7347655458e-05 * P1, SPV401 = -4.3209400767e-06 * P1;
constexpr double SPV011 = 1.5355844621e-05 * (T1 * P1), SPV111 = 2.0914122241e-06 * (T1 * P1),
                 SPV211 = -5.7751479725e-06 * (T1 * P1), SPV311 = 1.0767234341e-06 * (T1 * P1);
constexpr double SPV021 = -9.6659393016e-06 * (T2 * P1), SPV121 = -7.0686982208e-07 * (T2 * P1),
                 SPV221 = 1.4488066593e-06 * (T2 * P1);
constexpr double SPV031 = 3.1134283336e-06 * (T3 * P1), SPV131 = 7.9562529879e-08 * (T3 * P1);
constexpr double SPV041 = -5.6590253863e-07 * (T4 * P1);
constexpr double SPV002 = 1.0500241168e-06 * P2, SPV102 = 1.9600661704e-06 * P2, SPV202 = -2.1666693382e-06 * P2;
constexpr double SPV012 = -3.8541359685e-06 * (T1 * P2), SPV112 = 1.0157632247e-06 * (T1 * P2);
constexpr double SPV022 = 1.7178343158e-06 * (T2 * P2);
constexpr double SPV003 = -4.1503454190e-07 * P3, SPV103 = 3.5627020989e-07 * P3;
constexpr double SPV013 = -1.1293871415e-07 * (T1 * P3);

// dSV/dCT coefficients: b * SPV_a(b)c -> ALP_a(b-1)c.
constexpr double ALP000 = SPV010, ALP100 = SPV110, ALP200 = SPV210, ALP300 = SPV310, ALP400 = SPV410,
                 ALP500 = SPV510;
constexpr double ALP010 = 2.0 * SPV020, ALP110 = 2.0 * SPV120, ALP210 = 2.0 * SPV220, ALP310 = 2.0 * SPV320,
                 ALP410 = 2.0 * SPV420;
constexpr double ALP020 = 3.0 * SPV030, ALP120 = 3.0 * SPV130, ALP220 = 3.0 * SPV230, ALP320 = 3.0 * SPV330;
constexpr double ALP030 = 4.0 * SPV040, ALP130 = 4.0 * SPV140, ALP230 = 4.0 * SPV240;
constexpr double ALP040 = 5.0 * SPV050, ALP140 = 5.0 * SPV150;
constexpr double ALP050 = 6.0 * SPV060;
constexpr double ALP001 = SPV011, ALP101 = SPV111, ALP201 = SPV211, ALP301 = SPV311;
constexpr double ALP011 = 2.0 * SPV021, ALP111 = 2.0 * SPV121, ALP211 = 2.0 * SPV221;
constexpr double ALP021 = 3.0 * SPV031, ALP121 = 3.0 * SPV131;
constexpr double ALP031 = 4.0 * SPV041;
constexpr double ALP002 = SPV012, ALP102 = SPV112;
constexpr double ALP012 = 2.0 * SPV022;
constexpr double ALP003 = SPV013;

// dSV/dSA coefficients with the 0.5*R1_S0 chain factor folded in
// (a * 0.5 * SPV_abc * R1_S0 -> BET_(a-1)bc); the residual 1/zs is applied
// where dSV/dSA is formed.
constexpr double BET000 = 0.5 * SPV100 * kR1S0, BET100 = SPV200 * kR1S0, BET200 = 1.5 * SPV300 * kR1S0,
                 BET300 = 2.0 * SPV400 * kR1S0, BET400 = 2.5 * SPV500 * kR1S0, BET500 = 3.0 * SPV600 * kR1S0;
constexpr double BET010 = 0.5 * SPV110 * kR1S0, BET110 = SPV210 * kR1S0, BET210 = 1.5 * SPV310 * kR1S0,
                 BET310 = 2.0 * SPV410 * kR1S0, BET410 = 2.5 * SPV510 * kR1S0;
constexpr double BET020 = 0.5 * SPV120 * kR1S0, BET120 = SPV220 * kR1S0, BET220 = 1.5 * SPV320 * kR1S0,
                 BET320 = 2.0 * SPV420 * kR1S0;
constexpr double BET030 = 0.5 * SPV130 * kR1S0, BET130 = SPV230 * kR1S0, BET230 = 1.5 * SPV330 * kR1S0;
constexpr double BET040 = 0.5 * SPV140 * kR1S0, BET140 = SPV240 * kR1S0;
constexpr double BET050 = 0.5 * SPV150 * kR1S0;
constexpr double BET001 = 0.5 * SPV101 * kR1S0, BET101 = SPV201 * kR1S0, BET201 = 1.5 * SPV301 * kR1S0,
                 BET301 = 2.0 * SPV401 * kR1S0;
constexpr double BET011 = 0.5 * SPV111 * kR1S0, BET111 = SPV211 * kR1S0, BET211 = 1.5 * SPV311 * kR1S0;
constexpr double BET021 = 0.5 * SPV121 * kR1S0, BET121 = SPV221 * kR1S0;
constexpr double BET031 = 0.5 * SPV131 * kR1S0;
constexpr double BET002 = 0.5 * SPV102 * kR1S0, BET102 = SPV202 * kR1S0;
constexpr double BET012 = 0.5 * SPV112 * kR1S0;
constexpr double BET003 = 0.5 * SPV103 * kR1S0;
}  // namespace roq

// roquet_spv_point (ocean_eos.F90:282-448) in model variables (potential
// temperature, practical salinity, pressure in Pa): specific volume and its
// derivatives, the salinity one carrying both the direct SA route and the
// conservative-temperature route (CT depends on SR = SP*35.16504/35).
__device__ __forceinline__ void roquet_spv(double T_pt, double S_sp, double p, double& sv, double& dsv_dt,
                                           double& dsv_ds) {
    using namespace roq;
    const double SR = S_sp * kSrFactor;
    const double x2 = fmax(kCtSfac * SR, 1.0e-20);
    const double xx = sqrt(x2);
    const double yy = T_pt * 0.025;
    // CT = ct_from_pt(SR, PT): coefficients c_k of yy^k as polynomials in xx,
    // and their xx-derivatives d_k.
    const double c0 = 61.01362420681071 +
                      x2 * (268.5520265845071 +
                            xx * (937.2099110620707 + xx * (-1687.914374187449 + xx * 246.9598888781377)));
    const double c1 = 168776.46138048015 +
                      x2 * (-12019.028203559312 +
                            xx * (588.1802812170108 + xx * (936.3206544460336 + xx * 123.59576582457964)));
    const double c2 = -2735.2785605119625 +
                      x2 * (3734.858026725145 +
                            xx * (248.39476522971285 + xx * (-942.7827304544439 + xx * (-48.5891069025409))));
    const double c3 =
        2574.2164453821433 + x2 * (-2046.7671145057618 + xx * (-3.871557904936333 + xx * 369.4389437509002));
    const double c4 =
        -1536.6644434977543 + x2 * (465.28655623126450 + xx * (-2.6268019854268356 + xx * (-33.83664947895248)));
    const double c5 = 545.7340497931629 + x2 * (-0.6370820302831379 + xx * (-9.987880382780322));
    const double c6 = -50.91091728474331 + x2 * (-10.650848542359153);
    const double c7 = -18.30489878927802;
    const double d0 = xx * (2.0 * 268.5520265845071 +
                            xx * (3.0 * 937.2099110620707 +
                                  xx * (4.0 * (-1687.914374187449) + xx * 5.0 * 246.9598888781377)));
    const double d1 = xx * (2.0 * (-12019.028203559312) +
                            xx * (3.0 * 588.1802812170108 +
                                  xx * (4.0 * 936.3206544460336 + xx * 5.0 * 123.59576582457964)));
    const double d2 = xx * (2.0 * 3734.858026725145 +
                            xx * (3.0 * 248.39476522971285 +
                                  xx * (4.0 * (-942.7827304544439) + xx * 5.0 * (-48.5891069025409))));
    const double d3 =
        xx * (2.0 * (-2046.7671145057618) + xx * (3.0 * (-3.871557904936333) + xx * 4.0 * 369.4389437509002));
    const double d4 =
        xx * (2.0 * 465.28655623126450 + xx * (3.0 * (-2.6268019854268356) + xx * 4.0 * (-33.83664947895248)));
    const double d5 = xx * (2.0 * (-0.6370820302831379) + xx * 3.0 * (-9.987880382780322));
    const double d6 = xx * 2.0 * (-10.650848542359153);
    const double d7 = 0.0;
    const double hh = c0 + yy * (c1 + yy * (c2 + yy * (c3 + yy * (c4 + yy * (c5 + yy * (c6 + yy * c7))))));
    const double dh_dy =
        c1 + yy * (2.0 * c2 + yy * (3.0 * c3 + yy * (4.0 * c4 + yy * (5.0 * c5 + yy * (6.0 * c6 + yy * 7.0 * c7)))));
    const double dh_dx = d0 + yy * (d1 + yy * (d2 + yy * (d3 + yy * (d4 + yy * (d5 + yy * (d6 + yy * d7))))));
    const double CT = hh / kCp0;
    const double dct_dpt = 0.025 * dh_dy / kCp0;
    const double dct_dsr = dh_dx * (kCtSfac / (2.0 * xx)) / kCp0;

    const double zt = CT;
    const double zs = sqrt(fabs(S_sp * kSrFactor + kRDeltaS) * kR1S0);
    const double zp = p;

    const double sv_ts3 = SPV003 + (zs * SPV103 + zt * SPV013);
    const double sv_ts2 = SPV002 + (zs * (SPV102 + zs * SPV202) + zt * (SPV012 + (zs * SPV112 + zt * SPV022)));
    const double sv_ts1 =
        SPV001 + (zs * (SPV101 + zs * (SPV201 + zs * (SPV301 + zs * SPV401))) +
                  zt * (SPV011 + (zs * (SPV111 + zs * (SPV211 + zs * SPV311)) +
                                  zt * (SPV021 + (zs * (SPV121 + zs * SPV221) +
                                                  zt * (SPV031 + (zs * SPV131 + zt * SPV041)))))));
    const double sv_ts0 =
        zt * (SPV010 +
              (zs * (SPV110 + zs * (SPV210 + zs * (SPV310 + zs * (SPV410 + zs * SPV510)))) +
               zt * (SPV020 + (zs * (SPV120 + zs * (SPV220 + zs * (SPV320 + zs * SPV420))) +
                               zt * (SPV030 + (zs * (SPV130 + zs * (SPV230 + zs * SPV330)) +
                                               zt * (SPV040 + (zs * (SPV140 + zs * SPV240) +
                                                               zt * (SPV050 + (zs * SPV150 + zt * SPV060))))))))));
    const double sv_0s0 =
        SPV000 + zs * (SPV100 + zs * (SPV200 + zs * (SPV300 + zs * (SPV400 + zs * (SPV500 + zs * SPV600)))));
    const double sv_00p = zp * (V00 + zp * (V01 + zp * (V02 + zp * (V03 + zp * (V04 + zp * V05)))));
    sv = ((sv_ts0 + sv_0s0) + zp * (sv_ts1 + zp * (sv_ts2 + zp * sv_ts3))) + sv_00p;

    const double dvdzt3 = ALP003;
    const double dvdzt2 = ALP002 + (zs * ALP102 + zt * ALP012);
    const double dvdzt1 =
        ALP001 + (zs * (ALP101 + zs * (ALP201 + zs * ALP301)) +
                  zt * (ALP011 + (zs * (ALP111 + zs * ALP211) + zt * (ALP021 + (zs * ALP121 + zt * ALP031)))));
    const double dvdzt0 =
        ALP000 + (zs * (ALP100 + zs * (ALP200 + zs * (ALP300 + zs * (ALP400 + zs * ALP500)))) +
                  zt * (ALP010 + (zs * (ALP110 + zs * (ALP210 + zs * (ALP310 + zs * ALP410))) +
                                  zt * (ALP020 + (zs * (ALP120 + zs * (ALP220 + zs * ALP320)) +
                                                  zt * (ALP030 + (zt * (ALP040 + (zs * ALP140 + zt * ALP050)) +
                                                                  zs * (ALP130 + zs * ALP230))))))));
    const double dsv_dct = dvdzt0 + zp * (dvdzt1 + zp * (dvdzt2 + zp * dvdzt3));

    const double dvdzs3 = BET003;
    const double dvdzs2 = BET002 + (zs * BET102 + zt * BET012);
    const double dvdzs1 =
        BET001 + (zs * (BET101 + zs * (BET201 + zs * BET301)) +
                  zt * (BET011 + (zs * (BET111 + zs * BET211) + zt * (BET021 + (zs * BET121 + zt * BET031)))));
    const double dvdzs0 =
        BET000 + (zs * (BET100 + zs * (BET200 + zs * (BET300 + zs * (BET400 + zs * BET500)))) +
                  zt * (BET010 + (zs * (BET110 + zs * (BET210 + zs * (BET310 + zs * BET410))) +
                                  zt * (BET020 + (zs * (BET120 + zs * (BET220 + zs * BET320)) +
                                                  zt * (BET030 + (zt * (BET040 + (zs * BET140 + zt * BET050)) +
                                                                  zs * (BET130 + zs * BET230))))))));
    const double dsv_dsa = (dvdzs0 + zp * (dvdzs1 + zp * (dvdzs2 + zp * dvdzs3))) / zs;

    dsv_dt = dsv_dct * dct_dpt;
    dsv_ds = (dsv_dsa + dsv_dct * dct_dsr) * kSrFactor;
}

// The non-linear variants at one interface: density and dSV/dT, dSV/dS.
__device__ __forceinline__ void nonlinear_point(int variant, double T, double S, double p, double& rho,
                                                double& dsv_dt, double& dsv_ds) {
    if (variant == kRoquetSpV) {
        double sv;
        roquet_spv(T, S, p, sv, dsv_dt, dsv_ds);
        rho = 1.0 / sv;
    } else {
        wright97(T, S, p, rho, dsv_dt, dsv_ds);
    }
}

}  // namespace eos
}  // namespace redi
