// Device building blocks of the Redi neutral-diffusion step, shared by the
// FP64 (plain) and mixed-precision kernels.
//
// Every helper reproduces one expression tree of the reference
// (redi/ocean_redi.F90, redi/ocean_eos.F90 LINEAR branch) with the same operand
// order and association, so a translation unit compiled with FMA contraction
// off (-fmad=false) produces the reference's IEEE-754 results bit for bit.
//
// The column reconstruction is split into an h-only "geometry" part, computed
// once per column and reused by every scalar (T and S in Phase A, all tracers
// in Phase B), and a per-scalar part. The split moves no operation across a
// rounding: each reciprocal and product the reference forms from thicknesses
// alone is formed here with the same operands, then fed to the same
// per-scalar expression.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace redi {

// Load paths. LdNC: the read-only (non-coherent) cache path, for data no
// thread of the running kernel writes. LdCG: cached in L2 only, coherent
// across the blocks of a running kernel, for data produced inside it.
struct LdNC {
    template <class T>
    __device__ static __forceinline__ T ld(const T* p) { return __ldg(p); }
};
struct LdCG {
    template <class T>
    __device__ static __forceinline__ T ld(const T* p) { return __ldcg(p); }
};

constexpr double kGravity = 9.80665;    // redi/constants.F90:19
constexpr double kHDivEps = 1.0e-20;    // redi/constants.F90:21
constexpr double kHNeglect = 1.0e-30;   // ocean_redi.F90:242

// ocean_eos_t (ocean_eos.F90:239-278): the variant (the reference's codes,
// :39-51: 1 LINEAR, 2 WRIGHT_97, 4 ROQUET_SPV; 0 is LINEAR) and the members the
// LINEAR branch reads. rho0 also sets the hydrostatic pressure in every
// variant (ocean_redi.F90:643-646).
struct EosParams {
    int variant;
    double rho0, T_ref, S_ref, alpha_T, beta_S;
};
__host__ __device__ inline bool eos_is_linear(int variant) { return variant == 0 || variant == 1; }

// -------------------------------------------------------------------------
// PLM slope geometry at top-down layer t (ocean_redi.F90:135-150, 174-176):
// redi_fv_diff's three reciprocals and the plm_diff "no vanished neighbour"
// test depend only on the thicknesses h(t-1), h(t), h(t+1).
// -------------------------------------------------------------------------
struct PlmGeom {
    double g0, g1, g2;  // (hk*h_sum), ((2hkm1+hk)*hp), ((2hkp1+hk)*hm)
    bool ok;            // (h(k+1)+h(k))*(h(k-1)+h(k)) > 0
};

__device__ __forceinline__ PlmGeom plm_geom(double hkm1, double hk, double hkp1) {
    PlmGeom g;
    g.ok = (hkp1 + hk) * (hkm1 + hk) > 0.0;
    double h_sum = (hkm1 + hkp1) + hk;
    if (h_sum != 0.0) h_sum = 1.0 / h_sum;
    double hm = hkm1 + hk;
    if (hm != 0.0) hm = 1.0 / hm;
    double hp = hkp1 + hk;
    if (hp != 0.0) hp = 1.0 / hp;
    g.g0 = hk * h_sum;
    g.g1 = (2.0 * hkm1 + hk) * hp;
    g.g2 = (2.0 * hkp1 + hk) * hm;
    return g;
}

// redi_signum(1, x) (ocean_redi.F90:153-160) as a value in {-1, 0, 1}.
__device__ __forceinline__ double signum1(double x) {
    double s = copysign(1.0, x);
    if (x == 0.0) s = 0.0;
    return s;
}

// signum1(a) * signum1(b) <= 0, decided without the product: a zero on either
// side, or opposite sign bits (the sign bit is what copysign transfers).
__device__ __forceinline__ bool signs_not_agree(double a, double b) {
    return a == 0.0 || b == 0.0 || (signbit(a) != signbit(b));
}

// redi_plm_diff body for one interior layer (ocean_redi.F90:175-186).
__device__ __forceinline__ double plm_slope(const PlmGeom& g, double skm1, double sk, double skp1) {
    if (!g.ok) return 0.0;
    double diff_c = g.g0 * (g.g1 * (skp1 - sk) + g.g2 * (sk - skm1));
    double diff_l = 2.0 * (sk - skm1);
    double diff_r = 2.0 * (skp1 - sk);
    if (signs_not_agree(diff_l, diff_r)) return 0.0;
    double am = fmin(fmin(fabs(diff_l), fabs(diff_c)), fabs(diff_r));
    return copysign(am, diff_c);
}

// -------------------------------------------------------------------------
// PPM edge geometry at the interface between top-down layers t-1 and t
// (ocean_redi.F90:194-225): hkm1 = h(max(1,t-2)), hk = h(t-1), hkp1 = h(t),
// hkp2 = h(min(nk,t+1)).
// -------------------------------------------------------------------------
struct EdgeGeom {
    double w, f1, f2, f3, f4;
    bool degenerate;  // hk + hkp1 <= 0 -> arithmetic mean
    bool lt;          // hk < hkp1 selects the interpolation anchor
};

__device__ __forceinline__ EdgeGeom edge_geom(double hkm1, double hk, double hkp1, double hkp2, double hn) {
    EdgeGeom g;
    double r = hk + hkp1;
    g.degenerate = r <= 0.0;
    g.lt = hk < hkp1;
    if (g.degenerate) {
        g.w = g.f1 = g.f2 = g.f3 = g.f4 = 0.0;
        return g;
    }
    r = 1.0 / r;
    g.w = g.lt ? hk * r : hkp1 * r;
    double r_2hk_hkp1 = 1.0 / ((2.0 * hk + hkp1) + hn);
    double r_hk_2hkp1 = 1.0 / ((hk + 2.0 * hkp1) + hn);
    g.f1 = 1.0 / ((hk + hkp1) + (hkm1 + hkp2));
    g.f2 = 2.0 * (hkp1 * hk) * r * ((hkm1 + hk) * r_2hk_hkp1 - (hkp2 + hkp1) * r_hk_2hkp1);
    g.f3 = hk * (hkm1 + hk) * r_2hk_hkp1;
    g.f4 = hkp1 * (hkp1 + hkp2) * r_hk_2hkp1;
    return g;
}

__device__ __forceinline__ double ppm_edge(const EdgeGeom& g, double ak, double akp1, double pk, double pkp1) {
    if (g.degenerate) return 0.5 * (ak + akp1);
    double e = g.lt ? ak + g.w * (akp1 - ak) : akp1 + g.w * (ak - akp1);
    return e + g.f1 * (g.f2 * (akp1 - ak) - (g.f3 * pkp1 - g.f4 * pk));
}

// -------------------------------------------------------------------------
// Phase A helpers
// -------------------------------------------------------------------------

// Interface state of one column used by the neutral sweep: top-down interface
// T, S and the EOS derivatives dR/dT, dR/dS (ocean_redi.F90:647-653).
struct alignas(32) IfcState {
    double T, S, dRdT, dRdS;
};

template <class LD>
__device__ __forceinline__ IfcState load_ifc(const IfcState* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = LD::ld(q), b = LD::ld(q + 1);
    IfcState r;
    r.T = a.x; r.S = a.y; r.dRdT = b.x; r.dRdS = b.y;
    return r;
}

// Cross-column secant density difference rho(b) - rho(a)
// (ocean_redi.F90:344-345, 367-371, 406-410): 0.5*((dRdT_b + dRdT_a)*(T_b - T_a)
// + (dRdS_b + dRdS_a)*(S_b - S_a)).
__device__ __forceinline__ double secant_drho(const IfcState& b, const IfcState& a) {
    return 0.5 * ((b.dRdT + a.dRdT) * (b.T - a.T) + (b.dRdS + a.dRdS) * (b.S - a.S));
}

// ocean_redi.F90:260-285 redi_interpolate_position.
__device__ __forceinline__ double interpolate_position(double dRhoNeg, double Pneg, double dRhoPos, double Ppos) {
    if ((Ppos > Pneg) && (dRhoPos - dRhoNeg >= 0.0)) {
        if (dRhoPos - dRhoNeg > 0.0) return fmin(1.0, fmax(0.0, -dRhoNeg / (dRhoPos - dRhoNeg)));
        if (dRhoNeg > 0.0) return 0.0;
        if (dRhoNeg < 0.0) return 1.0;
        return 0.5;
    }
    return 0.5;  // Ppos == Pneg (vanished/inverted) and the device-safe clamp both give 0.5
}

// -------------------------------------------------------------------------
// Phase B helpers
// -------------------------------------------------------------------------

// PPM parabola of one top-down layer, prepared for redi_ppm_ave
// (ocean_redi.F90:833-850): the limited edges aL, aR and the layer mean enter
// ppm_ave only through aL, (aR - aL), a6o3 = 2*aMean - (aL + aR) and
// (aR - aL) + 3*a6o3, which are the same values on every call for a layer.
struct alignas(32) PpmLayer {
    double aL, dA, a6o3, B;
};

__device__ __forceinline__ PpmLayer make_ppm_layer(double alk, double ark, double tlk) {
    PpmLayer q;
    q.aL = alk;
    q.dA = ark - alk;
    q.a6o3 = 2.0 * tlk - (alk + ark);
    q.B = q.dA + 3.0 * q.a6o3;
    return q;
}

template <class LD>
__device__ __forceinline__ PpmLayer load_ppm(const PpmLayer* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = LD::ld(q), b = LD::ld(q + 1);
    PpmLayer r;
    r.aL = a.x; r.dA = a.y; r.a6o3 = b.x; r.B = b.y;
    return r;
}

// redi_ppm_ave(xL, xR, aL, aR, aMean).
__device__ __forceinline__ double ppm_ave(double xL, double xR, const PpmLayer& q) {
    double dx = xR - xL;
    double xave = 0.5 * (xR + xL);
    if (dx > 0.0 && dx <= 1.0) return (q.aL + xave * q.B) - q.a6o3 * (xR * xR + xR * xL + xL * xL);
    double a6 = 3.0 * q.a6o3;
    return q.aL + q.dA * xR + a6 * xR * (1.0 - xR);
}

// PPM edge limiter of redi_tracer_column (ocean_redi.F90:876-890).
__device__ __forceinline__ void ppm_limit(double& alk, double& ark, double tlk) {
    if (signs_not_agree(ark - tlk, tlk - alk)) {
        alk = tlk;
        ark = tlk;
    } else if (copysign(3.0, ark - alk) * ((tlk - alk) + (tlk - ark)) > fabs(ark - alk)) {
        alk = tlk + 2.0 * (tlk - ark);
    } else if (copysign(3.0, ark - alk) * ((tlk - alk) + (tlk - ark)) < -fabs(ark - alk)) {
        ark = tlk + 2.0 * (tlk - alk);
    }
}

// redi_sublayer_dT's down-gradient guard (ocean_redi.F90:919-924).
__device__ __forceinline__ double guarded_dT(double dT_top, double dT_bot, double dT_layer) {
    double dT_ave = 0.5 * (dT_top + dT_bot);
    if (signs_not_agree(dT_top, dT_bot) || signs_not_agree(dT_ave, dT_layer)) return 0.0;
    return dT_layer;
}

}  // namespace redi
