// Per-item device functions of the Redi step: one column, one face or one cell
// per call. Shared by the standalone kernels (redi_plain.cu) and the
// multi-domain persistent kernel (redi_domains.cu). LD is the load path
// (LdNC for data no running thread writes, LdCG for data produced inside the
// running kernel). Include only from translation units compiled with FMA
// contraction off.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "redi_device.cuh"
#include "redi_eos.cuh"
#include "redi_kernels.h"

namespace redi {
namespace plain {

// ---------------------------------------------------------------------------
// Streaming top-down PPM interface reconstruction (redi_interface_scalar,
// ocean_redi.F90:231-254) of NS scalars that share one thickness column.
//
// Layers are pulled from the surface down, t = 1..nk top-down: `fetch(t, r)`
// issues the raw loads of layer t (thickness and the NS thickness-weighted
// scalars) into r; the layer's means (hTr / max(h, eps)) are formed one
// iteration later, so every load has a full iteration to arrive. edge(t)
// needs layers t-2..t+1, so a four-layer register window replaces the
// reference's column arrays. `emit(t, e, s_above, h_t)` receives interface t
// (1..nk+1), its NS edge values, the NS means of the layer just above it
// (layer t-1; undefined for t = 1) and the thickness of layer t (t <= nk).
// ---------------------------------------------------------------------------
template <int NS>
struct RawLayer {
    double h;
    double s[NS];
};

template <int NS>
__device__ __forceinline__ void finish_layer(const RawLayer<NS>& r, double& hv, double (&sv)[NS]) {
    const double he = fmax(r.h, kHDivEps);
    hv = r.h;
#pragma unroll
    for (int n = 0; n < NS; ++n) sv[n] = r.s[n] / he;
}

// AHEAD = 2 keeps a second raw layer in flight (layer t+3 requested while t is
// formed), so every load has two iterations to arrive.
template <int NS, class Fetch, class Emit, int AHEAD = 1>
__device__ __forceinline__ void stream_edges(int nk, Fetch fetch, Emit emit) {
    static_assert(AHEAD == 1 || AHEAD == 2, "one or two raw layers in flight");
    double hA = 0.0, hB, hC, hD = 0.0;  // h(t-2), h(t-1), h(t), h(t+1)
    double sB[NS], sC[NS], sD[NS];      // layer scalars t-1, t, t+1
    double dB[NS], dC[NS];              // PLM slopes of layers t-1, t
    double e[NS];
    RawLayer<NS> r1, r2, rn, rn2;       // rn: raw layer t+2 in flight; rn2: t+3 (AHEAD 2)

    // t = 1: edge(1) = tr(1) - 0.5*diff(1), diff(1) = 0.
    fetch(1, r1);
    if (nk >= 2) fetch(2, r2);
    if (nk >= 3) fetch(3, rn);
    if constexpr (AHEAD == 2) {
        if (nk >= 4) fetch(4, rn2);
    }
    finish_layer(r1, hC, sC);
    if (nk >= 2) finish_layer(r2, hD, sD);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        dC[n] = 0.0;
        e[n] = sC[n] - 0.5 * dC[n];
        sB[n] = 0.0;
    }
    emit(1, e, sB, hC);

    for (int t = 2; t <= nk; ++t) {
        // shift the window down one layer: (t-1) <- t, t <- t+1
        hA = (t >= 3) ? hB : hA;
        hB = hC;
        hC = hD;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            sB[n] = sC[n];
            sC[n] = sD[n];
            dB[n] = dC[n];
        }
        if (t + 1 <= nk) {
            finish_layer(rn, hD, sD);
            if constexpr (AHEAD == 2) {
                if (t + 2 <= nk) rn = rn2;
                if (t + 3 <= nk) fetch(t + 3, rn2);
            } else {
                if (t + 2 <= nk) fetch(t + 2, rn);
            }
        }
        // diff(t): PLM slope for 2 <= t <= nk-1, PCM (0) at t = nk.
        if (t <= nk - 1) {
            const PlmGeom pg = plm_geom(hB, hC, hD);
#pragma unroll
            for (int n = 0; n < NS; ++n) dC[n] = plm_slope(pg, sB[n], sC[n], sD[n]);
        } else {
#pragma unroll
            for (int n = 0; n < NS; ++n) dC[n] = 0.0;
        }
        const double hkm1 = (t >= 3) ? hA : hB;   // h(max(1, t-2))
        const double hkp2 = (t + 1 <= nk) ? hD : hC;  // h(min(nk, t+1))
        const EdgeGeom eg = edge_geom(hkm1, hB, hC, hkp2, kHNeglect);
#pragma unroll
        for (int n = 0; n < NS; ++n) e[n] = ppm_edge(eg, sB[n], sC[n], dB[n], dC[n]);
        emit(t, e, sB, hC);
    }
    // edge(nk+1) = tr(nk) + 0.5*diff(nk), diff(nk) = 0.
#pragma unroll
    for (int n = 0; n < NS; ++n) e[n] = sC[n] + 0.5 * dC[n];
    emit(nk + 1, e, sC, 0.0);
}

// ---------------------------------------------------------------------------
// Phase A, step 1: per-column interface state (redi_build_column,
// ocean_redi.F90:609-654), written in [interface][column] order.
// ---------------------------------------------------------------------------
// Raw layers in flight per column thread (stream_edges' AHEAD) in the column
// state and reconstruction passes.
constexpr int kColumnAhead = 1;
constexpr int kReconAhead = 1;

// Whether a column is read by the sweep or the face flux: whether any of the
// faces it borders (u faces i and i+1, v faces j and j+1, where they are
// interior) passes `wet(face offset)`.
template <class WetU, class WetV>
__device__ __forceinline__ bool column_needed(int col, int nx, int ny, WetU wet_u, WetV wet_v) {
    const int i = col % nx, j = col / nx;
    return (i >= 1 && wet_u(i + (nx + 1) * j)) || (i + 1 <= nx - 1 && wet_u(i + 1 + (nx + 1) * j)) ||
           (j >= 1 && wet_v(i + nx * j)) || (j + 1 <= ny - 1 && wet_v(i + nx * (j + 1)));
}

template <class LD>
__device__ __forceinline__ void column_state_item(const ColumnStateArgs& a, int col) {
    const int ncol = a.nx * a.ny;
    const int nz = a.nz;
    if (a.wet_u) {  // the sweep reads a column only for a face with wet > 0 (its inert branch reads nothing)
        const double* wu = a.wet_u;
        const double* wv = a.wet_v;
        if (!column_needed(col, a.nx, a.ny, [wu](int f) { return LD::ld(wu + f) > 0.0; },
                           [wv](int f) { return LD::ld(wv + f) > 0.0; }))
            return;
    }
    const double* __restrict__ h = a.h + col;
    const double* __restrict__ th = a.th + col;
    const double* __restrict__ sh = a.sh + col;
    IfcState* __restrict__ ifc = a.ifc + col;
    double* __restrict__ pint = a.pint + col;

    const EosParams eos = a.eos;
    const bool linear = eos_is_linear(eos.variant);  // uniform over the launch
    const double dsv_dt = eos.alpha_T / (eos.rho0 * eos.rho0);  // ocean_eos.F90:511
    const double dsv_ds = -eos.beta_S / (eos.rho0 * eos.rho0);  // ocean_eos.F90:512
    const double grho = kGravity * eos.rho0;
    double P = 0.0;
    double h_layer_above = 0.0;

    auto fetch = [&](int t, RawLayer<2>& r) {
        const size_t off = (size_t)(nz - t) * ncol;  // native k = nz+1-t (1-based)
        r.h = LD::ld(h + off);
        r.s[0] = LD::ld(th + off);
        r.s[1] = LD::ld(sh + off);
    };
    auto emit = [&](int t, const double (&e)[2], const double (&)[2], double h_t) {
        if (t >= 2) P = P + grho * h_layer_above;  // Pint(t) = Pint(t-1) + g*rho0*h(t-1)
        double rho_i, sv_t = dsv_dt, sv_s = dsv_ds;
        if (linear)
            rho_i = eos.rho0 + eos.beta_S * (e[1] - eos.S_ref) - eos.alpha_T * (e[0] - eos.T_ref);
        else  // WRIGHT_97 / ROQUET_SPV at the interface pressure (ocean_redi.F90:649-650)
            eos::nonlinear_point(eos.variant, e[0], e[1], P, rho_i, sv_t, sv_s);
        double2* q = reinterpret_cast<double2*>(ifc + (size_t)(t - 1) * ncol);
        q[0] = make_double2(e[0], e[1]);
        q[1] = make_double2(-(rho_i * rho_i) * sv_t, -(rho_i * rho_i) * sv_s);
        pint[(size_t)(t - 1) * ncol] = P;
        h_layer_above = h_t;
    };
    stream_edges<2, decltype(fetch), decltype(emit), kColumnAhead>(nz, fetch, emit);
}

// ---------------------------------------------------------------------------
// Phase A, step 2: the continuous neutral-surface sweep per face
// (redi_neutral_positions_continuous + redi_face_coeffs, ocean_redi.F90:307-464,
// 656-692) and the slot writes of redi_calc_coeffs_x/_y (:694-812).
//
// Each column is read through a three-interface register window anchored at
// km1 = max(k-1, 1) (the reference's klm1/krm1): interfaces km1, km1+1 and
// km1+2 with their pressures. The pointer's own interface is km1 (k = 1) or
// km1+1 (k >= 2). When a pointer advances the window slides by one and one
// interface is fetched ahead, so a step waits on no load it has just issued.
// The two search directions share one code path: the searched column S and
// the anchor column A are selected per step (with the reference's asymmetric
// `dRhoTop > 0` / `dRhoTop >= 0` tests kept).
// ---------------------------------------------------------------------------
struct ColWin {
    IfcState a, b, c;   // interfaces km1, km1+1, km1+2 (1-based)
    double pa, pb, pc;  // pressures at the same interfaces
    int k;              // the pointer (1-based, 1..nk+1)
    int side;           // 0 left column, 1 right column (its ring)
};

// Look-ahead of the window: interfaces km1+3 and km1+4 of each column are in
// flight into a per-thread ring in shared memory (cp.async), issued two shifts
// before they enter the registers. A register window that loaded its next
// interface straight into the slot it rotates from would make the rotation
// itself wait on that load whenever one column advances on consecutive steps;
// here registers only ever receive settled values. Blocks of 128 threads.
constexpr int kSweepRing = 4;
constexpr int kSweepThreads = 128;
struct SweepRing {
    IfcState x[kSweepRing][2][kSweepThreads];
    double p[kSweepRing][2][kSweepThreads];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Ring slot q (0-based interface index, taken mod the ring) <- interface
// min(q, nk) of the column.
__device__ __forceinline__ void ring_fetch(SweepRing& r, int side, int q, const IfcState* X, const double* P, int nk,
                                           size_t ld) {
    const int slot = q % kSweepRing, qi = min(q, nk), tid = threadIdx.x;
    const IfcState* src = X + (size_t)qi * ld;
    cp_async16(&r.x[slot][side][tid], src);
    cp_async16(reinterpret_cast<char*>(&r.x[slot][side][tid]) + 16, reinterpret_cast<const char*>(src) + 16);
    cp_async8(&r.p[slot][side][tid], P + (size_t)qi * ld);
}

template <class LD>
__device__ __forceinline__ void win_init(ColWin& w, SweepRing& r, int side, const IfcState* X, const double* P, int nk,
                                         size_t ld) {
    w.k = 1;
    w.side = side;
    const int i1 = min(1, nk), i2 = min(2, nk);
    w.a = load_ifc<LD>(X);
    w.b = load_ifc<LD>(X + (size_t)i1 * ld);
    w.c = load_ifc<LD>(X + (size_t)i2 * ld);
    w.pa = LD::ld(P);
    w.pb = LD::ld(P + (size_t)i1 * ld);
    w.pc = LD::ld(P + (size_t)i2 * ld);
    ring_fetch(r, side, 3, X, P, nk, ld);
    ring_fetch(r, side, 4, X, P, nk, ld);
}

// k -> k+1: the anchor km1 moves only when k was >= 2. The interface that
// enters the window was requested two shifts ago (or at set-up); every group
// but the newest is complete after wait_group 1, and that group is never the
// one needed (the column's previous shift, or the empty group that closes the
// set-up, came after it).
__device__ __forceinline__ void win_advance(ColWin& w, SweepRing& r, const IfcState* X, const double* P, int nk,
                                            size_t ld) {
    if (w.k >= 2) {
        w.a = w.b;
        w.b = w.c;
        w.pa = w.pb;
        w.pb = w.pc;
        cp_async_wait<1>();
        const int q = w.k + 1;  // 0-based index of interface km1_new + 2
        w.c = r.x[q % kSweepRing][w.side][threadIdx.x];
        w.pc = r.p[q % kSweepRing][w.side][threadIdx.x];
        ring_fetch(r, w.side, q + 2, X, P, nk, ld);
        cp_async_commit();
    }
    w.k += 1;
}

// Register-only variant of the window (the persistent multi-domain kernel):
// the interface entering the window is loaded straight into it.
template <class LD>
__device__ __forceinline__ void win_init_reg(ColWin& w, const IfcState* X, const double* P, int nk, size_t ld) {
    w.k = 1;
    w.side = 0;
    const int i1 = min(1, nk), i2 = min(2, nk);
    w.a = load_ifc<LD>(X);
    w.b = load_ifc<LD>(X + (size_t)i1 * ld);
    w.c = load_ifc<LD>(X + (size_t)i2 * ld);
    w.pa = LD::ld(P);
    w.pb = LD::ld(P + (size_t)i1 * ld);
    w.pc = LD::ld(P + (size_t)i2 * ld);
}

template <class LD>
__device__ __forceinline__ void win_advance_reg(ColWin& w, const IfcState* X, const double* P, int nk, size_t ld) {
    if (w.k >= 2) {
        w.a = w.b;
        w.b = w.c;
        w.pa = w.pb;
        w.pb = w.pc;
        const int inext = min(w.k + 1, nk);  // 0-based index of interface km1_new + 2
        w.c = load_ifc<LD>(X + (size_t)inext * ld);
        w.pc = LD::ld(P + (size_t)inext * ld);
    }
    w.k += 1;
}

__device__ __forceinline__ IfcState sel(bool c, const IfcState& x, const IfcState& y) {
    IfcState r;
    r.T = c ? x.T : y.T;
    r.S = c ? x.S : y.S;
    r.dRdT = c ? x.dRdT : y.dRdT;
    r.dRdS = c ? x.dRdS : y.dRdS;
    return r;
}

__device__ __forceinline__ IfcState win_own(const ColWin& w) { return sel(w.k == 1, w.a, w.b); }

// STAGED: the window's look-ahead goes through the shared-memory ring (the
// standalone sweep kernel); otherwise registers only (the persistent kernel).
template <class P, class LD, bool STAGED>
__device__ __forceinline__ void sweep_item(const SweepArgsT<P>& a, int dir, int t) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    const size_t ld = (size_t)nx * ny;  // interface stride of the scratch
    int colL, colR, fo, nface;
    size_t fstride;
    if (dir == 0) {  // Fortran faces i = 2..nx, j = 1..ny
        nface = (nx - 1) * ny;
        if (t >= nface) return;
        const int j = t / (nx - 1), fi = 1 + t % (nx - 1);
        colL = (fi - 1) + nx * j;
        colR = fi + nx * j;
        fo = fi + (nx + 1) * j;
        fstride = (size_t)(nx + 1) * ny;
    } else {  // Fortran faces j = 2..ny, i = 1..nx
        nface = nx * (ny - 1);
        if (t >= nface) return;
        const int fj = 1 + t / nx, i = t % nx;
        colL = i + nx * (fj - 1);
        colR = i + nx * fj;
        fo = i + nx * fj;
        fstride = (size_t)nx * (ny + 1);
    }
    using Po = typename P::Po;
    using Ko = typename P::Ko;
    using He = typename P::He;
    const FaceOutT<P> o = dir == 0 ? a.u : a.v;
    Po* __restrict__ PoL = o.PoL + fo;
    Po* __restrict__ PoR = o.PoR + fo;
    Ko* __restrict__ KoL = o.KoL + fo;
    Ko* __restrict__ KoR = o.KoR + fo;
    He* __restrict__ hEff = o.hEff + fo;
    const double wet = LD::ld((dir == 0 ? a.wet_u : a.wet_v) + fo);
    if (o.dry) {
        const bool was_dry = o.keep && LD::ld(o.dry + fo);
        o.dry[fo] = wet > 0.0 ? 0 : 1;
        if (was_dry && !(wet > 0.0)) return;  // its slots still hold the inert coefficients
    }

    if (!(wet > 0.0)) {  // ocean_redi.F90:722-730: inert coefficients
        for (int s = 0; s < ns; ++s) {
            PoL[s * fstride] = Po(0);
            PoR[s * fstride] = Po(0);
            KoL[s * fstride] = Ko(1);
            KoR[s * fstride] = Ko(1);
        }
        for (int s = 0; s < ns - 1; ++s) hEff[s * fstride] = He(0);
        return;
    }

    const IfcState* XL = a.ifc + colL;
    const IfcState* XR = a.ifc + colR;
    const double* PL = a.pint + colL;
    const double* PR = a.pint + colR;
    const double pa_to_h = 1.0 / (kGravity * a.rho0);
    const int nk = nz;

    __shared__ SweepRing ring;
    ColWin wl, wr;
    if constexpr (STAGED) {
        win_init<LD>(wl, ring, 0, XL, PL, nk, ld);
        win_init<LD>(wr, ring, 1, XR, PR, nk, ld);
        cp_async_commit();  // the set-up group
        cp_async_commit();  // an empty group: the set-up group is never the newest
    } else {
        win_init_reg<LD>(wl, XL, PL, nk, ld);
        win_init_reg<LD>(wr, XR, PR, nk, ld);
    }
    double lastP_left = 0.0, lastP_right = 0.0;
    int lastK_left = 1, lastK_right = 1;
    bool reached_bottom = false, search_left = false, search_right = false;
    double absL_prev = 0.0, absR_prev = 0.0;

    for (int ks = 1; ks <= ns; ++ks) {
        const int kl = wl.k, kr = wr.k;
        const double dRho = secant_drho(win_own(wr), win_own(wl));
        if (!reached_bottom) {
            if (dRho < 0.0) {
                search_left = true;
                search_right = false;
            } else if (dRho > 0.0) {
                search_right = true;
                search_left = false;
            } else if (kl + kr == 2) {
                search_left = true;
                search_right = false;
            } else {
                search_left = !search_left;
                search_right = !search_right;
            }
        }
        // Exactly one direction is set. S: searched column, A: anchor column
        // (selected field by field so both windows stay in registers).
        const bool L = search_left;
        const IfcState Sa = sel(L, wl.a, wr.a), Sb = sel(L, wl.b, wr.b);
        const double Spa = L ? wl.pa : wr.pa, Spb = L ? wl.pb : wr.pb, Spc = L ? wl.pc : wr.pc;
        const int Sk = L ? kl : kr;
        const IfcState anc = L ? (kr == 1 ? wr.a : wr.b) : (kl == 1 ? wl.a : wl.b);
        const double Apa = L ? wr.pa : wl.pa, Apb = L ? wr.pb : wl.pb;
        const int ka = L ? kr : kl;
        const double dRhoTop = secant_drho(Sa, anc);
        const double dRhoBot = secant_drho(Sb, anc);
        const int km1 = Sk - 1 > 1 ? Sk - 1 : 1;
        double po_s;
        const bool top_zero = (L ? (dRhoTop > 0.0) : (dRhoTop >= 0.0)) || kr + kl == 2;
        if (top_zero) po_s = 0.0;
        else if (dRhoTop >= dRhoBot) po_s = 1.0;
        else po_s = interpolate_position(dRhoTop, Spa, dRhoBot, Spb);
        int ko_s = km1;
        bool carried = false;
        if (po_s >= 1.0 && km1 < nk) {
            ko_s = km1 + 1;
            po_s = po_s - 1.0;
            carried = true;
        }
        const int lastK_s = L ? lastK_left : lastK_right;
        const double lastP_s = L ? lastP_left : lastP_right;
        bool backstop = false;
        if ((double)(ko_s - lastK_s) + (po_s - lastP_s) < 0.0) {
            po_s = lastP_s;
            ko_s = lastK_s;
            backstop = true;
        }
        // absolute position of the searched side (redi_absolute_position)
        double abs_s;
        if (backstop) abs_s = L ? absL_prev : absR_prev;
        else if (carried) abs_s = Spb + po_s * (Spc - Spb);
        else abs_s = Spa + po_s * (Spb - Spa);
        // anchor side: its own interface, or the bed once exhausted
        double po_a, abs_a;
        int ko_a;
        if (ka <= nk) {
            // redi_absolute_position at po = 0: P(k) + 0*(P(k+1) - P(k)) is
            // P(k) itself for finite pressures, so the next interface's
            // pressure (often fetched by the previous step) is not waited on.
            po_a = 0.0;
            ko_a = ka;
            abs_a = (ka == 1) ? Apa : Apb;
        } else {
            po_a = 1.0;
            ko_a = nk;
            abs_a = Apa + po_a * (Apb - Apa);  // km1 = nk: interfaces nk, nk+1
        }
        if (ka <= nk) {
            if constexpr (STAGED) {
                if (L) win_advance(wr, ring, XR, PR, nk, ld);
                else   win_advance(wl, ring, XL, PL, nk, ld);
            } else {
                if (L) win_advance_reg<LD>(wr, XR, PR, nk, ld);
                else   win_advance_reg<LD>(wl, XL, PL, nk, ld);
            }
        } else {
            reached_bottom = true;
            search_left = !L;
            search_right = L;
        }
        const double pol = L ? po_s : po_a, por = L ? po_a : po_s;
        const int kol = L ? ko_s : ko_a, kor = L ? ko_a : ko_s;
        const double absL = L ? abs_s : abs_a, absR = L ? abs_a : abs_s;
        lastK_left = kol;
        lastP_left = pol;
        lastK_right = kor;
        lastP_right = por;
        const size_t so = (size_t)(ks - 1) * fstride;
        PoL[so] = Po(pol);
        PoR[so] = Po(por);
        KoL[so] = Ko(kol);
        KoR[so] = Ko(kor);
        if (ks > 1) {  // harmonic-mean effective thickness (:452-462), Pa -> m (:688-691)
            const double hL = absL - absL_prev;
            const double hR = absR - absR_prev;
            double he = 0.0;
            if (hL + hR > 0.0) he = 2.0 * hL * hR / (hL + hR);
            hEff[so - fstride] = He(he * pa_to_h);
        }
        absL_prev = absL;
        absR_prev = absR;
    }
    if constexpr (STAGED) cp_async_wait<0>();  // no copy may land in the ring after this face is done
}

// ---------------------------------------------------------------------------
// The same sweep with both columns' windows held in a per-thread ring in
// shared memory instead of registers (the standalone sweep kernel's default).
//
// Slot q % NR of side s holds interface min(q, nk) (0-based) of that column.
// A column with pointer k (1-based) reads interfaces max(k-2, 0) ..
// max(k-2, 0) + 2: its own interface is always k-1, the reference's km1 is
// max(k-2, 0). Both columns are read through the same index arithmetic, so the
// anchor's advance is one code path whichever column it is (the register form
// duplicates it per column, and a warp whose lanes search in different
// directions runs both copies). NR = 5 keeps two interfaces in flight per
// column (fetched two advances before they are read, wait_group 1); NR = 4
// keeps one (wait_group 0 at each advance); NR = 3 fetches the entering
// interface at the advance and waits for it at the top of the next step
// (the smallest ring: more resident blocks, one round trip per advance).
//
// The bottom density difference of a searched column with k >= 2 is the step's
// own dRho with its sign set by the direction: rho(S_k) - rho(A_k) and
// rho(A_k) - rho(S_k) are exact negatives (a commuted sum, an exactly negated
// difference, an exactly negated product), and the sign of a zero never
// reaches a decision (every use compares with 0 or forms a difference with a
// non-zero value).
// ---------------------------------------------------------------------------
constexpr int kSweepWinThreads = 128;  // block size of the shared-memory-window sweep
template <int NR>
struct SweepWin {
    double2 ts[NR][2][kSweepWinThreads];  // (T, S)
    double2 dd[NR][2][kSweepWinThreads];  // (dR/dT, dR/dS)
    double p[NR][2][kSweepWinThreads];    // pressure
};

template <int NR>
__device__ __forceinline__ void sw_fetch(SweepWin<NR>& r, int side, int q, const IfcState* X, const double* P, int nk,
                                         size_t ld) {
    const int slot = q % NR, qi = min(q, nk), tid = threadIdx.x;
    const double2* src = reinterpret_cast<const double2*>(X + (size_t)qi * ld);
    cp_async16(&r.ts[slot][side][tid], src);
    cp_async16(&r.dd[slot][side][tid], src + 1);
    cp_async8(&r.p[slot][side][tid], P + (size_t)qi * ld);
}

template <int NR>
__device__ __forceinline__ IfcState sw_ifc(const SweepWin<NR>& r, int side, int q) {
    const int slot = q % NR, tid = threadIdx.x;
    const double2 a = r.ts[slot][side][tid], b = r.dd[slot][side][tid];
    IfcState s;
    s.T = a.x;
    s.S = a.y;
    s.dRdT = b.x;
    s.dRdS = b.y;
    return s;
}

template <int NR>
__device__ __forceinline__ double sw_p(const SweepWin<NR>& r, int side, int q) {
    return r.p[q % NR][side][threadIdx.x];
}

// Ordered compaction across a block of NT threads: the threads whose `keep`
// is set write `value` to list[0 .. n) in thread order; returns n. Every
// thread of the block must call it (two block barriers).
template <int NT>
__device__ __forceinline__ int block_compact(bool keep, int value, int* list, int* warp_n, int tid = -1) {
    if (tid < 0) tid = threadIdx.x;  // the thread's linear index in the block
    const int lane = tid & 31, w = tid >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_n[w] = __popc(m);
    __syncthreads();
    int off = 0, total = 0;
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) {
        const int c = warp_n[i];
        off += i < w ? c : 0;
        total += c;
    }
    if (keep) list[off + __popc(m & ((1u << lane) - 1u))] = value;
    __syncthreads();
    return total;
}

// The part of the sweep for a face that is not wet (ocean_redi.F90:722-730:
// inert coefficients, and the dry-face record); returns whether face t of
// direction dir is wet, i.e. whether it needs the sweep.
template <class P, class LD>
__device__ __forceinline__ bool sweep_face_dry(const SweepArgsT<P>& a, int dir, int t) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    int fo;
    size_t fstride;
    if (dir == 0) {
        if (t >= (nx - 1) * ny) return false;
        fo = 1 + t % (nx - 1) + (nx + 1) * (t / (nx - 1));
        fstride = (size_t)(nx + 1) * ny;
    } else {
        if (t >= nx * (ny - 1)) return false;
        fo = t % nx + nx * (1 + t / nx);
        fstride = (size_t)nx * (ny + 1);
    }
    const FaceOutT<P> o = dir == 0 ? a.u : a.v;
    const double wet = LD::ld((dir == 0 ? a.wet_u : a.wet_v) + fo);
    if (o.dry) {
        const bool was_dry = o.keep && LD::ld(o.dry + fo);
        o.dry[fo] = wet > 0.0 ? 0 : 1;
        if (was_dry && !(wet > 0.0)) return false;  // its slots still hold the inert coefficients
    }
    if (wet > 0.0) return true;
    using Po = typename P::Po;
    using Ko = typename P::Ko;
    using He = typename P::He;
    for (int s = 0; s < ns; ++s) {
        o.PoL[fo + s * fstride] = Po(0);
        o.PoR[fo + s * fstride] = Po(0);
        o.KoL[fo + s * fstride] = Ko(1);
        o.KoR[fo + s * fstride] = Ko(1);
    }
    for (int s = 0; s < ns - 1; ++s) o.hEff[fo + s * fstride] = He(0);
    return false;
}

// r: this block's ring (dynamic shared memory, blocks of kSweepThreads).
// WET_ONLY: the caller has run sweep_face_dry and t is a wet face.
template <class P, class LD, int NR, bool WET_ONLY = false>
__device__ __forceinline__ void sweep_item_win(const SweepArgsT<P>& a, int dir, int t, SweepWin<NR>& r) {
    static_assert(NR >= 3 && NR <= 5, "ring of 3 (none in flight), 4 (one) or 5 (two)");
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    const size_t ld = (size_t)nx * ny;
    int colL, colR, fo;
    size_t fstride;
    if (dir == 0) {
        if (t >= (nx - 1) * ny) return;
        const int j = t / (nx - 1), fi = 1 + t % (nx - 1);
        colL = (fi - 1) + nx * j;
        colR = fi + nx * j;
        fo = fi + (nx + 1) * j;
        fstride = (size_t)(nx + 1) * ny;
    } else {
        if (t >= nx * (ny - 1)) return;
        const int fj = 1 + t / nx, i = t % nx;
        colL = i + nx * (fj - 1);
        colR = i + nx * fj;
        fo = i + nx * fj;
        fstride = (size_t)nx * (ny + 1);
    }
    using Po = typename P::Po;
    using Ko = typename P::Ko;
    using He = typename P::He;
    const FaceOutT<P> o = dir == 0 ? a.u : a.v;
    Po* __restrict__ PoL = o.PoL + fo;
    Po* __restrict__ PoR = o.PoR + fo;
    Ko* __restrict__ KoL = o.KoL + fo;
    Ko* __restrict__ KoR = o.KoR + fo;
    He* __restrict__ hEff = o.hEff + fo;
    if constexpr (!WET_ONLY) {
        if (!sweep_face_dry<P, LD>(a, dir, t)) return;
    }

    const IfcState* XL = a.ifc + colL;
    const IfcState* XR = a.ifc + colR;
    const double* PL = a.pint + colL;
    const double* PR = a.pint + colR;
    const double pa_to_h = 1.0 / (kGravity * a.rho0);
    const int nk = nz;
    constexpr int kAhead = NR - 3;  // interfaces in flight beyond the window

#pragma unroll
    for (int q = 0; q < 3 + kAhead; ++q) {
        sw_fetch(r, 0, q, XL, PL, nk, ld);
        sw_fetch(r, 1, q, XR, PR, nk, ld);
    }
    cp_async_commit();
    cp_async_wait<0>();

    int kL = 1, kR = 1;
    double lastP_left = 0.0, lastP_right = 0.0;
    int lastK_left = 1, lastK_right = 1;
    bool reached_bottom = false, search_left = false, search_right = false;
    double absL_prev = 0.0, absR_prev = 0.0;

    for (int ks = 1; ks <= ns; ++ks) {
        if constexpr (kAhead == 0) cp_async_wait<0>();
        const int kl = kL, kr = kR;
        const IfcState oL = sw_ifc(r, 0, kl - 1), oR = sw_ifc(r, 1, kr - 1);
        const double dRho = secant_drho(oR, oL);
        if (!reached_bottom) {
            if (dRho < 0.0) {
                search_left = true;
                search_right = false;
            } else if (dRho > 0.0) {
                search_right = true;
                search_left = false;
            } else if (kl + kr == 2) {
                search_left = true;
                search_right = false;
            } else {
                search_left = !search_left;
                search_right = !search_right;
            }
        }
        const bool L = search_left;
        const int sS = L ? 0 : 1, sA = L ? 1 : 0;
        const int Sk = L ? kl : kr, ka = L ? kr : kl;
        const int w0 = Sk > 2 ? Sk - 2 : 0;  // the searched column's km1, 0-based
        const IfcState Sa = sw_ifc(r, sS, w0);
        const IfcState anc = sw_ifc(r, sA, ka - 1);
        const double dRhoTop = secant_drho(Sa, anc);
        const double dRhoBot = Sk >= 2 ? (L ? -dRho : dRho) : secant_drho(sw_ifc(r, sS, w0 + 1), anc);
        const double Spa = sw_p(r, sS, w0), Spb = sw_p(r, sS, w0 + 1);
        const int km1 = w0 + 1;
        double po_s;
        const bool top_zero = (L ? (dRhoTop > 0.0) : (dRhoTop >= 0.0)) || kr + kl == 2;
        if (top_zero) po_s = 0.0;
        else if (dRhoTop >= dRhoBot) po_s = 1.0;
        else po_s = interpolate_position(dRhoTop, Spa, dRhoBot, Spb);
        int ko_s = km1;
        bool carried = false;
        if (po_s >= 1.0 && km1 < nk) {
            ko_s = km1 + 1;
            po_s = po_s - 1.0;
            carried = true;
        }
        const int lastK_s = L ? lastK_left : lastK_right;
        const double lastP_s = L ? lastP_left : lastP_right;
        bool backstop = false;
        if ((double)(ko_s - lastK_s) + (po_s - lastP_s) < 0.0) {
            po_s = lastP_s;
            ko_s = lastK_s;
            backstop = true;
        }
        double abs_s;
        if (backstop) abs_s = L ? absL_prev : absR_prev;
        else if (carried) abs_s = Spb + po_s * (sw_p(r, sS, w0 + 2) - Spb);
        else abs_s = Spa + po_s * (Spb - Spa);
        double po_a, abs_a;
        int ko_a;
        if (ka <= nk) {
            po_a = 0.0;
            ko_a = ka;
            abs_a = sw_p(r, sA, ka - 1);
            // the anchor column advances: its window slides once k >= 2, and
            // the slot that left it receives the interface kAhead + 2 below
            // the one that entered
            if (ka >= 2) {
                if constexpr (kAhead == 2) cp_async_wait<1>();
                else if constexpr (kAhead == 1) cp_async_wait<0>();
                sw_fetch(r, sA, ka + kAhead + 1, L ? XR : XL, L ? PR : PL, nk, ld);
                cp_async_commit();
            }
            if (L) kR = ka + 1;
            else kL = ka + 1;
        } else {
            po_a = 1.0;
            ko_a = nk;
            const double Apa = sw_p(r, sA, ka - 2), Apb = sw_p(r, sA, ka - 1);
            abs_a = Apa + po_a * (Apb - Apa);  // km1 = nk: interfaces nk, nk+1
            reached_bottom = true;
            search_left = !L;
            search_right = L;
        }
        const double pol = L ? po_s : po_a, por = L ? po_a : po_s;
        const int kol = L ? ko_s : ko_a, kor = L ? ko_a : ko_s;
        const double absL = L ? abs_s : abs_a, absR = L ? abs_a : abs_s;
        lastK_left = kol;
        lastP_left = pol;
        lastK_right = kor;
        lastP_right = por;
        const size_t so = (size_t)(ks - 1) * fstride;
        PoL[so] = Po(pol);
        PoR[so] = Po(por);
        KoL[so] = Ko(kol);
        KoR[so] = Ko(kor);
        if (ks > 1) {  // harmonic-mean effective thickness (:452-462), Pa -> m (:688-691)
            const double hL = absL - absL_prev;
            const double hR = absR - absR_prev;
            double he = 0.0;
            if (hL + hR > 0.0) he = 2.0 * hL * hR / (hL + hR);
            hEff[so - fstride] = He(he * pa_to_h);
        }
        absL_prev = absL;
        absR_prev = absR;
    }
    cp_async_wait<0>();  // no copy may land in the ring after this face is done
}

// ---------------------------------------------------------------------------
// Phase B, step 1: per-column tracer reconstruction for a group of NT tracers
// (redi_tracer_column, ocean_redi.F90:852-891). Writes, per tracer, the nz+1
// interface values Tint and the nz prepared PPM layers in [layer][column]
// order, so that threads of neighbouring columns touch neighbouring addresses.
// ---------------------------------------------------------------------------
template <class P>
__device__ __forceinline__ void store_ppm(typename P::Ppm* p, const PpmLayer& q);
template <>
__device__ __forceinline__ void store_ppm<PlainPrec>(PpmLayer* p, const PpmLayer& q) {
    double2* d = reinterpret_cast<double2*>(p);
    d[0] = make_double2(q.aL, q.dA);
    d[1] = make_double2(q.a6o3, q.B);
}
template <>
__device__ __forceinline__ void store_ppm<MixedPrec>(PpmLayerF* p, const PpmLayer& q) {
    *reinterpret_cast<float4*>(p) = make_float4((float)q.aL, (float)q.dA, (float)q.a6o3, (float)q.B);
}

template <int NT, class P, class LD>
// gid enumerates (tracer group, column) over the columns [c0, c0 + nb).
__device__ __forceinline__ void recon_item(const ReconArgsT<P>& a, int gid, int c0, int nb) {
    const int ncol = a.nx * a.ny;
    const int ngroups = (a.ntr + NT - 1) / NT;
    if (gid >= nb * ngroups) return;
    const int col = c0 + gid % nb;
    if (a.dry_u) {  // the face flux reads a column only for a face that is not dry
        const uint8_t* du = a.dry_u;
        const uint8_t* dv = a.dry_v;
        if (!column_needed(col, a.nx, a.ny, [du](int f) { return LD::ld(du + f) == 0; },
                           [dv](int f) { return LD::ld(dv + f) == 0; }))
            return;
    }
    const int g = gid / nb;
    const int tr0 = g * NT;
    const int nt = min(NT, a.ntr - tr0);
    const int nz = a.nz;
    const double* __restrict__ h = a.h + col;
    const double* htr[NT];
    double* ti[NT];
    typename P::Ppm* ppm[NT];
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        const int tr = tr0 + (n < nt ? n : 0);
        htr[n] = a.htr[tr] + col;
        ti[n] = a.ti + (size_t)tr * ncol * (nz + 1) + col;
        ppm[n] = a.ppm + (size_t)tr * ncol * nz + col;
    }
    double e_prev[NT];

    auto fetch = [&](int t, RawLayer<NT>& r) {
        const size_t off = (size_t)(nz - t) * ncol;
        r.h = LD::ld(h + off);
#pragma unroll
        for (int n = 0; n < NT; ++n) r.s[n] = LD::ld(htr[n] + off);
    };
    auto emit = [&](int t, const double (&e)[NT], const double (&s_above)[NT], double) {
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            if (n < nt) {
                ti[n][(size_t)(t - 1) * ncol] = e[n];
                if (t >= 2) {  // layer t-1 is complete: limit its edges
                    double alk = e_prev[n], ark = e[n];
                    const double tlk = s_above[n];
                    ppm_limit(alk, ark, tlk);
                    store_ppm<P>(ppm[n] + (size_t)(t - 2) * ncol, make_ppm_layer(alk, ark, tlk));
                }
            }
            e_prev[n] = e[n];
        }
    };
    stream_edges<NT, decltype(fetch), decltype(emit), kReconAhead>(nz, fetch, emit);
}

// ---------------------------------------------------------------------------
// Phase A's column state and Phase B's reconstruction of T and S in one pass
// (a whole step in one call: nothing can change the tracers in between).
// Both passes stream the same top-down PPM edges of hT and hS over the same
// thicknesses (stream_edges), so one stream feeds both: the EOS state and
// pressure of every interface (column_state_item) and the interface values and
// limited PPM layers of tracers 0 and 1 of the reconstruction buffer
// (recon_item), which are T and S (ts_swap: tracer 0 is S). The values are
// those of the two passes bit for bit. A column none of whose faces is wet is
// read by neither the sweep nor the face flux, and is skipped.
// ---------------------------------------------------------------------------
template <class P, class LD>
__device__ __forceinline__ void column_recon_item(const ColumnStateArgs& a, const ReconArgsT<P>& rc, int ts_swap,
                                                  int col) {
    const int ncol = a.nx * a.ny;
    const int nz = a.nz;
    if (a.wet_u) {
        const double* wu = a.wet_u;
        const double* wv = a.wet_v;
        if (!column_needed(col, a.nx, a.ny, [wu](int f) { return LD::ld(wu + f) > 0.0; },
                           [wv](int f) { return LD::ld(wv + f) > 0.0; }))
            return;
    }
    const double* __restrict__ h = a.h + col;
    const double* __restrict__ tr0 = rc.htr[0] + col;
    const double* __restrict__ tr1 = rc.htr[1] + col;
    IfcState* __restrict__ ifc = a.ifc + col;
    double* __restrict__ pint = a.pint + col;
    double* __restrict__ ti[2] = {rc.ti + col, rc.ti + (size_t)ncol * (nz + 1) + col};
    typename P::Ppm* __restrict__ ppm[2] = {rc.ppm + col, rc.ppm + (size_t)ncol * nz + col};

    const EosParams eos = a.eos;
    const bool linear = eos_is_linear(eos.variant);
    const double dsv_dt = eos.alpha_T / (eos.rho0 * eos.rho0);  // ocean_eos.F90:511
    const double dsv_ds = -eos.beta_S / (eos.rho0 * eos.rho0);  // ocean_eos.F90:512
    const double grho = kGravity * eos.rho0;
    const int iT = ts_swap ? 1 : 0, iS = ts_swap ? 0 : 1;
    double pres = 0.0;  // interface pressure
    double h_layer_above = 0.0;
    double e_prev[2];

    auto fetch = [&](int t, RawLayer<2>& r) {
        const size_t off = (size_t)(nz - t) * ncol;  // native k = nz+1-t (1-based)
        r.h = LD::ld(h + off);
        r.s[0] = LD::ld(tr0 + off);
        r.s[1] = LD::ld(tr1 + off);
    };
    auto emit = [&](int t, const double (&e)[2], const double (&s_above)[2], double h_t) {
        // column state (column_state_item)
        if (t >= 2) pres = pres + grho * h_layer_above;
        const double eT = e[iT], eS = e[iS];
        double rho_i, sv_t = dsv_dt, sv_s = dsv_ds;
        if (linear)
            rho_i = eos.rho0 + eos.beta_S * (eS - eos.S_ref) - eos.alpha_T * (eT - eos.T_ref);
        else
            eos::nonlinear_point(eos.variant, eT, eS, pres, rho_i, sv_t, sv_s);
        double2* q = reinterpret_cast<double2*>(ifc + (size_t)(t - 1) * ncol);
        q[0] = make_double2(eT, eS);
        q[1] = make_double2(-(rho_i * rho_i) * sv_t, -(rho_i * rho_i) * sv_s);
        pint[(size_t)(t - 1) * ncol] = pres;
        h_layer_above = h_t;
        // reconstruction (recon_item)
#pragma unroll
        for (int n = 0; n < 2; ++n) {
            ti[n][(size_t)(t - 1) * ncol] = e[n];
            if (t >= 2) {
                double alk = e_prev[n], ark = e[n];
                const double tlk = s_above[n];
                ppm_limit(alk, ark, tlk);
                store_ppm<P>(ppm[n] + (size_t)(t - 2) * ncol, make_ppm_layer(alk, ark, tlk));
            }
            e_prev[n] = e[n];
        }
    };
    stream_edges<2, decltype(fetch), decltype(emit), kColumnAhead>(nz, fetch, emit);
}

// ---------------------------------------------------------------------------
// Phase B, step 2: the along-neutral flux of every face, computed once
// (redi_face_flux + redi_sublayer_dT, ocean_redi.F90:893-925, 1037-1092).
//
// One thread per interior, non-wall face; all lanes of a warp walk the same
// sublayer ks, so each coefficient load is one contiguous row. The flux
// flx(ks) = dT * hEff * coef of every tracer is stored in F[tracer][ks][face];
// sublayers with hEff == 0 store +0.0. The reference evaluates each interior
// face twice (once from each adjacent cell, with identical operands and hence
// identical bits); here it is evaluated once and read by both cells.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double interp(double P, double a, double b) { return (1.0 - P) * a + P * b; }

// Layer mean of the PPM parabola and the flux product, per precision. `load`
// fetches a prepared layer, `mean` evaluates it (split so that every load of a
// sublayer can be issued before any of them is used).
template <class P>
struct FluxOps;

template <>
struct FluxOps<PlainPrec> {
    using Mean = double;
    using Raw = PpmLayer;
    template <class LD>
    __device__ static __forceinline__ Raw load(const PpmLayer* p) {
        return load_ppm<LD>(p);
    }
    __device__ static __forceinline__ double mean(double xL, double xR, const Raw& q) { return ppm_ave(xL, xR, q); }
    __device__ static __forceinline__ double flux(double dT, double he, double coef) { return dT * he * coef; }
};

template <>
struct FluxOps<MixedPrec> {
    using Mean = float;
    using Raw = float4;  // aL, dA, a6o3, B
    template <class LD>
    __device__ static __forceinline__ Raw load(const PpmLayerF* p) {
        return LD::ld(reinterpret_cast<const float4*>(p));
    }
    // redi_ppm_ave in FP32; the branch (a discrete decision) is taken on the
    // FP64 positions exactly as in the plain form.
    __device__ static __forceinline__ float mean(double xL, double xR, const Raw& q) {
        const float xl = (float)xL, xr = (float)xR;
        const double dx = xR - xL;
        if (dx > 0.0 && dx <= 1.0) {
            const float xave = 0.5f * (xr + xl);
            return (q.x + xave * q.w) - q.z * (xr * xr + xr * xl + xl * xl);
        }
        const float a6 = 3.0f * q.z;
        return q.x + q.y * xr + a6 * xr * (1.0f - xr);
    }
    __device__ static __forceinline__ float flux(double dT, float he, double coef) {
        return (float)dT * he * (float)coef;
    }
};

// Whether face t of direction dir (t < t_end) is one flux_item computes:
// an interior face of the launch's range that is neither a wall nor dry.
template <class P>
__device__ __forceinline__ bool flux_face_valid(const FaceFluxArgsT<P>& a, int dir, int t, int t_end) {
    const int nx = a.nx, ny = a.ny;
    if (dir == 0) {
        if (!(t < min(t_end, (nx - 1) * ny))) return false;
        const int j = t / (nx - 1), fi = 1 + t % (nx - 1), I = fi + 1;
        if ((a.wall_w && I == a.nghost + 1) || (a.wall_e && I == a.nghost + a.nxp + 1)) return false;
        return !(a.u.dry && a.u.dry[fi + (nx + 1) * j]);
    }
    if (!(t < min(t_end, nx * (ny - 1)))) return false;
    const int fj = 1 + t / nx, i = t % nx, J = fj + 1;
    if ((a.wall_s && J == a.nghost + 1) || (a.wall_n && J == a.nghost + a.nyp + 1)) return false;
    return !(a.v.dry && a.v.dry[i + nx * fj]);
}

// Every lane of the warp must call this (no lane may have exited): lanes
// without a face of their own (grid tail, wall faces) walk face 0 of their
// direction as a stand-in, load like the others and store nothing, so the
// warp-wide vote below is well defined. A warp whose every lane has
// hEff == 0 at a sublayer (land, outcropped layers) skips that sublayer's
// loads; otherwise the whole warp issues a pair of tracers' loads for the
// sublayer (bottom surface tracer values, PPM layers, and top values after a
// skip) as one batch before any of them is used, so each sublayer costs one
// memory round trip per tracer pair.
template <int NT, class P, class LD>
// t enumerates the faces of direction dir; faces at t >= t_end (the end of the
// launch's band, at most the direction's face count) are not this call's.
__device__ __forceinline__ void flux_item(const FaceFluxArgsT<P>& a, int dir, int t, int tr0, int t_end) {
    using Ops = FluxOps<P>;
    using Raw = typename Ops::Raw;
    using He = typename P::He;
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    const size_t ncol = (size_t)nx * ny;
    int colL, colR, fo;
    size_t fstride;
    bool valid;
    if ((dir == 0 ? (nx - 1) * ny : nx * (ny - 1)) <= 0) return;  // no face 0 to stand in
    if (dir == 0) {  // Fortran faces I = 2..nx, excluding walls
        valid = t < min(t_end, (nx - 1) * ny);
        const int tt = valid ? t : 0;
        const int j = tt / (nx - 1), fi = 1 + tt % (nx - 1);
        const int I = fi + 1;
        valid = valid && !((a.wall_w && I == a.nghost + 1) || (a.wall_e && I == a.nghost + a.nxp + 1));
        colL = (fi - 1) + nx * j;
        colR = fi + nx * j;
        fo = fi + (nx + 1) * j;
        fstride = (size_t)(nx + 1) * ny;
    } else {  // Fortran faces J = 2..ny, excluding walls
        valid = t < min(t_end, nx * (ny - 1));
        const int tt = valid ? t : 0;
        const int fj = 1 + tt / nx, i = tt % nx;
        const int J = fj + 1;
        valid = valid && !((a.wall_s && J == a.nghost + 1) || (a.wall_n && J == a.nghost + a.nyp + 1));
        colL = i + nx * (fj - 1);
        colR = i + nx * fj;
        fo = i + nx * fj;
        fstride = (size_t)nx * (ny + 1);
    }
    {   // a dry face (inert coefficients) has only +0.0 fluxes: nothing is
        // stored and the gather skips it
        const uint8_t* dry = dir == 0 ? a.u.dry : a.v.dry;
        if (dry && valid && LD::ld(dry + fo)) valid = false;
    }
    if (!__any_sync(0xffffffffu, valid)) return;  // warp-uniform
    const FaceInT<P>& c = dir == 0 ? a.u : a.v;
    const He* __restrict__ hEff = c.hEff + fo;
    const typename P::Po* __restrict__ PoL = c.PoL + fo;
    const typename P::Po* __restrict__ PoR = c.PoR + fo;
    const typename P::Ko* __restrict__ KoL = c.KoL + fo;
    const typename P::Ko* __restrict__ KoR = c.KoR + fo;
    const double* kh = dir == 0 ? a.khtr_u : a.khtr_v;
    const double khv = kh ? LD::ld(kh + fo) : a.khtr;
    // ((dt*khtr)*dy)*idx, ocean_redi.F90:1156/1168
    const double coef = a.dt * khv * LD::ld((dir == 0 ? a.dy_cu : a.dx_cv) + fo) *
                        LD::ld((dir == 0 ? a.idxCu : a.idyCv) + fo);
    const int nt = min(NT, a.ntr - tr0);
    // Tracers of the group sit at fixed strides in the scratch; a tracer slot
    // beyond nt reads tracer tr0 and stores nothing.
    const size_t ti_stride = ncol * (nz + 1), pp_stride = ncol * nz, f_stride = (size_t)(ns - 1) * fstride;
    const double* const tiL0 = a.ti + (size_t)tr0 * ti_stride + colL;
    const double* const tiR0 = a.ti + (size_t)tr0 * ti_stride + colR;
    const typename P::Ppm* const ppL0 = a.ppm + (size_t)tr0 * pp_stride + colL;
    const typename P::Ppm* const ppR0 = a.ppm + (size_t)tr0 * pp_stride + colR;
    typename P::Flux* const Fo0 = (dir == 0 ? a.Fu : a.Fv) + fo + (size_t)a.fslot0 * f_stride;
    auto trc = [nt](int n) { return (size_t)(n < nt ? n : 0); };

    // Register rotation: while sublayer s is evaluated, hEff(s+1) and the
    // bottom surface of s+1 (surface s+2) are already being fetched. The top
    // surface of s is the bottom surface of s-1 (tl/tr carry its tracer
    // values unless the previous sublayer was skipped by the whole warp).
    bool have_t = false;  // warp-uniform
    int kl_t = min(max((int)LD::ld(KoL), 1), nz), kr_t = min(max((int)LD::ld(KoR), 1), nz);
    double pl_t = LD::ld(PoL), pr_t = LD::ld(PoR);
    He he_c = LD::ld(hEff);
    int klr_c = LD::ld(KoL + fstride), krr_c = LD::ld(KoR + fstride);
    double pl_c = LD::ld(PoL + fstride), pr_c = LD::ld(PoR + fstride);
    double tl[NT], tr[NT];
    for (int s = 0; s < ns - 1; ++s) {
        const size_t s0 = (size_t)s * fstride;
        He he_n = He(0);
        int klr_n = 1, krr_n = 1;
        double pl_n = 0.0, pr_n = 0.0;
        if (s + 1 < ns - 1) {
            const size_t s2 = s0 + 2 * fstride;
            he_n = LD::ld(hEff + s0 + fstride);
            klr_n = LD::ld(KoL + s2);
            krr_n = LD::ld(KoR + s2);
            pl_n = LD::ld(PoL + s2);
            pr_n = LD::ld(PoR + s2);
        }
        const int kl_b = min(max(klr_c, 1), nz);
        const int kr_b = min(max(krr_c, 1), nz);
        const double pl_b = pl_c, pr_b = pr_c;
        const bool live = valid && he_c != He(0);
        if (!__any_sync(0xffffffffu, live)) {
#pragma unroll
            for (int n = 0; n < NT; ++n)
                if (valid && n < nt) Fo0[(size_t)n * f_stride + s0] = typename P::Flux(0);
            have_t = false;
        } else {
            const double xRl = pl_b + (double)(kl_b - kl_t);
            const double xRr = pr_b + (double)(kr_b - kr_t);
            // Tracers in pairs, one load batch per pair: bottom-surface tracer
            // values and the top layer's PPM, then (after a skip) the
            // top-surface values; the compiler barrier keeps the next pair's
            // loads from being hoisted into this batch (register budget).
#pragma unroll
            for (int p = 0; p < NT; p += 2) {
                constexpr int W = NT < 2 ? NT : 2;
                double b0L[W], b1L[W], b0R[W], b1R[W];
                Raw qL[W], qR[W];
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    const int n = p + w;
                    b0L[w] = LD::ld(tiL0 + trc(n) * ti_stride + (size_t)(kl_b - 1) * ncol);
                    b1L[w] = LD::ld(tiL0 + trc(n) * ti_stride + (size_t)kl_b * ncol);
                    b0R[w] = LD::ld(tiR0 + trc(n) * ti_stride + (size_t)(kr_b - 1) * ncol);
                    b1R[w] = LD::ld(tiR0 + trc(n) * ti_stride + (size_t)kr_b * ncol);
                    qL[w] = Ops::template load<LD>(ppL0 + trc(n) * pp_stride + (size_t)(kl_t - 1) * ncol);
                    qR[w] = Ops::template load<LD>(ppR0 + trc(n) * pp_stride + (size_t)(kr_t - 1) * ncol);
                }
                if (!have_t) {
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const int n = p + w;
                        tl[n] = interp(pl_t, LD::ld(tiL0 + trc(n) * ti_stride + (size_t)(kl_t - 1) * ncol),
                                       LD::ld(tiL0 + trc(n) * ti_stride + (size_t)kl_t * ncol));
                        tr[n] = interp(pr_t, LD::ld(tiR0 + trc(n) * ti_stride + (size_t)(kr_t - 1) * ncol),
                                       LD::ld(tiR0 + trc(n) * ti_stride + (size_t)kr_t * ncol));
                    }
                }
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    const int n = p + w;
                    const double bl = interp(pl_b, b0L[w], b1L[w]);
                    const double br = interp(pr_b, b0R[w], b1R[w]);
                    if (valid && n < nt) {
                        const typename Ops::Mean tlay = Ops::mean(pl_t, xRl, qL[w]);
                        const typename Ops::Mean trlay = Ops::mean(pr_t, xRr, qR[w]);
                        const double dT = guarded_dT(tr[n] - tl[n], br - bl, (double)(trlay - tlay));
                        Fo0[(size_t)n * f_stride + s0] = he_c == He(0) ? typename P::Flux(0) : Ops::flux(dT, he_c, coef);
                    }
                    tl[n] = bl;
                    tr[n] = br;
                }
                if (p + 2 < NT) asm volatile("" ::: "memory");
            }
            have_t = true;
        }
        kl_t = kl_b;
        kr_t = kr_b;
        pl_t = pl_b;
        pr_t = pr_b;
        he_c = he_n;
        klr_c = klr_n;
        krr_c = krr_n;
        pl_c = pl_n;
        pr_c = pr_n;
    }
}

// ---------------------------------------------------------------------------
// The face flux with its reconstruction loads staged one sublayer ahead.
//
// flux_item waits one memory round trip per sublayer: the reconstruction
// values a sublayer needs sit at layers given by its own Ko. Here the Ko of
// the next sublayer is known one iteration early (the coefficients run two
// surfaces ahead), so its reconstruction values are copied into this thread's
// slots in shared memory with cp.async while the current sublayer is
// evaluated from the other slot; the copies hold no registers while in
// flight. The arithmetic, the values and the stores are exactly flux_item's.
// Per thread and slot (sublayer parity), structure of arrays so that the
// threads of a warp touch consecutive words:
//   ti [slot][tracer][8][kFluxThreads] doubles: bottom-surface interface
//      values L0, L1, R0, R1, then the top-surface ones (staged only after a
//      sublayer that the whole warp skipped);
//   pp [slot][tracer][side][kU][kFluxThreads] 16-byte units: the prepared PPM
//      layer of the top layer, left then right column.
// ---------------------------------------------------------------------------
constexpr int kFluxThreads = 128;

template <class P>
struct PpmUnits;
template <>
struct PpmUnits<PlainPrec> {
    static constexpr int n = 2;
};
template <>
struct PpmUnits<MixedPrec> {
    static constexpr int n = 1;
};

template <int NT, class P>
struct FluxStage {
    static constexpr int kU = PpmUnits<P>::n;
    static constexpr size_t ti_doubles = (size_t)2 * NT * 8 * kFluxThreads;
    static constexpr size_t pp_units = (size_t)2 * NT * 2 * kU * kFluxThreads;
    static constexpr size_t bytes = ti_doubles * 8 + pp_units * 16;
};

template <class P>
__device__ __forceinline__ typename FluxOps<P>::Raw ld_stage_ppm(const double2* u);
template <>
__device__ __forceinline__ PpmLayer ld_stage_ppm<PlainPrec>(const double2* u) {
    const double2 a = u[0], b = u[kFluxThreads];
    PpmLayer r;
    r.aL = a.x; r.dA = a.y; r.a6o3 = b.x; r.B = b.y;
    return r;
}
template <>
__device__ __forceinline__ float4 ld_stage_ppm<MixedPrec>(const double2* u) {
    return *reinterpret_cast<const float4*>(u);
}

template <int NT, class P>
__device__ __forceinline__ void flux_item_staged(const FaceFluxArgsT<P>& a, int dir, int t, int tr0, int t_end,
                                                 double* __restrict__ sti, double2* __restrict__ spp) {
    using Ops = FluxOps<P>;
    using Raw = typename Ops::Raw;
    using He = typename P::He;
    constexpr int kU = PpmUnits<P>::n;
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    const size_t ncol = (size_t)nx * ny;
    const int tid = threadIdx.x;
    int colL, colR, fo;
    size_t fstride;
    bool valid;
    if ((dir == 0 ? (nx - 1) * ny : nx * (ny - 1)) <= 0) return;  // no face 0 to stand in
    if (dir == 0) {
        valid = t < min(t_end, (nx - 1) * ny);
        const int tt = valid ? t : 0;
        const int j = tt / (nx - 1), fi = 1 + tt % (nx - 1);
        const int I = fi + 1;
        valid = valid && !((a.wall_w && I == a.nghost + 1) || (a.wall_e && I == a.nghost + a.nxp + 1));
        colL = (fi - 1) + nx * j;
        colR = fi + nx * j;
        fo = fi + (nx + 1) * j;
        fstride = (size_t)(nx + 1) * ny;
    } else {
        valid = t < min(t_end, nx * (ny - 1));
        const int tt = valid ? t : 0;
        const int fj = 1 + tt / nx, i = tt % nx;
        const int J = fj + 1;
        valid = valid && !((a.wall_s && J == a.nghost + 1) || (a.wall_n && J == a.nghost + a.nyp + 1));
        colL = i + nx * (fj - 1);
        colR = i + nx * fj;
        fo = i + nx * fj;
        fstride = (size_t)nx * (ny + 1);
    }
    {   // a dry face (inert coefficients) has only +0.0 fluxes: nothing is
        // stored and the gather skips it
        const uint8_t* dry = dir == 0 ? a.u.dry : a.v.dry;
        if (dry && valid && dry[fo]) valid = false;
    }
    if (!__any_sync(0xffffffffu, valid)) return;  // warp-uniform
    const FaceInT<P>& c = dir == 0 ? a.u : a.v;
    const He* __restrict__ hEff = c.hEff + fo;
    const typename P::Po* __restrict__ PoL = c.PoL + fo;
    const typename P::Po* __restrict__ PoR = c.PoR + fo;
    const typename P::Ko* __restrict__ KoL = c.KoL + fo;
    const typename P::Ko* __restrict__ KoR = c.KoR + fo;
    const double* kh = dir == 0 ? a.khtr_u : a.khtr_v;
    const double khv = kh ? __ldg(kh + fo) : a.khtr;
    // ((dt*khtr)*dy)*idx, ocean_redi.F90:1156/1168
    const double coef = a.dt * khv * __ldg((dir == 0 ? a.dy_cu : a.dx_cv) + fo) *
                        __ldg((dir == 0 ? a.idxCu : a.idyCv) + fo);
    const int nt = min(NT, a.ntr - tr0);
    const size_t ti_stride = ncol * (nz + 1), pp_stride = ncol * nz, f_stride = (size_t)(ns - 1) * fstride;
    const double* const tiL0 = a.ti + (size_t)tr0 * ti_stride + colL;
    const double* const tiR0 = a.ti + (size_t)tr0 * ti_stride + colR;
    const typename P::Ppm* const ppL0 = a.ppm + (size_t)tr0 * pp_stride + colL;
    const typename P::Ppm* const ppR0 = a.ppm + (size_t)tr0 * pp_stride + colR;
    typename P::Flux* const Fo0 = (dir == 0 ? a.Fu : a.Fv) + fo + (size_t)a.fslot0 * f_stride;
    auto trc = [nt](int n) { return (size_t)(n < nt ? n : 0); };
    auto sti_at = [&](int slot, int n, int w) { return sti + ((size_t)((slot * NT + n) * 8 + w)) * kFluxThreads + tid; };
    auto spp_at = [&](int slot, int n, int side) {
        return spp + ((size_t)(((slot * NT + n) * 2 + side) * kU)) * kFluxThreads + tid;
    };
    // The staged loads of one sublayer: the bottom surface's interface values
    // at (klb, krb), the top layer's PPM at (klt, krt) and, if top, the top
    // surface's interface values.
    auto issue = [&](int slot, int klt, int krt, int klb, int krb, bool top) {
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            const double* tL = tiL0 + trc(n) * ti_stride;
            const double* tR = tiR0 + trc(n) * ti_stride;
            cp_async8(sti_at(slot, n, 0), tL + (size_t)(klb - 1) * ncol);
            cp_async8(sti_at(slot, n, 1), tL + (size_t)klb * ncol);
            cp_async8(sti_at(slot, n, 2), tR + (size_t)(krb - 1) * ncol);
            cp_async8(sti_at(slot, n, 3), tR + (size_t)krb * ncol);
            if (top) {
                cp_async8(sti_at(slot, n, 4), tL + (size_t)(klt - 1) * ncol);
                cp_async8(sti_at(slot, n, 5), tL + (size_t)klt * ncol);
                cp_async8(sti_at(slot, n, 6), tR + (size_t)(krt - 1) * ncol);
                cp_async8(sti_at(slot, n, 7), tR + (size_t)krt * ncol);
            }
            const char* pL = reinterpret_cast<const char*>(ppL0 + trc(n) * pp_stride + (size_t)(klt - 1) * ncol);
            const char* pR = reinterpret_cast<const char*>(ppR0 + trc(n) * pp_stride + (size_t)(krt - 1) * ncol);
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                cp_async16(spp_at(slot, n, 0) + (size_t)u * kFluxThreads, pL + 16 * u);
                cp_async16(spp_at(slot, n, 1) + (size_t)u * kFluxThreads, pR + 16 * u);
            }
        }
    };

    // Coefficients: top surface s, bottom s+1 (hEff(s)), next s+2 (hEff(s+1)),
    // and s+3 (hEff(s+2)) in flight.
    int kl_t = min(max((int)__ldg(KoL), 1), nz), kr_t = min(max((int)__ldg(KoR), 1), nz);
    double pl_t = __ldg(PoL), pr_t = __ldg(PoR);
    He he_c = __ldg(hEff);
    int klr_c = __ldg(KoL + fstride), krr_c = __ldg(KoR + fstride);
    double pl_c = __ldg(PoL + fstride), pr_c = __ldg(PoR + fstride);
    He he_n = He(0);
    int klr_n = 1, krr_n = 1;
    double pl_n = 0.0, pr_n = 0.0;
    if (ns - 1 > 1) {
        he_n = __ldg(hEff + fstride);
        klr_n = __ldg(KoL + 2 * fstride);
        krr_n = __ldg(KoR + 2 * fstride);
        pl_n = __ldg(PoL + 2 * fstride);
        pr_n = __ldg(PoR + 2 * fstride);
    }
    bool staged = __any_sync(0xffffffffu, valid && he_c != He(0));  // sublayer 0 staged (warp-uniform)
    if (staged) issue(0, kl_t, kr_t, min(max(klr_c, 1), nz), min(max(krr_c, 1), nz), true);
    cp_async_commit();
    bool have_t = false;  // tl / tr hold the top surface's values (warp-uniform)
    double tl[NT], tr[NT];
    for (int s = 0; s < ns - 1; ++s) {
        const size_t s0 = (size_t)s * fstride;
        He he_nn = He(0);
        int klr_nn = 1, krr_nn = 1;
        double pl_nn = 0.0, pr_nn = 0.0;
        if (s + 2 < ns - 1) {
            const size_t s3 = s0 + 3 * fstride;
            he_nn = __ldg(hEff + s0 + 2 * fstride);
            klr_nn = __ldg(KoL + s3);
            krr_nn = __ldg(KoR + s3);
            pl_nn = __ldg(PoL + s3);
            pr_nn = __ldg(PoR + s3);
        }
        const int kl_b = min(max(klr_c, 1), nz), kr_b = min(max(krr_c, 1), nz);
        const double pl_b = pl_c, pr_b = pr_c;
        // the next sublayer's loads: its top surface is this one's bottom
        bool staged_next = false;
        if (s + 1 < ns - 1) {
            staged_next = __any_sync(0xffffffffu, valid && he_n != He(0));
            if (staged_next)
                issue((s + 1) & 1, kl_b, kr_b, min(max(klr_n, 1), nz), min(max(krr_n, 1), nz), !staged);
        }
        cp_async_commit();
        const int slot = s & 1;
        if (staged) {
            cp_async_wait<1>();  // this sublayer's group (only the next one may still be in flight)
            const double xRl = pl_b + (double)(kl_b - kl_t);
            const double xRr = pr_b + (double)(kr_b - kr_t);
#pragma unroll
            for (int n = 0; n < NT; ++n) {
                if (!have_t) {
                    tl[n] = interp(pl_t, *sti_at(slot, n, 4), *sti_at(slot, n, 5));
                    tr[n] = interp(pr_t, *sti_at(slot, n, 6), *sti_at(slot, n, 7));
                }
                const double bl = interp(pl_b, *sti_at(slot, n, 0), *sti_at(slot, n, 1));
                const double br = interp(pr_b, *sti_at(slot, n, 2), *sti_at(slot, n, 3));
                if (valid && n < nt) {
                    const Raw qL = ld_stage_ppm<P>(spp_at(slot, n, 0));
                    const Raw qR = ld_stage_ppm<P>(spp_at(slot, n, 1));
                    const typename Ops::Mean tlay = Ops::mean(pl_t, xRl, qL);
                    const typename Ops::Mean trlay = Ops::mean(pr_t, xRr, qR);
                    const double dT = guarded_dT(tr[n] - tl[n], br - bl, (double)(trlay - tlay));
                    Fo0[(size_t)n * f_stride + s0] = he_c == He(0) ? typename P::Flux(0) : Ops::flux(dT, he_c, coef);
                }
                tl[n] = bl;
                tr[n] = br;
            }
            have_t = true;
        } else {
#pragma unroll
            for (int n = 0; n < NT; ++n)
                if (valid && n < nt) Fo0[(size_t)n * f_stride + s0] = typename P::Flux(0);
            have_t = false;
        }
        kl_t = kl_b;
        kr_t = kr_b;
        pl_t = pl_b;
        pr_t = pr_b;
        he_c = he_n;
        klr_c = klr_n;
        krr_c = krr_n;
        pl_c = pl_n;
        pr_c = pr_n;
        he_n = he_nn;
        klr_n = klr_nn;
        krr_n = krr_nn;
        pl_n = pl_nn;
        pr_n = pr_nn;
        staged = staged_next;
    }
    cp_async_wait<0>();  // nothing may land in the slots after this face is done
}

// ---------------------------------------------------------------------------
// The face flux reading each column's reconstruction through a two-layer ring
// in shared memory.
//
// Along a face the layer of each column's bottom surface never decreases and
// moves by one layer at a time, so per column side the sublayer walk needs the
// record of its current layer c (the prepared PPM layer and the interface value
// at the layer's bottom, Ti[c]) and, when the next surface moves down, the
// record of layer c + 1; Ti[c - 1] (the current layer's top interface) stays in
// a register. Record c + 1 is copied into the ring (cp.async) when the side
// enters layer c, so a sublayer that advances finds it in shared memory instead
// of waiting on a global load whose address its own Ko gives; every layer record
// is fetched once per face side instead of once per sublayer.
// A sublayer whose layers the ring does not hold (the first live sublayer of a
// face, the first after a run the whole warp skipped, a jump of more than one
// layer) loads as flux_item does and re-primes the ring. The arithmetic, the
// values and the stores are exactly flux_item's.
// Per thread, structure of arrays over the block's threads:
//   rpp [slot][side][tracer][kU][kFluxThreads] 16-byte units (PPM record),
//   rti [slot][side][tracer][kFluxThreads] doubles (Ti at the layer's bottom),
// slot = layer & 1.
// ---------------------------------------------------------------------------
template <int NT, class P>
struct FluxRing {
    static constexpr int kU = PpmUnits<P>::n;
    static constexpr size_t pp_units = (size_t)2 * 2 * NT * kU * kFluxThreads;
    static constexpr size_t ti_doubles = (size_t)2 * 2 * NT * kFluxThreads;
    static constexpr size_t bytes = pp_units * 16 + ti_doubles * 8;
};

template <int NT, class P>
__device__ __forceinline__ void flux_item_ring(const FaceFluxArgsT<P>& a, int dir, int t, int tr0, int t_end,
                                               double2* __restrict__ rpp, double* __restrict__ rti) {
    using Ops = FluxOps<P>;
    using Raw = typename Ops::Raw;
    using He = typename P::He;
    using Ppm = typename P::Ppm;
    constexpr int kU = PpmUnits<P>::n;
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    const size_t ncol = (size_t)nx * ny;
    const int tid = threadIdx.x;
    int colL, colR, fo;
    size_t fstride;
    bool valid;
    if ((dir == 0 ? (nx - 1) * ny : nx * (ny - 1)) <= 0) return;  // no face 0 to stand in
    if (dir == 0) {
        valid = t < min(t_end, (nx - 1) * ny);
        const int tt = valid ? t : 0;
        const int j = tt / (nx - 1), fi = 1 + tt % (nx - 1);
        const int I = fi + 1;
        valid = valid && !((a.wall_w && I == a.nghost + 1) || (a.wall_e && I == a.nghost + a.nxp + 1));
        colL = (fi - 1) + nx * j;
        colR = fi + nx * j;
        fo = fi + (nx + 1) * j;
        fstride = (size_t)(nx + 1) * ny;
    } else {
        valid = t < min(t_end, nx * (ny - 1));
        const int tt = valid ? t : 0;
        const int fj = 1 + tt / nx, i = tt % nx;
        const int J = fj + 1;
        valid = valid && !((a.wall_s && J == a.nghost + 1) || (a.wall_n && J == a.nghost + a.nyp + 1));
        colL = i + nx * (fj - 1);
        colR = i + nx * fj;
        fo = i + nx * fj;
        fstride = (size_t)nx * (ny + 1);
    }
    {   // a dry face (inert coefficients) has only +0.0 fluxes: nothing is
        // stored and the gather skips it
        const uint8_t* dry = dir == 0 ? a.u.dry : a.v.dry;
        if (dry && valid && dry[fo]) valid = false;
    }
    if (!__any_sync(0xffffffffu, valid)) return;  // warp-uniform
    const FaceInT<P>& c = dir == 0 ? a.u : a.v;
    const He* __restrict__ hEff = c.hEff + fo;
    const typename P::Po* __restrict__ PoL = c.PoL + fo;
    const typename P::Po* __restrict__ PoR = c.PoR + fo;
    const typename P::Ko* __restrict__ KoL = c.KoL + fo;
    const typename P::Ko* __restrict__ KoR = c.KoR + fo;
    const double* kh = dir == 0 ? a.khtr_u : a.khtr_v;
    const double khv = kh ? __ldg(kh + fo) : a.khtr;
    // ((dt*khtr)*dy)*idx, ocean_redi.F90:1156/1168
    const double coef = a.dt * khv * __ldg((dir == 0 ? a.dy_cu : a.dx_cv) + fo) *
                        __ldg((dir == 0 ? a.idxCu : a.idyCv) + fo);
    const int nt = min(NT, a.ntr - tr0);
    const size_t ti_stride = ncol * (nz + 1), pp_stride = ncol * nz, f_stride = (size_t)(ns - 1) * fstride;
    const double* const ti0[2] = {a.ti + (size_t)tr0 * ti_stride + colL, a.ti + (size_t)tr0 * ti_stride + colR};
    const Ppm* const pp0[2] = {a.ppm + (size_t)tr0 * pp_stride + colL, a.ppm + (size_t)tr0 * pp_stride + colR};
    typename P::Flux* const Fo0 = (dir == 0 ? a.Fu : a.Fv) + fo + (size_t)a.fslot0 * f_stride;
    auto trc = [nt](int n) { return (size_t)(n < nt ? n : 0); };
    auto pp_at = [&](int layer, int side, int n) {
        return rpp + ((size_t)((((layer & 1) * 2 + side) * NT + n) * kU)) * kFluxThreads + tid;
    };
    auto ti_at = [&](int layer, int side, int n) {
        return rti + ((size_t)(((layer & 1) * 2 + side) * NT + n)) * kFluxThreads + tid;
    };
    // record of layer k (1-based; clamped to the column) of one side
    auto fetch = [&](int side, int k) {
        const int kc = min(k, nz);
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            const char* src = reinterpret_cast<const char*>(pp0[side] + trc(n) * pp_stride + (size_t)(kc - 1) * ncol);
#pragma unroll
            for (int u = 0; u < kU; ++u) cp_async16(pp_at(k, side, n) + (size_t)u * kFluxThreads, src + 16 * u);
            cp_async8(ti_at(k, side, n), ti0[side] + trc(n) * ti_stride + (size_t)kc * ncol);
        }
    };
    auto gti = [&](int side, int n, int k) { return __ldg(ti0[side] + trc(n) * ti_stride + (size_t)k * ncol); };

    bool have_t = false;  // warp-uniform
    int kl_t = min(max((int)__ldg(KoL), 1), nz), kr_t = min(max((int)__ldg(KoR), 1), nz);
    double pl_t = __ldg(PoL), pr_t = __ldg(PoR);
    He he_c = __ldg(hEff);
    int klr_c = __ldg(KoL + fstride), krr_c = __ldg(KoR + fstride);
    double pl_c = __ldg(PoL + fstride), pr_c = __ldg(PoR + fstride);
    int cur[2] = {0, 0};    // layer whose record the ring holds as current (0: none)
    // what the newest copy group (the last live sublayer's) holds per side:
    // 1 the record below the current layer (an advance), 2 both (a re-prime)
    int newest[2] = {0, 0};
    double ttop[2][NT];     // Ti at the current layer's top interface
    double tl[NT], tr[NT];  // the top surface's tracer values
#pragma unroll
    for (int n = 0; n < NT; ++n) ttop[0][n] = ttop[1][n] = 0.0;
    for (int s = 0; s < ns - 1; ++s) {
        const size_t s0 = (size_t)s * fstride;
        He he_n = He(0);
        int klr_n = 1, krr_n = 1;
        double pl_n = 0.0, pr_n = 0.0;
        if (s + 1 < ns - 1) {
            const size_t s2 = s0 + 2 * fstride;
            he_n = __ldg(hEff + s0 + fstride);
            klr_n = __ldg(KoL + s2);
            krr_n = __ldg(KoR + s2);
            pl_n = __ldg(PoL + s2);
            pr_n = __ldg(PoR + s2);
        }
        const int kb[2] = {min(max(klr_c, 1), nz), min(max(krr_c, 1), nz)};
        const int kt[2] = {kl_t, kr_t};
        const double pt[2] = {pl_t, pr_t}, pb[2] = {pl_c, pr_c};
        const bool live = valid && he_c != He(0);
        if (!__any_sync(0xffffffffu, live)) {
#pragma unroll
            for (int n = 0; n < NT; ++n)
                if (valid && n < nt) Fo0[(size_t)n * f_stride + s0] = typename P::Flux(0);
            have_t = false;
        } else {
            bool fast[2], adv[2];
#pragma unroll
            for (int d = 0; d < 2; ++d) {
                fast[d] = cur[d] == kt[d] && (kb[d] == kt[d] || kb[d] == kt[d] + 1);
                adv[d] = fast[d] && kb[d] != kt[d];
            }
            const double xR[2] = {pb[0] + (double)(kb[0] - kt[0]), pb[1] + (double)(kb[1] - kt[1])};
            if (__all_sync(0xffffffffu, fast[0] && fast[1])) {
                // Every lane reads its ring. Every group but the newest is
                // complete after wait_group 1; the newest is waited for when
                // this sublayer reads from it: the current record after a
                // re-prime, the one below after an advance.
                bool need0 = false;
#pragma unroll
                for (int d = 0; d < 2; ++d) need0 = need0 || newest[d] == 2 || (adv[d] && newest[d] == 1);
                if (need0) cp_async_wait<0>();
                else cp_async_wait<1>();
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    double b0[2], b1[2];
                    Raw q[2];
#pragma unroll
                    for (int d = 0; d < 2; ++d) {
                        const double tk = *ti_at(kt[d], d, n);                       // Ti[kt]
                        b1[d] = *ti_at(adv[d] ? kt[d] + 1 : kt[d], d, n);            // Ti[kb]
                        b0[d] = adv[d] ? tk : ttop[d][n];                            // Ti[kb - 1]
                        q[d] = ld_stage_ppm<P>(pp_at(kt[d], d, n));
                        if (!have_t) {
                            const double top = interp(pt[d], ttop[d][n], tk);
                            if (d == 0) tl[n] = top;
                            else tr[n] = top;
                        }
                        ttop[d][n] = b0[d];
                    }
                    const double bl = interp(pb[0], b0[0], b1[0]);
                    const double br = interp(pb[1], b0[1], b1[1]);
                    if (valid && n < nt) {
                        const typename Ops::Mean tlay = Ops::mean(pt[0], xR[0], q[0]);
                        const typename Ops::Mean trlay = Ops::mean(pt[1], xR[1], q[1]);
                        const double dT = guarded_dT(tr[n] - tl[n], br - bl, (double)(trlay - tlay));
                        Fo0[(size_t)n * f_stride + s0] = he_c == He(0) ? typename P::Flux(0) : Ops::flux(dT, he_c, coef);
                    }
                    tl[n] = bl;
                    tr[n] = br;
                    // shared-memory reads wait tens of cycles: one tracer's at a
                    // time keeps the registers of the others free
                    if (n + 1 < NT) asm volatile("" ::: "memory");
                }
                // an advancing side fetches the layer below its new one into the
                // slot it leaves (read above, so its copy is complete)
#pragma unroll
                for (int d = 0; d < 2; ++d) {
                    newest[d] = adv[d] ? 1 : 0;
                    if (adv[d]) {
                        fetch(d, kb[d] + 1);
                        cur[d] = kb[d];
                    }
                }
            } else {
                // Some lane is off its ring: every lane loads as flux_item does,
                // then re-primes both sides at their bottom layers once none of
                // its copies is in flight (no slot may have two).
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    double b0[2], b1[2];
                    Raw q[2];
#pragma unroll
                    for (int d = 0; d < 2; ++d) {
                        b0[d] = gti(d, n, kb[d] - 1);
                        b1[d] = gti(d, n, kb[d]);
                        q[d] = Ops::template load<LdNC>(pp0[d] + trc(n) * pp_stride + (size_t)(kt[d] - 1) * ncol);
                    }
                    if (!have_t) {
                        tl[n] = interp(pt[0], gti(0, n, kt[0] - 1), gti(0, n, kt[0]));
                        tr[n] = interp(pt[1], gti(1, n, kt[1] - 1), gti(1, n, kt[1]));
                    }
                    const double bl = interp(pb[0], b0[0], b1[0]);
                    const double br = interp(pb[1], b0[1], b1[1]);
                    if (valid && n < nt) {
                        const typename Ops::Mean tlay = Ops::mean(pt[0], xR[0], q[0]);
                        const typename Ops::Mean trlay = Ops::mean(pt[1], xR[1], q[1]);
                        const double dT = guarded_dT(tr[n] - tl[n], br - bl, (double)(trlay - tlay));
                        Fo0[(size_t)n * f_stride + s0] = he_c == He(0) ? typename P::Flux(0) : Ops::flux(dT, he_c, coef);
                    }
                    tl[n] = bl;
                    tr[n] = br;
#pragma unroll
                    for (int d = 0; d < 2; ++d) ttop[d][n] = b0[d];
                    // one tracer's loads at a time: this path is rare, and its
                    // register peak would otherwise set the kernel's
                    if (n + 1 < NT) asm volatile("" ::: "memory");
                }
                cp_async_wait<0>();
#pragma unroll
                for (int d = 0; d < 2; ++d) {
                    fetch(d, kb[d]);
                    fetch(d, kb[d] + 1);
                    cur[d] = kb[d];
                    newest[d] = 2;
                }
            }
            cp_async_commit();
            have_t = true;
        }
        kl_t = kb[0];
        kr_t = kb[1];
        pl_t = pl_c;
        pr_t = pr_c;
        he_c = he_n;
        klr_c = klr_n;
        krr_c = krr_n;
        pl_c = pl_n;
        pr_c = pr_n;
    }
    cp_async_wait<0>();  // nothing may land in the ring after this face is done
}

// ---------------------------------------------------------------------------
// Phase B, step 3: per-cell flux divergence (redi_apply_flux_impl,
// ocean_redi.F90:1094-1181).
//
// One thread per T-cell column; a block is a BX x BY tile of columns. The
// reference adds, for each native layer of a cell, the flux of the W face
// (sublayers ks ascending, -flx into layer nz+1-KoR), then E (+flx at
// nz+1-KoL), S (-flx at KoR) and N (+flx at KoL) to dTr(k) starting from
// zero, then hTr(k) += dTr(k)*(1/areaT). Along one face the cell-side Ko is
// non-decreasing in ks (the sweep's monotonic-position backstop,
// ocean_redi.F90:385-388, 424-427), so one face's contributions to a block of
// CH layers form a contiguous run of sublayers. The kernel walks the column in
// chunks of CH layers and, per chunk, folds the W, E, S and N runs that land in
// it, in that order: every layer receives exactly the reference's additions in
// the reference's sequence (stored zero fluxes of skipped sublayers add +0.0,
// which leaves any dTr value unchanged: dTr starts at +0.0 and an IEEE sum or
// difference never turns it into -0.0). Consecutive additions to one layer run
// in a register. A flux whose cell-side layer lies behind the chunk (not
// possible for sweep-produced coefficients) is counted in the device error
// word and skipped.
// ---------------------------------------------------------------------------
// U sublayers are fetched per batch; the best depth depends on the kernel's
// register budget (the standalone gather uses 3 with 4-layer chunks and 4 with
// deeper ones, the persistent kernel 4).
template <int NT, int CH, class P, class LD, int U = 4>
__device__ __forceinline__ void gather_run(const typename P::Flux* const (&F)[NT],
                                           const typename P::Ko* __restrict__ KoS, size_t stride, bool left, int ns,
                                           int& ptr, int k0, int k1, double (&dTr)[NT][CH], int& bad) {
    // Sublayers are fetched U at a time (independent loads in flight), then
    // consumed in order until the first one beyond the chunk. The per-layer
    // sums stay in registers (see below).
    int s = ptr;
    while (s < ns - 1) {
        int kk[U];
        double ff[U][NT];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int su = s + u;
            if (su < ns - 1) {
                const size_t so = (size_t)su * stride;
                kk[u] = (int)LD::ld(KoS + so);
#pragma unroll
                for (int n = 0; n < NT; ++n) ff[u][n] = (double)LD::ld(F[n] + so);
            } else {
                kk[u] = 0x7fffffff;
#pragma unroll
                for (int n = 0; n < NT; ++n) ff[u][n] = 0.0;
            }
        }
        bool stop = false;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = kk[u];
            stop = stop || k >= k1;  // also the end of the face (s >= ns-1)
            if (!stop) {
                ++s;
                if (k < k0) ++bad;
                // Every slot takes a term: the flux where the index matches,
                // +0.0 elsewhere, which leaves the slot unchanged (it is never
                // -0.0) -- the same additions in the same order as an indexed
                // update, without a dynamically indexed array.
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    const bool hit = k - k0 == c;
#pragma unroll
                    for (int n = 0; n < NT; ++n) {
                        const double f = hit ? ff[u][n] : 0.0;
                        dTr[n][c] = left ? dTr[n][c] + f : dTr[n][c] - f;
                    }
                }
            }
        }
        if (stop) break;
    }
    ptr = s;
}

template <int NT, int CH, class P, class LD, int U = 4>
// Tracers tr0 .. tr0+NT-1 of the state; their fluxes sit at slots
// fslot .. fslot+NT-1 of the flux buffer.
__device__ __forceinline__ void gather_item(const CellGatherArgsT<P>& a, int i, int j, int tr0, int fslot) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    if (i >= nx || j >= ny) return;
    const size_t ncol = (size_t)nx * ny;
    const int col = i + nx * j;
    const int nt = min(NT, a.ntr - tr0);
    const int I = i + 1, J = j + 1;  // Fortran indices
    const int wuf_w = a.nghost + 1, wuf_e = a.nghost + a.nxp + 1;
    const int wvf_s = a.nghost + 1, wvf_n = a.nghost + a.nyp + 1;
    const size_t ustride = (size_t)(nx + 1) * ny, vstride = (size_t)nx * (ny + 1);
    // Faces in the reference order: W (u-face I, this cell RIGHT), E (u-face
    // I+1, LEFT), S (v-face J, RIGHT), N (v-face J+1, LEFT).
    bool on[4] = {I >= 2 && !((a.wall_w && I == wuf_w) || (a.wall_e && I == wuf_e)),
                  I <= nx - 1 && !((a.wall_w && I + 1 == wuf_w) || (a.wall_e && I + 1 == wuf_e)),
                  J >= 2 && !((a.wall_s && J == wvf_s) || (a.wall_n && J == wvf_n)),
                  J <= ny - 1 && !((a.wall_s && J + 1 == wvf_s) || (a.wall_n && J + 1 == wvf_n))};
    const int fo[4] = {i + (nx + 1) * j, i + 1 + (nx + 1) * j, i + nx * j, i + nx * (j + 1)};
    // dry faces (inert coefficients, recorded by the sweep) carry only +0.0
    // fluxes, which the face flux does not store: adding them would leave
    // every sum unchanged, so the walk skips them
    if (a.u.dry) {
        on[0] = on[0] && !LD::ld(a.u.dry + fo[0]);
        on[1] = on[1] && !LD::ld(a.u.dry + fo[1]);
    }
    if (a.v.dry) {
        on[2] = on[2] && !LD::ld(a.v.dry + fo[2]);
        on[3] = on[3] && !LD::ld(a.v.dry + fo[3]);
    }
    const double iaij = 1.0 / LD::ld(a.areaT + col);
    int ptr[4] = {0, 0, 0, 0};
    int bad = 0;
    double dTr[NT][CH];
    for (int k0 = 1; k0 <= nz; k0 += CH) {
        const int k1 = min(k0 + CH, nz + 1);
#pragma unroll
        for (int n = 0; n < NT; ++n)
#pragma unroll
            for (int c = 0; c < CH; ++c) dTr[n][c] = 0.0;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (!on[f]) continue;
            const bool u = f < 2, left = (f & 1) != 0;
            const size_t stride = u ? ustride : vstride;
            const typename P::Flux* F[NT];
#pragma unroll
            for (int n = 0; n < NT; ++n)
                F[n] = (u ? a.Fu : a.Fv) + (size_t)(fslot + (n < nt ? n : 0)) * (size_t)(ns - 1) * stride + fo[f];
            const FaceInT<P>& c = u ? a.u : a.v;
            gather_run<NT, CH, P, LD, U>(F, (left ? c.KoL : c.KoR) + fo[f], stride, left, ns, ptr[f], k0, k1, dTr,
                                         bad);
        }
        // Layers k0..k1-1 are complete: hTr(knat) += dTr(knat) * (1/areaT), knat = nz + 1 - k.
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            if (n >= nt) break;
            double* __restrict__ out = a.htr[tr0 + n] + col;
            const double* __restrict__ in = a.htr_in[tr0 + n] + col;  // == out for an in-place update
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const int k = k0 + c;
                if (k < k1) {
                    const size_t o = (size_t)(nz - k) * ncol;
                    out[o] = in[o] + dTr[n][c] * iaij;
                }
            }
        }
    }
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (on[f] && ptr[f] < ns - 1) ++bad;  // fluxes whose cell-side layer is beyond nz
    if (bad && a.err) atomicAdd(a.err, bad);
}

// The same fold with the chunk's per-layer sums of this thread in shared
// memory (acc: [CH][NT] doubles at a stride of kGatherThreads, this thread's
// column): each term is one load-add-store at its own layer, so neither the
// instruction count nor the registers grow with CH x NT. The additions and
// their order are exactly those of gather_run.
constexpr int kGatherThreads = 128;

// The walk with its batches software-pipelined: the batch after the current
// one is requested before the current one is folded, so one face's round
// trips overlap instead of following one another. A batch past the face's
// stop is fetched in vain (those sublayers belong to the next chunk; their
// lines are read again there). The additions and their order are exactly those
// of gather_run_s.
template <int NT, class P, class LD, int U>
__device__ __forceinline__ void gather_batch_ld(const typename P::Flux* const (&F)[NT],
                                                const typename P::Ko* __restrict__ KoS, size_t stride, int ns, int s0,
                                                int (&kk)[U], typename P::Flux (&ff)[U][NT]) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int su = s0 + u;
        if (su < ns - 1) {
            const size_t so = (size_t)su * stride;
            kk[u] = (int)LD::ld(KoS + so);
#pragma unroll
            for (int n = 0; n < NT; ++n) ff[u][n] = LD::ld(F[n] + so);
        } else {
            kk[u] = 0x7fffffff;
#pragma unroll
            for (int n = 0; n < NT; ++n) ff[u][n] = typename P::Flux(0);
        }
    }
}

template <int NT, int CH, class P, class LD, int U>
__device__ __forceinline__ void gather_run_sp(const typename P::Flux* const (&F)[NT],
                                              const typename P::Ko* __restrict__ KoS, size_t stride, bool left, int ns,
                                              int& ptr, int k0, int k1, double* __restrict__ acc, int& bad) {
    int s = ptr;
    if (s >= ns - 1) return;
    int kk[U];
    typename P::Flux ff[U][NT];
    gather_batch_ld<NT, P, LD, U>(F, KoS, stride, ns, s, kk, ff);
    while (true) {
        int kn[U];
        typename P::Flux fn[U][NT];
        gather_batch_ld<NT, P, LD, U>(F, KoS, stride, ns, s + U, kn, fn);
        bool stop = false;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = kk[u];
            stop = stop || k >= k1;  // also the end of the face (s >= ns-1)
            if (!stop) {
                ++s;
                if (k < k0) {
                    ++bad;
                } else {
                    double* d = acc + (size_t)(k - k0) * NT * kGatherThreads;
#pragma unroll
                    for (int n = 0; n < NT; ++n) {
                        const double v = d[n * kGatherThreads];
                        const double f = (double)ff[u][n];
                        d[n * kGatherThreads] = left ? v + f : v - f;
                    }
                }
            }
        }
        if (stop) break;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            kk[u] = kn[u];
#pragma unroll
            for (int n = 0; n < NT; ++n) ff[u][n] = fn[u][n];
        }
    }
    ptr = s;
}

template <int NT, int CH, class P, class LD, int U = 4>
__device__ __forceinline__ void gather_run_s(const typename P::Flux* const (&F)[NT],
                                             const typename P::Ko* __restrict__ KoS, size_t stride, bool left, int ns,
                                             int& ptr, int k0, int k1, double* __restrict__ acc, int& bad) {
    int s = ptr;
    while (s < ns - 1) {
        int kk[U];
        typename P::Flux ff[U][NT];  // widened to FP64 where added (exact)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int su = s + u;
            if (su < ns - 1) {
                const size_t so = (size_t)su * stride;
                kk[u] = (int)LD::ld(KoS + so);
#pragma unroll
                for (int n = 0; n < NT; ++n) ff[u][n] = LD::ld(F[n] + so);
            } else {
                kk[u] = 0x7fffffff;
#pragma unroll
                for (int n = 0; n < NT; ++n) ff[u][n] = typename P::Flux(0);
            }
        }
        bool stop = false;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = kk[u];
            stop = stop || k >= k1;  // also the end of the face (s >= ns-1)
            if (!stop) {
                ++s;
                if (k < k0) {
                    ++bad;
                } else {
                    double* d = acc + (size_t)(k - k0) * NT * kGatherThreads;
#pragma unroll
                    for (int n = 0; n < NT; ++n) {
                        const double v = d[n * kGatherThreads];
                        const double f = (double)ff[u][n];
                        d[n * kGatherThreads] = left ? v + f : v - f;
                    }
                }
            }
        }
        if (stop) break;
    }
    ptr = s;
}

template <int NT, int CH, class P, class LD, int U = 4, bool PIPE = false>
__device__ __forceinline__ void gather_item_s(const CellGatherArgsT<P>& a, int i, int j, int tr0, int fslot,
                                              double* __restrict__ acc) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, ns = 2 * nz + 2;
    if (i >= nx || j >= ny) return;
    const size_t ncol = (size_t)nx * ny;
    const int col = i + nx * j;
    const int nt = min(NT, a.ntr - tr0);
    const int I = i + 1, J = j + 1;  // Fortran indices
    const int wuf_w = a.nghost + 1, wuf_e = a.nghost + a.nxp + 1;
    const int wvf_s = a.nghost + 1, wvf_n = a.nghost + a.nyp + 1;
    const size_t ustride = (size_t)(nx + 1) * ny, vstride = (size_t)nx * (ny + 1);
    bool on[4] = {I >= 2 && !((a.wall_w && I == wuf_w) || (a.wall_e && I == wuf_e)),
                  I <= nx - 1 && !((a.wall_w && I + 1 == wuf_w) || (a.wall_e && I + 1 == wuf_e)),
                  J >= 2 && !((a.wall_s && J == wvf_s) || (a.wall_n && J == wvf_n)),
                  J <= ny - 1 && !((a.wall_s && J + 1 == wvf_s) || (a.wall_n && J + 1 == wvf_n))};
    const int fo[4] = {i + (nx + 1) * j, i + 1 + (nx + 1) * j, i + nx * j, i + nx * (j + 1)};
    // dry faces (inert coefficients, recorded by the sweep) carry only +0.0
    // fluxes, which the face flux does not store: adding them would leave
    // every sum unchanged, so the walk skips them
    if (a.u.dry) {
        on[0] = on[0] && !LD::ld(a.u.dry + fo[0]);
        on[1] = on[1] && !LD::ld(a.u.dry + fo[1]);
    }
    if (a.v.dry) {
        on[2] = on[2] && !LD::ld(a.v.dry + fo[2]);
        on[3] = on[3] && !LD::ld(a.v.dry + fo[3]);
    }
    const double iaij = 1.0 / LD::ld(a.areaT + col);
    int ptr[4] = {0, 0, 0, 0};
    int bad = 0;
    for (int k0 = 1; k0 <= nz; k0 += CH) {
        const int k1 = min(k0 + CH, nz + 1);
#pragma unroll
        for (int x = 0; x < CH * NT; ++x) acc[x * kGatherThreads] = 0.0;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (!on[f]) continue;
            const bool u = f < 2, left = (f & 1) != 0;
            const size_t stride = u ? ustride : vstride;
            const typename P::Flux* F[NT];
#pragma unroll
            for (int n = 0; n < NT; ++n)
                F[n] = (u ? a.Fu : a.Fv) + (size_t)(fslot + (n < nt ? n : 0)) * (size_t)(ns - 1) * stride + fo[f];
            const FaceInT<P>& c = u ? a.u : a.v;
            if constexpr (PIPE)
                gather_run_sp<NT, CH, P, LD, U>(F, (left ? c.KoL : c.KoR) + fo[f], stride, left, ns, ptr[f], k0, k1,
                                                acc, bad);
            else
                gather_run_s<NT, CH, P, LD, U>(F, (left ? c.KoL : c.KoR) + fo[f], stride, left, ns, ptr[f], k0, k1,
                                               acc, bad);
        }
        // Layers k0..k1-1 are complete: hTr(knat) += dTr(knat) * (1/areaT), knat = nz + 1 - k.
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            if (n >= nt) break;
            double* __restrict__ out = a.htr[tr0 + n] + col;
            const double* __restrict__ in = a.htr_in[tr0 + n] + col;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const int k = k0 + c;
                if (k < k1) {
                    const size_t o = (size_t)(nz - k) * ncol;
                    out[o] = in[o] + acc[(c * NT + n) * kGatherThreads] * iaij;
                }
            }
        }
    }
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (on[f] && ptr[f] < ns - 1) ++bad;
    if (bad && a.err) atomicAdd(a.err, bad);
}

}  // namespace plain
}  // namespace redi
