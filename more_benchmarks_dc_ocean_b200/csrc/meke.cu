// The MEKE step on sm_100a: meke_step_ext (meke/meke.F90:60-131) in two
// kernels, three with the biharmonic term.
//
//   pass A  k_meke_column   one thread per column: the column mass over nz
//                           layers (the only 3-D stream of the step), the
//                           structure factors and mixing length, the source
//                           bump and the first implicit-drag half; it also
//                           zeroes the staged rd / SN slots. Writes every
//                           per-cell workspace and the post-drag energy E1
//                           to scratch, so pass B reads a stable stencil.
//   (k4 >= 0) k_meke_del2   the bare-gradient Laplacian of E1 (the first half
//                           of meke_lateral's biharmonic block).
//   pass B  k_meke_lateral  one thread per cell: the four face fluxes of E1
//                           recomputed in registers (each interior face by
//                           both of its cells, the same arithmetic, the same
//                           bits), the flux divergence, the biharmonic
//                           tendency, the second drag half and the kh / ku
//                           closures. The west and south faces (and the edge
//                           faces) are stored to uflux / vflux.
//
// Pass B is launched with programmatic stream serialisation: its blocks are
// scheduled while pass A's last wave runs and wait in
// cudaGridDependencySynchronize() until pass A's writes are visible.
//
// Every expression keeps the Fortran operand order and the file is compiled
// with -fmad=false, so results are the reference's IEEE sequence bit for bit.
// Terms the step provably cannot reach are skipped without changing a bit:
// rd and SN are zeroed by the step itself (meke/meke.F90:81-83), so the
// deformation and Eady scales never contribute to 1/Lmix and pow() is only
// ever evaluated at 1; beta only matters when alpha_rhines > 0; the
// khmeke_fac * kh_diff face term is exactly zero when khmeke_fac == 0 and
// kh_diff is finite (it is a closure output: sqrt(max(0, .)) * Lmix).

#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>

#include "meke_b200.h"
#include "redi_kernels.h"

namespace {

constexpr double kMassNeglect = 1.0e-30;  // meke/meke.F90:51 MASS_NEGLECT
constexpr double kHVanished = 1.5e-4;     // meke/constants.F90:15 H_VANISHED
constexpr int kThreadsA = 256;  // pass A block: one column per thread
constexpr int kThreads = 128;   // pass B and Laplacian block: one cell per thread
constexpr int kMinBlocksB = 8;  // pass B register cap: the whole benchmark grid in one wave
constexpr int kColumnBatch = 8; // layers whose loads are in flight together

thread_local std::string g_err;

// Host-derived scalars, gates and scratch of one step.
struct Plan {
    int nt, nu, nv;
    double sdt, sdt_damp;
    int kh_flux;     // Laplacian flux: kh >= 0 (meke/meke.F90:79)
    int biharmonic;  // k4 >= 0
    int drag2;       // second drag half: kh >= 0 or k4 >= 0 (:119)
    int rhines;      // alpha_rhines > 0: beta = |grad f| is needed
    int kh_face;     // khmeke_fac != 0: fluxes read the pre-step kh_diff
    int pdl;         // pass B waits on pass A through the programmatic edge
    double* e1;      // post-drag energy (nt)
    double* kh0;     // pre-step kh_diff (nt), when kh_face
    double* lap;     // biharmonic Laplacian of E1 (nt), when biharmonic
    double* del2;    // ocean_meke_t%del2: the biharmonic tendency (nt)
};

__device__ __forceinline__ double drag_half(double e, double imass, double bf2, double ubbl2, double cdrag,
                                            double uscale, double damping, double sdt_damp) {
    // meke_drag (meke/meke.F90:532-556)
    const double cd2 = cdrag * cdrag;
    const double drag_rate = imass * sqrt(cd2 * ((fmax(0.0, 2.0 * bf2 * e) + ubbl2) + uscale * uscale));
    double damp_rate = damping + drag_rate * bf2;
    if (e < 0.0) damp_rate = 0.0;
    return e / (1.0 + sdt_damp * damp_rate);
}

__device__ __forceinline__ double inv_lmix(double ueddy, double sn, double beta, double area, double rd_over_dx,
                                           double depth, double cdrag, double a_deform, double a_rhines,
                                           double a_eady, double a_frict, double a_grid) {
    // meke_inv_lmix (meke/meke.F90:390-418)
    const double lgrid = sqrt(fmax(area, 0.0));
    const double ldeform = lgrid * rd_over_dx;
    double lfrict = 0.0;
    if (cdrag > 0.0) lfrict = depth / cdrag;
    double lrhines = 0.0;
    if (beta > 0.0) lrhines = sqrt(fmax(ueddy, 0.0) / beta);
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

__device__ __forceinline__ double harmonic_mass(double m1, double m2) {
    return 2.0 * m1 * m2 / ((m1 + m2) + kMassNeglect);  // meke/meke.F90:700-701
}

// ---------------------------------------------------------------- pass A ----
__global__ void __launch_bounds__(kThreadsA) k_meke_column(const MekeArgs a, const Plan p) {
    const int t = blockIdx.x * kThreadsA + threadIdx.x;
    // pass B's blocks may be scheduled as soon as every block of this grid runs
    cudaTriggerProgrammaticLaunchCompletion();
    // meke_zero_2d of the staged SN faces (meke/meke.F90:82-83)
    if (t < p.nu) a.sn_u_ws[t] = 0.0;
    if (t < p.nv) a.sn_v_ws[t] = 0.0;
    if (t >= p.nt) return;

    // per-cell inputs first, so their latency hides under the column stream
    const double kd = __ldg(a.ke_diss_ext + t);
    const double area = __ldg(a.areaT + t);
    const double ubbl2 = __ldg(a.u_bbl2 + t);
    const double gm = a.gmcoeff >= 0.0 ? __ldg(a.gm_src + t) : 0.0;
    const double e0 = a.meke[t];
    const double kh_prev = p.kh_face ? a.kh_diff[t] : 0.0;

    // meke_mass (meke/meke.F90:355-388), have_rho: one in-order sum per column.
    const size_t plane = (size_t)p.nt;
    const double* __restrict__ hcol = a.h_layer + t;
    const double* __restrict__ rcol = a.rho_layer + t;
    const int nz = a.nz;
    double mass = 0.0, dsum = 0.0;
    int k = 0;
    for (; k + kColumnBatch <= nz; k += kColumnBatch) {
        double hv[kColumnBatch], rv[kColumnBatch];
#pragma unroll
        for (int u = 0; u < kColumnBatch; ++u) {
            hv[u] = __ldg(hcol + (size_t)(k + u) * plane);
            rv[u] = __ldg(rcol + (size_t)(k + u) * plane);
        }
#pragma unroll
        for (int u = 0; u < kColumnBatch; ++u) {
            mass = mass + rv[u] * fmax(hv[u], kHVanished);
            dsum = dsum + hv[u];
        }
    }
    for (; k < nz; ++k) {
        const double hk = __ldg(hcol + (size_t)k * plane);
        const double rk = __ldg(rcol + (size_t)k * plane);
        mass = mass + rk * fmax(hk, kHVanished);
        dsum = dsum + hk;
    }
    const double imass = mass > 0.0 ? 1.0 / mass : 0.0;
    a.depth_tot[t] = dsum;
    a.mass_ws[t] = mass;
    a.i_mass[t] = imass;

    // meke_zero_2d of rd (:81) and meke_stage_rd of ke_diss (:100)
    const double rd = 0.0;
    a.rd_ws[t] = rd;
    a.ke_diss_ws[t] = kd;

    // meke_length_scales (meke/meke.F90:420-505)
    const double lgrid = sqrt(fmax(area, 0.0));
    const double ldeform = lgrid * rd;
    double lfrict = 0.0;
    if (a.cdrag > 0.0) lfrict = dsum / a.cdrag;
    double bf2 = a.cd_scale * a.cd_scale;
    if (lfrict * a.cb > 0.0) {
        const double ratio = ldeform / lfrict;
        const double base = 1.0 + a.cb * ratio;  // exactly 1 here: rd is zero in this step
        bf2 = bf2 + 1.0 / (base == 1.0 ? 1.0 : pow(base, 0.8));  // pow(+1, y) == 1 for every y
    }
    bf2 = fmax(bf2, a.min_gamma2);
    double tf2 = 1.0;
    if (lfrict * a.ct > 0.0) {
        const double ratio = ldeform / lfrict;
        const double base = 1.0 + a.ct * ratio;
        tf2 = 1.0 / (base == 1.0 ? 1.0 : pow(base, 0.25));
    }
    tf2 = fmax(tf2, a.min_gamma2);
    const double ueddy = sqrt(2.0 * fmax(0.0, tf2 * e0));
    double beta = 0.0;
    if (p.rhines) {
        const int nx = a.nx, ny = a.ny;
        const int i = t % nx, j = t / nx;
        if (i > 0 && i < nx - 1) {
            const double d = 0.5 * (__ldg(a.f_centre + t + 1) - __ldg(a.f_centre + t - 1)) * __ldg(a.idxT + t);
            beta = beta + d * d;
        }
        if (j > 0 && j < ny - 1) {
            const double d = 0.5 * (__ldg(a.f_centre + t + nx) - __ldg(a.f_centre + t - nx)) * __ldg(a.idyT + t);
            beta = beta + d * d;
        }
        beta = sqrt(beta);
    }
    const double sn = 0.0;  // the SN faces were zeroed above
    const double il = inv_lmix(ueddy, sn, beta, area, rd, dsum, a.cdrag, a.a_deform, a.a_rhines, a.a_eady,
                               a.a_frict, a.a_grid);
    a.bottom_fac2[t] = bf2;
    a.barotr_fac2[t] = tf2;
    a.le[t] = il > 0.0 ? 1.0 / il : 0.0;

    // meke_source (meke/meke.F90:507-530) and the first drag half (:532-556)
    double s = a.bgsrc;
    if (a.gmcoeff >= 0.0) s = s + a.gmcoeff * imass * gm;
    if (a.frcoeff >= 0.0) s = s - a.frcoeff * imass * kd;
    a.src[t] = s;
    const double e = e0 + p.sdt * s;
    p.e1[t] = drag_half(e, imass, bf2, ubbl2, a.cdrag, a.uscale, a.damping, p.sdt_damp);
    if (p.kh_face) p.kh0[t] = kh_prev;
}

// ------------------------------------------------- biharmonic Laplacian -----
__global__ void __launch_bounds__(kThreads) k_meke_del2(const MekeArgs a, const Plan p) {
    // meke/meke.F90:676-693: bare-gradient fluxes of E1 and their divergence
    const int t = blockIdx.x * kThreads + threadIdx.x;
    if (t >= p.nt) return;
    const int nx = a.nx, ny = a.ny;
    const int i = t % nx, j = t / nx;
    const double* __restrict__ e1 = p.e1;
    const int fu = t + j;  // u face west of cell t
    const double e = e1[t];
    double gw = 0.0, ge = 0.0, gs = 0.0, gn = 0.0;
    if (i > 0) gw = (__ldg(a.dy_cu + fu) * __ldg(a.idxCu + fu)) * (e - e1[t - 1]);
    if (i < nx - 1) ge = (__ldg(a.dy_cu + fu + 1) * __ldg(a.idxCu + fu + 1)) * (e1[t + 1] - e);
    if (j > 0) gs = (__ldg(a.dx_cv + t) * __ldg(a.idyCv + t)) * (e - e1[t - nx]);
    if (j < ny - 1) gn = (__ldg(a.dx_cv + t + nx) * __ldg(a.idyCv + t + nx)) * (e1[t + nx] - e);
    p.lap[t] = __ldg(a.iareaT + t) * ((ge - gw) + (gn - gs));
}

// ---------------------------------------------------------------- pass B ----
// Laplacian flux through a face from the values of its left / lower cell (l)
// and right / upper cell (r) (meke/meke.F90:736-745).
__device__ __forceinline__ double lap_face(const MekeArgs& a, const Plan& p, double geo, double ia_l, double ia_r,
                                           double m_l, double m_r, double e_l, double e_r, double k_l, double k_r) {
    double kh = fmax(0.0, a.kh_bg);
    if (p.kh_face) kh = kh + a.khmeke_fac * 0.5 * (k_l + k_r);
    const double inv_max = 2.0 * p.sdt * (geo * fmax(ia_l, ia_r));
    if (kh * inv_max > 0.25) kh = 0.25 / inv_max;
    return (kh * geo) * harmonic_mass(m_l, m_r) * (e_l - e_r);
}

// Biharmonic flux of the Laplacian through the same face (meke/meke.F90:697-724).
__device__ __forceinline__ double bih_face(const MekeArgs& a, const Plan& p, double geo, double ia_l, double ia_r,
                                           double m_l, double m_r, double l_l, double l_r) {
    const double g = geo * fmax(ia_l, ia_r);
    const double inv_max = 64.0 * p.sdt * (g * g);
    double k4 = a.k4;
    if (k4 * inv_max > 0.3) k4 = 0.3 / inv_max;
    return (k4 * geo) * harmonic_mass(m_l, m_r) * (l_r - l_l);
}

// Every load of a thread is issued up front: neighbour indices are clamped into
// the domain (an edge neighbour stands in as the cell itself, and that face's
// flux is replaced by 0, the value meke_lateral gives edge faces), and the face
// metrics of the edge faces exist (u faces have nx+1 columns, v faces ny+1
// rows). Interior faces see exactly the reference's operands.
__global__ void __launch_bounds__(kThreads, kMinBlocksB) k_meke_lateral(const MekeArgs a, const Plan p) {
    const int t = blockIdx.x * kThreads + threadIdx.x;
    if (p.pdl) cudaGridDependencySynchronize();
    if (t >= p.nt) return;
    const int nx = a.nx, ny = a.ny;
    const int i = t % nx, j = t / nx;
    const int fu = t + j;  // u face west of cell t; the v face south of it is t
    const bool west = i > 0, east = i < nx - 1, south = j > 0, north = j < ny - 1;
    const int tw = west ? t - 1 : t, te = east ? t + 1 : t, ts = south ? t - nx : t, tn = north ? t + nx : t;

    const double geo_w = __ldg(a.dy_cu + fu) * __ldg(a.idxCu + fu);
    const double geo_e = __ldg(a.dy_cu + fu + 1) * __ldg(a.idxCu + fu + 1);
    const double geo_s = __ldg(a.dx_cv + t) * __ldg(a.idyCv + t);
    const double geo_n = __ldg(a.dx_cv + t + nx) * __ldg(a.idyCv + t + nx);
    const double* __restrict__ iar = a.iareaT;
    const double* __restrict__ mws = a.mass_ws;
    const double* __restrict__ e1 = p.e1;
    const double ia_c = __ldg(iar + t), ia_w = __ldg(iar + tw), ia_e = __ldg(iar + te), ia_s = __ldg(iar + ts),
                 ia_n = __ldg(iar + tn);
    const double m_c = __ldg(mws + t), m_w = __ldg(mws + tw), m_e = __ldg(mws + te), m_s = __ldg(mws + ts),
                 m_n = __ldg(mws + tn);
    const double imass = __ldg(a.i_mass + t);
    const double bf2 = __ldg(a.bottom_fac2 + t);
    const double ubbl2 = __ldg(a.u_bbl2 + t);
    const double tf2 = __ldg(a.barotr_fac2 + t);
    const double lmix = __ldg(a.le + t);
    double e = __ldg(e1 + t);

    if (p.kh_flux) {
        // meke_lateral, Laplacian block (meke/meke.F90:732-746)
        const double e_w = __ldg(e1 + tw), e_e = __ldg(e1 + te), e_s = __ldg(e1 + ts), e_n = __ldg(e1 + tn);
        double k_c = 0.0, k_w = 0.0, k_e = 0.0, k_s = 0.0, k_n = 0.0;
        if (p.kh_face) {
            k_c = __ldg(p.kh0 + t);
            k_w = __ldg(p.kh0 + tw);
            k_e = __ldg(p.kh0 + te);
            k_s = __ldg(p.kh0 + ts);
            k_n = __ldg(p.kh0 + tn);
        }
        const double fw = west ? lap_face(a, p, geo_w, ia_w, ia_c, m_w, m_c, e_w, e, k_w, k_c) : 0.0;
        const double fe = east ? lap_face(a, p, geo_e, ia_c, ia_e, m_c, m_e, e, e_e, k_c, k_e) : 0.0;
        const double fs = south ? lap_face(a, p, geo_s, ia_s, ia_c, m_s, m_c, e_s, e, k_s, k_c) : 0.0;
        const double fn = north ? lap_face(a, p, geo_n, ia_c, ia_n, m_c, m_n, e, e_n, k_c, k_n) : 0.0;
        if (a.uflux) {
            a.uflux[fu] = fw;
            if (!east) a.uflux[fu + 1] = 0.0;
        }
        if (a.vflux) {
            a.vflux[t] = fs;
            if (!north) a.vflux[t + nx] = 0.0;
        }
        const double mke = p.sdt * (ia_c * imass) * ((fw - fe) + (fs - fn));
        e = e + mke;
    }
    if (p.biharmonic) {
        const double* __restrict__ lap = p.lap;
        const double l_c = __ldg(lap + t), l_w = __ldg(lap + tw), l_e = __ldg(lap + te), l_s = __ldg(lap + ts),
                     l_n = __ldg(lap + tn);
        const double gw = west ? bih_face(a, p, geo_w, ia_w, ia_c, m_w, m_c, l_w, l_c) : 0.0;
        const double ge = east ? bih_face(a, p, geo_e, ia_c, ia_e, m_c, m_e, l_c, l_e) : 0.0;
        const double gs = south ? bih_face(a, p, geo_s, ia_s, ia_c, m_s, m_c, l_s, l_c) : 0.0;
        const double gn = north ? bih_face(a, p, geo_n, ia_c, ia_n, m_c, m_n, l_c, l_n) : 0.0;
        if (!p.kh_flux) {  // the biharmonic fluxes are then the last ones meke_lateral stores
            if (a.uflux) {
                a.uflux[fu] = gw;
                if (!east) a.uflux[fu + 1] = 0.0;
            }
            if (a.vflux) {
                a.vflux[t] = gs;
                if (!north) a.vflux[t + nx] = 0.0;
            }
        }
        const double mke4 = p.sdt * (ia_c * imass) * ((gw - ge) + (gs - gn));
        p.del2[t] = mke4;
        e = e + mke4;
    }
    if (p.drag2) e = drag_half(e, imass, bf2, ubbl2, a.cdrag, a.uscale, a.damping, p.sdt_damp);
    a.meke[t] = e;

    // meke_kh_closure and meke_ku_closure (meke/meke.F90:575-622)
    double kh = 0.0;
    if (a.khcoeff > 0.0) {
        const double ueddy = sqrt(2.0 * fmax(0.0, tf2 * e));
        kh = a.khcoeff * ueddy * lmix;
    }
    a.kh_diff[t] = kh;
    double ku = 0.0;
    if (a.backscatter && a.visc_coeff_ku != 0.0) {
        const double ueddy = sqrt(2.0 * fmax(0.0, e));
        ku = a.visc_coeff_ku * ueddy * lmix;
    }
    a.ku[t] = ku;
}

// ---------------------------------------------------------------- host ------

int fail(int code, const std::string& msg) {
    g_err = msg;
    redi::set_last_error(msg);
    return code;
}

int cuda_fail(const char* what, cudaError_t e) {
    return fail(MEKE_B200_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_args(const MekeArgs* a) {
    if (!a) return fail(MEKE_B200_E_ARG, "meke: NULL argument block");
    if (a->nx < 1 || a->ny < 1 || a->nz < 0) return fail(MEKE_B200_E_ARG, "meke: nx, ny must be >= 1 and nz >= 0");
    if ((long long)(a->nx + 1) * (long long)(a->ny + 1) > (long long)INT_MAX - kThreads)
        return fail(MEKE_B200_E_ARG, "meke: domain too large for 32-bit cell indices");
    const void* need[] = {a->meke, a->kh_diff, a->le, a->ku, a->i_mass, a->depth_tot, a->bottom_fac2,
                          a->barotr_fac2, a->src, a->mass_ws, a->rd_ws, a->sn_u_ws, a->sn_v_ws, a->ke_diss_ws,
                          a->u_bbl2, a->ke_diss_ext, a->areaT, a->iareaT, a->dy_cu, a->dx_cv, a->idxCu, a->idyCv};
    for (const void* q : need)
        if (!q) return fail(MEKE_B200_E_ARG, "meke: a required array pointer is NULL");
    if (a->nz > 0 && (!a->h_layer || !a->rho_layer)) return fail(MEKE_B200_E_ARG, "meke: h_layer / rho_layer NULL");
    if (a->gmcoeff >= 0.0 && !a->gm_src) return fail(MEKE_B200_E_ARG, "meke: gm_src NULL with gmcoeff >= 0");
    if (a->a_rhines > 0.0 && (!a->f_centre || !a->idxT || !a->idyT))
        return fail(MEKE_B200_E_ARG, "meke: f_centre / idxT / idyT NULL with alpha_rhines > 0");
    return MEKE_B200_OK;
}

Plan make_plan(const MekeArgs& a) {
    Plan p{};
    p.nt = a.nx * a.ny;
    p.nu = (a.nx + 1) * a.ny;
    p.nv = a.nx * (a.ny + 1);
    p.sdt = a.dt * a.dtscale;
    double damp_step = 1.0;
    if (a.kh_bg >= 0.0 || a.k4 >= 0.0) damp_step = 0.5;
    p.sdt_damp = p.sdt * damp_step;
    p.kh_flux = a.kh_bg >= 0.0;
    p.biharmonic = a.k4 >= 0.0;
    p.drag2 = a.kh_bg >= 0.0 || a.k4 >= 0.0;
    p.rhines = a.a_rhines > 0.0;
    p.kh_face = p.kh_flux && a.khmeke_fac != 0.0;
    return p;
}

int blocks(int n) { return (n + kThreads - 1) / kThreads; }

// The kernels of one step on `st`. Inside stream capture pdl and instrument
// are off: the graph holds plain edges and its replays are counted instead.
int launch_step(const MekeArgs& a, Plan p, cudaStream_t st, bool pdl, bool instrument) {
    const int na = p.nu > p.nv ? p.nu : p.nv;  // >= nt
    if (instrument) redi::launch_begin(redi::K_MEKE_COLUMN, st);
    k_meke_column<<<(na + kThreadsA - 1) / kThreadsA, kThreadsA, 0, st>>>(a, p);
    if (instrument) redi::launch_end(redi::K_MEKE_COLUMN, st);
    if (p.biharmonic) {
        if (instrument) redi::launch_begin(redi::K_MEKE_DEL2, st);
        k_meke_del2<<<blocks(p.nt), kThreads, 0, st>>>(a, p);
        if (instrument) redi::launch_end(redi::K_MEKE_DEL2, st);
        pdl = false;  // pass B then follows the Laplacian kernel, which has no trigger
    }
    p.pdl = pdl ? 1 : 0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks(p.nt));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    if (instrument) redi::launch_begin(redi::K_MEKE_LATERAL, st);
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_meke_lateral, a, p);
    if (instrument) redi::launch_end(redi::K_MEKE_LATERAL, st);
    if (e != cudaSuccess) return cuda_fail("meke: launch", e);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("meke: launch", e);
    return MEKE_B200_OK;
}

}  // namespace

struct meke_b200 {
    int nx = 0, ny = 0, device = -1;
    double* buf = nullptr;  // e1 | kh0 | lap | del2, nx*ny doubles each
    size_t cells() const { return (size_t)nx * (size_t)ny; }
    double* e1() const { return buf; }
    double* kh0() const { return buf + cells(); }
    double* lap() const { return buf + 2 * cells(); }
    double* del2() const { return buf + 3 * cells(); }
};

namespace {

int run_step(meke_b200* h, const MekeArgs* a, double* del2, double* e1_override, cudaStream_t st, bool pdl,
             bool instrument = true) {
    int rc = check_args(a);
    if (rc < 0) return rc;
    if (!h) return fail(MEKE_B200_E_ARG, "meke_b200_step: NULL handle");
    if ((size_t)a->nx * (size_t)a->ny > h->cells())
        return fail(MEKE_B200_E_ARG, "meke_b200_step: domain larger than the handle was created for");
    Plan p = make_plan(*a);
    p.e1 = e1_override ? e1_override : h->e1();
    p.kh0 = h->kh0();
    p.lap = h->lap();
    p.del2 = del2 ? del2 : h->del2();
    return launch_step(*a, p, st, pdl, instrument);
}

// Scratch for the reference-signature launchers, one per device and domain size.
std::mutex g_mu;
std::map<std::tuple<int, int, int>, std::unique_ptr<meke_b200, int (*)(meke_b200*)>> g_scratch;

meke_b200* shared_scratch(const MekeArgs* a) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    auto key = std::make_tuple(dev, a->nx, a->ny);
    auto it = g_scratch.find(key);
    if (it != g_scratch.end()) return it->second.get();
    meke_b200* h = nullptr;
    if (meke_b200_create(a->nx, a->ny, 1, &h) != MEKE_B200_OK) return nullptr;
    g_scratch.emplace(key, std::unique_ptr<meke_b200, int (*)(meke_b200*)>(h, meke_b200_destroy));
    return h;
}

// The captured step of meke_cuda_launch mode 2 and the argument block it was captured with.
struct GraphCache {
    bool valid = false;
    int device = -1;
    MekeArgs args{};
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        if (stream) cudaStreamDestroy(stream);
        exec = nullptr;
        stream = nullptr;
        valid = false;
    }
} g_graph;

void report(const char* who, int rc) {
    if (rc < 0) std::fprintf(stderr, "%s: %s\n", who, g_err.c_str());
}

}  // namespace

extern "C" {

int meke_b200_create(int nx, int ny, int nz, meke_b200** out) {
    if (!out) return fail(MEKE_B200_E_ARG, "meke_b200_create: NULL output");
    *out = nullptr;
    if (nx < 1 || ny < 1 || nz < 0) return fail(MEKE_B200_E_ARG, "meke_b200_create: nx, ny must be >= 1, nz >= 0");
    if ((long long)(nx + 1) * (long long)(ny + 1) > (long long)INT_MAX - kThreads)
        return fail(MEKE_B200_E_ARG, "meke_b200_create: domain too large for 32-bit cell indices");
    auto* h = new meke_b200;
    h->nx = nx;
    h->ny = ny;
    cudaGetDevice(&h->device);
    cudaError_t e = cudaMalloc(&h->buf, 4 * h->cells() * sizeof(double));
    if (e != cudaSuccess) {
        delete h;
        cudaGetLastError();
        return fail(MEKE_B200_E_NOMEM, std::string("meke_b200_create: ") + cudaGetErrorString(e));
    }
    e = cudaMemset(h->buf, 0, 4 * h->cells() * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(h->buf);
        delete h;
        return cuda_fail("meke_b200_create", e);
    }
    *out = h;
    g_err.clear();
    return MEKE_B200_OK;
}

int meke_b200_destroy(meke_b200* self) {
    if (!self) return MEKE_B200_OK;
    if (self->buf) cudaFree(self->buf);
    delete self;
    return MEKE_B200_OK;
}

int meke_b200_step(meke_b200* self, const MekeArgs* args, double* del2, void* stream) {
    const int rc = run_step(self, args, del2, nullptr, static_cast<cudaStream_t>(stream), true);
    if (rc == MEKE_B200_OK) g_err.clear();
    return rc;
}

const double* meke_b200_scratch_energy(const meke_b200* self) { return self ? self->e1() : nullptr; }

const char* meke_b200_last_error(void) { return g_err.c_str(); }

void meke_cuda_launch(const MekeArgs* ap, int mode) {
    int rc = check_args(ap);
    meke_b200* h = rc < 0 ? nullptr : shared_scratch(ap);
    if (rc == MEKE_B200_OK && !h) rc = fail(MEKE_B200_E_NOMEM, "meke_cuda_launch: scratch allocation failed");
    if (rc == MEKE_B200_OK && mode != 2) {
        rc = run_step(h, ap, nullptr, nullptr, nullptr, true);
        const cudaError_t e = cudaDeviceSynchronize();
        if (rc == MEKE_B200_OK && e != cudaSuccess) rc = cuda_fail("meke_cuda_launch", e);
    } else if (rc == MEKE_B200_OK) {
        std::lock_guard<std::mutex> lock(g_mu);
        int dev = 0;
        cudaGetDevice(&dev);
        if (g_graph.valid && (g_graph.device != dev || std::memcmp(&g_graph.args, ap, sizeof(MekeArgs)) != 0))
            g_graph.reset();
        cudaError_t e = cudaSuccess;
        if (!g_graph.valid) {
            // a blocking stream, as the reference's: ordered with the legacy default stream
            e = cudaStreamCreate(&g_graph.stream);
            cudaGraph_t g = nullptr;
            if (e == cudaSuccess) e = cudaStreamBeginCapture(g_graph.stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                rc = run_step(h, ap, nullptr, nullptr, g_graph.stream, false, false);
                e = cudaStreamEndCapture(g_graph.stream, &g);
            }
            if (e == cudaSuccess && rc == MEKE_B200_OK) e = cudaGraphInstantiate(&g_graph.exec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e == cudaSuccess && rc == MEKE_B200_OK) {
                g_graph.valid = true;
                g_graph.device = dev;
                g_graph.args = *ap;
            } else {
                g_graph.reset();
            }
        }
        if (rc == MEKE_B200_OK && e == cudaSuccess) {
            redi::count_launches(redi::K_MEKE_COLUMN, 1);
            if (ap->k4 >= 0.0) redi::count_launches(redi::K_MEKE_DEL2, 1);
            redi::count_launches(redi::K_MEKE_LATERAL, 1);
            e = cudaGraphLaunch(g_graph.exec, g_graph.stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(g_graph.stream);
        }
        if (rc == MEKE_B200_OK && e != cudaSuccess) rc = cuda_fail("meke_cuda_launch (graph)", e);
    }
    report("meke_cuda_launch", rc);
}

void meke_cuda_graph_reset(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_graph.reset();
}

void meke_opt_launch(const MekeArgs* ap, double* meke_scratch) {
    int rc = check_args(ap);
    if (rc == MEKE_B200_OK && !meke_scratch) rc = fail(MEKE_B200_E_ARG, "meke_opt_launch: NULL meke_scratch");
    meke_b200* h = rc < 0 ? nullptr : shared_scratch(ap);
    if (rc == MEKE_B200_OK && !h) rc = fail(MEKE_B200_E_NOMEM, "meke_opt_launch: scratch allocation failed");
    if (rc == MEKE_B200_OK) {
        rc = run_step(h, ap, nullptr, meke_scratch, nullptr, true);
        const cudaError_t e = cudaDeviceSynchronize();
        if (rc == MEKE_B200_OK && e != cudaSuccess) rc = cuda_fail("meke_opt_launch", e);
    }
    report("meke_opt_launch", rc);
}

void meke_opt_launch_flat(double* meke, double* kh_diff, double* le, double* ku, double* i_mass, double* depth_tot,
                          double* bottom_fac2, double* barotr_fac2, double* src, double* uflux, double* vflux,
                          double* mass_ws, double* rd_ws, double* sn_u_ws, double* sn_v_ws, double* ke_diss_ws,
                          const double* u_bbl2, const double* f_centre, const double* gm_src,
                          const double* ke_diss_ext, const double* h_layer, const double* rho_layer,
                          const double* areaT, const double* iareaT, const double* idxT, const double* idyT,
                          const double* dy_cu, const double* dx_cv, const double* idxCu, const double* idyCv, int nx,
                          int ny, int nz, double dt, double dtscale, double cd_scale, double cb, double ct,
                          double min_gamma2, double cdrag, double uscale, double a_deform, double a_rhines,
                          double a_eady, double a_frict, double a_grid, double bgsrc, double gmcoeff, double frcoeff,
                          double damping, double kh_bg, double k4, double khmeke_fac, double khcoeff,
                          double visc_coeff_ku, double rho0, int backscatter, double* meke_scratch) {
    MekeArgs a{meke,      kh_diff,  le,        ku,        i_mass,     depth_tot, bottom_fac2, barotr_fac2,
               src,       uflux,    vflux,     mass_ws,   rd_ws,      sn_u_ws,   sn_v_ws,     ke_diss_ws,
               u_bbl2,    f_centre, gm_src,    ke_diss_ext, h_layer,  rho_layer, areaT,       iareaT,
               idxT,      idyT,     dy_cu,     dx_cv,     idxCu,      idyCv,     nx,          ny,
               nz,        dt,       dtscale,   cd_scale,  cb,         ct,        min_gamma2,  cdrag,
               uscale,    a_deform, a_rhines,  a_eady,    a_frict,    a_grid,    bgsrc,       gmcoeff,
               frcoeff,   damping,  kh_bg,     k4,        khmeke_fac, khcoeff,   visc_coeff_ku, rho0,
               backscatter};
    meke_opt_launch(&a, meke_scratch);
}

}  // extern "C"
