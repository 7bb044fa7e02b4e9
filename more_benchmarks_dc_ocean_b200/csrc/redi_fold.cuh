// Phase B of the Redi step as one fused pass per cell tile: every face's
// sublayer fluxes (redi_face_flux + redi_sublayer_dT, ocean_redi.F90:893-925,
// 1037-1092) are computed once per tile and folded into the cells' tracer
// tendencies in shared memory, in exactly the order redi_apply_flux_impl
// (:1094-1181) adds them, then hTr += dTr * (1/areaT). Nothing between the face
// walk and the fold goes through global memory.
//
// Tile: kTileW = 31 cells along i times BY rows. Its warps:
//   warps 0 .. BY-1    u walkers of rows 0 .. BY-1: lane l walks u face i0+l,
//                      the WEST face of cell l (its right column) and the EAST
//                      face of cell l-1 (its left column);
//   warps BY .. 2BY    v walkers of v-face rows g = 0 .. BY: lane l walks the
//                      v face below tile row g, the SOUTH face of cell (l, g)
//                      (its right column) and the NORTH face of cell (l, g-1)
//                      (its left column).
// Faces on the tile's edge are also walked by the neighbouring tile for its own
// cells (same operands, so the same bits); interior faces are walked once.
//
// Order. The reference forms dTr(k) of a cell from +0.0 by adding, in this
// order, the W face's terms (sublayers ks ascending), then E's, S's and N's. A
// face side's terms land at the cell-side layer Ko(ks), which never decreases
// along a face (the sweep's monotonic-position backstop, :385-388, 424-427).
// So per cell the four face sides form a chain W -> E -> S -> N, and a term of
// one side at layer m may be added once no earlier side has a term left at a
// layer <= m. Each side publishes a frontier, the layer of its next unadded
// term (every term above it is added); a side's effective frontier is the
// minimum of its own and its predecessor's. W waits for nobody; E waits for W
// (the neighbouring lane, by warp shuffle); S waits for E (the u warp of the
// same row, through shared memory); N waits for S (the v warp below, through
// shared memory). The waits form no cycle, so every walk completes; a warp
// leaves its walk only when every frontier it forwards has reached its final
// value (a v warp with no face of its own still relays PE into PS). A term
// that may not be added yet waits in its side's queue (kQ entries); a walker
// whose queue is full pauses. The accumulators hold every layer of every cell
// of the tile, so the lag between the two sides of a face (the two columns
// can be tens of layers apart at a seamount flank) never blocks a walk.
//
// Each accumulator is FP64 and receives exactly the reference's additions in
// the reference's order, so results are bit-identical to the reference
// (compiled with FMA contraction off). A Ko outside 1..nz, or decreasing along
// a face, is counted in the device error word (never the case for
// coefficients made by the sweep), as is a walk that waited longer than
// kStallNs for a frontier; after such a wait every block of the launch stops
// early (the abort word), so a fault in the ordering cannot hold the GPU.
#pragma once

#include <cuda/atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "redi_items.cuh"

namespace redi {
namespace fold {

constexpr int kTileW = 31;                  // cells of a tile row (lane 31 walks the 32nd u face)
constexpr int kQ = 8;                       // queued terms per face side
constexpr int kInf = 1 << 24;               // frontier of a side with no term left
constexpr long long kStallNs = 50000000LL;  // longest wait for a frontier (50 ms; a whole walk takes ~0.1 ms)

template <class P>
struct FoldArgsT {
    int nx, ny, nz, ntr;
    int nghost, nxp, nyp;
    int wall_w, wall_e, wall_s, wall_n;
    double dt;
    double khtr;  // used where khtr_u / khtr_v is null (scalar path)
    const double* khtr_u;
    const double* khtr_v;
    const double* dy_cu;
    const double* dx_cv;
    const double* idxCu;
    const double* idyCv;
    const double* areaT;
    FaceInT<P> u, v;
    const double* ti;                   // [tracer][nz+1][column]
    const typename P::Ppm* ppm;         // [tracer][nz][column]
    double* htr[kMaxTracers];           // updated tracers
    const double* htr_in[kMaxTracers];  // pre-step tracers (the same arrays for an in-place update)
    int* err;                           // device error word, may be null
    int* abort;                         // set once a walk gave up waiting: every block stops early; may be null
};

// Shared memory of one tile (bytes) for NT tracers per pass: the accumulators
// [NT][nz][BY][32] (FP64), 1/areaT [BY][32], the frontiers PE, PS [BY][32],
// and the queues, kSlots rings of kQ entries per lane (layer, NT fluxes).
template <class P, int NT, int BY, bool ORD = true>
struct FoldLayout {
    using Flux = typename P::Flux;
    static constexpr int kSlots = ORD ? 3 * BY : 0;  // E per u row; S and N per v row where the side is in the tile
    __host__ __device__ static size_t ia_off(int nz) { return (size_t)NT * nz * BY * 32 * sizeof(double); }
    __host__ __device__ static size_t front_off(int nz) { return ia_off(nz) + (size_t)BY * 32 * sizeof(double); }
    __host__ __device__ static size_t qlay_off(int nz) { return front_off(nz) + (size_t)2 * BY * 32 * sizeof(int); }
    __host__ __device__ static size_t qf_off(int nz) { return qlay_off(nz) + (size_t)kSlots * kQ * 32 * sizeof(int); }
    __host__ __device__ static size_t bytes(int nz) {
        return qf_off(nz) + (size_t)kSlots * kQ * NT * 32 * sizeof(Flux);
    }
};

// The deferred terms of one face side: a ring in shared memory, one column per lane.
template <int NT, class Flux>
struct SideQueue {
    int* lay;  // [kQ][32]
    Flux* f;   // [kQ][NT][32]
    int head, n;
    __device__ __forceinline__ int head_layer() const { return lay[head * 32 + (threadIdx.x & 31)]; }
    __device__ __forceinline__ void push(int m, const Flux (&v)[NT]) {
        const int lane = threadIdx.x & 31;
        int slot = head + n;
        if (slot >= kQ) slot -= kQ;
        lay[slot * 32 + lane] = m;
#pragma unroll
        for (int t = 0; t < NT; ++t) f[(slot * NT + t) * 32 + lane] = v[t];
        ++n;
    }
    __device__ __forceinline__ void head_flux(Flux (&v)[NT]) const {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int t = 0; t < NT; ++t) v[t] = f[(head * NT + t) * 32 + lane];
    }
    __device__ __forceinline__ void pop() {
        head = head + 1 == kQ ? 0 : head + 1;
        --n;
    }
};

__device__ __forceinline__ int ld_acquire(const int* p) {
    return cuda::atomic_ref<int, cuda::thread_scope_block>(*const_cast<int*>(p)).load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void st_release(int* p, int v) {
    cuda::atomic_ref<int, cuda::thread_scope_block>(*p).store(v, cuda::memory_order_release);
}
__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// dTr(m) of one cell, tracer by tracer: dTr + flx for the face's left column,
// dTr - flx for its right column (ocean_redi.F90:1082-1088).
template <int NT, class Flux>
__device__ __forceinline__ void add_term(double* cell, size_t tstride, size_t lstride, int m, const Flux (&v)[NT],
                                         bool left) {
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        double* d = cell + t * tstride + (size_t)m * lstride;
        const double f = (double)v[t];
        *d = left ? *d + f : *d - f;
    }
}

// A term of a side: range and order checks; a term at a layer outside 0..nz-1
// is dropped, one below the side's previous term is added where it lands.
__device__ __forceinline__ bool term_ok(int m, int nz, int& last, int& bad) {
    if (m < 0 || m >= nz) {
        ++bad;
        return false;
    }
    if (m < last) ++bad;
    last = m;
    return true;
}

// The deferred terms of a side whose predecessor's frontier is `front`: the new
// term (if any) is added at once when nothing waits before it and the
// predecessor is past its layer, else queued; then the queue drains in order.
template <int NT, class Flux>
__device__ __forceinline__ void side_step(SideQueue<NT, Flux>& q, bool term, int m, const Flux (&f)[NT], int front,
                                          double* cell, size_t tstride, size_t lstride, bool left, int nz, int& last,
                                          int& bad, bool& progress) {
    if (term) {
        if (q.n == 0 && m < front) {
            if (term_ok(m, nz, last, bad)) add_term<NT>(cell, tstride, lstride, m, f, left);
        } else {
            q.push(m, f);
        }
    }
    while (q.n > 0 && q.head_layer() < front) {
        const int mh = q.head_layer();
        Flux v[NT];
        q.head_flux(v);
        if (term_ok(mh, nz, last, bad)) add_term<NT>(cell, tstride, lstride, mh, v, left);
        q.pop();
        progress = true;
    }
}

// dTr(m) (+|-)= flx through shared-memory atomics: the unordered fold (mixed
// form only; the additions of a layer land in whatever order the walks reach it).
template <int NT, class Flux>
__device__ __forceinline__ void add_term_any(double* cell, size_t tstride, size_t lstride, int m, const Flux (&v)[NT],
                                             bool left) {
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const double f = (double)v[t];
        atomicAdd(cell + t * tstride + (size_t)m * lstride, left ? f : -f);
    }
}

// ORD: the reference's addition order (the chain of frontiers and queues);
// otherwise every term is added as soon as it is computed (the mixed form,
// whose result is checked against the FP64 reference within a tolerance and
// needs no particular order).
template <int NT, class P, int BY, bool ORD>
__global__ void __launch_bounds__(32 * (2 * BY + 1)) k_flux_fold(FoldArgsT<P> a, int jlo, int jhi) {
    using Ops = plain::FluxOps<P>;
    using Raw = typename Ops::Raw;
    using He = typename P::He;
    using Flux = typename P::Flux;
    using L = FoldLayout<P, NT, BY, ORD>;
    constexpr unsigned kFull = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char smem[];

    const int nx = a.nx, ny = a.ny, nz = a.nz, nsub = 2 * nz + 1;
    const size_t ncol = (size_t)nx * ny;
    double* acc = reinterpret_cast<double*>(smem);
    double* ia = reinterpret_cast<double*>(smem + L::ia_off(nz));
    int* PE = reinterpret_cast<int*>(smem + L::front_off(nz));
    int* PS = PE + BY * 32;
    int* qlay = reinterpret_cast<int*>(smem + L::qlay_off(nz));
    Flux* qf = reinterpret_cast<Flux*>(smem + L::qf_off(nz));
    const size_t lstride = (size_t)BY * 32;       // accumulators: layer stride
    const size_t tstride = (size_t)nz * lstride;  // accumulators: tracer stride

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kWarps = 2 * BY + 1;
    const int i0 = blockIdx.x * kTileW;
    const int j0 = jlo + blockIdx.y * BY;

    // ---- this lane's face and the tile cells on its two sides
    const bool is_u = warp < BY;
    const int g = is_u ? warp : warp - BY;  // u: tile row; v: v-face row (below tile row g)
    bool face, rcell, lcell;
    int colL = 0, colR = 0, fo = 0;
    size_t fstride;
    double* cellR;  // accumulators of the right column's cell (if in the tile)
    double* cellL;  // ... of the left column's cell
    if (is_u) {
        const int j = j0 + g;
        const int fi = i0 + lane;  // u face between columns fi-1 and fi
        const int I = fi + 1;      // Fortran index
        const bool rowok = j < jhi;
        face = rowok && fi >= 1 && fi <= nx - 1 &&
               !((a.wall_w && I == a.nghost + 1) || (a.wall_e && I == a.nghost + a.nxp + 1));
        rcell = rowok && lane < kTileW && fi < nx;
        lcell = rowok && lane >= 1 && fi - 1 < nx;
        fstride = (size_t)(nx + 1) * ny;
        if (face) {
            colL = fi - 1 + nx * j;
            colR = fi + nx * j;
            fo = fi + (nx + 1) * j;
        }
        cellR = acc + g * 32 + lane;
        cellL = acc + g * 32 + (lane >= 1 ? lane - 1 : 0);
    } else {
        const int jf = j0 + g;  // v face between cell rows jf-1 and jf
        const int i = i0 + lane;
        const int J = jf + 1;
        const bool lok = lane < kTileW && i < nx;
        face = lok && jf >= 1 && jf <= ny - 1 &&
               !((a.wall_s && J == a.nghost + 1) || (a.wall_n && J == a.nghost + a.nyp + 1));
        rcell = lok && g < BY && jf < jhi;
        lcell = lok && g >= 1 && jf - 1 < jhi;
        fstride = (size_t)nx * (ny + 1);
        if (face) {
            colL = i + nx * (jf - 1);
            colR = i + nx * jf;
            fo = i + nx * jf;
        }
        cellR = acc + (g < BY ? g : 0) * 32 + lane;
        cellL = acc + (g >= 1 ? g - 1 : 0) * 32 + lane;
    }
    const bool walk = face && (rcell || lcell);
    const bool qL_on = ORD && walk && lcell;           // E (u walker) or N (v walker)
    const bool qR_on = ORD && walk && rcell && !is_u;  // S (v walker); W is added at once
    SideQueue<NT, Flux> qL, qR;
    {
        const int sL = is_u ? g : BY + 2 * g - 1;  // N queue of v row g (g >= 1)
        const int sR = BY + 2 * g;                 // S queue of v row g (g < BY)
        qL.lay = qlay + (size_t)(sL < 0 ? 0 : sL) * kQ * 32;
        qL.f = qf + (size_t)(sL < 0 ? 0 : sL) * kQ * NT * 32;
        qR.lay = qlay + (size_t)(sR >= L::kSlots ? 0 : sR) * kQ * 32;
        qR.f = qf + (size_t)(sR >= L::kSlots ? 0 : sR) * kQ * NT * 32;
    }

    // ---- the face's coefficient stream and flux coefficient
    const FaceInT<P>& c = is_u ? a.u : a.v;
    const He* __restrict__ hEff = c.hEff + fo;
    const typename P::Po* __restrict__ PoL = c.PoL + fo;
    const typename P::Po* __restrict__ PoR = c.PoR + fo;
    const typename P::Ko* __restrict__ KoL = c.KoL + fo;
    const typename P::Ko* __restrict__ KoR = c.KoR + fo;
    double coef = 0.0;
    if (walk) {
        const double* kh = is_u ? a.khtr_u : a.khtr_v;
        const double khv = kh ? __ldg(kh + fo) : a.khtr;
        // ((dt*khtr)*dy)*idx, ocean_redi.F90:1156/1168
        coef = a.dt * khv * __ldg((is_u ? a.dy_cu : a.dx_cv) + fo) * __ldg((is_u ? a.idxCu : a.idyCv) + fo);
    }
    const size_t ti_stride = ncol * (nz + 1), pp_stride = ncol * nz;

    // 1/areaT of the tile's cells
    for (int x = threadIdx.x; x < BY * 32; x += blockDim.x) {
        const int r = x / 32, l = x % 32, i = i0 + l, j = j0 + r;
        ia[x] = (l < kTileW && i < nx && j < jhi) ? 1.0 / __ldg(a.areaT + i + (size_t)nx * j) : 0.0;
    }

    int bad = 0;
    for (int tr0 = 0; tr0 < a.ntr; tr0 += NT) {
        if (__syncthreads_or(a.abort && *(volatile int*)a.abort != 0)) break;  // block-uniform
        const int nt = min(NT, a.ntr - tr0);
        for (size_t x = threadIdx.x; x < (size_t)NT * tstride; x += blockDim.x) acc[x] = 0.0;
        for (int x = threadIdx.x; x < 2 * BY * 32; x += blockDim.x) PE[x] = 0;
        __syncthreads();

        // tracers of the group (a slot beyond nt repeats tracer tr0; its
        // accumulators are not written back)
        const double* tiL0 = a.ti + (size_t)tr0 * ti_stride + colL;
        const double* tiR0 = a.ti + (size_t)tr0 * ti_stride + colR;
        const typename P::Ppm* ppL0 = a.ppm + (size_t)tr0 * pp_stride + colL;
        const typename P::Ppm* ppR0 = a.ppm + (size_t)tr0 * pp_stride + colR;
        auto trc = [nt](int n) { return (size_t)(n < nt ? n : 0); };

        // Coefficient rotation (as in the face-flux walk): the top surface ks,
        // the bottom surface ks+1 with hEff(ks), and the next pair in flight.
        int ks = walk ? 0 : nsub;
        int klt_raw = 1, krt_raw = 1, kl_t = 1, kr_t = 1;
        double pl_t = 0.0, pr_t = 0.0;
        He he_c = He(0);
        int klr_c = 1, krr_c = 1;
        double pl_c = 0.0, pr_c = 0.0;
        if (walk) {
            klt_raw = (int)__ldg(KoL);
            krt_raw = (int)__ldg(KoR);
            kl_t = min(max(klt_raw, 1), nz);
            kr_t = min(max(krt_raw, 1), nz);
            pl_t = __ldg(PoL);
            pr_t = __ldg(PoR);
            he_c = __ldg(hEff);
            klr_c = (int)__ldg(KoL + fstride);
            krr_c = (int)__ldg(KoR + fstride);
            pl_c = __ldg(PoL + fstride);
            pr_c = __ldg(PoR + fstride);
        }
        double tl[NT], tr[NT];
        bool have_t = false;
        qL.head = qL.n = 0;
        qR.head = qR.n = 0;
        int lastL = -1, lastR = -1;
        long long t_prog = 0;
        bool timed = false;
        // A side that forwards another warp's frontier (S: min(PE, own)) may stop
        // only once it has forwarded the final value, even with no face to walk.
        bool fwd_done = is_u || !rcell;

        // Every warp runs at least one iteration, so every frontier of the tile
        // is published even where no lane of a warp has a face to walk.
        for (;;) {
            const bool more = ks < nsub;
            bool progress = false;
            const bool comp = more && (!qL_on || qL.n < kQ) && (!qR_on || qR.n < kQ);
            Flux f[NT];
            bool term = false;
            int mL = 0, mR = 0;
            if (__any_sync(kFull, comp)) {
                He he_n = He(0);
                int klr_n = 1, krr_n = 1;
                double pl_n = 0.0, pr_n = 0.0;
                if (comp && ks + 1 < nsub) {
                    const size_t s1 = (size_t)(ks + 1) * fstride, s2 = s1 + fstride;
                    he_n = __ldg(hEff + s1);
                    klr_n = (int)__ldg(KoL + s2);
                    krr_n = (int)__ldg(KoR + s2);
                    pl_n = __ldg(PoL + s2);
                    pr_n = __ldg(PoR + s2);
                }
                const int kl_b = min(max(klr_c, 1), nz), kr_b = min(max(krr_c, 1), nz);
                const double pl_b = pl_c, pr_b = pr_c;
                if (__any_sync(kFull, comp && he_c != He(0))) {
                    if (comp) {
                        const double xRl = pl_b + (double)(kl_b - kl_t);
                        const double xRr = pr_b + (double)(kr_b - kr_t);
                        double b0L[NT], b1L[NT], b0R[NT], b1R[NT];
                        Raw qLr[NT], qRr[NT];
#pragma unroll
                        for (int n = 0; n < NT; ++n) {
                            const double* tL = tiL0 + trc(n) * ti_stride;
                            const double* tR = tiR0 + trc(n) * ti_stride;
                            b0L[n] = __ldg(tL + (size_t)(kl_b - 1) * ncol);
                            b1L[n] = __ldg(tL + (size_t)kl_b * ncol);
                            b0R[n] = __ldg(tR + (size_t)(kr_b - 1) * ncol);
                            b1R[n] = __ldg(tR + (size_t)kr_b * ncol);
                            qLr[n] = Ops::template load<LdNC>(ppL0 + trc(n) * pp_stride + (size_t)(kl_t - 1) * ncol);
                            qRr[n] = Ops::template load<LdNC>(ppR0 + trc(n) * pp_stride + (size_t)(kr_t - 1) * ncol);
                        }
                        if (!have_t) {
#pragma unroll
                            for (int n = 0; n < NT; ++n) {
                                const double* tL = tiL0 + trc(n) * ti_stride;
                                const double* tR = tiR0 + trc(n) * ti_stride;
                                tl[n] = plain::interp(pl_t, __ldg(tL + (size_t)(kl_t - 1) * ncol),
                                                      __ldg(tL + (size_t)kl_t * ncol));
                                tr[n] = plain::interp(pr_t, __ldg(tR + (size_t)(kr_t - 1) * ncol),
                                                      __ldg(tR + (size_t)kr_t * ncol));
                            }
                        }
#pragma unroll
                        for (int n = 0; n < NT; ++n) {
                            const double bl = plain::interp(pl_b, b0L[n], b1L[n]);
                            const double br = plain::interp(pr_b, b0R[n], b1R[n]);
                            const typename Ops::Mean tlay = Ops::mean(pl_t, xRl, qLr[n]);
                            const typename Ops::Mean trlay = Ops::mean(pr_t, xRr, qRr[n]);
                            const double dT = guarded_dT(tr[n] - tl[n], br - bl, (double)(trlay - tlay));
                            f[n] = Ops::flux(dT, he_c, coef);
                            tl[n] = bl;
                            tr[n] = br;
                        }
                        have_t = true;
                    }
                } else if (comp) {
                    have_t = false;
                }
                if (comp) {
                    term = he_c != He(0);
                    mL = klt_raw - 1;
                    mR = krt_raw - 1;
                    kl_t = kl_b;
                    kr_t = kr_b;
                    klt_raw = klr_c;
                    krt_raw = krr_c;
                    pl_t = pl_b;
                    pr_t = pr_b;
                    he_c = he_n;
                    klr_c = klr_n;
                    krr_c = krr_n;
                    pl_c = pl_n;
                    pr_c = pr_n;
                    ++ks;
                    progress = true;
                }
            }
            if constexpr (!ORD) {
                if (term && rcell && term_ok(mR, nz, lastR, bad)) add_term_any<NT>(cellR, tstride, lstride, mR, f, false);
                if (term && lcell && term_ok(mL, nz, lastL, bad)) add_term_any<NT>(cellL, tstride, lstride, mL, f, true);
                if (__all_sync(kFull, ks >= nsub)) break;
                continue;
            }
            // Layer of each side's next term once its queue is empty.
            const int nxtL = ks < nsub ? klt_raw - 1 : kInf;
            const int nxtR = ks < nsub ? krt_raw - 1 : kInf;
            if (is_u) {
                // W: the first side of the chain, added at once.
                if (term && rcell && term_ok(mR, nz, lastR, bad)) add_term<NT>(cellR, tstride, lstride, mR, f, false);
                __syncwarp();
                const int frW = (walk && rcell) ? nxtR : kInf;
                const int pW = __shfl_up_sync(kFull, frW, 1);  // W frontier of cell lane-1
                if (lcell) {
                    if (qL_on) side_step<NT>(qL, term, mL, f, pW, cellL, tstride, lstride, true, nz, lastL, bad, progress);
                    const int frE = qL.n > 0 ? qL.head_layer() : (qL_on ? nxtL : kInf);
                    st_release(&PE[g * 32 + lane - 1], min(pW, frE));
                }
            } else {
                if (rcell) {  // S side of cell (lane, g): after E
                    const int pe = ld_acquire(&PE[g * 32 + lane]);
                    if (qR_on) side_step<NT>(qR, term, mR, f, pe, cellR, tstride, lstride, false, nz, lastR, bad, progress);
                    const int frS = qR.n > 0 ? qR.head_layer() : (qR_on ? nxtR : kInf);
                    const int ps_out = min(pe, frS);
                    st_release(&PS[g * 32 + lane], ps_out);
                    fwd_done = ps_out >= kInf;
                }
                if (qL_on) {  // N side of cell (lane, g-1): after S
                    const int ps = ld_acquire(&PS[(g - 1) * 32 + lane]);
                    side_step<NT>(qL, term, mL, f, ps, cellL, tstride, lstride, true, nz, lastL, bad, progress);
                }
            }
            if (__all_sync(kFull, ks >= nsub && qL.n == 0 && qR.n == 0 && fwd_done)) break;
            // A warp that made no progress waits for its predecessors' frontiers:
            // back off, and give up after kStallNs (counted as an error).
            if (__any_sync(kFull, progress)) {
                timed = false;
            } else {
                const long long now = __shfl_sync(kFull, global_ns(), 0);
                const int stop = a.abort ? __shfl_sync(kFull, *(volatile int*)a.abort, 0) : 0;
                if (!timed) {
                    t_prog = now;
                    timed = true;
                }
                if (now - t_prog > kStallNs || stop != 0) {
                    if (lane == 0) {
                        ++bad;
                        if (a.abort) atomicExch(a.abort, 1);
                    }
                    break;
                }
                __nanosleep(100);
            }
        }
        __syncthreads();

        // hTr(knat) += dTr(knat) * (1/areaT), knat = nz + 1 - Ko (ocean_redi.F90:1175-1178)
        for (int row = warp; row < nt * BY * nz; row += kWarps) {
            const int t = row / (BY * nz), rem = row - t * (BY * nz), m = rem / BY, r = rem - m * BY;
            const int i = i0 + lane, j = j0 + r;
            if (lane < kTileW && i < nx && j < jhi) {
                const size_t o = (size_t)i + (size_t)nx * j + (size_t)(nz - 1 - m) * ncol;
                a.htr[tr0 + t][o] =
                    a.htr_in[tr0 + t][o] + acc[t * tstride + m * lstride + r * 32 + lane] * ia[r * 32 + lane];
            }
        }
        __syncthreads();
    }
    if (bad && a.err) atomicAdd(a.err, bad);
}

}  // namespace fold
}  // namespace redi
