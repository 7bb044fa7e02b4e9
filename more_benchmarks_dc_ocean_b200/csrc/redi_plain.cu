// Redi neutral-diffusion step for sm_100a: the plain FP64 form and the
// mixed-precision form (precision policies in redi_kernels.h).
//
// Compiled with FMA contraction off (-fmad=false): every FP64 operation is the
// reference's (redi/ocean_redi.F90), in the reference's order, so the plain
// form is bit-identical to the CPU oracle and to the reference's own CUDA ports
// built the same way, and the mixed form takes every discrete decision exactly
// as the plain form does.
//
// Decomposition (one column = all nz layers of one (i,j) T-cell); the
// per-item bodies live in redi_items.cuh:
//
//   Phase A  redi_calc_coeffs (ocean_redi.F90:572-812)
//     k_column_state   one thread per column: top-down PPM interface T, S
//                      (thickness geometry shared by T and S), hydrostatic
//                      interface pressure and the EOS derivatives, written once
//                      per column (the reference rebuilds each column for each
//                      of its up to four faces).
//     k_neutral_sweep  one thread per interior wet face: the 2nz+2-surface
//                      continuous sweep (ocean_redi.F90:307-464), writing
//                      PoL/PoR/KoL/KoR/hEff in the reference layout
//                      (k_neutral_sweep_w: both columns' windows in a
//                      shared-memory ring, the default).
//
//   Phase B  redi_apply_flux (ocean_redi.F90:927-1181), all tracers fused
//     k_tracer_recon   one thread per (column, tracer pair): top-down PPM tracer
//                      edges + limiter (ocean_redi.F90:852-891).
//     k_face_flux      one thread per interior non-wall face: the sublayer
//                      fluxes of a group of tracers, each face once.
//     k_cell_gather    one thread per T-cell column: the fluxes of its four
//                      faces folded into its own layers in the reference's
//                      W, E, S, N / ks order, then hTr += dTr * (1/areaT).
//
// Layouts: cell fields (nx, ny, nz) column-major (i fastest); face fields as in
// the reference ((nx+1, ny, ns) u, (nx, ny+1, ns) v); scratch [layer][column].

#include <cstdint>
#include <cuda_runtime.h>

#include "redi_fold.cuh"
#include "redi_items.cuh"

namespace redi {
namespace plain {

// ---------------------------------------------------------------------------
// Standalone kernels: one launch per stage, read-only inputs through the
// non-coherent cache path.
// ---------------------------------------------------------------------------
// Face index ranges of one launch, per direction: faces lo[d] <= t < hi[d].
struct FaceRange {
    int lo[2], hi[2];
};

__global__ void __launch_bounds__(128) k_column_state(ColumnStateArgs a, int c0, int c1) {
    const int col = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (col < c1) column_state_item<LdNC>(a, col);
}

template <class P>
__global__ void __launch_bounds__(128) k_column_recon(ColumnStateArgs a, ReconArgsT<P> rc, int ts_swap, int ncol) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col < ncol) column_recon_item<P, LdNC>(a, rc, ts_swap, col);
}

template <class P>
__global__ void __launch_bounds__(128) k_neutral_sweep(SweepArgsT<P> a, FaceRange r) {
    const int d = blockIdx.x & 1;  // blocks alternate between u and v faces, as in k_face_flux
    const int t = r.lo[d] + (int)(blockIdx.x >> 1) * blockDim.x + threadIdx.x;
    if (t < r.hi[d]) sweep_item<P, LdNC, true>(a, d, t);
}

// The sweep with both windows in a shared-memory ring of NR interfaces per
// column (dynamic shared memory: sizeof(SweepWin<NR>)).
// A block's faces are first sorted into dry ones (handled at once) and wet
// ones, which are compacted onto the block's leading threads in face order, so
// the sweeps of a block with land run in as few warps as its wet faces fill.
template <class P, int NR>
__global__ void __launch_bounds__(kSweepWinThreads) k_neutral_sweep_w(SweepArgsT<P> a, FaceRange r) {
    extern __shared__ __align__(16) unsigned char sweep_win[];
    __shared__ int list[kSweepWinThreads];
    __shared__ int warp_n[kSweepWinThreads / 32];
    const int d = blockIdx.x & 1;
    const int t = r.lo[d] + (int)(blockIdx.x >> 1) * blockDim.x + threadIdx.x;
    const bool wet = t < r.hi[d] && sweep_face_dry<P, LdNC>(a, d, t);
    const int n = block_compact<kSweepWinThreads>(wet, t, list, warp_n);
    if ((int)threadIdx.x < n)
        sweep_item_win<P, LdNC, NR, true>(a, d, list[threadIdx.x], *reinterpret_cast<SweepWin<NR>*>(sweep_win));
}

template <int NT, class P>
__global__ void __launch_bounds__(128) k_tracer_recon(ReconArgsT<P> a, int c0, int nb) {
    recon_item<NT, P, LdNC>(a, blockIdx.x * blockDim.x + threadIdx.x, c0, nb);
}

// Every thread of the block reaches flux_item (its warp-wide votes need all lanes).
// Blocks alternate between the directions (even: u faces, odd: v faces), so the
// u and v faces of the same rows are in flight together and the second reads of
// a column's reconstruction are served from L2 instead of HBM.
// The block's faces that need a flux (not walls, not dry) are compacted onto
// its leading threads in face order; the others walk as stand-ins or, in warps
// with no face left, return at once.
template <int NT, class P>
__global__ void __launch_bounds__(128) k_face_flux(FaceFluxArgsT<P> a, int tr0, FaceRange r) {
    __shared__ int list[128];
    __shared__ int warp_n[4];
    const int d = blockIdx.x & 1;
    const int t = r.lo[d] + (int)(blockIdx.x >> 1) * blockDim.x + threadIdx.x;
    const int n = block_compact<128>(flux_face_valid(a, d, t, r.hi[d]), t, list, warp_n);
    flux_item<NT, P, LdNC>(a, d, (int)threadIdx.x < n ? list[threadIdx.x] : r.hi[d], tr0, r.hi[d]);
}

// The face flux with its reconstruction loads staged one sublayer ahead
// through shared memory (flux_item_staged); the same block order.
// The face flux reading each column's reconstruction through a two-layer ring
// in shared memory (flux_item_ring); the same block order.
template <int NT, class P>
__global__ void __launch_bounds__(kFluxThreads) k_face_flux_r(FaceFluxArgsT<P> a, int tr0, FaceRange r) {
    extern __shared__ __align__(16) unsigned char ring[];
    __shared__ int list[kFluxThreads];
    __shared__ int warp_n[kFluxThreads / 32];
    double2* rpp = reinterpret_cast<double2*>(ring);
    double* rti = reinterpret_cast<double*>(ring + FluxRing<NT, P>::pp_units * sizeof(double2));
    const int d = blockIdx.x & 1;
    const int t = r.lo[d] + (int)(blockIdx.x >> 1) * blockDim.x + threadIdx.x;
    const int n = block_compact<kFluxThreads>(flux_face_valid(a, d, t, r.hi[d]), t, list, warp_n);
    flux_item_ring<NT, P>(a, d, (int)threadIdx.x < n ? list[threadIdx.x] : r.hi[d], tr0, r.hi[d], rpp, rti);
}

template <int NT, class P>
__global__ void __launch_bounds__(kFluxThreads) k_face_flux_s(FaceFluxArgsT<P> a, int tr0, FaceRange r) {
    extern __shared__ __align__(16) unsigned char stage[];
    double* sti = reinterpret_cast<double*>(stage);
    double2* spp = reinterpret_cast<double2*>(stage + FluxStage<NT, P>::ti_doubles * sizeof(double));
    const int d = blockIdx.x & 1;
    flux_item_staged<NT, P>(a, d, r.lo[d] + (int)(blockIdx.x >> 1) * blockDim.x + threadIdx.x, tr0, r.hi[d], sti,
                            spp);
}

template <int NT, int CH, class P>
__global__ void __launch_bounds__(128) k_cell_gather(CellGatherArgsT<P> a, int tr0, int fslot, int j0, int j1) {
    const int j = j0 + blockIdx.y * blockDim.y + threadIdx.y;
    // sublayers fetched per round trip: 3 with 4-layer chunks, 4 with deeper chunks (measured)
    if (j < j1) gather_item<NT, CH, P, LdNC, (CH <= 4 ? 3 : 4)>(a, blockIdx.x * blockDim.x + threadIdx.x, j, tr0, fslot);
}

// The gather with its per-layer sums in shared memory (gather_item_s).
// U: sublayers fetched per round trip (0: 3 for 4-layer chunks, 4 otherwise).
// PIPE: the walk's batches software-pipelined (gather_run_sp).
template <int NT, int CH, class P, int U = 0, bool PIPE = false>
__global__ void __launch_bounds__(kGatherThreads) k_cell_gather_s(CellGatherArgsT<P> a, int tr0, int fslot, int j0,
                                                                  int j1) {
    __shared__ double acc[CH * NT * kGatherThreads];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int j = j0 + blockIdx.y * blockDim.y + threadIdx.y;
    constexpr int kU = U ? U : (CH <= 4 ? 3 : 4);
    if (j < j1)
        gather_item_s<NT, CH, P, LdNC, kU, PIPE>(a, blockIdx.x * blockDim.x + threadIdx.x, j, tr0, fslot, acc + tid);
}

// The point EOS at n independent points, as the column state evaluates it at
// each interface (eos_density_point + eos_specvol_derivs).
__global__ void __launch_bounds__(128) k_eos_points(EosParams e, int n, const double* __restrict__ T,
                                                    const double* __restrict__ S, const double* __restrict__ p,
                                                    double* __restrict__ rho, double* __restrict__ dsv_dt,
                                                    double* __restrict__ dsv_ds) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r, a = e.alpha_T / (e.rho0 * e.rho0), b = -e.beta_S / (e.rho0 * e.rho0);
    if (eos_is_linear(e.variant))
        r = e.rho0 + e.beta_S * (S[i] - e.S_ref) - e.alpha_T * (T[i] - e.T_ref);
    else
        eos::nonlinear_point(e.variant, T[i], S[i], p[i], r, a, b);
    rho[i] = r;
    dsv_dt[i] = a;
    dsv_ds[i] = b;
}

}  // namespace plain

// ---------------------------------------------------------------------------
// Host launchers (stream-ordered, no synchronisation).
// ---------------------------------------------------------------------------
namespace {

// The index ranges a band of T-cell rows needs (see Band in redi_kernels.h).
struct BandRanges {
    int j0, j1;        // cell rows
    int c0, c1;        // columns (rows j0-1 .. j1, clamped)
    plain::FaceRange f;
};

BandRanges band_ranges(int nx, int ny, Band b) {
    BandRanges r;
    r.j0 = max(b.row0, 0);
    r.j1 = b.row1 < 0 ? ny : min(b.row1, ny);
    r.c0 = max(r.j0 - 1, 0) * nx;
    r.c1 = min(r.j1 + 1, ny) * nx;
    r.f.lo[0] = r.j0 * (nx - 1);  // u faces of rows j0 .. j1-1
    r.f.hi[0] = r.j1 * (nx - 1);
    const int f0 = max(r.j0, 1), f1 = min(r.j1, ny - 1);  // v faces between rows f-1 and f, f0 <= f <= f1
    r.f.lo[1] = (f0 - 1) * nx;
    r.f.hi[1] = f1 >= f0 ? f1 * nx : r.f.lo[1];
    if (r.j1 <= r.j0) r.c1 = r.c0, r.f.hi[0] = r.f.lo[0], r.f.hi[1] = r.f.lo[1];
    return r;
}

unsigned face_blocks(const plain::FaceRange& f) {
    const int n = max(f.hi[0] - f.lo[0], f.hi[1] - f.lo[1]);
    return (unsigned)((max(n, 0) + 127) / 128);
}

}  // namespace

cudaError_t launch_column_state(const ColumnStateArgs& cs, cudaStream_t st, Band band) {
    const BandRanges r = band_ranges(cs.nx, cs.ny, band);
    if (r.c1 > r.c0) {
        launch_begin(K_COLUMN_STATE, st);
        plain::k_column_state<<<(r.c1 - r.c0 + 127) / 128, 128, 0, st>>>(cs, r.c0, r.c1);
        launch_end(K_COLUMN_STATE, st);
    }
    return cudaGetLastError();
}

template <class P>
cudaError_t launch_column_recon(const ColumnStateArgs& cs, const ReconArgsT<P>& rc, int ts_swap, cudaStream_t st) {
    const int ncol = cs.nx * cs.ny;
    launch_begin(K_COLUMN_RECON, st);
    plain::k_column_recon<P><<<(ncol + 127) / 128, 128, 0, st>>>(cs, rc, ts_swap, ncol);
    launch_end(K_COLUMN_RECON, st);
    return cudaGetLastError();
}
template cudaError_t launch_column_recon<PlainPrec>(const ColumnStateArgs&, const ReconArgsT<PlainPrec>&, int,
                                                    cudaStream_t);
template cudaError_t launch_column_recon<MixedPrec>(const ColumnStateArgs&, const ReconArgsT<MixedPrec>&, int,
                                                    cudaStream_t);

cudaError_t launch_eos_points(const EosParams& e, int n, const double* T, const double* S, const double* p,
                              double* rho, double* dsv_dt, double* dsv_ds, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    launch_begin(K_AUX, st);
    plain::k_eos_points<<<(n + 127) / 128, 128, 0, st>>>(e, n, T, S, p, rho, dsv_dt, dsv_ds);
    launch_end(K_AUX, st);
    return cudaGetLastError();
}

template <class P, int NR>
static cudaError_t launch_sweep_w(const SweepArgsT<P>& sw, const plain::FaceRange& f, unsigned nb, cudaStream_t st) {
    const size_t smem = sizeof(plain::SweepWin<NR>);
    cudaError_t e =
        cudaFuncSetAttribute(plain::k_neutral_sweep_w<P, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned nbw = (unsigned)(((size_t)nb * 128 + plain::kSweepWinThreads - 1) / plain::kSweepWinThreads);
    plain::k_neutral_sweep_w<P, NR><<<2 * nbw, plain::kSweepWinThreads, smem, st>>>(sw, f);
    return cudaSuccess;
}

template <class P>
cudaError_t launch_sweep(const SweepArgsT<P>& sw, cudaStream_t st, Band band) {
    const BandRanges r = band_ranges(sw.nx, sw.ny, band);
    const unsigned nb = face_blocks(r.f);
    if (nb > 0) {
        const int kid = P::kMixed ? K_MIXED_SWEEP : K_NEUTRAL_SWEEP;
        const int form = cell_tuning().sweep_form;
        launch_begin(kid, st);
        if (form >= 3 && form <= 5) {
            cudaError_t e = form == 3   ? launch_sweep_w<P, 3>(sw, r.f, nb, st)
                            : form == 4 ? launch_sweep_w<P, 4>(sw, r.f, nb, st)
                                        : launch_sweep_w<P, 5>(sw, r.f, nb, st);
            if (e != cudaSuccess) return e;
        } else {
            plain::k_neutral_sweep<P><<<2 * nb, 128, 0, st>>>(sw, r.f);
        }
        launch_end(kid, st);
    }
    return cudaGetLastError();
}

template <int GNT, class P>
static void launch_gather(const CellGatherArgsT<P>& cg, int tr, int slot, const BandRanges& r, const CellTuning& tune,
                          dim3 cgrid, dim3 block, cudaStream_t st) {
    launch_begin(K_CELL_UPDATE, st);
    // shared-memory sums: CH x GNT x 128 doubles must stay within the 48 KB of static shared memory
    if (tune.gather_smem && block.x * block.y == plain::kGatherThreads && tune.chunk * GNT <= 32) {
        const bool deep = tune.gather_batch >= 8;  // 8 sublayers per round trip instead of 3-4
        if (tune.gather_pipe) {  // batches of 4, the next one in flight
            switch (tune.chunk) {
                case 4: plain::k_cell_gather_s<GNT, 4, P, 4, true><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1); break;
                case 16:
                    if constexpr (GNT <= 2)
                        plain::k_cell_gather_s<GNT, 16, P, 4, true><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1);
                    break;
                default: plain::k_cell_gather_s<GNT, 8, P, 4, true><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1); break;
            }
            launch_end(K_CELL_UPDATE, st);
            return;
        }
        switch (tune.chunk) {
            case 4:
                if (deep) plain::k_cell_gather_s<GNT, 4, P, 8><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1);
                else plain::k_cell_gather_s<GNT, 4, P><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1);
                break;
            case 16:
                if constexpr (GNT <= 2) {
                    if (deep) plain::k_cell_gather_s<GNT, 16, P, 8><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1);
                    else plain::k_cell_gather_s<GNT, 16, P><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1);
                }
                break;
            default:
                if (deep) plain::k_cell_gather_s<GNT, 8, P, 8><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1);
                else plain::k_cell_gather_s<GNT, 8, P><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1);
                break;
        }
    } else {
        switch (tune.chunk) {
            case 4: plain::k_cell_gather<GNT, 4, P><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1); break;
            case 16: plain::k_cell_gather<GNT, 16, P><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1); break;
            default: plain::k_cell_gather<GNT, 8, P><<<cgrid, block, 0, st>>>(cg, tr, slot, r.j0, r.j1); break;
        }
    }
    launch_end(K_CELL_UPDATE, st);
}

// 8 tracers per gather: only the shared-memory sums with 4-layer chunks fit
// (32 KB); gather_spans_two admits no other shape.
template <class P>
static void launch_gather_8(const CellGatherArgsT<P>& cg, int tr, const BandRanges& r, const CellTuning& tune,
                            dim3 cgrid, dim3 block, cudaStream_t st) {
    launch_begin(K_CELL_UPDATE, st);
    if (tune.gather_batch >= 8) plain::k_cell_gather_s<8, 4, P, 8><<<cgrid, block, 0, st>>>(cg, tr, 0, r.j0, r.j1);
    else plain::k_cell_gather_s<8, 4, P><<<cgrid, block, 0, st>>>(cg, tr, 0, r.j0, r.j1);
    launch_end(K_CELL_UPDATE, st);
}

// The face flux of tracers tr0 .. tr0+NT-1 into flux-buffer slots
// ff.fslot0 .. ff.fslot0+NT-1.
template <int NT, class P>
static void launch_flux(const FaceFluxArgsT<P>& ff, int tr0, const BandRanges& r, const CellTuning& tune,
                        cudaStream_t st) {
    const unsigned nb = face_blocks(r.f);
    if (nb == 0) return;
    const int kid = P::kMixed ? K_MIXED_FLUX : K_FACE_FLUX;
    if constexpr (NT <= 4) {
        if (tune.flux_staged == 2) {
            static int opted[64] = {};
            int dev = 0;
            cudaGetDevice(&dev);
            const int bytes = (int)plain::FluxRing<NT, P>::bytes;
            if (dev >= 0 && dev < 64 && !opted[dev]) {
                cudaFuncSetAttribute(plain::k_face_flux_r<NT, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
                opted[dev] = 1;
            }
            launch_begin(kid, st);
            plain::k_face_flux_r<NT, P><<<2 * nb, plain::kFluxThreads, bytes, st>>>(ff, tr0, r.f);
            launch_end(kid, st);
            return;
        }
    }
    if constexpr (NT <= 2) {
        if (tune.flux_staged == 1) {
            // opt into more than 48 KB of dynamic shared memory once per device
            static int opted[64] = {};
            int dev = 0;
            cudaGetDevice(&dev);
            const int bytes = (int)plain::FluxStage<NT, P>::bytes;
            if (dev >= 0 && dev < 64 && !opted[dev]) {
                cudaFuncSetAttribute(plain::k_face_flux_s<NT, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
                opted[dev] = 1;
            }
            launch_begin(kid, st);
            plain::k_face_flux_s<NT, P><<<2 * nb, plain::kFluxThreads, bytes, st>>>(ff, tr0, r.f);
            launch_end(kid, st);
            return;
        }
    }
    launch_begin(kid, st);
    plain::k_face_flux<NT, P><<<2 * nb, 128, 0, st>>>(ff, tr0, r.f);
    launch_end(kid, st);
}

// The gathers of tracers tr0 .. tr0+NS-1, whose fluxes sit in slots 0 .. NS-1:
// one launch of 8 tracers (WIDE: the fluxes of two face-flux launches), or
// launches of 4 or 2 tracers, which read consecutive slots.
template <int NS, class P, bool WIDE = false>
static void launch_gathers(const CellGatherArgsT<P>& cg, int tr0, const BandRanges& r, const CellTuning& tune,
                           cudaStream_t st) {
    const dim3 block(tune.bx, tune.by);
    const dim3 cgrid((cg.nx + tune.bx - 1) / tune.bx, (r.j1 - r.j0 + tune.by - 1) / tune.by);
    if (cgrid.y == 0) return;
    if constexpr (WIDE) {
        launch_gather_8<P>(cg, tr0, r, tune, cgrid, block, st);
        return;
    }
    const int gnt = (tune.gather_tracers >= 4 && NS >= 4) ? 4 : (NS < 2 ? NS : 2);
    for (int g = 0; g < NS; g += gnt) {
        if (tr0 + g >= cg.ntr) break;
        if (gnt == 4) {
            launch_gather<(NS >= 4 ? 4 : 1), P>(cg, tr0 + g, g, r, tune, cgrid, block, st);
        } else {
            launch_gather<(NS < 2 ? NS : 2), P>(cg, tr0 + g, g, r, tune, cgrid, block, st);
        }
    }
}

// The tracer reconstruction over the band's columns, two tracers per thread.
template <class P>
void launch_recon(const ReconArgsT<P>& rc, const BandRanges& r, cudaStream_t st) {
    const int ngroups = (rc.ntr + 1) / 2;
    const int nb = r.c1 - r.c0;
    const long long n = (long long)nb * ngroups;
    const int kid = P::kMixed ? K_MIXED_RECON : K_TRACER_RECON;
    launch_begin(kid, st);
    plain::k_tracer_recon<2, P><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(rc, r.c0, nb);
    launch_end(kid, st);
}

// ---------------------------------------------------------------------------
// The fused face-flux + fold pass (redi_fold.cuh).
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kFoldSmemMax = 232448;      // dynamic shared memory a block may opt into on sm_100a
constexpr size_t kFoldSmemTwo = 113 * 1024;  // two blocks per SM

template <int NT, class P, int BY, bool ORD>
cudaError_t launch_fold_o(const fold::FoldArgsT<P>& fa, int jlo, int jhi, cudaStream_t st) {
    using L = fold::FoldLayout<P, NT, BY, ORD>;
    const size_t smem = L::bytes(fa.nz);
    // opt into large dynamic shared memory once per device
    static int opted[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !opted[dev]) {
        cudaError_t e = cudaFuncSetAttribute(fold::k_flux_fold<NT, P, BY, ORD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kFoldSmemMax);
        if (e != cudaSuccess) return e;
        opted[dev] = 1;
    }
    if (fa.abort) {
        cudaError_t e = cudaMemsetAsync(fa.abort, 0, sizeof(int), st);
        if (e != cudaSuccess) return e;
    }
    const dim3 grid((unsigned)((fa.nx + fold::kTileW - 1) / fold::kTileW), (unsigned)((jhi - jlo + BY - 1) / BY));
    const int kid = P::kMixed ? K_MIXED_FOLD : K_FLUX_FOLD;
    launch_begin(kid, st);
    fold::k_flux_fold<NT, P, BY, ORD><<<grid, 32 * (2 * BY + 1), smem, st>>>(fa, jlo, jhi);
    launch_end(kid, st);
    return cudaGetLastError();
}

// The plain form always folds in the reference's order; the mixed form folds
// in any order unless the ordered fold is asked for.
template <int NT, class P, int BY>
cudaError_t launch_fold_t(const fold::FoldArgsT<P>& fa, int jlo, int jhi, cudaStream_t st) {
    if (P::kMixed && !fold_tuning().ordered_mixed) return launch_fold_o<NT, P, BY, false>(fa, jlo, jhi, st);
    return launch_fold_o<NT, P, BY, true>(fa, jlo, jhi, st);
}

template <class P, bool ORD>
size_t fold_smem_o(int nt, int by, int nz) {
    if (by == 1) {
        return nt == 4 ? fold::FoldLayout<P, 4, 1, ORD>::bytes(nz)
             : nt == 2 ? fold::FoldLayout<P, 2, 1, ORD>::bytes(nz) : fold::FoldLayout<P, 1, 1, ORD>::bytes(nz);
    }
    return nt == 4 ? fold::FoldLayout<P, 4, 2, ORD>::bytes(nz)
         : nt == 2 ? fold::FoldLayout<P, 2, 2, ORD>::bytes(nz) : fold::FoldLayout<P, 1, 2, ORD>::bytes(nz);
}
template <class P>
size_t fold_smem(int nt, int by, int nz) {
    return (P::kMixed && !fold_tuning().ordered_mixed) ? fold_smem_o<P, false>(nt, by, nz)
                                                       : fold_smem_o<P, true>(nt, by, nz);
}

}  // namespace

template <class P>
FoldShape fold_shape(int nz, int ntr) {
    const FoldTuning t = fold_tuning();
    FoldShape s{0, 0};
    if (!(P::kMixed ? t.enable_mixed : t.enable)) return s;
    const int want_by = t.rows == 1 ? 1 : 2;
    const int cap_nt = t.tracers > 0 ? t.tracers : 4;
    // the rows asked for first, then the most tracers per pass that keep two
    // blocks per SM (one block if nothing else fits), never more than needed
    for (int pass = 0; pass < 2 && s.nt == 0; ++pass) {
        const size_t budget = pass == 0 ? kFoldSmemTwo : kFoldSmemMax;
        for (int by : {want_by, 3 - want_by}) {
            for (int nt : {4, 2, 1}) {
                if (nt > cap_nt || (nt > 1 && nt / 2 >= ntr)) continue;
                if (fold_smem<P>(nt, by, nz) <= budget) {
                    s.nt = nt;
                    s.by = by;
                    break;
                }
            }
            if (s.nt) break;
        }
    }
    return s;
}

template <class P>
cudaError_t launch_phase_b(const ReconArgsT<P>& rc_all, const FaceFluxArgsT<P>& ff, const CellGatherArgsT<P>& cg,
                           cudaStream_t st, Band band, int recon_from) {
    const BandRanges r = band_ranges(rc_all.nx, rc_all.ny, band);
    // the tracers still to reconstruct: rc_all's from recon_from on
    ReconArgsT<P> rc = rc_all;
    if (recon_from > 0) {
        const size_t ncol = (size_t)rc_all.nx * rc_all.ny;
        rc.ntr = rc_all.ntr > recon_from ? rc_all.ntr - recon_from : 0;
        for (int n = 0; n < rc.ntr; ++n) rc.htr[n] = rc_all.htr[n + recon_from];
        rc.ti = rc_all.ti + (size_t)recon_from * ncol * (rc_all.nz + 1);
        rc.ppm = rc_all.ppm + (size_t)recon_from * ncol * rc_all.nz;
    }
    const FoldShape fs = fold_shape<P>(rc.nz, ff.ntr);
    if (fs.nt > 0) {
        if (r.c1 > r.c0 && rc.ntr > 0) {
            launch_recon<P>(rc, r, st);
        }
        if (r.j1 <= r.j0) return cudaGetLastError();
        fold::FoldArgsT<P> fa{};
        fa.nx = ff.nx; fa.ny = ff.ny; fa.nz = ff.nz; fa.ntr = ff.ntr;
        fa.nghost = ff.nghost; fa.nxp = ff.nxp; fa.nyp = ff.nyp;
        fa.wall_w = ff.wall_w; fa.wall_e = ff.wall_e; fa.wall_s = ff.wall_s; fa.wall_n = ff.wall_n;
        fa.dt = ff.dt; fa.khtr = ff.khtr; fa.khtr_u = ff.khtr_u; fa.khtr_v = ff.khtr_v;
        fa.dy_cu = ff.dy_cu; fa.dx_cv = ff.dx_cv; fa.idxCu = ff.idxCu; fa.idyCv = ff.idyCv; fa.areaT = cg.areaT;
        fa.u = ff.u; fa.v = ff.v; fa.ti = ff.ti; fa.ppm = ff.ppm; fa.err = cg.err;
        fa.abort = cg.err ? cg.err + 1 : nullptr;  // the word after the error count (both in a scratch header)
        for (int n = 0; n < ff.ntr; ++n) {
            fa.htr[n] = cg.htr[n];
            fa.htr_in[n] = cg.htr_in[n];
        }
        if (fs.by == 1) {
            switch (fs.nt) {
                case 4: return launch_fold_t<4, P, 1>(fa, r.j0, r.j1, st);
                case 2: return launch_fold_t<2, P, 1>(fa, r.j0, r.j1, st);
                default: return launch_fold_t<1, P, 1>(fa, r.j0, r.j1, st);
            }
        }
        switch (fs.nt) {
            case 4: return launch_fold_t<4, P, 2>(fa, r.j0, r.j1, st);
            case 2: return launch_fold_t<2, P, 2>(fa, r.j0, r.j1, st);
            default: return launch_fold_t<1, P, 2>(fa, r.j0, r.j1, st);
        }
    }
    // Reconstruct in groups of two tracers (register window of 2 scalars).
    if (r.c1 > r.c0 && rc.ntr > 0) {
        launch_recon<P>(rc, r, st);
    }
    const CellTuning tune = cell_tuning();
    const int group = flux_group(ff.ntr, tune);
    if (gather_spans_two(ff.ntr, tune)) {
        // two face-flux launches of 4 tracers (slots 0-3 and 4-7), one gather of 8
        for (int tr0 = 0; tr0 < ff.ntr; tr0 += 8) {
            launch_flux<4, P>(ff, tr0, r, tune, st);
            if (tr0 + 4 < ff.ntr) {
                FaceFluxArgsT<P> f2 = ff;
                f2.fslot0 = 4;
                launch_flux<4, P>(f2, tr0 + 4, r, tune, st);
            }
            launch_gathers<8, P, true>(cg, tr0, r, tune, st);
        }
        return cudaGetLastError();
    }
    for (int tr0 = 0; tr0 < ff.ntr; tr0 += group) {
        switch (group) {
            case 8: launch_flux<8, P>(ff, tr0, r, tune, st); launch_gathers<8, P>(cg, tr0, r, tune, st); break;
            case 4: launch_flux<4, P>(ff, tr0, r, tune, st); launch_gathers<4, P>(cg, tr0, r, tune, st); break;
            case 2: launch_flux<2, P>(ff, tr0, r, tune, st); launch_gathers<2, P>(cg, tr0, r, tune, st); break;
            default: launch_flux<1, P>(ff, tr0, r, tune, st); launch_gathers<1, P>(cg, tr0, r, tune, st); break;
        }
    }
    return cudaGetLastError();
}

template cudaError_t launch_sweep<PlainPrec>(const SweepArgsT<PlainPrec>&, cudaStream_t, Band);
template cudaError_t launch_sweep<MixedPrec>(const SweepArgsT<MixedPrec>&, cudaStream_t, Band);
template cudaError_t launch_phase_b<PlainPrec>(const ReconArgsT<PlainPrec>&, const FaceFluxArgsT<PlainPrec>&,
                                               const CellGatherArgsT<PlainPrec>&, cudaStream_t, Band, int);
template FoldShape fold_shape<PlainPrec>(int, int);
template FoldShape fold_shape<MixedPrec>(int, int);
template cudaError_t launch_phase_b<MixedPrec>(const ReconArgsT<MixedPrec>&, const FaceFluxArgsT<MixedPrec>&,
                                               const CellGatherArgsT<MixedPrec>&, cudaStream_t, Band, int);

}  // namespace redi
