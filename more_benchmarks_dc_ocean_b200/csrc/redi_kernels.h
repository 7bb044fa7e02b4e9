// Internal launch interface of the Redi kernels (not part of the public C-ABI).
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "redi_device.cuh"

namespace redi {

constexpr int kNzMax = 1024;      // layers per column accepted by the kernels
constexpr int kMaxTracers = 64;   // tracers per fused launch (larger sets are split)

// ---------------------------------------------------------------------------
// Precision policies.
//
// Plain: the reference's FP64 everywhere, coefficients in the reference layout
// and types (bit-identical results).
// Mixed: every quantity that feeds a discrete decision of the algorithm (the
// sweep's density differences, interpolation denominators and positions; the
// tracer values at neutral surfaces whose signs the down-gradient guard tests)
// stays FP64 and is computed exactly as in the plain form; the PPM layer means
// (redi_ppm_ave), the flux product and their storage are FP32; Ko is stored as
// int16 and hEff as FP32; the flux divergence accumulates in FP64.
// ---------------------------------------------------------------------------
struct alignas(16) PpmLayerF {
    float aL, dA, a6o3, B;
};

struct PlainPrec {
    using Po = double;
    using Ko = int;
    using He = double;
    using Ppm = PpmLayer;
    using Flux = double;
    static constexpr bool kMixed = false;
};

struct MixedPrec {
    using Po = double;
    using Ko = int16_t;
    using He = float;
    using Ppm = PpmLayerF;
    using Flux = float;
    static constexpr bool kMixed = true;
};

template <class P>
struct FaceOutT {
    typename P::Po* PoL;
    typename P::Po* PoR;
    typename P::Ko* KoL;
    typename P::Ko* KoR;
    typename P::He* hEff;
    // per face: 1 where the sweep wrote inert coefficients (a dry face: every
    // flux is +0.0), else 0; may be null (not recorded)
    uint8_t* dry = nullptr;
    // the slots are the library's own, and a face recorded dry still holds its
    // inert coefficients: a face that stays dry is not written again
    bool keep = false;
};

template <class P>
struct FaceInT {
    const typename P::Po* PoL;
    const typename P::Po* PoR;
    const typename P::Ko* KoL;
    const typename P::Ko* KoR;
    const typename P::He* hEff;
    // the sweep's dry-face record (may be null): the face flux stores nothing
    // for a dry face and the gather skips it, which adds exactly the +0.0
    // fluxes the face would have had
    const uint8_t* dry = nullptr;
};

using FaceOut = FaceOutT<PlainPrec>;
using FaceIn = FaceInT<PlainPrec>;

struct ColumnStateArgs {
    int nx, ny, nz;
    EosParams eos;
    const double* h;
    const double* th;
    const double* sh;
    IfcState* ifc;   // [nz+1][column]
    double* pint;    // [nz+1][column]
    // the sweep's face masks (may be null): a column none of whose sweep faces
    // is wet is never read by the sweep, and is not computed
    const double* wet_u = nullptr;
    const double* wet_v = nullptr;
};

template <class P>
struct SweepArgsT {
    int nx, ny, nz;
    double rho0;
    const double* wet_u;
    const double* wet_v;
    const IfcState* ifc;
    const double* pint;
    FaceOutT<P> u, v;
};
using SweepArgs = SweepArgsT<PlainPrec>;

template <class P>
struct ReconArgsT {
    int nx, ny, nz, ntr;
    const double* h;
    const double* htr[kMaxTracers];
    double* ti;               // [tracer][nz+1][column]
    typename P::Ppm* ppm;     // [tracer][nz][column]
    // the sweep's dry-face record (may be null): a column all of whose faces
    // are dry is never read by the face flux, and is not reconstructed
    const uint8_t* dry_u = nullptr;
    const uint8_t* dry_v = nullptr;
};
using ReconArgs = ReconArgsT<PlainPrec>;

template <class P>
struct FaceFluxArgsT {
    int nx, ny, nz, ntr;
    int nghost, nxp, nyp;
    int wall_w, wall_e, wall_s, wall_n;
    double dt;
    double khtr;            // used where khtr_u / khtr_v is null (scalar path)
    const double* khtr_u;   // (nx+1, ny) or null
    const double* khtr_v;   // (nx, ny+1) or null
    const double* dy_cu;
    const double* dx_cv;
    const double* idxCu;
    const double* idyCv;
    FaceInT<P> u, v;
    const double* ti;                 // [tracer][nz+1][column]
    const typename P::Ppm* ppm;       // [tracer][nz][column]
    typename P::Flux* Fu;             // [slot][ns-1][(nx+1)*ny]
    typename P::Flux* Fv;             // [slot][ns-1][nx*(ny+1)]
    int fslot0 = 0;                   // slot of the launch's first tracer
};
using FaceFluxArgs = FaceFluxArgsT<PlainPrec>;

template <class P>
struct CellGatherArgsT {
    int nx, ny, nz, ntr;
    int nghost, nxp, nyp;
    int wall_w, wall_e, wall_s, wall_n;
    const double* areaT;
    FaceInT<P> u, v;                  // only KoL / KoR are read
    const typename P::Flux* Fu;
    const typename P::Flux* Fv;
    double* htr[kMaxTracers];         // updated tracers
    const double* htr_in[kMaxTracers];  // pre-step tracers (the same arrays for an in-place update)
    int* err;                         // device error word (fluxes out of order), may be null
};
using CellGatherArgs = CellGatherArgsT<PlainPrec>;

// Scratch bytes each phase needs for an (nx, ny, nz) domain.
inline size_t phase_a_scratch(int nx, int ny, int nz) {
    const size_t nifc = (size_t)nx * ny * (nz + 1);
    return nifc * sizeof(IfcState) + nifc * sizeof(double);
}
// Byte offset of the PPM layers behind the interface values in a Phase-B
// reconstruction buffer; 256-byte aligned, the layers are read as 16-byte vectors.
inline size_t recon_ppm_offset(int nx, int ny, int nz, int ntr) {
    return ((size_t)ntr * nx * ny * (nz + 1) * sizeof(double) + 255) & ~size_t(255);
}
template <class P>
inline size_t recon_bytes(int nx, int ny, int nz, int ntr) {
    return recon_ppm_offset(nx, ny, nz, ntr) + (size_t)ntr * nx * ny * nz * sizeof(typename P::Ppm);
}
template <class P>
inline size_t flux_bytes(int nx, int ny, int nz, int group) {
    const size_t faces = (size_t)(nx + 1) * ny + (size_t)nx * (ny + 1);
    return (size_t)group * (size_t)(2 * nz + 1) * faces * sizeof(typename P::Flux);
}
// Tracers per face-flux launch for a set of ntr tracers, at most cap (1, 2,
// 4 or 8): a larger group reads the coefficients fewer times, a smaller one
// needs fewer registers.
inline int tracer_group(int ntr, int cap = 8) {
    const int g = ntr >= 8 ? 8 : ntr >= 4 ? 4 : ntr >= 2 ? 2 : 1;
    return g < cap ? g : cap;
}

// Kernel identities for the launch counter and the optional event timing.
enum KernelId : int {
    K_COLUMN_STATE = 0,
    K_NEUTRAL_SWEEP = 1,
    K_TRACER_RECON = 2,
    K_CELL_UPDATE = 3,   // the per-cell gather
    K_FACE_FLUX = 4,
    K_MIXED_RECON = 5,
    K_MIXED_FLUX = 6,
    K_MIXED_SWEEP = 7,
    K_DOMAIN_PERSISTENT = 8,
    K_AUX = 9,
    K_MEKE_COLUMN = 10,   // MEKE pass A
    K_MEKE_DEL2 = 11,     // MEKE biharmonic Laplacian
    K_MEKE_LATERAL = 12,  // MEKE pass B
    K_ALE_COLUMNS = 13,   // ALE remap: targets, snapshot, tracers and the commit
    K_ALE_FACES = 14,     // ALE remap: face velocities
    K_FLUX_FOLD = 15,     // Phase B fused face flux + fold (FP64)
    K_MIXED_FOLD = 16,    // Phase B fused face flux + fold (mixed)
    K_COLUMN_RECON = 17,  // column state + T/S reconstruction in one pass (whole-step call)
    K_NUM = 18
};

// Sets the message redi_b200_last_error() returns on the calling thread.
void set_last_error(const std::string& msg);

// Launch bracketing: counts every kernel launch of the library and, while
// timing is switched on (redi_b200_profile_begin), records a CUDA event pair
// around it on the launching stream.
void launch_begin(int kid, cudaStream_t st);
void launch_end(int kid, cudaStream_t st);
// Adds n launches of kernel kid to the counter without timing them (CUDA graph
// replays, whose launches happen inside the graph).
void count_launches(int kid, unsigned long long n);

// Launch shape of Phase B: the cell gather's bx x by tile of columns per
// block (bx * by <= 128) and vertical chunk (layers per pass, 4, 8 or 16),
// the largest tracer group of one face-flux launch (1, 2, 4 or 8) and the
// tracers one gather launch folds (2 or 4).
struct CellTuning {
    int bx, by, chunk, group;
    int gather_tracers = 2;
    int gather_smem = 0;  // per-layer sums in shared memory (128-thread tiles) instead of registers
    int flux_staged = 0;  // face flux with its reconstruction loads staged one sublayer ahead (groups <= 2)
    int gather_batch = 0;  // shared-memory gather: sublayers per round trip (8, or 0: 3 / 4 by chunk)
    int sweep_form = 4;    // neutral sweep: 0 register windows, 3 / 4 / 5 windows in a shared-memory ring of that size
    int gather_pipe = 0;   // shared-memory gather: batches of 4 software-pipelined (the next one in flight)
};
CellTuning cell_tuning();
void set_cell_tuning(const CellTuning& t);

// Tracers per face-flux launch for ntr tracers under tuning t (the staged
// face flux holds at most 2 tracers in shared memory, the ring form 4).
inline int flux_group(int ntr, const CellTuning& t) {
    const int cap = t.flux_staged == 1 ? 2 : (t.flux_staged == 2 ? 4 : 8);
    return tracer_group(ntr, t.group < cap ? t.group : cap);
}
// Whether one gather folds the fluxes of two face-flux launches of 4 tracers
// (8 tracers per gather: the shared-memory gather with 4-layer chunks).
inline bool gather_spans_two(int ntr, const CellTuning& t) {
    return t.gather_tracers >= 8 && flux_group(ntr, t) == 4 && ntr > 4 && t.gather_smem && t.chunk == 4 &&
           t.bx * t.by == 128;
}
// Slots of the flux buffer Phase B needs for ntr tracers.
inline int flux_slots(int ntr, const CellTuning& t) { return gather_spans_two(ntr, t) ? 8 : flux_group(ntr, t); }

// Phase B as one fused face-flux + fold pass (redi_fold.cuh) instead of the
// face-flux / cell-gather pair: enable, tile rows (1 or 2) and tracers per
// pass (1, 2, 4; 0 picks the most that keep two blocks per SM), per form
// (plain FP64, mixed); ordered_mixed: the mixed form folds in the reference's
// order too (otherwise in any order, through shared-memory atomics).
struct FoldTuning {
    int enable, rows, tracers;
    int enable_mixed, ordered_mixed;
};
FoldTuning fold_tuning();
void set_fold_tuning(const FoldTuning& t);
// Tile rows and tracers per pass of the fused pass for a problem; nt == 0:
// it is off or its shared memory does not fit, and the pair runs.
struct FoldShape {
    int nt, by;
};
template <class P>
FoldShape fold_shape(int nz, int ntr);

// A band of T-cell rows [row0, row1) of the domain (row1 < 0: to the last
// row). A step restricted to a band touches the u faces of its rows, the v
// faces between rows row0-1 .. row1 and the columns of rows row0-1 .. row1:
// everything the band's cells need, and bands can be stepped one after
// another with identical results when the tracers are read from pre-step
// copies (CellGatherArgsT::htr_in).
struct Band {
    int row0 = 0, row1 = -1;
};

cudaError_t launch_column_state(const ColumnStateArgs& cs, cudaStream_t st, Band band = Band{});
// The column state and the reconstruction of rc's tracers 0 and 1 (T and S,
// or S and T when ts_swap) in one pass over every column.
template <class P>
cudaError_t launch_column_recon(const ColumnStateArgs& cs, const ReconArgsT<P>& rc, int ts_swap, cudaStream_t st);
// Density and dSV/dT, dSV/dS at n points (T, S, p device arrays).
cudaError_t launch_eos_points(const EosParams& e, int n, const double* T, const double* S, const double* p,
                              double* rho, double* dsv_dt, double* dsv_ds, cudaStream_t st);
template <class P>
cudaError_t launch_sweep(const SweepArgsT<P>& sw, cudaStream_t st, Band band = Band{});
template <class P>
// recon_from: the first tracer of rc to reconstruct (tracers before it were
// reconstructed already, by launch_column_recon).
cudaError_t launch_phase_b(const ReconArgsT<P>& rc, const FaceFluxArgsT<P>& ff, const CellGatherArgsT<P>& cg,
                           cudaStream_t st, Band band = Band{}, int recon_from = 0);

}  // namespace redi
