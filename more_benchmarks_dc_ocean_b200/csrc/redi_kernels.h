// Internal launch interface of the Redi kernels (not part of the public C-ABI).
#pragma once

#include <cuda_runtime.h>

#include "redi_device.cuh"

namespace redi {

constexpr int kNzMax = 128;       // layers per column supported by the FP64 kernels
constexpr int kMaxTracers = 64;   // tracers per fused launch (larger sets are split)
constexpr int kCellGroup = 2;     // tracers accumulated together per cell thread

struct FaceOut {
    double* PoL;
    double* PoR;
    int* KoL;
    int* KoR;
    double* hEff;
};

struct FaceIn {
    const double* PoL;
    const double* PoR;
    const int* KoL;
    const int* KoR;
    const double* hEff;
};

struct ColumnStateArgs {
    int nx, ny, nz;
    EosLin eos;
    const double* h;
    const double* th;
    const double* sh;
    IfcState* ifc;   // [nz+1][column]
    double* pint;    // [nz+1][column]
};

struct SweepArgs {
    int nx, ny, nz;
    double rho0;
    const double* wet_u;
    const double* wet_v;
    const IfcState* ifc;
    const double* pint;
    FaceOut u, v;
};

struct ReconArgs {
    int nx, ny, nz, ntr;
    const double* h;
    const double* htr[kMaxTracers];
    double* ti;      // [tracer][nz+1][column]
    PpmLayer* ppm;   // [tracer][nz][column]
};

struct FaceFluxArgs {
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
    FaceIn u, v;
    const double* ti;       // [tracer][nz+1][column]
    const PpmLayer* ppm;    // [tracer][nz][column]
    double* Fu;             // [group tracer][ns-1][(nx+1)*ny]
    double* Fv;             // [group tracer][ns-1][nx*(ny+1)]
};

struct CellGatherArgs {
    int nx, ny, nz, ntr;
    int nghost, nxp, nyp;
    int wall_w, wall_e, wall_s, wall_n;
    const double* areaT;
    FaceIn u, v;            // only KoL / KoR are read
    const double* Fu;
    const double* Fv;
    double* htr[kMaxTracers];
    int* err;               // device error word (fluxes out of order), may be null
};

// Scratch bytes each phase needs for an (nx, ny, nz) domain with ntr tracers.
inline size_t plain_phase_a_scratch(int nx, int ny, int nz) {
    const size_t nifc = (size_t)nx * ny * (nz + 1);
    return nifc * sizeof(IfcState) + nifc * sizeof(double);
}
inline size_t plain_recon_bytes(int nx, int ny, int nz, int ntr) {
    const size_t ncol = (size_t)nx * ny;
    return (size_t)ntr * ncol * ((nz + 1) * sizeof(double) + nz * sizeof(PpmLayer));
}
inline size_t plain_flux_bytes(int nx, int ny, int nz, int group) {
    const size_t faces = (size_t)(nx + 1) * ny + (size_t)nx * (ny + 1);
    return (size_t)group * (size_t)(2 * nz + 1) * faces * sizeof(double);
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
    K_NUM = 10
};

// Launch bracketing: counts every kernel launch of the library and, while
// timing is switched on (redi_b200_profile_begin), records a CUDA event pair
// around it on the launching stream.
void launch_begin(int kid, cudaStream_t st);
void launch_end(int kid, cudaStream_t st);

// Launch shape of the FP64 cell update: a bx x by tile of columns per block
// (bx * by <= 128) and the vertical chunk (layers per pass, 4, 8 or 16).
struct CellTuning {
    int bx, by, chunk;
};
CellTuning cell_tuning();
void set_cell_tuning(const CellTuning& t);

cudaError_t launch_plain_phase_a(const ColumnStateArgs& cs, const SweepArgs& sw, cudaStream_t st);
cudaError_t launch_plain_phase_b(const ReconArgs& rc, const FaceFluxArgs& ff, const CellGatherArgs& cg,
                                 cudaStream_t st);

}  // namespace redi
