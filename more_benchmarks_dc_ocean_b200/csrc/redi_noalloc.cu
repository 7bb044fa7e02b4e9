// A Redi step that allocates no device memory.
//
// Who needs it: a caller that must not call cudaMalloc or cudaFree while it
// steps the model. cudaFree (and cudaMalloc when the pool has to grow) can
// synchronise the whole device, which stalls every other stream of the
// process; neither may run while a stream is being captured into a CUDA graph;
// and some host models own all device memory through their own pool (an
// OpenACC runtime, a framework allocator) and forbid raw allocations after
// start-up. The regular entry points grow a scratch buffer with cudaMalloc on
// first use, which such callers cannot accept.
//
// How: all scratch of the step lives in one fixed array in the library's own
// device memory (kScratchBytes below). Every GPU that loads the library holds
// that array until the process exits. Its device address is looked up once per
// device, on the first call made on that device (cudaGetSymbolAddress); make
// that first call before any stream capture. A step whose scratch would not fit
// is refused with REDI_B200_E_UNSUPPORTED and the size limit in the message.
//
// All calls share the one array, so calls that overlap on the GPU (on
// different streams or from different host threads without ordering) race on
// it and corrupt each other's results; issue them in stream order. The array
// keeps the last call's contents; the only part that must start at zero, the
// error words, is cleared on the caller's stream by every call. (The words
// count coefficients found out of order; this entry point makes its own
// coefficients in Phase A, where that never happens, so it reports none.)
//
// The address is cached per device index for the life of the process: after
// cudaDeviceReset the module is loaded again at a new address, so do not reset
// a device that this library has stepped on and then call it again.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/redi_b200.h"
#include "redi_kernels.h"

namespace {

// 64 MiB: room for a domain of about 18 000 columns at nz = 25, 6 000 at
// nz = 75 (Phase A needs 40 B per interface; Phase B 2 x (8 B per interface +
// 32 B per layer) of reconstructions plus 2 x 8 B per face and sublayer of
// fluxes; the two phases reuse the same bytes).
constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr size_t kHeader = 256;  // error word
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

int set_error(int code, const std::string& msg) {
    redi::set_last_error("redi_b200_opt_launch_noalloc: " + msg);
    return code;
}

// Per-device set-up: the device address of the scratch array.
int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(REDI_B200_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(REDI_B200_E_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(REDI_B200_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return REDI_B200_OK;
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int redi_b200_opt_launch_noalloc(const int* nx_, const int* ny_, const int* nz_, const int* ns_, const double* dt_,
                                 const int* nghost_, const int* nxp_, const int* nyp_, const int* ww_,
                                 const int* we_, const int* wsz_, const int* wn_, const double* rho0_,
                                 const double* T_ref_, const double* S_ref_, const double* alpha_T_,
                                 const double* beta_S_, const double* h_layer, double* t_htr, double* s_htr,
                                 const double* wet_u, const double* wet_v, double* uPoL, double* uPoR, int* uKoL,
                                 int* uKoR, double* uhEff, double* vPoL, double* vPoR, int* vKoL, int* vKoR,
                                 double* vhEff, const double* khtr_u_ext, const double* khtr_v_ext, double* khtr_u,
                                 double* khtr_v, const double* dy_cu, const double* dx_cv, const double* idxCu,
                                 const double* idyCv, const double* areaT, double* tr_snap, void* stream) {
    (void)tr_snap;
    redi::set_last_error("");
    const void* scalars[] = {nx_, ny_, nz_, ns_, dt_, nghost_, nxp_, nyp_, ww_, we_, wsz_, wn_,
                             rho0_, T_ref_, S_ref_, alpha_T_, beta_S_};
    for (const void* p : scalars)
        if (!p) return set_error(REDI_B200_E_ARG, "NULL scalar argument");
    // the same checks as redi_opt_launch: doubles 8-byte aligned, the int Ko slots 4-byte aligned
    const void* reals[] = {h_layer, t_htr, s_htr, wet_u, wet_v, uPoL, uPoR, uhEff, vPoL, vPoR, vhEff,
                           khtr_u_ext, khtr_v_ext, khtr_u, khtr_v, dy_cu, dx_cv, idxCu, idyCv, areaT};
    for (const void* p : reals)
        if (!p || (reinterpret_cast<uintptr_t>(p) % alignof(double)) != 0)
            return set_error(REDI_B200_E_ARG, "NULL or misaligned array");
    const void* ints[] = {uKoL, uKoR, vKoL, vKoR};
    for (const void* p : ints)
        if (!p || (reinterpret_cast<uintptr_t>(p) % alignof(int)) != 0)
            return set_error(REDI_B200_E_ARG, "NULL or misaligned array");
    const int nx = *nx_, ny = *ny_, nz = *nz_, ns = *ns_;
    if (nx < 1 || ny < 1 || nz < 1 || nz > redi::kNzMax) return set_error(REDI_B200_E_ARG, "invalid domain extents");
    if (ns != 2 * nz + 2) return set_error(REDI_B200_E_ARG, "ns must equal 2*nz+2");

    // Scratch of each phase, laid out from the start of the array (after the header).
    const size_t ncol = (size_t)nx * ny;
    const size_t ifc_b = round256(ncol * (nz + 1) * sizeof(redi::IfcState));
    const size_t pint_b = round256(ncol * (nz + 1) * sizeof(double));
    const size_t ti_b = round256(2 * ncol * (nz + 1) * sizeof(double));
    const size_t ppm_b = round256(2 * ncol * nz * sizeof(redi::PpmLayer));
    const size_t fu_b = round256((size_t)2 * (2 * nz + 1) * (size_t)(nx + 1) * ny * sizeof(double));
    const size_t fv_b = round256((size_t)2 * (2 * nz + 1) * (size_t)nx * (ny + 1) * sizeof(double));
    const size_t need_a = ifc_b + pint_b, need_b = ti_b + ppm_b + fu_b + fv_b;
    // the sweep's dry-face record lives behind both phases' scratch (it is
    // written in Phase A and read in Phase B)
    const size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1);
    const size_t dry_off = need_a > need_b ? need_a : need_b;
    const size_t need = dry_off + round256(nu + nv);
    if (need > kScratchBytes - kHeader)
        return set_error(REDI_B200_E_UNSUPPORTED,
                         "domain needs " + std::to_string(need) + " bytes of scratch; this entry point is limited to " +
                             std::to_string(kScratchBytes - kHeader) +
                             " bytes (use redi_opt_launch or the handle API for larger domains)");
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc < 0) return rc;
    char* data = static_cast<char*>(base) + kHeader;
    int* err = static_cast<int*>(base);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(err, 0, 2 * sizeof(int), st);

    // Phase A (redi_calc_coeffs).
    redi::EosParams eos{1, *rho0_, *T_ref_, *S_ref_, *alpha_T_, *beta_S_};  // the launcher's LINEAR EOS
    redi::ColumnStateArgs cs{};
    cs.nx = nx; cs.ny = ny; cs.nz = nz; cs.eos = eos; cs.h = h_layer; cs.th = t_htr; cs.sh = s_htr;
    cs.ifc = reinterpret_cast<redi::IfcState*>(data);
    cs.pint = reinterpret_cast<double*>(data + ifc_b);
    cs.wet_u = wet_u; cs.wet_v = wet_v;
    redi::SweepArgs sw{};
    sw.nx = nx; sw.ny = ny; sw.nz = nz; sw.rho0 = eos.rho0; sw.wet_u = wet_u; sw.wet_v = wet_v;
    sw.ifc = cs.ifc; sw.pint = cs.pint;
    uint8_t* udry = reinterpret_cast<uint8_t*>(data + dry_off);
    uint8_t* vdry = udry + nu;
    sw.u = redi::FaceOut{uPoL, uPoR, uKoL, uKoR, uhEff, udry};
    sw.v = redi::FaceOut{vPoL, vPoR, vKoL, vKoR, vhEff, vdry};
    if (e == cudaSuccess) e = redi::launch_column_state(cs, st);
    if (e == cudaSuccess) e = redi::launch_sweep<redi::PlainPrec>(sw, st);
    // Per-face diffusivities resolved into the caller's slots (redi_face_copy).
    if (e == cudaSuccess) e = cudaMemcpyAsync(khtr_u, khtr_u_ext, (size_t)(nx + 1) * ny * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(khtr_v, khtr_v_ext, (size_t)nx * (ny + 1) * 8, cudaMemcpyDeviceToDevice, st);

    // Phase B (redi_apply_flux) for T and S.
    redi::ReconArgs r{};
    r.nx = nx; r.ny = ny; r.nz = nz; r.ntr = 2; r.h = h_layer;
    r.ti = reinterpret_cast<double*>(data);
    r.ppm = reinterpret_cast<redi::PpmLayer*>(data + ti_b);
    r.dry_u = udry; r.dry_v = vdry;
    r.htr[0] = t_htr;
    r.htr[1] = s_htr;
    redi::FaceFluxArgs ff{};
    ff.nx = nx; ff.ny = ny; ff.nz = nz; ff.ntr = 2;
    ff.nghost = *nghost_; ff.nxp = *nxp_; ff.nyp = *nyp_;
    ff.wall_w = *ww_; ff.wall_e = *we_; ff.wall_s = *wsz_; ff.wall_n = *wn_;
    ff.dt = *dt_; ff.khtr = 0.0; ff.khtr_u = khtr_u; ff.khtr_v = khtr_v;
    ff.dy_cu = dy_cu; ff.dx_cv = dx_cv; ff.idxCu = idxCu; ff.idyCv = idyCv;
    ff.u = redi::FaceIn{uPoL, uPoR, uKoL, uKoR, uhEff, udry};
    ff.v = redi::FaceIn{vPoL, vPoR, vKoL, vKoR, vhEff, vdry};
    ff.ti = r.ti; ff.ppm = r.ppm;
    ff.Fu = reinterpret_cast<double*>(data + ti_b + ppm_b);
    ff.Fv = reinterpret_cast<double*>(data + ti_b + ppm_b + fu_b);
    redi::CellGatherArgs cg{};
    cg.nx = nx; cg.ny = ny; cg.nz = nz; cg.ntr = 2;
    cg.nghost = ff.nghost; cg.nxp = ff.nxp; cg.nyp = ff.nyp;
    cg.wall_w = ff.wall_w; cg.wall_e = ff.wall_e; cg.wall_s = ff.wall_s; cg.wall_n = ff.wall_n;
    cg.areaT = areaT; cg.u = ff.u; cg.v = ff.v; cg.Fu = ff.Fu; cg.Fv = ff.Fv; cg.err = err;
    cg.htr[0] = t_htr;
    cg.htr[1] = s_htr;
    cg.htr_in[0] = t_htr;
    cg.htr_in[1] = s_htr;
    if (e == cudaSuccess) e = redi::launch_phase_b<redi::PlainPrec>(r, ff, cg, st);
    if (e != cudaSuccess) return set_error(REDI_B200_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return REDI_B200_OK;
}

}  // extern "C"
