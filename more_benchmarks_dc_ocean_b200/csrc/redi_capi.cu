// C-ABI of the B200 Redi step (include/redi_b200.h): the ocean_redi_t handle,
// the reference's gates and argument checks, scratch management and the
// reference-compatible launcher exports.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/redi_b200.h"
#include "redi_kernels.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(REDI_B200_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
bool aligned(const T* p) {
    return (reinterpret_cast<uintptr_t>(p) % alignof(T)) == 0;
}

__global__ void k_fill(double* p, size_t n, double v) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < n) p[t] = v;
}
__global__ void k_fill_int(int* p, size_t n, int v) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < n) p[t] = v;
}

cudaError_t fill(double* p, size_t n, double v, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_fill<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}
cudaError_t fill_int(int* p, size_t n, int v, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_fill_int<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}
__global__ void k_fill_short(int16_t* p, size_t n, int16_t v) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < n) p[t] = v;
}
cudaError_t fill_short(int16_t* p, size_t n, int16_t v, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_fill_short<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

// Grow-only device scratch. The first 256 bytes hold the device error word
// (count of out-of-order coefficient sublayers seen by the cell update); phase
// data starts at data().
struct Scratch {
    static constexpr size_t kHeader = 256;
    void* ptr = nullptr;
    size_t bytes = 0;
    int device = -1;
    cudaError_t reserve(size_t need) {
        need += kHeader;
        if (need <= bytes) return cudaSuccess;
        int err_keep = 0;
        if (ptr) {
            cudaMemcpy(&err_keep, ptr, sizeof(int), cudaMemcpyDeviceToHost);
            cudaError_t e = cudaFree(ptr);
            ptr = nullptr;
            bytes = 0;
            if (e != cudaSuccess) return e;
        }
        cudaError_t e = cudaMalloc(&ptr, need);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return e;
        }
        bytes = need;
        return cudaMemcpy(ptr, &err_keep, sizeof(int), cudaMemcpyHostToDevice);
    }
    void* data() const { return static_cast<char*>(ptr) + kHeader; }
    int* err() const { return static_cast<int*>(ptr); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

bool dims_ok(int nx, int ny, int nz, std::string& why) {
    if (nx < 1 || ny < 1) { why = "nx_total and ny_total must be >= 1"; return false; }
    if (nz < 1) { why = "nz must be >= 1"; return false; }
    if (nz > redi::kNzMax) {
        why = "nz = " + std::to_string(nz) + " exceeds the supported maximum of " + std::to_string(redi::kNzMax) +
              " layers (the reference's init stops for 2*nz+2 > NZ_STACK_MAX in the same way)";
        return false;
    }
    const long long ns = 2LL * nz + 2;
    if ((long long)(nx + 1) * (ny + 1) * ns >= (1LL << 31)) { why = "domain too large for 32-bit face indexing"; return false; }
    return true;
}

// Phase A into caller-provided or handle-owned coefficient slots.
template <class P>
int run_phase_a(int nx, int ny, int nz, const redi::EosParams& eos, const double* h, const double* th,
                const double* sh, const double* wet_u, const double* wet_v, const redi::FaceOutT<P>& u,
                const redi::FaceOutT<P>& v, Scratch& ws, cudaStream_t st, redi::Band band = redi::Band{}) {
    cudaError_t e = ws.reserve(redi::phase_a_scratch(nx, ny, nz));
    if (e != cudaSuccess) return cuda_fail(e, "scratch allocation (phase A)");
    const size_t nifc = (size_t)nx * ny * (nz + 1);
    redi::ColumnStateArgs cs{};
    cs.nx = nx; cs.ny = ny; cs.nz = nz; cs.eos = eos;
    cs.h = h; cs.th = th; cs.sh = sh;
    cs.ifc = reinterpret_cast<redi::IfcState*>(ws.data());
    cs.pint = reinterpret_cast<double*>(cs.ifc + nifc);
    cs.wet_u = wet_u; cs.wet_v = wet_v;
    redi::SweepArgsT<P> sw{};
    sw.nx = nx; sw.ny = ny; sw.nz = nz; sw.rho0 = eos.rho0;
    sw.wet_u = wet_u; sw.wet_v = wet_v; sw.ifc = cs.ifc; sw.pint = cs.pint;
    sw.u = u; sw.v = v;
    e = redi::launch_column_state(cs, st, band);
    if (e == cudaSuccess) e = redi::launch_sweep<P>(sw, st, band);
    if (e != cudaSuccess) return cuda_fail(e, "phase A launch");
    return REDI_B200_OK;
}

template <class P>
struct PhaseBInputs {
    int nx, ny, nz, nghost, nxp, nyp;
    int walls[4];
    double dt, khtr;
    const double *khtr_u, *khtr_v, *dy_cu, *dx_cv, *idxCu, *idyCv, *areaT, *h;
    redi::FaceInT<P> u, v;
};

// htr_in (may be null: in place) holds the pre-step tracers, htr receives the
// updated ones; band restricts the launches to a band of rows.
template <class P>
int run_phase_b(const PhaseBInputs<P>& in, int ntr, double* const* htr, Scratch& ws, cudaStream_t st,
                const double* const* htr_in = nullptr, redi::Band band = redi::Band{}, int recon_from = 0) {
    const int batch = ntr < redi::kMaxTracers ? ntr : redi::kMaxTracers;
    const size_t recon = redi::recon_bytes<P>(in.nx, in.ny, in.nz, batch);
    const int group = redi::flux_slots(batch, redi::cell_tuning());
    const size_t flux = redi::flux_bytes<P>(in.nx, in.ny, in.nz, group);
    cudaError_t e = ws.reserve(recon + flux);
    if (e != cudaSuccess) return cuda_fail(e, "scratch allocation (phase B)");
    const size_t ns1 = (size_t)(2 * in.nz + 1);
    using Flux = typename P::Flux;
    Flux* Fu = reinterpret_cast<Flux*>(static_cast<char*>(ws.data()) + recon);
    Flux* Fv = Fu + (size_t)group * ns1 * (size_t)(in.nx + 1) * in.ny;
    for (int t0 = 0; t0 < ntr; t0 += batch) {
        const int nt = (ntr - t0) < batch ? (ntr - t0) : batch;
        redi::ReconArgsT<P> rc{};
        rc.nx = in.nx; rc.ny = in.ny; rc.nz = in.nz; rc.ntr = nt; rc.h = in.h;
        rc.ti = reinterpret_cast<double*>(ws.data());
        rc.ppm = reinterpret_cast<typename P::Ppm*>(static_cast<char*>(ws.data()) +
                                                    redi::recon_ppm_offset(in.nx, in.ny, in.nz, nt));
        rc.dry_u = in.u.dry; rc.dry_v = in.v.dry;
        redi::FaceFluxArgsT<P> ff{};
        ff.nx = in.nx; ff.ny = in.ny; ff.nz = in.nz; ff.ntr = nt;
        ff.nghost = in.nghost; ff.nxp = in.nxp; ff.nyp = in.nyp;
        ff.wall_w = in.walls[0]; ff.wall_e = in.walls[1]; ff.wall_s = in.walls[2]; ff.wall_n = in.walls[3];
        ff.dt = in.dt; ff.khtr = in.khtr; ff.khtr_u = in.khtr_u; ff.khtr_v = in.khtr_v;
        ff.dy_cu = in.dy_cu; ff.dx_cv = in.dx_cv; ff.idxCu = in.idxCu; ff.idyCv = in.idyCv;
        ff.u = in.u; ff.v = in.v; ff.ti = rc.ti; ff.ppm = rc.ppm; ff.Fu = Fu; ff.Fv = Fv;
        redi::CellGatherArgsT<P> cg{};
        cg.nx = in.nx; cg.ny = in.ny; cg.nz = in.nz; cg.ntr = nt;
        cg.nghost = in.nghost; cg.nxp = in.nxp; cg.nyp = in.nyp;
        cg.wall_w = in.walls[0]; cg.wall_e = in.walls[1]; cg.wall_s = in.walls[2]; cg.wall_n = in.walls[3];
        cg.areaT = in.areaT; cg.u = in.u; cg.v = in.v; cg.Fu = Fu; cg.Fv = Fv; cg.err = ws.err();
        for (int n = 0; n < nt; ++n) {
            rc.htr[n] = htr_in ? htr_in[t0 + n] : htr[t0 + n];
            cg.htr[n] = htr[t0 + n];
            cg.htr_in[n] = htr_in ? htr_in[t0 + n] : htr[t0 + n];
        }
        e = redi::launch_phase_b<P>(rc, ff, cg, st, band, t0 == 0 ? recon_from : 0);
        if (e != cudaSuccess) return cuda_fail(e, "phase B launch");
    }
    return REDI_B200_OK;
}

// Device side of the host-state step: h and the tracers' pre-step and updated
// copies (the gather reads one and writes the other, so bands can be stepped
// one after another while their rows stream in and out), and the three
// streams of the pipeline. Grow-only; released with the handle.
struct HostPipeline {
    double* h = nullptr;
    std::vector<double*> tin, tout;
    size_t ncell = 0;
    cudaStream_t up = nullptr, comp = nullptr, down = nullptr;
    std::vector<cudaEvent_t> ev;

    cudaError_t ensure(size_t n, int ntr, int nevents) {
        cudaError_t e = cudaSuccess;
        if (n != ncell || (int)tin.size() < ntr) {
            release_buffers();
            ncell = n;
            e = cudaMalloc((void**)&h, n * 8);
            tin.assign(ntr, nullptr);
            tout.assign(ntr, nullptr);
            for (int t = 0; t < ntr && e == cudaSuccess; ++t) {
                e = cudaMalloc((void**)&tin[t], n * 8);
                if (e == cudaSuccess) e = cudaMalloc((void**)&tout[t], n * 8);
            }
            if (e != cudaSuccess) {
                release_buffers();
                return e;
            }
        }
        if (!up) e = cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
        if (e == cudaSuccess && !comp) e = cudaStreamCreateWithFlags(&comp, cudaStreamNonBlocking);
        if (e == cudaSuccess && !down) e = cudaStreamCreateWithFlags(&down, cudaStreamNonBlocking);
        while (e == cudaSuccess && (int)ev.size() < nevents) {
            cudaEvent_t x;
            e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
            if (e == cudaSuccess) ev.push_back(x);
        }
        return e;
    }
    void release_buffers() {
        if (h) cudaFree(h);
        for (double* p : tin) if (p) cudaFree(p);
        for (double* p : tout) if (p) cudaFree(p);
        h = nullptr;
        tin.clear();
        tout.clear();
        ncell = 0;
    }
    void release() {
        release_buffers();
        for (cudaEvent_t x : ev) cudaEventDestroy(x);
        ev.clear();
        for (cudaStream_t* s : {&up, &comp, &down})
            if (*s) cudaStreamDestroy(*s), *s = nullptr;
    }
};

// Rows [r0, r1) of an (nx, ny, nz) column-major field: nz slabs of r1-r0
// consecutive rows, one strided copy.
cudaError_t copy_rows(double* dst, const double* src, int nx, int ny, int nz, int r0, int r1, cudaMemcpyKind kind,
                      cudaStream_t st) {
    if (r1 <= r0) return cudaSuccess;
    const size_t pitch = (size_t)nx * ny * 8;
    return cudaMemcpy2DAsync(dst + (size_t)r0 * nx, pitch, src + (size_t)r0 * nx, pitch, (size_t)(r1 - r0) * nx * 8,
                             nz, kind, st);
}

// ---------------------------------------------------------------------------
// Launch counter and optional per-kernel event timing.
// ---------------------------------------------------------------------------
struct Profiler {
    std::mutex mu;
    bool active = false;
    struct Rec { int kid; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    unsigned long long launches[redi::K_NUM] = {};
    cudaEvent_t take() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
};
Profiler g_prof;

}  // namespace

namespace redi {
void set_last_error(const std::string& msg) { g_last_error = msg; }

// the autotuner's usual gather choice at config 1; the sweep's windows in a
// shared-memory ring of 4 interfaces
static CellTuning g_cell_tuning{64, 2, 8, 8, 2, 1, 0, 0, 4};
CellTuning cell_tuning() { return g_cell_tuning; }
void set_cell_tuning(const CellTuning& t) { g_cell_tuning = t; }
static FoldTuning g_fold_tuning{0, 2, 0, 0, 0};  // the pair stays the default until the fused pass is faster
FoldTuning fold_tuning() { return g_fold_tuning; }
void set_fold_tuning(const FoldTuning& t) { g_fold_tuning = t; }

void launch_begin(int kid, cudaStream_t st) {
    std::lock_guard<std::mutex> lock(g_prof.mu);
    __atomic_add_fetch(&g_prof.launches[kid], 1ULL, __ATOMIC_RELAXED);
    if (!g_prof.active) return;
    Profiler::Rec r{kid, g_prof.take(), nullptr};
    cudaEventRecord(r.a, st);
    g_prof.recs.push_back(r);
}
void count_launches(int kid, unsigned long long n) {
    __atomic_add_fetch(&g_prof.launches[kid], n, __ATOMIC_RELAXED);
}
void launch_end(int kid, cudaStream_t st) {
    std::lock_guard<std::mutex> lock(g_prof.mu);
    if (!g_prof.active) return;
    for (auto it = g_prof.recs.rbegin(); it != g_prof.recs.rend(); ++it) {
        if (it->kid == kid && it->b == nullptr) {
            it->b = g_prof.take();
            cudaEventRecord(it->b, st);
            return;
        }
    }
}
}  // namespace redi

// ---------------------------------------------------------------------------
// ocean_redi_t
// ---------------------------------------------------------------------------
struct redi_b200 {
    bool is_init = false;
    bool enable = false;
    bool continuous = true;
    double khtr = 0.0;
    double ref_pres = -1.0;
    int nx_total = 0, ny_total = 0, nz_ml = 0, nsurf = 0;
    int precision = REDI_B200_FP64;
    int device = -1;
    // Coefficient slots (ocean_redi.F90:105-116): Po f64, Ko i32 (FP64) or
    // i16 (MIXED), hEff f64 (FP64) or f32 (MIXED).
    double *uPoL = nullptr, *uPoR = nullptr, *vPoL = nullptr, *vPoR = nullptr;
    void *uKoL = nullptr, *uKoR = nullptr, *vKoL = nullptr, *vKoR = nullptr;
    void *uhEff = nullptr, *vhEff = nullptr;
    double *khtr_u = nullptr, *khtr_v = nullptr;
    // dry-face record written by the sweep next to the coefficients: 1 at
    // init (every slot holds the inert coefficients), cleared whenever the
    // slots are handed out (the caller may write into them)
    uint8_t *udry = nullptr, *vdry = nullptr;
    template <class P>
    redi::FaceOutT<P> out_u() {
        return {uPoL, uPoR, static_cast<typename P::Ko*>(uKoL), static_cast<typename P::Ko*>(uKoR),
                static_cast<typename P::He*>(uhEff), udry, true};
    }
    template <class P>
    redi::FaceOutT<P> out_v() {
        return {vPoL, vPoR, static_cast<typename P::Ko*>(vKoL), static_cast<typename P::Ko*>(vKoR),
                static_cast<typename P::He*>(vhEff), vdry, true};
    }
    template <class P>
    redi::FaceInT<P> in_u() {
        auto o = out_u<P>();
        return {o.PoL, o.PoR, o.KoL, o.KoR, o.hEff, o.dry};
    }
    template <class P>
    redi::FaceInT<P> in_v() {
        auto o = out_v<P>();
        return {o.PoL, o.PoR, o.KoL, o.KoR, o.hEff, o.dry};
    }
    Scratch ws;
    HostPipeline host;
    std::vector<void*> allocations;

    cudaError_t alloc(void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) allocations.push_back(*p);
        return e;
    }
    void free_all() {
        for (void* p : allocations) cudaFree(p);
        allocations.clear();
        ws.release();
        host.release();
    }
};

extern "C" {

int redi_b200_version(void) { return 100; }

int redi_b200_kernel_count(void) { return redi::K_NUM; }

int redi_b200_set_tuning(int bx, int by, int chunk) {
    if (bx < 1 || by < 1 || bx * by > 128 || (bx * by) % 32 != 0)
        return fail(REDI_B200_E_ARG, "redi_b200_set_tuning: bx*by must be a multiple of 32 and at most 128");
    if (chunk != 4 && chunk != 8 && chunk != 16)
        return fail(REDI_B200_E_ARG, "redi_b200_set_tuning: chunk must be 4, 8 or 16");
    redi::CellTuning t = redi::cell_tuning();
    t.bx = bx;
    t.by = by;
    t.chunk = chunk;
    redi::set_cell_tuning(t);
    return REDI_B200_OK;
}

int redi_b200_set_tracer_group(int max_group) {
    if (max_group != 1 && max_group != 2 && max_group != 4 && max_group != 8)
        return fail(REDI_B200_E_ARG, "redi_b200_set_tracer_group: max_group must be 1, 2, 4 or 8");
    redi::CellTuning t = redi::cell_tuning();
    t.group = max_group;
    redi::set_cell_tuning(t);
    return REDI_B200_OK;
}

int redi_b200_get_tracer_group(void) { return redi::cell_tuning().group; }

int redi_b200_set_gather_tracers(int n, int smem) {
    if (n != 2 && n != 4 && n != 8) return fail(REDI_B200_E_ARG, "redi_b200_set_gather_tracers: n must be 2, 4 or 8");
    if (smem < 0 || smem > 3) return fail(REDI_B200_E_ARG, "redi_b200_set_gather_tracers: smem must be 0, 1, 2 or 3");
    redi::CellTuning t = redi::cell_tuning();
    t.gather_tracers = n;
    t.gather_smem = smem ? 1 : 0;
    t.gather_batch = smem == 2 ? 8 : 0;
    t.gather_pipe = smem == 3 ? 1 : 0;
    redi::set_cell_tuning(t);
    return REDI_B200_OK;
}

int redi_b200_set_flux_staged(int on) {
    if (on < 0 || on > 2) return fail(REDI_B200_E_ARG, "redi_b200_set_flux_staged: on must be 0, 1 or 2");
    redi::CellTuning t = redi::cell_tuning();
    t.flux_staged = on;
    redi::set_cell_tuning(t);
    return REDI_B200_OK;
}

int redi_b200_get_flux_staged(void) { return redi::cell_tuning().flux_staged; }

int redi_b200_set_sweep_form(int form) {
    if (form != 0 && (form < 3 || form > 5))
        return fail(REDI_B200_E_ARG, "redi_b200_set_sweep_form: form must be 0, 3, 4 or 5");
    redi::CellTuning t = redi::cell_tuning();
    t.sweep_form = form;
    redi::set_cell_tuning(t);
    return REDI_B200_OK;
}

int redi_b200_get_sweep_form(void) { return redi::cell_tuning().sweep_form; }


int redi_b200_get_gather_tracers(int* smem) {
    const redi::CellTuning t = redi::cell_tuning();
    if (smem) *smem = t.gather_smem ? (t.gather_pipe ? 3 : (t.gather_batch >= 8 ? 2 : 1)) : 0;
    return redi::cell_tuning().gather_tracers;
}

int redi_b200_set_fold(int enable, int rows, int tracers) {
    if (rows != 1 && rows != 2) return fail(REDI_B200_E_ARG, "redi_b200_set_fold: rows must be 1 or 2");
    if (tracers != 0 && tracers != 1 && tracers != 2 && tracers != 4)
        return fail(REDI_B200_E_ARG, "redi_b200_set_fold: tracers must be 0 (automatic), 1, 2 or 4");
    if (enable < 0 || enable > 7) return fail(REDI_B200_E_ARG, "redi_b200_set_fold: enable is a mask of bits 0..2");
    redi::set_fold_tuning(redi::FoldTuning{enable & 1, rows, tracers, (enable >> 1) & 1, (enable >> 2) & 1});
    return REDI_B200_OK;
}

int redi_b200_get_fold(int* enable, int* rows, int* tracers) {
    if (!enable || !rows || !tracers) return fail(REDI_B200_E_ARG, "redi_b200_get_fold: NULL argument");
    const redi::FoldTuning t = redi::fold_tuning();
    *enable = t.enable | (t.enable_mixed << 1) | (t.ordered_mixed << 2);
    *rows = t.rows;
    *tracers = t.tracers;
    return REDI_B200_OK;
}

int redi_b200_fold_shape(int precision, int nz, int ntracers, int* rows, int* tracers) {
    if (!rows || !tracers || nz < 1 || ntracers < 1) return fail(REDI_B200_E_ARG, "redi_b200_fold_shape: bad argument");
    const redi::FoldShape s = precision == REDI_B200_MIXED ? redi::fold_shape<redi::MixedPrec>(nz, ntracers)
                                                           : redi::fold_shape<redi::PlainPrec>(nz, ntracers);
    *rows = s.by;
    *tracers = s.nt;
    return REDI_B200_OK;
}

int redi_b200_eos_points(const redi_b200_eos* eos, int n, const double* T, const double* S, const double* p,
                         double* rho, double* dsv_dt, double* dsv_ds, void* stream) {
    if (!eos || n < 0) return fail(REDI_B200_E_ARG, "redi_b200_eos_points: NULL eos or negative count");
    if (eos->variant == 3)
        return fail(REDI_B200_E_UNSUPPORTED, "redi_b200_eos_points: EOS variant 3 (TEOS-10) is reserved, not implemented");
    if (eos->variant != 0 && eos->variant != 1 && eos->variant != 2 && eos->variant != 4)
        return fail(REDI_B200_E_ARG, "redi_b200_eos_points: unknown EOS variant (1 LINEAR, 2 WRIGHT_97, 4 ROQUET_SPV)");
    if (n == 0) return REDI_B200_OK;
    if (!T || !S || !p || !rho || !dsv_dt || !dsv_ds) return fail(REDI_B200_E_ARG, "redi_b200_eos_points: NULL array");
    const redi::EosParams e{eos->variant, eos->rho0, eos->T_ref, eos->S_ref, eos->alpha_T, eos->beta_S};
    cudaError_t err = redi::launch_eos_points(e, n, T, S, p, rho, dsv_dt, dsv_ds, reinterpret_cast<cudaStream_t>(stream));
    return err == cudaSuccess ? REDI_B200_OK : cuda_fail(err, "redi_b200_eos_points launch");
}

int redi_b200_get_tuning(int* bx, int* by, int* chunk) {
    if (!bx || !by || !chunk) return fail(REDI_B200_E_ARG, "redi_b200_get_tuning: NULL argument");
    const redi::CellTuning t = redi::cell_tuning();
    *bx = t.bx; *by = t.by; *chunk = t.chunk;
    return REDI_B200_OK;
}

unsigned long long redi_b200_launch_count(int kernel) {
    if (kernel < 0) {
        unsigned long long t = 0;
        for (int k = 0; k < redi::K_NUM; ++k) t += __atomic_load_n(&g_prof.launches[k], __ATOMIC_RELAXED);
        return t;
    }
    if (kernel >= redi::K_NUM) return 0;
    return __atomic_load_n(&g_prof.launches[kernel], __ATOMIC_RELAXED);
}

int redi_b200_profile_begin(void) {
    std::lock_guard<std::mutex> lock(g_prof.mu);
    for (auto& r : g_prof.recs) {
        g_prof.pool.push_back(r.a);
        if (r.b) g_prof.pool.push_back(r.b);
    }
    g_prof.recs.clear();
    g_prof.active = true;
    return REDI_B200_OK;
}

int redi_b200_profile_end(double* total_ms, unsigned long long* counts, int n) {
    std::lock_guard<std::mutex> lock(g_prof.mu);
    g_prof.active = false;
    if (!total_ms || !counts || n < redi::K_NUM) return fail(REDI_B200_E_ARG, "redi_b200_profile_end: output arrays too small");
    for (int k = 0; k < n; ++k) { total_ms[k] = 0.0; counts[k] = 0; }
    for (auto& r : g_prof.recs) {
        if (!r.b) continue;
        cudaError_t e = cudaEventSynchronize(r.b);
        if (e != cudaSuccess) return cuda_fail(e, "redi_b200_profile_end");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        total_ms[r.kid] += ms;
        counts[r.kid] += 1;
    }
    return REDI_B200_OK;
}

const char* redi_b200_last_error(void) { return g_last_error.c_str(); }

int redi_b200_init(const redi_b200_grid* grid, int nz_ml, int precision, redi_b200** out) {
    if (!out) return fail(REDI_B200_E_ARG, "redi_b200_init: out is NULL");
    *out = nullptr;
    if (!grid) return fail(REDI_B200_E_ARG, "redi_b200_init: grid is NULL");
    if (precision != REDI_B200_FP64 && precision != REDI_B200_MIXED)
        return fail(REDI_B200_E_ARG, "redi_b200_init: precision must be REDI_B200_FP64 or REDI_B200_MIXED");
    int nz = nz_ml < 1 ? 1 : nz_ml;  // ocean_redi.F90:478-480
    std::string why;
    if (!dims_ok(grid->nx_total, grid->ny_total, nz, why)) {
        return fail(nz > redi::kNzMax ? REDI_B200_E_UNSUPPORTED : REDI_B200_E_ARG, "redi_b200_init: " + why);
    }
    redi_b200* s = new (std::nothrow) redi_b200();
    if (!s) return fail(REDI_B200_E_NOMEM, "redi_b200_init: host allocation failed");
    cudaGetDevice(&s->device);
    const int nx = grid->nx_total, ny = grid->ny_total, ns = 2 * nz + 2;
    s->nx_total = nx; s->ny_total = ny; s->nz_ml = nz; s->nsurf = ns; s->precision = precision;
    const size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1);
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = s->alloc(p, bytes); };
    const size_t kb = precision == REDI_B200_FP64 ? 4 : 2, hb = precision == REDI_B200_FP64 ? 8 : 4;
    A((void**)&s->uPoL, nu * ns * 8); A((void**)&s->uPoR, nu * ns * 8); A(&s->uhEff, nu * (ns - 1) * hb);
    A(&s->uKoL, nu * ns * kb); A(&s->uKoR, nu * ns * kb);
    A((void**)&s->vPoL, nv * ns * 8); A((void**)&s->vPoR, nv * ns * 8); A(&s->vhEff, nv * (ns - 1) * hb);
    A(&s->vKoL, nv * ns * kb); A(&s->vKoR, nv * ns * kb);
    A((void**)&s->khtr_u, nu * 8); A((void**)&s->khtr_v, nv * 8);
    A((void**)&s->udry, nu); A((void**)&s->vdry, nv);
    if (e != cudaSuccess) {
        s->free_all();
        delete s;
        return fail(REDI_B200_E_NOMEM, std::string("redi_b200_init: device allocation failed: ") + cudaGetErrorString(e));
    }
    // ocean_redi.F90:493-505: Po = 0, Ko = 1, hEff = 0, khtr_* = 0.
    cudaStream_t st = 0;
    cudaMemsetAsync(s->uPoL, 0, nu * ns * 8, st); cudaMemsetAsync(s->uPoR, 0, nu * ns * 8, st);
    cudaMemsetAsync(s->uhEff, 0, nu * (ns - 1) * hb, st);
    cudaMemsetAsync(s->vPoL, 0, nv * ns * 8, st); cudaMemsetAsync(s->vPoR, 0, nv * ns * 8, st);
    cudaMemsetAsync(s->vhEff, 0, nv * (ns - 1) * hb, st);
    if (precision == REDI_B200_FP64) {
        fill_int((int*)s->uKoL, nu * ns, 1, st); fill_int((int*)s->uKoR, nu * ns, 1, st);
        fill_int((int*)s->vKoL, nv * ns, 1, st); fill_int((int*)s->vKoR, nv * ns, 1, st);
    } else {
        fill_short((int16_t*)s->uKoL, nu * ns, 1, st); fill_short((int16_t*)s->uKoR, nu * ns, 1, st);
        fill_short((int16_t*)s->vKoL, nv * ns, 1, st); fill_short((int16_t*)s->vKoR, nv * ns, 1, st);
    }
    cudaMemsetAsync(s->khtr_u, 0, nu * 8, st);
    cudaMemsetAsync(s->khtr_v, 0, nv * 8, st);
    cudaMemsetAsync(s->udry, 1, nu, st);  // every face holds inert coefficients
    cudaMemsetAsync(s->vdry, 1, nv, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        s->free_all();
        delete s;
        return cuda_fail(e, "redi_b200_init");
    }
    s->is_init = true;
    *out = s;
    g_last_error.clear();
    return REDI_B200_OK;
}

int redi_b200_destroy(redi_b200* s) {
    if (!s) return REDI_B200_OK;
    s->is_init = false;
    s->free_all();
    delete s;
    return REDI_B200_OK;
}

int redi_b200_set_enable(redi_b200* s, int enable) {
    if (!s) return fail(REDI_B200_E_ARG, "redi_b200_set_enable: handle is NULL");
    s->enable = enable != 0;
    return REDI_B200_OK;
}

int redi_b200_set_khtr(redi_b200* s, double khtr) {
    if (!s) return fail(REDI_B200_E_ARG, "redi_b200_set_khtr: handle is NULL");
    s->khtr = khtr;
    return REDI_B200_OK;
}

int redi_b200_get_coeffs(const redi_b200* s, redi_b200_coeffs* out) {
    if (!s || !out) return fail(REDI_B200_E_ARG, "redi_b200_get_coeffs: NULL argument");
    if (s->precision != REDI_B200_FP64)
        return fail(REDI_B200_E_STATE, "redi_b200_get_coeffs: mixed-precision handles keep packed coefficients");
    out->uPoL = s->uPoL; out->uPoR = s->uPoR; out->uhEff = (double*)s->uhEff;
    out->uKoL = (int*)s->uKoL; out->uKoR = (int*)s->uKoR;
    out->vPoL = s->vPoL; out->vPoR = s->vPoR; out->vhEff = (double*)s->vhEff;
    out->vKoL = (int*)s->vKoL; out->vKoR = (int*)s->vKoR;
    out->khtr_u = s->khtr_u; out->khtr_v = s->khtr_v; out->nsurf = s->nsurf;
    // The caller may write into the slots: forget which faces hold inert
    // coefficients, so the next redi_calc_coeffs writes every face again and
    // redi_apply_flux skips no face it has not seen dry.
    const size_t nu = (size_t)(s->nx_total + 1) * s->ny_total, nv = (size_t)s->nx_total * (s->ny_total + 1);
    cudaError_t e = cudaMemset(s->udry, 0, nu);
    if (e == cudaSuccess) e = cudaMemset(s->vdry, 0, nv);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "redi_b200_get_coeffs");
    return REDI_B200_OK;
}

long long redi_b200_workspace_bytes(const redi_b200* s) { return s ? (long long)s->ws.bytes : 0; }

int redi_b200_error_count(const redi_b200* s, int reset) {
    if (!s) return fail(REDI_B200_E_ARG, "redi_b200_error_count: handle is NULL");
    if (!s->ws.ptr) return 0;
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, s->ws.err(), sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "redi_b200_error_count");
    if (reset) cudaMemset(s->ws.err(), 0, sizeof(int));
    return v;
}

// The gates and argument checks of redi_b200_calc_coeffs: OK, SKIPPED or an error.
static int check_calc(const redi_b200_grid* grid, const redi_b200_metrics* metrics, const redi_b200_eos* eos,
                      redi_b200* s, const redi_b200_state* ms) {
    if (!grid || !metrics || !eos || !s || !ms) return fail(REDI_B200_E_ARG, "redi_b200_calc_coeffs: NULL argument");
    // Gates of ocean_redi.F90:585-593.
    if (!s->is_init) return REDI_B200_SKIPPED;
    if (!s->enable) return REDI_B200_SKIPPED;
    if (ms->idx_temperature <= 0 || ms->idx_salinity <= 0) return REDI_B200_SKIPPED;
    if (!ms->h_layer) return REDI_B200_SKIPPED;
    const int nx = grid->nx_total, ny = grid->ny_total, nz = ms->nz_ml;
    if (s->nz_ml != nz) return REDI_B200_SKIPPED;
    if (nx != s->nx_total || ny != s->ny_total)
        return fail(REDI_B200_E_ARG, "redi_b200_calc_coeffs: grid extents differ from the handle's");
    if (eos->variant == 3)
        return fail(REDI_B200_E_UNSUPPORTED, "redi_b200_calc_coeffs: EOS variant 3 (TEOS-10) is reserved, not implemented");
    if (eos->variant != 0 && eos->variant != 1 && eos->variant != 2 && eos->variant != 4)
        return fail(REDI_B200_E_ARG, "redi_b200_calc_coeffs: unknown EOS variant (1 LINEAR, 2 WRIGHT_97, 4 ROQUET_SPV)");
    if (ms->idx_temperature > ms->ntracers || ms->idx_salinity > ms->ntracers || !ms->hTr)
        return fail(REDI_B200_E_ARG, "redi_b200_calc_coeffs: temperature/salinity index outside the tracer table");
    const double* th = ms->hTr[ms->idx_temperature - 1];
    const double* sh = ms->hTr[ms->idx_salinity - 1];
    if (!th || !sh || !metrics->wet_u || !metrics->wet_v)
        return fail(REDI_B200_E_ARG, "redi_b200_calc_coeffs: NULL device array");
    if (!aligned(ms->h_layer) || !aligned(th) || !aligned(sh) || !aligned(metrics->wet_u) || !aligned(metrics->wet_v))
        return fail(REDI_B200_E_ARG, "redi_b200_calc_coeffs: misaligned device array");
    return REDI_B200_OK;
}

int redi_b200_calc_coeffs(const redi_b200_grid* grid, const redi_b200_metrics* metrics, const redi_b200_eos* eos,
                          redi_b200* s, const redi_b200_state* ms, void* stream) {
    const int chk = check_calc(grid, metrics, eos, s, ms);
    if (chk != REDI_B200_OK) return chk;
    const int nx = grid->nx_total, ny = grid->ny_total, nz = ms->nz_ml;
    const double* th = ms->hTr[ms->idx_temperature - 1];
    const double* sh = ms->hTr[ms->idx_salinity - 1];
    redi::EosParams e{eos->variant, eos->rho0, eos->T_ref, eos->S_ref, eos->alpha_T, eos->beta_S};
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (s->precision == REDI_B200_MIXED)
        return run_phase_a<redi::MixedPrec>(nx, ny, nz, e, ms->h_layer, th, sh, metrics->wet_u, metrics->wet_v,
                                            s->out_u<redi::MixedPrec>(), s->out_v<redi::MixedPrec>(), s->ws, st);
    return run_phase_a<redi::PlainPrec>(nx, ny, nz, e, ms->h_layer, th, sh, metrics->wet_u, metrics->wet_v,
                                        s->out_u<redi::PlainPrec>(), s->out_v<redi::PlainPrec>(), s->ws, st);
}

// The gates and argument checks of redi_b200_apply_flux: OK, SKIPPED or an
// error; walls receives the boundary walls.
static int check_apply(const redi_b200_grid* grid, const redi_b200_metrics* metrics, redi_b200* s,
                       const redi_b200_state* ms, const double* khtr_u_ext, const double* khtr_v_ext,
                       const redi_b200_bc* bc, int walls[4]) {
    if (!grid || !metrics || !s || !ms) return fail(REDI_B200_E_ARG, "redi_b200_apply_flux: NULL argument");
    // Gates of ocean_redi.F90:951-959.
    if (!s->is_init) return REDI_B200_SKIPPED;
    if (!s->enable) return REDI_B200_SKIPPED;
    if (!ms->h_layer) return REDI_B200_SKIPPED;
    if (!ms->hTr || ms->ntracers <= 0) return REDI_B200_SKIPPED;
    const int nx = grid->nx_total, ny = grid->ny_total, nz = ms->nz_ml;
    if (s->nz_ml != nz) return REDI_B200_SKIPPED;
    if (nx != s->nx_total || ny != s->ny_total)
        return fail(REDI_B200_E_ARG, "redi_b200_apply_flux: grid extents differ from the handle's");
    // ocean_redi.F90:964-973: walls default closed.
    walls[0] = walls[1] = walls[2] = walls[3] = 1;
    if (bc) {
        walls[0] = bc->west == REDI_B200_OBC_WALL;
        walls[1] = bc->east == REDI_B200_OBC_WALL;
        walls[2] = bc->south == REDI_B200_OBC_WALL;
        walls[3] = bc->north == REDI_B200_OBC_WALL;
    }
    const bool use_ext = khtr_u_ext && khtr_v_ext;  // :975
    if (!use_ext && s->khtr <= 0.0) return REDI_B200_SKIPPED;  // :978
    const double* need[] = {metrics->dy_cu, metrics->dx_cv, metrics->idxCu, metrics->idyCv, metrics->areaT};
    for (const double* p : need)
        if (!p || !aligned(p)) return fail(REDI_B200_E_ARG, "redi_b200_apply_flux: NULL or misaligned metric array");
    for (int t = 0; t < ms->ntracers; ++t)
        if (!ms->hTr[t] || !aligned(ms->hTr[t]))
            return fail(REDI_B200_E_ARG, "redi_b200_apply_flux: NULL or misaligned tracer " + std::to_string(t + 1));
    return REDI_B200_OK;
}

// Phase B of a step whose arguments passed check_apply: the per-face KhTr
// into the slots, then the fluxes of every tracer (recon_from: tracers of the
// first batch already reconstructed).
static int run_apply(const redi_b200_grid* grid, const redi_b200_metrics* metrics, redi_b200* s,
                     const redi_b200_state* ms, double dt, const double* khtr_u_ext, const double* khtr_v_ext,
                     const int walls[4], cudaStream_t st, int recon_from) {
    const int nx = grid->nx_total, ny = grid->ny_total, nz = ms->nz_ml;
    const bool use_ext = khtr_u_ext && khtr_v_ext;
    const size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1);
    // Resolve the per-face KhTr into the slots (:981-987).
    cudaError_t e;
    if (use_ext) {
        e = cudaMemcpyAsync(s->khtr_u, khtr_u_ext, nu * 8, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->khtr_v, khtr_v_ext, nv * 8, cudaMemcpyDeviceToDevice, st);
    } else {
        e = fill(s->khtr_u, nu, s->khtr, st);
        if (e == cudaSuccess) e = fill(s->khtr_v, nv, s->khtr, st);
    }
    if (e != cudaSuccess) return cuda_fail(e, "redi_b200_apply_flux: khtr resolve");
    auto fill_in = [&](auto& in) {
        in.nx = nx; in.ny = ny; in.nz = nz; in.nghost = grid->nghost; in.nxp = grid->nx_phys; in.nyp = grid->ny_phys;
        for (int w = 0; w < 4; ++w) in.walls[w] = walls[w];
        in.dt = dt; in.khtr = s->khtr; in.khtr_u = s->khtr_u; in.khtr_v = s->khtr_v;
        in.dy_cu = metrics->dy_cu; in.dx_cv = metrics->dx_cv; in.idxCu = metrics->idxCu; in.idyCv = metrics->idyCv;
        in.areaT = metrics->areaT; in.h = ms->h_layer;
    };
    if (s->precision == REDI_B200_MIXED) {
        PhaseBInputs<redi::MixedPrec> in{};
        fill_in(in);
        in.u = s->in_u<redi::MixedPrec>();
        in.v = s->in_v<redi::MixedPrec>();
        return run_phase_b<redi::MixedPrec>(in, ms->ntracers, ms->hTr, s->ws, st, nullptr, redi::Band{}, recon_from);
    }
    PhaseBInputs<redi::PlainPrec> in{};
    fill_in(in);
    in.u = s->in_u<redi::PlainPrec>();
    in.v = s->in_v<redi::PlainPrec>();
    return run_phase_b<redi::PlainPrec>(in, ms->ntracers, ms->hTr, s->ws, st, nullptr, redi::Band{}, recon_from);
}

int redi_b200_apply_flux(const redi_b200_grid* grid, const redi_b200_metrics* metrics, redi_b200* s,
                         const redi_b200_state* ms, double dt, const double* khtr_u_ext, const double* khtr_v_ext,
                         const redi_b200_bc* bc, void* stream) {
    int walls[4];
    const int chk = check_apply(grid, metrics, s, ms, khtr_u_ext, khtr_v_ext, bc, walls);
    if (chk != REDI_B200_OK) return chk;
    return run_apply(grid, metrics, s, ms, dt, khtr_u_ext, khtr_v_ext, walls, reinterpret_cast<cudaStream_t>(stream), 0);
}


}  // extern "C"

// Phase A of a whole step whose tracers 1 and 2 are T and S (either order):
// the column state and the reconstruction of T and S in one pass, then the
// sweep. Phase B's buffers come first in the scratch (as run_phase_b lays them
// out for ntr tracers) and Phase A's behind them, so both live until the
// fluxes are done; run_phase_b with recon_from = 2 follows.
template <class P>
static int run_fused_phase_a(int nx, int ny, int nz, int ntr, const redi::EosParams& eos, const double* h,
                             const double* tr0, const double* tr1, int ts_swap, const double* wet_u,
                             const double* wet_v, const redi::FaceOutT<P>& u, const redi::FaceOutT<P>& v,
                             Scratch& ws, cudaStream_t st) {
    const int batch = ntr < redi::kMaxTracers ? ntr : redi::kMaxTracers;
    const size_t recon = redi::recon_bytes<P>(nx, ny, nz, batch);
    const size_t flux = redi::flux_bytes<P>(nx, ny, nz, redi::flux_slots(batch, redi::cell_tuning()));
    const size_t b_end = (recon + flux + 255) & ~size_t(255);
    cudaError_t e = ws.reserve(b_end + redi::phase_a_scratch(nx, ny, nz));
    if (e != cudaSuccess) return cuda_fail(e, "scratch allocation (whole step)");
    char* base = static_cast<char*>(ws.data());
    const size_t nifc = (size_t)nx * ny * (nz + 1);
    redi::ColumnStateArgs cs{};
    cs.nx = nx; cs.ny = ny; cs.nz = nz; cs.eos = eos;
    cs.h = h; cs.th = ts_swap ? tr1 : tr0; cs.sh = ts_swap ? tr0 : tr1;
    cs.ifc = reinterpret_cast<redi::IfcState*>(base + b_end);
    cs.pint = reinterpret_cast<double*>(cs.ifc + nifc);
    cs.wet_u = wet_u; cs.wet_v = wet_v;
    redi::ReconArgsT<P> rc{};
    rc.nx = nx; rc.ny = ny; rc.nz = nz; rc.ntr = batch; rc.h = h;
    rc.ti = reinterpret_cast<double*>(base);
    rc.ppm = reinterpret_cast<typename P::Ppm*>(base + redi::recon_ppm_offset(nx, ny, nz, batch));
    rc.htr[0] = tr0;
    rc.htr[1] = tr1;
    e = redi::launch_column_recon<P>(cs, rc, ts_swap, st);
    redi::SweepArgsT<P> sw{};
    sw.nx = nx; sw.ny = ny; sw.nz = nz; sw.rho0 = eos.rho0;
    sw.wet_u = wet_u; sw.wet_v = wet_v; sw.ifc = cs.ifc; sw.pint = cs.pint;
    sw.u = u; sw.v = v;
    if (e == cudaSuccess) e = redi::launch_sweep<P>(sw, st);
    if (e != cudaSuccess) return cuda_fail(e, "phase A launch (whole step)");
    return REDI_B200_OK;
}

template <class P>
static int run_step_phase_a(const redi_b200_grid* grid, const redi_b200_metrics* metrics, const redi_b200_eos* eos,
                            redi_b200* s, const redi_b200_state* ms, int ts_swap, cudaStream_t st) {
    const redi::EosParams e{eos->variant, eos->rho0, eos->T_ref, eos->S_ref, eos->alpha_T, eos->beta_S};
    return run_fused_phase_a<P>(grid->nx_total, grid->ny_total, ms->nz_ml, ms->ntracers, e, ms->h_layer, ms->hTr[0],
                                ms->hTr[1], ts_swap, metrics->wet_u, metrics->wet_v, s->out_u<P>(), s->out_v<P>(),
                                s->ws, st);
}

extern "C" {

int redi_b200_step(const redi_b200_grid* grid, const redi_b200_metrics* metrics, const redi_b200_eos* eos,
                   redi_b200* s, const redi_b200_state* ms, double dt, const double* khtr_u_ext,
                   const double* khtr_v_ext, const redi_b200_bc* bc, void* stream) {
    const int ca = check_calc(grid, metrics, eos, s, ms);
    if (ca < 0) return ca;
    int walls[4];
    const int cb = check_apply(grid, metrics, s, ms, khtr_u_ext, khtr_v_ext, bc, walls);
    if (cb < 0) return cb;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int iT = ms->idx_temperature, iS = ms->idx_salinity;
    const bool fused = ca == REDI_B200_OK && cb == REDI_B200_OK && ((iT == 1 && iS == 2) || (iT == 2 && iS == 1));
    if (!fused) {  // the two calls, each with its own gates
        if (ca == REDI_B200_OK) {
            const int r = redi_b200_calc_coeffs(grid, metrics, eos, s, ms, stream);
            if (r < 0) return r;
        }
        if (cb == REDI_B200_OK) {
            const int r = run_apply(grid, metrics, s, ms, dt, khtr_u_ext, khtr_v_ext, walls, st, 0);
            if (r < 0) return r;
        }
        return (ca == REDI_B200_OK || cb == REDI_B200_OK) ? REDI_B200_OK : REDI_B200_SKIPPED;
    }
    const int ts_swap = iT == 2 ? 1 : 0;
    const int ra = s->precision == REDI_B200_MIXED
                       ? run_step_phase_a<redi::MixedPrec>(grid, metrics, eos, s, ms, ts_swap, st)
                       : run_step_phase_a<redi::PlainPrec>(grid, metrics, eos, s, ms, ts_swap, st);
    if (ra < 0) return ra;
    return run_apply(grid, metrics, s, ms, dt, khtr_u_ext, khtr_v_ext, walls, st, 2);
}

}  // extern "C"

// First row of band b of nbands over ny rows (b == nbands gives ny). With
// nbands >= 3 and ny >= 4 nbands the bands weigh 1, ..., 1, 1/2, 1/4 (in
// quarters: 4, ..., 4, 2, 1; total 4 nbands - 5 <= ny, so every band has a
// row): the last band's kernels and download wait for the last upload, and a
// short last band shortens that tail. Otherwise the bands are equal.
static int band_edge(int b, int nbands, int ny) {
    if (nbands >= 3 && ny >= 4 * nbands) {
        const long long total = 4LL * nbands - 5;
        const long long acc = b <= nbands - 2 ? 4LL * b : (b == nbands - 1 ? total - 1 : total);
        return (int)(acc * ny / total);
    }
    return (int)((long long)b * ny / nbands);
}

// redi_calc_coeffs followed by redi_apply_flux on a model state that lives in
// host memory, pipelined over bands of rows: rows stream in on one stream,
// each band is stepped on a second as soon as its rows (and the row after
// them) are on the device, and finished rows stream back on a third.
template <class P>
int step_host_impl(const redi_b200_grid* grid, const redi_b200_metrics* metrics, const redi::EosParams& eos,
                   redi_b200* s, const redi_b200_state* ms, double dt, bool doA, bool doB, int walls[4],
                   bool use_ext, const double* khtr_u_ext, const double* khtr_v_ext, int nbands, cudaStream_t caller) {
    const int nx = grid->nx_total, ny = grid->ny_total, nz = ms->nz_ml, ntr = ms->ntracers;
    const size_t ncell = (size_t)nx * ny * nz;
    HostPipeline& hp = s->host;
    cudaError_t e = hp.ensure(ncell, ntr, 2 * nbands + 3);
    if (e != cudaSuccess) return fail(REDI_B200_E_NOMEM, std::string("redi_b200_step_host: ") + cudaGetErrorString(e));
    // Scratch for both phases up front: no reallocation while the pipeline runs.
    const int batch = ntr < redi::kMaxTracers ? ntr : redi::kMaxTracers;
    const size_t need_b = redi::recon_bytes<P>(nx, ny, nz, batch) +
                          redi::flux_bytes<P>(nx, ny, nz, redi::flux_slots(batch, redi::cell_tuning()));
    const size_t need_a = redi::phase_a_scratch(nx, ny, nz);
    e = s->ws.reserve(need_a > need_b ? need_a : need_b);
    if (e != cudaSuccess) return cuda_fail(e, "redi_b200_step_host: scratch allocation");
    cudaEvent_t start = hp.ev[0], done = hp.ev[1];
    e = cudaEventRecord(start, caller);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.up, start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.comp, start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.down, start, 0);
    if (doB && e == cudaSuccess) {  // per-face KhTr into the slots (ocean_redi.F90:981-987)
        const size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1);
        if (use_ext) {
            e = cudaMemcpyAsync(s->khtr_u, khtr_u_ext, nu * 8, cudaMemcpyDeviceToDevice, hp.comp);
            if (e == cudaSuccess) e = cudaMemcpyAsync(s->khtr_v, khtr_v_ext, nv * 8, cudaMemcpyDeviceToDevice, hp.comp);
        } else {
            e = fill(s->khtr_u, nu, s->khtr, hp.comp);
            if (e == cudaSuccess) e = fill(s->khtr_v, nv, s->khtr, hp.comp);
        }
    }
    if (e != cudaSuccess) return cuda_fail(e, "redi_b200_step_host: set-up");
    PhaseBInputs<P> in{};
    in.nx = nx; in.ny = ny; in.nz = nz; in.nghost = grid->nghost; in.nxp = grid->nx_phys; in.nyp = grid->ny_phys;
    for (int w = 0; w < 4; ++w) in.walls[w] = walls[w];
    in.dt = dt; in.khtr = s->khtr; in.khtr_u = s->khtr_u; in.khtr_v = s->khtr_v;
    in.dy_cu = metrics->dy_cu; in.dx_cv = metrics->dx_cv; in.idxCu = metrics->idxCu; in.idyCv = metrics->idyCv;
    in.areaT = metrics->areaT; in.h = hp.h;
    in.u = s->in_u<P>();
    in.v = s->in_v<P>();
    const double* th = hp.tin[ms->idx_temperature > 0 ? ms->idx_temperature - 1 : 0];
    const double* sh = hp.tin[ms->idx_salinity > 0 ? ms->idx_salinity - 1 : 0];
    int copied = 0;  // rows already on the device
    for (int b = 0; b < nbands; ++b) {
        const int j0 = band_edge(b, nbands, ny), j1 = band_edge(b + 1, nbands, ny);
        const int need = j1 + 1 < ny ? j1 + 1 : ny;  // the band's cells read one row beyond it
        cudaEvent_t up_b = hp.ev[2 + 2 * b], comp_b = hp.ev[3 + 2 * b];
        if (need > copied) {
            e = copy_rows(hp.h, ms->h_layer, nx, ny, nz, copied, need, cudaMemcpyHostToDevice, hp.up);
            for (int t = 0; t < ntr && e == cudaSuccess; ++t)
                e = copy_rows(hp.tin[t], ms->hTr[t], nx, ny, nz, copied, need, cudaMemcpyHostToDevice, hp.up);
            copied = need;
        }
        if (e == cudaSuccess) e = cudaEventRecord(up_b, hp.up);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.comp, up_b, 0);
        if (e != cudaSuccess) return cuda_fail(e, "redi_b200_step_host: upload");
        const redi::Band band{j0, j1};
        if (doA) {
            const int rc = run_phase_a<P>(nx, ny, nz, eos, hp.h, th, sh, metrics->wet_u, metrics->wet_v, s->out_u<P>(),
                                          s->out_v<P>(), s->ws, hp.comp, band);
            if (rc < 0) return rc;
        }
        if (doB) {
            const int rc = run_phase_b<P>(in, ntr, hp.tout.data(), s->ws, hp.comp, hp.tin.data(), band);
            if (rc < 0) return rc;
            e = cudaEventRecord(comp_b, hp.comp);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.down, comp_b, 0);
            for (int t = 0; t < ntr && e == cudaSuccess; ++t)
                e = copy_rows(ms->hTr[t], hp.tout[t], nx, ny, nz, j0, j1, cudaMemcpyDeviceToHost, hp.down);
            if (e != cudaSuccess) return cuda_fail(e, "redi_b200_step_host: download");
        }
    }
    cudaEvent_t last = hp.ev[2 + 2 * nbands];
    e = cudaEventRecord(last, hp.comp);  // the last band's kernels, even without downloads
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.down, last, 0);
    if (e == cudaSuccess) e = cudaEventRecord(done, hp.down);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(caller, done, 0);
    return e == cudaSuccess ? REDI_B200_OK : cuda_fail(e, "redi_b200_step_host: join");
}

extern "C" {

int redi_b200_step_host(const redi_b200_grid* grid, const redi_b200_metrics* metrics, const redi_b200_eos* eos,
                        redi_b200* s, const redi_b200_state* ms, double dt, const double* khtr_u_ext,
                        const double* khtr_v_ext, const redi_b200_bc* bc, int nbands, void* stream) {
    if (!grid || !metrics || !eos || !s || !ms) return fail(REDI_B200_E_ARG, "redi_b200_step_host: NULL argument");
    if (!s->is_init || !s->enable || !ms->h_layer) return REDI_B200_SKIPPED;
    const int nx = grid->nx_total, ny = grid->ny_total, nz = ms->nz_ml;
    if (s->nz_ml != nz) return REDI_B200_SKIPPED;
    if (nx != s->nx_total || ny != s->ny_total)
        return fail(REDI_B200_E_ARG, "redi_b200_step_host: grid extents differ from the handle's");
    if (eos->variant == 3)
        return fail(REDI_B200_E_UNSUPPORTED, "redi_b200_step_host: EOS variant 3 (TEOS-10) is reserved, not implemented");
    if (eos->variant != 0 && eos->variant != 1 && eos->variant != 2 && eos->variant != 4)
        return fail(REDI_B200_E_ARG, "redi_b200_step_host: unknown EOS variant (1 LINEAR, 2 WRIGHT_97, 4 ROQUET_SPV)");
    if (nbands < 1) return fail(REDI_B200_E_ARG, "redi_b200_step_host: nbands must be >= 1");
    if (nbands > ny) nbands = ny;
    if (nbands > 64) nbands = 64;
    // The two entry points' gates (ocean_redi.F90:585-593, 951-978), each on its own phase.
    const bool ts = ms->idx_temperature > 0 && ms->idx_salinity > 0 && ms->hTr &&
                    ms->idx_temperature <= ms->ntracers && ms->idx_salinity <= ms->ntracers;
    if ((ms->idx_temperature > ms->ntracers || ms->idx_salinity > ms->ntracers) && ms->ntracers > 0)
        return fail(REDI_B200_E_ARG, "redi_b200_step_host: temperature/salinity index outside the tracer table");
    const bool use_ext = khtr_u_ext && khtr_v_ext;
    const bool doA = ts;
    const bool doB = ms->hTr && ms->ntracers > 0 && (use_ext || s->khtr > 0.0);
    if (!doA && !doB) return REDI_B200_SKIPPED;
    if (ms->ntracers > 0 && !ms->hTr) return fail(REDI_B200_E_ARG, "redi_b200_step_host: NULL tracer table");
    for (int t = 0; t < ms->ntracers; ++t)
        if (!ms->hTr[t]) return fail(REDI_B200_E_ARG, "redi_b200_step_host: NULL host tracer " + std::to_string(t + 1));
    const double* need[] = {metrics->wet_u, metrics->wet_v, metrics->dy_cu, metrics->dx_cv, metrics->idxCu,
                            metrics->idyCv, metrics->areaT};
    for (const double* p : need)
        if (!p || !aligned(p)) return fail(REDI_B200_E_ARG, "redi_b200_step_host: NULL or misaligned metric array");
    int walls[4] = {1, 1, 1, 1};
    if (bc) {
        walls[0] = bc->west == REDI_B200_OBC_WALL;
        walls[1] = bc->east == REDI_B200_OBC_WALL;
        walls[2] = bc->south == REDI_B200_OBC_WALL;
        walls[3] = bc->north == REDI_B200_OBC_WALL;
    }
    const redi::EosParams e{eos->variant, eos->rho0, eos->T_ref, eos->S_ref, eos->alpha_T, eos->beta_S};
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (s->precision == REDI_B200_MIXED)
        return step_host_impl<redi::MixedPrec>(grid, metrics, e, s, ms, dt, doA, doB, walls, use_ext, khtr_u_ext,
                                               khtr_v_ext, nbands, st);
    return step_host_impl<redi::PlainPrec>(grid, metrics, e, s, ms, dt, doA, doB, walls, use_ext, khtr_u_ext,
                                           khtr_v_ext, nbands, st);
}

// ---------------------------------------------------------------------------
// Reference-compatible launchers (redi/opt_kernel.cu:534-574,
// redi/redi_kernel.cu:537-580).
// ---------------------------------------------------------------------------
static std::mutex g_compat_mu;
static std::vector<Scratch> g_compat_ws;  // one per device
// the sweep's dry-face record between the two phases of a compat call, one
// grow-only buffer per device (the phases share g_compat_ws)
static std::vector<Scratch> g_compat_dry;

static void compat_launch(const char* name, const int* nx_, const int* ny_, const int* nz_, const int* ns_,
                          const double* dt_, const int* nghost_, const int* nxp_, const int* nyp_, const int* ww_,
                          const int* we_, const int* wsz_, const int* wn_, const double* rho0_, const double* T_ref_,
                          const double* S_ref_, const double* alpha_T_, const double* beta_S_, const double* h_layer,
                          double* t_htr, double* s_htr, const double* wet_u, const double* wet_v, double* uPoL,
                          double* uPoR, int* uKoL, int* uKoR, double* uhEff, double* vPoL, double* vPoR, int* vKoL,
                          int* vKoR, double* vhEff, const double* khtr_u_ext, const double* khtr_v_ext,
                          double* khtr_u, double* khtr_v, const double* dy_cu, const double* dx_cv,
                          const double* idxCu, const double* idyCv, const double* areaT) {
    auto report = [&](int code, const std::string& msg) {
        fail(code, std::string(name) + ": " + msg);
        std::fprintf(stderr, "%s: %s\n", name, msg.c_str());
    };
    const void* scalars[] = {nx_, ny_, nz_, ns_, dt_, nghost_, nxp_, nyp_, ww_, we_, wsz_, wn_,
                             rho0_, T_ref_, S_ref_, alpha_T_, beta_S_};
    for (const void* p : scalars)
        if (!p) { report(REDI_B200_E_ARG, "NULL scalar argument"); return; }
    const int nx = *nx_, ny = *ny_, nz = *nz_, ns = *ns_;
    std::string why;
    if (!dims_ok(nx, ny, nz, why)) { report(REDI_B200_E_ARG, why); return; }
    if (ns != 2 * nz + 2) { report(REDI_B200_E_ARG, "ns must equal 2*nz+2"); return; }
    const void* arrays[] = {h_layer, t_htr, s_htr, wet_u, wet_v, uPoL, uPoR, uKoL, uKoR, uhEff, vPoL, vPoR,
                            vKoL, vKoR, vhEff, khtr_u_ext, khtr_v_ext, khtr_u, khtr_v, dy_cu, dx_cv, idxCu,
                            idyCv, areaT};
    for (const void* p : arrays)
        if (!p || (reinterpret_cast<uintptr_t>(p) % 4) != 0) { report(REDI_B200_E_ARG, "NULL or misaligned array"); return; }
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_compat_mu);
    if ((int)g_compat_ws.size() <= dev) g_compat_ws.resize(dev + 1);
    Scratch& ws = g_compat_ws[dev];
    if ((int)g_compat_dry.size() <= dev) g_compat_dry.resize(dev + 1);
    Scratch& dry = g_compat_dry[dev];
    const size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1);
    if (dry.reserve(nu + nv) != cudaSuccess) { report(REDI_B200_E_NOMEM, "scratch allocation (dry faces)"); return; }
    uint8_t* udry = static_cast<uint8_t*>(dry.data());
    uint8_t* vdry = udry + nu;
    cudaStream_t st = 0;  // the reference launches on the legacy default stream
    redi::EosParams e{1, *rho0_, *T_ref_, *S_ref_, *alpha_T_, *beta_S_};  // the launcher's LINEAR EOS
    redi::FaceOut u{uPoL, uPoR, uKoL, uKoR, uhEff, udry}, v{vPoL, vPoR, vKoL, vKoR, vhEff, vdry};
    // both phases in this call: the column state and the T/S reconstruction in one pass
    int rc = run_fused_phase_a<redi::PlainPrec>(nx, ny, nz, 2, e, h_layer, t_htr, s_htr, 0, wet_u, wet_v, u, v, ws, st);
    if (rc < 0) { report(rc, g_last_error); return; }
    cudaMemcpyAsync(khtr_u, khtr_u_ext, nu * 8, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(khtr_v, khtr_v_ext, nv * 8, cudaMemcpyDeviceToDevice, st);
    PhaseBInputs<redi::PlainPrec> in{};
    in.nx = nx; in.ny = ny; in.nz = nz; in.nghost = *nghost_; in.nxp = *nxp_; in.nyp = *nyp_;
    in.walls[0] = *ww_; in.walls[1] = *we_; in.walls[2] = *wsz_; in.walls[3] = *wn_;
    in.dt = *dt_; in.khtr = 0.0; in.khtr_u = khtr_u; in.khtr_v = khtr_v;
    in.dy_cu = dy_cu; in.dx_cv = dx_cv; in.idxCu = idxCu; in.idyCv = idyCv; in.areaT = areaT; in.h = h_layer;
    in.u = redi::FaceIn{uPoL, uPoR, uKoL, uKoR, uhEff, udry};
    in.v = redi::FaceIn{vPoL, vPoR, vKoL, vKoR, vhEff, vdry};
    double* trs[2] = {t_htr, s_htr};
    rc = run_phase_b<redi::PlainPrec>(in, 2, trs, ws, st, nullptr, redi::Band{}, 2);
    if (rc < 0) { report(rc, g_last_error); return; }
    cudaDeviceSynchronize();
}

void redi_opt_launch(const int* nx, const int* ny, const int* nz, const int* ns, const double* dt, const int* nghost,
                     const int* nxp, const int* nyp, const int* ww, const int* we, const int* wsz, const int* wn,
                     const double* rho0, const double* T_ref, const double* S_ref, const double* alpha_T,
                     const double* beta_S, const double* h_layer, double* t_htr, double* s_htr, const double* wet_u,
                     const double* wet_v, double* uPoL, double* uPoR, int* uKoL, int* uKoR, double* uhEff,
                     double* vPoL, double* vPoR, int* vKoL, int* vKoR, double* vhEff, const double* khtr_u_ext,
                     const double* khtr_v_ext, double* khtr_u, double* khtr_v, const double* dy_cu,
                     const double* dx_cv, const double* idxCu, const double* idyCv, const double* areaT,
                     double* tr_snap) {
    (void)tr_snap;
    compat_launch("redi_opt_launch", nx, ny, nz, ns, dt, nghost, nxp, nyp, ww, we, wsz, wn, rho0, T_ref, S_ref,
                  alpha_T, beta_S, h_layer, t_htr, s_htr, wet_u, wet_v, uPoL, uPoR, uKoL, uKoR, uhEff, vPoL, vPoR,
                  vKoL, vKoR, vhEff, khtr_u_ext, khtr_v_ext, khtr_u, khtr_v, dy_cu, dx_cv, idxCu, idyCv, areaT);
}

void redi_cuda_launch_(const int* nx, const int* ny, const int* nz, const int* ns, const double* dt,
                       const int* nghost, const int* nxp, const int* nyp, const int* ww, const int* we,
                       const int* wsz, const int* wn, const double* rho0, const double* T_ref, const double* S_ref,
                       const double* alpha_T, const double* beta_S, const double* h_layer, double* t_htr,
                       double* s_htr, const double* wet_u, const double* wet_v, double* uPoL, double* uPoR,
                       int* uKoL, int* uKoR, double* uhEff, double* vPoL, double* vPoR, int* vKoL, int* vKoR,
                       double* vhEff, const double* khtr_u_ext, const double* khtr_v_ext, double* khtr_u,
                       double* khtr_v, const double* dy_cu, const double* dx_cv, const double* idxCu,
                       const double* idyCv, const double* areaT, double* tr_snap) {
    (void)tr_snap;
    compat_launch("redi_cuda_launch_", nx, ny, nz, ns, dt, nghost, nxp, nyp, ww, we, wsz, wn, rho0, T_ref, S_ref,
                  alpha_T, beta_S, h_layer, t_htr, s_htr, wet_u, wet_v, uPoL, uPoR, uKoL, uKoR, uhEff, vPoL,
                  vPoR, vKoL, vKoR, vhEff, khtr_u_ext, khtr_v_ext, khtr_u, khtr_v, dy_cu, dx_cv, idxCu, idyCv,
                  areaT);
}

}  // extern "C"
