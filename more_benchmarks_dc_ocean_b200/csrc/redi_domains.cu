// Many independent regional domains of uneven size in one persistent kernel.
//
// A step of every domain (Phase A then Phase B, all tracers) is cut into work
// items: tiles of columns (interface state, tracer reconstruction), tiles of
// faces (neutral sweep, face fluxes of one tracer pair) and 2-D tiles of cells
// (the ordered gather of one tracer pair). The host builds the item queue once:
// stage by stage, and within a stage domain by domain, largest domain first
// (longest-processing-time order), so an item's predecessors always sit earlier
// in the queue. One persistent grid (as many blocks as fit on the GPU at once)
// claims items through an atomic cursor.
//
// Dependencies: the stages of one domain run in order (column state, sweep,
// reconstruction, then flux and gather per tracer pair, the flux buffer being
// reused by the next pair); a tile of stage s of domain d starts once every tile
// of stage s-1 of d is done. Thread 0 of the block polls the per-(domain,
// stage) completion counter with acquire semantics and releases its own
// counter after a block barrier and a device fence; data produced inside the
// kernel is read through L2 (LdCG), never through the non-coherent path.
// Progress is guaranteed: a block only ever waits on items claimed before its
// own, by blocks already running. Every wait is bounded by a time limit
// (default 2 s); on expiry the kernel records TIMEOUT with the domain and stage
// in a status word, and every block returns.
//
// Compiled with FMA contraction off: the arithmetic is the plain form's (or the
// mixed form's) exactly, so a batched domain's result equals a single-domain
// call's bit for bit.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/redi_b200.h"
#include "redi_items.cuh"

namespace redi {
namespace domains {

constexpr int kThreads = 128;
constexpr int kPairs = kMaxTracers / 2;           // tracer pairs per domain
constexpr int kMaxStages = 3 + 2 * kPairs;        // column, sweep, recon, (flux, gather) x pairs

enum Stage : int { S_COLUMN = 0, S_SWEEP = 1, S_RECON = 2, S_PAIR0 = 3 };

template <class P>
struct DomainDev {
    ColumnStateArgs cs;
    SweepArgsT<P> sw;
    ReconArgsT<P> rc;
    FaceFluxArgsT<P> ff;
    CellGatherArgsT<P> cg;
    int nstages;
    int ntiles[kMaxStages];
    int nu_tiles;   // face stages: tiles < nu_tiles are u-faces
    int gx;         // gather tiles along x
};

struct Item {
    int16_t domain;
    int16_t stage;
    int32_t tile;
};

constexpr int kStageKinds = 5;  // column state, sweep, reconstruction, face flux, gather

struct Control {
    int cursor;
    int status;   // 0 ok, REDI_B200_STATUS_TIMEOUT
    int t_domain;
    int t_stage;
    int bad;      // fluxes the gather found out of order (always 0 for coefficients made in the step)
    int pad;
    // Per stage kind, summed over blocks when accounting is on: time spent
    // waiting for predecessors, time spent on tiles, and tiles processed.
    unsigned long long wait_ns[kStageKinds];
    unsigned long long busy_ns[kStageKinds];
    unsigned long long tiles[kStageKinds];
};

__device__ __forceinline__ int stage_kind(int st) { return st < S_PAIR0 ? st : 3 + ((st - S_PAIR0) & 1); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait until *flag >= target (acquire); false on timeout or when
// another block has already recorded a failure.
__device__ __forceinline__ bool wait_at_least(int* flag, int target, int* status, unsigned long long limit_ns) {
    cuda::atomic_ref<int, cuda::thread_scope_device> f(*flag);
    if (f.load(cuda::memory_order_acquire) >= target) return true;
    cuda::atomic_ref<int, cuda::thread_scope_device> st(*status);
    const unsigned long long t0 = global_ns();
    while (true) {
        __nanosleep(256);
        if (f.load(cuda::memory_order_acquire) >= target) return true;
        if (st.load(cuda::memory_order_relaxed) != 0) return false;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// A held domain (fault injection from the host: its input is never
// published) makes the block wait for the release flag, which nothing sets
// during the launch, until the time limit.
__device__ __forceinline__ bool wait_released(const int* held, int* status, unsigned long long limit_ns) {
    cuda::atomic_ref<int, cuda::thread_scope_device> st(*status);
    const unsigned long long t0 = global_ns();
    while (*((const volatile int*)held) != 0) {
        __nanosleep(256);
        if (st.load(cuda::memory_order_relaxed) != 0) return false;
        if (global_ns() - t0 > limit_ns) return false;
    }
    return true;
}

// OCC is the residency the registers are budgeted for (blocks per SM).
template <class P, int CH, int OCC>
__global__ void __launch_bounds__(kThreads, OCC) k_domains(const DomainDev<P>* __restrict__ doms,
                                                           const Item* __restrict__ queue, int nitems, int* done,
                                                           const int* held, Control* ctl, unsigned long long limit_ns,
                                                           int bx, int account) {
    __shared__ int s_idx;
    __shared__ int s_go;
    const int tid = threadIdx.x;
    unsigned long long t_claim = 0, t_start = 0;
    while (true) {
        if (tid == 0) {
            int go = 1;
            if (account) t_claim = global_ns();
            const int idx = atomicAdd(&ctl->cursor, 1);
            s_idx = idx;
            if (idx >= nitems) {
                go = 0;
            } else if (*((volatile int*)&ctl->status) != 0) {
                go = 0;
            } else {
                const Item it = queue[idx];
                bool ok = true;
                if (it.stage == S_COLUMN) {
                    ok = wait_released(held + it.domain, &ctl->status, limit_ns);
                } else {
                    ok = wait_at_least(&done[it.domain * kMaxStages + it.stage - 1],
                                       doms[it.domain].ntiles[it.stage - 1], &ctl->status, limit_ns);
                }
                if (ok) {
                    __threadfence();  // the predecessors' writes before this block's reads
                    if (account) t_start = global_ns();
                } else {
                    if (atomicCAS(&ctl->status, 0, REDI_B200_STATUS_TIMEOUT) == 0) {
                        ctl->t_domain = it.domain;
                        ctl->t_stage = it.stage;
                    }
                    go = 0;
                }
            }
            s_go = go;
        }
        __syncthreads();
        if (!s_go) return;
        const Item it = queue[s_idx];
        const DomainDev<P>& d = doms[it.domain];
        const int st = it.stage;
        if (st == S_COLUMN) {
            const int col = it.tile * kThreads + tid;
            if (col < d.cs.nx * d.cs.ny) plain::column_state_item<LdCG>(d.cs, col);
        } else if (st == S_SWEEP) {
            const int dir = it.tile < d.nu_tiles ? 0 : 1;
            const int t = (dir == 0 ? it.tile : it.tile - d.nu_tiles) * kThreads + tid;
            plain::sweep_item<P, LdCG, false>(d.sw, dir, t);
        } else if (st == S_RECON) {
            plain::recon_item<2, P, LdCG>(d.rc, it.tile * kThreads + tid, 0, d.rc.nx * d.rc.ny);
        } else {
            const int pair = (st - S_PAIR0) >> 1;
            if (((st - S_PAIR0) & 1) == 0) {
                const int dir = it.tile < d.nu_tiles ? 0 : 1;
                const int t = (dir == 0 ? it.tile : it.tile - d.nu_tiles) * kThreads + tid;
                plain::flux_item<2, P, LdCG>(d.ff, dir, t, 2 * pair, INT_MAX);
            } else {
                const int by = kThreads / bx;
                const int i = (it.tile % d.gx) * bx + tid % bx;
                const int j = (it.tile / d.gx) * by + tid / bx;
                plain::gather_item<2, CH, P, LdCG>(d.cg, i, j, 2 * pair, 0);
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            cuda::atomic_ref<int, cuda::thread_scope_device> c(done[it.domain * kMaxStages + st]);
            c.fetch_add(1, cuda::memory_order_release);
            if (account) {
                const int kind = stage_kind(st);
                atomicAdd(&ctl->wait_ns[kind], t_start - t_claim);
                atomicAdd(&ctl->busy_ns[kind], global_ns() - t_start);
                atomicAdd(&ctl->tiles[kind], 1ULL);
            }
        }
    }
}

}  // namespace domains
}  // namespace redi

using redi::domains::Control;
using redi::domains::DomainDev;
using redi::domains::Item;
using redi::domains::kMaxStages;
using redi::domains::kThreads;

struct redi_b200_batch {
    int precision = REDI_B200_FP64;
    int ndomains = 0;
    int bx = 32, by = 4, chunk = 8;
    int use_graph = 1;
    int occ = 4;       // register budget: blocks per SM (4, 5 or 6)
    int account = 0;   // per-stage time accounting in the kernel
    int grid = 0;
    int nitems = 0;
    unsigned long long limit_ns = 2000000000ULL;
    void* d_doms = nullptr;       // DomainDev<P>[ndomains]
    Item* d_queue = nullptr;
    int* d_done = nullptr;        // ndomains * kMaxStages
    int* d_held = nullptr;        // ndomains
    Control* d_ctl = nullptr;
    std::vector<void*> allocs;    // per-domain coefficients and scratch
    std::vector<long long> updates;  // tracer-cell updates per step, per domain
    std::vector<double> cost;        // work estimate per domain (queue order)
    std::vector<unsigned char> host_doms;  // host copy of d_doms
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

int bfail(int code, const std::string& m) {
    redi::set_last_error(m);
    return code;
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

void drop_graph(redi_b200_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

void free_batch(redi_b200_batch* b) {
    drop_graph(b);
    for (void* p : b->allocs) cudaFree(p);
    b->allocs.clear();
    if (b->d_queue) cudaFree(b->d_queue);
    b->d_queue = nullptr;
}

template <class P>
using DomainKernel = void (*)(const DomainDev<P>*, const Item*, int, int*, const int*, Control*, unsigned long long, int,
                              int);

template <class P, int CH>
DomainKernel<P> kernel_occ(int occ) {
    switch (occ) {
        case 5: return redi::domains::k_domains<P, CH, 5>;
        case 6: return redi::domains::k_domains<P, CH, 6>;
        default: return redi::domains::k_domains<P, CH, 4>;
    }
}

template <class P>
DomainKernel<P> kernel_for(int chunk, int occ) {
    switch (chunk) {
        case 4: return kernel_occ<P, 4>(occ);
        case 16: return kernel_occ<P, 16>(occ);
        default: return kernel_occ<P, 8>(occ);
    }
}

// Queue position p of a face stage's ntiles tiles -> tile index (tiles < nu are
// u faces): u and v tiles alternate while both remain, so the two directions of
// the same rows are in flight together and a column's data is read from HBM once.
inline int face_tile_at(int p, int nu, int ntiles) {
    const int nv = ntiles - nu, m = nu < nv ? nu : nv;
    if (p < 2 * m) return (p & 1) ? nu + (p >> 1) : (p >> 1);
    return nu > nv ? p - m : nu + (p - m);
}

inline bool face_stage(int st) {
    return st == redi::domains::S_SWEEP || (st >= redi::domains::S_PAIR0 && ((st - redi::domains::S_PAIR0) & 1) == 0);
}

// Gather tiling, work queue and persistent grid for the current launch shape.
template <class P>
int layout(redi_b200_batch* b) {
    const int n = b->ndomains;
    DomainDev<P>* hd = reinterpret_cast<DomainDev<P>*>(b->host_doms.data());
    for (int k = 0; k < n; ++k) {
        DomainDev<P>& d = hd[k];
        d.gx = (d.cg.nx + b->bx - 1) / b->bx;
        const int gy = (d.cg.ny + b->by - 1) / b->by;
        for (int st = redi::domains::S_PAIR0 + 1; st < d.nstages; st += 2) d.ntiles[st] = d.gx * gy;
    }
    // Queue: stage-major, domains in decreasing cost within a stage.
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->cost[x] > b->cost[y]; });
    std::vector<Item> q;
    for (int st = 0; st < kMaxStages; ++st)
        for (int k : order)
            if (st < hd[k].nstages)
                for (int t = 0; t < hd[k].ntiles[st]; ++t)
                    q.push_back(Item{(int16_t)k, (int16_t)st,
                                     face_stage(st) ? face_tile_at(t, hd[k].nu_tiles, hd[k].ntiles[st]) : t});
    drop_graph(b);
    if (b->d_queue) cudaFree(b->d_queue);
    b->d_queue = nullptr;
    b->nitems = (int)q.size();
    cudaError_t e = cudaMalloc((void**)&b->d_queue, sizeof(Item) * q.size());
    if (e != cudaSuccess) return bfail(REDI_B200_E_NOMEM, std::string("redi_b200_batch: queue: ") + cudaGetErrorString(e));
    e = cudaMemcpy(b->d_queue, q.data(), sizeof(Item) * q.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_doms, hd, sizeof(DomainDev<P>) * n, cudaMemcpyHostToDevice);
    // Persistent grid: every block resident at once.
    int dev = 0, sms = 0, per_sm = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return bfail(REDI_B200_E_CUDA, std::string("redi_b200_batch: ") + cudaGetErrorString(e));
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_for<P>(b->chunk, b->occ), kThreads, 0);
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    b->grid = sms * per_sm;
    return REDI_B200_OK;
}

int layout_any(redi_b200_batch* b) {
    return b->precision == REDI_B200_MIXED ? layout<redi::MixedPrec>(b) : layout<redi::PlainPrec>(b);
}

template <class P>
int build(redi_b200_batch* b, int n, const redi_b200_domain* dom) {
    using Ko = typename P::Ko;
    using He = typename P::He;
    b->host_doms.assign(sizeof(DomainDev<P>) * n, 0);
    DomainDev<P>* hd = reinterpret_cast<DomainDev<P>*>(b->host_doms.data());
    b->cost.assign(n, 0.0);
    cudaError_t e0 = cudaMalloc((void**)&b->d_ctl, sizeof(Control));
    if (e0 != cudaSuccess) return bfail(REDI_B200_E_NOMEM, std::string("redi_b200_batch_create: ") + cudaGetErrorString(e0));
    b->allocs.push_back(b->d_ctl);
    for (int k = 0; k < n; ++k) {
        const redi_b200_domain& D = dom[k];
        const int nx = D.grid.nx_total, ny = D.grid.ny_total, nz = D.ms.nz_ml, ntr = D.ms.ntracers;
        const int ns = 2 * nz + 2;
        if (nx < 2 || ny < 2 || nz < 1 || nz > redi::kNzMax)
            return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: domain " + std::to_string(k) + " has invalid extents");
        if (ntr < 2 || ntr > redi::kMaxTracers || !D.ms.hTr || !D.ms.h_layer)
            return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: domain " + std::to_string(k) +
                                              " needs 2..64 tracers and a thickness field");
        if (D.ms.idx_temperature < 1 || D.ms.idx_salinity < 1 || D.ms.idx_temperature > ntr || D.ms.idx_salinity > ntr)
            return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: domain " + std::to_string(k) + " has no T/S");
        if (D.eos.variant != 0 && D.eos.variant != 1 && D.eos.variant != 2 && D.eos.variant != 4)
            return bfail(D.eos.variant == 3 ? REDI_B200_E_UNSUPPORTED : REDI_B200_E_ARG,
                         "redi_b200_batch_create: domain " + std::to_string(k) +
                             ": EOS variant must be 1 LINEAR, 2 WRIGHT_97 or 4 ROQUET_SPV");
        if (!D.khtr_u_ext || !D.khtr_v_ext || !D.metrics.dy_cu || !D.metrics.dx_cv || !D.metrics.idxCu ||
            !D.metrics.idyCv || !D.metrics.areaT || !D.metrics.wet_u || !D.metrics.wet_v)
            return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: domain " + std::to_string(k) + " has a NULL array");
        if ((long long)(nx + 1) * (ny + 1) * ns >= (1LL << 31))
            return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: domain too large");
        const size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1), ncol = (size_t)nx * ny;
        // coefficient slots (their initial state is irrelevant: the dry-face
        // record starts at 0, so the first step writes every interior face) and
        // the record itself
        const size_t coef_b = up256(nu * ns * 8) * 2 + up256(nv * ns * 8) * 2 + up256(nu * ns * sizeof(Ko)) * 2 +
                              up256(nv * ns * sizeof(Ko)) * 2 + up256(nu * (ns - 1) * sizeof(He)) +
                              up256(nv * (ns - 1) * sizeof(He)) + up256(nu) + up256(nv);
        const size_t a_b = redi::phase_a_scratch(nx, ny, nz);
        const size_t rb = redi::recon_bytes<P>(nx, ny, nz, ntr), fb = redi::flux_bytes<P>(nx, ny, nz, 2);
        const size_t scratch = std::max(a_b, up256(rb) + fb);
        char* base = nullptr;
        cudaError_t e = cudaMalloc((void**)&base, coef_b + up256(scratch));
        if (e != cudaSuccess) return bfail(REDI_B200_E_NOMEM, std::string("redi_b200_batch_create: ") + cudaGetErrorString(e));
        b->allocs.push_back(base);
        cudaMemset(base, 0, coef_b);
        char* q = base;
        auto take = [&](size_t bytes) { char* r = q; q += up256(bytes); return r; };
        redi::FaceOutT<P> u{(double*)take(nu * ns * 8), (double*)take(nu * ns * 8), (Ko*)take(nu * ns * sizeof(Ko)),
                            (Ko*)take(nu * ns * sizeof(Ko)), (He*)take(nu * (ns - 1) * sizeof(He))};
        redi::FaceOutT<P> v{(double*)take(nv * ns * 8), (double*)take(nv * ns * 8), (Ko*)take(nv * ns * sizeof(Ko)),
                            (Ko*)take(nv * ns * sizeof(Ko)), (He*)take(nv * (ns - 1) * sizeof(He))};
        // the batch's own slots: a face that stays dry keeps its inert coefficients
        u.dry = (uint8_t*)take(nu);
        v.dry = (uint8_t*)take(nv);
        u.keep = v.keep = true;
        char* sc = base + coef_b;
        DomainDev<P>& d = hd[k];
        std::memset(&d, 0, sizeof(d));
        const double* th = D.ms.hTr[D.ms.idx_temperature - 1];
        const double* sh = D.ms.hTr[D.ms.idx_salinity - 1];
        d.cs = redi::ColumnStateArgs{nx, ny, nz, redi::EosParams{D.eos.variant, D.eos.rho0, D.eos.T_ref, D.eos.S_ref,
                                                                  D.eos.alpha_T, D.eos.beta_S},
                                     D.ms.h_layer, th, sh, (redi::IfcState*)sc, nullptr};
        d.cs.pint = (double*)(d.cs.ifc + ncol * (nz + 1));
        d.cs.wet_u = D.metrics.wet_u; d.cs.wet_v = D.metrics.wet_v;
        d.sw.nx = nx; d.sw.ny = ny; d.sw.nz = nz; d.sw.rho0 = D.eos.rho0;
        d.sw.wet_u = D.metrics.wet_u; d.sw.wet_v = D.metrics.wet_v; d.sw.ifc = d.cs.ifc; d.sw.pint = d.cs.pint;
        d.sw.u = u; d.sw.v = v;
        d.rc.nx = nx; d.rc.ny = ny; d.rc.nz = nz; d.rc.ntr = ntr; d.rc.h = D.ms.h_layer;
        d.rc.ti = (double*)sc;
        d.rc.ppm = (typename P::Ppm*)(sc + redi::recon_ppm_offset(nx, ny, nz, ntr));
        d.rc.dry_u = u.dry; d.rc.dry_v = v.dry;
        int walls[4] = {1, 1, 1, 1};
        walls[0] = D.bc.west == REDI_B200_OBC_WALL; walls[1] = D.bc.east == REDI_B200_OBC_WALL;
        walls[2] = D.bc.south == REDI_B200_OBC_WALL; walls[3] = D.bc.north == REDI_B200_OBC_WALL;
        auto& ff = d.ff;
        ff.nx = nx; ff.ny = ny; ff.nz = nz; ff.ntr = ntr; ff.nghost = D.grid.nghost; ff.nxp = D.grid.nx_phys;
        ff.nyp = D.grid.ny_phys; ff.wall_w = walls[0]; ff.wall_e = walls[1]; ff.wall_s = walls[2]; ff.wall_n = walls[3];
        ff.dt = D.dt; ff.khtr = 0.0; ff.khtr_u = D.khtr_u_ext; ff.khtr_v = D.khtr_v_ext;
        ff.dy_cu = D.metrics.dy_cu; ff.dx_cv = D.metrics.dx_cv; ff.idxCu = D.metrics.idxCu; ff.idyCv = D.metrics.idyCv;
        ff.u = redi::FaceInT<P>{u.PoL, u.PoR, u.KoL, u.KoR, u.hEff, u.dry};
        ff.v = redi::FaceInT<P>{v.PoL, v.PoR, v.KoL, v.KoR, v.hEff, v.dry};
        ff.ti = d.rc.ti; ff.ppm = d.rc.ppm;
        ff.Fu = (typename P::Flux*)(sc + up256(rb));
        ff.Fv = ff.Fu + (size_t)2 * (2 * nz + 1) * nu;
        auto& cg = d.cg;
        cg.nx = nx; cg.ny = ny; cg.nz = nz; cg.ntr = ntr; cg.nghost = ff.nghost; cg.nxp = ff.nxp; cg.nyp = ff.nyp;
        cg.wall_w = walls[0]; cg.wall_e = walls[1]; cg.wall_s = walls[2]; cg.wall_n = walls[3];
        cg.areaT = D.metrics.areaT; cg.u = ff.u; cg.v = ff.v; cg.Fu = ff.Fu; cg.Fv = ff.Fv; cg.err = &b->d_ctl->bad;
        for (int t = 0; t < ntr; ++t) {
            d.rc.htr[t] = D.ms.hTr[t];
            cg.htr[t] = D.ms.hTr[t];
            cg.htr_in[t] = D.ms.hTr[t];
        }
        const int npairs = (ntr + 1) / 2;
        const int nuf = (nx - 1) * ny, nvf = nx * (ny - 1);
        d.nu_tiles = (nuf + kThreads - 1) / kThreads;
        const int face_tiles = d.nu_tiles + (nvf + kThreads - 1) / kThreads;
        d.nstages = redi::domains::S_PAIR0 + 2 * npairs;
        d.ntiles[redi::domains::S_COLUMN] = (int)((ncol + kThreads - 1) / kThreads);
        d.ntiles[redi::domains::S_SWEEP] = face_tiles;
        d.ntiles[redi::domains::S_RECON] = (int)((ncol * npairs + kThreads - 1) / kThreads);
        for (int g = 0; g < npairs; ++g) d.ntiles[redi::domains::S_PAIR0 + 2 * g] = face_tiles;
        b->cost[k] = (double)ncol * nz * (2.0 + ntr);
        b->updates.push_back((long long)D.grid.nx_phys * D.grid.ny_phys * nz * ntr);
    }
    cudaError_t e = cudaMalloc(&b->d_doms, sizeof(DomainDev<P>) * n);
    if (e == cudaSuccess) b->allocs.push_back(b->d_doms), e = cudaMalloc((void**)&b->d_done, sizeof(int) * n * kMaxStages);
    if (e == cudaSuccess) b->allocs.push_back(b->d_done), e = cudaMalloc((void**)&b->d_held, sizeof(int) * n);
    if (e == cudaSuccess) b->allocs.push_back(b->d_held);
    if (e != cudaSuccess) return bfail(REDI_B200_E_NOMEM, std::string("redi_b200_batch_create: ") + cudaGetErrorString(e));
    cudaMemset(b->d_held, 0, sizeof(int) * n);
    cudaMemset(b->d_ctl, 0, sizeof(Control));
    const int rc = layout<P>(b);
    if (rc < 0) return rc;
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return bfail(REDI_B200_E_CUDA, std::string("redi_b200_batch_create: ") + cudaGetErrorString(e));
    return REDI_B200_OK;
}

// The counter reset and the persistent kernel. `instrument` brackets the
// kernel for the launch counter and event timing; a graph replay is bracketed
// by the caller instead (nothing runs on the host when a graph replays).
template <class P>
cudaError_t enqueue(redi_b200_batch* b, cudaStream_t st, bool instrument) {
    cudaError_t e = cudaMemsetAsync(b->d_done, 0, sizeof(int) * b->ndomains * kMaxStages, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_ctl, 0, sizeof(Control), st);
    if (e != cudaSuccess) return e;
    const auto* doms = static_cast<const DomainDev<P>*>(b->d_doms);
    if (instrument) redi::launch_begin(redi::K_DOMAIN_PERSISTENT, st);
    kernel_for<P>(b->chunk, b->occ)<<<b->grid, kThreads, 0, st>>>(doms, b->d_queue, b->nitems, b->d_done, b->d_held,
                                                                  b->d_ctl, b->limit_ns, b->bx, b->account);
    if (instrument) redi::launch_end(redi::K_DOMAIN_PERSISTENT, st);
    return cudaGetLastError();
}

cudaError_t enqueue_any(redi_b200_batch* b, cudaStream_t st, bool instrument) {
    return b->precision == REDI_B200_MIXED ? enqueue<redi::MixedPrec>(b, st, instrument)
                                           : enqueue<redi::PlainPrec>(b, st, instrument);
}

}  // namespace

extern "C" {

int redi_b200_batch_create(int ndomains, const redi_b200_domain* domains, int precision, int tile_bx, int tile_by,
                           int chunk, int use_graph, redi_b200_batch** out) {
    if (!out) return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: out is NULL");
    *out = nullptr;
    if (ndomains < 1 || ndomains > 32767 || !domains)
        return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: need 1..32767 domains");
    if (precision != REDI_B200_FP64 && precision != REDI_B200_MIXED)
        return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: bad precision");
    if (tile_bx < 1 || tile_by < 1 || tile_bx * tile_by != kThreads)
        return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: the gather tile must hold 128 cells");
    if (chunk != 4 && chunk != 8 && chunk != 16) return bfail(REDI_B200_E_ARG, "redi_b200_batch_create: chunk must be 4, 8 or 16");
    redi_b200_batch* b = new (std::nothrow) redi_b200_batch();
    if (!b) return bfail(REDI_B200_E_NOMEM, "redi_b200_batch_create: host allocation failed");
    b->precision = precision;
    b->ndomains = ndomains;
    b->bx = tile_bx;
    b->by = tile_by;
    b->chunk = chunk;
    b->use_graph = use_graph != 0;
    const int rc = precision == REDI_B200_MIXED ? build<redi::MixedPrec>(b, ndomains, domains)
                                                : build<redi::PlainPrec>(b, ndomains, domains);
    if (rc < 0) {
        free_batch(b);
        delete b;
        return rc;
    }
    *out = b;
    return REDI_B200_OK;
}

int redi_b200_batch_step(redi_b200_batch* b, void* stream) {
    if (!b) return bfail(REDI_B200_E_ARG, "redi_b200_batch_step: NULL batch");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (!b->use_graph) {
        cudaError_t e = enqueue_any(b, st, true);
        return e == cudaSuccess ? REDI_B200_OK : bfail(REDI_B200_E_CUDA, cudaGetErrorString(e));
    }
    if (!b->exec) {
        // Capture the step (counter reset + persistent kernel) once on a private stream.
        cudaStream_t cap;
        cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t ee = enqueue_any(b, cap, false);
            e = cudaStreamEndCapture(cap, &b->graph);
            if (ee != cudaSuccess) e = ee;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) return bfail(REDI_B200_E_CUDA, std::string("redi_b200_batch_step: graph: ") + cudaGetErrorString(e));
    }
    redi::launch_begin(redi::K_DOMAIN_PERSISTENT, st);
    cudaError_t e = cudaGraphLaunch(b->exec, st);
    redi::launch_end(redi::K_DOMAIN_PERSISTENT, st);
    return e == cudaSuccess ? REDI_B200_OK : bfail(REDI_B200_E_CUDA, cudaGetErrorString(e));
}

int redi_b200_batch_status(const redi_b200_batch* b, int* status, int* domain, int* stage, int* bad) {
    if (!b || !status) return bfail(REDI_B200_E_ARG, "redi_b200_batch_status: NULL argument");
    Control c{};
    cudaError_t e = cudaMemcpy(&c, b->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bfail(REDI_B200_E_CUDA, cudaGetErrorString(e));
    *status = c.status;
    if (domain) *domain = c.t_domain;
    if (stage) *stage = c.t_stage;
    if (bad) *bad = c.bad;
    return REDI_B200_OK;
}

int redi_b200_batch_set_wait_limit(redi_b200_batch* b, long long ns) {
    if (!b || ns <= 0) return bfail(REDI_B200_E_ARG, "redi_b200_batch_set_wait_limit: bad argument");
    drop_graph(b);
    b->limit_ns = (unsigned long long)ns;
    return REDI_B200_OK;
}

int redi_b200_batch_set_tuning(redi_b200_batch* b, int tile_bx, int tile_by, int chunk, int occupancy) {
    if (!b) return bfail(REDI_B200_E_ARG, "redi_b200_batch_set_tuning: NULL batch");
    if (tile_bx < 1 || tile_by < 1 || tile_bx * tile_by != kThreads)
        return bfail(REDI_B200_E_ARG, "redi_b200_batch_set_tuning: the gather tile must hold 128 cells");
    if (chunk != 4 && chunk != 8 && chunk != 16)
        return bfail(REDI_B200_E_ARG, "redi_b200_batch_set_tuning: chunk must be 4, 8 or 16");
    if (occupancy != 0 && (occupancy < 4 || occupancy > 6))
        return bfail(REDI_B200_E_ARG, "redi_b200_batch_set_tuning: occupancy must be 4, 5 or 6 (0: keep)");
    cudaError_t e = cudaDeviceSynchronize();  // the queue may be in use by a step in flight
    if (e != cudaSuccess) return bfail(REDI_B200_E_CUDA, cudaGetErrorString(e));
    b->bx = tile_bx;
    b->by = tile_by;
    b->chunk = chunk;
    if (occupancy) b->occ = occupancy;
    return layout_any(b);
}

int redi_b200_batch_get_tuning(const redi_b200_batch* b, int* tile_bx, int* tile_by, int* chunk, int* occupancy,
                               int* grid) {
    if (!b) return bfail(REDI_B200_E_ARG, "redi_b200_batch_get_tuning: NULL batch");
    if (tile_bx) *tile_bx = b->bx;
    if (tile_by) *tile_by = b->by;
    if (chunk) *chunk = b->chunk;
    if (occupancy) *occupancy = b->occ;
    if (grid) *grid = b->grid;
    return REDI_B200_OK;
}

int redi_b200_batch_set_accounting(redi_b200_batch* b, int on) {
    if (!b) return bfail(REDI_B200_E_ARG, "redi_b200_batch_set_accounting: NULL batch");
    if ((on != 0) != (b->account != 0)) drop_graph(b);
    b->account = on != 0;
    return REDI_B200_OK;
}

int redi_b200_batch_stage_times(const redi_b200_batch* b, double* wait_ms, double* busy_ms, long long* tiles) {
    if (!b) return bfail(REDI_B200_E_ARG, "redi_b200_batch_stage_times: NULL batch");
    Control c{};
    cudaError_t e = cudaMemcpy(&c, b->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bfail(REDI_B200_E_CUDA, cudaGetErrorString(e));
    for (int k = 0; k < redi::domains::kStageKinds; ++k) {
        if (wait_ms) wait_ms[k] = c.wait_ns[k] * 1e-6;
        if (busy_ms) busy_ms[k] = c.busy_ns[k] * 1e-6;
        if (tiles) tiles[k] = (long long)c.tiles[k];
    }
    return REDI_B200_OK;
}

int redi_b200_batch_hold(redi_b200_batch* b, int domain, int hold) {
    if (!b || domain < 0 || domain >= b->ndomains) return bfail(REDI_B200_E_ARG, "redi_b200_batch_hold: bad domain");
    const int v = hold != 0;
    cudaError_t e = cudaMemcpy(b->d_held + domain, &v, sizeof(int), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? REDI_B200_OK : bfail(REDI_B200_E_CUDA, cudaGetErrorString(e));
}

long long redi_b200_batch_updates(const redi_b200_batch* b) {
    if (!b) return 0;
    long long s = 0;
    for (long long u : b->updates) s += u;
    return s;
}

long long redi_b200_batch_items(const redi_b200_batch* b) { return b ? b->nitems : 0; }

int redi_b200_batch_destroy(redi_b200_batch* b) {
    if (!b) return REDI_B200_OK;
    free_batch(b);
    delete b;
    return REDI_B200_OK;
}

}  // extern "C"
