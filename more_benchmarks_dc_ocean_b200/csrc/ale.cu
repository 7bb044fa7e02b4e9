// The ALE remap step on sm_100a: ale_remap_step (ale_remap/ale_remap.F90:76-188)
// in two kernels over tiles of columns staged in shared memory.
//
//   k_ale_columns  a block per tile of adjacent cell columns: the column total
//                  (L1), h_ref (L2), the h_old snapshot (L3) and the zstar
//                  targets (L4, :478-527); every tracer of the launch remapped
//                  over the tile's geometry (L5/L6, ocean_remap_tracer_field
//                  :530-581, heat / salt budgets); the commit (L9 mass budget,
//                  h_layer = target_h, L10 bt_eta).
//   k_ale_faces    a block per tile of u faces or v faces: face thicknesses
//                  from the two adjacent cells, remap of the velocity, optional
//                  KE-conserving rescale (L7/L8, :584-724).
//
// The column remap is remap_column (ale_remap/kernel_remap.F90:43-376) for PCM,
// PLM and PPM. The reference sweeps each column serially: for new layer k it
// walks the old layers from a start index carried over from layer k-1 and sums
// the pieces whose overlap is positive. When every old and new thickness of a
// column is >= 0 both sets of interface depths are non-decreasing, and the old
// layers with positive overlap with new layer k are exactly those in the
// contiguous range [first old layer whose top lies above z_new(k-1), last old
// layer whose bottom lies below z_new(k)]; summed in increasing order they give
// the reference's integral bit for bit. So each (column, new layer) is computed
// by its own thread from the tile in shared memory (a binary search finds the
// range). A column with a negative or NaN thickness takes the reference's serial
// sweep instead, on one thread, from the same tile. PLM slopes and PPM edge /
// limiter coefficients of an old layer depend only on the averages two layers
// either side (the reference's limiter loop has no dependency between layers)
// and are evaluated where a piece needs them. The column total is the last old
// interface depth: the same additions in the same order.
// Compiled with -fmad=false: results are the reference's IEEE sequence.

#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <string>
#include <vector>

#include "ale_b200.h"
#include "redi_kernels.h"

namespace {

constexpr double kHFloor = 1.5e-4;  // ale_remap/ale_remap.F90:70 H_FLOOR
constexpr int kNzMax = ALE_B200_NZ_MAX;
constexpr int kThreads = 256;  // with a 64-register cap: four blocks per SM
constexpr int kMaxTracers = 8;  // tracers remapped by one launch
constexpr int kPCM = 1, kPLM = 2, kPPM = 3;

thread_local std::string g_err;

struct Dims {
    int nx, ny, nz, conserve_ke;
    int n2;  // cells per layer (every offset of a step fits in 32 bits: checked on the host)
};

struct TracerSet {
    int n;
    double* tr[kMaxTracers];
    double* budget[kMaxTracers];
};

// A column of a tile in shared memory: element k at p[k * S].
template <int S>
struct Col {
    const double* p;
    __device__ __forceinline__ double operator[](int k) const { return p[k * S]; }
};

// Tile width (columns) for a column capacity: the staged arrays stay within the shared memory of a block.
template <int CAP>
struct Tile {
    static constexpr int W = CAP <= 64 ? 32 : 16;
};

// PLM slope of old layer ko (1-based), kernel_remap.F90:163-174
template <class A>
__device__ __forceinline__ double plm_slope(const A& q, int nz, int ko) {
    if (ko == 1 || ko == nz) return 0.0;
    const double dq_l = q[ko - 1] - q[ko - 2];
    const double dq_r = q[ko] - q[ko - 1];
    if (dq_l * dq_r > 0.0) return 0.5 * copysign(fmin(fabs(dq_l), fabs(dq_r)), dq_l);
    return 0.0;
}

// Limited PPM edges and curvature of old layer ko (1-based), nz >= 3:
// kernel_remap.F90:257-328 evaluated for one layer.
template <class A>
__device__ __forceinline__ void ppm_coeffs(const A& q, int nz, int ko, double& qL, double& qR, double& q6) {
    const double qc = q[ko - 1];
    double l, r;
    if (ko == 1) {
        l = qc;
    } else if (ko == 2) {
        l = 0.5 * (q[0] + q[1]);  // q_L(2) = q_R(1)
    } else {                      // the interior edge between layers ko-1 and ko
        const int k = ko - 1;
        l = 0.5 * (q[k - 1] + q[k]);
        if (k + 2 <= nz) l = (7.0 / 12.0) * (q[k - 1] + q[k]) - (1.0 / 12.0) * (q[k - 2] + q[k + 1]);
    }
    if (ko == nz) {
        r = qc;
    } else if (ko == 1) {
        r = 0.5 * (q[0] + q[1]);
    } else {  // the interior edge between layers ko and ko+1
        const int k = ko;
        r = 0.5 * (q[k - 1] + q[k]);
        if (k + 2 <= nz) r = (7.0 / 12.0) * (q[k - 1] + q[k]) - (1.0 / 12.0) * (q[k - 2] + q[k + 1]);
    }
    double q_min = qc, q_max = qc;
    if (ko > 1) {
        q_min = fmin(q_min, q[ko - 2]);
        q_max = fmax(q_max, q[ko - 2]);
    }
    if (ko < nz) {
        q_min = fmin(q_min, q[ko]);
        q_max = fmax(q_max, q[ko]);
    }
    l = fmax(q_min, fmin(q_max, l));
    r = fmax(q_min, fmin(q_max, r));
    const double dq = r - l;
    const double dq_l = qc - l;
    const double dq_r = r - qc;
    if (dq_l * dq_r <= 0.0) {
        l = qc;
        r = qc;
    } else {
        const double s6 = 6.0 * qc - 3.0 * (l + r);
        if (fabs(s6) > fabs(dq)) {
            if (s6 * dq > 0.0)
                l = 3.0 * qc - 2.0 * r;
            else
                r = 3.0 * qc - 2.0 * l;
        }
    }
    qL = l;
    qR = r;
    q6 = 6.0 * qc - 3.0 * (l + r);
}

// Old layer ko's contribution to a new layer: the integral of its
// reconstruction over [z_lo, z_hi] (kernel_remap.F90:107, 193-204, 349-362).
template <int M, class A>
__device__ __forceinline__ double piece(const A& q, const A& dz_old, int nz, int ko, double zo_lo, double z_lo,
                                        double z_hi, double overlap) {
    const double qo = q[ko - 1];
    if (M == kPCM) return qo * overlap;
    const double d = dz_old[ko - 1];
    if (!(d > 0.0)) return qo * overlap;
    const double xi_lo = (z_lo - zo_lo) / d;
    const double xi_hi = (z_hi - zo_lo) / d;
    if (M == kPLM) return overlap * (qo + plm_slope(q, nz, ko) * (xi_lo + xi_hi - 1.0));
    double cL, cR, c6;
    ppm_coeffs(q, nz, ko, cL, cR, c6);
    return d * ((xi_hi - xi_lo) * cL + 0.5 * (xi_hi * xi_hi - xi_lo * xi_lo) * (cR - cL + c6) -
                (xi_hi * xi_hi * xi_hi - xi_lo * xi_lo * xi_lo) * c6 / 3.0);
}

// The new average of layer k (0-based) of a monotone column: the pieces of the
// old layers overlapping it, summed in increasing order. z_old / z_new hold the
// interface depths 0..nz.
template <int METHOD, class A>
__device__ __forceinline__ double new_layer(int nz, const A& dz_old, const A& z_old, const A& dz_new, const A& z_new,
                                            const A& q, int k) {
    if (METHOD != kPCM && nz == 1) return q[0];
    constexpr int M2 = METHOD == kPPM ? kPLM : METHOD;  // two layers: PPM reduces to PLM
    const double dzn = dz_new[k];
    if (dzn <= 0.0) return 0.0;
    const double zn_lo = z_new[k], zn_hi = z_new[k + 1];
    int lo = 1, hi = nz + 1;  // first ko in [1, nz] with z_old[ko] > zn_lo (nz + 1: none)
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (z_old[mid] > zn_lo)
            hi = mid;
        else
            lo = mid + 1;
    }
    double integral = 0.0;
    for (int ko = lo; ko <= nz; ++ko) {
        const double zo_lo = z_old[ko - 1];
        if (!(zo_lo < zn_hi)) break;
        const double zo_hi = z_old[ko];
        const double z_lo = fmax(zn_lo, zo_lo);
        const double z_hi = fmin(zn_hi, zo_hi);
        const double overlap = z_hi - z_lo;
        if (overlap <= 0.0) continue;
        integral = integral + (METHOD == kPPM && nz == 2 ? piece<M2>(q, dz_old, nz, ko, zo_lo, z_lo, z_hi, overlap)
                                                         : piece<METHOD>(q, dz_old, nz, ko, zo_lo, z_lo, z_hi, overlap));
    }
    return integral / dzn;
}

// The reference's serial sweep (remap_column), for columns with a negative or NaN thickness.
template <int METHOD, class A, class Emit>
__device__ void serial_column(int nz, const A& dz_old, const A& z_old, const A& dz_new, const A& q, Emit emit) {
    if (METHOD != kPCM && nz == 1) {
        emit(0, q[0]);
        return;
    }
    constexpr int M2 = METHOD == kPPM ? kPLM : METHOD;
    int ko_start = 1;
    double zn_prev = 0.0;
    for (int k = 1; k <= nz; ++k) {
        const double dzn = dz_new[k - 1];
        const double zn = zn_prev + dzn;
        if (dzn <= 0.0) {
            emit(k - 1, 0.0);
            zn_prev = zn;
            continue;
        }
        double integral = 0.0;
        for (int ko = ko_start; ko <= nz; ++ko) {
            const double zo_lo = z_old[ko - 1];
            const double zo_hi = z_old[ko];
            const double z_lo = fmax(zn_prev, zo_lo);
            const double z_hi = fmin(zn, zo_hi);
            const double overlap = z_hi - z_lo;
            if (overlap <= 0.0) {
                if (zo_hi > zn) break;
                continue;
            }
            integral = integral + (METHOD == kPPM && nz == 2
                                       ? piece<M2>(q, dz_old, nz, ko, zo_lo, z_lo, z_hi, overlap)
                                       : piece<METHOD>(q, dz_old, nz, ko, zo_lo, z_lo, z_hi, overlap));
            if (zo_hi <= zn) ko_start = ko;
        }
        emit(k - 1, integral / dzn);
        zn_prev = zn;
    }
}

// rescale_anomaly_ke (ale_remap/ale_remap.F90:684-724) on one column of a tile
template <int stride>
__device__ void rescale_anomaly_ke(int nz, const Col<stride>& h_old, const Col<stride>& h_new,
                                   const Col<stride>& u_old, double* u_new) {
    double h_old_sum = 0.0, h_new_sum = 0.0, mom_old = 0.0, mom_new = 0.0;
    for (int k = 0; k < nz; ++k) {
        h_old_sum = h_old_sum + h_old[k];
        h_new_sum = h_new_sum + h_new[k];
        mom_old = mom_old + h_old[k] * u_old[k];
        mom_new = mom_new + h_new[k] * u_new[k * stride];
    }
    if (h_old_sum <= kHFloor || h_new_sum <= kHFloor) return;
    const double u_bar_old = mom_old / h_old_sum;
    const double u_bar_new = mom_new / h_new_sum;
    double ke_old = 0.0, ke_new = 0.0;
    for (int k = 0; k < nz; ++k) {
        double anom = u_old[k] - u_bar_old;
        ke_old = ke_old + 0.5 * h_old[k] * anom * anom;
        anom = u_new[k * stride] - u_bar_new;
        ke_new = ke_new + 0.5 * h_new[k] * anom * anom;
    }
    if (ke_new <= 0.0 || ke_old <= 0.0) return;
    double scale_fac = sqrt(ke_old / ke_new);
    if (scale_fac > 1.25) scale_fac = 1.25;
    if (scale_fac < 0.0) scale_fac = 0.0;
    for (int k = 0; k < nz; ++k) u_new[k * stride] = u_bar_new + scale_fac * (u_new[k * stride] - u_bar_new);
}

// Interface depths of every column of the tile (one thread per column), and
// whether the column is monotone (every thickness >= 0).
template <int W>
__device__ __forceinline__ void tile_depths(int nz, int ncol, const double* dzo, const double* dzn, double* zo,
                                            double* zn, int* serial) {
    const int c = threadIdx.x;
    if (c >= ncol) return;
    double a = 0.0, b = 0.0;
    bool mono = true;
    zo[c] = 0.0;
    zn[c] = 0.0;
    for (int k = 0; k < nz; ++k) {
        const double x = dzo[k * W + c], y = dzn[k * W + c];
        mono = mono && x >= 0.0 && y >= 0.0;
        a = a + x;
        b = b + y;
        zo[(k + 1) * W + c] = a;
        zn[(k + 1) * W + c] = b;
    }
    serial[c] = mono ? 0 : 1;
}

// ----------------------------------------------------------------- kernels --
// Tile of cell columns. pre: compute the snapshot and the targets from h_layer
// (the first launch of a step); otherwise read them back. commit: the last launch.
template <int METHOD, int CAP>
__global__ void __launch_bounds__(kThreads, 4) k_ale_columns(const Dims d, const TracerSet ts, int pre, int commit,
                                                          double* h_layer, double* bt_eta,
                                                          const double* __restrict__ bt_H_ref,
                                                          const double* __restrict__ dsig, double* total_h,
                                                          double* h_ref, double* h_old, double* target_h,
                                                          double* mass_budget) {
    constexpr int W = Tile<CAP>::W;
    extern __shared__ double sm[];
    double* dzo = sm;                 // [CAP][W]
    double* dzn = dzo + CAP * W;      // [CAP][W]
    double* zo = dzn + CAP * W;       // [CAP + 1][W]
    double* zn = zo + (CAP + 1) * W;  // [CAP + 1][W]
    double* q = zn + (CAP + 1) * W;   // [CAP][W]
    __shared__ int serial[W];
    __shared__ double ct[W];  // column total h_ref + eta of the zstar target
    const int nz = d.nz;
    const int n2 = d.n2;
    const int t0 = blockIdx.x * W;
    const int ncol = (int)(n2 - t0 < W ? n2 - t0 : W);
    const int ne = nz * W;

    for (int e = threadIdx.x; e < ne; e += kThreads) {
        const int k = e / W, c = e - k * W;
        if (c < ncol) dzo[e] = pre ? h_layer[t0 + c + n2 * k] : __ldg(h_old + t0 + c + n2 * k);
    }
    __syncthreads();
    if (pre) {
        // L1 total (the running sum of the column: the last interface depth), L2 h_ref, L4 column total
        if (threadIdx.x < ncol) {
            const int c = threadIdx.x;
            double s = 0.0;
            for (int k = 0; k < nz; ++k) s = s + dzo[k * W + c];
            const double e = bt_eta[t0 + c];
            const double hr = s - e;
            if (total_h) total_h[t0 + c] = s;
            if (h_ref) h_ref[t0 + c] = hr;
            ct[c] = hr + e;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < ne; e += kThreads) {  // L3 snapshot, L4 targets
            const int k = e / W, c = e - k * W;
            if (c >= ncol) continue;
            const double tg = ct[c] * __ldg(dsig + k);
            dzn[e] = tg;
            h_old[t0 + c + n2 * k] = dzo[e];
            target_h[t0 + c + n2 * k] = tg;
        }
    } else {
        for (int e = threadIdx.x; e < ne; e += kThreads) {
            const int k = e / W, c = e - k * W;
            if (c < ncol) dzn[e] = __ldg(target_h + t0 + c + n2 * k);
        }
    }
    __syncthreads();
    tile_depths<W>(nz, ncol, dzo, dzn, zo, zn, serial);
    __syncthreads();

    for (int n = 0; n < ts.n; ++n) {
        double* hTr = ts.tr[n];
        double* budget = ts.budget[n];
        for (int e = threadIdx.x; e < ne; e += kThreads) {
            const int k = e / W, c = e - k * W;
            if (c >= ncol) continue;
            const double h = dzo[e];
            q[e] = h > kHFloor ? hTr[t0 + c + n2 * k] / h : 0.0;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < ne; e += kThreads) {
            const int k = e / W, c = e - k * W;
            if (c >= ncol || serial[c]) continue;
            const double cn = new_layer<METHOD>(nz, Col<W>{dzo + c}, Col<W>{zo + c}, Col<W>{dzn + c},
                                                Col<W>{zn + c}, Col<W>{q + c}, k);
            const int o = t0 + c + n2 * k;
            const double hTr_new = cn * dzn[e];
            if (budget) budget[o] = budget[o] + (hTr_new - hTr[o]);
            hTr[o] = hTr_new;
        }
        if (threadIdx.x < ncol && serial[threadIdx.x]) {
            const int c = threadIdx.x;
            serial_column<METHOD>(nz, Col<W>{dzo + c}, Col<W>{zo + c}, Col<W>{dzn + c}, Col<W>{q + c},
                                  [&](int k, double cn) {
                                      const int o = t0 + c + n2 * k;
                                      const double hTr_new = cn * dzn[k * W + c];
                                      if (budget) budget[o] = budget[o] + (hTr_new - hTr[o]);
                                      hTr[o] = hTr_new;
                                  });
        }
        __syncthreads();  // q is reused by the next tracer
    }

    if (commit) {
        for (int e = threadIdx.x; e < ne; e += kThreads) {  // L9
            const int k = e / W, c = e - k * W;
            if (c >= ncol) continue;
            const int o = t0 + c + n2 * k;
            mass_budget[o] = mass_budget[o] + (dzn[e] - dzo[e]);
            h_layer[o] = dzn[e];
        }
        if (threadIdx.x < ncol) {  // L10
            const int c = threadIdx.x;
            double e = -__ldg(bt_H_ref + t0 + c);
            for (int k = 0; k < nz; ++k) e = e + dzn[k * W + c];
            bt_eta[t0 + c] = e;
        }
    }
}

// Tile of u faces (blocks [0, nbu)) or v faces (the rest).
template <int METHOD, int CAP>
__global__ void __launch_bounds__(kThreads, 4) k_ale_faces(const Dims d, int nbu, const double* __restrict__ h_old,
                                                        const double* __restrict__ target_h, double* u, double* v) {
    constexpr int W = Tile<CAP>::W;
    extern __shared__ double sm[];
    double* dzo = sm;
    double* dzn = dzo + CAP * W;
    double* zo = dzn + CAP * W;
    double* zn = zo + (CAP + 1) * W;
    double* q = zn + (CAP + 1) * W;
    double* qn = q + CAP * W;  // new values, when the KE rescale needs the whole column
    __shared__ int serial[W];
    __shared__ int cell_l[W], cell_r[W];
    __shared__ int edge[W];
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int n2 = d.n2;
    const bool xface = (int)blockIdx.x < nbu;
    const int nf = xface ? (nx + 1) * ny : nx * (ny + 1);
    const int f0 = (xface ? (int)blockIdx.x : (int)blockIdx.x - nbu) * W;
    const int ncol = (int)(nf - f0 < W ? nf - f0 : W);
    double* field = xface ? u : v;
    const int ne = nz * W;

    if (threadIdx.x < ncol) {
        const int f = f0 + threadIdx.x;
        if (xface) {  // remap_x_face_velocity
            const int I = (int)(f % (nx + 1)), j = (int)(f / (nx + 1));
            edge[threadIdx.x] = I == 0 || I == nx;
            cell_l[threadIdx.x] = (I == 0 ? 0 : I - 1) + nx * j;
            cell_r[threadIdx.x] = (I == nx ? nx - 1 : I) + nx * j;
        } else {  // remap_y_face_velocity
            const int i = (int)(f % nx), J = (int)(f / nx);
            edge[threadIdx.x] = J == 0 || J == ny;
            cell_l[threadIdx.x] = i + nx * (J == 0 ? 0 : J - 1);
            cell_r[threadIdx.x] = i + nx * (J == ny ? ny - 1 : J);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ne; e += kThreads) {
        const int k = e / W, c = e - k * W;
        if (c >= ncol) continue;
        const int l = cell_l[c] + n2 * k, r = cell_r[c] + n2 * k;
        if (edge[c]) {
            dzo[e] = __ldg(h_old + l);
            dzn[e] = __ldg(target_h + l);
        } else {
            dzo[e] = 0.5 * (__ldg(h_old + l) + __ldg(h_old + r));
            dzn[e] = 0.5 * (__ldg(target_h + l) + __ldg(target_h + r));
        }
        q[e] = field[f0 + c + nf * k];
    }
    __syncthreads();
    tile_depths<W>(nz, ncol, dzo, dzn, zo, zn, serial);
    __syncthreads();
    const bool ke = d.conserve_ke != 0;
    for (int e = threadIdx.x; e < ne; e += kThreads) {
        const int k = e / W, c = e - k * W;
        if (c >= ncol || serial[c]) continue;
        const double val = new_layer<METHOD>(nz, Col<W>{dzo + c}, Col<W>{zo + c}, Col<W>{dzn + c}, Col<W>{zn + c},
                                             Col<W>{q + c}, k);
        if (ke)
            qn[e] = val;
        else
            field[f0 + c + nf * k] = val;
    }
    if (threadIdx.x < ncol && serial[threadIdx.x]) {
        const int c = threadIdx.x;
        serial_column<METHOD>(nz, Col<W>{dzo + c}, Col<W>{zo + c}, Col<W>{dzn + c}, Col<W>{q + c},
                              [&](int k, double val) {
                                  if (ke)
                                      qn[k * W + c] = val;
                                  else
                                      field[f0 + c + nf * k] = val;
                              });
    }
    if (!ke) return;
    __syncthreads();
    if (threadIdx.x < ncol) {
        const int c = threadIdx.x;
        rescale_anomaly_ke<W>(nz, Col<W>{dzo + c}, Col<W>{dzn + c}, Col<W>{q + c}, qn + c);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ne; e += kThreads) {
        const int k = e / W, c = e - k * W;
        if (c < ncol) field[f0 + c + nf * k] = qn[e];
    }
}

// -------------------------------------------------------------------- host --
int fail(int code, const std::string& msg) {
    g_err = msg;
    redi::set_last_error(msg);
    return code;
}

template <int CAP>
constexpr size_t column_smem() {
    return sizeof(double) * (size_t)Tile<CAP>::W * (3 * CAP + 2 * (CAP + 1));
}
template <int CAP>
constexpr size_t face_smem() {
    return column_smem<CAP>() + sizeof(double) * (size_t)Tile<CAP>::W * CAP;
}

template <int METHOD, int CAP>
cudaError_t allow_smem() {
    static cudaError_t once = [] {
        cudaError_t e = cudaFuncSetAttribute(k_ale_columns<METHOD, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)column_smem<CAP>());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_ale_faces<METHOD, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)face_smem<CAP>());
        return e;
    }();
    return once;
}

template <int METHOD, int CAP>
int launch(const ale_b200_step_args& a, cudaStream_t st) {
    constexpr int W = Tile<CAP>::W;
    cudaError_t e = allow_smem<METHOD, CAP>();
    if (e != cudaSuccess) return fail(ALE_B200_E_CUDA, std::string("ale: shared memory: ") + cudaGetErrorString(e));
    const Dims d{a.nx, a.ny, a.nz, a.conserve_ke ? 1 : 0, a.nx * a.ny};
    std::vector<TracerSet> sets;
    TracerSet cur{};
    for (int n = 0; n < a.ntracers; ++n) {
        if (!a.tracers[n]) continue;
        cur.tr[cur.n] = a.tracers[n];
        cur.budget[cur.n] = n == a.idx_temperature ? a.heat_budget : n == a.idx_salinity ? a.salt_budget : nullptr;
        if (++cur.n == kMaxTracers) {
            sets.push_back(cur);
            cur = TracerSet{};
        }
    }
    if (cur.n > 0 || sets.empty()) sets.push_back(cur);
    const int nb = (int)((d.n2 + W - 1) / W);
    for (size_t s = 0; s < sets.size(); ++s) {
        redi::launch_begin(redi::K_ALE_COLUMNS, st);
        k_ale_columns<METHOD, CAP><<<nb, kThreads, column_smem<CAP>(), st>>>(
            d, sets[s], s == 0 ? 1 : 0, s + 1 == sets.size() ? 1 : 0, a.h_layer, a.bt_eta, a.bt_H_ref, a.dsig,
            a.total_h, a.h_ref, a.h_old, a.target_h, a.mass_budget);
        redi::launch_end(redi::K_ALE_COLUMNS, st);
    }
    if (a.u && a.v) {
        const long long nu = (long long)(a.nx + 1) * a.ny, nv = (long long)a.nx * (a.ny + 1);
        const int nbu = (int)((nu + W - 1) / W), nbv = (int)((nv + W - 1) / W);
        redi::launch_begin(redi::K_ALE_FACES, st);
        k_ale_faces<METHOD, CAP><<<nbu + nbv, kThreads, face_smem<CAP>(), st>>>(d, nbu, a.h_old, a.target_h, a.u,
                                                                                a.v);
        redi::launch_end(redi::K_ALE_FACES, st);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ALE_B200_E_CUDA, std::string("ale: launch: ") + cudaGetErrorString(e));
    return ALE_B200_OK;
}

template <int METHOD>
int launch_cap(const ale_b200_step_args& a, cudaStream_t st) {
    if (a.nz <= 32) return launch<METHOD, 32>(a, st);
    if (a.nz <= 64) return launch<METHOD, 64>(a, st);
    return launch<METHOD, kNzMax>(a, st);
}

int run(const ale_b200_step_args* a, cudaStream_t st) {
    if (!a) return fail(ALE_B200_E_ARG, "ale: NULL argument block");
    if (a->nx < 1 || a->ny < 1 || a->nz < 1) return fail(ALE_B200_E_ARG, "ale: nx, ny, nz must be >= 1");
    if (a->nz > kNzMax) return fail(ALE_B200_E_ARG, "ale: nz exceeds ALE_B200_NZ_MAX (the reference's NZ_STACK_MAX)");
    if ((long long)(a->nx + 1) * (a->ny + 1) * a->nz > (long long)INT_MAX - 1024)
        return fail(ALE_B200_E_ARG, "ale: domain too large for 32-bit offsets");
    if (a->method == 4 || a->method == 5)
        return fail(ALE_B200_E_UNSUPPORTED, "ale: REMAP_PPM_H4 and REMAP_PQM are not implemented");
    if (!a->h_layer || !a->mass_budget || !a->bt_eta || !a->bt_H_ref || !a->dsig || !a->h_old || !a->target_h)
        return fail(ALE_B200_E_ARG, "ale: a required array pointer is NULL");
    if (a->ntracers < 0 || (a->ntracers > 0 && !a->tracers)) return fail(ALE_B200_E_ARG, "ale: bad tracer table");
    for (int n = 0; n < a->ntracers; ++n) {
        if (!a->tracers[n]) continue;
        if ((n == a->idx_temperature && !a->heat_budget) || (n == a->idx_salinity && !a->salt_budget))
            return fail(ALE_B200_E_ARG, "ale: heat / salt budget NULL for the temperature / salinity slot");
    }
    int rc;
    if (a->method == kPCM)
        rc = launch_cap<kPCM>(*a, st);
    else if (a->method == kPPM)
        rc = launch_cap<kPPM>(*a, st);
    else
        rc = launch_cap<kPLM>(*a, st);  // REMAP_PLM and the select-case default
    if (rc == ALE_B200_OK) g_err.clear();
    return rc;
}

void report(const char* who, int rc) {
    if (rc < 0) std::fprintf(stderr, "%s: %s\n", who, g_err.c_str());
}

}  // namespace

extern "C" {

int ale_b200_remap_step(const ale_b200_step_args* args, void* stream) {
    return run(args, static_cast<cudaStream_t>(stream));
}

const char* ale_b200_last_error(void) { return g_err.c_str(); }

void ale_remap_cuda(int nx, int ny, int nz, int method, int fused, double* h_layer, double* h_old, double* target_h,
                    double* total_h, double* h_ref, double* hTr_t, double* hTr_s, double* u, double* v,
                    double* mass_b, double* heat_b, double* salt_b, double* eta, double* H_ref, double* dsig) {
    (void)fused;  // the reference's faithful and fused forms give the same results
    double* tr[2] = {hTr_t, hTr_s};
    const ale_b200_step_args a{nx,     ny,     nz,     method, 0,      2,     0,      1,      h_layer, tr,
                               u,      v,      mass_b, heat_b, salt_b, eta,   H_ref,  dsig,   total_h, h_ref,
                               h_old,  target_h};
    report("ale_remap_cuda", run(&a, nullptr));
}

void ale_remap_opt(int nx, int ny, int nz, double* h_layer, double* h_old, double* target_h, double* hTr_t,
                   double* hTr_s, double* u, double* v, double* mass_b, double* heat_b, double* salt_b, double* eta,
                   double* H_ref, double* dsig) {
    double* tr[2] = {hTr_t, hTr_s};
    const ale_b200_step_args a{nx,     ny,     nz,     kPPM,   0,      2,       0,      1,       h_layer, tr,
                               u,      v,      mass_b, heat_b, salt_b, eta,     H_ref,  dsig,    nullptr, nullptr,
                               h_old,  target_h};
    report("ale_remap_opt", run(&a, nullptr));
}

void cuda_sync(void) { cudaDeviceSynchronize(); }

}  // extern "C"
