// TEST INFRASTRUCTURE ONLY — the CPU oracle for the ALE remap step. Nothing in
// the product path links or calls this file; tests, smoke() and the CPU
// baseline of bench.py use it as the checker.
//
// A plain C++ restatement of `ale_remap_step` (ale_remap/ale_remap.F90:76-188),
// loop by loop, in the reference's order:
//   L1  column total            remap_total_h = sum_k h_layer
//   L2  h_ref                   remap_h_ref = total_h - bt_eta
//   L3  snapshot                remap_h_old = h_layer
//   L4  zstar target            target_h(k) = (h_ref + bt_eta) * dsig(k)   (:478-527)
//   L5/L6 tracers               ocean_remap_tracer_field (:530-581): c = hTr/h (0 below
//                               H_FLOOR), remap_column, hTr = c*h_new, heat / salt budgets
//   L7/L8 face velocities       remap_x/y_face_velocity (:584-681), optional
//                               rescale_anomaly_ke (:684-724)
//   L9  commit                  mass budget += target_h - h_old; h_layer = target_h
//   L10 bt_eta                  bt_eta = -bt_H_ref + sum_k h_layer
// with remap_column (ale_remap/kernel_remap.F90:43-68) for REMAP_PCM (:70-123),
// REMAP_PLM (:125-212) and REMAP_PPM (:214-376); the select-case default is PLM.
// REMAP_PPM_H4 and REMAP_PQM are not restated (status -2).
//
// Arithmetic follows the Fortran expressions operand for operand and the file
// is compiled with -ffp-contract=off. MIN / MAX / SIGN / ABS are fmin / fmax /
// copysign / fabs, as the reference's CUDA port writes them (ale_remap/ale_kernel.cu).

#include <cmath>
#include <cstddef>
#include <vector>

namespace {

constexpr double H_FLOOR = 1.5e-4;  // ale_remap/ale_remap.F90:70
enum { REMAP_PCM = 1, REMAP_PLM = 2, REMAP_PPM = 3, REMAP_PPM_H4 = 4, REMAP_PQM = 5 };

// The overlap sweep shared by the three methods (kernel_remap.F90:96-121,
// 176-210, 330-374): `piece(ko, z_lo, z_hi, overlap)` is old layer ko's
// contribution to the integral.
template <class Piece>
void sweep(int nz, const double* dz_old, const double* dz_new, double* q_new, Piece piece) {
    std::vector<double> z_old(nz + 1), z_new(nz + 1);
    z_old[0] = 0.0;
    z_new[0] = 0.0;
    for (int k = 1; k <= nz; ++k) {
        z_old[k] = z_old[k - 1] + dz_old[k - 1];
        z_new[k] = z_new[k - 1] + dz_new[k - 1];
    }
    int ko_start = 1;
    for (int k = 1; k <= nz; ++k) {
        if (dz_new[k - 1] <= 0.0) {
            q_new[k - 1] = 0.0;
            continue;
        }
        double integral = 0.0;
        for (int ko = ko_start; ko <= nz; ++ko) {
            const double z_lo = std::fmax(z_new[k - 1], z_old[ko - 1]);
            const double z_hi = std::fmin(z_new[k], z_old[ko]);
            const double overlap = z_hi - z_lo;
            if (overlap <= 0.0) {
                if (z_old[ko] > z_new[k]) break;
                continue;
            }
            integral = integral + piece(ko, z_lo, z_hi, overlap, z_old[ko - 1]);
            if (z_old[ko] <= z_new[k]) ko_start = ko;
        }
        q_new[k - 1] = integral / dz_new[k - 1];
    }
}

void remap_pcm(int nz, const double* dz_old, const double* dz_new, const double* q_old, double* q_new) {
    sweep(nz, dz_old, dz_new, q_new,
          [&](int ko, double, double, double overlap, double) { return q_old[ko - 1] * overlap; });
}

void remap_plm(int nz, const double* dz_old, const double* dz_new, const double* q_old, double* q_new) {
    if (nz == 1) {
        q_new[0] = q_old[0];
        return;
    }
    std::vector<double> slope(nz);
    slope[0] = 0.0;
    for (int k = 2; k <= nz - 1; ++k) {
        const double dq_l = q_old[k - 1] - q_old[k - 2];
        const double dq_r = q_old[k] - q_old[k - 1];
        if (dq_l * dq_r > 0.0)
            slope[k - 1] = 0.5 * std::copysign(std::fmin(std::fabs(dq_l), std::fabs(dq_r)), dq_l);
        else
            slope[k - 1] = 0.0;
    }
    slope[nz - 1] = 0.0;
    sweep(nz, dz_old, dz_new, q_new, [&](int ko, double z_lo, double z_hi, double overlap, double z_base) {
        const double d = dz_old[ko - 1];
        if (d > 0.0) {
            const double xi_lo = (z_lo - z_base) / d;
            const double xi_hi = (z_hi - z_base) / d;
            return overlap * (q_old[ko - 1] + slope[ko - 1] * (xi_lo + xi_hi - 1.0));
        }
        return q_old[ko - 1] * overlap;
    });
}

void remap_ppm(int nz, const double* dz_old, const double* dz_new, const double* q_old, double* q_new) {
    if (nz == 1) {
        q_new[0] = q_old[0];
        return;
    }
    if (nz == 2) {
        remap_plm(nz, dz_old, dz_new, q_old, q_new);
        return;
    }
    std::vector<double> qL(nz), qR(nz), q6(nz, 0.0);
    // step 1: edge values (1-based k in the comments of kernel_remap.F90:257-287)
    qL[0] = q_old[0];
    qR[nz - 1] = q_old[nz - 1];
    qR[0] = 0.5 * (q_old[0] + q_old[1]);
    qL[nz - 1] = 0.5 * (q_old[nz - 2] + q_old[nz - 1]);
    for (int k = 2; k <= nz - 1; ++k) {
        double edge = 0.5 * (q_old[k - 1] + q_old[k]);
        if (k - 1 >= 1 && k + 2 <= nz)
            edge = (7.0 / 12.0) * (q_old[k - 1] + q_old[k]) - (1.0 / 12.0) * (q_old[k - 2] + q_old[k + 1]);
        qR[k - 1] = edge;
        qL[k] = edge;
    }
    if (nz >= 3) qL[1] = qR[0];
    // step 2: Colella-Woodward limiting
    for (int k = 1; k <= nz; ++k) {
        double q_min = q_old[k - 1], q_max = q_old[k - 1];
        if (k > 1) {
            q_min = std::fmin(q_min, q_old[k - 2]);
            q_max = std::fmax(q_max, q_old[k - 2]);
        }
        if (k < nz) {
            q_min = std::fmin(q_min, q_old[k]);
            q_max = std::fmax(q_max, q_old[k]);
        }
        qL[k - 1] = std::fmax(q_min, std::fmin(q_max, qL[k - 1]));
        qR[k - 1] = std::fmax(q_min, std::fmin(q_max, qR[k - 1]));
        const double dq = qR[k - 1] - qL[k - 1];
        const double dq_l = q_old[k - 1] - qL[k - 1];
        const double dq_r = qR[k - 1] - q_old[k - 1];
        if (dq_l * dq_r <= 0.0) {
            qL[k - 1] = q_old[k - 1];
            qR[k - 1] = q_old[k - 1];
        } else {
            q6[k - 1] = 6.0 * q_old[k - 1] - 3.0 * (qL[k - 1] + qR[k - 1]);
            if (std::fabs(q6[k - 1]) > std::fabs(dq)) {
                if (q6[k - 1] * dq > 0.0)
                    qL[k - 1] = 3.0 * q_old[k - 1] - 2.0 * qR[k - 1];
                else
                    qR[k - 1] = 3.0 * q_old[k - 1] - 2.0 * qL[k - 1];
            }
        }
        q6[k - 1] = 6.0 * q_old[k - 1] - 3.0 * (qL[k - 1] + qR[k - 1]);
    }
    // step 3: integrate the parabolas over the new layers
    sweep(nz, dz_old, dz_new, q_new, [&](int ko, double z_lo, double z_hi, double overlap, double z_base) {
        const double d = dz_old[ko - 1];
        if (d > 0.0) {
            const double xi_lo = (z_lo - z_base) / d;
            const double xi_hi = (z_hi - z_base) / d;
            return d * ((xi_hi - xi_lo) * qL[ko - 1] +
                        0.5 * (xi_hi * xi_hi - xi_lo * xi_lo) * (qR[ko - 1] - qL[ko - 1] + q6[ko - 1]) -
                        (xi_hi * xi_hi * xi_hi - xi_lo * xi_lo * xi_lo) * q6[ko - 1] / 3.0);
        }
        return q_old[ko - 1] * overlap;
    });
}

bool remap_column(int method, int nz, const double* dz_old, const double* dz_new, const double* q_old,
                  double* q_new) {
    switch (method) {
        case REMAP_PCM: remap_pcm(nz, dz_old, dz_new, q_old, q_new); return true;
        case REMAP_PPM: remap_ppm(nz, dz_old, dz_new, q_old, q_new); return true;
        case REMAP_PPM_H4:
        case REMAP_PQM: return false;
        default: remap_plm(nz, dz_old, dz_new, q_old, q_new); return true;  // REMAP_PLM and the default case
    }
}

// rescale_anomaly_ke (ale_remap/ale_remap.F90:684-724)
void rescale_anomaly_ke(int nz, const double* h_old, const double* h_new, const double* u_old, double* u_new) {
    double h_old_sum = 0.0, h_new_sum = 0.0, mom_old = 0.0, mom_new = 0.0;
    for (int k = 0; k < nz; ++k) {
        h_old_sum = h_old_sum + h_old[k];
        h_new_sum = h_new_sum + h_new[k];
        mom_old = mom_old + h_old[k] * u_old[k];
        mom_new = mom_new + h_new[k] * u_new[k];
    }
    if (h_old_sum <= H_FLOOR || h_new_sum <= H_FLOOR) return;
    const double u_bar_old = mom_old / h_old_sum;
    const double u_bar_new = mom_new / h_new_sum;
    double ke_old = 0.0, ke_new = 0.0;
    for (int k = 0; k < nz; ++k) {
        double anom = u_old[k] - u_bar_old;
        ke_old = ke_old + 0.5 * h_old[k] * anom * anom;
        anom = u_new[k] - u_bar_new;
        ke_new = ke_new + 0.5 * h_new[k] * anom * anom;
    }
    if (ke_new <= 0.0 || ke_old <= 0.0) return;
    double scale_fac = std::sqrt(ke_old / ke_new);
    if (scale_fac > 1.25) scale_fac = 1.25;
    if (scale_fac < 0.0) scale_fac = 0.0;
    for (int k = 0; k < nz; ++k) u_new[k] = u_bar_new + scale_fac * (u_new[k] - u_bar_new);
}

}  // namespace

// Arrays are Fortran column-major: cells (nx, ny), layers (nx, ny, nz), u faces
// (nx+1, ny, nz), v faces (nx, ny+1, nz). tracers[t] may be null (an
// unallocated slot); heat / salt budgets go with tracers idx_temperature /
// idx_salinity (0-based; -1 = none). u / v null skips the face remap.
struct AleOracleArgs {
    int nx, ny, nz, method, conserve_ke, ntracers, idx_temperature, idx_salinity;
    double* h_layer;
    double** tracers;
    double *u, *v;
    double *mass_budget, *heat_budget, *salt_budget;
    double *bt_eta;
    const double *bt_H_ref, *dsig;
    double *total_h, *h_ref, *h_old, *target_h;  // vcoord workspaces (outputs)
};

extern "C" {

// One ale_remap_step. Returns 0, or -2 for a method that is not restated.
int ale_oracle_step(const AleOracleArgs* ap) {
    const AleOracleArgs& a = *ap;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const size_t n2 = (size_t)nx * ny;
    if (a.method == REMAP_PPM_H4 || a.method == REMAP_PQM) return -2;
    auto c3 = [&](int i, int j, int k) { return (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * (size_t)k); };
    // L1-L3
    for (size_t t = 0; t < n2; ++t) {
        double s = 0.0;
        for (int k = 0; k < nz; ++k) s = s + a.h_layer[t + n2 * k];
        a.total_h[t] = s;
    }
    for (size_t t = 0; t < n2; ++t) a.h_ref[t] = a.total_h[t] - a.bt_eta[t];
    for (size_t t = 0; t < n2 * nz; ++t) a.h_old[t] = a.h_layer[t];
    // L4 (zstar)
    for (int k = 0; k < nz; ++k)
        for (size_t t = 0; t < n2; ++t) {
            const double column_total = a.h_ref[t] + a.bt_eta[t];
            a.target_h[t + n2 * k] = column_total * a.dsig[k];
        }
    // L5/L6
    std::vector<double> ho(nz), hn(nz), co(nz), cn(nz), uo(nz), un(nz);
    for (int tr = 0; tr < a.ntracers; ++tr) {
        double* hTr = a.tracers[tr];
        if (!hTr) continue;
        double* budget = tr == a.idx_temperature ? a.heat_budget : tr == a.idx_salinity ? a.salt_budget : nullptr;
#pragma omp parallel for firstprivate(ho, hn, co, cn)
        for (long long t = 0; t < (long long)n2; ++t) {
            for (int k = 0; k < nz; ++k) {
                ho[k] = a.h_old[t + n2 * k];
                hn[k] = a.target_h[t + n2 * k];
                co[k] = ho[k] > H_FLOOR ? hTr[t + n2 * k] / ho[k] : 0.0;
            }
            remap_column(a.method, nz, ho.data(), hn.data(), co.data(), cn.data());
            for (int k = 0; k < nz; ++k) {
                const double hTr_new = cn[k] * hn[k];
                if (budget) budget[t + n2 * k] = budget[t + n2 * k] + (hTr_new - hTr[t + n2 * k]);
                hTr[t + n2 * k] = hTr_new;
            }
        }
    }
    // L7/L8
    if (a.u && a.v) {
#pragma omp parallel for firstprivate(ho, hn, uo, un)
        for (int j = 0; j < ny; ++j)
            for (int I = 0; I <= nx; ++I) {
                for (int k = 0; k < nz; ++k) {
                    if (I == 0) {
                        ho[k] = a.h_old[c3(0, j, k)];
                        hn[k] = a.target_h[c3(0, j, k)];
                    } else if (I == nx) {
                        ho[k] = a.h_old[c3(nx - 1, j, k)];
                        hn[k] = a.target_h[c3(nx - 1, j, k)];
                    } else {
                        ho[k] = 0.5 * (a.h_old[c3(I - 1, j, k)] + a.h_old[c3(I, j, k)]);
                        hn[k] = 0.5 * (a.target_h[c3(I - 1, j, k)] + a.target_h[c3(I, j, k)]);
                    }
                    uo[k] = a.u[(size_t)I + (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k)];
                }
                remap_column(a.method, nz, ho.data(), hn.data(), uo.data(), un.data());
                if (a.conserve_ke) rescale_anomaly_ke(nz, ho.data(), hn.data(), uo.data(), un.data());
                for (int k = 0; k < nz; ++k) a.u[(size_t)I + (size_t)(nx + 1) * ((size_t)j + (size_t)ny * k)] = un[k];
            }
#pragma omp parallel for firstprivate(ho, hn, uo, un)
        for (int J = 0; J <= ny; ++J)
            for (int i = 0; i < nx; ++i) {
                for (int k = 0; k < nz; ++k) {
                    if (J == 0) {
                        ho[k] = a.h_old[c3(i, 0, k)];
                        hn[k] = a.target_h[c3(i, 0, k)];
                    } else if (J == ny) {
                        ho[k] = a.h_old[c3(i, ny - 1, k)];
                        hn[k] = a.target_h[c3(i, ny - 1, k)];
                    } else {
                        ho[k] = 0.5 * (a.h_old[c3(i, J - 1, k)] + a.h_old[c3(i, J, k)]);
                        hn[k] = 0.5 * (a.target_h[c3(i, J - 1, k)] + a.target_h[c3(i, J, k)]);
                    }
                    uo[k] = a.v[(size_t)i + (size_t)nx * ((size_t)J + (size_t)(ny + 1) * k)];
                }
                remap_column(a.method, nz, ho.data(), hn.data(), uo.data(), un.data());
                if (a.conserve_ke) rescale_anomaly_ke(nz, ho.data(), hn.data(), uo.data(), un.data());
                for (int k = 0; k < nz; ++k) a.v[(size_t)i + (size_t)nx * ((size_t)J + (size_t)(ny + 1) * k)] = un[k];
            }
    }
    // L9-L10
    for (size_t t = 0; t < n2 * nz; ++t) {
        a.mass_budget[t] = a.mass_budget[t] + (a.target_h[t] - a.h_old[t]);
        a.h_layer[t] = a.target_h[t];
    }
    for (size_t t = 0; t < n2; ++t) {
        double e = -a.bt_H_ref[t];
        for (int k = 0; k < nz; ++k) e = e + a.h_layer[t + n2 * k];
        a.bt_eta[t] = e;
    }
    return 0;
}

}  // extern "C"
