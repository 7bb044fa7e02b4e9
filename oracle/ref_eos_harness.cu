// TEST INFRASTRUCTURE ONLY — never linked into the product.
//
// Runs the reference's own CUDA transcription of eos_specvol_derivs
// (redi/ocean_eos.F90, LINEAR and WRIGHT_97 branches) over caller-supplied
// points, so that its outputs pin the oracle's Wright derivatives
// (oracle/redi_eos_oracle.h, wright_dsv) bit for bit. The reference keeps two
// copies of that device routine, one per model that evaluates a non-linear EOS
// on the GPU:
//
//   REF_EOS_EPBL  epbl/epbl_kernel.cu:112-137      (takes EpblParams, epbl/epbl_params.h:19)
//   REF_EOS_KS    kappa_shear/ks_kernel.cu:108-134 (takes KsPar, ks_kernel.cu:79-87)
//
// The reference file is compiled where it lies: oracle/ref_build.sh passes its
// directory with -I and selects it with one of the macros above; nothing of it
// is copied here. Built with -fmad=false so the result is the IEEE sequence of
// the source.
#include <cstring>

#if defined(REF_EOS_EPBL)
#include "epbl_kernel.cu"
using RefEosPar = EpblParams;
#elif defined(REF_EOS_KS)
#include "ks_kernel.cu"
using RefEosPar = KsPar;
#else
#error "define REF_EOS_EPBL or REF_EOS_KS"
#endif

__global__ void k_ref_eos_specvol_derivs(RefEosPar par, int n, const double* T, const double* S, const double* p,
                                         double* dsv_dt, double* dsv_ds) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a, b;
    eos_specvol_derivs(par, T[i], S[i], p[i], &a, &b);
    dsv_dt[i] = a;
    dsv_ds[i] = b;
}

// Host arrays of n points in, host arrays out. Returns 0, or the CUDA error code.
extern "C" int ref_eos_specvol_derivs(int variant, double rho0, double alpha_T, double beta_S, int n,
                                      const double* T, const double* S, const double* p, double* dsv_dt,
                                      double* dsv_ds) {
    if (n <= 0) return 0;
    RefEosPar par;
    std::memset(&par, 0, sizeof par);
    par.eos_variant = variant;
    par.eos_rho0 = rho0;
    par.eos_alpha_T = alpha_T;
    par.eos_beta_S = beta_S;
    const size_t bytes = (size_t)n * sizeof(double);
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 5 * bytes);
    if (e != cudaSuccess) return (int)e;
    double *dT = d, *dS = d + n, *dp = d + 2 * (size_t)n, *o1 = d + 3 * (size_t)n, *o2 = d + 4 * (size_t)n;
    cudaMemcpy(dT, T, bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dS, S, bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dp, p, bytes, cudaMemcpyHostToDevice);
    k_ref_eos_specvol_derivs<<<(n + 127) / 128, 128>>>(par, n, dT, dS, dp, o1, o2);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(dsv_dt, o1, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(dsv_ds, o2, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return (int)e;
}
