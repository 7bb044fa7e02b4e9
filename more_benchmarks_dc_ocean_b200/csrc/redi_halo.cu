// Halo packing for the horizontal domain decomposition (halo.py): one launch
// copies one column (or row) of every field of a tile into a contiguous buffer
// for a neighbour, or back from the buffer it received, instead of one copy per
// field. Fields are (nx, ny, nz) column-major like the Fortran arrays (i
// fastest); the buffer holds field f's nz x ny (column) or nz x nx (row)
// values at f * n, layer-major, in the order torch slicing of the (nz, ny, nx)
// array gives.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/redi_b200.h"
#include "redi_kernels.h"

namespace {

struct HaloFields {
    double* f[redi::kMaxTracers + 1];
};

__global__ void k_halo_copy(HaloFields hf, int nf, int nx, int ny, int nz, int axis, int index, double* buf,
                            int to_buf) {
    const int along = axis == 0 ? ny : nx;  // a column runs along j, a row along i
    const long long n = (long long)along * nz;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n * nf) return;
    const int f = (int)(t / n);
    const long long r = t - (long long)f * n;
    const int k = (int)(r / along), a = (int)(r - (long long)k * along);
    const size_t o = axis == 0 ? (size_t)index + (size_t)nx * a + (size_t)nx * ny * k
                               : (size_t)a + (size_t)nx * index + (size_t)nx * ny * k;
    if (to_buf)
        buf[t] = hf.f[f][o];
    else
        hf.f[f][o] = buf[t];
}

}  // namespace

extern "C" int redi_b200_halo_copy(double* const* fields, int nfields, int nx, int ny, int nz, int axis, int index,
                                   double* buf, int to_buf, void* stream) {
    if (!fields || !buf || nfields < 1 || nfields > redi::kMaxTracers + 1 || nx < 1 || ny < 1 || nz < 1 ||
        (axis != 0 && axis != 1) || index < 0 || index >= (axis == 0 ? nx : ny)) {
        redi::set_last_error("redi_b200_halo_copy: bad argument");
        return REDI_B200_E_ARG;
    }
    HaloFields hf{};
    for (int f = 0; f < nfields; ++f) {
        if (!fields[f]) {
            redi::set_last_error("redi_b200_halo_copy: NULL field");
            return REDI_B200_E_ARG;
        }
        hf.f[f] = fields[f];
    }
    const long long n = (long long)(axis == 0 ? ny : nx) * nz * nfields;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    redi::launch_begin(redi::K_AUX, st);
    k_halo_copy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(hf, nfields, nx, ny, nz, axis, index, buf, to_buf);
    redi::launch_end(redi::K_AUX, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        redi::set_last_error(std::string("redi_b200_halo_copy: ") + cudaGetErrorString(e));
        return REDI_B200_E_CUDA;
    }
    return REDI_B200_OK;
}
