// cnm_noalloc.cu -- the radial block solve for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: host codes that hand the
// solver a fixed, pre-reserved device arena and forbid any other allocation (so
// that a long run can never fail half-way on an out-of-memory), drivers that
// issue work from inside a region where allocation is not allowed, and plug-ins
// that only ever receive device pointers from their host application.  The
// handle API (cnm_create) allocates its working vectors, so it is closed to them.
// cnm_radial_solve_noalloc gives them the preconditioner's per-mode tridiagonal
// solve with no allocation at all: the caller passes the inputs and the output,
// and the one piece of scratch the solve needs -- the inverse Thomas pivots --
// lives in the file-scope device array below, of fixed size.
#include "../../include/cnm_gpu.h"
#include "cnm_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <mutex>

namespace cnm {

// Pivots for at most CNM_NOALLOC_MAX_UNKNOWNS complex unknowns, plus one trailing
// element whose first int is the solve's status word.  Every GPU that loads the
// library holds this array (16 MiB + 16 bytes) until the process exits.
static __device__ __align__(256) double2 g_noalloc_scratch[CNM_NOALLOC_MAX_UNKNOWNS + 1];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double2 *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device.  In host code the
// symbol g_noalloc_scratch is only a host-side stand-in, so its address has to be
// asked for once per device, with that device current.
cudaError_t scratch_for_current_device(double2 **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k_precond_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<double2 *>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

// Warm-up window of the chunked scans for an off-diagonal of modulus kappa (the same
// rule as the handle's windowed preconditioner): the forward and backward sweeps
// contract by rho = kappa / |p+| per node, p+ the attracting pivot of a diagonal
// 1 + 2 i kappa 0.99, and the window is long enough to forget the start value to
// exp(-40) at that rate.  `rho` returns the rate the window assumes; the factorisation
// flags any interior pivot whose actual rate |off / p_i| exceeds it.
int scan_window(double kappa, double &rho)
{
    const std::complex<double> a(1.0, 2.0 * kappa * 0.99), c(-kappa * kappa, 0.0);
    const std::complex<double> sq = std::sqrt(a * a - 4.0 * c);
    const double pp = std::max(std::abs((a + sq) * 0.5), std::abs((a - sq) * 0.5));
    rho = kappa / pp;
    const int w = rho < 1.0 ? (int)std::ceil(40.0 / -std::log(rho)) + 16 : 4096;
    const int wc = std::max(32, std::min(4096, w));
    // the rate the clamped window still forgets to exp(-40)
    rho = std::min(rho < 1.0 ? rho : 1.0, std::exp(-40.0 / (double)(wc - 16)));
    return wc;
}

}  // namespace
}  // namespace cnm

extern "C" int cnm_radial_solve_noalloc(const double *diag, double off_re, double off_im, int32_t Nr,
                                        int32_t n_modes, const double *b, double *x, void *stream)
{
    using namespace cnm;
    if (!diag || !b || !x || Nr < 3 || n_modes < 1) return CNM_EINVAL;
    if ((int64_t)Nr * (int64_t)n_modes > (int64_t)CNM_NOALLOC_MAX_UNKNOWNS) return CNM_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double2 *scratch = nullptr;
    if (scratch_for_current_device(&scratch) != cudaSuccess) return CNM_ECUDA;
    int *status = reinterpret_cast<int *>(scratch + CNM_NOALLOC_MAX_UNKNOWNS);
    // the array keeps the previous call's contents: the status word must start at zero
    if (cudaMemsetAsync(status, 0, sizeof(int), st) != cudaSuccess) return CNM_ECUDA;
    const double2 off = make_double2(off_re, off_im);
    const int chunk = 2048;
    double rho = 0.0;
    const int window = scan_window(std::hypot(off_re, off_im), rho);
    const int chunks = (Nr + chunk - 1) / chunk;
    // one chunk per mode: the sweeps start at the boundary and are exact, nothing to check
    const double rho_max = chunks > 1 ? rho : INFINITY;
    k_precond_factor_diag<<<dim3(chunks, n_modes), SCAN_THREADS, 0, st>>>(
        reinterpret_cast<const double2 *>(diag), Nr, off, chunk, window / 2 + 16, rho_max, scratch, status);
    if (cudaGetLastError() != cudaSuccess) return CNM_ECUDA;
    const size_t smem = (size_t)(std::min(Nr, chunk + 2 * window) + SCAN_THREADS) * sizeof(double2);
    k_precond_solve<<<dim3(chunks, n_modes), SCAN_THREADS, smem, st>>>(
        Nr, chunk, window, off, scratch, reinterpret_cast<const double2 *>(b), reinterpret_cast<double2 *>(x));
    if (cudaGetLastError() != cudaSuccess) return CNM_ECUDA;
    int host_status = 0;
    if (cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return CNM_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CNM_ECUDA;
    return host_status ? CNM_EDEVICE : CNM_OK;
}
