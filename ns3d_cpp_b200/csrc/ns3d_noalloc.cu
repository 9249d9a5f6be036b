// ns3d_compute_rhs_noalloc: the right-hand side of a periodic box held in
// caller-owned device memory, computed without allocating anything.
//
// Who needs it: hosts whose device memory belongs to somebody else's
// allocator. A framework with a caching allocator or a job with a fixed,
// pre-reserved memory budget cannot let a library call cudaMalloc behind its
// back (the memory would be invisible to its accounting and could fail with
// out-of-memory in the middle of a run), and a time loop that must never stall
// on the driver's allocation path cannot either. Such a caller passes its
// input and output buffers; the intermediate arrays of the RHS live in a
// fixed-size array of this library's own device memory.
//
// The scratch (temperature + the inviscid accumulator + the viscous fluxes)
// is the file-scope array below: 15 doubles per cell for at most
// NS3D_NOALLOC_MAX_CELLS cells, 7.5 MiB, held on every GPU that loads the
// library until the process exits. Every call shares it and it keeps the last
// call's contents; each kernel overwrites what it reads later in the same
// call, so nothing needs clearing, but calls that overlap on the GPU (other
// streams, other threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "ns3d_internal.h"

using namespace ns3d;

namespace ns3d {
extern template cudaError_t launch_sweep<double>(const LaunchCfg&, int, StateView, double*, const Ctrl*);
extern template cudaError_t launch_visc_flux<double>(const LaunchCfg&, StateView, double*, const Ctrl*);
extern template cudaError_t launch_rhs_out<double>(const LaunchCfg&, const double*, const double*, double*);
extern template cudaError_t launch_sweep<float>(const LaunchCfg&, int, StateView, float*, const Ctrl*);
extern template cudaError_t launch_visc_flux<float>(const LaunchCfg&, StateView, float*, const Ctrl*);
extern template cudaError_t launch_rhs_out<float>(const LaunchCfg&, const float*, const float*, double*);
}  // namespace ns3d

// 15 doubles per cell: T (double) + 5 accumulator values + the viscous fluxes
// (9 doubles in the FP64 form; 5 + 12 floats in the FP32-stencil form).
static __device__ __align__(256) double g_noalloc_scratch[15 * (long long)NS3D_NOALLOC_MAX_CELLS];

namespace {

constexpr int kMaxDevices = 256;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device. In host code the symbol names a host-side shadow, not device
// memory, so kernels must be given this address.
ns3d_status scratch_address(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ns3d_compute_rhs_noalloc: cudaGetDevice: %s\n", cudaGetErrorString(e));
        return NS3D_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return NS3D_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "ns3d_compute_rhs_noalloc: cudaGetSymbolAddress: %s\n",
                         cudaGetErrorString(e));
            return NS3D_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return NS3D_OK;
}

// T = p / (rho Rgas) with primitiveToConserved's density clamp.
__global__ void k_noalloc_temperature(long long n, const double* __restrict__ rho,
                                      const double* __restrict__ p, double Rgas,
                                      double* __restrict__ T) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    double rr = rho[id];
    if (rr <= 0.0) rr = 1e-12;
    T[id] = p[id] / (rr * Rgas);
}

template <class R>
cudaError_t rhs_into(const LaunchCfg& L, StateView W, double* scratch, double* rhs) {
    const long long n = L.P.n;
    R* tacc = reinterpret_cast<R*>(scratch + n);
    // fv on a 16-byte boundary (the FP32 form reads it as float4); FP32 needs
    // 8 + 20 + 48 bytes per cell (+12 of padding) of the 120 the array holds
    R* fv = reinterpret_cast<R*>((reinterpret_cast<uintptr_t>(tacc + 5 * n) + 15) & ~uintptr_t(15));
    cudaError_t e = cudaSuccess;
    for (int dir = 0; dir < 3 && e == cudaSuccess; ++dir) e = launch_sweep<R>(L, dir, W, tacc, nullptr);
    if (e == cudaSuccess) e = launch_visc_flux<R>(L, W, fv, nullptr);
    if (e == cudaSuccess) e = launch_rhs_out<R>(L, tacc, fv, rhs);
    return e;
}

}  // namespace

extern "C" ns3d_status ns3d_compute_rhs_noalloc(const ns3d_params* p, const double* rho,
                                                const double* u, const double* v, const double* w,
                                                const double* pres, double* rhs, void* stream) {
    if (!p || !rho || !u || !v || !w || !pres || !rhs) return NS3D_ERR_INVALID;
    LaunchCfg L;
    std::string msg;
    ns3d_status s = build_launch_cfg(p, &L, &msg);
    if (s != NS3D_OK) {
        std::fprintf(stderr, "ns3d_compute_rhs_noalloc: %s\n", msg.c_str());
        return s;
    }
    if (L.P.n > NS3D_NOALLOC_MAX_CELLS) {
        std::fprintf(stderr,
                     "ns3d_compute_rhs_noalloc: %lld cells exceed the fixed scratch of %d cells; "
                     "use ns3d_create + ns3d_compute_rhs for larger boxes\n",
                     L.P.n, NS3D_NOALLOC_MAX_CELLS);
        return NS3D_ERR_INVALID;
    }
    double* scratch = nullptr;
    if ((s = scratch_address(&scratch)) != NS3D_OK) return s;
    L.stream = static_cast<cudaStream_t>(stream);
    double* T = scratch;
    const long long n = L.P.n;
    k_noalloc_temperature<<<(unsigned)((n + 255) / 256), 256, 0, L.stream>>>(n, rho, pres, L.P.Rgas, T);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        const StateView W{rho, u, v, w, pres, T};
        e = p->precision == NS3D_PREC_FP64 ? rhs_into<double>(L, W, scratch, rhs)
                                           : rhs_into<float>(L, W, scratch, rhs);
    }
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ns3d_compute_rhs_noalloc: %s\n", cudaGetErrorString(e));
        return NS3D_ERR_CUDA;
    }
    return NS3D_OK;
}
