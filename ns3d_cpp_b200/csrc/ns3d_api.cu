// C ABI implementation: context, device buffers, transfers and the
// sequencing of the stage kernels. Declarations and reference citations are
// in include/ns3d_gpu.h.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <type_traits>
#include <thread>
#include <vector>

#include "ns3d_gpu.h"
#define NS3D_API_KERNELS
#include "ns3d_internal.h"
#include "ns3d_launch.cuh"

using namespace ns3d;

namespace ns3d {
// explicit instantiations live in ns3d_fp64.cu / ns3d_fp32.cu
extern template cudaError_t launch_sweep<double>(const LaunchCfg&, int, StateView, double*, const Ctrl*);
extern template cudaError_t launch_visc_flux<double>(const LaunchCfg&, StateView, double*, const Ctrl*);
extern template cudaError_t launch_update<double>(const LaunchCfg&, int, StateView, StateView,
                                                  const double*, const double*, StateOut, Ctrl*);
extern template cudaError_t launch_rhs_out<double>(const LaunchCfg&, const double*, const double*, double*);
extern template cudaError_t launch_sweep<float>(const LaunchCfg&, int, StateView, float*, const Ctrl*);
extern template cudaError_t launch_visc_flux<float>(const LaunchCfg&, StateView, float*, const Ctrl*);
extern template cudaError_t launch_update<float>(const LaunchCfg&, int, StateView, StateView,
                                                 const float*, const float*, StateOut, Ctrl*);
extern template cudaError_t launch_rhs_out<float>(const LaunchCfg&, const float*, const float*, double*);
extern template cudaError_t launch_sweep_z_update<double>(const LaunchCfg&, int, StateView, StateView,
                                                          const double*, const double*, StateOut, Ctrl*);
extern template cudaError_t launch_sweep_z_update<float>(const LaunchCfg&, int, StateView, StateView,
                                                         const float*, const float*, StateOut, Ctrl*);
}  // namespace ns3d

// Steps one run call can record before the record grows (synchronously).
constexpr int kStepTimesCap0 = 8192;

struct ns3d_ctx {
    ns3d_params p;
    LaunchCfg L;
    int device = 0;
    cudaStream_t stream = nullptr;
    // the viscous flux can run beside the sweeps on a second stream (NS3D_OVERLAP=1;
    // measured at 256^3 FP32: 8.13 -> 8.04 ms per step, the sweep it shares the
    // SMs with stretching by about the viscous kernel's time, so it is off by default)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool overlap = false;
    // the z sweep fused with the stage update (NS3D_FUSE=1) or the two kernels
    // (NS3D_FUSE=0); the same bits either way
    bool fuse = false;
    long long n = 0;
    double* wmem = nullptr;      // 3 state buffers x 6 arrays x n
    double* slot[3] = {nullptr, nullptr, nullptr};  // state buffer b: 6 arrays of n from slot[b]
    // ns3d_prefetch_primitive: a fourth 6 n block that host copies land in on
    // the copy stream; the upload that uses it swaps it with the current
    // buffer's block (no device copy)
    double* stage_mem = nullptr;
    double* stage = nullptr;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_staged = nullptr, ev_consumed = nullptr;
    const double* pre_h[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    bool prefetched = false;
    int cur = 0, rec = 0;        // current state buffer, recorded (U0) buffer
    void* tacc = nullptr;        // 5 n (R)
    void* fv = nullptr;          // viscous fluxes: 9 n doubles (FP64) or 3 n float4 (FP32)
    size_t rsize = 8;            // sizeof(R)
    Ctrl* ctrl = nullptr;
    Ctrl* ctrl_host = nullptr;   // pinned mirror
    double* sums_part = nullptr; // partial sums
    double* sums_out = nullptr;
    int sums_blocks = 0;
    bool dtmin_valid = false;
    double* step_times = nullptr;  // current_time after each step of the last run call
    // device scratch of the adjoint entry points, kept between calls (grown,
    // never shrunk; freed with the context)
    double* adj_buf[10] = {};
    size_t adj_cap[10] = {};
    int step_times_cap = 0, step_times_n = 0;
    double time = 0.0, out_next = 0.0;
    long long steps = 0;         // completed steps (the time_advance step count beside `time`)
    int last_events = 0;         // NS3D_EVENT_* of the last stepping call
    // spectrum
    cufftHandle fft = 0;
    bool fft_ready = false;
    cufftDoubleComplex* spec = nullptr;
    double* bins = nullptr;
    double* spec_part = nullptr;  // per-block bin partials of the spectrum
    // instrumentation
    long long launches = 0;
    bool prof_on = false;
    struct ProfRec { int cls; cudaEvent_t a, b; };
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::string err;
};

namespace {

const char* kStaticErr = "invalid context";

ns3d_status fail(ns3d_ctx* c, ns3d_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

#define NS3D_CK(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(ctx, NS3D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

double* warr(ns3d_ctx* c, int buf, int a) { return c->slot[buf] + (long long)a * c->n; }

cudaEvent_t pool_event(ns3d_ctx* c) {
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}

// Launch `nk` kernels through `f` (returns cudaError_t) as kernel class `cls`:
// counted, and bracketed by an event pair when profiling is on.
template <class F>
ns3d_status launch_on(ns3d_ctx* ctx, cudaStream_t st, int cls, int nk, F&& f) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (ctx->prof_on) {
        a = pool_event(ctx);
        b = pool_event(ctx);
        if (a && b) cudaEventRecord(a, st);
    }
    const cudaError_t e = f();
    if (e != cudaSuccess) return fail(ctx, NS3D_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    if (a && b) {
        cudaEventRecord(b, st);
        ctx->prof.push_back({cls, a, b});
    }
    ctx->launches += nk;
    return NS3D_OK;
}

template <class F>
ns3d_status launch(ns3d_ctx* ctx, int cls, int nk, F&& f) {
    return launch_on(ctx, ctx->stream, cls, nk, f);
}

// The status of `expr`: a launcher's own cudaError_t (an attribute or
// configuration failure it returns) or, for raw <<<>>> launches (void), the
// launch error.
template <class F>
cudaError_t launch_result(F&& f) {
    if constexpr (std::is_void_v<decltype(f())>) {
        f();
        return cudaGetLastError();
    } else {
        const cudaError_t e = f();
        const cudaError_t e2 = cudaGetLastError();
        return e != cudaSuccess ? e : e2;
    }
}

#define NS3D_LAUNCH(cls, nk, expr)                                                   \
    do {                                                                             \
        ns3d_status s_ = launch(ctx, (cls), (nk), [&]() -> cudaError_t {             \
            return launch_result([&]() { return expr; });                            \
        });                                                                          \
        if (s_ != NS3D_OK) return s_;                                                \
    } while (0)

StateView view(ns3d_ctx* c, int buf) {
    return StateView{warr(c, buf, 0), warr(c, buf, 1), warr(c, buf, 2),
                     warr(c, buf, 3), warr(c, buf, 4), warr(c, buf, 5)};
}
StateOut outv(ns3d_ctx* c, int buf) {
    return StateOut{warr(c, buf, 0), warr(c, buf, 1), warr(c, buf, 2),
                    warr(c, buf, 3), warr(c, buf, 4), warr(c, buf, 5)};
}

int recon_kind(int recon) {
    switch (recon) {
    case NS3D_RECON_WENO5: return RC_WENO5;
    case NS3D_RECON_LINEAR: return RC_LINEAR;
    case NS3D_RECON_MDCD: return RC_LIN6;
    case NS3D_RECON_MDCD_HYBRID: return RC_MDCD_HYBRID;
    case NS3D_RECON_UPWIND_7TH: case NS3D_RECON_UD7L: return RC_LIN8;
    default: return -1;
    }
}

// Linear reconstruction coefficients evaluated with the reference's own
// expressions (reconstruction.cpp:126-135, 227-249).
void linear_coefficients(const ns3d_params& p, double lin[8]) {
    for (int m = 0; m < 8; ++m) lin[m] = 0.0;
    if (p.recon == NS3D_RECON_MDCD || p.recon == NS3D_RECON_MDCD_HYBRID) {
        const double diss = p.mdcd_diss, disp = p.mdcd_disp;
        lin[0] = (1.0 / 2.0 * disp + 1.0 / 2.0 * diss);
        lin[1] = (-3.0 / 2.0 * disp - 5.0 / 2.0 * diss - 1.0 / 12.0);
        lin[2] = (7.0 / 12.0 + disp + 5.0 * diss);
        lin[3] = (7.0 / 12.0 + disp - 5.0 * diss);
        lin[4] = (-3.0 / 2.0 * disp + 5.0 / 2.0 * diss - 1.0 / 12.0);
        lin[5] = (1.0 / 2.0 * disp - 1.0 / 2.0 * diss);
    } else if (p.recon == NS3D_RECON_UPWIND_7TH) {
        // a0*s0 + ... with a2, a5 negative: x - c*s == x + (-c)*s exactly, and
        // the a7*s7 = 0*s7 term adds a signed zero, which changes nothing.
        lin[0] = -1.0 / 140.0;
        lin[1] = 5.0 / 84.0;
        lin[2] = -(101.0 / 420.0);
        lin[3] = 319.0 / 420.0;
        lin[4] = 107.0 / 210.0;
        lin[5] = -(19.0 / 210.0);
        lin[6] = 1.0 / 105.0;
        lin[7] = 0.0;
    } else if (p.recon == NS3D_RECON_UD7L) {
        const double alpha = p.ud7l_alpha;
        lin[0] = -3.0 / 420.0 * alpha - 3.0 / 840.0 * (1.0 - alpha);
        lin[1] = 25.0 / 420.0 * alpha + 29.0 / 840.0 * (1.0 - alpha);
        lin[2] = -101.0 / 420.0 * alpha - 139.0 / 840.0 * (1.0 - alpha);
        lin[3] = 319.0 / 420.0 * alpha + 533.0 / 840.0 * (1.0 - alpha);
        lin[4] = 214.0 / 420.0 * alpha + 533.0 / 840.0 * (1.0 - alpha);
        lin[5] = -38.0 / 420.0 * alpha - 139.0 / 840.0 * (1.0 - alpha);
        lin[6] = 4.0 / 420.0 * alpha + 29.0 / 840.0 * (1.0 - alpha);
        lin[7] = (-3.0 / 840.0) * (1.0 - alpha);
    }
}

// ---- small kernels of the API layer (FP64, this TU is built with -fmad=false)

// primitiveToConserved's density clamp and T after an upload of primitives.
__global__ void k_prim_finish(DevParams P, StateOut W) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    double rr = W.rho[id];
    if (rr <= 0.0) { rr = 1e-12; W.rho[id] = rr; }
    W.T[id] = W.p[id] / (rr * P.Rgas);
}

// ---- isotropic initial field (generate_full_turbulence, isotropic_ini.cpp:25-122)

// Fourier coefficients of the three velocity components at every mode:
// amplitude sqrt(2/3) sqrt(A kk exp(-2 kk / k0^2) / 4 pi), three random phases
// 2 pi r, projection normal to k. r: the uniform draws of the reference's
// loop order (z outermost, x innermost = this layout's order), 3 per cell,
// none for k = 0. Same expressions and operation order as the reference.
__global__ void k_iso_modes(int NX, int NY, int NZ, int k0, double A, const double* __restrict__ r,
                            cufftDoubleComplex* __restrict__ U, cufftDoubleComplex* __restrict__ V,
                            cufftDoubleComplex* __restrict__ Wc) {
    const long long n = (long long)NX * NY * NZ;
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const double PI = 3.14159265358979323846;
    const int i = (int)(id % NX), j = (int)((id / NX) % NY), k = (int)(id / ((long long)NX * NY));
    const int k1 = (i <= NX / 2 ? i : i - NX);
    const int k2 = (j <= NY / 2 ? j : j - NY);
    const int k3 = (k <= NZ / 2 ? k : k - NZ);
    const int kk = k1 * k1 + k2 * k2 + k3 * k3;
    if (kk == 0) {
        U[id] = make_cuDoubleComplex(0.0, 0.0);
        V[id] = make_cuDoubleComplex(0.0, 0.0);
        Wc[id] = make_cuDoubleComplex(0.0, 0.0);
        return;
    }
    const double Ak = sqrt(2.0 / 3.0) * sqrt(A * kk * exp(-2.0 * kk / (double)(k0 * k0)) / (4.0 * PI));
    const double a1 = 2 * PI * r[3 * id], a2 = 2 * PI * r[3 * id + 1], a3 = 2 * PI * r[3 * id + 2];
    const double v1r = Ak * sin(a1), v1i = Ak * cos(a1);
    const double v2r = Ak * sin(a2), v2i = Ak * cos(a2);
    const double v3r = Ak * sin(a3), v3i = Ak * cos(a3);
    const double vkr = k1 * v1r + k2 * v2r + k3 * v3r;
    const double vki = k1 * v1i + k2 * v2i + k3 * v3i;
    U[id] = make_cuDoubleComplex(k1 * vkr / kk - v1r, k1 * vki / kk - v1i);
    V[id] = make_cuDoubleComplex(k2 * vkr / kk - v2r, k2 * vki / kk - v2i);
    Wc[id] = make_cuDoubleComplex(k3 * vkr / kk - v3r, k3 * vki / kk - v3i);
}

// Real parts of the inverse transforms as the velocity, rho = 1, T = 1,
// p = Rgas rho T (init_isotropic_turbulence, isotropic_ini.cpp:184-189).
__global__ void k_iso_state(DevParams P, const cufftDoubleComplex* __restrict__ U,
                            const cufftDoubleComplex* __restrict__ V,
                            const cufftDoubleComplex* __restrict__ Wc, StateOut W) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    W.rho[id] = 1.0;
    W.u[id] = U[id].x;
    W.v[id] = V[id].x;
    W.w[id] = Wc[id].x;
    W.p[id] = P.Rgas * 1.0 * 1.0;
    W.T[id] = 1.0;
}

__global__ void k_iso_scale(long long n, double s, StateOut W) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    W.u[id] *= s;
    W.v[id] *= s;
    W.w[id] *= s;
}

// ---- residual monitor (compute_diagnostics, postprocess.cpp:7-98)

// Per block: sum over cells of (U - U0)^2 dx^3 and max |U| for the five
// conserved variables (U of the current state, U0 of the recorded one, both as
// primitiveToConserved computes them). part[block * 10 + q]: sums q = 0..4,
// maxima 5..9.
__global__ void __launch_bounds__(256)
k_resid_partial(DevParams P, StateView Wc, StateView W0, double* __restrict__ part) {
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, m[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double dx3 = P.dx * P.dx * P.dx;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < P.n;
         id += (long long)gridDim.x * blockDim.x) {
        double U[5], U0[5];
        prim2cons_cell(Wc, id, P.gamma, U);
        prim2cons_cell(W0, id, P.gamma, U0);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double r = U[q] - U0[q];
            s[q] += r * r * dx3;
            m[q] = fmax(m[q], fabs(U[q]));
        }
    }
    __shared__ double red[10][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 10; ++q) {
        double x = q < 5 ? s[q] : m[q - 5];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = q < 5 ? x + y : fmax(x, y);
        }
        if (lane == 0) red[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        const int q = threadIdx.x;
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            x = q < 5 ? x + red[q][w] : fmax(x, red[q][w]);
        part[(long long)blockIdx.x * 10 + q] = x;
    }
}

__global__ void k_resid_final(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= 10) return;
    double x = 0.0;
    for (int b = 0; b < nblocks; ++b)
        x = q < 5 ? x + part[(long long)b * 10 + q] : fmax(x, part[(long long)b * 10 + q]);
    out[q] = x;
}

// conservedToPrimitive (+ T) of an uploaded conserved state held in `U`.
__global__ void k_cons2prim(DevParams P, const double* __restrict__ U, StateOut W) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    const long long n = P.n;
    double rr = U[id];
    if (rr <= 0.0) rr = 1e-12;
    const double u = U[n + id] / rr, v = U[2 * n + id] / rr, w = U[3 * n + id] / rr;
    const double kinetic = 0.5 * (u * u + v * v + w * w);
    const double e_internal = U[4 * n + id] / rr - kinetic;
    const double p = (P.gamma - 1.0) * rr * e_internal;
    W.rho[id] = rr; W.u[id] = u; W.v[id] = v; W.w[id] = w; W.p[id] = p;
    W.T[id] = p / (rr * P.Rgas);
}

// primitiveToConserved of the state into 5 blocks; c into `c` when non-null.
__global__ void k_prim2cons(DevParams P, StateView W, double* __restrict__ U, double* __restrict__ c) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    double Uc[5];
    prim2cons_cell(W, id, P.gamma, Uc);
    for (int q = 0; q < 5; ++q) U[q * P.n + id] = Uc[q];
    if (c) c[id] = sqrt(P.gamma * W.p[id] / Uc[0]);
}

// Shell binning of one velocity component's half spectrum (cuFFT D2Z of the
// component, EnergySpectrum.cpp:108-125: E(k) += 0.5 |u_hat|^2 with
// u_hat = X / N and k = floor(|k|); modes strictly inside the x half-space
// stand for their conjugates and count twice), in a fixed order so that E(k)
// is the same to the last bit on every call.
//
// A warp takes whole x rows (fixed (j, k), ic = 0 .. nx/2) of the half
// spectrum in a fixed assignment. Along a row the shell index is
// non-decreasing in ic, so the 32 values of a chunk fall into contiguous runs
// of equal shell: a segmented shuffle reduction leaves each run's sum in its
// first lane, which adds it to the warp's own shared bin array (no two lanes
// write one bin in the same step). The block then sums its warps' arrays in
// warp order into part[block][bin].
constexpr int SPEC_WARPS = 4;
constexpr int SPEC_BLOCKS = 4 * 148;

// Shells a half spectrum can reach: floor(|k|) <= floor(sqrt((nx/2)^2 +
// (ny/2)^2 + (nz/2)^2)); one more for safety, at most the reference's 2 nx + 1.
inline int spectrum_bins_used(int nx, int ny, int nz) {
    const double k2 = (double)(nx / 2) * (nx / 2) + (double)(ny / 2) * (ny / 2) +
                      (double)(nz / 2) * (nz / 2);
    const int nb = (int)std::sqrt(k2) + 2;
    return nb < 2 * nx + 1 ? nb : 2 * nx + 1;
}

__global__ void __launch_bounds__(32 * SPEC_WARPS)
k_spectrum_part(const cufftDoubleComplex* __restrict__ X, int nx, int ny, int nz, double scale,
                int nbu, double* __restrict__ part) {
    extern __shared__ double sb[];  // [SPEC_WARPS][nbu]
    for (int b = threadIdx.x; b < SPEC_WARPS * nbu; b += blockDim.x) sb[b] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    double* wb = sb + wq * nbu;
    const int nxh = nx / 2 + 1;
    const long long rows = (long long)ny * nz;
    const long long warps = (long long)gridDim.x * SPEC_WARPS;
    for (long long r = (long long)blockIdx.x * SPEC_WARPS + wq; r < rows; r += warps) {
        const int j = (int)(r % ny), k = (int)(r / ny);
        const int k2 = j <= ny / 2 ? j : j - ny;
        const int k3 = k <= nz / 2 ? k : k - nz;
        const int kt = k2 * k2 + k3 * k3;
        for (int c0 = 0; c0 < nxh; c0 += 32) {
            const int ic = c0 + lane;
            double e = 0.0;
            int kk = -1;
            if (ic < nxh) {
                const cufftDoubleComplex z = X[r * nxh + ic];
                const double re = z.x * scale, im = z.y * scale;
                e = 0.5 * (re * re + im * im);
                const bool self_conj = (ic == 0) || ((nx % 2 == 0) && ic == nx / 2);
                if (!self_conj) e *= 2.0;
                kk = (int)sqrt(1.0 * (ic * ic + kt));
            }
            // segmented sum over runs of equal kk (contiguous: kk non-decreasing in ic)
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double ev = __shfl_down_sync(0xffffffffu, e, off);
                const int kv = __shfl_down_sync(0xffffffffu, kk, off);
                if (lane + off < 32 && kv == kk) e += ev;
            }
            const int kprev = __shfl_up_sync(0xffffffffu, kk, 1);
            const bool head = kk >= 0 && (lane == 0 || kprev != kk);
            if (head && kk < nbu) wb[kk] += e;
            __syncwarp();
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbu; b += blockDim.x) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < SPEC_WARPS; ++w) x += sb[w * nbu + b];
        part[(long long)blockIdx.x * nbu + b] = x;
    }
}

// bins[b] += sum over blocks of part[.][b], blocks in order.
__global__ void k_spectrum_final(const double* __restrict__ part, int nblocks, int nbu,
                                 double* __restrict__ bins) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbu) return;
    double x = 0.0;
    for (int k = 0; k < nblocks; ++k) x += part[(long long)k * nbu + b];
    bins[b] += x;
}

ns3d_status validate(const ns3d_params* p, std::string& msg) {
    for (int f = 0; f < 6; ++f)
        if (p->bc[f] != NS3D_BC_PERIODIC) {
            msg = "only periodic boundaries are built (boundary.cpp:56-207 is out of scope)";
            return NS3D_ERR_UNSUPPORTED;
        }
    if (recon_kind(p->recon) < 0) {
        msg = "reconstruction WCNS has no implementation in the reference either";
        return NS3D_ERR_UNSUPPORTED;
    }
    if (p->fvs_type != NS3D_FVS_STEGER_WARMING && p->fvs_type != NS3D_FVS_LAX_FRIEDRICHS) {
        msg = "unknown fvs_type";
        return NS3D_ERR_INVALID;
    }
    if (p->vis_scheme < NS3D_VIS_C8TH || p->vis_scheme > NS3D_VIS_C4TH) {
        msg = "unknown vis_scheme";
        return NS3D_ERR_INVALID;
    }
    if (p->global_nx < 8 || p->global_ny < 8 || p->global_nz < 8) {
        msg = "each extent must be at least 8 cells";
        return NS3D_ERR_INVALID;
    }
    if ((long long)p->global_nx * p->global_ny * p->global_nz > (1ll << 31)) {
        msg = "grid larger than 2^31 cells";
        return NS3D_ERR_INVALID;
    }
    if (p->precision != NS3D_PREC_FP64 && p->precision != NS3D_PREC_FP32_ACC64) {
        msg = "unknown precision";
        return NS3D_ERR_INVALID;
    }
    if (!(p->gamma > 1.0) || !(p->Ma > 0.0) || !(p->Re > 0.0) || !(p->Pr > 0.0)) {
        msg = "gamma > 1, Ma > 0, Re > 0 and Pr > 0 are required";
        return NS3D_ERR_INVALID;
    }
    return NS3D_OK;
}

inline unsigned blocks_for(long long n, int th) { return (unsigned)((n + th - 1) / th); }

ns3d_status reset_ctrl(ns3d_ctx* ctx) {
    Ctrl h{};
    h.dtmin_bits = 0;
    std::memcpy(&h.dtmin_bits, &CFL_INIT, sizeof(double));
    h.time = ctx->time;
    h.out_next = ctx->out_next;
    h.bad_cell = ctx->n;
    *ctx->ctrl_host = h;
    NS3D_CK(cudaMemcpyAsync(ctx->ctrl, ctx->ctrl_host, sizeof(Ctrl), cudaMemcpyHostToDevice,
                            ctx->stream));
    return NS3D_OK;
}

ns3d_status read_ctrl(ns3d_ctx* ctx) {
    NS3D_CK(cudaMemcpyAsync(ctx->ctrl_host, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                            ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

// The RHS pieces of the current state into tacc/fv: the sweeps along x, y and
// (unless `dirs` is 2, when the z sweep is left to the fused stage kernel) z,
// and the viscous flux.
template <class R>
ns3d_status rhs_parts_t(ns3d_ctx* ctx, StateView W, const Ctrl* ctrl, int dirs = 3) {
    R* tacc = (R*)ctx->tacc;
    if (ctx->overlap) {
        // the viscous flux (state -> fv) beside the sweeps (state -> T_acc):
        // fork after the work already queued, join before the update
        NS3D_CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
        NS3D_CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
        LaunchCfg Ls = ctx->L;
        Ls.stream = ctx->side;
        ns3d_status s = launch_on(ctx, ctx->side, NS3D_KERNEL_VISC_FLUX, 1, [&]() -> cudaError_t {
            return launch_result([&]() { return launch_visc_flux<R>(Ls, W, (R*)ctx->fv, ctrl); });
        });
        if (s != NS3D_OK) return s;
        NS3D_CK(cudaEventRecord(ctx->ev_join, ctx->side));
        for (int dir = 0; dir < dirs; ++dir)
            NS3D_LAUNCH(NS3D_KERNEL_SWEEP_X + dir, 1, launch_sweep<R>(ctx->L, dir, W, tacc, ctrl));
        NS3D_CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
        return NS3D_OK;
    }
    for (int dir = 0; dir < dirs; ++dir)
        NS3D_LAUNCH(NS3D_KERNEL_SWEEP_X + dir, 1, launch_sweep<R>(ctx->L, dir, W, tacc, ctrl));
    NS3D_LAUNCH(NS3D_KERNEL_VISC_FLUX, 1, launch_visc_flux<R>(ctx->L, W, (R*)ctx->fv, ctrl));
    return NS3D_OK;
}

// The RHS pieces of the current state (sweeps + viscous flux) into tacc/fv.
ns3d_status launch_rhs_parts(ns3d_ctx* ctx, StateView W, const Ctrl* ctrl) {
    return ctx->p.precision == NS3D_PREC_FP64 ? rhs_parts_t<double>(ctx, W, ctrl)
                                              : rhs_parts_t<float>(ctx, W, ctrl);
}

// One Shu-Osher stage Wc -> Wn (recorded state W0): the three sweeps, the
// viscous flux and k_update; or, with ctx->fuse (component-wise schemes), the
// x and y sweeps, the viscous flux and the z sweep fused with the update
// (k_sweep_ring<2, ..., FUSE>). Both give the same bits.
template <class R>
ns3d_status stage_t(ns3d_ctx* ctx, int stage, StateView Wc, StateView W0, StateOut Wn) {
    const R* tacc = (const R*)ctx->tacc;
    const R* fv = (const R*)ctx->fv;
    if (ctx->L.chr || !ctx->fuse) {
        ns3d_status s = rhs_parts_t<R>(ctx, Wc, ctx->ctrl);
        if (s != NS3D_OK) return s;
        NS3D_LAUNCH(NS3D_KERNEL_UPDATE, 1,
                    launch_update<R>(ctx->L, stage, Wc, W0, tacc, fv, Wn, ctx->ctrl));
        return NS3D_OK;
    }
    ns3d_status s = rhs_parts_t<R>(ctx, Wc, ctx->ctrl, 2);
    if (s != NS3D_OK) return s;
    NS3D_LAUNCH(NS3D_KERNEL_SWEEP_Z_UPDATE, 1,
                launch_sweep_z_update<R>(ctx->L, stage, Wc, W0, tacc, fv, Wn, ctx->ctrl));
    return NS3D_OK;
}

// A stage on explicit state arrays (6 blocks of n each); FP64 form.
StateView view_at(double* base, long long n) {
    return StateView{base, base + n, base + 2 * n, base + 3 * n, base + 4 * n, base + 5 * n};
}
StateOut out_at(double* base, long long n) {
    return StateOut{base, base + n, base + 2 * n, base + 3 * n, base + 4 * n, base + 5 * n};
}

ns3d_status stage_at(ns3d_ctx* ctx, int stage, double* wc, double* w0, double* wn) {
    return stage_t<double>(ctx, stage, view_at(wc, ctx->n), view_at(w0, ctx->n),
                           out_at(wn, ctx->n));
}

ns3d_status launch_stage(ns3d_ctx* ctx, int stage, int bc, int b0, int bn) {
    const StateView Wc = view(ctx, bc), W0 = view(ctx, b0);
    return ctx->p.precision == NS3D_PREC_FP64 ? stage_t<double>(ctx, stage, Wc, W0, outv(ctx, bn))
                                              : stage_t<float>(ctx, stage, Wc, W0, outv(ctx, bn));
}

// One runge_kutta_3 on the device with dt from ctrl->dt. Buffer rotation keeps
// the recorded state intact, so U0 stays valid exactly as rho0.. do.
ns3d_status enqueue_rk3(ns3d_ctx* ctx) {
    int a = ctx->cur, r = ctx->rec, x, y;
    if (a == r) {
        x = (a + 1) % 3;
        y = (a + 2) % 3;
        ns3d_status s;
        if ((s = launch_stage(ctx, 1, a, r, x)) != NS3D_OK) return s;
        if ((s = launch_stage(ctx, 2, x, r, y)) != NS3D_OK) return s;
        if ((s = launch_stage(ctx, 3, y, r, x)) != NS3D_OK) return s;
        ctx->cur = x;
    } else {
        const int z = 3 - a - r;
        ns3d_status s;
        if ((s = launch_stage(ctx, 1, a, r, z)) != NS3D_OK) return s;
        if ((s = launch_stage(ctx, 2, z, r, a)) != NS3D_OK) return s;
        if ((s = launch_stage(ctx, 3, a, r, z)) != NS3D_OK) return s;
        ctx->cur = z;
    }
    return NS3D_OK;
}

ns3d_status enqueue_cfl(ns3d_ctx* ctx) {
    NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1,
                (k_cfl<<<blocks_for(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->L.P, view(ctx, ctx->cur),
                                                                       ctx->ctrl)));
    ctx->dtmin_valid = true;
    return NS3D_OK;
}

// Host layout conversions ---------------------------------------------------

void gather_interior(const ns3d_params& p, const double* src, double* dst) {
    const int g = p.ghost_layers;
    const long long sx = p.global_nx + 2 * g, sy = p.global_ny + 2 * g;
    long long q = 0;
    for (int k = 0; k < p.global_nz; ++k)
        for (int j = 0; j < p.global_ny; ++j) {
            const double* row = src + ((k + g) * sy + (j + g)) * sx + g;
            std::memcpy(dst + q, row, sizeof(double) * p.global_nx);
            q += p.global_nx;
        }
}

// Interior -> Field3D layout: face ghosts get periodic images (apply_boundary),
// edges and corners get `fill` (what Field3D keeps there).
void scatter_ghosted(const ns3d_params& p, const double* src, double* dst, double fill) {
    const int g = p.ghost_layers, nx = p.global_nx, ny = p.global_ny, nz = p.global_nz;
    const long long sx = nx + 2 * g, sy = ny + 2 * g, sz = nz + 2 * g;
    for (long long t = 0; t < sx * sy * sz; ++t) dst[t] = fill;
    auto wrapi = [](int a, int n) { return ((a % n) + n) % n; };
    for (int k = 0; k < (int)sz; ++k)
        for (int j = 0; j < (int)sy; ++j)
            for (int i = 0; i < (int)sx; ++i) {
                const int gi = (i < g || i >= g + nx), gj = (j < g || j >= g + ny),
                          gk = (k < g || k >= g + nz);
                if (gi + gj + gk > 1) continue;  // edge or corner ghost
                const int ii = wrapi(i - g, nx), jj = wrapi(j - g, ny), kk = wrapi(k - g, nz);
                dst[(k * sy + j) * sx + i] = src[((long long)kk * ny + jj) * nx + ii];
            }
}

long long ghosted_count(const ns3d_params& p) {
    const int g = p.ghost_layers;
    return (long long)(p.global_nx + 2 * g) * (p.global_ny + 2 * g) * (p.global_nz + 2 * g);
}

// Upload 5 host arrays into 5 consecutive device arrays starting at dst.
ns3d_status upload5(ns3d_ctx* ctx, const double* const* h, double* const* d, int layout) {
    if (layout == NS3D_LAYOUT_INTERIOR) {
        for (int q = 0; q < 5; ++q) {
            if (!h[q]) return fail(ctx, NS3D_ERR_INVALID, "null host pointer");
            NS3D_CK(cudaMemcpyAsync(d[q], h[q], sizeof(double) * ctx->n, cudaMemcpyHostToDevice,
                                    ctx->stream));
        }
        return NS3D_OK;
    }
    if (layout != NS3D_LAYOUT_GHOSTED) return fail(ctx, NS3D_ERR_INVALID, "unknown layout");
    std::vector<double> tmp(ctx->n);
    for (int q = 0; q < 5; ++q) {
        if (!h[q]) return fail(ctx, NS3D_ERR_INVALID, "null host pointer");
        gather_interior(ctx->p, h[q], tmp.data());
        NS3D_CK(cudaMemcpyAsync(d[q], tmp.data(), sizeof(double) * ctx->n, cudaMemcpyHostToDevice,
                                ctx->stream));
        NS3D_CK(cudaStreamSynchronize(ctx->stream));
    }
    return NS3D_OK;
}

ns3d_status download_arrays(ns3d_ctx* ctx, const double* const* d, double* const* h,
                            const double* fills, int count, int layout) {
    if (layout == NS3D_LAYOUT_INTERIOR) {
        for (int q = 0; q < count; ++q)
            if (h[q])
                NS3D_CK(cudaMemcpyAsync(h[q], d[q], sizeof(double) * ctx->n, cudaMemcpyDeviceToHost,
                                        ctx->stream));
        NS3D_CK(cudaStreamSynchronize(ctx->stream));
        return NS3D_OK;
    }
    if (layout != NS3D_LAYOUT_GHOSTED) return fail(ctx, NS3D_ERR_INVALID, "unknown layout");
    std::vector<double> tmp(ctx->n);
    for (int q = 0; q < count; ++q) {
        if (!h[q]) continue;
        NS3D_CK(cudaMemcpyAsync(tmp.data(), d[q], sizeof(double) * ctx->n, cudaMemcpyDeviceToHost,
                                ctx->stream));
        NS3D_CK(cudaStreamSynchronize(ctx->stream));
        scatter_ghosted(ctx->p, tmp.data(), h[q], fills[q]);
    }
    return NS3D_OK;
}

ns3d_status compute_sums(ns3d_ctx* ctx, double out[NSUMS]) {
    NS3D_LAUNCH(NS3D_KERNEL_OTHER, 2, (k_sums_partial<<<ctx->sums_blocks, 256, 0, ctx->stream>>>(
                                           ctx->L.P, view(ctx, ctx->cur), ctx->sums_part),
                                       k_sums_final<<<1, 32, 0, ctx->stream>>>(
                                           ctx->sums_part, ctx->sums_blocks, ctx->sums_out)));
    NS3D_CK(cudaMemcpyAsync(out, ctx->sums_out, sizeof(double) * NSUMS, cudaMemcpyDeviceToHost,
                            ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

}  // namespace

namespace ns3d {

// Measured at 256^3 (B200): the 2.5-D viscous flux with 16 planes per block is
// the fastest shape (FP64 1.15 -> 1.01 ms, FP32 unchanged); smaller boxes take
// fewer planes per block (detail::zb_for) so that the grid fills the SMs.
void default_tiling(LaunchCfg& L) {
    L.zb = 0;
    L.tiled = 3;  // 2.5-D viscous flux, pipelined plane loads (k_visc_flux_pipe)
    L.pipe = 3;   // FP32 sweeps with the software-pipelined split (k_sweep_x_pipe, k_sweep_pipe)
    if (const char* e = std::getenv("NS3D_PIPE")) L.pipe = std::atoi(e);
    if (const char* e = std::getenv("NS3D_TILE_ZB")) L.zb = std::atoi(e);
    if (const char* e = std::getenv("NS3D_TILED")) L.tiled = std::atoi(e);
    if (const char* e = std::getenv("NS3D_SEG"))
        for (int d = 0; d < 3; ++d) L.seg[d] = std::atoi(e);
}

ns3d_status build_launch_cfg(const ns3d_params* p, LaunchCfg* L, std::string* msg) {
    if (!p || !L) return NS3D_ERR_INVALID;
    ns3d_params q = *p;
    ns3d_status s = ns3d_params_derive(&q);
    if (s != NS3D_OK) return s;
    std::string m;
    if ((s = validate(&q, m)) != NS3D_OK) {
        if (msg) *msg = m;
        return s;
    }
    std::memset(L, 0, sizeof(*L));
    DevParams& P = L->P;
    P.nx = q.global_nx; P.ny = q.global_ny; P.nz = q.global_nz;
    P.n = (long long)q.global_nx * q.global_ny * q.global_nz;
    P.gamma = q.gamma; P.Rgas = q.Rgas; P.mu = q.mu; P.Cp = q.Cp; P.Pr = q.Pr;
    P.sutherland_s = q.sutherland_s_over_tref; P.sw_eps = q.sw_entropy_eps;
    P.dx = q.dx; P.dy = q.dy; P.dz = q.dz;
    P.inv_dx = 1.0 / q.dx; P.inv_dy = 1.0 / q.dy; P.inv_dz = 1.0 / q.dz;
    P.cfl = q.cfl; P.dt_fixed = q.dt_fixed;
    linear_coefficients(q, P.lin);
    P.mdcd_disp = q.mdcd_disp; P.mdcd_diss = q.mdcd_diss;
    P.vis_order = q.vis_scheme == NS3D_VIS_C4TH ? 4 : (q.vis_scheme == NS3D_VIS_C6TH ? 6 : 8);
    L->fvs = q.fvs_type == NS3D_FVS_STEGER_WARMING ? FV_SW : FV_LF;
    L->rc = recon_kind(q.recon);
    L->chr = q.char_recon ? 1 : 0;
    for (int d = 0; d < 3; ++d) L->seg[d] = 0;  // chosen per launch from the grid
    default_tiling(*L);
    L->stream = nullptr;
    return NS3D_OK;
}

}  // namespace ns3d

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char* ns3d_last_error(const ns3d_ctx* ctx) { return ctx ? ctx->err.c_str() : kStaticErr; }

ns3d_status ns3d_create(const ns3d_params* p, int device, ns3d_ctx** out) {
    if (!p || !out) return NS3D_ERR_INVALID;
    *out = nullptr;
    ns3d_params q = *p;
    ns3d_status s = ns3d_params_derive(&q);
    if (s != NS3D_OK) return s;
    std::string msg;
    s = validate(&q, msg);
    if (s != NS3D_OK) {
        std::fprintf(stderr, "ns3d_create: %s\n", msg.c_str());
        return s;
    }
    auto* ctx = new ns3d_ctx;
    ctx->p = q;
    ctx->device = device;
    ctx->n = (long long)q.global_nx * q.global_ny * q.global_nz;
    ctx->time = 0.0;
    ctx->out_next = q.output_Timefreq;
    DevParams& P = ctx->L.P;
    std::memset(&P, 0, sizeof(P));
    P.nx = q.global_nx; P.ny = q.global_ny; P.nz = q.global_nz; P.n = ctx->n;
    P.gamma = q.gamma; P.Rgas = q.Rgas; P.mu = q.mu; P.Cp = q.Cp; P.Pr = q.Pr;
    P.sutherland_s = q.sutherland_s_over_tref; P.sw_eps = q.sw_entropy_eps;
    P.dx = q.dx; P.dy = q.dy; P.dz = q.dz;
    P.inv_dx = 1.0 / q.dx; P.inv_dy = 1.0 / q.dy; P.inv_dz = 1.0 / q.dz;  // range_kutta.cpp:14-16
    P.cfl = q.cfl; P.dt_fixed = q.dt_fixed;
    linear_coefficients(q, P.lin);
    P.mdcd_disp = q.mdcd_disp; P.mdcd_diss = q.mdcd_diss;
    P.vis_order = q.vis_scheme == NS3D_VIS_C4TH ? 4 : (q.vis_scheme == NS3D_VIS_C6TH ? 6 : 8);
    ctx->L.fvs = q.fvs_type == NS3D_FVS_STEGER_WARMING ? FV_SW : FV_LF;
    ctx->L.rc = recon_kind(q.recon);
    ctx->L.chr = q.char_recon ? 1 : 0;
    for (int d = 0; d < 3; ++d) ctx->L.seg[d] = 0;  // chosen per launch from the grid
    default_tiling(ctx->L);
    ctx->rsize = q.precision == NS3D_PREC_FP64 ? sizeof(double) : sizeof(float);

    auto bail = [&](ns3d_status st, const std::string& m) {
        std::fprintf(stderr, "ns3d_create: %s\n", m.c_str());
        ns3d_destroy(ctx);
        return st;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(NS3D_ERR_CUDA, cudaGetErrorString(e));
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(NS3D_ERR_CUDA, cudaGetErrorString(e));
    ctx->L.stream = ctx->stream;
    if (const char* ov = std::getenv("NS3D_OVERLAP")) ctx->overlap = std::atoi(ov) != 0;
    if (const char* fu = std::getenv("NS3D_FUSE")) ctx->fuse = std::atoi(fu) != 0;
    if (ctx->overlap &&
        (cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess ||
         cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
         cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess))
        return bail(NS3D_ERR_CUDA, "second stream for the overlapped viscous flux");
    const size_t n = (size_t)ctx->n;
    if (cudaMalloc(&ctx->wmem, sizeof(double) * 18 * n) != cudaSuccess ||
        cudaMalloc(&ctx->tacc, ctx->rsize * 5 * n) != cudaSuccess ||
        cudaMalloc(&ctx->fv, ctx->rsize * (ctx->rsize == 4 ? fv_values_per_cell<float>() : fv_values_per_cell<double>()) * n) != cudaSuccess ||
        cudaMalloc(&ctx->ctrl, sizeof(Ctrl)) != cudaSuccess) {
        cudaGetLastError();
        return bail(NS3D_ERR_NOMEM, "device allocation failed");
    }
    if (cudaMallocHost(&ctx->ctrl_host, sizeof(Ctrl)) != cudaSuccess)
        return bail(NS3D_ERR_NOMEM, "pinned allocation failed");
    ctx->sums_blocks = (int)std::min<long long>(4 * 148, (ctx->n + 255) / 256);
    if (cudaMalloc(&ctx->sums_part, sizeof(double) * NSUMS * ctx->sums_blocks) != cudaSuccess ||
        cudaMalloc(&ctx->sums_out, sizeof(double) * NSUMS) != cudaSuccess ||
        cudaMalloc(&ctx->step_times, sizeof(double) * kStepTimesCap0) != cudaSuccess)
        return bail(NS3D_ERR_NOMEM, "device allocation failed");
    ctx->step_times_cap = kStepTimesCap0;
    for (int b = 0; b < 3; ++b) ctx->slot[b] = ctx->wmem + (size_t)b * 6 * n;
    // a uniform quiescent state until the first upload (Field3D::allocate, :232-236)
    cudaMemsetAsync(ctx->wmem, 0, sizeof(double) * 18 * n, ctx->stream);
    if (reset_ctrl(ctx) != NS3D_OK) return bail(NS3D_ERR_CUDA, ctx->err);
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return bail(NS3D_ERR_CUDA, cudaGetErrorString(e));
    *out = ctx;
    return NS3D_OK;
}

ns3d_status ns3d_destroy(ns3d_ctx* ctx) {
    if (!ctx) return NS3D_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->fft_ready) cufftDestroy(ctx->fft);
    cudaFree(ctx->spec);
    cudaFree(ctx->bins);
    cudaFree(ctx->spec_part);
    cudaFree(ctx->wmem);
    cudaFree(ctx->stage_mem);
    cudaFree(ctx->tacc);
    cudaFree(ctx->fv);
    cudaFree(ctx->ctrl);
    cudaFree(ctx->sums_part);
    cudaFree(ctx->sums_out);
    cudaFree(ctx->step_times);
    for (double* b : ctx->adj_buf) cudaFree(b);
    if (ctx->ctrl_host) cudaFreeHost(ctx->ctrl_host);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->ev_staged) cudaEventDestroy(ctx->ev_staged);
    if (ctx->ev_consumed) cudaEventDestroy(ctx->ev_consumed);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return NS3D_OK;
}

ns3d_status ns3d_get_params(const ns3d_ctx* ctx, ns3d_params* out) {
    if (!ctx || !out) return NS3D_ERR_INVALID;
    *out = ctx->p;
    return NS3D_OK;
}

ns3d_status ns3d_device_bytes(const ns3d_ctx* ctx, size_t* bytes) {
    if (!ctx || !bytes) return NS3D_ERR_INVALID;
    *bytes = sizeof(double) * (ctx->stage_mem ? 24 : 18) * (size_t)ctx->n +
             ctx->rsize * 14 * (size_t)ctx->n;
    for (size_t c : ctx->adj_cap) *bytes += sizeof(double) * c;
    return NS3D_OK;
}

ns3d_status ns3d_synchronize(ns3d_ctx* ctx) {
    if (!ctx) return NS3D_ERR_INVALID;
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->copy_stream) NS3D_CK(cudaStreamSynchronize(ctx->copy_stream));
    return NS3D_OK;
}

ns3d_status ns3d_prefetch_primitive(ns3d_ctx* ctx, const double* rho, const double* u,
                                    const double* v, const double* w, const double* p,
                                    int layout) {
    if (!ctx) return NS3D_ERR_INVALID;
    const double* h[5] = {rho, u, v, w, p};
    for (int q = 0; q < 5; ++q)
        if (!h[q]) return fail(ctx, NS3D_ERR_INVALID, "null host pointer");
    if (layout == NS3D_LAYOUT_GHOSTED) return NS3D_OK;  // gathered on the host at upload time
    if (layout != NS3D_LAYOUT_INTERIOR) return fail(ctx, NS3D_ERR_INVALID, "unknown layout");
    NS3D_CK(cudaSetDevice(ctx->device));
    const size_t n = (size_t)ctx->n;
    if (!ctx->stage_mem) {
        if (cudaMalloc(&ctx->stage_mem, sizeof(double) * 6 * n) != cudaSuccess) {
            cudaGetLastError();
            ctx->stage_mem = nullptr;
            return fail(ctx, NS3D_ERR_NOMEM, "prefetch staging allocation failed");
        }
        ctx->stage = ctx->stage_mem;
        NS3D_CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        NS3D_CK(cudaEventCreateWithFlags(&ctx->ev_staged, cudaEventDisableTiming));
        NS3D_CK(cudaEventCreateWithFlags(&ctx->ev_consumed, cudaEventDisableTiming));
    }
    // the staging block was the current buffer's until the last upload that
    // used a prefetch: wait until the work queued before that upload is done
    NS3D_CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_consumed, 0));
    for (int q = 0; q < 5; ++q)
        NS3D_CK(cudaMemcpyAsync(ctx->stage + q * n, h[q], sizeof(double) * n,
                                cudaMemcpyHostToDevice, ctx->copy_stream));
    NS3D_CK(cudaEventRecord(ctx->ev_staged, ctx->copy_stream));
    for (int q = 0; q < 5; ++q) ctx->pre_h[q] = h[q];
    ctx->prefetched = true;
    return NS3D_OK;
}

ns3d_status ns3d_upload_primitive(ns3d_ctx* ctx, const double* rho, const double* u,
                                  const double* v, const double* w, const double* p, int layout) {
    if (!ctx) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    const double* h[5] = {rho, u, v, w, p};
    bool staged = ctx->prefetched && layout == NS3D_LAYOUT_INTERIOR;
    for (int q = 0; q < 5; ++q) staged = staged && h[q] == ctx->pre_h[q];
    ctx->prefetched = false;
    if (staged) {
        // the prefetched arrays become the current buffer's
        NS3D_CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_staged, 0));
        std::swap(ctx->slot[ctx->cur], ctx->stage);
    } else {
        double* d[5];
        for (int q = 0; q < 5; ++q) d[q] = warr(ctx, ctx->cur, q);
        ns3d_status s = upload5(ctx, h, d, layout);
        if (s != NS3D_OK) return s;
    }
    k_prim_finish<<<blocks_for(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->L.P, outv(ctx, ctx->cur));
    NS3D_CK(cudaGetLastError());
    if (staged) NS3D_CK(cudaEventRecord(ctx->ev_consumed, ctx->stream));
    ctx->rec = ctx->cur;
    ctx->dtmin_valid = false;
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

ns3d_status ns3d_upload_conserved(ns3d_ctx* ctx, const double* rho, const double* rhou,
                                  const double* rhov, const double* rhow, const double* E,
                                  int layout) {
    if (!ctx) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    const int tmpb = (ctx->cur + 1) % 3;  // a free state buffer as staging (5 of its 6 arrays)
    const double* h[5] = {rho, rhou, rhov, rhow, E};
    double* d[5];
    for (int q = 0; q < 5; ++q) d[q] = warr(ctx, tmpb, q);
    ns3d_status s = upload5(ctx, h, d, layout);
    if (s != NS3D_OK) return s;
    k_cons2prim<<<blocks_for(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->L.P, warr(ctx, tmpb, 0),
                                                                 outv(ctx, ctx->cur));
    NS3D_CK(cudaGetLastError());
    ctx->rec = ctx->cur;
    ctx->dtmin_valid = false;
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

ns3d_status ns3d_download_primitive(ns3d_ctx* ctx, double* rho, double* u, double* v, double* w,
                                    double* p, double* T, double* c, int layout) {
    if (!ctx) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    const double* d[7];
    for (int q = 0; q < 6; ++q) d[q] = warr(ctx, ctx->cur, q);
    d[6] = nullptr;
    if (c) {
        // c from primitiveToConserved; staged in a free buffer
        const int tmpb = ctx->cur == ctx->rec ? (ctx->cur + 1) % 3 : 3 - ctx->cur - ctx->rec;
        k_prim2cons<<<blocks_for(ctx->n, 256), 256, 0, ctx->stream>>>(
            ctx->L.P, view(ctx, ctx->cur), warr(ctx, tmpb, 0), warr(ctx, tmpb, 5));
        NS3D_CK(cudaGetLastError());
        d[6] = warr(ctx, tmpb, 5);
    }
    double* h[7] = {rho, u, v, w, p, T, c};
    const double fills[7] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    return download_arrays(ctx, d, h, fills, 7, layout);
}

ns3d_status ns3d_download_conserved(ns3d_ctx* ctx, double* rho, double* rhou, double* rhov,
                                    double* rhow, double* E, int layout) {
    if (!ctx) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    const int tmpb = ctx->cur == ctx->rec ? (ctx->cur + 1) % 3 : 3 - ctx->cur - ctx->rec;
    k_prim2cons<<<blocks_for(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->L.P, view(ctx, ctx->cur),
                                                                 warr(ctx, tmpb, 0), nullptr);
    NS3D_CK(cudaGetLastError());
    const double* d[5];
    for (int q = 0; q < 5; ++q) d[q] = warr(ctx, tmpb, 0) + q * ctx->n;
    double* h[5] = {rho, rhou, rhov, rhow, E};
    const double fills[5] = {1.0, 0.0, 0.0, 0.0, 0.0};
    return download_arrays(ctx, d, h, fills, 5, layout);
}

ns3d_status ns3d_record_conserved0(ns3d_ctx* ctx) {
    if (!ctx) return NS3D_ERR_INVALID;
    ctx->rec = ctx->cur;
    return NS3D_OK;
}

ns3d_status ns3d_compute_rhs(ns3d_ctx* ctx, double* r0, double* r1, double* r2, double* r3,
                             double* r4, int layout) {
    if (!ctx) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    ns3d_status s = launch_rhs_parts(ctx, view(ctx, ctx->cur), nullptr);
    if (s != NS3D_OK) return s;
    // rhs staged in a free state buffer (5 of its 6 arrays)
    const int tmpb = ctx->cur == ctx->rec ? (ctx->cur + 1) % 3 : 3 - ctx->cur - ctx->rec;
    double* rhs = warr(ctx, tmpb, 0);
    if (ctx->p.precision == NS3D_PREC_FP64)
        NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1,
                    launch_rhs_out<double>(ctx->L, (const double*)ctx->tacc, (const double*)ctx->fv, rhs));
    else
        NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1,
                    launch_rhs_out<float>(ctx->L, (const float*)ctx->tacc, (const float*)ctx->fv, rhs));
    const double* d[5];
    for (int q = 0; q < 5; ++q) d[q] = rhs + q * ctx->n;
    double* h[5] = {r0, r1, r2, r3, r4};
    const double fills[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    return download_arrays(ctx, d, h, fills, 5, layout);
}

ns3d_status ns3d_compute_timestep(ns3d_ctx* ctx, double* dt) {
    if (!ctx || !dt) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    ns3d_status s = reset_ctrl(ctx);
    if (s != NS3D_OK) return s;
    if ((s = enqueue_cfl(ctx)) != NS3D_OK) return s;
    if ((s = read_ctrl(ctx)) != NS3D_OK) return s;
    double m;
    std::memcpy(&m, &ctx->ctrl_host->dtmin_bits, sizeof(double));
    *dt = ctx->p.cfl * m;
    return NS3D_OK;
}

ns3d_status ns3d_runge_kutta_3(ns3d_ctx* ctx, double dt) {
    if (!ctx) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    ns3d_status s = reset_ctrl(ctx);
    if (s != NS3D_OK) return s;
    NS3D_CK(cudaMemcpyAsync(&ctx->ctrl->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if ((s = enqueue_rk3(ctx)) != NS3D_OK) return s;
    ctx->dtmin_valid = true;  // stage 3 left the CFL minimum of the new state in ctrl
    if ((s = read_ctrl(ctx)) != NS3D_OK) return s;
    if (ctx->ctrl_host->bad_cell < ctx->n) {
        char buf[160];
        const long long b = ctx->ctrl_host->bad_cell;
        std::snprintf(buf, sizeof(buf), "non-physical value at cell (%lld,%lld,%lld)",
                      b % ctx->p.global_nx, (b / ctx->p.global_nx) % ctx->p.global_ny,
                      b / ((long long)ctx->p.global_nx * ctx->p.global_ny));
        return fail(ctx, NS3D_ERR_NONPHYSICAL, buf);
    }
    return NS3D_OK;
}

static ns3d_status run_steps(ns3d_ctx* ctx, int mode, int nsteps, int* steps_done) {
    NS3D_CK(cudaSetDevice(ctx->device));
    ctx->step_times_n = 0;
    if (nsteps > ctx->step_times_cap) {
        // grown once to the longest call (cudaMalloc synchronises)
        NS3D_CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->step_times);
        ctx->step_times = nullptr;
        ctx->step_times_cap = 0;
        if (cudaMalloc(&ctx->step_times, sizeof(double) * (size_t)nsteps) != cudaSuccess)
            return fail(ctx, NS3D_ERR_NOMEM, "step time record allocation failed");
        ctx->step_times_cap = nsteps;
    }
    // keep the CFL minimum of the current state across calls when valid
    unsigned long long keep = 0;
    bool have = false;
    if (ctx->dtmin_valid) {
        NS3D_CK(cudaMemcpyAsync(&keep, &ctx->ctrl->dtmin_bits, sizeof(keep), cudaMemcpyDeviceToHost,
                                ctx->stream));
        NS3D_CK(cudaStreamSynchronize(ctx->stream));
        have = true;
    }
    ns3d_status s = reset_ctrl(ctx);
    if (s != NS3D_OK) return s;
    if (have)
        NS3D_CK(cudaMemcpyAsync(&ctx->ctrl->dtmin_bits, &keep, sizeof(keep), cudaMemcpyHostToDevice,
                                ctx->stream));
    else if ((s = enqueue_cfl(ctx)) != NS3D_OK)
        return s;
    const ns3d_params& p = ctx->p;
    const int cur0 = ctx->cur, rec0 = ctx->rec;
    for (int step = 0; step < nsteps; ++step) {
        ctx->rec = ctx->cur;  // recordConservedTo0 (maincycle.cpp:22)
        NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1,
                    (k_control_pre<<<1, 1, 0, ctx->stream>>>(ctx->ctrl, mode, p.cfl, p.dt_fixed,
                                                              p.TotalTime, p.output_Timefreq)));
        if ((s = enqueue_rk3(ctx)) != NS3D_OK) return s;
        NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1,
                    (k_control_post<<<1, 1, 0, ctx->stream>>>(ctx->ctrl, mode, p.TotalTime, ctx->n,
                                                               ctx->step_times)));
    }
    if ((s = read_ctrl(ctx)) != NS3D_OK) return s;
    const Ctrl& h = *ctx->ctrl_host;
    // Kernels of the iterations after a device-side stop returned at entry, so
    // the buffer rotation is that of the completed steps only: each step with
    // U0 recorded from the current buffer moves `cur` one buffer forward.
    const int d = h.steps_done;
    ctx->cur = (cur0 + d) % 3;
    if (nsteps == 0) ctx->rec = rec0;
    else if (d < nsteps && h.stop_in_pre) ctx->rec = ctx->cur;  // recorded, then stopped
    else ctx->rec = d > 0 ? (cur0 + d - 1) % 3 : rec0;
    if (steps_done) *steps_done = d;
    // a step that left a non-physical state is counted but, like the
    // reference's aborted step, records no time
    ctx->step_times_n = (h.stop && h.stop_reason == STOP_NONPHYSICAL && d > 0) ? d - 1 : d;
    ctx->steps += d;
    ctx->time = h.time;
    ctx->out_next = h.out_next;
    ctx->dtmin_valid = true;
    // if_output of the last completed step (mode 2 stops right after one), and
    // whether time_advance's loop has reached TotalTime
    ctx->last_events = (d > 0 && h.output && !h.stop_in_pre ? NS3D_EVENT_OUTPUT : 0) |
                       (h.stop && h.stop_reason == STOP_TOTAL_TIME ? NS3D_EVENT_END : 0);
    if (h.stop && h.stop_reason == STOP_NONPHYSICAL) return fail(ctx, NS3D_ERR_NONPHYSICAL, "non-physical state");
    if (h.stop && h.stop_reason == STOP_DT_SMALL) return fail(ctx, NS3D_ERR_DT, "dt too small");
    return NS3D_OK;
}

ns3d_status ns3d_step(ns3d_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return NS3D_ERR_INVALID;
    return run_steps(ctx, 0, nsteps, nullptr);
}

ns3d_status ns3d_time_advance(ns3d_ctx* ctx, int max_steps, double* time, int* steps_done) {
    if (!ctx || max_steps < 0) return NS3D_ERR_INVALID;
    int done = 0;
    ns3d_status s = run_steps(ctx, 1, max_steps, &done);
    if (time) *time = ctx->time;
    if (steps_done) *steps_done = done;
    return s;
}

ns3d_status ns3d_time_advance_segment(ns3d_ctx* ctx, int max_steps, double* time,
                                      int* steps_done, int* events) {
    if (!ctx || max_steps < 0) return NS3D_ERR_INVALID;
    int done = 0;
    ctx->last_events = 0;
    ns3d_status s = run_steps(ctx, 2, max_steps, &done);
    if (time) *time = ctx->time;
    if (steps_done) *steps_done = done;
    if (events) *events = s == NS3D_OK ? ctx->last_events : 0;
    return s;
}

ns3d_status ns3d_step_times(ns3d_ctx* ctx, double* times, int cap, int* n) {
    if (!ctx || cap < 0 || (cap > 0 && !times) || !n) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    *n = ctx->step_times_n;
    const int m = std::min(cap, ctx->step_times_n);
    if (m > 0) {
        NS3D_CK(cudaMemcpyAsync(times, ctx->step_times, sizeof(double) * m, cudaMemcpyDeviceToHost,
                                ctx->stream));
        NS3D_CK(cudaStreamSynchronize(ctx->stream));
    }
    return NS3D_OK;
}

ns3d_status ns3d_last_dt(ns3d_ctx* ctx, double* dt) {
    if (!ctx || !dt) return NS3D_ERR_INVALID;
    ns3d_status s = read_ctrl(ctx);
    if (s != NS3D_OK) return s;
    *dt = ctx->ctrl_host->dt;
    return NS3D_OK;
}

ns3d_status ns3d_residuals(ns3d_ctx* ctx, double* res) {
    if (!ctx || !res) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    static_assert(NSUMS >= 10, "the residual partials share the sums buffers");
    NS3D_LAUNCH(NS3D_KERNEL_OTHER, 2,
                (k_resid_partial<<<ctx->sums_blocks, 256, 0, ctx->stream>>>(
                     ctx->L.P, view(ctx, ctx->cur), view(ctx, ctx->rec), ctx->sums_part),
                 k_resid_final<<<1, 32, 0, ctx->stream>>>(ctx->sums_part, ctx->sums_blocks,
                                                          ctx->sums_out)));
    double h[10];
    NS3D_CK(cudaMemcpyAsync(h, ctx->sums_out, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < 5; ++q) res[q] = std::sqrt(h[q]) / h[5 + q];
    return NS3D_OK;
}

// ---- binary checkpoint
//
// The reference restarts from its Tecplot field (9 significant digits). The
// checkpoint keeps the current state buffer's six arrays (rho, u, v, w, p, T)
// bit for bit, the clock (time, next output time) and the CFL minimum of the
// state, so a run continued from it repeats the uninterrupted run exactly.
// Layout: a 96-byte header (CkptHeader, little-endian), then the six arrays of
// nx*ny*nz doubles each, x fastest.

namespace {

struct CkptHeader {
    char magic[8];               // "NS3DCKPT"
    uint32_t version, header_bytes;
    int32_t nx, ny, nz, precision;
    double time, out_next;
    uint64_t dtmin_bits;         // the CFL minimum's bit pattern when dtmin_valid
    uint32_t dtmin_valid, reserved;
    double dx, dy, dz;
    // the gas the state belongs to: T = p / (rho Rgas) is stored, and the CFL
    // minimum carries the sound speed sqrt(gamma p / rho)
    double gamma, Rgas, mu, Pr, Cp, sutherland_s;
    int64_t steps;               // completed time_advance steps (ns3d_run numbers on from it)
    uint64_t payload_hash;       // hash_words over the six arrays
};
static_assert(sizeof(CkptHeader) == 152, "checkpoint header layout");
constexpr char kCkptMagic[8] = {'N', 'S', '3', 'D', 'C', 'K', 'P', 'T'};
constexpr uint32_t kCkptVersion = 2;

// FNV-1a over 64-bit words: chunks of 2^17 words hashed on the host's threads,
// the chunk hashes folded in order, so the value does not depend on the
// thread count.
uint64_t hash_words(const uint64_t* w, long long n) {
    constexpr uint64_t kOffset = 0xcbf29ce484222325ull, kPrime = 0x100000001b3ull;
    constexpr long long C = 1ll << 17;
    const long long nch = (n + C - 1) / C;
    std::vector<uint64_t> hs((size_t)nch);
    const long long hw = std::max(1u, std::thread::hardware_concurrency());
    const int T = (int)std::max(1ll, std::min({nch, hw, 64ll}));
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
        th.emplace_back([&, t] {
            for (long long c = t; c < nch; c += T) {
                uint64_t h = kOffset;
                const long long e = std::min(n, (c + 1) * C);
                for (long long i = c * C; i < e; ++i) h = (h ^ w[i]) * kPrime;
                hs[(size_t)c] = h;
            }
        });
    for (auto& x : th) x.join();
    uint64_t h = kOffset;
    for (uint64_t x : hs) h = (h ^ x) * kPrime;
    return h;
}

bool same_bits(double a, double b) { return std::memcmp(&a, &b, sizeof a) == 0; }

}  // namespace

ns3d_status ns3d_checkpoint_write(ns3d_ctx* ctx, const char* path) {
    if (!ctx || !path) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    CkptHeader h{};
    std::memcpy(h.magic, kCkptMagic, sizeof h.magic);
    h.version = kCkptVersion;
    h.header_bytes = sizeof h;
    h.nx = ctx->p.global_nx;
    h.ny = ctx->p.global_ny;
    h.nz = ctx->p.global_nz;
    h.precision = ctx->p.precision;
    h.time = ctx->time;
    h.out_next = ctx->out_next;
    h.dtmin_valid = ctx->dtmin_valid ? 1u : 0u;
    h.dx = ctx->p.dx;
    h.dy = ctx->p.dy;
    h.dz = ctx->p.dz;
    h.gamma = ctx->p.gamma;
    h.Rgas = ctx->p.Rgas;
    h.mu = ctx->p.mu;
    h.Pr = ctx->p.Pr;
    h.Cp = ctx->p.Cp;
    h.sutherland_s = ctx->p.sutherland_s_over_tref;
    h.steps = ctx->steps;
    const long long nw = 6 * ctx->n;
    std::vector<double> buf((size_t)nw);
    if (ctx->dtmin_valid)
        NS3D_CK(cudaMemcpyAsync(&h.dtmin_bits, &ctx->ctrl->dtmin_bits, sizeof h.dtmin_bits,
                                cudaMemcpyDeviceToHost, ctx->stream));
    NS3D_CK(cudaMemcpyAsync(buf.data(), warr(ctx, ctx->cur, 0), sizeof(double) * nw,
                            cudaMemcpyDeviceToHost, ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    h.payload_hash = hash_words(reinterpret_cast<const uint64_t*>(buf.data()), nw);
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(ctx, NS3D_ERR_FILE, std::string("cannot open ") + path);
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
              std::fwrite(buf.data(), sizeof(double), (size_t)nw, f) == (size_t)nw;
    ok = std::fclose(f) == 0 && ok;
    return ok ? NS3D_OK : fail(ctx, NS3D_ERR_FILE, std::string("write failed: ") + path);
}

namespace {

// Opens `path` and checks its header against `p`; on NS3D_OK *f is positioned
// at the payload.
ns3d_status checkpoint_open(const char* path, const ns3d_params* p, CkptHeader* h, FILE** f,
                            std::string* msg) {
    *f = std::fopen(path, "rb");
    if (!*f) {
        *msg = std::string("cannot open ") + path;
        return NS3D_ERR_FILE;
    }
    ns3d_status s = NS3D_OK;
    if (std::fread(h, sizeof *h, 1, *f) != 1 || std::memcmp(h->magic, kCkptMagic, sizeof h->magic) ||
        h->version != kCkptVersion || h->header_bytes != sizeof *h) {
        *msg = std::string("not a version 2 checkpoint: ") + path;
        s = NS3D_ERR_FILE;
    } else if (h->nx != p->global_nx || h->ny != p->global_ny || h->nz != p->global_nz ||
               !same_bits(h->dx, p->dx) || !same_bits(h->dy, p->dy) || !same_bits(h->dz, p->dz)) {
        *msg = "the checkpoint's grid differs from the parameters'";
        s = NS3D_ERR_INVALID;
    } else if (!same_bits(h->gamma, p->gamma) || !same_bits(h->Rgas, p->Rgas) ||
               !same_bits(h->mu, p->mu) || !same_bits(h->Pr, p->Pr) || !same_bits(h->Cp, p->Cp) ||
               !same_bits(h->sutherland_s, p->sutherland_s_over_tref)) {
        *msg = "the checkpoint's gas (gamma, Rgas, mu, Pr, Cp or Sutherland S) differs from the "
               "parameters'";
        s = NS3D_ERR_INVALID;
    }
    if (s != NS3D_OK) {
        std::fclose(*f);
        *f = nullptr;
    }
    return s;
}

}  // namespace

ns3d_status ns3d_checkpoint_check(const char* path, const ns3d_params* p) {
    if (!path || !p) return NS3D_ERR_INVALID;
    ns3d_params q = *p;
    ns3d_params_derive(&q);
    CkptHeader h{};
    FILE* f = nullptr;
    std::string msg;
    const ns3d_status s = checkpoint_open(path, &q, &h, &f, &msg);
    if (f) std::fclose(f);
    if (s != NS3D_OK) std::fprintf(stderr, "ns3d_checkpoint_check: %s\n", msg.c_str());
    return s;
}

ns3d_status ns3d_checkpoint_read(ns3d_ctx* ctx, const char* path) {
    if (!ctx || !path) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    CkptHeader h{};
    FILE* f = nullptr;
    std::string msg;
    const ns3d_status hs = checkpoint_open(path, &ctx->p, &h, &f, &msg);
    if (hs != NS3D_OK) return fail(ctx, hs, msg);
    const long long nw = 6 * ctx->n;
    std::vector<double> buf((size_t)nw);
    const size_t got = std::fread(buf.data(), sizeof(double), (size_t)nw, f);
    std::fclose(f);
    if (got != (size_t)nw) return fail(ctx, NS3D_ERR_FILE, std::string("truncated checkpoint: ") + path);
    if (hash_words(reinterpret_cast<const uint64_t*>(buf.data()), nw) != h.payload_hash)
        return fail(ctx, NS3D_ERR_FILE, std::string("checkpoint checksum mismatch: ") + path);
    NS3D_CK(cudaMemcpyAsync(warr(ctx, ctx->cur, 0), buf.data(), sizeof(double) * nw,
                            cudaMemcpyHostToDevice, ctx->stream));
    // the CFL minimum only carries over between contexts of the same form
    ctx->dtmin_valid = h.dtmin_valid != 0 && h.precision == ctx->p.precision;
    if (ctx->dtmin_valid)
        NS3D_CK(cudaMemcpyAsync(&ctx->ctrl->dtmin_bits, &h.dtmin_bits, sizeof h.dtmin_bits,
                                cudaMemcpyHostToDevice, ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    ctx->rec = ctx->cur;
    ctx->time = h.time;
    ctx->out_next = h.out_next;
    ctx->steps = h.steps;
    return NS3D_OK;
}

ns3d_status ns3d_completed_steps(ns3d_ctx* ctx, long long* steps) {
    if (!ctx || !steps) return NS3D_ERR_INVALID;
    *steps = ctx->steps;
    return NS3D_OK;
}

ns3d_status ns3d_total_energy(ns3d_ctx* ctx, double* etot) {
    if (!ctx || !etot) return NS3D_ERR_INVALID;
    double s[NSUMS];
    ns3d_status st = compute_sums(ctx, s);
    if (st != NS3D_OK) return st;
    *etot = s[0] * (ctx->p.dx * ctx->p.dy * ctx->p.dz);
    return NS3D_OK;
}

ns3d_status ns3d_energy_spectrum(ns3d_ctx* ctx, double* Ek, int nbins) {
    if (!ctx || !Ek || nbins <= 0 || nbins > 2 * ctx->p.global_nx + 1) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    const int nx = ctx->p.global_nx, ny = ctx->p.global_ny, nz = ctx->p.global_nz;
    const int kmax = 2 * nx + 1;
    if (!ctx->fft_ready) {
        if (cufftPlan3d(&ctx->fft, nz, ny, nx, CUFFT_D2Z) != CUFFT_SUCCESS)
            return fail(ctx, NS3D_ERR_CUDA, "cufftPlan3d failed");
        cufftSetStream(ctx->fft, ctx->stream);
        NS3D_CK(cudaMalloc(&ctx->spec, sizeof(cufftDoubleComplex) * (size_t)(nx / 2 + 1) * ny * nz));
        NS3D_CK(cudaMalloc(&ctx->bins, sizeof(double) * kmax));
        const int nbu = spectrum_bins_used(nx, ny, nz);
        NS3D_CK(cudaMalloc(&ctx->spec_part, sizeof(double) * (size_t)SPEC_BLOCKS * nbu));
        if (sizeof(double) * SPEC_WARPS * nbu > 48 * 1024)
            NS3D_CK(cudaFuncSetAttribute(k_spectrum_part, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(double) * SPEC_WARPS * nbu)));
        ctx->fft_ready = true;
    }
    NS3D_CK(cudaMemsetAsync(ctx->bins, 0, sizeof(double) * kmax, ctx->stream));
    const double scale = 1.0 / (double)ctx->n;  // EnergySpectrum.cpp:88-96
    const int nbu = spectrum_bins_used(nx, ny, nz);
    for (int comp = 1; comp <= 3; ++comp) {
        if (cufftExecD2Z(ctx->fft, warr(ctx, ctx->cur, comp), ctx->spec) != CUFFT_SUCCESS)
            return fail(ctx, NS3D_ERR_CUDA, "cufftExecD2Z failed");
        NS3D_LAUNCH(NS3D_KERNEL_OTHER, 2,
                    (k_spectrum_part<<<SPEC_BLOCKS, 32 * SPEC_WARPS,
                                       sizeof(double) * SPEC_WARPS * nbu, ctx->stream>>>(
                         ctx->spec, nx, ny, nz, scale, nbu, ctx->spec_part),
                     k_spectrum_final<<<(nbu + 127) / 128, 128, 0, ctx->stream>>>(
                         ctx->spec_part, SPEC_BLOCKS, nbu, ctx->bins)));
    }
    NS3D_CK(cudaMemcpyAsync(Ek, ctx->bins, sizeof(double) * nbins, cudaMemcpyDeviceToHost, ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

// ---- discrete adjoint -------------------------------------------------------

namespace {

// Device scratch of one adjoint call, released when it goes out of scope.
struct DevBuf {
    double* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    bool alloc(size_t count) { return cudaMalloc(&p, sizeof(double) * count) == cudaSuccess; }
};

// The adjoint's scratch arrays, by role.
enum { AB_CK, AB_WS, AB_LA, AB_LB, AB_LU0, AB_LR, AB_G, AB_LG, AB_DTD, AB_LW, AB_COUNT };

// `count` doubles of adjoint scratch `slot`, kept in the context: a call that
// needs no more than an earlier one allocates nothing (allocating and freeing
// ~1 GB per call cost 0.1-0.7 s of the call, varying from call to call).
double* adj_scratch(ns3d_ctx* c, int slot, size_t count) {
    if (count > c->adj_cap[slot]) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->adj_buf[slot]);
        c->adj_buf[slot] = nullptr;
        c->adj_cap[slot] = 0;
        if (cudaMalloc(&c->adj_buf[slot], sizeof(double) * count) != cudaSuccess) {
            cudaGetLastError();
            c->adj_buf[slot] = nullptr;
            return nullptr;
        }
        c->adj_cap[slot] = count;
    }
    return c->adj_buf[slot];
}

ns3d_status adjoint_supported(ns3d_ctx* ctx) {
    if (ctx->p.precision != NS3D_PREC_FP64)
        return fail(ctx, NS3D_ERR_UNSUPPORTED, "the adjoint differentiates the FP64 form");
    if (ctx->L.rc == RC_MDCD_HYBRID)
        return fail(ctx, NS3D_ERR_UNSUPPORTED, "no adjoint for MDCD_HYBRID");
    if (ctx->L.chr)
        return fail(ctx, NS3D_ERR_UNSUPPORTED, "no adjoint for characteristic-wise reconstruction");
    return NS3D_OK;
}

ns3d_status set_dt(ns3d_ctx* ctx, double dt) {
    NS3D_CK(cudaMemcpyAsync(&ctx->ctrl->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    // a pageable source: the copy has been staged when cudaMemcpyAsync returns
    return NS3D_OK;
}

}  // namespace

ns3d_status ns3d_rhs_vjp(ns3d_ctx* ctx, const double* lam_rhs, double* lam_w) {
    if (!ctx || !lam_rhs || !lam_w) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    ns3d_status s = adjoint_supported(ctx);
    if (s != NS3D_OK) return s;
    const long long n = ctx->n;
    double* lr = adj_scratch(ctx, AB_LR, 5 * n);
    double* lw = adj_scratch(ctx, AB_LW, 5 * n);
    double* G = adj_scratch(ctx, AB_G, (size_t)adj_scratch_blocks(ctx->L) * n);
    double* lg = adj_scratch(ctx, AB_LG, 16 * n);
    if (!lr || !lw || !G || !lg) return fail(ctx, NS3D_ERR_NOMEM, "adjoint scratch allocation failed");
    NS3D_CK(cudaMemcpyAsync(lr, lam_rhs, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, ctx->stream));
    NS3D_CK(cudaMemsetAsync(lw, 0, sizeof(double) * 5 * n, ctx->stream));
    NS3D_LAUNCH(NS3D_KERNEL_OTHER, 11, adj_rhs_vjp(ctx->L, view(ctx, ctx->cur), lr, G, lg, lw));
    NS3D_CK(cudaMemcpyAsync(lam_w, lw, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

ns3d_status ns3d_step_dts(ns3d_ctx* ctx, int nsteps, const double* dts) {
    if (!ctx || nsteps < 0 || (nsteps > 0 && !dts)) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    ns3d_status s = reset_ctrl(ctx);
    if (s != NS3D_OK) return s;
    for (int k = 0; k < nsteps; ++k) {
        ctx->rec = ctx->cur;
        if ((s = set_dt(ctx, dts[k])) != NS3D_OK) return s;
        if ((s = enqueue_rk3(ctx)) != NS3D_OK) return s;
    }
    ctx->dtmin_valid = false;
    if ((s = read_ctrl(ctx)) != NS3D_OK) return s;
    if (ctx->ctrl_host->bad_cell < ctx->n) return fail(ctx, NS3D_ERR_NONPHYSICAL, "non-physical state");
    return NS3D_OK;
}

ns3d_status ns3d_adjoint(ns3d_ctx* ctx, int nsteps, int K, const double* dts_in, double* dts_out,
                         const double* lam_final, double* grad, double* J) {
    if (!ctx || nsteps < 1 || K < 1 || !grad) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    ns3d_status s = adjoint_supported(ctx);
    if (s != NS3D_OK) return s;
    const long long n = ctx->n;
    const size_t st = 6 * (size_t)n;  // one state: rho,u,v,w,p,T
    const int nseg = (nsteps + K - 1) / K;
    double* ck = adj_scratch(ctx, AB_CK, st * nseg);
    double* ws = adj_scratch(ctx, AB_WS, st * (3 * (size_t)K + 1));
    double* la = adj_scratch(ctx, AB_LA, 5 * n);
    double* lb = adj_scratch(ctx, AB_LB, 5 * n);
    double* lu0 = adj_scratch(ctx, AB_LU0, 5 * n);
    double* lr = adj_scratch(ctx, AB_LR, 5 * n);
    double* G = adj_scratch(ctx, AB_G, (size_t)adj_scratch_blocks(ctx->L) * n);
    double* lg = adj_scratch(ctx, AB_LG, 16 * n);
    double* dtd = adj_scratch(ctx, AB_DTD, nsteps);
    if (!ck || !ws || !la || !lb || !lu0 || !lr || !G || !lg || !dtd)
        return fail(ctx, NS3D_ERR_NOMEM, "adjoint checkpoint/scratch allocation failed");
    std::vector<double> dts(nsteps);

    // ---- forward run, a checkpoint every K steps, dt recorded ----
    if ((s = reset_ctrl(ctx)) != NS3D_OK) return s;
    for (int k = 0; k < nsteps; ++k) {
        if (k % K == 0)
            NS3D_CK(cudaMemcpyAsync(ck + (size_t)(k / K) * st, warr(ctx, ctx->cur, 0),
                                    sizeof(double) * st, cudaMemcpyDeviceToDevice, ctx->stream));
        ctx->rec = ctx->cur;
        if (dts_in) {
            if ((s = set_dt(ctx, dts_in[k])) != NS3D_OK) return s;
        } else {
            std::memcpy(&ctx->ctrl_host->dtmin_bits, &CFL_INIT, sizeof(double));
            NS3D_CK(cudaMemcpyAsync(&ctx->ctrl->dtmin_bits, &ctx->ctrl_host->dtmin_bits,
                                    sizeof(unsigned long long), cudaMemcpyHostToDevice, ctx->stream));
            if ((s = enqueue_cfl(ctx)) != NS3D_OK) return s;
            NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1,
                        (k_control_pre<<<1, 1, 0, ctx->stream>>>(ctx->ctrl, 0, ctx->p.cfl,
                                                                  ctx->p.dt_fixed, 0.0, 0.0)));
        }
        NS3D_CK(cudaMemcpyAsync(dtd + k, &ctx->ctrl->dt, sizeof(double), cudaMemcpyDeviceToDevice,
                                ctx->stream));
        if ((s = enqueue_rk3(ctx)) != NS3D_OK) return s;
    }
    NS3D_CK(cudaMemcpyAsync(dts.data(), dtd, sizeof(double) * nsteps, cudaMemcpyDeviceToHost,
                            ctx->stream));
    if ((s = read_ctrl(ctx)) != NS3D_OK) return s;
    if (ctx->ctrl_host->bad_cell < n) return fail(ctx, NS3D_ERR_NONPHYSICAL, "non-physical state");
    ctx->dtmin_valid = false;
    if (dts_out) std::memcpy(dts_out, dts.data(), sizeof(double) * nsteps);
    double sums[NSUMS];
    if ((s = compute_sums(ctx, sums)) != NS3D_OK) return s;
    if (J) *J = sums[0] * (ctx->p.dx * ctx->p.dy * ctx->p.dz);

    // ---- seed: dJ/dw at the end state ----
    double* A = la;
    double* B = lb;
    if (lam_final)
        NS3D_CK(cudaMemcpyAsync(A, lam_final, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, ctx->stream));
    else
        NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1,
                    adj_seed_ke(ctx->L, view(ctx, ctx->cur), A, ctx->p.dx * ctx->p.dy * ctx->p.dz));

    // ---- reverse sweep, segment by segment ----
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * K, m = std::min(K, nsteps - s0);
        NS3D_CK(cudaMemcpyAsync(ws, ck + (size_t)seg * st, sizeof(double) * st,
                                cudaMemcpyDeviceToDevice, ctx->stream));
        for (int j = 0; j < m; ++j) {  // recompute the segment's stage states
            double* w0 = ws + (size_t)(3 * j) * st;
            if ((s = set_dt(ctx, dts[s0 + j])) != NS3D_OK) return s;
            if ((s = stage_at(ctx, 1, w0, w0, w0 + st)) != NS3D_OK) return s;
            if ((s = stage_at(ctx, 2, w0 + st, w0, w0 + 2 * st)) != NS3D_OK) return s;
            if ((s = stage_at(ctx, 3, w0 + 2 * st, w0, w0 + 3 * st)) != NS3D_OK) return s;
        }
        for (int j = m - 1; j >= 0; --j) {  // A: adjoint of the step's end state
            double* w0 = ws + (size_t)(3 * j) * st;
            const double dt = dts[s0 + j];
            for (int stg = 3; stg >= 1; --stg) {
                const StateView Wk = view_at(w0 + (size_t)stg * st, n);
                const StateView Wp = view_at(w0 + (size_t)(stg - 1) * st, n);
                NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1, adj_stage(ctx->L, stg, Wk, Wp, A, lu0, lr, B, dt));
                NS3D_LAUNCH(NS3D_KERNEL_OTHER, 11, adj_rhs_vjp(ctx->L, Wp, lr, G, lg, B));
                std::swap(A, B);
            }
            NS3D_LAUNCH(NS3D_KERNEL_OTHER, 1, adj_finish(ctx->L, view_at(w0, n), lu0, A));
        }
    }
    NS3D_CK(cudaMemcpyAsync(grad, A, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, ctx->stream));
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

ns3d_status ns3d_get_stream(ns3d_ctx* ctx, void** stream) {
    if (!ctx || !stream) return NS3D_ERR_INVALID;
    *stream = (void*)ctx->stream;
    return NS3D_OK;
}

ns3d_status ns3d_profile(ns3d_ctx* ctx, int enable) {
    if (!ctx) return NS3D_ERR_INVALID;
    if (enable) {
        NS3D_CK(cudaStreamSynchronize(ctx->stream));
        ctx->prof.clear();
        ctx->ev_used = 0;
    }
    ctx->prof_on = enable != 0;
    return NS3D_OK;
}

ns3d_status ns3d_profile_read(ns3d_ctx* ctx, double* ms, long long* launches) {
    if (!ctx || !ms || !launches) return NS3D_ERR_INVALID;
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    for (int c = 0; c < NS3D_KERNEL_CLASSES; ++c) {
        ms[c] = 0.0;
        launches[c] = 0;
    }
    for (const auto& r : ctx->prof) {
        float t = 0.f;
        NS3D_CK(cudaEventElapsedTime(&t, r.a, r.b));
        ms[r.cls] += t;
        launches[r.cls] += 1;
    }
    return NS3D_OK;
}

ns3d_status ns3d_launch_count(const ns3d_ctx* ctx, long long* count) {
    if (!ctx || !count) return NS3D_ERR_INVALID;
    *count = ctx->launches;
    return NS3D_OK;
}

// compute_turbulence_statistics (ana_isotropic.cpp:196-314) from the state's
// sums and the spectrum Ek[0..kmax).
static ns3d_status stats_from(ns3d_ctx* ctx, const double* Ek, int kmax, ns3d_turb_stats* out) {
    double s[NSUMS];
    ns3d_status st = compute_sums(ctx, s);
    if (st != NS3D_OK) return st;
    const double N = (double)ctx->n;
    std::memset(out, 0, sizeof(*out));
    out->total_energy = s[0] * (ctx->p.dx * ctx->p.dy * ctx->p.dz);
    out->mean_mu = s[2] / N;
    out->mean_rho = s[3] / N;
    out->nu = out->mean_mu / out->mean_rho;
    out->kinetic_energy = s[1] / N;
    out->u_rms = std::sqrt(s[4] / (3.0 * N));
    const double mu_ = s[5] / N, mv = s[6] / N, mw = s[7] / N;
    out->tke = 0.5 * ((s[8] / N - mu_ * mu_) + (s[9] / N - mv * mv) + (s[10] / N - mw * mw));
    out->mach_t = std::sqrt(out->kinetic_energy * 2) / (s[11] / N);
    double eps = 0.0;
    for (int k = 0; k < kmax; ++k) eps += 2.0 * out->nu * (double)k * (double)k * Ek[k];
    out->dissipation = eps;
    // ana_isotropic.cpp:286-303
    out->dudx2 = s[12] / N;
    out->taylor_li = out->u_rms / std::sqrt(out->dudx2);
    out->re_lambda = out->u_rms * out->taylor_li / out->nu;
    out->eta = std::pow(out->nu * out->nu * out->nu / eps, 0.25);
    out->u_eta = std::pow(out->nu * eps, 0.25);
    out->tau_eta = std::pow(out->nu / eps, 0.5);
    out->taylor = std::sqrt(15.0 * out->nu * out->u_rms * out->u_rms / eps);
    return NS3D_OK;
}

ns3d_status ns3d_turbulence_stats(ns3d_ctx* ctx, ns3d_turb_stats* out) {
    if (!ctx || !out) return NS3D_ERR_INVALID;
    const int kmax = 2 * ctx->p.global_nx + 1;
    std::vector<double> Ek(kmax);
    ns3d_status st = ns3d_energy_spectrum(ctx, Ek.data(), kmax);
    if (st != NS3D_OK) return st;
    return stats_from(ctx, Ek.data(), kmax, out);
}

ns3d_status ns3d_turbulence_stats_spectrum(ns3d_ctx* ctx, const double* Ek, int nbins,
                                           ns3d_turb_stats* out) {
    if (!ctx || !Ek || nbins < 1 || !out) return NS3D_ERR_INVALID;
    return stats_from(ctx, Ek, nbins, out);
}

ns3d_status ns3d_init_isotropic(ns3d_ctx* ctx, int k0, double A, unsigned long long seed,
                                double mach_t) {
    if (!ctx || k0 <= 0 || !(A > 0.0)) return NS3D_ERR_INVALID;
    NS3D_CK(cudaSetDevice(ctx->device));
    const int NX = ctx->p.global_nx, NY = ctx->p.global_ny, NZ = ctx->p.global_nz;
    const long long n = ctx->n;
    const size_t plane = (size_t)3 * NX * NY;
    DevBuf r, spec;
    double* host = nullptr;
    if (!r.alloc((size_t)3 * n) || !spec.alloc((size_t)6 * n) ||
        cudaMallocHost(&host, sizeof(double) * plane) != cudaSuccess)
        return fail(ctx, NS3D_ERR_NOMEM, "init_isotropic: scratch allocation failed");
    // the uniform draws, in the reference's order (rnd01: mt19937_64 + uniform [0,1))
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    ns3d_status st = NS3D_OK;
    for (int k = 0; k < NZ && st == NS3D_OK; ++k) {
        size_t q = 0;
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                if (i == 0 && j == 0 && k == 0) {  // kk == 0: no draws
                    host[q++] = 0.0; host[q++] = 0.0; host[q++] = 0.0;
                    continue;
                }
                host[q++] = dist(rng);
                host[q++] = dist(rng);
                host[q++] = dist(rng);
            }
        if (cudaMemcpyAsync(r.p + (size_t)k * plane, host, sizeof(double) * plane,
                            cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
            st = fail(ctx, NS3D_ERR_CUDA, "init_isotropic: copy of the phases failed");
    }
    cudaFreeHost(host);
    if (st != NS3D_OK) return st;
    auto* U = reinterpret_cast<cufftDoubleComplex*>(spec.p);
    auto* V = U + n;
    auto* Wc = V + n;
    k_iso_modes<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(NX, NY, NZ, k0, A, r.p, U, V, Wc);
    NS3D_CK(cudaGetLastError());
    // inverse (backward, unnormalised) transforms, as fftw_plan_dft_3d(..., FFTW_BACKWARD)
    cufftHandle plan;
    if (cufftPlan3d(&plan, NZ, NY, NX, CUFFT_Z2Z) != CUFFT_SUCCESS)
        return fail(ctx, NS3D_ERR_CUDA, "init_isotropic: cufftPlan3d failed");
    cufftSetStream(plan, ctx->stream);
    bool ok = true;
    for (cufftDoubleComplex* c : {U, V, Wc}) ok = ok && cufftExecZ2Z(plan, c, c, CUFFT_INVERSE) == CUFFT_SUCCESS;
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    cufftDestroy(plan);
    if (!ok) return fail(ctx, NS3D_ERR_CUDA, "init_isotropic: cufftExecZ2Z failed");
    k_iso_state<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(ctx->L.P, U, V, Wc, outv(ctx, ctx->cur));
    NS3D_CK(cudaGetLastError());
    // energy normalisation: mean 0.5|u|^2 -> Ek0 = 3A/64 sqrt(2 pi) k0^5 (isotropic_ini.cpp:36,
    // 106-118), or the turbulent Mach number sqrt(2 KE) / <c> -> mach_t
    double sums[NSUMS];
    if ((st = compute_sums(ctx, sums)) != NS3D_OK) return st;
    const double PI = 3.14159265358979323846;
    const double Er = sums[1] / (double)n;
    double scale;
    if (mach_t > 0.0) {
        const double c_mean = sums[11] / (double)n;
        scale = mach_t * c_mean / std::sqrt(2.0 * Er);
    } else {
        const double Ek0 = 3.0 * A / 64.0 * std::sqrt(2 * PI) * std::pow(k0, 5);
        scale = std::sqrt(Ek0 / Er);
    }
    k_iso_scale<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(n, scale, outv(ctx, ctx->cur));
    NS3D_CK(cudaGetLastError());
    k_prim_finish<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(ctx->L.P, outv(ctx, ctx->cur));
    NS3D_CK(cudaGetLastError());
    ctx->rec = ctx->cur;
    ctx->dtmin_valid = false;
    NS3D_CK(cudaStreamSynchronize(ctx->stream));
    return NS3D_OK;
}

}  // extern "C"
