// Launchers for the stage kernels. Included by exactly one translation unit
// per compute type (ns3d_fp64.cu: double, -fmad=false; ns3d_fp32.cu: float),
// which instantiates them explicitly.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "ns3d_kernels.cuh"

namespace ns3d {

struct LaunchCfg {
    DevParams P;
    int fvs;      // FV_SW / FV_LF
    int rc;       // RC_* of the reconstruction
    int chr;      // 1: characteristic-wise reconstruction (char_recon)
    int seg[3];   // cells per thread segment along x, y, z
    cudaStream_t stream;
    int zb;       // planes per block of the 2.5-D viscous kernels (0: from the grid)
    int tiled;    // bit 0: 2.5-D visc_flux (when the box tiles); bit 1: its pipelined form
    int pipe;     // FP32 sweeps with the software-pipelined split: bit 0 the x sweep
                  // (k_sweep_x_pipe, rows of >= 128 cells), bit 1 the y / z sweeps (k_sweep_pipe)
};

// Launch-shape defaults, overridable by NS3D_TILE_ZB / NS3D_TILED / NS3D_SEG / NS3D_PIPE for
// tuning.
void default_tiling(LaunchCfg& L);

// One inviscid sweep (dir 0, 1, 2 in this order per RHS evaluation).
template <class R>
cudaError_t launch_sweep(const LaunchCfg& L, int dir, StateView W, R* tacc, const Ctrl* ctrl);
template <class R>
cudaError_t launch_visc_flux(const LaunchCfg& L, StateView W, R* fv, const Ctrl* ctrl);
template <class R>
cudaError_t launch_update(const LaunchCfg& L, int stage, StateView Wc, StateView W0,
                          const R* tacc, const R* fv, StateOut Wn, Ctrl* ctrl);
template <class R>
cudaError_t launch_rhs_out(const LaunchCfg& L, const R* tacc, const R* fv, double* rhs);
// The z sweep fused with the stage update (k_sweep_ring<2, ..., FUSE>): T_acc
// holds the x + y terms, fv the viscous fluxes of Wc; writes Wn. Component-wise
// reconstruction only (L.chr == 0; cudaErrorNotSupported otherwise).
template <class R>
cudaError_t launch_sweep_z_update(const LaunchCfg& L, int stage, StateView Wc, StateView W0,
                                  const R* tacc, const R* fv, StateOut Wn, Ctrl* ctrl);

namespace detail {

inline int threads_for(int ext) { return ext >= 128 ? 128 : (ext >= 64 ? 64 : 32); }

inline dim3 cell_grid(const DevParams& P, int th) { return dim3((P.nx + th - 1) / th, P.ny, P.nz); }

// Cells per marching segment: long segments amortise the S-1 halo splits at
// the segment start, short ones give enough threads to fill 148 SMs. One cell
// per 1024 lines, within [1, 64] (and <= len): the fastest lengths measured on
// a B200 were 1 at 32^3 (1024 lines), 4 at 64^3, 16 at 128^3 and 64 at 256^3.
inline int segment_for(int len, long long lines) {
    long long seg = lines / 1024;
    seg = seg < 1 ? 1 : (seg > 64 ? 64 : seg);
    return seg > len ? len : (int)seg;
}

}  // namespace detail

#ifdef NS3D_LAUNCH_IMPL

namespace detail {

// Launch shape of a marching sweep along DIR (threads over the line index of
// `ext`, blockIdx.y over `other`, blockIdx.z over segments of `seg` cells).
struct MarchShape {
    dim3 grid;
    int th, seg;
};
template <int DIR>
inline MarchShape march_shape(const LaunchCfg& L, int max_threads) {
    const DevParams& P = L.P;
    const int ext = DIR == 0 ? P.ny : P.nx;        // thread dimension
    const int other = DIR == 2 ? P.ny : P.nz;     // blockIdx.y dimension
    const int len = DIR == 0 ? P.nx : (DIR == 1 ? P.ny : P.nz);
    MarchShape m;
    m.seg = L.seg[DIR] > 0 ? L.seg[DIR] : segment_for(len, (long long)ext * other);
    m.th = threads_for(ext);
    if (m.th > max_threads) m.th = max_threads;
    m.grid = dim3((ext + m.th - 1) / m.th, other, (len + m.seg - 1) / m.seg);
    return m;
}

template <int DIR, class R, int FVS, int RC, bool CHR>
cudaError_t sweep_dir(const LaunchCfg& L, StateView W, R* tacc, const Ctrl* ctrl) {
    const DevParams& P = L.P;
    if (DIR == 0 && P.nx % 32 == 0) {
        const long long rows = (long long)P.ny * P.nz;
        const unsigned blocks = (unsigned)((rows + XW_WARPS - 1) / XW_WARPS);
        if constexpr (sizeof(R) == 4 && !CHR) {
            if ((L.pipe & 1) && P.nx >= 128) {
                if constexpr (FVS == FV_SW) {
                    if (P.sw_eps > 0.0) {  // the entropy fix, compiled in
                        k_sweep_x_pipe<FVS, RC, 1><<<blocks, 32 * XW_WARPS, 0, L.stream>>>(P, W, tacc, ctrl);
                        return cudaGetLastError();
                    }
                }
                k_sweep_x_pipe<FVS, RC, 0><<<blocks, 32 * XW_WARPS, 0, L.stream>>>(P, W, tacc, ctrl);
                return cudaGetLastError();
            }
            k_sweep_x_warp_f32<FVS, RC><<<blocks, 32 * XW_WARPS, 0, L.stream>>>(P, W, tacc, ctrl);
        }
        else
            k_sweep_x_warp<R, FVS, RC, CHR><<<blocks, 32 * XW_WARPS, 0, L.stream>>>(P, W, tacc, ctrl);
        return cudaGetLastError();
    }
    if constexpr (DIR != 0 && !CHR) {
        const MarchShape m = march_shape<DIR>(L, RingCfg<R>::T);
        if constexpr (sizeof(R) == 4) {
            if (L.pipe & 2) {
                if constexpr (FVS == FV_SW) {
                    if (P.sw_eps > 0.0) {  // the entropy fix, compiled in
                        k_sweep_pipe<DIR, FVS, RC, 1><<<m.grid, m.th, 0, L.stream>>>(P, W, tacc, m.seg, ctrl);
                        return cudaGetLastError();
                    }
                }
                k_sweep_pipe<DIR, FVS, RC, 0><<<m.grid, m.th, 0, L.stream>>>(P, W, tacc, m.seg, ctrl);
                return cudaGetLastError();
            }
        }
        k_sweep_ring<DIR, R, FVS, RC, false><<<m.grid, m.th, 0, L.stream>>>(
            P, W, tacc, m.seg, ctrl, FuseArgs<R>{});
        return cudaGetLastError();
    } else {
        const MarchShape m = march_shape<DIR>(L, 128);
        k_sweep<DIR, R, FVS, RC, CHR><<<m.grid, m.th, 0, L.stream>>>(P, W, tacc, m.seg, ctrl);
        return cudaGetLastError();
    }
}

template <class R, int FVS, int RC>
cudaError_t sweep_z_update(const LaunchCfg& L, const FuseArgs<R>& F, StateView Wc,
                           const R* tacc) {
    const MarchShape m = march_shape<2>(L, RingCfg<R>::T);
    k_sweep_ring<2, R, FVS, RC, true><<<m.grid, m.th, 0, L.stream>>>(
        L.P, Wc, const_cast<R*>(tacc), m.seg, F.ctrl, F);
    return cudaGetLastError();
}

// L.chr selects the characteristic-wise sweeps (du_inviscous_character).
template <class R, int FVS, int RC>
cudaError_t sweeps(const LaunchCfg& L, int dir, StateView W, R* tacc, const Ctrl* ctrl) {
    if (L.chr) {
        if (dir == 0) return sweep_dir<0, R, FVS, RC, true>(L, W, tacc, ctrl);
        if (dir == 1) return sweep_dir<1, R, FVS, RC, true>(L, W, tacc, ctrl);
        return sweep_dir<2, R, FVS, RC, true>(L, W, tacc, ctrl);
    }
    if (dir == 0) return sweep_dir<0, R, FVS, RC, false>(L, W, tacc, ctrl);
    if (dir == 1) return sweep_dir<1, R, FVS, RC, false>(L, W, tacc, ctrl);
    return sweep_dir<2, R, FVS, RC, false>(L, W, tacc, ctrl);
}

template <class R, int FVS>
cudaError_t sweeps_rc(const LaunchCfg& L, int dir, StateView W, R* tacc, const Ctrl* ctrl) {
    switch (L.rc) {
    case RC_WENO5: return sweeps<R, FVS, RC_WENO5>(L, dir, W, tacc, ctrl);
    case RC_LINEAR: return sweeps<R, FVS, RC_LINEAR>(L, dir, W, tacc, ctrl);
    case RC_LIN6: return sweeps<R, FVS, RC_LIN6>(L, dir, W, tacc, ctrl);
    case RC_MDCD_HYBRID: return sweeps<R, FVS, RC_MDCD_HYBRID>(L, dir, W, tacc, ctrl);
    case RC_LIN8: return sweeps<R, FVS, RC_LIN8>(L, dir, W, tacc, ctrl);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace detail

template <class R>
cudaError_t launch_sweep(const LaunchCfg& L, int dir, StateView W, R* tacc, const Ctrl* ctrl) {
    return L.fvs == FV_SW ? detail::sweeps_rc<R, FV_SW>(L, dir, W, tacc, ctrl)
                          : detail::sweeps_rc<R, FV_LF>(L, dir, W, tacc, ctrl);
}

template <class R>
cudaError_t launch_sweep_z_update(const LaunchCfg& L, int stage, StateView Wc, StateView W0,
                                  const R* tacc, const R* fv, StateOut Wn, Ctrl* ctrl) {
    if (L.chr) return cudaErrorNotSupported;
    const FuseArgs<R> F{stage, W0, fv, Wn, ctrl};
    auto by_rc = [&](auto fvs) -> cudaError_t {
        constexpr int FVS = decltype(fvs)::value;
        switch (L.rc) {
        case RC_WENO5: return detail::sweep_z_update<R, FVS, RC_WENO5>(L, F, Wc, tacc);
        case RC_LINEAR: return detail::sweep_z_update<R, FVS, RC_LINEAR>(L, F, Wc, tacc);
        case RC_LIN6: return detail::sweep_z_update<R, FVS, RC_LIN6>(L, F, Wc, tacc);
        case RC_MDCD_HYBRID: return detail::sweep_z_update<R, FVS, RC_MDCD_HYBRID>(L, F, Wc, tacc);
        case RC_LIN8: return detail::sweep_z_update<R, FVS, RC_LIN8>(L, F, Wc, tacc);
        default: return cudaErrorInvalidValue;
        }
    };
    return L.fvs == FV_SW ? by_rc(std::integral_constant<int, FV_SW>{})
                          : by_rc(std::integral_constant<int, FV_LF>{});
}

namespace detail {
template <class R>
inline bool tiles_25d(const LaunchCfg& L, int bit) {
    return (L.tiled & bit) && L.zb >= 0 && L.P.nx % VTile<R>::X == 0 && L.P.ny % VTile<R>::Y == 0;
}
// Planes per block of the 2.5-D kernels: L.zb when set, else 16 halved until
// the grid has at least 4 blocks per SM (32^3: 1 plane, 128^3: 8, 256^3: 16).
template <class R>
inline int zb_for(const LaunchCfg& L) {
    if (L.zb > 0) return L.zb;
    const long long tiles = (long long)(L.P.nx / VTile<R>::X) * (L.P.ny / VTile<R>::Y);
    int zb = 16;
    while (zb > 1 && tiles * ((L.P.nz + zb - 1) / zb) < 4 * 148) zb >>= 1;
    return zb;
}
template <class R>
inline dim3 grid_25d(const LaunchCfg& L) {
    const int zb = zb_for<R>(L);
    return dim3(L.P.nx / VTile<R>::X, L.P.ny / VTile<R>::Y, (L.P.nz + zb - 1) / zb);
}
// k_visc_flux_pipe<R, ORD>: more than 48 KB of dynamic shared memory, opted
// in once per instantiation and device (setting it twice is harmless).
template <class R, int ORD>
cudaError_t visc_pipe(const LaunchCfg& L, StateView W, R* fv, const Ctrl* ctrl) {
    constexpr int sm = (int)VPipe<R>::smem_bytes;
    static bool opted[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !opted[dev]) {
        e = cudaFuncSetAttribute(k_visc_flux_pipe<R, ORD>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) opted[dev] = true;
    }
    const dim3 g = grid_25d<R>(L), b(VTile<R>::X, VTile<R>::Y);
    k_visc_flux_pipe<R, ORD><<<g, b, sm, L.stream>>>(L.P, W, fv, ctrl, zb_for<R>(L));
    return cudaGetLastError();
}
}  // namespace detail

template <class R>
cudaError_t launch_visc_flux(const LaunchCfg& L, StateView W, R* fv, const Ctrl* ctrl) {
    if (detail::tiles_25d<R>(L, 1) && (L.tiled & 2)) {
        switch (L.P.vis_order) {
        case 4: return detail::visc_pipe<R, 4>(L, W, fv, ctrl);
        case 6: return detail::visc_pipe<R, 6>(L, W, fv, ctrl);
        default: return detail::visc_pipe<R, 8>(L, W, fv, ctrl);
        }
    }
    if (detail::tiles_25d<R>(L, 1)) {
        const dim3 g = detail::grid_25d<R>(L), b(VTile<R>::X, VTile<R>::Y);
        switch (L.P.vis_order) {
        case 4: k_visc_flux_25d<R, 4><<<g, b, 0, L.stream>>>(L.P, W, fv, ctrl, detail::zb_for<R>(L)); break;
        case 6: k_visc_flux_25d<R, 6><<<g, b, 0, L.stream>>>(L.P, W, fv, ctrl, detail::zb_for<R>(L)); break;
        default: k_visc_flux_25d<R, 8><<<g, b, 0, L.stream>>>(L.P, W, fv, ctrl, detail::zb_for<R>(L)); break;
        }
        return cudaGetLastError();
    }
    const int th = detail::threads_for(L.P.nx);
    const dim3 g = detail::cell_grid(L.P, th);
    switch (L.P.vis_order) {
    case 4: k_visc_flux<R, 4><<<g, th, 0, L.stream>>>(L.P, W, fv, ctrl); break;
    case 6: k_visc_flux<R, 6><<<g, th, 0, L.stream>>>(L.P, W, fv, ctrl); break;
    default: k_visc_flux<R, 8><<<g, th, 0, L.stream>>>(L.P, W, fv, ctrl); break;
    }
    return cudaGetLastError();
}

template <class R, int ORD>
static cudaError_t update_ord(const LaunchCfg& L, int stage, StateView Wc, StateView W0,
                              const R* tacc, const R* fv, StateOut Wn, Ctrl* ctrl) {
    const int th = detail::threads_for(L.P.nx);
    const dim3 g = detail::cell_grid(L.P, th);
    if (stage == 1) k_update<R, ORD, 1><<<g, th, 0, L.stream>>>(L.P, Wc, W0, tacc, fv, Wn, ctrl);
    else if (stage == 2) k_update<R, ORD, 2><<<g, th, 0, L.stream>>>(L.P, Wc, W0, tacc, fv, Wn, ctrl);
    else k_update<R, ORD, 3><<<g, th, 0, L.stream>>>(L.P, Wc, W0, tacc, fv, Wn, ctrl);
    return cudaGetLastError();
}

template <class R>
cudaError_t launch_update(const LaunchCfg& L, int stage, StateView Wc, StateView W0,
                          const R* tacc, const R* fv, StateOut Wn, Ctrl* ctrl) {
    switch (L.P.vis_order) {
    case 4: return update_ord<R, 4>(L, stage, Wc, W0, tacc, fv, Wn, ctrl);
    case 6: return update_ord<R, 6>(L, stage, Wc, W0, tacc, fv, Wn, ctrl);
    default: return update_ord<R, 8>(L, stage, Wc, W0, tacc, fv, Wn, ctrl);
    }
}

template <class R>
cudaError_t launch_rhs_out(const LaunchCfg& L, const R* tacc, const R* fv, double* rhs) {
    const int th = detail::threads_for(L.P.nx);
    const dim3 g = detail::cell_grid(L.P, th);
    switch (L.P.vis_order) {
    case 4: k_rhs_out<R, 4><<<g, th, 0, L.stream>>>(L.P, tacc, fv, rhs); break;
    case 6: k_rhs_out<R, 6><<<g, th, 0, L.stream>>>(L.P, tacc, fv, rhs); break;
    default: k_rhs_out<R, 8><<<g, th, 0, L.stream>>>(L.P, tacc, fv, rhs); break;
    }
    return cudaGetLastError();
}

#define NS3D_INSTANTIATE_LAUNCHERS(R)                                                          \
    template cudaError_t launch_sweep<R>(const LaunchCfg&, int, StateView, R*, const Ctrl*);   \
    template cudaError_t launch_visc_flux<R>(const LaunchCfg&, StateView, R*, const Ctrl*);    \
    template cudaError_t launch_update<R>(const LaunchCfg&, int, StateView, StateView,         \
                                          const R*, const R*, StateOut, Ctrl*);                \
    template cudaError_t launch_rhs_out<R>(const LaunchCfg&, const R*, const R*, double*);   \
    template cudaError_t launch_sweep_z_update<R>(const LaunchCfg&, int, StateView, StateView, \
                                                  const R*, const R*, StateOut, Ctrl*);

#endif  // NS3D_LAUNCH_IMPL

}  // namespace ns3d
