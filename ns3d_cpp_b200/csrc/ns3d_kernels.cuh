// Kernels of one RK3 stage, templated on the compute type R (double or float).
//
// Device layout (HBM): interior-only SoA arrays of n = nx*ny*nz doubles,
// x fastest. The periodic ghost fill of the reference (apply_boundary +
// primitiveToConserved, field_structures.h:795-853) becomes index wrap-around
// in the loaders: a ghost value of the reference is bit-identical to its
// periodic image, so nothing is copied.
//
// State per buffer: primitives rho,u,v,w,p plus T (= p/(rho Rgas) exactly as
// primitiveToConserved computes it). Conserved values (rhou, E) and c are
// recomputed on the fly with the reference's expressions, which reproduces
// the cons->prim->cons round trip of every stage bit for bit.
//
// One stage = sweep_x, sweep_y, sweep_z (inviscid, accumulating
// T_acc = ((ax*idx + ay*idy) + az*idz) in the reference's order), visc_flux
// (gradients + stresses), update (viscous divergence, rhs, Shu-Osher stage in
// double, conservedToPrimitive, next-step CFL candidates and positivity after
// stage 3).
#pragma once

#include "ns3d_device.cuh"
#include <type_traits>

namespace ns3d {

struct StateView {
    const double *rho, *u, *v, *w, *p, *T;
};
struct StateOut {
    double *rho, *u, *v, *w, *p, *T;
};

// Device-side control block of the time loop (maincycle.cpp:14-52).
struct Ctrl {
    unsigned long long dtmin_bits;   // running min of the CFL candidates (bit pattern)
    unsigned long long pad0;
    double dt;                       // dt of the step in flight
    double time;                     // current_time
    double out_next;                 // next scheduled output time
    int stop;                        // 1: the loop has ended, kernels return at entry
    int stop_reason;                 // NS3D_STOP_*
    int steps_done;
    int active;                      // a step is in flight
    long long bad_cell;              // first non-physical cell (linear index), or n
    int stop_in_pre;                 // the stop came from the start-of-iteration checks
    int output;                      // if_output of the last iteration begun (maincycle.cpp:33-45)
};

enum : int { STOP_NONE = 0, STOP_TOTAL_TIME = 1, STOP_DT_SMALL = 2, STOP_NONPHYSICAL = 3,
             STOP_OUTPUT = 4 };

constexpr double CFL_INIT = 1e9;     // timestep.cpp:8

__device__ __forceinline__ int wrap1(int s, int len) {
    return s < 0 ? s + len : (s >= len ? s - len : s);
}

// ---------------------------------------------------------------------------
// One face of du_inviscous_character (InviscousFlux_new.cpp:165-437): the Roe
// state of the face's two cells wl, wr (primitives, rho as stored), the
// eigenvector matrices along DIR, the windows projected on the left
// eigenvectors (sums from 0 in the reference's order), one reconstruction per
// characteristic field and the result mapped back by the right ones.
// FP(m, r) / FM(m, r): split flux component r of window cell m (unreversed;
// the minus window is reversed here as reconstruct_select does). In the FP32
// form the windows are deviations from a common offset, which the projection
// and reconstruction carry through (R L ref = ref cancels in the difference).
// ---------------------------------------------------------------------------
template <int DIR, class R, int RC, class GP, class GM>
__device__ __forceinline__ void char_face(double gamma, const double* wl, const double* wr,
                                          GP FP, GM FM, const R* lin, R disp, R diss,
                                          R face[5]) {
    constexpr int S = Stencil<RC>::S;
    double ua[5], Lm[5][5], Rm[5][5];
    roe_state(gamma, wl, wr, ua);
    eigen_LR<DIR == 0, DIR == 1, DIR == 2>(gamma, ua, Lm, Rm);
    R wc[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        R a[S], bc[S], b[S];
#pragma unroll
        for (int m = 0; m < S; ++m) {
            R sp = R(0.0), sm = R(0.0);
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                sp += R(Lm[q][r]) * FP(m, r);
                sm += R(Lm[q][r]) * FM(m, r);
            }
            a[m] = sp;
            bc[m] = sm;
        }
#pragma unroll
        for (int m = 0; m < S; ++m) b[m] = bc[S - 1 - m];
        const R plus_face = reconstruct<R, RC>(a, lin, disp, diss);
        const R minus_face = reconstruct<R, RC>(b, lin, disp, diss);
        wc[q] = plus_face + minus_face;
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        R sum = R(0.0);
#pragma unroll
        for (int r = 0; r < 5; ++r) sum += R(Rm[q][r]) * wc[r];
        face[q] = sum;
    }
}

// ---------------------------------------------------------------------------
// Split-flux storage of the sweeps in shared memory. A slot holds one cell's
// split fluxes, FP32: (F+0..3) float4, (F-0..3) float4, (F+4, F-4) float2 --
// exactly the operand pairs of the paired WENO5; FP64: five double2. The
// arrays are [slot][t]: threads with consecutive t read consecutive 8- or
// 16-byte words (no bank conflicts).
// ---------------------------------------------------------------------------
// Blocks per SM the ring sweeps are compiled for (register cap 65536 / (T MINB)).
#ifndef NS3D_RING_MINB_F32
#define NS3D_RING_MINB_F32 4
#endif
#ifndef NS3D_RING_MINB_F64
#define NS3D_RING_MINB_F64 6
#endif
#ifndef NS3D_RING_T_F32
#define NS3D_RING_T_F32 128
#endif
template <class R> struct RingCfg;
template <> struct RingCfg<float> { static constexpr int T = NS3D_RING_T_F32, MINB = NS3D_RING_MINB_F32; };
template <> struct RingCfg<double> { static constexpr int T = 64, MINB = NS3D_RING_MINB_F64; };

template <class R, int S, int T> struct SplitRing;
template <int S, int T> struct SplitRing<float, S, T> {
    float4 p[S][T];   // F+0..3
    float4 m[S][T];   // F-0..3
    float2 e[S][T];   // F+4, F-4
    __device__ __forceinline__ void put(int slot, int t, const float* Fp, const float* Fm) {
        p[slot][t] = make_float4(Fp[0], Fp[1], Fp[2], Fp[3]);
        m[slot][t] = make_float4(Fm[0], Fm[1], Fm[2], Fm[3]);
        e[slot][t] = make_float2(Fp[4], Fm[4]);
    }
    __device__ __forceinline__ void get(int slot, int t, float* Fp, float* Fm) const {
        const float4 a = p[slot][t], b = m[slot][t];
        const float2 c = e[slot][t];
        Fp[0] = a.x; Fp[1] = a.y; Fp[2] = a.z; Fp[3] = a.w; Fp[4] = c.x;
        Fm[0] = b.x; Fm[1] = b.y; Fm[2] = b.z; Fm[3] = b.w; Fm[4] = c.y;
    }
    // component q of F+ (minus = false) or F- of one slot (one scalar load)
    __device__ __forceinline__ float comp(int slot, int t, int q, bool minus) const {
        if (q == 4) return reinterpret_cast<const float*>(&e[slot][t])[minus ? 1 : 0];
        return reinterpret_cast<const float*>(minus ? &m[slot][t] : &p[slot][t])[q];
    }
};
template <int S, int T> struct SplitRing<double, S, T> {
    double2 a[S][5][T];   // (F+0,F+1) (F+2,F+3) (F-0,F-1) (F-2,F-3) (F+4,F-4)
    __device__ __forceinline__ void put(int slot, int t, const double* Fp, const double* Fm) {
        a[slot][0][t] = make_double2(Fp[0], Fp[1]);
        a[slot][1][t] = make_double2(Fp[2], Fp[3]);
        a[slot][2][t] = make_double2(Fm[0], Fm[1]);
        a[slot][3][t] = make_double2(Fm[2], Fm[3]);
        a[slot][4][t] = make_double2(Fp[4], Fm[4]);
    }
    __device__ __forceinline__ void get(int slot, int t, double* Fp, double* Fm) const {
        const double2 x0 = a[slot][0][t], x1 = a[slot][1][t], x2 = a[slot][2][t];
        const double2 x3 = a[slot][3][t], x4 = a[slot][4][t];
        Fp[0] = x0.x; Fp[1] = x0.y; Fp[2] = x1.x; Fp[3] = x1.y; Fp[4] = x4.x;
        Fm[0] = x2.x; Fm[1] = x2.y; Fm[2] = x3.x; Fm[3] = x3.y; Fm[4] = x4.y;
    }
    __device__ __forceinline__ double comp(int slot, int t, int q, bool minus) const {
        if (q == 4) return reinterpret_cast<const double*>(&a[slot][4][t])[minus ? 1 : 0];
        return reinterpret_cast<const double*>(&a[slot][(minus ? 2 : 0) + (q >> 1)][t])[q & 1];
    }
};

// The window of phase PH (window position m in slot (PH + m) mod S) into
// registers; the slots are compile-time, so every load has an immediate offset.
template <int PH, class R, int S, int T>
__device__ __forceinline__ void ring_window(const SplitRing<R, S, T>& rg, int t, R fp[][5],
                                            R fm[][5]) {
#pragma unroll
    for (int m = 0; m < S; ++m) rg.get((PH + m) % S, t, fp[m], fm[m]);
}
template <class R, int S, int T>
__device__ __forceinline__ void ring_window_at(int ph, const SplitRing<R, S, T>& rg, int t,
                                               R fp[][5], R fm[][5]) {
    switch (ph) {
    case 0: ring_window<0>(rg, t, fp, fm); break;
    case 1: ring_window<1 % S>(rg, t, fp, fm); break;
    case 2: ring_window<2 % S>(rg, t, fp, fm); break;
    case 3: ring_window<3 % S>(rg, t, fp, fm); break;
    case 4: ring_window<4 % S>(rg, t, fp, fm); break;
    case 5: ring_window<5 % S>(rg, t, fp, fm); break;
    case 6: ring_window<6 % S>(rg, t, fp, fm); break;
    default: ring_window<7 % S>(rg, t, fp, fm); break;
    }
}

// ---------------------------------------------------------------------------
// Inviscid sweep along DIR (du_inviscous, InviscousFlux_new.cpp:4-163, and the
// divergence of range_kutta.cpp:51-98).
//
// One thread marches along one line segment of `seg` cells, holding the split
// fluxes of the S cells of the current face window in registers: each cell is
// split once, every face is reconstructed once, and the face flux of the
// previous face is kept for the difference. Split fluxes never touch memory.
//   DIR 0: lines over (j,k), threads over j        (march along x)
//   DIR 1: lines over (i,k), threads over i        (coalesced along x)
//   DIR 2: lines over (i,j), threads over i        (coalesced along x)
// T_acc (5 blocks of n, type R): DIR 0 writes ax*idx, DIR 1 and 2 add.
// ---------------------------------------------------------------------------
template <int DIR, class R, int FVS, int RC, bool CHR = false>
__global__ void __launch_bounds__(128)
k_sweep(DevParams P, StateView W, R* __restrict__ tacc, int seg, const Ctrl* __restrict__ ctrl) {
    if (ctrl && ctrl->stop) return;
    constexpr int S = Stencil<RC>::S;
    constexpr int MID = (S - 1) / 2;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = P.n;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    long long base, stride;
    int len;
    if constexpr (DIR == 0) {
        if (t0 >= ny) return;
        base = ((long long)blockIdx.y * ny + t0) * nx;
        stride = 1;
        len = nx;
    } else if constexpr (DIR == 1) {
        if (t0 >= nx) return;
        base = (long long)blockIdx.y * ny * nx + t0;
        stride = nx;
        len = ny;
    } else {
        if (t0 >= nx) return;
        base = (long long)blockIdx.y * nx + t0;
        stride = (long long)nx * ny;
        len = nz;
    }
    const int c0 = blockIdx.z * seg;
    if (c0 >= len) return;
    const int c1 = min(c0 + seg, len);

    const R gamma = R(P.gamma), eps = R(P.sw_eps);
    R lin[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) lin[m] = R(P.lin[m]);
    const R disp = R(P.mdcd_disp), diss = R(P.mdcd_diss);
    const R inv_h = R(DIR == 0 ? P.inv_dx : (DIR == 1 ? P.inv_dy : P.inv_dz));

    R fp[S][5], fm[S][5];
    // FP32-stencil form: the split is evaluated in double from the double
    // state and the segment's first split flux is subtracted before rounding
    // to float, so the float reconstruction works on deviations of size
    // O(variation) instead of O(value) (p ~ 1/(gamma Ma^2) otherwise leaves
    // ~1e-4 relative error in pressure gradients). Every reconstruction is
    // shift-invariant (weights from differences, coefficients summing to 1)
    // and the offset is the same for both faces of a cell, so it cancels in the
    // face-flux difference. The FP64 form keeps the reference's arithmetic.
    constexpr bool kDeviation = sizeof(R) < sizeof(double);
    double refp[5], refm[5];
    const double inv_gm1 = kDeviation ? 1.0 / (P.gamma - 1.0) : 0.0;
    const double inv_2g = kDeviation ? 1.0 / (2.0 * P.gamma) : 0.0;
    // Loads of one cell's primitives are issued a step before the cell is
    // split (`load_raw` into registers), so their latency hides behind the
    // reconstruction of the current face instead of stalling the march.
    auto load_raw = [&](int s, double* raw) {
        const long long id = base + (long long)wrap1(s, len) * stride;
        raw[0] = W.rho[id];
        raw[1] = W.u[id];
        raw[2] = W.v[id];
        raw[3] = W.w[id];
        raw[4] = W.p[id];
    };
    auto split_raw = [&](const double* raw, R* Fp, R* Fm, bool set_ref) {
        if constexpr (!kDeviation) {
            R rr = R(raw[0]);
            const R u = R(raw[1]), v = R(raw[2]), w = R(raw[3]), p = R(raw[4]);
            if (rr <= R(0)) rr = R(1e-12);
            R E, c;
            p2c_Ec(rr, u, v, w, p, gamma, E, c);
            if constexpr (FVS == FV_SW)
                split_sw<R, DIR == 0, DIR == 1, DIR == 2>(rr, u, v, w, E, p, c, gamma, eps, Fp, Fm);
            else
                split_lf<R, DIR == 0, DIR == 1, DIR == 2>(rr, u, v, w, E, p, c, Fp, Fm);
        } else {
            double Fpd[5], Fmd[5];
            split_fast<FVS, DIR == 0, DIR == 1, DIR == 2>(P, inv_gm1, inv_2g, raw, Fpd, Fmd);
            if (set_ref) {
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    refp[q] = Fpd[q];
                    refm[q] = Fmd[q];
                }
            }
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                Fp[q] = R(Fpd[q] - refp[q]);
                Fm[q] = R(Fmd[q] - refm[q]);
            }
        }
    };
    (void)gamma;
    (void)eps;
    // CHR: the face's two cells are reloaded (L1/L2 hits); rho as stored.
    auto char_face_at = [&](int f, R* face) {
        double wl[5], wr[5];
        load_raw(f, wl);
        load_raw(f + 1, wr);
        char_face<DIR, R, RC>(P.gamma, wl, wr, [&](int m, int r) { return fp[m][r]; },
                              [&](int m, int r) { return fm[m][r]; }, lin, disp, diss, face);
    };
    (void)char_face_at;

    int f = c0 - 1;  // face f sits between cells f and f+1 (the reference's i_face = f + ng)
    double nxt[5];
#pragma unroll
    for (int m = 0; m < S - 1; ++m) {
        load_raw(f - MID + m, nxt);
        split_raw(nxt, fp[m], fm[m], m == 0);
    }
    load_raw(f - MID + S - 1, nxt);
    R prev[5];
    for (int t = 0; f < c1; ++t, ++f) {
        double cur[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) cur[q] = nxt[q];
        // the following cell (in range by wrap-around even past the segment end)
        load_raw(f - MID + S, nxt);
        R old[5];
        const long long oid = base + (long long)f * stride;
        if constexpr (DIR != 0) {
            if (t > 0) {
#pragma unroll
                for (int q = 0; q < 5; ++q) old[q] = tacc[q * n + oid];
            }
        }
        split_raw(cur, fp[S - 1], fm[S - 1], false);
        R face[5];
        if constexpr (CHR) {
            char_face_at(f, face);
        } else if constexpr (kDeviation && RC == RC_WENO5) {
            // reconstruct_select reverses the minus window (flag < 0)
            weno5_face_x2([&](int m, int q) { return fp[m][q]; },
                          [&](int m, int q) { return fm[S - 1 - m][q]; }, face);
        } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                R a[S], b[S];
#pragma unroll
                for (int m = 0; m < S; ++m) {
                    a[m] = fp[m][q];
                    b[m] = fm[S - 1 - m][q];  // reconstruct_select reverses for flag < 0
                }
                const R plus_face = reconstruct<R, RC>(a, lin, disp, diss);
                const R minus_face = reconstruct<R, RC>(b, lin, disp, diss);
                face[q] = plus_face + minus_face;
            }
        }
        if (t > 0) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const R d = face[q] - prev[q];
                if constexpr (DIR == 0)
                    tacc[q * n + oid] = d * inv_h;
                else
                    tacc[q * n + oid] = old[q] + d * inv_h;
            }
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) prev[q] = face[q];
#pragma unroll
        for (int m = 0; m < S - 1; ++m)
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                fp[m][q] = fp[m + 1][q];
                fm[m][q] = fm[m + 1][q];
            }
    }
}

// ---------------------------------------------------------------------------
// x sweep, warp per periodic row (nx a multiple of 32). Lanes hold 32
// consecutive cells, so loads and stores are coalesced; the split fluxes of
// the previous, current and next 32-cell chunks live in a per-warp shared
// ring, and every lane reconstructs one face per chunk. The face on the -x
// side of a lane's cell comes from the neighbouring lane (shuffle). Each cell
// of the row is split exactly once: the last and first chunks, needed twice by
// periodicity, are kept in registers. Same arithmetic per face and cell as
// k_sweep<0> (the FP64 results are identical); in the FP32-stencil form the
// split-flux offset is the row's first cell.
// ---------------------------------------------------------------------------
#ifndef NS3D_XW_WARPS
#define NS3D_XW_WARPS 4
#endif
constexpr int XW_WARPS = NS3D_XW_WARPS;

template <class R, int FVS, int RC, bool CHR>
__device__ __forceinline__ void x_sweep_row(const DevParams& P, const StateView& W,
                                            R* __restrict__ tacc, SplitRing<R, XW_WARPS, 96>& ring,
                                            int wq, int lane, long long row);

template <class R, int FVS, int RC, bool CHR = false>
__global__ void __launch_bounds__(32 * XW_WARPS)
k_sweep_x_warp(DevParams P, StateView W, R* __restrict__ tacc, const Ctrl* __restrict__ ctrl) {
    if (ctrl && ctrl->stop) return;
    __shared__ SplitRing<R, XW_WARPS, 96> ring;  // [warp][3 chunks x 32 cells]
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const long long row = (long long)blockIdx.x * XW_WARPS + wq;
    if (row >= (long long)P.ny * P.nz) return;  // warp-uniform
    x_sweep_row<R, FVS, RC, CHR>(P, W, tacc, ring, wq, lane, row);
}

// The FP32 component-wise form of k_sweep_x_warp, capped at 128 registers
// (4 blocks of 128 threads per SM): left to itself the compiler takes 154 and
// fits 3 blocks (measured at 256^3: 0.502 ms uncapped, 0.483 ms capped, with
// 8 / 12 bytes of spills).
template <int FVS, int RC>
__global__ void __maxnreg__(128)
k_sweep_x_warp_f32(DevParams P, StateView W, float* __restrict__ tacc, const Ctrl* __restrict__ ctrl) {
    if (ctrl && ctrl->stop) return;
    __shared__ SplitRing<float, XW_WARPS, 96> ring;
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const long long row = (long long)blockIdx.x * XW_WARPS + wq;
    if (row >= (long long)P.ny * P.nz) return;  // warp-uniform
    x_sweep_row<float, FVS, RC, false>(P, W, tacc, ring, wq, lane, row);
}

// FP32-form x sweep with the split software-pipelined (rows of at least four
// 32-cell chunks). A warp's ring has four rotating chunk slots (chunk k in
// slot k mod 4) and a fifth that keeps chunk 0 for the last chunk's +x
// neighbour. While the faces of chunk c are reconstructed from chunks c-1, c,
// c+1, the split of chunk c+2 runs beside them (independent chains, no
// branch: ENT fixes the entropy-fix choice, square roots from sqrt_nr_nb) and
// goes into the slot of chunk c-2, which no lane reads any more; one
// __syncwarp per chunk then makes it visible. Chunk 0's double split serves
// as the row's offset (lane 0's value). Faces, the periodic seam and the
// T_acc writes as in x_sweep_row.
template <int FVS, int RC, int ENT>
__global__ void __launch_bounds__(32 * XW_WARPS, 4)
k_sweep_x_pipe(DevParams P, StateView W, float* __restrict__ tacc, const Ctrl* __restrict__ ctrl) {
    if (ctrl && ctrl->stop) return;
    constexpr int S = Stencil<RC>::S;
    constexpr int MID = (S - 1) / 2;
    __shared__ SplitRing<float, XW_WARPS, 160> ring;  // [warp][5 slots x 32 cells]
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const long long row = (long long)blockIdx.x * XW_WARPS + wq;
    if (row >= (long long)P.ny * P.nz) return;  // warp-uniform
    const int nx = P.nx;
    const long long n = P.n;
    const long long base = row * nx;
    const int nch = nx >> 5;  // >= 4 (the launcher's condition)
    float lin[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) lin[m] = float(P.lin[m]);
    const float disp = float(P.mdcd_disp), diss = float(P.mdcd_diss);
    const float inv_h = float(P.inv_dx);
    const double inv_gm1 = 1.0 / (P.gamma - 1.0);
    const double inv_2g = 1.0 / (2.0 * P.gamma);
    double refp[5], refm[5];
    auto load_raw = [&](int chunk, double* raw) {
        const long long id = base + (chunk << 5) + lane;
        raw[0] = W.rho[id];
        raw[1] = W.u[id];
        raw[2] = W.v[id];
        raw[3] = W.w[id];
        raw[4] = W.p[id];
    };
    auto split_d = [&](const double* raw, double* Fpd, double* Fmd) {
        split_fast<FVS, 1, 0, 0, 1, ENT, true>(P, inv_gm1, inv_2g, raw, Fpd, Fmd);
    };
    auto split_raw = [&](const double* raw, float* Fp, float* Fm) {
        double Fpd[5], Fmd[5];
        split_d(raw, Fpd, Fmd);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            Fp[q] = float(Fpd[q] - refp[q]);
            Fm[q] = float(Fmd[q] - refm[q]);
        }
    };
    auto put = [&](int slot, const float* Fp, const float* Fm) {
        ring.put(wq, slot * 32 + lane, Fp, Fm);
    };

    // prologue: chunk 0 (slots 0 and 4; lane 0's split is the offset), the last
    // chunk (slot 3, as chunk -1) and chunk 1 (slot 1); chunk 2's loads issued
    double raw[5], nxt[5];
    {
        float Fp[5], Fm[5];
        double Fpd[5], Fmd[5];
        load_raw(0, raw);
        split_d(raw, Fpd, Fmd);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            refp[q] = __shfl_sync(0xffffffffu, Fpd[q], 0);
            refm[q] = __shfl_sync(0xffffffffu, Fmd[q], 0);
            Fp[q] = float(Fpd[q] - refp[q]);
            Fm[q] = float(Fmd[q] - refm[q]);
        }
        put(0, Fp, Fm);
        put(4, Fp, Fm);
        load_raw(nch - 1, raw);
        split_raw(raw, Fp, Fm);
        put(3, Fp, Fm);
        load_raw(1, raw);
        split_raw(raw, Fp, Fm);
        put(1, Fp, Fm);
    }
    load_raw(2, nxt);
    __syncwarp();
    float carry[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    // one chunk: faces of chunk c from chunks c-1, c, c+1; with SPLIT, chunk
    // c+2's split beside them
    auto chunk_step = [&](int c, auto split_tag) {
        constexpr bool SPLIT = decltype(split_tag)::value;
        const int sp = (c + 3) & 3, sc = c & 3, sn = c + 1 == nch ? 4 : ((c + 1) & 3);
        double cr[5];
        if constexpr (SPLIT) {
#pragma unroll
            for (int q = 0; q < 5; ++q) cr[q] = nxt[q];
            load_raw(min(c + 3, nch - 1), nxt);
        }
        int cell[S];
#pragma unroll
        for (int m = 0; m < S; ++m) {
            const int o = lane - MID + m;
            const int sl = o < 0 ? sp : (o >= 32 ? sn : sc);
            cell[m] = sl * 32 + (o & 31);
        }
        float face[5], Fp[5], Fm[5];
        if constexpr (RC == RC_WENO5) {
            float fp[S][5], fm[S][5];
#pragma unroll
            for (int m = 0; m < S; ++m) ring.get(wq, cell[m], fp[m], fm[m]);
            if constexpr (SPLIT) split_raw(cr, Fp, Fm);
            weno5_face_x2([&](int m, int q) { return fp[m][q]; },
                          [&](int m, int q) { return fm[S - 1 - m][q]; }, face);
        } else {
            if constexpr (SPLIT) split_raw(cr, Fp, Fm);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                float a[S], b[S];
#pragma unroll
                for (int m = 0; m < S; ++m) {
                    a[m] = ring.comp(wq, cell[m], q, false);
                    b[m] = ring.comp(wq, cell[S - 1 - m], q, true);
                }
                const float plus_face = reconstruct<float, RC>(a, lin, disp, diss);
                const float minus_face = reconstruct<float, RC>(b, lin, disp, diss);
                face[q] = plus_face + minus_face;
            }
        }
        if constexpr (SPLIT) {
            put((c + 2) & 3, Fp, Fm);  // the slot of chunk c-2
            __syncwarp();
        }
        const long long id = base + (c << 5) + lane;
        const bool park = c == 0 && lane == 0;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            float left = __shfl_up_sync(0xffffffffu, face[q], 1);
            const float last = __shfl_sync(0xffffffffu, face[q], 31);
            if (lane == 0) left = carry[q];
            carry[q] = last;
            tacc[q * n + id] = park ? face[q] : (face[q] - left) * inv_h;
        }
    };
    for (int c = 0; c + 2 < nch; ++c) chunk_step(c, std::true_type{});
    for (int c = nch - 2; c < nch; ++c) chunk_step(c, std::false_type{});
    if (lane == 0) {
        // cell 0: its parked face minus face nx-1 (the last chunk's lane 31)
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const float d = tacc[q * n + base] - carry[q];
            tacc[q * n + base] = d * inv_h;
        }
    }
}

// The x sweep of one periodic row by one warp (the body of k_sweep_x_warp).
template <class R, int FVS, int RC, bool CHR>
__device__ __forceinline__ void x_sweep_row(const DevParams& P, const StateView& W,
                                            R* __restrict__ tacc, SplitRing<R, XW_WARPS, 96>& ring,
                                            int wq, int lane, long long row) {
    constexpr int S = Stencil<RC>::S;
    constexpr int MID = (S - 1) / 2;
    constexpr bool kDeviation = sizeof(R) < sizeof(double);
    const int nx = P.nx;
    const long long n = P.n;
    const long long base = row * nx;
    const int nch = nx >> 5;
    const R gamma = R(P.gamma), eps = R(P.sw_eps);
    R lin[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) lin[m] = R(P.lin[m]);
    const R disp = R(P.mdcd_disp), diss = R(P.mdcd_diss);
    const R inv_h = R(P.inv_dx);
    (void)gamma;
    (void)eps;

    double refp[5], refm[5];
    const double inv_gm1 = kDeviation ? 1.0 / (P.gamma - 1.0) : 0.0;
    const double inv_2g = kDeviation ? 1.0 / (2.0 * P.gamma) : 0.0;
    auto load_raw = [&](int chunk, double* raw) {
        const long long id = base + (chunk << 5) + lane;
        raw[0] = W.rho[id];
        raw[1] = W.u[id];
        raw[2] = W.v[id];
        raw[3] = W.w[id];
        raw[4] = W.p[id];
    };
    auto split_raw = [&](const double* raw, R* Fp, R* Fm) {
        if constexpr (!kDeviation) {
            R rr = R(raw[0]);
            const R u = R(raw[1]), v = R(raw[2]), w = R(raw[3]), p = R(raw[4]);
            if (rr <= R(0)) rr = R(1e-12);
            R E, c;
            p2c_Ec(rr, u, v, w, p, gamma, E, c);
            if constexpr (FVS == FV_SW) split_sw<R, 1, 0, 0>(rr, u, v, w, E, p, c, gamma, eps, Fp, Fm);
            else split_lf<R, 1, 0, 0>(rr, u, v, w, E, p, c, Fp, Fm);
        } else {
            double Fpd[5], Fmd[5];
            split_fast<FVS, 1, 0, 0>(P, inv_gm1, inv_2g, raw, Fpd, Fmd);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                Fp[q] = R(Fpd[q] - refp[q]);
                Fm[q] = R(Fmd[q] - refm[q]);
            }
        }
    };
    // the FP32 form's offset: the split flux of the row's first cell
    if constexpr (kDeviation) {
        double raw[5];
        load_raw(0, raw);
        double Fpd[5], Fmd[5];
        split_fast<FVS, 1, 0, 0>(P, inv_gm1, inv_2g, raw, Fpd, Fmd);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            refp[q] = __shfl_sync(0xffffffffu, Fpd[q], 0);
            refm[q] = __shfl_sync(0xffffffffu, Fmd[q], 0);
        }
    }
    auto put = [&](int slot, const R* Fp, const R* Fm) { ring.put(wq, slot * 32 + lane, Fp, Fm); };
    // face at chunk-relative position `pos` (face pos sits between cells pos and
    // pos+1 of chunk `chunk`, held in slot `cs`); window cells pos-MID .. pos-MID+S-1
    auto face_at = [&](int cs, int pos, int chunk, R* face) {
        int cell[S];
#pragma unroll
        for (int m = 0; m < S; ++m) {
            const int k = cs * 32 + pos - MID + m;
            cell[m] = k < 0 ? k + 96 : (k >= 96 ? k - 96 : k);
        }
        if constexpr (CHR || (kDeviation && RC == RC_WENO5)) {
            R fp[S][5], fm[S][5];
#pragma unroll
            for (int m = 0; m < S; ++m) ring.get(wq, cell[m], fp[m], fm[m]);
            if constexpr (CHR) {
                // the face's two cells, loaded coalesced over the warp (rho as stored)
                int gl = chunk * 32 + pos;
                gl = gl < 0 ? gl + nx : gl;
                const int gr = gl + 1 == nx ? 0 : gl + 1;
                const double wl[5] = {W.rho[base + gl], W.u[base + gl], W.v[base + gl],
                                      W.w[base + gl], W.p[base + gl]};
                const double wr[5] = {W.rho[base + gr], W.u[base + gr], W.v[base + gr],
                                      W.w[base + gr], W.p[base + gr]};
                char_face<0, R, RC>(P.gamma, wl, wr, [&](int m, int r) { return fp[m][r]; },
                                    [&](int m, int r) { return fm[m][r]; }, lin, disp, diss,
                                    face);
            } else {
                weno5_face_x2([&](int m, int q) { return fp[m][q]; },
                              [&](int m, int q) { return fm[S - 1 - m][q]; }, face);
            }
        } else {
            // scalar reconstructions: one component of the window at a time
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                R a[S], b[S];
#pragma unroll
                for (int m = 0; m < S; ++m) {
                    a[m] = ring.comp(wq, cell[m], q, false);
                    b[m] = ring.comp(wq, cell[S - 1 - m], q, true);
                }
                const R plus_face = reconstruct<R, RC>(a, lin, disp, diss);
                const R minus_face = reconstruct<R, RC>(b, lin, disp, diss);
                face[q] = plus_face + minus_face;
            }
        }
    };

    // prologue: slot 0 <- last chunk, slot 1 <- chunk 0
    R lastp[5], lastm[5], firstp[5], firstm[5];
    double raw[5], nxt[5];
    load_raw(nch - 1, raw);
    split_raw(raw, lastp, lastm);
    if (nch > 1) {
        load_raw(0, raw);
        split_raw(raw, firstp, firstm);
    } else {  // one chunk per row: the first chunk is the last
#pragma unroll
        for (int q = 0; q < 5; ++q) { firstp[q] = lastp[q]; firstm[q] = lastm[q]; }
    }
    put(0, lastp, lastm);
    put(1, firstp, firstm);
    if (nch > 1) load_raw(1, nxt);
    __syncwarp();
    // the face on the -x side of cell 0 is face nx-1 (periodicity): the last
    // chunk's lane 31 computes it from the same window, so lane 0 parks its
    // chunk-0 face in T_acc and finishes that cell after the last chunk; with
    // one chunk per row it is lane 31's own face, taken by shuffle below
    R carry[5] = {R(0), R(0), R(0), R(0), R(0)};
    int cur = 1;
    for (int c = 0; c < nch; ++c) {
        const int nslot = cur == 2 ? 0 : cur + 1;
        R Fp[5], Fm[5];
        if (c + 1 == nch) {
#pragma unroll
            for (int q = 0; q < 5; ++q) { Fp[q] = firstp[q]; Fm[q] = firstm[q]; }
        } else if (c + 2 == nch) {
#pragma unroll
            for (int q = 0; q < 5; ++q) { Fp[q] = lastp[q]; Fm[q] = lastm[q]; }
        } else {
            split_raw(nxt, Fp, Fm);
        }
        __syncwarp();
        put(nslot, Fp, Fm);
        if (c + 2 < nch - 1) load_raw(c + 2, nxt);
        const long long id = base + (c << 5) + lane;
        __syncwarp();
        R face[5];
        face_at(cur, lane, c, face);
        const bool park = c == 0 && lane == 0 && nch > 1;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            R left = __shfl_up_sync(0xffffffffu, face[q], 1);
            const R last = __shfl_sync(0xffffffffu, face[q], 31);
            if (lane == 0) left = nch == 1 ? last : carry[q];
            carry[q] = last;
            const R d = face[q] - left;
            tacc[q * n + id] = park ? face[q] : d * inv_h;
        }
        cur = nslot;
    }
    if (nch > 1 && lane == 0) {
        // cell 0: its parked face minus face nx-1 (the last chunk's lane 31)
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const R d = tacc[q * n + base] - carry[q];
            tacc[q * n + base] = d * inv_h;
        }
    }
}

// ---------------------------------------------------------------------------
// Viscous flux storage (fv). FP64 form: 9 blocks of n in the order 0 xx, 1 yy,
// 2 zz, 3 xy, 4 xz, 5 yz, 6 ex, 7 ey, 8 ez. FP32 form: three float4 blocks of
// n, one per direction compute_vis_flux differentiates,
//   X = (xx, xy, xz, ex) (Fv), Y = (xy, yy, yz, ey) (Hv), Z = (xz, yz, zz, ez) (Gv),
// so the update reads the four values of one stencil offset with one 16-byte
// load (24 loads per cell instead of 96) for 12 floats stored instead of 9.
// ---------------------------------------------------------------------------
template <class R>
constexpr int fv_values_per_cell() { return sizeof(R) == 4 ? 12 : 9; }

template <class R>
__device__ __forceinline__ void store_fv(R* fv, long long n, long long id, R txx, R tyy, R tzz,
                                         R txy, R txz, R tyz, R ex, R ey, R ez) {
    if constexpr (sizeof(R) == 4) {
        float4* F = reinterpret_cast<float4*>(fv);
        F[id] = make_float4(txx, txy, txz, ex);
        F[n + id] = make_float4(txy, tyy, tyz, ey);
        F[2 * n + id] = make_float4(txz, tyz, tzz, ez);
    } else {
        fv[0 * n + id] = txx;
        fv[1 * n + id] = tyy;
        fv[2 * n + id] = tzz;
        fv[3 * n + id] = txy;
        fv[4 * n + id] = txz;
        fv[5 * n + id] = tyz;
        fv[6 * n + id] = ex;
        fv[7 * n + id] = ey;
        fv[8 * n + id] = ez;
    }
}

// ---------------------------------------------------------------------------
// Viscous flux (compute_gradients ViscousFlux.cpp:240-279 +
// compute_viscous_flux :282-339). Output fv (type R) in the layout of store_fv:
// the stresses tau_xx..tau_yz and the energy fluxes ex, ey, ez. The
// reference's 12 flux arrays map onto these (Fv = {xx, xy, xz, ex},
// Hv = {xy, yy, yz, ey}, Gv = {xz, yz, zz, ez}); the mass fluxes are zero.
// ---------------------------------------------------------------------------
template <class R, int ORD>
__global__ void __launch_bounds__(128)
k_visc_flux(DevParams P, StateView W, R* __restrict__ fv, const Ctrl* __restrict__ ctrl) {
    if (ctrl && ctrl->stop) return;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long n = P.n;
    const long long id = ((long long)k * ny + j) * nx + i;
    const long long sxy = (long long)nx * ny;
    // FP32-stencil form: differentiate deviations from the centre value, formed
    // in double (the central stencils' coefficients sum to zero, so the
    // derivative is unchanged while T ~ 1 +- small keeps its low-order digits).
    constexpr bool kDeviation = sizeof(R) < sizeof(double);
    auto gx = [&](const double* a) {
        const double c0 = kDeviation ? a[id] : 0.0;
        return [=](int o) { return R(a[id + (wrap1(i + o, nx) - i)] - c0); };
    };
    auto gy = [&](const double* a) {
        const double c0 = kDeviation ? a[id] : 0.0;
        return [=](int o) { return R(a[id + (long long)(wrap1(j + o, ny) - j) * nx] - c0); };
    };
    auto gz = [&](const double* a) {
        const double c0 = kDeviation ? a[id] : 0.0;
        return [=](int o) { return R(a[id + (long long)(wrap1(k + o, nz) - k) * sxy] - c0); };
    };
    const R dx = R(P.dx), dy = R(P.dy), dz = R(P.dz);
    const R du_dx = dcentral<R, ORD>(gx(W.u), dx);
    const R du_dy = dcentral<R, ORD>(gy(W.u), dy);
    const R du_dz = dcentral<R, ORD>(gz(W.u), dz);
    const R dv_dx = dcentral<R, ORD>(gx(W.v), dx);
    const R dv_dy = dcentral<R, ORD>(gy(W.v), dy);
    const R dv_dz = dcentral<R, ORD>(gz(W.v), dz);
    const R dw_dx = dcentral<R, ORD>(gx(W.w), dx);
    const R dw_dy = dcentral<R, ORD>(gy(W.w), dy);
    const R dw_dz = dcentral<R, ORD>(gz(W.w), dz);
    const R dT_dx = dcentral<R, ORD>(gx(W.T), dx);
    const R dT_dy = dcentral<R, ORD>(gy(W.T), dy);
    const R dT_dz = dcentral<R, ORD>(gz(W.T), dz);

    const R mu = get_mu<R>(R(W.T[id]), R(P.mu), R(P.sutherland_s));
    const R Cp = R(P.Cp), Pr = R(P.Pr);
    const R divU = du_dx + dv_dy + dw_dz;
    const R tau_xx = R(2.0) * mu * du_dx - R(2.0 / 3.0) * mu * divU;
    const R tau_yy = R(2.0) * mu * dv_dy - R(2.0 / 3.0) * mu * divU;
    const R tau_zz = R(2.0) * mu * dw_dz - R(2.0 / 3.0) * mu * divU;
    const R tau_xy = mu * (du_dy + dv_dx);
    const R tau_xz = mu * (du_dz + dw_dx);
    const R tau_yz = mu * (dv_dz + dw_dy);
    const R qx = mu * Cp / Pr * dT_dx;
    const R qy = mu * Cp / Pr * dT_dy;
    const R qz = mu * Cp / Pr * dT_dz;
    const R u = R(W.u[id]), v = R(W.v[id]), w = R(W.w[id]);
    store_fv<R>(fv, n, id, tau_xx, tau_yy, tau_zz, tau_xy, tau_xz, tau_yz,
                u * tau_xx + v * tau_xy + w * tau_xz + qx, u * tau_xy + v * tau_yy + w * tau_yz + qy,
                u * tau_xz + v * tau_yz + w * tau_zz + qz);
}

// ---------------------------------------------------------------------------
// 2.5-D forms of the viscous kernels (nx % 32 == 0, ny % 8 == 0): a 32 x 8
// thread tile marches along z. The x and y neighbours of a plane come from a
// shared tile with a 4-cell halo, the z neighbours from a 9-deep register
// queue per thread, so each input value is read from L2 about 2.5 times per
// plane instead of 12 or more. Per cell the arithmetic is the same as in
// k_visc_flux / k_update (same values, same order).
// ---------------------------------------------------------------------------
// Tile shape per compute type. FP32: 32 x 16 (halo loads 1.9x the outputs),
// at most 64 registers and 2 blocks of 512 threads per SM (68 registers and
// fewer blocks measured 14% slower). FP64: 32 x 8, 128 registers, 2 blocks of
// 256 threads (a 32 x 16 tile would leave one block per SM).
template <class R>
struct VTile {
    static constexpr int X = 32, Y = sizeof(R) == 4 ? 16 : 8, H = 4;
    static constexpr int SX = X + 2 * H, SY = Y + 2 * H;
};

template <class R, int ORD>
__global__ void __launch_bounds__(VTile<R>::X * VTile<R>::Y, 2)
k_visc_flux_25d(DevParams P, StateView W, R* __restrict__ fv, const Ctrl* __restrict__ ctrl,
                int zb) {
    constexpr int VT_X = VTile<R>::X, VT_Y = VTile<R>::Y, VT_H = VTile<R>::H;
    constexpr int VT_SX = VTile<R>::SX, VT_SY = VTile<R>::SY;
    if (ctrl && ctrl->stop) return;
    // FP32-stencil form: values enter the tile and the z queue as float
    // deviations from one reference per block and variable (formed in
    // double), so each value is converted once; central stencils' weights sum
    // to zero, so the reference drops out of every derivative. FP64 form: the
    // reference is 0 and x - 0.0 == x, the reference's arithmetic unchanged.
    constexpr bool kDeviation = sizeof(R) < sizeof(double);
    using TT = R;
    __shared__ TT tile[4][VT_SY][VT_SX];
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = P.n, sxy = (long long)nx * ny;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * VT_X + tx;
    const int i0 = blockIdx.x * VT_X, j0 = blockIdx.y * VT_Y;
    const int i = i0 + tx, j = j0 + ty;
    const int k0 = blockIdx.z * zb, k1 = min(k0 + zb, nz);
    const double* src[4] = {W.u, W.v, W.w, W.T};
    double ref[4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
        ref[v] = kDeviation ? src[v][(long long)k0 * sxy + (long long)j0 * nx + i0] : 0.0;
    TT q[4][9];  // z queue: q[v][m] = value at k - 4 + m (minus ref[v])
    const long long col = (long long)j * nx + i;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const long long off = (long long)wrap1(k0 - 4 + m, nz) * sxy + col;
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v][m] = TT(src[v][off] - ref[v]);
    }
    const R dx = R(P.dx), dy = R(P.dy), dz = R(P.dz);
    const R mu_ref = R(P.mu), Ss = R(P.sutherland_s), Cp = R(P.Cp), Pr = R(P.Pr);
    for (int k = k0; k < k1; ++k) {
        const long long plane = (long long)k * sxy;
        {
            const long long off = (long long)wrap1(k + 4, nz) * sxy + col;
#pragma unroll
            for (int v = 0; v < 4; ++v) q[v][8] = TT(src[v][off] - ref[v]);
        }
        for (int t = tid; t < VT_SX * VT_SY; t += VT_X * VT_Y) {
            const int ly = t / VT_SX, lx = t - ly * VT_SX;
            const long long off = plane + (long long)wrap1(j0 - VT_H + ly, ny) * nx + wrap1(i0 - VT_H + lx, nx);
#pragma unroll
            for (int v = 0; v < 4; ++v) tile[v][ly][lx] = TT(src[v][off] - ref[v]);
        }
        __syncthreads();
        const int cx = tx + VT_H, cy = ty + VT_H;
        R g[4][3];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            g[v][0] = dcentral<R, ORD>([&](int o) { return tile[v][cy][cx + o]; }, dx);
            g[v][1] = dcentral<R, ORD>([&](int o) { return tile[v][cy + o][cx]; }, dy);
            g[v][2] = dcentral<R, ORD>([&](int o) { return q[v][4 + o]; }, dz);
        }
        const R du_dx = g[0][0], du_dy = g[0][1], du_dz = g[0][2];
        const R dv_dx = g[1][0], dv_dy = g[1][1], dv_dz = g[1][2];
        const R dw_dx = g[2][0], dw_dy = g[2][1], dw_dz = g[2][2];
        const R dT_dx = g[3][0], dT_dy = g[3][1], dT_dz = g[3][2];
        const R mu = get_mu<R>(R(ref[3]) + q[3][4], mu_ref, Ss);
        const R divU = du_dx + dv_dy + dw_dz;
        const R tau_xx = R(2.0) * mu * du_dx - R(2.0 / 3.0) * mu * divU;
        const R tau_yy = R(2.0) * mu * dv_dy - R(2.0 / 3.0) * mu * divU;
        const R tau_zz = R(2.0) * mu * dw_dz - R(2.0 / 3.0) * mu * divU;
        const R tau_xy = mu * (du_dy + dv_dx);
        const R tau_xz = mu * (du_dz + dw_dx);
        const R tau_yz = mu * (dv_dz + dw_dy);
        const R qx = mu * Cp / Pr * dT_dx;
        const R qy = mu * Cp / Pr * dT_dy;
        const R qz = mu * Cp / Pr * dT_dz;
        const R u = R(ref[0]) + q[0][4], v = R(ref[1]) + q[1][4], w = R(ref[2]) + q[2][4];
        const long long id = plane + col;
        store_fv<R>(fv, n, id, tau_xx, tau_yy, tau_zz, tau_xy, tau_xz, tau_yz,
                    u * tau_xx + v * tau_xy + w * tau_xz + qx,
                    u * tau_xy + v * tau_yy + w * tau_yz + qy,
                    u * tau_xz + v * tau_yz + w * tau_zz + qz);
#pragma unroll
        for (int v2 = 0; v2 < 4; ++v2)
#pragma unroll
            for (int m = 0; m < 8; ++m) q[v2][m] = q[v2][m + 1];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// The 2.5-D viscous kernel with its plane loads pipelined (same arithmetic per
// cell as k_visc_flux_25d, same results). Per z step:
//   * the tile of the next plane is written into the second of two shared
//     tiles while the current one is read, so one barrier per plane suffices;
//   * its interior comes from the thread's own z queue (the value was loaded
//     four planes earlier as the queue's head), only the 4-cell halo ring is
//     loaded again (448 of 960 tile cells in the FP32 form);
//   * the halo values and the queue head of the plane after next are copied
//     asynchronously (cp.async, 8 bytes each) into per-thread staging slots in
//     shared memory, so their latency hides behind a whole plane of compute
//     and they take no registers while in flight.
// Each thread owns its staging slots (halo cells h = tid, tid + NT, ...), so
// the staged values need no barrier, only the thread's own wait.
// ---------------------------------------------------------------------------
// Two values of type R in one 8- / 16-byte word.
template <class R> struct Pair;
template <> struct Pair<float> {
    using type = float2;
    __device__ static float2 make(float a, float b) { return make_float2(a, b); }
};
template <> struct Pair<double> {
    using type = double2;
    __device__ static double2 make(double a, double b) { return make_double2(a, b); }
};

template <class R>
struct VPipe {
    using T = VTile<R>;
    static constexpr int NT = T::X * T::Y;                 // threads = interior cells
    static constexpr int NH = T::SX * T::SY - NT;          // halo cells of a tile
    static constexpr int HPT = (NH + NT - 1) / NT;         // halo cells per thread
    static constexpr size_t tile_bytes = 2 * 4 * T::SY * T::SX * sizeof(R);
    static constexpr size_t smem_bytes = tile_bytes + sizeof(double) * 4 * (NH + NT);
    // tile coordinates (ly, lx) of halo cell h: the H top rows, the H bottom
    // rows, then the H left and H right columns of the middle rows
    __device__ static void halo_cell(int h, int& ly, int& lx) {
        constexpr int H = T::H, SX = T::SX, SY = T::SY, X = T::X;
        if (h < H * SX) {
            ly = h / SX; lx = h - ly * SX;
        } else if (h < 2 * H * SX) {
            h -= H * SX; ly = SY - H + h / SX; lx = h - (h / SX) * SX;
        } else {
            h -= 2 * H * SX; ly = H + h / (2 * H);
            const int c = h - (h / (2 * H)) * (2 * H);
            lx = c < H ? c : X + c;
        }
    }
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <class R, int ORD>
__global__ void __launch_bounds__(VTile<R>::X * VTile<R>::Y, 2)
k_visc_flux_pipe(DevParams P, StateView W, R* __restrict__ fv, const Ctrl* __restrict__ ctrl,
                 int zb) {
    using VT = VTile<R>;
    using VP = VPipe<R>;
    constexpr int X = VT::X, Y = VT::Y, H = VT::H, SX = VT::SX, SY = VT::SY;
    constexpr int NT = VP::NT, NH = VP::NH, HPT = VP::HPT;
    if (ctrl && ctrl->stop) return;
    constexpr bool kDeviation = sizeof(R) < sizeof(double);
    extern __shared__ __align__(16) unsigned char vsm[];
    // FP32: the tile holds (u, v) and (w, T) as float2 pairs, so one 8-byte
    // shared load feeds two derivatives (0.400 -> 0.380 ms at 256^3); FP64
    // keeps one array per variable (16-byte pairs measured slower, 0.79 -> 0.83)
    constexpr bool kPairs = sizeof(R) == 4;
    using R2 = typename Pair<R>::type;
    R2 (*tile2)[2][SY][SX] = reinterpret_cast<R2 (*)[2][SY][SX]>(vsm);       // [2][2][SY][SX]
    R (*tile)[4][SY][SX] = reinterpret_cast<R (*)[4][SY][SX]>(vsm);          // [2][4][SY][SX]
    // tile cell (flat index t of buffer buf) <- the four values of one cell
    auto put = [&](int buf, int t, R a, R b, R c, R d) {
        if constexpr (kPairs) {
            (&tile2[buf][0][0][0])[t] = Pair<R>::make(a, b);
            (&tile2[buf][1][0][0])[t] = Pair<R>::make(c, d);
        } else {
            (&tile[buf][0][0][0])[t] = a;
            (&tile[buf][1][0][0])[t] = b;
            (&tile[buf][2][0][0])[t] = c;
            (&tile[buf][3][0][0])[t] = d;
        }
    };
    double (*sth)[NH] = reinterpret_cast<double (*)[NH]>(vsm + VP::tile_bytes);  // [4][NH]
    double (*stq)[NT] = reinterpret_cast<double (*)[NT]>(vsm + VP::tile_bytes + sizeof(double) * 4 * NH);
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = P.n, sxy = (long long)nx * ny;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * X + tx;
    const int i0 = blockIdx.x * X, j0 = blockIdx.y * Y;
    const int i = i0 + tx, j = j0 + ty;
    const int k0 = blockIdx.z * zb, k1 = min(k0 + zb, nz);
    const double* src[4] = {W.u, W.v, W.w, W.T};
    double ref[4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
        ref[v] = kDeviation ? src[v][(long long)k0 * sxy + (long long)j0 * nx + i0] : 0.0;
    auto wrapz = [&](int k) { k %= nz; return k < 0 ? k + nz : k; };
    // this thread's halo cells: in-plane offsets (a plane has < 2^31 cells)
    // and flat tile positions
    int hoff[HPT], hti[HPT];
#pragma unroll
    for (int c = 0; c < HPT; ++c) {
        const int h = tid + c * NT;
        int ly = 0, lx = 0;
        if (h < NH) VP::halo_cell(h, ly, lx);
        hti[c] = ly * SX + lx;
        hoff[c] = wrap1(j0 - H + ly, ny) * nx + wrap1(i0 - H + lx, nx);
    }
    const long long col = (long long)j * nx + i;
    auto issue = [&](int kh, int kq) {  // halo of plane kh, queue head of plane kq
#pragma unroll
        for (int c = 0; c < HPT; ++c) {
            const int h = tid + c * NT;
            if (h < NH) {
                const long long off = (long long)wrapz(kh) * sxy + hoff[c];
#pragma unroll
                for (int v = 0; v < 4; ++v) cp_async8(&sth[v][h], src[v] + off);
            }
        }
        const long long offq = (long long)wrapz(kq) * sxy + col;
#pragma unroll
        for (int v = 0; v < 4; ++v) cp_async8(&stq[v][tid], src[v] + offq);
        cp_async_commit();
    };
    // prologue: queue planes k0-4 .. k0+3, tile 0 = plane k0, staging = (halo k0+1, head k0+4)
    R q[4][9];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const long long off = (long long)wrapz(k0 - 4 + m) * sxy + col;
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v][m] = R(src[v][off] - ref[v]);
    }
#pragma unroll
    for (int c = 0; c < HPT; ++c) {
        const int h = tid + c * NT;
        if (h < NH) {
            const long long off = (long long)k0 * sxy + hoff[c];
            put(0, hti[c], R(src[0][off] - ref[0]), R(src[1][off] - ref[1]), R(src[2][off] - ref[2]),
                R(src[3][off] - ref[3]));
        }
    }
    const int tc = (ty + H) * SX + tx + H;  // this thread's cell in the tile
    put(0, tc, q[0][4], q[1][4], q[2][4], q[3][4]);
    issue(k0 + 1, k0 + 4);
    __syncthreads();
    const R dx = R(P.dx), dy = R(P.dy), dz = R(P.dz);
    const R mu_ref = R(P.mu), Ss = R(P.sutherland_s), Cp = R(P.Cp), Pr = R(P.Pr);
    int b = 0;
    for (int k = k0; k < k1; ++k) {
        // the staged halo of plane k+1 and head of plane k+4 (this thread's own copies)
        cp_async_wait_all();
#pragma unroll
        for (int v = 0; v < 4; ++v) q[v][8] = R(stq[v][tid] - ref[v]);
        if (k + 1 < k1) {
            // tile of plane k+1 into the other buffer (everyone finished reading it)
#pragma unroll
            for (int c = 0; c < HPT; ++c) {
                const int h = tid + c * NT;
                if (h < NH)
                    put(b ^ 1, hti[c], R(sth[0][h] - ref[0]), R(sth[1][h] - ref[1]),
                        R(sth[2][h] - ref[2]), R(sth[3][h] - ref[3]));
            }
            put(b ^ 1, tc, q[0][5], q[1][5], q[2][5], q[3][5]);
            issue(k + 2, k + 5);
        }
        const int cx = tx + H, cy = ty + H;
        R g[4][3];
        if constexpr (kPairs) {
#pragma unroll
            for (int pr = 0; pr < 2; ++pr) {
#pragma unroll
                for (int d = 0; d < 2; ++d) {  // x, then y taps of one pair
                    R2 t2[2 * H + 1];
#pragma unroll
                    for (int o = -H; o <= H; ++o)
                        if (o != 0) t2[o + H] = d == 0 ? tile2[b][pr][cy][cx + o] : tile2[b][pr][cy + o][cx];
                    const R h = d == 0 ? dx : dy;
                    g[2 * pr][d] = dcentral<R, ORD>([&](int o) { return t2[o + H].x; }, h);
                    g[2 * pr + 1][d] = dcentral<R, ORD>([&](int o) { return t2[o + H].y; }, h);
                }
            }
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                g[v][0] = dcentral<R, ORD>([&](int o) { return tile[b][v][cy][cx + o]; }, dx);
                g[v][1] = dcentral<R, ORD>([&](int o) { return tile[b][v][cy + o][cx]; }, dy);
            }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) g[v][2] = dcentral<R, ORD>([&](int o) { return q[v][4 + o]; }, dz);
        const R du_dx = g[0][0], du_dy = g[0][1], du_dz = g[0][2];
        const R dv_dx = g[1][0], dv_dy = g[1][1], dv_dz = g[1][2];
        const R dw_dx = g[2][0], dw_dy = g[2][1], dw_dz = g[2][2];
        const R dT_dx = g[3][0], dT_dy = g[3][1], dT_dz = g[3][2];
        const R mu = get_mu<R>(R(ref[3]) + q[3][4], mu_ref, Ss);
        const R divU = du_dx + dv_dy + dw_dz;
        const R tau_xx = R(2.0) * mu * du_dx - R(2.0 / 3.0) * mu * divU;
        const R tau_yy = R(2.0) * mu * dv_dy - R(2.0 / 3.0) * mu * divU;
        const R tau_zz = R(2.0) * mu * dw_dz - R(2.0 / 3.0) * mu * divU;
        const R tau_xy = mu * (du_dy + dv_dx);
        const R tau_xz = mu * (du_dz + dw_dx);
        const R tau_yz = mu * (dv_dz + dw_dy);
        const R qx = mu * Cp / Pr * dT_dx;
        const R qy = mu * Cp / Pr * dT_dy;
        const R qz = mu * Cp / Pr * dT_dz;
        const R u = R(ref[0]) + q[0][4], v = R(ref[1]) + q[1][4], w = R(ref[2]) + q[2][4];
        const long long id = (long long)k * sxy + col;
        store_fv<R>(fv, n, id, tau_xx, tau_yy, tau_zz, tau_xy, tau_xz, tau_yz,
                    u * tau_xx + v * tau_xy + w * tau_xz + qx,
                    u * tau_xy + v * tau_yy + w * tau_yz + qy,
                    u * tau_xz + v * tau_yz + w * tau_zz + qz);
#pragma unroll
        for (int v2 = 0; v2 < 4; ++v2)
#pragma unroll
            for (int m = 0; m < 8; ++m) q[v2][m] = q[v2][m + 1];
        b ^= 1;
        __syncthreads();
    }
    cp_async_wait_all();
}

// Viscous part of the rhs at one cell: compute_vis_flux (ViscousFlux.cpp:370-384,
// x then y then z added to 0); r[0] = 0.
template <class R, int ORD>
__device__ __forceinline__ void cell_visc(const DevParams& P, const R* __restrict__ fv, int i,
                                          int j, int k, long long id, R r[5]) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = P.n, sxy = (long long)nx * ny;
    const R dx = R(P.dx), dy = R(P.dy), dz = R(P.dz);
    r[0] = R(0.0);
    if constexpr (sizeof(R) == 4) {
        // three float4 blocks: one 16-byte load per stencil offset and direction
        constexpr int H = ORD / 2;
        const float4* X = reinterpret_cast<const float4*>(fv);
        const float4* Y = X + n;
        const float4* Z = Y + n;
        float4 vx[2 * H + 1], vy[2 * H + 1], vz[2 * H + 1];
#pragma unroll
        for (int o = -H; o <= H; ++o) {
            if (o == 0) continue;
            vx[o + H] = X[id + (wrap1(i + o, nx) - i)];
            vy[o + H] = Y[id + (long long)(wrap1(j + o, ny) - j) * nx];
            vz[o + H] = Z[id + (long long)(wrap1(k + o, nz) - k) * sxy];
        }
        auto comp = [](const float4& a, int m) { return m == 0 ? a.x : (m == 1 ? a.y : (m == 2 ? a.z : a.w)); };
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            R acc = R(0.0);
            acc += dcentral<R, ORD>([&](int o) { return comp(vx[o + H], m); }, dx);
            acc += dcentral<R, ORD>([&](int o) { return comp(vy[o + H], m); }, dy);
            acc += dcentral<R, ORD>([&](int o) { return comp(vz[o + H], m); }, dz);
            r[m + 1] = acc;
        }
    } else {
        auto gx = [&](int a) {
            return [=](int o) { return fv[a * n + id + (wrap1(i + o, nx) - i)]; };
        };
        auto gy = [&](int a) {
            return [=](int o) { return fv[a * n + id + (long long)(wrap1(j + o, ny) - j) * nx]; };
        };
        auto gz = [&](int a) {
            return [=](int o) { return fv[a * n + id + (long long)(wrap1(k + o, nz) - k) * sxy]; };
        };
        // flux blocks: 0 xx, 1 yy, 2 zz, 3 xy, 4 xz, 5 yz, 6 ex, 7 ey, 8 ez
        constexpr int FX[4] = {0, 3, 4, 6};  // Fv_momx, Fv_momy, Fv_momz, Fv_E
        constexpr int FY[4] = {3, 1, 5, 7};  // Hv_*
        constexpr int FZ[4] = {4, 5, 2, 8};  // Gv_*
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            R acc = R(0.0);
            acc += dcentral<R, ORD>(gx(FX[m]), dx);
            acc += dcentral<R, ORD>(gy(FY[m]), dy);
            acc += dcentral<R, ORD>(gz(FZ[m]), dz);
            r[m + 1] = acc;
        }
    }
}

// rhs at one cell: the viscous part followed by the inviscid divergence
// (range_kutta.cpp:61-97) accumulated in tacc.
template <class R, int ORD>
__device__ __forceinline__ void cell_rhs(const DevParams& P, const R* __restrict__ tacc,
                                         const R* __restrict__ fv, int i, int j, int k,
                                         long long id, R r[5]) {
    cell_visc<R, ORD>(P, fv, i, j, k, id, r);
    const long long n = P.n;
#pragma unroll
    for (int q = 0; q < 5; ++q) r[q] += -tacc[q * n + id];
}

// compute_rhs output (5 blocks of n, double).
template <class R, int ORD>
__global__ void __launch_bounds__(128)
k_rhs_out(DevParams P, const R* __restrict__ tacc, const R* __restrict__ fv,
          double* __restrict__ rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.nx) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long id = ((long long)k * P.ny + j) * P.nx + i;
    R r[5];
    cell_rhs<R, ORD>(P, tacc, fv, i, j, k, id, r);
#pragma unroll
    for (int q = 0; q < 5; ++q) rhs[q * P.n + id] = double(r[q]);
}

// Conserved state of primitive cell values (primitiveToConserved).
__device__ __forceinline__ void prim2cons_cell(const StateView& W, long long id, double gamma,
                                               double U[5]) {
    double rr = W.rho[id];
    if (rr <= 0.0) rr = 1e-12;
    const double u = W.u[id], v = W.v[id], w = W.w[id], p = W.p[id];
    U[0] = rr;
    U[1] = rr * u;
    U[2] = rr * v;
    U[3] = rr * w;
    const double kinetic = 0.5 * (u * u + v * v + w * w);
    const double e_internal = p / ((gamma - 1.0) * rr);
    U[4] = rr * (e_internal + kinetic);
}

// Per-cell CFL candidate of compute_timestep (timestep.cpp:18-30), std::min
// semantics (a NaN candidate never replaces the running minimum).
__device__ __forceinline__ double cfl_candidate(const DevParams& P, double rho, double u,
                                                double v, double w, double p) {
    const double a = sqrt(P.gamma * p / (rho < 1e-14 ? 1e-14 : rho));
    const double dt_x = P.dx / (fabs(u) + a);
    const double dt_y = P.dy / (fabs(v) + a);
    const double dt_z = P.dz / (fabs(w) + a);
    double m = (dt_z < dt_y) ? dt_z : dt_y;
    m = (m < dt_x) ? m : dt_x;
    return m;
}

// Block-wide min of non-negative doubles, one atomicMin per block.
__device__ __forceinline__ void block_min_to(double v, unsigned long long* dst) {
    unsigned long long b = (v == v) ? pos_double_bits(v) : ~0ull;  // NaN never wins
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
        b = x < b ? x : b;
    }
    __shared__ unsigned long long red[32];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;  // 1-D or 2-D blocks
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) red[wid] = b;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x * blockDim.y + 31) >> 5;
        b = lane < nw ? red[lane] : ~0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
            b = x < b ? x : b;
        }
        if (lane == 0 && b != ~0ull) atomicMin(dst, b);
    }
}

// ---------------------------------------------------------------------------
// Stage update (range_kutta.cpp:107-147) fused with the viscous divergence
// and, after stage 3, the positivity check (:149-162) and the next step's CFL
// candidates. Wc: current state, W0: recorded state (U0 = prim2cons(W0)),
// Wn: output. Stage 3 may write Wn == W0 in place (each thread reads its own
// cell of W0 before writing it), so no pointer here is __restrict__.
// ---------------------------------------------------------------------------
// The FP32-stencil form (R = float) keeps the state in double but takes the
// divisions by rho as multiplications by one Newton-refined reciprocal (see
// rcp_nr): its rhs already carries float rounding, so the reference's exact
// cons->prim->cons round trip is only kept in the FP64 form.
__device__ __forceinline__ void prim2cons_fast(const StateView& W, long long id, double inv_gm1,
                                               double U[5]) {
    double rr = W.rho[id];
    if (rr <= 0.0) rr = 1e-12;
    const double u = W.u[id], v = W.v[id], w = W.w[id], p = W.p[id];
    U[0] = rr;
    U[1] = rr * u;
    U[2] = rr * v;
    U[3] = rr * w;
    U[4] = p * inv_gm1 + rr * (0.5 * (u * u + v * v + w * w));
}

// Shu-Osher stage of one cell from its rhs r, conservedToPrimitive of the
// result and, after stage 3, the positivity test and the CFL candidate
// (folded into `cand` with std::min semantics: a NaN never wins).
template <class R, int STAGE>
__device__ __forceinline__ void stage_cell(const DevParams& P, const StateView& Wc,
                                           const StateView& W0, long long id, const R r[5],
                                           double dt, const StateOut& Wn, Ctrl* ctrl,
                                           double& cand) {
    constexpr bool kFast = sizeof(R) < sizeof(double);
    const double gamma = P.gamma;
    double U0[5], U[5];
    if constexpr (kFast) {
        const double inv_gm1 = 1.0 / (gamma - 1.0);
        prim2cons_fast(W0, id, inv_gm1, U0);
        if (STAGE != 1) prim2cons_fast(Wc, id, inv_gm1, U);
    } else {
        prim2cons_cell(W0, id, gamma, U0);
        if (STAGE != 1) prim2cons_cell(Wc, id, gamma, U);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const double rq = double(r[q]);
        if (STAGE == 1)
            U[q] = U0[q] + dt * rq;
        else if (STAGE == 2)
            U[q] = 0.75 * U0[q] + 0.25 * (U[q] + dt * rq);
        else
            U[q] = (1.0 / 3.0) * U0[q] + (2.0 / 3.0) * (U[q] + dt * rq);
    }
    // conservedToPrimitive (field_structures.h:405-427)
    double rr = U[0];
    if (rr <= 0.0) rr = 1e-12;
    double u, v, w, p, T;
    if constexpr (kFast) {
        const double ir = rcp_nr(rr);
        u = U[1] * ir;
        v = U[2] * ir;
        w = U[3] * ir;
        p = (gamma - 1.0) * (U[4] - rr * (0.5 * (u * u + v * v + w * w)));
        T = p * ir * (1.0 / P.Rgas);
    } else {
        u = U[1] / rr;
        v = U[2] / rr;
        w = U[3] / rr;
        const double kinetic = 0.5 * (u * u + v * v + w * w);
        const double e_internal = U[4] / rr - kinetic;
        p = (gamma - 1.0) * rr * e_internal;
        T = p / (rr * P.Rgas);  // primitiveToConserved's T
    }
    Wn.rho[id] = rr;
    Wn.u[id] = u;
    Wn.v[id] = v;
    Wn.w[id] = w;
    Wn.p[id] = p;
    Wn.T[id] = T;
    if (STAGE == 3) {
        // range_kutta.cpp:154 tests rho <= 0 || p <= 0 || T <= 0, which a
        // NaN passes; the negated form below also reports NaN.
        if (!(rr > 0.0) || !(p > 0.0) || !(T > 0.0)) atomicMin(&ctrl->bad_cell, id);
        double c;
        if constexpr (kFast) {
            const double a = sqrt_nr(gamma * p * rcp_nr(rr));
            const double cx = P.dx * rcp_nr(fabs(u) + a);
            const double cy = P.dy * rcp_nr(fabs(v) + a);
            const double cz = P.dz * rcp_nr(fabs(w) + a);
            c = (cz < cy) ? cz : cy;
            c = (c < cx) ? c : cx;
        } else {
            c = cfl_candidate(P, rr, u, v, w, p);
        }
        cand = (c < cand) ? c : cand;
    }
}

// 8 blocks of 128 threads per SM (at most 64 registers): the neighbour loads
// are latency-bound, and more resident warps beat more loads in flight per
// thread. Measured at 256^3: FP32 0.713 -> 0.578 ms (5 blocks 0.630, 7 blocks
// 0.609, 10 blocks 0.680); FP64 1.80 -> 1.39 ms (6 blocks 1.52, 10 blocks 1.55).
template <class R, int ORD, int STAGE>
__global__ void __launch_bounds__(128, 8)
k_update(DevParams P, StateView Wc, StateView W0, const R* __restrict__ tacc,
         const R* __restrict__ fv, StateOut Wn, Ctrl* ctrl) {
    if (ctrl->stop) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < P.nx;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long id = ((long long)k * P.ny + j) * P.nx + (live ? i : 0);
    double cand = CFL_INIT;
    if (live) {
        R r[5];
        cell_rhs<R, ORD>(P, tacc, fv, i, j, k, id, r);
        stage_cell<R, STAGE>(P, Wc, W0, id, r, ctrl->dt, Wn, ctrl, cand);
    }
    if (STAGE == 3) block_min_to(cand, &ctrl->dtmin_bits);
}

// ---------------------------------------------------------------------------
// y and z sweeps with the face window in shared memory (component-wise
// reconstruction; du_inviscous, InviscousFlux_new.cpp:4-163, and the
// divergence of range_kutta.cpp:51-98).
//
// Same march as k_sweep (one thread per line segment, threads over x, every
// cell split once, one reconstruction per face), but the split fluxes of the
// S window cells sit in a per-thread ring of S shared-memory slots instead of
// registers: the new cell's split overwrites the slot of the cell that left
// the window, so nothing is shifted per step (the register window cost 10(S-1)
// moves per cell) and the ~10 S registers of the window are freed for more
// resident warps. Each thread touches only its own column of the ring, so no
// barrier is needed.
//
// FUSE (z sweep only): after the z difference of a cell, the rest of the
// stage runs on it in the same thread -- the viscous divergence of the fluxes
// fv, rhs = visc + (-(T_acc + az idz)) in the reference's order, the
// Shu-Osher stage, conservedToPrimitive and (stage 3) positivity and the next
// step's CFL candidates -- so T_acc's z term is never stored and the
// memory-bound update runs under the compute-bound sweep. Results equal
// k_sweep<2> followed by k_update bit for bit.
// ---------------------------------------------------------------------------

// Stage-update operands of the fused z sweep.
template <class R>
struct FuseArgs {
    int stage;            // 1, 2, 3
    StateView W0;         // recorded state (U0 = prim2cons(W0))
    const R* fv;          // viscous fluxes (store_fv layout)
    StateOut Wn;          // output state
    Ctrl* ctrl;           // dt, bad_cell, dtmin_bits
};

template <class R, int STAGE>
__device__ __forceinline__ void fused_cell(const DevParams& P, const StateView& Wc,
                                           const FuseArgs<R>& F, int i, int j, int k,
                                           long long id, const R tz[5], double dt, double& cand) {
    R r[5];
    if (P.vis_order == 4) cell_visc<R, 4>(P, F.fv, i, j, k, id, r);
    else if (P.vis_order == 6) cell_visc<R, 6>(P, F.fv, i, j, k, id, r);
    else cell_visc<R, 8>(P, F.fv, i, j, k, id, r);
#pragma unroll
    for (int q = 0; q < 5; ++q) r[q] += -tz[q];
    stage_cell<R, STAGE>(P, Wc, F.W0, id, r, dt, F.Wn, F.ctrl, cand);
}

template <int DIR, class R, int FVS, int RC, bool FUSE>
#ifdef NS3D_RING_MAXREG
__global__ void __launch_bounds__(RingCfg<R>::T) __maxnreg__(sizeof(R) == 4 ? NS3D_RING_MAXREG : 255)
#else
__global__ void __launch_bounds__(RingCfg<R>::T, RingCfg<R>::MINB)
#endif
k_sweep_ring(DevParams P, StateView W, R* __restrict__ tacc, int seg, const Ctrl* __restrict__ ctrl,
             FuseArgs<R> F) {
    static_assert(DIR == 1 || DIR == 2, "y and z sweeps");
    static_assert(!FUSE || DIR == 2, "the stage update follows the last (z) sweep");
    constexpr int S = Stencil<RC>::S;
    constexpr int MID = (S - 1) / 2;
    constexpr int T = RingCfg<R>::T;
    constexpr bool kDeviation = sizeof(R) < sizeof(double);
    __shared__ SplitRing<R, S, T> ring;
    if (ctrl && ctrl->stop) return;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = P.n;
    const int tid = threadIdx.x;
    const int t0 = blockIdx.x * blockDim.x + tid;
    const bool live = t0 < nx;
    const int len = DIR == 1 ? ny : nz;
    const long long stride = DIR == 1 ? (long long)nx : (long long)nx * ny;
    const long long base = DIR == 1 ? (long long)blockIdx.y * ny * nx + (live ? t0 : 0)
                                    : (long long)blockIdx.y * nx + (live ? t0 : 0);
    const int c0 = blockIdx.z * seg;
    if (c0 >= len) return;  // block-uniform
    const int c1 = min(c0 + seg, len);

    R lin[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) lin[m] = R(P.lin[m]);
    const R disp = R(P.mdcd_disp), diss = R(P.mdcd_diss);
    const R inv_h = R(DIR == 1 ? P.inv_dy : P.inv_dz);
    const R gamma = R(P.gamma), eps = R(P.sw_eps);
    (void)gamma;
    (void)eps;
    double refp[5], refm[5];
    const double inv_gm1 = kDeviation ? 1.0 / (P.gamma - 1.0) : 0.0;
    const double inv_2g = kDeviation ? 1.0 / (2.0 * P.gamma) : 0.0;
    auto load_raw = [&](int s, double* raw) {
        const long long id = base + (long long)wrap1(s, len) * stride;
        raw[0] = W.rho[id];
        raw[1] = W.u[id];
        raw[2] = W.v[id];
        raw[3] = W.w[id];
        raw[4] = W.p[id];
    };
    // the split of k_sweep (FP32 form: double split, minus the segment's first
    // cell's split flux, rounded to float)
    auto split_raw = [&](const double* raw, R* Fp, R* Fm, bool set_ref) {
        if constexpr (!kDeviation) {
            R rr = R(raw[0]);
            const R u = R(raw[1]), v = R(raw[2]), w = R(raw[3]), p = R(raw[4]);
            if (rr <= R(0)) rr = R(1e-12);
            R E, c;
            p2c_Ec(rr, u, v, w, p, gamma, E, c);
            if constexpr (FVS == FV_SW)
                split_sw<R, 0, DIR == 1, DIR == 2>(rr, u, v, w, E, p, c, gamma, eps, Fp, Fm);
            else
                split_lf<R, 0, DIR == 1, DIR == 2>(rr, u, v, w, E, p, c, Fp, Fm);
        } else {
            double Fpd[5], Fmd[5];
            split_fast<FVS, 0, DIR == 1, DIR == 2>(P, inv_gm1, inv_2g, raw, Fpd, Fmd);
            if (set_ref) {
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    refp[q] = Fpd[q];
                    refm[q] = Fmd[q];
                }
            }
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                Fp[q] = R(Fpd[q] - refp[q]);
                Fm[q] = R(Fmd[q] - refm[q]);
            }
        }
    };

    double cand = CFL_INIT;
    double dt = 0.0;
    if constexpr (FUSE) dt = F.ctrl->dt;
    if (live) {
        int f = c0 - 1;  // face f sits between cells f and f+1
        double nxt[5];
#pragma unroll
        for (int m = 0; m < S - 1; ++m) {
            load_raw(f - MID + m, nxt);
            R Fp[5], Fm[5];
            split_raw(nxt, Fp, Fm, m == 0);
            ring.put(m, tid, Fp, Fm);
        }
        load_raw(f - MID + S - 1, nxt);
        R prev[5];
        int ph = 0;  // window position m of this face sits in slot (ph + m) mod S
        for (int t = 0; f < c1; ++t, ++f) {
            double cur[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) cur[q] = nxt[q];
            load_raw(f - MID + S, nxt);  // the following cell, one step ahead
            const long long oid = base + (long long)f * stride;
            R old[5];
            if (t > 0) {
#pragma unroll
                for (int q = 0; q < 5; ++q) old[q] = tacc[q * n + oid];
            }
            {
                R Fp[5], Fm[5];
                split_raw(cur, Fp, Fm, false);
                ring.put(ph == 0 ? S - 1 : ph - 1, tid, Fp, Fm);
            }
            R face[5];
            if constexpr (kDeviation && RC == RC_WENO5) {
                R fp[S][5], fm[S][5];
                ring_window_at(ph, ring, tid, fp, fm);
                // reconstruct_select reverses the minus window (flag < 0)
                weno5_face_x2([&](int m, int q) { return fp[m][q]; },
                              [&](int m, int q) { return fm[S - 1 - m][q]; }, face);
            } else {
                // scalar reconstructions: one component of the window at a time
                int sl[S];
#pragma unroll
                for (int m = 0; m < S; ++m) sl[m] = ph + m < S ? ph + m : ph + m - S;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    R a[S], b[S];
#pragma unroll
                    for (int m = 0; m < S; ++m) {
                        a[m] = ring.comp(sl[m], tid, q, false);
                        b[m] = ring.comp(sl[S - 1 - m], tid, q, true);
                    }
                    const R plus_face = reconstruct<R, RC>(a, lin, disp, diss);
                    const R minus_face = reconstruct<R, RC>(b, lin, disp, diss);
                    face[q] = plus_face + minus_face;
                }
            }
            if (t > 0) {
                R tz[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) tz[q] = old[q] + (face[q] - prev[q]) * inv_h;
                if constexpr (FUSE) {
                    const int i = t0, j = blockIdx.y;
                    if (F.stage == 1) fused_cell<R, 1>(P, W, F, i, j, f, oid, tz, dt, cand);
                    else if (F.stage == 2) fused_cell<R, 2>(P, W, F, i, j, f, oid, tz, dt, cand);
                    else fused_cell<R, 3>(P, W, F, i, j, f, oid, tz, dt, cand);
                } else {
#pragma unroll
                    for (int q = 0; q < 5; ++q) tacc[q * n + oid] = tz[q];
                }
            }
#pragma unroll
            for (int q = 0; q < 5; ++q) prev[q] = face[q];
            ph = ph + 1 == S ? 0 : ph + 1;
        }
    }
    if constexpr (FUSE) {
        if (F.stage == 3) block_min_to(cand, &F.ctrl->dtmin_bits);
    }
}

// FP32-form y / z sweep with the split software-pipelined (k_sweep_ring's
// march and arithmetic, reordered): when face f is reconstructed its whole
// window (cells f-MID .. f-MID+S-1) is already in the ring, and the split of
// cell f-MID+S, which enters the window of face f+1, runs in the same
// iteration, beside the reconstruction and with no branch between the two
// chains (ENT fixes the entropy-fix choice, square roots from sqrt_nr_nb); its
// split flux goes into the slot of cell f-MID once the window has been read.
// The interleaved chains need more registers than the 126 of the plain ring
// at 4 blocks per SM, so this kernel is compiled for NS3D_PIPE_MINB blocks.
#ifndef NS3D_PIPE_MINB
#define NS3D_PIPE_MINB 3
#endif
template <int DIR, int FVS, int RC, int ENT>
__global__ void __launch_bounds__(RingCfg<float>::T, NS3D_PIPE_MINB)
k_sweep_pipe(DevParams P, StateView W, float* __restrict__ tacc, int seg,
             const Ctrl* __restrict__ ctrl) {
    static_assert(DIR == 1 || DIR == 2, "y and z sweeps");
    constexpr int S = Stencil<RC>::S;
    constexpr int MID = (S - 1) / 2;
    constexpr int T = RingCfg<float>::T;
    __shared__ SplitRing<float, S, T> ring;
    if (ctrl && ctrl->stop) return;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const long long n = P.n;
    const int tid = threadIdx.x;
    const int t0 = blockIdx.x * blockDim.x + tid;
    if (t0 >= nx) return;  // each thread owns its ring column: no barrier follows
    const int len = DIR == 1 ? ny : nz;
    const long long stride = DIR == 1 ? (long long)nx : (long long)nx * ny;
    const long long base = DIR == 1 ? (long long)blockIdx.y * ny * nx + t0
                                    : (long long)blockIdx.y * nx + t0;
    const int c0 = blockIdx.z * seg;
    if (c0 >= len) return;
    const int c1 = min(c0 + seg, len);

    float lin[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) lin[m] = float(P.lin[m]);
    const float disp = float(P.mdcd_disp), diss = float(P.mdcd_diss);
    const float inv_h = float(DIR == 1 ? P.inv_dy : P.inv_dz);
    const double inv_gm1 = 1.0 / (P.gamma - 1.0);
    const double inv_2g = 1.0 / (2.0 * P.gamma);
    double refp[5], refm[5];
    // cells f-MID .. f-MID+S+1 of every face: within (-len, 2 len) for
    // extents >= 8, so one wrap suffices
    auto load_raw = [&](int s, double* raw) {
        const long long id = base + (long long)wrap1(s, len) * stride;
        raw[0] = W.rho[id];
        raw[1] = W.u[id];
        raw[2] = W.v[id];
        raw[3] = W.w[id];
        raw[4] = W.p[id];
    };
    auto split_d = [&](const double* raw, double* Fpd, double* Fmd) {
        split_fast<FVS, 0, DIR == 1, DIR == 2, 1, ENT, true>(P, inv_gm1, inv_2g, raw, Fpd, Fmd);
    };
    auto split_raw = [&](const double* raw, float* Fp, float* Fm) {
        double Fpd[5], Fmd[5];
        split_d(raw, Fpd, Fmd);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            Fp[q] = float(Fpd[q] - refp[q]);
            Fm[q] = float(Fmd[q] - refm[q]);
        }
    };

    int f = c0 - 1;  // face f sits between cells f and f+1
    double nxt[5];
    {
        // the window of face c0-1 into slots 0..S-1; its first cell's split
        // flux is the segment's offset
        float Fp[5], Fm[5];
        load_raw(f - MID, nxt);
        split_d(nxt, refp, refm);
#pragma unroll
        for (int q = 0; q < 5; ++q) Fp[q] = Fm[q] = 0.f;
        ring.put(0, tid, Fp, Fm);
#pragma unroll
        for (int m = 1; m < S; ++m) {
            load_raw(f - MID + m, nxt);
            split_raw(nxt, Fp, Fm);
            ring.put(m, tid, Fp, Fm);
        }
    }
    load_raw(f - MID + S, nxt);
    float prev[5];
    int ph = 0;  // window position m of the current face sits in slot (ph + m) mod S
    for (int t = 0; f < c1; ++t, ++f) {
        double cur[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) cur[q] = nxt[q];
        load_raw(f - MID + S + 1, nxt);  // split in the next iteration
        const long long oid = base + (long long)f * stride;
        float old[5];
        if (t > 0) {
#pragma unroll
            for (int q = 0; q < 5; ++q) old[q] = tacc[q * n + oid];
        }
        float face[5], Fp[5], Fm[5];
        if constexpr (RC == RC_WENO5) {
            float fp[S][5], fm[S][5];
            ring_window_at(ph, ring, tid, fp, fm);
            split_raw(cur, Fp, Fm);
            weno5_face_x2([&](int m, int q) { return fp[m][q]; },
                          [&](int m, int q) { return fm[S - 1 - m][q]; }, face);
        } else {
            int sl[S];
#pragma unroll
            for (int m = 0; m < S; ++m) sl[m] = ph + m < S ? ph + m : ph + m - S;
            split_raw(cur, Fp, Fm);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                float a[S], b[S];
#pragma unroll
                for (int m = 0; m < S; ++m) {
                    a[m] = ring.comp(sl[m], tid, q, false);
                    b[m] = ring.comp(sl[S - 1 - m], tid, q, true);
                }
                const float plus_face = reconstruct<float, RC>(a, lin, disp, diss);
                const float minus_face = reconstruct<float, RC>(b, lin, disp, diss);
                face[q] = plus_face + minus_face;
            }
        }
        // cell f-MID leaves the window: its slot takes cell f-MID+S
        ring.put(ph, tid, Fp, Fm);
        if (t > 0) {
#pragma unroll
            for (int q = 0; q < 5; ++q) tacc[q * n + oid] = old[q] + (face[q] - prev[q]) * inv_h;
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) prev[q] = face[q];
        ph = ph + 1 == S ? 0 : ph + 1;
    }
}

// Sums of the reductions below (see k_sums_partial).
constexpr int NSUMS = 13;

// The kernels from here on are not templates; only the API translation unit
// (which defines NS3D_API_KERNELS) instantiates them.
#ifdef NS3D_API_KERNELS

// compute_timestep candidates of the current state (standalone).
__global__ void __launch_bounds__(256)
k_cfl(DevParams P, StateView W, Ctrl* ctrl) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double cand = CFL_INIT;
    if (id < P.n) cand = cfl_candidate(P, W.rho[id], W.u[id], W.v[id], W.w[id], W.p[id]);
    block_min_to(cand, &ctrl->dtmin_bits);
}

// Start of one time_advance iteration (maincycle.cpp:14-47). mode 0: plain
// step (dt from CFL or dt_fixed); mode 1: with the TotalTime / output-time
// clipping and stop conditions of time_advance; mode 2: as mode 1, and the
// loop also ends after a step whose if_output is set, so that the host can
// write that step's output.
__global__ void k_control_pre(Ctrl* c, int mode, double cfl, double dt_fixed, double total_time,
                              double out_freq) {
    if (c->stop) return;
    const double eps = 1e-12;
    c->output = 0;
    if (mode >= 1 && fabs(total_time - c->time) <= eps) {
        c->stop = 1;
        c->stop_reason = STOP_TOTAL_TIME;
        c->stop_in_pre = 1;
        c->active = 0;
        return;
    }
    double dt = dt_fixed;
    if (dt_fixed < 0.0) dt = cfl * __longlong_as_double((long long)c->dtmin_bits);
    if (mode >= 1) {
        double t = c->time;
        if (t >= c->out_next - eps) {
            c->out_next += out_freq;
            c->output = 1;
        }
        if (t + dt > total_time) dt = total_time - t;
        if (t + dt > c->out_next) {
            dt = c->out_next - t;
            c->out_next += out_freq;
            c->output = 1;
        }
        if (dt <= eps) {
            // the state is unchanged: its CFL minimum stays valid
            c->stop = 1;
            c->stop_reason = STOP_DT_SMALL;
            c->stop_in_pre = 1;
            c->active = 0;
            return;
        }
    }
    // the step runs: its stage 3 collects the next state's CFL minimum
    c->dtmin_bits = pos_double_bits(CFL_INIT);
    c->time += dt;
    c->dt = dt;
    c->active = 1;
}

// End of one iteration (maincycle.cpp:250 + 298-300, range_kutta.cpp:149-162).
__global__ void k_control_post(Ctrl* c, int mode, double total_time, long long n,
                               double* times) {
    if (c->stop || !c->active) return;
    c->active = 0;
    c->steps_done += 1;
    if (c->bad_cell < n) {
        c->stop = 1;
        c->stop_reason = STOP_NONPHYSICAL;
        return;
    }
    times[c->steps_done - 1] = c->time;  // current_time after the step
    if (mode >= 1 && c->time >= total_time) {
        c->stop = 1;
        c->stop_reason = STOP_TOTAL_TIME;
    } else if (mode == 2 && c->output) {
        c->stop = 1;
        c->stop_reason = STOP_OUTPUT;
    }
}

// ---------------------------------------------------------------------------
// Reductions (FP64)
// ---------------------------------------------------------------------------

// compute_total_energy (postprocess.cpp:103-128) and the sums of
// compute_turbulence_statistics (ana_isotropic.cpp:241-255), per block, then
// a second pass sums the block partials in double. Outputs 12 sums:
// [0] sum 0.5 rho |u|^2, [1] sum 0.5|u|^2, [2] sum mu(T), [3] sum rho,
// [4] sum |u|^2, [5..7] sum u,v,w, [8..10] sum u^2,v^2,w^2, [11] sum sqrt(g R T),
// [12] sum (du/dx)^2 with du/dx of compute_gradients_dudx (ViscousFlux.cpp:389-410):
// the viscous scheme's central derivative.
template <int ORD>
__device__ __forceinline__ double dudx_at(const DevParams& P, const double* __restrict__ u,
                                          long long id) {
    const int nx = P.nx;
    const int i = (int)(id % nx);
    return dcentral<double, ORD>([&](int o) { return u[id + (wrap1(i + o, nx) - i)]; }, P.dx);
}

__global__ void __launch_bounds__(256)
k_sums_partial(DevParams P, StateView W, double* __restrict__ part) {
    double s[NSUMS];
#pragma unroll
    for (int q = 0; q < NSUMS; ++q) s[q] = 0.0;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < P.n;
         id += (long long)gridDim.x * blockDim.x) {
        const double rho = W.rho[id], u = W.u[id], v = W.v[id], w = W.w[id], T = W.T[id];
        const double q2 = u * u + v * v + w * w;
        s[0] += 0.5 * rho * q2;
        s[1] += 0.5 * q2;
        s[2] += get_mu<double>(T, P.mu, P.sutherland_s);
        s[3] += rho;
        s[4] += q2;
        s[5] += u;
        s[6] += v;
        s[7] += w;
        s[8] += u * u;
        s[9] += v * v;
        s[10] += w * w;
        s[11] += sqrt(P.gamma * P.Rgas * T);
        const double dudx = P.vis_order == 4 ? dudx_at<4>(P, W.u, id)
                          : (P.vis_order == 6 ? dudx_at<6>(P, W.u, id) : dudx_at<8>(P, W.u, id));
        s[12] += dudx * dudx;
    }
    __shared__ double red[NSUMS][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NSUMS; ++q) {
        double x = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < NSUMS) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[threadIdx.x][w];
        part[(long long)blockIdx.x * NSUMS + threadIdx.x] = x;
    }
}

__global__ void k_sums_final(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= NSUMS) return;
    double x = 0.0;
    for (int b = 0; b < nblocks; ++b) x += part[(long long)b * NSUMS + q];
    out[q] = x;
}

#endif  // NS3D_API_KERNELS

}  // namespace ns3d
