// Discrete adjoint kernels (FP64): the vector-Jacobian product of the RHS and
// of one Shu-Osher stage with its cons<->prim conversions. No counterpart in
// the reference (it has no derivative code).
//
// RHS VJP, per direction d (R = V - sum_d inv_h_d (F_d(f) - F_d(f-1))):
//   lamF(f) = inv_h (lamR(f+1) - lamR(f))                     (face f = f+1/2)
//   k_adj_face: reconstruction VJP of every face into G (2 x S x 5 arrays)
//   k_adj_cell: lamF+-(c) = sum over the faces whose windows hold c, then the
//               transposed split Jacobian -> lamW(c) +=
// Viscous part: lam of the fluxes = D^T lamR = -D lamR (antisymmetric central
// stencils on a periodic line), pointwise flux VJP (tau, q, mu(T)), then the
// gradient transpose -D again.
#include <cuda_runtime.h>

#include "ns3d_adjoint.cuh"
#include "ns3d_internal.h"
#include "ns3d_kernels.cuh"

namespace ns3d {

namespace {

// index of the cell at line position s (wrapped) given the cell id at position p
struct Line {
    long long id;
    long long stride;
    int pos, len;
    __device__ long long at(int s) const { return id + (long long)(wrap1(s, len) - pos) * stride; }
};

template <int DIR>
__device__ __forceinline__ Line line_of(const DevParams& P, int i, int j, int k, long long id) {
    if constexpr (DIR == 0) return Line{id, 1, i, P.nx};
    else if constexpr (DIR == 1) return Line{id, (long long)P.nx, j, P.ny};
    else return Line{id, (long long)P.nx * P.ny, k, P.nz};
}

__device__ __forceinline__ void load_w5(const StateView& W, long long id, double* w) {
    double rr = W.rho[id];
    if (rr <= 0.0) rr = 1e-12;
    w[0] = rr;
    w[1] = W.u[id];
    w[2] = W.v[id];
    w[3] = W.w[id];
    w[4] = W.p[id];
}

// Forward split at the windows' cells, with Newton-refined reciprocal and
// square roots (split_fast, two steps: about an ulp).
template <int FVS, int DIR>
__device__ __forceinline__ void split_fwd(const double* w5, const DevParams& P, double* Fp,
                                          double* Fm) {
    split_fast<FVS, DIR == 0, DIR == 1, DIR == 2, 2>(P, 1.0 / (P.gamma - 1.0), 0.5 / P.gamma,
                                                     w5, Fp, Fm);
}

// Index of face/cell position f of a line in the split-flux cotangent array G.
// x lines (threads over j) use a j-fastest layout so that a warp's stores are
// contiguous; y and z lines (threads over i) use the cell index itself.
template <int DIR>
__device__ __forceinline__ long long g_index(const DevParams& P, int i, int j, int k) {
    if constexpr (DIR == 0) return ((long long)k * P.nx + i) * P.ny + j;
    else return ((long long)k * P.ny + j) * P.nx + i;
}

// Reconstruction VJP of every face: marches a line segment like k_sweep,
// holding the split fluxes of the face window in registers.
template <int DIR, int FVS, int RC>
__global__ void __launch_bounds__(128)
k_adj_face(DevParams P, StateView W, const double* __restrict__ lamR, double* __restrict__ G,
           int seg) {
    constexpr int S = Stencil<RC>::S;
    constexpr int MID = (S - 1) / 2;
    const int nx = P.nx, ny = P.ny;
    const long long n = P.n;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    long long base, stride;
    int len;
    if constexpr (DIR == 0) {
        if (t0 >= ny) return;
        base = ((long long)blockIdx.y * ny + t0) * nx; stride = 1; len = nx;
    } else if constexpr (DIR == 1) {
        if (t0 >= nx) return;
        base = (long long)blockIdx.y * ny * nx + t0; stride = nx; len = ny;
    } else {
        if (t0 >= nx) return;
        base = (long long)blockIdx.y * nx + t0; stride = (long long)nx * ny; len = P.nz;
    }
    const int c0 = blockIdx.z * seg;
    if (c0 >= len) return;
    const int c1 = min(c0 + seg, len);
    double lin[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) lin[m] = P.lin[m];
    const double inv_h = DIR == 0 ? P.inv_dx : (DIR == 1 ? P.inv_dy : P.inv_dz);
    auto idx = [&](int s) { return base + (long long)wrap1(s, len) * stride; };
    double fp[S][5], fm[S][5];
#pragma unroll
    for (int m = 0; m < S - 1; ++m) {
        double w5[5];
        load_w5(W, idx(c0 - MID + m), w5);
        split_fwd<FVS, DIR>(w5, P, fp[m], fm[m]);
    }
    double lr_here[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) lr_here[q] = lamR[q * n + idx(c0)];
    for (int f = c0; f < c1; ++f) {
        double w5[5];
        load_w5(W, idx(f - MID + S - 1), w5);
        split_fwd<FVS, DIR>(w5, P, fp[S - 1], fm[S - 1]);
        const long long nid = idx(f + 1);
        const long long fid = DIR == 0 ? g_index<0>(P, f, t0, blockIdx.y) : idx(f);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double lr_next = lamR[q * n + nid];
            const double lamF = inv_h * (lr_next - lr_here[q]);
            lr_here[q] = lr_next;
            double a[S], b[S], ga[S], gb[S];
#pragma unroll
            for (int m = 0; m < S; ++m) {
                a[m] = fp[m][q];
                b[m] = fm[S - 1 - m][q];
                ga[m] = 0.0;
                gb[m] = 0.0;
            }
            reconstruct_vjp<RC>(a, lin, lamF, ga);
            reconstruct_vjp<RC>(b, lin, lamF, gb);
#pragma unroll
            for (int m = 0; m < S; ++m) {
                G[((long long)(0 * S + m) * 5 + q) * n + fid] = ga[m];
                G[((long long)(1 * S + m) * 5 + q) * n + fid] = gb[m];
            }
        }
#pragma unroll
        for (int m = 0; m < S - 1; ++m)
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                fp[m][q] = fp[m + 1][q];
                fm[m][q] = fm[m + 1][q];
            }
    }
}

// Gather of the split-flux cotangents of each cell and the transposed split
// Jacobian: lamW(c) += (dF+/dw)^T lamF+(c) + (dF-/dw)^T lamF-(c).
template <int DIR, int FVS, int RC>
__global__ void __launch_bounds__(128)
k_adj_cell(DevParams P, StateView W, const double* __restrict__ G, double* __restrict__ lamW) {
    constexpr int S = Stencil<RC>::S;
    constexpr int MID = (S - 1) / 2;
    // x: threads over j (G's x layout is j-fastest); y, z: threads over i
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (DIR == 0 ? P.ny : P.nx)) return;
    const int i = DIR == 0 ? (int)blockIdx.y : t, j = DIR == 0 ? t : (int)blockIdx.y;
    const int k = blockIdx.z;
    const long long n = P.n;
    const long long id = ((long long)k * P.ny + j) * P.nx + i;
    const int pos = DIR == 0 ? i : (DIR == 1 ? j : k);
    const int len = DIR == 0 ? P.nx : (DIR == 1 ? P.ny : P.nz);
    auto gat = [&](int s) {
        const int w = wrap1(s, len);
        return DIR == 0 ? g_index<0>(P, w, j, k) : (DIR == 1 ? g_index<1>(P, i, w, k)
                                                             : g_index<2>(P, i, j, w));
    };
    double gp[5], gm[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        double sp = 0.0, sm = 0.0;
#pragma unroll
        for (int m = 0; m < S; ++m) {
            // cell c = f - MID + m in the plus window of face f = c + MID - m
            sp += G[((long long)(0 * S + m) * 5 + q) * n + gat(pos + MID - m)];
            // cell c = f - MID + (S-1-m) in the minus window of face f = c + MID - S + 1 + m
            sm += G[((long long)(1 * S + m) * 5 + q) * n + gat(pos + MID - S + 1 + m)];
        }
        gp[q] = sp;
        gm[q] = sm;
    }
    double w5[5], gw[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    load_w5(W, id, w5);
    split_vjp<FVS, DIR>(w5, P.gamma, P.sw_eps, gp, gm, gw);
#pragma unroll
    for (int q = 0; q < 5; ++q) lamW[q * n + id] += gw[q];
}

// Viscous VJP, part 1: lam of the 12 gradients and the direct lam of u,v,w,T.
// lg blocks: 0..11 gradients (du/dx du/dy du/dz dv/.. dw/.. dT/..), 12..15 u,v,w,T.
template <int ORD>
__global__ void __launch_bounds__(128)
k_adj_visc1(DevParams P, StateView W, const double* __restrict__ lamR, double* __restrict__ lg) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long n = P.n;
    const long long id = ((long long)k * ny + j) * nx + i;
    const Line Lx = line_of<0>(P, i, j, k, id), Ly = line_of<1>(P, i, j, k, id),
               Lz = line_of<2>(P, i, j, k, id);
    auto d = [&](const double* a, const Line& L, double h) {
        return dcentral<double, ORD>([&](int o) { return a[L.at(L.pos + o)]; }, h);
    };
    const double dx = P.dx, dy = P.dy, dz = P.dz;
    // lam of the fluxes (D^T = -D)
    double lF[4], lH[4], lGz[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const double* lr = lamR + (long long)(m + 1) * n;
        lF[m] = -d(lr, Lx, dx);
        lH[m] = -d(lr, Ly, dy);
        lGz[m] = -d(lr, Lz, dz);
    }
    // forward gradients and stresses at the cell
    const double ux = d(W.u, Lx, dx), uy = d(W.u, Ly, dy), uz = d(W.u, Lz, dz);
    const double vx = d(W.v, Lx, dx), vy = d(W.v, Ly, dy), vz = d(W.v, Lz, dz);
    const double wx = d(W.w, Lx, dx), wy = d(W.w, Ly, dy), wz = d(W.w, Lz, dz);
    const double Tx = d(W.T, Lx, dx), Ty = d(W.T, Ly, dy), Tz = d(W.T, Lz, dz);
    const double T = W.T[id];
    const double mu = get_mu<double>(T, P.mu, P.sutherland_s);
    const double kq = P.Cp / P.Pr;
    const double div = ux + vy + wz;
    const double txx = 2.0 * mu * ux - 2.0 / 3.0 * mu * div;
    const double tyy = 2.0 * mu * vy - 2.0 / 3.0 * mu * div;
    const double tzz = 2.0 * mu * wz - 2.0 / 3.0 * mu * div;
    const double txy = mu * (uy + vx), txz = mu * (uz + wx), tyz = mu * (vz + wy);
    const double u = W.u[id], v = W.v[id], w = W.w[id];
    // flux entries: Fv = {txx, txy, txz, ex}, Hv = {txy, tyy, tyz, ey}, Gv = {txz, tyz, tzz, ez}
    double ltxx = lF[0], ltxy = lF[1] + lH[0], ltxz = lF[2] + lGz[0];
    double ltyy = lH[1], ltyz = lH[2] + lGz[1], ltzz = lGz[2];
    const double lex = lF[3], ley = lH[3], lez = lGz[3];
    // e_x = u txx + v txy + w txz + qx, e_y = u txy + v tyy + w tyz + qy, e_z = ...
    double lu = lex * txx + ley * txy + lez * txz;
    double lv = lex * txy + ley * tyy + lez * tyz;
    double lw = lex * txz + ley * tyz + lez * tzz;
    ltxx += lex * u; ltxy += lex * v + ley * u; ltxz += lex * w + lez * u;
    ltyy += ley * v; ltyz += ley * w + lez * v; ltzz += lez * w;
    // q_d = mu Cp/Pr dT_d
    double lmu = kq * (lex * Tx + ley * Ty + lez * Tz);
    const double lTx = lex * mu * kq, lTy = ley * mu * kq, lTz = lez * mu * kq;
    // stresses
    double lux = 2.0 * mu * ltxx, lvy = 2.0 * mu * ltyy, lwz = 2.0 * mu * ltzz;
    const double ldiv = -2.0 / 3.0 * mu * (ltxx + ltyy + ltzz);
    lux += ldiv; lvy += ldiv; lwz += ldiv;
    lmu += ltxx * (2.0 * ux - 2.0 / 3.0 * div) + ltyy * (2.0 * vy - 2.0 / 3.0 * div) +
           ltzz * (2.0 * wz - 2.0 / 3.0 * div);
    lmu += ltxy * (uy + vx) + ltxz * (uz + wx) + ltyz * (vz + wy);
    const double luy = mu * ltxy, lvx = mu * ltxy, luz = mu * ltxz, lwx = mu * ltxz;
    const double lvz = mu * ltyz, lwy = mu * ltyz;
    const double lT = lmu * dmu_dT(T, P.mu, P.sutherland_s);
    const double out[16] = {lux, luy, luz, lvx, lvy, lvz, lwx, lwy, lwz, lTx, lTy, lTz,
                            lu, lv, lw, lT};
#pragma unroll
    for (int q = 0; q < 16; ++q) lg[(long long)q * n + id] = out[q];
}

// Viscous VJP, part 2: gradient transpose (-D) plus the direct parts; T = p/(rho R).
template <int ORD>
__global__ void __launch_bounds__(128)
k_adj_visc2(DevParams P, StateView W, const double* __restrict__ lg, double* __restrict__ lamW) {
    const int nx = P.nx, ny = P.ny;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    const int j = blockIdx.y, k = blockIdx.z;
    const long long n = P.n;
    const long long id = ((long long)k * ny + j) * nx + i;
    const Line Lx = line_of<0>(P, i, j, k, id), Ly = line_of<1>(P, i, j, k, id),
               Lz = line_of<2>(P, i, j, k, id);
    auto d = [&](int blk, const Line& L, double h) {
        const double* a = lg + (long long)blk * n;
        return dcentral<double, ORD>([&](int o) { return a[L.at(L.pos + o)]; }, h);
    };
    double lv4[4];
#pragma unroll
    for (int m = 0; m < 4; ++m)
        lv4[m] = lg[(long long)(12 + m) * n + id] - d(3 * m, Lx, P.dx) - d(3 * m + 1, Ly, P.dy) -
                 d(3 * m + 2, Lz, P.dz);
    double rr = W.rho[id];
    if (rr <= 0.0) rr = 1e-12;
    const double T = W.T[id];
    lamW[1 * n + id] += lv4[0];
    lamW[2 * n + id] += lv4[1];
    lamW[3 * n + id] += lv4[2];
    lamW[4 * n + id] += lv4[3] / (rr * P.Rgas);
    lamW[0 * n + id] += -lv4[3] * T / rr;
}

// Adjoint of one stage. Wk: the stage's output state, Wp: its input state.
// Stage coefficients (U_k = a U0 + bU U(Wp) + bR dt R(Wp)): (1, 0, 1),
// (3/4, 1/4, 1/4), (1/3, 2/3, 2/3). Writes lamR, initialises lamWp with the
// U(Wp) part and accumulates lamU0 (set at stage 3, the first one reversed).
template <int STAGE>
__global__ void __launch_bounds__(256)
k_adj_stage(DevParams P, StateView Wk, StateView Wp, const double* __restrict__ lamWk,
            double* __restrict__ lamU0, double* __restrict__ lamR, double* __restrict__ lamWp,
            double dt) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    const long long n = P.n;
    const double a = STAGE == 1 ? 1.0 : (STAGE == 2 ? 0.75 : 1.0 / 3.0);
    const double bU = STAGE == 1 ? 0.0 : (STAGE == 2 ? 0.25 : 2.0 / 3.0);
    const double bR = STAGE == 1 ? 1.0 : bU;
    double wk[5], lw[5], lU[5];
    load_w5(Wk, id, wk);
#pragma unroll
    for (int q = 0; q < 5; ++q) lw[q] = lamWk[q * n + id];
    c2p_vjp(wk, P.gamma, lw, lU);
    double lp[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (STAGE != 1) {
        double wp[5], lUp[5];
        load_w5(Wp, id, wp);
#pragma unroll
        for (int q = 0; q < 5; ++q) lUp[q] = bU * lU[q];
        p2c_vjp(wp, P.gamma, lUp, lp);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        if (STAGE == 3) lamU0[q * n + id] = a * lU[q];
        else lamU0[q * n + id] += a * lU[q];
        lamR[q * n + id] = bR * dt * lU[q];
        lamWp[q * n + id] = lp[q];
    }
}

// lamW0 += (dU0/dW0)^T lamU0 (U0 = primitiveToConserved of the step's start).
__global__ void __launch_bounds__(256)
k_adj_finish(DevParams P, StateView W0, const double* __restrict__ lamU0, double* __restrict__ lamW0) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    const long long n = P.n;
    double w0[5], lU[5], lw[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    load_w5(W0, id, w0);
#pragma unroll
    for (int q = 0; q < 5; ++q) lU[q] = lamU0[q * n + id];
    p2c_vjp(w0, P.gamma, lU, lw);
#pragma unroll
    for (int q = 0; q < 5; ++q) lamW0[q * n + id] += lw[q];
}

// d/dW of J = sum 0.5 rho |u|^2 dV (compute_total_energy, postprocess.cpp:103).
__global__ void __launch_bounds__(256)
k_adj_seed_ke(DevParams P, StateView W, double* __restrict__ lamW, double dV) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    const long long n = P.n;
    const double rho = W.rho[id], u = W.u[id], v = W.v[id], w = W.w[id];
    lamW[0 * n + id] = 0.5 * (u * u + v * v + w * w) * dV;
    lamW[1 * n + id] = rho * u * dV;
    lamW[2 * n + id] = rho * v * dV;
    lamW[3 * n + id] = rho * w * dV;
    lamW[4 * n + id] = 0.0;
}

template <int DIR, int FVS, int RC>
cudaError_t adj_dir(const LaunchCfg& L, StateView W, const double* lamR, double* G, double* lamW) {
    const DevParams& P = L.P;
    const int ext = DIR == 0 ? P.ny : P.nx;
    const int other = DIR == 2 ? P.ny : P.nz;
    const int len = DIR == 0 ? P.nx : (DIR == 1 ? P.ny : P.nz);
    const int seg = detail::segment_for(len, (long long)ext * other);
    const int th = detail::threads_for(ext);
    dim3 grid((ext + th - 1) / th, other, (len + seg - 1) / seg);
    k_adj_face<DIR, FVS, RC><<<grid, th, 0, L.stream>>>(P, W, lamR, G, seg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int cext = DIR == 0 ? P.ny : P.nx;
    const int tc = detail::threads_for(cext);
    const dim3 cg((cext + tc - 1) / tc, DIR == 0 ? P.nx : P.ny, P.nz);
    k_adj_cell<DIR, FVS, RC><<<cg, tc, 0, L.stream>>>(P, W, G, lamW);
    return cudaGetLastError();
}

template <int FVS, int RC>
cudaError_t adj_inviscid(const LaunchCfg& L, StateView W, const double* lamR, double* G,
                         double* lamW) {
    cudaError_t e = adj_dir<0, FVS, RC>(L, W, lamR, G, lamW);
    if (e == cudaSuccess) e = adj_dir<1, FVS, RC>(L, W, lamR, G, lamW);
    if (e == cudaSuccess) e = adj_dir<2, FVS, RC>(L, W, lamR, G, lamW);
    return e;
}

template <int FVS>
cudaError_t adj_inviscid_rc(const LaunchCfg& L, StateView W, const double* lamR, double* G,
                            double* lamW) {
    switch (L.rc) {
    case RC_WENO5: return adj_inviscid<FVS, RC_WENO5>(L, W, lamR, G, lamW);
    case RC_LINEAR: return adj_inviscid<FVS, RC_LINEAR>(L, W, lamR, G, lamW);
    case RC_LIN6: return adj_inviscid<FVS, RC_LIN6>(L, W, lamR, G, lamW);
    case RC_LIN8: return adj_inviscid<FVS, RC_LIN8>(L, W, lamR, G, lamW);
    default: return cudaErrorNotSupported;
    }
}

}  // namespace

int adj_scratch_blocks(const LaunchCfg& L) {
    const int S = L.rc == RC_LIN8 ? 8 : (L.rc == RC_LINEAR ? 2 : 6);
    return 2 * S * 5;
}

cudaError_t adj_rhs_vjp(const LaunchCfg& L, StateView W, const double* lamR, double* G,
                        double* lg, double* lamW) {
    cudaError_t e = L.fvs == FV_SW ? adj_inviscid_rc<FV_SW>(L, W, lamR, G, lamW)
                                   : adj_inviscid_rc<FV_LF>(L, W, lamR, G, lamW);
    if (e != cudaSuccess) return e;
    const int th = detail::threads_for(L.P.nx);
    const dim3 g = detail::cell_grid(L.P, th);
    switch (L.P.vis_order) {
    case 4:
        k_adj_visc1<4><<<g, th, 0, L.stream>>>(L.P, W, lamR, lg);
        k_adj_visc2<4><<<g, th, 0, L.stream>>>(L.P, W, lg, lamW);
        break;
    case 6:
        k_adj_visc1<6><<<g, th, 0, L.stream>>>(L.P, W, lamR, lg);
        k_adj_visc2<6><<<g, th, 0, L.stream>>>(L.P, W, lg, lamW);
        break;
    default:
        k_adj_visc1<8><<<g, th, 0, L.stream>>>(L.P, W, lamR, lg);
        k_adj_visc2<8><<<g, th, 0, L.stream>>>(L.P, W, lg, lamW);
        break;
    }
    return cudaGetLastError();
}

cudaError_t adj_stage(const LaunchCfg& L, int stage, StateView Wk, StateView Wp,
                      const double* lamWk, double* lamU0, double* lamR, double* lamWp, double dt) {
    const unsigned b = (unsigned)((L.P.n + 255) / 256);
    if (stage == 1) k_adj_stage<1><<<b, 256, 0, L.stream>>>(L.P, Wk, Wp, lamWk, lamU0, lamR, lamWp, dt);
    else if (stage == 2) k_adj_stage<2><<<b, 256, 0, L.stream>>>(L.P, Wk, Wp, lamWk, lamU0, lamR, lamWp, dt);
    else k_adj_stage<3><<<b, 256, 0, L.stream>>>(L.P, Wk, Wp, lamWk, lamU0, lamR, lamWp, dt);
    return cudaGetLastError();
}

cudaError_t adj_finish(const LaunchCfg& L, StateView W0, const double* lamU0, double* lamW0) {
    k_adj_finish<<<(unsigned)((L.P.n + 255) / 256), 256, 0, L.stream>>>(L.P, W0, lamU0, lamW0);
    return cudaGetLastError();
}

cudaError_t adj_seed_ke(const LaunchCfg& L, StateView W, double* lamW, double dV) {
    k_adj_seed_ke<<<(unsigned)((L.P.n + 255) / 256), 256, 0, L.stream>>>(L.P, W, lamW, dV);
    return cudaGetLastError();
}

}  // namespace ns3d
