// Hand-written reverse-mode (vector-Jacobian) forms of the per-cell functions
// of the RHS and the RK3 stage, in FP64. No counterpart in the reference: this
// is the discrete adjoint of the FP64 forward path (the derivative of exactly
// the arithmetic the forward kernels perform, up to rounding).
#pragma once

#include "ns3d_device.cuh"

namespace ns3d {

// d rec / d a_j of weno5(a0..a4), times lam, added to g[0..4].
// rec = sum w_k p_k, w_k = alpha_k / sum alpha, alpha_k = d_k / (eps + beta_k)^2:
// d rec / d beta_l = -2 w_l (p_l - rec) / (eps + beta_l).
// Reciprocals are Newton-refined estimates (rcp_nr, two steps: about an ulp).
__device__ __forceinline__ void weno5_vjp(const double* a, double lam, double* g) {
    const double eps = 1e-6;
    const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3], a4 = a[4];
    const double D0 = a0 - 2.0 * a1 + a2, E0 = a0 - 4.0 * a1 + 3.0 * a2;
    const double D1 = a1 - 2.0 * a2 + a3, E1 = a1 - a3;
    const double D2 = a2 - 2.0 * a3 + a4, E2 = 3.0 * a2 - 4.0 * a3 + a4;
    const double b0 = 13.0 / 12.0 * D0 * D0 + 0.25 * E0 * E0;
    const double b1 = 13.0 / 12.0 * D1 * D1 + 0.25 * E1 * E1;
    const double b2 = 13.0 / 12.0 * D2 * D2 + 0.25 * E2 * E2;
    const double r0 = rcp_nr<2>(eps + b0), r1 = rcp_nr<2>(eps + b1), r2 = rcp_nr<2>(eps + b2);
    const double al0 = 0.1 * r0 * r0, al1 = 0.6 * r1 * r1, al2 = 0.3 * r2 * r2;
    const double inv = rcp_nr<2>(al0 + al1 + al2);
    const double w0 = al0 * inv, w1 = al1 * inv, w2 = al2 * inv;
    const double p0 = (2.0 * a0 - 7.0 * a1 + 11.0 * a2) * (1.0 / 6.0);
    const double p1 = (-a1 + 5.0 * a2 + 2.0 * a3) * (1.0 / 6.0);
    const double p2 = (2.0 * a2 + 5.0 * a3 - a4) * (1.0 / 6.0);
    const double rec = w0 * p0 + w1 * p1 + w2 * p2;
    const double s0 = -2.0 * w0 * (p0 - rec) * r0 * lam;
    const double s1 = -2.0 * w1 * (p1 - rec) * r1 * lam;
    const double s2 = -2.0 * w2 * (p2 - rec) * r2 * lam;
    const double c = 13.0 / 6.0;
    g[0] += lam * (w0 * (2.0 / 6.0)) + s0 * (c * D0 + 0.5 * E0);
    g[1] += lam * (w0 * (-7.0 / 6.0) + w1 * (-1.0 / 6.0)) + s0 * (-2.0 * c * D0 - 2.0 * E0) +
            s1 * (c * D1 + 0.5 * E1);
    g[2] += lam * (w0 * (11.0 / 6.0) + w1 * (5.0 / 6.0) + w2 * (2.0 / 6.0)) +
            s0 * (c * D0 + 1.5 * E0) + s1 * (-2.0 * c * D1) + s2 * (c * D2 + 1.5 * E2);
    g[3] += lam * (w1 * (2.0 / 6.0) + w2 * (5.0 / 6.0)) + s1 * (c * D1 - 0.5 * E1) +
            s2 * (-2.0 * c * D2 - 2.0 * E2);
    g[4] += lam * (w2 * (-1.0 / 6.0)) + s2 * (c * D2 + 0.5 * E2);
}

// VJP of one reconstruction with respect to its (already oriented) window.
template <int RC>
__device__ __forceinline__ void reconstruct_vjp(const double* s, const double* lin, double lam,
                                                double* g) {
    if constexpr (RC == RC_WENO5) {
        weno5_vjp(s, lam, g);
    } else if constexpr (RC == RC_LINEAR) {
        g[0] += lam;
    } else {
        constexpr int S = Stencil<RC>::S;
#pragma unroll
        for (int m = 0; m < S; ++m) g[m] += lam * lin[m];
    }
}

// Split fluxes of one primitive state w = (rho,u,v,w,p) along DIR and the
// VJP: gw[5] += (dF+/dw)^T gp + (dF-/dw)^T gm. The forward part repeats
// p2c_Ec + split_sw / split_lf in FP64, with Newton-refined reciprocals and
// square roots (rcp_nr, sqrt_nr, two steps) in place of IEEE division and sqrt.
template <int FVS, int DIR>
__device__ __forceinline__ void split_vjp(const double* w5, double gamma, double eps,
                                          const double* gp, const double* gm, double* gw) {
    const double rho = w5[0], u = w5[1], v = w5[2], w = w5[3], p = w5[4];
    const double vel[3] = {u, v, w};
    const double k = 0.5 * (u * u + v * v + w * w);
    const double ir = rcp_nr<2>(rho);
    const double E = p / (gamma - 1.0) + rho * k;
    const double c = sqrt_nr<2>(gamma * p * ir);
    const double un = vel[DIR];
    double grho = 0.0, gvel[3] = {0.0, 0.0, 0.0}, gp_ = 0.0, gE = 0.0, gc = 0.0, gk = 0.0,
           gun = 0.0;
    if constexpr (FVS == FV_SW) {
        const double l[3] = {un - c, un, un + c};
        double a[3], lp[3], lm[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            a[i] = eps > 0.0 ? sqrt_nr<2>(l[i] * l[i] + eps * eps) : fabs(l[i]);
            lp[i] = 0.5 * (l[i] + a[i]);
            lm[i] = 0.5 * (l[i] - a[i]);
        }
        const double S1p = lp[0] + lp[2], S1m = lm[0] + lm[2];
        const double S2p = lp[2] - lp[0], S2m = lm[2] - lm[0];
        const double H = (E + p) * ir;
        const double ga1 = rho / (2.0 * gamma), ga2 = 2.0 * (gamma - 1.0);
        const double V = k;
        double gS1p = 0, gS1m = 0, gS2p = 0, gS2m = 0, glp2 = 0, glm2 = 0, gH = 0, gV = 0,
               gga1 = 0;
        // F+- = ga1 * (bracket); bracket per component
        auto side = [&](const double* g, double S1, double l2, double S2, double& gS1,
                        double& gl2, double& gS2) {
            double br[5];
            br[0] = S1 + ga2 * l2;
#pragma unroll
            for (int j = 0; j < 3; ++j)
                br[1 + j] = S1 * vel[j] + ga2 * l2 * vel[j] + (j == DIR ? S2 * c : 0.0);
            br[4] = S1 * H + ga2 * l2 * V + S2 * un * c;
#pragma unroll
            for (int q = 0; q < 5; ++q) gga1 += g[q] * br[q];
            const double G0 = g[0] * ga1, G4 = g[4] * ga1;
            gS1 += G0;
            gl2 += G0 * ga2;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double Gj = g[1 + j] * ga1;
                gS1 += Gj * vel[j];
                gvel[j] += Gj * (S1 + ga2 * l2);
                gl2 += Gj * ga2 * vel[j];
                if (j == DIR) {
                    gS2 += Gj * c;
                    gc += Gj * S2;
                }
            }
            gS1 += G4 * H;
            gH += G4 * S1;
            gl2 += G4 * ga2 * V;
            gV += G4 * ga2 * l2;
            gS2 += G4 * un * c;
            gun += G4 * S2 * c;
            gc += G4 * S2 * un;
        };
        side(gp, S1p, lp[1], S2p, gS1p, glp2, gS2p);
        side(gm, S1m, lm[1], S2m, gS1m, glm2, gS2m);
        double glp[3] = {gS1p - gS2p, glp2, gS1p + gS2p};
        double glm[3] = {gS1m - gS2m, glm2, gS1m + gS2m};
        double gl[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double ga = 0.5 * (glp[i] - glm[i]);
            gl[i] = 0.5 * (glp[i] + glm[i]);
            const double dadl = eps > 0.0 ? l[i] * rcp_nr<2>(a[i]) : (l[i] > 0.0 ? 1.0 : (l[i] < 0.0 ? -1.0 : 0.0));
            gl[i] += ga * dadl;
        }
        gun += gl[0] + gl[1] + gl[2];
        gc += -gl[0] + gl[2];
        gE += gH * ir;
        gp_ += gH * ir;
        grho += -gH * H * ir;
        gk += gV;
        grho += gga1 / (2.0 * gamma);
    } else {
        const double n[3] = {DIR == 0 ? 1.0 : 0.0, DIR == 1 ? 1.0 : 0.0, DIR == 2 ? 1.0 : 0.0};
        const double amax = fabs(un) + c;
        const double U[5] = {rho, rho * u, rho * v, rho * w, E};
        double gF[5], gaU[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            gF[q] = 0.5 * (gp[q] + gm[q]);
            gaU[q] = 0.5 * (gp[q] - gm[q]);
        }
        double gamax = 0.0, gU[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            gamax += gaU[q] * U[q];
            gU[q] = gaU[q] * amax;
        }
        // F1 = rho un; F2..4 = rho vel_j un + p n_j; F5 = (E + p) un
        grho += gF[0] * un;
        gun += gF[0] * rho;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            grho += gF[1 + j] * vel[j] * un;
            gvel[j] += gF[1 + j] * rho * un;
            gun += gF[1 + j] * rho * vel[j];
            gp_ += gF[1 + j] * n[j];
        }
        gE += gF[4] * un;
        gp_ += gF[4] * un;
        gun += gF[4] * (E + p);
        // U
        grho += gU[0];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            grho += gU[1 + j] * vel[j];
            gvel[j] += gU[1 + j] * rho;
        }
        gE += gU[4];
        gun += gamax * (un > 0.0 ? 1.0 : (un < 0.0 ? -1.0 : 0.0));
        gc += gamax;
    }
    gvel[DIR] += gun;
    // c = sqrt(gamma p / rho)
    gp_ += gc * gamma * 0.5 * rcp_nr<2>(c) * ir;
    grho += -gc * c * 0.5 * ir;
    // E = p/(gamma-1) + rho k
    gp_ += gE / (gamma - 1.0);
    grho += gE * k;
    gk += gE * rho;
    // k = |vel|^2 / 2
#pragma unroll
    for (int j = 0; j < 3; ++j) gvel[j] += gk * vel[j];
    gw[0] += grho;
    gw[1] += gvel[0];
    gw[2] += gvel[1];
    gw[3] += gvel[2];
    gw[4] += gp_;
}

// conservedToPrimitive VJP evaluated at the primitive result w: lam_w -> lam_U.
__device__ __forceinline__ void c2p_vjp(const double* w5, double gamma, const double* lw,
                                        double* lU) {
    const double rho = w5[0], u = w5[1], v = w5[2], w = w5[3];
    const double g1 = gamma - 1.0;
    const double k = 0.5 * (u * u + v * v + w * w);
    lU[0] = lw[0] - (lw[1] * u + lw[2] * v + lw[3] * w) / rho + lw[4] * g1 * k;
    lU[1] = lw[1] / rho - lw[4] * g1 * u;
    lU[2] = lw[2] / rho - lw[4] * g1 * v;
    lU[3] = lw[3] / rho - lw[4] * g1 * w;
    lU[4] = lw[4] * g1;
}

// primitiveToConserved VJP at w: lam_U -> lam_w (added).
__device__ __forceinline__ void p2c_vjp(const double* w5, double gamma, const double* lU,
                                        double* lw) {
    const double rho = w5[0], u = w5[1], v = w5[2], w = w5[3];
    const double k = 0.5 * (u * u + v * v + w * w);
    lw[0] += lU[0] + lU[1] * u + lU[2] * v + lU[3] * w + lU[4] * k;
    lw[1] += lU[1] * rho + lU[4] * rho * u;
    lw[2] += lU[2] * rho + lU[4] * rho * v;
    lw[3] += lU[3] * rho + lU[4] * rho * w;
    lw[4] += lU[4] / (gamma - 1.0);
}

// d mu / d T of get_mu: mu (1.5 / T - 1 / (T + S)).
__device__ __forceinline__ double dmu_dT(double T, double mu_ref, double S) {
    const double mu = get_mu<double>(T, mu_ref, S);
    return mu * (1.5 / T - 1.0 / (T + S));
}

}  // namespace ns3d
