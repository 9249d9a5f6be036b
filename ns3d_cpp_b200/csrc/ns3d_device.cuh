// Per-cell device functions of the RHS: thermodynamics, flux vector splitting,
// scalar reconstructions, central differences.
//
// Templated on the compute type R. The FP64 instantiation is compiled with
// -fmad=false and keeps the reference's expression order term by term, so it
// reproduces the reference's rounding (IEEE division and sqrt are correctly
// rounded on both sides; T^1.5 is rounded once from a value accurate far
// beyond double, which glibc's pow matches on all but ~0.2% of arguments and
// differs from there by an ulp). The FP32 instantiation
// runs the same algebra in float (the FP32-stencil form).
#pragma once

#include <cstdint>

namespace ns3d {

// Scheme identifiers used as template arguments. Linear schemes share one
// code path: MDCD (reconstruction.cpp:126-135) is a 6-point linear stencil and
// UPWIND_7TH / UD7L (:227-249) are 8-point linear stencils whose coefficients
// are evaluated on the host with the reference's expressions.
enum : int { RC_WENO5 = 0, RC_LINEAR = 2, RC_LIN6 = 3, RC_MDCD_HYBRID = 4, RC_LIN8 = 5 };
enum : int { FV_SW = 0, FV_LF = 1 };

template <int RC> struct Stencil;
template <> struct Stencil<RC_WENO5> { static constexpr int S = 6; };
template <> struct Stencil<RC_LINEAR> { static constexpr int S = 2; };
template <> struct Stencil<RC_LIN6> { static constexpr int S = 6; };
template <> struct Stencil<RC_MDCD_HYBRID> { static constexpr int S = 6; };
template <> struct Stencil<RC_LIN8> { static constexpr int S = 8; };

// Parameters every kernel receives by value.
struct DevParams {
    int nx, ny, nz;
    long long n;
    double gamma, Rgas, mu, Cp, Pr, sutherland_s, sw_eps;
    double dx, dy, dz, inv_dx, inv_dy, inv_dz;
    double cfl, dt_fixed;
    double lin[8];   // linear reconstruction coefficients (LIN6 / LIN8)
    double mdcd_disp, mdcd_diss;
    int vis_order;   // 4, 6, 8
};

// ---------------------------------------------------------------------------
// Thermodynamics (field_structures.h:94-105, 405-451)
// ---------------------------------------------------------------------------

// T^1.5 rounded once from a ~2^-104-accurate value (so correctly rounded but
// for results within that distance of a rounding midpoint, such as T a few
// ulps from 1, which may land one ulp off), by error-free
// transformations (Dekker 1971; the FMA residual of a square root, Markstein
// 1990): s = RN(sqrt T) and r = T - s^2 exactly (one FMA), so
// sqrt T = s + r / (2 s) to relative O((r / s^2)^2); p = RN(T s) and its
// error e = T s - p exactly (one FMA), so T^1.5 = p + e + T r / (2 s), where
// T r / (2 s) = r s / 2 + r^2 / (2 s) and the last term is ~2^-106 of the
// result; only the final addition rounds at the result's scale. The reference's libm
// pow (glibc) is correctly rounded on all but ~0.2% of the temperatures the
// solver meets, against which a general-purpose pow differs by an ulp on
// several percent. Zero, negative, infinite and NaN arguments go to pow.
__device__ __forceinline__ double pow_1p5(double T) {
    const double s = sqrt(T);
    if (!(s > 0.0) || !(s < 1.0e300)) return pow(T, 1.5);
    const double r = fma(-s, s, T);
    const double p = T * s;
    const double e = fma(T, s, -p);
    return p + (e + 0.5 * (r * s));
}

// SolverParams::get_mu (field_structures.h:94-105): Sutherland.
template <class R>
__device__ __forceinline__ R get_mu(R T, R mu_ref, R S) {
    return mu_ref * pow_1p5(T) * (R(1.0) + S) / (T + S);
}

// FP32-stencil form: T^1.5 as T sqrt(T) (the difference from pow is far below
// the float rounding this form carries; pow costs several times more).
template <>
__device__ __forceinline__ float get_mu<float>(float T, float mu_ref, float S) {
    return mu_ref * (T * sqrtf(T)) * (1.0f + S) / (T + S);
}

// primitiveToConserved (field_structures.h:430-451) for one cell: E and c.
template <class R>
__device__ __forceinline__ void p2c_Ec(R rr, R u, R v, R w, R p, R gamma, R& E, R& c) {
    R kinetic = R(0.5) * (u * u + v * v + w * w);
    R e_internal = p / ((gamma - R(1.0)) * rr);
    E = rr * (e_internal + kinetic);
    c = sqrt(gamma * p / rr);
}

// ---------------------------------------------------------------------------
// Flux vector splitting (InviscousFlux_new.cpp:439-530)
// ---------------------------------------------------------------------------

template <class R>
__device__ __forceinline__ R abs_fix(R l, R eps) {
    // README.md:177-180 entropy fix; eps == 0 is the reference's plain |l|.
    return eps > R(0) ? sqrt(l * l + eps * eps) : fabs(l);
}

// split_StagerWarming (InviscousFlux_new.cpp:439-489). N1,N2,N3: direction.
template <class R, int N1, int N2, int N3>
__device__ __forceinline__ void split_sw(R rho, R u, R v, R w, R E, R p, R c, R gamma, R eps,
                                         R Fp[5], R Fm[5]) {
    const R n1 = R(N1), n2 = R(N2), n3 = R(N3);
    R un = u * n1 + v * n2 + w * n3;
    R lambda1 = un - c, lambda2 = un, lambda3 = un + c;
    R a1 = abs_fix(lambda1, eps), a2 = abs_fix(lambda2, eps), a3 = abs_fix(lambda3, eps);
    R lambda1_plus = R(0.5) * (lambda1 + a1);
    R lambda1_minus = R(0.5) * (lambda1 - a1);
    R lambda2_plus = R(0.5) * (lambda2 + a2);
    R lambda2_minus = R(0.5) * (lambda2 - a2);
    R lambda3_plus = R(0.5) * (lambda3 + a3);
    R lambda3_minus = R(0.5) * (lambda3 - a3);
    R S1_p = lambda1_plus + lambda3_plus;
    R S1_m = lambda1_minus + lambda3_minus;
    R S2_p = lambda3_plus - lambda1_plus;
    R S2_m = lambda3_minus - lambda1_minus;
    R H = (E + p) / rho;
    R ga1 = rho / (R(2.0) * gamma);
    R ga2 = R(2.0) * (gamma - R(1.0));
    R V = R(0.5) * (u * u + v * v + w * w);
    Fp[0] = ga1 * (S1_p + ga2 * lambda2_plus);
    Fp[1] = ga1 * (S1_p * u + ga2 * lambda2_plus * u + S2_p * n1 * c);
    Fp[2] = ga1 * (S1_p * v + ga2 * lambda2_plus * v + S2_p * n2 * c);
    Fp[3] = ga1 * (S1_p * w + ga2 * lambda2_plus * w + S2_p * n3 * c);
    Fp[4] = ga1 * (S1_p * H + ga2 * lambda2_plus * V + S2_p * un * c);
    Fm[0] = ga1 * (S1_m + ga2 * lambda2_minus);
    Fm[1] = ga1 * (S1_m * u + ga2 * lambda2_minus * u + S2_m * n1 * c);
    Fm[2] = ga1 * (S1_m * v + ga2 * lambda2_minus * v + S2_m * n2 * c);
    Fm[3] = ga1 * (S1_m * w + ga2 * lambda2_minus * w + S2_m * n3 * c);
    Fm[4] = ga1 * (S1_m * H + ga2 * lambda2_minus * V + S2_m * un * c);
}

// split_LaxFriedrichs (InviscousFlux_new.cpp:491-530), local wave speed.
template <class R, int N1, int N2, int N3>
__device__ __forceinline__ void split_lf(R rho, R u, R v, R w, R E, R p, R c, R Fp[5],
                                         R Fm[5]) {
    const R n1 = R(N1), n2 = R(N2), n3 = R(N3);
    R un = u * n1 + v * n2 + w * n3;
    R a_max = fabs(un) + c;
    R F1 = rho * un;
    R F2 = rho * u * un + p * n1;
    R F3 = rho * v * un + p * n2;
    R F4 = rho * w * un + p * n3;
    R F5 = (E + p) * un;
    Fp[0] = R(0.5) * (F1 + a_max * rho);
    Fp[1] = R(0.5) * (F2 + a_max * rho * u);
    Fp[2] = R(0.5) * (F3 + a_max * rho * v);
    Fp[3] = R(0.5) * (F4 + a_max * rho * w);
    Fp[4] = R(0.5) * (F5 + a_max * E);
    Fm[0] = R(0.5) * (F1 - a_max * rho);
    Fm[1] = R(0.5) * (F2 - a_max * rho * u);
    Fm[2] = R(0.5) * (F3 - a_max * rho * v);
    Fm[3] = R(0.5) * (F4 - a_max * rho * w);
    Fm[4] = R(0.5) * (F5 - a_max * E);
}

// ---------------------------------------------------------------------------
// FP32-stencil form of the split (double, feeding the float reconstructions).
//
// Same formulas as p2c_Ec + split_sw / split_lf, with the divisions by rho
// replaced by one reciprocal and the square roots (sound speed, entropy fix)
// taken from the hardware estimates refined by one Newton-Raphson step:
//   1/b:     x <- x + x (1 - b x)
//   sqrt(b): s = b y (y ~ 1/sqrt b), s <- s + (y/2) (b - s^2)   (Heron)
// Each step squares the estimate's relative error (2^-23 or better on entry):
// one step leaves ~1e-14, far below the float rounding of the deviations that
// the FP32 form's reconstructions see (measured: the same FP32-vs-FP64 error
// after 100 steps at 256^3 as with IEEE operations); two steps (with the
// 1/sqrt estimate refined first, y <- y (3 - b y^2) / 2) leave about an ulp,
// which the FP64 adjoint needs because the entropy fix's 0.5 (l - sqrt(l^2 +
// eps^2)) amplifies the square root's error by ~l^2/eps^2. The FP64 forward
// form keeps the reference's IEEE divisions and square roots.
// ---------------------------------------------------------------------------
template <int STEPS = 1>
__device__ __forceinline__ double rcp_nr(double b) {
    double x;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(b));
#pragma unroll
    for (int s = 0; s < STEPS; ++s) x = fma(x, fma(-b, x, 1.0), x);
    return x;
}

template <int STEPS = 1>
__device__ __forceinline__ double sqrt_nr(double b) {
    // zero, negative, NaN and huge arguments take the IEEE path
    if (!(b > 0.0 && b < 1.0e300)) return sqrt(b);
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
#pragma unroll
    for (int s = 1; s < STEPS; ++s) y = y * fma(-0.5 * b * y, y, 1.5);
    const double s = b * y;
    return fma(0.5 * y, fma(-s, s, b), s);
}

// sqrt_nr<1> without a branch, for code whose instructions the compiler should
// be free to interleave with independent work (a branch ends the scheduling
// region). Equal to sqrt_nr<1> for b in (0, 1e300); +-0 and NaN as IEEE sqrt;
// negative b gives NaN like sqrt; b >= 1e300 or subnormal also gives NaN
// (a sound speed or entropy-fix argument outside (1e-308, 1e300) belongs to a
// nonphysical state, which the stage update's positivity check then reports).
__device__ __forceinline__ double sqrt_nr_nb(double b) {
    const bool ok = b > 0.0 && b < 1.0e300;
    const double bs = ok ? b : 1.0;
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(bs));
    const double s = bs * y;
    const double r = fma(0.5 * y, fma(-s, s, bs), s);
    return ok ? r : (b == 0.0 ? b : __longlong_as_double(0x7ff8000000000000LL));
}

// raw = (rho, u, v, w, p) of one cell; inv_gm1 = 1/(gamma-1), inv_2g = 1/(2 gamma).
// The face normal (N1, N2, N3) is a coordinate axis, so the normal velocity is
// one component and the c-terms enter only the normal momentum; the products
// with the zero components (which IEEE arithmetic cannot drop by itself) are
// left out. ENT: -1 reads whether the entropy fix is on from P.sw_eps at run
// time, 0 / 1 fix it at compile time; NB (with STEPS = 1) takes the square
// roots from sqrt_nr_nb, so that with ENT >= 0 the split has no branch.
template <int FVS, int N1, int N2, int N3, int STEPS = 1, int ENT = -1, bool NB = false>
__device__ __forceinline__ void split_fast(const DevParams& P, double inv_gm1, double inv_2g,
                                           const double* raw, double Fp[5], double Fm[5]) {
    static_assert(N1 + N2 + N3 == 1, "axis-aligned face normal");
    static_assert(!NB || STEPS == 1, "the branch-free square root takes one Newton step");
    auto root = [](double b) { return NB ? sqrt_nr_nb(b) : sqrt_nr<STEPS>(b); };
    double rho = raw[0];
    if (rho <= 0.0) rho = 1e-12;
    const double u = raw[1], v = raw[2], w = raw[3], p = raw[4];
    const double gamma = P.gamma;
    const double ir = rcp_nr<STEPS>(rho);
    const double kinetic = 0.5 * (u * u + v * v + w * w);
    const double E = rho * (p * ir * inv_gm1 + kinetic);
    const double c = root(gamma * p * ir);
    const double un = N1 ? u : (N2 ? v : w);
    if constexpr (FVS == FV_SW) {
        const double eps = P.sw_eps;
        const bool fix = ENT < 0 ? eps > 0.0 : ENT == 1;
        const double l1 = un - c, l2 = un, l3 = un + c;
        const double a1 = fix ? root(l1 * l1 + eps * eps) : fabs(l1);
        const double a2 = fix ? root(l2 * l2 + eps * eps) : fabs(l2);
        const double a3 = fix ? root(l3 * l3 + eps * eps) : fabs(l3);
        const double l1p = 0.5 * (l1 + a1), l1m = 0.5 * (l1 - a1);
        const double l2p = 0.5 * (l2 + a2), l2m = 0.5 * (l2 - a2);
        const double l3p = 0.5 * (l3 + a3), l3m = 0.5 * (l3 - a3);
        const double S1p = l1p + l3p, S1m = l1m + l3m;
        const double S2p = l3p - l1p, S2m = l3m - l1m;
        const double H = (E + p) * ir;
        const double ga1 = rho * inv_2g;
        const double ga2 = 2.0 * (gamma - 1.0);
        const double cp = S2p * c, cm = S2m * c;
        const double bp = S1p + ga2 * l2p, bm = S1m + ga2 * l2m;  // common factor of u, v, w
        Fp[0] = ga1 * bp;
        Fp[1] = ga1 * (N1 ? bp * u + cp : bp * u);
        Fp[2] = ga1 * (N2 ? bp * v + cp : bp * v);
        Fp[3] = ga1 * (N3 ? bp * w + cp : bp * w);
        Fp[4] = ga1 * (S1p * H + ga2 * l2p * kinetic + cp * un);
        Fm[0] = ga1 * bm;
        Fm[1] = ga1 * (N1 ? bm * u + cm : bm * u);
        Fm[2] = ga1 * (N2 ? bm * v + cm : bm * v);
        Fm[3] = ga1 * (N3 ? bm * w + cm : bm * w);
        Fm[4] = ga1 * (S1m * H + ga2 * l2m * kinetic + cm * un);
    } else {
        // split_lf with the pressure only in the normal momentum
        const double a_max = fabs(un) + c;
        const double F1 = rho * un;
        const double F2 = rho * u * un + (N1 ? p : 0.0);
        const double F3 = rho * v * un + (N2 ? p : 0.0);
        const double F4 = rho * w * un + (N3 ? p : 0.0);
        const double F5 = (E + p) * un;
        Fp[0] = 0.5 * (F1 + a_max * rho);
        Fp[1] = 0.5 * (F2 + a_max * rho * u);
        Fp[2] = 0.5 * (F3 + a_max * rho * v);
        Fp[3] = 0.5 * (F4 + a_max * rho * w);
        Fp[4] = 0.5 * (F5 + a_max * E);
        Fm[0] = 0.5 * (F1 - a_max * rho);
        Fm[1] = 0.5 * (F2 - a_max * rho * u);
        Fm[2] = 0.5 * (F3 - a_max * rho * v);
        Fm[3] = 0.5 * (F4 - a_max * rho * w);
        Fm[4] = 0.5 * (F5 - a_max * E);
    }
}

// ---------------------------------------------------------------------------
// Characteristic-wise reconstruction (du_inviscous_character,
// InviscousFlux_new.cpp:165-437): at each face the Roe-averaged state of its
// two cells, the left / right eigenvector matrices along the face normal, the
// split-flux windows projected on the left eigenvectors, one reconstruction
// per characteristic field, and the result mapped back by the right ones.
// ---------------------------------------------------------------------------

// computeRoeAveragedState_new (InviscousFlux_new.cpp:628-659): (rho, u, v, w, H)
// of two primitive states (rho, u, v, w, p); same operation order.
__device__ __forceinline__ void roe_state(double gamma, const double* l, const double* r,
                                          double* ua) {
    const double EL = l[0] * (0.5 * (l[1] * l[1] + l[2] * l[2] + l[3] * l[3]) +
                              l[4] / ((gamma - 1.0) * l[0]));
    const double ER = r[0] * (0.5 * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) +
                              r[4] / ((gamma - 1.0) * r[0]));
    const double sl = sqrt(l[0]), sr = sqrt(r[0]);
    ua[0] = sl * sr;
    const double den = 1.0 / (sl + sr);
    ua[1] = (sl * l[1] + sr * r[1]) * den;
    ua[2] = (sl * l[2] + sr * r[2]) * den;
    ua[3] = (sl * l[3] + sr * r[3]) * den;
    const double HL = (EL + l[4]) / l[0];
    const double HR = (ER + r[4]) / r[0];
    ua[4] = (sl * HL + sr * HR) * den;
}

// build_eigen_matrices_new (InviscousFlux_new.cpp:532-625) along the unit normal
// (N1, N2, N3): the same entries in the same operation order.
template <int N1, int N2, int N3>
__device__ __forceinline__ void eigen_LR(double gamma, const double* ua, double Lm[5][5],
                                         double Rm[5][5]) {
    const double nx = N1, ny = N2, nz = N3;
    const double u0 = ua[1], v0 = ua[2], w0 = ua[3], h0 = ua[4];
    const double V = 0.5 * (u0 * u0 + v0 * v0 + w0 * w0);
    const double un = u0 * nx + v0 * ny + w0 * nz;
    const double c = sqrt((gamma - 1.0) * (h0 - V));
    const double t2 = u0 * nz + v0 * nx + w0 * ny;  // the two transverse velocities
    const double t3 = u0 * ny + v0 * nz + w0 * nx;
    Rm[0][0] = 1.0;         Rm[0][1] = 1.0; Rm[0][2] = 0.0; Rm[0][3] = 0.0; Rm[0][4] = 1.0;
    Rm[1][0] = u0 - c * nx; Rm[1][1] = u0;  Rm[1][2] = nz;  Rm[1][3] = ny;  Rm[1][4] = u0 + c * nx;
    Rm[2][0] = v0 - c * ny; Rm[2][1] = v0;  Rm[2][2] = nx;  Rm[2][3] = nz;  Rm[2][4] = v0 + c * ny;
    Rm[3][0] = w0 - c * nz; Rm[3][1] = w0;  Rm[3][2] = ny;  Rm[3][3] = nx;  Rm[3][4] = w0 + c * nz;
    Rm[4][0] = h0 - un * c; Rm[4][1] = V;   Rm[4][2] = t2;  Rm[4][3] = t3;  Rm[4][4] = h0 + un * c;
    const double chi = 0.5 / c;
    const double K = (gamma - 1.0) / (c * c);
    const double K1 = K / 2;
    Lm[0][0] = K1 * V + chi * un;    Lm[0][1] = -chi * nx - K1 * u0; Lm[0][2] = -chi * ny - K1 * v0;
    Lm[0][3] = -chi * nz - K1 * w0;  Lm[0][4] = K1;
    Lm[1][0] = 1.0 - K * V;  Lm[1][1] = K * u0;  Lm[1][2] = K * v0;  Lm[1][3] = K * w0;  Lm[1][4] = -K;
    Lm[2][0] = -t2;  Lm[2][1] = nz;  Lm[2][2] = nx;  Lm[2][3] = ny;  Lm[2][4] = 0.0;
    Lm[3][0] = -t3;  Lm[3][1] = ny;  Lm[3][2] = nz;  Lm[3][3] = nx;  Lm[3][4] = 0.0;
    Lm[4][0] = K1 * V - chi * un;    Lm[4][1] = chi * nx - K1 * u0;  Lm[4][2] = chi * ny - K1 * v0;
    Lm[4][3] = chi * nz - K1 * w0;   Lm[4][4] = K1;
}

// ---------------------------------------------------------------------------
// Scalar reconstructions (reconstruction.cpp). `s` is the window after the
// reversal that reconstruct_select applies for the minus flux (:24-31).
// ---------------------------------------------------------------------------

// a / b for a divisor b known in advance, with y = RN(1/b) precomputed (an IEEE
// division): Markstein's theorem (P. Markstein, IBM J. Res. Dev. 34(1), 1990)
// -- if y is 1/b correctly rounded and q is within one ulp of a/b, then
// r = a - b q is a double (one exact FMA) and RN(q + r y) = RN(a/b). Here
// q = RN(a y) is within one ulp, so the result equals the IEEE quotient a / b
// bit for bit (finite a/b in the normal range), in three operations.
__device__ __forceinline__ double div_rcp(double a, double b, double y) {
    const double q = a * y;
    const double r = fma(-b, q, a);
    return fma(r, y, q);
}

// weno5_reconstruction (reconstruction.cpp:93-124): WENO5-JS, eps 1e-6, p = 2.
template <class R>
__device__ __forceinline__ R weno5(R f0, R f1, R f2, R f3, R f4) {
    const R eps = R(1e-6);
    R beta0 = R(13.0 / 12.0) * (f0 - R(2) * f1 + f2) * (f0 - R(2) * f1 + f2)
            + R(0.25) * (f0 - R(4) * f1 + R(3) * f2) * (f0 - R(4) * f1 + R(3) * f2);
    R beta1 = R(13.0 / 12.0) * (f1 - R(2) * f2 + f3) * (f1 - R(2) * f2 + f3)
            + R(0.25) * (f1 - f3) * (f1 - f3);
    R beta2 = R(13.0 / 12.0) * (f2 - R(2) * f3 + f4) * (f2 - R(2) * f3 + f4)
            + R(0.25) * (R(3) * f2 - R(4) * f3 + f4) * (R(3) * f2 - R(4) * f3 + f4);
    R alpha0 = R(0.1) / ((eps + beta0) * (eps + beta0));
    R alpha1 = R(0.6) / ((eps + beta1) * (eps + beta1));
    R alpha2 = R(0.3) / ((eps + beta2) * (eps + beta2));
    R asum = alpha0 + alpha1 + alpha2;
    R w0 = alpha0 / asum;
    R w1 = alpha1 / asum;
    R w2 = alpha2 / asum;
    // the reference's division by 6, as the IEEE quotient (div_rcp)
    const double six = 6.0, rcp6 = 1.0 / 6.0;
    R p0 = div_rcp(R(2) * f0 - R(7) * f1 + R(11) * f2, six, rcp6);
    R p1 = div_rcp(-f1 + R(5) * f2 + R(2) * f3, six, rcp6);
    R p2 = div_rcp(R(2) * f2 + R(5) * f3 - f4, six, rcp6);
    return w0 * p0 + w1 * p1 + w2 * p2;
}

// FP32-stencil form of weno5 (preferred over the template for float): the same
// indicators z_k = eps + beta_k and the same normalised combination of the
// three candidate stencils, with the nonlinear weights taken over a common
// denominator. With y_k = z_k^2, alpha_k = d_k / y_k; multiplying every
// alpha_k by y0 y1 y2 gives e_k = d_k m_k (m0 = y1 y2, m1 = y0 y2, m2 = y0 y1)
// and w_k = e_k / (e0 + e1 + e2): one reciprocal per reconstruction instead
// of four divisions. z_k >= eps = 1e-6, so the products stay >= 1e-25, well
// inside float's normal range for any deviation below ~1e4. The candidate
// stencils keep their integer coefficients (summing to exactly 6) and the 1/6
// is applied once to the combination: coefficients pre-divided by 6 do not sum
// to 1 in float and were measured to bias the faces by the deviation's size.
__device__ __forceinline__ float rcp_approx(float x);
__device__ __forceinline__ float weno5(float f0, float f1, float f2, float f3, float f4) {
    const float eps = 1e-6f;
    const float t0 = f0 - 2.f * f1 + f2, s0 = f0 - 4.f * f1 + 3.f * f2;
    const float t1 = f1 - 2.f * f2 + f3, s1 = f1 - f3;
    const float t2 = f2 - 2.f * f3 + f4, s2 = 3.f * f2 - 4.f * f3 + f4;
    const float z0 = eps + ((13.f / 12.f) * t0 * t0 + 0.25f * s0 * s0);
    const float z1 = eps + ((13.f / 12.f) * t1 * t1 + 0.25f * s1 * s1);
    const float z2 = eps + ((13.f / 12.f) * t2 * t2 + 0.25f * s2 * s2);
    const float y0 = z0 * z0, y1 = z1 * z1, y2 = z2 * z2;
    const float e0 = 0.1f * (y1 * y2), e1 = 0.6f * (y0 * y2), e2 = 0.3f * (y0 * y1);
    const float P0 = 2.f * f0 - 7.f * f1 + 11.f * f2;
    const float P1 = -f1 + 5.f * f2 + 2.f * f3;
    const float P2 = 2.f * f2 + 5.f * f3 - f4;
    const float num = e0 * P0 + e1 * P1 + e2 * P2;
    return (num * (1.f / 6.f)) * rcp_approx(e0 + e1 + e2);
}

// Approximate float reciprocal (the hardware estimate, ~1 ulp).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Two float weno5 reconstructions at once in sm_100's paired FP32 arithmetic
// (one FFMA2/FADD2/FMUL2 instruction per operation on both lanes of a float2):
// the same indicators, common-denominator weights, candidate stencils and
// normalised sum as weno5(float), operation for operation; only the one
// approximate reciprocal runs per lane. The sweeps are instruction-issue
// bound, so halving the reconstructions' instruction count shortens them.
__device__ __forceinline__ float2 weno5x2(float2 f0, float2 f1, float2 f2, float2 f3, float2 f4) {
    auto c = [](float v) { return make_float2(v, v); };
    const float2 t0 = __fadd2_rn(__ffma2_rn(c(-2.f), f1, f0), f2);
    const float2 s0 = __ffma2_rn(c(3.f), f2, __ffma2_rn(c(-4.f), f1, f0));
    const float2 t1 = __fadd2_rn(__ffma2_rn(c(-2.f), f2, f1), f3);
    const float2 s1 = __ffma2_rn(c(-1.f), f3, f1);
    const float2 t2 = __fadd2_rn(__ffma2_rn(c(-2.f), f3, f2), f4);
    const float2 s2 = __fadd2_rn(__ffma2_rn(c(-4.f), f3, __fmul2_rn(c(3.f), f2)), f4);
    // z = eps + (13/12 t^2 + s^2 / 4)
    const float2 z0 = __fadd2_rn(c(1e-6f), __ffma2_rn(__fmul2_rn(c(13.f / 12.f), t0), t0,
                                                      __fmul2_rn(__fmul2_rn(c(0.25f), s0), s0)));
    const float2 z1 = __fadd2_rn(c(1e-6f), __ffma2_rn(__fmul2_rn(c(13.f / 12.f), t1), t1,
                                                      __fmul2_rn(__fmul2_rn(c(0.25f), s1), s1)));
    const float2 z2 = __fadd2_rn(c(1e-6f), __ffma2_rn(__fmul2_rn(c(13.f / 12.f), t2), t2,
                                                      __fmul2_rn(__fmul2_rn(c(0.25f), s2), s2)));
    const float2 y0 = __fmul2_rn(z0, z0), y1 = __fmul2_rn(z1, z1), y2 = __fmul2_rn(z2, z2);
    // e_k = d_k m_k over the common denominator y0 y1 y2 (see weno5(float))
    const float2 e0 = __fmul2_rn(c(0.1f), __fmul2_rn(y1, y2));
    const float2 e1 = __fmul2_rn(c(0.6f), __fmul2_rn(y0, y2));
    const float2 e2 = __fmul2_rn(c(0.3f), __fmul2_rn(y0, y1));
    const float2 den = __fadd2_rn(__fadd2_rn(e0, e1), e2);
    // integer-coefficient stencils (coefficients summing to exactly 6), 1/6 once
    const float2 P0 = __ffma2_rn(c(11.f), f2, __ffma2_rn(c(-7.f), f1, __fmul2_rn(c(2.f), f0)));
    const float2 P1 = __ffma2_rn(c(2.f), f3, __ffma2_rn(c(5.f), f2, __fmul2_rn(c(-1.f), f1)));
    const float2 P2 = __ffma2_rn(c(-1.f), f4, __ffma2_rn(c(5.f), f3, __fmul2_rn(c(2.f), f2)));
    const float2 num = __ffma2_rn(e2, P2, __ffma2_rn(e1, P1, __fmul2_rn(e0, P0)));
    const float2 inv = make_float2(rcp_approx(den.x), rcp_approx(den.y));
    return __fmul2_rn(__fmul2_rn(num, c(1.f / 6.f)), inv);
}

// The 10 WENO5 reconstructions of one face in the FP32 form, paired as
// (plus q0, plus q1), (plus q2, plus q3), (minus q0, minus q1), (minus q2,
// minus q3) and (plus q4, minus q4). P(m, q) / M(m, q): the plus / minus
// window value (minus already reversed) at position m of component q.
template <class GP, class GM>
__device__ __forceinline__ void weno5_face_x2(GP P, GM M, float face[5]) {
    auto pr = [](float x, float y) { return make_float2(x, y); };
    const float2 p01 = weno5x2(pr(P(0, 0), P(0, 1)), pr(P(1, 0), P(1, 1)), pr(P(2, 0), P(2, 1)),
                               pr(P(3, 0), P(3, 1)), pr(P(4, 0), P(4, 1)));
    const float2 p23 = weno5x2(pr(P(0, 2), P(0, 3)), pr(P(1, 2), P(1, 3)), pr(P(2, 2), P(2, 3)),
                               pr(P(3, 2), P(3, 3)), pr(P(4, 2), P(4, 3)));
    const float2 m01 = weno5x2(pr(M(0, 0), M(0, 1)), pr(M(1, 0), M(1, 1)), pr(M(2, 0), M(2, 1)),
                               pr(M(3, 0), M(3, 1)), pr(M(4, 0), M(4, 1)));
    const float2 m23 = weno5x2(pr(M(0, 2), M(0, 3)), pr(M(1, 2), M(1, 3)), pr(M(2, 2), M(2, 3)),
                               pr(M(3, 2), M(3, 3)), pr(M(4, 2), M(4, 3)));
    const float2 pm4 = weno5x2(pr(P(0, 4), M(0, 4)), pr(P(1, 4), M(1, 4)), pr(P(2, 4), M(2, 4)),
                               pr(P(3, 4), M(3, 4)), pr(P(4, 4), M(4, 4)));
    face[0] = p01.x + m01.x;
    face[1] = p01.y + m01.y;
    face[2] = p23.x + m23.x;
    face[3] = p23.y + m23.y;
    face[4] = pm4.x + pm4.y;
}

// mdcd_hybrid_reconstruction (reconstruction.cpp:151-225).
template <class R>
__device__ __forceinline__ R mdcd_hybrid(const R* s, const R* lin6, R disp, R diss) {
    const R eps_small = R(1e-40);
    R f0 = s[0], f1 = s[1], f2 = s[2], f3 = s[3], f4 = s[4], f5 = s[5];
    const R eps = R(0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4);
    R a1 = fabs(f2 - f1) + fabs(f2 - R(2) * f1 + f0);
    R b1 = fabs(f2 - f3) + fabs(f2 - R(2) * f3 + f4);
    R a2 = fabs(f3 - f2) + fabs(f3 - R(2) * f2 + f1);
    R b2 = fabs(f3 - f4) + fabs(f3 - R(2) * f4 + f5);
    R sai1 = (R(2) * a1 * b1 + eps) / (a1 * a1 + b1 * b1 + eps);
    R sai2 = (R(2) * a2 * b2 + eps) / (a2 * a2 + b2 * b2 + eps);
    R sai = sai2 < sai1 ? sai2 : sai1;
    if (sai > R(0.4)) {
        return lin6[0] * s[0] + lin6[1] * s[1] + lin6[2] * s[2] + lin6[3] * s[3] +
               lin6[4] * s[4] + lin6[5] * s[5];
    }
    R q0 = (R(2) * f0 - R(7) * f1 + R(11) * f2) / R(6.0);
    R q1 = (-f1 + R(5) * f2 + R(2) * f3) / R(6.0);
    R q2 = (R(2) * f2 + R(5) * f3 - f4) / R(6.0);
    R q3 = (R(11) * f3 - R(7) * f4 + R(2) * f5) / R(6.0);
    R d0 = R(1.5) * (disp + diss);
    R d1 = R(0.5) - R(1.5) * (disp - R(3) * diss);
    R d2 = R(0.5) - R(1.5) * (disp + R(3) * diss);
    R d3 = R(1.5) * (disp - diss);
    R t;
    t = f0 - R(2) * f1 + f2; R e0 = t * t; t = f0 - R(4) * f1 + R(3) * f2; R g0 = t * t;
    R beta0 = R(13.0 / 12.0) * e0 + R(0.25) * g0;
    t = f1 - R(2) * f2 + f3; R e1 = t * t; t = f1 - f3; R g1 = t * t;
    R beta1 = R(13.0 / 12.0) * e1 + R(0.25) * g1;
    t = f2 - R(2) * f3 + f4; R e2 = t * t; t = R(3) * f2 - R(4) * f3 + f4; R g2 = t * t;
    R beta2 = R(13.0 / 12.0) * e2 + R(0.25) * g2;
    R beta3 = (R(271799) * (f0 * f0)
        + f0 * (R(-2380800) * f1 + R(4086352) * f2 - R(3462252) * f3 + R(1458762) * f4 - R(245620) * f5)
        + f1 * (R(5653317) * f1 - R(20427884) * f2 + R(17905032) * f3 - R(7727988) * f4 + R(1325006) * f5)
        + f2 * (R(19510972) * f2 - R(35817664) * f3 + R(15929912) * f4 - R(2792660) * f5)
        + f3 * (R(17195652) * f3 - R(15880404) * f4 + R(2863984) * f5)
        + f4 * (R(3824847) * f4 - R(1429976) * f5)
        + R(139633) * (f5 * f5)) / R(120960.0);
    R tau6 = fabs(beta3 - (beta0 + R(4) * beta1 + beta2) / R(6.0));
    t = R(20) + tau6 / (beta0 + eps_small); R aa0 = d0 * (t * t);
    t = R(20) + tau6 / (beta1 + eps_small); R aa1 = d1 * (t * t);
    t = R(20) + tau6 / (beta2 + eps_small); R aa2 = d2 * (t * t);
    t = R(20) + tau6 / (beta3 + eps_small); R aa3 = d3 * (t * t);
    return (aa0 * q0 + aa1 * q1 + aa2 * q2 + aa3 * q3) / (aa0 + aa1 + aa2 + aa3);
}

// One reconstruction of a window s[0..S-1] (already oriented).
template <class R, int RC>
__device__ __forceinline__ R reconstruct(const R* s, const R* lin, R disp, R diss) {
    if constexpr (RC == RC_WENO5) {
        return weno5(s[0], s[1], s[2], s[3], s[4]);
    } else if constexpr (RC == RC_LINEAR) {
        return s[0];  // linear_reconstruction, reconstruction.cpp:88-90
    } else if constexpr (RC == RC_LIN6) {
        return lin[0] * s[0] + lin[1] * s[1] + lin[2] * s[2] + lin[3] * s[3] + lin[4] * s[4] +
               lin[5] * s[5];
    } else if constexpr (RC == RC_MDCD_HYBRID) {
        return mdcd_hybrid(s, lin, disp, diss);
    } else {
        return lin[0] * s[0] + lin[1] * s[1] + lin[2] * s[2] + lin[3] * s[3] + lin[4] * s[4] +
               lin[5] * s[5] + lin[6] * s[6] + lin[7] * s[7];
    }
}

// ---------------------------------------------------------------------------
// Central first derivatives (ViscousFlux.cpp:23-40); periodic => full order.
// f(o) returns the value at offset o along the line.
// ---------------------------------------------------------------------------
template <class R, int ORD, class F>
__device__ __forceinline__ R dcentral(F f, R h) {
    if constexpr (ORD == 4) {
        return (-f(2) + R(8.0) * f(1) - R(8.0) * f(-1) + f(-2)) / (R(12.0) * h);
    } else if constexpr (ORD == 6) {
        return (f(3) - R(9.0) * f(2) + R(45.0) * f(1) - R(45.0) * f(-1) + R(9.0) * f(-2) - f(-3)) /
               (R(60.0) * h);
    } else {
        const R c1 = R(0.8), c2 = R(-0.2), c3 = R(0.0380952380952381), c4 = R(-0.00357142857142857);
        return (c1 * (f(1) - f(-1)) + c2 * (f(2) - f(-2)) + c3 * (f(3) - f(-3)) +
                c4 * (f(4) - f(-4))) / h;
    }
}

// Order-preserving bit pattern of a non-negative double (for atomicMin).
__device__ __forceinline__ unsigned long long pos_double_bits(double x) {
    return (unsigned long long)__double_as_longlong(x);
}

}  // namespace ns3d
