/*
 * ns3d_oracle.c -- CPU restatement of ns3d_cpp's RHS + RK3 time-step loop.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle). Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg use it, and only as the checker. The product
 * (ns3d_cpp_b200/) never links, loads or calls it.
 *
 * Pinned against the reference's own sources compiled here (oracle/_ref, see
 * oracle/Makefile) and against the golden fixtures in tests/golden/ that were
 * generated from that build (tests/golden/make_golden.py).
 *
 * Layout: interior-only periodic box, SoA, x fastest: a[(k*ny + j)*nx + i].
 * The reference stores g ghost layers per side and fills them by a periodic
 * halo exchange of (rho,u,v,w,p) followed by primitiveToConserved
 * (field_structures.h:795-853, range_kutta.cpp:117-119). Every ghost value is
 * then bit-identical to its periodic image, so indexing with wrap-around is the
 * same computation. The corner/edge ghosts the reference never fills are never
 * read by the sweeps (lines run over interior (j,k) only).
 *
 * Floating-point operation order follows the reference expression by
 * expression (no FMA contraction: built with -ffp-contract=off), so FP64
 * results agree with the reference to the last bit or so.
 *
 * State model: the reference carries conserved U and primitives (u,v,w,p,T,c)
 * side by side; after every stage the conserved state is rebuilt from the
 * primitives (primitiveToConserved). Hence U == prim2cons(W) holds at every
 * RHS evaluation and the primitive tuple W = (rho,u,v,w,p) is the whole state.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Enumerations use the reference's enum order (field_structures.h:112-131). */
enum { ORC_SW = 0, ORC_LF = 1 };
enum { ORC_WENO5 = 0, ORC_WCNS = 1, ORC_LINEAR = 2, ORC_MDCD = 3, ORC_MDCD_HYBRID = 4,
       ORC_UPWIND_7TH = 5, ORC_UD7L = 6 };
enum { ORC_C8 = 0, ORC_C6 = 1, ORC_C4 = 2 };

typedef struct orc_params {
    double gamma, Pr, Ma, Re;
    double Cv, Cp, Rgas, mu;     /* derived as initialization.cpp:374-377 */
    double dx, dy, dz;           /* L/N as initialization.cpp:324-326 */
    double mdcd_diss, mdcd_disp, ud7l_alpha;
    double sw_eps;               /* entropy fix; 0 reproduces split_StagerWarming exactly */
    double sutherland_s;         /* S/Tref; 110.4/288.15 as field_structures.h:100 */
    int nx, ny, nz;
    int fvs, recon, vis;
    int mu_variant;              /* 0: pow(T, 1.5) as the reference; 1: T*sqrt(T) (a
                                    1-ulp perturbation, for sensitivity controls) */
    int char_recon;              /* 1: characteristic-wise reconstruction
                                    (du_inviscous_character, InviscousFlux_new.cpp:165-437) */
} orc_params;

#define IDX(i, j, k) (((long)(k) * ny + (j)) * nx + (i))

static inline int wrap(int i, int n) { i %= n; return i < 0 ? i + n : i; }

/* ------------------------------------------------------------------------ */
/* Thermodynamics: field_structures.h:94-105, 405-451                       */
/* ------------------------------------------------------------------------ */

/* SolverParams::get_mu, field_structures.h:94-105 (Sutherland). */
static inline double get_mu(const orc_params *P, double T) {
    double S_ref = P->sutherland_s;
    double t15 = P->mu_variant ? T * sqrt(T) : pow(T, 1.5);
    return P->mu * t15 * (1.0 + S_ref) / (T + S_ref);
}

/* primitiveToConserved, field_structures.h:430-451 (one cell). */
static inline void p2c(const orc_params *P, double rr, double u, double v, double w, double p,
                       double *ru, double *rv, double *rw, double *E, double *T, double *c) {
    const double gamma = P->gamma;
    *ru = rr * u;
    *rv = rr * v;
    *rw = rr * w;
    double kinetic = 0.5 * (u * u + v * v + w * w);
    double e_internal = p / ((gamma - 1.0) * rr);
    *E = rr * (e_internal + kinetic);
    *T = p / (rr * P->Rgas);
    *c = sqrt(gamma * p / rr);
}

/* conservedToPrimitive, field_structures.h:405-427 (one cell, incl. clamp). */
static inline void c2p(const orc_params *P, double *rho, double ru, double rv, double rw, double E,
                       double *u, double *v, double *w, double *p) {
    const double gamma = P->gamma;
    double rr = *rho;
    if (rr <= 0.0) { rr = 1e-12; *rho = rr; }
    *u = ru / rr;
    *v = rv / rr;
    *w = rw / rr;
    double kinetic = 0.5 * (*u * *u + *v * *v + *w * *w);
    double e_internal = E / rr - kinetic;
    *p = (gamma - 1.0) * rr * e_internal;
}

void orc_prim2cons(const orc_params *P, const double *W, double *U, double *T, double *c) {
    const long n = (long)P->nx * P->ny * P->nz;
    for (long q = 0; q < n; ++q) {
        double rr = W[q];
        if (rr <= 0.0) rr = 1e-12;
        U[q] = rr;
        p2c(P, rr, W[n + q], W[2 * n + q], W[3 * n + q], W[4 * n + q], &U[n + q], &U[2 * n + q],
            &U[3 * n + q], &U[4 * n + q], T ? &T[q] : &(double){0}, c ? &c[q] : &(double){0});
    }
}

void orc_cons2prim(const orc_params *P, const double *U, double *W) {
    const long n = (long)P->nx * P->ny * P->nz;
    for (long q = 0; q < n; ++q) {
        double rr = U[q];
        c2p(P, &rr, U[n + q], U[2 * n + q], U[3 * n + q], U[4 * n + q], &W[n + q], &W[2 * n + q],
            &W[3 * n + q], &W[4 * n + q]);
        W[q] = rr;
    }
}

/* ------------------------------------------------------------------------ */
/* Flux vector splitting: InviscousFlux_new.cpp:439-530                     */
/* ------------------------------------------------------------------------ */

/* split_StagerWarming, InviscousFlux_new.cpp:439-489, with the optional
 * entropy fix |lambda| -> sqrt(lambda^2 + eps^2) of README.md:177-180. */
static inline double absfix(double l, double eps) {
    return eps > 0.0 ? sqrt(l * l + eps * eps) : fabs(l);
}

static void split_sw(const orc_params *P, double rho, double u, double v, double w, double E,
                     double p, double c, int n1, int n2, int n3, double Fp[5], double Fm[5]) {
    const double gamma = P->gamma, eps = P->sw_eps;
    double un = u * n1 + v * n2 + w * n3;
    double lambda1 = un - c, lambda2 = un, lambda3 = un + c;
    double a1 = absfix(lambda1, eps), a2 = absfix(lambda2, eps), a3 = absfix(lambda3, eps);
    double lambda1_plus = 0.5 * (lambda1 + a1);
    double lambda1_minus = 0.5 * (lambda1 - a1);
    double lambda2_plus = 0.5 * (lambda2 + a2);
    double lambda2_minus = 0.5 * (lambda2 - a2);
    double lambda3_plus = 0.5 * (lambda3 + a3);
    double lambda3_minus = 0.5 * (lambda3 - a3);
    double S1_p = lambda1_plus + lambda3_plus;
    double S1_m = lambda1_minus + lambda3_minus;
    double S2_p = lambda3_plus - lambda1_plus;
    double S2_m = lambda3_minus - lambda1_minus;
    double H = (E + p) / rho;
    double ga1 = rho / (2.0 * gamma);
    double ga2 = 2.0 * (gamma - 1.0);
    double V = 0.5 * (u * u + v * v + w * w);
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

/* split_LaxFriedrichs, InviscousFlux_new.cpp:491-530 (local wave speed). */
static void split_lf(const orc_params *P, double rho, double u, double v, double w, double E,
                     double p, double c, int n1, int n2, int n3, double Fp[5], double Fm[5]) {
    (void)P;
    double un = u * n1 + v * n2 + w * n3;
    double a_max = fabs(un) + c;
    double F1 = rho * un;
    double F2 = rho * u * un + p * n1;
    double F3 = rho * v * un + p * n2;
    double F4 = rho * w * un + p * n3;
    double F5 = (E + p) * un;
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

/* Split fluxes of one cell state (rho,u,v,w,p) along direction dir. */
void orc_split(const orc_params *P, const double *w5, int dir, double *Fp, double *Fm) {
    double rr = w5[0], ru, rv, rw, E, T, c;
    p2c(P, rr, w5[1], w5[2], w5[3], w5[4], &ru, &rv, &rw, &E, &T, &c);
    if (P->fvs == ORC_SW)
        split_sw(P, rr, w5[1], w5[2], w5[3], E, w5[4], c, dir == 0, dir == 1, dir == 2, Fp, Fm);
    else
        split_lf(P, rr, w5[1], w5[2], w5[3], E, w5[4], c, dir == 0, dir == 1, dir == 2, Fp, Fm);
}

/* ------------------------------------------------------------------------ */
/* Scalar reconstructions: reconstruction.cpp                               */
/* ------------------------------------------------------------------------ */

/* weno5_reconstruction, reconstruction.cpp:93-124 (points 0..4 of 6). */
static double weno5(const double *s) {
    double f0 = s[0], f1 = s[1], f2 = s[2], f3 = s[3], f4 = s[4];
    double eps = 1e-6;
    double beta0 = 13.0 / 12.0 * (f0 - 2 * f1 + f2) * (f0 - 2 * f1 + f2)
                 + 0.25 * (f0 - 4 * f1 + 3 * f2) * (f0 - 4 * f1 + 3 * f2);
    double beta1 = 13.0 / 12.0 * (f1 - 2 * f2 + f3) * (f1 - 2 * f2 + f3)
                 + 0.25 * (f1 - f3) * (f1 - f3);
    double beta2 = 13.0 / 12.0 * (f2 - 2 * f3 + f4) * (f2 - 2 * f3 + f4)
                 + 0.25 * (3 * f2 - 4 * f3 + f4) * (3 * f2 - 4 * f3 + f4);
    double alpha0 = 0.1 / ((eps + beta0) * (eps + beta0));
    double alpha1 = 0.6 / ((eps + beta1) * (eps + beta1));
    double alpha2 = 0.3 / ((eps + beta2) * (eps + beta2));
    double asum = alpha0 + alpha1 + alpha2;
    double w0 = alpha0 / asum, w1 = alpha1 / asum, w2 = alpha2 / asum;
    double p0 = (2 * f0 - 7 * f1 + 11 * f2) / 6.0;
    double p1 = (-f1 + 5 * f2 + 2 * f3) / 6.0;
    double p2 = (2 * f2 + 5 * f3 - f4) / 6.0;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

/* mdcd_reconstruction, reconstruction.cpp:126-135 (linear, 6 points). */
static double mdcd(const orc_params *P, const double *s) {
    double diss = P->mdcd_diss, disp = P->mdcd_disp;
    return (1.0 / 2.0 * disp + 1.0 / 2.0 * diss) * s[0] +
           (-3.0 / 2.0 * disp - 5.0 / 2.0 * diss - 1.0 / 12.0) * s[1] +
           (7.0 / 12.0 + disp + 5.0 * diss) * s[2] +
           (7.0 / 12.0 + disp - 5.0 * diss) * s[3] +
           (-3.0 / 2.0 * disp + 5.0 / 2.0 * diss - 1.0 / 12.0) * s[4] +
           (1.0 / 2.0 * disp - 1.0 / 2.0 * diss) * s[5];
}

/* mdcd_hybrid_reconstruction, reconstruction.cpp:151-225. */
static double mdcd_hybrid(const orc_params *P, const double *s) {
    double diss = P->mdcd_diss, disp = P->mdcd_disp;
    double eps_small = 1e-40;
    double f0 = s[0], f1 = s[1], f2 = s[2], f3 = s[3], f4 = s[4], f5 = s[5];
    double eps = 0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4;
    double a1 = fabs(f2 - f1) + fabs(f2 - 2 * f1 + f0);
    double b1 = fabs(f2 - f3) + fabs(f2 - 2 * f3 + f4);
    double a2 = fabs(f3 - f2) + fabs(f3 - 2 * f2 + f1);
    double b2 = fabs(f3 - f4) + fabs(f3 - 2 * f4 + f5);
    double sai1 = (2 * a1 * b1 + eps) / (a1 * a1 + b1 * b1 + eps);
    double sai2 = (2 * a2 * b2 + eps) / (a2 * a2 + b2 * b2 + eps);
    double sai = sai2 < sai1 ? sai2 : sai1;
    if (sai > 0.4) return mdcd(P, s);
    double q0 = (2 * f0 - 7 * f1 + 11 * f2) / 6.0;
    double q1 = (-f1 + 5 * f2 + 2 * f3) / 6.0;
    double q2 = (2 * f2 + 5 * f3 - f4) / 6.0;
    double q3 = (11 * f3 - 7 * f4 + 2 * f5) / 6.0;
    double d0 = 1.5 * (disp + diss);
    double d1 = 0.5 - 1.5 * (disp - 3 * diss);
    double d2 = 0.5 - 1.5 * (disp + 3 * diss);
    double d3 = 1.5 * (disp - diss);
    double t;
    t = f0 - 2 * f1 + f2; double e0 = t * t; t = f0 - 4 * f1 + 3 * f2; double g0 = t * t;
    double beta0 = 13.0 / 12.0 * e0 + 0.25 * g0;
    t = f1 - 2 * f2 + f3; double e1 = t * t; t = f1 - f3; double g1 = t * t;
    double beta1 = 13.0 / 12.0 * e1 + 0.25 * g1;
    t = f2 - 2 * f3 + f4; double e2 = t * t; t = 3 * f2 - 4 * f3 + f4; double g2 = t * t;
    double beta2 = 13.0 / 12.0 * e2 + 0.25 * g2;
    double beta3 = (271799 * (f0 * f0)
        + f0 * (-2380800 * f1 + 4086352 * f2 - 3462252 * f3 + 1458762 * f4 - 245620 * f5)
        + f1 * (5653317 * f1 - 20427884 * f2 + 17905032 * f3 - 7727988 * f4 + 1325006 * f5)
        + f2 * (19510972 * f2 - 35817664 * f3 + 15929912 * f4 - 2792660 * f5)
        + f3 * (17195652 * f3 - 15880404 * f4 + 2863984 * f5)
        + f4 * (3824847 * f4 - 1429976 * f5)
        + 139633 * (f5 * f5)) / 120960.0;
    double tau6 = fabs(beta3 - (beta0 + 4 * beta1 + beta2) / 6.0);
    t = 20 + tau6 / (beta0 + eps_small); double aa0 = d0 * (t * t);
    t = 20 + tau6 / (beta1 + eps_small); double aa1 = d1 * (t * t);
    t = 20 + tau6 / (beta2 + eps_small); double aa2 = d2 * (t * t);
    t = 20 + tau6 / (beta3 + eps_small); double aa3 = d3 * (t * t);
    return (aa0 * q0 + aa1 * q1 + aa2 * q2 + aa3 * q3) / (aa0 + aa1 + aa2 + aa3);
}

/* UpWind_7th_reconstruction, reconstruction.cpp:227-232 (points 0..6 of 8). */
static double upwind7(const double *s) {
    return (-1.0 / 140.0) * s[0] + (5.0 / 84.0) * s[1] - (101.0 / 420.0) * s[2]
         + (319.0 / 420.0) * s[3] + (107.0 / 210.0) * s[4]
         - (19.0 / 210.0) * s[5] + (1.0 / 105.0) * s[6];
}

/* ud7l_reconstruction, reconstruction.cpp:234-249. */
static double ud7l(const orc_params *P, const double *s) {
    double alpha = P->ud7l_alpha;
    double a0 = -3.0 / 420.0 * alpha - 3.0 / 840.0 * (1.0 - alpha);
    double a1 = 25.0 / 420.0 * alpha + 29.0 / 840.0 * (1.0 - alpha);
    double a2 = -101.0 / 420.0 * alpha - 139.0 / 840.0 * (1.0 - alpha);
    double a3 = 319.0 / 420.0 * alpha + 533.0 / 840.0 * (1.0 - alpha);
    double a4 = 214.0 / 420.0 * alpha + 533.0 / 840.0 * (1.0 - alpha);
    double a5 = -38.0 / 420.0 * alpha - 139.0 / 840.0 * (1.0 - alpha);
    double a6 = 4.0 / 420.0 * alpha + 29.0 / 840.0 * (1.0 - alpha);
    double a7 = (-3.0 / 840.0) * (1.0 - alpha);
    return a0 * s[0] + a1 * s[1] + a2 * s[2] + a3 * s[3]
         + a4 * s[4] + a5 * s[5] + a6 * s[6] + a7 * s[7];
}

/* Stencil width per scheme, initialization.cpp:329-357. */
int orc_stencil(int recon) {
    switch (recon) {
    case ORC_LINEAR: return 2;
    case ORC_UPWIND_7TH: case ORC_UD7L: return 8;
    default: return 6;
    }
}

/* reconstruct_select, reconstruction.cpp:13-85: `flag < 0` reverses the window. */
static double recon_select(const orc_params *P, const double *win, int S, double flag) {
    double a[8];
    for (int m = 0; m < S; ++m) a[m] = flag < 0.0 ? win[S - 1 - m] : win[m];
    switch (P->recon) {
    case ORC_WENO5: return weno5(a);
    case ORC_LINEAR: return a[0];
    case ORC_MDCD: return mdcd(P, a);
    case ORC_MDCD_HYBRID: return mdcd_hybrid(P, a);
    case ORC_UPWIND_7TH: return upwind7(a);
    case ORC_UD7L: return ud7l(P, a);
    default: {   /* reconstruction.cpp:77-84 fallback */
        int mid = S / 2;
        return flag >= 0.0 ? 0.5 * (win[mid] + win[mid - 1]) : 0.5 * (win[mid] + win[mid + 1]);
    }
    }
}

double orc_recon_scalar(const orc_params *P, const double *win, int S, double flag) {
    return recon_select(P, win, S, flag);
}

/* ------------------------------------------------------------------------ */
/* Inviscid face fluxes: du_inviscous, InviscousFlux_new.cpp:4-163           */
/* ------------------------------------------------------------------------ */

/* Roe-averaged state (rho, u, v, w, H) of two primitive states
 * (computeRoeAveragedState_new, InviscousFlux_new.cpp:628-659), same operation order. */
static void roe_state(const orc_params *P, const double *l, const double *r, double *ua) {
    const double g = P->gamma;
    const double EL = l[0] * (0.5 * (l[1] * l[1] + l[2] * l[2] + l[3] * l[3]) + l[4] / ((g - 1.0) * l[0]));
    const double ER = r[0] * (0.5 * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) + r[4] / ((g - 1.0) * r[0]));
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

/* Left and right eigenvector matrices of the Euler flux Jacobian along the
 * unit normal (nx, ny, nz) at the Roe state (build_eigen_matrices_new,
 * InviscousFlux_new.cpp:532-625): same entries, same operation order. */
static void eigen_LR(const orc_params *P, const double *ua, double nx, double ny, double nz,
                     double Lm[5][5], double Rm[5][5]) {
    const double g = P->gamma;
    const double u0 = ua[1], v0 = ua[2], w0 = ua[3], h0 = ua[4];
    const double V = 0.5 * (u0 * u0 + v0 * v0 + w0 * w0);
    const double un = u0 * nx + v0 * ny + w0 * nz;
    const double c = sqrt((g - 1.0) * (h0 - V));
    const double t2 = u0 * nz + v0 * nx + w0 * ny;   /* the two transverse velocities */
    const double t3 = u0 * ny + v0 * nz + w0 * nx;
    Rm[0][0] = 1.0;          Rm[0][1] = 1.0; Rm[0][2] = 0.0; Rm[0][3] = 0.0; Rm[0][4] = 1.0;
    Rm[1][0] = u0 - c * nx;  Rm[1][1] = u0;  Rm[1][2] = nz;  Rm[1][3] = ny;  Rm[1][4] = u0 + c * nx;
    Rm[2][0] = v0 - c * ny;  Rm[2][1] = v0;  Rm[2][2] = nx;  Rm[2][3] = nz;  Rm[2][4] = v0 + c * ny;
    Rm[3][0] = w0 - c * nz;  Rm[3][1] = w0;  Rm[3][2] = ny;  Rm[3][3] = nx;  Rm[3][4] = w0 + c * nz;
    Rm[4][0] = h0 - un * c;  Rm[4][1] = V;   Rm[4][2] = t2;  Rm[4][3] = t3;  Rm[4][4] = h0 + un * c;
    const double chi = 0.5 / c;
    const double K = (g - 1.0) / (c * c);
    const double K1 = K / 2;
    Lm[0][0] = K1 * V + chi * un;  Lm[0][1] = -chi * nx - K1 * u0;  Lm[0][2] = -chi * ny - K1 * v0;
    Lm[0][3] = -chi * nz - K1 * w0;  Lm[0][4] = K1;
    Lm[1][0] = 1.0 - K * V;  Lm[1][1] = K * u0;  Lm[1][2] = K * v0;  Lm[1][3] = K * w0;  Lm[1][4] = -K;
    Lm[2][0] = -t2;  Lm[2][1] = nz;  Lm[2][2] = nx;  Lm[2][3] = ny;  Lm[2][4] = 0.0;
    Lm[3][0] = -t3;  Lm[3][1] = ny;  Lm[3][2] = nz;  Lm[3][3] = nx;  Lm[3][4] = 0.0;
    Lm[4][0] = K1 * V - chi * un;  Lm[4][1] = chi * nx - K1 * u0;  Lm[4][2] = chi * ny - K1 * v0;
    Lm[4][3] = chi * nz - K1 * w0;  Lm[4][4] = K1;
}

/* Face fluxes of direction `dir` (0=x,1=y,2=z) for every line. Output F has
 * 5 blocks of n; F[q*n + idx(cell)] is the flux through the face on the +side
 * of that cell (face i+1/2 for dir x), i.e. the reference's flux_f? at index
 * i_face = i + ng. The face on the -side of cell 0 is that of cell n-1 by
 * periodicity. */
void orc_face_fluxes(const orc_params *P, const double *W, int dir, double *Fout) {
    const int nx = P->nx, ny = P->ny, nz = P->nz;
    const long n = (long)nx * ny * nz;
    const int S = orc_stencil(P->recon);
    const int mid = (S - 1) / 2;
    const int nl[3] = {nx, ny, nz};
    const int len = nl[dir];
    const int n1 = dir == 0, n2 = dir == 1, n3 = dir == 2;
    const int na = dir == 0 ? ny : nx;           /* the two transverse extents */
    const int nb = dir == 2 ? ny : nz;
#pragma omp parallel
    {
        /* cells of the line plus S on each side */
        double *Fp = (double *)malloc(sizeof(double) * 5 * (len + 2 * S));
        double *Fm = (double *)malloc(sizeof(double) * 5 * (len + 2 * S));
#pragma omp for collapse(2) schedule(static)
        for (int b = 0; b < nb; ++b)
            for (int a = 0; a < na; ++a) {
                for (int t = -S; t < len + S; ++t) {
                    int s = wrap(t, len);
                    int i = dir == 0 ? s : a, j = dir == 1 ? s : (dir == 0 ? a : b),
                        k = dir == 2 ? s : b;
                    long id = IDX(i, j, k);
                    double rr = W[id], u = W[n + id], v = W[2 * n + id], w = W[3 * n + id],
                           p = W[4 * n + id];
                    if (rr <= 0.0) rr = 1e-12;
                    double ru, rv, rw, E, T, c;
                    p2c(P, rr, u, v, w, p, &ru, &rv, &rw, &E, &T, &c);
                    double fp[5], fm[5];
                    if (P->fvs == ORC_SW) split_sw(P, rr, u, v, w, E, p, c, n1, n2, n3, fp, fm);
                    else split_lf(P, rr, u, v, w, E, p, c, n1, n2, n3, fp, fm);
                    for (int q = 0; q < 5; ++q) {
                        Fp[5 * (t + S) + q] = fp[q];
                        Fm[5 * (t + S) + q] = fm[q];
                    }
                }
                for (int f = 0; f < len; ++f) {
                    int i = dir == 0 ? f : a, j = dir == 1 ? f : (dir == 0 ? a : b),
                        k = dir == 2 ? f : b;
                    long id = IDX(i, j, k);
                    if (P->char_recon) {
                        /* du_inviscous_character: Roe state of the face's two cells,
                         * windows projected on the left eigenvectors, one
                         * reconstruction per characteristic field, back by R. */
                        const int f1 = wrap(f + 1, len);
                        const long idr = IDX(dir == 0 ? f1 : i, dir == 1 ? f1 : j, dir == 2 ? f1 : k);
                        double wl[5], wr[5], ua[5], Lm[5][5], Rm[5][5], wc[5];
                        for (int q = 0; q < 5; ++q) {
                            wl[q] = W[q * n + id];
                            wr[q] = W[q * n + idr];
                        }
                        roe_state(P, wl, wr, ua);
                        eigen_LR(P, ua, (double)n1, (double)n2, (double)n3, Lm, Rm);
                        for (int q = 0; q < 5; ++q) {
                            double wp[8], wm[8];
                            for (int m = 0; m < S; ++m) {
                                const double *fp = &Fp[5 * (f + (m - mid) + S)];
                                const double *fm = &Fm[5 * (f + (m - mid) + S)];
                                double sp = 0.0, sm = 0.0;
                                for (int r = 0; r < 5; ++r) {
                                    sp += Lm[q][r] * fp[r];
                                    sm += Lm[q][r] * fm[r];
                                }
                                wp[m] = sp;
                                wm[m] = sm;
                            }
                            wc[q] = recon_select(P, wp, S, +1.0) + recon_select(P, wm, S, -1.0);
                        }
                        for (int q = 0; q < 5; ++q) {
                            double sum = 0.0;
                            for (int r = 0; r < 5; ++r) sum += Rm[q][r] * wc[r];
                            Fout[q * n + id] = sum;
                        }
                        continue;
                    }
                    for (int q = 0; q < 5; ++q) {
                        double wp[8], wm[8];
                        for (int m = 0; m < S; ++m) {
                            wp[m] = Fp[5 * (f + (m - mid) + S) + q];
                            wm[m] = Fm[5 * (f + (m - mid) + S) + q];
                        }
                        double plus_face = recon_select(P, wp, S, +1.0);
                        double minus_face = recon_select(P, wm, S, -1.0);
                        Fout[q * n + id] = plus_face + minus_face;
                    }
                }
            }
        free(Fp);
        free(Fm);
    }
}

/* ------------------------------------------------------------------------ */
/* Viscous terms: ViscousFlux.cpp                                           */
/* ------------------------------------------------------------------------ */

/* Central first derivative of a periodic line at offset stride `st`, order
 * 4/6/8 (diff_4th/6th/8th_central, ViscousFlux.cpp:23-40; with periodic
 * neighbours choose_scheme always returns the full order, :45,62,81). */
static inline double dcentral(const double *f, long id, long st, int pos, int len, int order,
                              double h) {
#define F_(o) f[id + (long)(wrap(pos + (o), len) - pos) * st]
    if (order == 4)
        return (-F_(2) + 8.0 * F_(1) - 8.0 * F_(-1) + F_(-2)) / (12.0 * h);
    if (order == 6)
        return (F_(3) - 9.0 * F_(2) + 45.0 * F_(1) - 45.0 * F_(-1) + 9.0 * F_(-2) - F_(-3)) /
               (60.0 * h);
    {
        double c1 = 0.8, c2 = -0.2, c3 = 0.0380952380952381, c4 = -0.00357142857142857;
        return (c1 * (F_(1) - F_(-1)) + c2 * (F_(2) - F_(-2)) + c3 * (F_(3) - F_(-3)) +
                c4 * (F_(4) - F_(-4))) / h;
    }
#undef F_
}

static int vis_order(int vis) { return vis == ORC_C4 ? 4 : vis == ORC_C6 ? 6 : 8; }

/* compute_gradients (ViscousFlux.cpp:240-279) then compute_viscous_flux
 * (:282-339). Output Fv: 12 blocks of n in the order
 * Fv(momx,momy,momz,E), Hv(momx,momy,momz,E), Gv(momx,momy,momz,E). */
void orc_viscous_flux(const orc_params *P, const double *W, double *Fv, double *grad12) {
    const int nx = P->nx, ny = P->ny, nz = P->nz;
    const long n = (long)nx * ny * nz;
    const int ord = vis_order(P->vis);
    const double Pr = P->Pr, Cp = P->Cp;
    double *T = (double *)malloc(sizeof(double) * n);
    for (long q = 0; q < n; ++q) {
        double rr = W[q];
        if (rr <= 0.0) rr = 1e-12;
        T[q] = W[4 * n + q] / (rr * P->Rgas);
    }
    const double *uu = W + n, *vv = W + 2 * n, *ww = W + 3 * n;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long id = IDX(i, j, k);
                double du_dx = dcentral(uu, id, 1, i, nx, ord, P->dx);
                double du_dy = dcentral(uu, id, nx, j, ny, ord, P->dy);
                double du_dz = dcentral(uu, id, (long)nx * ny, k, nz, ord, P->dz);
                double dv_dx = dcentral(vv, id, 1, i, nx, ord, P->dx);
                double dv_dy = dcentral(vv, id, nx, j, ny, ord, P->dy);
                double dv_dz = dcentral(vv, id, (long)nx * ny, k, nz, ord, P->dz);
                double dw_dx = dcentral(ww, id, 1, i, nx, ord, P->dx);
                double dw_dy = dcentral(ww, id, nx, j, ny, ord, P->dy);
                double dw_dz = dcentral(ww, id, (long)nx * ny, k, nz, ord, P->dz);
                double dT_dx = dcentral(T, id, 1, i, nx, ord, P->dx);
                double dT_dy = dcentral(T, id, nx, j, ny, ord, P->dy);
                double dT_dz = dcentral(T, id, (long)nx * ny, k, nz, ord, P->dz);
                if (grad12) {
                    double g[12] = {du_dx, du_dy, du_dz, dv_dx, dv_dy, dv_dz,
                                    dw_dx, dw_dy, dw_dz, dT_dx, dT_dy, dT_dz};
                    for (int q = 0; q < 12; ++q) grad12[q * n + id] = g[q];
                }
                double mu = get_mu(P, T[id]);
                double divU = du_dx + dv_dy + dw_dz;
                double tau_xx = 2.0 * mu * du_dx - (2.0 / 3.0) * mu * divU;
                double tau_yy = 2.0 * mu * dv_dy - (2.0 / 3.0) * mu * divU;
                double tau_zz = 2.0 * mu * dw_dz - (2.0 / 3.0) * mu * divU;
                double tau_xy = mu * (du_dy + dv_dx);
                double tau_xz = mu * (du_dz + dw_dx);
                double tau_yz = mu * (dv_dz + dw_dy);
                double qx = mu * Cp / Pr * dT_dx;
                double qy = mu * Cp / Pr * dT_dy;
                double qz = mu * Cp / Pr * dT_dz;
                double u = uu[id], v = vv[id], w = ww[id];
                Fv[0 * n + id] = tau_xx;
                Fv[1 * n + id] = tau_xy;
                Fv[2 * n + id] = tau_xz;
                Fv[3 * n + id] = u * tau_xx + v * tau_xy + w * tau_xz + qx;
                Fv[4 * n + id] = tau_xy;
                Fv[5 * n + id] = tau_yy;
                Fv[6 * n + id] = tau_yz;
                Fv[7 * n + id] = u * tau_xy + v * tau_yy + w * tau_yz + qy;
                Fv[8 * n + id] = tau_xz;
                Fv[9 * n + id] = tau_yz;
                Fv[10 * n + id] = tau_zz;
                Fv[11 * n + id] = u * tau_xz + v * tau_yz + w * tau_zz + qz;
            }
    free(T);
}

/* ------------------------------------------------------------------------ */
/* compute_rhs, range_kutta.cpp:11-99                                       */
/* ------------------------------------------------------------------------ */

void orc_rhs(const orc_params *P, const double *W, double *rhs) {
    const int nx = P->nx, ny = P->ny, nz = P->nz;
    const long n = (long)nx * ny * nz;
    const int ord = vis_order(P->vis);
    double *FX = (double *)malloc(sizeof(double) * 5 * n);
    double *FY = (double *)malloc(sizeof(double) * 5 * n);
    double *FZ = (double *)malloc(sizeof(double) * 5 * n);
    double *Fv = (double *)malloc(sizeof(double) * 12 * n);
    orc_face_fluxes(P, W, 0, FX);
    orc_face_fluxes(P, W, 1, FY);
    orc_face_fluxes(P, W, 2, FZ);
    orc_viscous_flux(P, W, Fv, NULL);
    const double idx = 1.0 / P->dx, idy = 1.0 / P->dy, idz = 1.0 / P->dz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long id = IDX(i, j, k);
                /* compute_vis_flux, ViscousFlux.cpp:341-386: rhs_m += dx + dy + dz */
                double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                for (int m = 0; m < 4; ++m) {
                    r[m + 1] += dcentral(Fv + (0 + m) * n, id, 1, i, nx, ord, P->dx);
                    r[m + 1] += dcentral(Fv + (4 + m) * n, id, nx, j, ny, ord, P->dy);
                    r[m + 1] += dcentral(Fv + (8 + m) * n, id, (long)nx * ny, k, nz, ord, P->dz);
                }
                long ixm = IDX(wrap(i - 1, nx), j, k), iym = IDX(i, wrap(j - 1, ny), k),
                     izm = IDX(i, j, wrap(k - 1, nz));
                /* range_kutta.cpp:51-98 */
                for (int q = 0; q < 5; ++q) {
                    double fx_r = FX[q * n + id], fx_l = FX[q * n + ixm];
                    double fy_t = FY[q * n + id], fy_b = FY[q * n + iym];
                    double fz_f = FZ[q * n + id], fz_b = FZ[q * n + izm];
                    r[q] += -((fx_r - fx_l) * idx + (fy_t - fy_b) * idy + (fz_f - fz_b) * idz);
                    rhs[q * n + id] = r[q];
                }
            }
    free(FX); free(FY); free(FZ); free(Fv);
}

/* ------------------------------------------------------------------------ */
/* runge_kutta_3, range_kutta.cpp:102-163                                   */
/* ------------------------------------------------------------------------ */

/* One Shu-Osher RK3 step of the primitive state W (5 blocks of n, in/out)
 * with recorded conserved U0 (5 blocks). Returns 0, or 1 + the first interior
 * cell (x fastest) that fails rho>0, p>0, T>0 (range_kutta.cpp:149-162). */
long orc_rk3(const orc_params *P, double *W, const double *U0, double dt) {
    const long n = (long)P->nx * P->ny * P->nz;
    double *rhs = (double *)malloc(sizeof(double) * 5 * n);
    double *U = (double *)malloc(sizeof(double) * 5 * n);
    for (int s = 0; s < 3; ++s) {
        orc_rhs(P, W, rhs);
        orc_prim2cons(P, W, U, NULL, NULL);
        for (int q = 0; q < 5; ++q)
            for (long t = 0; t < n; ++t) {
                long a = q * n + t;
                if (s == 0) U[a] = U0[a] + dt * rhs[a];
                else if (s == 1) U[a] = 0.75 * U0[a] + 0.25 * (U[a] + dt * rhs[a]);
                else U[a] = (1.0 / 3.0) * U0[a] + (2.0 / 3.0) * (U[a] + dt * rhs[a]);
            }
        orc_cons2prim(P, U, W);
    }
    long bad = 0;
    for (long t = 0; t < n; ++t) {
        double rr = W[t], p = W[4 * n + t];
        double T = p / (rr * P->Rgas);
        if (rr <= 0.0 || p <= 0.0 || T <= 0.0) { bad = t + 1; break; }
    }
    free(rhs);
    free(U);
    return bad;
}

/* compute_timestep, timestep.cpp:5-33 (std::min semantics kept). */
double orc_timestep(const orc_params *P, const double *W, double cfl) {
    const long n = (long)P->nx * P->ny * P->nz;
    double dt_local = 1e9;
    for (long t = 0; t < n; ++t) {
        double rho = W[t], u = W[n + t], v = W[2 * n + t], w = W[3 * n + t], p = W[4 * n + t];
        double a = sqrt(P->gamma * p / (rho < 1e-14 ? 1e-14 : rho));
        double dt_x = P->dx / (fabs(u) + a);
        double dt_y = P->dy / (fabs(v) + a);
        double dt_z = P->dz / (fabs(w) + a);
        double m = (dt_z < dt_y) ? dt_z : dt_y;
        m = (m < dt_x) ? m : dt_x;
        dt_local = (m < dt_local) ? m : dt_local;
    }
    return cfl * dt_local;
}

/* compute_total_energy, postprocess.cpp:103-128: sum of 0.5 rho |u|^2 dV. */
double orc_total_energy(const orc_params *P, const double *W) {
    const long n = (long)P->nx * P->ny * P->nz;
    const double cell_vol = P->dx * P->dy * P->dz;
    double s = 0.0;
    for (long t = 0; t < n; ++t) {
        double rho = W[t], u = W[n + t], v = W[2 * n + t], w = W[3 * n + t];
        double kinetic = 0.5 * rho * (u * u + v * v + w * w);
        double eint = 0;
        s += (kinetic + eint) * cell_vol;
    }
    return s;
}

/* Sums of compute_turbulence_statistics, ana_isotropic.cpp:241-255:
 * out = [sum 0.5|u|^2, sum mu(T), sum rho, sum |u|^2, sum u, sum v, sum w,
 *        sum u^2, sum v^2, sum w^2, sum sqrt(gamma Rgas T)]. */
void orc_turb_sums(const orc_params *P, const double *W, double *out) {
    const int nx = P->nx, ny = P->ny;
    const long n = (long)P->nx * P->ny * P->nz;
    const int ord = vis_order(P->vis);
    double s[12] = {0};
    for (long t = 0; t < n; ++t) {
        double rho = W[t], uu = W[n + t], vv = W[2 * n + t], ww = W[3 * n + t], p = W[4 * n + t];
        double T = p / (rho * P->Rgas);
        s[0] += 0.5 * (uu * uu + vv * vv + ww * ww);
        s[1] += get_mu(P, T);
        s[2] += rho;
        s[3] += (uu * uu + vv * vv + ww * ww);
        s[4] += uu; s[5] += vv; s[6] += ww;
        s[7] += uu * uu; s[8] += vv * vv; s[9] += ww * ww;
        s[10] += sqrt(P->gamma * P->Rgas * T);
        /* du/dx of compute_gradients_dudx (ViscousFlux.cpp:389-410), the viscous order */
        const double dudx = dcentral(W + n, t, 1, (int)(t % nx), nx, ord, P->dx);
        s[11] += dudx * dudx;
    }
    (void)ny;
    memcpy(out, s, sizeof(s));
}
