/*
 * CPU ORACLE — test infrastructure only.
 *
 * A plain-C, double-precision restatement of the reference's explicit
 * (symplectic Euler) APIC MPM substep, written to check the CUDA path.  Only
 * tests/, the smoke check and bench.py's CPU-baseline leg load it, and only
 * as a checker: the product path (physbam_b200/csrc) never calls it and
 * fails loudly when its CUDA library is missing.
 *
 * It is pinned against the reference itself: tests/golden/ holds dumps made
 * by oracle/ref_scene.cpp (the reference's MPM_DRIVER compiled from its own
 * sources by oracle/ref.mk), and the CPU tests require this restatement to
 * reproduce them.  Operation order follows the reference wherever that is
 * cheap, so the two agree to a few ulps, not just to a tolerance.
 *
 * Each function cites the reference (paths inside the PhysBAM tree).
 * Matrices are column-major, x[i + d*j], as MATRIX<T,d> stores them
 * (Core/Matrices/MATRIX_3X3.h:115-119).  Grids cover the ghosted domain
 * [-3, G+3)^d with the last index fastest (Core/Math_Tools/RANGE_ITERATOR.h:
 * 110-120), as ARRAY<T,TV_INT> lays them out.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GHOST 3
#define MAXOBJ 32

typedef struct {
    int kind;            /* 0 = RANGE box, 1 = PLANE, 2 = SPHERE */
    int type;            /* 0 = stick, 1 = slip, 2 = separate */
    double friction;
    double a[3], b[3];   /* box: min, max corners;  plane: unit normal, point;  sphere: center, radius */
    /* a moving object (func_frame / func_twist, MPM_COLLISION_OBJECT.cpp:23-71): its frame at the
       substep's start (R0, x0) and end (R1, x1), R column-major d x d, and its twist at the end */
    int moving;
    double R0[9], x0[3], R1[9], x1[3], v[3], w[3];
} oracle_object;

typedef struct {
    int dim;
    int counts[3];
    double dmin[3], dmax[3];
    int model;           /* 0 = COROTATED_FIXED, 1 = NEO_HOOKEAN, 2 = ST_VENANT_KIRCHHOFF_HENCKY_STRAIN */
    double gravity[3];
    int nobj;
    oracle_object obj[MAXOBJ];
    int npen;            /* penalty collision objects (IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES) */
    double pen_stiffness, pen_separation;
    oracle_object pen[MAXOBJ];
    const unsigned char* models;   /* per-particle model (one MPM_FINITE_ELEMENTS per model), or NULL */
} oracle_scene;

/* ------------------------------------------------------------------ */
/* small dense algebra (column-major)                                   */
/* ------------------------------------------------------------------ */
static inline double sqr(double x) { return x * x; }
#define M3(A, i, j) (A)[(i) + 3 * (j)]

static void mat3_mul(const double* A, const double* B, double* C)
{   /* C = A*B ; Core/Matrices/MATRIX_3X3.h operator* */
    double t[9];
    for(int j = 0; j < 3; j++)
        for(int i = 0; i < 3; i++)
            t[i + 3 * j] = A[i] * B[3 * j] + A[i + 3] * B[3 * j + 1] + A[i + 6] * B[3 * j + 2];
    memcpy(C, t, sizeof t);
}

/* Givens vector (a,-b).Normalized(): MATRIX_3X3.cpp:37-41; VECTOR_2D Normalized */
static void givens(double a, double b, double g[2])
{
    double m = sqrt(a * a + b * b);
    if(m) { double s = 1 / m; g[0] = a * s; g[1] = -b * s; }
    else { g[0] = 1; g[1] = 0; }
}
/* rows i,j <- u.x*v+u.y*w, u.x*w-u.y*v : MATRIX_3X3.cpp:44-49 */
static void apply_l(double* A, const double g[2], int i, int j)
{
    for(int c = 0; c < 3; c++) {
        double v = M3(A, i, c), w = M3(A, j, c);
        M3(A, i, c) = g[0] * v + g[1] * w;
        M3(A, j, c) = g[0] * w - g[1] * v;
    }
}
/* columns i,j : MATRIX_3X3.cpp:52-57 */
static void apply_r(double* A, const double g[2], int i, int j)
{
    for(int r = 0; r < 3; r++) {
        double v = M3(A, r, i), w = M3(A, r, j);
        M3(A, r, i) = g[0] * v + g[1] * w;
        M3(A, r, j) = g[0] * w - g[1] * v;
    }
}
static void zero_l(double* U, double* A, int r0, int r1, int c)
{   /* MATRIX_3X3.cpp:60-66 */
    double g[2];
    givens(M3(A, r0, c), M3(A, r1, c), g);
    apply_l(A, g, r1, r0);
    apply_r(U, g, r1, r0);
    M3(A, r1, c) = 0;
}
static void zero_r(double* V, double* A, int c0, int c1, int r)
{   /* MATRIX_3X3.cpp:68-75 */
    double g[2];
    givens(M3(A, r, c0), M3(A, r, c1), g);
    apply_r(A, g, c1, c0);
    apply_r(V, g, c1, c0);
    M3(A, r, c1) = 0;
}
static void zero_chasing(double* U, double* A, double* V)
{   /* MATRIX_3X3.cpp:76-83 */
    zero_l(U, A, 0, 1, 0);
    zero_r(V, A, 1, 2, 0);
    zero_l(U, A, 1, 2, 1);
}
static void swap_col(double* U, int i, int j)
{   /* MATRIX_3X3.cpp:85-91: (u,v) -> (v,-u) */
    for(int r = 0; r < 3; r++) { double u = M3(U, r, i), v = M3(U, r, j); M3(U, r, i) = v; M3(U, r, j) = -u; }
}
static void swap_row(double* U, int i, int j)
{
    for(int c = 0; c < 3; c++) { double u = M3(U, i, c), v = M3(U, j, c); M3(U, i, c) = v; M3(U, j, c) = -u; }
}
static void sv_swap(double* U, double* D, double* V, int i, int j)
{
    swap_col(U, i, j); swap_col(V, i, j);
    double t = D[i]; D[i] = D[j]; D[j] = t;
}
static void flip_sign(double* U, double* D, int i, int j)
{   /* MATRIX_3X3.cpp:107-114 */
    D[i] = -D[i]; D[j] = -D[j];
    for(int r = 0; r < 3; r++) { M3(U, r, i) = -M3(U, r, i); M3(U, r, j) = -M3(U, r, j); }
}
static int argmax3(double a, double b, double c)
{   /* Core/Math_Tools/argmax.h:17-18 */
    return a >= c ? (a >= b ? 0 : 1) : (b >= c ? 1 : 2);
}
static void sort_sv(double* U, double* D, double* V)
{   /* MATRIX_3X3.cpp:115-123 */
    int i = argmax3(fabs(D[0]), fabs(D[1]), fabs(D[2]));
    if(i > 0) sv_swap(U, D, V, 0, i);
    if(fabs(D[1]) < fabs(D[2])) sv_swap(U, D, V, 1, 2);
    if(D[0] < 0) flip_sign(U, D, 0, D[1] < 0 ? 1 : 2);
    else if(D[1] < 0) flip_sign(U, D, 1, 2);
}

/* 2x2 symmetric eigenproblem, SYMMETRIC_MATRIX_2X2.h:364-375.
 * S = (x00, x10, x11); returns eigenvalues l[0] >= l[1] and column-major V. */
static void sym2_eigen(double x00, double x10, double x11, double l[2], double V[4])
{
    double a = .5 * (x00 + x11), b = .5 * (x00 - x11), c = x10;
    double c2 = sqr(c), m = sqrt(sqr(b) + c2), k = x00 * x11 - c2;
    if(a >= 0) { l[0] = a + m; l[1] = l[0] ? k / l[0] : 0; }
    else { l[1] = a - m; l[0] = l[1] ? k / l[1] : 0; }
    if(l[1] > l[0]) { double t = l[0]; l[0] = l[1]; l[1] = t; }
    double v0, v1;
    if(b >= 0) { v0 = m + b; v1 = c; } else { v0 = -c; v1 = b - m; }
    double n = sqrt(v0 * v0 + v1 * v1);
    if(n) { double s = 1 / n; v0 *= s; v1 *= s; } else { v0 = 1; v1 = 0; }
    V[0] = v0; V[1] = v1; V[2] = -v1; V[3] = v0;
}

/* 2x2 SVD via indefinite polar decomposition, MATRIX_2X2.h:313-322.
 * F column-major (x[0..3]); U, V column-major rotations; s[1] may be negative. */
static void svd2(const double* x, double* U, double* s, double* V)
{
    double x03 = x[0] + x[3], cs, sn;
    if(x03 == 0) { cs = 0; sn = 1; }
    else { double t = (x[1] - x[2]) / x03; cs = 1 / sqrt(1 + t * t); sn = t * cs; }
    double Q[4] = {cs, sn, -sn, cs};
    double S00 = Q[0] * x[0] + Q[1] * x[1], S10 = Q[0] * x[2] + Q[1] * x[3], S11 = Q[2] * x[2] + Q[3] * x[3];
    sym2_eigen(S00, S10, S11, s, V);
    if(s[1] < 0 && fabs(s[1]) >= fabs(s[0])) {
        double a = -s[1], b = -s[0];
        s[0] = a; s[1] = b;
        for(int i = 0; i < 4; i++) Q[i] = -Q[i];
        double W[4] = {V[2], V[3], -V[0], -V[1]};
        memcpy(V, W, sizeof W);
    }
    /* U = Q*V */
    U[0] = Q[0] * V[0] + Q[2] * V[1]; U[1] = Q[1] * V[0] + Q[3] * V[1];
    U[2] = Q[0] * V[2] + Q[2] * V[3]; U[3] = Q[1] * V[2] + Q[3] * V[3];
}

static void top_block(double* U, double* B, double* V, double* D)
{   /* MATRIX_3X3.cpp:124-136 */
    double a[4] = {M3(B, 0, 0), M3(B, 1, 0), M3(B, 0, 1), M3(B, 1, 1)}, u[4], d[2], v[4];
    svd2(a, u, d, v);
    apply_r(U, u, 0, 1);
    apply_r(V, v, 0, 1);
    D[0] = d[0]; D[1] = d[1]; D[2] = M3(B, 2, 2);
    sort_sv(U, D, V);
}
static void bot_block(double* U, double* B, double* V, double* D)
{   /* MATRIX_3X3.cpp:138-150 */
    double a[4] = {M3(B, 1, 1), M3(B, 2, 1), M3(B, 1, 2), M3(B, 2, 2)}, u[4], d[2], v[4];
    svd2(a, u, d, v);
    apply_r(U, u, 1, 2);
    apply_r(V, v, 1, 2);
    D[0] = M3(B, 0, 0); D[1] = d[0]; D[2] = d[1];
    sort_sv(U, D, V);
}
static int check_tolerances(double* B, double* U, double* D, double* V, double tau)
{   /* MATRIX_3X3.cpp:152-180 */
    if(fabs(M3(B, 1, 2)) <= tau) { top_block(U, B, V, D); return 1; }
    if(fabs(M3(B, 0, 1)) <= tau) { bot_block(U, B, V, D); return 1; }
    if(fabs(M3(B, 1, 1)) <= tau) {
        double g[2], o[2];
        givens(M3(B, 1, 2), M3(B, 2, 2), g);
        o[0] = -g[1]; o[1] = g[0];          /* VECTOR_2D Orthogonal_Vector: (-y, x) */
        apply_l(B, o, 2, 1);
        apply_r(U, o, 2, 1);
        top_block(U, B, V, D);
        return 1;
    }
    if(fabs(M3(B, 2, 2)) <= tau) {
        zero_r(V, B, 1, 2, 1);
        zero_r(V, B, 0, 2, 0);
        top_block(U, B, V, D);
        return 1;
    }
    if(fabs(M3(B, 0, 0)) <= tau) {
        zero_l(U, B, 1, 0, 1);
        zero_l(U, B, 2, 0, 2);
        bot_block(U, B, V, D);
        return 1;
    }
    return 0;
}
static int lazy_sort(double* U, double* B, double* V, int i, int j)
{   /* MATRIX_3X3.cpp:182-193 */
    if(fabs(M3(B, i, i)) * 100 >= fabs(M3(B, j, j))) return 0;
    swap_row(B, i, j); swap_col(U, i, j); swap_col(B, i, j); swap_col(V, i, j);
    return 1;
}
static void bidiagonalize(double* U, double* B, double* V)
{   /* MATRIX_3X3.cpp:195-200 */
    zero_l(U, B, 1, 2, 0);
    zero_chasing(U, B, V);
}

/* 3x3 SVD, implicit-shift QR (Gast, Fu, Jiang, Teran 2016), MATRIX_3X3.cpp:202-236.
 * U, V rotations; smallest singular value possibly negative.  Returns the
 * iteration count, or -1 if it did not converge in 1000 sweeps (the reference
 * loops without bound). */
int oracle_svd3(const double* F, double* U, double* D, double* V)
{
    double B[9];
    memcpy(B, F, sizeof B);
    for(int i = 0; i < 9; i++) U[i] = V[i] = (i % 4 == 0);
    bidiagonalize(U, B, V);
    double fro = 0;
    for(int i = 0; i < 9; i++) fro += B[i] * B[i];
    double nu = 16 * DBL_EPSILON;
    double tau = nu * fmax(.5 * sqrt(fro), 1.);
    for(int it = 0; it < 1000; it++) {
        if(check_tolerances(B, U, D, V, tau)) return it;
        int ls = lazy_sort(U, B, V, 0, 1);
        ls |= lazy_sort(U, B, V, 0, 2);
        ls |= lazy_sort(U, B, V, 1, 2);
        if(ls) {
            bidiagonalize(U, B, V);
            if(check_tolerances(B, U, D, V, tau)) return it;
        }
        double al0 = M3(B, 0, 0), al1 = M3(B, 1, 1), al2 = M3(B, 2, 2);
        double be0 = M3(B, 0, 1), be1 = M3(B, 1, 2);
        double ga0 = al0 * be0, ga1 = al1 * be1;
        double a0 = al1 * al1 + be0 * be0;
        double a1 = al2 * al2 + be1 * be1;
        double b0 = ga1;
        double d = .5 * (a0 - a1);
        double mu = a1 - b0 * b0 / (d + (d >= 0 ? 1. : -1.) * sqrt(d * d + b0 * b0));
        double g[2];
        givens(al0 * al0 - mu, ga0, g);
        apply_r(B, g, 1, 0);
        apply_r(V, g, 1, 0);
        zero_chasing(U, B, V);
    }
    return -1;
}

/* ------------------------------------------------------------------ */
/* constitutive models on singular values                               */
/* ------------------------------------------------------------------ */
/* COROTATED_FIXED::P_From_Strain, COROTATED_FIXED.cpp:59-65 */
static void corotated_phat(int d, const double* s, double mu, double la, double* P)
{
    double J = d == 2 ? s[0] * s[1] : s[0] * s[1] * s[2];
    double cof[3];
    if(d == 2) { cof[0] = s[1]; cof[1] = s[0]; }
    else { cof[0] = s[1] * s[2]; cof[1] = s[0] * s[2]; cof[2] = s[0] * s[1]; }
    double k = la * (J - 1);
    for(int a = 0; a < d; a++) P[a] = 2 * mu * (s[a] - 1) + k * cof[a];
}

/* NEO_HOOKEAN::Clamp_To_Hyperbola + P_From_Strain, NEO_HOOKEAN.cpp:42-82,
 * failure_threshold .25 (STANDARD_TESTS_BASE.cpp:377-381 via the header default). */
static void neohookean_phat(int d, const double* s, double mu, double la, double* P)
{
    const double ft = .25;
    double J = d == 2 ? s[0] * s[1] : s[0] * s[1] * s[2];
    if(J >= ft) {
        double c = mu - la * log(J);
        for(int a = 0; a < d; a++) P[a] = mu * s[a] - c * (1 / s[a]);
        return;
    }
    double Fc[3];
    if(d == 2) {
        double root = sqrt(ft);
        if(sqr(s[0]) > ft) { Fc[0] = s[0]; Fc[1] = ft / s[0]; }
        else { Fc[0] = Fc[1] = root; }
    } else {
        double root = cbrt(ft);
        if(s[0] * s[1] * s[1] > ft) { Fc[0] = s[0]; Fc[1] = s[1]; Fc[2] = ft / (s[0] * s[1]); }
        else if(s[0] * s[0] * s[0] > ft) { double c = sqrt(ft / s[0]); Fc[0] = s[0]; Fc[1] = Fc[2] = c; }
        else { Fc[0] = Fc[1] = Fc[2] = root; }
    }
    double Fi[3], dF[3], inner = 0;
    for(int a = 0; a < d; a++) { Fi[a] = 1 / Fc[a]; dF[a] = s[a] - Fc[a]; inner += Fi[a] * dF[a]; }
    double c = mu - la * log(ft);
    for(int a = 0; a < d; a++) P[a] = mu * s[a] + c * (sqr(Fi[a]) * dF[a] - Fi[a]) + la * inner * Fi[a];
}

/* ST_VENANT_KIRCHHOFF_HENCKY_STRAIN::P_From_Strain
 * (Deformables/Constitutive_Models/ST_VENANT_KIRCHHOFF_HENCKY_STRAIN.cpp:67-78):
 * Phat = (2 mu ln S + lambda tr(ln S)) S^-1, zero once the smallest signed
 * singular value is <= 0. */
static void hencky_phat(int d, const double* s, double mu, double la, double* P)
{
    if(s[d - 1] <= 0) {
        for(int a = 0; a < d; a++) P[a] = 0;
        return;
    }
    double l[3], tr = 0;
    for(int a = 0; a < d; a++) { l[a] = log(s[a]); tr += l[a]; }
    for(int a = 0; a < d; a++) P[a] = (2 * mu * l[a] + la * tr) / s[a];
}

/* MPM_FINITE_ELEMENTS::Precompute, MPM_FINITE_ELEMENTS.cpp:47-67:
 * PFT = U * Phat(sigma) * (Fn*V)^T with Fn = F (MPM_EXAMPLE::Capture_Stress). */
void oracle_pft(int d, int model, const double* F, double mu, double la, double* PFT)
{
    double U[9], V[9], s[3], P[3];
    if(d == 2) {
        svd2(F, U, s, V);
    } else {
        oracle_svd3(F, U, s, V);
    }
    if(model == 0) corotated_phat(d, s, mu, la, P);
    else if(model == 1) neohookean_phat(d, s, mu, la, P);
    else hencky_phat(d, s, mu, la, P);
    if(d == 2) {
        double FV[4];
        FV[0] = F[0] * V[0] + F[2] * V[1]; FV[1] = F[1] * V[0] + F[3] * V[1];
        FV[2] = F[0] * V[2] + F[2] * V[3]; FV[3] = F[1] * V[2] + F[3] * V[3];
        double PT[4] = {P[0] * FV[0], P[1] * FV[2], P[0] * FV[1], P[1] * FV[3]};   /* diag(P) * FV^T */
        PFT[0] = U[0] * PT[0] + U[2] * PT[1]; PFT[1] = U[1] * PT[0] + U[3] * PT[1];
        PFT[2] = U[0] * PT[2] + U[2] * PT[3]; PFT[3] = U[1] * PT[2] + U[3] * PT[3];
    } else {
        double FV[9], PT[9];
        mat3_mul(F, V, FV);
        for(int i = 0; i < 3; i++)
            for(int j = 0; j < 3; j++) PT[i + 3 * j] = P[i] * FV[j + 3 * i];
        mat3_mul(U, PT, PFT);
    }
}

/* ------------------------------------------------------------------ */
/* collision objects                                                    */
/* ------------------------------------------------------------------ */
/* RANGE::Signed_Distance, Core/Math_Tools/RANGE.cpp:37-45 */
static double box_phi(int d, const oracle_object* o, const double* X)
{
    double phi[3], mx = -DBL_MAX, out = 0;
    int all_le = 1;
    for(int a = 0; a < d; a++) {
        double len = o->b[a] - o->a[a], c = (o->a[a] + o->b[a]) * .5;
        phi[a] = fabs(X[a] - c) - .5 * len;
        if(!(phi[a] <= 0)) all_le = 0;
        if(phi[a] > mx) mx = phi[a];
    }
    if(!all_le) {
        for(int a = 0; a < d; a++) { double p = phi[a] > 0 ? phi[a] : 0; out += p * p; }
        return sqrt(out);
    }
    return mx;
}
/* RANGE::Normal, Core/Math_Tools/RANGE.cpp:49-63 */
static void box_normal(int d, const oracle_object* o, const double* X, double* n)
{
    int inside = 1;
    for(int a = 0; a < d; a++) if(!(X[a] >= o->a[a] && X[a] <= o->b[a])) inside = 0;
    double pmax[3], pmin[3];
    for(int a = 0; a < d; a++) { pmax[a] = X[a] - o->b[a]; pmin[a] = o->a[a] - X[a]; }
    if(inside) {
        double m[3];
        for(int a = 0; a < d; a++) m[a] = pmin[a] > pmax[a] ? pmin[a] : pmax[a];
        int ax = d == 2 ? (m[0] >= m[1] ? 0 : 1) : argmax3(m[0], m[1], m[2]);
        for(int a = 0; a < d; a++) n[a] = 0;
        n[ax] = pmax[ax] > pmin[ax] ? 1 : -1;
        return;
    }
    double mag = 0;
    for(int a = 0; a < d; a++) {
        double p = pmin[a] > pmax[a] ? pmin[a] : pmax[a];
        n[a] = p > 0 ? (pmax[a] > pmin[a] ? p : -p) : 0;
        mag += n[a] * n[a];
    }
    mag = sqrt(mag);
    if(mag) { double s = 1 / mag; for(int a = 0; a < d; a++) n[a] *= s; }
    else { for(int a = 0; a < d; a++) n[a] = a == 0; }
}
static double obj_phi(int d, const oracle_object* o, const double* X)
{
    if(o->kind == 0) return box_phi(d, o, X);
    if(o->kind == 2) {   /* SPHERE::Signed_Distance, Geometry/Basic_Geometry/SPHERE.h:59-60 */
        double r2 = 0;
        for(int a = 0; a < d; a++) r2 += (X[a] - o->a[a]) * (X[a] - o->a[a]);
        return sqrt(r2) - o->b[0];
    }
    double s = 0;  /* PLANE::Signed_Distance, Geometry/Basic_Geometry/PLANE.h:62-63 */
    for(int a = 0; a < d; a++) s += o->a[a] * (X[a] - o->b[a]);
    return s;
}
static void obj_normal(int d, const oracle_object* o, const double* X, double* n)
{
    if(o->kind == 0) { box_normal(d, o, X, n); return; }
    if(o->kind == 2) {   /* SPHERE::Normal: (X - center).Normalized() */
        double mag = 0;
        for(int a = 0; a < d; a++) { n[a] = X[a] - o->a[a]; mag += n[a] * n[a]; }
        mag = sqrt(mag);
        if(mag) { double s = 1 / mag; for(int a = 0; a < d; a++) n[a] *= s; }
        else { for(int a = 0; a < d; a++) n[a] = a == 0; }
        return;
    }
    for(int a = 0; a < d; a++) n[a] = o->a[a];
}

/* MPM_COLLISION_OBJECT::Phi / Normal / Velocity (MPM_COLLISION_OBJECT.cpp:23-71):
 * a moving object is evaluated in its own frame, Z = R^T (X - x). */
static void obj_local(int d, const oracle_object* o, int end, const double* X, double* Z)
{
    const double* R = end ? o->R1 : o->R0;
    const double* x = end ? o->x1 : o->x0;
    for(int c = 0; c < d; c++) {
        double z = 0;
        for(int a = 0; a < d; a++) z += R[a + d * c] * (X[a] - x[a]);
        Z[c] = z;
    }
}
static double obj_phi_at(int d, const oracle_object* o, int end, const double* X)
{
    if(!o->moving) return obj_phi(d, o, X);
    double Z[3];
    obj_local(d, o, end, X, Z);
    return obj_phi(d, o, Z);
}
static void obj_normal_at(int d, const oracle_object* o, const double* X, double* n)
{
    if(!o->moving) { obj_normal(d, o, X, n); return; }
    double Z[3], nl[3];
    obj_local(d, o, 1, X, Z);
    obj_normal(d, o, Z, nl);
    for(int r = 0; r < d; r++) {
        double s = 0;
        for(int c = 0; c < d; c++) s += o->R1[r + d * c] * nl[c];
        n[r] = s;
    }
}
static void obj_velocity_at(int d, const oracle_object* o, const double* X, double* V)
{
    double r[3];
    if(!o->moving) { for(int a = 0; a < d; a++) V[a] = 0; return; }
    for(int a = 0; a < d; a++) r[a] = X[a] - o->x1[a];
    if(d == 3) {
        V[0] = o->v[0] + (o->w[1] * r[2] - o->w[2] * r[1]);
        V[1] = o->v[1] + (o->w[2] * r[0] - o->w[0] * r[2]);
        V[2] = o->v[2] + (o->w[0] * r[1] - o->w[1] * r[0]);
    } else {
        V[0] = o->v[0] + -o->w[0] * r[1];
        V[1] = o->v[1] + o->w[0] * r[0];
    }
}

/* The force of the penalty collision objects on a particle at X, one
 * IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES per object in order
 * (Deformables/Collisions_And_Interactions/IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES.cpp:49-60,
 * 82-85): where phi <= separation, x = separation - phi, a = k x^2,
 * grad pe = -3 a n and F -= grad pe. */
static void penalty_force(const oracle_scene* sc, const double* X, double* f)
{
    const int d = sc->dim;
    for(int j = 0; j < sc->npen; j++) {
        const oracle_object* o = sc->pen + j;
        double phi = obj_phi(d, o, X);
        if(phi > sc->pen_separation) continue;
        double n[3];
        obj_normal(d, o, X, n);
        double x = sc->pen_separation - phi, a = sc->pen_stiffness * x * x;
        for(int c = 0; c < d; c++) f[c] -= -3 * a * n[c];
    }
}

/* ------------------------------------------------------------------ */
/* the substep                                                          */
/* ------------------------------------------------------------------ */
typedef struct {
    int base[3];
    double w[3][3], dw[3][3];      /* [stencil offset][axis] */
} weights_t;

/* PARTICLE_GRID_WEIGHTS_SPLINE<TV,2>::Compute_Precompute_Data + Compute_Weights,
 * PARTICLE_GRID_WEIGHTS_SPLINE.cpp:93-105,133-139; GRID::Cell/Center, Grid_Tools/Grids/GRID.h:123,189-190 */
static void spline_weights(const oracle_scene* sc, const double* dX, const double* inv, const double* X, weights_t* W)
{
    for(int a = 0; a < sc->dim; a++) {
        double y = X[a] - dX[a];   /* X - .5*degree*DX */
        W->base[a] = (int)floor((y - sc->dmin[a]) * inv[a]);
        double c = sc->dmin[a] + ((double)W->base[a] + .5) * dX[a];
        double x = (X[a] - c) * inv[a];
        W->w[0][a] = .5 * sqr(x - 1.5);
        W->dw[0][a] = (x - 1.5) * inv[a];
        x -= 1;
        W->w[1][a] = -x * x + .75;
        W->dw[1][a] = -2 * x * inv[a];
        x -= 1;
        W->w[2][a] = .5 * sqr(x + 1.5);
        W->dw[2][a] = (x + 1.5) * inv[a];
    }
}

typedef struct { int idx; double w; double g[3]; double Z[3]; } node_t;

/* PARTICLE_GRID_WEIGHTS_SPLINE::Compute, PARTICLE_GRID_WEIGHTS_SPLINE.cpp:33-56:
 * tensor-product weights and gradients in RANGE_ITERATOR order (last axis fastest). */
static int stencil(const oracle_scene* sc, const double* dX, const weights_t* W, const int* gs, node_t* out)
{
    int d = sc->dim, k = 0;
    int n2 = d == 3 ? 3 : 1;
    for(int i = 0; i < 3; i++)
        for(int j = 0; j < 3; j++)
            for(int l = 0; l < n2; l++) {
                int off[3] = {i, j, l};
                int idx[3];
                double all_w[3];
                for(int a = 0; a < d; a++) { idx[a] = W->base[a] + off[a]; all_w[a] = W->w[off[a]][a]; }
                double w = all_w[0] * all_w[1];
                if(d == 3) w *= all_w[2];
                double g[3] = {1, 1, 1};
                for(int jj = 0; jj < d; jj++) {
                    double dj = W->dw[off[jj]][jj];
                    for(int ii = 0; ii < d; ii++) g[ii] *= ii == jj ? dj : all_w[jj];
                }
                int flat = 0;
                for(int a = 0; a < d; a++) {
                    int c = idx[a] + GHOST;
                    if(c < 0 || c >= gs[a]) return -1;
                    flat = flat * gs[a] + c;
                }
                out[k].idx = flat;
                out[k].w = w;
                for(int a = 0; a < d; a++) {
                    out[k].g[a] = g[a];
                    out[k].Z[a] = sc->dmin[a] + ((double)idx[a] + .5) * dX[a];
                }
                k++;
            }
    return k;
}

/*
 * One substep, MPM_DRIVER::Advance_One_Time_Step (MPM_DRIVER.cpp:141-157) with
 * use_symplectic_euler, use_affine, flip=0, quadratic weights, no reflection
 * boundaries and no plasticity.
 *
 * X, V (n*d), F, B (n*d*d column-major) are updated in place; valid (n bytes)
 * is cleared for particles that leave the domain.  The grid outputs are
 * optional ((G+6)^d nodes each; NULL = not wanted): mass and velocity after
 * P2G, velocity and friction velocity after the forces.
 * Returns 0, or -1 on a stencil outside the ghosted grid, -2 on allocation failure.
 */
int oracle_substep(const oracle_scene* sc, long long n, double* X, double* V, double* F, double* B,
    const double* mass, const double* vol, const double* mu, const double* la, unsigned char* valid,
    double dt, double time, double* out_m, double* out_v0, double* out_v, double* out_vf)
{
    const int d = sc->dim, dd = d * d;
    int gs[3] = {1, 1, 1};
    long long gn = 1;
    double dX[3], inv[3];
    for(int a = 0; a < d; a++) {
        gs[a] = sc->counts[a] + 2 * GHOST;
        gn *= gs[a];
        dX[a] = (sc->dmax[a] - sc->dmin[a]) / sc->counts[a];   /* GRID::Initialize, GRID.cpp:23-24 */
        inv[a] = 1 / dX[a];
    }
    int rc = 0;
    double* gm = calloc(gn, sizeof(double));
    double* gv = calloc(gn * d, sizeof(double));      /* velocity (momentum, then v) */
    double* gv0 = calloc(gn * d, sizeof(double));     /* velocity_save == objective v0 */
    double* gf = calloc(gn * d, sizeof(double));      /* force, then dv */
    double* gvf = calloc(gn * d, sizeof(double));     /* velocity_friction_save */
    double* dvb = calloc(gn * d, sizeof(double));     /* tmp1: dv before collisions */
    double* v1 = calloc(gn * d, sizeof(double));
    unsigned char* coll = calloc(gn, 1);
    long long* simulated = malloc(sizeof(long long) * (n ? n : 1));
    weights_t* W = malloc(sizeof(weights_t) * (n ? n : 1));
    double* PFT = malloc(sizeof(double) * dd * (n ? n : 1));
    /* per-node collision records, in object order, for Apply_Friction */
    int* ncol = calloc(gn, sizeof(int));
    int* cobj = malloc(sizeof(int) * gn * (sc->nobj ? sc->nobj : 1));
    double* cn = malloc(sizeof(double) * gn * (sc->nobj ? sc->nobj : 1) * 3);
    unsigned char* stuck = calloc(gn, 1);
    double* sv = calloc(gn * d, sizeof(double));      /* stuck_velocity */
    if(!sv || !gm || !gv || !gv0 || !gf || !gvf || !dvb || !v1 || !coll || !simulated || !W || !PFT || !ncol || !cobj || !cn || !stuck) {
        rc = -2; goto done;
    }
    node_t nodes[27];

    /* Update_Simulated_Particles, MPM_DRIVER.cpp:1142-1157 */
    long long ns = 0;
    for(long long p = 0; p < n; p++) if(valid[p]) simulated[ns++] = p;

    /* Update_Particle_Weights (MPM_DRIVER.cpp:233-241): all particles */
    for(long long p = 0; p < n; p++) spline_weights(sc, dX, inv, X + p * d, W + p);
    double Dp_inv[3];
    for(int a = 0; a < d; a++) Dp_inv[a] = 4 * inv[a] * inv[a];   /* Dp_Inverse_Helper, l.152-158 */

    /* Particle_To_Grid, MPM_DRIVER.cpp:245-306 (serial scatter order) */
    for(long long k = 0; k < ns; k++) {
        long long p = simulated[k];
        int nn = stencil(sc, dX, W + p, gs, nodes);
        if(nn < 0) { rc = -1; goto done; }
        const double* Xp = X + p * d;
        const double* Bp = B + p * dd;
        for(int q = 0; q < nn; q++) {
            double w = nodes[q].w;
            int i = nodes[q].idx;
            gm[i] += w * mass[p];
            double Vn[3], Y[3], BY[3];
            for(int a = 0; a < d; a++) Vn[a] = w * V[p * d + a];
            for(int a = 0; a < d; a++) Y[a] = (nodes[q].Z[a] - Xp[a]) * Dp_inv[a];
            for(int a = 0; a < d; a++) {
                double s = 0;
                for(int c = 0; c < d; c++) s += Bp[a + d * c] * Y[c];
                BY[a] = s;
            }
            for(int a = 0; a < d; a++) Vn[a] += BY[a] * w;
            for(int a = 0; a < d; a++) gv[(long long)i * d + a] += mass[p] * Vn[a];
        }
    }
    for(long long i = 0; i < gn; i++) {
        if(gm[i] != 0) {
            for(int a = 0; a < d; a++) {
                double v = gv[i * d + a] / gm[i];
                gv[i * d + a] = v;
                gv0[i * d + a] = v;
            }
        } else for(int a = 0; a < d; a++) gv[i * d + a] = 0;
    }
    if(out_m) memcpy(out_m, gm, sizeof(double) * gn);
    if(out_v0) memcpy(out_v0, gv0, sizeof(double) * gn * d);

    /* Apply_Forces, symplectic branch, MPM_DRIVER.cpp:959-1023 */
    if(sc->npen) {   /* Apply_Particle_Forces, l.933-945: the penalty objects' particle forces, scattered */
        for(long long k = 0; k < ns; k++) {
            long long p = simulated[k];
            double fp[3] = {0, 0, 0};
            penalty_force(sc, X + p * d, fp);
            int nn = stencil(sc, dX, W + p, gs, nodes);
            for(int q = 0; q < nn; q++) {
                long long i = nodes[q].idx;
                for(int a = 0; a < d; a++) gf[i * d + a] += nodes[q].w * fp[a];
            }
        }
    }
    for(long long k = 0; k < ns; k++) {       /* MPM_FINITE_ELEMENTS::Precompute */
        long long p = simulated[k];
        oracle_pft(d, sc->models ? sc->models[p] : sc->model, F + p * dd, mu[p], la[p], PFT + p * dd);
    }
    for(long long k = 0; k < ns; k++) {       /* MPM_FINITE_ELEMENTS::Add_Forces, l.84-99 */
        long long p = simulated[k];
        double A[9];
        for(int e = 0; e < dd; e++) A[e] = PFT[p * dd + e] * vol[p];
        int nn = stencil(sc, dX, W + p, gs, nodes);
        for(int q = 0; q < nn; q++) {
            long long i = nodes[q].idx;
            for(int a = 0; a < d; a++) {
                double s = 0;
                for(int c = 0; c < d; c++) s += A[a + d * c] * nodes[q].g[c];
                gf[i * d + a] -= s;
            }
        }
    }
    for(long long k = 0; k < ns; k++) {       /* MPM_GRAVITY::Add_Forces, MPM_GRAVITY.cpp:62-68 */
        long long p = simulated[k];
        int nn = stencil(sc, dX, W + p, gs, nodes);
        for(int q = 0; q < nn; q++) {
            long long i = nodes[q].idx;
            double wm = nodes[q].w * mass[p];
            for(int a = 0; a < d; a++) gf[i * d + a] += wm * sc->gravity[a];
        }
    }
    double t1 = time + dt;
    for(long long i = 0; i < gn; i++) {
        if(gm[i] == 0) continue;
        double* dv = gf + i * d;
        double s = dt / gm[i];
        for(int a = 0; a < d; a++) { dv[a] = s * dv[a]; dvb[i * d + a] = dv[a]; }
        /* MPM_OBJECTIVE::Adjust_For_Collision + Test_Add_Collision, MPM_OBJECTIVE.cpp:150-225 */
        int idx[3];
        long long r = i;
        for(int a = d - 1; a >= 0; a--) { idx[a] = (int)(r % gs[a]) - GHOST; r /= gs[a]; }
        double X0[3];
        for(int a = 0; a < d; a++) X0[a] = sc->dmin[a] + ((double)idx[a] + .5) * dX[a];
        for(int j = 0; j < sc->nobj; j++) {
            const oracle_object* o = sc->obj + j;
            double Vn[3], Xn[3], nrm[3];
            for(int a = 0; a < d; a++) { Vn[a] = gv0[i * d + a] + dv[a]; Xn[a] = X0[a] + dt * Vn[a]; }
            double phi0 = obj_phi_at(d, o, 0, X0);
            double phi = obj_phi_at(d, o, 1, Xn) - fmin(phi0, 0.);
            if(o->type == 0 && phi0 > 0) continue;
            if(o->type == 1 && phi0 > 0) continue;
            if(o->type == 2 && phi > 1e-15) continue;
            if(o->type != 0 && phi > FLT_MAX) continue;
            obj_normal_at(d, o, Xn, nrm);
            int c = ncol[i]++;
            cobj[i * sc->nobj + c] = j;
            for(int a = 0; a < d; a++) cn[(i * sc->nobj + c) * 3 + a] = nrm[a];
            for(int a = 0; a < d; a++) Xn[a] -= phi * nrm[a];
            for(int a = 0; a < d; a++) Vn[a] = (Xn[a] - X0[a]) / dt;
            if(o->type == 0) {   /* at the object's velocity (stuck_velocity) */
                obj_velocity_at(d, o, Xn, Vn);
                for(int a = 0; a < d; a++) sv[i * d + a] = Vn[a];
                stuck[i] = 1;
            }
            for(int a = 0; a < d; a++) dv[a] = Vn[a] - gv0[i * d + a];
        }
        (void)t1;
    }
    /* Apply_Friction, MPM_DRIVER.cpp:1064-1094 */
    for(long long i = 0; i < gn; i++) {
        if(gm[i] == 0) continue;
        for(int a = 0; a < d; a++) gvf[i * d + a] = gf[i * d + a];
    }
    if(sc->nobj) {
        for(long long i = 0; i < gn; i++) {
            if(gm[i] == 0) continue;
            for(int a = 0; a < d; a++) v1[i * d + a] = gv0[i * d + a] + gf[i * d + a];
            if(stuck[i]) for(int a = 0; a < d; a++) v1[i * d + a] = 0;
            for(int c = 0; c < ncol[i]; c++) {
                const oracle_object* o = sc->obj + cobj[i * sc->nobj + c];
                const double* nrm = cn + (i * sc->nobj + c) * 3;
                double* v = v1 + i * d;
                double nf = 0, vn = 0, t[3], tm = 0;
                for(int a = 0; a < d; a++) nf += nrm[a] * (gf[i * d + a] - dvb[i * d + a]);
                for(int a = 0; a < d; a++) vn += v[a] * nrm[a];
                for(int a = 0; a < d; a++) { t[a] = v[a] - vn * nrm[a]; tm += t[a] * t[a]; }
                tm = sqrt(tm);
                if(tm) { double s = 1 / tm; for(int a = 0; a < d; a++) t[a] *= s; }
                else for(int a = 0; a < d; a++) t[a] = a == 0;
                double kf = o->friction * nf;
                if(tm <= kf) { double vv = 0; for(int a = 0; a < d; a++) vv += v[a] * nrm[a]; for(int a = 0; a < d; a++) v[a] = vv * nrm[a]; }
                else for(int a = 0; a < d; a++) v[a] -= kf * t[a];
                for(int a = 0; a < d; a++) gvf[i * d + a] = v[a] - gv0[i * d + a];
            }
        }
    }
    /* final assembly, MPM_DRIVER.cpp:1050-1056 */
    for(long long i = 0; i < gn; i++) {
        if(gm[i] == 0) continue;
        for(int a = 0; a < d; a++) {
            gv[i * d + a] = gf[i * d + a] + gv0[i * d + a];
            gvf[i * d + a] += gv0[i * d + a];
        }
        if(stuck[i]) for(int a = 0; a < d; a++) gvf[i * d + a] = sv[i * d + a];
    }
    if(out_v) memcpy(out_v, gv, sizeof(double) * gn * d);
    if(out_vf) memcpy(out_vf, gvf, sizeof(double) * gn * d);

    /* Grid_To_Particle, MPM_DRIVER.cpp:450-515 */
    double eps[3], lo[3], hi[3];
    for(int a = 0; a < d; a++) {
        eps[a] = DBL_EPSILON * 4 * (sc->dmax[a] - sc->dmin[a]);
        lo[a] = sc->dmin[a] + eps[a];
        hi[a] = sc->dmax[a] - eps[a];
    }
    for(long long k = 0; k < ns; k++) {
        long long p = simulated[k];
        double Vpic[3] = {0, 0, 0}, Vpf[3] = {0, 0, 0}, G[9] = {0}, Bh[9] = {0};
        int nn = stencil(sc, dX, W + p, gs, nodes);
        for(int q = 0; q < nn; q++) {
            long long i = nodes[q].idx;
            double w = nodes[q].w;
            const double* vn = gv + i * d;
            const double* vf = gvf + i * d;
            for(int a = 0; a < d; a++) { Vpic[a] += w * vn[a]; Vpf[a] += w * vf[a]; }
            for(int c = 0; c < d; c++) for(int a = 0; a < d; a++) G[a + d * c] += vn[a] * nodes[q].g[c];
            double Zp[3], Zm[3];
            for(int a = 0; a < d; a++) {
                double xi = nodes[q].Z[a] + dt * vn[a];
                Zp[a] = nodes[q].Z[a] + xi;
                Zm[a] = nodes[q].Z[a] - xi;
            }
            double hw = w / 2;
            for(int c = 0; c < d; c++) for(int a = 0; a < d; a++)
                Bh[a + d * c] += hw * (vf[a] * Zp[c] + Zm[a] * vf[c]);
        }
        double* Fp = F + p * dd;
        double A[9], Fn[9];
        for(int e = 0; e < dd; e++) A[e] = dt * G[e];
        for(int a = 0; a < d; a++) A[a + d * a] += 1;
        for(int c = 0; c < d; c++) for(int a = 0; a < d; a++) {
            double s = 0;
            for(int e = 0; e < d; e++) s += A[a + d * e] * Fp[e + d * c];
            Fn[a + d * c] = s;
        }
        memcpy(Fp, Fn, sizeof(double) * dd);
        double* Xp = X + p * d;
        double xn[3];
        for(int a = 0; a < d; a++) xn[a] = Xp[a] + dt * Vpic[a];
        double* Bp = B + p * dd;
        for(int c = 0; c < d; c++) for(int a = 0; a < d; a++)
            Bp[a + d * c] = Bh[a + d * c] - .5 * (Vpf[a] * (Xp[c] + xn[c]) + (Xp[a] - xn[a]) * Vpf[c]);
        for(int a = 0; a < d; a++) { Xp[a] = xn[a]; V[p * d + a] = Vpf[a]; }
        /* Reflect_Or_Invalidate_Particle, MPM_DRIVER.cpp:1219-1239 (all sides free) */
        for(int a = 0; a < d; a++) {
            if(Xp[a] < lo[a]) valid[p] = 0;
            else if(Xp[a] > hi[a]) valid[p] = 0;
        }
    }
done:
    free(gm); free(gv); free(gv0); free(gf); free(gvf); free(dvb); free(v1); free(coll);
    free(simulated); free(W); free(PFT); free(ncol); free(cobj); free(cn); free(stuck); free(sv);
    return rc;
}

/* Runs nsteps substeps; used by the CPU baseline and the multi-step parity tests. */
int oracle_run(const oracle_scene* sc, long long n, double* X, double* V, double* F, double* B,
    const double* mass, const double* vol, const double* mu, const double* la, unsigned char* valid,
    double dt, double time, int nsteps)
{
    for(int s = 0; s < nsteps; s++) {
        int rc = oracle_substep(sc, n, X, V, F, B, mass, vol, mu, la, valid, dt, time + s * dt, 0, 0, 0, 0);
        if(rc) return rc;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* plasticity                                                           */
/* ------------------------------------------------------------------ */
static double det_cm(int d, const double* A)
{
    if(d == 2) return A[0] * A[3] - A[2] * A[1];
    return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) + A[6] * (A[1] * A[5] - A[4] * A[2]);
}

/* C = A B, column-major d x d */
static void mul_cm(int d, const double* A, const double* B, double* C)
{
    for(int c = 0; c < d; c++)
        for(int r = 0; r < d; r++) {
            double s = 0;
            for(int k = 0; k < d; k++) s += A[r + d * k] * B[k + d * c];
            C[r + d * c] = s;
        }
}

/* MPM_PLASTICITY_MODEL::Update_Particles (Hybrid_Methods/Forces/MPM_PLASTICITY_MODEL.cpp:35-49)
 * with MPM_PLASTICITY_CLAMP::Compute (Hybrid_Methods/Forces/MPM_PLASTICITY_CLAMP.cpp:28-45),
 * after G2P over the particles simulated in the substep (`valid` holds their
 * validity at its start).  prm = theta_c, theta_s, max_hardening,
 * hardening_factor.  F, Fp column-major per particle. */
void oracle_plastic_clamp(int d, long long n, double* F, double* Fp, double* mu, double* la,
    const double* mu0, const double* la0, const unsigned char* valid, const double* prm)
{
    const double lo = 1 - prm[0], hi = 1 + prm[1];
    const int dd = d * d;
    for(long long p = 0; p < n; p++) {
        if(!valid[p]) continue;
        double* Fe = F + p * dd;
        double U[9], S[3], V[9];
        if(d == 3) oracle_svd3(Fe, U, S, V);
        else svd2(Fe, U, S, V);
        double st[3];
        int same = 1;
        for(int a = 0; a < d; a++) {
            st[a] = S[a] < lo ? lo : (S[a] > hi ? hi : S[a]);
            if(st[a] != S[a]) same = 0;
        }
        if(same) continue;
        /* hardening from det of the new Fp: det(Fe) / det(strain) * det(Fp) */
        double pf = 1, ps = 1;
        for(int a = 0; a < d; a++) { pf *= S[a]; ps *= st[a]; }
        double det = pf / ps * det_cm(d, Fp + p * dd);
        double e = prm[3] * (1 - det);
        double coeff = exp(e < prm[2] ? e : prm[2]);
        if(coeff < 1e-8) coeff = 1e-8;
        mu[p] = mu0[p] * coeff;
        la[p] = la0[p] * coeff;
        /* F = U strain V^T;  Fp = V strain^-1 U^T Fe Fp */
        double Us[9], Vi[9], Fn[9], T1[9], T2[9], Fe0[9];
        memcpy(Fe0, Fe, dd * sizeof(double));
        for(int c = 0; c < d; c++)
            for(int r = 0; r < d; r++) { Us[r + d * c] = U[r + d * c] * st[c]; Vi[r + d * c] = V[r + d * c] / st[c]; }
        for(int c = 0; c < d; c++)
            for(int r = 0; r < d; r++) {
                double s = 0, t = 0;
                for(int k = 0; k < d; k++) { s += Us[r + d * k] * V[c + d * k]; t += Vi[r + d * k] * U[c + d * k]; }
                Fn[r + d * c] = s;
                T1[r + d * c] = t;
            }
        mul_cm(d, T1, Fe0, T2);
        mul_cm(d, T2, Fp + p * dd, T1);
        memcpy(Fe, Fn, dd * sizeof(double));
        memcpy(Fp + p * dd, T1, dd * sizeof(double));
    }
}

/* MPM_DRUCKER_PRAGER::Update_Hardening (Hybrid_Methods/Forces/MPM_DRUCKER_PRAGER.cpp:118-125):
 * q += increment; phi = pi/180 (a0 + (a1 q - a4) exp(-a3 q));
 * rho_F = sqrt(2/3) 2 sin(phi) / (3 - sin(phi)).  prm = a0, a1, a3, a4, use_vc. */
static const double kPi = 3.14159265358979323846;

static void dp_hardening(double* pdef, double* rho_F, double inc, const double* prm)
{
    *pdef += inc;
    const double q = *pdef;
    const double phi = kPi / 180 * (prm[0] + (prm[1] * q - prm[3]) * exp(-prm[2] * q));
    const double sp = sin(phi);
    *rho_F = sqrt(2.0 / 3.0) * 2 * sp / (3 - sp);
}

/* MPM_DRUCKER_PRAGER::Initialize_Particles (MPM_DRUCKER_PRAGER.cpp:42-58): sigma_Y = sigma_Y0,
 * rho_F from a zero hardening increment; plastic_def and vc start at 0. */
void oracle_dp_init(long long n, double* pdef, double* rho_F, double* sigma_Y, double* vc, double sigma_Y0,
    const double* prm)
{
    for(long long p = 0; p < n; p++) {
        pdef[p] = 0;
        vc[p] = 0;
        sigma_Y[p] = sigma_Y0;
        dp_hardening(pdef + p, rho_F + p, 0, prm);
    }
}

/* MPM_PLASTICITY_MODEL::Update_Particles (MPM_PLASTICITY_MODEL.cpp:35-49) with
 * MPM_DRUCKER_PRAGER::Compute (MPM_DRUCKER_PRAGER.cpp:62-89, store_hardening on):
 * the trial Hencky strain ln|S| + beta + vc/d, beta = -sigma_Y g / (rho_F d),
 * g = 1 / (d lambda + 2 mu), b = 1 / (2 mu); k its trace, sh its deviator,
 * q = |sh|, r = rho_F k / g, dg = q + b r.  dg <= 0: elastic, unchanged.
 * q = 0 or k > 0 (the tip): strain = exp(-beta) (or 1 without cohesion),
 * vc += tr ln|S| + d beta, hardening by |ln|S||.  Else onto the cone:
 * strain = exp(k/d - (r b / q) sh - beta), vc = 0, hardening by dg.
 * Then F = U strain V^T, Fp = V strain^-1 U^T Fe Fp, over the particles simulated
 * in the substep.  F, Fp column-major per particle. */
void oracle_plastic_dp(int d, long long n, double* F, double* Fp, const double* mu, const double* la,
    double* pdef, double* rho_F, double* sigma_Y, double* vc, const unsigned char* valid, const double* prm)
{
    const int dd = d * d;
    const int use_vc = prm[4] != 0;
    for(long long p = 0; p < n; p++) {
        if(!valid[p]) continue;
        double* Fe = F + p * dd;
        double U[9], S[3], V[9];
        if(d == 3) oracle_svd3(Fe, U, S, V);
        else svd2(Fe, U, S, V);
        const double g = 1 / (d * la[p] + 2 * mu[p]), b = 1 / (2 * mu[p]);
        const double beta = -sigma_Y[p] * g / (rho_F[p] * d);
        double lf[3], st[3], k = 0, lsum = 0, lmag = 0;
        for(int a = 0; a < d; a++) {
            lf[a] = log(fabs(S[a]));
            st[a] = lf[a] + beta + vc[p] / d;
            k += st[a];
            lsum += lf[a];
            lmag += lf[a] * lf[a];
        }
        double sh[3], q = 0;
        for(int a = 0; a < d; a++) { sh[a] = st[a] - k / d; q += sh[a] * sh[a]; }
        q = sqrt(q);
        const double r = rho_F[p] * k / g, dg = q + b * r;
        if(dg <= 0) continue;
        double strain[3];
        if(q == 0 || k > 0) {
            for(int a = 0; a < d; a++) strain[a] = sigma_Y[p] != 0 ? exp(-beta) : 1;
            if(use_vc) vc[p] += lsum + beta * d;
            dp_hardening(pdef + p, rho_F + p, sqrt(lmag), prm);
        } else {
            const double pp = r * b / q;
            for(int a = 0; a < d; a++) strain[a] = exp(k / d - pp * sh[a] - beta);
            vc[p] = 0;
            dp_hardening(pdef + p, rho_F + p, dg, prm);
        }
        double Us[9], Vi[9], Fn[9], T1[9], T2[9], Fe0[9];
        memcpy(Fe0, Fe, dd * sizeof(double));
        for(int c = 0; c < d; c++)
            for(int rr = 0; rr < d; rr++) { Us[rr + d * c] = U[rr + d * c] * strain[c]; Vi[rr + d * c] = V[rr + d * c] / strain[c]; }
        for(int c = 0; c < d; c++)
            for(int rr = 0; rr < d; rr++) {
                double s1 = 0, t = 0;
                for(int kk = 0; kk < d; kk++) { s1 += Us[rr + d * kk] * V[c + d * kk]; t += Vi[rr + d * kk] * U[c + d * kk]; }
                Fn[rr + d * c] = s1;
                T1[rr + d * c] = t;
            }
        mul_cm(d, T1, Fe0, T2);
        mul_cm(d, T2, Fp + p * dd, T1);
        memcpy(Fe, Fn, dd * sizeof(double));
        memcpy(Fp + p * dd, T1, dd * sizeof(double));
    }
}
