// Device math for the explicit MPM substep: quadratic B-spline weights, the
// 3x3 / 2x2 signed SVD, the constitutive models, and the collision objects.
// Templated on the scalar type so the FP64 path and the FP64 fallbacks inside
// the FP32 path share one implementation.
//
// Matrices are column-major, a[i + d*j], the layout of PhysBAM's MATRIX<T,d>
// (Core/Matrices/MATRIX_3X3.h:115-119).
#pragma once
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_types.h"

namespace mpm {

template<class T> struct Lim;
template<> struct Lim<double> { static constexpr double eps = DBL_EPSILON; };
template<> struct Lim<float> { static constexpr float eps = FLT_EPSILON; };

template<class T> __host__ __device__ __forceinline__ T sqr(T x) { return x * x; }

// ---------------------------------------------------------------------------
// Quadratic B-spline weights.
// PARTICLE_GRID_WEIGHTS_SPLINE<TV,2>::Compute_Precompute_Data / Compute_Weights
// (Hybrid_Methods/Iterators/PARTICLE_GRID_WEIGHTS_SPLINE.cpp:93-105,133-139):
// base = Cell(X - dX), x = (X - Center(base)) / dX, and per axis
//   w0 = .5 (x-1.5)^2, w1 = .75 - (x-1)^2, w2 = .5 (x-2.5)^2  with derivatives / dX.
// ---------------------------------------------------------------------------
template<class T> struct Axis {
    int base;
    T w[3], dw[3];
};

template<class T> __device__ __forceinline__ Axis<T> spline_axis(T X, T dmin, T dx, T inv)
{
    Axis<T> a;
    T y = X - dx;
    a.base = (int)floor((y - dmin) * inv);
    T c = dmin + ((T)a.base + (T).5) * dx;
    T x = (X - c) * inv;
    a.w[0] = (T).5 * sqr(x - (T)1.5);
    a.dw[0] = (x - (T)1.5) * inv;
    x -= (T)1;
    a.w[1] = -x * x + (T).75;
    a.dw[1] = (T)-2 * x * inv;
    x -= (T)1;
    a.w[2] = (T).5 * sqr(x + (T)1.5);
    a.dw[2] = (x + (T)1.5) * inv;
    return a;
}

// ---------------------------------------------------------------------------
// Signed SVD, U and V rotations, the smallest singular value possibly
// negative.  3x3: implicit-shift QR of Gast, Fu, Jiang & Teran (2016,
// "Implicit-shifted Symmetric QR Singular Value Decomposition of 3x3
// Matrices", UCLA tech report), the method the reference uses
// (Core/Matrices/MATRIX_3X3.cpp:202-236).  2x2: indefinite polar
// decomposition then a symmetric eigenproblem (MATRIX_2X2.h:313-322,
// SYMMETRIC_MATRIX_2X2.h:364-375).
// ---------------------------------------------------------------------------
#define M3(A, i, j) (A)[(i) + 3 * (j)]

template<class T> __device__ __forceinline__ void givens(T a, T b, T g[2])
{
    T m = sqrt(a * a + b * b);
    if(m != 0) { T s = (T)1 / m; g[0] = a * s; g[1] = -b * s; }
    else { g[0] = 1; g[1] = 0; }
}
template<class T> __device__ __forceinline__ void apply_l(T* A, const T g[2], int i, int j)
{
#pragma unroll
    for(int c = 0; c < 3; c++) {
        T v = M3(A, i, c), w = M3(A, j, c);
        M3(A, i, c) = g[0] * v + g[1] * w;
        M3(A, j, c) = g[0] * w - g[1] * v;
    }
}
template<class T> __device__ __forceinline__ void apply_r(T* A, const T g[2], int i, int j)
{
#pragma unroll
    for(int r = 0; r < 3; r++) {
        T v = M3(A, r, i), w = M3(A, r, j);
        M3(A, r, i) = g[0] * v + g[1] * w;
        M3(A, r, j) = g[0] * w - g[1] * v;
    }
}
template<class T> __device__ void zero_l(T* U, T* A, int r0, int r1, int c)
{
    T g[2];
    givens(M3(A, r0, c), M3(A, r1, c), g);
    apply_l(A, g, r1, r0);
    apply_r(U, g, r1, r0);
    M3(A, r1, c) = 0;
}
template<class T> __device__ void zero_r(T* V, T* A, int c0, int c1, int r)
{
    T g[2];
    givens(M3(A, r, c0), M3(A, r, c1), g);
    apply_r(A, g, c1, c0);
    apply_r(V, g, c1, c0);
    M3(A, r, c1) = 0;
}
template<class T> __device__ void zero_chasing(T* U, T* A, T* V)
{
    zero_l(U, A, 0, 1, 0);
    zero_r(V, A, 1, 2, 0);
    zero_l(U, A, 1, 2, 1);
}
template<class T> __device__ void swap_col(T* U, int i, int j)
{
#pragma unroll
    for(int r = 0; r < 3; r++) { T u = M3(U, r, i), v = M3(U, r, j); M3(U, r, i) = v; M3(U, r, j) = -u; }
}
template<class T> __device__ void swap_row(T* U, int i, int j)
{
#pragma unroll
    for(int c = 0; c < 3; c++) { T u = M3(U, i, c), v = M3(U, j, c); M3(U, i, c) = v; M3(U, j, c) = -u; }
}
template<class T> __device__ void sv_swap(T* U, T* D, T* V, int i, int j)
{
    swap_col(U, i, j);
    swap_col(V, i, j);
    T t = D[i]; D[i] = D[j]; D[j] = t;
}
template<class T> __device__ void flip_sign(T* U, T* D, int i, int j)
{
    D[i] = -D[i]; D[j] = -D[j];
#pragma unroll
    for(int r = 0; r < 3; r++) { M3(U, r, i) = -M3(U, r, i); M3(U, r, j) = -M3(U, r, j); }
}
template<class T> __device__ __forceinline__ int argmax3(T a, T b, T c)
{
    return a >= c ? (a >= b ? 0 : 1) : (b >= c ? 1 : 2);
}
template<class T> __device__ void sort_sv(T* U, T* D, T* V)
{
    int i = argmax3(fabs(D[0]), fabs(D[1]), fabs(D[2]));
    if(i > 0) sv_swap(U, D, V, 0, i);
    if(fabs(D[1]) < fabs(D[2])) sv_swap(U, D, V, 1, 2);
    if(D[0] < 0) flip_sign(U, D, 0, D[1] < 0 ? 1 : 2);
    else if(D[1] < 0) flip_sign(U, D, 1, 2);
}
template<class T> __device__ void sym2_eigen(T x00, T x10, T x11, T l[2], T V[4])
{
    T a = (T).5 * (x00 + x11), b = (T).5 * (x00 - x11), c = x10;
    T c2 = sqr(c), m = sqrt(sqr(b) + c2), k = x00 * x11 - c2;
    if(a >= 0) { l[0] = a + m; l[1] = l[0] != 0 ? k / l[0] : 0; }
    else { l[1] = a - m; l[0] = l[1] != 0 ? k / l[1] : 0; }
    if(l[1] > l[0]) { T t = l[0]; l[0] = l[1]; l[1] = t; }
    T v0, v1;
    if(b >= 0) { v0 = m + b; v1 = c; } else { v0 = -c; v1 = b - m; }
    T n = sqrt(v0 * v0 + v1 * v1);
    if(n != 0) { T s = (T)1 / n; v0 *= s; v1 *= s; } else { v0 = 1; v1 = 0; }
    V[0] = v0; V[1] = v1; V[2] = -v1; V[3] = v0;
}
template<class T> __device__ void svd2(const T* x, T* U, T* s, T* V)
{
    T x03 = x[0] + x[3], cs, sn;
    if(x03 == 0) { cs = 0; sn = 1; }
    else { T t = (x[1] - x[2]) / x03; cs = (T)1 / sqrt(1 + t * t); sn = t * cs; }
    T Q[4] = {cs, sn, -sn, cs};
    T S00 = Q[0] * x[0] + Q[1] * x[1], S10 = Q[0] * x[2] + Q[1] * x[3], S11 = Q[2] * x[2] + Q[3] * x[3];
    sym2_eigen(S00, S10, S11, s, V);
    if(s[1] < 0 && fabs(s[1]) >= fabs(s[0])) {
        T a = -s[1], b = -s[0];
        s[0] = a; s[1] = b;
#pragma unroll
        for(int i = 0; i < 4; i++) Q[i] = -Q[i];
        T W0 = V[2], W1 = V[3], W2 = -V[0], W3 = -V[1];
        V[0] = W0; V[1] = W1; V[2] = W2; V[3] = W3;
    }
    U[0] = Q[0] * V[0] + Q[2] * V[1]; U[1] = Q[1] * V[0] + Q[3] * V[1];
    U[2] = Q[0] * V[2] + Q[2] * V[3]; U[3] = Q[1] * V[2] + Q[3] * V[3];
}
template<class T> __device__ void top_block(T* U, T* B, T* V, T* D)
{
    T a[4] = {M3(B, 0, 0), M3(B, 1, 0), M3(B, 0, 1), M3(B, 1, 1)}, u[4], d[2], v[4];
    svd2(a, u, d, v);
    apply_r(U, u, 0, 1);
    apply_r(V, v, 0, 1);
    D[0] = d[0]; D[1] = d[1]; D[2] = M3(B, 2, 2);
    sort_sv(U, D, V);
}
template<class T> __device__ void bot_block(T* U, T* B, T* V, T* D)
{
    T a[4] = {M3(B, 1, 1), M3(B, 2, 1), M3(B, 1, 2), M3(B, 2, 2)}, u[4], d[2], v[4];
    svd2(a, u, d, v);
    apply_r(U, u, 1, 2);
    apply_r(V, v, 1, 2);
    D[0] = M3(B, 0, 0); D[1] = d[0]; D[2] = d[1];
    sort_sv(U, D, V);
}
template<class T> __device__ bool check_tolerances(T* B, T* U, T* D, T* V, T tau)
{
    if(fabs(M3(B, 1, 2)) <= tau) { top_block(U, B, V, D); return true; }
    if(fabs(M3(B, 0, 1)) <= tau) { bot_block(U, B, V, D); return true; }
    if(fabs(M3(B, 1, 1)) <= tau) {
        T g[2], o[2];
        givens(M3(B, 1, 2), M3(B, 2, 2), g);
        o[0] = -g[1]; o[1] = g[0];
        apply_l(B, o, 2, 1);
        apply_r(U, o, 2, 1);
        top_block(U, B, V, D);
        return true;
    }
    if(fabs(M3(B, 2, 2)) <= tau) {
        zero_r(V, B, 1, 2, 1);
        zero_r(V, B, 0, 2, 0);
        top_block(U, B, V, D);
        return true;
    }
    if(fabs(M3(B, 0, 0)) <= tau) {
        zero_l(U, B, 1, 0, 1);
        zero_l(U, B, 2, 0, 2);
        bot_block(U, B, V, D);
        return true;
    }
    return false;
}
template<class T> __device__ bool lazy_sort(T* U, T* B, T* V, int i, int j)
{
    if(fabs(M3(B, i, i)) * 100 >= fabs(M3(B, j, j))) return false;
    swap_row(B, i, j); swap_col(U, i, j); swap_col(B, i, j); swap_col(V, i, j);
    return true;
}

// The bound on svd3's sweeps (the reference iterates without bound; a bounded
// loop keeps the GPU safe).  One device variable per compiled module, set on
// the current device through mpm_debug_set_svd_iterations, a test hook that
// makes the non-convergence flag reachable.
static __device__ int g_svd_max_it = 64;
#define MPM_SVD_LIMIT_SETTER(name) \
    cudaError_t name(int v) { return cudaMemcpyToSymbol(mpm::g_svd_max_it, &v, sizeof v); }

// Returns false when the iteration did not converge within max_it sweeps
// (g_svd_max_it when max_it < 0).
template<class T> __device__ bool svd3(const T* F, T* U, T* D, T* V, int max_it = -1)
{
    if(max_it < 0) max_it = g_svd_max_it;
    T B[9];
#pragma unroll
    for(int i = 0; i < 9; i++) { B[i] = F[i]; U[i] = V[i] = (i % 4 == 0) ? (T)1 : (T)0; }
    zero_l(U, B, 1, 2, 0);
    zero_chasing(U, B, V);
    T fro = 0;
#pragma unroll
    for(int i = 0; i < 9; i++) fro += B[i] * B[i];
    T tau = (T)16 * Lim<T>::eps * fmax((T).5 * sqrt(fro), (T)1);
    for(int it = 0; it < max_it; it++) {
        if(check_tolerances(B, U, D, V, tau)) return true;
        bool ls = lazy_sort(U, B, V, 0, 1);
        ls |= lazy_sort(U, B, V, 0, 2);
        ls |= lazy_sort(U, B, V, 1, 2);
        if(ls) {
            zero_l(U, B, 1, 2, 0);
            zero_chasing(U, B, V);
            if(check_tolerances(B, U, D, V, tau)) return true;
        }
        T al0 = M3(B, 0, 0), al1 = M3(B, 1, 1), al2 = M3(B, 2, 2);
        T be0 = M3(B, 0, 1), be1 = M3(B, 1, 2);
        T ga0 = al0 * be0, ga1 = al1 * be1;
        T a0 = al1 * al1 + be0 * be0;
        T a1 = al2 * al2 + be1 * be1;
        T b0 = ga1;
        T d = (T).5 * (a0 - a1);
        T mu = a1 - b0 * b0 / (d + (d >= 0 ? (T)1 : (T)-1) * sqrt(d * d + b0 * b0));
        T g[2];
        givens(al0 * al0 - mu, ga0, g);
        apply_r(B, g, 1, 0);
        apply_r(V, g, 1, 0);
        zero_chasing(U, B, V);
    }
    D[0] = M3(B, 0, 0); D[1] = M3(B, 1, 1); D[2] = M3(B, 2, 2);
    return false;
}

// ---------------------------------------------------------------------------
// Constitutive models on singular values.
// COROTATED_FIXED::P_From_Strain (Deformables/Constitutive_Models/COROTATED_FIXED.cpp:59-65):
//   Phat = 2 mu (S - I) + lambda (J - 1) cof(S)
// NEO_HOOKEAN::P_From_Strain with Clamp_To_Hyperbola (NEO_HOOKEAN.cpp:42-82),
// failure threshold .25 (the header default the reference's scenes use).
// ---------------------------------------------------------------------------
constexpr double kNeoHookeanThreshold = 0.25;

template<class T, int d> __device__ void phat(int model, const T* s, T mu, T la, T* P)
{
    T J = d == 2 ? s[0] * s[1] : s[0] * s[1] * s[2];
    if(model == MPM_STVK_HENCKY) {
        // ST_VENANT_KIRCHHOFF_HENCKY_STRAIN::P_From_Strain (ST_VENANT_KIRCHHOFF_HENCKY_STRAIN.cpp:67-78):
        // Phat = (2 mu ln S + lambda tr ln S) S^-1, zero once the last signed singular value is <= 0
        if(!(s[d - 1] > 0)) {
#pragma unroll
            for(int a = 0; a < d; a++) P[a] = 0;
            return;
        }
        T l[3], tr = 0;
#pragma unroll
        for(int a = 0; a < d; a++) { l[a] = log(s[a]); tr += l[a]; }
#pragma unroll
        for(int a = 0; a < d; a++) P[a] = (2 * mu * l[a] + la * tr) / s[a];
        return;
    }
    if(model == MPM_COROTATED_FIXED) {
        T cof[3];
        if(d == 2) { cof[0] = s[1]; cof[1] = s[0]; }
        else { cof[0] = s[1] * s[2]; cof[1] = s[0] * s[2]; cof[2] = s[0] * s[1]; }
        T k = la * (J - 1);
#pragma unroll
        for(int a = 0; a < d; a++) P[a] = 2 * mu * (s[a] - 1) + k * cof[a];
        return;
    }
    const T ft = (T)kNeoHookeanThreshold;
    if(J >= ft) {
        T c = mu - la * log(J);
#pragma unroll
        for(int a = 0; a < d; a++) P[a] = mu * s[a] - c * ((T)1 / s[a]);
        return;
    }
    T Fc[3];
    if(d == 2) {
        if(sqr(s[0]) > ft) { Fc[0] = s[0]; Fc[1] = ft / s[0]; }
        else { Fc[0] = Fc[1] = sqrt(ft); }
    } else {
        if(s[0] * s[1] * s[1] > ft) { Fc[0] = s[0]; Fc[1] = s[1]; Fc[2] = ft / (s[0] * s[1]); }
        else if(s[0] * s[0] * s[0] > ft) { T c = sqrt(ft / s[0]); Fc[0] = s[0]; Fc[1] = Fc[2] = c; }
        else { Fc[0] = Fc[1] = Fc[2] = cbrt(ft); }
    }
    T Fi[3], dF[3], inner = 0;
#pragma unroll
    for(int a = 0; a < d; a++) { Fi[a] = (T)1 / Fc[a]; dF[a] = s[a] - Fc[a]; inner += Fi[a] * dF[a]; }
    T c = mu - la * log(ft);
#pragma unroll
    for(int a = 0; a < d; a++) P[a] = mu * s[a] + c * (sqr(Fi[a]) * dF[a] - Fi[a]) + la * inner * Fi[a];
}

// ---------------------------------------------------------------------------
// Second derivatives on singular values for the implicit solve: the
// DIAGONALIZED_ISOTROPIC_STRESS_DERIVATIVE blocks H (H[i + d k] = x_iikk,
// symmetric), B (x_ikik) and C (x_ikki) in the reference's pair order (2D: 01;
// 3D: 12 20 01), with enforce_definiteness off (the constitutive models' default,
// CONSTITUTIVE_MODEL.cpp:16).
//   COROTATED_FIXED::Isotropic_Stress_Derivative_Helper (COROTATED_FIXED.cpp:125-163), panic 1e-6
//   NEO_HOOKEAN::Isotropic_Stress_Derivative_Helper (NEO_HOOKEAN.cpp:144-179), on the
//     hyperbola-clamped F below J = .25
//   ST_VENANT_KIRCHHOFF_HENCKY_STRAIN::Isotropic_Stress_Derivative_Helper
//     (ST_VENANT_KIRCHHOFF_HENCKY_STRAIN.cpp:92-150), zero once the last signed value is <= 0
// (log(y) - log(x)) / (y - x) without cancellation: log1p(u)/u with u = (y - x)/x.
template<class T> __device__ __forceinline__ T diff_log_over_diff(T x, T y)
{
    const T u = (y - x) / x;
    const T r = fabs(u) < (T)1e-18 ? (T)1 : log1p(u) / u;
    return r / x;
}

template<class T, int d> __device__ void stress_derivative(int model, const T* s, T mu, T la, T* H, T* Bv, T* Cv)
{
    const int P0[3] = {1, 2, 0}, P1[3] = {2, 0, 1};   // pair k of 3D: (1,2) (2,0) (0,1)
    for(int e = 0; e < 9; e++) H[e] = 0;
    for(int e = 0; e < 3; e++) Bv[e] = Cv[e] = 0;
    if(model == MPM_COROTATED_FIXED) {
        const T panic = (T)1e-6, mu2 = 2 * mu;
        auto guard = [&](T x) { return fabs(x) < panic ? (x < 0 ? -panic : panic) : x; };
        if(d == 2) {
            const T J = s[0] * s[1], d01 = guard(s[0] + s[1]);
            H[0] = mu2 + la * s[1] * s[1];
            H[3] = mu2 + la * s[0] * s[0];
            H[1] = H[2] = la * (2 * J - 1);
            Cv[0] = mu2 / d01 - la * (J - 1);
            Bv[0] = mu2 * (1 - 1 / d01);
        } else {
            const T J = s[0] * s[1] * s[2];
            const T cof[3] = {s[1] * s[2], s[0] * s[2], s[0] * s[1]};
            for(int a = 0; a < 3; a++) H[a + 3 * a] = mu2 + la * cof[a] * cof[a];
            H[1] = H[3] = la * s[2] * (2 * J - 1);
            H[2] = H[6] = la * s[1] * (2 * J - 1);
            H[5] = H[7] = la * s[0] * (2 * J - 1);
            for(int k = 0; k < 3; k++) {
                const T dk = guard(s[P0[k]] + s[P1[k]]);
                Cv[k] = mu2 / dk + la * s[k] * (1 - J);
                Bv[k] = mu2 * (1 - 1 / dk);
            }
        }
        return;
    }
    if(model == MPM_NEO_HOOKEAN) {
        const T ft = (T)kNeoHookeanThreshold;
        T J = 1;
        for(int a = 0; a < d; a++) J *= s[a];
        T Fc[3];
        for(int a = 0; a < d; a++) Fc[a] = s[a];
        if(!(J >= ft)) {   // NEO_HOOKEAN::Clamp_To_Hyperbola
            if(d == 2) {
                if(s[0] * s[0] > ft) { Fc[0] = s[0]; Fc[1] = ft / s[0]; }
                else { Fc[0] = Fc[1] = sqrt(ft); }
            } else {
                if(s[0] * s[1] * s[1] > ft) { Fc[0] = s[0]; Fc[1] = s[1]; Fc[2] = ft / (s[0] * s[1]); }
                else if(s[0] * s[0] * s[0] > ft) { T c = sqrt(ft / s[0]); Fc[0] = s[0]; Fc[1] = Fc[2] = c; }
                else { Fc[0] = Fc[1] = Fc[2] = cbrt(ft); }
            }
        }
        T Fi[3], detFi = 1;
        for(int a = 0; a < d; a++) { Fi[a] = 1 / Fc[a]; detFi *= Fi[a]; }
        const T mlj = mu + la * log(detFi);
        for(int a = 0; a < d; a++) H[a + d * a] = mu + (la + mlj) * Fi[a] * Fi[a];
        for(int a = 0; a < d; a++)
            for(int b = 0; b < d; b++)
                if(a != b) H[a + d * b] = la * Fi[a] * Fi[b];
        if(d == 2) { Bv[0] = mu; Cv[0] = mlj * Fi[1] * Fi[0]; }
        else
            for(int k = 0; k < 3; k++) { Bv[k] = mu; Cv[k] = mlj * Fi[P0[k]] * Fi[P1[k]]; }
        return;
    }
    // ST_VENANT_KIRCHHOFF_HENCKY_STRAIN (failure_threshold 0)
    if(!(s[d - 1] > 0)) return;
    const T l2m = la + 2 * mu, mu2 = 2 * mu;
    T l[3], sum = 0;
    for(int a = 0; a < d; a++) { l[a] = log(s[a]); sum += l[a]; }
    for(int a = 0; a < d; a++) H[a + d * a] = (l2m - mu2 * l[a] - la * sum) / (s[a] * s[a]);
    for(int a = 0; a < d; a++)
        for(int b = 0; b < d; b++)
            if(a != b) H[a + d * b] = la / (s[a] * s[b]);
    auto pair = [&](int i, int j, T& B, T& C) {
        const T m = (mu2 / s[i]) * (diff_log_over_diff(s[i], s[j]) - l[j] / s[j]) - la * sum / (s[i] * s[j]);
        T p;
        if(d == 2) p = ((la * s[0] + l2m * s[1]) * l[0] + (la * s[1] + l2m * s[0]) * l[1]) / (s[0] * s[1] * (s[0] + s[1]));
        else p = (mu2 * (s[j] * l[i] + s[i] * l[j]) + la * (s[i] + s[j]) * sum) / (s[i] * s[j] * (s[i] + s[j]));
        B = (T).5 * (m + p);
        C = (T).5 * (m - p);
    };
    if(d == 2) pair(0, 1, Bv[0], Cv[0]);
    else {
        pair(0, 1, Bv[2], Cv[2]);
        pair(0, 2, Bv[1], Cv[1]);
        pair(1, 2, Bv[0], Cv[0]);
    }
}

// DIAGONALIZED_ISOTROPIC_STRESS_DERIVATIVE::Differential: dP = dPhat/dF : dF in
// the SVD frame (column-major d x d).
template<class T, int d> __device__ __forceinline__ void stress_differential(const T* H, const T* Bv, const T* Cv, const T* G, T* dP)
{
    if(d == 2) {
        dP[0] = H[0] * G[0] + H[1] * G[3];
        dP[3] = H[1] * G[0] + H[3] * G[3];
        dP[1] = Bv[0] * G[1] + Cv[0] * G[2];
        dP[2] = Cv[0] * G[1] + Bv[0] * G[2];
        return;
    }
    dP[0] = H[0] * G[0] + H[1] * G[4] + H[2] * G[8];
    dP[4] = H[1] * G[0] + H[4] * G[4] + H[5] * G[8];
    dP[8] = H[2] * G[0] + H[5] * G[4] + H[8] * G[8];
    dP[1] = Bv[2] * G[1] + Cv[2] * G[3];
    dP[3] = Cv[2] * G[1] + Bv[2] * G[3];
    dP[2] = Bv[1] * G[2] + Cv[1] * G[6];
    dP[6] = Cv[1] * G[2] + Bv[1] * G[6];
    dP[5] = Bv[0] * G[5] + Cv[0] * G[7];
    dP[7] = Cv[0] * G[5] + Bv[0] * G[7];
}

// Energy_Density on singular values:
//   COROTATED_FIXED (COROTATED_FIXED.cpp:179-185): mu |S - I|^2 + lambda/2 (J - 1)^2
//   NEO_HOOKEAN (NEO_HOOKEAN.cpp:191-199): mu (|S|^2/2 - d/2 - ln J) + lambda/2 ln^2 J, 1e16 for J <= 0
//   ST_VENANT_KIRCHHOFF_HENCKY_STRAIN (l.52-63): mu |ln S|^2 + lambda/2 (tr ln S)^2, FLT_MAX
//     once the last signed value is <= 0
template<class T, int d> __device__ T energy_density(int model, const T* s, T mu, T la)
{
    T J = 1;
    for(int a = 0; a < d; a++) J *= s[a];
    if(model == MPM_COROTATED_FIXED) {
        T e = 0;
        for(int a = 0; a < d; a++) e += (s[a] - 1) * (s[a] - 1);
        return mu * e + (T).5 * la * (J - 1) * (J - 1);
    }
    if(model == MPM_NEO_HOOKEAN) {
        if(J <= 0) return (T)1e16;
        T I1 = 0;
        for(int a = 0; a < d; a++) I1 += s[a] * s[a];
        const T lj = log(J);
        return mu * ((T).5 * (I1 - d) - lj) + (T).5 * la * lj * lj;
    }
    if(s[d - 1] <= 0) return (T)FLT_MAX;
    T n2 = 0, tr = 0;
    for(int a = 0; a < d; a++) { const T l = log(s[a]); n2 += l * l; tr += l; }
    return mu * n2 + (T).5 * la * tr * tr;
}

// ISOTROPIC_CONSTITUTIVE_MODEL::Sound_Speed (ISOTROPIC_CONSTITUTIVE_MODEL.cpp:150-161)
// from the singular values and the stress derivative blocks.
template<class T, int d> __device__ T sound_speed(const T* S, const T* H, const T* Bv, T density)
{
    T F2[3], cm = -(T)INFINITY;
    for(int a = 0; a < d; a++) { F2[a] = S[a] * S[a]; cm = fmax(cm, H[a + d * a] * F2[a]); }
    const int spin = d == 3 ? 3 : 1;
    for(int k = 0; k < spin; k++)
        for(int i = 0; i < 2; i++) cm = fmax(cm, Bv[k] * F2[(k + i + 1) % spin]);
    return sqrt(cm / density);
}


// MPM_FINITE_ELEMENTS::Precompute (Hybrid_Methods/Forces/MPM_FINITE_ELEMENTS.cpp:47-67):
// PFT = U Phat(S) (F V)^T, i.e. P(F) F^T.  Returns false if the SVD did not converge.
template<class T, int d> __device__ bool pft_svd(int model, const T* F, T mu, T la, T* PFT)
{
    T U[9], V[9], s[3], P[3];
    bool ok = true;
    if(d == 2) {
        svd2(F, U, s, V);
        phat<T, 2>(model, s, mu, la, P);
        T FV[4];
        FV[0] = F[0] * V[0] + F[2] * V[1]; FV[1] = F[1] * V[0] + F[3] * V[1];
        FV[2] = F[0] * V[2] + F[2] * V[3]; FV[3] = F[1] * V[2] + F[3] * V[3];
        T PT[4] = {P[0] * FV[0], P[1] * FV[2], P[0] * FV[1], P[1] * FV[3]};
        PFT[0] = U[0] * PT[0] + U[2] * PT[1]; PFT[1] = U[1] * PT[0] + U[3] * PT[1];
        PFT[2] = U[0] * PT[2] + U[2] * PT[3]; PFT[3] = U[1] * PT[2] + U[3] * PT[3];
        return true;
    }
    ok = svd3(F, U, s, V);
    phat<T, 3>(model, s, mu, la, P);
    T FV[9], PT[9];
#pragma unroll
    for(int j = 0; j < 3; j++)
#pragma unroll
        for(int i = 0; i < 3; i++)
            FV[i + 3 * j] = F[i] * V[3 * j] + F[i + 3] * V[3 * j + 1] + F[i + 6] * V[3 * j + 2];
#pragma unroll
    for(int i = 0; i < 3; i++)
#pragma unroll
        for(int j = 0; j < 3; j++) PT[i + 3 * j] = P[i] * FV[j + 3 * i];
#pragma unroll
    for(int j = 0; j < 3; j++)
#pragma unroll
        for(int i = 0; i < 3; i++)
            PFT[i + 3 * j] = U[i] * PT[3 * j] + U[i + 3] * PT[3 * j + 1] + U[i + 6] * PT[3 * j + 2];
    return ok;
}

// ---------------------------------------------------------------------------
// Static collision objects (MPM_COLLISION_OBJECT, Hybrid_Methods/Collisions/
// MPM_COLLISION_OBJECT.cpp:27-48, with ANALYTIC_IMPLICIT_OBJECT forwarding to
// RANGE::Signed_Distance / RANGE::Normal, Core/Math_Tools/RANGE.cpp:37-63, or
// PLANE, Geometry/Basic_Geometry/PLANE.h:52-63).
// ---------------------------------------------------------------------------
struct DevObject {
    int kind, type;
    double friction;
    double a[3], b[3];
};

// The same object with its numbers rounded to float once (the FP32 path
// rounds each of them to float where it uses them, so results are the same).
struct DevObjectF {
    int kind, type;
    float friction;
    float a[3], b[3];
};

template<class T, int d, class O> __device__ T object_phi(const O& o, const T* X)
{
    if(o.kind == MPM_SPHERE) {   // SPHERE::Signed_Distance (Geometry/Basic_Geometry/SPHERE.h:59-60)
        T r2 = 0;
#pragma unroll
        for(int a = 0; a < d; a++) r2 += (X[a] - (T)o.a[a]) * (X[a] - (T)o.a[a]);
        return sqrt(r2) - (T)o.b[0];
    }
    if(o.kind == MPM_PLANE) {
        T s = 0;
#pragma unroll
        for(int a = 0; a < d; a++) s += (T)o.a[a] * (X[a] - (T)o.b[a]);
        return s;
    }
    T phi[3], mx = -(T)INFINITY, out = 0;
    bool all_le = true;
#pragma unroll
    for(int a = 0; a < d; a++) {
        T lo = (T)o.a[a], hi = (T)o.b[a];
        T len = hi - lo, c = (lo + hi) * (T).5;
        phi[a] = fabs(X[a] - c) - (T).5 * len;
        if(!(phi[a] <= 0)) all_le = false;
        mx = phi[a] > mx ? phi[a] : mx;
    }
    if(!all_le) {
#pragma unroll
        for(int a = 0; a < d; a++) { T p = phi[a] > 0 ? phi[a] : 0; out += p * p; }
        return sqrt(out);
    }
    return mx;
}

template<class T, int d, class O> __device__ void object_normal(const O& o, const T* X, T* n)
{
    if(o.kind == MPM_SPHERE) {   // SPHERE::Normal: (X - center).Normalized()
        T mag = 0;
#pragma unroll
        for(int a = 0; a < d; a++) { n[a] = X[a] - (T)o.a[a]; mag += n[a] * n[a]; }
        mag = sqrt(mag);
        if(mag != 0) {
            const T s = (T)1 / mag;
#pragma unroll
            for(int a = 0; a < d; a++) n[a] *= s;
        } else {
#pragma unroll
            for(int a = 0; a < d; a++) n[a] = a == 0 ? (T)1 : (T)0;
        }
        return;
    }
    if(o.kind == MPM_PLANE) {
#pragma unroll
        for(int a = 0; a < d; a++) n[a] = (T)o.a[a];
        return;
    }
    bool inside = true;
    T pmax[3], pmin[3];
#pragma unroll
    for(int a = 0; a < d; a++) {
        T lo = (T)o.a[a], hi = (T)o.b[a];
        if(!(X[a] >= lo && X[a] <= hi)) inside = false;
        pmax[a] = X[a] - hi;
        pmin[a] = lo - X[a];
    }
    if(inside) {
        T m[3];
#pragma unroll
        for(int a = 0; a < d; a++) m[a] = pmin[a] > pmax[a] ? pmin[a] : pmax[a];
        int ax = d == 2 ? (m[0] >= m[1] ? 0 : 1) : argmax3(m[0], m[1], m[2]);
#pragma unroll
        for(int a = 0; a < d; a++) n[a] = 0;
        n[ax] = pmax[ax] > pmin[ax] ? (T)1 : (T)-1;
        return;
    }
    T mag = 0;
#pragma unroll
    for(int a = 0; a < d; a++) {
        T p = pmin[a] > pmax[a] ? pmin[a] : pmax[a];
        n[a] = p > 0 ? (pmax[a] > pmin[a] ? p : -p) : 0;
        mag += n[a] * n[a];
    }
    mag = sqrt(mag);
    if(mag != 0) {
        T s = (T)1 / mag;
#pragma unroll
        for(int a = 0; a < d; a++) n[a] *= s;
    } else {
#pragma unroll
        for(int a = 0; a < d; a++) n[a] = a == 0 ? (T)1 : (T)0;
    }
}

// Hessian of the signed distance, H[a + d b] (the implicit solve's collision
// curvature): zero for a plane and inside a box; outside a box
// RANGE::Hessian (Core/Math_Tools/RANGE.cpp:67-81) (D - n n^T)/|n| over the
// axes the point is beyond; SPHERE::Hessian (SPHERE.h:38-39) (I - z z^T)/|X - c|.
template<class T, int d, class O> __device__ void object_hessian(const O& o, const T* X, T* H)
{
#pragma unroll
    for(int e = 0; e < d * d; e++) H[e] = 0;
    if(o.kind == MPM_PLANE) return;
    T z[3], D[3], w = 0;
    if(o.kind == MPM_SPHERE) {
#pragma unroll
        for(int a = 0; a < d; a++) { z[a] = X[a] - (T)o.a[a]; w += z[a] * z[a]; D[a] = 1; }
    } else {
        bool inside = true;
#pragma unroll
        for(int a = 0; a < d; a++) if(!(X[a] >= (T)o.a[a] && X[a] <= (T)o.b[a])) inside = false;
        if(inside) return;
#pragma unroll
        for(int a = 0; a < d; a++) {
            const T pmax = X[a] - (T)o.b[a], pmin = (T)o.a[a] - X[a];
            const T phi = pmin > pmax ? pmin : pmax;
            z[a] = 0; D[a] = 0;
            if(phi > 0) { z[a] = pmax > pmin ? phi : -phi; D[a] = 1; }
            w += z[a] * z[a];
        }
    }
    w = sqrt(w);
    if(w != 0) {
        const T s = (T)1 / w;
#pragma unroll
        for(int a = 0; a < d; a++) z[a] *= s;
    } else {
#pragma unroll
        for(int a = 0; a < d; a++) z[a] = a == 0 ? (T)1 : (T)0;
    }
#pragma unroll
    for(int a = 0; a < d; a++)
#pragma unroll
        for(int b = 0; b < d; b++) H[a + d * b] = ((a == b ? D[a] : (T)0) - z[a] * z[b]) / w;
}

// A moving collision object over one substep: MPM_COLLISION_OBJECT's
// func_frame at the substep's start (R0, x0) and end (R1, x1) and func_twist
// at its end (v, w) (Hybrid_Methods/Collisions/MPM_COLLISION_OBJECT.cpp:23-71).
// The object's geometry is given in its own frame: a point Z of it sits at
// R Z + x.  R is column-major d x d; in 2D w[0] is the spin.
template<class S> struct ObjMotionT {
    S R0[9], x0[3], R1[9], x1[3], v[3], w[3];
};
typedef ObjMotionT<double> ObjMotion;
typedef ObjMotionT<float> ObjMotionF;

// FRAME::Inverse_Times: Z = R^T (X - x), the frame at the substep's end when `end`.
template<class T, int d, class S> __device__ __forceinline__ void to_local(const ObjMotionT<S>& m, bool end, const T* X, T* Z)
{
    const S* R = end ? m.R1 : m.R0;
    const S* x = end ? m.x1 : m.x0;
    T y[3];
#pragma unroll
    for(int a = 0; a < d; a++) y[a] = X[a] - (T)x[a];
#pragma unroll
    for(int c = 0; c < d; c++) {
        T z = 0;
#pragma unroll
        for(int a = 0; a < d; a++) z += (T)R[a + d * c] * y[a];
        Z[c] = z;
    }
}

// MPM_COLLISION_OBJECT::Phi / Normal / Hessian (l.23-59) of object j at the
// substep's start or end; `mo` null or bit j of `moving` clear: a static object.
template<class T, int d, class O, class S> __device__ T phi_at(const O& o, const ObjMotionT<S>* mo, unsigned moving, int j,
    bool end, const T* X)
{
    if(!mo || !((moving >> j) & 1u)) return object_phi<T, d>(o, X);
    T Z[3];
    to_local<T, d>(mo[j], end, X, Z);
    return object_phi<T, d>(o, Z);
}

template<class T, int d, class O, class S> __device__ void normal_at(const O& o, const ObjMotionT<S>* mo, unsigned moving, int j,
    const T* X, T* n)
{
    if(!mo || !((moving >> j) & 1u)) { object_normal<T, d>(o, X, n); return; }
    T Z[3], nl[3];
    to_local<T, d>(mo[j], true, X, Z);
    object_normal<T, d>(o, Z, nl);
    const S* R = mo[j].R1;
#pragma unroll
    for(int r = 0; r < d; r++) {
        T s = 0;
#pragma unroll
        for(int c = 0; c < d; c++) s += (T)R[r + d * c] * nl[c];
        n[r] = s;
    }
}

// SYMMETRIC_MATRIX::Conjugate(R, H) = R H R^T for a moving object.
template<class T, int d, class O, class S> __device__ void hessian_at(const O& o, const ObjMotionT<S>* mo, unsigned moving, int j,
    const T* X, T* H)
{
    if(!mo || !((moving >> j) & 1u)) { object_hessian<T, d>(o, X, H); return; }
    T Z[3], Hl[9], RH[9];
    to_local<T, d>(mo[j], true, X, Z);
    object_hessian<T, d>(o, Z, Hl);
    const S* R = mo[j].R1;
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T s = 0;
#pragma unroll
            for(int k = 0; k < d; k++) s += (T)R[r + d * k] * Hl[k + d * c];
            RH[r + d * c] = s;
        }
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T s = 0;
#pragma unroll
            for(int k = 0; k < d; k++) s += RH[r + d * k] * (T)R[c + d * k];
            H[r + d * c] = s;
        }
}

// MPM_COLLISION_OBJECT::Velocity (l.63-71): v + w x (X - x1); zero when static.
template<class T, int d, class S> __device__ void velocity_at(const ObjMotionT<S>* mo, unsigned moving, int j, const T* X, T* V)
{
    if(!mo || !((moving >> j) & 1u)) {
#pragma unroll
        for(int a = 0; a < d; a++) V[a] = 0;
        return;
    }
    const ObjMotionT<S>& m = mo[j];
    T r[3];
#pragma unroll
    for(int a = 0; a < d; a++) r[a] = X[a] - (T)m.x1[a];
    if(d == 3) {
        V[0] = (T)m.v[0] + ((T)m.w[1] * r[2] - (T)m.w[2] * r[1]);
        V[1] = (T)m.v[1] + ((T)m.w[2] * r[0] - (T)m.w[0] * r[2]);
        V[2] = (T)m.v[2] + ((T)m.w[0] * r[1] - (T)m.w[1] * r[0]);
    } else {   // VECTOR<T,1>::Cross(VECTOR<T,2>): the spin times the perpendicular (-y, x)
        V[0] = (T)m.v[0] + -(T)m.w[0] * r[1];
        V[1] = (T)m.v[1] + (T)m.w[0] * r[0];
    }
}

// Penalty collision objects at one particle position, one
// IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES per object, in object order
// (Update_Position_Based_State_Particle,
// Deformables/Collisions_And_Interactions/IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES.cpp:49-60):
// where phi <= sep, x = sep - phi and a = k x^2, the energy a x, the force
// -grad pe = 3 a n (Add_Velocity_Independent_Forces, l.82-85) added to f, and
// the Hessian 6 k x n n^T - 3 a Hess(phi) added to H (when H is not null).
// Returns the energy.
template<class T, int d, class O> __device__ T penalty_particle(const O* objs, int nobj, T k, T sep, const T* X, T* f, T* H)
{
    T e = 0;
    for(int j = 0; j < nobj; j++) {
        const T phi = object_phi<T, d>(objs[j], X);
        if(phi > sep) continue;
        T n[3];
        object_normal<T, d>(objs[j], X, n);
        const T x = sep - phi, a = k * x * x;
        e += a * x;
        const T ga = (T)-3 * a;   // grad pe = -3 a n
#pragma unroll
        for(int r = 0; r < d; r++) f[r] -= ga * n[r];
        if(H) {
            T Hp[9];
            object_hessian<T, d>(objs[j], X, Hp);
            const T s = (T)6 * k * x, t = (T)3 * a;
#pragma unroll
            for(int c = 0; c < d; c++)
#pragma unroll
                for(int r = 0; r < d; r++) H[r + d * c] += s * (n[r] * n[c]) - t * Hp[r + d * c];
        }
    }
    return e;
}

// Grid-node collision projection and Coulomb friction for one node.
// MPM_OBJECTIVE::Test_Add_Collision / Adjust_For_Collision
// (Hybrid_Methods/System/MPM_OBJECTIVE.cpp:150-225), MPM_DRIVER::Apply_Friction
// (Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.cpp:1064-1094) and the final
// assembly of Apply_Forces (l.1050-1056).  Objects are static, or move as
// `mo` gives them (bit j of `moving`): the start test at the substep's start
// frame, the projection at its end frame, a sticky node at the object's
// velocity there.
//
// In: v0 (grid velocity after P2G), dv (dt/m f), node centre X0.
// Out: vnew (velocity), vfric (velocity_friction_save).
//
// FP32 state: the reference's projection moves the node to X = X0 + dt V,
// projects X and takes V = (X - X0) / dt, which in FP32 keeps only a few bits
// of V once |dt V| is far below |X0| (dt 2e-5 and |X0| ~ 1 quantise V to
// ~3e-3 m/s).  So with T = float, a node that may touch an object during the
// substep is collided in FP64 (the same formulas, exact inputs promoted);
// a static object whose signed distance at the node exceeds dt |V| plus the
// FP32 rounding of that distance is out of reach, as the FP64 test decides
// too (signed distances are 1-Lipschitz), and a node out of every object's
// reach keeps V.
template<class T, int d, class O, class S = double> __device__ void collide_node(const O* objs, int nobj, const T* X0,
    const T* v0, T* dv, T dt, T* vnew, T* vfric, const ObjMotionT<S>* mo = nullptr, unsigned moving = 0)
{
    if constexpr(sizeof(T) == 4) {
        T speed = 0, xmax = 1;
#pragma unroll
        for(int a = 0; a < d; a++) {
            const T va = v0[a] + dv[a];
            speed += va * va;
            xmax = fmaxf(xmax, fabsf(X0[a]));
        }
        const T step = dt * sqrtf(speed);
        bool near = false;
        for(int j = 0; j < nobj && !near; j++) {
            T scale = xmax;
#pragma unroll
            for(int a = 0; a < 3; a++) scale = fmaxf(scale, fmaxf(fabsf((T)objs[j].a[a]), fabsf((T)objs[j].b[a])));
            near = (mo && ((moving >> j) & 1u)) || !(object_phi<T, d>(objs[j], X0) > step + (T)64 * FLT_EPSILON * scale);
        }
        if(!near) {
#pragma unroll
            for(int a = 0; a < d; a++) vnew[a] = vfric[a] = v0[a] + dv[a];
            return;
        }
        double X0d[3] = {0, 0, 0}, v0d[3] = {0, 0, 0}, dvd[3] = {0, 0, 0}, vnd[3], vfd[3];
#pragma unroll
        for(int a = 0; a < d; a++) { X0d[a] = X0[a]; v0d[a] = v0[a]; dvd[a] = dv[a]; }
        collide_node<double, d, O, S>(objs, nobj, X0d, v0d, dvd, (double)dt, vnd, vfd, mo, moving);
#pragma unroll
        for(int a = 0; a < d; a++) { dv[a] = (T)dvd[a]; vnew[a] = (T)vnd[a]; vfric[a] = (T)vfd[a]; }
        return;
    }
    T dvb[3], nrm[MPM_MAX_OBJECTS][3], sv[3] = {0, 0, 0};
    int cobj[MPM_MAX_OBJECTS];
    int ncol = 0;
    bool stuck = false;
#pragma unroll
    for(int a = 0; a < d; a++) dvb[a] = dv[a];
    for(int j = 0; j < nobj; j++) {
        const O& o = objs[j];
        const T phi0 = phi_at<T, d>(o, mo, moving, j, false, X0);
        // stick and slip test only nodes that start inside the object
        if((o.type == MPM_STICK || o.type == MPM_SLIP) && phi0 > 0) continue;
        T Vn[3], Xn[3];
#pragma unroll
        for(int a = 0; a < d; a++) { Vn[a] = v0[a] + dv[a]; Xn[a] = X0[a] + dt * Vn[a]; }
        T phi = phi_at<T, d>(o, mo, moving, j, true, Xn) - fmin(phi0, (T)0);
        if(o.type == MPM_SEPARATE && phi > (T)1e-15) continue;
        if(o.type != MPM_STICK && phi > (T)FLT_MAX) continue;
        T n[3];
        normal_at<T, d>(o, mo, moving, j, Xn, n);
#pragma unroll
        for(int a = 0; a < d; a++) nrm[ncol][a] = n[a];
        cobj[ncol] = j;
        ncol++;
#pragma unroll
        for(int a = 0; a < d; a++) Xn[a] -= phi * n[a];
#pragma unroll
        for(int a = 0; a < d; a++) Vn[a] = (Xn[a] - X0[a]) / dt;
        if(o.type == MPM_STICK) {   // at the object's velocity (stuck_velocity)
            velocity_at<T, d>(mo, moving, j, Xn, Vn);
#pragma unroll
            for(int a = 0; a < d; a++) sv[a] = Vn[a];
            stuck = true;
        }
#pragma unroll
        for(int a = 0; a < d; a++) dv[a] = Vn[a] - v0[a];
    }
    T gvf[3], v[3];
#pragma unroll
    for(int a = 0; a < d; a++) gvf[a] = dv[a];
    if(nobj) {
#pragma unroll
        for(int a = 0; a < d; a++) v[a] = stuck ? (T)0 : v0[a] + dv[a];
        for(int c = 0; c < ncol; c++) {
            const T* n = nrm[c];
            T nf = 0, vn = 0, t[3], tm = 0;
#pragma unroll
            for(int a = 0; a < d; a++) nf += n[a] * (dv[a] - dvb[a]);
#pragma unroll
            for(int a = 0; a < d; a++) vn += v[a] * n[a];
#pragma unroll
            for(int a = 0; a < d; a++) { t[a] = v[a] - vn * n[a]; tm += t[a] * t[a]; }
            tm = sqrt(tm);
            if(tm != 0) {
                T s = (T)1 / tm;
#pragma unroll
                for(int a = 0; a < d; a++) t[a] *= s;
            } else {
#pragma unroll
                for(int a = 0; a < d; a++) t[a] = a == 0 ? (T)1 : (T)0;
            }
            T kf = (T)objs[cobj[c]].friction * nf;
            if(tm <= kf) {
                T vv = 0;
#pragma unroll
                for(int a = 0; a < d; a++) vv += v[a] * n[a];
#pragma unroll
                for(int a = 0; a < d; a++) v[a] = vv * n[a];
            } else {
#pragma unroll
                for(int a = 0; a < d; a++) v[a] -= kf * t[a];
            }
#pragma unroll
            for(int a = 0; a < d; a++) gvf[a] = v[a] - v0[a];
        }
    }
#pragma unroll
    for(int a = 0; a < d; a++) {
        vnew[a] = dv[a] + v0[a];
        vfric[a] = stuck ? sv[a] : gvf[a] + v0[a];
    }
}

// ---------------------------------------------------------------------------
// Snow plasticity for one particle after G2P: MPM_PLASTICITY_MODEL::
// Update_Particles (Hybrid_Methods/Forces/MPM_PLASTICITY_MODEL.cpp:35-49) with
// MPM_PLASTICITY_CLAMP::Compute (MPM_PLASTICITY_CLAMP.cpp:28-45).  The
// singular values of F are clamped to [1 - theta_c, 1 + theta_s]; when any
// moved, mu and lambda harden to mu0, lambda0 times
// exp(min(max_hardening, hardening_factor (1 - det Fp_new))) (at least 1e-8),
// F becomes U strain V^T and Fp becomes V strain^-1 U^T F_old Fp.  F and Fp
// are column-major.  prm = theta_c, theta_s, max_hardening, hardening_factor.
// Returns whether the particle changed; `ok` is false if the SVD did not
// converge (the particle is left as it is).
template<class T, int d> __device__ bool plastic_clamp(T* F, T* Fp, T& mu, T& la, T mu0, T la0, const T* prm, bool& ok)
{
    T U[9], S[3], V[9];
    ok = true;
    if(d == 3) ok = svd3<T>(F, U, S, V);
    else svd2<T>(F, U, S, V);
    if(!ok) return false;
    const T lo = (T)1 - prm[0], hi = (T)1 + prm[1];
    T st[3];
    bool same = true;
#pragma unroll
    for(int a = 0; a < d; a++) {
        st[a] = S[a] < lo ? lo : (S[a] > hi ? hi : S[a]);
        if(st[a] != S[a]) same = false;
    }
    if(same) return false;
    T pf = 1, ps = 1;
#pragma unroll
    for(int a = 0; a < d; a++) { pf *= S[a]; ps *= st[a]; }
    const T* P = Fp;
    const T detp = d == 2 ? P[0] * P[3] - P[2] * P[1]
                          : P[0] * (P[4] * P[8] - P[7] * P[5]) - P[3] * (P[1] * P[8] - P[7] * P[2]) + P[6] * (P[1] * P[5] - P[4] * P[2]);
    const T e = prm[3] * ((T)1 - pf / ps * detp);
    T coeff = exp(e < prm[2] ? e : prm[2]);
    if(coeff < (T)1e-8) coeff = (T)1e-8;
    mu = mu0 * coeff;
    la = la0 * coeff;
    T Fe[9], T1[9], T2[9];
#pragma unroll
    for(int k = 0; k < d * d; k++) Fe[k] = F[k];
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T f = 0, t = 0;
#pragma unroll
            for(int k = 0; k < d; k++) {
                f += U[r + d * k] * st[k] * V[c + d * k];
                t += V[r + d * k] / st[k] * U[c + d * k];
            }
            F[r + d * c] = f;
            T1[r + d * c] = t;
        }
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T s2 = 0;
#pragma unroll
            for(int k = 0; k < d; k++) s2 += T1[r + d * k] * Fe[k + d * c];
            T2[r + d * c] = s2;
        }
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T s2 = 0;
#pragma unroll
            for(int k = 0; k < d; k++) s2 += T2[r + d * k] * P[k + d * c];
            T1[r + d * c] = s2;
        }
#pragma unroll
    for(int k = 0; k < d * d; k++) Fp[k] = T1[k];
    return true;
}

// ---------------------------------------------------------------------------
// Eigensystem of a symmetric 3x3 matrix in FP32 registers by cyclic Jacobi
// rotations (Golub & Van Loan, Matrix Computations, 4th ed., 8.5.2: the
// symmetric Schur rotation): A <- V^T A V becomes diagonal, V accumulates the
// rotations (columns = eigenvectors), unsorted.  Used for the SVD-free
// plasticity updates (eigensystem of F^T F) and the Hencky stress (of F F^T).
// ---------------------------------------------------------------------------
template<int P, int Q>
__device__ __forceinline__ void jacobi_rotate(float (&A)[3][3], float (&V)[3][3])
{
    constexpr int R = 3 - P - Q;
    const float apq = A[P][Q];
    const float d = A[Q][Q] - A[P][P];
    // t = tan of the rotation angle: an approximate t still gives an exact
    // rotation (c and s come from t) and only leaves a residual that the next
    // sweep removes; c to full precision keeps V orthogonal
    const float h = d * d + 4.f * apq * apq;
    const float den = fabsf(d) + h * rsqrtf(h);
    float t = h > 0.f ? __fdividef(2.f * apq, den) : 0.f;
    if(d < 0.f) t = -t;
    const float x = 1.f + t * t;
    float c = rsqrtf(x);
    c = c * (1.5f - 0.5f * x * c * c);   // one Newton step
    const float s = t * c;
    A[P][P] -= t * apq;
    A[Q][Q] += t * apq;
    A[P][Q] = A[Q][P] = 0.f;
    const float arp = A[R][P], arq = A[R][Q];
    A[R][P] = A[P][R] = c * arp - s * arq;
    A[R][Q] = A[Q][R] = s * arp + c * arq;
#pragma unroll
    for(int k = 0; k < 3; k++) {
        const float vp = V[k][P], vq = V[k][Q];
        V[k][P] = c * vp - s * vq;
        V[k][Q] = s * vp + c * vq;
    }
}


__device__ __forceinline__ void sym_eig3f(float (&A)[3][3], float (&V)[3][3])
{
#pragma unroll
    for(int i = 0; i < 3; i++)
#pragma unroll
        for(int k = 0; k < 3; k++) V[i][k] = i == k ? 1.f : 0.f;
    // three sweeps reach FP32 accuracy for eigenvalue ratios up to 100; a
    // fourth runs where the off-diagonal part is not yet at rounding level
#pragma unroll
    for(int sweep = 0; sweep < 3; sweep++) {
        jacobi_rotate<0, 1>(A, V);
        jacobi_rotate<0, 2>(A, V);
        jacobi_rotate<1, 2>(A, V);
    }
    const float off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const float dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if(off > 1e-14f * dia) {
        jacobi_rotate<0, 1>(A, V);
        jacobi_rotate<0, 2>(A, V);
        jacobi_rotate<1, 2>(A, V);
    }
}

// ---------------------------------------------------------------------------
// MPM_DRUCKER_PRAGER (Hybrid_Methods/Forces/MPM_DRUCKER_PRAGER.cpp).
// prm = a0, a1, a3, a4, use_vc.  Per particle: q = plastic_def, rho_F,
// sigma_Y (cohesion), vc.
// ---------------------------------------------------------------------------
// Update_Hardening (l.118-125): q += inc; phi = pi/180 (a0 + (a1 q - a4) exp(-a3 q));
// rho_F = sqrt(2/3) 2 sin(phi) / (3 - sin(phi)).
template<class T> __device__ __forceinline__ void dp_hardening(T& q, T& rho_F, T inc, const T* prm)
{
    q += inc;
    const T phi = (T)(3.14159265358979323846 / 180) * (prm[0] + (prm[1] * q - prm[3]) * exp(-prm[2] * q));
    const T sp = sin(phi);
    rho_F = (T)0.81649658092772603 * 2 * sp / (3 - sp);   // sqrt(2/3)
}

// Compute with store_hardening (l.62-89) on the singular values S (the last
// may be negative): writes the projected strain and returns true, or returns
// false where the trial state is elastic (dg <= 0: no change at all).
template<class T, int d> __device__ bool dp_strain(const T* S, T mu, T la, T& q, T& rho_F, T sigma_Y, T& vc,
    const T* prm, T* strain)
{
    const T g = 1 / (d * la + 2 * mu), b = 1 / (2 * mu);
    const T beta = -sigma_Y * g / (rho_F * d);
    T lf[3], st[3], k = 0, lsum = 0, lmag = 0;
#pragma unroll
    for(int a = 0; a < d; a++) {
        lf[a] = log(fabs(S[a]));
        st[a] = lf[a] + beta + vc / d;
        k += st[a];
        lsum += lf[a];
        lmag += lf[a] * lf[a];
    }
    T sh[3], qq = 0;
#pragma unroll
    for(int a = 0; a < d; a++) { sh[a] = st[a] - k / d; qq += sh[a] * sh[a]; }
    qq = sqrt(qq);
    const T r = rho_F * k / g, dg = qq + b * r;
    if(!(dg > 0)) return false;
    if(qq == 0 || k > 0) {
        const T e = sigma_Y != 0 ? exp(-beta) : (T)1;
#pragma unroll
        for(int a = 0; a < d; a++) strain[a] = e;
        if(prm[4] != 0) vc += lsum + beta * d;
        dp_hardening(q, rho_F, sqrt(lmag), prm);
        return true;
    }
    const T pp = r * b / qq;
#pragma unroll
    for(int a = 0; a < d; a++) strain[a] = exp(k / d - pp * sh[a] - beta);
    vc = 0;
    dp_hardening(q, rho_F, dg, prm);
    return true;
}

// MPM_PLASTICITY_MODEL::Update_Particles (MPM_PLASTICITY_MODEL.cpp:35-49) with
// Drucker-Prager on the signed SVD: F = U strain V^T, Fp = V strain^-1 U^T Fe Fp.
// `st` = q, rho_F, sigma_Y, vc.  Returns whether F and Fp changed.
template<class T, int d> __device__ bool plastic_dp(T* F, T* Fp, T mu, T la, T* st, const T* prm, bool& ok)
{
    T U[9], S[3], V[9], strain[3];
    ok = true;
    if(d == 3) ok = svd3<T>(F, U, S, V);
    else svd2<T>(F, U, S, V);
    if(!ok) return false;
    if(!dp_strain<T, d>(S, mu, la, st[0], st[1], st[2], st[3], prm, strain)) return false;
    T Fe[9], T1[9], T2[9];
#pragma unroll
    for(int k = 0; k < d * d; k++) Fe[k] = F[k];
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T f = 0, t = 0;
#pragma unroll
            for(int k = 0; k < d; k++) {
                f += U[r + d * k] * strain[k] * V[c + d * k];
                t += V[r + d * k] / strain[k] * U[c + d * k];
            }
            F[r + d * c] = f;
            T1[r + d * c] = t;
        }
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T s2 = 0;
#pragma unroll
            for(int k = 0; k < d; k++) s2 += T1[r + d * k] * Fe[k + d * c];
            T2[r + d * c] = s2;
        }
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T s2 = 0;
#pragma unroll
            for(int k = 0; k < d; k++) s2 += T2[r + d * k] * Fp[k + d * c];
            T1[r + d * c] = s2;
        }
#pragma unroll
    for(int k = 0; k < d * d; k++) Fp[k] = T1[k];
    return true;
}

}  // namespace mpm
