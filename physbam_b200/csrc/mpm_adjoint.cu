// Reverse-mode derivative of the explicit substep (3D; static frictionless
// collision objects), written by hand for the plain path's data layout.
//
// The reference has no reverse mode; its linearisations of the same maps are
// MPM_FINITE_ELEMENTS::Add_Hessian_Times (Hybrid_Methods/Forces/
// MPM_FINITE_ELEMENTS.cpp:103-132: gather, stress differential in the SVD
// frame, scatter) and MPM_OBJECTIVE::Update_F (System/MPM_OBJECTIVE.cpp:95-134).
// The stress differential is DIAGONALIZED_ISOTROPIC_STRESS_DERIVATIVE::
// Differential (Deformables/Constitutive_Models/DIAGONALIZED_ISOTROPIC_STRESS_
// DERIVATIVE.h:16-43) with the blocks of COROTATED_FIXED (COROTATED_FIXED.cpp:
// 144-167) and NEO_HOOKEAN (NEO_HOOKEAN.cpp:162ff); it is the Hessian of the
// energy density, a symmetric operator, so it is its own transpose.
//
// Substep (v_fric = v_new without friction):
//   m_i = sum w m_p,   p_i = sum w m_p (V + B D (Z_i - X)) - dt vol S g,   S = P(F) F^T
//   u_i = p_i / m_i + dt gravity,   v_i = C_i(u_i)   (collision projection)
//   V' = sum w v_i,  G = sum v_i g^T,  B' = sum w v_i (Z_i - X)^T,  F' = (I + dt G) F,  X' = X + dt V'
// with w = w_ip(X), g = dw_ip/dX, Hw = d^2 w_ip / dX^2, D = 4/dx^2.
// C_i applies the node's collisions in object order (MPM_OBJECTIVE::
// Test_Add_Collision, System/MPM_OBJECTIVE.cpp:150-183): a slip or
// separating object moves the node's end point X = X0 + dt u onto its surface,
// u <- u - (phi / dt) n, phi = Phi(X) - min(Phi(X0), 0), n = grad Phi(X), whose
// derivative is I - n n^T - phi Hess Phi(X) (symmetric); a sticking static
// object sets u = 0.  Which objects act is held fixed (the projection is
// differentiated where it acts), as for any piecewise-smooth map.
// Adjoint per substep, last to first:
//   adj_g2p  (per particle; the adjoint of the gather is a scatter to the grid)
//   adj_grid (per node)
//   adj_p2g  (per particle; the adjoint of the scatter is a gather), incl. the stress.
// The forward is recomputed segment by segment from checkpoints taken every k
// substeps; inside a segment each substep's particle state, grid mass and
// velocity and P F^T are kept.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include <algorithm>

#include "mpm_internal.h"

namespace {

using namespace mpm;

template<class T> struct AdjArgs {
    SceneParams sp;
    int64_t n, gn;
    int gs[3];
    const T *X, *V, *F, *B;        // state at the start of the substep
    const uint8_t* valid;
    const T *mass, *vol, *mu, *lam;
    const T* pft;                   // P F^T of the substep
    const T *gm, *gv;               // grid mass, velocity after the forces (v_new)
    const T* gu;                    // grid velocity before the collision projection (u)
    const T *aX1, *aV1, *aB1, *aF1; // adjoints of the substep's outputs
    T *aX0, *aV0, *aB0, *aF0;       // adjoints of its inputs
    T *amu, *alam;                  // accumulated over substeps
    T* ga;                          // grid: v-bar, then p-bar in place
    T* gma;                         // grid: m-bar
    T dt;
    unsigned* flags;
};

template<class T> struct Axis2 {
    int base;
    T w[3], dw[3], ddw[3];
};

template<class T> __device__ __forceinline__ Axis2<T> axis2(T X, T dmin, T dx, T inv)
{
    Axis<T> a = spline_axis<T>(X, dmin, dx, inv);
    Axis2<T> b;
    b.base = a.base;
#pragma unroll
    for(int o = 0; o < 3; o++) { b.w[o] = a.w[o]; b.dw[o] = a.dw[o]; }
    T i2 = inv * inv;
    b.ddw[0] = i2; b.ddw[1] = -2 * i2; b.ddw[2] = i2;
    return b;
}

template<class T> __device__ __forceinline__ bool stencil_ok(const AdjArgs<T>& a, const Axis2<T>* ax)
{
#pragma unroll
    for(int k = 0; k < 3; k++) {
        int lo = ax[k].base + MPM_GHOST;
        if(lo < 0 || lo + 2 >= a.gs[k]) return false;
    }
    return true;
}

// node q of the 27: flat index, weight, gradient, Hessian (row-major 3x3), offset Z - X
template<class T> __device__ __forceinline__ void node3(const AdjArgs<T>& a, const Axis2<T>* ax, const T* X, int q,
    int64_t& flat, T& w, T* g, T* H, T* d)
{
    int o[3] = {q / 9, (q / 3) % 3, q % 3};
    T wx = ax[0].w[o[0]], wy = ax[1].w[o[1]], wz = ax[2].w[o[2]];
    T dx = ax[0].dw[o[0]], dy = ax[1].dw[o[1]], dz = ax[2].dw[o[2]];
    T hx = ax[0].ddw[o[0]], hy = ax[1].ddw[o[1]], hz = ax[2].ddw[o[2]];
    w = wx * wy * wz;
    g[0] = dx * wy * wz; g[1] = wx * dy * wz; g[2] = wx * wy * dz;
    H[0] = hx * wy * wz; H[4] = wx * hy * wz; H[8] = wx * wy * hz;
    H[1] = H[3] = dx * dy * wz;
    H[2] = H[6] = dx * wy * dz;
    H[5] = H[7] = wx * dy * dz;
    flat = 0;
#pragma unroll
    for(int k = 0; k < 3; k++) {
        int idx = ax[k].base + o[k];
        flat = flat * a.gs[k] + (idx + MPM_GHOST);
        d[k] = (T)a.sp.dmin[k] + ((T)idx + (T).5) * (T)a.sp.dx[k] - X[k];
    }
}

template<class T> __global__ void k_adj_g2p(AdjArgs<T> a)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(p >= a.n) return;
    const T *aX1 = a.aX1 + 3 * p, *aV1 = a.aV1 + 3 * p, *aB1 = a.aB1 + 9 * p, *aF1 = a.aF1 + 9 * p;
    if(!a.valid[p]) {   // frozen particle: identity
        for(int k = 0; k < 3; k++) { a.aX0[3 * p + k] = aX1[k]; a.aV0[3 * p + k] = aV1[k]; }
        for(int k = 0; k < 9; k++) { a.aB0[9 * p + k] = aB1[k]; a.aF0[9 * p + k] = aF1[k]; }
        return;
    }
    const T* X = a.X + 3 * p;
    const T* F = a.F + 9 * p;
    Axis2<T> ax[3];
#pragma unroll
    for(int k = 0; k < 3; k++) ax[k] = axis2<T>(X[k], (T)a.sp.dmin[k], (T)a.sp.dx[k], (T)a.sp.inv_dx[k]);
    if(!stencil_ok(a, ax)) { atomicOr(a.flags, MPM_FLAG_DOMAIN); return; }
    // recompute G = sum v g^T
    T G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for(int q = 0; q < 27; q++) {
        int64_t i;
        T w, g[3], H[9], d[3];
        node3(a, ax, X, q, i, w, g, H, d);
        const T* v = a.gv + 3 * i;
#pragma unroll
        for(int c = 0; c < 3; c++)
#pragma unroll
            for(int r = 0; r < 3; r++) G[r + 3 * c] += v[r] * g[c];
    }
    // F' = (I + dt G) F  ->  F-bar = (I + dt G)^T F'-bar,  G-bar = dt F'-bar F^T
    T Fb[9], Gb[9];
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
        for(int r = 0; r < 3; r++) {
            T s = aF1[r + 3 * c], t = 0;
#pragma unroll
            for(int e = 0; e < 3; e++) {
                s += a.dt * G[e + 3 * r] * aF1[e + 3 * c];
                t += aF1[r + 3 * e] * F[c + 3 * e];
            }
            Fb[r + 3 * c] = s;
            Gb[r + 3 * c] = a.dt * t;
        }
    T Vt[3], Xb[3];
#pragma unroll
    for(int k = 0; k < 3; k++) { Vt[k] = aV1[k] + a.dt * aX1[k]; Xb[k] = aX1[k]; }
    for(int q = 0; q < 27; q++) {
        int64_t i;
        T w, g[3], H[9], d[3];
        node3(a, ax, X, q, i, w, g, H, d);
        const T* v = a.gv + 3 * i;
        T vb[3], u[3], Bd[3], BTv[3];
#pragma unroll
        for(int r = 0; r < 3; r++) {
            Bd[r] = aB1[r] * d[0] + aB1[r + 3] * d[1] + aB1[r + 6] * d[2];
            vb[r] = w * Vt[r] + Gb[r] * g[0] + Gb[r + 3] * g[1] + Gb[r + 6] * g[2] + w * Bd[r];
        }
#pragma unroll
        for(int c = 0; c < 3; c++) {
            u[c] = Gb[3 * c] * v[0] + Gb[3 * c + 1] * v[1] + Gb[3 * c + 2] * v[2];
            BTv[c] = aB1[3 * c] * v[0] + aB1[3 * c + 1] * v[1] + aB1[3 * c + 2] * v[2];
        }
        T s = v[0] * (Vt[0] + Bd[0]) + v[1] * (Vt[1] + Bd[1]) + v[2] * (Vt[2] + Bd[2]);
#pragma unroll
        for(int e = 0; e < 3; e++)
            Xb[e] += s * g[e] + H[3 * e] * u[0] + H[3 * e + 1] * u[1] + H[3 * e + 2] * u[2] - w * BTv[e];
#pragma unroll
        for(int r = 0; r < 3; r++) atomicAdd(a.ga + 3 * i + r, vb[r]);
    }
#pragma unroll
    for(int k = 0; k < 3; k++) a.aX0[3 * p + k] = Xb[k];
#pragma unroll
    for(int k = 0; k < 9; k++) a.aF0[9 * p + k] = Fb[k];
}

// The adjoint of a node's collision projection C(u): replay the projections
// to find which objects act and their normals, then apply the transposed
// (symmetric) derivatives in reverse object order to vb.
template<class T> __device__ void adj_collide(const AdjArgs<T>& a, int64_t i, const T* u, T* vb)
{
    int64_t r = i;
    int idx[3];
    for(int k = 2; k >= 0; k--) { idx[k] = (int)(r % a.gs[k]) - MPM_GHOST; r /= a.gs[k]; }
    T X0[3], v[3], J[MPM_MAX_OBJECTS][6];   // per acting object: symmetric derivative (xx yy zz xy xz yz)
    bool stick[MPM_MAX_OBJECTS];
    int ncol = 0;
    for(int k = 0; k < 3; k++) { X0[k] = (T)a.sp.dmin[k] + ((T)idx[k] + (T).5) * (T)a.sp.dx[k]; v[k] = u[k]; }
    for(int j = 0; j < a.sp.nobj; j++) {
        const DevObject& o = a.sp.objs[j];
        const T phi0 = object_phi<T, 3>(o, X0);
        if((o.type == MPM_STICK || o.type == MPM_SLIP) && phi0 > 0) continue;
        T X[3];
        for(int k = 0; k < 3; k++) X[k] = X0[k] + a.dt * v[k];
        const T phi = object_phi<T, 3>(o, X) - fmin(phi0, (T)0);
        if(o.type == MPM_SEPARATE && phi > (T)1e-15) continue;
        if(o.type != MPM_STICK && phi > (T)FLT_MAX) continue;
        T n[3], H[9];
        object_normal<T, 3>(o, X, n);
        object_hessian<T, 3>(o, X, H);
        J[ncol][0] = 1 - n[0] * n[0] - phi * H[0];
        J[ncol][1] = 1 - n[1] * n[1] - phi * H[4];
        J[ncol][2] = 1 - n[2] * n[2] - phi * H[8];
        J[ncol][3] = -n[0] * n[1] - phi * H[1];
        J[ncol][4] = -n[0] * n[2] - phi * H[2];
        J[ncol][5] = -n[1] * n[2] - phi * H[5];
        stick[ncol] = o.type == MPM_STICK;
        ncol++;
        for(int k = 0; k < 3; k++) v[k] -= phi * n[k] / a.dt;
        if(o.type == MPM_STICK)
            for(int k = 0; k < 3; k++) v[k] = 0;   // a static object's velocity
    }
    for(int c = ncol - 1; c >= 0; c--) {
        if(stick[c]) { vb[0] = vb[1] = vb[2] = 0; continue; }
        const T* M = J[c];
        const T x = M[0] * vb[0] + M[3] * vb[1] + M[4] * vb[2];
        const T y = M[3] * vb[0] + M[1] * vb[1] + M[5] * vb[2];
        const T z = M[4] * vb[0] + M[5] * vb[1] + M[2] * vb[2];
        vb[0] = x; vb[1] = y; vb[2] = z;
    }
}

template<class T> __global__ void k_adj_grid(AdjArgs<T> a)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.gn; i += (int64_t)gridDim.x * blockDim.x) {
        T m = a.gm[i];
        if(m == 0) { a.gma[i] = 0; continue; }
        T vb[3] = {a.ga[3 * i], a.ga[3 * i + 1], a.ga[3 * i + 2]};
        const T* u = a.gu + 3 * i;
        if(a.sp.nobj) adj_collide<T>(a, i, u, vb);
        T im = (T)1 / m, s = 0;
#pragma unroll
        for(int k = 0; k < 3; k++) {
            s += vb[k] * (u[k] - a.dt * (T)a.sp.gravity[k]);
            a.ga[3 * i + k] = vb[k] * im;
        }
        a.gma[i] = -s * im;
    }
}

// The grid velocity before the collision projection, as the grid update forms
// it: u = v0 + (dt / m) f.
template<class T> __global__ void k_grid_u(const T* gv0, const T* gf, const T* gm, T dt, int64_t gn, T* u)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < gn; i += (int64_t)gridDim.x * blockDim.x) {
        const T m = gm[i];
        const T s = m != 0 ? dt / m : (T)0;
        for(int k = 0; k < 3; k++) u[3 * i + k] = gv0[3 * i + k] + s * gf[3 * i + k];
    }
}

// Stress blocks in the SVD frame (the reference's Isotropic_Stress_Derivative_Helper)
// and dPhat/dmu, dPhat/dlambda.
__device__ void stress_blocks(int model, const double* s, double mu, double la, double* Hs, double* Bk, double* Ck,
    double* P, double* dPmu, double* dPla)
{
    double J = s[0] * s[1] * s[2];
    if(model == MPM_COROTATED_FIXED) {
        const double panic = 1e-6;
        double cof[3] = {s[1] * s[2], s[0] * s[2], s[0] * s[1]};
        double mu2 = 2 * mu;
        for(int k = 0; k < 3; k++) {
            P[k] = mu2 * (s[k] - 1) + la * (J - 1) * cof[k];
            dPmu[k] = 2 * (s[k] - 1);
            dPla[k] = (J - 1) * cof[k];
        }
        auto guard = [&](double x) { return fabs(x) < panic ? (x < 0 ? -panic : panic) : x; };
        double d01 = guard(s[0] + s[1]), d02 = guard(s[0] + s[2]), d12 = guard(s[1] + s[2]);
        Hs[0] = mu2 + la * cof[0] * cof[0]; Hs[4] = mu2 + la * cof[1] * cof[1]; Hs[8] = mu2 + la * cof[2] * cof[2];
        Hs[1] = Hs[3] = la * s[2] * (2 * J - 1);
        Hs[2] = Hs[6] = la * s[1] * (2 * J - 1);
        Hs[5] = Hs[7] = la * s[0] * (2 * J - 1);
        Ck[2] = mu2 / d01 + la * s[2] * (1 - J);
        Ck[1] = mu2 / d02 + la * s[1] * (1 - J);
        Ck[0] = mu2 / d12 + la * s[0] * (1 - J);
        Bk[2] = mu2 * (1 - 1 / d01);
        Bk[1] = mu2 * (1 - 1 / d02);
        Bk[0] = mu2 * (1 - 1 / d12);
        return;
    }
    // NEO_HOOKEAN, J >= threshold branch (NEO_HOOKEAN.cpp:73-82 and its 3D derivative helper)
    double Fi[3] = {1 / s[0], 1 / s[1], 1 / s[2]};
    double lJ = log(J);
    for(int k = 0; k < 3; k++) {
        P[k] = mu * s[k] - (mu - la * lJ) * Fi[k];
        dPmu[k] = s[k] - Fi[k];
        dPla[k] = lJ * Fi[k];
    }
    double mlj = mu + la * log(Fi[0] * Fi[1] * Fi[2]);
    Hs[0] = mu + (la + mlj) * Fi[0] * Fi[0];
    Hs[4] = mu + (la + mlj) * Fi[1] * Fi[1];
    Hs[8] = mu + (la + mlj) * Fi[2] * Fi[2];
    Hs[1] = Hs[3] = la * Fi[1] * Fi[0];
    Hs[2] = Hs[6] = la * Fi[2] * Fi[0];
    Hs[5] = Hs[7] = la * Fi[2] * Fi[1];
    Bk[0] = Bk[1] = Bk[2] = mu;
    Ck[2] = mlj * Fi[1] * Fi[0];
    Ck[1] = mlj * Fi[2] * Fi[0];
    Ck[0] = mlj * Fi[2] * Fi[1];
}

template<class T> __global__ void k_adj_p2g(AdjArgs<T> a)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(p >= a.n || !a.valid[p]) return;
    const T* X = a.X + 3 * p;
    const T* V = a.V + 3 * p;
    const T* Bm = a.B + 9 * p;
    const T* S = a.pft + 9 * p;
    const T m = a.mass[p], vol = a.vol[p];
    const T D = 4 * (T)a.sp.inv_dx[0] * (T)a.sp.inv_dx[0];
    Axis2<T> ax[3];
#pragma unroll
    for(int k = 0; k < 3; k++) ax[k] = axis2<T>(X[k], (T)a.sp.dmin[k], (T)a.sp.dx[k], (T)a.sp.inv_dx[k]);
    if(!stencil_ok(a, ax)) return;
    T Vb[3] = {0, 0, 0}, Bb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Sb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Xb[3] = {0, 0, 0};
    for(int q = 0; q < 27; q++) {
        int64_t i;
        T w, g[3], H[9], d[3];
        node3(a, ax, X, q, i, w, g, H, d);
        const T pb[3] = {a.ga[3 * i], a.ga[3 * i + 1], a.ga[3 * i + 2]};
        const T mb = a.gma[i];
        T mom[3], BTp[3], STp[3];
#pragma unroll
        for(int r = 0; r < 3; r++) mom[r] = m * (V[r] + D * (Bm[r] * d[0] + Bm[r + 3] * d[1] + Bm[r + 6] * d[2]));
#pragma unroll
        for(int c = 0; c < 3; c++) {
            BTp[c] = Bm[3 * c] * pb[0] + Bm[3 * c + 1] * pb[1] + Bm[3 * c + 2] * pb[2];
            STp[c] = S[3 * c] * pb[0] + S[3 * c + 1] * pb[1] + S[3 * c + 2] * pb[2];
        }
        T s = m * mb + pb[0] * mom[0] + pb[1] * mom[1] + pb[2] * mom[2];
#pragma unroll
        for(int e = 0; e < 3; e++)
            Xb[e] += s * g[e] - w * m * D * BTp[e] - a.dt * vol * (H[3 * e] * STp[0] + H[3 * e + 1] * STp[1] + H[3 * e + 2] * STp[2]);
#pragma unroll
        for(int r = 0; r < 3; r++) {
            Vb[r] += w * m * pb[r];
#pragma unroll
            for(int c = 0; c < 3; c++) {
                Bb[r + 3 * c] += w * m * D * pb[r] * d[c];
                Sb[r + 3 * c] -= a.dt * vol * pb[r] * g[c];
            }
        }
    }
    // stress adjoint through the SVD (FP64)
    double Fd[9], U[9], Vv[9], sg[3], Sbd[9];
#pragma unroll
    for(int k = 0; k < 9; k++) { Fd[k] = a.F[9 * p + k]; Sbd[k] = Sb[k]; }
    if(!svd3<double>(Fd, U, sg, Vv)) atomicOr(a.flags, MPM_FLAG_NOT_CONVERGED);
    double Hs[9], Bk[3], Ck[3], Ph[3], dPmu[3], dPla[3];
    stress_blocks(a.sp.model, sg, (double)a.mu[p], (double)a.lam[p], Hs, Bk, Ck, Ph, dPmu, dPla);
    // P = U Phat V^T ; Pbar = Sbar F ; Fbar += Sbar^T P + U Diff(U^T Pbar V) V^T
    double P[9], Pb[9], Fb[9];
    for(int c = 0; c < 3; c++)
        for(int r = 0; r < 3; r++) {
            double s = 0, t = 0;
            for(int e = 0; e < 3; e++) {
                s += U[r + 3 * e] * Ph[e] * Vv[c + 3 * e];
                t += Sbd[r + 3 * e] * Fd[e + 3 * c];
            }
            P[r + 3 * c] = s;
            Pb[r + 3 * c] = t;
        }
    double W[9], T1[9];   // W = U^T Pbar V
    for(int c = 0; c < 3; c++)
        for(int r = 0; r < 3; r++) {
            double s = 0;
            for(int e = 0; e < 3; e++) s += Pb[r + 3 * e] * Vv[e + 3 * c];
            T1[r + 3 * c] = s;
        }
    for(int c = 0; c < 3; c++)
        for(int r = 0; r < 3; r++) {
            double s = 0;
            for(int e = 0; e < 3; e++) s += U[e + 3 * r] * T1[e + 3 * c];
            W[r + 3 * c] = s;
        }
    double dW[9];
    dW[0] = Hs[0] * W[0] + Hs[1] * W[4] + Hs[2] * W[8];
    dW[4] = Hs[3] * W[0] + Hs[4] * W[4] + Hs[5] * W[8];
    dW[8] = Hs[6] * W[0] + Hs[7] * W[4] + Hs[8] * W[8];
    dW[1] = Bk[2] * W[1] + Ck[2] * W[3]; dW[3] = Ck[2] * W[1] + Bk[2] * W[3];
    dW[2] = Bk[1] * W[2] + Ck[1] * W[6]; dW[6] = Ck[1] * W[2] + Bk[1] * W[6];
    dW[5] = Bk[0] * W[5] + Ck[0] * W[7]; dW[7] = Ck[0] * W[5] + Bk[0] * W[7];
    for(int c = 0; c < 3; c++)
        for(int r = 0; r < 3; r++) {
            double s = 0;
            for(int e = 0; e < 3; e++) s += dW[r + 3 * e] * Vv[c + 3 * e];
            T1[r + 3 * c] = s;
        }
    for(int c = 0; c < 3; c++)
        for(int r = 0; r < 3; r++) {
            double s = 0, t = 0;
            for(int e = 0; e < 3; e++) {
                s += U[r + 3 * e] * T1[e + 3 * c];
                t += Sbd[e + 3 * r] * P[e + 3 * c];
            }
            Fb[r + 3 * c] = s + t;
        }
    // dS/dmu = U diag(dPhat/dmu * sigma) U^T (S = U Phat Sigma U^T); likewise lambda
    double bmu = 0, bla = 0;
    for(int k = 0; k < 3; k++) {
        double sk = 0;   // (U^T Sbar U)_kk
        for(int r = 0; r < 3; r++)
            for(int c = 0; c < 3; c++) sk += U[r + 3 * k] * Sbd[r + 3 * c] * U[c + 3 * k];
        bmu += sk * dPmu[k] * sg[k];
        bla += sk * dPla[k] * sg[k];
    }
#pragma unroll
    for(int k = 0; k < 3; k++) { a.aX0[3 * p + k] += Xb[k]; a.aV0[3 * p + k] = Vb[k]; }
#pragma unroll
    for(int k = 0; k < 9; k++) { a.aB0[9 * p + k] = Bb[k]; a.aF0[9 * p + k] += (T)Fb[k]; }
    a.amu[p] += (T)bmu;
    a.alam[p] += (T)bla;
}

template<class T> __global__ void k_zero(T* p, int64_t n)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = 0;
}

int blocks_for(mpm_handle* h, int64_t n, int t, bool cap)
{
    int64_t b = (n + t - 1) / t;
    if(cap && b > (int64_t)h->sm_count * 8) b = (int64_t)h->sm_count * 8;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

// State snapshot sizes (elements of T): X 3n, V 3n, F 9n, B 9n, valid n bytes.
struct DiffTape {
    bool recorded = false;           // holds the forward pass of the current particles
    int64_t n = 0, gn = 0;
    int nsteps = 0, every = 0;
    double dt = 0;
    size_t esz = 0;
    void* ckpt = nullptr;            // (nsteps/every + 1) states
    uint8_t* ckpt_valid = nullptr;
    bool full = false;               // every substep recorded by the forward (no recompute)
    void* seg = nullptr;             // every (or, full, nsteps) states
    uint8_t* seg_valid = nullptr;
    void *seg_gm = nullptr, *seg_gv = nullptr, *seg_gu = nullptr, *seg_pft = nullptr;
    void* final_state = nullptr;
    uint8_t* final_valid = nullptr;
    void *adj[2] = {nullptr, nullptr};   // X V F B adjoints, double-buffered
    void *amu = nullptr, *alam = nullptr, *ga = nullptr, *gma = nullptr;
};

static DiffTape* tape(mpm_handle* h) { return reinterpret_cast<DiffTape*>(h->diff); }

// New particles: the recorded rollout no longer applies; its buffers are kept
// for the next mpm_diff_forward of the same shape.
void diff_invalidate(mpm_handle* h)
{
    DiffTape* t = tape(h);
    if(t) t->recorded = false;
}

void diff_free(mpm_handle* h)
{
    DiffTape* t = tape(h);
    if(!t) return;
    void* ps[] = {t->ckpt, t->ckpt_valid, t->seg, t->seg_valid, t->seg_gm, t->seg_gv, t->seg_gu, t->seg_pft, t->final_state,
                  t->final_valid, t->adj[0], t->adj[1], t->amu, t->alam, t->ga, t->gma};
    for(void* p: ps) cudaFree(p);
    delete t;
    h->diff = nullptr;
}

static int state_copy(mpm_handle* h, void* dst, uint8_t* dvalid, bool to_tape)
{
    PlainState& s = h->plain;
    size_t e = h->model.precision == MPM_FP64 ? 8 : 4;
    int64_t n = s.n;
    char* d = (char*)dst;
    void* parts[4] = {s.X, s.V, s.F, s.B};
    int64_t cnt[4] = {3 * n, 3 * n, 9 * n, 9 * n};
    for(int k = 0; k < 4; k++) {
        if(to_tape) MPM_CUDA(h, cudaMemcpyAsync(d, parts[k], cnt[k] * e, cudaMemcpyDeviceToDevice, h->stream));
        else MPM_CUDA(h, cudaMemcpyAsync(parts[k], d, cnt[k] * e, cudaMemcpyDeviceToDevice, h->stream));
        d += cnt[k] * e;
    }
    if(to_tape) MPM_CUDA(h, cudaMemcpyAsync(dvalid, s.valid, n, cudaMemcpyDeviceToDevice, h->stream));
    else MPM_CUDA(h, cudaMemcpyAsync(s.valid, dvalid, n, cudaMemcpyDeviceToDevice, h->stream));
    return MPM_OK;
}

// One substep of the rollout with its intermediates into tape slot j: the
// state before it, the node masses and velocities after the forces, the grid
// update's velocity map (k_grid_u) and P F^T; `advance`: the G2P that ends it.
template<class T> static int record_substep(mpm_handle* h, DiffTape* t, int j, bool advance)
{
    PlainState& s = h->plain;
    const int64_t n = t->n, gn = t->gn;
    const size_t e = sizeof(T), st = 24 * n * e;
    int rc;
    if((rc = state_copy(h, (char*)t->seg + j * st, t->seg_valid + j * n, true))) return rc;
    if((rc = plain_p2g(h, t->dt, 0))) return rc;
    if((rc = plain_forces(h, t->dt, 0))) return rc;
    MPM_CUDA(h, cudaMemcpyAsync((T*)t->seg_gm + j * gn, s.gm, gn * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync((T*)t->seg_gv + j * gn * 3, s.gv, gn * 3 * e, cudaMemcpyDeviceToDevice, h->stream));
    k_grid_u<T><<<blocks_for(h, gn, 256, true), 256, 0, h->stream>>>((const T*)s.gv0, (const T*)s.gf, (const T*)s.gm,
                                                                   (T)t->dt, gn, (T*)t->seg_gu + j * gn * 3);
    MPM_LAUNCHED(h, "k_grid_u");
    MPM_CUDA(h, cudaMemcpyAsync((T*)t->seg_pft + j * 9 * n, s.pft, 9 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    if(advance && (rc = plain_g2p(h, t->dt, 0))) return rc;
    return MPM_OK;
}

// Tape slots for `slots` substeps (the segment buffers the backward reads).
static int alloc_segments(mpm_handle* h, DiffTape* t, int slots)
{
    const int64_t n = t->n, gn = t->gn;
    const size_t e = t->esz, st = 24 * n * e;
    MPM_CUDA(h, cudaMalloc(&t->seg, slots * st + 1));
    MPM_CUDA(h, cudaMalloc(&t->seg_valid, slots * n + 1));
    MPM_CUDA(h, cudaMalloc(&t->seg_gm, slots * gn * e));
    MPM_CUDA(h, cudaMalloc(&t->seg_gv, slots * gn * 3 * e));
    MPM_CUDA(h, cudaMalloc(&t->seg_gu, slots * gn * 3 * e));
    MPM_CUDA(h, cudaMalloc(&t->seg_pft, slots * 9 * n * e + 1));
    return MPM_OK;
}

// Bytes of the tape slots of one substep.
static size_t slot_bytes(int64_t n, int64_t gn, size_t e) { return (24 * n + 9 * n) * e + n + 7 * gn * e; }

int diff_forward(mpm_handle* h, double dt, int nsteps, int every)
{
    if(h->model.path != MPM_PATH_PLAIN || h->sp.dim != 3)
        return set_error(h, MPM_ERR_ARG, "the adjoint runs on the 3D plain path");
    if(h->sp.npen) return set_error(h, MPM_ERR_ARG, "the adjoint does not differentiate penalty collision objects");
    if(h->moving) return set_error(h, MPM_ERR_ARG, "the adjoint differentiates static collision objects");
    for(int j = 0; j < h->sp.nobj; j++)
        if(h->sp.objs[j].friction != 0)
            return set_error(h, MPM_ERR_ARG, "the adjoint differentiates frictionless collision objects");
    if(h->reflect.enabled) return set_error(h, MPM_ERR_ARG, "the adjoint does not differentiate reflection boundaries");
    if(h->plastic.kind) return set_error(h, MPM_ERR_ARG, "the adjoint does not differentiate plasticity");
    if(h->plain.pmodel) return set_error(h, MPM_ERR_ARG, "the adjoint takes one constitutive model");
    if(h->implicit.enabled) return set_error(h, MPM_ERR_ARG, "the adjoint differentiates the explicit substep");
    if(h->sp.model == MPM_STVK_HENCKY) return set_error(h, MPM_ERR_ARG, "the adjoint covers COROTATED_FIXED and NEO_HOOKEAN");
    if(nsteps < 1 || every < 1) return set_error(h, MPM_ERR_ARG, "nsteps and checkpoint interval must be >= 1");
    PlainState& s = h->plain;
    const size_t esz = h->model.precision == MPM_FP64 ? 8 : 4;
    DiffTape* t = tape(h);
    // every substep's intermediates kept when the tape budget allows (by default
    // a quarter of the free device memory): the backward then recomputes nothing
    size_t free_b = 0, total_b = 0;
    if(cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    const double budget = h->diff_budget < 0 ? 0.25 * (double)free_b : std::min((double)h->diff_budget, 0.9 * (double)free_b);
    const bool want_full = nsteps > every && (double)slot_bytes(s.n, s.gn, esz) * nsteps <= budget;
    // a tape of the same shape is reused as it is (no allocation)
    const bool reuse = t && t->n == s.n && t->gn == s.gn && t->nsteps == nsteps && t->every == every && t->esz == esz &&
                       t->full == want_full;
    if(!reuse) {
        diff_free(h);
        t = new DiffTape();
        h->diff = t;
        t->n = s.n; t->gn = s.gn; t->nsteps = nsteps; t->every = every;
        t->esz = esz;
        t->full = want_full;
        if(t->full) {
            int arc = alloc_segments(h, t, nsteps);
            if(arc) return arc;
        }
    }
    t->recorded = false;
    t->dt = dt;
    size_t st = 24 * s.n * t->esz;
    int nck = (nsteps + every - 1) / every;
    if(!reuse) {
        MPM_CUDA(h, cudaMalloc(&t->ckpt, nck * st + 1));
        MPM_CUDA(h, cudaMalloc(&t->ckpt_valid, nck * s.n + 1));
        MPM_CUDA(h, cudaMalloc(&t->final_state, st + 1));
        MPM_CUDA(h, cudaMalloc(&t->final_valid, s.n + 1));
    }
    int rc;
    for(int k = 0; k < nsteps; k++) {
        if(t->full) {
            rc = esz == 8 ? record_substep<double>(h, t, k, true) : record_substep<float>(h, t, k, true);
            if(rc) return rc;
            continue;
        }
        if(k % every == 0) {
            int c = k / every;
            if((rc = state_copy(h, (char*)t->ckpt + c * st, t->ckpt_valid + c * s.n, true))) return rc;
        }
        if((rc = plain_p2g(h, dt, 0))) return rc;
        if((rc = plain_forces(h, dt, 0))) return rc;
        if((rc = plain_g2p(h, dt, 0))) return rc;
    }
    if((rc = state_copy(h, t->final_state, t->final_valid, true))) return rc;
    t->recorded = true;
    return MPM_OK;
}

template<class T> static int backward_t(mpm_handle* h, const void* gX, const void* gV, const void* gF, const void* gB,
    void* oX, void* oV, void* oF, void* oB, void* omu, void* olam)
{
    DiffTape* t = tape(h);
    PlainState& s = h->plain;
    const int64_t n = t->n, gn = t->gn;
    const size_t e = sizeof(T);
    const size_t st = 24 * n * e;
    const int every = t->every;
    if(!t->seg) {
        int arc = alloc_segments(h, t, every);
        if(arc) return arc;
    }
    if(!t->adj[0]) {
        for(int k = 0; k < 2; k++) MPM_CUDA(h, cudaMalloc(&t->adj[k], st + 1));
        MPM_CUDA(h, cudaMalloc(&t->amu, n * e + 1));
        MPM_CUDA(h, cudaMalloc(&t->alam, n * e + 1));
        MPM_CUDA(h, cudaMalloc(&t->ga, gn * 3 * e));
        MPM_CUDA(h, cudaMalloc(&t->gma, gn * e));
    }
    // seed: adjoint of the final state (device arrays of T)
    T* a1 = (T*)t->adj[0];
    T* a0 = (T*)t->adj[1];
    MPM_CUDA(h, cudaMemcpyAsync(a1, gX, 3 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(a1 + 3 * n, gV, 3 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(a1 + 6 * n, gF, 9 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(a1 + 15 * n, gB, 9 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemsetAsync(t->amu, 0, n * e, h->stream));
    MPM_CUDA(h, cudaMemsetAsync(t->alam, 0, n * e, h->stream));
    const int tb = 128;
    // a full tape is one segment, recorded by the forward; otherwise each
    // checkpoint's segment is recomputed from it, keeping what the adjoint needs
    const int nck = t->full ? 1 : (t->nsteps + every - 1) / every;
    const int span = t->full ? t->nsteps : every;
    int rc;
    for(int c = nck - 1; c >= 0; c--) {
        int k0 = c * span, k1 = k0 + span < t->nsteps ? k0 + span : t->nsteps;
        if(!t->full) {
            if((rc = state_copy(h, (char*)t->ckpt + c * st, t->ckpt_valid + c * n, false))) return rc;
            for(int k = k0; k < k1; k++)
                if((rc = record_substep<T>(h, t, k - k0, k + 1 < k1))) return rc;
        }
        for(int k = k1 - 1; k >= k0; k--) {
            int j = k - k0;
            const T* base = (const T*)((char*)t->seg + j * st);
            AdjArgs<T> a;
            a.sp = h->sp;
            a.n = n; a.gn = gn;
            for(int q = 0; q < 3; q++) a.gs[q] = h->sp.counts[q] + 2 * MPM_GHOST;
            a.X = base; a.V = base + 3 * n; a.F = base + 6 * n; a.B = base + 15 * n;
            a.valid = t->seg_valid + j * n;
            a.mass = (const T*)s.mass; a.vol = (const T*)s.vol; a.mu = (const T*)s.mu; a.lam = (const T*)s.lam;
            a.pft = (const T*)t->seg_pft + j * 9 * n;
            a.gm = (const T*)t->seg_gm + j * gn;
            a.gv = (const T*)t->seg_gv + j * gn * 3;
            a.gu = (const T*)t->seg_gu + j * gn * 3;
            a.aX1 = a1; a.aV1 = a1 + 3 * n; a.aF1 = a1 + 6 * n; a.aB1 = a1 + 15 * n;
            a.aX0 = a0; a.aV0 = a0 + 3 * n; a.aF0 = a0 + 6 * n; a.aB0 = a0 + 15 * n;
            a.amu = (T*)t->amu; a.alam = (T*)t->alam;
            a.ga = (T*)t->ga; a.gma = (T*)t->gma;
            a.dt = (T)t->dt;
            a.flags = h->d_flags;
            int slot = timer_begin(h, "adj_zero");
            k_zero<T><<<blocks_for(h, gn * 3, 256, true), 256, 0, h->stream>>>(a.ga, gn * 3);
            timer_end(h, slot);
            MPM_LAUNCHED(h, "k_zero");
            slot = timer_begin(h, "adj_g2p");
            k_adj_g2p<T><<<blocks_for(h, n, tb, false), tb, 0, h->stream>>>(a);
            timer_end(h, slot);
            MPM_LAUNCHED(h, "k_adj_g2p");
            slot = timer_begin(h, "adj_grid");
            k_adj_grid<T><<<blocks_for(h, gn, 256, true), 256, 0, h->stream>>>(a);
            timer_end(h, slot);
            MPM_LAUNCHED(h, "k_adj_grid");
            slot = timer_begin(h, "adj_p2g");
            k_adj_p2g<T><<<blocks_for(h, n, tb, false), tb, 0, h->stream>>>(a);
            timer_end(h, slot);
            MPM_LAUNCHED(h, "k_adj_p2g");
            T* tmp = a1; a1 = a0; a0 = tmp;
        }
    }
    // a1 now holds the adjoint of the initial state
    MPM_CUDA(h, cudaMemcpyAsync(oX, a1, 3 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(oV, a1 + 3 * n, 3 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(oF, a1 + 6 * n, 9 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(oB, a1 + 15 * n, 9 * n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(omu, t->amu, n * e, cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(olam, t->alam, n * e, cudaMemcpyDeviceToDevice, h->stream));
    // leave the handle at the final state again
    return state_copy(h, t->final_state, t->final_valid, false);
}

// grad views: X, V, F, B of n particles in the reference layout, device or host,
// dtype must equal the path's precision.
int diff_backward(mpm_handle* h, const mpm_particles_view* gout, mpm_particles_view* gin, void* gmu, void* glam)
{
    DiffTape* t = tape(h);
    if(!t || !t->recorded) return set_error(h, MPM_ERR_STATE, "mpm_diff_backward needs a recorded mpm_diff_forward");
    int prec = h->model.precision;
    if(gout->n != t->n || gin->n != t->n) return set_error(h, MPM_ERR_ARG, "particle count");
    if(gout->dtype != prec || gin->dtype != prec) return set_error(h, MPM_ERR_ARG, "gradient dtype must match the path precision");
    if(!gout->X || !gout->V || !gout->F || !gout->B || !gin->X || !gin->V || !gin->F || !gin->B || !gmu || !glam)
        return set_error(h, MPM_ERR_ARG, "null gradient array");
    const size_t e = prec == MPM_FP64 ? 8 : 4;
    const int64_t n = t->n;
    // stage host arrays
    const void* src[4] = {gout->X, gout->V, gout->F, gout->B};
    int64_t cnt[6] = {3 * n, 3 * n, 9 * n, 9 * n, n, n};
    void* dsrc[4];
    void* dout[6];
    std::vector<void*> owned;
    for(int k = 0; k < 4; k++) {
        if(gout->on_device) dsrc[k] = const_cast<void*>(src[k]);
        else {
            MPM_CUDA(h, cudaMallocAsync(&dsrc[k], cnt[k] * e + 1, h->stream));
            owned.push_back(dsrc[k]);
            MPM_CUDA(h, cudaMemcpyAsync(dsrc[k], src[k], cnt[k] * e, cudaMemcpyHostToDevice, h->stream));
        }
    }
    void* dst[6] = {gin->X, gin->V, gin->F, gin->B, gmu, glam};
    for(int k = 0; k < 6; k++) {
        if(gin->on_device) dout[k] = dst[k];
        else {
            MPM_CUDA(h, cudaMallocAsync(&dout[k], cnt[k] * e + 1, h->stream));
            owned.push_back(dout[k]);
        }
    }
    int rc = prec == MPM_FP64 ? backward_t<double>(h, dsrc[0], dsrc[1], dsrc[2], dsrc[3], dout[0], dout[1], dout[2], dout[3], dout[4], dout[5])
                              : backward_t<float>(h, dsrc[0], dsrc[1], dsrc[2], dsrc[3], dout[0], dout[1], dout[2], dout[3], dout[4], dout[5]);
    if(rc) return rc;
    if(!gin->on_device)
        for(int k = 0; k < 6; k++) MPM_CUDA(h, cudaMemcpyAsync(dst[k], dout[k], cnt[k] * e, cudaMemcpyDeviceToHost, h->stream));
    for(void* p: owned) MPM_CUDA(h, cudaFreeAsync(p, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

// This module's copy of the SVD sweep bound (mpm_debug_set_svd_iterations).
MPM_SVD_LIMIT_SETTER(svd_limit_adjoint)
