// Backward-Euler force solve of the plain path: the reference's default
// Apply_Forces when use_symplectic_euler is off (MPM_DRIVER.cpp:1024-1048).
//
// Newton's method (Tools/Nonlinear_Equations/NEWTONS_METHOD.cpp:20-85) on
// MPM_OBJECTIVE (Hybrid_Methods/System/MPM_OBJECTIVE.cpp) over the grid
// velocity increments dv of the nodes with mass, with the mass-weighted inner
// product and Hessian of MPM_KRYLOV_SYSTEM (MPM_KRYLOV_SYSTEM.cpp:40-95),
// conjugate gradients (Tools/Krylov_Solvers/CONJUGATE_GRADIENT.cpp:20-85) and
// the strong-Wolfe line search (Tools/Nonlinear_Equations/LINE_SEARCH.cpp:188-250),
// with NEWTONS_METHOD's default flags as MPM_DRIVER sets them.  The device
// does every grid and particle pass (the force and Hessian scatters are those
// of MPM_FINITE_ELEMENTS, Add_Forces / Add_Hessian_Times, l.84-132); the host
// runs the Newton / CG / line-search control flow, reading back one or two
// reduced scalars per step (deterministic two-stage reductions in FP64).
//
// Collision objects are the static boxes, planes and spheres of the explicit
// path; the curvature terms of the projection use the Hessian of the signed
// distance at the tested position.  A node's collisions are kept per object,
// in object order (the reference appends them per node in that order).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "mpm_internal.h"
#include "mpm_plain.cuh"

namespace {

using namespace mpm;
using namespace plain;

constexpr int kRedBlocks = 256, kRedThreads = 256;
constexpr double kCollisionThickness = 1e-15;   // MPM_OBJECTIVE::collision_thickness

template<class T> struct ImpArgs {
    PlainArgs<T> a;
    T *F0, *X0;                 // particle state at the start of the step (Fn = F0)
    T *U, *FV, *sig, *dP;       // SVD of the current F: U, Fn V, singular values, stress derivative (9 + 3 + 3)
    double* pe;                 // per-particle potential energy
    uint8_t *cmask, *stuck;     // per node: collision objects (bit j), stuck flag
    T* cdat;                    // per node and object: phi, n_dE, normal, position, H g (2 + 3d)
    T* pen;                     // per particle: penalty force (d) and Hessian (d x d) at the current X
    T* svel;                    // per node: the velocity of the sticky object holding it (stuck_velocity)
    int nobj;
    const uint32_t* order;      // particles sorted by cell (the passes visit them in this order)
};

// The t-th particle of a pass: neighbours in the grid run in neighbouring
// threads, so the stencil gathers and the atomic scatters stay in cache.
template<class T> __device__ __forceinline__ int64_t particle_at(const ImpArgs<T>& ia, int64_t t)
{
    return ia.order ? (int64_t)ia.order[t] : t;
}

// Sort key of a particle: the flat index of its stencil's first node; invalid
// particles and stencils outside the grid go last.
template<class T, int d> __global__ void k_imp_keys(ImpArgs<T> ia, uint32_t* keys)
{
    const PlainArgs<T>& a = ia.a;
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        uint32_t k = 0xffffffffu;
        Stencil<T, d> s;
        if(a.valid[p] && make_stencil<T, d>(a, a.X + p * d, s)) {
            int64_t flat = 0;
            for(int c = 0; c < d; c++) flat = flat * a.gs[c] + (s.base[c] + MPM_GHOST);
            k = (uint32_t)flat;
        }
        keys[p] = k;
    }
}

template<class T, int d> __device__ __forceinline__ bool node_valid(const ImpArgs<T>& ia, int64_t i) { return ia.a.gm[i] != 0; }

template<class T, int d> __device__ __forceinline__ void node_position(const ImpArgs<T>& ia, int64_t i, T* X)
{
    int64_t r = i;
    for(int k = d - 1; k >= 0; k--) {
        const int idx = (int)(r % ia.a.gs[k]) - MPM_GHOST;
        r /= ia.a.gs[k];
        X[k] = (T)ia.a.sp.dmin[k] + ((T)idx + (T).5) * (T)ia.a.sp.dx[k];
    }
}

// ---------------------------------------------------------------------------
// particle passes (weights of the particle positions at the start of the step)
// ---------------------------------------------------------------------------
template<class T, int d> __global__ void k_imp_save(ImpArgs<T> ia)
{
    const PlainArgs<T>& a = ia.a;
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        for(int e = 0; e < d * d; e++) ia.F0[p * d * d + e] = a.F[p * d * d + e];
        for(int e = 0; e < d; e++) ia.X0[p * d + e] = a.X[p * d + e];
    }
}

// MPM_OBJECTIVE::Restore_F
template<class T, int d> __global__ void k_imp_restore(ImpArgs<T> ia)
{
    const PlainArgs<T>& a = ia.a;
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        for(int e = 0; e < d * d; e++) a.F[p * d * d + e] = ia.F0[p * d * d + e];
        for(int e = 0; e < d; e++) a.X[p * d + e] = ia.X0[p * d + e];
    }
}

// MPM_OBJECTIVE::Update_F (l.96-131): F = (I + dt grad v) F0, X = X0 + dt V_p.
template<class T, int d> __global__ void k_imp_update_F(ImpArgs<T> ia, const T* v)
{
    const PlainArgs<T>& a = ia.a;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(t >= a.n) return;
    const int64_t p = particle_at(ia, t);
    if(!a.valid[p]) return;
    Stencil<T, d> s;
    if(!make_stencil<T, d>(a, ia.X0 + p * d, s)) return;
    T Vp[3] = {0, 0, 0}, G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int nq = d == 3 ? 27 : 9;
    for(int q = 0; q < nq; q++) {
        int64_t i;
        T w, g[3], Z[3];
        node<T, d>(a, s, q, i, w, g, Z);
#pragma unroll
        for(int r = 0; r < d; r++) {
            const T vr = v[i * d + r];
            Vp[r] += w * vr;
#pragma unroll
            for(int c = 0; c < d; c++) G[r + d * c] += vr * g[c];
        }
    }
    const T* F0 = ia.F0 + p * d * d;
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = F0[r + d * c];
#pragma unroll
            for(int k = 0; k < d; k++) sum += a.dt * G[r + d * k] * F0[k + d * c];
            a.F[p * d * d + r + d * c] = sum;
        }
#pragma unroll
    for(int r = 0; r < d; r++) a.X[p * d + r] = ia.X0[p * d + r] + a.dt * Vp[r];
}

// MPM_FINITE_ELEMENTS::Precompute (l.47-67) on the current F with Fn = F0, the
// stress derivative, and the potential energy of the particle (Energy_Density
// times volume, l.71-80, plus MPM_GRAVITY::Potential_Energy, MPM_GRAVITY.cpp:48-57).
template<class T, int d> __global__ void k_imp_precompute(ImpArgs<T> ia)
{
    const PlainArgs<T>& a = ia.a;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(t >= a.n) return;
    const int64_t p = particle_at(ia, t);
    // IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES::Update_Position_Based_State
    // runs over every particle, simulated or not (its energy counts them all).
    double epen = 0;
    if(a.sp.npen) {
        T fp[3] = {0, 0, 0}, Hp[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        epen = (double)penalty_particle<T, d>(a.sp.pen, a.sp.npen, (T)a.sp.pen_stiffness, (T)a.sp.pen_separation,
                                              a.X + p * d, fp, Hp);
        T* q = ia.pen + p * (d + d * d);
        for(int e = 0; e < d; e++) q[e] = fp[e];
        for(int e = 0; e < d * d; e++) q[d + e] = Hp[e];
    }
    if(!a.valid[p]) { ia.pe[p] = epen; return; }
    T F[9], U[9], V[9], S[3], P[3];
#pragma unroll
    for(int e = 0; e < d * d; e++) F[e] = a.F[p * d * d + e];
    bool ok = true;
    if(d == 3) ok = svd3<T>(F, U, S, V);
    else svd2<T>(F, U, S, V);
    if(!ok) atomicOr(a.flags, MPM_FLAG_NOT_CONVERGED);
    const T mu = a.mu[p], la = a.lam[p];
    const int model = model_of(a, p);
    phat<T, d>(model, S, mu, la, P);
    const T* F0 = ia.F0 + p * d * d;
    T FV[9];
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int k = 0; k < d; k++) sum += F0[r + d * k] * V[k + d * c];
            FV[r + d * c] = sum;
        }
    // PFT = U Phat FV^T
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int k = 0; k < d; k++) sum += U[r + d * k] * P[k] * FV[c + d * k];
            a.pft[p * d * d + r + d * c] = sum;
        }
    T H[9], Bv[3], Cv[3];
    stress_derivative<T, d>(model, S, mu, la, H, Bv, Cv);
    for(int e = 0; e < d * d; e++) { ia.U[p * d * d + e] = U[e]; ia.FV[p * d * d + e] = FV[e]; }
    for(int e = 0; e < d; e++) ia.sig[p * d + e] = S[e];
    for(int e = 0; e < 9; e++) ia.dP[p * 15 + e] = H[e];
    for(int e = 0; e < 3; e++) { ia.dP[p * 15 + 9 + e] = Bv[e]; ia.dP[p * 15 + 12 + e] = Cv[e]; }
    double e = (double)a.vol[p] * (double)energy_density<T, d>(model, S, mu, la);
    for(int k = 0; k < d; k++) e -= (double)a.mass[p] * (double)a.X[p * d + k] * a.sp.gravity[k];
    ia.pe[p] = e + epen;
}

// MPM_FINITE_ELEMENTS::Add_Forces (l.84-99) + MPM_GRAVITY::Add_Forces (l.62-68)
// + the penalty forces of MPM_EXAMPLE::Add_Forces (MPM_EXAMPLE.cpp:139-153).
template<class T, int d> __global__ void k_imp_forces(ImpArgs<T> ia, T* f)
{
    const PlainArgs<T>& a = ia.a;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(t >= a.n) return;
    const int64_t p = particle_at(ia, t);
    if(!a.valid[p]) return;
    Stencil<T, d> s;
    if(!make_stencil<T, d>(a, ia.X0 + p * d, s)) return;
    T A[9];
#pragma unroll
    for(int e = 0; e < d * d; e++) A[e] = a.pft[p * d * d + e] * a.vol[p];
    const T mp = a.mass[p];
    T fp[3] = {0, 0, 0};
    if(a.sp.npen)
        for(int e = 0; e < d; e++) fp[e] = ia.pen[p * (d + d * d) + e];
    const int nq = d == 3 ? 27 : 9;
    for(int q = 0; q < nq; q++) {
        int64_t i;
        T w, g[3], Z[3];
        node<T, d>(a, s, q, i, w, g, Z);
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int c = 0; c < d; c++) sum += A[r + d * c] * g[c];
            atomicAdd(f + i * d + r, -sum + w * mp * (T)a.sp.gravity[r] + w * fp[r]);
        }
    }
}

// MPM_FINITE_ELEMENTS::Add_Hessian_Times (l.103-132): W = sum z_i grad w_i^T,
// M = U dPhat(U^T W FV) FV^T vol, f_i += M grad w_i; with penalty objects also
// MPM_EXAMPLE::Add_Hessian_Times' Lagrangian part (MPM_EXAMPLE.cpp:157-177):
// z_p = sum w_i z_i, f_i += w_i H_p z_p.
template<class T, int d> __global__ void k_imp_hessian(ImpArgs<T> ia, const T* z, T* f)
{
    const PlainArgs<T>& a = ia.a;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(t >= a.n) return;
    const int64_t p = particle_at(ia, t);
    if(!a.valid[p]) return;
    Stencil<T, d> s;
    if(!make_stencil<T, d>(a, ia.X0 + p * d, s)) return;
    T W[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, zp[3] = {0, 0, 0};
    const bool pen = a.sp.npen != 0;
    const int nq = d == 3 ? 27 : 9;
    for(int q = 0; q < nq; q++) {
        int64_t i;
        T w, g[3], Z[3];
        node<T, d>(a, s, q, i, w, g, Z);
#pragma unroll
        for(int r = 0; r < d; r++) {
#pragma unroll
            for(int c = 0; c < d; c++) W[r + d * c] += z[i * d + r] * g[c];
            if(pen) zp[r] += w * z[i * d + r];
        }
    }
    T Hz[3] = {0, 0, 0};
    if(pen) {
        const T* Hp = ia.pen + p * (d + d * d) + d;
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int c = 0; c < d; c++) sum += Hp[r + d * c] * zp[c];
            Hz[r] = sum;
        }
    }
    const T* U = ia.U + p * d * d;
    const T* FV = ia.FV + p * d * d;
    T WF[9], G[9], dPh[9], UD[9], M[9];
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int k = 0; k < d; k++) sum += W[r + d * k] * FV[k + d * c];
            WF[r + d * c] = sum;
        }
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int k = 0; k < d; k++) sum += U[k + d * r] * WF[k + d * c];
            G[r + d * c] = sum;
        }
    const T* blk = ia.dP + p * 15;
    stress_differential<T, d>(blk, blk + 9, blk + 12, G, dPh);
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int k = 0; k < d; k++) sum += U[r + d * k] * dPh[k + d * c];
            UD[r + d * c] = sum;
        }
    const T vol = a.vol[p];
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int k = 0; k < d; k++) sum += UD[r + d * k] * FV[c + d * k];
            M[r + d * c] = sum * vol;
        }
    for(int q = 0; q < nq; q++) {
        int64_t i;
        T w, g[3], Z[3];
        node<T, d>(a, s, q, i, w, g, Z);
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int c = 0; c < d; c++) sum += M[r + d * c] * g[c];
            atomicAdd(f + i * d + r, sum + w * Hz[r]);
        }
    }
}

// ---------------------------------------------------------------------------
// node passes (nodes with mass: MPM_EXAMPLE::valid_grid_indices)
// ---------------------------------------------------------------------------
#define NODE_LOOP(ia) \
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (ia).a.gn; i += (int64_t)gridDim.x * blockDim.x) \
        if(node_valid<T, d>(ia, i))

// MPM_KRYLOV_VECTOR::Copy: out = c x + y (y may be null)
template<class T, int d> __global__ void k_imp_copy(ImpArgs<T> ia, T* out, T c, const T* x, const T* y)
{
    NODE_LOOP(ia) {
        for(int k = 0; k < d; k++) out[i * d + k] = c * x[i * d + k] + (y ? y[i * d + k] : (T)0);
    }
}

// gradient of MPM_OBJECTIVE::Compute_Unconstrained (l.71-91): g = dv - dt/m f
template<class T, int d> __global__ void k_imp_grad(ImpArgs<T> ia, T* g, const T* dv, const T* f)
{
    NODE_LOOP(ia) {
        const T s = ia.a.dt / ia.a.gm[i];
        for(int k = 0; k < d; k++) g[i * d + k] = dv[i * d + k] - s * f[i * d + k];
    }
}

// MPM_OBJECTIVE::Adjust_For_Collision (l.180-222) with Test_Add_Collision
// (l.143-176), prune and stick on, objects in order: each test moves dv of
// the node onto the object (or to the object's velocity for a sticky one) and
// records the collision; an earlier object's projection feeds the next one's
// test.  A moving object is tested at its frames of the substep's start and end.
template<class T, int d> __global__ void k_imp_adjust(ImpArgs<T> ia, T* dv)
{
    NODE_LOOP(ia) {
        const PlainArgs<T>& a = ia.a;
        uint8_t mask = 0, stuck = 0;
        T X0[3];
        node_position<T, d>(ia, i, X0);
        for(int j = 0; j < ia.nobj; j++) {
            const DevObject& o = a.sp.objs[j];
            T V[3], X[3];
#pragma unroll
            for(int k = 0; k < d; k++) { V[k] = a.gv0[i * d + k] + dv[i * d + k]; X[k] = X0[k] + a.dt * V[k]; }
            const T phi0 = phi_at<T, d>(o, a.motion, a.moving, j, false, X0);
            const T phi = phi_at<T, d>(o, a.motion, a.moving, j, true, X) - fmin(phi0, (T)0);
            if(o.type == MPM_STICK && phi0 > 0) continue;
            if(o.type == MPM_SLIP && phi0 > 0) continue;
            if(o.type == MPM_SEPARATE && phi > (T)kCollisionThickness) continue;
            if(o.type != MPM_STICK && phi > (T)FLT_MAX) continue;
            T n[3];
            normal_at<T, d>(o, a.motion, a.moving, j, X, n);
            T* cd = ia.cdat + (i * ia.nobj + j) * (2 + 3 * d);
            cd[0] = phi;
            cd[1] = 0;
            for(int k = 0; k < d; k++) { cd[2 + k] = n[k]; cd[2 + d + k] = X[k]; cd[2 + 2 * d + k] = 0; }
            mask |= (uint8_t)(1u << j);
            for(int k = 0; k < d; k++) { X[k] -= phi * n[k]; V[k] = (X[k] - X0[k]) / a.dt; }
            if(o.type == MPM_STICK) {
                velocity_at<T, d>(a.motion, a.moving, j, X, V);
                for(int k = 0; k < d; k++) ia.svel[i * d + k] = V[k];
                stuck = 1;
            }
            for(int k = 0; k < d; k++) dv[i * d + k] = V[k] - a.gv0[i * d + k];
        }
        ia.cmask[i] = mask;
        ia.stuck[i] = stuck;
    }
}

// MPM_OBJECTIVE::Project_Gradient_And_Prune_Constraints (l.226-248): the
// collisions in reverse order; one whose node may leave the object (separate
// with allow_sep, or not penetrating) and whose gradient points out of it is
// dropped, else the normal part of the gradient is removed.
template<class T, int d> __global__ void k_imp_project(ImpArgs<T> ia, T* g, int allow_sep)
{
    NODE_LOOP(ia) {
        uint8_t mask = ia.cmask[i];
        if(!mask && !ia.stuck[i]) continue;
        if(ia.stuck[i])
            for(int k = 0; k < d; k++) g[i * d + k] = 0;
        for(int j = ia.nobj - 1; j >= 0; j--) {
            if(!(mask & (1u << j))) continue;
            T* cd = ia.cdat + (i * ia.nobj + j) * (2 + 3 * d);
            T ndE = 0;
            for(int k = 0; k < d; k++) ndE += g[i * d + k] * cd[2 + k];
            cd[1] = ndE;
            const bool sep = ia.a.sp.objs[j].type == MPM_SEPARATE;
            if(((allow_sep && sep) || cd[0] <= (T)kCollisionThickness) && ndE < 0) {
                mask &= (uint8_t)~(1u << j);
                continue;
            }
            // H_dE = H g; g -= n_dE n + phi H_dE
            T H[9], gv[3];
            hessian_at<T, d>(ia.a.sp.objs[j], ia.a.motion, ia.a.moving, j, cd + 2 + d, H);
            for(int k = 0; k < d; k++) gv[k] = g[i * d + k];
            for(int r = 0; r < d; r++) {
                T hd = 0;
                for(int c = 0; c < d; c++) hd += H[r + d * c] * gv[c];
                cd[2 + 2 * d + r] = hd;
            }
            for(int k = 0; k < d; k++) g[i * d + k] -= ndE * cd[2 + k] + cd[0] * cd[2 + 2 * d + k];
        }
        ia.cmask[i] = mask;
    }
}

// MPM_KRYLOV_SYSTEM::Multiply (l.40-78), before the Hessian: tmp = v with the
// stuck nodes zeroed and the colliding nodes' normal parts removed.
template<class T, int d> __global__ void k_imp_mult_pre(ImpArgs<T> ia, T* tmp, const T* v)
{
    NODE_LOOP(ia) {
        T x[3];
        for(int k = 0; k < d; k++) x[k] = ia.stuck[i] ? (T)0 : v[i * d + k];
        const uint8_t mask = ia.cmask[i];
        for(int j = 0; j < ia.nobj; j++) {
            if(!(mask & (1u << j))) continue;
            const T* n = ia.cdat + (i * ia.nobj + j) * (2 + 3 * d) + 2;
            T dn = 0;
            for(int k = 0; k < d; k++) dn += x[k] * n[k];
            for(int k = 0; k < d; k++) x[k] -= dn * n[k];
        }
        for(int k = 0; k < d; k++) tmp[i * d + k] = x[k];
    }
}

// ... and after it: f = (dt^2/m) H tmp + tmp, with the stuck nodes zeroed and
// per collision f -= n (n.f) + dt (Hc v n_dE + (n.v) H_dE + (H_dE.v) n), v the
// unprojected input (the curvature terms of MPM_KRYLOV_SYSTEM::Multiply).
template<class T, int d> __global__ void k_imp_mult_post(ImpArgs<T> ia, T* f, const T* tmp, const T* v)
{
    NODE_LOOP(ia) {
        const T s = ia.a.dt * ia.a.dt / ia.a.gm[i];
        T x[3];
        for(int k = 0; k < d; k++) x[k] = s * f[i * d + k] + tmp[i * d + k];
        if(ia.stuck[i])
            for(int k = 0; k < d; k++) x[k] = 0;
        const uint8_t mask = ia.cmask[i];
        for(int j = 0; j < ia.nobj; j++) {
            if(!(mask & (1u << j))) continue;
            const T* cd = ia.cdat + (i * ia.nobj + j) * (2 + 3 * d);
            const T* n = cd + 2;
            const T* hde = cd + 2 + 2 * d;
            T H[9];
            hessian_at<T, d>(ia.a.sp.objs[j], ia.a.motion, ia.a.moving, j, cd + 2 + d, H);
            T dn = 0, nv = 0, hv = 0, Hv[3];
            for(int k = 0; k < d; k++) { dn += x[k] * n[k]; nv += n[k] * v[i * d + k]; hv += hde[k] * v[i * d + k]; }
            for(int r = 0; r < d; r++) {
                Hv[r] = 0;
                for(int c = 0; c < d; c++) Hv[r] += H[r + d * c] * v[i * d + c];
            }
            for(int k = 0; k < d; k++)
                x[k] -= n[k] * dn + ia.a.dt * (Hv[k] * cd[1] + nv * hde[k] + hv * n[k]);
        }
        for(int k = 0; k < d; k++) f[i * d + k] = x[k];
    }
}

// MPM_DRIVER::Apply_Friction, implicit branch (MPM_DRIVER.cpp:1064-1094):
// Coulomb friction on the colliding nodes from the normal force the
// projection removed (tmp0 unprojected, tmp1 projected gradient).  vfs is
// velocity_friction_save relative to v0.
template<class T, int d> __global__ void k_imp_friction(ImpArgs<T> ia, const T* dv, const T* tmp0, const T* tmp1, T* vfs)
{
    NODE_LOOP(ia) {
        const PlainArgs<T>& a = ia.a;
        T v[3];
        for(int k = 0; k < d; k++) {
            vfs[i * d + k] = dv[i * d + k];
            v[k] = ia.stuck[i] ? (T)0 : dv[i * d + k] + a.gv0[i * d + k];
        }
        const uint8_t mask = ia.cmask[i];
        for(int j = 0; j < ia.nobj; j++) {
            if(!(mask & (1u << j))) continue;
            const T* n = ia.cdat + (i * ia.nobj + j) * (2 + 3 * d) + 2;
            T nf = 0, vn = 0;
            for(int k = 0; k < d; k++) { nf += n[k] * (tmp0[i * d + k] - tmp1[i * d + k]); vn += v[k] * n[k]; }
            T t[3], tm = 0;
            for(int k = 0; k < d; k++) { t[k] = v[k] - vn * n[k]; tm += t[k] * t[k]; }
            tm = sqrt(tm);
            if(tm) {   // VECTOR::Normalize: a zero vector becomes the first axis
                const T inv = 1 / tm;
                for(int k = 0; k < d; k++) t[k] *= inv;
            } else {
                for(int k = 0; k < d; k++) t[k] = k == 0 ? (T)1 : (T)0;
            }
            const T kf = (T)a.sp.objs[j].friction * nf;
            if(tm <= kf) for(int k = 0; k < d; k++) v[k] = vn * n[k];
            else for(int k = 0; k < d; k++) v[k] -= kf * t[k];
            for(int k = 0; k < d; k++) vfs[i * d + k] = v[k] - a.gv0[i * d + k];
        }
    }
}

// The end of Apply_Forces (MPM_DRIVER.cpp:1049-1056): velocity = dv + v0,
// velocity_friction_save += v0, stuck nodes at the object's velocity.
template<class T, int d> __global__ void k_imp_finish(ImpArgs<T> ia, const T* dv, const T* vfs)
{
    NODE_LOOP(ia) {
        const PlainArgs<T>& a = ia.a;
        for(int k = 0; k < d; k++) {
            a.gv[i * d + k] = dv[i * d + k] + a.gv0[i * d + k];
            a.gvf[i * d + k] = ia.stuck[i] ? ia.svel[i * d + k] : vfs[i * d + k] + a.gv0[i * d + k];
        }
    }
}

// Deterministic reductions: a fixed grid writes one partial per block, one
// block sums them in order.
template<class T> __device__ double block_sum(double v)
{
    __shared__ double sh[kRedThreads];
    sh[threadIdx.x] = v;
    __syncthreads();
    for(int s = kRedThreads / 2; s > 0; s >>= 1) {
        if(threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    return sh[0];
}

// MPM_KRYLOV_SYSTEM::Inner_Product (l.82-95): sum over nodes with mass of m x.y
template<class T, int d> __global__ void k_imp_dot(ImpArgs<T> ia, const T* x, const T* y, double* partial)
{
    double acc = 0;
    NODE_LOOP(ia) {
        double s = 0;
        for(int k = 0; k < d; k++) s += (double)x[i * d + k] * (double)y[i * d + k];
        acc += (double)ia.a.gm[i] * s;
    }
    const double t = block_sum<T>(acc);
    if(threadIdx.x == 0) partial[blockIdx.x] = t;
}

template<class T> __global__ void k_imp_sum_particles(const double* pe, int64_t n, double* partial)
{
    double acc = 0;
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) acc += pe[p];
    const double t = block_sum<T>(acc);
    if(threadIdx.x == 0) partial[blockIdx.x] = t;
}

__device__ double block_sum_max(double v)
{
    __shared__ double sh[kRedThreads];
    sh[threadIdx.x] = v;
    __syncthreads();
    for(int s = kRedThreads / 2; s > 0; s >>= 1) {
        if(threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    return sh[0];
}

__global__ void k_imp_max_final(const double* partial, int count, double* out)
{
    if(threadIdx.x) return;
    double r = partial[0];
    for(int b = 1; b < count; b++) r = fmax(r, partial[b]);
    *out = r;
}

// one block per result slot; the partials (count == blockDim.x) summed by a
// fixed tree, so the result does not depend on scheduling
__global__ void k_imp_final(const double* partial, int count, int slots, double* out)
{
    __shared__ double sh[kRedThreads];
    const int s = blockIdx.x;
    sh[threadIdx.x] = threadIdx.x < count ? partial[s * count + threadIdx.x] : 0.0;
    __syncthreads();
    for(int st = kRedThreads / 2; st > 0; st >>= 1) {
        if(threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
        __syncthreads();
    }
    if(threadIdx.x == 0) out[s] = sh[0];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
enum { V_DV, V_GRAD, V_DX, V_TM, V_Q, V_S, V_R, V_TMP0, V_TMP1, V_TMP2, V_V1, V_STMP, V_VFS, V_SVEL, V_COUNT };

}  // namespace

struct ImplicitState {
    int64_t gn = 0, n = 0;
    int nobj = 0, d = 0;
    size_t esz = 0;
    void* vec = nullptr;           // V_COUNT node vectors of gn * d scalars
    void* part = nullptr;          // F0, X0, U, FV, sig, dP, pen
    double* pe = nullptr;
    uint8_t* cmask = nullptr;
    uint8_t* stuck = nullptr;
    void* cdat = nullptr;
    double* partial = nullptr;     // 2 * kRedBlocks
    double* dout = nullptr;        // 2 results
    double* hout = nullptr;        // pinned copy
    uint32_t *keys = nullptr, *sorted = nullptr, *perm = nullptr, *alt_k = nullptr, *alt_v = nullptr, *scratch = nullptr;
    int key_bits = 1;
};

namespace {

template<class T, int d> struct Solver {
    mpm_handle* h;
    ImpArgs<T> ia;
    T* v[V_COUNT];
    cudaStream_t st;
    int pb, gb;
    const mpm_implicit_desc& prm;
    int rc = MPM_OK;
    int krylov_total = 0;

    Solver(mpm_handle* h_, double dt) : h(h_), st(h_->stream), prm(h_->implicit)
    {
        ImplicitState& s = *h->imp;
        ia.a = args<T>(h, dt);
        const int64_t n = s.n ? s.n : 1;
        T* P = (T*)s.part;
        ia.F0 = P; ia.X0 = P + n * d * d; ia.U = ia.X0 + n * d; ia.FV = ia.U + n * d * d;
        ia.sig = ia.FV + n * d * d; ia.dP = ia.sig + n * d; ia.pen = ia.dP + n * 15;
        ia.pe = s.pe; ia.cmask = s.cmask; ia.stuck = s.stuck; ia.cdat = (T*)s.cdat; ia.nobj = h->sp.nobj;
        ia.order = nullptr;
        for(int k = 0; k < V_COUNT; k++) v[k] = (T*)s.vec + (size_t)k * s.gn * d;
        ia.svel = v[V_SVEL];
        pb = pblocks(s.n, 128);
        gb = gblocks(h, s.gn, 256);
    }
    static int pblocks(int64_t n, int t) { int64_t b = (n + t - 1) / t; return (int)(b < 1 ? 1 : b); }
    static int gblocks(mpm_handle* h, int64_t n, int t)
    {
        int64_t b = (n + t - 1) / t, cap = (int64_t)h->sm_count * 8;
        return (int)(b < 1 ? 1 : (b > cap ? cap : b));
    }
    bool failed() { return rc != MPM_OK; }
    void check(const char* what)
    {
        cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess && !rc) rc = check_cuda(h, e, what);
    }

    // reductions ----------------------------------------------------------
    double dot(const T* x, const T* y)
    {
        ImplicitState& s = *h->imp;
        k_imp_dot<T, d><<<kRedBlocks, kRedThreads, 0, st>>>(ia, x, y, s.partial);
        k_imp_final<<<1, kRedThreads, 0, st>>>(s.partial, kRedBlocks, 1, s.dout);
        cudaMemcpyAsync(s.hout, s.dout, sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        check("implicit dot");
        return s.hout[0];
    }
    // m-weighted |x|^2 / 2 + potential energy, in one read-back
    double energy(const T* x)
    {
        ImplicitState& s = *h->imp;
        k_imp_dot<T, d><<<kRedBlocks, kRedThreads, 0, st>>>(ia, x, x, s.partial);
        k_imp_sum_particles<T><<<kRedBlocks, kRedThreads, 0, st>>>(s.pe, s.n, s.partial + kRedBlocks);
        k_imp_final<<<2, kRedThreads, 0, st>>>(s.partial, kRedBlocks, 2, s.dout);
        cudaMemcpyAsync(s.hout, s.dout, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        check("implicit energy");
        return s.hout[0] / 2 + s.hout[1];
    }

    // vector ops on nodes with mass ---------------------------------------
    void copy(T* out, T c, const T* x, const T* y = nullptr) { k_imp_copy<T, d><<<gb, 256, 0, st>>>(ia, out, c, x, y); }
    void zero(T* x) { cudaMemsetAsync(x, 0, (size_t)ia.a.gn * d * sizeof(T), st); }

    // MPM_OBJECTIVE ----------------------------------------------------------
    void adjust(T* x)
    {
        if(!ia.nobj) return;
        k_imp_adjust<T, d><<<gb, 256, 0, st>>>(ia, x);
    }
    void project(T* g, bool allow_sep)
    {
        if(!ia.nobj) return;
        k_imp_project<T, d><<<gb, 256, 0, st>>>(ia, g, allow_sep ? 1 : 0);
    }
    // Compute_Unconstrained: F, X at v0 + dv; forces, gradient and energy as asked
    void compute_unconstrained(const T* dv, T* g, double* e)
    {
        copy(v[V_V1], 1, dv, ia.a.gv0);
        k_imp_update_F<T, d><<<pb, 128, 0, st>>>(ia, v[V_V1]);
        k_imp_precompute<T, d><<<pb, 128, 0, st>>>(ia);
        if(e) *e = energy(dv);
        if(g) {
            zero(v[V_TMP2]);
            k_imp_forces<T, d><<<pb, 128, 0, st>>>(ia, v[V_TMP2]);
            k_imp_grad<T, d><<<gb, 256, 0, st>>>(ia, g, dv, v[V_TMP2]);
        }
        check("compute_unconstrained");
    }
    // Compute (l.48-65): at the feasible copy of dv; the gradient projected
    void compute(const T* dv, bool hess, T* g, double* e)
    {
        copy(v[V_TMP1], 1, dv);
        adjust(v[V_TMP1]);
        compute_unconstrained(v[V_TMP1], g, e);
        if(g) project(g, hess);
    }
    void make_feasible(T* x) { adjust(x); }

    // MPM_KRYLOV_SYSTEM::Multiply
    void multiply(const T* x, T* out)
    {
        k_imp_mult_pre<T, d><<<gb, 256, 0, st>>>(ia, v[V_STMP], x);
        zero(out);
        k_imp_hessian<T, d><<<pb, 128, 0, st>>>(ia, v[V_STMP], out);
        k_imp_mult_post<T, d><<<gb, 256, 0, st>>>(ia, out, v[V_STMP], x);
    }

    // CONJUGATE_GRADIENT::Solve with relative tolerance and
    // finish_before_indefiniteness; x = 0 on entry.
    bool cg(T* x, const T* b, double tolerance, int max_iterations, int& used)
    {
        T *q = v[V_Q], *s = v[V_S], *r = v[V_R];
        double rho_old = FLT_MAX;
        copy(r, 1, b);                // r = b - A 0
        int it;
        for(it = 0;; it++) {
            const double rho = dot(r, r);      // no preconditioner: rho = |r|^2
            const double cn = sqrt(rho);
            if(failed()) return false;
            if(it == 0) tolerance *= cn;
            if(cn <= tolerance) { used = it; return true; }   // min_iterations 0
            if(it == max_iterations) break;
            if(it == 0) copy(s, 1, r);
            else copy(s, (T)(rho / rho_old), s, r);
            multiply(s, q);
            const double sq = dot(s, q);
            if(sq <= 0) {
                if(it == 0) copy(x, 1, b);
                used = it;
                return true;
            }
            const double alpha = sq ? rho / sq : (double)FLT_MAX;
            copy(x, (T)alpha, s, x);
            copy(r, (T)-alpha, q, r);
            rho_old = rho;
        }
        used = it;
        return false;
    }

    // PARAMETRIC_LINE::Compute for the line search: objective along x + t dx
    void line_eval(const T* x, const T* dx, double t, double& f, double& df)
    {
        copy(v[V_GRAD], (T)t, dx, x);              // the reference reuses grad as the point
        compute(v[V_GRAD], false, v[V_TM], &f);
        df = dot(v[V_TM], dx);
    }

    struct Wolfe { double a, fa, dfa; };
    static double interpolate(const Wolfe& lo, const Wolfe& hi)
    {
        const double k = hi.fa - lo.fa, a = -2 * k + lo.dfa + hi.dfa, b = 3 * k - 2 * lo.dfa - hi.dfa, c = lo.dfa;
        const double r = b * b - 3 * a * c;
        if(r > 0) {
            double s = sqrt(r), num = s - b, den = 3 * a;
            if(den < 0) { num = -num; den = -den; }
            if(num > .1 * den && num < .9 * den) return lo.a + num / den * (hi.a - lo.a);
        }
        return (lo.a + hi.a) / 2;
    }
    // LINE_SEARCH::Line_Search_Wolfe_Conditions_Zoom
    bool zoom(const T* x, const T* dx, Wolfe lo, Wolfe hi, Wolfe x0, double& out, double c1, double c2)
    {
        const double eps = std::numeric_limits<T>::epsilon();
        const double min_interval = fabs(hi.a - lo.a) * eps;
        while(fabs(hi.a - lo.a) > min_interval && !failed()) {
            Wolfe xj = {interpolate(lo, hi), 0, 0};
            line_eval(x, dx, xj.a, xj.fa, xj.dfa);
            if(xj.fa > x0.fa + c1 * xj.a * x0.dfa || xj.fa >= x0.fa) hi = xj;
            else if(fabs(xj.dfa) <= -c2 * x0.dfa) { out = xj.a; return true; }
            else {
                if((hi.a > lo.a && xj.dfa >= 0) || (hi.a < lo.a && xj.dfa <= 0)) hi = lo;
                lo = xj;
            }
        }
        if(lo.a - x0.a >= min_interval * 100) { out = lo.a; return true; }
        return false;
    }
    // LINE_SEARCH::Line_Search_Wolfe_Conditions on [0, 1], c1 1e-4, c2 .9
    double line_search(const T* x, const T* dx)
    {
        const double c1 = 1e-4, c2 = .9;
        Wolfe a0 = {0, 0, 0};
        line_eval(x, dx, 0, a0.fa, a0.dfa);
        if(!(a0.dfa < 0)) return 0;      // the reference asserts a descent direction
        Wolfe x0 = a0, x1 = {1, 0, 0};
        double out = 0;
        for(int guard = 0; x1.a <= (double)FLT_MAX && guard < 200 && !failed(); guard++) {
            line_eval(x, dx, x1.a, x1.fa, x1.dfa);
            if(x1.fa > a0.fa + c1 * x1.a * a0.dfa || x1.fa >= x0.fa) return zoom(x, dx, x0, x1, a0, out, c1, c2) ? out : 0;
            if(fabs(x1.dfa) <= -c2 * a0.dfa) return x1.a;
            if(x1.dfa >= 0) return zoom(x, dx, x1, x0, a0, out, c1, c2) ? out : 0;
            x0 = x1;
            x1.a = 2 * x1.a - x0.a;
        }
        return 0;
    }

    // MPM_OBJECTIVE::Initial_Guess (l.268-288)
    bool initial_guess(T* dv, double tolerance)
    {
        double e0 = 0, e1 = 0;
        zero(dv);
        compute(dv, false, v[V_TMP0], &e0);
        copy(dv, -1, v[V_TMP0]);
        const double g0 = sqrt(dot(v[V_TMP0], v[V_TMP0]));
        compute(dv, false, v[V_TMP0], &e1);
        const double g1 = sqrt(dot(v[V_TMP0], v[V_TMP0]));
        if(e1 < std::max(e0, e0 * 1.1)) return true;
        if(g1 < g0 * 1.1 || g1 < tolerance) return true;
        zero(dv);
        return false;
    }

    // NEWTONS_METHOD::Newtons_Method with MPM_DRIVER's settings: CG, Wolfe
    // search, gradient-descent failsafe, step norm <= 100, countdown at the
    // default 5e-10 for 5 iterations.
    bool newton(T* x, double tolerance, bool require_one, int& iterations)
    {
        const double countdown_tolerance = 5e-10, angle_tolerance = 1e-2, max_step = 100;
        const int countdown_iterations = 5;
        T *grad = v[V_GRAD], *dx = v[V_DX], *tm = v[V_TM];
        bool result = false;
        int local_max = prm.newton_iterations;
        make_feasible(x);
        int it;
        for(it = 0; it < local_max && !failed(); it++) {
            compute(x, true, grad, nullptr);   // the energy only feeds the reference's log
            const double norm_grad = sqrt(dot(grad, grad)), conv = norm_grad;
            h->imp_stats.residual = conv;
            if(conv < tolerance && (it || !require_one || !conv)) { result = true; break; }
            if(conv < countdown_tolerance) { result = true; local_max = std::min(local_max, it + countdown_iterations); }
            zero(dx);
            copy(tm, -1, grad);
            const double ktol = std::min(.5, prm.solver_tolerance * sqrt(std::max(conv, tolerance)));
            int used = 0;
            cg(dx, tm, ktol, prm.solver_iterations, used);
            krylov_total += used;
            // Make_Downhill_Direction
            const double ndx = sqrt(dot(dx, dx)), inner = dot(dx, grad);
            if(inner > angle_tolerance * ndx * norm_grad) copy(dx, -1, dx);
            else if(inner >= -angle_tolerance * ndx * norm_grad) copy(dx, (T)(-ndx / norm_grad), grad);
            const double nrm = sqrt(dot(dx, dx));
            if(nrm > max_step) copy(dx, (T)(max_step / nrm), dx);
            const double a = line_search(x, dx);
            if(a <= 0) break;
            copy(x, (T)a, dx, x);
            make_feasible(x);
        }
        iterations = it;
        return result;
    }

    int solve(double dt)
    {
        ImplicitState& s = *h->imp;
        if(s.n) {
            // the particles in cell order for every pass of the solve (their weights
            // are those of the step's start, so one sort serves the whole solve)
            k_imp_keys<T, d><<<pb, 128, 0, st>>>(ia, s.keys);
            check("implicit keys");
            if((rc = sort_keys_device(h, s.keys, s.n, s.key_bits, s.sorted, s.perm, s.alt_k, s.alt_v, s.scratch))) return rc;
            ia.order = s.perm;
            k_imp_save<T, d><<<pb, 128, 0, st>>>(ia);
        }
        for(int k = 0; k < V_COUNT; k++) zero(v[k]);
        if(ia.nobj) {
            cudaMemsetAsync(s.cmask, 0, s.gn, st);
            cudaMemsetAsync(s.stuck, 0, s.gn, st);
        }
        T* dv = v[V_DV];
        const double tolerance = prm.newton_tolerance * dt;
        const bool require_one = !initial_guess(dv, tolerance);
        int iters = 0;
        const bool converged = newton(dv, tolerance, require_one, iters);
        if(failed()) return rc;
        // Apply_Friction: velocity_friction_save = dv; Coulomb friction on the collisions
        if(ia.nobj) {
            compute_unconstrained(dv, v[V_TMP0], nullptr);
            copy(v[V_TMP1], 1, v[V_TMP0]);
            project(v[V_TMP1], true);
            k_imp_friction<T, d><<<gb, 256, 0, st>>>(ia, dv, v[V_TMP0], v[V_TMP1], v[V_VFS]);
        } else {
            copy(v[V_VFS], 1, dv);
        }
        if(s.n) k_imp_restore<T, d><<<pb, 128, 0, st>>>(ia);
        k_imp_finish<T, d><<<gb, 256, 0, st>>>(ia, dv, v[V_VFS]);
        // Reflect_Boundary_Velocity on velocity and velocity_friction_save (MPM_DRIVER.cpp:1055-1057)
        if(h->reflect.enabled && !h->reflect.full_reflection) plain_reflect_velocity(h);
        check("implicit finish");
        h->imp_stats.newton_iterations = iters;
        h->imp_stats.krylov_iterations = krylov_total;
        h->imp_stats.converged = converged ? 1 : 0;
        return rc;
    }
};

template<class T> int ensure_state(mpm_handle* h)
{
    PlainState& ps = h->plain;
    const int d = h->sp.dim;
    if(!h->imp) h->imp = new ImplicitState();
    ImplicitState& s = *h->imp;
    const size_t e = sizeof(T);
    if(s.gn == ps.gn && s.n == ps.n && s.nobj == h->sp.nobj && s.d == d && s.esz == e && s.vec) return MPM_OK;
    implicit_free(h);
    h->imp = new ImplicitState();
    ImplicitState& t = *h->imp;
    t.gn = ps.gn; t.n = ps.n; t.nobj = h->sp.nobj; t.d = d; t.esz = e;
    const int64_t n = t.n ? t.n : 1;
    MPM_CUDA(h, cudaMalloc(&t.vec, (size_t)V_COUNT * t.gn * d * e));
    MPM_CUDA(h, cudaMalloc(&t.part, (size_t)n * (d * d * 4 + d * 3 + 15) * e));
    MPM_CUDA(h, cudaMalloc(&t.pe, (size_t)n * sizeof(double)));
    MPM_CUDA(h, cudaMalloc(&t.cmask, (size_t)t.gn));
    MPM_CUDA(h, cudaMalloc(&t.stuck, (size_t)t.gn));
    MPM_CUDA(h, cudaMemset(t.cmask, 0, (size_t)t.gn));
    MPM_CUDA(h, cudaMemset(t.stuck, 0, (size_t)t.gn));
    if(t.nobj) MPM_CUDA(h, cudaMalloc(&t.cdat, (size_t)t.gn * t.nobj * (2 + 3 * d) * e));
    MPM_CUDA(h, cudaMalloc(&t.partial, 2 * kRedBlocks * sizeof(double)));
    MPM_CUDA(h, cudaMalloc(&t.dout, 2 * sizeof(double)));
    MPM_CUDA(h, cudaMallocHost(&t.hout, 2 * sizeof(double)));
    uint32_t** sb[] = {&t.keys, &t.sorted, &t.perm, &t.alt_k, &t.alt_v};
    for(uint32_t** p: sb) MPM_CUDA(h, cudaMalloc(p, (size_t)n * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMalloc(&t.scratch, (size_t)sort_scratch_words(n) * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMemset(t.scratch, 0, (size_t)sort_scratch_words(n) * sizeof(uint32_t)));
    t.key_bits = 1;
    while((int64_t)((1ull << t.key_bits) - 1) < t.gn) t.key_bits++;
    return MPM_OK;
}

template<class T> int implicit_t(mpm_handle* h, double dt)
{
    int rc = ensure_state<T>(h);
    if(rc) return rc;
    int slot = timer_begin(h, "plain_implicit");
    if(h->sp.dim == 3) { Solver<T, 3> sv(h, dt); rc = sv.solve(dt); }
    else { Solver<T, 2> sv(h, dt); rc = sv.solve(dt); }
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_imp_*");
    return rc;
}

}  // namespace

namespace {
// Compute_Max_Sound_Speed on the singular values and stress derivative of the
// solve's last force evaluation (what the reference's force holds then).
template<class T, int d> __global__ void k_imp_sound(ImpArgs<T> ia, double* partial)
{
    const PlainArgs<T>& a = ia.a;
    double smax = 0;
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        if(!a.valid[p]) continue;
        const T* blk = ia.dP + p * 15;
        smax = fmax(smax, (double)sound_speed<T, d>(ia.sig + p * d, blk, blk + 9, a.mass[p] / a.vol[p]));
    }
    const double r = block_sum_max(smax);
    if(threadIdx.x == 0) partial[blockIdx.x] = r;
}

template<class T> int implicit_sound_t(mpm_handle* h, double* partial, double* out)
{
    if(!h->imp) return set_error(h, MPM_ERR_STATE, "no implicit solve yet");
    if(h->sp.dim == 3) {
        Solver<T, 3> sv(h, 0.0);
        k_imp_sound<T, 3><<<kRedBlocks, kRedThreads, 0, h->stream>>>(sv.ia, partial);
    } else {
        Solver<T, 2> sv(h, 0.0);
        k_imp_sound<T, 2><<<kRedBlocks, kRedThreads, 0, h->stream>>>(sv.ia, partial);
    }
    k_imp_max_final<<<1, 32, 0, h->stream>>>(partial, kRedBlocks, out);
    return MPM_OK;
}
}  // namespace

int implicit_max_sound_speed(mpm_handle* h, double* partial, double* out)
{
    return h->model.precision == MPM_FP64 ? implicit_sound_t<double>(h, partial, out) : implicit_sound_t<float>(h, partial, out);
}

void implicit_free(mpm_handle* h)
{
    if(!h->imp) return;
    ImplicitState& s = *h->imp;
    cudaFree(s.vec); cudaFree(s.part); cudaFree(s.pe); cudaFree(s.cmask); cudaFree(s.stuck); cudaFree(s.cdat);
    cudaFree(s.partial); cudaFree(s.dout);
    cudaFree(s.keys); cudaFree(s.sorted); cudaFree(s.perm); cudaFree(s.alt_k); cudaFree(s.alt_v); cudaFree(s.scratch);
    if(s.hout) cudaFreeHost(s.hout);
    delete h->imp;
    h->imp = nullptr;
}

int plain_implicit_forces(mpm_handle* h, double dt, double)
{
    return h->model.precision == MPM_FP64 ? implicit_t<double>(h, dt) : implicit_t<float>(h, dt);
}

// This module's copy of the SVD sweep bound (mpm_debug_set_svd_iterations).
MPM_SVD_LIMIT_SETTER(svd_limit_implicit)
