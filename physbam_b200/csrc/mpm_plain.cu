// Plain path: a direct GPU port of the reference's explicit substep, one thread
// per particle (or grid node), global atomics for every scatter, particles in
// the reference's MPM_PARTICLES layout and arrival order.  Templated on the
// scalar type; in FP64 it is the baseline the FP32 fast path is measured
// against, and the path whose grids are checked node-for-node against the
// reference (it keeps velocity_save and separate force arrays like the
// reference does).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "mpm_internal.h"
#include "mpm_plain.cuh"

namespace {

using namespace mpm;
using namespace plain;

template<class T> struct Vec4 { T v[4]; };
template<class T> struct Vec5 { T v[5]; };

template<class T> __global__ void k_clear(PlainArgs<T> a)
{
    const int d = a.sp.dim;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.gn; i += (int64_t)gridDim.x * blockDim.x) {
        a.gm[i] = 0;
        for(int k = 0; k < d; k++) {
            a.gmv[i * d + k] = 0; a.gf[i * d + k] = 0; a.gv0[i * d + k] = 0;
            a.gv[i * d + k] = 0; a.gvf[i * d + k] = 0;
        }
    }
}

// MPM_DRIVER::Particle_To_Grid scatter (MPM_DRIVER.cpp:259-271).
template<class T, int d> __global__ void k_p2g(PlainArgs<T> a)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(p >= a.n || !a.valid[p]) return;
    const T* X = a.X + p * d;
    Stencil<T, d> s;
    if(!make_stencil<T, d>(a, X, s)) { atomicOr(a.flags, MPM_FLAG_DOMAIN); return; }
    T Dp_inv[3];
#pragma unroll
    for(int k = 0; k < d; k++) Dp_inv[k] = 4 * (T)a.sp.inv_dx[k] * (T)a.sp.inv_dx[k];
    const T* Bp = a.B + p * d * d;
    T mp = a.mass[p];
    const int nq = d == 3 ? 27 : 9;
    for(int q = 0; q < nq; q++) {
        int64_t i;
        T w, g[3], Z[3];
        node<T, d>(a, s, q, i, w, g, Z);
        atomicAdd(a.gm + i, w * mp);
        T Vn[3], Y[3];
#pragma unroll
        for(int k = 0; k < d; k++) { Vn[k] = w * a.V[p * d + k]; Y[k] = (Z[k] - X[k]) * Dp_inv[k]; }
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int c = 0; c < d; c++) sum += Bp[r + d * c] * Y[c];
            Vn[r] += sum * w;
        }
#pragma unroll
        for(int k = 0; k < d; k++) atomicAdd(a.gmv + i * d + k, mp * Vn[k]);
    }
}

// v = mv / m on nodes with mass (MPM_DRIVER.cpp:282-305).
template<class T> __global__ void k_normalize(PlainArgs<T> a)
{
    const int d = a.sp.dim;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.gn; i += (int64_t)gridDim.x * blockDim.x) {
        T m = a.gm[i];
        for(int k = 0; k < d; k++) a.gv0[i * d + k] = m != 0 ? a.gmv[i * d + k] / m : (T)0;
    }
}

// MPM_FINITE_ELEMENTS::Precompute (MPM_FINITE_ELEMENTS.cpp:47-67).
template<class T, int d> __global__ void k_stress(PlainArgs<T> a)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(p >= a.n || !a.valid[p]) return;
    T F[9], PFT[9];
#pragma unroll
    for(int e = 0; e < d * d; e++) F[e] = a.F[p * d * d + e];
    if(!pft_svd<T, d>(model_of(a, p), F, a.mu[p], a.lam[p], PFT)) atomicOr(a.flags, MPM_FLAG_NOT_CONVERGED);
#pragma unroll
    for(int e = 0; e < d * d; e++) a.pft[p * d * d + e] = PFT[e];
}

// MPM_FINITE_ELEMENTS::Add_Forces (MPM_FINITE_ELEMENTS.cpp:84-99),
// MPM_GRAVITY::Add_Forces (MPM_GRAVITY.cpp:62-68) and the penalty collision
// forces of Apply_Particle_Forces (MPM_DRIVER.cpp:933-945) in one pass.
template<class T, int d> __global__ void k_forces(PlainArgs<T> a)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(p >= a.n || !a.valid[p]) return;
    Stencil<T, d> s;
    if(!make_stencil<T, d>(a, a.X + p * d, s)) return;
    T A[9];
#pragma unroll
    for(int e = 0; e < d * d; e++) A[e] = a.pft[p * d * d + e] * a.vol[p];
    T mp = a.mass[p];
    T fp[3] = {0, 0, 0};   // the particle's penalty force
    if(a.sp.npen)
        penalty_particle<T, d>(a.sp.pen, a.sp.npen, (T)a.sp.pen_stiffness, (T)a.sp.pen_separation, a.X + p * d, fp,
                               (T*)nullptr);
    const int nq = d == 3 ? 27 : 9;
    for(int q = 0; q < nq; q++) {
        int64_t i;
        T w, g[3], Z[3];
        node<T, d>(a, s, q, i, w, g, Z);
        T wm = w * mp;
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int c = 0; c < d; c++) sum += A[r + d * c] * g[c];
            atomicAdd(a.gf + i * d + r, -sum + wm * (T)a.sp.gravity[r] + w * fp[r]);
        }
    }
}

// Apply_Forces grid update: dv = dt/m f, collision projection, friction,
// assembly (MPM_DRIVER.cpp:989-1056, MPM_OBJECTIVE.cpp:150-225).
template<class T, int d> __global__ void k_grid_update(PlainArgs<T> a)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.gn; i += (int64_t)gridDim.x * blockDim.x) {
        T m = a.gm[i];
        if(m == 0) continue;
        T dv[3], v0[3], X0[3], vn[3], vf[3];
        T s = a.dt / m;
        int64_t r = i;
        int idx[3];
        for(int k = d - 1; k >= 0; k--) { idx[k] = (int)(r % a.gs[k]) - MPM_GHOST; r /= a.gs[k]; }
#pragma unroll
        for(int k = 0; k < d; k++) {
            dv[k] = s * a.gf[i * d + k];
            v0[k] = a.gv0[i * d + k];
            X0[k] = (T)a.sp.dmin[k] + ((T)idx[k] + (T).5) * (T)a.sp.dx[k];
        }
        collide_node<T, d>(a.sp.objs, a.sp.nobj, X0, v0, dv, a.dt, vn, vf, a.motion, a.moving);
#pragma unroll
        for(int k = 0; k < d; k++) { a.gv[i * d + k] = vn[k]; a.gvf[i * d + k] = vf[k]; }
    }
}

// MPM_DRIVER::Grid_To_Particle (MPM_DRIVER.cpp:450-515) and
// Reflect_Or_Invalidate_Particle (l.1219-1239, all sides free).
template<class T, int d> __global__ void k_g2p(PlainArgs<T> a)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if(p >= a.n || !a.valid[p]) return;
    T* X = a.X + p * d;
    Stencil<T, d> s;
    if(!make_stencil<T, d>(a, X, s)) return;
    T Vpic[3] = {0, 0, 0}, Vpf[3] = {0, 0, 0}, G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Bh[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int nq = d == 3 ? 27 : 9;
    for(int q = 0; q < nq; q++) {
        int64_t i;
        T w, g[3], Z[3];
        node<T, d>(a, s, q, i, w, g, Z);
        T vn[3], vf[3], Zp[3], Zm[3];
#pragma unroll
        for(int k = 0; k < d; k++) {
            vn[k] = a.gv[i * d + k];
            vf[k] = a.gvf[i * d + k];
            Vpic[k] += w * vn[k];
            Vpf[k] += w * vf[k];
            T xi = Z[k] + a.dt * vn[k];
            Zp[k] = Z[k] + xi;
            Zm[k] = Z[k] - xi;
        }
#pragma unroll
        for(int c = 0; c < d; c++)
#pragma unroll
            for(int r = 0; r < d; r++) G[r + d * c] += vn[r] * g[c];
        T hw = w / 2;
#pragma unroll
        for(int c = 0; c < d; c++)
#pragma unroll
            for(int r = 0; r < d; r++) Bh[r + d * c] += hw * (vf[r] * Zp[c] + Zm[r] * vf[c]);
    }
    T* Fp = a.F + p * d * d;
    T A[9], Fn[9];
#pragma unroll
    for(int e = 0; e < d * d; e++) A[e] = a.dt * G[e];
#pragma unroll
    for(int k = 0; k < d; k++) A[k + d * k] += 1;
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++) {
            T sum = 0;
#pragma unroll
            for(int e = 0; e < d; e++) sum += A[r + d * e] * Fp[e + d * c];
            Fn[r + d * c] = sum;
        }
    T xn[3];
    bool finite = true;
#pragma unroll
    for(int k = 0; k < d; k++) xn[k] = X[k] + a.dt * Vpic[k];
    T* Bp = a.B + p * d * d;
#pragma unroll
    for(int c = 0; c < d; c++)
#pragma unroll
        for(int r = 0; r < d; r++)
            Bp[r + d * c] = Bh[r + d * c] - (T).5 * (Vpf[r] * (X[c] + xn[c]) + (X[r] - xn[r]) * Vpf[c]);
#pragma unroll
    for(int e = 0; e < d * d; e++) { Fp[e] = Fn[e]; finite = finite && isfinite(Fn[e]); }
    // Reflect_Or_Invalidate_Particle (l.1219-1239): mirrored back across a
    // non-free face, invalidated across a free one
    bool keep = true;
#pragma unroll
    for(int k = 0; k < d; k++) {
        finite = finite && isfinite(xn[k]) && isfinite(Vpf[k]);
        T eps = Lim<T>::eps * 4 * ((T)a.sp.dmax[k] - (T)a.sp.dmin[k]);
        const T A = (T)a.sp.dmin[k] + eps, B = (T)a.sp.dmax[k] - eps;
        T x = xn[k], v = Vpf[k];
        if(x < A) {
            if(a.side[2 * k] != MPM_BC_FREE) { x = 2 * A - x; v = -v; }
            else keep = false;
        } else if(x > B) {
            if(a.side[2 * k + 1] != MPM_BC_FREE) { x = 2 * B - x; v = -v; }
            else keep = false;
        }
        X[k] = x;
        a.V[p * d + k] = v;
    }
    if(!finite) { atomicOr(a.flags, MPM_FLAG_NAN); keep = false; }
    // a particle that leaves is marked 2 while plasticity still has to see it
    // (the reference updates every particle simulated in this substep)
    if(!keep) a.valid[p] = a.mark_left ? 2 : 0;
}

template<class T> __global__ void k_count_valid(const uint8_t* valid, int64_t n, unsigned long long* out)
{
    unsigned long long c = 0;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) c += valid[i] ? 1 : 0;
    atomicAdd(out, c);
}

int pblocks(int64_t n, int t) { int64_t b = (n + t - 1) / t; return (int)(b < 1 ? 1 : b); }
int gblocks(mpm_handle* h, int64_t n, int t)
{
    int64_t b = (n + t - 1) / t, cap = (int64_t)h->sm_count * 8;
    if(b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

size_t esize(mpm_handle* h) { return h->model.precision == MPM_FP64 ? 8 : 4; }

// ---------------------------------------------------------------------------
// Reflection boundary conditions (MPM_DRIVER.cpp:307-446).  One launch per
// side, in side order, over that side's ghost slab including the corner
// blocks (RANGE_ITERATOR with RI::ghost | RI::duplicate_corners): each ghost
// node pairs with its mirror image across the face, image = 2 face - index - 1
// along the side's axis.  No velocity boundary function (bc = 0).
// ---------------------------------------------------------------------------
template<class T, int d> __device__ __forceinline__ bool slab_node(const PlainArgs<T>& a, int side, int64_t t,
    int64_t& ghost, int64_t& image)
{
    const int axis = side / 2, hi = side % 2;
    int idx[3];
    int64_t r = t;
    for(int k = d - 1; k >= 0; k--) {
        const int ext = k == axis ? MPM_GHOST : a.gs[k];
        idx[k] = (int)(r % ext);
        r /= ext;
    }
    if(r) return false;
    const int G = a.gs[axis] - 2 * MPM_GHOST;
    // ghost layer along the axis, in cell coordinates, and its mirror
    const int c = hi ? G + idx[axis] : idx[axis] - MPM_GHOST;
    const int cm = hi ? 2 * G - c - 1 : -c - 1;
    int gi[3], ii[3];
    for(int k = 0; k < d; k++) { gi[k] = idx[k]; ii[k] = idx[k]; }
    gi[axis] = c + MPM_GHOST;
    ii[axis] = cm + MPM_GHOST;
    ghost = image = 0;
    for(int k = 0; k < d; k++) { ghost = ghost * a.gs[k] + gi[k]; image = image * a.gs[k] + ii[k]; }
    return true;
}

template<class T, int d> __device__ __forceinline__ int64_t slab_size(const PlainArgs<T>& a, int side)
{
    int64_t n = MPM_GHOST;
    for(int k = 0; k < d; k++) if(k != side / 2) n *= a.gs[k];
    return n;
}

// Reflect_Boundary_Mass_Momentum (l.310-341): both nodes take the total mass;
// momentum sums (free), differences (no-slip) or sums with the normal part
// differenced (slip, separate).
template<class T, int d> __global__ void k_reflect_mm(PlainArgs<T> a, int side)
{
    const int type = a.side[side], axis = side / 2;
    for(int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < slab_size<T, d>(a, side); t += (int64_t)gridDim.x * blockDim.x) {
        int64_t o, i;
        if(!slab_node<T, d>(a, side, t, o, i)) continue;
        const T mt = a.gm[i] + a.gm[o];
        T vi[3], vo[3];
        for(int k = 0; k < d; k++) {
            const T mi = a.gmv[i * d + k], mo = a.gmv[o * d + k];
            T id = mi - mo, od = -id, in = mi + mo, on = in;
            if(type == MPM_BC_SLIP && k == axis) { in = id; on = od; }
            if(type == MPM_BC_NOSLIP) { vi[k] = id; vo[k] = od; }
            else { vi[k] = in; vo[k] = on; }
        }
        for(int k = 0; k < d; k++) { a.gmv[i * d + k] = vi[k]; a.gmv[o * d + k] = vo[k]; }
        a.gm[i] = a.gm[o] = mt;
    }
}

// Reflect_Boundary_Force (l.424-446), the same folding on the forces.
template<class T, int d> __global__ void k_reflect_force(PlainArgs<T> a, int side)
{
    const int type = a.side[side], axis = side / 2;
    for(int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < slab_size<T, d>(a, side); t += (int64_t)gridDim.x * blockDim.x) {
        int64_t o, i;
        if(!slab_node<T, d>(a, side, t, o, i)) continue;
        T fi[3], fo[3];
        for(int k = 0; k < d; k++) {
            const T xi = a.gf[i * d + k], xo = a.gf[o * d + k];
            T id = xi - xo, od = -id, in = xi + xo, on = in;
            if(type == MPM_BC_SLIP && k == axis) { in = id; on = od; }
            if(type == MPM_BC_NOSLIP) { fi[k] = id; fo[k] = od; }
            else { fi[k] = in; fo[k] = on; }
        }
        for(int k = 0; k < d; k++) { a.gf[i * d + k] = fi[k]; a.gf[o * d + k] = fo[k]; }
    }
}

// Reflect_Boundary_Velocity (l.397-421): the ghost node (with mass) takes its
// image's velocity, reversed (no-slip) or with the normal part reversed (slip).
template<class T, int d> __global__ void k_reflect_vel(PlainArgs<T> a, int side, T* u)
{
    const int type = a.side[side], axis = side / 2;
    for(int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < slab_size<T, d>(a, side); t += (int64_t)gridDim.x * blockDim.x) {
        int64_t o, i;
        if(!slab_node<T, d>(a, side, t, o, i) || a.gm[o] == 0) continue;
        for(int k = 0; k < d; k++) {
            const T vi = u[i * d + k];
            T od = -vi, on = vi;
            if(type == MPM_BC_SLIP && k == axis) on = od;
            u[o * d + k] = type == MPM_BC_NOSLIP ? od : on;
        }
    }
}

// Reflect_Boundary_Friction with Reflect_Helper (l.342-395): the mass-weighted
// pair velocities, separated with Coulomb friction for BC_SEP.
template<class T, int d> __global__ void k_reflect_friction(PlainArgs<T> a, int side, T mu)
{
    const int type = a.side[side], axis = side / 2, hi = side % 2;
    for(int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < slab_size<T, d>(a, side); t += (int64_t)gridDim.x * blockDim.x) {
        int64_t o, i;
        if(!slab_node<T, d>(a, side, t, o, i)) continue;
        const T mi = a.gm[i], mo = a.gm[o];
        if(!mi || !mo) continue;
        T vi[3], vo[3], ri[3], ro[3];
        for(int k = 0; k < d; k++) { vi[k] = a.gv[i * d + k]; vo[k] = a.gv[o * d + k]; }
        const T mt = mi + mo, ai = mi / mt, ao = 1 - ai;
        T in[3], id[3], od[3];
        for(int k = 0; k < d; k++) {
            in[k] = ai * vi[k] + ao * vo[k];
            id[k] = ai * vi[k] + ao * (-vo[k]);
            od[k] = ao * vo[k] + ai * (-vi[k]);
        }
        if(type == MPM_BC_FREE) {
            for(int k = 0; k < d; k++) ri[k] = ro[k] = in[k];
        } else if(type == MPM_BC_NOSLIP) {
            for(int k = 0; k < d; k++) { ri[k] = id[k]; ro[k] = od[k]; }
        } else if(type == MPM_BC_SLIP) {
            for(int k = 0; k < d; k++) { ri[k] = ro[k] = in[k]; }
            ri[axis] = id[axis];
            ro[axis] = od[axis];
        } else {
            const T dv = 2 * ao * ai * (-vi[axis] - vo[axis]);
            const T dvn = hi ? -dv : dv;
            if(dvn < 0) {
                for(int k = 0; k < d; k++) { ri[k] = vi[k]; ro[k] = vo[k]; }
            } else {
                T idn[3] = {0, 0, 0}, odn[3] = {0, 0, 0}, tv[3];
                idn[axis] = id[axis];
                odn[axis] = od[axis];
                for(int k = 0; k < d; k++) tv[k] = in[k];
                tv[axis] = 0;
                T mag = 0;
                for(int k = 0; k < d; k++) mag += tv[k] * tv[k];
                mag = sqrt(mag);
                if(mag) { const T inv = 1 / mag; for(int k = 0; k < d; k++) tv[k] *= inv; }
                else for(int k = 0; k < d; k++) tv[k] = k == 0 ? (T)1 : (T)0;   // VECTOR::Normalize
                const T r = mag - mu * dvn;
                for(int k = 0; k < d; k++) {
                    ri[k] = r < 0 ? idn[k] : idn[k] + r * tv[k];
                    ro[k] = r < 0 ? odn[k] : odn[k] + r * tv[k];
                }
            }
        }
        for(int k = 0; k < d; k++) { a.gv[i * d + k] = ri[k]; a.gv[o * d + k] = ro[k]; }
    }
}

template<class T> __global__ void k_copy_vf(PlainArgs<T> a)
{
    const int d = a.sp.dim;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.gn * d; i += (int64_t)gridDim.x * blockDim.x) a.gvf[i] = a.gv[i];
}

enum ReflectPass { REFLECT_MM, REFLECT_FORCE, REFLECT_VEL, REFLECT_FRICTION };

template<class T> int reflect_pass(mpm_handle* h, const PlainArgs<T>& a, ReflectPass pass)
{
    const int d = h->sp.dim, t = 256;
    for(int side = 0; side < 2 * d; side++) {
        int64_t n = MPM_GHOST;
        for(int k = 0; k < d; k++) if(k != side / 2) n *= a.gs[k];
        const int b = gblocks(h, n, t);
        if(d == 3) {
            if(pass == REFLECT_MM) k_reflect_mm<T, 3><<<b, t, 0, h->stream>>>(a, side);
            else if(pass == REFLECT_FORCE) k_reflect_force<T, 3><<<b, t, 0, h->stream>>>(a, side);
            else if(pass == REFLECT_FRICTION) k_reflect_friction<T, 3><<<b, t, 0, h->stream>>>(a, side, (T)h->reflect.friction);
            else { k_reflect_vel<T, 3><<<b, t, 0, h->stream>>>(a, side, a.gv); k_reflect_vel<T, 3><<<b, t, 0, h->stream>>>(a, side, a.gvf); }
        } else {
            if(pass == REFLECT_MM) k_reflect_mm<T, 2><<<b, t, 0, h->stream>>>(a, side);
            else if(pass == REFLECT_FORCE) k_reflect_force<T, 2><<<b, t, 0, h->stream>>>(a, side);
            else if(pass == REFLECT_FRICTION) k_reflect_friction<T, 2><<<b, t, 0, h->stream>>>(a, side, (T)h->reflect.friction);
            else { k_reflect_vel<T, 2><<<b, t, 0, h->stream>>>(a, side, a.gv); k_reflect_vel<T, 2><<<b, t, 0, h->stream>>>(a, side, a.gvf); }
        }
    }
    MPM_LAUNCHED(h, "k_reflect_*");
    return MPM_OK;
}

template<class T> int p2g_t(mpm_handle* h, double dt)
{
    PlainArgs<T> a = args<T>(h, dt);
    const int t = 128;
    int slot = timer_begin(h, "plain_clear");
    k_clear<T><<<gblocks(h, a.gn, t), t, 0, h->stream>>>(a);
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_clear");
    if(a.n) {
        slot = timer_begin(h, "plain_p2g");
        if(h->sp.dim == 3) k_p2g<T, 3><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
        else k_p2g<T, 2><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
        timer_end(h, slot);
        MPM_LAUNCHED(h, "k_p2g");
    }
    if(a.reflect && !h->reflect.full_reflection) {
        int rc = reflect_pass<T>(h, a, REFLECT_MM);
        if(rc) return rc;
    }
    slot = timer_begin(h, "plain_normalize");
    k_normalize<T><<<gblocks(h, a.gn, t), t, 0, h->stream>>>(a);
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_normalize");
    return MPM_OK;
}

template<class T> int forces_t(mpm_handle* h, double dt)
{
    PlainArgs<T> a = args<T>(h, dt);
    const int t = 128;
    if(a.n) {
        int slot = timer_begin(h, "plain_stress");
        if(h->sp.dim == 3) k_stress<T, 3><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
        else k_stress<T, 2><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
        timer_end(h, slot);
        MPM_LAUNCHED(h, "k_stress");
        slot = timer_begin(h, "plain_forces");
        if(h->sp.dim == 3) k_forces<T, 3><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
        else k_forces<T, 2><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
        timer_end(h, slot);
        MPM_LAUNCHED(h, "k_forces");
    }
    if(a.reflect && !h->reflect.full_reflection) {
        int rc = reflect_pass<T>(h, a, REFLECT_FORCE);
        if(rc) return rc;
    }
    int slot = timer_begin(h, "plain_grid_update");
    if(h->sp.dim == 3) k_grid_update<T, 3><<<gblocks(h, a.gn, t), t, 0, h->stream>>>(a);
    else k_grid_update<T, 2><<<gblocks(h, a.gn, t), t, 0, h->stream>>>(a);
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_grid_update");
    if(a.reflect) {
        if(h->reflect.full_reflection) {   // no collision objects: the friction velocity is the velocity
            int rc = reflect_pass<T>(h, a, REFLECT_FRICTION);
            if(rc) return rc;
            k_copy_vf<T><<<gblocks(h, a.gn * h->sp.dim, t), t, 0, h->stream>>>(a);
            MPM_LAUNCHED(h, "k_copy_vf");
        } else {
            return reflect_pass<T>(h, a, REFLECT_VEL);
        }
    }
    return MPM_OK;
}

// ---------------------------------------------------------------------------
// MPM_DRIVER::Reduce_Dt (MPM_DRIVER.cpp:519-545) after the forces.
// ---------------------------------------------------------------------------
// Enforce_Limit_Max (l.547-574): lower s so that t (a + t b) stays within the bound.
template<class T> __device__ void limit_max(T& s, T bound, T a, T b)
{
    if(a < 0) { a = -a; b = -b; }
    if(a * a + 4 * b * bound >= 0) {
        if(s * (a + s * b) > bound) s = (2 * bound) / (a + sqrt(a * a + 4 * b * bound));
    } else {
        if(s * (a + s * b) < -bound) s = -(a + sqrt(a * a - 4 * b * bound)) / (2 * b);
    }
}

__device__ __forceinline__ double block_reduce(double v, bool take_min)
{
    __shared__ double sh[256];
    sh[threadIdx.x] = v;
    __syncthreads();
    for(int st = blockDim.x / 2; st > 0; st >>= 1) {
        if(threadIdx.x < st) sh[threadIdx.x] = take_min ? fmin(sh[threadIdx.x], sh[threadIdx.x + st]) : fmax(sh[threadIdx.x], sh[threadIdx.x + st]);
        __syncthreads();
    }
    return sh[0];
}

// Grid_To_Particle_Limit_Dt (l.577-625) per particle, min over particles:
// the scale s <= 100 of dt at which the F change (cfl_F, entrywise) and the
// displacement (cfl) of the G2P update reach their bounds.  velocity_save is
// the velocity after P2G.
template<class T, int d> __global__ void k_strong_cfl(PlainArgs<T> a, T cfl, T cfl_F, double* partial)
{
    double smin = 100;
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        if(!a.valid[p]) continue;
        Stencil<T, d> st;
        if(!make_stencil<T, d>(a, a.X + p * d, st)) continue;
        T Vp[3] = {0, 0, 0}, Vs[3] = {0, 0, 0}, G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Gs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const int nq = d == 3 ? 27 : 9;
        for(int q = 0; q < nq; q++) {
            int64_t i;
            T w, g[3], Z[3];
            node<T, d>(a, st, q, i, w, g, Z);
            for(int r = 0; r < d; r++) {
                const T vo = a.gv0[i * d + r], dvr = a.gv[i * d + r] - vo;
                Vp[r] += w * vo;
                Vs[r] += w * dvr;
                for(int c = 0; c < d; c++) { G[r + d * c] += vo * g[c]; Gs[r + d * c] += dvr * g[c]; }
            }
        }
        T s = 100;
        for(int i = 0; i < d; i++)
            for(int j = 0; j < d; j++) limit_max<T>(s, cfl_F, a.dt * G[i + d * j], a.dt * Gs[i + d * j]);
        for(int i = 0; i < d; i++) limit_max<T>(s, cfl, a.dt * Vp[i], a.dt * Vs[i]);
        smin = fmin(smin, (double)s);
    }
    const double r = block_reduce(smin, true);
    if(threadIdx.x == 0) partial[blockIdx.x] = r;
}

// Compute_Max_Sound_Speed (MPM_DRIVER.cpp:893-918): max over particles of
// ISOTROPIC_CONSTITUTIVE_MODEL::Sound_Speed of the stress derivative of F.
template<class T, int d> __global__ void k_sound_speed(PlainArgs<T> a, double* partial)
{
    double smax = 0;
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        if(!a.valid[p]) continue;
        T F[9], U[9], V[9], S[3], H[9], Bv[3], Cv[3];
        for(int e = 0; e < d * d; e++) F[e] = a.F[p * d * d + e];
        if(d == 3) svd3<T>(F, U, S, V);
        else svd2<T>(F, U, S, V);
        stress_derivative<T, d>(model_of(a, p), S, a.mu[p], a.lam[p], H, Bv, Cv);
        smax = fmax(smax, (double)sound_speed<T, d>(S, H, Bv, a.mass[p] / a.vol[p]));
    }
    const double r = block_reduce(smax, false);
    if(threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void k_fold(const double* partial, int count, int take_min, double* out)
{
    if(threadIdx.x) return;
    double r = partial[0];
    for(int b = 1; b < count; b++) r = take_min ? fmin(r, partial[b]) : fmax(r, partial[b]);
    *out = r;
}

// v = (v - vs) s + vs for the velocity and the friction velocity (l.536-544)
template<class T> __global__ void k_scale_dt(PlainArgs<T> a, T s)
{
    const int d = a.sp.dim;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.gn; i += (int64_t)gridDim.x * blockDim.x) {
        if(a.gm[i] == 0) continue;
        for(int k = 0; k < d; k++) {
            const T vs = a.gv0[i * d + k];
            a.gv[i * d + k] = (a.gv[i * d + k] - vs) * s + vs;
            a.gvf[i * d + k] = (a.gvf[i * d + k] - vs) * s + vs;
        }
    }
}

template<class T> int reduce_dt_t(mpm_handle* h, double dt, double* dt_out)
{
    PlainArgs<T> a = args<T>(h, dt);
    const mpm_dt_control& c = h->dt_control;
    *dt_out = dt;
    if(!a.n || (!c.strong_cfl && !c.sound_cfl)) return MPM_OK;
    constexpr int blocks = 128, t = 256, room = 256;   // room: partials per reduction (the implicit one uses 256)
    double *partial = nullptr, res[2] = {100, 0};
    MPM_CUDA(h, cudaMallocAsync(&partial, (2 * room + 2) * sizeof(double), h->stream));
    double* out = partial + 2 * room;
    if(c.strong_cfl) {
        if(h->sp.dim == 3) k_strong_cfl<T, 3><<<blocks, t, 0, h->stream>>>(a, (T)c.cfl, (T)c.cfl_F, partial);
        else k_strong_cfl<T, 2><<<blocks, t, 0, h->stream>>>(a, (T)c.cfl, (T)c.cfl_F, partial);
        k_fold<<<1, 32, 0, h->stream>>>(partial, blocks, 1, out);
        MPM_LAUNCHED(h, "k_strong_cfl");
    }
    if(c.sound_cfl) {
        if(h->implicit.enabled) {
            int rc = implicit_max_sound_speed(h, partial + room, out + 1);
            if(rc) return rc;
        } else {
            if(h->sp.dim == 3) k_sound_speed<T, 3><<<blocks, t, 0, h->stream>>>(a, partial + room);
            else k_sound_speed<T, 2><<<blocks, t, 0, h->stream>>>(a, partial + room);
            k_fold<<<1, 32, 0, h->stream>>>(partial + room, blocks, 0, out + 1);
            MPM_LAUNCHED(h, "k_sound_speed");
        }
    }
    MPM_CUDA(h, cudaMemcpyAsync(res, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaFreeAsync(partial, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    double nd = dt;
    if(c.strong_cfl && (T)(dt * res[0]) < (T)nd) nd = (T)(dt * res[0]);
    if(c.sound_cfl) {   // Limit_Dt_Sound_Speed, with Robust_Divide
        T dxm = (T)h->sp.dx[0];
        for(int k = 1; k < h->sp.dim; k++) dxm = dxm < (T)h->sp.dx[k] ? dxm : (T)h->sp.dx[k];
        const T sp = (T)res[1];
        T q;
        if(fabs(sp) == (T)FLT_MAX) q = 0;
        else if(fabs(sp) > 1 || fabs(dxm) < (T)FLT_MAX * fabs(sp)) q = dxm / sp;
        else q = ((dxm > 0) == (sp >= 0)) ? (T)FLT_MAX : -(T)FLT_MAX;
        const T nds = q * (T)c.cfl_sound;
        nd = (T)nd < nds ? nd : (double)nds;
    }
    nd = (T)nd > (T)c.min_dt ? nd : c.min_dt;
    if((T)nd >= (T)dt * (T)0.99) return MPM_OK;
    const T sc = (T)nd / (T)dt;
    k_scale_dt<T><<<gblocks(h, a.gn, t), t, 0, h->stream>>>(a, sc);
    MPM_LAUNCHED(h, "k_scale_dt");
    *dt_out = (double)(T)nd;
    return MPM_OK;
}

// MPM_DRIVER::Update_Plasticity_And_Hardening (MPM_DRIVER.cpp:922-928) with
// MPM_PLASTICITY_CLAMP, over the valid particles after G2P.
template<class T, int d> __global__ void k_plastic_clamp(PlainArgs<T> a, T* Fp, const T* mu0, const T* lam0, Vec4<T> prm)
{
    T* mu = const_cast<T*>(a.mu);
    T* lam = const_cast<T*>(a.lam);
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        if(!a.valid[p]) continue;
        if(a.valid[p] == 2) a.valid[p] = 0;   // left the domain in this G2P: updated once more
        if(a.pmask && !a.pmask[p]) continue;
        T F[d * d], P[d * d];
#pragma unroll
        for(int k = 0; k < d * d; k++) { F[k] = a.F[p * d * d + k]; P[k] = Fp[p * d * d + k]; }
        T m = mu[p], l = lam[p];
        bool ok;
        if(plastic_clamp<T, d>(F, P, m, l, mu0[p], lam0[p], prm.v, ok)) {
#pragma unroll
            for(int k = 0; k < d * d; k++) { a.F[p * d * d + k] = F[k]; Fp[p * d * d + k] = P[k]; }
            mu[p] = m;
            lam[p] = l;
        }
        if(!ok) atomicOr(a.flags, MPM_FLAG_NOT_CONVERGED);
    }
}

// MPM_DRUCKER_PRAGER after G2P over the particles simulated in the substep.
template<class T, int d> __global__ void k_plastic_dp(PlainArgs<T> a, T* Fp, T* q, T* rhoF, T* sigY, T* vc, Vec5<T> prm)
{
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        if(!a.valid[p]) continue;
        if(a.valid[p] == 2) a.valid[p] = 0;
        if(a.pmask && !a.pmask[p]) continue;
        T F[d * d], P[d * d], st[4] = {q[p], rhoF[p], sigY[p], vc[p]};
#pragma unroll
        for(int k = 0; k < d * d; k++) { F[k] = a.F[p * d * d + k]; P[k] = Fp[p * d * d + k]; }
        bool ok;
        const bool changed = plastic_dp<T, d>(F, P, a.mu[p], a.lam[p], st, prm.v, ok);
        if(changed) {
#pragma unroll
            for(int k = 0; k < d * d; k++) { a.F[p * d * d + k] = F[k]; Fp[p * d * d + k] = P[k]; }
        }
        q[p] = st[0]; rhoF[p] = st[1]; vc[p] = st[3];
        if(!ok) atomicOr(a.flags, MPM_FLAG_NOT_CONVERGED);
    }
}

// Drucker-Prager start (MPM_DRUCKER_PRAGER::Initialize_Particles): Fp = I,
// plastic_def = vc = 0, sigma_Y = cohesion, rho_F at zero plastic deformation;
// particles outside `mask` keep the arrays' zero state.
template<class T, int d> __global__ void k_dp_init(int64_t n, T* Fp, T* q, T* rhoF, T* sigY, T* vc, T cohesion, Vec5<T> prm,
    const uint8_t* mask)
{
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for(int k = 0; k < d * d; k++) Fp[p * d * d + k] = k % (d + 1) == 0 ? (T)1 : (T)0;
        T qq = 0, r = 0;
        const bool on = !mask || mask[p];
        if(on) dp_hardening<T>(qq, r, (T)0, prm.v);
        q[p] = qq; rhoF[p] = r; sigY[p] = on ? cohesion : (T)0; vc[p] = 0;
    }
}

template<class T> Vec5<T> dp_params(const mpm_plasticity_desc& pl)
{
    return {{(T)pl.dp_a0, (T)pl.dp_a1, (T)pl.dp_a3, (T)pl.dp_a4, (T)(pl.use_vc ? 1 : 0)}};
}

// Unplastic start: Fp = I, mu0 = mu, lambda0 = lambda.
template<class T, int d> __global__ void k_plastic_init(int64_t n, T* Fp, T* mu0, T* lam0, const T* mu, const T* lam)
{
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for(int k = 0; k < d * d; k++) Fp[p * d * d + k] = k % (d + 1) == 0 ? (T)1 : (T)0;
        mu0[p] = mu[p];
        lam0[p] = lam[p];
    }
}

template<class T> int g2p_t(mpm_handle* h, double dt)
{
    PlainArgs<T> a = args<T>(h, dt);
    if(!a.n) return MPM_OK;
    const int t = 128;
    int slot = timer_begin(h, "plain_g2p");
    if(h->sp.dim == 3) k_g2p<T, 3><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
    else k_g2p<T, 2><<<pblocks(a.n, t), t, 0, h->stream>>>(a);
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_g2p");
    if(h->plastic.kind == MPM_PLASTICITY_CLAMP) {
        PlainState& s = h->plain;
        Vec4<T> prm = {{(T)h->plastic.theta_c, (T)h->plastic.theta_s, (T)h->plastic.max_hardening, (T)h->plastic.hardening_factor}};
        slot = timer_begin(h, "plain_plasticity");
        if(h->sp.dim == 3) k_plastic_clamp<T, 3><<<pblocks(a.n, t), t, 0, h->stream>>>(a, (T*)s.Fp, (const T*)s.mu0, (const T*)s.lam0, prm);
        else k_plastic_clamp<T, 2><<<pblocks(a.n, t), t, 0, h->stream>>>(a, (T*)s.Fp, (const T*)s.mu0, (const T*)s.lam0, prm);
        timer_end(h, slot);
        MPM_LAUNCHED(h, "k_plastic_clamp");
    } else if(h->plastic.kind == MPM_PLASTICITY_DRUCKER_PRAGER) {
        PlainState& s = h->plain;
        const Vec5<T> prm = dp_params<T>(h->plastic);
        slot = timer_begin(h, "plain_plasticity");
        if(h->sp.dim == 3)
            k_plastic_dp<T, 3><<<pblocks(a.n, t), t, 0, h->stream>>>(a, (T*)s.Fp, (T*)s.pdef, (T*)s.rhoF, (T*)s.sigY, (T*)s.vc, prm);
        else
            k_plastic_dp<T, 2><<<pblocks(a.n, t), t, 0, h->stream>>>(a, (T*)s.Fp, (T*)s.pdef, (T*)s.rhoF, (T*)s.sigY, (T*)s.vc, prm);
        timer_end(h, slot);
        MPM_LAUNCHED(h, "k_plastic_dp");
    }
    return MPM_OK;
}

template<class Tin, class Tout> __global__ void k_convert(const Tin* in, Tout* out, int64_t n)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) out[i] = (Tout)in[i];
}

}  // namespace

int plain_alloc(mpm_handle* h, int64_t n)
{
    PlainState& s = h->plain;
    const int d = h->sp.dim;
    size_t e = esize(h);
    int64_t gn = 1;
    for(int k = 0; k < d; k++) gn *= h->sp.counts[k] + 2 * MPM_GHOST;
    if(s.gn != gn) {
        void** g[] = {&s.gm, &s.gmv, &s.gv0, &s.gf, &s.gv, &s.gvf};
        for(void** p: g) { cudaFree(*p); *p = nullptr; }
        MPM_CUDA(h, cudaMalloc(&s.gm, gn * e));
        for(int i = 1; i < 6; i++) MPM_CUDA(h, cudaMalloc(g[i], gn * d * e));
        s.gn = gn;
        for(void** p: g) MPM_CUDA(h, cudaMemsetAsync(*p, 0, (p == &s.gm ? gn : gn * d) * e, h->stream));
    }
    if(s.n != n) {
        void** pa[] = {&s.X, &s.V, &s.F, &s.B, &s.mass, &s.vol, &s.mu, &s.lam, &s.pft, &s.Fp, &s.mu0, &s.lam0,
                       &s.pdef, &s.rhoF, &s.sigY, &s.vc};
        for(void** p: pa) { cudaFree(*p); *p = nullptr; }
        cudaFree(s.valid); s.valid = nullptr;
        cudaFree(s.pmodel); s.pmodel = nullptr;
        cudaFree(s.pmask); s.pmask = nullptr;
        int64_t m = n ? n : 1;
        MPM_CUDA(h, cudaMalloc(&s.X, m * d * e));
        MPM_CUDA(h, cudaMalloc(&s.V, m * d * e));
        MPM_CUDA(h, cudaMalloc(&s.F, m * d * d * e));
        MPM_CUDA(h, cudaMalloc(&s.B, m * d * d * e));
        MPM_CUDA(h, cudaMalloc(&s.pft, m * d * d * e));
        MPM_CUDA(h, cudaMalloc(&s.mass, m * e));
        MPM_CUDA(h, cudaMalloc(&s.vol, m * e));
        MPM_CUDA(h, cudaMalloc(&s.mu, m * e));
        MPM_CUDA(h, cudaMalloc(&s.lam, m * e));
        MPM_CUDA(h, cudaMalloc(&s.valid, m));
        s.n = n;
    }
    return MPM_OK;
}

void plain_free(mpm_handle* h)
{
    PlainState& s = h->plain;
    void* ps[] = {s.X, s.V, s.F, s.B, s.mass, s.vol, s.mu, s.lam, s.pft, s.valid, s.gm, s.gmv, s.gv0, s.gf, s.gv, s.gvf,
                  s.Fp, s.mu0, s.lam0, s.pdef, s.rhoF, s.sigY, s.vc, s.pmodel, s.pmask};
    for(void* p: ps) cudaFree(p);
    s = PlainState();
}

// Copy one array in, converting between the caller's and the path's scalar type.
static int copy_in(mpm_handle* h, void* dst, const void* src, int64_t count, int src_dtype, bool src_dev)
{
    size_t e = esize(h), se = src_dtype == MPM_FP64 ? 8 : 4;
    if(!src) return set_error(h, MPM_ERR_ARG, "null particle array");
    if(se == e) {
        MPM_CUDA(h, cudaMemcpyAsync(dst, src, count * e, src_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
        return MPM_OK;
    }
    void* tmp = const_cast<void*>(src);
    void* owned = nullptr;
    if(!src_dev) {
        MPM_CUDA(h, cudaMallocAsync(&owned, count * se, h->stream));
        MPM_CUDA(h, cudaMemcpyAsync(owned, src, count * se, cudaMemcpyHostToDevice, h->stream));
        tmp = owned;
    }
    int b = (int)((count + 255) / 256);
    if(b > 4096) b = 4096;
    if(b < 1) b = 1;
    if(se == 8) k_convert<double, float><<<b, 256, 0, h->stream>>>((const double*)tmp, (float*)dst, count);
    else k_convert<float, double><<<b, 256, 0, h->stream>>>((const float*)tmp, (double*)dst, count);
    MPM_LAUNCHED(h, "k_convert");
    if(owned) MPM_CUDA(h, cudaFreeAsync(owned, h->stream));
    return MPM_OK;
}

static int copy_out(mpm_handle* h, void* dst, const void* src, int64_t count, int dst_dtype, bool dst_dev)
{
    size_t e = esize(h), de = dst_dtype == MPM_FP64 ? 8 : 4;
    if(!dst) return MPM_OK;
    if(de == e) {
        MPM_CUDA(h, cudaMemcpyAsync(dst, src, count * e, dst_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
        return MPM_OK;
    }
    void* tmp = dst;
    void* owned = nullptr;
    if(!dst_dev) {
        MPM_CUDA(h, cudaMallocAsync(&owned, count * de, h->stream));
        tmp = owned;
    }
    int b = (int)((count + 255) / 256);
    if(b > 4096) b = 4096;
    if(b < 1) b = 1;
    if(e == 8) k_convert<double, float><<<b, 256, 0, h->stream>>>((const double*)src, (float*)tmp, count);
    else k_convert<float, double><<<b, 256, 0, h->stream>>>((const float*)src, (double*)tmp, count);
    MPM_LAUNCHED(h, "k_convert");
    if(owned) {
        MPM_CUDA(h, cudaMemcpyAsync(dst, owned, count * de, cudaMemcpyDeviceToHost, h->stream));
        MPM_CUDA(h, cudaFreeAsync(owned, h->stream));
    }
    return MPM_OK;
}

int plain_set_particles(mpm_handle* h, const mpm_particles_view* v)
{
    int rc = plain_alloc(h, v->n);
    if(rc) return rc;
    PlainState& s = h->plain;
    const int d = h->sp.dim;
    bool dev = v->on_device != 0;
    int64_t n = v->n;
    if(!n) return MPM_OK;
    if((rc = copy_in(h, s.X, v->X, n * d, v->dtype, dev))) return rc;
    if((rc = copy_in(h, s.V, v->V, n * d, v->dtype, dev))) return rc;
    if((rc = copy_in(h, s.F, v->F, n * d * d, v->dtype, dev))) return rc;
    if((rc = copy_in(h, s.B, v->B, n * d * d, v->dtype, dev))) return rc;
    if((rc = copy_in(h, s.mass, v->mass, n, v->dtype, dev))) return rc;
    if((rc = copy_in(h, s.vol, v->volume, n, v->dtype, dev))) return rc;
    if((rc = copy_in(h, s.mu, v->mu, n, v->dtype, dev))) return rc;
    if((rc = copy_in(h, s.lam, v->lambda, n, v->dtype, dev))) return rc;
    if(v->valid) MPM_CUDA(h, cudaMemcpyAsync(s.valid, v->valid, n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
    else MPM_CUDA(h, cudaMemsetAsync(s.valid, 1, n, h->stream));
    if(h->plastic.kind) return plain_plastic_init(h);
    return MPM_OK;
}

// Allocate the plastic state if needed and start it unplastic.
int plain_plastic_init(mpm_handle* h)
{
    PlainState& s = h->plain;
    const int d = h->sp.dim;
    const size_t e = esize(h);
    const int64_t m = s.n ? s.n : 1;
    if(!s.Fp) {
        MPM_CUDA(h, cudaMalloc(&s.Fp, m * d * d * e));
        void** pa[] = {&s.mu0, &s.lam0, &s.pdef, &s.rhoF, &s.sigY, &s.vc};
        for(void** p: pa) MPM_CUDA(h, cudaMalloc(p, m * e));
    }
    if(!s.n) return MPM_OK;
    const int b = gblocks(h, s.n, 256);
    if(h->plastic.kind == MPM_PLASTICITY_DRUCKER_PRAGER) {
        const double c = h->plastic.cohesion;
        if(e == 8) {
            const Vec5<double> prm = dp_params<double>(h->plastic);
            if(d == 3) k_dp_init<double, 3><<<b, 256, 0, h->stream>>>(s.n, (double*)s.Fp, (double*)s.pdef, (double*)s.rhoF, (double*)s.sigY, (double*)s.vc, c, prm, s.pmask);
            else k_dp_init<double, 2><<<b, 256, 0, h->stream>>>(s.n, (double*)s.Fp, (double*)s.pdef, (double*)s.rhoF, (double*)s.sigY, (double*)s.vc, c, prm, s.pmask);
        } else {
            const Vec5<float> prm = dp_params<float>(h->plastic);
            if(d == 3) k_dp_init<float, 3><<<b, 256, 0, h->stream>>>(s.n, (float*)s.Fp, (float*)s.pdef, (float*)s.rhoF, (float*)s.sigY, (float*)s.vc, (float)c, prm, s.pmask);
            else k_dp_init<float, 2><<<b, 256, 0, h->stream>>>(s.n, (float*)s.Fp, (float*)s.pdef, (float*)s.rhoF, (float*)s.sigY, (float*)s.vc, (float)c, prm, s.pmask);
        }
        MPM_LAUNCHED(h, "k_dp_init");
        return MPM_OK;
    }
    if(e == 8) {
        if(d == 3) k_plastic_init<double, 3><<<b, 256, 0, h->stream>>>(s.n, (double*)s.Fp, (double*)s.mu0, (double*)s.lam0, (const double*)s.mu, (const double*)s.lam);
        else k_plastic_init<double, 2><<<b, 256, 0, h->stream>>>(s.n, (double*)s.Fp, (double*)s.mu0, (double*)s.lam0, (const double*)s.mu, (const double*)s.lam);
    } else {
        if(d == 3) k_plastic_init<float, 3><<<b, 256, 0, h->stream>>>(s.n, (float*)s.Fp, (float*)s.mu0, (float*)s.lam0, (const float*)s.mu, (const float*)s.lam);
        else k_plastic_init<float, 2><<<b, 256, 0, h->stream>>>(s.n, (float*)s.Fp, (float*)s.mu0, (float*)s.lam0, (const float*)s.mu, (const float*)s.lam);
    }
    MPM_LAUNCHED(h, "k_plastic_init");
    return MPM_OK;
}

int plain_get_plastic(mpm_handle* h, mpm_plastic_view* v)
{
    PlainState& s = h->plain;
    const int d = h->sp.dim;
    if(v->n != s.n) return set_error(h, MPM_ERR_ARG, "particle count differs from mpm_set_particles");
    if(!v->n) return MPM_OK;
    const bool dev = v->on_device != 0;
    const int64_t n = v->n;
    int rc;
    if(v->Fp && (rc = copy_out(h, v->Fp, s.Fp, n * d * d, v->dtype, dev))) return rc;
    if(v->mu && (rc = copy_out(h, v->mu, s.mu, n, v->dtype, dev))) return rc;
    if(v->lambda && (rc = copy_out(h, v->lambda, s.lam, n, v->dtype, dev))) return rc;
    if(v->mu0 && (rc = copy_out(h, v->mu0, s.mu0, n, v->dtype, dev))) return rc;
    if(v->lambda0 && (rc = copy_out(h, v->lambda0, s.lam0, n, v->dtype, dev))) return rc;
    if(v->plastic_def && (rc = copy_out(h, v->plastic_def, s.pdef, n, v->dtype, dev))) return rc;
    if(v->rho_F && (rc = copy_out(h, v->rho_F, s.rhoF, n, v->dtype, dev))) return rc;
    if(v->cohesion && (rc = copy_out(h, v->cohesion, s.sigY, n, v->dtype, dev))) return rc;
    if(v->vc && (rc = copy_out(h, v->vc, s.vc, n, v->dtype, dev))) return rc;
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

int plain_set_plastic(mpm_handle* h, const mpm_plastic_view* v)
{
    PlainState& s = h->plain;
    const int d = h->sp.dim;
    if(v->n != s.n) return set_error(h, MPM_ERR_ARG, "particle count differs from mpm_set_particles");
    if(!v->n) return MPM_OK;
    const bool dev = v->on_device != 0;
    const int64_t n = v->n;
    int rc;
    if(v->Fp && (rc = copy_in(h, s.Fp, v->Fp, n * d * d, v->dtype, dev))) return rc;
    if(v->mu && (rc = copy_in(h, s.mu, v->mu, n, v->dtype, dev))) return rc;
    if(v->lambda && (rc = copy_in(h, s.lam, v->lambda, n, v->dtype, dev))) return rc;
    if(v->mu0 && (rc = copy_in(h, s.mu0, v->mu0, n, v->dtype, dev))) return rc;
    if(v->lambda0 && (rc = copy_in(h, s.lam0, v->lambda0, n, v->dtype, dev))) return rc;
    if(v->plastic_def && (rc = copy_in(h, s.pdef, v->plastic_def, n, v->dtype, dev))) return rc;
    if(v->rho_F && (rc = copy_in(h, s.rhoF, v->rho_F, n, v->dtype, dev))) return rc;
    if(v->cohesion && (rc = copy_in(h, s.sigY, v->cohesion, n, v->dtype, dev))) return rc;
    if(v->vc && (rc = copy_in(h, s.vc, v->vc, n, v->dtype, dev))) return rc;
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

int plain_get_particles(mpm_handle* h, mpm_particles_view* v)
{
    PlainState& s = h->plain;
    const int d = h->sp.dim;
    if(v->n != s.n) return set_error(h, MPM_ERR_ARG, "particle count differs from mpm_set_particles");
    bool dev = v->on_device != 0;
    int64_t n = v->n;
    if(!n) return MPM_OK;
    int rc;
    if((rc = copy_out(h, v->X, s.X, n * d, v->dtype, dev))) return rc;
    if((rc = copy_out(h, v->V, s.V, n * d, v->dtype, dev))) return rc;
    if((rc = copy_out(h, v->F, s.F, n * d * d, v->dtype, dev))) return rc;
    if((rc = copy_out(h, v->B, s.B, n * d * d, v->dtype, dev))) return rc;
    if(v->valid) MPM_CUDA(h, cudaMemcpyAsync(v->valid, s.valid, n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

int plain_p2g(mpm_handle* h, double dt, double)
{
    return h->model.precision == MPM_FP64 ? p2g_t<double>(h, dt) : p2g_t<float>(h, dt);
}
int plain_forces(mpm_handle* h, double dt, double)
{
    return h->model.precision == MPM_FP64 ? forces_t<double>(h, dt) : forces_t<float>(h, dt);
}
int plain_reflect_velocity(mpm_handle* h)
{
    if(h->model.precision == MPM_FP64) return reflect_pass<double>(h, args<double>(h, 0.0), REFLECT_VEL);
    return reflect_pass<float>(h, args<float>(h, 0.0), REFLECT_VEL);
}
int plain_reduce_dt(mpm_handle* h, double dt, double* dt_out)
{
    return h->model.precision == MPM_FP64 ? reduce_dt_t<double>(h, dt, dt_out) : reduce_dt_t<float>(h, dt, dt_out);
}
int plain_g2p(mpm_handle* h, double dt, double)
{
    return h->model.precision == MPM_FP64 ? g2p_t<double>(h, dt) : g2p_t<float>(h, dt);
}

int plain_get_grid(mpm_handle* h, double* m, double* v0, double* v, double* vf)
{
    PlainState& s = h->plain;
    const int d = h->sp.dim;
    int rc;
    if(m && (rc = copy_out(h, m, s.gm, s.gn, MPM_FP64, false))) return rc;
    if(v0 && (rc = copy_out(h, v0, s.gv0, s.gn * d, MPM_FP64, false))) return rc;
    if(v && (rc = copy_out(h, v, s.gv, s.gn * d, MPM_FP64, false))) return rc;
    if(vf && (rc = copy_out(h, vf, s.gvf, s.gn * d, MPM_FP64, false))) return rc;
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

namespace {
// Extra node forces into the grid force array of the current substep (after
// P2G cleared it and before the grid update reads it).
template<class T, class S> __global__ void k_add_forces(T* gf, const S* f, int64_t count)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        gf[i] += (T)f[i];
}
}  // namespace

int plain_add_forces(mpm_handle* h, const void* f, int dtype, bool on_device)
{
    PlainState& s = h->plain;
    const int64_t count = s.gn * h->sp.dim;
    const size_t e = dtype == MPM_FP64 ? 8 : 4;
    if(!count) return MPM_OK;
    const void* src = f;
    void* stage = nullptr;
    if(!on_device) {
        MPM_CUDA(h, cudaMallocAsync(&stage, count * e, h->stream));
        MPM_CUDA(h, cudaMemcpyAsync(stage, f, count * e, cudaMemcpyHostToDevice, h->stream));
        src = stage;
    }
    const int blocks = gblocks(h, count, 256);
    if(h->model.precision == MPM_FP64) {
        if(e == 8) k_add_forces<double, double><<<blocks, 256, 0, h->stream>>>((double*)s.gf, (const double*)src, count);
        else k_add_forces<double, float><<<blocks, 256, 0, h->stream>>>((double*)s.gf, (const float*)src, count);
    } else {
        if(e == 8) k_add_forces<float, double><<<blocks, 256, 0, h->stream>>>((float*)s.gf, (const double*)src, count);
        else k_add_forces<float, float><<<blocks, 256, 0, h->stream>>>((float*)s.gf, (const float*)src, count);
    }
    MPM_LAUNCHED(h, "k_add_forces");
    if(stage) MPM_CUDA(h, cudaFreeAsync(stage, h->stream));
    return MPM_OK;
}

int plain_count_valid(mpm_handle* h, int64_t* c)
{
    unsigned long long* d = nullptr;
    MPM_CUDA(h, cudaMallocAsync(&d, sizeof(*d), h->stream));
    MPM_CUDA(h, cudaMemsetAsync(d, 0, sizeof(*d), h->stream));
    if(h->plain.n) {
        k_count_valid<float><<<gblocks(h, h->plain.n, 256), 256, 0, h->stream>>>(h->plain.valid, h->plain.n, d);
        MPM_LAUNCHED(h, "k_count_valid");
    }
    unsigned long long r = 0;
    MPM_CUDA(h, cudaMemcpyAsync(&r, d, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaFreeAsync(d, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    *c = (int64_t)r;
    return MPM_OK;
}

// ---------------------------------------------------------------------------
// Diagnostics in FP64 (MPM_EXAMPLE::Total_Particle_* / Total_Grid_*,
// MPM_EXAMPLE.cpp:209-327; MPM_DRIVER::Max_Particle_Speed / Grid_V_Upper_Bound,
// MPM_DRIVER.cpp:1112-1138).  2D angular momentum goes to component 0.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ void pwarp_add(double* acc, double v)
{
#pragma unroll
    for(int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if((threadIdx.x & 31) == 0 && v != 0) atomicAdd(acc, v);
}
__device__ __forceinline__ void pwarp_max(unsigned long long* mx, double v)
{
#pragma unroll
    for(int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if((threadIdx.x & 31) == 0) atomicMax(mx, (unsigned long long)__double_as_longlong(v));
}

template<class T> __global__ void k_plain_particle_totals(PlainArgs<T> a, double* acc, unsigned long long* mx)
{
    const int d = a.sp.dim;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, vmax = 0, amax = 0;
    double inv_min = a.sp.inv_dx[0];
    for(int k = 1; k < d; k++) inv_min = fmin(inv_min, a.sp.inv_dx[k]);
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        if(!a.valid[p]) continue;
        double X[3] = {0, 0, 0}, V[3] = {0, 0, 0}, B[9];
        for(int k = 0; k < d; k++) { X[k] = a.X[p * d + k]; V[k] = a.V[p * d + k]; }
        for(int k = 0; k < d * d; k++) B[k] = a.B[p * d * d + k];
        double m = a.mass[p];
        s[0] += m;
        for(int k = 0; k < d; k++) s[1 + k] += m * V[k];
        if(d == 3) {
            s[4] += m * (X[1] * V[2] - X[2] * V[1]) - m * (B[7] - B[5]);
            s[5] += m * (X[2] * V[0] - X[0] * V[2]) - m * (B[2] - B[6]);
            s[6] += m * (X[0] * V[1] - X[1] * V[0]) - m * (B[3] - B[1]);
        } else {
            s[4] += m * (X[0] * V[1] - X[1] * V[0]) - m * (B[2] - B[1]);
        }
        double v2 = 0, bd = 0, bf = 0;
        for(int k = 0; k < d; k++) v2 += V[k] * V[k];
        for(int c = 0; c < d; c++)
            for(int r = 0; r < d; r++) {
                double b2 = B[r + d * c] * B[r + d * c];
                bd += b2 * 4.0 * a.sp.inv_dx[c] * a.sp.inv_dx[c];
                bf += b2;
            }
        s[7] += 0.5 * m * v2 + 0.5 * m * bd;
        s[8] += 1;
        double sp = sqrt(v2);
        vmax = fmax(vmax, sp);
        amax = fmax(amax, sp + sqrt(bf) * 6.0 * sqrt((double)d) * inv_min);
    }
    for(int k = 0; k < 9; k++) pwarp_add(acc + k, s[k]);
    pwarp_max(mx, vmax);
    pwarp_max(mx + 1, amax);
}

template<class T> __global__ void k_plain_grid_totals(PlainArgs<T> a, double* acc)
{
    const int d = a.sp.dim;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.gn; i += (int64_t)gridDim.x * blockDim.x) {
        double m = a.gm[i];
        if(m == 0) continue;
        int64_t r = i;
        int idx[3] = {0, 0, 0};
        for(int k = d - 1; k >= 0; k--) { idx[k] = (int)(r % a.gs[k]) - MPM_GHOST; r /= a.gs[k]; }
        double X[3] = {0, 0, 0}, v[3] = {0, 0, 0};
        for(int k = 0; k < d; k++) {
            X[k] = a.sp.dmin[k] + ((double)idx[k] + 0.5) * a.sp.dx[k];
            v[k] = a.gv[i * d + k];
        }
        s[0] += m;
        for(int k = 0; k < d; k++) s[1 + k] += m * v[k];
        if(d == 3) {
            s[4] += m * (X[1] * v[2] - X[2] * v[1]);
            s[5] += m * (X[2] * v[0] - X[0] * v[2]);
            s[6] += m * (X[0] * v[1] - X[1] * v[0]);
        } else {
            s[4] += m * (X[0] * v[1] - X[1] * v[0]);
        }
        s[7] += 0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        s[8] += 1;
    }
    for(int k = 0; k < 9; k++) pwarp_add(acc + k, s[k]);
}
}  // namespace

static int plain_totals(mpm_handle* h, bool grid, mpm_totals* out)
{
    double* d = nullptr;
    MPM_CUDA(h, cudaMallocAsync((void**)&d, 16 * sizeof(double), h->stream));
    MPM_CUDA(h, cudaMemsetAsync(d, 0, 16 * sizeof(double), h->stream));
    const int t = 256;
    if(h->model.precision == MPM_FP64) {
        PlainArgs<double> a = args<double>(h, 0.0);
        if(grid) k_plain_grid_totals<double><<<gblocks(h, a.gn, t), t, 0, h->stream>>>(a, d);
        else if(a.n) k_plain_particle_totals<double><<<gblocks(h, a.n, t), t, 0, h->stream>>>(a, d, (unsigned long long*)(d + 12));
    } else {
        PlainArgs<float> a = args<float>(h, 0.0);
        if(grid) k_plain_grid_totals<float><<<gblocks(h, a.gn, t), t, 0, h->stream>>>(a, d);
        else if(a.n) k_plain_particle_totals<float><<<gblocks(h, a.n, t), t, 0, h->stream>>>(a, d, (unsigned long long*)(d + 12));
    }
    MPM_LAUNCHED(h, "k_plain_totals");
    double acc[9];
    unsigned long long mx[2];
    MPM_CUDA(h, cudaMemcpyAsync(acc, d, sizeof acc, cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(mx, d + 12, sizeof mx, cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaFreeAsync(d, h->stream);
    out->mass = acc[0];
    for(int k = 0; k < 3; k++) { out->momentum[k] = acc[1 + k]; out->angular_momentum[k] = acc[4 + k]; }
    out->kinetic_energy = acc[7];
    out->count = (int64_t)acc[8];
    memcpy(&out->max_speed, &mx[0], 8);
    memcpy(&out->max_affine_speed, &mx[1], 8);
    if(grid) out->max_speed = out->max_affine_speed = 0;
    return MPM_OK;
}

int plain_particle_totals(mpm_handle* h, mpm_totals* out) { return plain_totals(h, false, out); }
int plain_grid_totals(mpm_handle* h, mpm_totals* out) { return plain_totals(h, true, out); }

// This module's copy of the SVD sweep bound (mpm_debug_set_svd_iterations).
MPM_SVD_LIMIT_SETTER(svd_limit_plain)
