// Reference-layout kernel arguments and the particle stencil shared by the
// plain path (mpm_plain.cu) and the implicit solve (mpm_implicit.cu).
#pragma once
#include "mpm_internal.h"

namespace plain {

using namespace mpm;

template<class T> struct PlainArgs {
    SceneParams sp;
    int64_t n, gn;
    int gs[3];
    T *X, *V, *F, *B;
    const T *mass, *vol, *mu, *lam;
    T* pft;
    uint8_t* valid;
    T *gm, *gmv, *gv0, *gf, *gv, *gvf;
    T dt;
    unsigned* flags;
    int mark_left;
    int reflect;          // reflection boundary conditions on
    int side[6];          // their types per side (mpm_bc_type)
    const ObjMotion* motion;   // moving collision objects (bit j of `moving`): their substep frames
    unsigned moving;
    const uint8_t* pmodel;     // per-particle constitutive model, or null (sp.model for all)
    const uint8_t* pmask;      // particles the plasticity acts on, or null (all)
};

// The constitutive model of particle p: its own, or the handle's.
template<class T> __device__ __forceinline__ int model_of(const PlainArgs<T>& a, int64_t p)
{
    return a.pmodel ? (int)a.pmodel[p] : a.sp.model;
}

template<class T, int d> struct Stencil {
    Axis<T> ax[3];
    int base[3];
};

// Weights of one particle; returns false if the 3^d stencil leaves the ghosted grid.
template<class T, int d> __device__ bool make_stencil(const PlainArgs<T>& a, const T* X, Stencil<T, d>& s)
{
    bool ok = true;
#pragma unroll
    for(int k = 0; k < d; k++) {
        s.ax[k] = spline_axis<T>(X[k], (T)a.sp.dmin[k], (T)a.sp.dx[k], (T)a.sp.inv_dx[k]);
        s.base[k] = s.ax[k].base;
        int lo = s.base[k] + MPM_GHOST, hi = lo + 2;
        if(lo < 0 || hi >= a.gs[k]) ok = false;
    }
    return ok;
}

// Tensor-product node q (RANGE_ITERATOR order, last axis fastest):
// PARTICLE_GRID_WEIGHTS_SPLINE::Compute (PARTICLE_GRID_WEIGHTS_SPLINE.cpp:33-56).
template<class T, int d> __device__ __forceinline__ void node(const PlainArgs<T>& a, const Stencil<T, d>& s, int q,
    int64_t& flat, T& w, T* g, T* Z)
{
    int off[3];
    if(d == 3) { off[0] = q / 9; off[1] = (q / 3) % 3; off[2] = q % 3; }
    else { off[0] = q / 3; off[1] = q % 3; off[2] = 0; }
    T aw[3];
#pragma unroll
    for(int k = 0; k < d; k++) aw[k] = s.ax[k].w[off[k]];
    w = aw[0] * aw[1];
    if(d == 3) w *= aw[2];
#pragma unroll
    for(int k = 0; k < d; k++) g[k] = 1;
#pragma unroll
    for(int j = 0; j < d; j++) {
        T dj = s.ax[j].dw[off[j]];
#pragma unroll
        for(int i = 0; i < d; i++) g[i] *= i == j ? dj : aw[j];
    }
    flat = 0;
#pragma unroll
    for(int k = 0; k < d; k++) {
        int idx = s.base[k] + off[k];
        flat = flat * a.gs[k] + (idx + MPM_GHOST);
        Z[k] = (T)a.sp.dmin[k] + ((T)idx + (T).5) * (T)a.sp.dx[k];
    }
}

template<class T> inline PlainArgs<T> args(mpm_handle* h, double dt)
{
    PlainArgs<T> a;
    PlainState& s = h->plain;
    a.sp = h->sp;
    a.n = s.n;
    a.gn = s.gn;
    for(int k = 0; k < 3; k++) a.gs[k] = k < h->sp.dim ? h->sp.counts[k] + 2 * MPM_GHOST : 1;
    a.X = (T*)s.X; a.V = (T*)s.V; a.F = (T*)s.F; a.B = (T*)s.B;
    a.mass = (const T*)s.mass; a.vol = (const T*)s.vol; a.mu = (const T*)s.mu; a.lam = (const T*)s.lam;
    a.pft = (T*)s.pft; a.valid = s.valid;
    a.gm = (T*)s.gm; a.gmv = (T*)s.gmv; a.gv0 = (T*)s.gv0; a.gf = (T*)s.gf; a.gv = (T*)s.gv; a.gvf = (T*)s.gvf;
    a.dt = (T)dt;
    a.flags = h->d_flags;
    a.mark_left = h->plastic.kind != MPM_PLASTICITY_NONE;
    a.reflect = h->reflect.enabled;
    for(int k = 0; k < 6; k++) a.side[k] = h->reflect.enabled ? h->reflect.side_type[k] : MPM_BC_FREE;
    a.pmodel = s.pmodel;
    a.pmask = s.pmask;
    a.motion = h->motion_dev;
    a.moving = h->motion_dev ? h->moving : 0u;
    return a;
}

}  // namespace plain
