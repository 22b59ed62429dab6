// C++ binding of libphysbam_mpm.so for PhysBAM code: the adapter a PhysBAM
// maintainer adds next to Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.h
// (whose public step functions, MPM_DRIVER.h:41-78, it stands in for) to run
// the explicit substep of an MPM_EXAMPLE on the GPU.  Header only; include it
// after the PhysBAM headers it uses and link libphysbam_mpm.so.
//
// The particle arrays of MPM_PARTICLES are handed to the C ABI in their own
// layout (ARRAY_VIEW<TV> AoS, MATRIX column-major, ARRAY_VIEW<bool> one byte
// each); the library keeps its own device copy between Upload and Download.
// PhysBAM errors are exceptions (PHYSBAM_FATAL_ERROR, Core/Log/
// DEBUG_UTILITIES.cpp:95-103); a non-zero status of the C ABI becomes one,
// with the library's message.
#pragma once

#include <Core/Log/DEBUG_UTILITIES.h>
#include <Core/Vectors/VECTOR.h>
#include <Hybrid_Methods/Examples_And_Drivers/MPM_EXAMPLE.h>
#include <Hybrid_Methods/Examples_And_Drivers/MPM_PARTICLES.h>

#include <string>
#include <vector>

#include "mpm_capi.h"

namespace PhysBAM {

template<class TV> struct B200_SUBSTEP
{
    typedef typename TV::SCALAR T;
    mpm_handle* h = nullptr;

    B200_SUBSTEP() = default;
    B200_SUBSTEP(const B200_SUBSTEP&) = delete;
    B200_SUBSTEP& operator=(const B200_SUBSTEP&) = delete;
    ~B200_SUBSTEP() { if(h) mpm_destroy(h); }

    void Check(int rc, const char* what) const
    {
        if(!rc) return;
        char msg[256] = "";
        if(h) mpm_last_error(h, msg, sizeof msg);
        PHYSBAM_FATAL_ERROR(std::string(what) + ": " + mpm_status_string(rc) + (msg[0] ? std::string(" (") + msg + ")" : ""));
    }

    // The example's grid (MPM_EXAMPLE::grid, ghost layers ex.ghost) and one
    // constitutive model for every particle (mpm_model: MPM_COROTATED_FIXED,
    // MPM_NEO_HOOKEAN, MPM_STVK_HENCKY), gravity, the fast FP32 path (3D) or
    // the plain path in T's precision; the example's particles are uploaded.
    void Initialize(MPM_EXAMPLE<TV>& ex, int model, const TV& gravity, bool fast = TV::m == 3)
    {
        mpm_grid_desc g = {};
        g.dim = TV::m;
        g.ghost = ex.ghost;
        for(int a = 0; a < TV::m; a++) {
            g.counts[a] = ex.grid.counts(a);
            g.domain_min[a] = ex.grid.domain.min_corner(a);
            g.domain_max[a] = ex.grid.domain.max_corner(a);
        }
        mpm_model_desc m = {};
        m.model = model;
        m.precision = fast || sizeof(T) == 4 ? MPM_FP32 : MPM_FP64;
        m.path = fast ? MPM_PATH_FAST : MPM_PATH_PLAIN;
        for(int a = 0; a < TV::m; a++) m.gravity[a] = gravity(a);
        Check(mpm_create(&g, &m, &h), "mpm_create");
        Upload(ex.particles);
    }

    // Collision objects as MPM_EXAMPLE::Add_Collision_Object receives them:
    // RANGE boxes (a = min corner, b = max corner), PLANEs (a = normal, b = a
    // point) and SPHEREs (a = centre, b[0] = radius), stick / slip / separate,
    // Coulomb friction.
    void Set_Collision_Objects(const std::vector<mpm_collision_object>& objects)
    {
        Check(mpm_set_collision_objects(h, objects.data(), (int)objects.size()), "mpm_set_collision_objects");
    }

    mpm_particles_view View(MPM_PARTICLES<TV>& p)
    {
        mpm_particles_view v = {};
        v.n = p.number;
        v.dtype = sizeof(T) == 8 ? MPM_FP64 : MPM_FP32;
        v.X = p.X.Get_Array_Pointer();
        v.V = p.V.Get_Array_Pointer();
        v.F = p.F.Get_Array_Pointer();
        v.B = p.B.Get_Array_Pointer();
        v.mass = p.mass.Get_Array_Pointer();
        v.volume = p.volume.Get_Array_Pointer();
        v.mu = p.mu.Get_Array_Pointer();
        v.lambda = p.lambda.Get_Array_Pointer();
        v.valid = (uint8_t*)p.valid.Get_Array_Pointer();
        return v;
    }

    void Upload(MPM_PARTICLES<TV>& p) { mpm_particles_view v = View(p); Check(mpm_set_particles(h, &v), "mpm_set_particles"); }
    void Download(MPM_PARTICLES<TV>& p) { mpm_particles_view v = View(p); Check(mpm_get_particles(h, &v), "mpm_get_particles"); }

    // MPM_DRIVER::Advance_One_Time_Step for the explicit (symplectic Euler) path.
    void Advance_One_Time_Step(T dt, T time) { Check(mpm_substep(h, dt, time), "mpm_substep"); }
    // n fixed-dt substeps (Simulate_To_Frame with min_dt = max_dt), replayed from a CUDA graph.
    void Advance(T dt, T time, int n) { Check(mpm_advance(h, dt, time, n), "mpm_advance"); }
    // Waits for the queued substeps; device-side errors (NaN, a stencil off the grid) surface here.
    void Synchronize() { Check(mpm_synchronize(h), "mpm_synchronize"); }
    // MPM_DRIVER::Compute_Dt with the affine CFL bound (use_affine_cfl), clamped below by min_dt.
    T Compute_Dt(const MPM_EXAMPLE<TV>& ex)
    {
        double dt = 0;
        Check(mpm_compute_dt(h, ex.cfl, ex.max_dt, &dt), "mpm_compute_dt");
        return std::max((T)dt, ex.min_dt);
    }
    // The -print_stats diagnostics (Total_Particle_Linear_Momentum etc.), FP64 on the GPU.
    mpm_totals Particle_Stats()
    {
        mpm_totals t;
        Check(mpm_particle_totals(h, &t), "mpm_particle_totals");
        return t;
    }
};

}  // namespace PhysBAM
