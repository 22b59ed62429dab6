// The reference-side binding, compiled and run: a scene file of
// physbam_b200/scenes.py is read into the reference's own MPM_EXAMPLE
// (oracle/ref_scene.h, as STANDARD_TESTS_BASE sets scenes up), then its
// substeps run on the GPU through include/mpm_physbam.hpp (B200_SUBSTEP<TV>,
// the adapter a PhysBAM maintainer adds) instead of MPM_DRIVER's CPU loop, and
// the particles downloaded back into MPM_PARTICLES are dumped.  Test
// infrastructure: tests/test_gpu_integration.py runs it.  Built by
// oracle/ref.mk against the reference's sources and libphysbam_mpm.so.
//
//   ref_b200 <scene.bin> <dump.bin> [-float] [-substeps]
//
// -float: TV = VECTOR<float,3> (the FP32 fast path reads float arrays), else
// double arrays handed to the same path.  -substeps: one mpm_substep call per
// substep instead of one mpm_advance over all of them.
// Dump: int32 n, then X (n x 3), V (n x 3), F (n x 9, column-major), B (n x 9)
// as doubles, then valid (n bytes); a JSON line with the GPU loop's seconds on stdout.
#include "ref_scene.h"
#include "mpm_physbam.hpp"

namespace {

template<class TV> int Run(const SCENE_FILE& s, const char* dump_path, bool per_substep)
{
    typedef typename TV::SCALAR T;
    FILE_SCENE<TV> example(s, 1);
    char tmpl[] = "/tmp/ref_b200_XXXXXX";
    example.viewer_dir.output_directory = mkdtemp(tmpl);
    MPM_DRIVER<TV> driver(example);
    driver.Initialize();             // grid, particles, forces and objects of the scene

    B200_SUBSTEP<TV> gpu;
    TV g;
    for(int a = 0; a < TV::m; a++) g(a) = (T)s.gravity[a];
    gpu.Initialize(example, s.model, g);
    std::vector<mpm_collision_object> objs;
    for(const OBJ& o: s.objs) {
        if(o.moving) throw std::runtime_error("the runner hands static objects only");
        mpm_collision_object c = {};
        c.kind = o.kind;
        c.type = o.type;
        c.friction = o.friction;
        for(int k = 0; k < 3; k++) { c.a[k] = o.a[k]; c.b[k] = o.b[k]; }
        objs.push_back(c);
    }
    gpu.Set_Collision_Objects(objs);
    auto t0 = std::chrono::steady_clock::now();
    if(per_substep)
        for(int k = 0; k < s.nsteps; k++) gpu.Advance_One_Time_Step((T)s.dt, (T)(s.t0 + k * s.dt));
    else gpu.Advance((T)s.dt, (T)s.t0, s.nsteps);
    gpu.Synchronize();
    auto t1 = std::chrono::steady_clock::now();
    gpu.Download(example.particles);

    FILE* f = fopen(dump_path, "wb");
    if(!f) throw std::runtime_error("cannot open dump");
    const MPM_PARTICLES<TV>& p = example.particles;
    const int n = p.number;
    fwrite(&n, sizeof n, 1, f);
    std::vector<double> buf;
    auto put = [&](int comps, auto get) {
        buf.resize((size_t)n * comps);
        for(int i = 0; i < n; i++) for(int c = 0; c < comps; c++) buf[(size_t)i * comps + c] = (double)get(i, c);
        fwrite(buf.data(), sizeof(double), buf.size(), f);
    };
    put(3, [&](int i, int c) { return p.X(i)(c); });
    put(3, [&](int i, int c) { return p.V(i)(c); });
    put(9, [&](int i, int c) { return p.F(i).x[c]; });
    put(9, [&](int i, int c) { return p.B(i).x[c]; });
    std::vector<unsigned char> valid(n);
    for(int i = 0; i < n; i++) valid[i] = p.valid(i) ? 1 : 0;
    fwrite(valid.data(), 1, n, f);
    fclose(f);
    printf("{\"gpu_seconds\": %.6f, \"substeps\": %d, \"particles\": %d}\n",
           std::chrono::duration<double>(t1 - t0).count(), s.nsteps, n);
    return 0;
}

}  // namespace

int main(int argc, char* argv[])
{
    if(argc < 3) { fprintf(stderr, "usage: ref_b200 scene.bin dump.bin [-float] [-substeps]\n"); return 2; }
    bool use_float = false, per_substep = false;
    for(int i = 3; i < argc; i++) {
        if(!strcmp(argv[i], "-float")) use_float = true;
        else if(!strcmp(argv[i], "-substeps")) per_substep = true;
    }
    LOG::Initialize_Logging(true, true, 0, false);
    SCENE_FILE s = Read_Scene(argv[1]);
    if(s.dim != 3) { fprintf(stderr, "ref_b200: 3D scenes only\n"); return 2; }
    int rc = 1;
    try {
        rc = use_float ? Run<VECTOR<float, 3> >(s, argv[2], per_substep) : Run<VECTOR<double, 3> >(s, argv[2], per_substep);
    } catch(const std::exception& e) {
        fprintf(stderr, "ref_b200: %s\n", e.what());
        rc = 1;
    }
    LOG::Finish_Logging();
    return rc;
}
