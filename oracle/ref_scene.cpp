// Reference runner: drives the reference's own MPM_DRIVER / MPM_EXAMPLE on a
// scene file written by physbam_b200/scenes.py, and dumps particle and grid
// state after chosen substeps.  Test infrastructure only (it pins the CPU
// restatement in oracle/ and produces the golden fixtures); the product never
// links or runs it.  Built by oracle/ref.mk against the reference's sources.
//
//   ref_scene <scene.bin> <dump.bin> [-threads T] [-float] [-time] [-totals CFL MAX_DT] [-output DIR]
//             [-restart DIR FRAME]
//
// The scene set-up (oracle/ref_scene.h) follows Projects/mpm/STANDARD_TESTS_BASE.cpp.
#include "ref_scene.h"

namespace {
template<class T> void wr(FILE* f, const T* p, size_t n) { fwrite(p, sizeof(T), n, f); }

struct TOTALS_REQUEST { bool on = false; double cfl = 1, max_dt = 1; };

std::string keep_output;   // -output DIR: the viewer directory the driver writes (kept)
int restart_frame = 0;     // -restart DIR FRAME: start from that frame of DIR (Read_Output_Files)

template<class TV> int Run(const SCENE_FILE& s, const char* dump_path, int threads, bool report_time,
    const TOTALS_REQUEST& totals)
{
    typedef typename TV::SCALAR T;
    typedef VECTOR<int, TV::m> TV_INT;
    const int d = TV::m;
    FILE_SCENE<TV> example(s, threads);
    char tmpl[] = "/tmp/ref_scene_XXXXXX";
    std::string outdir = keep_output.empty() ? std::string(mkdtemp(tmpl)) : keep_output;
    example.viewer_dir.output_directory = outdir;
    if(restart_frame) example.restart = restart_frame;
    MPM_DRIVER<TV> driver(example);
    driver.Initialize();

    std::vector<double> gm, gv0, gv, gvf;
    int current = -1;
    auto want = [&](int step){for(int x: s.dumps) if(x == step) return true; return false;};
    auto grab = [&](const ARRAY<TV, TV_INT>& u, std::vector<double>& out)
    {
        out.resize((size_t)u.array.m * d);
        for(int i = 0; i < u.array.m; i++) for(int a = 0; a < d; a++) out[(size_t)i * d + a] = u.array(i)(a);
    };
    example.Add_Callbacks(false, "p2g", [&]()
    {
        if(!want(current)) return;
        gm.resize(example.mass.array.m);
        for(int i = 0; i < example.mass.array.m; i++) gm[i] = example.mass.array(i);
        grab(example.velocity, gv0);
    });
    example.Add_Callbacks(false, "forces", [&]()
    {
        if(!want(current)) return;
        grab(example.velocity, gv);
        grab(example.velocity_friction_save, gvf);
    });

    FILE* f = fopen(dump_path, "wb");
    if(!f) { fprintf(stderr, "cannot open dump\n"); return 1; }
    double total = 0;
    std::vector<double> step_seconds;
    int substeps = 0;
    example.Add_Callbacks(false, "time-step", [&]() { substeps++; });
    std::vector<int> frame_substeps;
    for(int step = 0; step < s.nsteps; step++) {
        current = step;
        auto t0 = std::chrono::steady_clock::now();
        if(s.dt_control) {   // one frame: `step` counts frames
            const int before = substeps;
            driver.Simulate_To_Frame(step + 1);
            frame_substeps.push_back(substeps - before);
        } else {
            example.dt = (T)s.dt;
            driver.Advance_One_Time_Step();
        }
        auto t1 = std::chrono::steady_clock::now();
        step_seconds.push_back(std::chrono::duration<double>(t1 - t0).count());
        total += step_seconds.back();
        if(!s.dt_control) example.time += example.dt;
        if(!want(step)) continue;
        wr(f, &step, 1);
        std::vector<double> buf;
        size_t n = s.n;
        buf.resize(n * d);
        for(size_t p = 0; p < n; p++) for(int a = 0; a < d; a++) buf[p * d + a] = example.particles.X(p)(a);
        wr(f, buf.data(), buf.size());
        for(size_t p = 0; p < n; p++) for(int a = 0; a < d; a++) buf[p * d + a] = example.particles.V(p)(a);
        wr(f, buf.data(), buf.size());
        buf.resize(n * d * d);
        for(size_t p = 0; p < n; p++) for(int k = 0; k < d * d; k++) buf[p * d * d + k] = example.particles.F(p).x[k];
        wr(f, buf.data(), buf.size());
        for(size_t p = 0; p < n; p++) for(int k = 0; k < d * d; k++) buf[p * d * d + k] = example.particles.B(p).x[k];
        wr(f, buf.data(), buf.size());
        std::vector<unsigned char> valid(n);
        for(size_t p = 0; p < n; p++) valid[p] = example.particles.valid(p) ? 1 : 0;
        wr(f, valid.data(), n);
        wr(f, gm.data(), gm.size());
        wr(f, gv0.data(), gv0.size());
        wr(f, gv.data(), gv.size());
        wr(f, gvf.data(), gvf.size());
        if(s.plasticity) {
            buf.resize(n * d * d);
            for(size_t p = 0; p < n; p++) for(int k = 0; k < d * d; k++) buf[p * d * d + k] = example.particles.Fp(p).x[k];
            wr(f, buf.data(), buf.size());
            buf.resize(n);
            auto put = [&](auto get){for(size_t p = 0; p < n; p++) buf[p] = get(p); wr(f, buf.data(), n);};
            if(s.plasticity == 1) {
                put([&](size_t p){return (double)example.particles.mu(p);});
                put([&](size_t p){return (double)example.particles.lambda(p);});
            } else {
                const MPM_DRUCKER_PRAGER<TV>& dp = *example.dp;
                put([&](size_t p){return (double)dp.plastic_def(p);});
                put([&](size_t p){return (double)dp.rho_F(p);});
                put([&](size_t p){return (double)dp.sigma_Y(p);});
                put([&](size_t p){return (double)dp.vc(p);});
            }
        }
    }
    fclose(f);
    if(totals.on) {
        // the reference's own diagnostics on the final particle state
        auto lin = example.Total_Particle_Linear_Momentum();
        auto ang = example.Total_Particle_Angular_Momentum();
        double mass = 0;
        for(int k = 0; k < example.simulated_particles.m; k++) mass += example.particles.mass(example.simulated_particles(k));
        example.cfl = (T)totals.cfl;
        example.max_dt = (T)totals.max_dt;
        printf("{\"mass\": %.17g, \"count\": %d, \"momentum\": [", mass, example.simulated_particles.m);
        for(int a = 0; a < d; a++) printf("%s%.17g", a ? ", " : "", (double)lin(a));
        printf("], \"angular_momentum\": [");
        for(int a = 0; a < ang.m; a++) printf("%s%.17g", a ? ", " : "", (double)ang(a));
        printf("], \"kinetic_energy\": %.17g, \"max_speed\": %.17g, \"max_affine_speed\": %.17g, \"dt\": %.17g}\n",
            (double)example.Total_Particle_Kinetic_Energy(), (double)driver.Max_Particle_Speed(),
            (double)driver.Grid_V_Upper_Bound(), (double)driver.Compute_Dt());
    }
    if(s.dt_control) {
        printf("{\"frame_substeps\": [");
        for(size_t i = 0; i < frame_substeps.size(); i++) printf("%s%d", i ? ", " : "", frame_substeps[i]);
        printf("], \"time\": %.17g}\n", (double)example.time);
    }
    if(report_time) {
        printf("{\"substeps\": %d, \"particles\": %lld, \"seconds\": %.9g, \"threads\": %d, \"step_seconds\": [",
            s.nsteps, s.n, total, threads);
        for(size_t i = 0; i < step_seconds.size(); i++) printf("%s%.9g", i ? ", " : "", step_seconds[i]);
        printf("]}\n");
    }
    if(keep_output.empty()) {
        std::string cmd = "rm -rf '" + outdir + "'";
        if(system(cmd.c_str())) {}
    }
    return 0;
}
}

int main(int argc, char* argv[])
{
    if(argc < 3) { fprintf(stderr, "usage: ref_scene scene.bin dump.bin [-threads T] [-float] [-time] [-totals CFL MAX_DT]\n"); return 2; }
    int threads = 1;
    bool use_float = false, report_time = false;
    TOTALS_REQUEST totals;
    for(int i = 3; i < argc; i++) {
        if(!strcmp(argv[i], "-threads") && i + 1 < argc) threads = atoi(argv[++i]);
        else if(!strcmp(argv[i], "-float")) use_float = true;
        else if(!strcmp(argv[i], "-time")) report_time = true;
        else if(!strcmp(argv[i], "-output") && i + 1 < argc) keep_output = argv[++i];
        else if(!strcmp(argv[i], "-restart") && i + 2 < argc) { keep_output = argv[++i]; restart_frame = atoi(argv[++i]); }
        else if(!strcmp(argv[i], "-totals") && i + 2 < argc) {
            totals.on = true;
            totals.cfl = atof(argv[++i]);
            totals.max_dt = atof(argv[++i]);
        }
    }
#ifdef USE_OPENMP
    omp_set_num_threads(threads);
#endif
    LOG::Initialize_Logging(true, true, 0, false);
    SCENE_FILE s = Read_Scene(argv[1]);
    int rc;
    if(use_float) rc = s.dim == 2 ? Run<VECTOR<float, 2> >(s, argv[2], threads, report_time, totals) : Run<VECTOR<float, 3> >(s, argv[2], threads, report_time, totals);
    else rc = s.dim == 2 ? Run<VECTOR<double, 2> >(s, argv[2], threads, report_time, totals) : Run<VECTOR<double, 3> >(s, argv[2], threads, report_time, totals);
    LOG::Finish_Logging();
    return rc;
}
