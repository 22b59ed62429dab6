// Handle layout and internal interfaces of libphysbam_mpm.so (not public).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "mpm_math.cuh"
#include "mpm_types.h"

// Everything a kernel needs about the scene, passed by value.
struct SceneParams {
    int dim;
    int counts[3];
    double dmin[3], dmax[3], dx[3], inv_dx[3];
    int model;
    double gravity[3];
    int nobj;
    mpm::DevObject objs[MPM_MAX_OBJECTS];
    int npen;                                   // penalty collision objects (plain path)
    double pen_stiffness, pen_separation;
    mpm::DevObject pen[MPM_MAX_OBJECTS];
};

// Reference-layout device arrays for the plain path (one thread per particle).
struct PlainState {
    int64_t n = 0, gn = 0;
    void *X = nullptr, *V = nullptr, *F = nullptr, *B = nullptr;
    void *mass = nullptr, *vol = nullptr, *mu = nullptr, *lam = nullptr, *pft = nullptr;
    uint8_t* valid = nullptr;
    void *gm = nullptr, *gmv = nullptr, *gv0 = nullptr, *gf = nullptr, *gv = nullptr, *gvf = nullptr;
    void *Fp = nullptr, *mu0 = nullptr, *lam0 = nullptr;   // plastic state (plasticity on): clamp
    void *pdef = nullptr, *rhoF = nullptr, *sigY = nullptr, *vc = nullptr;   // Drucker-Prager
    uint8_t* pmodel = nullptr;   // per-particle constitutive model (null: the handle's model)
    uint8_t* pmask = nullptr;    // particles the plasticity acts on (null: all)
};

// One scene of a batch, as the fast-path kernels see it.
struct SceneDev {
    float dmin[3], dmax[3], dx[3], inv[3], gravity[3];
    int counts[3];
    int NB[3];              // particle blocks (4^3 cells) per axis
    int NN[3];              // node blocks (4^3 nodes) per axis
    int GA[3];              // grid node extent per axis (4 NN >= G + 6)
    uint32_t block_base;    // first global particle-block id of the scene
    uint32_t nb_base;       // first global node-block id of the scene
    int64_t node_base;      // first node of the scene's grid in the pooled grid
    int model;
    int obj_begin, nobj;    // collision objects [obj_begin, obj_begin + nobj)
    int pad;
};

// Fast path: cell-sorted SoA particles (double-buffered), block-sparse grids of
// one or more scenes.
struct FastState {
    int64_t n = 0, npad = 0;
    int key_bits = 0;
    int cur = 0;
    bool batch = false;                       // created by mpm_batch_create
    int nscenes = 0;
    std::vector<SceneDev> scenes_h;
    std::vector<int64_t> pbase_h;             // particle offset of each scene, nscenes + 1
    std::vector<mpm::DevObject> objs_h;
    int64_t total_blocks = 0, total_nblocks = 0, total_nodes = 0;
    SceneDev* scenes = nullptr;
    uint16_t* block_scene = nullptr;          // global particle block -> scene
    uint16_t* nb_scene = nullptr;             // global node block -> scene
    int64_t* pbase = nullptr;
    mpm::DevObject* objs = nullptr;
    float* soa[2] = {nullptr, nullptr};       // 24 * npad floats: x y z, vx vy vz, F0..8, B0..8
    float4* attr[2] = {nullptr, nullptr};     // mass, volume, mu, lambda
    int* pid[2] = {nullptr, nullptr};         // caller's particle index
    float* plas[2] = {nullptr, nullptr};      // plasticity on: 13 * npad floats: Fp0..8, then mu0, lambda0
                                              // (clamp) or plastic_def, rho_F, sigma_Y, vc (Drucker-Prager)
    uint32_t* keys[2] = {nullptr, nullptr};   // cell keys of each buffer's slots
    uint8_t* dirs[2] = {nullptr, nullptr};    // each slot's move direction from its previous block (G2P)
    uint32_t* sorted_keys = nullptr;
    uint32_t* perm = nullptr;                 // sorted position -> slot in the current buffer
    uint32_t* sort_keys_alt = nullptr;
    uint32_t* sort_vals_alt = nullptr;
    uint32_t* sort_scratch = nullptr;         // histograms, tickets, epoch, look-back status words
    // the particle blocks of a substep's sorted order, one set per buffer parity
    // (the next substep's routing reads the previous set)
    uint32_t* bstart[2] = {nullptr, nullptr}; // per particle block
    uint32_t* bend[2] = {nullptr, nullptr};
    uint4* active[2] = {nullptr, nullptr};    // active particle blocks: (block, start, count, scene)
    uint4* chunks[2] = {nullptr, nullptr};    // work items, two uint4 each: (block, part, parts, scene), (block start, block count, 0, 0)
    int64_t chunk_cap = 0;
    // routing from one substep's order to the next (mpm_fast.cu, k_bins / k_route):
    // per block a row of arrival counts by direction (G2P) and the row of their
    // sorted offsets, per block its arrivals and departures out of the domain,
    // look-back status of the block scan
    uint32_t* dcount = nullptr;               // total_blocks x 32
    uint32_t* doff = nullptr;                 // total_blocks x 32
    unsigned long long* bcount = nullptr;     // total_blocks: arrivals (low word), invalidated (high word)
    uint32_t* scan = nullptr;                 // epoch word, then the look-back status words (two chains)
    void* tmaps = nullptr;                    // per scene: CUtensorMap of its node grid (G2P tiles by TMA)
    bool order_ready = false;                 // the previous set + dcount describe the current slots
    bool sorted_now = false;                  // this substep's order is built (P2G may repeat)
    uint32_t* nb_flag = nullptr;              // node-block touched this substep
    uint32_t* nb_list = nullptr;              // touched node blocks
    uint32_t* counters = nullptr;             // 2 x 16 words, one set per parity: see FastCounter
    int grid_set = 0;                         // counter set of the last grid update (its node blocks)
    float4* acc = nullptr;                    // P2G accumulator: momentum+dt*force (xyz), mass (w)
    float4* vel = nullptr;                    // per node 2 x float4: vnew.xyz, vfric.x | vfric.yz, mass, 0
    float* vkick = nullptr;                   // penalty objects on: 3 * npad floats, V + dt f / m per slot
    uint8_t* pmodel = nullptr;                // constitutive model per caller particle index (null: the scene's)
    uint8_t* pmask = nullptr;                 // plasticity on per caller particle index (null: all)
    bool keys_ready = false;
    uint64_t generation = 0;   // bumped whenever device buffers are (re)allocated
    int64_t grid_nodes = 0;
    uint32_t grid_node_blocks = 0;
    bool grid_dirty = false;   // the accumulator holds a P2G that no grid update consumed
    void* staging = nullptr;   // device copies of host particle arrays (set / get)
    size_t staging_bytes = 0;   // size of `staging`
    // launch shapes (mpm_autotune)
    int p2g_variant = MPM_P2G_FIXED256;       // P2G launch shape (MPM_P2G_*)
    int route_variant = MPM_P2G_FIXED256;     // the shape whose work-item size the current order has
    int g2p_threads = 128;
    int cta_mult = 1;
};

// One set of per-substep counters (two sets, one per buffer parity).
enum FastCounter {
    CNT_ACTIVE_BLOCKS = 0,
    CNT_ACTIVE_PARTICLES = 1,      // valid particles of the substep's order
    CNT_P2G_WORK = 2,
    CNT_G2P_WORK = 3,
    CNT_NODE_BLOCKS = 4,
    CNT_GRID_WORK = 5,
    CNT_FALLBACK = 6,
    CNT_P2G_DONE = 7,
    CNT_CHUNKS = 8,                // work items in the set's chunk list
    CNT_NEW_INVALID = 9,           // particles the last G2P invalidated
    CNT_SPARE = 10,                // (unused)
    CNT_FAR = 11,                  // particles that moved past a neighbour block
    CNT_COUNT = 16
};

struct ImplicitState;   // mpm_implicit.cu

struct KernelTimer {
    std::string name;
    double ms = 0;
    int64_t launches = 0;
};

struct PendingEvent {
    int timer;
    cudaEvent_t start, stop;
};

struct mpm_handle {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    mpm_grid_desc grid{};
    mpm_model_desc model{};
    SceneParams sp{};
    mpm::DevObjectF* pen_f = nullptr;   // penalty objects rounded to float (fast path), MPM_MAX_OBJECTS
    int64_t n = 0;
    bool have_particles = false;
    unsigned* d_flags = nullptr;
    PlainState plain;
    FastState fast;
    mpm_plasticity_desc plastic{};   // kind MPM_PLASTICITY_NONE: off
    mpm_implicit_desc implicit{};    // enabled 0: symplectic Euler
    mpm_dt_control dt_control{};     // Compute_Dt / Reduce_Dt controls
    mpm_reflection_desc reflect{};   // reflection boundary conditions (enabled 0: none)
    double last_dt = 0;              // step the last substep took (Reduce_Dt may shorten it)
    // moving collision objects: host callbacks, and their frames for the current substep
    mpm_motion_fn motion_fn[MPM_MAX_OBJECTS] = {};
    void* motion_user[MPM_MAX_OBJECTS] = {};
    unsigned moving = 0;                      // bit j: object j moves
    mpm::ObjMotion* motion_dev = nullptr;     // MPM_MAX_OBJECTS, plain path and implicit solve
    mpm::ObjMotionF* motion_dev_f = nullptr;  // the same in float, fast path
    // mpm_advance over moving objects: the frames of every substep, filled before the
    // graph replays; each replay's first kernel copies the next slot into motion_dev
    mpm::ObjMotion* motion_table = nullptr;
    mpm::ObjMotionF* motion_table_f = nullptr;
    unsigned* motion_slot = nullptr;          // device counter of the slot to take next
    int motion_cap = 0;                       // substeps the tables hold
    bool motion_from_table = false;
    mpm_implicit_stats imp_stats{};  // of the last implicit solve
    ImplicitState* imp = nullptr;
    // timing
    bool timing = false;
    std::vector<KernelTimer> timers;
    std::vector<PendingEvent> pending;
    std::vector<cudaEvent_t> event_pool;
    // one captured substep per particle-buffer parity (the fast path swaps buffers)
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};   // one captured substep per buffer parity
    double graph_dt = 0;
    // checkpoints of the last mpm_diff_forward (mpm_adjoint.cu)
    void* diff = nullptr;
    int64_t diff_budget = -1;                 // mpm_set_diff_tape_budget
    std::string last_error;
};

// frames and twists of the moving objects for the substep [time, time + dt] (mpm_capi.cu)
int update_motion(mpm_handle* h, double time, double dt);

// timing helpers (mpm_capi.cu)
int timer_begin(mpm_handle* h, const char* name);
void timer_end(mpm_handle* h, int slot);

// plain path (mpm_plain.cu)
int plain_alloc(mpm_handle* h, int64_t n);
void plain_free(mpm_handle* h);
int plain_set_particles(mpm_handle* h, const mpm_particles_view* v);
int plain_get_particles(mpm_handle* h, mpm_particles_view* v);
int plain_p2g(mpm_handle* h, double dt, double time);
int plain_forces(mpm_handle* h, double dt, double time);
int plain_g2p(mpm_handle* h, double dt, double time);
int plain_get_grid(mpm_handle* h, double* m, double* v0, double* v, double* vf);
int plain_count_valid(mpm_handle* h, int64_t* c);
int plain_add_forces(mpm_handle* h, const void* f, int dtype, bool on_device);
int fast_add_forces(mpm_handle* h, double dt, const void* f, int dtype, bool on_device);

// fast path (mpm_fast.cu)
int fast_alloc(mpm_handle* h, int64_t n);
void fast_free(mpm_handle* h);
int fast_penalty_buffers(mpm_handle* h);
int fast_set_particles(mpm_handle* h, const mpm_particles_view* v);
int fast_get_particles(mpm_handle* h, mpm_particles_view* v);
int fast_p2g(mpm_handle* h, double dt, double time);
int fast_forces(mpm_handle* h, double dt, double time);
int fast_g2p(mpm_handle* h, double dt, double time);
int fast_get_grid(mpm_handle* h, int scene, double* m, double* v0, double* v, double* vf);
// Each compiled module's copy of the SVD sweep bound (mpm_math.cuh, g_svd_max_it).
cudaError_t svd_limit_plain(int v);
cudaError_t svd_limit_adjoint(int v);
cudaError_t svd_limit_implicit(int v);
cudaError_t svd_limit_fast(int v);
cudaError_t svd_limit_capi(int v);
int debug_sort_stall(const uint32_t* keys, int64_t n, int bits, uint32_t spin_limit);
int debug_set_sort_epoch(mpm_handle* h, uint32_t epoch);
int fast_count_valid(mpm_handle* h, int64_t* c);
int fast_debug_sort_state(mpm_handle* h, uint32_t* slot_keys, uint32_t* sorted_keys, uint32_t* perm);
int fast_setup_scenes(mpm_handle* h, const mpm_scene_desc* descs, int count, const mpm_collision_object* objs, int nobjs);
int fast_autotune(mpm_handle* h, double dt, int substeps, int flags, char* report, int report_len);
int radix_sort_host(const uint32_t* keys, int64_t n, int bits, uint32_t* sorted_keys, uint32_t* perm);
int64_t sort_scratch_words(int64_t n);
int sort_keys_device(mpm_handle* h, const uint32_t* keys, int64_t n, int bits, uint32_t* sorted, uint32_t* perm,
    uint32_t* alt_keys, uint32_t* alt_vals, uint32_t* scratch);
int fast_prepare(mpm_handle* h);
int fast_particle_totals(mpm_handle* h, mpm_totals* out);
int fast_grid_totals(mpm_handle* h, mpm_totals* out);
int plain_particle_totals(mpm_handle* h, mpm_totals* out);
int plain_plastic_init(mpm_handle* h);
int fast_plastic_init(mpm_handle* h);
int fast_get_plastic(mpm_handle* h, mpm_plastic_view* v);
int fast_set_plastic(mpm_handle* h, const mpm_plastic_view* v);
int plain_get_plastic(mpm_handle* h, mpm_plastic_view* v);
int plain_set_plastic(mpm_handle* h, const mpm_plastic_view* v);
int plain_grid_totals(mpm_handle* h, mpm_totals* out);

// implicit solve (mpm_implicit.cu)
int plain_implicit_forces(mpm_handle* h, double dt, double time);
int implicit_max_sound_speed(mpm_handle* h, double* partial, double* out);
int plain_reduce_dt(mpm_handle* h, double dt, double* dt_out);
int plain_reflect_velocity(mpm_handle* h);
void implicit_free(mpm_handle* h);

// adjoint (mpm_adjoint.cu)
int diff_forward(mpm_handle* h, double dt, int nsteps, int every);
int diff_backward(mpm_handle* h, const mpm_particles_view* gout, mpm_particles_view* gin, void* gmu, void* glam);
void diff_free(mpm_handle* h);
void diff_invalidate(mpm_handle* h);

// helpers
int set_error(mpm_handle* h, int code, const std::string& msg);
int check_cuda(mpm_handle* h, cudaError_t e, const char* what);
#define MPM_CUDA(h, call)                                   \
    do {                                                    \
        cudaError_t e__ = (call);                           \
        if(e__ != cudaSuccess) return check_cuda(h, e__, #call); \
    } while(0)
#define MPM_LAUNCHED(h, what)                               \
    do {                                                    \
        cudaError_t e__ = cudaGetLastError();               \
        if(e__ != cudaSuccess) return check_cuda(h, e__, what); \
    } while(0)
