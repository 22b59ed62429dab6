// C ABI entry points (include/mpm_capi.h).  No exception crosses this file's
// boundary; every entry point returns an mpm_status.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "mpm_internal.h"

int set_error(mpm_handle* h, int code, const std::string& msg)
{
    if(h) h->last_error = msg;
    return code;
}

int check_cuda(mpm_handle* h, cudaError_t e, const char* what)
{
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if(e == cudaErrorMemoryAllocation) return set_error(h, MPM_ERR_NOMEM, msg);
    return set_error(h, MPM_ERR_CUDA, msg);
}

int timer_begin(mpm_handle* h, const char* name)
{
    if(!h->timing) return -1;
    int slot = -1;
    for(size_t i = 0; i < h->timers.size(); i++)
        if(h->timers[i].name == name) slot = (int)i;
    if(slot < 0) {
        KernelTimer t;
        t.name = name;
        h->timers.push_back(t);
        slot = (int)h->timers.size() - 1;
    }
    PendingEvent p;
    p.timer = slot;
    for(int k = 0; k < 2; k++) {
        cudaEvent_t ev;
        if(!h->event_pool.empty()) { ev = h->event_pool.back(); h->event_pool.pop_back(); }
        else cudaEventCreate(&ev);
        (k ? p.stop : p.start) = ev;
    }
    cudaEventRecord(p.start, h->stream);
    h->pending.push_back(p);
    return (int)h->pending.size() - 1;
}

void timer_end(mpm_handle* h, int slot)
{
    if(slot < 0 || !h->timing) return;
    cudaEventRecord(h->pending[slot].stop, h->stream);
}

static void drain_timers(mpm_handle* h)
{
    for(PendingEvent& p: h->pending) {
        float ms = 0;
        cudaEventSynchronize(p.stop);
        if(cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
            h->timers[p.timer].ms += ms;
            h->timers[p.timer].launches++;
        }
        h->event_pool.push_back(p.start);
        h->event_pool.push_back(p.stop);
    }
    h->pending.clear();
}

static bool fast(const mpm_handle* h) { return h->model.path == MPM_PATH_FAST; }

static int read_flags(mpm_handle* h)
{
    unsigned f = 0;
    MPM_CUDA(h, cudaMemcpyAsync(&f, h->d_flags, sizeof(f), cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    if(!f) return MPM_OK;
    MPM_CUDA(h, cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned), h->stream));
    if(f & MPM_FLAG_NAN) return set_error(h, MPM_ERR_NAN, "non-finite particle state");
    if(f & MPM_FLAG_DOMAIN) return set_error(h, MPM_ERR_DOMAIN, "particle stencil outside the ghosted grid");
    if(f & MPM_FLAG_TIMEOUT) return set_error(h, MPM_ERR_TIMEOUT, "device wait gave up");
    if(f & MPM_FLAG_NOT_CONVERGED) return set_error(h, MPM_ERR_NOT_CONVERGED, "SVD did not converge");
    if(f & MPM_FLAG_ORDER) return set_error(h, MPM_ERR_CUDA, "particle order out of step with its block counts");
    return MPM_OK;
}

static int release_graph(mpm_handle* h)
{
    for(cudaGraphExec_t& g: h->graphs) {
        if(g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    h->graph_dt = 0;
    return MPM_OK;
}

// ROTATION<TV>::Rotation_Matrix of a unit quaternion (w, x, y, z), or in 2D of
// the unit complex number (cos, sin), column-major d x d.
static void rotation_matrix(int d, const double* q, double* R)
{
    if(d == 2) {
        double m = std::sqrt(q[0] * q[0] + q[1] * q[1]);
        double c = m > 0 ? q[0] / m : 1, s = m > 0 ? q[1] / m : 0;
        R[0] = c; R[1] = s; R[2] = -s; R[3] = c;
        return;
    }
    double m = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    double w = 1, x = 0, y = 0, z = 0;
    if(m > 0) { w = q[0] / m; x = q[1] / m; y = q[2] / m; z = q[3] / m; }
    R[0] = 1 - 2 * (y * y + z * z); R[3] = 2 * (x * y - w * z);     R[6] = 2 * (x * z + w * y);
    R[1] = 2 * (x * y + w * z);     R[4] = 1 - 2 * (x * x + z * z); R[7] = 2 * (y * z - w * x);
    R[2] = 2 * (x * z - w * y);     R[5] = 2 * (y * z + w * x);     R[8] = 1 - 2 * (x * x + y * y);
}

// The frames of one substep from the objects' callbacks (double and float).
static int eval_motion(mpm_handle* h, double time, double dt, mpm::ObjMotion* m, mpm::ObjMotionF* mf)
{
    const int d = h->sp.dim;
    for(int j = 0; j < h->sp.nobj && j < MPM_MAX_OBJECTS; j++) {
        if(!((h->moving >> j) & 1u)) continue;
        mpm_object_state s0{}, s1{};
        if(h->motion_fn[j](h->motion_user[j], j, time, &s0) || h->motion_fn[j](h->motion_user[j], j, time + dt, &s1))
            return set_error(h, MPM_ERR_ARG, "an object motion callback failed");
        rotation_matrix(d, s0.rotation, m[j].R0);
        rotation_matrix(d, s1.rotation, m[j].R1);
        for(int k = 0; k < 3; k++) {
            m[j].x0[k] = s0.translation[k]; m[j].x1[k] = s1.translation[k];
            m[j].v[k] = s1.linear[k]; m[j].w[k] = s1.angular[k];
        }
        for(int k = 0; k < 9; k++) { mf[j].R0[k] = (float)m[j].R0[k]; mf[j].R1[k] = (float)m[j].R1[k]; }
        for(int k = 0; k < 3; k++) {
            mf[j].x0[k] = (float)m[j].x0[k]; mf[j].x1[k] = (float)m[j].x1[k];
            mf[j].v[k] = (float)m[j].v[k]; mf[j].w[k] = (float)m[j].w[k];
        }
    }
    return MPM_OK;
}

// Copy slot *slot of the tables into the substep's frames and step the slot.
__global__ void k_motion_pick(const mpm::ObjMotion* tab, const mpm::ObjMotionF* tabf, unsigned* slot, int cap,
    mpm::ObjMotion* out, mpm::ObjMotionF* outf)
{
    const unsigned s = *slot < (unsigned)cap ? *slot : (unsigned)cap - 1u;
    const int nd = (int)(sizeof(mpm::ObjMotion) * MPM_MAX_OBJECTS / sizeof(double));
    const int nf = (int)(sizeof(mpm::ObjMotionF) * MPM_MAX_OBJECTS / sizeof(float));
    const double* src = (const double*)(tab + (size_t)s * MPM_MAX_OBJECTS);
    const float* srcf = (const float*)(tabf + (size_t)s * MPM_MAX_OBJECTS);
    for(int k = threadIdx.x; k < nd; k += blockDim.x) ((double*)out)[k] = src[k];
    for(int k = threadIdx.x; k < nf; k += blockDim.x) ((float*)outf)[k] = srcf[k];
    __syncthreads();
    if(threadIdx.x == 0) *slot = s + 1u;
}

// The frames of the substeps of one mpm_advance, before its graph replays.
static int fill_motion_table(mpm_handle* h, double dt, double time, int nsteps)
{
    const size_t one = sizeof(mpm::ObjMotion) * MPM_MAX_OBJECTS, onef = sizeof(mpm::ObjMotionF) * MPM_MAX_OBJECTS;
    if(nsteps > h->motion_cap) {   // the replayed graphs hold the table pointers
        release_graph(h);
        MPM_CUDA(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->motion_table); cudaFree(h->motion_table_f);
        h->motion_table = nullptr; h->motion_table_f = nullptr; h->motion_cap = 0;
        MPM_CUDA(h, cudaMalloc(&h->motion_table, one * nsteps));
        MPM_CUDA(h, cudaMalloc(&h->motion_table_f, onef * nsteps));
        h->motion_cap = nsteps;
    }
    if(!h->motion_slot) MPM_CUDA(h, cudaMalloc(&h->motion_slot, sizeof(unsigned)));
    if(!h->motion_dev) MPM_CUDA(h, cudaMalloc(&h->motion_dev, one));
    if(!h->motion_dev_f) MPM_CUDA(h, cudaMalloc(&h->motion_dev_f, onef));
    std::vector<mpm::ObjMotion> m((size_t)nsteps * MPM_MAX_OBJECTS);
    std::vector<mpm::ObjMotionF> mf((size_t)nsteps * MPM_MAX_OBJECTS);
    for(int s = 0; s < nsteps; s++) {
        int rc = eval_motion(h, time + s * dt, dt, &m[(size_t)s * MPM_MAX_OBJECTS], &mf[(size_t)s * MPM_MAX_OBJECTS]);
        if(rc) return rc;
    }
    // in stream order after the earlier replays that read the tables; a copy from
    // pageable memory has staged it before it returns
    MPM_CUDA(h, cudaMemcpyAsync(h->motion_table, m.data(), one * nsteps, cudaMemcpyHostToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(h->motion_table_f, mf.data(), onef * nsteps, cudaMemcpyHostToDevice, h->stream));
    MPM_CUDA(h, cudaMemsetAsync(h->motion_slot, 0, sizeof(unsigned), h->stream));
    return MPM_OK;
}

// The moving objects' frames at time and time + dt and twists at time + dt,
// from their callbacks, copied to the device in stream order (from host memory
// the copy has staged before it returns, so the next substep may refill it);
// inside mpm_advance the next slot of the prepared tables instead.
int update_motion(mpm_handle* h, double time, double dt)
{
    if(!h->moving) return MPM_OK;
    if(h->motion_from_table) {
        k_motion_pick<<<1, 256, 0, h->stream>>>(h->motion_table, h->motion_table_f, h->motion_slot, h->motion_cap,
                                                h->motion_dev, h->motion_dev_f);
        MPM_LAUNCHED(h, "k_motion_pick");
        return MPM_OK;
    }
    mpm::ObjMotion m[MPM_MAX_OBJECTS] = {};
    mpm::ObjMotionF mf[MPM_MAX_OBJECTS] = {};
    int rc = eval_motion(h, time, dt, m, mf);
    if(rc) return rc;
    if(!h->motion_dev) MPM_CUDA(h, cudaMalloc(&h->motion_dev, sizeof(m)));
    if(!h->motion_dev_f) MPM_CUDA(h, cudaMalloc(&h->motion_dev_f, sizeof(mf)));
    MPM_CUDA(h, cudaMemcpyAsync(h->motion_dev, m, sizeof(m), cudaMemcpyHostToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(h->motion_dev_f, mf, sizeof(mf), cudaMemcpyHostToDevice, h->stream));
    return MPM_OK;
}

// One substep: the three phases back to back.
static bool reduces_dt(const mpm_handle* h) { return h->dt_control.strong_cfl || h->dt_control.sound_cfl; }

// Advance_One_Time_Step: p2g, forces, Reduce_Dt (plain path, when asked), g2p
static int enqueue_substep(mpm_handle* h, double dt, double time)
{
    int rc = mpm_particle_to_grid(h, dt, time);
    if(!rc) rc = mpm_apply_forces(h, dt, time);
    double taken = dt;
    if(!rc && !fast(h) && reduces_dt(h)) rc = plain_reduce_dt(h, dt, &taken);
    if(!rc) rc = mpm_grid_to_particle(h, taken, time);
    h->last_dt = taken;
    return rc;
}

// Run a substep from its captured graph (captured on first use), or eagerly
// when per-kernel timing is on (events cannot live inside a graph).  The fast
// path alternates its particle buffers, so it keeps one graph per parity.
static int run_substep(mpm_handle* h, double dt, double time)
{
    if(h->timing || h->implicit.enabled || (h->moving && !h->motion_from_table) || (!fast(h) && reduces_dt(h)))
        return enqueue_substep(h, dt, time);
    // the fast path's full sort after new particles runs eagerly, never in a graph
    int prc = fast(h) ? fast_prepare(h) : MPM_OK;
    if(prc) return prc;
    const int par = fast(h) ? h->fast.cur : 0;
    cudaGraphExec_t& ge = h->graphs[par];
    if(!ge) {
        cudaGraph_t g;
        MPM_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int crc = enqueue_substep(h, dt, time);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if(fast(h)) h->fast.cur = par;     // capture executed nothing
        if(crc) { if(e == cudaSuccess) cudaGraphDestroy(g); return crc; }
        if(e != cudaSuccess) return check_cuda(h, e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if(e != cudaSuccess) { ge = nullptr; return check_cuda(h, e, "cudaGraphInstantiate"); }
        h->graph_dt = dt;
    }
    MPM_CUDA(h, cudaGraphLaunch(ge, h->stream));
    h->last_dt = dt;
    if(fast(h)) h->fast.cur = 1 - par;
    return MPM_OK;
}

extern "C" {

const char* mpm_status_string(int s)
{
    switch(s) {
        case MPM_OK: return "ok";
        case MPM_ERR_ARG: return "bad argument";
        case MPM_ERR_CUDA: return "CUDA error";
        case MPM_ERR_NAN: return "non-finite value";
        case MPM_ERR_DOMAIN: return "particle outside the grid";
        case MPM_ERR_TIMEOUT: return "device wait timed out";
        case MPM_ERR_NOMEM: return "out of device memory";
        case MPM_ERR_STATE: return "call out of order";
        case MPM_ERR_NOT_CONVERGED: return "SVD did not converge";
    }
    return "unknown status";
}

int mpm_last_error(mpm_handle* h, char* buf, int len)
{
    if(!h || !buf || len <= 0) return MPM_ERR_ARG;
    snprintf(buf, (size_t)len, "%s", h->last_error.c_str());
    return MPM_OK;
}

int mpm_create(const mpm_grid_desc* g, const mpm_model_desc* m, mpm_handle** out)
{
    if(!g || !m || !out) return MPM_ERR_ARG;
    *out = nullptr;
    if(g->dim != 2 && g->dim != 3) return MPM_ERR_ARG;
    if(g->ghost != MPM_GHOST) return MPM_ERR_ARG;
    if(m->model != MPM_COROTATED_FIXED && m->model != MPM_NEO_HOOKEAN && m->model != MPM_STVK_HENCKY) return MPM_ERR_ARG;
    if(m->precision != MPM_FP32 && m->precision != MPM_FP64) return MPM_ERR_ARG;
    if(m->path != MPM_PATH_FAST && m->path != MPM_PATH_PLAIN) return MPM_ERR_ARG;
    if(m->path == MPM_PATH_FAST && (g->dim != 3 || m->precision != MPM_FP32)) return MPM_ERR_ARG;
    for(int k = 0; k < g->dim; k++) {
        if(g->counts[k] < 1 || g->counts[k] > 4096) return MPM_ERR_ARG;
        if(!(g->domain_max[k] > g->domain_min[k])) return MPM_ERR_ARG;
    }
    mpm_handle* h = new(std::nothrow) mpm_handle();
    if(!h) return MPM_ERR_NOMEM;
    if(cudaGetDevice(&h->device) != cudaSuccess) { delete h; return MPM_ERR_CUDA; }
    if(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess) { delete h; return MPM_ERR_CUDA; }
    if(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return MPM_ERR_CUDA; }
    h->own_stream = true;
    h->grid = *g;
    h->model = *m;
    SceneParams& sp = h->sp;
    memset(&sp, 0, sizeof(sp));
    sp.dim = g->dim;
    for(int k = 0; k < 3; k++) {
        bool on = k < g->dim;
        sp.counts[k] = on ? g->counts[k] : 1;
        sp.dmin[k] = on ? g->domain_min[k] : 0;
        sp.dmax[k] = on ? g->domain_max[k] : 1;
        sp.dx[k] = (sp.dmax[k] - sp.dmin[k]) / sp.counts[k];   // GRID::Initialize, GRID.cpp:23-24
        sp.inv_dx[k] = 1 / sp.dx[k];
        sp.gravity[k] = on ? m->gravity[k] : 0;
    }
    sp.model = m->model;
    if(cudaMalloc(&h->d_flags, sizeof(unsigned)) != cudaSuccess ||
       cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned), h->stream) != cudaSuccess) {
        cudaStreamDestroy(h->stream);
        delete h;
        return MPM_ERR_CUDA;
    }
    *out = h;
    return MPM_OK;
}

int mpm_destroy(mpm_handle* h)
{
    if(!h) return MPM_ERR_ARG;
    cudaStreamSynchronize(h->stream);
    release_graph(h);
    drain_timers(h);
    for(cudaEvent_t e: h->event_pool) cudaEventDestroy(e);
    diff_free(h);
    implicit_free(h);
    plain_free(h);
    fast_free(h);
    cudaFree(h->pen_f);
    cudaFree(h->motion_dev);
    cudaFree(h->motion_dev_f);
    cudaFree(h->motion_table);
    cudaFree(h->motion_table_f);
    cudaFree(h->motion_slot);
    cudaFree(h->d_flags);
    if(h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return MPM_OK;
}

int mpm_set_stream(mpm_handle* h, void* stream)
{
    if(!h) return MPM_ERR_ARG;
    cudaStreamSynchronize(h->stream);
    release_graph(h);
    if(h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
    return MPM_OK;
}

int mpm_set_collision_objects(mpm_handle* h, const mpm_collision_object* objs, int count)
{
    if(!h || count < 0 || count > MPM_MAX_OBJECTS || (count && !objs)) return MPM_ERR_ARG;
    if(count && h->reflect.enabled && h->reflect.full_reflection)
        return set_error(h, MPM_ERR_ARG, "full reflection is built for scenes without collision objects");
    for(int i = 0; i < count; i++) {
        const mpm_collision_object& o = objs[i];
        if(o.kind != MPM_BOX && o.kind != MPM_PLANE && o.kind != MPM_SPHERE) return set_error(h, MPM_ERR_ARG, "unknown object kind");
        if(o.kind == MPM_SPHERE && !(o.b[0] > 0)) return set_error(h, MPM_ERR_ARG, "sphere radius must be positive");
        if(o.type < MPM_STICK || o.type > MPM_SEPARATE) return set_error(h, MPM_ERR_ARG, "unknown collision type");
        if(o.kind == MPM_BOX)
            for(int k = 0; k < h->sp.dim; k++)
                if(!(o.b[k] > o.a[k])) return set_error(h, MPM_ERR_ARG, "box with an empty side (RANGE::Signed_Distance)");
    }
    if(fast(h) && h->fast.batch) return set_error(h, MPM_ERR_ARG, "a batch takes its objects at mpm_batch_create");
    release_graph(h);
    h->moving = 0;   // a new object list starts static
    for(int j = 0; j < MPM_MAX_OBJECTS; j++) { h->motion_fn[j] = nullptr; h->motion_user[j] = nullptr; }
    h->sp.nobj = count;
    for(int i = 0; i < count; i++) {
        mpm::DevObject& d = h->sp.objs[i];
        d.kind = objs[i].kind;
        d.type = objs[i].type;
        d.friction = objs[i].friction;
        for(int k = 0; k < 3; k++) { d.a[k] = objs[i].a[k]; d.b[k] = objs[i].b[k]; }
    }
    if(fast(h) && h->fast.scenes) {   // particles already set: refresh the device tables of scene 0
        FastState& f = h->fast;
        f.objs_h.assign(count > 0 ? count : 1, mpm::DevObject{});
        for(int i = 0; i < count; i++) f.objs_h[i] = h->sp.objs[i];
        f.scenes_h[0].obj_begin = 0;
        f.scenes_h[0].nobj = count;
        cudaFree(f.objs);
        f.objs = nullptr;
        MPM_CUDA(h, cudaMalloc(&f.objs, f.objs_h.size() * sizeof(mpm::DevObject)));
        MPM_CUDA(h, cudaMemcpy(f.objs, f.objs_h.data(), f.objs_h.size() * sizeof(mpm::DevObject), cudaMemcpyHostToDevice));
        MPM_CUDA(h, cudaMemcpy(f.scenes, f.scenes_h.data(), sizeof(SceneDev), cudaMemcpyHostToDevice));
    }
    return MPM_OK;
}

int mpm_set_particles(mpm_handle* h, const mpm_particles_view* v)
{
    if(!h || !v || v->n < 0) return MPM_ERR_ARG;
    if(v->dtype != MPM_FP32 && v->dtype != MPM_FP64) return set_error(h, MPM_ERR_ARG, "dtype");
    diff_invalidate(h);
    const uint64_t gen = h->fast.generation;
    int rc = fast(h) ? fast_set_particles(h, v) : plain_set_particles(h, v);
    // captured substeps hold buffer addresses: keep them only if none moved
    if(!fast(h) || h->fast.generation != gen || rc) release_graph(h);
    if(rc) return rc;
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    h->n = v->n;
    h->have_particles = true;
    return read_flags(h);
}

int mpm_get_particles(mpm_handle* h, mpm_particles_view* v)
{
    if(!h || !v) return MPM_ERR_ARG;
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    if(v->dtype != MPM_FP32 && v->dtype != MPM_FP64) return set_error(h, MPM_ERR_ARG, "dtype");
    return fast(h) ? fast_get_particles(h, v) : plain_get_particles(h, v);
}

static int check_dt(mpm_handle* h, double dt)
{
    if(!h) return MPM_ERR_ARG;
    if(!(dt > 0) || !std::isfinite(dt)) return set_error(h, MPM_ERR_ARG, "dt must be positive");
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    return MPM_OK;
}

int mpm_particle_to_grid(mpm_handle* h, double dt, double time)
{
    int rc = check_dt(h, dt);
    if(rc) return rc;
    return fast(h) ? fast_p2g(h, dt, time) : plain_p2g(h, dt, time);
}

int mpm_apply_forces(mpm_handle* h, double dt, double time)
{
    int rc = check_dt(h, dt);
    if(!rc) rc = update_motion(h, time, dt);
    if(rc) return rc;
    if(fast(h)) return fast_forces(h, dt, time);
    return h->implicit.enabled ? plain_implicit_forces(h, dt, time) : plain_forces(h, dt, time);
}

int mpm_grid_to_particle(mpm_handle* h, double dt, double time)
{
    int rc = check_dt(h, dt);
    if(rc) return rc;
    return fast(h) ? fast_g2p(h, dt, time) : plain_g2p(h, dt, time);
}

int mpm_substep(mpm_handle* h, double dt, double time)
{
    int rc = check_dt(h, dt);
    if(rc) return rc;
    return enqueue_substep(h, dt, time);
}

int mpm_advance(mpm_handle* h, double dt, double time, int nsteps)
{
    int rc = check_dt(h, dt);
    if(rc) return rc;
    if(nsteps < 0) return set_error(h, MPM_ERR_ARG, "nsteps < 0");
    if(h->graph_dt != dt) release_graph(h);
    if(fast(h) && nsteps && (rc = fast_prepare(h))) return rc;
    // moving objects: their frames go into tables first, so the substeps can replay a graph
    const bool table = h->moving && nsteps > 1 && !h->timing && !h->implicit.enabled && !(!fast(h) && reduces_dt(h));
    if(table && (rc = fill_motion_table(h, dt, time, nsteps))) return rc;
    h->motion_from_table = table;
    for(int s = 0; s < nsteps && !rc; s++) rc = run_substep(h, dt, time + s * dt);
    h->motion_from_table = false;
    return rc;
}

int mpm_synchronize(mpm_handle* h)
{
    if(!h) return MPM_ERR_ARG;
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    MPM_CUDA(h, cudaGetLastError());
    return read_flags(h);
}

int mpm_get_grid(mpm_handle* h, double* m, double* v0, double* v, double* vf)
{
    if(!h) return MPM_ERR_ARG;
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    if(fast(h) && h->fast.nscenes != 1) return set_error(h, MPM_ERR_ARG, "a batch returns its grids per scene: mpm_batch_get_grid");
    return fast(h) ? fast_get_grid(h, 0, m, v0, v, vf) : plain_get_grid(h, m, v0, v, vf);
}

int mpm_add_grid_forces(mpm_handle* h, double dt, const void* force, int dtype, int on_device)
{
    if(!h || !force) return MPM_ERR_ARG;
    if(!(dt > 0) || !std::isfinite(dt)) return set_error(h, MPM_ERR_ARG, "dt must be positive");
    if(dtype != MPM_FP32 && dtype != MPM_FP64) return set_error(h, MPM_ERR_ARG, "dtype");
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    if(h->implicit.enabled) return set_error(h, MPM_ERR_ARG, "extra node forces enter the explicit substep");
    if(fast(h) && h->fast.nscenes != 1) return set_error(h, MPM_ERR_ARG, "extra node forces take single-scene handles");
    return fast(h) ? fast_add_forces(h, dt, force, dtype, on_device != 0) : plain_add_forces(h, force, dtype, on_device != 0);
}

int mpm_batch_get_grid(mpm_handle* h, int scene, double* m, double* v, double* vf)
{
    if(!h) return MPM_ERR_ARG;
    if(!fast(h)) return set_error(h, MPM_ERR_ARG, "grids per scene belong to fast-path handles");
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    return fast_get_grid(h, scene, m, nullptr, v, vf);
}

int mpm_count_valid(mpm_handle* h, int64_t* count)
{
    if(!h || !count) return MPM_ERR_ARG;
    if(!h->have_particles) { *count = 0; return MPM_OK; }
    return fast(h) ? fast_count_valid(h, count) : plain_count_valid(h, count);
}

int mpm_batch_create(const mpm_scene_desc* scenes, int count, const mpm_collision_object* objects, int object_count,
    mpm_handle** out)
{
    if(!scenes || !out || count < 1 || object_count < 0 || (object_count && !objects)) return MPM_ERR_ARG;
    *out = nullptr;
    for(int i = 0; i < count; i++)
        if(scenes[i].model < MPM_COROTATED_FIXED || scenes[i].model > MPM_STVK_HENCKY) return MPM_ERR_ARG;
    mpm_model_desc m;
    memset(&m, 0, sizeof(m));
    m.model = scenes[0].model;
    m.precision = MPM_FP32;
    m.path = MPM_PATH_FAST;
    mpm_handle* h = nullptr;
    int rc = mpm_create(&scenes[0].grid, &m, &h);
    if(rc) return rc;
    h->fast.batch = true;
    if((rc = fast_setup_scenes(h, scenes, count, objects, object_count))) {
        mpm_destroy(h);
        return rc;
    }
    *out = h;
    return MPM_OK;
}

int mpm_autotune_ex(mpm_handle* h, double dt, int substeps, int flags, char* report, int report_len)
{
    int rc = check_dt(h, dt);
    if(rc) return rc;
    if(!fast(h)) return set_error(h, MPM_ERR_ARG, "the autotuner tunes the fast path");
    if(flags & ~MPM_AUTOTUNE_COLD_L2) return set_error(h, MPM_ERR_ARG, "unknown autotune flag");
    release_graph(h);
    if((rc = fast_autotune(h, dt, substeps, flags, report, report_len))) return rc;
    return read_flags(h);
}

int mpm_autotune(mpm_handle* h, double dt, int substeps, char* report, int report_len)
{
    return mpm_autotune_ex(h, dt, substeps, 0, report, report_len);
}

int mpm_set_launch_shape(mpm_handle* h, int p2g_variant, int g2p_threads, int cta_mult)
{
    if(!h) return MPM_ERR_ARG;
    if(!fast(h)) return set_error(h, MPM_ERR_ARG, "launch shapes belong to the fast path");
    if(p2g_variant < MPM_P2G_GROUPS128 || p2g_variant > MPM_P2G_FIXED256) return set_error(h, MPM_ERR_ARG, "unknown P2G variant");
    if(g2p_threads != 64 && g2p_threads != 128 && g2p_threads != 256) return set_error(h, MPM_ERR_ARG, "G2P threads: 64, 128 or 256");
    if(cta_mult != 1 && cta_mult != 2) return set_error(h, MPM_ERR_ARG, "CTA multiplier: 1 or 2");
    release_graph(h);
    h->fast.p2g_variant = p2g_variant;
    h->fast.g2p_threads = g2p_threads;
    h->fast.cta_mult = cta_mult;
    return MPM_OK;
}

int mpm_get_launch_shape(mpm_handle* h, int* p2g_variant, int* g2p_threads, int* cta_mult)
{
    if(!h || !p2g_variant || !g2p_threads || !cta_mult) return MPM_ERR_ARG;
    if(!fast(h)) return set_error(h, MPM_ERR_ARG, "launch shapes belong to the fast path");
    *p2g_variant = h->fast.p2g_variant;
    *g2p_threads = h->fast.g2p_threads;
    *cta_mult = h->fast.cta_mult;
    return MPM_OK;
}

int mpm_set_diff_tape_budget(mpm_handle* h, int64_t bytes)
{
    if(!h) return MPM_ERR_ARG;
    h->diff_budget = bytes;
    return MPM_OK;
}

int mpm_diff_forward(mpm_handle* h, double dt, int nsteps, int checkpoint_every)
{
    int rc = check_dt(h, dt);
    if(rc) return rc;
    release_graph(h);
    if((rc = diff_forward(h, dt, nsteps, checkpoint_every))) return rc;
    return mpm_synchronize(h);
}

int mpm_diff_backward(mpm_handle* h, const mpm_particles_view* grad_final, mpm_particles_view* grad_initial,
    void* grad_mu, void* grad_lambda)
{
    if(!h || !grad_final || !grad_initial) return MPM_ERR_ARG;
    int rc = diff_backward(h, grad_final, grad_initial, grad_mu, grad_lambda);
    if(rc) return rc;
    return read_flags(h);
}

int mpm_radix_sort_u32(const uint32_t* keys, int64_t n, int bits, uint32_t* sorted_keys, uint32_t* perm)
{
    return radix_sort_host(keys, n, bits, sorted_keys, perm);
}

int mpm_debug_sort_stall(const uint32_t* keys, int64_t n, int bits, uint32_t spin_limit)
{
    return debug_sort_stall(keys, n, bits, spin_limit);
}

int mpm_debug_set_sort_epoch(mpm_handle* h, uint32_t epoch)
{
    if(!h) return MPM_ERR_ARG;
    if(!fast(h)) return set_error(h, MPM_ERR_ARG, "the sort scratch exists on the fast path only");
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    return debug_set_sort_epoch(h, epoch);
}

int mpm_debug_set_svd_iterations(int max_it)
{
    if(max_it < 0 || max_it > 1000000) return MPM_ERR_ARG;
    cudaError_t (*set[])(int) = {svd_limit_plain, svd_limit_adjoint, svd_limit_implicit, svd_limit_fast, svd_limit_capi};
    for(auto f: set)
        if(f(max_it) != cudaSuccess) return MPM_ERR_CUDA;
    return MPM_OK;
}

int mpm_debug_sort_state(mpm_handle* h, uint32_t* slot_keys, uint32_t* sorted_keys, uint32_t* perm)
{
    if(!h) return MPM_ERR_ARG;
    if(!fast(h)) return set_error(h, MPM_ERR_ARG, "sort state exists on the fast path only");
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    return fast_debug_sort_state(h, slot_keys, sorted_keys, perm);
}

int mpm_set_implicit(mpm_handle* h, const mpm_implicit_desc* d)
{
    if(!h || !d) return MPM_ERR_ARG;
    if(d->enabled) {
        if(fast(h)) return set_error(h, MPM_ERR_ARG, "the implicit solve runs on the plain path");
        if(!(d->newton_tolerance >= 0) || !std::isfinite(d->newton_tolerance) || d->newton_iterations < 1 ||
           !(d->solver_tolerance > 0) || !std::isfinite(d->solver_tolerance) || d->solver_iterations < 1)
            return set_error(h, MPM_ERR_ARG, "implicit solve parameters");
    }
    release_graph(h);
    h->implicit = *d;
    h->implicit.enabled = d->enabled ? 1 : 0;
    return MPM_OK;
}

int mpm_set_reflection(mpm_handle* h, const mpm_reflection_desc* r)
{
    if(!h || !r) return MPM_ERR_ARG;
    if(r->enabled) {
        if(fast(h)) return set_error(h, MPM_ERR_ARG, "reflection boundary conditions run on the plain path");
        for(int k = 0; k < 2 * h->sp.dim; k++)
            if(r->side_type[k] < MPM_BC_FREE || r->side_type[k] > MPM_BC_SEP) return set_error(h, MPM_ERR_ARG, "side type");
        if(!(r->friction >= 0) || !std::isfinite(r->friction)) return set_error(h, MPM_ERR_ARG, "reflection friction");
        if(r->full_reflection && h->sp.nobj)
            return set_error(h, MPM_ERR_ARG, "full reflection is built for scenes without collision objects");
    }
    release_graph(h);
    h->reflect = *r;
    h->reflect.enabled = r->enabled ? 1 : 0;
    for(int k = 2 * h->sp.dim; k < 6; k++) h->reflect.side_type[k] = MPM_BC_FREE;
    return MPM_OK;
}

int mpm_set_penalty_objects(mpm_handle* h, const mpm_collision_object* objs, int count, double stiffness,
                            double separation)
{
    if(!h || count < 0 || count > MPM_MAX_OBJECTS || (count && !objs)) return MPM_ERR_ARG;
    if(count) {
        if(fast(h) && h->fast.batch) return set_error(h, MPM_ERR_ARG, "a batch takes no penalty objects");
        if(!(stiffness >= 0) || !std::isfinite(stiffness) || !std::isfinite(separation))
            return set_error(h, MPM_ERR_ARG, "penalty stiffness must be finite and >= 0, separation finite");
    }
    for(int i = 0; i < count; i++) {
        const mpm_collision_object& o = objs[i];
        if(o.kind != MPM_BOX && o.kind != MPM_PLANE && o.kind != MPM_SPHERE) return set_error(h, MPM_ERR_ARG, "unknown object kind");
        if(o.kind == MPM_SPHERE && !(o.b[0] > 0)) return set_error(h, MPM_ERR_ARG, "sphere radius must be positive");
        if(o.kind == MPM_BOX)
            for(int k = 0; k < h->sp.dim; k++)
                if(!(o.b[k] > o.a[k])) return set_error(h, MPM_ERR_ARG, "box with an empty side (RANGE::Signed_Distance)");
    }
    release_graph(h);
    h->sp.npen = count;
    h->sp.pen_stiffness = stiffness;
    h->sp.pen_separation = separation;
    for(int i = 0; i < count; i++) {
        mpm::DevObject& d = h->sp.pen[i];
        d.kind = objs[i].kind;
        d.type = objs[i].type;
        d.friction = objs[i].friction;
        for(int k = 0; k < 3; k++) { d.a[k] = objs[i].a[k]; d.b[k] = objs[i].b[k]; }
    }
    if(fast(h) && count) {   // the fast path reads them from device memory, in float
        mpm::DevObjectF tab[MPM_MAX_OBJECTS] = {};
        for(int i = 0; i < count; i++) {
            const mpm::DevObject& o = h->sp.pen[i];
            tab[i].kind = o.kind;
            tab[i].type = o.type;
            tab[i].friction = (float)o.friction;
            for(int k = 0; k < 3; k++) { tab[i].a[k] = (float)o.a[k]; tab[i].b[k] = (float)o.b[k]; }
        }
        if(!h->pen_f) MPM_CUDA(h, cudaMalloc(&h->pen_f, sizeof(tab)));
        MPM_CUDA(h, cudaMemcpy(h->pen_f, tab, sizeof(tab), cudaMemcpyHostToDevice));
        return fast_penalty_buffers(h);
    }
    return MPM_OK;
}

int mpm_set_object_motion(mpm_handle* h, int object, mpm_motion_fn fn, void* user)
{
    if(!h) return MPM_ERR_ARG;
    if(object < 0 || object >= h->sp.nobj) return set_error(h, MPM_ERR_ARG, "no collision object with that index");
    if(fast(h) && h->fast.batch) return set_error(h, MPM_ERR_ARG, "a batch takes no moving objects");
    release_graph(h);
    h->motion_fn[object] = fn;
    h->motion_user[object] = fn ? user : nullptr;
    if(fn) h->moving |= 1u << object;
    else h->moving &= ~(1u << object);
    return MPM_OK;
}

// A per-particle byte array (caller order) on the device: the plain path's
// particles are in caller order, the fast path looks it up by caller index.
static int set_particle_bytes(mpm_handle* h, uint8_t*& dst, const uint8_t* src, int64_t n)
{
    release_graph(h);
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    if(!src) {
        cudaFree(dst);
        dst = nullptr;
        return MPM_OK;
    }
    if(!dst) MPM_CUDA(h, cudaMalloc(&dst, (size_t)(n ? n : 1)));
    MPM_CUDA(h, cudaMemcpy(dst, src, (size_t)n, cudaMemcpyHostToDevice));
    return MPM_OK;
}

int mpm_set_particle_models(mpm_handle* h, const uint8_t* models, int64_t n)
{
    if(!h) return MPM_ERR_ARG;
    if(fast(h) && h->fast.batch) return set_error(h, MPM_ERR_ARG, "a batch takes one model per scene");
    const int64_t count = fast(h) ? h->fast.n : h->plain.n;
    if(models) {
        if(!h->have_particles || n != count) return set_error(h, MPM_ERR_ARG, "one model per particle, after mpm_set_particles");
        for(int64_t p = 0; p < n; p++)
            if(models[p] != MPM_COROTATED_FIXED && models[p] != MPM_NEO_HOOKEAN && models[p] != MPM_STVK_HENCKY)
                return set_error(h, MPM_ERR_ARG, "unknown constitutive model");
    }
    return set_particle_bytes(h, fast(h) ? h->fast.pmodel : h->plain.pmodel, models, n);
}

int mpm_set_plastic_particles(mpm_handle* h, const uint8_t* mask, int64_t n)
{
    if(!h) return MPM_ERR_ARG;
    if(fast(h) && h->fast.batch) return set_error(h, MPM_ERR_ARG, "a batch takes one plasticity for all particles");
    const int64_t count = fast(h) ? h->fast.n : h->plain.n;
    if(mask && (!h->have_particles || n != count)) return set_error(h, MPM_ERR_ARG, "one flag per particle, after mpm_set_particles");
    int rc = set_particle_bytes(h, fast(h) ? h->fast.pmask : h->plain.pmask, mask, n);
    if(rc) return rc;
    if(h->plastic.kind != MPM_PLASTICITY_NONE && h->have_particles) return fast(h) ? fast_plastic_init(h) : plain_plastic_init(h);
    return MPM_OK;
}

int mpm_set_dt_control(mpm_handle* h, const mpm_dt_control* c)
{
    if(!h || !c) return MPM_ERR_ARG;
    if(!(c->cfl > 0) || !(c->min_dt >= 0) || !(c->max_dt > 0) || !(c->max_dt >= c->min_dt) || !std::isfinite(c->max_dt))
        return set_error(h, MPM_ERR_ARG, "dt control: cfl > 0, 0 <= min_dt <= max_dt");
    if((c->strong_cfl && !(c->cfl_F > 0)) || (c->sound_cfl && !(c->cfl_sound > 0)))
        return set_error(h, MPM_ERR_ARG, "dt control: CFL numbers must be positive");
    if(fast(h) && (c->strong_cfl || c->sound_cfl))
        return set_error(h, MPM_ERR_ARG, "the strong and sound-speed CFL reductions run on the plain path");
    release_graph(h);
    h->dt_control = *c;
    return MPM_OK;
}

int mpm_last_dt(mpm_handle* h, double* dt)
{
    if(!h || !dt) return MPM_ERR_ARG;
    *dt = h->last_dt;
    return MPM_OK;
}

int mpm_simulate_frame(mpm_handle* h, double time, double frame_dt, double* time_out, int* substeps)
{
    if(!h || !(frame_dt > 0)) return MPM_ERR_ARG;
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    const mpm_dt_control& c = h->dt_control;
    if(!(c.max_dt > 0)) return set_error(h, MPM_ERR_STATE, "mpm_set_dt_control first");
    const double time_at_frame = time + frame_dt;
    int count = 0;
    for(bool done = false; !done; count++) {
        double dt = 0;
        int rc = mpm_compute_dt(h, c.cfl, c.max_dt, &dt);
        if(rc) return rc;
        dt = dt < c.min_dt ? c.min_dt : (dt > c.max_dt ? c.max_dt : dt);
        double next = time + dt;
        if(next + .0001 * dt > time_at_frame) { next = time_at_frame; done = true; }   // roundoff
        else if(next + dt > time_at_frame) next = (time + time_at_frame) / 2;
        dt = next - time;
        if(!(dt > 0)) return set_error(h, MPM_ERR_ARG, "substep dt is not positive");
        const double original = dt;
        if((rc = mpm_substep(h, dt, time))) return rc;
        if(h->last_dt < original) {   // Reduce_Dt shortened the step
            next = time + h->last_dt;
            done = false;
        }
        time = next;
    }
    if(time_out) *time_out = time;
    if(substeps) *substeps = count;
    return MPM_OK;
}

int mpm_get_implicit_stats(mpm_handle* h, mpm_implicit_stats* s)
{
    if(!h || !s) return MPM_ERR_ARG;
    *s = h->imp_stats;
    return MPM_OK;
}

int mpm_set_plasticity(mpm_handle* h, const mpm_plasticity_desc* p)
{
    if(!h || !p) return MPM_ERR_ARG;
    if(p->kind != MPM_PLASTICITY_NONE && p->kind != MPM_PLASTICITY_CLAMP && p->kind != MPM_PLASTICITY_DRUCKER_PRAGER)
        return set_error(h, MPM_ERR_ARG, "unknown plasticity kind");
    if(p->kind == MPM_PLASTICITY_CLAMP) {
        if(!(p->theta_c >= 0 && p->theta_c < 1) || !(p->theta_s >= 0) || !std::isfinite(p->theta_s))
            return set_error(h, MPM_ERR_ARG, "clamp bounds: 0 <= theta_c < 1, 0 <= theta_s");
        if(std::isnan(p->max_hardening) || !std::isfinite(p->hardening_factor))
            return set_error(h, MPM_ERR_ARG, "hardening parameters");
    }
    if(p->kind == MPM_PLASTICITY_DRUCKER_PRAGER) {
        const double v[] = {p->dp_a0, p->dp_a1, p->dp_a3, p->dp_a4, p->cohesion};
        for(double x: v)
            if(!std::isfinite(x)) return set_error(h, MPM_ERR_ARG, "Drucker-Prager parameters must be finite");
        // rho_F divides the cohesion term: the friction angle must stay in (0, 90) degrees at q = 0
        const double phi0 = p->dp_a0 - p->dp_a4;
        if(!(phi0 > 0 && phi0 < 90)) return set_error(h, MPM_ERR_ARG, "friction angle a0 - a4 outside (0, 90) degrees");
    }
    release_graph(h);
    const int was = h->plastic.kind;
    h->plastic = *p;
    if(p->kind && p->kind != was && h->have_particles) {
        int rc = fast(h) ? fast_plastic_init(h) : plain_plastic_init(h);
        if(rc) return rc;
        MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    return MPM_OK;
}

// mu0 / lambda0 belong to the clamp, plastic_def .. vc to Drucker-Prager
static bool plastic_view_matches(const mpm_handle* h, const mpm_plastic_view* v)
{
    if(h->plastic.kind == MPM_PLASTICITY_CLAMP) return !v->plastic_def && !v->rho_F && !v->cohesion && !v->vc;
    return !v->mu0 && !v->lambda0;
}

int mpm_get_plastic_state(mpm_handle* h, mpm_plastic_view* v)
{
    if(!h || !v) return MPM_ERR_ARG;
    if(!h->plastic.kind) return set_error(h, MPM_ERR_STATE, "plasticity is off");
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    if(v->dtype != MPM_FP32 && v->dtype != MPM_FP64) return set_error(h, MPM_ERR_ARG, "dtype");
    if(!plastic_view_matches(h, v)) return set_error(h, MPM_ERR_ARG, "plastic state arrays of the other plasticity kind");
    return fast(h) ? fast_get_plastic(h, v) : plain_get_plastic(h, v);
}

int mpm_set_plastic_state(mpm_handle* h, const mpm_plastic_view* v)
{
    if(!h || !v) return MPM_ERR_ARG;
    if(!h->plastic.kind) return set_error(h, MPM_ERR_STATE, "plasticity is off");
    if(!h->have_particles) return set_error(h, MPM_ERR_STATE, "no particles set");
    if(v->dtype != MPM_FP32 && v->dtype != MPM_FP64) return set_error(h, MPM_ERR_ARG, "dtype");
    if(!plastic_view_matches(h, v)) return set_error(h, MPM_ERR_ARG, "plastic state arrays of the other plasticity kind");
    release_graph(h);
    return fast(h) ? fast_set_plastic(h, v) : plain_set_plastic(h, v);
}

int mpm_particle_totals(mpm_handle* h, mpm_totals* out)
{
    if(!h || !out) return MPM_ERR_ARG;
    memset(out, 0, sizeof(*out));
    if(!h->have_particles) return MPM_OK;
    return fast(h) ? fast_particle_totals(h, out) : plain_particle_totals(h, out);
}

int mpm_grid_totals(mpm_handle* h, mpm_totals* out)
{
    if(!h || !out) return MPM_ERR_ARG;
    memset(out, 0, sizeof(*out));
    if(!h->have_particles) return MPM_OK;
    return fast(h) ? fast_grid_totals(h, out) : plain_grid_totals(h, out);
}

int mpm_compute_dt(mpm_handle* h, double cfl, double max_dt, double* dt)
{
    if(!h || !dt || !(cfl > 0) || !(max_dt > 0)) return MPM_ERR_ARG;
    mpm_totals t;
    int rc = mpm_particle_totals(h, &t);
    if(rc) return rc;
    double dx_min = h->sp.dx[0];
    for(int k = 1; k < h->sp.dim; k++) dx_min = std::min(dx_min, h->sp.dx[k]);
    if(fast(h) && h->fast.batch)   // smallest cell of any scene
        for(const SceneDev& s: h->fast.scenes_h)
            for(int k = 0; k < 3; k++) dx_min = std::min(dx_min, (double)s.dx[k]);
    double critical = cfl * dx_min / max_dt, v = t.max_affine_speed;
    *dt = v > critical ? cfl * dx_min / v : max_dt;
    return MPM_OK;
}

int mpm_set_timing(mpm_handle* h, int enable)
{
    if(!h) return MPM_ERR_ARG;
    cudaStreamSynchronize(h->stream);
    drain_timers(h);
    h->timing = enable != 0;
    for(KernelTimer& t: h->timers) { t.ms = 0; t.launches = 0; }
    return MPM_OK;
}

int mpm_get_timing(mpm_handle* h, char* names, int names_len, double* ms, int64_t* launches, int max_entries, int* count)
{
    if(!h || !count) return MPM_ERR_ARG;
    drain_timers(h);
    std::string all;
    int c = 0;
    for(const KernelTimer& t: h->timers) {
        if(c < max_entries) {
            if(ms) ms[c] = t.ms;
            if(launches) launches[c] = t.launches;
            if(c) all += ",";
            all += t.name;
        }
        c++;
    }
    *count = c < max_entries ? c : max_entries;
    if(names && names_len > 0) snprintf(names, (size_t)names_len, "%s", all.c_str());
    return MPM_OK;
}

}  // extern "C"

// This module's copy of the SVD sweep bound (mpm_debug_set_svd_iterations).
MPM_SVD_LIMIT_SETTER(svd_limit_capi)
