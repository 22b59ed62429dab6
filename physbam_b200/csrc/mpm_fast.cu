// Fast path: the explicit MPM substep in FP32 with block-sorted particles, for
// one scene or a batch of independent scenes (a single scene is a batch of one).
//
// Per substep (MPM_DRIVER::Advance_One_Time_Step, MPM_DRIVER.cpp:141-157), each
// phase is ONE launch over the blocks of all scenes:
//   bins     the substep's order from the previous one: per particle block
//            (4^3 cells) its arrivals, counted by the last G2P in the block's
//            row by direction, a scan into block ranges, the work items (parts
//            of a block's particles) and where each group of moved particles
//            lands.
//   route    every particle slot to its place in that order (a stable sort by
//            block; invalid particles go to the tail).
//   p2g      persistent CTAs over the work items: B-spline weights, the stress P(F) F^T (fused;
//            MPM_FINITE_ELEMENTS::Precompute, .cpp:47-67), APIC momentum plus
//            dt * force into a 6^3-node shared fixed-point tile, flushed with
//            one float4 atomic per touched node (Particle_To_Grid l.245-306 with
//            MPM_FINITE_ELEMENTS::Add_Forces folded in).  It marks the node
//            blocks its tile covers.
//   grid     one thread per node of the marked node blocks: v = (mv + dt f)/m
//            + dt g, collision projection and friction (Apply_Forces
//            l.959-1060); clears the accumulator for the next substep.
//   g2p      persistent CTAs over the work items: the tile of (v, v_fric) by TMA
//            (the next item's copy in flight), gather, update F,
//            X, V and the APIC B (Grid_To_Particle l.450-515), write the
//            particle to its slot in the other buffer with its next key, and
//            count where the part's particles move (the next bins' input).
// After new particles (or a restore) a full radix sort of the keys orders the
// slots once (fast_prepare).  Scenes differ in grid size, domain, model and
// collision objects; blocks and node blocks of all scenes share one
// numbering, and a CTA looks up the scene of the block it works on.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "mpm_internal.h"
#include "mpm_sort.cuh"

namespace {

using namespace mpm;

constexpr int BS = 4;                      // cells per particle-block edge
constexpr int TE = BS + 2;                 // tile edge in nodes
constexpr int TN = TE * TE * TE;           // 216 nodes per tile
// P2G tile layout: node (x, y, z) of the 6^3 tile at x PSX + y PSY + z.  With
// these strides the 32 cells of a warp-aligned half block (cell = lx << 4 |
// ly << 2 | lz, lx in {0, 1} or {2, 3}) reach 32 distinct shared-memory banks
// at every node offset (52 lx + 8 ly + lz is distinct mod 32), where the
// dense 6-stride layout put up to four lanes on one bank.
constexpr int PSY = 8, PSX = 52;
constexpr int PTN = (TE - 1) * PSX + (TE - 1) * PSY + TE;   // 306 floats per quantity
__host__ __device__ constexpr int ptile(int x, int y, int z) { return x * PSX + y * PSY + z; }
constexpr uint32_t SENTINEL = 0xffffffffu;
constexpr int NCOMP = 24;                  // x3 v3 F9 B9 floats per particle
constexpr int C_X = 0, C_V = 3, C_F = 6, C_B = 15;
constexpr int NPLAS = 13;                  // plastic state floats per particle: Fp0..8, then
                                           // mu0, lambda0 (clamp) or plastic_def, rho_F, sigma_Y, vc

// Move directions of a particle between two substeps' orders: the 27
// neighbour blocks (dx, dy, dz in -1..1, index (dx+1) 9 + (dy+1) 3 + dz+1),
// then farther than a neighbour, then invalidated.
constexpr int NDIR = 29;
constexpr int DIR_STAY = 13, DIR_FAR = 27, DIR_INVALID = 28;
// Row of a block in the arrival counts (dcount): one 128-byte line, entries
// 0..26 the arrivals from each neighbour direction, 27 the arrivals from
// farther away.  Row of a block in the offsets (doff): entries 0..26 the first
// sorted position of the group of its particles that moved in direction d,
// 27 the next sorted position of an arrival from farther away, 28 the first
// tail slot of the particles it lost out of the domain.
constexpr int ROW = 32;
constexpr int SCAN_TILE = 256;             // allocation unit of the block scan's status words (>= its tiles)
// Largest work item (particles of one block) of each P2G launch shape.
constexpr int kPartSize[4] = {512, 1024, 128, 256};

struct FastArgs {
    int64_t n, npad;
    const float* src;
    const float4* src_attr;
    const int* src_pid;
    float* dst;
    float4* dst_attr;
    int* dst_pid;
    uint32_t* perm;
    uint32_t* sorted_keys;
    const uint32_t* keys_cur;   // cell keys of the current buffer's slots
    uint32_t* keys_next;        // cell keys of the other buffer's slots (G2P writes them)
    const uint8_t* dir_cur;     // move directions of the current buffer's slots
    uint8_t* dir_next;          // move directions of the other buffer's slots (G2P writes them)
    // this substep's order: block ranges, active blocks, work items, counters
    uint32_t *bstart, *bend, *ctr;
    uint4* active;              // active blocks: (block, start, count or SENTINEL, scene)
    uint4* chunks;
    // the previous substep's order (routing input)
    const uint32_t *obstart, *obend, *octr;
    const uint4* oactive;
    uint32_t* nctr;             // the next substep's counters (the same storage as octr; G2P clears it)
    uint32_t *dcount, *doff, *scan;
    unsigned long long* bcount;
    int64_t nblk;               // particle blocks of all scenes
    int part;                   // P2G work-item size (particles)
    uint32_t chunk_cap;         // capacity of the work-item lists
    uint32_t *nb_flag, *nb_list;
    uint32_t* fallback;   // sorted positions whose stress takes the FP64 route (P2G)
    const CUtensorMap* tmaps;   // per scene: its grid of 8-float nodes as a 4D tensor (G2P tiles)
    float4* acc;
    float4* vel;
    const SceneDev* scenes;
    const uint16_t* block_scene;
    const uint16_t* nb_scene;
    const int64_t* pbase;
    const DevObject* objs;
    int nscenes;
    float dt;
    unsigned* flags;
    const float* psrc;    // plastic state (null: plasticity off), current and next buffer
    float* pdst;
    int pkind, nplas;     // plasticity kind; plastic floats per particle
    float prm[5];         // clamp: theta_c, theta_s, max_hardening, hardening_factor;
                          // Drucker-Prager: a0, a1, a3, a4, use_vc
    const DevObjectF* pen;    // penalty collision objects (npen of them)
    int npen;
    float pen_k, pen_sep;     // their stiffness and separation
    const float* vsrc;        // the velocities P2G reads (3 x npad): src's, or V + dt f / m with penalty objects
    float* vkick;             // where k_penalty_kick writes V + dt f / m
    const ObjMotionF* motion; // moving collision objects (bit j of `moving`, single-scene handles)
    unsigned moving;
    const uint8_t* pmodel;    // constitutive model per caller particle index, or null (the scene's)
    const uint8_t* pmask;     // plasticity on, per caller particle index, or null (all)
};

// The constitutive model of the particle in slot i of the current buffer.
__device__ __forceinline__ int slot_model(const FastArgs& a, const SceneDev& sc, uint32_t i)
{
    return a.pmodel ? (int)a.pmodel[a.src_pid[i]] : sc.model;
}

__device__ __forceinline__ int64_t node_index(const SceneDev& sc, int qx, int qy, int qz)
{
    return sc.node_base + ((int64_t)qx * sc.GA[1] + qy) * sc.GA[2] + qz;
}

// Cell key of a position in scene sc: its global block and in-block cell of the
// first stencil node (base + 3 in ghosted node coordinates).  SENTINEL when the
// stencil would leave the ghosted grid.
__device__ __forceinline__ uint32_t cell_key(const SceneDev& sc, const float* X)
{
    int cc[3];
#pragma unroll
    for(int k = 0; k < 3; k++) {
        float y = X[k] - sc.dx[k];
        int base = (int)floorf((y - sc.dmin[k]) * sc.inv[k]);
        cc[k] = base + MPM_GHOST;
        if(cc[k] < 0 || cc[k] > sc.counts[k] + MPM_GHOST) return SENTINEL;
    }
    uint32_t b = ((uint32_t)(cc[0] >> 2) * sc.NB[1] + (uint32_t)(cc[1] >> 2)) * sc.NB[2] + (uint32_t)(cc[2] >> 2);
    return ((sc.block_base + b) << 6) | ((cc[0] & 3) << 4) | ((cc[1] & 3) << 2) | (cc[2] & 3);
}

__device__ __forceinline__ void block_coords(const SceneDev& sc, uint32_t lb, int& bx, int& by, int& bz)
{
    bz = lb % sc.NB[2];
    uint32_t r = lb / sc.NB[2];
    by = r % sc.NB[1];
    bx = r / sc.NB[1];
}

// Copy scene s into shared memory (the caller synchronises before use).
__device__ __forceinline__ void stage_scene(const FastArgs& a, int s, SceneDev* out)
{
    constexpr int words = (int)(sizeof(SceneDev) / 4);
    if(threadIdx.x < words) ((uint32_t*)out)[threadIdx.x] = ((const uint32_t*)(a.scenes + s))[threadIdx.x];
}

// ---------------------------------------------------------------------------
// Stress P(F) F^T in FP32 without an SVD where that is exact in exact
// arithmetic and well conditioned; otherwise (inverted or nearly degenerate
// F, or the neo-Hookean clamp region) the caller falls back to the FP64 SVD.
//   NEO_HOOKEAN, J >= .25:  P F^T = mu (F F^T - I) + lambda ln J I
//   COROTATED_FIXED, J > 0: P F^T = 2 mu (b - sqrt(b)) + lambda J (J-1) I,
//     b = F F^T; sqrt(b) = R F^T is the left stretch, from the eigenvalues of
//     b and the closed form of Hoger & Carlson (1984):
//     sqrt(b) = (-b^2 + (I1^2 - I2) b + I1 I3 I) / (I1 I2 - I3)
//     with I1, I2, I3 the invariants of sqrt(b).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool stress_fast(int model, const float* F, float mu, float la, float* PFT)
{
    float b00 = F[0] * F[0] + F[3] * F[3] + F[6] * F[6];
    float b11 = F[1] * F[1] + F[4] * F[4] + F[7] * F[7];
    float b22 = F[2] * F[2] + F[5] * F[5] + F[8] * F[8];
    float b01 = F[0] * F[1] + F[3] * F[4] + F[6] * F[7];
    float b02 = F[0] * F[2] + F[3] * F[5] + F[6] * F[8];
    float b12 = F[1] * F[2] + F[4] * F[5] + F[7] * F[8];
    float J = F[0] * (F[4] * F[8] - F[7] * F[5]) - F[3] * (F[1] * F[8] - F[7] * F[2]) + F[6] * (F[1] * F[5] - F[4] * F[2]);
    if(model == MPM_STVK_HENCKY) {
        // P F^T = U diag(2 mu ln S + lambda tr ln S) U^T = mu ln b + (lambda / 2) tr(ln b) I,
        // U diag(S^2) U^T = b = F F^T; zero stress once det F <= 0 (the reference's
        // test on the last signed singular value)
        if(!(J > 0.f)) {
#pragma unroll
            for(int e = 0; e < 9; e++) PFT[e] = 0.f;
            return true;
        }
        float A[3][3] = {{b00, b01, b02}, {b01, b11, b12}, {b02, b12, b22}}, W[3][3];
        sym_eig3f(A, W);
        const float lmax = fmaxf(A[0][0], fmaxf(A[1][1], A[2][2])), lmin = fminf(A[0][0], fminf(A[1][1], A[2][2]));
        if(!(lmin > 1e-4f * lmax)) return false;     // sigma_min / sigma_max < 1e-2: FP64 SVD
        float l[3];
#pragma unroll
        for(int i = 0; i < 3; i++) l[i] = mu * logf(A[i][i]);
        const float pr = 0.5f * la * (logf(A[0][0]) + logf(A[1][1]) + logf(A[2][2]));
#pragma unroll
        for(int r = 0; r < 3; r++)
#pragma unroll
            for(int c = 0; c < 3; c++)
                PFT[r + 3 * c] = W[r][0] * l[0] * W[c][0] + W[r][1] * l[1] * W[c][1] + W[r][2] * l[2] * W[c][2] + (r == c ? pr : 0.f);
        return true;
    }
    if(model == MPM_NEO_HOOKEAN) {
        if(!(J >= (float)kNeoHookeanThreshold)) return false;
        float d = la * logf(J) - mu;
        PFT[0] = mu * b00 + d; PFT[4] = mu * b11 + d; PFT[8] = mu * b22 + d;
        PFT[1] = PFT[3] = mu * b01;
        PFT[2] = PFT[6] = mu * b02;
        PFT[5] = PFT[7] = mu * b12;
        return true;
    }
    if(!(J > 0.f)) return false;
    // eigenvalues of b (trigonometric form); only symmetric functions of their
    // square roots are used, which stay accurate for repeated eigenvalues
    float q = (b00 + b11 + b22) * (1.f / 3.f);
    float c00 = b00 - q, c11 = b11 - q, c22 = b22 - q;
    float off = b01 * b01 + b02 * b02 + b12 * b12;
    float p2 = (c00 * c00 + c11 * c11 + c22 * c22 + 2.f * off) * (1.f / 6.f);
    float l1, l2, l3;
    if(p2 <= 1e-14f * q * q) {
        l1 = l2 = l3 = q;
    } else {
        float p = sqrtf(p2), ip = 1.f / p;
        float e00 = c00 * ip, e11 = c11 * ip, e22 = c22 * ip, e01 = b01 * ip, e02 = b02 * ip, e12 = b12 * ip;
        float det = e00 * (e11 * e22 - e12 * e12) - e01 * (e01 * e22 - e12 * e02) + e02 * (e01 * e12 - e11 * e02);
        float r = fminf(fmaxf(0.5f * det, -1.f), 1.f);
        float phi = acosf(r) * (1.f / 3.f);
        l1 = q + 2.f * p * cosf(phi);
        l3 = q + 2.f * p * cosf(phi + 2.0943951023931953f);
        l2 = 3.f * q - l1 - l3;
    }
    if(!(l3 > 1e-4f * l1)) return false;     // sigma_min / sigma_max < 1e-2: FP64 SVD
    float m1 = sqrtf(l1), m2 = sqrtf(fmaxf(l2, 0.f)), m3 = sqrtf(l3);
    float I1 = m1 + m2 + m3, I2 = m1 * m2 + m2 * m3 + m3 * m1, I3 = J;
    float den = I1 * I2 - I3;
    if(!(den > 0.f)) return false;
    float ca = I1 * I1 - I2, cb = I1 * I3, id = 1.f / den;
    float s00 = b00 * b00 + b01 * b01 + b02 * b02;
    float s11 = b01 * b01 + b11 * b11 + b12 * b12;
    float s22 = b02 * b02 + b12 * b12 + b22 * b22;
    float s01 = b00 * b01 + b01 * b11 + b02 * b12;
    float s02 = b00 * b02 + b01 * b12 + b02 * b22;
    float s12 = b01 * b02 + b11 * b12 + b12 * b22;
    float u00 = (-s00 + ca * b00 + cb) * id, u11 = (-s11 + ca * b11 + cb) * id, u22 = (-s22 + ca * b22 + cb) * id;
    float u01 = (-s01 + ca * b01) * id, u02 = (-s02 + ca * b02) * id, u12 = (-s12 + ca * b12) * id;
    float mu2 = 2.f * mu, pr = la * J * (J - 1.f);
    PFT[0] = mu2 * (b00 - u00) + pr; PFT[4] = mu2 * (b11 - u11) + pr; PFT[8] = mu2 * (b22 - u22) + pr;
    PFT[1] = PFT[3] = mu2 * (b01 - u01);
    PFT[2] = PFT[6] = mu2 * (b02 - u02);
    PFT[5] = PFT[7] = mu2 * (b12 - u12);
    return true;
}

// FP64 fallback: the reference's signed SVD route, out of line so its
// registers do not weigh on the common path.
__device__ __noinline__ bool stress_fp64(int model, const float* Ff, float mu, float la, float* PFT)
{
    double F[9], P[9];
#pragma unroll
    for(int e = 0; e < 9; e++) F[e] = Ff[e];
    bool ok = pft_svd<double, 3>(model, F, (double)mu, (double)la, P);
#pragma unroll
    for(int e = 0; e < 9; e++) PFT[e] = (float)P[e];
    return ok;
}

// ---------------------------------------------------------------------------
__global__ void k_init_keys(FastArgs a, const uint8_t* valid_by_slot, uint32_t* out)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        // scene of particle i: pbase[s] <= i < pbase[s + 1] (particles arrive in scene order)
        int lo = 0, hi = a.nscenes - 1;
        while(lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if(a.pbase[mid] <= i) lo = mid; else hi = mid - 1;
        }
        float X[3] = {a.src[(C_X + 0) * a.npad + i], a.src[(C_X + 1) * a.npad + i], a.src[(C_X + 2) * a.npad + i]};
        uint32_t k = valid_by_slot[i] ? cell_key(a.scenes[lo], X) : SENTINEL;
        if(valid_by_slot[i] && k == SENTINEL) atomicOr(a.flags, MPM_FLAG_DOMAIN);
        out[i] = k;
    }
}

// ---------------------------------------------------------------------------
// The substep's particle order, built from the previous one.
//
// The previous G2P wrote every particle's new cell key to its slot and
// counted, in the row of each block, how many particles arrived from each
// neighbour block (dcount[block][d], d the move direction, d = DIR_FAR for
// arrivals from farther away), and per block the particles it received and
// the particles it lost out of the domain (bcount).  Slots are grouped by
// their previous block, in block order.  A stable sort by block key is then:
// new block b holds the particles that came from block b - delta(d) with
// direction d, group after group in the order of those previous blocks (each
// group in slot order), then its far arrivals; all valid particles come
// first, in block order, then the particles the last G2P invalidated (in slot
// order), then those invalid before.  k_bins scans the per-block counts into
// block ranges (one pass of decoupled look-back over tiles of blocks), turns
// each block's row of counts into the row of its groups' offsets and hands out
// the work items; k_route moves every slot to its place.  This takes the place of a radix
// sort of the keys every substep: the order equals a stable sort by block key
// whenever no particle crossed more than one block (4 cells) in the substep;
// far arrivals go to the end of their block in arrival order.  The
// reference's analogue is the binning of GATHER_SCATTER::Prepare_Scatter
// (Hybrid_Methods/Iterators/GATHER_SCATTER.cpp:33-87).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int dir_dx(int d) { return d / 9 - 1; }
__device__ __forceinline__ int dir_dy(int d) { return (d / 3) % 3 - 1; }
__device__ __forceinline__ int dir_dz(int d) { return d % 3 - 1; }

// Direction of a move from block (ox, oy, oz) to block (nx, ny, nz) of a scene.
__device__ __forceinline__ int move_dir(int ox, int oy, int oz, int nx, int ny, int nz)
{
    const int dx = nx - ox, dy = ny - oy, dz = nz - oz;
    if(dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) return DIR_FAR;
    return (dx + 1) * 9 + (dy + 1) * 3 + dz + 1;
}

// Direction of the particle with new cell key `key`, previously in block `b`
// (local coordinates bx, by, bz) of scene sc.
__device__ __forceinline__ int key_dir(const SceneDev& sc, uint32_t b, int bx, int by, int bz, uint32_t key)
{
    if(key == SENTINEL) return DIR_INVALID;
    const uint32_t nb = key >> 6;
    if(nb == b) return DIR_STAY;
    int nx, ny, nz;
    block_coords(sc, nb - sc.block_base, nx, ny, nz);
    return move_dir(bx, by, bz, nx, ny, nz);
}

// Decoupled look-back of one running count by one warp: publish the tile's
// aggregate, add the predecessors' aggregates until an inclusive prefix, then
// publish the inclusive prefix; returns the exclusive prefix (every lane).
// Each round reads a window of 32 predecessors.  Status word of tile t at
// status[t * STATUS_STRIDE], one per 32-byte sector (the polling of all tiles
// then spreads over many L2 lines): epoch (30 bits) | flag (2 bits: 1
// aggregate, 2 inclusive) | value (32 bits).  The wait is bounded: past the
// limit the tile sets the timeout flag and goes on with what it has summed.
constexpr int STATUS_STRIDE = 4;

__device__ uint32_t warp_lookback(uint64_t* status, int64_t tile, uint32_t agg, uint64_t epoch, unsigned* flags)
{
    using ref = cuda::atomic_ref<uint64_t, cuda::thread_scope_device>;
    const int lane = threadIdx.x & 31;
    if(tile == 0) {
        if(lane == 0) ref(status[0]).store((epoch << 34) | (2ull << 32) | agg, cuda::memory_order_relaxed);
        return 0;
    }
    if(lane == 0) ref(status[tile * STATUS_STRIDE]).store((epoch << 34) | (1ull << 32) | agg, cuda::memory_order_relaxed);
    uint32_t excl = 0, spins = 0;
    int64_t j = tile - 1;
    for(;;) {
        const int64_t t = j - lane;
        uint64_t w = (epoch << 34) | (2ull << 32);          // before tile 0: an inclusive zero
        if(t >= 0) w = ref(status[t * STATUS_STRIDE]).load(cuda::memory_order_relaxed);
        const uint32_t fl = (w >> 34) == epoch ? (uint32_t)(w >> 32) & 3u : 0u;
        const unsigned pending = __ballot_sync(0xffffffffu, fl == 0);
        const unsigned incl = __ballot_sync(0xffffffffu, fl == 2);
        const int np = pending ? __ffs(pending) - 1 : 32;
        const int ni = incl ? __ffs(incl) - 1 : 32;
        const int take = ni < np ? ni + 1 : np;             // lanes 0 .. take - 1 count
        uint32_t v = lane < take ? (uint32_t)w : 0u;
#pragma unroll
        for(int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if(ni < np) break;
        j -= np;
        if(np == 0 && ++spins > mpm_sort::kSpinLimit) {
            if(lane == 0) atomicOr(flags, MPM_FLAG_TIMEOUT);
            break;
        }
    }
    if(lane == 0) ref(status[tile * STATUS_STRIDE]).store((epoch << 34) | (2ull << 32) | (excl + agg), cuda::memory_order_relaxed);
    return excl;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if(lane >= o) x += y;
    }
    return x;
}

// Work items (P2G and G2P): part k of the `parts` parts of a block, two uint4
// each, (block, k, parts, scene) and (block start, block count, 0, 0), so that
// a kernel needs no other load to begin an item.  CTAs take items by ticket
// (an atomic counter: CTAs that finish early take more) ahead of need: P2G
// starts on the item of its CTA index, then holds the next item's descriptor
// in flight and the ticket after it, so neither round trip falls between two
// items.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;"
                 :: "r"((uint32_t)__cvta_generic_to_shared(smem)), "l"(gmem) : "memory");
}

// Thread 0: start the copy of item w's descriptor into dst[0..1] (nothing past the last item).
__device__ __forceinline__ void work_prefetch(const FastArgs& a, uint32_t w, uint32_t nwork, uint4* dst)
{
    if(w < nwork) {
        cp_async16(dst, a.chunks + 2 * (size_t)w);
        cp_async16(dst + 1, a.chunks + 2 * (size_t)w + 1);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Thread 0: wait for the copy; past the last item dst holds the end mark.
__device__ __forceinline__ void work_arrive(uint32_t w, uint32_t nwork, uint4* dst)
{
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if(w >= nwork) dst[0] = make_uint4(SENTINEL, 0u, 0u, 0u);
}

// Tiles of BIN_TILE blocks of all scenes, one per CTA in launch order (a
// tile waits only on tiles of lower index, whose CTAs start first), BIN_PER
// consecutive blocks per thread: each block's arrivals and departures out of
// the domain, the exclusive prefix over all blocks (block ranges, tail slots
// of the departed), the active blocks and the work items (parts of at most
// a.part particles); for an active block its row of group offsets, from its
// row of arrival counts (loaded while the tile looks back, so that no tile
// publishes its aggregate late).  Consumed counts are zeroed for the next G2P.
constexpr int BIN_THREADS = 512, BIN_PER = 2, BIN_TILE = BIN_THREADS * BIN_PER;

__global__ void __launch_bounds__(BIN_THREADS) k_bins(FastArgs a)
{
    constexpr int NW = BIN_THREADS / 32;
    __shared__ uint32_t s_warp[NW][4];
    __shared__ uint32_t s_pre[4];         // prefixes of the tile: count, invalid (look-back); parts, active (bases)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t tile = blockIdx.x, ntiles = (a.nblk + BIN_TILE - 1) / BIN_TILE;
    const int64_t b0 = tile * BIN_TILE + threadIdx.x * BIN_PER;
    const uint64_t epoch = a.scan[0] & mpm_sort::kEpochMask;
    uint64_t* status = reinterpret_cast<uint64_t*>(a.scan + 8);
    uint32_t cnt[BIN_PER], inv[BIN_PER], sid[BIN_PER], v[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for(int u = 0; u < BIN_PER; u++) {
        const int64_t b = b0 + u;
        const unsigned long long c = b < a.nblk ? a.bcount[b] : 0ull;
        sid[u] = b < a.nblk ? a.block_scene[b] : 0u;
        cnt[u] = (uint32_t)c;
        inv[u] = (uint32_t)(c >> 32);
        v[0] += cnt[u];
        v[1] += inv[u];
        v[2] += cnt[u] ? (cnt[u] + a.part - 1) / a.part : 0u;
        v[3] += cnt[u] ? 1u : 0u;
    }
    uint32_t x[4];
#pragma unroll
    for(int q = 0; q < 4; q++) {
        x[q] = warp_incl_scan(v[q]);
        if(lane == 31) s_warp[warp][q] = x[q];
    }
    __syncthreads();
    if(warp == 0) {
#pragma unroll
        for(int q = 0; q < 4; q++) {
            const uint32_t t = lane < NW ? s_warp[lane][q] : 0u;
            const uint32_t ti = warp_incl_scan(t);
            if(lane < NW) s_warp[lane][q] = ti - t;                  // exclusive warp offset
            const uint32_t tot = __shfl_sync(0xffffffffu, ti, NW - 1);
            if(lane == 0) s_pre[q] = tot;                            // tile total, for now
        }
    }
    __syncthreads();
    uint32_t tot[4];
#pragma unroll
    for(int q = 0; q < 4; q++) tot[q] = s_pre[q];
    __syncthreads();
    if(warp == 0) {
        const uint32_t p = warp_lookback(status, tile, tot[0], epoch, a.flags);
        if(lane == 0) s_pre[0] = p;
    } else if(warp == 1) {
        const uint32_t p = warp_lookback(status + ntiles * STATUS_STRIDE, tile, tot[1], epoch, a.flags);
        if(lane == 0) s_pre[1] = p;
    } else if(threadIdx.x == 64) {
        s_pre[2] = tot[2] ? atomicAdd(&a.ctr[CNT_CHUNKS], tot[2]) : 0u;
        s_pre[3] = tot[3] ? atomicAdd(&a.ctr[CNT_ACTIVE_BLOCKS], tot[3]) : 0u;
    }
    // the arrival rows of the active blocks, as offsets within the block: the
    // groups in the order of their previous blocks (direction falling), then the far arrivals
    uint32_t rel[BIN_PER][28], nz[BIN_PER];
    bool consistent = true;
#pragma unroll
    for(int u = 0; u < BIN_PER; u++) nz[u] = 0u;
#pragma unroll
    for(int u = 0; u < BIN_PER; u++) {
        if(!cnt[u]) continue;
        const uint4* row = reinterpret_cast<const uint4*>(a.dcount + (size_t)(b0 + u) * ROW);
#pragma unroll
        for(int k = 0; k < 7; k++) {
            const uint4 r4 = row[k];
            rel[u][4 * k] = r4.x; rel[u][4 * k + 1] = r4.y; rel[u][4 * k + 2] = r4.z; rel[u][4 * k + 3] = r4.w;
        }
        uint32_t run = 0;
#pragma unroll
        for(int d = 26; d >= 0; d--) {
            const uint32_t c = rel[u][d];
            rel[u][d] = run;
            run += c;
            nz[u] |= (c ? 1u : 0u) << d;
        }
        consistent &= run + rel[u][DIR_FAR] == cnt[u];
        rel[u][DIR_FAR] = run;
    }
    if(!consistent) atomicOr(a.flags, MPM_FLAG_ORDER);   // counts out of step: report
    __syncthreads();
    if(tile == ntiles - 1 && threadIdx.x == 0) {
        a.ctr[CNT_ACTIVE_PARTICLES] = s_pre[0] + tot[0];
        a.ctr[CNT_NEW_INVALID] = s_pre[1] + tot[1];
    }
    uint32_t ex[4];
#pragma unroll
    for(int q = 0; q < 4; q++) ex[q] = s_pre[q] + s_warp[warp][q] + x[q] - v[q];
    // ranges, offset rows, work items and the active list
#pragma unroll
    for(int u = 0; u < BIN_PER; u++) {
        const int64_t b = b0 + u;
        if(!cnt[u] && !inv[u]) continue;
        a.bcount[b] = 0ull;
        if(!cnt[u]) {
            a.doff[(size_t)b * ROW + DIR_INVALID] = ex[1];
            ex[1] += inv[u];
            continue;
        }
        const uint32_t start = ex[0], parts = (cnt[u] + a.part - 1) / a.part;
        ex[0] += cnt[u];
        a.bstart[b] = start;
        a.bend[b] = start + cnt[u];
        // each group's offset into the row of the block it came from (b - delta(d), entry d)
        const SceneDev& sc = a.scenes[sid[u]];
        const int64_t sy = sc.NB[2], sx = (int64_t)sc.NB[1] * sc.NB[2];
#pragma unroll
        for(int d = 0; d < 27; d++)
            if((nz[u] >> d) & 1u)
                a.doff[(size_t)(b - dir_dx(d) * sx - dir_dy(d) * sy - dir_dz(d)) * ROW + d] = start + rel[u][d];
        a.doff[(size_t)b * ROW + DIR_FAR] = start + rel[u][DIR_FAR];
        if(inv[u]) a.doff[(size_t)b * ROW + DIR_INVALID] = ex[1];   // the departed's first tail slot
        ex[1] += inv[u];
        uint4* crow = reinterpret_cast<uint4*>(a.dcount + (size_t)b * ROW);
#pragma unroll
        for(int k = 0; k < 7; k++) crow[k] = make_uint4(0u, 0u, 0u, 0u);
        a.active[ex[3]++] = make_uint4((uint32_t)b, start, cnt[u], sid[u]);
        for(uint32_t k = 0; k < parts; k++, ex[2]++)
            if(ex[2] < a.chunk_cap) {
                a.chunks[2 * (size_t)ex[2]] = make_uint4((uint32_t)b, k, parts, sid[u]);
                a.chunks[2 * (size_t)ex[2] + 1] = make_uint4(start, cnt[u], 0u, 0u);
            }
    }
}

// Slot j of the current buffer to slot `dest` of the other (state, attributes,
// caller index, plastic state) with key `key`.
__device__ __forceinline__ void copy_slot(const FastArgs& a, uint32_t j, uint32_t dest, uint32_t key)
{
#pragma unroll 4
    for(int c = 0; c < NCOMP; c++) a.dst[c * a.npad + dest] = a.src[c * a.npad + j];
    a.dst_attr[dest] = a.src_attr[j];
    a.dst_pid[dest] = a.src_pid[j];
    if(a.psrc)
        for(int c = 0; c < a.nplas; c++) a.pdst[c * a.npad + dest] = a.psrc[c * a.npad + j];
    a.keys_next[dest] = key;
}

// Every slot of the current buffer to its place in the new order (perm[dest]
// = slot, sorted key).  Valid particles keep their state in place (P2G and
// G2P read it through perm); invalid ones are copied to their tail slot of
// the other buffer, which G2P does not write.
//
// A group of G warps per previous block, G (1, 2, 4 or 8) as large as keeps
// every block in flight at once: many blocks per SM when there are many, many
// warps per block when there are few.  Per batch, warp k of the group takes
// RW rounds of 32 consecutive slots (keys and the move directions G2P
// recorded, loaded together) after those of warps 0..k-1, counts each round's
// directions into its rows of shared memory and turns them into ranks; the
// group then offsets each warp's ranks by the counts of the warps before it
// and by the direction's next destination (first: entry d of the block's
// offset row, which k_bins wrote), so that ranks follow slot order.  The
// group synchronises on its own named barrier, never the whole CTA.
__global__ void __launch_bounds__(256) k_route(FastArgs a)
{
    constexpr int W = 8, RW = 4, CS = 33;       // warps per CTA, rounds per warp and batch, padded row
    __shared__ uint32_t s_cnt[W * RW][CS];      // per warp and round: count per direction, then rank
    __shared__ uint32_t s_tot[W][32];           // per warp: its batch's count per direction
    __shared__ uint32_t s_next[W][32];          // per group (its last warp): next destination per direction
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const uint32_t nold = a.octr[CNT_ACTIVE_BLOCKS], nvalid_old = a.octr[CNT_ACTIVE_PARTICLES];
    const uint32_t nvalid = a.ctr[CNT_ACTIVE_PARTICLES], ninv = a.ctr[CNT_NEW_INVALID];
    int G = 1;
    while(G < W && (uint64_t)nold * (uint64_t)(2 * G) <= (uint64_t)gridDim.x * W) G *= 2;
    const int gw = warp % G, g0 = warp - gw, last = g0 + G - 1;
    const uint32_t groups = gridDim.x * (uint32_t)(W / G);
    auto gsync = [&]() {
        if(G == 1) __syncwarp();
        else asm volatile("bar.sync %0, %1;" :: "r"(1 + warp / G), "r"(32 * G) : "memory");
    };
    for(uint32_t w = blockIdx.x * (uint32_t)(W / G) + (uint32_t)(warp / G); w < nold; w += groups) {
        const uint4 od = a.oactive[w];
        const uint32_t o = od.x, s = od.y, e = od.z != SENTINEL ? od.y + od.z : a.obend[o];
        if(warp == last) {   // lane d: the first destination of direction d (other entries are not read)
            const uint32_t first = a.doff[(size_t)o * ROW + lane];
            s_next[g0][lane] = lane == DIR_INVALID ? nvalid + first : first;
        }
        for(uint32_t jb = s; jb < e; jb += (uint32_t)(32 * RW * G)) {
            const uint32_t jw = jb + (uint32_t)(32 * RW * gw);
            uint32_t key[RW], intra[RW];
            int dr[RW];
#pragma unroll
            for(int r = 0; r < RW; r++) {
                const uint32_t j = jw + 32 * r + lane;
                key[r] = j < e ? a.keys_cur[j] : SENTINEL;
                dr[r] = j < e ? a.dir_cur[j] : 31;
                s_cnt[warp * RW + r][lane] = 0u;
            }
            __syncwarp();
#pragma unroll
            for(int r = 0; r < RW; r++) {
                const unsigned peers = __match_any_sync(0xffffffffu, dr[r]);
                intra[r] = __popc(peers & below);
                if(dr[r] != 31 && (__ffs(peers) - 1) == lane) s_cnt[warp * RW + r][dr[r]] = __popc(peers);
            }
            __syncwarp();
            uint32_t run = 0;                    // lane d: this warp's ranks of direction d
#pragma unroll
            for(int r = 0; r < RW; r++) {
                const uint32_t c = s_cnt[warp * RW + r][lane];
                s_cnt[warp * RW + r][lane] = run;
                run += c;
            }
            s_tot[warp][lane] = run;
            gsync();
            uint32_t base = s_next[g0][lane];
            for(int k = g0; k < warp; k++) base += s_tot[k][lane];
#pragma unroll
            for(int r = 0; r < RW; r++) s_cnt[warp * RW + r][lane] += base;
            __syncwarp();
#pragma unroll
            for(int r = 0; r < RW; r++) {
                const int d = dr[r];
                if(d == 31) continue;
                const uint32_t j = jw + 32 * r + lane;
                uint32_t dest;
                if(d == DIR_FAR) {
                    dest = atomicAdd(&a.doff[(size_t)(key[r] >> 6) * ROW + DIR_FAR], 1u);
                    atomicAdd(&a.ctr[CNT_FAR], 1u);
                } else dest = s_cnt[warp * RW + r][d] + intra[r];
                if(dest < a.n) {
                    if(d == DIR_INVALID) copy_slot(a, j, dest, SENTINEL);
                    a.perm[dest] = j;
                    a.sorted_keys[dest] = key[r];
                } else atomicOr(a.flags, MPM_FLAG_ORDER);   // counts out of step: report, write nothing
            }
            gsync();
            if(warp == last) s_next[g0][lane] = base + run;
        }
    }
    // the particles invalid before the last G2P follow, in slot order
    for(int64_t j = nvalid_old + blockIdx.x * 256ll + threadIdx.x; j < a.n; j += (int64_t)gridDim.x * 256) {
        const uint32_t dest = (uint32_t)(nvalid + ninv + (j - nvalid_old));
        if(dest >= a.n) {
            atomicOr(a.flags, MPM_FLAG_ORDER);
            break;
        }
        copy_slot(a, (uint32_t)j, dest, SENTINEL);
        a.perm[dest] = (uint32_t)j;
        a.sorted_keys[dest] = SENTINEL;
    }
    if(blockIdx.x == 0 && threadIdx.x == 0) a.scan[0] += 1u;   // the next block scan's epoch
}

// After a full radix sort of the current slots' keys (particles just set, or
// the autotuner's restore): the particles are copied to the other buffer in
// sorted order, and that order is recorded as the previous substep's (block
// ranges and active blocks into the given set, every particle counted as
// staying in its block), so the next substep's routing is the identity.
__global__ void k_prepare(FastArgs a, uint32_t* pbstart, uint32_t* pbend, uint4* pactive, uint32_t* pctr)
{
    const int lane = threadIdx.x & 31;
    const int64_t end = (a.n + 31) & ~(int64_t)31;      // whole warps stay in the loop
    for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < end; j += (int64_t)gridDim.x * blockDim.x) {
        const bool in = j < a.n;
        const uint32_t k = in ? a.sorted_keys[j] : SENTINEL;
        if(in) {
            copy_slot(a, a.perm[j], (uint32_t)j, k);
            a.dir_next[j] = k != SENTINEL ? (uint8_t)DIR_STAY : (uint8_t)DIR_INVALID;
        }
        const bool valid = k != SENTINEL;
        const uint32_t b = k >> 6;
        const unsigned peers = __match_any_sync(0xffffffffu, valid ? b : 0xffffffffu);
        if(valid && (__ffs(peers) - 1) == lane) {
            atomicAdd(&a.dcount[(size_t)b * ROW + DIR_STAY], (uint32_t)__popc(peers));
            atomicAdd(&a.bcount[b], (unsigned long long)__popc(peers));
        }
        if(!in) continue;
        const uint32_t kp = j ? a.sorted_keys[j - 1] : SENTINEL;
        if(!valid) {
            if(j == 0 || kp != SENTINEL) pctr[CNT_ACTIVE_PARTICLES] = (uint32_t)j;
            continue;
        }
        if(j == 0 || (kp >> 6) != b) {
            pbstart[b] = (uint32_t)j;
            pactive[atomicAdd(&pctr[CNT_ACTIVE_BLOCKS], 1u)] = make_uint4(b, (uint32_t)j, SENTINEL, a.block_scene[b]);
        }
        const uint32_t kn = j + 1 < a.n ? a.sorted_keys[j + 1] : SENTINEL;
        if(kn == SENTINEL || (kn >> 6) != b) pbend[b] = (uint32_t)(j + 1);
        if(j + 1 == a.n) pctr[CNT_ACTIVE_PARTICLES] = (uint32_t)a.n;
    }
}


// Every node quantity of a particle has the separable form (w = wx wy wz at
// node (i, j, k))
//   q_node = Hx[i] wy[j] wz[k] + wx[i] Hy[j] wz[k] + wx[i] wy[j] Hz[k]
// with, for momentum component r and axis a,
//   Ha[o] = wa[o] m B(r,a) Dinv_a (x_a(o) - X_a) - dt vol PF^T(r,a) wa'(o)
//           (+ wa[o] m V_r on the x axis),
// i.e. w m (V + B Dinv (x - X)) - dt vol PF^T grad w; mass is the same form
// with V_r = 1, B = 0 and PF^T = 0 (MPM_DRIVER::Particle_To_Grid,
// MPM_DRIVER.cpp:245-306, with MPM_FINITE_ELEMENTS::Add_Forces,
// MPM_FINITE_ELEMENTS.cpp:84-99, folded in as dt f).
struct PairSlot {
    float Hx[3], Hy[3], Hz[3];
};

__device__ __forceinline__ void pair_slot(const Axis<float>& wx, const Axis<float>& wy, const Axis<float>& wz,
    const float dX[3][3], float mV, const float mBD[3], const float S[3], PairSlot& q)
{
#pragma unroll
    for(int o = 0; o < 3; o++) {
        q.Hx[o] = wx.w[o] * fmaf(mBD[0], dX[0][o], mV) - S[0] * wx.dw[o];
        q.Hy[o] = wy.w[o] * (mBD[1] * dX[1][o]) - S[1] * wy.dw[o];
        q.Hz[o] = wz.w[o] * (mBD[2] * dX[2][o]) - S[2] * wz.dw[o];
    }
}

// Weights and separable factors of all four node quantities of the particle
// at sorted position j (mass: Hx = m wx, Hy = Hz = 0).  A particle whose
// stress needs the FP64 route is listed for p2g_finish and contributes
// mass and momentum here.
struct P2GFactors {
    float w[9];            // wx[3], wy[3], wz[3]
    float mwx[3];          // mass factor m wx
    PairSlot q[3];         // momentum components x, y, z
    int base[3];           // first stencil node - ghost, per axis
};

// Factors from a particle state held in registers (X, V, F, B, attributes);
// `j` is the sorted position recorded if the stress needs the FP64 route.
__device__ __forceinline__ void factors_from(const FastArgs& a, const SceneDev& sc, const float* X, const float* V,
    const float* F, const float* B, const float4 at, uint32_t j, P2GFactors& P, int model)
{
    float S[9];
    if(!stress_fast(model, F, at.z, at.w, S)) {
        a.fallback[atomicAdd(&a.ctr[CNT_FALLBACK], 1u)] = j;
#pragma unroll
        for(int r = 0; r < 9; r++) S[r] = 0.f;
    }
    const float sv = a.dt * at.y, m = at.x;
    const Axis<float> wx = spline_axis<float>(X[0], sc.dmin[0], sc.dx[0], sc.inv[0]);
    const Axis<float> wy = spline_axis<float>(X[1], sc.dmin[1], sc.dx[1], sc.inv[1]);
    const Axis<float> wz = spline_axis<float>(X[2], sc.dmin[2], sc.dx[2], sc.inv[2]);
    P.base[0] = wx.base; P.base[1] = wy.base; P.base[2] = wz.base;
    float dX[3][3];
    const float bx = (float)wx.base + 0.5f, by = (float)wy.base + 0.5f, bz = (float)wz.base + 0.5f;
#pragma unroll
    for(int o = 0; o < 3; o++) {
        dX[0][o] = sc.dmin[0] + (bx + (float)o) * sc.dx[0] - X[0];
        dX[1][o] = sc.dmin[1] + (by + (float)o) * sc.dx[1] - X[1];
        dX[2][o] = sc.dmin[2] + (bz + (float)o) * sc.dx[2] - X[2];
    }
    const float Dm[3] = {4.f * sc.inv[0] * sc.inv[0] * m, 4.f * sc.inv[1] * sc.inv[1] * m, 4.f * sc.inv[2] * sc.inv[2] * m};
#pragma unroll
    for(int r = 0; r < 3; r++) {
        const float mBD[3] = {B[r] * Dm[0], B[r + 3] * Dm[1], B[r + 6] * Dm[2]};
        const float Sr[3] = {S[r] * sv, S[r + 3] * sv, S[r + 6] * sv};
        pair_slot(wx, wy, wz, dX, m * V[r], mBD, Sr, P.q[r]);
    }
#pragma unroll
    for(int o = 0; o < 3; o++) {
        P.mwx[o] = m * wx.w[o];
        P.w[o] = wx.w[o]; P.w[3 + o] = wy.w[o]; P.w[6 + o] = wz.w[o];
    }
}

// i = perm[j], the slot of sorted position j (callers load it early).
__device__ __forceinline__ void particle_factors(const FastArgs& a, const SceneDev& sc, uint32_t j, uint32_t i, P2GFactors& P)
{
    float X[3], V[3], F[9], B[9];
#pragma unroll
    for(int r = 0; r < 3; r++) { X[r] = a.src[(C_X + r) * a.npad + i]; V[r] = a.vsrc[r * a.npad + i]; }
#pragma unroll
    for(int r = 0; r < 9; r++) { F[r] = a.src[(C_F + r) * a.npad + i]; B[r] = a.src[(C_B + r) * a.npad + i]; }
    factors_from(a, sc, X, V, F, B, a.src_attr[i], j, P, slot_model(a, sc, i));   // attributes: mass, volume, mu, lambda
}

// The 27 node values of one particle: f(ii, jj, kk, mass, px, py, pz).
template<class FN> __device__ __forceinline__ void factor_nodes(const P2GFactors& P, FN&& f)
{
#pragma unroll
    for(int ii = 0; ii < 3; ii++)
#pragma unroll
        for(int jj = 0; jj < 3; jj++) {
            const float wxy = P.w[ii] * P.w[3 + jj], mxy = P.mwx[ii] * P.w[3 + jj];
            float A[3];
#pragma unroll
            for(int r2 = 0; r2 < 3; r2++) A[r2] = fmaf(P.q[r2].Hx[ii], P.w[3 + jj], P.w[ii] * P.q[r2].Hy[jj]);
#pragma unroll
            for(int kk = 0; kk < 3; kk++) {
                const float wz = P.w[6 + kk];
                f(ii, jj, kk, mxy * wz, fmaf(A[0], wz, wxy * P.q[0].Hz[kk]), fmaf(A[1], wz, wxy * P.q[1].Hz[kk]),
                  fmaf(A[2], wz, wxy * P.q[2].Hz[kk]));
            }
        }
}

// The elastic force of the particles the P2G kernels listed for the FP64
// stress route: -dt vol PF^T grad w added to the momentum of their 27 nodes.
// Their nodes lie in their block's tile, whose node blocks P2G already
// marked.  The CTA of the P2G launch that finishes last does this, once every
// other CTA has listed its particles.  Inlined: an out-of-line call here made
// the whole P2G kernel keep a stack frame and move about 230 B per particle
// through local memory in its main loop (P2G 16 % slower at the headline).
__device__ __forceinline__ void p2g_fallback_force(const FastArgs& a, uint32_t k)
{
    const uint32_t j = a.fallback[k], i = a.perm[j];
    const SceneDev& sc = a.scenes[a.block_scene[a.sorted_keys[j] >> 6]];
    float X[3], F[9], S[9];
#pragma unroll
    for(int r = 0; r < 3; r++) X[r] = a.src[(C_X + r) * a.npad + i];
#pragma unroll
    for(int r = 0; r < 9; r++) F[r] = a.src[(C_F + r) * a.npad + i];
    const float4 at = a.src_attr[i];
    if(!stress_fp64(slot_model(a, sc, i), F, at.z, at.w, S)) atomicOr(a.flags, MPM_FLAG_NOT_CONVERGED);
    const float sv = a.dt * at.y;
    const Axis<float> wx = spline_axis<float>(X[0], sc.dmin[0], sc.dx[0], sc.inv[0]);
    const Axis<float> wy = spline_axis<float>(X[1], sc.dmin[1], sc.dx[1], sc.inv[1]);
    const Axis<float> wz = spline_axis<float>(X[2], sc.dmin[2], sc.dx[2], sc.inv[2]);
    for(int ii = 0; ii < 3; ii++)
        for(int jj = 0; jj < 3; jj++)
            for(int kk = 0; kk < 3; kk++) {
                const float g0 = wx.dw[ii] * wy.w[jj] * wz.w[kk], g1 = wx.w[ii] * wy.dw[jj] * wz.w[kk],
                            g2 = wx.w[ii] * wy.w[jj] * wz.dw[kk];
                float f[3];
#pragma unroll
                for(int r = 0; r < 3; r++) f[r] = -sv * (S[r] * g0 + S[r + 3] * g1 + S[r + 6] * g2);
                const int qx = wx.base + MPM_GHOST + ii, qy = wy.base + MPM_GHOST + jj, qz = wz.base + MPM_GHOST + kk;
                atomicAdd(&a.acc[node_index(sc, qx, qy, qz)], make_float4(f[0], f[1], f[2], 0.f));
            }
}

__device__ __forceinline__ void p2g_finish(const FastArgs& a, int* s_last)
{
    __syncthreads();
    if(threadIdx.x == 0) {
        __threadfence();
        *s_last = atomicAdd(&a.ctr[CNT_P2G_DONE], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if(!*s_last) return;
    __threadfence();
    const uint32_t count = *(volatile uint32_t*)&a.ctr[CNT_FALLBACK];
    for(uint32_t k = threadIdx.x; k < count; k += blockDim.x) p2g_fallback_force(a, k);
}

// Penalty collision objects (Apply_Particle_Forces, MPM_DRIVER.cpp:933-945):
// per slot of the current buffer, V + dt f / m with f the objects' force at X
// (penalty_particle in FP32).  P2G reads these velocities in place of V, so
// the node accumulator of momentum plus impulse gains dt sum_p w_ip f_p, the
// reference's scattered particle force times dt.
__global__ void k_penalty_kick(FastArgs a)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        float X[3], f[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for(int r = 0; r < 3; r++) X[r] = a.src[(C_X + r) * a.npad + i];
        penalty_particle<float, 3>(a.pen, a.npen, a.pen_k, a.pen_sep, X, f, (float*)nullptr);
        const float s = a.dt / a.src_attr[i].x;
#pragma unroll
        for(int r = 0; r < 3; r++) a.vkick[r * a.npad + i] = fmaf(s, f[r], a.src[(C_V + r) * a.npad + i]);
    }
}

// ---------------------------------------------------------------------------
// P2G (MPM_DRIVER::Particle_To_Grid, MPM_DRIVER.cpp:245-306, with
// MPM_FINITE_ELEMENTS::Add_Forces, MPM_FINITE_ELEMENTS.cpp:84-99, folded in as
// dt f): one work item is part k of a block, the particles bstart + k,
// bstart + k + parts, ... (a strided part samples every cell of the block),
// one thread per particle.
//
// The part's node values are summed in a shared tile of fixed-point
// integers: shared-memory integer adds run at three times the rate of float
// adds to shared memory, and integer sums do not depend on their order.  Each
// quantity (mass, momentum x, y, z) has its own power-of-two scale, chosen
// after every particle of the part has bounded its largest node value: the
// bounds' sum B maps below 2^21, so no node sum can overflow.  A contribution
// goes in as its nearest integer plus its rounding residual in units of 2^-23
// (a second 32-bit sum: at most 256 residuals of at most 2^22), both formed by
// float adds rather than conversion instructions, so a node keeps B 2^-45
// absolutely: nodes that only the edges of a few stencils reach, with masses
// many orders below the part's, keep their velocities to FP32 accuracy.  The
// tile goes out as floats (hi + lo 2^-23 combined in FP64) with one float4
// atomic per touched node.
//
// Lanes must hit different nodes in each shared add, so the part's particles
// are first binned by cell and handed out round by round (round r: the
// (r+1)-th particle of every cell that has one), cells in index order.
// ---------------------------------------------------------------------------
template<int T> struct P2GSmem {
    int q[4][PTN];                        // fixed-point tile: mass, momentum x, y, z (units of 1 / scale)
    int ql[4][PTN];                       // the rounding residuals, units of 2^-22 / scale
    uint32_t ccount[64];                  // particles per cell of the part
    uint32_t rsize[T];                    // particles in round r
    uint32_t roff[T];                     // first list position of round r
    unsigned long long rmask[T];          // cells with more than r particles
    uint32_t list[T];                     // the part's sorted positions, round by round
    float bound[4];
    float scale[4];
    int maxc;
    int scene;
    uint4 work[2][2];                     // this item's descriptor and the next one's
    SceneDev sc;
};

// Largest |node value| of a particle over its 27 nodes, per quantity.
__device__ __forceinline__ void factor_bounds(const P2GFactors& P, float* bnd)
{
    const float mx = fmaxf(P.w[0], fmaxf(P.w[1], P.w[2]));
    const float my = fmaxf(P.w[3], fmaxf(P.w[4], P.w[5]));
    const float mz = fmaxf(P.w[6], fmaxf(P.w[7], P.w[8]));
    bnd[0] = fmaxf(P.mwx[0], fmaxf(P.mwx[1], P.mwx[2])) * my * mz;
#pragma unroll
    for(int r = 0; r < 3; r++) {
        const PairSlot& s = P.q[r];
        const float hx = fmaxf(fabsf(s.Hx[0]), fmaxf(fabsf(s.Hx[1]), fabsf(s.Hx[2])));
        const float hy = fmaxf(fabsf(s.Hy[0]), fmaxf(fabsf(s.Hy[1]), fabsf(s.Hy[2])));
        const float hz = fmaxf(fabsf(s.Hz[0]), fmaxf(fabsf(s.Hz[1]), fabsf(s.Hz[2])));
        bnd[1 + r] = hx * my * mz + mx * hy * mz + mx * my * hz;
    }
}

// The factors of a particle in shared memory, one array of T per value (so the
// thread that reads slot t reads consecutive words).
constexpr int NFAC = 39;   // w[9], mass factor m wx[3], momentum Hx, Hy, Hz of x, y, z

constexpr float kRoundMagic = 12582912.f;       // 1.5 2^23
constexpr int kRoundMagicBits = 0x4B400000;     // its bit pattern

__device__ __forceinline__ void store_factors(float* FS, int T, int pos, const P2GFactors& P)
{
#pragma unroll
    for(int e = 0; e < 9; e++) FS[e * T + pos] = P.w[e];
#pragma unroll
    for(int o = 0; o < 3; o++) FS[(9 + o) * T + pos] = P.mwx[o];
#pragma unroll
    for(int r = 0; r < 3; r++)
#pragma unroll
        for(int o = 0; o < 3; o++) {
            FS[(12 + 9 * r + o) * T + pos] = P.q[r].Hx[o];
            FS[(15 + 9 * r + o) * T + pos] = P.q[r].Hy[o];
            FS[(18 + 9 * r + o) * T + pos] = P.q[r].Hz[o];
        }
}

__device__ __forceinline__ void load_factors(const float* FS, int T, int pos, P2GFactors& P)
{
#pragma unroll
    for(int e = 0; e < 9; e++) P.w[e] = FS[e * T + pos];
#pragma unroll
    for(int o = 0; o < 3; o++) P.mwx[o] = FS[(9 + o) * T + pos];
#pragma unroll
    for(int r = 0; r < 3; r++)
#pragma unroll
        for(int o = 0; o < 3; o++) {
            P.q[r].Hx[o] = FS[(12 + 9 * r + o) * T + pos];
            P.q[r].Hy[o] = FS[(15 + 9 * r + o) * T + pos];
            P.q[r].Hz[o] = FS[(18 + 9 * r + o) * T + pos];
        }
}

// Each thread first prepares the particle its own slot of the part holds
// (loads through perm stay close to consecutive), then the factors move
// through shared memory to the thread of the particle's place in the
// round-by-round cell order, which adds them to the tile.
template<int T> __global__ void __launch_bounds__(T, 768 / T) k_p2g(FastArgs a)
{
    constexpr int NW = T / 32;
    __shared__ P2GSmem<T> S;
    extern __shared__ __align__(16) float FS[];    // NFAC x T factors, in place order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nwork = min(a.ctr[CNT_CHUNKS], a.chunk_cap);
    // thread 0: this item and the next; the first item by CTA index (every CTA
    // starts on one), later ones by ticket
    uint32_t w = 0, wnext = 0;
    if(threadIdx.x == 0) {
        S.scene = -1;
        w = blockIdx.x;
        work_prefetch(a, w, nwork, S.work[0]);
        wnext = gridDim.x + atomicAdd(&a.ctr[CNT_P2G_WORK], 1u);
    }
    for(int cur = 0;; cur ^= 1) {
        __syncthreads();
        if(threadIdx.x == 0) {
            work_arrive(w, nwork, S.work[cur]);
            work_prefetch(a, wnext, nwork, S.work[cur ^ 1]);
            w = wnext;
            wnext = gridDim.x + atomicAdd(&a.ctr[CNT_P2G_WORK], 1u);
            S.maxc = 0;
        }
        for(int t = threadIdx.x; t < 4 * PTN; t += T) { (&S.q[0][0])[t] = 0; (&S.ql[0][0])[t] = 0; }
        if(threadIdx.x < 64) S.ccount[threadIdx.x] = 0u;
        if(threadIdx.x < 4) S.bound[threadIdx.x] = 0.f;
        __syncthreads();
        const uint4 wk = S.work[cur][0], wr = S.work[cur][1];
        if(wk.x == SENTINEL) break;
        const uint32_t b = wk.x, part = wk.y, parts = wk.z;
        const int sid = (int)wk.w;
        if(sid != S.scene) stage_scene(a, sid, &S.sc);
        const uint32_t s = wr.x, e = wr.x + wr.y;
        const uint32_t cnt = e - s > part ? min((e - s - part + parts - 1) / parts, (uint32_t)T) : 0u;
        // this thread's slot of the (strided) part: cell, rank in its cell, factors, bounds
        const bool mine = threadIdx.x < cnt;
        uint32_t cell = 0, r = 0;
        float bnd[4] = {0.f, 0.f, 0.f, 0.f};
        P2GFactors P;
        uint32_t slot = 0;
        if(mine) {   // the slot with the key: one round trip before the particle loads, not two
            const uint32_t j = s + part + threadIdx.x * parts;
            cell = a.sorted_keys[j] & 63u;
            slot = a.perm[j];
            r = atomicAdd(&S.ccount[cell], 1u);
        }
        __syncthreads();
        if(threadIdx.x == 0) S.scene = sid;
        // the block's 8 node blocks for the grid update: flags exchanged now,
        // first touches listed after the flush (the round trip overlaps the item)
        uint32_t nb = 0, nb_prev = 1;
        if(threadIdx.x >= T - 8) {
            const int o = threadIdx.x - (T - 8);
            int bx, by, bz;
            block_coords(S.sc, b - S.sc.block_base, bx, by, bz);
            nb = S.sc.nb_base + ((uint32_t)(bx + (o >> 2)) * S.sc.NN[1] + by + ((o >> 1) & 1)) * S.sc.NN[2] + bz + (o & 1);
            nb_prev = atomicExch(&a.nb_flag[nb], 1u);
        }
        // the part's rounds: every warp reduces the 64 cell counts itself (no
        // barrier) and writes the masks of its rounds
        const uint32_t cc0 = S.ccount[lane], cc1 = S.ccount[lane + 32];
        uint32_t mc = max(cc0, cc1);
#pragma unroll
        for(int o = 16; o; o >>= 1) mc = max(mc, __shfl_xor_sync(0xffffffffu, mc, o));
        const int maxc = (int)mc;
        for(int rr = warp; rr < maxc; rr += NW) {
            const unsigned lo = __ballot_sync(0xffffffffu, cc0 > (uint32_t)rr);
            const unsigned hi = __ballot_sync(0xffffffffu, cc1 > (uint32_t)rr);
            if(lane == 0) {
                S.rmask[rr] = lo | ((unsigned long long)hi << 32);
                S.rsize[rr] = __popc(lo) + __popc(hi);
            }
        }
        if(mine) {
            particle_factors(a, S.sc, s + part + threadIdx.x * parts, slot, P);
            factor_bounds(P, bnd);
        }
#pragma unroll
        for(int q = 0; q < 4; q++) {
            float v = bnd[q];
#pragma unroll
            for(int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if(lane == 0 && v != 0.f) atomicAdd(&S.bound[q], v);
        }
        __syncthreads();
        if(threadIdx.x >= T - 4) {   // the scale of each quantity
            const int q = threadIdx.x - (T - 4);
            const float B = S.bound[q];
            float sc = 0.f;
            if(!isfinite(B)) atomicOr(a.flags, MPM_FLAG_NAN);
            else if(B > 0.f) {
                int ex;
                frexpf(B, &ex);                      // B < 2^ex
                sc = ldexpf(1.f, 21 - max(ex, -90));
            }
            S.scale[q] = sc;
        }
        if(warp == 0) {   // exclusive scan of the round sizes
            uint32_t carry = 0;
            for(int r0 = 0; r0 < maxc; r0 += 32) {
                const uint32_t x = r0 + lane < maxc ? S.rsize[r0 + lane] : 0u;
                const uint32_t xi = warp_incl_scan(x);
                if(r0 + lane < maxc) S.roff[r0 + lane] = carry + xi - x;
                carry += __shfl_sync(0xffffffffu, xi, 31);
            }
        }
        __syncthreads();
        if(mine) {
            const int pos = (int)(S.roff[r] + __popcll(S.rmask[r] & ((1ull << cell) - 1ull)));
            store_factors(FS, T, pos, P);
            S.list[pos] = cell;
        }
        __syncthreads();
        if(mine) {   // the particle at place threadIdx.x of the round-by-round order
            load_factors(FS, T, threadIdx.x, P);
            const int pc = (int)S.list[threadIdx.x];
            const float s0 = S.scale[0], s1 = S.scale[1], s2 = S.scale[2], s3 = S.scale[3];
            const int t0 = ptile(pc >> 4, (pc >> 2) & 3, pc & 3);
            // y = rint(y) + residual, both as integers without a conversion
            // instruction: for |x| <= 2^22, x + 1.5 2^23 rounds x to an integer
            // held in the low mantissa bits (|y| < 2^21 by the scale; the
            // residual, |y - rint(y)| <= 1/2, goes in units of 2^-23, and
            // y - rint(y) is exact in float)
            auto add = [&](int q, int t, float y) {
                const float m1 = y + kRoundMagic;
                const float r = y - (m1 - kRoundMagic);
                atomicAdd(&S.q[q][t], __float_as_int(m1) - kRoundMagicBits);
                atomicAdd(&S.ql[q][t], __float_as_int(fmaf(r, 8388608.f, kRoundMagic)) - kRoundMagicBits);
            };
            factor_nodes(P, [&](int ii, int jj, int kk, float m, float px, float py, float pz) {
                const int t = t0 + ptile(ii, jj, kk);
                add(0, t, m * s0);
                add(1, t, px * s1);
                add(2, t, py * s2);
                add(3, t, pz * s3);
            });
        }
        __syncthreads();
        // out: one float4 atomic per touched node, and the node blocks for the grid update
        const SceneDev& sc = S.sc;
        int bx, by, bz;
        block_coords(sc, b - sc.block_base, bx, by, bz);
        double inv[4];
#pragma unroll
        for(int q = 0; q < 4; q++) inv[q] = S.scale[q] > 0.f ? 1.0 / S.scale[q] : 0.0;
        for(int t = threadIdx.x; t < TN; t += T) {
            const int tx = t / (TE * TE), ty = (t / TE) % TE, tz = t % TE, u = ptile(tx, ty, tz);
            float v[4];
            bool any = false;
#pragma unroll
            for(int q = 0; q < 4; q++) {
                const int hi = S.q[q][u], lo = S.ql[q][u];
                any |= (hi | lo) != 0;
                v[q] = (float)(((double)hi + (double)lo * 1.1920928955078125e-07) * inv[q]);
            }
            if(any)
                atomicAdd(&a.acc[node_index(sc, 4 * bx + tx, 4 * by + ty, 4 * bz + tz)], make_float4(v[1], v[2], v[3], v[0]));
        }
        if(nb_prev == 0u) a.nb_list[atomicAdd(&a.ctr[CNT_NODE_BLOCKS], 1u)] = nb;
    }
    p2g_finish(a, &S.maxc);
}

// ---------------------------------------------------------------------------
// P2G by lane groups: a work item is a contiguous part of a block (at most
// 4 T particles for T threads), binned by cell in shared memory; groups of 4
// lanes walk balanced ranges of the cell-sorted part.  Per round each lane of
// a group prepares one particle (stress, weights, the separable factors of
// all four node quantities); in four rotating sub-steps lane k takes from the
// group's lane (k + p) mod 4 that particle's weights and the factors of
// quantity k (mass, momentum x, y, z) and adds its 27 node values into 27
// registers.  A lane writes its registers to the shared float tile only when
// its particles move to another cell, so a cell of ~8 particles costs 27
// shared atomics per quantity instead of 27 per particle; the tile goes out
// with one float4 atomic per touched node.
// ---------------------------------------------------------------------------
template<int T> struct P2GGroupSmem {
    float q[4][PTN];                      // node sums: mass, momentum + dt force x, y, z
    uint32_t ccount[64], cstart[64];
    uint32_t list[4 * T];                 // the part's sorted positions, cell by cell
    uint8_t lcell[4 * T];
    int scene;
    uint4 work[2][2];                     // this item's descriptor and the next one's
};

// The 9 separable factors of quantity `qn` (0 mass, 1-3 momentum) of P.
__device__ __forceinline__ void quantity_factors(const P2GFactors& P, int qn, float* h)
{
#pragma unroll
    for(int o = 0; o < 3; o++) {
        const float m = P.mwx[o];
        const float x0 = P.q[0].Hx[o], x1 = P.q[1].Hx[o], x2 = P.q[2].Hx[o];
        const float y0 = P.q[0].Hy[o], y1 = P.q[1].Hy[o], y2 = P.q[2].Hy[o];
        const float z0 = P.q[0].Hz[o], z1 = P.q[1].Hz[o], z2 = P.q[2].Hz[o];
        h[o] = qn == 0 ? m : (qn == 1 ? x0 : (qn == 2 ? x1 : x2));
        h[3 + o] = qn == 0 ? 0.f : (qn == 1 ? y0 : (qn == 2 ? y1 : y2));
        h[6 + o] = qn == 0 ? 0.f : (qn == 1 ? z0 : (qn == 2 ? z1 : z2));
    }
}

template<int T> __global__ void __launch_bounds__(T, 512 / T) k_p2g_groups(FastArgs a)
{
    constexpr int G = T / 4;              // lane groups
    __shared__ P2GGroupSmem<T> S;
    __shared__ SceneDev s_sc;
    const int lane = threadIdx.x & 31, k = threadIdx.x & 3, g = threadIdx.x >> 2;
    const unsigned gmask = 0xfu << (lane & ~3);
    const uint32_t nwork = min(a.ctr[CNT_CHUNKS], a.chunk_cap);
    // thread 0: this item and the next; the first item by CTA index (every CTA
    // starts on one), later ones by ticket
    uint32_t w = 0, wnext = 0;
    if(threadIdx.x == 0) {
        S.scene = -1;
        w = blockIdx.x;
        work_prefetch(a, w, nwork, S.work[0]);
        wnext = gridDim.x + atomicAdd(&a.ctr[CNT_P2G_WORK], 1u);
    }
    for(int cur = 0;; cur ^= 1) {
        __syncthreads();
        if(threadIdx.x == 0) {
            work_arrive(w, nwork, S.work[cur]);
            work_prefetch(a, wnext, nwork, S.work[cur ^ 1]);
            w = wnext;
            wnext = gridDim.x + atomicAdd(&a.ctr[CNT_P2G_WORK], 1u);
        }
        for(int t = threadIdx.x; t < 4 * PTN; t += T) (&S.q[0][0])[t] = 0.f;
        if(threadIdx.x < 64) S.ccount[threadIdx.x] = 0u;
        __syncthreads();
        const uint4 wk = S.work[cur][0], wr = S.work[cur][1];
        if(wk.x == SENTINEL) break;
        const uint32_t b = wk.x, part = wk.y, parts = wk.z;
        const int sid = (int)wk.w;
        if(sid != S.scene) stage_scene(a, sid, &s_sc);
        const uint32_t s = wr.x, c = wr.y;
        const uint32_t j0 = s + (uint32_t)((uint64_t)c * part / parts);
        const uint32_t cnt = min((uint32_t)((uint64_t)c * (part + 1) / parts) + s - j0, (uint32_t)(4 * T));
        // bin by cell: up to 4 particles per thread
        uint32_t cl[4], rk[4];
#pragma unroll
        for(int u = 0; u < 4; u++) {
            const uint32_t i = threadIdx.x + u * T;
            cl[u] = i < cnt ? a.sorted_keys[j0 + i] & 63u : 0u;
            rk[u] = i < cnt ? atomicAdd(&S.ccount[cl[u]], 1u) : 0u;
        }
        __syncthreads();
        if(threadIdx.x == 0) S.scene = sid;
        // the block's 8 node blocks for the grid update: flags exchanged now,
        // first touches listed after the flush (the round trip overlaps the item)
        uint32_t nb = 0, nb_prev = 1;
        if(threadIdx.x >= T - 8) {
            const int o = threadIdx.x - (T - 8);
            int bx, by, bz;
            block_coords(s_sc, b - s_sc.block_base, bx, by, bz);
            nb = s_sc.nb_base + ((uint32_t)(bx + (o >> 2)) * s_sc.NN[1] + by + ((o >> 1) & 1)) * s_sc.NN[2] + bz + (o & 1);
            nb_prev = atomicExch(&a.nb_flag[nb], 1u);
        }
        if(threadIdx.x < 32) {   // exclusive scan of the 64 cell counts
            const uint32_t c0 = S.ccount[2 * lane], c1 = S.ccount[2 * lane + 1];
            const uint32_t x = warp_incl_scan(c0 + c1);
            S.cstart[2 * lane] = x - c0 - c1;
            S.cstart[2 * lane + 1] = x - c1;
        }
        __syncthreads();
#pragma unroll
        for(int u = 0; u < 4; u++) {
            const uint32_t i = threadIdx.x + u * T;
            if(i < cnt) {
                const uint32_t pos = S.cstart[cl[u]] + rk[u];
                S.list[pos] = j0 + i;
                S.lcell[pos] = (uint8_t)cl[u];
            }
        }
        __syncthreads();
        // this group's balanced range of the cell-sorted part
        const uint32_t r0 = (uint32_t)((uint64_t)cnt * g / G), r1 = (uint32_t)((uint64_t)cnt * (g + 1) / G);
        const SceneDev& sc = s_sc;
        float acc[27];
#pragma unroll
        for(int q = 0; q < 27; q++) acc[q] = 0.f;
        int cell = -1;
        float* const tq = S.q[k];
        auto flush = [&]() {
            const int t0 = ptile(cell >> 4, (cell >> 2) & 3, cell & 3);
#pragma unroll
            for(int q = 0; q < 27; q++) {
                atomicAdd(&tq[t0 + ptile(q / 9, (q / 3) % 3, q % 3)], acc[q]);
                acc[q] = 0.f;
            }
        };
        for(uint32_t rb = r0; rb < r1; rb += 4) {   // a round: one particle per lane of the group
            const uint32_t mine = rb + k;
            P2GFactors P;
            int pc = -1;
            if(mine < r1) {
                pc = S.lcell[mine];
                particle_factors(a, sc, S.list[mine], a.perm[S.list[mine]], P);
            } else {
#pragma unroll
                for(int e = 0; e < 9; e++) P.w[e] = 0.f;
#pragma unroll
                for(int o = 0; o < 3; o++) {
                    P.mwx[o] = 0.f;
#pragma unroll
                    for(int r = 0; r < 3; r++) P.q[r].Hx[o] = P.q[r].Hy[o] = P.q[r].Hz[o] = 0.f;
                }
            }
#pragma unroll
            for(int p = 0; p < 4; p++) {
                // lane k reads lane (k + p) mod 4, which sends the factors of quantity (its index - p) mod 4
                const int src = (lane & ~3) | ((k + p) & 3);
                float h[9];
                quantity_factors(P, (k - p) & 3, h);
                float w[9], f[9];
#pragma unroll
                for(int e = 0; e < 9; e++) {
                    w[e] = __shfl_sync(gmask, P.w[e], src);
                    f[e] = __shfl_sync(gmask, h[e], src);
                }
                const int rc = __shfl_sync(gmask, pc, src);
                if(rc < 0) continue;                  // past the group's range
                if(rc != cell) {
                    if(cell >= 0) flush();
                    cell = rc;
                }
                // node (i, j, l): Hx[i] wy[j] wz[l] + wx[i] Hy[j] wz[l] + wx[i] wy[j] Hz[l]
#pragma unroll
                for(int ii = 0; ii < 3; ii++)
#pragma unroll
                    for(int jj = 0; jj < 3; jj++) {
                        const float wxy = w[ii] * w[3 + jj];
                        const float A = fmaf(f[ii], w[3 + jj], w[ii] * f[3 + jj]);
#pragma unroll
                        for(int ll = 0; ll < 3; ll++) {
                            const int q = (ii * 3 + jj) * 3 + ll;
                            acc[q] = fmaf(A, w[6 + ll], fmaf(wxy, f[6 + ll], acc[q]));
                        }
                    }
            }
        }
        if(cell >= 0) flush();
        __syncthreads();
        // out: one float4 atomic per touched node, and the node blocks for the grid update
        int bx, by, bz;
        block_coords(sc, b - sc.block_base, bx, by, bz);
        for(int t = threadIdx.x; t < TN; t += T) {
            const int tx = t / (TE * TE), ty = (t / TE) % TE, tz = t % TE, u = ptile(tx, ty, tz);
            const float m = S.q[0][u];
            if(m != 0.f)
                atomicAdd(&a.acc[node_index(sc, 4 * bx + tx, 4 * by + ty, 4 * bz + tz)],
                          make_float4(S.q[1][u], S.q[2][u], S.q[3][u], m));
        }
        if(nb_prev == 0u) a.nb_list[atomicAdd(&a.ctr[CNT_NODE_BLOCKS], 1u)] = nb;
    }
    __shared__ int s_last;
    p2g_finish(a, &s_last);
}

// One thread per node of the listed node blocks (4^3 nodes each, 64
// consecutive threads), grid-stride with CTA-uniform trip counts.  Each group
// of 64 threads (one node block) copies its scene record and collision
// objects into shared memory before use; a one-scene handle does that once
// per CTA.  Nodes within reach of an object are collided in FP64
// (collide_node).
__global__ void __launch_bounds__(256) k_grid(FastArgs a)
{
    constexpr int kGroups = 4;   // node blocks per CTA pass
    __shared__ SceneDev s_sc[kGroups];
    __shared__ DevObject s_obj[kGroups][MPM_MAX_OBJECTS];
    __shared__ int s_scene[kGroups];
    const int grp = threadIdx.x >> 6, t = threadIdx.x & 63;
    const uint64_t total = (uint64_t)a.ctr[CNT_NODE_BLOCKS] * 64u;
    const uint64_t stride = (uint64_t)gridDim.x * 256u;
    if(threadIdx.x < kGroups) s_scene[threadIdx.x] = -1;
    __syncthreads();
    for(uint64_t g0 = blockIdx.x * 256ull; g0 < total; g0 += stride) {
        const uint64_t g = g0 + threadIdx.x;
        const bool live = g < total;
        const uint32_t nb = live ? a.nb_list[g >> 6] : 0u;
        const int scene = live ? (int)a.nb_scene[nb] : s_scene[grp];
        // restage when this group's scene changed (all 64 threads agree)
        if(scene != s_scene[grp] && scene >= 0) {
            constexpr int words = (int)(sizeof(SceneDev) / 4);
            if(t < words) ((uint32_t*)&s_sc[grp])[t] = ((const uint32_t*)(a.scenes + scene))[t];
            const SceneDev& gs = a.scenes[scene];
            if(t < gs.nobj) s_obj[grp][t] = a.objs[gs.obj_begin + t];
        }
        __syncthreads();
        if(t == 0 && live) s_scene[grp] = scene;
        if(live) {
            const SceneDev& sc = s_sc[grp];
            const uint32_t lnb = nb - sc.nb_base;
            int nz = lnb % sc.NN[2], r = lnb / sc.NN[2], ny = r % sc.NN[1], nx = r / sc.NN[1];
            int qx = 4 * nx + (t >> 4), qy = 4 * ny + ((t >> 2) & 3), qz = 4 * nz + (t & 3);
            int64_t q = node_index(sc, qx, qy, qz);
            float4 c = a.acc[q];
            float4 o0 = make_float4(0, 0, 0, 0), o1 = make_float4(0, 0, 0, 0);
            if(c.w != 0.f) {
                float im = 1.f / c.w;
                float V[3] = {c.x * im + a.dt * sc.gravity[0], c.y * im + a.dt * sc.gravity[1], c.z * im + a.dt * sc.gravity[2]};
                float vn[3], vf[3];
                if(sc.nobj) {
                    float X0[3] = {sc.dmin[0] + ((float)(qx - MPM_GHOST) + 0.5f) * sc.dx[0],
                                   sc.dmin[1] + ((float)(qy - MPM_GHOST) + 0.5f) * sc.dx[1],
                                   sc.dmin[2] + ((float)(qz - MPM_GHOST) + 0.5f) * sc.dx[2]};
                    float zero[3] = {0.f, 0.f, 0.f};
                    collide_node<float, 3>(s_obj[grp], sc.nobj, X0, zero, V, a.dt, vn, vf, a.motion, a.moving);
                } else {
#pragma unroll
                    for(int k = 0; k < 3; k++) vn[k] = vf[k] = V[k];
                }
                o0 = make_float4(vn[0], vn[1], vn[2], vf[0]);
                o1 = make_float4(vf[1], vf[2], c.w, 0.f);
                a.acc[q] = make_float4(0, 0, 0, 0);
            }
            a.vel[2 * q] = o0;
            a.vel[2 * q + 1] = o1;
            if(t == 0) a.nb_flag[nb] = 0u;
        }
        __syncthreads();
    }
}

// G2P, one thread per particle in sorted order (coalesced).  The tile of
// (v_new, v_fric) is copied to shared memory by TMA; the sums over the 27 nodes are
// taken separably (z first, then y, then x), so each node costs two 16-byte
// shared loads and twelve FMAs:
//   V' = sum w vn,  G = sum vn g^T,  Vf = sum w vf,  Bv = sum w vf (Z - X)^T.
// The antisymmetric part of the reference's B (MPM_DRIVER.cpp:482-485,503-508),
//   dt/2 [sum w (vf vn^T - vn vf^T) - (Vf V'^T - V' Vf^T)],
// is non-zero only where the grid update changed v_fric against v_new (nodes
// that met a collision object), so it is summed only for tiles holding such
// nodes.
// G2P of the particle at sorted position j against the staged tile `tv`
// (origin node (ox, oy, oz)): writes its new state to slot j of the other
// buffer and its next key; also returns it in `out`.
struct G2PState {
    float xn[3], Vf[3], Fn[9], Bn[9];
    float4 at;
    uint32_t key;
    bool ok;
};

// MPM_DRIVER::Update_Plasticity_And_Hardening (MPM_DRIVER.cpp:922-928) with
// MPM_PLASTICITY_CLAMP through the SVD, for the particle already written to
// slot j (F, Fp and the Lame parameters rewritten in place).  Out of line and
// fed from memory, so that neither its registers nor a stack copy of its
// operands weigh on the G2P loop; G2P calls it only where the SVD-free form
// below does not apply (det F <= 0 or sigma_max / sigma_min > 10).
__device__ __noinline__ void plastic_svd_slot(float* dst, float* pdst, float4* dst_attr, int64_t npad, uint32_t j,
    float tc, float ts, float mh, float hf, unsigned* flags)
{
    float F[9], Fp[9];
    for(int k = 0; k < 9; k++) { F[k] = dst[(C_F + k) * npad + j]; Fp[k] = pdst[k * npad + j]; }
    float4 at = dst_attr[j];
    const float prm[4] = {tc, ts, mh, hf};
    bool ok;
    float mu = at.z, la = at.w;
    if(plastic_clamp<float, 3>(F, Fp, mu, la, pdst[9 * npad + j], pdst[10 * npad + j], prm, ok)) {
        for(int k = 0; k < 9; k++) { dst[(C_F + k) * npad + j] = F[k]; pdst[k * npad + j] = Fp[k]; }
        at.z = mu;
        at.w = la;
        dst_attr[j] = at;
    }
    if(!ok) atomicOr(flags, MPM_FLAG_NOT_CONVERGED);
}

// True when every singular value of F lies strictly inside the clamp band
// [1 - theta_c, 1 + theta_s] with a relative margin of 1e-5 and det F > 0:
// the clamp then leaves F, Fp, mu and lambda unchanged, so the SVD is skipped.
// Test: C - a I and b I - C positive definite (LDL^T pivots > 0) for
// C = F^T F, a = (1 - theta_c)^2 (1 + 1e-5), b = (1 + theta_s)^2 (1 - 1e-5).
// FP32 rounding in C and in the pivots is ~1e-7, well inside the margin.
__device__ __forceinline__ bool pd3(float m00, float m01, float m02, float m11, float m12, float m22)
{
    if(!(m00 > 0.f)) return false;
    const float i0 = __fdividef(1.f, m00);
    const float d1 = m11 - m01 * m01 * i0;
    if(!(d1 > 0.f)) return false;
    const float e12 = m12 - m01 * m02 * i0;
    return m22 - m02 * m02 * i0 - __fdividef(e12 * e12, d1) > 0.f;
}

__device__ __forceinline__ bool clamp_inactive(const float* F, const float* prm)
{
    const float J = F[0] * (F[4] * F[8] - F[7] * F[5]) - F[3] * (F[1] * F[8] - F[7] * F[2]) + F[6] * (F[1] * F[5] - F[4] * F[2]);
    if(!(J > 0.f)) return false;
    float c[6];   // C = F^T F: 00 01 02 11 12 22
    const int I[6] = {0, 0, 0, 1, 1, 2}, K[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for(int e = 0; e < 6; e++)
        c[e] = F[3 * I[e]] * F[3 * K[e]] + F[3 * I[e] + 1] * F[3 * K[e] + 1] + F[3 * I[e] + 2] * F[3 * K[e] + 2];
    const float lo = 1.f - prm[0], hi = 1.f + prm[1];
    const float a = lo * lo * (1.f + 1e-5f), b = hi * hi * (1.f - 1e-5f);
    return pd3(c[0] - a, c[1], c[2], c[3] - a, c[4], c[5] - a) && pd3(b - c[0], -c[1], -c[2], b - c[3], -c[4], b - c[5]);
}

// The clamp without an SVD, for det F > 0 and sigma_min / sigma_max > 0.1.
// With F = U S V^T (det U = det V = 1) and S' the clamped singular values,
// the reference's updates only need V and S (U^T F = S V^T):
//   F  <- U S' V^T       = F  (V diag(S'/S) V^T)
//   Fp <- V S'^-1 U^T F Fp = (V diag(S/S') V^T) Fp
// V diag(S^2) V^T is the eigensystem of C = F^T F (sym_eig3f).  Both matrix
// functions depend only on C, so they are stable for repeated singular values
// (and the Drucker-Prager strain, an isotropic function of S, keeps that).
// plastic_eig / plastic_dp_eig return 0 (unchanged), 1 (projected) or -1
// (outside the conditions above: the caller takes the SVD route).
// Singular values S and right singular vectors V of F from the eigensystem of
// F^T F (sym_eig3f); false where det F <= 0 or sigma_max / sigma_min > 10 (the
// caller takes the SVD route).
__device__ __forceinline__ bool ftf_eig(const float* F, float* S, float (&V)[3][3])
{
    const float J = F[0] * (F[4] * F[8] - F[7] * F[5]) - F[3] * (F[1] * F[8] - F[7] * F[2]) + F[6] * (F[1] * F[5] - F[4] * F[2]);
    if(!(J > 0.f)) return false;
    float A[3][3];
#pragma unroll
    for(int i = 0; i < 3; i++)
#pragma unroll
        for(int k = 0; k < 3; k++) A[i][k] = F[3 * i] * F[3 * k] + F[3 * i + 1] * F[3 * k + 1] + F[3 * i + 2] * F[3 * k + 2];
    sym_eig3f(A, V);
    const float lmax = fmaxf(A[0][0], fmaxf(A[1][1], A[2][2])), lmin = fminf(A[0][0], fminf(A[1][1], A[2][2]));
    if(!(lmin > 1e-2f * lmax)) return false;
#pragma unroll
    for(int i = 0; i < 3; i++) S[i] = sqrtf(A[i][i]);
    return true;
}

// F <- U St V^T = F (V diag(St/S) V^T),  Fp <- V St^-1 U^T F Fp = (V diag(S/St) V^T) Fp.
__device__ __forceinline__ void apply_strain(float* F, float* Fp, const float* S, const float* St, const float (&V)[3][3])
{
    float g[3], h[3];
#pragma unroll
    for(int i = 0; i < 3; i++) { g[i] = __fdividef(St[i], S[i]); h[i] = __fdividef(S[i], St[i]); }
    float M[3][3], N[3][3];
#pragma unroll
    for(int j = 0; j < 3; j++)
#pragma unroll
        for(int k = 0; k < 3; k++) {
            M[j][k] = V[j][0] * g[0] * V[k][0] + V[j][1] * g[1] * V[k][1] + V[j][2] * g[2] * V[k][2];
            N[j][k] = V[j][0] * h[0] * V[k][0] + V[j][1] * h[1] * V[k][1] + V[j][2] * h[2] * V[k][2];
        }
    float Fo[9], Po[9];
#pragma unroll
    for(int k = 0; k < 9; k++) { Fo[k] = F[k]; Po[k] = Fp[k]; }
#pragma unroll
    for(int r = 0; r < 3; r++)
#pragma unroll
        for(int c = 0; c < 3; c++) {
            F[r + 3 * c] = Fo[r] * M[0][c] + Fo[r + 3] * M[1][c] + Fo[r + 6] * M[2][c];
            Fp[r + 3 * c] = N[r][0] * Po[3 * c] + N[r][1] * Po[3 * c + 1] + N[r][2] * Po[3 * c + 2];
        }
}

__device__ __forceinline__ int plastic_eig(float* F, float* Fp, float4& at, float mu0, float la0, const float* prm)
{
    float S[3], V[3][3];
    if(!ftf_eig(F, S, V)) return -1;
    const float lo = 1.f - prm[0], hi = 1.f + prm[1];
    float St[3];
    bool same = true;
#pragma unroll
    for(int i = 0; i < 3; i++) {
        St[i] = fminf(fmaxf(S[i], lo), hi);
        same = same && St[i] == S[i];
    }
    if(same) return 0;
    const float* P = Fp;
    const float detp = P[0] * (P[4] * P[8] - P[7] * P[5]) - P[3] * (P[1] * P[8] - P[7] * P[2]) + P[6] * (P[1] * P[5] - P[4] * P[2]);
    const float e = prm[3] * (1.f - S[0] * S[1] * S[2] / (St[0] * St[1] * St[2]) * detp);
    const float coeff = fmaxf(expf(fminf(e, prm[2])), 1e-8f);
    at.z = mu0 * coeff;
    at.w = la0 * coeff;
    apply_strain(F, Fp, S, St, V);
    return 1;
}

// Drucker-Prager by the same SVD-free route (det F > 0, well conditioned):
// the return mapping on S, then F and Fp as for the clamp.  `st` = plastic_def,
// rho_F, sigma_Y, vc, updated in place.  Returns 0 (elastic), 1 or -1.
__device__ __forceinline__ int plastic_dp_eig(float* F, float* Fp, float mu, float la, float* st, const float* prm)
{
    float S[3], V[3][3], strain[3];
    if(!ftf_eig(F, S, V)) return -1;
    if(!dp_strain<float, 3>(S, mu, la, st[0], st[1], st[2], st[3], prm, strain)) return 0;
    apply_strain(F, Fp, S, strain, V);
    return 1;
}

// The Drucker-Prager update through the SVD for the particle already written
// to slot j, out of line and fed from memory (as plastic_svd_slot).
__device__ __noinline__ void plastic_dp_svd_slot(float* dst, float* pdst, const float4* dst_attr, int64_t npad, uint32_t j,
    float a0, float a1, float a3, float a4, float use_vc, unsigned* flags)
{
    float F[9], Fp[9], st[4];
    for(int k = 0; k < 9; k++) { F[k] = dst[(C_F + k) * npad + j]; Fp[k] = pdst[k * npad + j]; }
    for(int k = 0; k < 4; k++) st[k] = pdst[(9 + k) * npad + j];
    const float4 at = dst_attr[j];
    const float prm[5] = {a0, a1, a3, a4, use_vc};
    bool ok;
    if(plastic_dp<float, 3>(F, Fp, at.z, at.w, st, prm, ok)) {
        for(int k = 0; k < 9; k++) { dst[(C_F + k) * npad + j] = F[k]; pdst[k * npad + j] = Fp[k]; }
    }
    for(int k = 0; k < 4; k++) pdst[(9 + k) * npad + j] = st[k];
    if(!ok) atomicOr(flags, MPM_FLAG_NOT_CONVERGED);
}

// PK: the plasticity fused after the update (0 none, 1 clamp, 2 Drucker-Prager).
template<int PK>
__device__ __forceinline__ void g2p_particle(const FastArgs& a, const SceneDev& sc, const float4* tv, bool anti,
    int ox, int oy, int oz, uint32_t j, G2PState& out)
{
    const float dt = a.dt;
    const uint32_t i = a.perm[j];
    float X[3], F[9];
#pragma unroll
    for(int k = 0; k < 3; k++) X[k] = a.src[(C_X + k) * a.npad + i];
#pragma unroll
    for(int k = 0; k < 9; k++) F[k] = a.src[(C_F + k) * a.npad + i];
    float4 at = a.src_attr[i];
    const int pid = a.src_pid[i];
    Axis<float> wx = spline_axis<float>(X[0], sc.dmin[0], sc.dx[0], sc.inv[0]);
    Axis<float> wy = spline_axis<float>(X[1], sc.dmin[1], sc.dx[1], sc.inv[1]);
    Axis<float> wz = spline_axis<float>(X[2], sc.dmin[2], sc.dx[2], sc.inv[2]);
    const int t0 = ((wx.base + MPM_GHOST - ox) * TE + (wy.base + MPM_GHOST - oy)) * TE + (wz.base + MPM_GHOST - oz);
    float dX[3], dY[3], wzd[3];
#pragma unroll
    for(int o = 0; o < 3; o++) {
        dX[o] = sc.dmin[0] + ((float)(wx.base + o) + 0.5f) * sc.dx[0] - X[0];
        dY[o] = sc.dmin[1] + ((float)(wy.base + o) + 0.5f) * sc.dx[1] - X[1];
        wzd[o] = wz.w[o] * (sc.dmin[2] + ((float)(wz.base + o) + 0.5f) * sc.dx[2] - X[2]);
    }
    float* const Vf = out.Vf;
    Vf[0] = Vf[1] = Vf[2] = 0.f;
    float Vp[3] = {0, 0, 0}, G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Bv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    float K01 = 0, K02 = 0, K12 = 0;
#pragma unroll
    for(int ii = 0; ii < 3; ii++)
#pragma unroll
        for(int jj = 0; jj < 3; jj++) {
            float Sw[3] = {0, 0, 0}, Sd[3] = {0, 0, 0}, Tw[3] = {0, 0, 0}, Td[3] = {0, 0, 0};
            float k01 = 0, k02 = 0, k12 = 0;
#pragma unroll
            for(int kk = 0; kk < 3; kk++) {
                const int t = t0 + (ii * TE + jj) * TE + kk;
                const float4 p0 = tv[2 * t], p1 = tv[2 * t + 1];
                const float vn[3] = {p0.x, p0.y, p0.z}, vf[3] = {p0.w, p1.x, p1.y};
#pragma unroll
                for(int r = 0; r < 3; r++) {
                    Sw[r] += vn[r] * wz.w[kk];
                    Sd[r] += vn[r] * wz.dw[kk];
                    Tw[r] += vf[r] * wz.w[kk];
                    Td[r] += vf[r] * wzd[kk];
                }
                if(anti) {
                    k01 += wz.w[kk] * (vf[0] * vn[1] - vf[1] * vn[0]);
                    k02 += wz.w[kk] * (vf[0] * vn[2] - vf[2] * vn[0]);
                    k12 += wz.w[kk] * (vf[1] * vn[2] - vf[2] * vn[1]);
                }
            }
            const float wxy = wx.w[ii] * wy.w[jj], gx0 = wx.dw[ii] * wy.w[jj], gy0 = wx.w[ii] * wy.dw[jj];
            K01 += wxy * k01;
            K02 += wxy * k02;
            K12 += wxy * k12;
            const float wxX = wxy * dX[ii], wxY = wxy * dY[jj];
#pragma unroll
            for(int r = 0; r < 3; r++) {
                Vp[r] += wxy * Sw[r];
                G[r] += gx0 * Sw[r];
                G[r + 3] += gy0 * Sw[r];
                G[r + 6] += wxy * Sd[r];
                Vf[r] += wxy * Tw[r];
                Bv[r] += wxX * Tw[r];
                Bv[r + 3] += wxY * Tw[r];
                Bv[r + 6] += wxy * Td[r];
            }
        }
    // F <- (I + dt grad v) F
    float* const Fn = out.Fn;
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
        for(int r = 0; r < 3; r++)
            Fn[r + 3 * c] = F[r + 3 * c] + dt * (G[r] * F[3 * c] + G[r + 3] * F[3 * c + 1] + G[r + 6] * F[3 * c + 2]);
    float* const xn = out.xn;
#pragma unroll
    for(int k = 0; k < 3; k++) xn[k] = X[k] + dt * Vp[k];
    const float h = 0.5f * dt;
    const float A01 = h * (K01 - (Vf[0] * Vp[1] - Vp[0] * Vf[1]));
    const float A02 = h * (K02 - (Vf[0] * Vp[2] - Vp[0] * Vf[2]));
    const float A12 = h * (K12 - (Vf[1] * Vp[2] - Vp[1] * Vf[2]));
    const float Bn[9] = {Bv[0], Bv[1] - A01, Bv[2] - A02,
                         Bv[3] + A01, Bv[4], Bv[5] - A12,
                         Bv[6] + A02, Bv[7] + A12, Bv[8]};
    bool ok = true;
#pragma unroll
    for(int k = 0; k < 3; k++) {
        float eps = FLT_EPSILON * 4.f * (sc.dmax[k] - sc.dmin[k]);
        if(!(xn[k] >= sc.dmin[k] + eps && xn[k] <= sc.dmax[k] - eps)) ok = false;
    }
    bool finite = true;
#pragma unroll
    for(int k = 0; k < 9; k++) finite = finite && isfinite(Fn[k]);
    finite = finite && isfinite(xn[0]) && isfinite(xn[1]) && isfinite(xn[2]);
    if(!finite) { atomicOr(a.flags, MPM_FLAG_NAN); ok = false; }
    bool svd = false;
    if(PK) {
        // every particle of this substep, including one that just left
        float Fp[9], st[4];
#pragma unroll
        for(int k = 0; k < 9; k++) Fp[k] = a.psrc[k * a.npad + i];
#pragma unroll
        for(int k = 0; k < (PK == 1 ? 2 : 4); k++) st[k] = a.psrc[(9 + k) * a.npad + i];
        const bool on = !a.pmask || a.pmask[pid];   // the plasticity's own particles
        if(PK == 1)   // st = mu0, lambda0
            svd = on && finite && !clamp_inactive(Fn, a.prm) && plastic_eig(Fn, Fp, at, st[0], st[1], a.prm) < 0;
        else
            svd = on && finite && plastic_dp_eig(Fn, Fp, at.z, at.w, st, a.prm) < 0;
#pragma unroll
        for(int k = 0; k < 9; k++) a.pdst[k * a.npad + j] = Fp[k];
#pragma unroll
        for(int k = 0; k < (PK == 1 ? 2 : 4); k++) a.pdst[(9 + k) * a.npad + j] = st[k];
    }
    const uint32_t key = ok ? cell_key(sc, xn) : SENTINEL;
#pragma unroll
    for(int k = 0; k < 3; k++) { a.dst[(C_X + k) * a.npad + j] = xn[k]; a.dst[(C_V + k) * a.npad + j] = Vf[k]; }
#pragma unroll
    for(int k = 0; k < 9; k++) { a.dst[(C_F + k) * a.npad + j] = Fn[k]; a.dst[(C_B + k) * a.npad + j] = Bn[k]; }
    a.dst_attr[j] = at;
    a.dst_pid[j] = pid;
    a.keys_next[j] = key;
    if(PK == 1 && svd)
        plastic_svd_slot(a.dst, a.pdst, a.dst_attr, a.npad, j, a.prm[0], a.prm[1], a.prm[2], a.prm[3], a.flags);
    if(PK == 2 && svd)
        plastic_dp_svd_slot(a.dst, a.pdst, a.dst_attr, a.npad, j, a.prm[0], a.prm[1], a.prm[2], a.prm[3], a.prm[4], a.flags);
#pragma unroll
    for(int k = 0; k < 9; k++) out.Bn[k] = Bn[k];
    out.at = at;
    out.key = key;
    out.ok = ok;
}

// ---------------------------------------------------------------------------
// G2P tiles by TMA.  Every scene's grid of (v_new, v_fric, mass) nodes, 8
// floats each, is described by a 4D tensor map {8 floats, z, y, x} over this
// GPU's own grid allocation (fast_setup_scenes encodes one per scene); a
// work item's 6^3-node tile is one cp.async.bulk.tensor copy into shared
// memory, completing on an mbarrier.  The copy of the next work item's tile
// is issued before the current item is computed (two tile buffers), so its
// latency hides behind the current particles' gather and arithmetic.
// ---------------------------------------------------------------------------
constexpr uint32_t TILE_BYTES = TN * 32;   // 6^3 nodes x 8 floats

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void fence_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done != 0;
}

// Bounded wait for phase `parity` of `bar`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    for(uint32_t spin = 0; spin < mpm_sort::kSpinLimit; spin++)
        if(mbar_try_wait(bar, parity)) return true;
    return false;
}

// One tile: box {8, 6, 6, 6} at node (ox, oy, oz) of the scene's map, into `dst`
// (128-byte aligned shared memory), completing `bar`'s current phase.
__device__ __forceinline__ void tma_tile(float4* dst, const CUtensorMap* map, uint64_t* bar, int ox, int oy, int oz)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %4, %5, %6}], [%2];"
                 :: "r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(0), "r"(oz), "r"(oy), "r"(ox)
                 : "memory");
}

// Thread 0: the next work item's descriptor into work[0..1] and its tile copy
// into `dst` started; returns whether there is such an item.
__device__ __forceinline__ bool g2p_take(const FastArgs& a, uint32_t nwork, uint4* work, float4* dst, uint64_t* bar)
{
    const uint32_t w = atomicAdd(&a.ctr[CNT_G2P_WORK], 1u);
    if(w >= nwork) {
        work[0] = make_uint4(SENTINEL, 0u, 0u, 0u);
        return false;
    }
    const uint4 wk = a.chunks[2 * (size_t)w], wr = a.chunks[2 * (size_t)w + 1];
    const SceneDev& sc = a.scenes[wk.w];
    int bx, by, bz;
    block_coords(sc, wk.x - sc.block_base, bx, by, bz);
    fence_async_shared();   // the CTA's reads of this buffer come before the copy's writes
    mbar_expect_tx(bar, TILE_BYTES);
    tma_tile(dst, a.tmaps + wk.w, bar, 4 * bx, 4 * by, 4 * bz);
    work[0] = wk;
    work[1] = wr;
    return true;
}

template<int THREADS, int PK> __global__ void __launch_bounds__(THREADS) k_g2p(FastArgs a)
{
    // the previous order's counters are read by nothing after the routing: they
    // become the next substep's, cleared here (no memset node between substeps)
    if(blockIdx.x == 0 && threadIdx.x < CNT_COUNT) a.nctr[threadIdx.x] = 0u;
    __shared__ alignas(128) float4 tv[2][2 * TN];
    __shared__ alignas(8) uint64_t s_bar[2];
    __shared__ uint4 s_work[2][2];
    __shared__ int s_scene;
    __shared__ SceneDev s_sc;
    // where this part's particles go next substep: per direction (k_bins, k_route)
    __shared__ uint32_t s_dc[32];
    const int lane = threadIdx.x & 31;
    const uint32_t nwork = min(a.ctr[CNT_CHUNKS], a.chunk_cap);
    if(threadIdx.x < 32) s_dc[threadIdx.x] = 0u;
    if(threadIdx.x == 0) {
        s_scene = -1;
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        fence_async_shared();
        g2p_take(a, nwork, s_work[0], tv[0], &s_bar[0]);
    }
    __syncthreads();
    uint32_t issued = 1u;               // bit b: a copy into buffer b is in flight (thread 0's view)
    bool failed = false;
    for(int k = 0;; k++) {
        const int buf = k & 1;
        const uint4 wk = s_work[buf][0], wr = s_work[buf][1];
        if(wk.x == SENTINEL) break;
        if(threadIdx.x == 0) {          // the next item's tile copy, overlapping this item
            const bool more = g2p_take(a, nwork, s_work[buf ^ 1], tv[buf ^ 1], &s_bar[buf ^ 1]);
            issued = (issued & ~(1u << buf)) | (more ? 1u << (buf ^ 1) : 0u);
        }
        const uint32_t b = wk.x, part = wk.y, parts = wk.z;
        const int sid = (int)wk.w;
        if(sid != s_scene) {
            stage_scene(a, sid, &s_sc);
            __syncthreads();
            if(threadIdx.x == 0) s_scene = sid;
        }
        const SceneDev& sc = s_sc;
        int bx, by, bz;
        block_coords(sc, b - sc.block_base, bx, by, bz);
        const int ox = 4 * bx, oy = 4 * by, oz = 4 * bz;
        // the tile: wait for its copy, then note nodes whose friction velocity differs
        const bool arrived = mbar_wait(&s_bar[buf], (uint32_t)(k >> 1) & 1u);
        int differs = 0;
        const float4* t4 = tv[buf];
        for(int t = threadIdx.x; t < TN; t += THREADS) {
            const float4 p0 = t4[2 * t], p1 = t4[2 * t + 1];
            differs |= (p0.w != p0.x) | (p1.x != p0.y) | (p1.y != p0.z);
        }
        if(__syncthreads_or(!arrived)) {
            failed = true;
            break;
        }
        const bool anti = __syncthreads_or(differs) != 0;
        // a contiguous part of the block (coalesced slots)
        const uint32_t s = wr.x, c = wr.y;
        const uint32_t j0 = s + (uint32_t)((uint64_t)c * part / parts), j1 = s + (uint32_t)((uint64_t)c * (part + 1) / parts);
        for(uint32_t j = j0 + threadIdx.x; j < j1; j += THREADS) {
            G2PState o;
            g2p_particle<PK>(a, sc, t4, anti, ox, oy, oz, j, o);
            const int d = key_dir(sc, b, bx, by, bz, o.key);
            a.dir_next[j] = (uint8_t)d;
            if(d == DIR_FAR) {
                atomicAdd(&a.dcount[(size_t)(o.key >> 6) * ROW + DIR_FAR], 1u);
                atomicAdd(&a.bcount[o.key >> 6], 1ull);
            }
            const unsigned act = __activemask();
            const unsigned peers = __match_any_sync(act, d);
            if((__ffs(peers) - 1) == lane) atomicAdd(&s_dc[d], (uint32_t)__popc(peers));
        }
        __syncthreads();
        if(threadIdx.x < NDIR) {
            const int d = threadIdx.x;
            const uint32_t c2 = s_dc[d];
            if(c2 && d == DIR_INVALID) atomicAdd(&a.bcount[b], (unsigned long long)c2 << 32);
            else if(c2 && d != DIR_FAR) {   // the neighbour block they moved to: block + delta(d)
                const uint32_t nb = b + ((dir_dx(d) * sc.NB[1]) + dir_dy(d)) * sc.NB[2] + dir_dz(d);
                atomicAdd(&a.dcount[(size_t)nb * ROW + d], c2);
                atomicAdd(&a.bcount[nb], (unsigned long long)c2);
            }
            s_dc[d] = 0u;
        }
    }
    if(threadIdx.x == 0) {
        if(failed) atomicOr(a.flags, MPM_FLAG_TIMEOUT);
        // copies still in flight land before the CTA's shared memory goes away
        for(int bb = 0; bb < 2; bb++)
            if(failed && ((issued >> bb) & 1u)) mbar_wait(&s_bar[bb], 0u), mbar_wait(&s_bar[bb], 1u);
    }
}

// Reference layout <-> sorted SoA
template<class T> __global__ void k_scatter_in(FastArgs a, const T* X, const T* V, const T* F, const T* B, const T* m,
    const T* vol, const T* mu, const T* la, const uint8_t* valid, uint8_t* valid_slot)
{
    for(int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
        float* d = a.dst;
        for(int k = 0; k < 3; k++) { d[(C_X + k) * a.npad + p] = (float)X[p * 3 + k]; d[(C_V + k) * a.npad + p] = (float)V[p * 3 + k]; }
        for(int k = 0; k < 9; k++) { d[(C_F + k) * a.npad + p] = (float)F[p * 9 + k]; d[(C_B + k) * a.npad + p] = (float)B[p * 9 + k]; }
        a.dst_attr[p] = make_float4((float)m[p], (float)vol[p], (float)mu[p], (float)la[p]);
        a.dst_pid[p] = (int)p;
        valid_slot[p] = valid ? valid[p] : 1;
    }
}

template<class T> __global__ void k_gather_out(FastArgs a, const uint32_t* keys, T* X, T* V, T* F, T* B, uint8_t* valid)
{
    for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < a.n; j += (int64_t)gridDim.x * blockDim.x) {
        int p = a.src_pid[j];
        const float* s = a.src;
        for(int k = 0; k < 3; k++) {
            if(X) X[(int64_t)p * 3 + k] = (T)s[(C_X + k) * a.npad + j];
            if(V) V[(int64_t)p * 3 + k] = (T)s[(C_V + k) * a.npad + j];
        }
        for(int k = 0; k < 9; k++) {
            if(F) F[(int64_t)p * 9 + k] = (T)s[(C_F + k) * a.npad + j];
            if(B) B[(int64_t)p * 9 + k] = (T)s[(C_B + k) * a.npad + j];
        }
        if(valid) valid[p] = keys[j] != SENTINEL;
    }
}

// Plastic state of the current buffer: unplastic start (Fp = I, mu0 = mu,
// lambda0 = lambda), and exchange with the caller's particle order.
__global__ void k_plastic_init(int64_t n, int64_t npad, float* P, const float4* attr)
{
    for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for(int k = 0; k < 9; k++) P[k * npad + j] = k % 4 == 0 ? 1.f : 0.f;
        const float4 at = attr[j];
        P[9 * npad + j] = at.z;
        P[10 * npad + j] = at.w;
    }
}

// Drucker-Prager start (MPM_DRUCKER_PRAGER::Initialize_Particles): Fp = I,
// plastic_def = vc = 0, sigma_Y = cohesion, rho_F at zero plastic deformation.
// Particles outside `mask` (by caller index `pid`) keep the arrays' zero state.
__global__ void k_dp_init(int64_t n, int64_t npad, float* P, float cohesion, float a0, float a1, float a3, float a4,
    const int* pid, const uint8_t* mask)
{
    const float prm[5] = {a0, a1, a3, a4, 0.f};
    float q = 0.f, rho = 0.f;
    dp_hardening<float>(q, rho, 0.f, prm);
    for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const bool on = !mask || mask[pid[j]];
#pragma unroll
        for(int k = 0; k < 9; k++) P[k * npad + j] = k % 4 == 0 ? 1.f : 0.f;
        P[9 * npad + j] = on ? q : 0.f;
        P[10 * npad + j] = on ? rho : 0.f;
        P[11 * npad + j] = on ? cohesion : 0.f;
        P[12 * npad + j] = 0.f;
    }
}

// Caller-order arrays of the plastic state: Fp, the Lame parameters (in the
// attributes) and the per-particle scalars at plastic components 9, 10, ...
template<class T> struct PlasticArrays {
    T* Fp;
    T* mu;
    T* la;
    T* sc[4];
};

template<class T> __global__ void k_plastic_out(int64_t n, int64_t npad, const float* P, const float4* attr, const int* pid,
    PlasticArrays<T> o)
{
    for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = pid[j];
        if(o.Fp)
            for(int k = 0; k < 9; k++) o.Fp[p * 9 + k] = (T)P[k * npad + j];
        if(o.mu) o.mu[p] = (T)attr[j].z;
        if(o.la) o.la[p] = (T)attr[j].w;
        for(int k = 0; k < 4; k++)
            if(o.sc[k]) o.sc[k][p] = (T)P[(9 + k) * npad + j];
    }
}

template<class T> __global__ void k_plastic_in(int64_t n, int64_t npad, float* P, float4* attr, const int* pid,
    PlasticArrays<T> in)
{
    for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = pid[j];
        if(in.Fp)
            for(int k = 0; k < 9; k++) P[k * npad + j] = (float)in.Fp[p * 9 + k];
        if(in.mu) attr[j].z = (float)in.mu[p];
        if(in.la) attr[j].w = (float)in.la[p];
        for(int k = 0; k < 4; k++)
            if(in.sc[k]) P[(9 + k) * npad + j] = (float)in.sc[k][p];
    }
}

// Grids of scene `s` in the reference's ghosted layout: the node blocks of the
// last substep's list that belong to the scene.
__global__ void k_grid_out(FastArgs a, const uint32_t* list, uint32_t count, int s, double* m, double* v, double* vf,
    int G0, int G1, int G2)
{
    const SceneDev& sc = a.scenes[s];
    for(uint32_t w = blockIdx.x; w < count; w += gridDim.x) {
        if(a.nb_scene[list[w]] != s) continue;
        uint32_t nb = list[w] - sc.nb_base;
        int nz = nb % sc.NN[2], r = nb / sc.NN[2], ny = r % sc.NN[1], nx = r / sc.NN[1];
        int t = threadIdx.x;
        int qx = 4 * nx + (t >> 4), qy = 4 * ny + ((t >> 2) & 3), qz = 4 * nz + (t & 3);
        if(qx >= G0 || qy >= G1 || qz >= G2) continue;
        int64_t q = node_index(sc, qx, qy, qz);
        int64_t o = ((int64_t)qx * G1 + qy) * G2 + qz;
        float4 p0 = a.vel[2 * q], p1 = a.vel[2 * q + 1];
        if(m) m[o] = p1.z;
        if(v) { v[3 * o] = p0.x; v[3 * o + 1] = p0.y; v[3 * o + 2] = p0.z; }
        if(vf) { vf[3 * o] = p0.w; vf[3 * o + 1] = p1.x; vf[3 * o + 2] = p1.y; }
    }
}

__global__ void k_count_keys(const uint32_t* keys, int64_t n, unsigned long long* out)
{
    unsigned long long c = 0;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) c += keys[i] != SENTINEL;
    atomicAdd(out, c);
}

FastArgs make_args(mpm_handle* h, double dt)
{
    FastArgs a;
    FastState& f = h->fast;
    a.n = f.n;
    a.npad = f.npad;
    int c = f.cur, o = 1 - f.cur;
    a.src = f.soa[c]; a.src_attr = f.attr[c]; a.src_pid = f.pid[c];
    a.dst = f.soa[o]; a.dst_attr = f.attr[o]; a.dst_pid = f.pid[o];
    a.perm = f.perm;
    a.sorted_keys = f.sorted_keys;
    a.keys_cur = f.keys[c];
    a.keys_next = f.keys[o];
    a.dir_cur = f.dirs[c];
    a.dir_next = f.dirs[o];
    // this substep's order is set c, the previous substep's set o
    a.bstart = f.bstart[c]; a.bend = f.bend[c]; a.active = f.active[c]; a.chunks = f.chunks[c];
    a.ctr = f.counters ? f.counters + CNT_COUNT * c : nullptr;
    a.obstart = f.bstart[o]; a.obend = f.bend[o]; a.oactive = f.active[o];
    a.octr = f.counters ? f.counters + CNT_COUNT * o : nullptr;
    a.nctr = f.counters ? f.counters + CNT_COUNT * o : nullptr;
    a.dcount = f.dcount; a.doff = f.doff; a.bcount = f.bcount; a.scan = f.scan;
    a.nblk = f.total_blocks;
    a.part = kPartSize[f.route_variant];
    a.chunk_cap = (uint32_t)f.chunk_cap;
    a.nb_flag = f.nb_flag; a.nb_list = f.nb_list;
    a.acc = f.acc; a.vel = f.vel;
    a.fallback = f.sort_keys_alt;   // the full sort's ping-pong buffer is free during substeps
    a.tmaps = (const CUtensorMap*)f.tmaps;
    a.scenes = f.scenes; a.block_scene = f.block_scene; a.nb_scene = f.nb_scene; a.pbase = f.pbase;
    a.objs = f.objs;
    a.nscenes = f.nscenes;
    a.pen = h->pen_f;
    a.npen = h->pen_f && f.vkick ? h->sp.npen : 0;
    a.pen_k = (float)h->sp.pen_stiffness;
    a.pen_sep = (float)h->sp.pen_separation;
    a.vkick = f.vkick;
    a.pmodel = f.pmodel;
    a.pmask = f.pmask;
    a.motion = h->motion_dev_f;
    a.moving = h->motion_dev_f ? h->moving : 0u;
    a.vsrc = a.npen ? f.vkick : a.src + (size_t)C_V * a.npad;
    a.dt = (float)dt;
    a.flags = h->d_flags;
    const bool plastic = h->plastic.kind != MPM_PLASTICITY_NONE && f.plas[0];
    a.psrc = plastic ? f.plas[c] : nullptr;
    a.pdst = plastic ? f.plas[o] : nullptr;
    const mpm_plasticity_desc& pl = h->plastic;
    a.pkind = pl.kind;
    a.nplas = pl.kind == MPM_PLASTICITY_CLAMP ? 11 : 13;
    if(pl.kind == MPM_PLASTICITY_DRUCKER_PRAGER) {
        a.prm[0] = (float)pl.dp_a0; a.prm[1] = (float)pl.dp_a1; a.prm[2] = (float)pl.dp_a3; a.prm[3] = (float)pl.dp_a4;
        a.prm[4] = pl.use_vc ? 1.f : 0.f;
    } else {
        a.prm[0] = (float)pl.theta_c; a.prm[1] = (float)pl.theta_s; a.prm[2] = (float)pl.max_hardening;
        a.prm[3] = (float)pl.hardening_factor; a.prm[4] = 0.f;
    }
    return a;
}

int grid_stride_blocks(mpm_handle* h, int64_t n, int t)
{
    int64_t b = (n + t - 1) / t, cap = (int64_t)h->sm_count * 16;
    if(b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

// Launch shapes the autotuner chooses among.  P2G: lane groups with 128 or
// 256 threads (work items of up to 512 / 1024 particles), or the fixed-point
// tile with 128 or 256 threads (one particle per thread).
const int kG2PThreads[] = {64, 128, 256};
const char* const kP2GNames[] = {"groups128", "groups256", "fixed128", "fixed256"};

int occupancy_ctas(mpm_handle* h, const void* fn, int threads, int mult)
{
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, 0);
    return h->sm_count * (occ > 0 ? occ : 1) * mult;
}

}  // namespace

// ---------------------------------------------------------------------------
// Scenes: block / node-block / grid numbering of the whole batch.
// ---------------------------------------------------------------------------
static int encode_tile_maps(mpm_handle* h);

int fast_setup_scenes(mpm_handle* h, const mpm_scene_desc* descs, int count, const mpm_collision_object* objs, int nobjs)
{
    h->fast.generation++;
    FastState& f = h->fast;
    if(count < 1 || count > 65535) return set_error(h, MPM_ERR_ARG, "between 1 and 65535 scenes");
    std::vector<SceneDev> sc(count);
    std::vector<int64_t> pb(count + 1, 0);
    int64_t blocks = 0, nblocks = 0, nodes = 0;
    for(int s = 0; s < count; s++) {
        const mpm_scene_desc& d = descs[s];
        if(d.grid.dim != 3 || d.grid.ghost != MPM_GHOST) return set_error(h, MPM_ERR_ARG, "batched scenes are 3D with ghost 3");
        if(d.model != MPM_COROTATED_FIXED && d.model != MPM_NEO_HOOKEAN && d.model != MPM_STVK_HENCKY)
            return set_error(h, MPM_ERR_ARG, "model");
        if(d.particle_count < 0) return set_error(h, MPM_ERR_ARG, "particle_count");
        if(d.object_count < 0 || d.object_count > MPM_MAX_OBJECTS || d.first_object < 0 || d.first_object + d.object_count > nobjs)
            return set_error(h, MPM_ERR_ARG, "scene collision-object range");
        SceneDev& c = sc[s];
        memset(&c, 0, sizeof(c));
        int64_t snodes = 1, sblocks = 1, snb = 1;
        for(int k = 0; k < 3; k++) {
            if(d.grid.counts[k] < 1 || d.grid.counts[k] > 4096 || !(d.grid.domain_max[k] > d.grid.domain_min[k]))
                return set_error(h, MPM_ERR_ARG, "scene grid");
            double dx = (d.grid.domain_max[k] - d.grid.domain_min[k]) / d.grid.counts[k];   // GRID.cpp:23-24
            c.dmin[k] = (float)d.grid.domain_min[k];
            c.dmax[k] = (float)d.grid.domain_max[k];
            c.dx[k] = (float)dx;
            c.inv[k] = (float)(1 / dx);
            c.gravity[k] = (float)d.gravity[k];
            c.counts[k] = d.grid.counts[k];
            c.NB[k] = (d.grid.counts[k] + 4 + 3) / 4;
            c.NN[k] = c.NB[k] + 1;
            c.GA[k] = 4 * c.NN[k];
            snodes *= c.GA[k];
            sblocks *= c.NB[k];
            snb *= c.NN[k];
        }
        c.block_base = (uint32_t)blocks;
        c.nb_base = (uint32_t)nblocks;
        c.node_base = nodes;
        c.model = d.model;
        c.obj_begin = d.first_object;
        c.nobj = d.object_count;
        blocks += sblocks;
        nblocks += snb;
        nodes += snodes;
        pb[s + 1] = pb[s] + d.particle_count;
    }
    int bits = 6;
    while((1LL << bits) <= blocks * 64) bits++;
    if(bits > 32) return set_error(h, MPM_ERR_ARG, "batch too large for 32-bit cell keys");
    fast_free(h);
    f.nscenes = count;
    f.scenes_h = sc;
    f.pbase_h = pb;
    f.key_bits = bits;
    f.total_blocks = blocks;
    f.total_nblocks = nblocks;
    f.total_nodes = nodes;
    std::vector<uint16_t> bs(blocks), ns(nblocks);
    for(int s = 0; s < count; s++) {
        int64_t b1 = s + 1 < count ? sc[s + 1].block_base : blocks;
        int64_t n1 = s + 1 < count ? sc[s + 1].nb_base : nblocks;
        for(int64_t b = sc[s].block_base; b < b1; b++) bs[b] = (uint16_t)s;
        for(int64_t b = sc[s].nb_base; b < n1; b++) ns[b] = (uint16_t)s;
    }
    MPM_CUDA(h, cudaMalloc(&f.scenes, count * sizeof(SceneDev)));
    MPM_CUDA(h, cudaMemcpy(f.scenes, sc.data(), count * sizeof(SceneDev), cudaMemcpyHostToDevice));
    MPM_CUDA(h, cudaMalloc(&f.pbase, (count + 1) * sizeof(int64_t)));
    MPM_CUDA(h, cudaMemcpy(f.pbase, pb.data(), (count + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
    MPM_CUDA(h, cudaMalloc(&f.block_scene, blocks * sizeof(uint16_t)));
    MPM_CUDA(h, cudaMemcpy(f.block_scene, bs.data(), blocks * sizeof(uint16_t), cudaMemcpyHostToDevice));
    MPM_CUDA(h, cudaMalloc(&f.nb_scene, nblocks * sizeof(uint16_t)));
    MPM_CUDA(h, cudaMemcpy(f.nb_scene, ns.data(), nblocks * sizeof(uint16_t), cudaMemcpyHostToDevice));
    f.objs_h.assign(nobjs > 0 ? nobjs : 1, DevObject{});
    for(int i = 0; i < nobjs; i++) {
        DevObject& o = f.objs_h[i];
        o.kind = objs[i].kind;
        o.type = objs[i].type;
        o.friction = objs[i].friction;
        for(int k = 0; k < 3; k++) { o.a[k] = objs[i].a[k]; o.b[k] = objs[i].b[k]; }
    }
    MPM_CUDA(h, cudaMalloc(&f.objs, f.objs_h.size() * sizeof(DevObject)));
    MPM_CUDA(h, cudaMemcpy(f.objs, f.objs_h.data(), f.objs_h.size() * sizeof(DevObject), cudaMemcpyHostToDevice));
    f.grid_nodes = nodes;
    f.grid_node_blocks = nblocks;
    f.grid_dirty = false;
    MPM_CUDA(h, cudaMalloc(&f.acc, nodes * sizeof(float4)));
    MPM_CUDA(h, cudaMalloc(&f.vel, nodes * 2 * sizeof(float4)));
    MPM_CUDA(h, cudaMemset(f.acc, 0, nodes * sizeof(float4)));
    MPM_CUDA(h, cudaMemset(f.vel, 0, nodes * 2 * sizeof(float4)));
    for(int k = 0; k < 2; k++) {
        MPM_CUDA(h, cudaMalloc(&f.bstart[k], blocks * sizeof(uint32_t)));
        MPM_CUDA(h, cudaMalloc(&f.bend[k], blocks * sizeof(uint32_t)));
        MPM_CUDA(h, cudaMalloc(&f.active[k], blocks * sizeof(uint4)));
    }
    MPM_CUDA(h, cudaMalloc(&f.nb_flag, nblocks * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMalloc(&f.nb_list, nblocks * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMemset(f.nb_flag, 0, nblocks * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMalloc(&f.counters, 2 * CNT_COUNT * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMemset(f.counters, 0, 2 * CNT_COUNT * sizeof(uint32_t)));
    // routing between substeps: direction counts and offsets, far arrivals,
    // the block scan's epoch word and look-back status words (two chains)
    MPM_CUDA(h, cudaMalloc(&f.dcount, (size_t)ROW * blocks * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMalloc(&f.doff, (size_t)ROW * blocks * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMalloc(&f.bcount, blocks * sizeof(unsigned long long)));
    MPM_CUDA(h, cudaMemset(f.bcount, 0, blocks * sizeof(unsigned long long)));
    MPM_CUDA(h, cudaMemset(f.dcount, 0, (size_t)ROW * blocks * sizeof(uint32_t)));
    const int64_t tiles = (blocks + SCAN_TILE - 1) / SCAN_TILE;
    MPM_CUDA(h, cudaMalloc(&f.scan, (8 + 4 * STATUS_STRIDE * tiles) * sizeof(uint32_t)));
    MPM_CUDA(h, cudaMemset(f.scan, 0, (8 + 4 * STATUS_STRIDE * tiles) * sizeof(uint32_t)));
    f.order_ready = false;
    f.sorted_now = false;
    return encode_tile_maps(h);
}

// G2P's tile copies: per scene, its slice of the node grid (GA[0] x GA[1] x
// GA[2] nodes, z fastest, 8 floats = 32 bytes per node: v_new, v_fric, mass)
// as a 4D tensor {8, z, y, x} with a box of {8, 6, 6, 6}.  The driver's
// encoder is looked up through the runtime, so the library does not link
// libcuda directly.
static int encode_tile_maps(mpm_handle* h)
{
    FastState& f = h->fast;
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if(!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
           q != cudaDriverEntryPointSuccess || !fn)
            return set_error(h, MPM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    std::vector<CUtensorMap> maps(f.nscenes);
    for(int s = 0; s < f.nscenes; s++) {
        const SceneDev& c = f.scenes_h[s];
        const cuuint64_t dim[4] = {8, (cuuint64_t)c.GA[2], (cuuint64_t)c.GA[1], (cuuint64_t)c.GA[0]};
        const cuuint64_t stride[3] = {32, 32ull * c.GA[2], 32ull * c.GA[2] * c.GA[1]};
        const cuuint32_t box[4] = {8, TE, TE, TE}, estride[4] = {1, 1, 1, 1};
        CUresult r = encode(&maps[s], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void*)(f.vel + 2 * c.node_base), dim, stride, box,
                            estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if(r != CUDA_SUCCESS) return set_error(h, MPM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    }
    cudaFree(f.tmaps);
    f.tmaps = nullptr;
    MPM_CUDA(h, cudaMalloc(&f.tmaps, maps.size() * sizeof(CUtensorMap)));
    MPM_CUDA(h, cudaMemcpy(f.tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    return MPM_OK;
}

// Single-scene handles: scene 0 from the handle's grid, model and objects.
int fast_single_scene(mpm_handle* h)
{
    mpm_scene_desc d;
    memset(&d, 0, sizeof(d));
    d.grid = h->grid;
    d.model = h->model.model;
    for(int k = 0; k < 3; k++) d.gravity[k] = h->model.gravity[k];
    d.particle_count = h->fast.n;
    d.first_object = 0;
    d.object_count = h->sp.nobj;
    mpm_collision_object objs[MPM_MAX_OBJECTS];
    for(int i = 0; i < h->sp.nobj; i++) {
        objs[i].kind = h->sp.objs[i].kind;
        objs[i].type = h->sp.objs[i].type;
        objs[i].friction = h->sp.objs[i].friction;
        for(int k = 0; k < 3; k++) { objs[i].a[k] = h->sp.objs[i].a[k]; objs[i].b[k] = h->sp.objs[i].b[k]; }
    }
    int64_t n = h->fast.n;
    int rc = fast_setup_scenes(h, &d, 1, objs, h->sp.nobj);
    h->fast.n = n;
    return rc;
}

int fast_alloc(mpm_handle* h, int64_t n)
{
    FastState& f = h->fast;
    if(h->sp.dim != 3) return set_error(h, MPM_ERR_ARG, "the fast path is 3D; use MPM_PATH_PLAIN for 2D");
    if(n >= (1LL << 30)) return set_error(h, MPM_ERR_ARG, "more than 2^30 - 1 particles");
    if(f.batch) {
        if(n != f.pbase_h.back()) return set_error(h, MPM_ERR_ARG, "particle count differs from the scenes' total");
    } else if(!f.scenes || f.n != n) {
        // a new particle count rebuilds the scene tables and every buffer;
        // re-uploading the same count keeps them (and the captured graphs)
        int rc;
        f.n = n;
        if((rc = fast_single_scene(h))) return rc;
    }
    if(f.n != n || !f.soa[0]) {
        f.generation++;
        for(int b = 0; b < 2; b++) {
            cudaFree(f.soa[b]); cudaFree(f.attr[b]); cudaFree(f.pid[b]); cudaFree(f.plas[b]);
            f.soa[b] = nullptr; f.attr[b] = nullptr; f.pid[b] = nullptr; f.plas[b] = nullptr;
        }
        uint32_t** ps[] = {&f.keys[0], &f.keys[1], &f.sorted_keys, &f.perm, &f.sort_keys_alt, &f.sort_vals_alt,
                           &f.sort_scratch};
        for(uint32_t** p: ps) { cudaFree(*p); *p = nullptr; }
        for(int k = 0; k < 2; k++) {
            cudaFree(f.chunks[k]); f.chunks[k] = nullptr;
            cudaFree(f.dirs[k]); f.dirs[k] = nullptr;
        }
        cudaFree(f.vkick);
        f.vkick = nullptr;
        cudaFree(f.pmodel); cudaFree(f.pmask);   // per caller index: a new count drops them
        f.pmodel = nullptr; f.pmask = nullptr;
        int64_t np = ((n ? n : 1) + 31) / 32 * 32;
        f.npad = np;
        for(int b = 0; b < 2; b++) {
            MPM_CUDA(h, cudaMalloc(&f.soa[b], NCOMP * np * sizeof(float)));
            MPM_CUDA(h, cudaMalloc(&f.attr[b], np * sizeof(float4)));
            MPM_CUDA(h, cudaMalloc(&f.pid[b], np * sizeof(int)));
        }
        for(int k = 0; k < 2; k++) {
            MPM_CUDA(h, cudaMalloc(&f.keys[k], np * sizeof(uint32_t)));
            MPM_CUDA(h, cudaMalloc(&f.dirs[k], np * sizeof(uint8_t)));
        }
        // work items: a block's particles in parts of at least 64
        f.chunk_cap = np / 64 + std::min<int64_t>(np, f.total_blocks) + 1;
        for(int k = 0; k < 2; k++) MPM_CUDA(h, cudaMalloc(&f.chunks[k], 2 * f.chunk_cap * sizeof(uint4)));
        MPM_CUDA(h, cudaMalloc(&f.sorted_keys, np * sizeof(uint32_t)));
        MPM_CUDA(h, cudaMalloc(&f.perm, np * sizeof(uint32_t)));
        MPM_CUDA(h, cudaMalloc(&f.sort_keys_alt, np * sizeof(uint32_t)));
        MPM_CUDA(h, cudaMalloc(&f.sort_vals_alt, np * sizeof(uint32_t)));
        MPM_CUDA(h, cudaMalloc(&f.sort_scratch, mpm_sort::scratch_words(np) * sizeof(uint32_t)));
        MPM_CUDA(h, cudaMemsetAsync(f.sort_scratch, 0, mpm_sort::scratch_words(np) * sizeof(uint32_t), h->stream));
        MPM_CUDA(h, mpm_sort::prepare());
        f.n = n;
        f.order_ready = false;
        f.sorted_now = false;
    }
    return fast_penalty_buffers(h);
}

// The side buffer of the penalty impulse, once there are penalty objects and particles.
int fast_penalty_buffers(mpm_handle* h)
{
    FastState& f = h->fast;
    if(h->sp.npen && f.npad && !f.vkick) {
        f.generation++;   // make_args changes: graphs captured without the buffer are stale
        MPM_CUDA(h, cudaMalloc(&f.vkick, 3 * f.npad * sizeof(float)));
    }
    return MPM_OK;
}

void fast_free(mpm_handle* h)
{
    FastState& f = h->fast;
    for(int b = 0; b < 2; b++) {
        cudaFree(f.soa[b]); cudaFree(f.attr[b]); cudaFree(f.pid[b]); cudaFree(f.plas[b]);
        f.soa[b] = nullptr; f.attr[b] = nullptr; f.pid[b] = nullptr; f.plas[b] = nullptr;
    }
    void** ps[] = {(void**)&f.keys[0], (void**)&f.keys[1], (void**)&f.dirs[0], (void**)&f.dirs[1],
                   (void**)&f.sorted_keys, (void**)&f.perm,
                   (void**)&f.sort_keys_alt, (void**)&f.sort_vals_alt, (void**)&f.sort_scratch, (void**)&f.bstart[0],
                   (void**)&f.bend[0], (void**)&f.active[0], (void**)&f.chunks[0], (void**)&f.bstart[1],
                   (void**)&f.bend[1], (void**)&f.active[1], (void**)&f.chunks[1], (void**)&f.nb_flag,
                   (void**)&f.nb_list, (void**)&f.counters, (void**)&f.acc, (void**)&f.vel, (void**)&f.scenes,
                   (void**)&f.block_scene, (void**)&f.nb_scene, (void**)&f.pbase, (void**)&f.objs, (void**)&f.vkick,
                   (void**)&f.pmodel, (void**)&f.pmask, (void**)&f.dcount, (void**)&f.doff,
                   (void**)&f.scan, (void**)&f.tmaps, (void**)&f.bcount};
    for(void** p: ps) { cudaFree(*p); *p = nullptr; }
    f.order_ready = false;
    f.sorted_now = false;
    cudaFree(f.staging);
    f.staging = nullptr;
    f.staging_bytes = 0;
    f.n = 0;
    f.npad = 0;
    f.keys_ready = false;
}

// The handle's staging buffer for host arrays, grown on demand and kept (the
// stream is drained before it is replaced, since queued copies may use it).
static int fast_staging(mpm_handle* h, size_t bytes, uint8_t** out)
{
    FastState& f = h->fast;
    if(f.staging_bytes < bytes) {
        MPM_CUDA(h, cudaStreamSynchronize(h->stream));
        cudaFree(f.staging);
        f.staging = nullptr;
        f.staging_bytes = 0;
        MPM_CUDA(h, cudaMalloc(&f.staging, bytes));
        f.staging_bytes = bytes;
    }
    *out = (uint8_t*)f.staging;
    return MPM_OK;
}

int fast_set_particles(mpm_handle* h, const mpm_particles_view* v)
{
    int rc = fast_alloc(h, v->n);
    if(rc) return rc;
    FastState& f = h->fast;
    int64_t n = v->n;
    if(f.grid_dirty) {   // a P2G without its grid update left mass in the kept accumulator
        MPM_CUDA(h, cudaMemsetAsync(f.acc, 0, f.grid_nodes * sizeof(float4), h->stream));
        MPM_CUDA(h, cudaMemsetAsync(f.nb_flag, 0, f.grid_node_blocks * sizeof(uint32_t), h->stream));
        f.grid_dirty = false;
    }
    f.cur = 0;
    f.keys_ready = n == 0;
    f.order_ready = false;
    f.sorted_now = false;
    if(!n) return MPM_OK;
    // stage caller arrays on the device if needed
    bool dev = v->on_device != 0;
    size_t e = v->dtype == MPM_FP64 ? 8 : 4;
    const void* src[8] = {v->X, v->V, v->F, v->B, v->mass, v->volume, v->mu, v->lambda};
    int64_t cnt[8] = {3 * n, 3 * n, 9 * n, 9 * n, n, n, n, n};
    void* dptr[8] = {};
    // host arrays go through the handle's staging buffer (kept between calls,
    // so a re-upload allocates nothing): 28 scalars and 2 bytes per particle
    uint8_t* stage = nullptr;
    rc = fast_staging(h, (size_t)n * (28 * e + 2) + 256, &stage);
    if(rc) return rc;
    size_t off = 0;
    for(int i = 0; i < 8; i++) {
        if(!src[i]) return set_error(h, MPM_ERR_ARG, "null particle array");
        if(dev) dptr[i] = const_cast<void*>(src[i]);
        else {
            dptr[i] = stage + off;
            off += cnt[i] * e;
            MPM_CUDA(h, cudaMemcpyAsync(dptr[i], src[i], cnt[i] * e, cudaMemcpyHostToDevice, h->stream));
        }
    }
    uint8_t *dvalid = nullptr, *valid_slot = stage + (size_t)n * 28 * e + n;
    if(v->valid) {
        if(dev) dvalid = v->valid;
        else {
            dvalid = stage + (size_t)n * 28 * e;
            MPM_CUDA(h, cudaMemcpyAsync(dvalid, v->valid, n, cudaMemcpyHostToDevice, h->stream));
        }
    }
    FastArgs a = make_args(h, 0.0);
    a.dst = f.soa[0]; a.dst_attr = f.attr[0]; a.dst_pid = f.pid[0];
    int blocks = grid_stride_blocks(h, n, 256);
    if(e == 8)
        k_scatter_in<double><<<blocks, 256, 0, h->stream>>>(a, (const double*)dptr[0], (const double*)dptr[1], (const double*)dptr[2],
            (const double*)dptr[3], (const double*)dptr[4], (const double*)dptr[5], (const double*)dptr[6], (const double*)dptr[7], dvalid, valid_slot);
    else
        k_scatter_in<float><<<blocks, 256, 0, h->stream>>>(a, (const float*)dptr[0], (const float*)dptr[1], (const float*)dptr[2],
            (const float*)dptr[3], (const float*)dptr[4], (const float*)dptr[5], (const float*)dptr[6], (const float*)dptr[7], dvalid, valid_slot);
    MPM_LAUNCHED(h, "k_scatter_in");
    a = make_args(h, 0.0);
    k_init_keys<<<blocks, 256, 0, h->stream>>>(a, valid_slot, f.keys[f.cur]);
    MPM_LAUNCHED(h, "k_init_keys");

    f.keys_ready = true;
    if(h->plastic.kind) return fast_plastic_init(h);
    return MPM_OK;
}

// Allocate the plastic state if needed and start it unplastic.
int fast_plastic_init(mpm_handle* h)
{
    FastState& f = h->fast;
    if(!f.soa[0]) return MPM_OK;
    if(!f.plas[0])
        for(int b = 0; b < 2; b++) MPM_CUDA(h, cudaMalloc(&f.plas[b], NPLAS * f.npad * sizeof(float)));
    if(!f.n) return MPM_OK;
    const mpm_plasticity_desc& pl = h->plastic;
    if(pl.kind == MPM_PLASTICITY_DRUCKER_PRAGER) {
        k_dp_init<<<grid_stride_blocks(h, f.n, 256), 256, 0, h->stream>>>(f.n, f.npad, f.plas[f.cur], (float)pl.cohesion,
            (float)pl.dp_a0, (float)pl.dp_a1, (float)pl.dp_a3, (float)pl.dp_a4, f.pid[f.cur], f.pmask);
        MPM_LAUNCHED(h, "k_dp_init");
        return MPM_OK;
    }
    k_plastic_init<<<grid_stride_blocks(h, f.n, 256), 256, 0, h->stream>>>(f.n, f.npad, f.plas[f.cur], f.attr[f.cur]);
    MPM_LAUNCHED(h, "k_plastic_init");
    return MPM_OK;
}

// The view's arrays in the order of PlasticArrays: Fp, mu, lambda, then the
// scalars at plastic components 9.. of the handle's kind.
static void plastic_view_arrays(const mpm_handle* h, const mpm_plastic_view* v, void* out[7])
{
    const bool dp = h->plastic.kind == MPM_PLASTICITY_DRUCKER_PRAGER;
    void* a[7] = {v->Fp, v->mu, v->lambda, dp ? v->plastic_def : v->mu0, dp ? v->rho_F : v->lambda0,
                  dp ? v->cohesion : nullptr, dp ? v->vc : nullptr};
    for(int i = 0; i < 7; i++) out[i] = a[i];
}

template<class T> static PlasticArrays<T> plastic_arrays(void* const* p)
{
    PlasticArrays<T> r;
    r.Fp = (T*)p[0]; r.mu = (T*)p[1]; r.la = (T*)p[2];
    for(int k = 0; k < 4; k++) r.sc[k] = (T*)p[3 + k];
    return r;
}

int fast_get_plastic(mpm_handle* h, mpm_plastic_view* v)
{
    FastState& f = h->fast;
    if(v->n != f.n) return set_error(h, MPM_ERR_ARG, "particle count differs from mpm_set_particles");
    if(!f.plas[0]) return set_error(h, MPM_ERR_STATE, "no plastic state");
    const int64_t n = v->n;
    if(!n) return MPM_OK;
    const bool dev = v->on_device != 0;
    const size_t e = v->dtype == MPM_FP64 ? 8 : 4;
    void* dst[7];
    plastic_view_arrays(h, v, dst);
    const int64_t cnt[7] = {9 * n, n, n, n, n, n, n};
    void* dptr[7] = {};
    uint8_t* stage = nullptr;
    if(!dev) {
        int rc = fast_staging(h, (size_t)n * 15 * e + 256, &stage);
        if(rc) return rc;
    }
    size_t off = 0;
    for(int i = 0; i < 7; i++) {
        if(!dst[i]) continue;
        if(dev) dptr[i] = dst[i];
        else { dptr[i] = stage + off; off += cnt[i] * e; }
    }
    const int blocks = grid_stride_blocks(h, n, 256), c = f.cur;
    if(e == 8) k_plastic_out<double><<<blocks, 256, 0, h->stream>>>(n, f.npad, f.plas[c], f.attr[c], f.pid[c], plastic_arrays<double>(dptr));
    else k_plastic_out<float><<<blocks, 256, 0, h->stream>>>(n, f.npad, f.plas[c], f.attr[c], f.pid[c], plastic_arrays<float>(dptr));
    MPM_LAUNCHED(h, "k_plastic_out");
    if(!dev)
        for(int i = 0; i < 7; i++)
            if(dst[i]) MPM_CUDA(h, cudaMemcpyAsync(dst[i], dptr[i], cnt[i] * e, cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

int fast_set_plastic(mpm_handle* h, const mpm_plastic_view* v)
{
    FastState& f = h->fast;
    if(v->n != f.n) return set_error(h, MPM_ERR_ARG, "particle count differs from mpm_set_particles");
    if(!f.plas[0]) return set_error(h, MPM_ERR_STATE, "no plastic state");
    const int64_t n = v->n;
    if(!n) return MPM_OK;
    const bool dev = v->on_device != 0;
    const size_t e = v->dtype == MPM_FP64 ? 8 : 4;
    void* src[7];
    plastic_view_arrays(h, v, src);
    const int64_t cnt[7] = {9 * n, n, n, n, n, n, n};
    void* dptr[7] = {};
    uint8_t* stage = nullptr;
    if(!dev) {
        int rc = fast_staging(h, (size_t)n * 15 * e + 256, &stage);
        if(rc) return rc;
    }
    size_t off = 0;
    for(int i = 0; i < 7; i++) {
        if(!src[i]) continue;
        if(dev) dptr[i] = src[i];
        else {
            dptr[i] = stage + off;
            MPM_CUDA(h, cudaMemcpyAsync(stage + off, src[i], cnt[i] * e, cudaMemcpyHostToDevice, h->stream));
            off += cnt[i] * e;
        }
    }
    const int blocks = grid_stride_blocks(h, n, 256), c = f.cur;
    if(e == 8) k_plastic_in<double><<<blocks, 256, 0, h->stream>>>(n, f.npad, f.plas[c], f.attr[c], f.pid[c], plastic_arrays<double>(dptr));
    else k_plastic_in<float><<<blocks, 256, 0, h->stream>>>(n, f.npad, f.plas[c], f.attr[c], f.pid[c], plastic_arrays<float>(dptr));
    MPM_LAUNCHED(h, "k_plastic_in");
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

int fast_get_particles(mpm_handle* h, mpm_particles_view* v)
{
    FastState& f = h->fast;
    if(v->n != f.n) return set_error(h, MPM_ERR_ARG, "particle count differs from mpm_set_particles");
    int64_t n = v->n;
    if(!n) return MPM_OK;
    bool dev = v->on_device != 0;
    size_t e = v->dtype == MPM_FP64 ? 8 : 4;
    void* dst[4] = {v->X, v->V, v->F, v->B};
    int64_t cnt[4] = {3 * n, 3 * n, 9 * n, 9 * n};
    void* dptr[4] = {};
    uint8_t* stage = nullptr;
    if(!dev) {
        int rc = fast_staging(h, (size_t)n * (24 * e + 1) + 256, &stage);
        if(rc) return rc;
    }
    size_t off = 0;
    for(int i = 0; i < 4; i++) {
        if(!dst[i]) continue;
        if(dev) dptr[i] = dst[i];
        else { dptr[i] = stage + off; off += cnt[i] * e; }
    }
    uint8_t* dvalid = nullptr;
    if(v->valid) dvalid = dev ? v->valid : stage + (size_t)n * 24 * e;
    FastArgs a = make_args(h, 0.0);
    int blocks = grid_stride_blocks(h, n, 256);
    if(e == 8) k_gather_out<double><<<blocks, 256, 0, h->stream>>>(a, f.keys[f.cur], (double*)dptr[0], (double*)dptr[1], (double*)dptr[2], (double*)dptr[3], dvalid);
    else k_gather_out<float><<<blocks, 256, 0, h->stream>>>(a, f.keys[f.cur], (float*)dptr[0], (float*)dptr[1], (float*)dptr[2], (float*)dptr[3], dvalid);
    MPM_LAUNCHED(h, "k_gather_out");
    if(!dev) {
        for(int i = 0; i < 4; i++) {
            if(!dst[i]) continue;
            MPM_CUDA(h, cudaMemcpyAsync(dst[i], dptr[i], cnt[i] * e, cudaMemcpyDeviceToHost, h->stream));
        }
        if(dvalid) MPM_CUDA(h, cudaMemcpyAsync(v->valid, dvalid, n, cudaMemcpyDeviceToHost, h->stream));
    }
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

// The order of the current slots when no G2P produced it (particles just
// set, or the autotuner's restore): a radix sort of the slots' cell keys,
// then the particles are copied to the other buffer in sorted order and that
// order is recorded as a previous substep's (k_prepare).  Runs eagerly, never
// inside a captured substep.
int fast_prepare(mpm_handle* h)
{
    FastState& f = h->fast;
    if(f.order_ready || !f.keys_ready || !f.n) return MPM_OK;
    const int64_t n = f.n;
    const int c = f.cur;
    int slot = timer_begin(h, "fast_full_sort");
    cudaError_t e = mpm_sort::radix_sort(f.keys[c], f.sorted_keys, f.perm, f.sort_keys_alt, f.sort_vals_alt, n, f.key_bits,
                                         f.sort_scratch, h->d_flags, MPM_FLAG_TIMEOUT, h->sm_count * 4, h->stream);
    if(e != cudaSuccess) return check_cuda(h, e, "radix_sort");
    timer_end(h, slot);
    MPM_CUDA(h, cudaMemsetAsync(f.dcount, 0, (size_t)ROW * f.total_blocks * sizeof(uint32_t), h->stream));
    MPM_CUDA(h, cudaMemsetAsync(f.bcount, 0, f.total_blocks * sizeof(unsigned long long), h->stream));
    MPM_CUDA(h, cudaMemsetAsync(f.counters, 0, 2 * CNT_COUNT * sizeof(uint32_t), h->stream));   // both sets
    FastArgs a = make_args(h, 0.0);
    k_prepare<<<grid_stride_blocks(h, n, 256), 256, 0, h->stream>>>(a, f.bstart[c], f.bend[c], f.active[c],
                                                                    f.counters + CNT_COUNT * c);
    MPM_LAUNCHED(h, "k_prepare");
    f.cur = 1 - c;       // the sorted copy is the current buffer; set c describes it
    f.order_ready = true;
    f.sorted_now = false;
    return MPM_OK;
}

// This substep's order from the previous one: block scan (ranges, routing
// offsets, work items) and routing of every slot.
static int fast_route(mpm_handle* h)
{
    FastState& f = h->fast;
    int slot = timer_begin(h, "fast_bins");
    FastArgs a = make_args(h, 0.0);   // a.ctr: cleared by the last G2P or by fast_prepare
    const int64_t tiles = (f.total_blocks + BIN_TILE - 1) / BIN_TILE;
    k_bins<<<(unsigned)tiles, BIN_THREADS, 0, h->stream>>>(a);
    MPM_LAUNCHED(h, "k_bins");
    timer_end(h, slot);
    slot = timer_begin(h, "fast_route");
    k_route<<<occupancy_ctas(h, (const void*)k_route, 256, 1), 256, 0, h->stream>>>(a);   // resident CTAs only
    MPM_LAUNCHED(h, "k_route");
    timer_end(h, slot);
    f.sorted_now = true;
    return MPM_OK;
}

template<int T> static void launch_p2g(mpm_handle* h, const FastArgs& a)
{
    const int smem = NFAC * T * (int)sizeof(float);
    static bool attr = false;
    if(!attr) {
        cudaFuncSetAttribute((const void*)k_p2g<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)k_p2g<T>, T, smem);
    k_p2g<T><<<h->sm_count * (occ > 0 ? occ : 1) * h->fast.cta_mult, T, smem, h->stream>>>(a);
}

template<int T> static void launch_p2g_groups(mpm_handle* h, const FastArgs& a)
{
    k_p2g_groups<T><<<occupancy_ctas(h, (const void*)k_p2g_groups<T>, T, h->fast.cta_mult), T, 0, h->stream>>>(a);
}

int fast_p2g(mpm_handle* h, double dt, double)
{
    FastState& f = h->fast;
    if(!f.keys_ready) return set_error(h, MPM_ERR_STATE, "particles not set");
    if(!f.n) return MPM_OK;
    int rc = fast_prepare(h);
    if(rc) return rc;
    const bool repeat = f.sorted_now;
    if(!repeat) {
        f.route_variant = f.p2g_variant;   // the work items' size; a repeated P2G keeps it
        if((rc = fast_route(h))) return rc;
    }
    FastArgs a = make_args(h, dt);
    if(a.npen) {
        const int ps = timer_begin(h, "fast_penalty");
        k_penalty_kick<<<grid_stride_blocks(h, f.n, 256), 256, 0, h->stream>>>(a);
        timer_end(h, ps);
        MPM_LAUNCHED(h, "k_penalty_kick");
    }
    if(repeat) {   // P2G again before a G2P (the phase entry points): its work tickets restart
        MPM_CUDA(h, cudaMemsetAsync(a.ctr + CNT_P2G_WORK, 0, sizeof(uint32_t), h->stream));
        MPM_CUDA(h, cudaMemsetAsync(a.ctr + CNT_FALLBACK, 0, 2 * sizeof(uint32_t), h->stream));
    }
    int slot = timer_begin(h, "fast_p2g");
    switch(f.route_variant) {
        case MPM_P2G_GROUPS256: launch_p2g_groups<256>(h, a); break;
        case MPM_P2G_FIXED128: launch_p2g<128>(h, a); break;
        case MPM_P2G_FIXED256: launch_p2g<256>(h, a); break;
        default: launch_p2g_groups<128>(h, a); break;
    }
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_p2g");
    f.grid_dirty = true;   // until the grid update reads and clears the accumulator
    return MPM_OK;
}

int fast_forces(mpm_handle* h, double dt, double)
{
    FastState& f = h->fast;
    if(!f.n) return MPM_OK;
    if(!f.sorted_now) return set_error(h, MPM_ERR_STATE, "grid update before P2G");
    FastArgs a = make_args(h, dt);
    f.grid_set = f.cur;
    int slot = timer_begin(h, "fast_grid");
    k_grid<<<h->sm_count * 8, 256, 0, h->stream>>>(a);
    f.grid_dirty = false;
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_grid");
    return MPM_OK;
}

template<int PK> static void launch_g2p(mpm_handle* h, const FastArgs& a)
{
    const FastState& f = h->fast;
    switch(f.g2p_threads) {
        case 64: k_g2p<64, PK><<<occupancy_ctas(h, (const void*)k_g2p<64, PK>, 64, f.cta_mult), 64, 0, h->stream>>>(a); break;
        case 256: k_g2p<256, PK><<<occupancy_ctas(h, (const void*)k_g2p<256, PK>, 256, f.cta_mult), 256, 0, h->stream>>>(a); break;
        default: k_g2p<128, PK><<<occupancy_ctas(h, (const void*)k_g2p<128, PK>, 128, f.cta_mult), 128, 0, h->stream>>>(a); break;
    }
}

int fast_g2p(mpm_handle* h, double dt, double)
{
    FastState& f = h->fast;
    if(!f.n) return MPM_OK;
    if(!f.sorted_now) return set_error(h, MPM_ERR_STATE, "G2P before P2G");
    FastArgs a = make_args(h, dt);
    int slot = timer_begin(h, "fast_g2p");
    if(!a.psrc) launch_g2p<0>(h, a);
    else if(a.pkind == MPM_PLASTICITY_CLAMP) launch_g2p<1>(h, a);
    else launch_g2p<2>(h, a);
    timer_end(h, slot);
    MPM_LAUNCHED(h, "k_g2p");
    f.cur = 1 - f.cur;
    f.sorted_now = false;
    f.order_ready = true;
    return MPM_OK;
}

namespace {
// Extra node forces (the caller's, in the reference's ghosted layout) into the
// P2G accumulator of the listed node blocks: momentum + dt f where the node
// has mass, which the grid update then turns into dv = dt f / m.
template<class S> __global__ void k_add_forces(FastArgs a, const S* f, float dt, int G0, int G1, int G2)
{
    const SceneDev& sc = a.scenes[0];
    const uint64_t total = (uint64_t)a.ctr[CNT_NODE_BLOCKS] * 64u;
    for(uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t nb = a.nb_list[g >> 6] - sc.nb_base;
        const int t = (int)(g & 63u);
        const int nz = nb % sc.NN[2], r = nb / sc.NN[2], ny = r % sc.NN[1], nx = r / sc.NN[1];
        const int qx = 4 * nx + (t >> 4), qy = 4 * ny + ((t >> 2) & 3), qz = 4 * nz + (t & 3);
        if(qx >= G0 || qy >= G1 || qz >= G2) continue;
        const int64_t q = node_index(sc, qx, qy, qz);
        float4 c = a.acc[q];
        if(c.w == 0.f) continue;
        const int64_t o = 3 * (((int64_t)qx * G1 + qy) * G2 + qz);
        c.x += dt * (float)f[o];
        c.y += dt * (float)f[o + 1];
        c.z += dt * (float)f[o + 2];
        a.acc[q] = c;
    }
}
}  // namespace

int fast_add_forces(mpm_handle* h, double dt, const void* f, int dtype, bool on_device)
{
    FastState& f_ = h->fast;
    if(!f_.n) return MPM_OK;
    if(!f_.sorted_now || !f_.grid_dirty) return set_error(h, MPM_ERR_STATE, "extra node forces go between P2G and the grid update");
    int G[3];
    int64_t gn = 1;
    for(int k = 0; k < 3; k++) { G[k] = h->sp.counts[k] + 2 * MPM_GHOST; gn *= G[k]; }
    const size_t e = dtype == MPM_FP64 ? 8 : 4;
    const void* src = f;
    void* stage = nullptr;
    if(!on_device) {
        MPM_CUDA(h, cudaMallocAsync(&stage, gn * 3 * e, h->stream));
        MPM_CUDA(h, cudaMemcpyAsync(stage, f, gn * 3 * e, cudaMemcpyHostToDevice, h->stream));
        src = stage;
    }
    FastArgs a = make_args(h, dt);
    if(e == 8) k_add_forces<double><<<h->sm_count * 8, 256, 0, h->stream>>>(a, (const double*)src, (float)dt, G[0], G[1], G[2]);
    else k_add_forces<float><<<h->sm_count * 8, 256, 0, h->stream>>>(a, (const float*)src, (float)dt, G[0], G[1], G[2]);
    MPM_LAUNCHED(h, "k_add_forces");
    if(stage) MPM_CUDA(h, cudaFreeAsync(stage, h->stream));
    return MPM_OK;
}

int fast_get_grid(mpm_handle* h, int scene, double* m, double* v0, double* v, double* vf)
{
    FastState& f = h->fast;
    if(v0) return set_error(h, MPM_ERR_ARG, "velocity after P2G is not kept on the fast path");
    if(scene < 0 || scene >= f.nscenes) return set_error(h, MPM_ERR_ARG, "scene index");
    int G[3];
    int64_t gn = 1;
    for(int k = 0; k < 3; k++) { G[k] = f.scenes_h[scene].counts[k] + 2 * MPM_GHOST; gn *= G[k]; }
    uint32_t count = 0;
    MPM_CUDA(h, cudaMemcpyAsync(&count, f.counters + CNT_COUNT * f.grid_set + CNT_NODE_BLOCKS, sizeof(count),
                                cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    double *dm = nullptr, *dv = nullptr, *dvf = nullptr;
    if(m) { MPM_CUDA(h, cudaMallocAsync((void**)&dm, gn * 8, h->stream)); MPM_CUDA(h, cudaMemsetAsync(dm, 0, gn * 8, h->stream)); }
    if(v) { MPM_CUDA(h, cudaMallocAsync((void**)&dv, gn * 24, h->stream)); MPM_CUDA(h, cudaMemsetAsync(dv, 0, gn * 24, h->stream)); }
    if(vf) { MPM_CUDA(h, cudaMallocAsync((void**)&dvf, gn * 24, h->stream)); MPM_CUDA(h, cudaMemsetAsync(dvf, 0, gn * 24, h->stream)); }
    FastArgs a = make_args(h, 0.0);
    if(count) {
        k_grid_out<<<count < 65535u ? count : 65535u, 64, 0, h->stream>>>(a, f.nb_list, count, scene, dm, dv, dvf, G[0], G[1], G[2]);
        MPM_LAUNCHED(h, "k_grid_out");
    }
    if(m) { MPM_CUDA(h, cudaMemcpyAsync(m, dm, gn * 8, cudaMemcpyDeviceToHost, h->stream)); MPM_CUDA(h, cudaFreeAsync(dm, h->stream)); }
    if(v) { MPM_CUDA(h, cudaMemcpyAsync(v, dv, gn * 24, cudaMemcpyDeviceToHost, h->stream)); MPM_CUDA(h, cudaFreeAsync(dv, h->stream)); }
    if(vf) { MPM_CUDA(h, cudaMemcpyAsync(vf, dvf, gn * 24, cudaMemcpyDeviceToHost, h->stream)); MPM_CUDA(h, cudaFreeAsync(dvf, h->stream)); }
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

int fast_count_valid(mpm_handle* h, int64_t* c)
{
    FastState& f = h->fast;
    unsigned long long* d = nullptr;
    MPM_CUDA(h, cudaMallocAsync(&d, sizeof(*d), h->stream));
    MPM_CUDA(h, cudaMemsetAsync(d, 0, sizeof(*d), h->stream));
    if(f.n) {
        k_count_keys<<<grid_stride_blocks(h, f.n, 256), 256, 0, h->stream>>>(f.keys[f.cur], f.n, d);
        MPM_LAUNCHED(h, "k_count_keys");
    }
    unsigned long long r = 0;
    MPM_CUDA(h, cudaMemcpyAsync(&r, d, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaFreeAsync(d, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    *c = (int64_t)r;
    return MPM_OK;
}

int fast_debug_sort_state(mpm_handle* h, uint32_t* slot_keys, uint32_t* sorted_keys, uint32_t* perm)
{
    FastState& f = h->fast;
    size_t bytes = f.n * sizeof(uint32_t);
    if(slot_keys) MPM_CUDA(h, cudaMemcpyAsync(slot_keys, f.keys[f.cur], bytes, cudaMemcpyDeviceToHost, h->stream));
    if(sorted_keys) MPM_CUDA(h, cudaMemcpyAsync(sorted_keys, f.sorted_keys, bytes, cudaMemcpyDeviceToHost, h->stream));
    if(perm) MPM_CUDA(h, cudaMemcpyAsync(perm, f.perm, bytes, cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: times every (P2G variant, G2P block size, persistent-CTA multiple)
// on the handle's own particles for a few substeps and keeps the fastest.  The
// particle state is restored afterwards (the trials run on a copy).
// ---------------------------------------------------------------------------
int fast_autotune(mpm_handle* h, double dt, int substeps, int flags, char* report, int report_len)
{
    FastState& f = h->fast;
    if(!f.keys_ready || !f.n) return set_error(h, MPM_ERR_STATE, "particles not set");
    if(substeps < 1) substeps = 1;
    if(substeps > 64) substeps = 64;
    // cold L2: a buffer twice the L2 is written before every timed substep
    const bool cold = flags & MPM_AUTOTUNE_COLD_L2;
    void* scrub = nullptr;
    size_t scrub_bytes = 0;
    if(cold) {
        int l2 = 0;
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, h->device);
        scrub_bytes = 2 * (size_t)(l2 > 0 ? l2 : (64 << 20));
        MPM_CUDA(h, cudaMalloc(&scrub, scrub_bytes));
    }
    // keep the current state: both buffers + keys
    const int64_t np = f.npad;
    float* save_soa = nullptr;
    float4* save_attr = nullptr;
    int* save_pid = nullptr;
    uint32_t* save_keys = nullptr;
    MPM_CUDA(h, cudaMalloc(&save_soa, NCOMP * np * sizeof(float)));
    MPM_CUDA(h, cudaMalloc(&save_attr, np * sizeof(float4)));
    MPM_CUDA(h, cudaMalloc(&save_pid, np * sizeof(int)));
    MPM_CUDA(h, cudaMalloc(&save_keys, np * sizeof(uint32_t)));
    const int cur0 = f.cur;
    MPM_CUDA(h, cudaMemcpyAsync(save_soa, f.soa[cur0], NCOMP * np * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(save_attr, f.attr[cur0], np * sizeof(float4), cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(save_pid, f.pid[cur0], np * sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(save_keys, f.keys[cur0], np * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
    float* save_plas = nullptr;
    const bool plastic = h->plastic.kind && f.plas[0];
    if(plastic) {
        MPM_CUDA(h, cudaMalloc(&save_plas, NPLAS * np * sizeof(float)));
        MPM_CUDA(h, cudaMemcpyAsync(save_plas, f.plas[cur0], NPLAS * np * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    }
    cudaEvent_t e0[64], e1[64];
    for(int k = 0; k < substeps; k++) { cudaEventCreate(&e0[k]); cudaEventCreate(&e1[k]); }
    std::string rep;
    float best = 1e30f;
    int best_v = f.p2g_variant, best_t = f.g2p_threads, best_m = f.cta_mult;
    const bool timing = h->timing;
    h->timing = false;
    int rc = MPM_OK;
    for(int variant = 0; variant <= MPM_P2G_FIXED256 && !rc; variant++)
        for(int ti = 0; ti < 3 && !rc; ti++)
            for(int mult = 1; mult <= 2 && !rc; mult++) {
                f.p2g_variant = variant;
                f.g2p_threads = kG2PThreads[ti];
                f.cta_mult = mult;
                // restore, warm up one substep, then time
                f.cur = cur0;
                cudaMemcpyAsync(f.soa[cur0], save_soa, NCOMP * np * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(f.attr[cur0], save_attr, np * sizeof(float4), cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(f.pid[cur0], save_pid, np * sizeof(int), cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(f.keys[cur0], save_keys, np * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream);
                if(plastic) cudaMemcpyAsync(f.plas[cur0], save_plas, NPLAS * np * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
                f.order_ready = false;
                f.sorted_now = false;
                if((rc = fast_p2g(h, dt, 0)) || (rc = fast_forces(h, dt, 0)) || (rc = fast_g2p(h, dt, 0))) break;
                for(int s = 0; s < substeps && !rc; s++) {
                    if(cold) cudaMemsetAsync(scrub, s & 0xff, scrub_bytes, h->stream);
                    cudaEventRecord(e0[s], h->stream);
                    if(!(rc = fast_p2g(h, dt, 0)) && !(rc = fast_forces(h, dt, 0))) rc = fast_g2p(h, dt, 0);
                    cudaEventRecord(e1[s], h->stream);
                }
                if(rc) break;
                if(cudaEventSynchronize(e1[substeps - 1]) != cudaSuccess) { rc = check_cuda(h, cudaGetLastError(), "autotune"); break; }
                float ms = 0;
                for(int s = 0; s < substeps; s++) {
                    float one = 0;
                    cudaEventElapsedTime(&one, e0[s], e1[s]);
                    ms += one;
                }
                ms /= substeps;
                char line[128];
                snprintf(line, sizeof line, "%sp2g=%s g2p=%d ctas=x%d: %.4f ms", rep.empty() ? "" : "; ",
                         kP2GNames[variant], kG2PThreads[ti], mult, ms);
                rep += line;
                if(ms < best) { best = ms; best_v = variant; best_t = kG2PThreads[ti]; best_m = mult; }
            }
    h->timing = timing;
    f.p2g_variant = best_v;
    f.g2p_threads = best_t;
    f.cta_mult = best_m;
    f.cur = cur0;
    cudaMemcpyAsync(f.soa[cur0], save_soa, NCOMP * np * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(f.attr[cur0], save_attr, np * sizeof(float4), cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(f.pid[cur0], save_pid, np * sizeof(int), cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(f.keys[cur0], save_keys, np * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream);
    if(plastic) cudaMemcpyAsync(f.plas[cur0], save_plas, NPLAS * np * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
    f.order_ready = false;
    f.sorted_now = false;
    cudaStreamSynchronize(h->stream);
    cudaFree(save_soa); cudaFree(save_attr); cudaFree(save_pid); cudaFree(save_keys); cudaFree(save_plas);
    for(int k = 0; k < substeps; k++) { cudaEventDestroy(e0[k]); cudaEventDestroy(e1[k]); }
    cudaFree(scrub);
    char tail[128];
    snprintf(tail, sizeof tail, " | chosen p2g=%s g2p=%d ctas=x%d (%.4f ms/substep%s)", kP2GNames[best_v], best_t, best_m, best,
             cold ? ", cold L2" : "");
    rep += tail;
    if(report && report_len > 0) snprintf(report, (size_t)report_len, "%s", rep.c_str());
    return rc;
}

int64_t sort_scratch_words(int64_t n) { return mpm_sort::scratch_words(n); }

// Stable LSD radix sort of device keys on the handle's stream (the fast path's
// sort), for the other paths: sorted keys and the permutation.
int sort_keys_device(mpm_handle* h, const uint32_t* keys, int64_t n, int bits, uint32_t* sorted, uint32_t* perm,
    uint32_t* alt_keys, uint32_t* alt_vals, uint32_t* scratch)
{
    MPM_CUDA(h, mpm_sort::prepare());
    cudaError_t e = mpm_sort::radix_sort(keys, sorted, perm, alt_keys, alt_vals, n, bits, scratch, h->d_flags,
                                         MPM_FLAG_TIMEOUT, h->sm_count * 4, h->stream);
    if(e != cudaSuccess) return check_cuda(h, e, "radix_sort");
    return MPM_OK;
}

int radix_sort_host(const uint32_t* keys, int64_t n, int bits, uint32_t* sorted_keys, uint32_t* perm)
{
    if(n < 0 || bits < 1 || bits > 32 || (n && (!keys || !sorted_keys || !perm))) return MPM_ERR_ARG;
    if(n >= (1LL << 30)) return MPM_ERR_ARG;
    if(!n) return MPM_OK;
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t st;
    if(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return MPM_ERR_CUDA;
    uint32_t *k = nullptr, *ko = nullptr, *vo = nullptr, *ka = nullptr, *va = nullptr, *scratch = nullptr;
    unsigned* flags = nullptr;
    int rc = MPM_OK;
    size_t b = n * sizeof(uint32_t);
    size_t sw = mpm_sort::scratch_words(n) * sizeof(uint32_t);
    if(cudaMalloc(&k, b) || cudaMalloc(&ko, b) || cudaMalloc(&vo, b) || cudaMalloc(&ka, b) || cudaMalloc(&va, b) ||
       cudaMalloc(&scratch, sw) || cudaMalloc(&flags, sizeof(unsigned))) rc = MPM_ERR_NOMEM;
    if(!rc && (cudaMemsetAsync(scratch, 0, sw, st) || cudaMemsetAsync(flags, 0, sizeof(unsigned), st) ||
               mpm_sort::prepare())) rc = MPM_ERR_CUDA;
    if(!rc) {
        cudaMemcpyAsync(k, keys, b, cudaMemcpyHostToDevice, st);
        if(mpm_sort::radix_sort(k, ko, vo, ka, va, n, bits, scratch, flags, MPM_FLAG_TIMEOUT, sms * 4, st) != cudaSuccess)
            rc = MPM_ERR_CUDA;
        else {
            unsigned fl = 0;
            cudaMemcpyAsync(sorted_keys, ko, b, cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(perm, vo, b, cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(&fl, flags, sizeof(fl), cudaMemcpyDeviceToHost, st);
            if(cudaStreamSynchronize(st) != cudaSuccess) rc = MPM_ERR_CUDA;
            else if(fl & MPM_FLAG_TIMEOUT) rc = MPM_ERR_TIMEOUT;
        }
    }
    cudaFree(k); cudaFree(ko); cudaFree(vo); cudaFree(ka); cudaFree(va); cudaFree(scratch); cudaFree(flags);
    cudaStreamDestroy(st);
    return rc;
}

// A sort pass whose first tile never runs: the pass's ticket counter starts at
// 1 and one CTA fewer than the tiles is launched, so every tile's look-back
// reaches tile 0, which never publishes, and gives up after `spin_limit` polls.
// Every output position stays inside [0, n): a tile that gave up misses tile
// 0's counts, which only lowers its positions.  Test hook for the timeout path.
int debug_sort_stall(const uint32_t* keys, int64_t n, int bits, uint32_t spin_limit)
{
    const int64_t tiles = mpm_sort::tiles_for(n, mpm_sort::kSmallTile);
    if(!keys || bits < 1 || bits > 32 || tiles < 2 || n > mpm_sort::kSmallSortMax || spin_limit > (1u << 22))
        return MPM_ERR_ARG;
    cudaStream_t st;
    if(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return MPM_ERR_CUDA;
    uint32_t *k = nullptr, *ko = nullptr, *vo = nullptr, *scratch = nullptr;
    unsigned* flags = nullptr;
    const size_t b = n * sizeof(uint32_t), sw = mpm_sort::scratch_words(n) * sizeof(uint32_t);
    int rc = MPM_OK;
    if(cudaMalloc(&k, b) || cudaMalloc(&ko, b) || cudaMalloc(&vo, b) || cudaMalloc(&scratch, sw) ||
       cudaMalloc(&flags, sizeof(unsigned))) rc = MPM_ERR_NOMEM;
    if(!rc && (cudaMemsetAsync(scratch, 0, sw, st) || cudaMemsetAsync(flags, 0, sizeof(unsigned), st) ||
               mpm_sort::prepare() || cudaMemcpyAsync(k, keys, b, cudaMemcpyHostToDevice, st))) rc = MPM_ERR_CUDA;
    if(!rc) {
        mpm_sort::k_upfront_hist<<<1, mpm_sort::kThreads, 0, st>>>(k, n, bits, scratch);   // epoch 1, tickets 0
        const uint32_t one = 1;
        cudaMemcpyAsync(scratch + mpm_sort::kTicketOff, &one, sizeof one, cudaMemcpyHostToDevice, st);
        mpm_sort::k_onesweep<mpm_sort::kSmallItems><<<(unsigned)(tiles - 1), mpm_sort::kThreads,
            mpm_sort::pass_smem<mpm_sort::kSmallItems>(), st>>>(k, nullptr, ko, vo, n, bits, 0, tiles, scratch, flags,
                                                                MPM_FLAG_TIMEOUT, spin_limit);
        unsigned fl = 0;
        cudaMemcpyAsync(&fl, flags, sizeof fl, cudaMemcpyDeviceToHost, st);
        if(cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = MPM_ERR_CUDA;
        else if(fl & MPM_FLAG_TIMEOUT) rc = MPM_ERR_TIMEOUT;
    }
    cudaFree(k); cudaFree(ko); cudaFree(vo); cudaFree(scratch); cudaFree(flags);
    cudaStreamDestroy(st);
    return rc;
}

// Seed the epoch words of the handle's radix-sort scratch and block scan (test
// hook: sorts and scans across the 2^30 wrap of the status words' epoch field).
int debug_set_sort_epoch(mpm_handle* h, uint32_t epoch)
{
    FastState& f = h->fast;
    if(!f.sort_scratch || !f.scan) return set_error(h, MPM_ERR_STATE, "no sort scratch");
    MPM_CUDA(h, cudaMemcpyAsync(f.sort_scratch + mpm_sort::kEpochOff, &epoch, sizeof epoch, cudaMemcpyHostToDevice, h->stream));
    MPM_CUDA(h, cudaMemcpyAsync(f.scan, &epoch, sizeof epoch, cudaMemcpyHostToDevice, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

// ---------------------------------------------------------------------------
// Radix sort without any allocation.
//
// Some callers cannot allocate device memory when they need to sort: hosts
// that give this library a fixed memory budget up front and forbid growth
// afterwards, and loops with latency limits that cannot absorb cudaMalloc /
// cudaFree and the device-wide synchronisation cudaFree implies.
// mpm_radix_sort_u32_noalloc serves them: the caller passes device arrays for
// the keys and both outputs, and every temporary the sort needs lives in one
// fixed array compiled into this file.  The call blocks until the sort is
// done (it reads back the timeout flag of the sort's bounded waits).
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (about 2.6 MB) until the process exits, whether or not the
// entry point is used.  It is shared by all calls on a device and keeps the
// previous call's contents; each call clears what must start at zero.  Calls
// that overlap on the GPU (two streams, or two host threads) race on it.
// ---------------------------------------------------------------------------
namespace {
constexpr int64_t kNoAllocMaxKeys = MPM_NOALLOC_MAX_KEYS;
constexpr int64_t kNoAllocSortWords =
    mpm_sort::kStatusOff + 2LL * mpm_sort::kMaxPasses * ((kNoAllocMaxKeys + mpm_sort::kTile - 1) / mpm_sort::kTile) * mpm_sort::kRadix;
constexpr int64_t kNoAllocKeysAlt = kNoAllocSortWords;                 // ping-pong keys
constexpr int64_t kNoAllocValsAlt = kNoAllocKeysAlt + kNoAllocMaxKeys;  // ping-pong payloads
constexpr int64_t kNoAllocFlag = kNoAllocValsAlt + kNoAllocMaxKeys;     // timeout flag word
constexpr int64_t kNoAllocWords = kNoAllocFlag + 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

// The host-side name g_noalloc_scratch is only a stand-in for the device
// variable; kernels get its device address, looked up once per device.
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Once per device, with that device current: find the array's device address
// and zero it (the look-back status words must start with epoch 0).
int noalloc_setup(int dev, uint32_t** out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if(!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        if(cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MPM_ERR_CUDA;
        if(cudaMemset(p, 0, sizeof(uint32_t) * kNoAllocWords) != cudaSuccess) return MPM_ERR_CUDA;
        if(mpm_sort::prepare() != cudaSuccess) return MPM_ERR_CUDA;
        g_noalloc_ptr[dev] = (uint32_t*)p;
    }
    *out = g_noalloc_ptr[dev];
    return MPM_OK;
}
}  // namespace

extern "C" int mpm_radix_sort_u32_noalloc(const uint32_t* keys, int64_t n, int bits, uint32_t* sorted_keys,
    uint32_t* perm, void* stream)
{
    if(n < 0 || bits < 1 || bits > 32) return MPM_ERR_ARG;
    if(n > kNoAllocMaxKeys) return MPM_ERR_ARG;     // beyond the fixed scratch: use mpm_radix_sort_u32
    if(n == 0) return MPM_OK;
    if(!keys || !sorted_keys || !perm || keys == sorted_keys || keys == perm || sorted_keys == perm) return MPM_ERR_ARG;
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return MPM_ERR_CUDA;
    uint32_t* base = nullptr;
    int rc = noalloc_setup(dev, &base);
    if(rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned* flag = (unsigned*)(base + kNoAllocFlag);
    if(cudaMemsetAsync(flag, 0, sizeof(unsigned), st) != cudaSuccess) return MPM_ERR_CUDA;
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // 4096-key tiles always: the fixed scratch holds the look-back words for those
    if(mpm_sort::radix_sort(keys, sorted_keys, perm, base + kNoAllocKeysAlt, base + kNoAllocValsAlt, n, bits, base,
                            flag, MPM_FLAG_TIMEOUT, sms * 4, st, false) != cudaSuccess) return MPM_ERR_CUDA;
    unsigned f = 0;
    if(cudaMemcpyAsync(&f, flag, sizeof(f), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MPM_ERR_CUDA;
    if(cudaStreamSynchronize(st) != cudaSuccess) return MPM_ERR_CUDA;
    return (f & MPM_FLAG_TIMEOUT) ? MPM_ERR_TIMEOUT : MPM_OK;
}

// ---------------------------------------------------------------------------
// Diagnostics in FP64 (MPM_EXAMPLE::Total_Particle_* / Total_Grid_*,
// MPM_EXAMPLE.cpp:209-327; MPM_DRIVER::Max_Particle_Speed / Grid_V_Upper_Bound,
// MPM_DRIVER.cpp:1112-1138).  acc: mass, momentum[3], angular[3], kinetic,
// count; mx: max speed, max affine speed (as ordered bits of non-negative doubles).
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ void warp_add(double* acc, double v)
{
#pragma unroll
    for(int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if((threadIdx.x & 31) == 0 && v != 0) atomicAdd(acc, v);
}
__device__ __forceinline__ void warp_max(unsigned long long* mx, double v)
{
#pragma unroll
    for(int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if((threadIdx.x & 31) == 0) atomicMax(mx, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_particle_totals(FastArgs a, double* acc, unsigned long long* mx)
{
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, vmax = 0, amax = 0;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t key = a.keys_cur[i];
        if(key == SENTINEL) continue;
        const SceneDev& sc = a.scenes[a.block_scene[key >> 6]];
        double X[3], V[3], B[9];
        for(int k = 0; k < 3; k++) { X[k] = a.src[(C_X + k) * a.npad + i]; V[k] = a.src[(C_V + k) * a.npad + i]; }
        for(int k = 0; k < 9; k++) B[k] = a.src[(C_B + k) * a.npad + i];
        double m = a.src_attr[i].x;
        s[0] += m;
        for(int k = 0; k < 3; k++) s[1 + k] += m * V[k];
        // m X x V - m B:epsilon  (Contract_Permutation_Tensor = (B12-B21, B20-B02, B01-B10))
        s[4] += m * (X[1] * V[2] - X[2] * V[1]) - m * (B[7] - B[5]);
        s[5] += m * (X[2] * V[0] - X[0] * V[2]) - m * (B[2] - B[6]);
        s[6] += m * (X[0] * V[1] - X[1] * V[0]) - m * (B[3] - B[1]);
        double v2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2], bd = 0, bf = 0;
        for(int c = 0; c < 3; c++)
            for(int r = 0; r < 3; r++) {
                double b2 = B[r + 3 * c] * B[r + 3 * c];
                bd += b2 * 4.0 * (double)sc.inv[c] * (double)sc.inv[c];
                bf += b2;
            }
        s[7] += 0.5 * m * v2 + 0.5 * m * bd;
        s[8] += 1;
        double inv_min = fmin((double)sc.inv[0], fmin((double)sc.inv[1], (double)sc.inv[2]));
        double sp = sqrt(v2);
        vmax = fmax(vmax, sp);
        amax = fmax(amax, sp + sqrt(bf) * 6.0 * sqrt(3.0) * inv_min);
    }
    for(int k = 0; k < 9; k++) warp_add(acc + k, s[k]);
    warp_max(mx, vmax);
    warp_max(mx + 1, amax);
}

// one node block per CTA of 64 threads, over the node blocks of the last substep
__global__ void k_grid_totals(FastArgs a, uint32_t count, double* acc)
{
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for(uint32_t w = blockIdx.x; w < count; w += gridDim.x) {
        const uint32_t nb = a.nb_list[w];
        const SceneDev& sc = a.scenes[a.nb_scene[nb]];
        const uint32_t lnb = nb - sc.nb_base;
        int nz = lnb % sc.NN[2], r = lnb / sc.NN[2], ny = r % sc.NN[1], nx = r / sc.NN[1];
        int t = threadIdx.x;
        int qx = 4 * nx + (t >> 4), qy = 4 * ny + ((t >> 2) & 3), qz = 4 * nz + (t & 3);
        int64_t q = node_index(sc, qx, qy, qz);
        float4 p0 = a.vel[2 * q], p1 = a.vel[2 * q + 1];
        double m = p1.z;
        if(m == 0) continue;
        double v[3] = {p0.x, p0.y, p0.z};
        double X[3] = {sc.dmin[0] + ((double)(qx - MPM_GHOST) + 0.5) * sc.dx[0], sc.dmin[1] + ((double)(qy - MPM_GHOST) + 0.5) * sc.dx[1],
                       sc.dmin[2] + ((double)(qz - MPM_GHOST) + 0.5) * sc.dx[2]};
        s[0] += m;
        for(int k = 0; k < 3; k++) s[1 + k] += m * v[k];
        s[4] += m * (X[1] * v[2] - X[2] * v[1]);
        s[5] += m * (X[2] * v[0] - X[0] * v[2]);
        s[6] += m * (X[0] * v[1] - X[1] * v[0]);
        s[7] += 0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        s[8] += 1;
    }
    for(int k = 0; k < 9; k++) warp_add(acc + k, s[k]);
}
}  // namespace

static int totals_out(mpm_handle* h, double* dacc, unsigned long long* dmx, mpm_totals* out)
{
    double acc[9];
    unsigned long long mx[2] = {0, 0};
    MPM_CUDA(h, cudaMemcpyAsync(acc, dacc, sizeof acc, cudaMemcpyDeviceToHost, h->stream));
    if(dmx) MPM_CUDA(h, cudaMemcpyAsync(mx, dmx, sizeof mx, cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    out->mass = acc[0];
    for(int k = 0; k < 3; k++) { out->momentum[k] = acc[1 + k]; out->angular_momentum[k] = acc[4 + k]; }
    out->kinetic_energy = acc[7];
    out->count = (int64_t)acc[8];
    double v0, v1;
    memcpy(&v0, &mx[0], 8);
    memcpy(&v1, &mx[1], 8);
    out->max_speed = v0;
    out->max_affine_speed = v1;
    return MPM_OK;
}

int fast_particle_totals(mpm_handle* h, mpm_totals* out)
{
    FastState& f = h->fast;
    double* d = nullptr;
    MPM_CUDA(h, cudaMallocAsync((void**)&d, 16 * sizeof(double), h->stream));
    MPM_CUDA(h, cudaMemsetAsync(d, 0, 16 * sizeof(double), h->stream));
    if(f.n) {
        FastArgs a = make_args(h, 0.0);
        k_particle_totals<<<grid_stride_blocks(h, f.n, 256), 256, 0, h->stream>>>(a, d, (unsigned long long*)(d + 12));
        MPM_LAUNCHED(h, "k_particle_totals");
    }
    int rc = totals_out(h, d, (unsigned long long*)(d + 12), out);
    cudaFreeAsync(d, h->stream);
    return rc;
}

int fast_grid_totals(mpm_handle* h, mpm_totals* out)
{
    FastState& f = h->fast;
    uint32_t count = 0;
    MPM_CUDA(h, cudaMemcpyAsync(&count, f.counters + CNT_COUNT * f.grid_set + CNT_NODE_BLOCKS, sizeof(count),
                                cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    double* d = nullptr;
    MPM_CUDA(h, cudaMallocAsync((void**)&d, 16 * sizeof(double), h->stream));
    MPM_CUDA(h, cudaMemsetAsync(d, 0, 16 * sizeof(double), h->stream));
    if(count) {
        FastArgs a = make_args(h, 0.0);
        k_grid_totals<<<count < 65535u ? count : 65535u, 64, 0, h->stream>>>(a, count, d);
        MPM_LAUNCHED(h, "k_grid_totals");
    }
    int rc = totals_out(h, d, nullptr, out);
    out->max_speed = out->max_affine_speed = 0;
    cudaFreeAsync(d, h->stream);
    return rc;
}

// This module's copy of the SVD sweep bound (mpm_debug_set_svd_iterations).
MPM_SVD_LIMIT_SETTER(svd_limit_fast)
