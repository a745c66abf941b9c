// Host side of the serving pool (include/ffs_pool.h).
//
// Memory: one device arena of `budget_bytes`, reserved at creation, holds the
// state of every admitted episode (moments, flags, wall masks, surface and
// force arrays).  Admission carves a block out of it first-fit and fails
// with FFS_ERR_CAPACITY when no block fits; eviction returns the block.  The
// fixed tables (episode descriptors, active table, parameters, outputs, the
// shared link table) are allocated once at creation as well, so admission,
// eviction and stepping never allocate device memory.
//
// Stepping: all admitted episodes advance together.  One control step is one
// CUDA-graph launch of `substeps` x {kinematics, link detection, dense pass,
// link cells, force reduction} plus the output kernel; every kernel covers
// all episodes and reads their number from the device-side active table, so
// the graph is captured once per (tile shape, starting buffer parity) and
// reused for every mix.  The active table is re-uploaded only after the mix
// changed; the per-step parameters (actions, wave phases) are one upload.
//
// Work unit of the dense pass: ffs_pool_tune times the candidate units
// (tiles and row-marching strips, kPoolShapes) on the current mix (CUDA
// events, a warm launch then five timed ones each) and keeps the fastest.
// Every unit gives the same bits, so the choice changes only the speed.  It
// runs by itself on the first advance and again when the number of cells has
// grown or shrunk by 2x since the last tuning.  FFS_POOL_SHAPE pins the unit.
//
// Ordering: every device operation of a pool is issued on the pool's stream,
// so an evicted episode's block is reused only after the work that read it.
// The pinned parameter and output buffers are double-buffered: control step
// k uses buffer k & 1, so ffs_pool_advance waits only for step k - 2 (the
// last user of the buffer it refills), not for step k - 1, and a caller can
// enqueue the next control step while the previous one runs.  The pinned
// active table is refilled only after its last upload has completed (its own
// event).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "ffs_lbm.h"
#include "ffs_pool.h"
#include "ffs_common.cuh"
#include "ffs_links.cuh"
#include "ffs_pool.cuh"

using namespace fflbm;

namespace fflbm {
ffs_status record_error(ffs_status s, const std::string &msg); // ffs_capi.cu: sets ffs_last_error()
}

namespace {

#define POOL_CK(expr)                                                                                                  \
    do {                                                                                                               \
        cudaError_t e_ = (expr);                                                                                       \
        if (e_ != cudaSuccess)                                                                                         \
            return record_error(e_ == cudaErrorMemoryAllocation ? FFS_ERR_OUT_OF_MEMORY : FFS_ERR_CUDA,                \
                                std::string(#expr) + ": " + cudaGetErrorString(e_));                                   \
    } while (0)

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

// First-fit allocator over the arena, with coalescing of free blocks.
struct Arena {
    char *base = nullptr;
    size_t size = 0;
    std::map<size_t, size_t> free_; // offset -> bytes

    void reset(char *b, size_t n)
    {
        base = b;
        size = n;
        free_.clear();
        if (n) free_[0] = n;
    }
    bool alloc(size_t bytes, size_t *off)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t roff = it->first + bytes;
            free_.erase(it);
            if (rest) free_[roff] = rest;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t free_bytes() const
    {
        size_t s = 0;
        for (auto &kv : free_) s += kv.second;
        return s;
    }
    size_t largest() const
    {
        size_t s = 0;
        for (auto &kv : free_) s = std::max(s, kv.second);
        return s;
    }
};

// Byte offsets of one episode's arrays inside its arena block.
struct Layout {
    size_t mom0, mom1, flags, wallmask, status, rest, amp, sin_kx, cos_kx, segment, elements, V, U, acc, force, sums;
    size_t total;
};

Layout layout_of(int64_t ncell, int nv, int ne, size_t esize)
{
    Layout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o += align_up(bytes); return at; };
    L.mom0 = take(esize * 6 * (size_t)ncell);
    L.mom1 = take(esize * 6 * (size_t)ncell);
    L.flags = take(((size_t)ncell + 3) & ~(size_t)3);
    L.wallmask = take(sizeof(uint32_t) * (size_t)ncell);
    L.status = take(sizeof(uint32_t));
    L.rest = take(sizeof(float) * 2 * (size_t)nv);
    L.amp = take(sizeof(float) * (size_t)nv);
    L.sin_kx = take(sizeof(float) * (size_t)nv);
    L.cos_kx = take(sizeof(float) * (size_t)nv);
    L.segment = take(sizeof(int32_t) * (size_t)nv);
    L.elements = take(sizeof(uint32_t) * 2 * (size_t)ne);
    L.V = take(sizeof(float) * 2 * (size_t)nv);
    L.U = take(sizeof(float) * 2 * (size_t)nv);
    L.acc = take(sizeof(long long) * 2 * (size_t)nv);
    L.force = take(sizeof(double) * 2 * (size_t)nv);
    L.sums = take(sizeof(double) * 4);
    L.total = o;
    return L;
}

// sin and cos of the body-wave phase omega t of episode substep q, formed in
// double and rounded to float: the one definition the device kinematics (via
// the per-step parameter upload) and ffs_swimmer_surface share.
void wave_phase(double omega, double t0, double dt, int64_t q, float *sb, float *cb)
{
    const double beta = omega * (t0 + (double)q * dt);
    *sb = (float)std::sin(beta);
    *cb = (float)std::cos(beta);
}

struct Slot {
    bool used = false;
    size_t off = 0, bytes = 0;
    int nx = 0, ny = 0, nv = 0, ne = 0;
    int64_t ncell = 0;
    double omega_wave = 0.0, t0 = 0.0, dt = 0.0;
    int64_t q = 0; // substeps done
    float actions[kPoolMaxActions] = {};
    PoolEpisode dev{};
};

} // namespace

struct ffs_pool {
    ffs_pool_desc d{};
    size_t esize = 2;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    Arena arena;
    char *arena_mem = nullptr;
    std::vector<Slot> slots;
    std::vector<int> order; // admitted slots, admission order
    PoolEpisode *d_eps = nullptr;
    PoolParams *d_prm = nullptr, *h_prm[2] = {};
    PoolActive *d_act = nullptr, *h_act = nullptr;
    PoolOutput *d_out = nullptr, *h_out[2] = {};
    LinkTable lt;
    uint32_t *owner = nullptr;
    int shape = 1;
    bool act_dirty = true;
    int64_t tuned_cells = 0; // cells of the mix at the last tuning (0: never)
    double tuned_ms = 0.0;   // one dense pass of the chosen shape at that tuning
    int parity = 0;
    cudaGraphExec_t graph[kPoolNumShapes][2] = {};
    // done[b]: the last control step that used pinned buffer b has finished
    // (its outputs are in h_out[b]); act_sent: the last active-table upload
    // has read h_act
    cudaEvent_t done[2] = {}, act_sent = nullptr, ev0 = nullptr, ev1 = nullptr;
    bool inflight[2] = {false, false};
    bool act_pending = false;
    int last = 0;             // buffer of the latest control step
    int64_t advances = 0, graph_builds = 0;
    int sms = 0;              // SMs of the device, queried at creation
    int grid_dense[kPoolNumShapes] = {};
    int grid_link = 0;        // resident CTAs of the link-cell kernel (one wave)
};

namespace {

ffs_status fail(ffs_status s, const std::string &m) { return record_error(s, m); }

int64_t mix_cells(const ffs_pool *p)
{
    int64_t c = 0;
    for (int s : p->order) c += p->slots[s].ncell;
    return c;
}

// Fills the host active table for the current tile shape.
void build_active(ffs_pool *p)
{
    PoolActive &A = *p->h_act;
    const PoolTileShape sh = kPoolShapes[p->shape];
    A.n = (uint32_t)p->order.size();
    A.tile_prefix[0] = A.elem_prefix[0] = A.vert_prefix[0] = 0;
    for (size_t a = 0; a < p->order.size(); ++a) {
        const Slot &s = p->slots[p->order[a]];
        const uint32_t tx = (uint32_t)((s.nx + sh.tx - 1) / sh.tx), ty = (uint32_t)((s.ny + sh.ty - 1) / sh.ty);
        A.slot[a] = (uint32_t)p->order[a];
        A.tiles_x[a] = tx;
        A.tile_prefix[a + 1] = A.tile_prefix[a] + tx * ty;
        A.elem_prefix[a + 1] = A.elem_prefix[a] + (uint32_t)s.ne;
        A.vert_prefix[a + 1] = A.vert_prefix[a] + (uint32_t)s.nv;
    }
}

ffs_status upload_active(ffs_pool *p)
{
    if (p->act_pending) {
        POOL_CK(cudaEventSynchronize(p->act_sent));
        p->act_pending = false;
    }
    build_active(p);
    POOL_CK(cudaMemcpyAsync(p->d_act, p->h_act, sizeof(PoolActive), cudaMemcpyHostToDevice, p->st));
    POOL_CK(cudaEventRecord(p->act_sent, p->st));
    p->act_pending = true;
    p->act_dirty = false;
    return FFS_OK;
}

// Waits for control step(s) in flight on pinned buffer b.
ffs_status wait_buffer(ffs_pool *p, int b)
{
    if (p->inflight[b]) {
        POOL_CK(cudaEventSynchronize(p->done[b]));
        p->inflight[b] = false;
    }
    return FFS_OK;
}

// Waits for every control step in flight (the latest one finishes last: one
// stream).
ffs_status wait_idle(ffs_pool *p)
{
    ffs_status r = wait_buffer(p, p->last);
    if (r != FFS_OK) return r;
    return wait_buffer(p, p->last ^ 1);
}

template <typename T> ffs_status capture(ffs_pool *p, int shape, int parity, cudaGraphExec_t *out)
{
    const int S = p->d.substeps;
    const int g_kin = p->sms * 4, g_det = p->sms * 4, g_link = p->grid_link, g_fin = p->sms * 2;
    cudaGraph_t graph = nullptr;
    POOL_CK(cudaStreamBeginCapture(p->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t err = cudaSuccess;
    int par = parity;
    for (int j = 0; j < S && err == cudaSuccess; ++j) {
        if ((err = launch_pool_kinematics(p->d_eps, p->d_prm, p->d_act, j, g_kin, p->st)) != cudaSuccess) break;
        if ((err = launch_pool_detect<T>(p->d_eps, p->d_act, p->lt, p->owner, par, g_det, p->st)) != cudaSuccess) break;
        if ((err = launch_pool_dense<T>(p->d_eps, p->d_act, par, shape, p->grid_dense[shape], p->st)) != cudaSuccess)
            break;
        if ((err = launch_pool_link_cells<T>(p->d_eps, p->lt, p->owner, par, g_link, p->st)) != cudaSuccess) break;
        if ((err = launch_pool_finalize(p->d_eps, p->d_act, p->lt, g_fin, p->st)) != cudaSuccess) break;
        par ^= 1;
    }
    if (err == cudaSuccess) err = launch_pool_outputs(p->d_eps, p->d_act, p->d_out, S, p->st);
    cudaError_t e2 = cudaStreamEndCapture(p->st, &graph);
    if (err == cudaSuccess) err = e2;
    if (err == cudaSuccess) err = cudaGraphInstantiate(out, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (err != cudaSuccess) return fail(FFS_ERR_CUDA, std::string("pool graph capture: ") + cudaGetErrorString(err));
    ++p->graph_builds;
    return FFS_OK;
}

// FFS_POOL_SHAPE pins the dense work unit (an index into kPoolShapes) for
// tests that check every unit; -1 when unset or out of range.
static int pinned_shape()
{
    const char *pin = std::getenv("FFS_POOL_SHAPE");
    if (!pin) return -1;
    const int v = std::atoi(pin);
    return (v >= 0 && v < kPoolNumShapes) ? v : -1;
}

template <typename T> ffs_status tune_impl(ffs_pool *p)
{
    if (p->order.empty()) return FFS_OK;
    float best = 1e30f;
    int best_shape = p->shape;
    const int pin = pinned_shape(); // a pinned shape is only timed
    for (int sh = pin >= 0 ? pin : 0; sh < (pin >= 0 ? pin + 1 : kPoolNumShapes); ++sh) {
        p->shape = sh;
        ffs_status r = upload_active(p);
        if (r != FFS_OK) return r;
        // the dense pass reads the current buffer and writes the other one,
        // which the next real step overwrites: repeating it changes no state
        POOL_CK((launch_pool_dense<T>(p->d_eps, p->d_act, p->parity, sh, p->grid_dense[sh], p->st)));
        POOL_CK(cudaEventRecord(p->ev0, p->st));
        for (int r2 = 0; r2 < 5; ++r2)
            POOL_CK((launch_pool_dense<T>(p->d_eps, p->d_act, p->parity, sh, p->grid_dense[sh], p->st)));
        POOL_CK(cudaEventRecord(p->ev1, p->st));
        POOL_CK(cudaEventSynchronize(p->ev1));
        float ms = 0.0f;
        POOL_CK(cudaEventElapsedTime(&ms, p->ev0, p->ev1));
        if (ms < best) { best = ms; best_shape = sh; }
    }
    p->shape = best_shape;
    p->act_dirty = true;
    p->tuned_cells = mix_cells(p);
    p->tuned_ms = best / 5.0;
    return FFS_OK;
}

ffs_status tune(ffs_pool *p)
{
    ffs_status r = wait_idle(p);
    if (r != FFS_OK) return r;
    switch (p->d.storage) {
    case FFS_STORAGE_F32: return tune_impl<float>(p);
    case FFS_STORAGE_F16: return tune_impl<__half>(p);
    default: return tune_impl<__nv_bfloat16>(p);
    }
}

template <typename T> ffs_status init_episode(ffs_pool *p, Slot &s, const float *bcvel)
{
    GridArgs<T> g{};
    g.nx = s.nx;
    g.ny = s.ny;
    g.nz = 1;
    g.ncell = (uint32_t)s.ncell;
    g.omega = s.dev.omega;
    g.codec = s.dev.codec;
    g.src = static_cast<const T *>(s.dev.mom[0]);
    g.dst = static_cast<T *>(s.dev.mom[0]);
    g.flags = s.dev.flags;
    g.wallmask = s.dev.wallmask;
    g.status = s.dev.status;
    POOL_CK((launch_initialize<2, T>(g, static_cast<T *>(s.dev.mom[1]), bcvel, p->st)));
    return FFS_OK;
}

ffs_status check_episode(const ffs_pool *p, const ffs_episode_desc *ep)
{
    if (!ep) return fail(FFS_ERR_INVALID_ARGUMENT, "null episode");
    const ffs_lbm_desc &d = ep->grid;
    const ffs_swimmer &w = ep->swimmer;
    if (d.dim != 2) return fail(FFS_ERR_UNSUPPORTED, "pool episodes are D2Q9 (dim 2)");
    if (d.nx <= 0 || d.ny <= 0) return fail(FFS_ERR_INVALID_ARGUMENT, "grid extents must be positive");
    if ((int64_t)d.nx * d.ny >= (int64_t)kPoolCellStride)
        return fail(FFS_ERR_UNSUPPORTED, "pool episodes hold fewer than 2^22 cells");
    if (!(d.fluid_viscosity > 0.0) || !(d.fluid_dx > 0.0) || !(d.dt > 0.0))
        return fail(FFS_ERR_INVALID_ARGUMENT, "viscosity, dx and dt must be positive");
    if (!ep->flags) return fail(FFS_ERR_INVALID_ARGUMENT, "episode flags are required");
    if (w.num_vertices <= 0 || w.num_elements <= 0 || !w.rest || !w.elements || !w.amplitude || !w.sin_kx ||
        !w.cos_kx)
        return fail(FFS_ERR_INVALID_ARGUMENT, "swimmer arrays are required");
    for (int v = 0; v < w.num_vertices && w.segment; ++v)
        if (w.segment[v] >= p->d.num_actions || w.segment[v] < -1)
            return fail(FFS_ERR_INVALID_ARGUMENT, "swimmer segment index outside the action vector");
    for (int e = 0; e < 2 * w.num_elements; ++e)
        if (w.elements[e] >= (uint32_t)w.num_vertices)
            return fail(FFS_ERR_INVALID_ARGUMENT, "swimmer element index outside the vertex array");
    return FFS_OK;
}

} // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

ffs_status ffs_pool_create(const ffs_pool_desc *desc, ffs_pool **out)
{
    if (!desc || !out) return fail(FFS_ERR_INVALID_ARGUMENT, "null descriptor or output");
    *out = nullptr;
    const ffs_pool_desc &d = *desc;
    if (d.storage < FFS_STORAGE_F32 || d.storage > FFS_STORAGE_BF16) return fail(FFS_ERR_INVALID_ARGUMENT, "bad storage");
    if (d.budget_bytes <= 0) return fail(FFS_ERR_INVALID_ARGUMENT, "budget_bytes must be positive");
    if (d.max_episodes < 1 || d.max_episodes > kPoolMaxSlots)
        return fail(FFS_ERR_INVALID_ARGUMENT, "max_episodes must be in 1..1000");
    if (d.substeps < 1 || d.substeps > kPoolMaxSubsteps) return fail(FFS_ERR_INVALID_ARGUMENT, "substeps must be in 1..64");
    if (d.num_actions < 0 || d.num_actions > kPoolMaxActions)
        return fail(FFS_ERR_INVALID_ARGUMENT, "num_actions must be in 0..16");
    ffs_pool *p = new (std::nothrow) ffs_pool();
    if (!p) return fail(FFS_ERR_OUT_OF_MEMORY, "host allocation failed");
    p->d = d;
    if (pinned_shape() >= 0) p->shape = pinned_shape();
    p->esize = d.storage == FFS_STORAGE_F32 ? 4 : 2;
    p->slots.resize(d.max_episodes);
    auto bail = [&](cudaError_t e, const char *what) {
        ffs_pool_destroy(p);
        return fail(e == cudaErrorMemoryAllocation ? FFS_ERR_OUT_OF_MEMORY : FFS_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return bail(e, "device");
    if ((e = cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return bail(e, "SMs");
    if (d.stream) {
        p->st = reinterpret_cast<cudaStream_t>(d.stream);
    } else {
        if ((e = cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
        p->own_stream = true;
    }
    if ((e = cudaMalloc(&p->arena_mem, (size_t)d.budget_bytes)) != cudaSuccess) return bail(e, "arena");
    p->arena.reset(p->arena_mem, (size_t)d.budget_bytes);
    if ((e = cudaMalloc(&p->d_eps, sizeof(PoolEpisode) * d.max_episodes)) != cudaSuccess) return bail(e, "episodes");
    if ((e = cudaMalloc(&p->d_prm, sizeof(PoolParams) * d.max_episodes)) != cudaSuccess) return bail(e, "params");
    for (int b = 0; b < 2; ++b)
        if ((e = cudaMallocHost(&p->h_prm[b], sizeof(PoolParams) * d.max_episodes)) != cudaSuccess) return bail(e, "params");
    if ((e = cudaMalloc(&p->d_act, sizeof(PoolActive))) != cudaSuccess) return bail(e, "active table");
    if ((e = cudaMallocHost(&p->h_act, sizeof(PoolActive))) != cudaSuccess) return bail(e, "active table");
    if ((e = cudaMalloc(&p->d_out, sizeof(PoolOutput) * d.max_episodes)) != cudaSuccess) return bail(e, "outputs");
    for (int b = 0; b < 2; ++b) {
        if ((e = cudaMallocHost(&p->h_out[b], sizeof(PoolOutput) * d.max_episodes)) != cudaSuccess)
            return bail(e, "outputs");
        std::memset(p->h_out[b], 0, sizeof(PoolOutput) * d.max_episodes);
    }
    std::memset(p->h_act, 0, sizeof(PoolActive));
    if ((e = cudaMemset(p->d_act, 0, sizeof(PoolActive))) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemset(p->d_out, 0, sizeof(PoolOutput) * d.max_episodes)) != cudaSuccess) return bail(e, "memset");
    // one link table for all episodes, keyed by slot * 2^22 + cell
    const int64_t link_cells = d.max_link_cells > 0 ? d.max_link_cells : (int64_t)2048 * d.max_episodes;
    uint64_t cap = 1024;
    while (cap < (uint64_t)link_cells * 2) cap <<= 1;
    if (cap > (1ull << 30)) return bail(cudaErrorInvalidValue, "link table too large");
    p->lt.cap = (uint32_t)cap;
    if ((e = cudaMalloc(&p->lt.keys, sizeof(uint32_t) * cap)) != cudaSuccess) return bail(e, "link keys");
    if ((e = cudaMalloc(&p->lt.links, sizeof(unsigned long long) * cap * 9)) != cudaSuccess) return bail(e, "links");
    if ((e = cudaMalloc(&p->lt.list, sizeof(uint32_t) * cap)) != cudaSuccess) return bail(e, "link list");
    if ((e = cudaMalloc(&p->lt.count, sizeof(uint32_t))) != cudaSuccess) return bail(e, "link count");
    if ((e = cudaMalloc(&p->owner, sizeof(uint32_t) * cap)) != cudaSuccess) return bail(e, "link owner");
    if ((e = cudaMemset(p->lt.keys, 0, sizeof(uint32_t) * cap)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemset(p->lt.links, 0xFF, sizeof(unsigned long long) * cap * 9)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemset(p->lt.count, 0, sizeof(uint32_t))) != cudaSuccess) return bail(e, "memset");
    p->lt.acc = nullptr; // per-episode accumulators live in the arena
    p->lt.acc_cap = 0;
    for (int sh = 0; sh < kPoolNumShapes; ++sh) {
        int b = 1;
        switch (d.storage) {
        case FFS_STORAGE_F32: b = pool_dense_blocks_per_sm<float>(sh); break;
        case FFS_STORAGE_F16: b = pool_dense_blocks_per_sm<__half>(sh); break;
        default: b = pool_dense_blocks_per_sm<__nv_bfloat16>(sh); break;
        }
        p->grid_dense[sh] = p->sms * b;
    }
    switch (d.storage) {
    case FFS_STORAGE_F32: p->grid_link = p->sms * pool_link_cells_blocks_per_sm<float>(); break;
    case FFS_STORAGE_F16: p->grid_link = p->sms * pool_link_cells_blocks_per_sm<__half>(); break;
    default: p->grid_link = p->sms * pool_link_cells_blocks_per_sm<__nv_bfloat16>(); break;
    }
    for (int b = 0; b < 2; ++b)
        if ((e = cudaEventCreateWithFlags(&p->done[b], cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
    if ((e = cudaEventCreateWithFlags(&p->act_sent, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
    if ((e = cudaEventCreate(&p->ev0)) != cudaSuccess) return bail(e, "event");
    if ((e = cudaEventCreate(&p->ev1)) != cudaSuccess) return bail(e, "event");
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(e, "create sync");
    *out = p;
    return FFS_OK;
}

ffs_status ffs_pool_destroy(ffs_pool *p)
{
    if (!p) return FFS_OK;
    if (p->st) cudaStreamSynchronize(p->st);
    for (auto &row : p->graph)
        for (auto &g : row)
            if (g) cudaGraphExecDestroy(g);
    for (int b = 0; b < 2; ++b)
        if (p->done[b]) cudaEventDestroy(p->done[b]);
    if (p->act_sent) cudaEventDestroy(p->act_sent);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    cudaFree(p->lt.keys); cudaFree(p->lt.links); cudaFree(p->lt.list); cudaFree(p->lt.count); cudaFree(p->owner);
    cudaFree(p->d_eps); cudaFree(p->d_prm); cudaFree(p->d_act); cudaFree(p->d_out); cudaFree(p->arena_mem);
    for (int b = 0; b < 2; ++b)
        if (p->h_prm[b]) cudaFreeHost(p->h_prm[b]);
    if (p->h_act) cudaFreeHost(p->h_act);
    for (int b = 0; b < 2; ++b)
        if (p->h_out[b]) cudaFreeHost(p->h_out[b]);
    if (p->own_stream && p->st) cudaStreamDestroy(p->st);
    delete p;
    return FFS_OK;
}

ffs_status ffs_pool_episode_bytes(const ffs_pool *p, const ffs_episode_desc *ep, int64_t *bytes)
{
    if (!p || !bytes) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    ffs_status r = check_episode(p, ep);
    if (r != FFS_OK) return r;
    *bytes = (int64_t)layout_of((int64_t)ep->grid.nx * ep->grid.ny, ep->swimmer.num_vertices,
                                ep->swimmer.num_elements, p->esize).total;
    return FFS_OK;
}

ffs_status ffs_pool_admit(ffs_pool *p, const ffs_episode_desc *ep, int *slot_out)
{
    if (!p || !slot_out) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    *slot_out = -1;
    ffs_status r = check_episode(p, ep);
    if (r != FFS_OK) return r;
    int si = -1;
    for (int i = 0; i < (int)p->slots.size(); ++i)
        if (!p->slots[i].used) { si = i; break; }
    if (si < 0) return fail(FFS_ERR_CAPACITY, "every episode slot is in use");
    const ffs_lbm_desc &d = ep->grid;
    const ffs_swimmer &w = ep->swimmer;
    const int64_t ncell = (int64_t)d.nx * d.ny;
    const Layout L = layout_of(ncell, w.num_vertices, w.num_elements, p->esize);
    size_t off = 0;
    if (!p->arena.alloc(L.total, &off))
        return fail(FFS_ERR_CAPACITY, "episode needs " + std::to_string(L.total) + " bytes; the pool has " +
                                          std::to_string(p->arena.largest()) + " contiguous bytes free");
    Slot &s = p->slots[si];
    s = Slot{};
    s.used = true;
    s.off = off;
    s.bytes = L.total;
    s.nx = d.nx;
    s.ny = d.ny;
    s.ncell = ncell;
    s.nv = w.num_vertices;
    s.ne = w.num_elements;
    s.omega_wave = w.omega;
    s.t0 = w.t0;
    s.dt = d.dt;
    char *b = p->arena.base + off;
    PoolEpisode &E = s.dev;
    E.nx = d.nx;
    E.ny = d.ny;
    E.ncell = (uint32_t)ncell;
    E.cell_base = (uint32_t)si * kPoolCellStride;
    // omega, Cf and the storage codec exactly as ffs_lbm_create forms them
    const float visf = (float)d.fluid_viscosity;
    E.omega = (float)(1.0 / ((double)visf * 3.0 + 0.5));
    E.cl = (float)d.fluid_dx;
    E.ct = (float)d.dt;
    const float cm = (float)(d.fluid_density * d.fluid_dx * d.fluid_dx);
    E.cf = (double)(float)((double)cm * d.fluid_dx / (d.dt * d.dt));
    const double tau = 3.0 * d.fluid_viscosity + 0.5;
    int k = (int)std::lround(std::log2(256.0 / tau));
    k = std::max(4, std::min(16, k));
    E.codec.su = 16.0f;
    E.codec.inv_su = 1.0f / 16.0f;
    E.codec.sp = std::ldexp(1.0f, k);
    E.codec.inv_sp = std::ldexp(1.0f, -k);
    E.mom[0] = b + L.mom0;
    E.mom[1] = b + L.mom1;
    E.flags = reinterpret_cast<uint8_t *>(b + L.flags);
    E.wallmask = reinterpret_cast<uint32_t *>(b + L.wallmask);
    E.status = reinterpret_cast<uint32_t *>(b + L.status);
    E.nv = w.num_vertices;
    E.ne = w.num_elements;
    E.rest = reinterpret_cast<const float *>(b + L.rest);
    E.amp = reinterpret_cast<const float *>(b + L.amp);
    E.sin_kx = reinterpret_cast<const float *>(b + L.sin_kx);
    E.cos_kx = reinterpret_cast<const float *>(b + L.cos_kx);
    E.segment = reinterpret_cast<const int32_t *>(b + L.segment);
    E.elements = reinterpret_cast<const uint32_t *>(b + L.elements);
    E.V = reinterpret_cast<float *>(b + L.V);
    E.U = reinterpret_cast<float *>(b + L.U);
    E.acc = reinterpret_cast<long long *>(b + L.acc);
    E.force = reinterpret_cast<double *>(b + L.force);
    E.sums = reinterpret_cast<double *>(b + L.sums);
    E.wave_omega = (float)w.omega;
    double cx = 0.0, cy = 0.0;
    for (int v = 0; v < w.num_vertices; ++v) { cx += w.rest[2 * v]; cy += w.rest[2 * v + 1]; }
    E.cx0 = (float)(cx / w.num_vertices);
    E.cy0 = (float)(cy / w.num_vertices);

    auto undo = [&](ffs_status st) {
        p->arena.release(s.off, s.bytes);
        s = Slot{};
        return st;
    };
    cudaStream_t st = p->st;
    const size_t nv = (size_t)w.num_vertices;
    std::vector<int32_t> seg(nv, -1);
    if (w.segment) std::memcpy(seg.data(), w.segment, sizeof(int32_t) * nv);
    cudaError_t e = cudaSuccess;
    auto cp = [&](void *dst, const void *src, size_t n) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st);
    };
    auto zero = [&](void *dst, size_t n) {
        if (e == cudaSuccess) e = cudaMemsetAsync(dst, 0, n, st);
    };
    zero(E.flags, ((size_t)ncell + 3) & ~(size_t)3);
    cp(E.flags, ep->flags, (size_t)ncell);
    zero(E.status, sizeof(uint32_t));
    cp(b + L.rest, w.rest, sizeof(float) * 2 * nv);
    cp(b + L.amp, w.amplitude, sizeof(float) * nv);
    cp(b + L.sin_kx, w.sin_kx, sizeof(float) * nv);
    cp(b + L.cos_kx, w.cos_kx, sizeof(float) * nv);
    cp(b + L.segment, seg.data(), sizeof(int32_t) * nv);
    cp(b + L.elements, w.elements, sizeof(uint32_t) * 2 * (size_t)w.num_elements);
    cp(E.V, w.rest, sizeof(float) * 2 * nv);
    zero(E.U, sizeof(float) * 2 * nv);
    zero(E.acc, sizeof(long long) * 2 * nv);
    zero(E.force, sizeof(double) * 2 * nv);
    zero(E.sums, sizeof(double) * 4);
    cp(p->d_eps + si, &E, sizeof(PoolEpisode));
    if (e != cudaSuccess) return undo(fail(FFS_ERR_CUDA, std::string("admission upload: ") + cudaGetErrorString(e)));
    if ((e = launch_prepare_flags<2>(E.flags, E.wallmask, d.nx, d.ny, 1, st)) != cudaSuccess)
        return undo(fail(FFS_ERR_CUDA, std::string("prepare flags: ") + cudaGetErrorString(e)));
    switch (p->d.storage) {
    case FFS_STORAGE_F32: r = init_episode<float>(p, s, d.boundary_velocities); break;
    case FFS_STORAGE_F16: r = init_episode<__half>(p, s, d.boundary_velocities); break;
    default: r = init_episode<__nv_bfloat16>(p, s, d.boundary_velocities); break;
    }
    if (r != FFS_OK) return undo(r);
    // pageable sources above are consumed before the calls return, but make
    // the admission complete before the caller reuses its arrays anyway
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
        return undo(fail(FFS_ERR_CUDA, std::string("admission: ") + cudaGetErrorString(e)));
    p->inflight[0] = p->inflight[1] = false;
    p->act_pending = false;
    p->order.push_back(si);
    p->act_dirty = true;
    *slot_out = si;
    return FFS_OK;
}

ffs_status ffs_pool_evict(ffs_pool *p, int slot)
{
    if (!p || slot < 0 || slot >= (int)p->slots.size() || !p->slots[slot].used)
        return fail(FFS_ERR_INVALID_ARGUMENT, "no such episode");
    Slot &s = p->slots[slot];
    p->arena.release(s.off, s.bytes);
    s = Slot{};
    p->order.erase(std::find(p->order.begin(), p->order.end(), slot));
    p->act_dirty = true;
    return FFS_OK;
}

ffs_status ffs_pool_set_action(ffs_pool *p, int slot, const float *actions, int n)
{
    if (!p || slot < 0 || slot >= (int)p->slots.size() || !p->slots[slot].used)
        return fail(FFS_ERR_INVALID_ARGUMENT, "no such episode");
    if (n < 0 || n > p->d.num_actions || (n > 0 && !actions))
        return fail(FFS_ERR_INVALID_ARGUMENT, "action vector longer than num_actions");
    for (int i = 0; i < n; ++i) p->slots[slot].actions[i] = actions[i];
    return FFS_OK;
}

ffs_status ffs_pool_set_actions(ffs_pool *p, int n, const int *slots, const float *actions)
{
    if (!p || n < 0 || (n > 0 && (!slots || !actions))) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    for (int i = 0; i < n; ++i)
        if (slots[i] < 0 || slots[i] >= (int)p->slots.size() || !p->slots[slots[i]].used)
            return fail(FFS_ERR_INVALID_ARGUMENT, "no such episode: slot " + std::to_string(slots[i]));
    const int na = p->d.num_actions;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < na; ++k) p->slots[slots[i]].actions[k] = actions[(size_t)i * na + k];
    return FFS_OK;
}

ffs_status ffs_pool_tune(ffs_pool *p)
{
    if (!p) return fail(FFS_ERR_INVALID_ARGUMENT, "null pool");
    return tune(p);
}

ffs_status ffs_pool_advance(ffs_pool *p)
{
    if (!p) return fail(FFS_ERR_INVALID_ARGUMENT, "null pool");
    if (p->order.empty()) return FFS_OK;
    // this step uses pinned buffer nb; wait only for the step that used it
    // last (two steps back), not for the previous one
    const int nb = (int)(p->advances & 1);
    ffs_status r = wait_buffer(p, nb);
    if (r != FFS_OK) return r;
    const int64_t cells = mix_cells(p);
    if (p->tuned_cells == 0 || cells > 2 * p->tuned_cells || 2 * cells < p->tuned_cells) {
        r = tune(p);
        if (r != FFS_OK) return r;
    }
    if (p->act_dirty) {
        r = upload_active(p);
        if (r != FFS_OK) return r;
    }
    const int S = p->d.substeps;
    for (size_t a = 0; a < p->order.size(); ++a) {
        Slot &s = p->slots[p->order[a]];
        PoolParams &P = p->h_prm[nb][a];
        std::memcpy(P.actions, s.actions, sizeof(P.actions));
        for (int j = 0; j < S; ++j) wave_phase(s.omega_wave, s.t0, s.dt, s.q + j, &P.sb[j], &P.cb[j]);
    }
    POOL_CK(cudaMemcpyAsync(p->d_prm, p->h_prm[nb], sizeof(PoolParams) * p->order.size(), cudaMemcpyHostToDevice,
                            p->st));
    cudaGraphExec_t &g = p->graph[p->shape][p->parity];
    if (!g) {
        // first use of this (shape, parity): capture with the stream idle
        if ((r = wait_idle(p)) != FFS_OK) return r;
        switch (p->d.storage) {
        case FFS_STORAGE_F32: r = capture<float>(p, p->shape, p->parity, &g); break;
        case FFS_STORAGE_F16: r = capture<__half>(p, p->shape, p->parity, &g); break;
        default: r = capture<__nv_bfloat16>(p, p->shape, p->parity, &g); break;
        }
        if (r != FFS_OK) return r;
    }
    POOL_CK(cudaGraphLaunch(g, p->st));
    POOL_CK(cudaMemcpyAsync(p->h_out[nb], p->d_out, sizeof(PoolOutput) * p->slots.size(), cudaMemcpyDeviceToHost,
                            p->st));
    POOL_CK(cudaEventRecord(p->done[nb], p->st));
    p->inflight[nb] = true;
    p->last = nb;
    p->parity ^= (S & 1);
    for (int si : p->order) p->slots[si].q += S;
    ++p->advances;
    return FFS_OK;
}

ffs_status ffs_pool_collect(ffs_pool *p, int slot, ffs_pool_output *out, double *forces)
{
    if (!p || slot < 0 || slot >= (int)p->slots.size() || !p->slots[slot].used)
        return fail(FFS_ERR_INVALID_ARGUMENT, "no such episode");
    ffs_status r = wait_idle(p);
    if (r != FFS_OK) return r;
    static_assert(sizeof(PoolOutput) == sizeof(ffs_pool_output), "output record layout");
    if (out) std::memcpy(out, p->h_out[p->last] + slot, sizeof(ffs_pool_output));
    if (forces) {
        const Slot &s = p->slots[slot];
        POOL_CK(cudaMemcpyAsync(forces, s.dev.force, sizeof(double) * 2 * s.nv, cudaMemcpyDeviceToHost, p->st));
        POOL_CK(cudaStreamSynchronize(p->st));
    }
    return FFS_OK;
}

ffs_status ffs_pool_collect_many(ffs_pool *p, int n, const int *slots, ffs_pool_output *out)
{
    if (!p || n < 0 || (n > 0 && (!slots || !out))) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    for (int i = 0; i < n; ++i)
        if (slots[i] < 0 || slots[i] >= (int)p->slots.size() || !p->slots[slots[i]].used)
            return fail(FFS_ERR_INVALID_ARGUMENT, "no such episode: slot " + std::to_string(slots[i]));
    ffs_status r = wait_idle(p);
    if (r != FFS_OK) return r;
    for (int i = 0; i < n; ++i) std::memcpy(out + i, p->h_out[p->last] + slots[i], sizeof(ffs_pool_output));
    return FFS_OK;
}

ffs_status ffs_pool_get_moments(ffs_pool *p, int slot, float *moments)
{
    if (!p || !moments || slot < 0 || slot >= (int)p->slots.size() || !p->slots[slot].used)
        return fail(FFS_ERR_INVALID_ARGUMENT, "no such episode");
    ffs_status r = wait_idle(p);
    if (r != FFS_OK) return r;
    const Slot &s = p->slots[slot];
    float *stage = nullptr;
    POOL_CK(cudaMalloc(&stage, sizeof(float) * 6 * (size_t)s.ncell));
    cudaError_t e;
    const void *src = s.dev.mom[p->parity];
    switch (p->d.storage) {
    case FFS_STORAGE_F32:
        e = launch_convert_out<2, float>(static_cast<const float *>(src), stage, true, (uint32_t)s.ncell, s.dev.codec, p->st);
        break;
    case FFS_STORAGE_F16:
        e = launch_convert_out<2, __half>(static_cast<const __half *>(src), stage, true, (uint32_t)s.ncell, s.dev.codec,
                                          p->st);
        break;
    default:
        e = launch_convert_out<2, __nv_bfloat16>(static_cast<const __nv_bfloat16 *>(src), stage, true,
                                                 (uint32_t)s.ncell, s.dev.codec, p->st);
        break;
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(moments, stage, sizeof(float) * 6 * (size_t)s.ncell, cudaMemcpyDeviceToHost, p->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->st);
    cudaFree(stage);
    if (e != cudaSuccess) return fail(FFS_ERR_CUDA, std::string("get_moments: ") + cudaGetErrorString(e));
    return FFS_OK;
}

ffs_status ffs_pool_get_info(const ffs_pool *p, ffs_pool_info *info)
{
    if (!p || !info) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    info->budget_bytes = p->d.budget_bytes;
    info->free_bytes = (int64_t)p->arena.free_bytes();
    info->largest_free_bytes = (int64_t)p->arena.largest();
    info->active_episodes = (int)p->order.size();
    const PoolTileShape sh = kPoolShapes[p->shape];
    int64_t tiles = 0;
    for (int si : p->order) {
        const Slot &s = p->slots[si];
        tiles += (int64_t)((s.nx + sh.tx - 1) / sh.tx) * ((s.ny + sh.ty - 1) / sh.ty);
    }
    info->tiles = (int)tiles;
    info->tile_x = sh.tx;
    info->tile_y = sh.ty;
    info->strip = sh.strip ? 1 : 0;
    info->advances = p->advances;
    info->graph_builds = p->graph_builds;
    info->cells = mix_cells(p);
    info->tuned_cells = p->tuned_cells;
    info->dense_ms = p->tuned_ms;
    return FFS_OK;
}

ffs_status ffs_swimmer_surface(const ffs_swimmer *sw, const float *actions, int num_actions, int64_t q, double dt,
                               float *vertices, float *velocities)
{
    if (!sw || !vertices || !velocities || (num_actions > 0 && !actions) || num_actions < 0 ||
        num_actions > kPoolMaxActions)
        return fail(FFS_ERR_INVALID_ARGUMENT, "bad swimmer surface arguments");
    float act[kPoolMaxActions] = {};
    for (int i = 0; i < num_actions; ++i) act[i] = actions[i];
    float sb, cb;
    wave_phase(sw->omega, sw->t0, dt, q, &sb, &cb);
    const float wom = (float)sw->omega;
    for (int v = 0; v < sw->num_vertices; ++v) {
        const int seg = sw->segment ? sw->segment[v] : -1;
        if (seg >= num_actions) return fail(FFS_ERR_INVALID_ARGUMENT, "swimmer segment index outside the action vector");
        swimmer_vertex(sw->rest[2 * v], sw->rest[2 * v + 1], sw->amplitude[v], sw->sin_kx[v], sw->cos_kx[v], seg, act,
                       sb, cb, wom, vertices[2 * v], vertices[2 * v + 1], velocities[2 * v], velocities[2 * v + 1]);
    }
    return FFS_OK;
}

} // extern "C"
