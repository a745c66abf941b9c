// C ABI of the fluid step (include/ffs_lbm.h): grid objects, their device
// memory, and the per-step launch sequence.
//
// Per step, on the caller's stream and without host synchronisation:
//   1. detect_links   (only with a surface)   O(surface), on a side stream,
//                                             concurrent with 2
//   2. dense2d/dense3d                         O(grid), the bandwidth-bound pass
//   3. link_cells     (only with a surface)   O(boundary cells), after 1 and 2
//   4. finalize_forces(only with a surface)   O(vertices); folded into the
//                                             last CTA of 3 for small surfaces
// then the host flips the current buffer, exactly where the reference calls
// flow_field.swapMoments() (FsiCoupling2D.cu:419, FsiCoupling3D.cu:476).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "ffs_lbm.h"
#include "ffs_common.cuh"
#include "ffs_dense2d.cuh"
#include "ffs_dense3d.cuh"
#include "ffs_links.cuh"

using namespace fflbm;

struct ffs_lbm {
    ffs_lbm_desc d;
    int dim = 2, Q = 9, NM = 6;
    int64_t ncell = 0;
    size_t esize = 4;
    void *mom[2] = {nullptr, nullptr};
    int cur = 0;
    uint8_t *flags = nullptr; // padded to a multiple of 4 bytes
    uint32_t *wallmask = nullptr;
    uint32_t *status = nullptr;
    float omega = 1.0f;
    double cf = 1.0;
    float cl = 1.0f, ct = 1.0f;
    Codec codec{};
    LinkTable lt;
    float *staging = nullptr; // ncell * NM floats, allocated on first host transfer
    uint32_t *fill_bits = nullptr; // D3Q27 solid fill: one parity bit per cell, zero between calls
    int dense_variant = -1;   // D3Q27 kernel variant chosen on the first step (tune_dense3d)
    // link detection runs on `side` while the dense pass runs on the caller's
    // stream; fork/join order them
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // stage timing (ffs_lbm_profile_*)
    int profiling = 0;  // 0 off, 1 stage events, 2 stage events with detection serialised
    struct Mark { int stage; cudaEvent_t a, b; };
    std::vector<Mark> marks;
    std::vector<cudaEvent_t> event_pool;
    double prof_ms[4] = {0, 0, 0, 0};
    int64_t prof_n[4] = {0, 0, 0, 0};
};

namespace {

thread_local std::string g_last_error;

ffs_status fail(ffs_status s, const std::string &msg)
{
    g_last_error = msg;
    return s;
}

} // namespace

// Error reporting shared with the other C-ABI translation units (ffs_pool.cu).
namespace fflbm {
ffs_status record_error(ffs_status s, const std::string &msg) { return fail(s, msg); }
} // namespace fflbm

namespace {

#define FFS_CK(expr)                                                                                                    \
    do {                                                                                                                \
        cudaError_t e_ = (expr);                                                                                        \
        if (e_ != cudaSuccess) return fail(FFS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));           \
    } while (0)

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

uint32_t next_pow2(uint64_t v)
{
    uint64_t p = 1;
    while (p < v) p <<= 1;
    return (uint32_t)std::min<uint64_t>(p, 1ull << 31);
}

template <typename T> GridArgs<T> args(ffs_lbm *h)
{
    GridArgs<T> g;
    g.nx = h->d.nx;
    g.ny = h->d.ny;
    g.nz = h->dim == 2 ? 1 : h->d.nz;
    g.ncell = (uint32_t)h->ncell;
    g.periodic = h->d.periodic_mask;
    g.half_pops = h->dim == 2 ? h->d.ref_half_populations : 0;
    g.wall_stream = h->dim == 2 ? h->d.ref_2d_wall_stream : 0;
    g.omega = h->omega;
    g.codec = h->codec;
    g.src = static_cast<const T *>(h->mom[h->cur]);
    g.dst = static_cast<T *>(h->mom[1 - h->cur]);
    g.flags = h->flags;
    g.wallmask = h->wallmask;
    g.status = h->status;
    return g;
}

void free_links(LinkTable &lt)
{
    cudaFree(lt.keys); cudaFree(lt.links); cudaFree(lt.list); cudaFree(lt.count); cudaFree(lt.acc);
    lt = LinkTable{};
}

ffs_status ensure_links(ffs_lbm *h, int64_t max_vertices, int64_t max_link_cells)
{
    LinkTable &lt = h->lt;
    uint32_t want_cap = next_pow2((uint64_t)std::max<int64_t>(max_link_cells, 1024) * 2);
    if (lt.cap < want_cap) {
        // a new table starts empty; the old one is empty between steps
        cudaFree(lt.keys); cudaFree(lt.links); cudaFree(lt.list);
        lt.keys = nullptr; lt.links = nullptr; lt.list = nullptr;
        FFS_CK(cudaMalloc(&lt.keys, sizeof(uint32_t) * want_cap));
        FFS_CK(cudaMalloc(&lt.links, sizeof(unsigned long long) * (size_t)want_cap * h->Q));
        FFS_CK(cudaMalloc(&lt.list, sizeof(uint32_t) * want_cap));
        FFS_CK(cudaMemset(lt.keys, 0, sizeof(uint32_t) * want_cap));
        FFS_CK(cudaMemset(lt.links, 0xFF, sizeof(unsigned long long) * (size_t)want_cap * h->Q));
        lt.cap = want_cap;
    }
    if (!lt.count) {
        // the list count and the finished-CTA count of link_cells_kernel
        FFS_CK(cudaMalloc(&lt.count, 2 * sizeof(uint32_t)));
        FFS_CK(cudaMemset(lt.count, 0, 2 * sizeof(uint32_t)));
        lt.done = lt.count + 1;
    }
    if ((int64_t)lt.acc_cap < max_vertices) {
        cudaFree(lt.acc);
        lt.acc = nullptr;
        FFS_CK(cudaMalloc(&lt.acc, sizeof(long long) * (size_t)max_vertices * h->dim));
        FFS_CK(cudaMemset(lt.acc, 0, sizeof(long long) * (size_t)max_vertices * h->dim));
        lt.acc_cap = (uint32_t)max_vertices;
    }
    return FFS_OK;
}

// link cells a surface can own at most: every element's grown bounding box,
// bounded by the grid; a generous default for the on-demand path
int64_t default_link_cells(const ffs_lbm *h, int64_t num_elements)
{
    int64_t per = h->dim == 2 ? 12 : 40;
    return std::min<int64_t>(num_elements * per + 4096, h->ncell);
}

ffs_status check_surface(const ffs_lbm *h, const ffs_surface *s)
{
    if (!s) return FFS_OK;
    if (s->num_elements < 0 || s->num_vertices < 0) return fail(FFS_ERR_INVALID_ARGUMENT, "negative surface size");
    if (s->num_elements == 0) return FFS_OK;
    if (s->dim != h->dim) return fail(FFS_ERR_INVALID_ARGUMENT, "surface dim differs from grid dim");
    if (!s->vertices || !s->velocities || !s->elements)
        return fail(FFS_ERR_INVALID_ARGUMENT, "surface arrays must be device pointers");
    if (s->num_elements > 0 && s->num_vertices <= 0) return fail(FFS_ERR_INVALID_ARGUMENT, "surface has no vertices");
    return FFS_OK;
}

SurfaceArgs surface_args(const ffs_surface *s)
{
    SurfaceArgs a{};
    if (s) {
        a.V = s->vertices; a.U = s->velocities; a.E = s->elements;
        a.nv = s->num_vertices; a.ne = s->num_elements;
        a.forces = s->forces; a.forces64 = s->forces64;
    }
    return a;
}

cudaEvent_t take_event(ffs_lbm *h)
{
    if (!h->event_pool.empty()) {
        cudaEvent_t e = h->event_pool.back();
        h->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Records an event pair around one stage when profiling is on.
struct StageTimer {
    ffs_lbm *h;
    int stage;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    StageTimer(ffs_lbm *h_, int stage_, cudaStream_t st_) : h(h_), stage(stage_), st(st_)
    {
        if (h->profiling) {
            a = take_event(h);
            cudaEventRecord(a, st);
        }
    }
    ~StageTimer()
    {
        if (a) {
            cudaEvent_t b = take_event(h);
            cudaEventRecord(b, st);
            h->marks.push_back({stage, a, b});
        }
    }
};

template <int DIM, typename T> ffs_status step_impl(ffs_lbm *h, const SurfaceArgs &sa, cudaStream_t st)
{
    GridArgs<T> g = args<T>(h);
    const bool surf = sa.ne > 0;
    StepScalars sc{h->cl, h->ct, h->cf};
    uint32_t *words = reinterpret_cast<uint32_t *>(h->flags);
    const bool serial = h->profiling == 2;
    if (DIM == 3 && h->dense_variant < 0) h->dense_variant = tune_dense3d<T>(g, st);
    if (surf) {
        if (h->lt.cap == 0 || (int64_t)h->lt.acc_cap < sa.nv) {
            ffs_status r = ensure_links(h, std::max<int64_t>(sa.nv, h->lt.acc_cap),
                                        std::max<int64_t>(default_link_cells(h, sa.ne), h->lt.cap / 2));
            if (r != FFS_OK) return r;
        }
        // Link detection and the dense pass overlap: the dense pass skips
        // cells whose LINK bit it sees, but any link cell it does update is
        // rewritten by link_cells, which runs after both.  Serial profiling
        // runs detection on the caller's stream first, so that each stage's
        // events time that stage alone (same results: the order only
        // changes which link cells the dense pass skips).
        const cudaStream_t ds = serial ? st : h->side;
        if (!serial) {
            FFS_CK(cudaEventRecord(h->fork, st));
            FFS_CK(cudaStreamWaitEvent(h->side, h->fork, 0));
        }
        {
            StageTimer t(h, 0, ds);
            FFS_CK((launch_detect_links<DIM, T>(g, words, h->lt, sa, sc, ds)));
        }
        if (!serial) FFS_CK(cudaEventRecord(h->join, h->side));
    }
    {
        StageTimer t(h, 1, st);
        if (DIM == 2) FFS_CK(launch_dense2d<T>(g, st));
        else FFS_CK(launch_dense3d<T>(g, st, h->dense_variant));
    }
    if (surf) {
        if (!serial) FFS_CK(cudaStreamWaitEvent(st, h->join, 0));
        const bool fold = (long long)sa.nv * DIM <= kFoldForcesMax;
        {
            StageTimer t(h, 2, st);
            FFS_CK((launch_link_cells<DIM, T>(g, words, h->lt, sa, sc, st, fold)));
        }
        if (!fold) {
            StageTimer t(h, 3, st);
            FFS_CK(launch_finalize_forces<DIM>(h->lt, sa, h->cf, st));
        }
    }
    h->cur ^= 1;
    return FFS_OK;
}

template <int DIM> ffs_status step_dim(ffs_lbm *h, const SurfaceArgs &sa, cudaStream_t st)
{
    switch (h->d.storage) {
    case FFS_STORAGE_F32: return step_impl<DIM, float>(h, sa, st);
    case FFS_STORAGE_F16: return step_impl<DIM, __half>(h, sa, st);
    default: return step_impl<DIM, __nv_bfloat16>(h, sa, st);
    }
}

template <int DIM, typename T> ffs_status init_impl(ffs_lbm *h, cudaStream_t st)
{
    h->cur = 0;
    GridArgs<T> g = args<T>(h);
    g.dst = static_cast<T *>(h->mom[0]);
    FFS_CK((launch_initialize<DIM, T>(g, static_cast<T *>(h->mom[1]), h->d.boundary_velocities, st)));
    return FFS_OK;
}

template <int DIM, typename T> cudaError_t conv_in(ffs_lbm *h, const float *src, bool aos, void *dst, cudaStream_t st)
{
    return launch_convert_in<DIM, T>(src, aos, static_cast<T *>(dst), (uint32_t)h->ncell, h->codec, st);
}
template <int DIM, typename T> cudaError_t conv_out(ffs_lbm *h, const void *src, float *dst, bool aos, cudaStream_t st)
{
    return launch_convert_out<DIM, T>(static_cast<const T *>(src), dst, aos, (uint32_t)h->ncell, h->codec, st);
}

cudaError_t convert_in(ffs_lbm *h, const float *src, bool aos, void *dst, cudaStream_t st)
{
    if (h->dim == 2) {
        if (h->d.storage == FFS_STORAGE_F32) return conv_in<2, float>(h, src, aos, dst, st);
        if (h->d.storage == FFS_STORAGE_F16) return conv_in<2, __half>(h, src, aos, dst, st);
        return conv_in<2, __nv_bfloat16>(h, src, aos, dst, st);
    }
    if (h->d.storage == FFS_STORAGE_F32) return conv_in<3, float>(h, src, aos, dst, st);
    if (h->d.storage == FFS_STORAGE_F16) return conv_in<3, __half>(h, src, aos, dst, st);
    return conv_in<3, __nv_bfloat16>(h, src, aos, dst, st);
}

cudaError_t convert_out(ffs_lbm *h, const void *src, float *dst, bool aos, cudaStream_t st)
{
    if (h->dim == 2) {
        if (h->d.storage == FFS_STORAGE_F32) return conv_out<2, float>(h, src, dst, aos, st);
        if (h->d.storage == FFS_STORAGE_F16) return conv_out<2, __half>(h, src, dst, aos, st);
        return conv_out<2, __nv_bfloat16>(h, src, dst, aos, st);
    }
    if (h->d.storage == FFS_STORAGE_F32) return conv_out<3, float>(h, src, dst, aos, st);
    if (h->d.storage == FFS_STORAGE_F16) return conv_out<3, __half>(h, src, dst, aos, st);
    return conv_out<3, __nv_bfloat16>(h, src, dst, aos, st);
}

ffs_status ensure_staging(ffs_lbm *h)
{
    if (!h->staging) FFS_CK(cudaMalloc(&h->staging, sizeof(float) * (size_t)h->ncell * h->NM));
    return FFS_OK;
}

int which_index(const ffs_lbm *h, int which)
{
    switch (which) {
    case FFS_BUF_CURRENT: return h->cur;
    case FFS_BUF_NEXT: return 1 - h->cur;
    case FFS_BUF_A: return 0;
    case FFS_BUF_B: return 1;
    default: return -1;
    }
}

ffs_status prepare_flags(ffs_lbm *h, cudaStream_t st)
{
    if (h->dim == 2) FFS_CK(launch_prepare_flags<2>(h->flags, h->wallmask, h->d.nx, h->d.ny, 1, st));
    else FFS_CK(launch_prepare_flags<3>(h->flags, h->wallmask, h->d.nx, h->d.ny, h->d.nz, st));
    return FFS_OK;
}

} // namespace

extern "C" {

int ffs_abi_version(void) { return FFS_ABI_VERSION; }

const char *ffs_last_error(void) { return g_last_error.c_str(); }

const char *ffs_status_string(ffs_status s)
{
    switch (s) {
    case FFS_OK: return "ok";
    case FFS_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FFS_ERR_OUT_OF_MEMORY: return "out of device memory";
    case FFS_ERR_CUDA: return "CUDA error";
    case FFS_ERR_CAPACITY: return "capacity exceeded";
    case FFS_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

ffs_status ffs_lbm_create(const ffs_lbm_desc *desc, ffs_lbm **out)
{
    if (!desc || !out) return fail(FFS_ERR_INVALID_ARGUMENT, "null descriptor or output");
    *out = nullptr;
    const ffs_lbm_desc &d = *desc;
    if (d.dim != 2 && d.dim != 3) return fail(FFS_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
    const int nz = d.dim == 2 ? 1 : d.nz;
    if (d.nx <= 0 || d.ny <= 0 || nz <= 0) return fail(FFS_ERR_INVALID_ARGUMENT, "grid extents must be positive");
    const int64_t ncell = (int64_t)d.nx * d.ny * nz;
    if (ncell >= (int64_t)1 << 31) return fail(FFS_ERR_UNSUPPORTED, "grids of 2^31 cells or more are not supported");
    if (d.storage < FFS_STORAGE_F32 || d.storage > FFS_STORAGE_BF16) return fail(FFS_ERR_INVALID_ARGUMENT, "bad storage");
    if (!(d.fluid_viscosity > 0.0) || !(d.fluid_dx > 0.0) || !(d.dt > 0.0))
        return fail(FFS_ERR_INVALID_ARGUMENT, "viscosity, dx and dt must be positive");
    if (d.ref_2d_wall_stream != 0 && d.ref_2d_wall_stream != 1)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ref_2d_wall_stream must be 0 or 1");
    ffs_lbm *h = new (std::nothrow) ffs_lbm();
    if (!h) return fail(FFS_ERR_OUT_OF_MEMORY, "host allocation failed");
    h->d = d;
    h->d.nz = nz;
    h->dim = d.dim;
    h->Q = d.dim == 2 ? 9 : 27;
    h->NM = d.dim == 2 ? 6 : 10;
    h->ncell = ncell;
    h->esize = d.storage == FFS_STORAGE_F32 ? 4 : 2;
    // omega = 1 / (3 nu + 1/2) formed in double from the float m_viscosity
    // (LbmFlowField2D.hpp:177; FsiCoupling2D.cu:236, FsiCoupling3D.cu:303)
    const float visf = (float)d.fluid_viscosity;
    h->omega = (float)(1.0 / ((double)visf * 3.0 + 0.5));
    // getCf (Config.hpp:96-100, :154-158), a float in the reference
    const float cm = (float)(d.dim == 2 ? d.fluid_density * d.fluid_dx * d.fluid_dx
                                        : d.fluid_density * d.fluid_dx * d.fluid_dx * d.fluid_dx);
    h->cf = (double)(float)((double)cm * d.fluid_dx / (d.dt * d.dt));
    h->cl = (float)d.fluid_dx;
    h->ct = (float)d.dt;
    // reduced-precision scales: u * 16, (pi - u u) * 2^k with k from tau so
    // that typical non-equilibrium stress sits in fp16's normal range
    const double tau = 3.0 * d.fluid_viscosity + 0.5;
    int k = (int)std::lround(std::log2(256.0 / tau));
    k = std::max(4, std::min(16, k));
    h->codec.su = 16.0f;
    h->codec.inv_su = 1.0f / 16.0f;
    h->codec.sp = std::ldexp(1.0f, k);
    h->codec.inv_sp = std::ldexp(1.0f, -k);

    auto bail = [&](cudaError_t e, const char *what) {
        ffs_lbm_destroy(h);
        return fail(e == cudaErrorMemoryAllocation ? FFS_ERR_OUT_OF_MEMORY : FFS_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
    };
    const size_t mbytes = h->esize * (size_t)ncell * h->NM;
    cudaError_t e;
    if ((e = cudaMalloc(&h->mom[0], mbytes)) != cudaSuccess) return bail(e, "moments A");
    if ((e = cudaMalloc(&h->mom[1], mbytes)) != cudaSuccess) return bail(e, "moments B");
    const size_t fbytes = ((size_t)ncell + 3) & ~(size_t)3;
    if ((e = cudaMalloc(&h->flags, fbytes)) != cudaSuccess) return bail(e, "flags");
    if ((e = cudaMalloc(&h->wallmask, sizeof(uint32_t) * (size_t)ncell)) != cudaSuccess) return bail(e, "wallmask");
    if ((e = cudaMalloc(&h->status, sizeof(uint32_t))) != cudaSuccess) return bail(e, "status");
    if ((e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    if ((e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
    if ((e = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
    if ((e = cudaMemset(h->mom[0], 0, mbytes)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemset(h->mom[1], 0, mbytes)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemset(h->flags, 0, fbytes)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemset(h->wallmask, 0, sizeof(uint32_t) * (size_t)ncell)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemset(h->status, 0, sizeof(uint32_t))) != cudaSuccess) return bail(e, "memset");
    // all cells Fluid (LbmInitializer2D.cu:103)
    std::vector<uint8_t> f((size_t)ncell, (uint8_t)kFluid);
    if ((e = cudaMemcpy(h->flags, f.data(), (size_t)ncell, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "flags upload");
    ffs_status st = prepare_flags(h, nullptr);
    if (st != FFS_OK) { ffs_lbm_destroy(h); return st; }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(e, "create sync");
    *out = h;
    return FFS_OK;
}

ffs_status ffs_lbm_destroy(ffs_lbm *h)
{
    if (!h) return FFS_OK;
    for (auto &m : h->marks) { cudaEventDestroy(m.a); cudaEventDestroy(m.b); }
    for (auto e : h->event_pool) cudaEventDestroy(e);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    if (h->side) cudaStreamDestroy(h->side);
    cudaFree(h->mom[0]); cudaFree(h->mom[1]); cudaFree(h->flags); cudaFree(h->wallmask); cudaFree(h->status);
    cudaFree(h->staging);
    cudaFree(h->fill_bits);
    free_links(h->lt);
    delete h;
    return FFS_OK;
}

ffs_status ffs_lbm_set_flags(ffs_lbm *h, const uint8_t *flags, int memory, void *stream)
{
    if (!h || !flags) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    cudaStream_t st = S(stream);
    if (memory == FFS_MEM_HOST) {
        for (int64_t c = 0; c < h->ncell; ++c)
            if (flags[c] > kSmoke) return fail(FFS_ERR_INVALID_ARGUMENT, "flag value is not an LbmNodeFlag");
        FFS_CK(cudaMemcpyAsync(h->flags, flags, (size_t)h->ncell, cudaMemcpyHostToDevice, st));
    } else if (memory == FFS_MEM_DEVICE) {
        FFS_CK(cudaMemcpyAsync(h->flags, flags, (size_t)h->ncell, cudaMemcpyDeviceToDevice, st));
    } else {
        return fail(FFS_ERR_INVALID_ARGUMENT, "memory must be FFS_MEM_HOST or FFS_MEM_DEVICE");
    }
    ffs_status r = prepare_flags(h, st);
    if (r != FFS_OK) return r;
    if (memory == FFS_MEM_HOST) FFS_CK(cudaStreamSynchronize(st));
    return FFS_OK;
}

ffs_status ffs_lbm_get_flags(ffs_lbm *h, uint8_t *flags, int memory, void *stream)
{
    if (!h || !flags) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    cudaStream_t st = S(stream);
    std::vector<uint8_t> tmp((size_t)h->ncell);
    FFS_CK(cudaMemcpyAsync(tmp.data(), h->flags, (size_t)h->ncell, cudaMemcpyDeviceToHost, st));
    FFS_CK(cudaStreamSynchronize(st));
    for (auto &v : tmp) v &= kTypeMask;
    if (memory == FFS_MEM_HOST) std::memcpy(flags, tmp.data(), tmp.size());
    else {
        FFS_CK(cudaMemcpyAsync(flags, tmp.data(), tmp.size(), cudaMemcpyHostToDevice, st));
        FFS_CK(cudaStreamSynchronize(st));
    }
    return FFS_OK;
}

ffs_status ffs_lbm_initialize(ffs_lbm *h, void *stream)
{
    if (!h) return fail(FFS_ERR_INVALID_ARGUMENT, "null grid");
    cudaStream_t st = S(stream);
    if (h->dim == 2) {
        if (h->d.storage == FFS_STORAGE_F32) return init_impl<2, float>(h, st);
        if (h->d.storage == FFS_STORAGE_F16) return init_impl<2, __half>(h, st);
        return init_impl<2, __nv_bfloat16>(h, st);
    }
    if (h->d.storage == FFS_STORAGE_F32) return init_impl<3, float>(h, st);
    if (h->d.storage == FFS_STORAGE_F16) return init_impl<3, __half>(h, st);
    return init_impl<3, __nv_bfloat16>(h, st);
}

ffs_status ffs_lbm_set_moments(ffs_lbm *h, const float *m, int layout, int memory, int which, void *stream)
{
    if (!h || !m) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    if (layout != FFS_LAYOUT_AOS && layout != FFS_LAYOUT_SOA) return fail(FFS_ERR_INVALID_ARGUMENT, "bad layout");
    cudaStream_t st = S(stream);
    const float *src = m;
    if (memory == FFS_MEM_HOST) {
        ffs_status r = ensure_staging(h);
        if (r != FFS_OK) return r;
        FFS_CK(cudaMemcpyAsync(h->staging, m, sizeof(float) * (size_t)h->ncell * h->NM, cudaMemcpyHostToDevice, st));
        src = h->staging;
    } else if (memory != FFS_MEM_DEVICE) {
        return fail(FFS_ERR_INVALID_ARGUMENT, "bad memory kind");
    }
    const bool aos = layout == FFS_LAYOUT_AOS;
    if (which == FFS_BUF_BOTH) {
        FFS_CK(convert_in(h, src, aos, h->mom[0], st));
        FFS_CK(convert_in(h, src, aos, h->mom[1], st));
    } else {
        int b = which_index(h, which);
        if (b < 0) return fail(FFS_ERR_INVALID_ARGUMENT, "bad buffer selector");
        FFS_CK(convert_in(h, src, aos, h->mom[b], st));
    }
    if (memory == FFS_MEM_HOST) FFS_CK(cudaStreamSynchronize(st));
    return FFS_OK;
}

ffs_status ffs_lbm_get_moments(ffs_lbm *h, float *m, int layout, int memory, int which, void *stream)
{
    if (!h || !m) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    if (layout != FFS_LAYOUT_AOS && layout != FFS_LAYOUT_SOA) return fail(FFS_ERR_INVALID_ARGUMENT, "bad layout");
    int b = which_index(h, which);
    if (b < 0) return fail(FFS_ERR_INVALID_ARGUMENT, "bad buffer selector");
    cudaStream_t st = S(stream);
    const bool aos = layout == FFS_LAYOUT_AOS;
    if (memory == FFS_MEM_DEVICE) {
        FFS_CK(convert_out(h, h->mom[b], m, aos, st));
        return FFS_OK;
    }
    if (memory != FFS_MEM_HOST) return fail(FFS_ERR_INVALID_ARGUMENT, "bad memory kind");
    ffs_status r = ensure_staging(h);
    if (r != FFS_OK) return r;
    FFS_CK(convert_out(h, h->mom[b], h->staging, aos, st));
    FFS_CK(cudaMemcpyAsync(m, h->staging, sizeof(float) * (size_t)h->ncell * h->NM, cudaMemcpyDeviceToHost, st));
    FFS_CK(cudaStreamSynchronize(st));
    return FFS_OK;
}

ffs_status ffs_lbm_reserve_surface(ffs_lbm *h, int max_vertices, int max_link_cells)
{
    if (!h || max_vertices < 0 || max_link_cells < 0) return fail(FFS_ERR_INVALID_ARGUMENT, "bad reservation");
    return ensure_links(h, max_vertices, max_link_cells);
}

ffs_status ffs_lbm_step(ffs_lbm *h, const ffs_surface *s, void *stream)
{
    if (!h) return fail(FFS_ERR_INVALID_ARGUMENT, "null grid");
    ffs_status r = check_surface(h, s);
    if (r != FFS_OK) return r;
    const SurfaceArgs sa = surface_args(s);
    return h->dim == 2 ? step_dim<2>(h, sa, S(stream)) : step_dim<3>(h, sa, S(stream));
}

ffs_status ffs_lbm_step_coupled(ffs_lbm *h, const ffs_volume_surface *s, void *stream)
{
    if (!h || !s) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    if (s->dim != h->dim) return fail(FFS_ERR_INVALID_ARGUMENT, "surface dim differs from grid dim");
    if (s->num_vertices < 0 || s->num_elements < 0 || s->num_volume_vertices < 0)
        return fail(FFS_ERR_INVALID_ARGUMENT, "negative surface size");
    if (s->num_vertices > 0 && (!s->volume_positions || !s->volume_velocities || !s->surface_to_volume ||
                                !s->surface_positions || !s->surface_velocities))
        return fail(FFS_ERR_INVALID_ARGUMENT, "surface arrays must be device pointers");
    if (s->num_elements > 0 && (!s->elements || s->num_vertices <= 0))
        return fail(FFS_ERR_INVALID_ARGUMENT, "surface has elements but no vertices");
    if (s->num_volume_vertices > 0 && !s->volume_forces)
        return fail(FFS_ERR_INVALID_ARGUMENT, "volume_forces must be a device pointer");
    cudaStream_t st = S(stream);
    FFS_CK(launch_gather_surface(h->dim, s->volume_positions, s->volume_velocities, s->surface_to_volume,
                                 s->num_vertices, s->num_volume_vertices, s->surface_positions, s->surface_velocities,
                                 s->volume_forces, h->status, st));
    SurfaceArgs sa{};
    sa.V = s->surface_positions; sa.U = s->surface_velocities; sa.E = s->elements;
    sa.nv = s->num_vertices; sa.ne = s->num_elements;
    sa.map = s->surface_to_volume; sa.vforces = s->volume_forces; sa.nvol = s->num_volume_vertices;
    return h->dim == 2 ? step_dim<2>(h, sa, st) : step_dim<3>(h, sa, st);
}

ffs_status ffs_lbm_fill_solid(ffs_lbm *h, const ffs_surface *s, void *stream)
{
    if (!h || !s) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    ffs_status r = check_surface(h, s);
    if (r != FFS_OK) return r;
    cudaStream_t st = S(stream);
    if (h->dim == 2) {
        FFS_CK(launch_fill_solid2(h->flags, h->d.nx, h->d.ny, h->cl, surface_args(s), st));
    } else {
        if (!h->fill_bits) {
            const size_t bytes = sizeof(uint32_t) * (size_t)h->d.ny * h->d.nz * ((h->d.nx + 31) / 32);
            FFS_CK(cudaMalloc(&h->fill_bits, bytes));
            FFS_CK(cudaMemsetAsync(h->fill_bits, 0, bytes, st));
        }
        FFS_CK(launch_fill_solid3(h->flags, h->fill_bits, h->d.nx, h->d.ny, h->d.nz, h->cl, surface_args(s), st));
    }
    return prepare_flags(h, st);
}

ffs_status ffs_lbm_get_status(ffs_lbm *h, uint32_t *status, int clear, void *stream)
{
    if (!h || !status) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    cudaStream_t st = S(stream);
    FFS_CK(cudaMemcpyAsync(status, h->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    if (clear) FFS_CK(cudaMemsetAsync(h->status, 0, sizeof(uint32_t), st));
    FFS_CK(cudaStreamSynchronize(st));
    return FFS_OK;
}

ffs_status ffs_lbm_get_info(ffs_lbm *h, int64_t *ncell, int *nm, int *q, double *omega, double *cf)
{
    if (!h) return fail(FFS_ERR_INVALID_ARGUMENT, "null grid");
    if (ncell) *ncell = h->ncell;
    if (nm) *nm = h->NM;
    if (q) *q = h->Q;
    if (omega) *omega = h->omega;
    if (cf) *cf = h->cf;
    return FFS_OK;
}

ffs_status ffs_lbm_debug_links(ffs_lbm *h, const ffs_surface *s, uint64_t *cell_dir, uint64_t *key, int64_t capacity,
                               int64_t *count, void *stream)
{
    if (!h || !s || !count) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    ffs_status r = check_surface(h, s);
    if (r != FFS_OK) return r;
    *count = 0;
    if (s->num_elements == 0) return FFS_OK;
    cudaStream_t st = S(stream);
    r = ensure_links(h, std::max<int64_t>(s->num_vertices, h->lt.acc_cap),
                     std::max<int64_t>(default_link_cells(h, s->num_elements), h->lt.cap / 2));
    if (r != FFS_OK) return r;
    SurfaceArgs sa = surface_args(s);
    StepScalars sc{h->cl, h->ct, h->cf};
    uint32_t *words = reinterpret_cast<uint32_t *>(h->flags);
    if (h->dim == 2) FFS_CK((launch_detect_links<2, float>(args<float>(h), words, h->lt, sa, sc, st)));
    else FFS_CK((launch_detect_links<3, float>(args<float>(h), words, h->lt, sa, sc, st)));
    uint32_t n = 0;
    FFS_CK(cudaMemcpyAsync(&n, h->lt.count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    FFS_CK(cudaStreamSynchronize(st));
    std::vector<uint32_t> list(n), keys(h->lt.cap);
    std::vector<unsigned long long> links((size_t)h->lt.cap * h->Q);
    if (n) FFS_CK(cudaMemcpyAsync(list.data(), h->lt.list, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
    FFS_CK(cudaMemcpyAsync(keys.data(), h->lt.keys, sizeof(uint32_t) * h->lt.cap, cudaMemcpyDeviceToHost, st));
    FFS_CK(cudaMemcpyAsync(links.data(), h->lt.links, sizeof(unsigned long long) * links.size(), cudaMemcpyDeviceToHost, st));
    FFS_CK(cudaStreamSynchronize(st));
    std::vector<std::pair<uint64_t, uint64_t>> out;
    for (uint32_t w = 0; w < n; ++w) {
        uint32_t slot = list[w];
        uint64_t cell = keys[slot] - 1;
        for (int l = 0; l < h->Q; ++l) {
            unsigned long long k = links[(size_t)slot * h->Q + l];
            if (k != ~0ull) out.emplace_back(cell * h->Q + l, k);
        }
    }
    std::sort(out.begin(), out.end());
    *count = (int64_t)out.size();
    for (int64_t i = 0; i < (int64_t)out.size() && i < capacity; ++i) {
        if (cell_dir) cell_dir[i] = out[i].first;
        if (key) key[i] = out[i].second;
    }
    if (h->dim == 2) FFS_CK(launch_reset_links<2>(h->lt, words, st));
    else FFS_CK(launch_reset_links<3>(h->lt, words, st));
    FFS_CK(cudaStreamSynchronize(st));
    return FFS_OK;
}

ffs_status ffs_lbm_profile_enable(ffs_lbm *h, int enable)
{
    if (!h) return fail(FFS_ERR_INVALID_ARGUMENT, "null grid");
    if (enable < 0 || enable > 2) return fail(FFS_ERR_INVALID_ARGUMENT, "profile mode must be 0, 1 or 2");
    h->profiling = enable;
    return FFS_OK;
}

ffs_status ffs_lbm_profile_read(ffs_lbm *h, ffs_profile *out, int reset)
{
    if (!h || !out) return fail(FFS_ERR_INVALID_ARGUMENT, "null argument");
    for (auto &m : h->marks) {
        FFS_CK(cudaEventSynchronize(m.b));
        float ms = 0.0f;
        FFS_CK(cudaEventElapsedTime(&ms, m.a, m.b));
        h->prof_ms[m.stage] += ms;
        h->prof_n[m.stage] += 1;
        h->event_pool.push_back(m.a);
        h->event_pool.push_back(m.b);
    }
    h->marks.clear();
    for (int i = 0; i < 4; ++i) { out->ms[i] = h->prof_ms[i]; out->launches[i] = h->prof_n[i]; }
    if (reset)
        for (int i = 0; i < 4; ++i) { h->prof_ms[i] = 0.0; h->prof_n[i] = 0; }
    return FFS_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// ffs_lbm_step_noalloc: ffs_lbm_step with its moving-boundary scratch (link
// table and per-vertex force accumulators) in a fixed device array of this
// library instead of memory from cudaMalloc.  It allocates nothing, ever: no
// cudaMalloc/cudaFree, no pool or library allocation.
//
// Callers that cannot allocate while stepping:
//  * hosts that reserved their device memory up front and admitted work
//    against that budget (a serving process packing many episodes into HBM,
//    or a caller whose pool allocator already holds the free memory): a
//    cudaMalloc in mid-run can fail with out-of-memory there;
//  * latency-bound step loops that share the device with other streams:
//    cudaMalloc/cudaFree synchronise the whole device and stall them.
// ffs_lbm_step allocates its scratch on the first step with a surface (and
// again for a larger one); this entry point never does.
//
// Scratch layout (one array shared by every grid and every call on a device;
// the table has twice as many slots as the supported link cells, so it is at
// most half full, like the table ffs_lbm_step sizes for itself):
//   keys  [kNoallocSlots]  u32, 0 = empty slot          must start at 0
//   list  [kNoallocSlots]  u32, claimed slots            no requirement
//   count, done u32 (own 256-byte line)                  must start at 0
//   links [kNoallocSlots * Q] u64, ~0 = no link          must start at ~0
//   acc   [kNoallocMaxVertices * DIM] i64 force sums     must start at 0
// Every call clears all four on its stream before its first kernel, so a
// call never depends on the previous one having finished cleanly.  Calls
// that overlap in time on one device (two streams, two threads, two grids)
// race on the array: the caller orders them.
namespace {

constexpr uint32_t kNoallocMaxLinkCells = 16384;          // link cells per step supported
constexpr uint32_t kNoallocSlots = 2 * kNoallocMaxLinkCells; // table slots (full at 32,768 link cells)
constexpr uint32_t kNoallocMaxVertices = 32768;           // surface vertices at most
constexpr size_t kNoallocKeysOff = 0;
constexpr size_t kNoallocListOff = kNoallocKeysOff + sizeof(uint32_t) * kNoallocSlots;
constexpr size_t kNoallocCountOff = kNoallocListOff + sizeof(uint32_t) * kNoallocSlots;
constexpr size_t kNoallocLinksOff = kNoallocCountOff + 256;
constexpr size_t kNoallocAccOff = kNoallocLinksOff + sizeof(unsigned long long) * kNoallocSlots * 27;
constexpr size_t kNoallocBytes = kNoallocAccOff + sizeof(long long) * kNoallocMaxVertices * 3; // 8,126,720
static_assert(kNoallocLinksOff % 256 == 0 && kNoallocAccOff % 256 == 0, "scratch sections stay 256-byte aligned");
static_assert((kNoallocSlots & (kNoallocSlots - 1)) == 0, "the link table wants a power-of-two slot count");
static_assert(kNoallocBytes == 8126720, "the header states the scratch size");
static_assert(kNoallocMaxLinkCells == FFS_NOALLOC_MAX_LINK_CELLS && kNoallocMaxVertices == FFS_NOALLOC_MAX_VERTICES,
              "limits as the header states them");

constexpr int kNoallocMaxDevices = 64;

} // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

namespace {

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_base[kNoallocMaxDevices] = {};

// Address of the scratch array on the current device, looked up once per
// device (the lookup may load this library's device code on that device).
// A cudaDeviceReset discards that code and with it the array, so the cached
// address is only valid until the device is reset (the header says so).
ffs_status noalloc_scratch(unsigned char **out)
{
    int dev = -1;
    FFS_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoallocMaxDevices) return fail(FFS_ERR_UNSUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
        unsigned char *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(FFS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_base[dev] = p;
    }
    *out = g_noalloc_base[dev];
    return FFS_OK;
}

template <int DIM, typename T> ffs_status noalloc_impl(ffs_lbm *h, const ffs_surface *s, unsigned char *base,
                                                       cudaStream_t st)
{
    constexpr int Q = Lattice<DIM>::Q;
    GridArgs<T> g = args<T>(h);
    const bool surf = s && s->num_elements > 0;
    SurfaceArgs sa = surface_args(s);
    StepScalars sc{h->cl, h->ct, h->cf};
    uint32_t *words = reinterpret_cast<uint32_t *>(h->flags);
    LinkTable lt;
    if (surf) {
        lt.cap = kNoallocSlots;
        lt.keys = reinterpret_cast<uint32_t *>(base + kNoallocKeysOff);
        lt.list = reinterpret_cast<uint32_t *>(base + kNoallocListOff);
        lt.count = reinterpret_cast<uint32_t *>(base + kNoallocCountOff);
        lt.done = lt.count + 1; // same 256-byte line, cleared with it
        lt.links = reinterpret_cast<unsigned long long *>(base + kNoallocLinksOff);
        lt.acc = reinterpret_cast<long long *>(base + kNoallocAccOff);
        lt.acc_cap = kNoallocMaxVertices;
        FFS_CK(cudaMemsetAsync(base, 0, kNoallocLinksOff, st)); // keys, list, count
        FFS_CK(cudaMemsetAsync(lt.links, 0xFF, sizeof(unsigned long long) * kNoallocSlots * Q, st));
        FFS_CK(cudaMemsetAsync(lt.acc, 0, sizeof(long long) * (size_t)s->num_vertices * DIM, st));
        // detection on the grid's side stream, beside the dense pass, as in
        // step_impl (the streams and events exist since the grid was created)
        FFS_CK(cudaEventRecord(h->fork, st));
        FFS_CK(cudaStreamWaitEvent(h->side, h->fork, 0));
        FFS_CK((launch_detect_links<DIM, T>(g, words, lt, sa, sc, h->side)));
        FFS_CK(cudaEventRecord(h->join, h->side));
    }
    if (DIM == 2) FFS_CK(launch_dense2d<T>(g, st));
    else FFS_CK(launch_dense3d<T>(g, st, h->dense_variant < 0 ? 0 : h->dense_variant));
    if (surf) {
        FFS_CK(cudaStreamWaitEvent(st, h->join, 0));
        const bool fold = (long long)sa.nv * DIM <= kFoldForcesMax;
        FFS_CK((launch_link_cells<DIM, T>(g, words, lt, sa, sc, st, fold)));
        if (!fold) FFS_CK(launch_finalize_forces<DIM>(lt, sa, h->cf, st));
    }
    h->cur ^= 1;
    return FFS_OK;
}

template <int DIM> ffs_status noalloc_dim(ffs_lbm *h, const ffs_surface *s, unsigned char *base, cudaStream_t st)
{
    switch (h->d.storage) {
    case FFS_STORAGE_F32: return noalloc_impl<DIM, float>(h, s, base, st);
    case FFS_STORAGE_F16: return noalloc_impl<DIM, __half>(h, s, base, st);
    default: return noalloc_impl<DIM, __nv_bfloat16>(h, s, base, st);
    }
}

} // namespace

extern "C" ffs_status ffs_lbm_step_noalloc(ffs_lbm *h, const ffs_surface *s, void *stream)
{
    if (!h) return fail(FFS_ERR_INVALID_ARGUMENT, "null grid");
    ffs_status r = check_surface(h, s);
    if (r != FFS_OK) return r;
    if (s && s->num_elements > 0 && (uint32_t)s->num_vertices > kNoallocMaxVertices)
        return fail(FFS_ERR_CAPACITY, "ffs_lbm_step_noalloc: " + std::to_string(s->num_vertices) +
                                          " surface vertices exceed its fixed scratch (at most " +
                                          std::to_string(kNoallocMaxVertices) + "); use ffs_lbm_step");
    unsigned char *base = nullptr;
    r = noalloc_scratch(&base);
    if (r != FFS_OK) return r;
    return h->dim == 2 ? noalloc_dim<2>(h, s, base, S(stream)) : noalloc_dim<3>(h, s, base, S(stream));
}
