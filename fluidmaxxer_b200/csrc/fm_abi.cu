// fm_abi.cu -- the C ABI of include/fm.h: lattice context, boundary-list
// set-up, the per-step launch schedule, getters and FP64 reductions.
//
// The host logic mirrors the reference's lattice/operator classes
// (include/core/lattice/NSLattice.hpp, include/core/lattice/ADLattice.hpp,
// include/boundary/**, include/reaction/**) and the loop order of
// src/main.cpp:319-357; the arithmetic lives in fm_kernels.cuh.
#include "../../include/fm.h"
#include "fm_kernels.cuh"
#include "fm_pair.cuh"
#include "fm_adjoint.cuh"

#include <cuda_runtime.h>
#if defined(__SSE2__) && !defined(__CUDA_ARCH__)
#include <emmintrin.h>
#define FM_SCAN_SSE2 1
#endif

#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace fm_internal {
// The driver's handle of the context current on this thread (null when the
// driver entry point is unavailable), looked up through the runtime so the
// library has no link-time dependency on the driver library.  Caches of
// per-device state compare it to notice a new context (after cudaDeviceReset).
__attribute__((visibility("hidden"))) void* current_context()
{
    using GetCurrent = int (*)(void**);
    static GetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        cudaGetLastError();
        return reinterpret_cast<GetCurrent>(p);
    }();
    void* ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}
}  // namespace fm_internal

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

#define FM_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(FM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

#define FM_CHECK_LAUNCH(what)                                                                  \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess)                                                                 \
            return fail(FM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_));       \
    } while (0)

constexpr int kBlock = 256;
// default L2 prefetch distance of the fused kernel: 54% of one resident wave
// (148 SMs x 5 blocks -> ~400 blocks), the best of a sweep at 512x256x256
constexpr int kPrefetchWavePct = 54;
inline int grid_for(long long n, int block = kBlock) { return (int)((n + block - 1) / block); }

enum BcKind { BC_NS_VEL_EQ, BC_NS_VEL_NEQ, BC_NS_PRESSURE, BC_NS_BOUNCEBACK, BC_AD_DIRICHLET, BC_AD_PULSE, BC_AD_NEUMANN };

struct Bc {
    int kind = 0;
    int* cells = nullptr;   // device list
    int* nei = nullptr;     // device list (NEQ inward neighbours)
    int count = 0;
    double v[5] = {0, 0, 0, 0, 0};
    int iv[2] = {0, 0};
};

}  // namespace

struct fm_lattice {
    fm_params p{};
    int precision = FM_F32;
    int n = 0;
    long long ns = 0;
    size_t nwords = 0;
    size_t elt = 4;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    void* f[2] = {nullptr, nullptr};
    void* g[2] = {nullptr, nullptr};
    int cur = 0;
    void* phi = nullptr;                // R per cell (R = float, or double for FM_F64)
    void* q = nullptr;
    size_t qelt = 4;
    uint32_t* solid = nullptr;
    uint32_t* region = nullptr;
    uint32_t* defer = nullptr;
    void* por = nullptr;                // R per cell
    void* tau = nullptr;                // R per cell
    bool tau_field = false;
    bool collision_set = false;
    int collision = FM_COLL_BGK;
    int coupling = 1;
    int isotherm = FM_ISO_NONE;
    double iso[3] = {0, 0, 0};
    std::vector<Bc> ns_pre, ns_post, ad_pre, ad_post;
    int* deferred = nullptr;
    int ndeferred = 0;
    int* probe = nullptr;
    int nprobe = 0;
    int probe_every = 0;
    double* d_bt = nullptr;
    int bt_cap = 0;
    int bt_count = 0;
    double* d_acc = nullptr;   // 8 doubles of reduction scratch
    void* d_tmp = nullptr;     // 4 planes of R for field getters
    long long step = 0;
    bool initialised = false;
    double f_shift = 0.0, g_shift = 0.0;
    size_t relt = 4;                    // bytes of the arithmetic type R
    int fuse_inlet = 0;                 // NEQ inlet on the full x = 0 plane, inside the fused kernel
    int inlet_state = 0;                // 1: f[cur] at x = 0 holds next-step NEQ values, x0post the populations
    void* x0post = nullptr;             // [19][rows_stride] in the population storage type
    uint32_t rows_stride = 0;
    uint32_t* cellw = nullptr;          // per-cell flag words (k_build_flags)
    bool dirty = true;                  // flags / fusion need rebuilding
    bool split_open = false;            // a step begun by fm_step_planes, not yet finished
    int fuse_outlet = 0, fuse_neumann = 0, fuse_dirichlet = 0;
    uint32_t pf_dist = 0;               // L2 prefetch distance of the fused kernel (blocks)
    bool pf_set = false;                // pf_dist fixed by fm_set_tuning
    double rho_out = 1.0, c_in = 0.0;
    bool profiling = false;
    double* d_wide = nullptr;           // FP64 staging plane of the field getters
    char* adj_arena = nullptr;          // adjoint workspace, kept between fm_adjoint_breakthrough calls
    size_t adj_bytes = 0;
    long long adj_forward_steps = 0;    // forward steps recomputed by the last adjoint call
    std::vector<cudaEvent_t> prof_ev;   // pairs: start, stop
    size_t prof_used = 0;               // events recorded since the last read
    int mon_every = 0;                  // step monitor period (fm_set_monitor; 0 = off)
    double* d_mon_part = nullptr;       // per-block partials of a monitored launch [blocks][kMonN]
    double* d_mon = nullptr;            // the monitor's rows [mon_cap][kMonN]
    int mon_cap = 0;
    std::vector<long long> mon_steps;   // step of each row
    int layout = 0;                     // storage of f[cur], g[cur]: 0 natural, 1 pair layout (fm_pair.cuh)
    int pair_pref = 0;                  // use the pair layout where it applies (fm_set_pair_layout; off by default)
    int in_batch = 0;                   // batches holding this lattice (they step the natural layout)
    int staged_pref = 1;                // pair layout: the staged kernel where it applies (fm_set_pair_kernel)
    int staged_grid[4] = {0, 0, 0, 0};  // its resident blocks (persistent grid) per variant: BGK / porous x monitored
    size_t staged_smem[4] = {0, 0, 0, 0};   // ... and the shared memory they were sized for
    int* d_status = nullptr;            // device status word of the step kernels (fm_step_status)
};

namespace {

// Device memory comes from a stream-ordered pool the library creates for each
// device (the device's default pool and its settings stay the host
// application's).  The pool keeps up to half of the device memory mapped when
// it is freed, so a lattice created after another reuses memory that is
// already mapped: plain cudaMalloc / cudaFree map and unmap it every time,
// which took 10-250 ms per 512x256x256 lattice and varied from call to call.
// fm_trim_memory hands the kept memory back.  A new context of the device
// (after cudaDeviceReset) gets a new pool.
struct PoolSlot {
    cudaMemPool_t pool = nullptr;
    void* ctx = nullptr;
};
std::mutex g_pool_mutex;
PoolSlot g_pools[64];

cudaError_t library_pool(cudaMemPool_t* out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    PoolSlot& s = g_pools[dev];
    void* ctx = fm_internal::current_context();
    if (!s.pool || (ctx && ctx != s.ctx)) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            uint64_t keep = total_b / 2;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        s.pool = pool;
        s.ctx = ctx ? ctx : fm_internal::current_context();
    }
    *out = s.pool;
    return cudaSuccess;
}

// Device memory from the library's own pool on `st`, then `st` is synchronised,
// so the memory is usable from any stream afterwards.
template <typename T>
int dev_alloc(T** p, size_t count, cudaStream_t st)
{
    *p = nullptr;
    if (count == 0) return FM_OK;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = library_pool(&pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void**)p, count * sizeof(T), pool, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(FM_ERR_NOMEM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
    }
    return FM_OK;
}

// Back to the pool in the order of `st`: after the work queued on `st` (the
// stream of the lattice or batch that owns p, on which all work using p runs
// or is joined), without synchronising the host or the device.
void dev_free(void* p, cudaStream_t st)
{
    if (!p) return;
    cudaFreeAsync(p, st);
}

int check_lattice(const fm_lattice* L)
{
    if (!L) return fail(FM_ERR_ARG, "null lattice");
    return FM_OK;
}

int check_mask(const fm_lattice* L, const void* mask, size_t n, const char* who)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!mask) return fail(FM_ERR_ARG, std::string(who) + ": null mask");
    if (n != (size_t)L->n) return fail(FM_ERR_ARG, std::string(who) + " mask mismatch");
    return FM_OK;
}

// 8 mask bytes -> 8 bits, bit i set iff byte i is nonzero: (x & 0x7f) + 0x7f
// sets the high bit of every byte with a low bit set (no carry leaves a
// byte), "| x" adds bytes with only the high bit; the multiply moves the
// high bit of byte i to bit 56 + i without carries into the top byte
inline uint32_t nonzero8(const uint8_t* p)
{
    uint64_t x;
    std::memcpy(&x, p, 8);
    const uint64_t lo7 = 0x7f7f7f7f7f7f7f7full, hi = 0x8080808080808080ull;
    const uint64_t t = (((x & lo7) + lo7) | x) & hi;
    return (uint32_t)(((t >> 7) * 0x0102040810204080ull) >> 56);
}

// 32 mask bytes -> 32 bits, bit i set iff byte i is nonzero (x86-64: two
// byte compares and movemasks; elsewhere four nonzero8)
inline uint32_t nonzero32(const uint8_t* p)
{
#ifdef FM_SCAN_SSE2
    const __m128i z = _mm_setzero_si128();
    const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(p));
    const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(p + 16));
    const uint32_t za = (uint32_t)_mm_movemask_epi8(_mm_cmpeq_epi8(a, z));
    const uint32_t zb = (uint32_t)_mm_movemask_epi8(_mm_cmpeq_epi8(b, z));
    return ~(za | zb << 16);
#else
    return nonzero8(p) | nonzero8(p + 8) << 8 | nonzero8(p + 16) << 16 | nonzero8(p + 24) << 24;
#endif
}

// Host worker threads for the set-up scans, started once and reused: starting
// and joining 16 threads per mask call cost about as much as the scan itself.
// A process forked after the threads started gets a new pool (the workers of
// the parent do not exist in the child).  Calls from several host threads at
// once take turns.
class HostPool {
public:
    static constexpr size_t kMax = 16;
    static HostPool& get()
    {
        static std::mutex m;
        static HostPool* pool = nullptr;
        std::lock_guard<std::mutex> lock(m);
        if (!pool || pool->pid_ != getpid()) pool = new HostPool();   // a forked child's pool is new
        return *pool;
    }
    size_t size() const { return nthreads_ + 1; }
    // runs job(t) for t in [0, nt), nt <= size(); the caller runs t = 0
    void run(size_t nt, const std::function<void(size_t)>& job)
    {
        std::lock_guard<std::mutex> one(call_);
        {
            std::lock_guard<std::mutex> lock(m_);
            job_ = &job;
            active_ = nt;
            pending_ = nt - 1;
            ++gen_;
        }
        cv_.notify_all();
        job(0);
        std::unique_lock<std::mutex> lock(m_);
        done_.wait(lock, [&] { return pending_ == 0; });
        job_ = nullptr;
    }

private:
    HostPool() : pid_(getpid())
    {
        nthreads_ = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), kMax) - 1;
        for (size_t i = 0; i < nthreads_; ++i) std::thread([this, i] { loop(i + 1); }).detach();
    }
    void loop(size_t t)
    {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(size_t)>* job = nullptr;
            {
                std::unique_lock<std::mutex> lock(m_);
                cv_.wait(lock, [&] { return gen_ != seen; });
                seen = gen_;
                if (t < active_) job = job_;
            }
            if (!job) continue;
            (*job)(t);
            std::lock_guard<std::mutex> lock(m_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    pid_t pid_;
    size_t nthreads_ = 0;
    std::mutex call_, m_;
    std::condition_variable cv_, done_;
    const std::function<void(size_t)>* job_ = nullptr;
    size_t active_ = 0, pending_ = 0;
    uint64_t gen_ = 0;
};

// Run body(lo, hi, t) over [0, n) in contiguous chunks on up to 16 host
// threads (one chunk below 64K elements): the set-up scans of full-lattice
// byte masks.
template <typename F>
void parallel_chunks(size_t n, F body)
{
    const size_t min_chunk = (size_t)1 << 16;
    HostPool& pool = HostPool::get();
    const size_t nt = std::max<size_t>(1, std::min(pool.size(), n / min_chunk));
    if (nt <= 1) {
        body(0, n, 0);
        return;
    }
    const size_t per = (n + nt - 1) / nt;
    const std::function<void(size_t)> job = [&](size_t t) {
        const size_t lo = std::min(n, t * per), hi = std::min(n, lo + per);
        body(lo, hi, t);
    };
    pool.run(nt, job);
}

std::vector<uint32_t> pack_bits(const uint8_t* m, size_t n, size_t nwords)
{
    std::vector<uint32_t> b(nwords, 0u);
    const size_t full = n / 32;
    parallel_chunks(full, [&](size_t lo, size_t hi, size_t) {
        for (size_t w = lo; w < hi; ++w) {
            const uint8_t* p = m + 32 * w;
            b[w] = nonzero32(p);
        }
    });
    for (size_t c = 32 * full; c < n; ++c)
        if (m[c]) b[c >> 5] |= 1u << (c & 31);
    return b;
}

int upload_list(const std::vector<int>& h, int** d, cudaStream_t st)
{
    if (h.empty()) { *d = nullptr; return FM_OK; }
    int rc = dev_alloc(d, h.size(), st);
    if (rc) return rc;
    FM_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    FM_CUDA(cudaStreamSynchronize(st));
    return FM_OK;
}

// indices of the nonzero bytes, in order (8 bytes per test, so sparse masks
// such as boundary planes cost one load and compare per 8 cells)
std::vector<int> compress(const uint8_t* m, size_t n)
{
    const size_t groups = n / 32;
    std::vector<std::vector<int>> part(16);
    parallel_chunks(groups, [&](size_t lo, size_t hi, size_t t) {
        std::vector<int>& v = part[t];
        for (size_t g = lo; g < hi; ++g) {
            uint32_t bits = nonzero32(m + 32 * g);
            while (bits) {
                v.push_back((int)(32 * g + (size_t)__builtin_ctz(bits)));
                bits &= bits - 1u;
            }
        }
    });
    std::vector<int> v;
    size_t total = 0;
    for (const auto& p : part) total += p.size();
    v.reserve(total + 8);
    for (const auto& p : part) v.insert(v.end(), p.begin(), p.end());
    for (size_t c = 32 * groups; c < n; ++c)
        if (m[c]) v.push_back((int)c);
    return v;
}

bool is_full_x_plane(const fm_lattice* L, const Bc& b, int x)
{
    if (b.count != L->p.ny * L->p.nz) return false;
    std::vector<int> h((size_t)b.count);
    if (cudaMemcpyAsync(h.data(), b.cells, h.size() * sizeof(int), cudaMemcpyDeviceToHost, L->stream) != cudaSuccess ||
        cudaStreamSynchronize(L->stream) != cudaSuccess)
        return false;
    for (size_t i = 0; i < h.size(); ++i)
        if (h[i] != x + L->p.nx * (int)i) return false;   // lists are in cell order: (x, y, z) with y fastest
    return true;
}

// Decide which boundary planes the fused kernel handles, build the list of
// cells whose AD update must follow the remaining post-stream NS boundaries,
// and build the per-cell flag words.  Runs before the first step after any
// change of geometry, region or boundaries.
int prepare(fm_lattice* L)
{
    if (!L->dirty) return FM_OK;
    const int nx = L->p.nx;
    // a full x = nx-1 plane can be fused when its x-1 neighbour is always the
    // previous lane of the same warp: every row ends at an odd cell index,
    // which holds for even nx
    const bool lanes_ok = nx >= 3 && nx % 2 == 0;
    L->fuse_outlet = 0;
    if (lanes_ok && L->ns_post.size() == 1 && L->ns_post[0].kind == BC_NS_PRESSURE &&
        is_full_x_plane(L, L->ns_post[0], nx - 1)) {
        L->fuse_outlet = 1;
        L->rho_out = L->ns_post[0].v[0];
    }
    L->fuse_neumann = 0;
    L->fuse_dirichlet = 0;
    {
        int nd = 0, nn = 0;
        bool planes = true;
        for (const Bc& b : L->ad_post) {
            if (b.kind == BC_AD_DIRICHLET) { ++nd; planes = planes && is_full_x_plane(L, b, 0); }
            else { ++nn; planes = planes && is_full_x_plane(L, b, nx - 1); }
        }
        // the in-kernel AD planes need every AD update in the fused kernel:
        // no cell may be deferred behind a list-path NS boundary
        const bool no_deferred = L->fuse_outlet || L->ns_post.empty();
        if (planes && nd <= 1 && nn <= 1 && lanes_ok && no_deferred) {
            for (const Bc& b : L->ad_post) {
                if (b.kind == BC_AD_DIRICHLET) { L->fuse_dirichlet = 1; L->c_in = b.v[0]; }
                else L->fuse_neumann = 1;
            }
        }
    }
    // the NEQ inlet plane: the x = 1 lane computes next step's x = 0 values in
    // the fused kernel; needs its final populations, so no list-path NS
    // boundary may rewrite x = 1 after the collision
    L->fuse_inlet = 0;
    if (lanes_ok && L->ns_pre.size() == 1 && L->ns_pre[0].kind == BC_NS_VEL_NEQ &&
        is_full_x_plane(L, L->ns_pre[0], 0) && (L->fuse_outlet || L->ns_post.empty())) {
        L->fuse_inlet = 1;
        if (!L->x0post) {
            L->rows_stride = (uint32_t)(((long long)L->p.ny * L->p.nz + 31) / 32 * 32);
            int rc0 = dev_alloc((char**)&L->x0post, (size_t)19 * L->rows_stride * L->elt, L->stream);
            if (rc0) return rc0;
        }
    }
    // deferred AD cells: those a non-fused post-stream NS boundary rewrites
    dev_free(L->deferred, L->stream);
    L->deferred = nullptr;
    L->ndeferred = 0;
    int rc = 0;
    bool any_deferred = false;
    if (!L->fuse_outlet)
        for (const Bc& b : L->ns_post) any_deferred = any_deferred || b.count > 0;
    if (any_deferred) {
        std::vector<uint8_t> mark((size_t)L->n, 0);
        for (const Bc& b : L->ns_post) {
            std::vector<int> h((size_t)b.count);
            if (b.count) {
                FM_CUDA(cudaMemcpyAsync(h.data(), b.cells, h.size() * sizeof(int), cudaMemcpyDeviceToHost, L->stream));
                FM_CUDA(cudaStreamSynchronize(L->stream));
            }
            for (int c : h) mark[(size_t)c] = 1;
        }
        std::vector<int> list = compress(mark.data(), mark.size());
        L->ndeferred = (int)list.size();
        rc = upload_list(list, &L->deferred, L->stream);
        if (rc) return rc;
        if (!L->defer) {
            rc = dev_alloc(&L->defer, L->nwords, L->stream);
            if (rc) return rc;
        }
        std::vector<uint32_t> bits = pack_bits(mark.data(), mark.size(), L->nwords);
        FM_CUDA(cudaMemcpyAsync(L->defer, bits.data(), bits.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, L->stream));
        FM_CUDA(cudaStreamSynchronize(L->stream));
    }
    if (!L->cellw) {
        rc = dev_alloc(&L->cellw, (size_t)L->ns, L->stream);
        if (rc) return rc;
    }
    fm::k_build_flags<<<grid_for(L->n), kBlock, 0, L->stream>>>(
        L->cellw, L->solid, L->isotherm != FM_ISO_NONE ? L->region : nullptr, L->ndeferred ? L->defer : nullptr, L->n,
        L->p.nx, L->p.ny, L->p.nz, L->p.periodic_x != 0, L->p.periodic_y != 0, L->p.periodic_z != 0,
        fm::fastdiv_magic((uint32_t)L->p.nx), fm::fastdiv_magic((uint32_t)(L->p.nx * L->p.ny)),
        L->collision == FM_COLL_BGK);
    FM_CHECK_LAUNCH("k_build_flags");
    if (!L->pf_set) {
        // FP32: about half a resident wave ahead.  FP64 and the 16-bit forms:
        // none.  Measured on 33.5M-cell lattices of three shapes, the prefetch
        // made FP64 17-20% and the 16-bit forms 5-9% slower; on 4M-cell
        // lattices it gained at most 4% (FP64, 40 blocks) and 1% (16-bit).
        int dev = 0, sms = 148;
        const int per_sm = 5;   // resident 256-thread blocks at 48 registers
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        L->pf_dist = L->elt == 4 ? (uint32_t)(kPrefetchWavePct * sms * per_sm / 100) : 0u;
    }
    L->dirty = false;
    return FM_OK;
}

template <typename T, typename QT>
fm::StepArgs<T, QT> make_args(const fm_lattice* L)
{
    using R = typename fm::Pop<T>::R;
    fm::StepArgs<T, QT> a{};
    const int A = L->cur, B = 1 - L->cur;
    a.fA = (const T*)L->f[A];
    a.fB = (T*)L->f[B];
    a.gA = (const T*)L->g[A];
    a.gB = (T*)L->g[B];
    a.phi = (R*)L->phi;
    a.q = (QT*)L->q;
    a.cellw = L->cellw;
    a.porosity = (const R*)L->por;
    a.tau_ad = L->tau_field ? (const R*)L->tau : nullptr;
    a.div_nx = fm::fastdiv_magic((uint32_t)L->p.nx);
    a.div_nxy = fm::fastdiv_magic((uint32_t)(L->p.nx * L->p.ny));
    a.ns = (uint32_t)L->ns;
    a.n = L->n;
    a.nx = L->p.nx; a.ny = L->p.ny; a.nz = L->p.nz;
    a.px = L->p.periodic_x != 0; a.py = L->p.periodic_y != 0; a.pz = L->p.periodic_z != 0;
    // omega with the 0.5001 clamp, in R as the reference forms it in DATA_TYPE
    // (src/collision/BGKCollision.cu:202-205)
    R tau = (R)L->p.tau;
    if (tau < R(0.5001)) tau = R(0.5001);
    a.omega = R(1) / tau;
    a.rho0 = (R)L->p.rho0;
    a.omega_ad = R(1) / (R)L->p.tau_ad;
    a.min_conc = (R)L->p.min_concentration;
    a.f_shift = (R)L->f_shift;
    a.g_shift = (R)L->g_shift;
    a.coupling = L->coupling;
    a.isotherm = L->isotherm;
    a.iso_a = (R)L->iso[0];
    a.iso_b = (R)L->iso[1];
    a.iso_k = (R)L->iso[2];
    a.fuse_outlet = L->fuse_outlet;
    a.rho_out = (R)L->rho_out;
    a.fuse_neumann = L->fuse_neumann;
    a.fuse_dirichlet = L->fuse_dirichlet;
    a.c_in = (R)L->c_in;
    a.pf_dist = L->pf_dist;
    a.fuse_inlet = L->fuse_inlet;
    if (L->fuse_inlet) {
        a.uin_x = (R)L->ns_pre[0].v[0];
        a.uin_y = (R)L->ns_pre[0].v[1];
        a.uin_z = (R)L->ns_pre[0].v[2];
    }
    a.x0post = (T*)L->x0post;
    a.rows_stride = L->rows_stride;
    a.div_h = fm::fastdiv_magic((uint32_t)(L->p.nx / 2));
    a.c_first = 0;
    a.c_end = (uint32_t)L->n;
    a.neg_zero = (typename fm::Pop<T>::R)-0.0;
    a.status = L->d_status;
    a.st_rows = 0;
    return a;
}

// h = nx / 2 when f[cur] and g[cur] are in the pair layout, else 0 (natural)
uint32_t pair_h(const fm_lattice* L) { return L->layout ? (uint32_t)(L->p.nx / 2) : 0u; }
unsigned long long div_nx(const fm_lattice* L) { return fm::fastdiv_magic((uint32_t)L->p.nx); }

// resident blocks per SM of the pair kernel, and its L2 prefetch distance
// (the same fraction of a resident wave as the one-cell kernel's)
uint32_t pair_prefetch(const fm_lattice* L)
{
    if (L->pf_set) return L->pf_dist;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int per_sm = L->collision == FM_COLL_BGK ? fm::kPairBlocks<false> : fm::kPairBlocks<true>;
    return (uint32_t)(kPrefetchWavePct * sms * per_sm / 100);
}

// The staged pair kernel (fm_pair.cuh) runs a pair-layout lattice whose
// x-rows fit one tile (nx / 2 <= 256 words) and start on 16-byte boundaries
// (nx % 8 == 0), unless fm_set_pair_kernel(lat, 0) asks for k_coupled_pair.
// Tiles hold 256 / (nx / 2) rows; the two stages of a block must fit its
// shared memory.
constexpr size_t kStageSmemMax = 227 * 1024;
bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
bool staged_shape(const fm_lattice* L)
{
    // bulk copies want 16-byte aligned sources: every row of nx % 8 == 0
    // cells is, when the arrays themselves are
    const bool aligned = aligned16(L->f[0]) && aligned16(L->f[1]) && aligned16(L->g[0]) && aligned16(L->g[1]) &&
                         aligned16(L->cellw) && aligned16(L->phi) && aligned16(L->q) && aligned16(L->por) &&
                         aligned16(L->tau);
    return L->layout == 1 && L->staged_pref && L->p.nx % 8 == 0 && L->p.nx / 2 <= fm::kStageThreads && aligned;
}
uint32_t staged_rows(const fm_lattice* L) { return (uint32_t)(fm::kStageThreads / (L->p.nx / 2)); }
// bytes of shared memory the staged kernel takes for `a` (stage_geom of fm_pair.cuh)
template <typename T, typename QT>
size_t staged_smem(const fm::StepArgs<T, QT>& a)
{
    using R = typename fm::Pop<T>::R;
    const fm::StageGeom g = fm::stage_geom(a.nx, a.st_rows, a.isotherm != 0, a.porosity != nullptr,
                                           a.tau_ad != nullptr, (uint32_t)sizeof(QT), (uint32_t)sizeof(R));
    return fm::kStageHeader + 2 * (size_t)g.bytes;
}

// The staged pair kernel over the words [a.c_first, a.c_end) when it applies
// to L (shape, alignment, shared memory): *launched tells whether it ran, and
// *grid receives its block count.
template <typename T, typename QT>
int launch_staged(fm_lattice* L, fm::StepArgs<T, QT> a, bool mon, cudaStream_t st, int* grid, bool* launched)
{
    *launched = false;
    if (!staged_shape(L)) return FM_OK;
    const bool bgk = L->collision == FM_COLL_BGK;
    a.st_rows = staged_rows(L);
    if (bgk) a.porosity = nullptr;   // BGK reads no porosity: keep it out of the stages
    const size_t smem = staged_smem(a);
    if (smem > kStageSmemMax) return FM_OK;
    void (*kern)(const fm::StepArgs<T, QT>) =
        mon ? (bgk ? fm::k_pair_staged<T, QT, false, true> : fm::k_pair_staged<T, QT, true, true>)
            : (bgk ? fm::k_pair_staged<T, QT, false, false> : fm::k_pair_staged<T, QT, true, false>);
    const int variant = (bgk ? 0 : 1) + (mon ? 2 : 0);
    if (L->staged_smem[variant] != smem) {
        // the attributes are the function's, for every lattice: allow the most
        // dynamic shared memory a block may take beside its static part, and
        // prefer the largest shared-memory carveout so several blocks fit an SM
        int dev = 0, sms = 148, optin = 0, per_sm = 0;
        FM_CUDA(cudaGetDevice(&dev));
        FM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        FM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa{};
        FM_CUDA(cudaFuncGetAttributes(&fa, kern));
        const int dyn_max = optin - (int)fa.sharedSizeBytes;
        if ((long long)smem > (long long)dyn_max) return FM_OK;
        FM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max));
        FM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
        FM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, fm::kStageThreads, smem));
        L->staged_grid[variant] = std::max(1, per_sm) * sms;
        L->staged_smem[variant] = smem;
    }
    const uint32_t rows = (a.c_end - a.c_first) / (uint32_t)(L->p.nx / 2);
    const uint32_t tiles = (rows + a.st_rows - 1) / a.st_rows;
    *grid = (int)std::min<long long>(tiles, L->staged_grid[variant]);
    kern<<<*grid, fm::kStageThreads, smem, st>>>(a);
    FM_CHECK_LAUNCH("k_pair_staged");
    *launched = true;
    return FM_OK;
}

// The pair kernel over the words [a.c_first, a.c_end) (whole x-rows): the
// staged kernel where it applies, else k_coupled_pair.  *grid receives the
// launch's block count (the monitor folds that many partials).
template <typename T, typename QT>
int launch_pair(fm_lattice* L, fm::StepArgs<T, QT> a, bool mon, cudaStream_t st, int* grid)
{
    if constexpr (fm::Pop<T>::kShifted) {
        bool launched = false;
        const int rc = launch_staged<T, QT>(L, a, mon, st, grid, &launched);
        if (rc || launched) return rc;
        const bool bgk = L->collision == FM_COLL_BGK;
        a.pf_dist = pair_prefetch(L);
        *grid = grid_for((long long)(a.c_end - a.c_first));
        if (mon && bgk) fm::k_coupled_pair<T, QT, false, true><<<*grid, kBlock, 0, st>>>(a);
        else if (mon) fm::k_coupled_pair<T, QT, true, true><<<*grid, kBlock, 0, st>>>(a);
        else if (bgk) fm::k_coupled_pair<T, QT, false><<<*grid, kBlock, 0, st>>>(a);
        else fm::k_coupled_pair<T, QT, true><<<*grid, kBlock, 0, st>>>(a);
        FM_CHECK_LAUNCH("k_coupled_pair");
        return FM_OK;
    }
    return fail(FM_ERR_STATE, "pair layout: 16-bit forms only");
}

// The 16-bit cell update addresses its pulls with signed 32-bit offsets
// (faster) unless 18 ns + nx*ny + 2 nx + 1 reaches 2^31 (fm::pull19_fast).
bool wide_offsets(const fm_lattice* L)
{
    return 18LL * L->ns + (long long)L->p.nx * L->p.ny + 2LL * L->p.nx + 1 >= (1LL << 31);
}

template <typename T, typename QT, bool POROUS, bool MON>
void launch_coupled(const fm_lattice* L, int grid, cudaStream_t st, const fm::StepArgs<T, QT>& a)
{
    if constexpr (fm::Pop<T>::kShifted) {
        if (wide_offsets(L)) {
            fm::k_coupled_step<T, QT, POROUS, MON, true><<<grid, kBlock, 0, st>>>(a);
            return;
        }
    }
    fm::k_coupled_step<T, QT, POROUS, MON><<<grid, kBlock, 0, st>>>(a);
}

template <typename T, typename QT>
int launch_step(fm_lattice* L)
{
    using R = typename fm::Pop<T>::R;
    const long long s = L->step + 1;
    const int A = L->cur, B = 1 - L->cur;
    cudaStream_t st = L->stream;
    const bool mon = L->mon_every > 0 && s % L->mon_every == 0;
    T* fA = (T*)L->f[A];
    T* fB = (T*)L->f[B];
    T* gA = (T*)L->g[A];
    T* gB = (T*)L->g[B];

    // NS pre-collision boundaries on f_A (Lattice::step, NSLattice.hpp:193-195)
    for (const Bc& b : L->ns_pre) {
        if (!b.count || L->fuse_inlet) continue;
        if (b.kind == BC_NS_VEL_EQ)
            fm::k_ns_velocity_eq<T><<<grid_for(b.count), kBlock, 0, st>>>(
                fA, L->ns, b.cells, b.count, (R)L->p.rho0, (R)b.v[0], (R)b.v[1], (R)b.v[2], (R)L->f_shift);
        else
            fm::k_ns_velocity_neq<T><<<grid_for(b.count), kBlock, 0, st>>>(
                fA, L->ns, b.cells, b.nei, b.count, (R)b.v[0], (R)b.v[1], (R)b.v[2], (R)L->f_shift);
    }
    // AD pre-collision boundaries on g_A (ADLattice::step, ADLattice.hpp:150-152);
    // the pulse value is formed on the host in double as
    // src/boundary/ad/ADDirichletTanhPulse.cu:126-138 does
    for (const Bc& b : L->ad_pre) {
        if (!b.count) continue;
        const double kk = (double)(R)b.v[2];
        const double pulse = 0.5 * (std::tanh(((double)s - (double)b.iv[0]) / kk) -
                                    std::tanh(((double)s - (double)b.iv[1]) / kk));
        const R phi_in = (R)b.v[0] + (R)pulse * (R)b.v[1];
        fm::k_ad_fill<T><<<grid_for(b.count), kBlock, 0, st>>>(gA, L->ns, b.cells, b.count, phi_in, (R)L->g_shift);
    }
    // the fused NS + coupling + LDF + AD step
    const fm::StepArgs<T, QT> a = make_args<T, QT>(L);
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (L->profiling) {
        if (L->prof_used + 2 > L->prof_ev.size()) {
            for (int i = 0; i < 256; ++i) {
                cudaEvent_t e;
                FM_CUDA(cudaEventCreate(&e));
                L->prof_ev.push_back(e);
            }
        }
        ev0 = L->prof_ev[L->prof_used];
        ev1 = L->prof_ev[L->prof_used + 1];
        L->prof_used += 2;
        FM_CUDA(cudaEventRecord(ev0, st));
    }
    int grid = 0;
    const bool bgk = L->collision == FM_COLL_BGK;
    if constexpr (fm::Pop<T>::kShifted) {
        if (L->layout == 1) {
            fm::StepArgs<T, QT> ap = a;
            ap.c_end = (uint32_t)(L->n / 2);
            ap.mon = L->d_mon_part;
            const int rc = launch_pair<T, QT>(L, ap, mon, st, &grid);
            if (rc) return rc;
        }
    }
    if (L->layout == 0) {
        fm::StepArgs<T, QT> am = a;
        am.mon = L->d_mon_part;
        grid = grid_for(L->n);
        if (mon && bgk) launch_coupled<T, QT, false, true>(L, grid, st, am);
        else if (mon) launch_coupled<T, QT, true, true>(L, grid, st, am);
        else if (bgk) launch_coupled<T, QT, false, false>(L, grid, st, a);
        else launch_coupled<T, QT, true, false>(L, grid, st, a);
    }
    if (ev1) FM_CUDA(cudaEventRecord(ev1, st));
    if (mon) {
        // the launch's partials folded into the next row of the monitor
        const int row = (int)L->mon_steps.size();
        if (row >= L->mon_cap) {
            const int cap = std::max(64, 2 * L->mon_cap);
            double* nb = nullptr;
            int rc = dev_alloc(&nb, (size_t)cap * fm::kMonN, st);
            if (rc) return rc;
            if (row)
                FM_CUDA(cudaMemcpyAsync(nb, L->d_mon, sizeof(double) * fm::kMonN * row, cudaMemcpyDeviceToDevice, st));
            dev_free(L->d_mon, st);
            L->d_mon = nb;
            L->mon_cap = cap;
        }
        fm::k_monitor_fold<<<1, kBlock, 0, st>>>(L->d_mon_part, grid, L->d_mon + (size_t)row * fm::kMonN);
        FM_CHECK_LAUNCH("k_monitor_fold");
        L->mon_steps.push_back(s);
    }
    // NS post-stream boundaries on f_B (NSLattice.hpp:203-205)
    for (const Bc& b : L->ns_post) {
        if (!b.count || L->fuse_outlet) continue;
        if (b.kind == BC_NS_PRESSURE)
            fm::k_ns_pressure<T><<<grid_for(b.count), kBlock, 0, st>>>(fB, L->ns, b.cells, b.count, (R)b.v[0], (R)L->f_shift);
        else
            fm::k_ns_bounceback<T><<<grid_for(b.count), kBlock, 0, st>>>(fB, L->ns, b.cells, b.count);
    }
    if (L->ndeferred)
        fm::k_ad_deferred<T, QT><<<grid_for(L->ndeferred), kBlock, 0, st>>>(a, L->deferred, L->ndeferred);
    // AD post-stream boundaries on g_B (ADLattice.hpp:157-159)
    for (const Bc& b : L->ad_post) {
        if (!b.count) continue;
        if (b.kind == BC_AD_DIRICHLET && L->fuse_dirichlet) continue;
        if (b.kind == BC_AD_NEUMANN && L->fuse_neumann) continue;
        if (b.kind == BC_AD_DIRICHLET)
            fm::k_ad_fill<T><<<grid_for(b.count), kBlock, 0, st>>>(gB, L->ns, b.cells, b.count, (R)b.v[0], (R)L->g_shift);
        else
            fm::k_ad_neumann<T><<<grid_for(b.count), kBlock, 0, st>>>(gB, L->ns, b.cells, b.count);
    }
    FM_CHECK_LAUNCH("fm_step");
    L->cur = B;
    L->step = s;
    return FM_OK;
}

// The fused step kernel of the next step over the z-planes [z0, z1) only
// (fm_step_planes): reads f[cur] / g[cur], writes f[1-cur] / g[1-cur] of
// those planes; the step is completed by fm_step_finish.
template <typename T, typename QT>
int launch_planes(fm_lattice* L, int z0, int z1)
{
    fm::StepArgs<T, QT> a = make_args<T, QT>(L);
    const uint32_t nxy = (uint32_t)L->p.nx * (uint32_t)L->p.ny;
    cudaStream_t st = L->stream;
    if constexpr (fm::Pop<T>::kShifted) {
        if (L->layout == 1) {
            a.c_first = (uint32_t)z0 * (nxy / 2);
            a.c_end = (uint32_t)z1 * (nxy / 2);
            int grid = 0;
            return launch_pair<T, QT>(L, a, false, st, &grid);
        }
    }
    a.c_first = (uint32_t)z0 * nxy;
    a.c_end = (uint32_t)z1 * nxy;
    const int grid = grid_for((long long)(a.c_end - a.c_first));
    if (L->collision == FM_COLL_BGK) launch_coupled<T, QT, false, false>(L, grid, st, a);
    else launch_coupled<T, QT, true, false>(L, grid, st, a);
    FM_CHECK_LAUNCH("k_coupled_step (planes)");
    return FM_OK;
}

// x = 0 inlet plane representation: plain (f[cur] holds the reference's
// post-step populations) or fused (f[cur] holds the NEQ values of the next
// step and x0post the populations).
template <typename T>
int inlet_to_fused(fm_lattice* L)
{
    using R = typename fm::Pop<T>::R;
    const Bc& b = L->ns_pre[0];
    fm::k_inlet_prime<T><<<grid_for(b.count), kBlock, 0, L->stream>>>(
        (T*)L->f[L->cur], L->ns, b.cells, b.nei, b.count, (R)b.v[0], (R)b.v[1], (R)b.v[2], (R)L->f_shift,
        (T*)L->x0post, L->rows_stride, pair_h(L), div_nx(L));
    FM_CHECK_LAUNCH("k_inlet_prime");
    L->inlet_state = 1;
    return FM_OK;
}

template <typename T>
int inlet_to_plain(fm_lattice* L)
{
    // the list that was fused is the only NS pre-collision boundary
    const Bc& b = L->ns_pre[0];
    fm::k_inlet_restore<T><<<grid_for(b.count), kBlock, 0, L->stream>>>((T*)L->f[L->cur], L->ns, b.cells, b.count,
                                                                      (const T*)L->x0post, L->rows_stride,
                                                                      pair_h(L), div_nx(L));
    FM_CHECK_LAUNCH("k_inlet_restore");
    L->inlet_state = 0;
    return FM_OK;
}

int ensure_bt_capacity(fm_lattice* L, int need)
{
    if (need <= L->bt_cap) return FM_OK;
    int cap = std::max(need, std::max(1024, 2 * L->bt_cap));
    double* nb = nullptr;
    int rc = dev_alloc(&nb, (size_t)cap, L->stream);
    if (rc) return rc;
    FM_CUDA(cudaMemsetAsync(nb, 0, sizeof(double) * (size_t)cap, L->stream));
    if (L->bt_count)
        FM_CUDA(cudaMemcpyAsync(nb, L->d_bt, sizeof(double) * (size_t)L->bt_count, cudaMemcpyDeviceToDevice, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    dev_free(L->d_bt, L->stream);
    L->d_bt = nb;
    L->bt_cap = cap;
    return FM_OK;
}

int probe_into(fm_lattice* L, double* dst)
{
    if (L->relt == 8)
        fm::k_probe_mean<double><<<std::min(grid_for(L->nprobe), 148), kBlock, 0, L->stream>>>(
            (const double*)L->phi, L->probe, L->nprobe, dst);
    else
        fm::k_probe_mean<float><<<std::min(grid_for(L->nprobe), 148), kBlock, 0, L->stream>>>(
            (const float*)L->phi, L->probe, L->nprobe, dst);
    FM_CHECK_LAUNCH("k_probe_mean");
    return FM_OK;
}

int take_sample(fm_lattice* L)
{
    if (!L->nprobe) return FM_OK;
    int rc = ensure_bt_capacity(L, L->bt_count + 1);
    if (rc) return rc;
    // the probe accumulates block sums: the slot may hold a sample of an
    // earlier run (fm_init_equilibrium restarts the series)
    FM_CUDA(cudaMemsetAsync(L->d_bt + L->bt_count, 0, sizeof(double), L->stream));
    rc = probe_into(L, L->d_bt + L->bt_count);
    if (rc) return rc;
    ++L->bt_count;
    return FM_OK;
}

template <typename T, typename QT>
int init_state(fm_lattice* L)
{
    using R = typename fm::Pop<T>::R;
    fm::k_init<T, QT><<<grid_for(L->n), kBlock, 0, L->stream>>>(
        (T*)L->f[0], (T*)L->g[0], (R*)L->phi, (QT*)L->q, L->ns, L->n, (R)L->p.rho0, (R)L->p.phi0,
        (R)L->f_shift, (R)L->g_shift);
    FM_CHECK_LAUNCH("k_init");
    // Lattice::initEquilibrium copies f into f_new (NSLattice.hpp:184)
    FM_CUDA(cudaMemcpyAsync(L->f[1], L->f[0], (size_t)19 * L->ns * L->elt, cudaMemcpyDeviceToDevice, L->stream));
    FM_CUDA(cudaMemcpyAsync(L->g[1], L->g[0], (size_t)7 * L->ns * L->elt, cudaMemcpyDeviceToDevice, L->stream));
    return FM_OK;
}

template <typename T, typename QT>
int macros_to_tmp(fm_lattice* L)
{
    using R = typename fm::Pop<T>::R;
    R* t = (R*)L->d_tmp;
    fm::k_macros<T><<<grid_for(L->n), kBlock, 0, L->stream>>>((const T*)L->f[L->cur], L->ns, L->n, (R)L->f_shift, t,
                                                             t + L->ns, t + 2 * L->ns, t + 3 * L->ns, pair_h(L),
                                                             div_nx(L));
    FM_CHECK_LAUNCH("k_macros");
    return FM_OK;
}

// sums of rho, phi, q over the z-planes [z0, z1) into d_acc[0..2] (a z-plane
// range is the same run of storage elements in either layout)
template <typename T, typename QT>
int range_sums(fm_lattice* L, int z0, int z1)
{
    using R = typename fm::Pop<T>::R;
    const long long nxy = (long long)L->p.nx * L->p.ny, c0 = z0 * nxy, cnt = (long long)(z1 - z0) * nxy;
    FM_CUDA(cudaMemsetAsync(L->d_acc, 0, 8 * sizeof(double), L->stream));
    if (cnt > 0) {
        fm::k_domain_sums<T, QT><<<std::min(grid_for(cnt), 148 * 8), kBlock, 0, L->stream>>>(
            (const T*)L->f[L->cur] + c0, (const R*)L->phi + c0, (const QT*)L->q + c0, L->ns, (int)cnt, (R)L->f_shift,
            L->d_acc);
        FM_CHECK_LAUNCH("k_domain_sums (planes)");
    }
    return FM_OK;
}

template <typename T, typename QT>
int domain_sums(fm_lattice* L)
{
    using R = typename fm::Pop<T>::R;
    FM_CUDA(cudaMemsetAsync(L->d_acc, 0, 8 * sizeof(double), L->stream));
    fm::k_domain_sums<T, QT><<<std::min(grid_for(L->n), 148 * 8), kBlock, 0, L->stream>>>(
        (const T*)L->f[L->cur], (const R*)L->phi, (const QT*)L->q, L->ns, L->n, (R)L->f_shift, L->d_acc);
    FM_CHECK_LAUNCH("k_domain_sums");
    if (L->nprobe) return probe_into(L, L->d_acc + 3);
    return FM_OK;
}

// population planes <-> FP64 host arrays, through planes of the arithmetic type R
template <typename T>
__global__ void k_pop_to_real(const T* __restrict__ src, typename fm::Pop<T>::R* __restrict__ dst, long long ns, int n,
                              int nq, int d3q19, typename fm::Pop<T>::R shift, uint32_t pair_h,
                              unsigned long long div_nx)
{
    using R = typename fm::Pop<T>::R;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)nq * n) return;
    const int k = (int)(i / n), c = (int)(i - (long long)k * n);
    const uint32_t e = fm::pair_element((uint32_t)c, pair_h, div_nx);
    dst[i] = d3q19 ? fm::Pop<T>::ld(src + (long long)k * ns + e, fm::fshift<T>(k, shift))
                   : fm::PopG<T>::ld(src + (long long)k * ns + e, k, shift);
}

template <typename T>
__global__ void k_real_to_pop(const typename fm::Pop<T>::R* __restrict__ src, T* __restrict__ dst, long long ns, int n,
                              int nq, int d3q19, typename fm::Pop<T>::R shift, uint32_t pair_h,
                              unsigned long long div_nx)
{
    using R = typename fm::Pop<T>::R;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)nq * n) return;
    const int k = (int)(i / n), c = (int)(i - (long long)k * n);
    const uint32_t e = fm::pair_element((uint32_t)c, pair_h, div_nx);
    if (d3q19) fm::Pop<T>::st(dst + (long long)k * ns + e, src[i], fm::fshift<T>(k, shift));
    else fm::PopG<T>::st(dst + (long long)k * ns + e, src[i], k, shift, (uint32_t)c);
}

template <typename T>
int pops_get(fm_lattice* L, double* f, double* g)
{
    using R = typename fm::Pop<T>::R;
    const int n = L->n;
    for (int which = 0; which < 2; ++which) {
        double* out = which == 0 ? f : g;
        if (!out) continue;
        const int nq = which == 0 ? 19 : 7;
        R* tmp = nullptr;
        int rc = dev_alloc(&tmp, (size_t)nq * n, L->stream);
        if (rc) return rc;
        const void* src = which == 0 ? L->f[L->cur] : L->g[L->cur];
        k_pop_to_real<T><<<grid_for((long long)nq * n), kBlock, 0, L->stream>>>(
            (const T*)src, tmp, L->ns, n, nq, which == 0, (R)(which == 0 ? L->f_shift : L->g_shift), pair_h(L),
            div_nx(L));
        std::vector<R> h((size_t)nq * n);
        cudaError_t e = cudaMemcpyAsync(h.data(), tmp, h.size() * sizeof(R), cudaMemcpyDeviceToHost, L->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
        dev_free(tmp, L->stream);
        if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("fm_get_state: ") + cudaGetErrorString(e));
        for (size_t i = 0; i < h.size(); ++i) out[i] = (double)h[i];
    }
    return FM_OK;
}

template <typename T>
int pops_set(fm_lattice* L, const double* f, const double* g)
{
    using R = typename fm::Pop<T>::R;
    const int n = L->n;
    for (int which = 0; which < 2; ++which) {
        const double* in = which == 0 ? f : g;
        if (!in) continue;
        const int nq = which == 0 ? 19 : 7;
        std::vector<R> h((size_t)nq * n);
        for (size_t i = 0; i < h.size(); ++i) h[i] = (R)in[i];
        R* tmp = nullptr;
        int rc = dev_alloc(&tmp, h.size(), L->stream);
        if (rc) return rc;
        cudaError_t e = cudaMemcpyAsync(tmp, h.data(), h.size() * sizeof(R), cudaMemcpyHostToDevice, L->stream);
        void* dst = which == 0 ? L->f[L->cur] : L->g[L->cur];
        if (e == cudaSuccess) {
            k_real_to_pop<T><<<grid_for((long long)nq * n), kBlock, 0, L->stream>>>(
                tmp, (T*)dst, L->ns, n, nq, which == 0, (R)(which == 0 ? L->f_shift : L->g_shift), pair_h(L),
                div_nx(L));
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
        dev_free(tmp, L->stream);
        if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("fm_set_state: ") + cudaGetErrorString(e));
    }
    return FM_OK;
}

// dispatch on the storage format
template <template <typename, typename> class F, typename... Args>
int dispatch(fm_lattice* L, Args... args)
{
    switch (L->precision) {
        case FM_F32: return F<float, float>::run(L, args...);
        case FM_F64: return F<double, double>::run(L, args...);
        case FM_F16_SHIFTED: return F<__half, double>::run(L, args...);
        case FM_BF16_SHIFTED: return F<__nv_bfloat16, double>::run(L, args...);
        case FM_F16_FIXED_AD: return F<fm::hq, double>::run(L, args...);
        default: return fail(FM_ERR_ARG, "unknown precision");
    }
}

// f[cur] and g[cur] between the natural and the pair layout, through the
// write buffers (the next step rewrites them whole); `cur` is kept
template <typename T, typename QT>
int convert_layout(fm_lattice* L, int to)
{
    if constexpr (sizeof(T) == 2) {
        for (int which = 0; which < 2; ++which) {
            const int nq = which ? 7 : 19;
            void** buf = which ? L->g : L->f;
            uint16_t* cur = (uint16_t*)buf[L->cur];
            uint16_t* tmp = (uint16_t*)buf[1 - L->cur];
            fm::k_pair_permute<uint16_t><<<grid_for((long long)nq * L->n), kBlock, 0, L->stream>>>(
                cur, tmp, L->ns, L->n, nq, (uint32_t)(L->p.nx / 2), div_nx(L), to);
            FM_CHECK_LAUNCH("k_pair_permute");
            FM_CUDA(cudaMemcpyAsync(cur, tmp, (size_t)nq * L->ns * 2, cudaMemcpyDeviceToDevice, L->stream));
        }
        L->layout = to;
        return FM_OK;
    }
    return fail(FM_ERR_STATE, "pair layout: 16-bit forms only");
}

template <typename T, typename QT> struct StepOp { static int run(fm_lattice* L) { return launch_step<T, QT>(L); } };
template <typename T, typename QT> struct PlanesOp {
    static int run(fm_lattice* L, int z0, int z1) { return launch_planes<T, QT>(L, z0, z1); }
};
template <typename T, typename QT> struct LayoutOp {
    static int run(fm_lattice* L, int to) { return convert_layout<T, QT>(L, to); }
};
template <typename T, typename QT> struct InletFusedOp { static int run(fm_lattice* L) { return inlet_to_fused<T>(L); } };
template <typename T, typename QT> struct InletPlainOp { static int run(fm_lattice* L) { return inlet_to_plain<T>(L); } };

// before reading f[cur] for outputs: the x = 0 plane as the reference holds it
int ensure_plain(fm_lattice* L)
{
    if (L->inlet_state == 1) return dispatch<InletPlainOp>(L);
    return FM_OK;
}
template <typename T, typename QT> struct InitOp { static int run(fm_lattice* L) { return init_state<T, QT>(L); } };
template <typename T, typename QT> struct MacroOp { static int run(fm_lattice* L) { return macros_to_tmp<T, QT>(L); } };
template <typename T, typename QT> struct SumOp { static int run(fm_lattice* L) { return domain_sums<T, QT>(L); } };
template <typename T, typename QT> struct RangeSumOp {
    static int run(fm_lattice* L, int z0, int z1) { return range_sums<T, QT>(L, z0, z1); }
};
template <typename T, typename QT> struct GetPops {
    static int run(fm_lattice* L, double* f, double* g) { return pops_get<T>(L, f, g); }
};
template <typename T, typename QT> struct SetPops {
    static int run(fm_lattice* L, const double* f, const double* g) { return pops_set<T>(L, f, g); }
};

// The layout the next step runs on: the pair layout (fm_pair.cuh) for a
// 16-bit form with nx % 4 == 0 and nx >= 8 whose boundaries all run inside the
// fused step, outside any batch, when fm_set_pair_layout enabled it; else
// natural.  Converts
// the stored populations when it changes.  Call after prepare().
int ensure_layout(fm_lattice* L)
{
    const bool is16 = L->precision == FM_F16_SHIFTED || L->precision == FM_BF16_SHIFTED ||
                      L->precision == FM_F16_FIXED_AD;
    int want = 0;
    if (is16 && L->pair_pref && !L->in_batch && L->p.nx % 4 == 0 && L->p.nx >= 8 && fm_launches_per_step(L) == 1)
        want = 1;
    if (want == L->layout) return FM_OK;
    return dispatch<LayoutOp>(L, want);
}

int add_bc(fm_lattice* L, std::vector<Bc>& into, Bc b, const std::vector<int>& cells, const std::vector<int>* nei)
{
    b.count = (int)cells.size();
    int rc = upload_list(cells, &b.cells, L->stream);
    if (rc) return rc;
    if (nei) {
        rc = upload_list(*nei, &b.nei, L->stream);
        if (rc) { dev_free(b.cells, L->stream); return rc; }
    }
    into.push_back(b);
    L->dirty = true;
    return FM_OK;
}

// reference launchers on raw device pointers
__global__ void k_ldf_source_u8(int n, const uint8_t* __restrict__ region, const float* __restrict__ phi,
                                float* __restrict__ S, float* __restrict__ q, int langmuir, float a, float b, float k,
                                float eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!region[i]) { S[i] = 0.0f; return; }
    float c = phi[i];
    if (c < eps) c = eps;
    const float ce = c - eps;
    float qeq;
    if (langmuir) { const float bc = b * ce; qeq = a * (bc / (1.0f + bc)); }
    else qeq = a * ce;
    const float qi = q[i];
    const float dq = k * (qeq - qi);
    q[i] = qi + dq;
    S[i] = -dq;
}

}  // namespace

namespace fm_internal {
// lets the other translation units of the library report through fm_last_error()
__attribute__((visibility("hidden"))) int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace fm_internal

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* fm_last_error(void) { return g_last_error.c_str(); }
int fm_abi_version(void) { return FM_ABI_VERSION; }

int fm_lattice_create(const fm_params* p, int precision, void* stream, fm_lattice** out)
{
    if (!p || !out) return fail(FM_ERR_ARG, "fm_lattice_create: null argument");
    *out = nullptr;
    // NSLattice.hpp:21-22 / ADLattice.hpp:23-24
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0) return fail(FM_ERR_ARG, "NSLattice: invalid dimensions");
    const long long n = (long long)p->nx * p->ny * p->nz;
    // population offsets k*ns + c are 32-bit: 19 planes must fit below 2^32
    if (19LL * ((n + 31) / 32 * 32) >= (1LL << 32))
        return fail(FM_ERR_UNSUPPORTED, "lattice larger than 226,050,000 cells");
    if (precision != FM_F32 && precision != FM_F16_SHIFTED && precision != FM_BF16_SHIFTED && precision != FM_F64 &&
        precision != FM_F16_FIXED_AD)
        return fail(FM_ERR_ARG, "unknown precision");
    fm_lattice* L = new fm_lattice();
    L->p = *p;
    L->precision = precision;
    L->n = (int)n;
    L->ns = (n + 31) / 32 * 32;
    L->nwords = (size_t)(L->ns / 32);
    L->elt = precision == FM_F32 ? 4 : (precision == FM_F64 ? 8 : 2);
    L->qelt = precision == FM_F32 ? 4 : 8;
    L->relt = precision == FM_F64 ? 8 : 4;
    if (precision == FM_F16_SHIFTED || precision == FM_BF16_SHIFTED || precision == FM_F16_FIXED_AD) {
        L->f_shift = p->rho0;
        L->g_shift = 0.5;   // unused by the fixed-point D3Q7 planes
    }
    if (stream) L->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete L;
            return fail(FM_ERR_CUDA, "cudaStreamCreate failed");
        }
        L->own_stream = true;
    }
    int rc = 0;
    for (int i = 0; i < 2 && !rc; ++i) {
        rc = dev_alloc((char**)&L->f[i], (size_t)19 * L->ns * L->elt, L->stream);
        if (!rc) rc = dev_alloc((char**)&L->g[i], (size_t)7 * L->ns * L->elt, L->stream);
    }
    if (!rc) rc = dev_alloc((char**)&L->phi, (size_t)L->ns * L->relt, L->stream);
    if (!rc) rc = dev_alloc((char**)&L->q, (size_t)L->ns * L->qelt, L->stream);
    if (!rc) rc = dev_alloc(&L->solid, L->nwords, L->stream);
    if (!rc) rc = dev_alloc((char**)&L->tau, (size_t)L->ns * L->relt, L->stream);
    if (!rc) rc = dev_alloc(&L->d_acc, 8, L->stream);
    if (!rc) rc = dev_alloc(&L->d_status, 4, L->stream);
    if (rc) { fm_lattice_destroy(L); return rc; }
    cudaMemsetAsync(L->d_status, 0, 4 * sizeof(int), L->stream);
    // zeroed fields as the constructors memset them (NSLattice.hpp:34-44,
    // ADLattice.hpp:49-53, AdsorbedField.hpp:18)
    cudaMemsetAsync(L->phi, 0, L->relt * L->ns, L->stream);
    cudaMemsetAsync(L->q, 0, L->qelt * L->ns, L->stream);
    cudaMemsetAsync(L->solid, 0, sizeof(uint32_t) * L->nwords, L->stream);
    for (int i = 0; i < 2; ++i) {
        cudaMemsetAsync(L->f[i], 0, (size_t)19 * L->ns * L->elt, L->stream);
        cudaMemsetAsync(L->g[i], 0, (size_t)7 * L->ns * L->elt, L->stream);
    }
    if (cudaStreamSynchronize(L->stream) != cudaSuccess) {
        fm_lattice_destroy(L);
        return fail(FM_ERR_CUDA, "memset failed");
    }
    *out = L;
    return FM_OK;
}

int fm_lattice_destroy(fm_lattice* L)
{
    if (!L) return FM_OK;
    if (L->in_batch) return fail(FM_ERR_STATE, "fm_lattice_destroy: a batch still holds the lattice (destroy it first)");
    if (L->stream) cudaStreamSynchronize(L->stream);
    for (int i = 0; i < 2; ++i) { dev_free(L->f[i], L->stream); dev_free(L->g[i], L->stream); }
    dev_free(L->phi, L->stream); dev_free(L->q, L->stream); dev_free(L->solid, L->stream); dev_free(L->region, L->stream); dev_free(L->defer, L->stream);
    dev_free(L->por, L->stream); dev_free(L->tau, L->stream); dev_free(L->deferred, L->stream); dev_free(L->probe, L->stream); dev_free(L->d_bt, L->stream);
    dev_free(L->d_acc, L->stream); dev_free(L->d_tmp, L->stream); dev_free(L->cellw, L->stream); dev_free(L->x0post, L->stream); dev_free(L->adj_arena, L->stream);
    dev_free(L->d_wide, L->stream);
    dev_free(L->d_mon_part, L->stream);
    dev_free(L->d_mon, L->stream);
    dev_free(L->d_status, L->stream);
    for (cudaEvent_t e : L->prof_ev) cudaEventDestroy(e);
    for (auto* v : {&L->ns_pre, &L->ns_post, &L->ad_pre, &L->ad_post})
        for (Bc& b : *v) { dev_free(b.cells, L->stream); dev_free(b.nei, L->stream); }
    if (L->own_stream) cudaStreamDestroy(L->stream);
    delete L;
    return FM_OK;
}

int fm_set_obstacle_mask(fm_lattice* L, const uint8_t* mask, size_t n)
{
    if (check_mask(L, mask, n, "NSLattice::setObstacleMask:")) return FM_ERR_ARG;
    std::vector<uint32_t> bits = pack_bits(mask, n, L->nwords);
    FM_CUDA(cudaMemcpyAsync(L->solid, bits.data(), bits.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    L->dirty = true;
    return FM_OK;
}

int fm_set_obstacle_bits(fm_lattice* L, const uint32_t* bits, size_t nwords)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!bits || nwords != ((size_t)L->n + 31) / 32) return fail(FM_ERR_ARG, "obstacle bits size mismatch");
    std::vector<uint32_t> b(L->nwords, 0u);
    std::memcpy(b.data(), bits, nwords * sizeof(uint32_t));
    const size_t tail = (size_t)L->n & 31;   // clear bits past the last cell
    if (tail) b[(size_t)L->n >> 5] &= (1u << tail) - 1u;
    FM_CUDA(cudaMemcpyAsync(L->solid, b.data(), b.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    L->dirty = true;
    return FM_OK;
}

// upload per-cell values as the arithmetic type R (float, or double for FM_F64)
static int upload_real_field(fm_lattice* L, void** dst, const std::vector<double>& h)
{
    if (!*dst) {
        int rc = dev_alloc((char**)dst, (size_t)L->ns * L->relt, L->stream);
        if (rc) return rc;
        FM_CUDA(cudaMemsetAsync(*dst, 0, L->relt * L->ns, L->stream));
    }
    if (L->relt == 8) {
        FM_CUDA(cudaMemcpyAsync(*dst, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, L->stream));
        FM_CUDA(cudaStreamSynchronize(L->stream));
    } else {
        std::vector<float> hf(h.size());
        for (size_t i = 0; i < h.size(); ++i) hf[i] = (float)h[i];
        FM_CUDA(cudaMemcpyAsync(*dst, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice, L->stream));
        FM_CUDA(cudaStreamSynchronize(L->stream));
    }
    return FM_OK;
}

// a value as the arithmetic type R would hold it
static double as_real(const fm_lattice* L, double v) { return L->relt == 8 ? v : (double)(float)v; }

int fm_set_porosity_from_mask(fm_lattice* L, const uint8_t* mask, size_t n, double phi_masked, double phi_else)
{
    // NSLattice.hpp:88-114
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!mask || n != (size_t)L->n) return fail(FM_ERR_ARG, "setPorosityFromMask: mask size != lattice size");
    std::vector<double> h(n);
    for (size_t c = 0; c < n; ++c) h[c] = mask[c] ? phi_masked : phi_else;
    return upload_real_field(L, &L->por, h);
}

int fm_set_porosity(fm_lattice* L, const double* porosity, size_t n)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!porosity || n != (size_t)L->n) return fail(FM_ERR_ARG, "porosity field size mismatch");
    std::vector<double> h(porosity, porosity + n);
    return upload_real_field(L, &L->por, h);
}

int fm_set_tau_field(fm_lattice* L, const double* tau, size_t n)
{
    // ADLattice.hpp:95-100
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!tau || n != (size_t)L->n) return fail(FM_ERR_ARG, "ADLattice: tau field size mismatch");
    const double t0 = as_real(L, tau[0]);
    bool uniform = true;
    for (size_t c = 1; c < n && uniform; ++c) uniform = as_real(L, tau[c]) == t0;
    if (uniform) {
        // one value everywhere: the scalar path computes the same 1/tau per cell
        L->p.tau_ad = t0;
        L->tau_field = false;
        return FM_OK;
    }
    std::vector<double> h(n);
    for (size_t c = 0; c < n; ++c) h[c] = as_real(L, tau[c]);
    int rc = upload_real_field(L, &L->tau, h);
    if (rc) return rc;
    L->tau_field = true;
    return FM_OK;
}

int fm_build_tau_field(int nx, int ny, int nz, double dx_phys, double dt_phys, const uint8_t* mask, size_t n,
                       double d_fluid_phys, double d_solid_phys, double* tau_out)
{
    // ADUnitConverter's constructor checks (ADUnitConverter.hpp:30-42)
    if (nx < 2) return fail(FM_ERR_ARG, "ADUnitConverter: Nx must be >= 2");
    if (!(dx_phys > 0.0)) return fail(FM_ERR_ARG, "ADUnitConverter: dx_phys must be > 0");
    if (!(dt_phys > 0.0)) return fail(FM_ERR_ARG, "ADUnitConverter: dt_phys must be > 0");
    // buildTauField (ADUnitConverter.hpp:63-104)
    if (ny <= 0 || nz <= 0 || !mask || !tau_out || n != (size_t)nx * (size_t)ny * (size_t)nz)
        return fail(FM_ERR_ARG, "ADUnitConverter: mask size mismatch");
    // tauFromDiffusivityPhys (ADUnitConverter.hpp:45-58): D_lbm = D dt / dx^2,
    // tau = D_lbm / cs2 + 1/2 with the D3Q7 cs2 = 1/4, all in double
    const double cs2 = 0.25;
    const double tf = d_fluid_phys * dt_phys / (dx_phys * dx_phys) / cs2 + 0.5;
    const double ts = d_solid_phys * dt_phys / (dx_phys * dx_phys) / cs2 + 0.5;
    if (!(tf > 0.5) || !(ts > 0.5)) return fail(FM_ERR_ARG, "ADUnitConverter: tau_ad <= 0.5 (unstable)");
    for (size_t c = 0; c < n; ++c) tau_out[c] = mask[c] ? ts : tf;
    return FM_OK;
}

int fm_set_collision(fm_lattice* L, int collision)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (collision != FM_COLL_BGK && collision != FM_COLL_POROUS) return fail(FM_ERR_ARG, "unknown collision operator");
    L->collision = collision;
    L->collision_set = true;
    L->dirty = true;
    if (collision == FM_COLL_POROUS && !L->por) {
        // the reference's porosity buffer starts zeroed (NSLattice.hpp:39-40)
        std::vector<double> h((size_t)L->n, 0.0);
        return upload_real_field(L, &L->por, h);
    }
    return FM_OK;
}

int fm_set_coupling(fm_lattice* L, int enabled)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    L->coupling = enabled ? 1 : 0;
    return FM_OK;
}

static int set_region(fm_lattice* L, const uint8_t* region, size_t n)
{
    std::vector<uint32_t> bits = pack_bits(region, n, L->nwords);
    if (!L->region) {
        int rc = dev_alloc(&L->region, L->nwords, L->stream);
        if (rc) return rc;
    }
    FM_CUDA(cudaMemcpyAsync(L->region, bits.data(), bits.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    L->dirty = true;
    return FM_OK;
}

int fm_set_isotherm_linear(fm_lattice* L, const uint8_t* region, size_t n, double k_henry, double k_ldf)
{
    if (check_mask(L, region, n, "LinearLDF region")) return FM_ERR_ARG;
    int rc = set_region(L, region, n);
    if (rc) return rc;
    L->isotherm = FM_ISO_LINEAR;
    L->dirty = true;
    L->iso[0] = k_henry; L->iso[1] = 0.0; L->iso[2] = k_ldf;
    return FM_OK;
}

int fm_set_isotherm_langmuir(fm_lattice* L, const uint8_t* region, size_t n, double q_max, double b, double k_ldf)
{
    if (check_mask(L, region, n, "LangmuirLDF region")) return FM_ERR_ARG;
    int rc = set_region(L, region, n);
    if (rc) return rc;
    L->isotherm = FM_ISO_LANGMUIR;
    L->dirty = true;
    L->iso[0] = q_max; L->iso[1] = b; L->iso[2] = k_ldf;
    return FM_OK;
}

int fm_clear_isotherm(fm_lattice* L)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    L->isotherm = FM_ISO_NONE;
    L->dirty = true;
    return FM_OK;
}

int fm_add_ns_velocity_eq(fm_lattice* L, const uint8_t* mask, size_t n, double ux, double uy, double uz)
{
    if (check_mask(L, mask, n, "VelocityDirichletEq")) return FM_ERR_ARG;
    Bc b; b.kind = BC_NS_VEL_EQ; b.v[0] = ux; b.v[1] = uy; b.v[2] = uz;
    return add_bc(L, L->ns_pre, b, compress(mask, n), nullptr);
}

int fm_add_ns_velocity_neq(fm_lattice* L, const uint8_t* mask, size_t n, double ux, double uy, double uz)
{
    // include/boundary/ns/VelocityDirichletNEQ.hpp:26-107
    if (check_mask(L, mask, n, "VelocityDirichletNEQ")) return FM_ERR_ARG;
    const int nx = L->p.nx, ny = L->p.ny, nz = L->p.nz;
    std::vector<int> cells = compress(mask, n), nei;
    Bc b; b.kind = BC_NS_VEL_NEQ; b.v[0] = ux; b.v[1] = uy; b.v[2] = uz;
    if (cells.empty()) return add_bc(L, L->ns_pre, b, cells, nullptr);
    int minx = nx - 1, maxx = 0, miny = ny - 1, maxy = 0, minz = nz - 1, maxz = 0;
    for (int c : cells) {
        const int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        minx = std::min(minx, x); maxx = std::max(maxx, x);
        miny = std::min(miny, y); maxy = std::max(maxy, y);
        minz = std::min(minz, z); maxz = std::max(maxz, z);
    }
    const bool isx = minx == maxx, isy = miny == maxy, isz = minz == maxz;
    if (int(isx) + int(isy) + int(isz) != 1)
        return fail(FM_ERR_ARG, "VelocityDirichletNEQ: mask must describe exactly one axis-aligned plane "
                                "(x=const OR y=const OR z=const).");
    int dx = 0, dy = 0, dz = 0;
    if (isx) { if (minx == 0) dx = 1; else if (minx == nx - 1) dx = -1; else return fail(FM_ERR_ARG, "VelocityDirichletNEQ: x-plane not at boundary"); }
    if (isy) { if (miny == 0) dy = 1; else if (miny == ny - 1) dy = -1; else return fail(FM_ERR_ARG, "VelocityDirichletNEQ: y-plane not at boundary"); }
    if (isz) { if (minz == 0) dz = 1; else if (minz == nz - 1) dz = -1; else return fail(FM_ERR_ARG, "VelocityDirichletNEQ: z-plane not at boundary"); }
    for (int c : cells) {
        const int x = c % nx + dx, y = (c / nx) % ny + dy, z = c / (nx * ny) + dz;
        if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz)
            return fail(FM_ERR_ARG, "VelocityDirichletNEQ: inferred neighbor out of domain.");
        nei.push_back(x + y * nx + z * nx * ny);
    }
    return add_bc(L, L->ns_pre, b, cells, &nei);
}

int fm_add_ns_pressure(fm_lattice* L, const uint8_t* mask, size_t n, double rho_out)
{
    if (check_mask(L, mask, n, "PressureDirichlet")) return FM_ERR_ARG;
    // the kernel skips x <= 0 (src/boundary/ns/PressureDirichlet.cu:46-47)
    std::vector<int> cells;
    for (int c : compress(mask, n))
        if (c % L->p.nx > 0) cells.push_back(c);
    Bc b; b.kind = BC_NS_PRESSURE; b.v[0] = rho_out;
    return add_bc(L, L->ns_post, b, cells, nullptr);
}

int fm_add_ns_bounceback(fm_lattice* L, const uint8_t* mask, size_t n)
{
    if (check_mask(L, mask, n, "BounceBack")) return FM_ERR_ARG;
    Bc b; b.kind = BC_NS_BOUNCEBACK;
    return add_bc(L, L->ns_post, b, compress(mask, n), nullptr);
}

int fm_add_ad_dirichlet(fm_lattice* L, const uint8_t* mask, size_t n, double phi)
{
    if (check_mask(L, mask, n, "ADDirichlet")) return FM_ERR_ARG;
    Bc b; b.kind = BC_AD_DIRICHLET; b.v[0] = phi;
    return add_bc(L, L->ad_post, b, compress(mask, n), nullptr);
}

int fm_add_ad_tanh_pulse(fm_lattice* L, const uint8_t* mask, size_t n, double phi_base, double phi_amp, int t_on_step,
                         int t_off_step, double k_step)
{
    if (check_mask(L, mask, n, "ADDirichletTanhPulse")) return FM_ERR_ARG;
    Bc b; b.kind = BC_AD_PULSE; b.v[0] = phi_base; b.v[1] = phi_amp; b.v[2] = k_step;
    b.iv[0] = t_on_step; b.iv[1] = t_off_step;
    return add_bc(L, L->ad_pre, b, compress(mask, n), nullptr);
}

int fm_add_ad_neumann(fm_lattice* L, const uint8_t* mask, size_t n)
{
    if (check_mask(L, mask, n, "ADNeumannOutlet")) return FM_ERR_ARG;
    // only x = Nx-1 cells copy from x = Nx-2 (src/boundary/ad/ADNeumannOutlet.cu:17-22)
    std::vector<int> cells;
    if (L->p.nx >= 2)
        for (int c : compress(mask, n))
            if (c % L->p.nx == L->p.nx - 1) cells.push_back(c);
    Bc b; b.kind = BC_AD_NEUMANN;
    return add_bc(L, L->ad_post, b, cells, nullptr);
}

int fm_init_equilibrium(fm_lattice* L)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!L->collision_set) return fail(FM_ERR_STATE, "NSLattice::initEquilibrium: collision operator not set");
    L->cur = 0;
    L->step = 0;
    L->bt_count = 0;
    L->inlet_state = 0;
    L->mon_steps.clear();
    int rc = dispatch<InitOp>(L);
    if (rc) return rc;
    L->initialised = true;
    if (L->nprobe && L->probe_every > 0) return take_sample(L);
    return FM_OK;
}

int fm_step(fm_lattice* L, int nsteps)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (nsteps < 0) return fail(FM_ERR_ARG, "fm_step: negative step count");
    if (!L->collision_set) return fail(FM_ERR_STATE, "NSLattice: collision operator not set, could not step()!");
    if (!L->initialised) return fail(FM_ERR_STATE, "fm_step: fm_init_equilibrium not called");
    if (L->isotherm != FM_ISO_NONE && !L->region) return fail(FM_ERR_STATE, "isotherm without region mask");
    if (L->split_open) return fail(FM_ERR_STATE, "fm_step: a step begun by fm_step_planes is not finished");
    int prc = prepare(L);
    if (!prc) prc = ensure_layout(L);
    if (prc) return prc;
    if (L->mon_every > 0 && fm_launches_per_step(L) != 1)
        return fail(FM_ERR_UNSUPPORTED, "fm_step: the step monitor needs every boundary inside the fused step");
    if (L->fuse_inlet && L->inlet_state == 0) prc = dispatch<InletFusedOp>(L);
    else if (!L->fuse_inlet && L->inlet_state == 1) prc = dispatch<InletPlainOp>(L);
    if (prc) return prc;
    for (int i = 0; i < nsteps; ++i) {
        int rc = dispatch<StepOp>(L);
        if (rc) return rc;
        if (L->nprobe && L->probe_every > 0 && L->step % L->probe_every == 0) {
            rc = take_sample(L);
            if (rc) return rc;
        }
    }
    return FM_OK;
}

int fm_synchronize(fm_lattice* L)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return FM_OK;
}

long long fm_step_count(const fm_lattice* L) { return L ? L->step : -1; }

// device plane of R -> host doubles
// FP32 plane -> FP64 plane on the device (the host output is FP64)
__global__ void k_widen(const float* __restrict__ src, double* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

// device plane of R (or FP32 q) -> host doubles: widened on the device, then
// one copy straight into the caller's buffer
// FM_ERR_DEVICE when a step kernel's bounded wait gave up since the last
// fm_step_status (the word stays set until that call reads it)
static int device_status(fm_lattice* L)
{
    int st = 0;
    FM_CUDA(cudaMemcpyAsync(&st, L->d_status, sizeof(int), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return st ? fail(FM_ERR_DEVICE, "a step kernel's wait for its shared-memory copies gave up (fm_step_status)")
              : FM_OK;
}

static int copy_real_plane(fm_lattice* L, const void* src, double* out, size_t N, bool is_double)
{
    if (is_double) {
        FM_CUDA(cudaMemcpyAsync(out, src, N * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
        FM_CUDA(cudaStreamSynchronize(L->stream));
        return device_status(L);
    }
    if (!L->d_wide) {
        int rc = dev_alloc(&L->d_wide, (size_t)L->ns, L->stream);
        if (rc) return rc;
    }
    k_widen<<<std::min(grid_for((long long)N), 148 * 16), kBlock, 0, L->stream>>>((const float*)src, L->d_wide,
                                                                                   (long long)N);
    FM_CHECK_LAUNCH("k_widen");
    FM_CUDA(cudaMemcpyAsync(out, L->d_wide, N * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return device_status(L);
}

// FP64 plane -> FP32 plane on the device
__global__ void k_narrow(const double* __restrict__ src, float* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

// device plane of R (or FP64 q) -> host floats: FP32 planes go straight into
// the caller's buffer, FP64 ones are narrowed on the device first
static int copy_real_plane_f32(fm_lattice* L, const void* src, float* out, size_t N, bool is_double)
{
    if (is_double) {
        if (!L->d_wide) {
            int rc = dev_alloc(&L->d_wide, (size_t)L->ns, L->stream);
            if (rc) return rc;
        }
        float* tmp = reinterpret_cast<float*>(L->d_wide);
        k_narrow<<<std::min(grid_for((long long)N), 148 * 16), kBlock, 0, L->stream>>>((const double*)src, tmp,
                                                                                       (long long)N);
        FM_CHECK_LAUNCH("k_narrow");
        src = tmp;
    }
    FM_CUDA(cudaMemcpyAsync(out, src, N * sizeof(float), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return device_status(L);
}

// All six fields (rho, ux, uy, uz, C, q; a null output is skipped) with one
// macroscopic pass and one synchronisation: each plane goes to the caller's
// buffer by one copy, after being widened or narrowed on the device into the
// staging plane when its type differs from the output's.  Every kernel and copy
// is queued on the lattice's stream, so the staging plane is reused in stream
// order and the copies run back to back.
}  // extern "C"

template <typename OutT>
static int get_fields_batched(fm_lattice* L, OutT* const out[6], size_t n)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!out || n != (size_t)L->n) return fail(FM_ERR_ARG, "fm_get_fields: size mismatch");
    const size_t N = (size_t)L->n;
    int rc = FM_OK;
    if (out[0] || out[1] || out[2] || out[3]) {
        if ((rc = ensure_plain(L))) return rc;
        if (!L->d_tmp && (rc = dev_alloc((char**)&L->d_tmp, (size_t)4 * L->ns * L->relt, L->stream))) return rc;
        if ((rc = dispatch<MacroOp>(L))) return rc;
    }
    if (!L->d_wide && (rc = dev_alloc(&L->d_wide, (size_t)L->ns, L->stream))) return rc;
    constexpr bool out_double = sizeof(OutT) == 8;
    const int grid = std::min(grid_for((long long)N), 148 * 16);
    for (int f = 0; f < 6; ++f) {
        if (!out[f]) continue;
        const void* src = f < 4 ? (const void*)((const char*)L->d_tmp + (size_t)f * L->ns * L->relt)
                                : (f == 4 ? L->phi : L->q);
        const bool src_double = (f == 5 ? L->qelt : L->relt) == 8;
        if (src_double == out_double) {
            FM_CUDA(cudaMemcpyAsync(out[f], src, N * sizeof(OutT), cudaMemcpyDeviceToHost, L->stream));
        } else if (out_double) {
            k_widen<<<grid, kBlock, 0, L->stream>>>((const float*)src, L->d_wide, (long long)N);
            FM_CHECK_LAUNCH("k_widen");
            FM_CUDA(cudaMemcpyAsync(out[f], L->d_wide, N * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
        } else {
            float* tmp = reinterpret_cast<float*>(L->d_wide);
            k_narrow<<<grid, kBlock, 0, L->stream>>>((const double*)src, tmp, (long long)N);
            FM_CHECK_LAUNCH("k_narrow");
            FM_CUDA(cudaMemcpyAsync(out[f], tmp, N * sizeof(float), cudaMemcpyDeviceToHost, L->stream));
        }
    }
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return device_status(L);
}

extern "C" {

int fm_get_field_f32(fm_lattice* L, int field, float* out, size_t n)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!out || n != (size_t)L->n) return fail(FM_ERR_ARG, "fm_get_field_f32: size mismatch");
    const size_t N = (size_t)L->n;
    if (field >= FM_FIELD_RHO && field <= FM_FIELD_UZ) {
        int prc = ensure_plain(L);
        if (prc) return prc;
        if (!L->d_tmp) {
            int rc = dev_alloc((char**)&L->d_tmp, (size_t)4 * L->ns * L->relt, L->stream);
            if (rc) return rc;
        }
        int rc = dispatch<MacroOp>(L);
        if (rc) return rc;
        return copy_real_plane_f32(L, (const char*)L->d_tmp + (size_t)field * L->ns * L->relt, out, N, L->relt == 8);
    }
    if (field == FM_FIELD_C) return copy_real_plane_f32(L, L->phi, out, N, L->relt == 8);
    if (field == FM_FIELD_Q) return copy_real_plane_f32(L, L->q, out, N, L->qelt == 8);
    return fail(FM_ERR_ARG, "fm_get_field_f32: unknown field");
}

int fm_get_fields(fm_lattice* L, double* const out[6], size_t n) { return get_fields_batched(L, out, n); }
int fm_get_fields_f32(fm_lattice* L, float* const out[6], size_t n) { return get_fields_batched(L, out, n); }

int fm_get_field(fm_lattice* L, int field, double* out, size_t n)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!out || n != (size_t)L->n) return fail(FM_ERR_ARG, "fm_get_field: size mismatch");
    const size_t N = (size_t)L->n;
    if (field >= FM_FIELD_RHO && field <= FM_FIELD_UZ) {
        int prc = ensure_plain(L);
        if (prc) return prc;
        if (!L->d_tmp) {
            int rc = dev_alloc((char**)&L->d_tmp, (size_t)4 * L->ns * L->relt, L->stream);
            if (rc) return rc;
        }
        int rc = dispatch<MacroOp>(L);
        if (rc) return rc;
        return copy_real_plane(L, (const char*)L->d_tmp + (size_t)field * L->ns * L->relt, out, N, L->relt == 8);
    }
    if (field == FM_FIELD_C) return copy_real_plane(L, L->phi, out, N, L->relt == 8);
    if (field == FM_FIELD_Q) return copy_real_plane(L, L->q, out, N, L->qelt == 8);
    return fail(FM_ERR_ARG, "fm_get_field: unknown field");
}

int fm_set_outlet_probe(fm_lattice* L, const uint8_t* mask, size_t n, int every)
{
    if (check_mask(L, mask, n, "OutletCSV outlet")) return FM_ERR_ARG;
    if (every < 0) return fail(FM_ERR_ARG, "fm_set_outlet_probe: negative period");
    std::vector<int> cells = compress(mask, n);
    dev_free(L->probe, L->stream);
    L->probe = nullptr;
    L->nprobe = (int)cells.size();
    L->probe_every = every;
    L->bt_count = 0;
    int rc = upload_list(cells, &L->probe, L->stream);
    if (rc) return rc;
    if (L->initialised && every > 0 && L->step % every == 0) return take_sample(L);
    return FM_OK;
}

int fm_outlet_stats(fm_lattice* L, double out[3])
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!out) return fail(FM_ERR_ARG, "fm_outlet_stats: null output");
    if (!L->initialised) return fail(FM_ERR_STATE, "fm_outlet_stats: lattice not initialised");
    if (!L->nprobe) {
        out[0] = out[1] = out[2] = 0.0;
        return FM_OK;
    }
    if (L->relt == 8)
        fm::k_probe_stats<double><<<1, 1024, 0, L->stream>>>((const double*)L->phi, L->probe, L->nprobe, L->d_acc);
    else
        fm::k_probe_stats<float><<<1, 1024, 0, L->stream>>>((const float*)L->phi, L->probe, L->nprobe, L->d_acc);
    FM_CHECK_LAUNCH("k_probe_stats");
    FM_CUDA(cudaMemcpyAsync(out, L->d_acc, 3 * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return FM_OK;
}

int fm_get_breakthrough(fm_lattice* L, double* out, int capacity, int* count)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (count) *count = L->bt_count;
    if (!out || capacity <= 0 || !L->bt_count) {
        FM_CUDA(cudaStreamSynchronize(L->stream));
        return FM_OK;
    }
    const int m = std::min(capacity, L->bt_count);
    FM_CUDA(cudaMemcpyAsync(out, L->d_bt, sizeof(double) * m, cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return FM_OK;
}

int fm_reduce(fm_lattice* L, double out[4])
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!out) return fail(FM_ERR_ARG, "fm_reduce: null output");
    int rc = ensure_plain(L);
    if (rc) return rc;
    rc = dispatch<SumOp>(L);
    if (rc) return rc;
    FM_CUDA(cudaMemcpyAsync(out, L->d_acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return device_status(L);
}

int fm_get_state(fm_lattice* L, double* f, double* g, double* phi, double* q)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    int rc = f ? ensure_plain(L) : FM_OK;
    if (rc) return rc;
    rc = dispatch<GetPops>(L, f, g);
    if (rc) return rc;
    if (phi && (rc = fm_get_field(L, FM_FIELD_C, phi, (size_t)L->n))) return rc;
    if (q && (rc = fm_get_field(L, FM_FIELD_Q, q, (size_t)L->n))) return rc;
    return FM_OK;
}

int fm_set_state(fm_lattice* L, const double* f, const double* g, const double* phi, const double* q)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!L->initialised) return fail(FM_ERR_STATE, "fm_set_state: fm_init_equilibrium not called");
    int rc = dispatch<SetPops>(L, f, g);
    if (!rc && f) L->inlet_state = 0;   // every population, x = 0 included, is the caller's
    if (rc) return rc;
    const size_t N = (size_t)L->n;
    if (phi) {
        rc = upload_real_field(L, &L->phi, std::vector<double>(phi, phi + N));
        if (rc) return rc;
    }
    if (q) {
        if (L->qelt == 8) {
            FM_CUDA(cudaMemcpyAsync(L->q, q, N * sizeof(double), cudaMemcpyHostToDevice, L->stream));
            FM_CUDA(cudaStreamSynchronize(L->stream));
        } else {
            std::vector<float> h(N);
            for (size_t c = 0; c < N; ++c) h[c] = (float)q[c];
            FM_CUDA(cudaMemcpyAsync(L->q, h.data(), N * sizeof(float), cudaMemcpyHostToDevice, L->stream));
            FM_CUDA(cudaStreamSynchronize(L->stream));
        }
    }
    return FM_OK;
}

int fm_launch_henry_ldf_source_d3q7(int n_cells, const uint8_t* d_region, const float* d_phi, float* d_sphi,
                                    float* d_q, float k_henry, float k_ldf, float phi_min_clamp, void* stream)
{
    if (n_cells < 0 || (n_cells && (!d_region || !d_phi || !d_sphi || !d_q)))
        return fail(FM_ERR_ARG, "launch_henry_ldf_source_d3q7: bad arguments");
    if (!n_cells) return FM_OK;
    k_ldf_source_u8<<<grid_for(n_cells), kBlock, 0, (cudaStream_t)stream>>>(n_cells, d_region, d_phi, d_sphi, d_q, 0,
                                                                          k_henry, 0.0f, k_ldf, phi_min_clamp);
    FM_CHECK_LAUNCH("k_henry_ldf_source");
    return FM_OK;
}

int fm_launch_langmuir_ldf_source_d3q7(int n_cells, const uint8_t* d_region, const float* d_phi, float* d_sphi,
                                       float* d_q, float q_max, float b, float k_ldf, float phi_min_clamp,
                                       void* stream)
{
    if (n_cells < 0 || (n_cells && (!d_region || !d_phi || !d_sphi || !d_q)))
        return fail(FM_ERR_ARG, "launch_langmuir_ldf_source_d3q7: bad arguments");
    if (!n_cells) return FM_OK;
    k_ldf_source_u8<<<grid_for(n_cells), kBlock, 0, (cudaStream_t)stream>>>(n_cells, d_region, d_phi, d_sphi, d_q, 1,
                                                                          q_max, b, k_ldf, phi_min_clamp);
    FM_CHECK_LAUNCH("k_langmuir_ldf_source");
    return FM_OK;
}

int fm_profile_enable(fm_lattice* L, int enabled)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    L->profiling = enabled != 0;
    L->prof_used = 0;
    return FM_OK;
}

int fm_profile_read(fm_lattice* L, double* kernel_ms, long long* launches)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    FM_CUDA(cudaStreamSynchronize(L->stream));
    double total = 0.0;
    for (size_t i = 0; i + 1 < L->prof_used; i += 2) {
        float ms = 0.0f;
        FM_CUDA(cudaEventElapsedTime(&ms, L->prof_ev[i], L->prof_ev[i + 1]));
        total += ms;
    }
    if (kernel_ms) *kernel_ms = total;
    if (launches) *launches = (long long)(L->prof_used / 2);
    L->prof_used = 0;
    return FM_OK;
}

}  // extern "C"

namespace {
template <typename T, typename QT>
int pull_copy_run(fm_lattice* L, int reps, double* ms_per_rep, double* bytes_per_rep)
{
    const long long nx = L->p.nx, nxy = (long long)L->p.nx * L->p.ny;
    const long long c_lo = nxy + nx + 1, c_hi = (long long)L->n - nxy - nx - 1;
    if (c_hi <= c_lo || (L->layout == 1 && c_hi <= c_lo + 2))
        return fail(FM_ERR_ARG, "fm_bench_pull_copy: lattice too small (needs more than two z-planes)");
    const int A = L->cur, B = 1 - L->cur;
    // the pair layout: whole words, every source off the fold points
    const long long h = nx / 2, hny = h * L->p.ny;
    const long long w_lo = hny + h + 1, w_hi = (long long)L->n / 2 - hny - h - 1;
    const bool pair = L->layout == 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    FM_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return fail(FM_ERR_CUDA, "cudaEventCreate failed"); }
    auto launch = [&]() {
        if (pair)
            fm::k_pull_copy_pair<<<grid_for(w_hi - w_lo), kBlock, 0, L->stream>>>(
                (const uint32_t*)L->f[A], (uint32_t*)L->f[B], (const uint32_t*)L->g[A], (uint32_t*)L->g[B],
                (uint32_t)(L->ns / 2), (int)h, (int)hny, (uint32_t)w_lo, (uint32_t)w_hi);
        else
            fm::k_pull_copy<T><<<grid_for(c_hi - c_lo), kBlock, 0, L->stream>>>(
                (const T*)L->f[A], (T*)L->f[B], (const T*)L->g[A], (T*)L->g[B], (uint32_t)L->ns, (int)nx, (int)nxy,
                (uint32_t)c_lo, (uint32_t)c_hi);
    };
    launch();
    cudaEventRecord(e0, L->stream);
    for (int i = 0; i < reps; ++i) launch();
    cudaEventRecord(e1, L->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("fm_bench_pull_copy: ") + cudaGetErrorString(e));
    if (ms_per_rep) *ms_per_rep = ms / reps;
    if (bytes_per_rep)
        *bytes_per_rep = pair ? 2.0 * 26.0 * 4.0 * (double)(w_hi - w_lo) : 2.0 * 26.0 * sizeof(T) * (double)(c_hi - c_lo);
    return FM_OK;
}
template <typename T, typename QT> struct PullCopyOp {
    static int run(fm_lattice* L, int reps, double* ms, double* bytes) { return pull_copy_run<T, QT>(L, reps, ms, bytes); }
};
}  // namespace

extern "C" {

int fm_bench_pull_copy(fm_lattice* L, int reps, double* ms_per_rep, double* bytes_per_rep)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (reps < 1) return fail(FM_ERR_ARG, "fm_bench_pull_copy: reps must be >= 1");
    return dispatch<PullCopyOp>(L, reps, ms_per_rep, bytes_per_rep);
}

int fm_set_monitor(fm_lattice* L, int every)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (every < 0) return fail(FM_ERR_ARG, "fm_set_monitor: negative period");
    if (every > 0 && !L->d_mon_part) {
        int rc = dev_alloc(&L->d_mon_part, (size_t)grid_for(L->n) * fm::kMonN, L->stream);
        if (rc) return rc;
    }
    L->mon_every = every;
    L->mon_steps.clear();
    return FM_OK;
}

int fm_get_monitor(fm_lattice* L, double* out, int capacity, int* count)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    const int rows = (int)L->mon_steps.size();
    if (count) *count = rows;
    if (!out || capacity <= 0 || !rows) return FM_OK;
    const int m = std::min(capacity, rows);
    std::vector<double> h((size_t)m * fm::kMonN);
    FM_CUDA(cudaMemcpyAsync(h.data(), L->d_mon, h.size() * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    for (int i = 0; i < m; ++i) {
        out[(size_t)i * (fm::kMonN + 1)] = (double)L->mon_steps[(size_t)i];
        for (int j = 0; j < fm::kMonN; ++j) out[(size_t)i * (fm::kMonN + 1) + 1 + j] = h[(size_t)i * fm::kMonN + j];
    }
    return FM_OK;
}

int fm_trim_memory(size_t keep_bytes)
{
    cudaMemPool_t pool = nullptr;
    cudaError_t e = library_pool(&pool);
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, keep_bytes);
    if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("fm_trim_memory: ") + cudaGetErrorString(e));
    return FM_OK;
}

int fm_set_pair_layout(fm_lattice* L, int enabled)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    L->pair_pref = enabled ? 1 : 0;
    return FM_OK;
}

int fm_storage_layout(fm_lattice* L)
{
    if (!L) return fail(FM_ERR_ARG, "null lattice");
    int rc = prepare(L);
    if (!rc) rc = ensure_layout(L);
    return rc ? rc : L->layout;
}

int fm_set_pair_kernel(fm_lattice* L, int staged)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    L->staged_pref = staged ? 1 : 0;
    return FM_OK;
}

int fm_step_kernel(fm_lattice* L)
{
    if (!L) return fail(FM_ERR_ARG, "null lattice");
    int rc = prepare(L);
    if (!rc) rc = ensure_layout(L);
    if (rc) return rc;
    if (L->layout == 0) return L->elt == 2 && wide_offsets(L) ? 3 : 0;
    if (!staged_shape(L)) return 1;
    // the stages of this lattice's set-up (16-bit forms: 4-byte C, 8-byte q)
    const uint32_t rows = staged_rows(L);
    const fm::StageGeom g = fm::stage_geom(L->p.nx, rows, L->isotherm != FM_ISO_NONE,
                                           L->collision != FM_COLL_BGK && L->por != nullptr, L->tau_field, 8u, 4u);
    return fm::kStageHeader + 2 * (size_t)g.bytes <= kStageSmemMax ? 2 : 1;
}

int fm_step_status(fm_lattice* L, int* status)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!status) return fail(FM_ERR_ARG, "fm_step_status: null output");
    FM_CUDA(cudaMemcpyAsync(status, L->d_status, sizeof(int), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaMemsetAsync(L->d_status, 0, sizeof(int), L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return FM_OK;
}

int fm_set_prefetch_distance(fm_lattice* L, int blocks)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (blocks < 0) { L->pf_set = false; L->dirty = true; return FM_OK; }
    L->pf_set = true;
    L->pf_dist = (uint32_t)blocks;
    return FM_OK;
}

// ===========================================================================
// batching
// ===========================================================================
}  // extern "C"

struct fm_batch {
    std::vector<fm_lattice*> lats;
    int precision = FM_F32;
    int collision = FM_COLL_BGK;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int block = 256, cpt = 1, pf = 0, grid = 0;
    int mode = 3;                            // 0: shared-memory persistent kernel (global tables)
                                             // 1: constant-memory persistent, 2: constant-memory flat
                                             // 3: one k_coupled_step launch per lattice (kernel parameters)
    bool use_const = false;                  // tables fit in constant memory
    int nitems = 0;                          // work items (chunks)
    std::vector<uint32_t> item_off;          // per-lattice first work item (prefix sums)
    void* d_items[2] = {nullptr, nullptr};   // StepArgs tables for lattice parity 0 / 1
    std::vector<unsigned char> h_args[2];    // host StepArgs per parity, the lattices' own prefetch (mode 3)
    // mode 3 runs the lattices' launches on kSideStreams streams forked from
    // `stream` and joined back each step: lattices are independent within a
    // step, so one lattice's last wave overlaps the next one's first
    static constexpr int kSideStreams = 4;
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kSideStreams] = {};
    std::vector<int> side_of;                // side stream of each lattice (largest first, least loaded)
    fm::WorkItem* d_work = nullptr;
    uint32_t* d_off = nullptr;
    int nwork = 0;
    fm::ProbeItem* d_probes = nullptr;
    int nprobes = 0;
    int* d_counters = nullptr;
    std::vector<int> probe_lat;              // lattice of each probe item
    int probe_every = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    cudaEvent_t ev = nullptr;
    long long cells = 0;
};

namespace {

template <typename T, typename QT>
int batch_items(fm_batch* B)
{
    const size_t nb = sizeof(fm::StepArgs<T, QT>) * B->lats.size();
    std::vector<fm::StepArgs<T, QT>> h(B->lats.size());
    for (int par = 0; par < 2; ++par) {
        for (size_t i = 0; i < B->lats.size(); ++i) {
            fm_lattice* L = B->lats[i];
            const int keep = L->cur;
            L->cur = par;
            h[i] = make_args<T, QT>(L);
            L->cur = keep;
        }
        B->h_args[par].resize(nb);
        std::memcpy(B->h_args[par].data(), h.data(), nb);
        for (auto& a : h) a.pf_dist = 0;
        if (!B->d_items[par]) {
            int rc = dev_alloc((char**)&B->d_items[par], nb, B->stream);
            if (rc) return rc;
        }
        FM_CUDA(cudaMemcpyAsync(B->d_items[par], h.data(), nb, cudaMemcpyHostToDevice, B->stream));
        FM_CUDA(cudaStreamSynchronize(B->stream));
    }
    B->use_const = 2 * nb <= (size_t)fm::kBatchConstBytes && B->lats.size() <= (size_t)fm::kBatchMaxLattices;
    if (!B->use_const && (B->mode == 1 || B->mode == 2)) B->mode = 0;
    return FM_OK;
}
template <typename T, typename QT> struct BatchItemsOp {
    static int run(fm_lattice*, fm_batch* B) { return batch_items<T, QT>(B); }
};

// the argument tables and the work-item offsets into constant memory
// (device-to-device, stream-ordered, captured with the step graph)
template <typename T, typename QT>
int batch_upload_const(fm_batch* B)
{
    const size_t nb = sizeof(fm::StepArgs<T, QT>) * B->lats.size();
    for (int par = 0; par < 2; ++par)
        FM_CUDA(cudaMemcpyToSymbolAsync(fm::c_batch_args, B->d_items[par], nb, par * nb, cudaMemcpyDeviceToDevice,
                                        B->stream));
    FM_CUDA(cudaMemcpyToSymbolAsync(fm::c_batch_off, B->d_off, sizeof(uint32_t) * (B->lats.size() + 1), 0,
                                    cudaMemcpyDeviceToDevice, B->stream));
    return FM_OK;
}

template <typename T, typename QT>
int batch_launch_step(fm_batch* B, int parity)
{
    if (B->mode == 3) {
        const auto* args = reinterpret_cast<const fm::StepArgs<T, QT>*>(B->h_args[parity].data());
        FM_CUDA(cudaEventRecord(B->fork_ev, B->stream));
        for (int k = 0; k < fm_batch::kSideStreams; ++k) FM_CUDA(cudaStreamWaitEvent(B->side[k], B->fork_ev, 0));
        for (size_t i = 0; i < B->lats.size(); ++i) {
            cudaStream_t st = B->side[B->side_of[i]];
            if (B->collision == FM_COLL_BGK)
                fm::k_coupled_step<T, QT, false><<<grid_for(B->lats[i]->n), kBlock, 0, st>>>(args[i]);
            else
                fm::k_coupled_step<T, QT, true><<<grid_for(B->lats[i]->n), kBlock, 0, st>>>(args[i]);
        }
        FM_CHECK_LAUNCH("k_coupled_step (batch)");
        for (int k = 0; k < fm_batch::kSideStreams; ++k) {
            FM_CUDA(cudaEventRecord(B->join_ev[k], B->side[k]));
            FM_CUDA(cudaStreamWaitEvent(B->stream, B->join_ev[k], 0));
        }
        return FM_OK;
    }
    if (B->mode == 0) {
        const auto* items = (const fm::StepArgs<T, QT>*)B->d_items[parity];
        if (B->collision == FM_COLL_BGK)
            fm::k_coupled_batch<T, QT, false><<<B->grid, B->block, 0, B->stream>>>(items, B->d_work, B->nwork, B->cpt, B->pf);
        else
            fm::k_coupled_batch<T, QT, true><<<B->grid, B->block, 0, B->stream>>>(items, B->d_work, B->nwork, B->cpt, B->pf);
        FM_CHECK_LAUNCH("k_coupled_batch");
        return FM_OK;
    }
    const int persistent = B->mode == 1;
    const int grid = persistent ? B->grid : B->nitems;
    const int nlat = (int)B->lats.size();
    if (B->collision == FM_COLL_BGK)
        fm::k_coupled_batch_c<T, QT, false><<<grid, B->block, 0, B->stream>>>(nlat, parity, B->cpt, B->pf, persistent);
    else
        fm::k_coupled_batch_c<T, QT, true><<<grid, B->block, 0, B->stream>>>(nlat, parity, B->cpt, B->pf, persistent);
    FM_CHECK_LAUNCH("k_coupled_batch_c");
    return FM_OK;
}
template <typename T, typename QT> struct BatchConstOp {
    static int run(fm_lattice*, fm_batch* B) { return batch_upload_const<T, QT>(B); }
};
template <typename T, typename QT> struct BatchStepOp {
    static int run(fm_lattice*, fm_batch* B, int parity) { return batch_launch_step<T, QT>(B, parity); }
};

template <typename T, typename QT>
int batch_grid(fm_batch* B)
{
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e;
    if (B->mode == 0)
        e = B->collision == FM_COLL_BGK
                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fm::k_coupled_batch<T, QT, false>, B->block, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fm::k_coupled_batch<T, QT, true>, B->block, 0);
    else
        e = B->collision == FM_COLL_BGK
                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fm::k_coupled_batch_c<T, QT, false>, B->block, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fm::k_coupled_batch_c<T, QT, true>, B->block, 0);
    if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("occupancy: ") + cudaGetErrorString(e));
    B->grid = std::max(1, std::min(B->nwork, sms * std::max(per, 1)));
    return FM_OK;
}
template <typename T, typename QT> struct BatchGridOp {
    static int run(fm_lattice*, fm_batch* B) { return batch_grid<T, QT>(B); }
};

int batch_dispatch_items(fm_batch* B) { return dispatch<BatchItemsOp>(B->lats[0], B); }
int batch_dispatch_grid(fm_batch* B) { return dispatch<BatchGridOp>(B->lats[0], B); }
int batch_dispatch_step(fm_batch* B, int parity) { return dispatch<BatchStepOp>(B->lats[0], B, parity); }
int batch_dispatch_const(fm_batch* B)
{
    return (B->mode == 1 || B->mode == 2) ? dispatch<BatchConstOp>(B->lats[0], B) : FM_OK;
}

// the cell-range work list: chunks of block*cpt cells, lattice by lattice
int batch_work(fm_batch* B)
{
    const uint32_t chunk = (uint32_t)B->block * (uint32_t)B->cpt;
    std::vector<fm::WorkItem> w;
    B->item_off.assign(1, 0u);
    for (size_t i = 0; i < B->lats.size(); ++i) {
        for (uint32_t c = 0; c < (uint32_t)B->lats[i]->n; c += chunk) w.push_back({(int)i, c});
        B->item_off.push_back((uint32_t)w.size());
    }
    dev_free(B->d_work, B->stream);
    dev_free(B->d_off, B->stream);
    B->d_work = nullptr;
    B->d_off = nullptr;
    B->nwork = (int)w.size();
    B->nitems = (int)w.size();
    int rc = dev_alloc(&B->d_work, w.size(), B->stream);
    if (!rc) rc = dev_alloc(&B->d_off, B->item_off.size(), B->stream);
    if (rc) return rc;
    FM_CUDA(cudaMemcpyAsync(B->d_work, w.data(), w.size() * sizeof(fm::WorkItem), cudaMemcpyHostToDevice, B->stream));
    FM_CUDA(cudaMemcpyAsync(B->d_off, B->item_off.data(), B->item_off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            B->stream));
    FM_CUDA(cudaStreamSynchronize(B->stream));
    return batch_dispatch_grid(B);
}

void batch_drop_graph(fm_batch* B)
{
    if (B->graph) cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
    B->graph_steps = 0;
}

// probe table with room for `more` samples per lattice beyond the current count
int batch_probes(fm_batch* B, int more)
{
    std::vector<fm::ProbeItem> h;
    B->probe_lat.clear();
    bool moved = false;
    for (size_t i = 0; i < B->lats.size(); ++i) {
        fm_lattice* L = B->lats[i];
        if (!L->nprobe || L->probe_every <= 0) continue;
        const double* before = L->d_bt;
        int rc = ensure_bt_capacity(L, L->bt_count + more + 1);
        if (rc) return rc;
        moved = moved || before != L->d_bt;
        B->probe_lat.push_back((int)i);
        h.push_back({L->phi, L->probe, L->nprobe, L->d_bt, nullptr, L->bt_cap});
    }
    if ((int)h.size() != B->nprobes || moved || !B->d_probes) {
        batch_drop_graph(B);
        dev_free(B->d_probes, B->stream);
        dev_free(B->d_counters, B->stream);
        B->d_probes = nullptr;
        B->d_counters = nullptr;
        B->nprobes = (int)h.size();
        if (!B->nprobes) return FM_OK;
        int rc = dev_alloc(&B->d_counters, h.size(), B->stream);
        if (rc) return rc;
        for (size_t i = 0; i < h.size(); ++i) h[i].counter = B->d_counters + i;
        rc = dev_alloc(&B->d_probes, h.size(), B->stream);
        if (rc) return rc;
        FM_CUDA(cudaMemcpyAsync(B->d_probes, h.data(), h.size() * sizeof(fm::ProbeItem), cudaMemcpyHostToDevice,
                                B->stream));
        FM_CUDA(cudaStreamSynchronize(B->stream));
    }
    return FM_OK;
}

int batch_launch_probes(fm_batch* B)
{
    if (!B->nprobes) return FM_OK;
    if (B->precision == FM_F64) fm::k_probe_batch<double><<<B->nprobes, kBlock, 0, B->stream>>>(B->d_probes);
    else fm::k_probe_batch<float><<<B->nprobes, kBlock, 0, B->stream>>>(B->d_probes);
    FM_CHECK_LAUNCH("k_probe_batch");
    return FM_OK;
}

// one step of every lattice; `s` is the step number being completed
int batch_one(fm_batch* B, long long s, int parity)
{
    int rc = batch_dispatch_step(B, parity);
    if (rc) return rc;
    if (B->probe_every > 0 && s % B->probe_every == 0) return batch_launch_probes(B);
    return FM_OK;
}

long long gcd_ll(long long a, long long b) { return b ? gcd_ll(b, a % b) : a; }

// Before a batch launches anything: every lattice at the same step, its own
// pending work (set-up, the natural layout a batch steps, the fused inlet's
// representation) queued, and the batch's stream ordered after it.
int batch_ready(fm_batch* B)
{
    fm_lattice* L0 = B->lats[0];
    for (fm_lattice* L : B->lats) {
        if (L->step != L0->step || L->cur != L0->cur)
            return fail(FM_ERR_STATE, "fm_batch_step: lattices are no longer at the same step");
        int rc = prepare(L);
        if (!rc) rc = ensure_layout(L);
        if (!rc && L->fuse_inlet && L->inlet_state == 0) rc = dispatch<InletFusedOp>(L);
        if (rc) return rc;
        FM_CUDA(cudaEventRecord(B->ev, L->stream));
        FM_CUDA(cudaStreamWaitEvent(B->stream, B->ev, 0));
    }
    return FM_OK;
}

}  // namespace

extern "C" {

int fm_batch_create(fm_lattice* const* lattices, int count, void* stream, fm_batch** out)
{
    if (!out || !lattices || count <= 0) return fail(FM_ERR_ARG, "fm_batch_create: bad arguments");
    *out = nullptr;
    fm_lattice* L0 = lattices[0];
    for (int i = 0; i < count; ++i) {
        fm_lattice* L = lattices[i];
        if (!L) return fail(FM_ERR_ARG, "fm_batch_create: null lattice");
        if (!L->initialised) return fail(FM_ERR_STATE, "fm_batch_create: lattice not initialised");
        if (L->precision != L0->precision || L->collision != L0->collision)
            return fail(FM_ERR_ARG, "fm_batch_create: lattices differ in precision or collision operator");
        if (L->step != L0->step) return fail(FM_ERR_STATE, "fm_batch_create: lattices are at different steps");
        if (L->elt == 2 && wide_offsets(L))
            return fail(FM_ERR_UNSUPPORTED, "fm_batch_create: a 16-bit lattice of more than ~119M cells steps on its own");
        if (fm_launches_per_step(L) != 1)
            return fail(FM_ERR_UNSUPPORTED, "fm_batch_create: a lattice needs boundary kernels besides the fused "
                                            "step (full x-plane boundaries and even Nx are required)");
        const int every = (L->nprobe && L->probe_every > 0) ? L->probe_every : 0;
        const int every0 = (L0->nprobe && L0->probe_every > 0) ? L0->probe_every : 0;
        if (every && every0 && every != every0)
            return fail(FM_ERR_ARG, "fm_batch_create: outlet probes with different periods");
    }
    fm_batch* B = new fm_batch();
    B->lats.assign(lattices, lattices + count);
    for (fm_lattice* L : B->lats) ++L->in_batch;
    B->precision = L0->precision;
    B->collision = L0->collision;
    for (fm_lattice* L : B->lats) {
        B->cells += L->n;
        if (L->nprobe && L->probe_every > 0) B->probe_every = L->probe_every;
    }
    if (stream) B->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete B;
            return fail(FM_ERR_CUDA, "cudaStreamCreate failed");
        }
        B->own_stream = true;
    }
    int rc = cudaEventCreateWithFlags(&B->ev, cudaEventDisableTiming) == cudaSuccess ? FM_OK : FM_ERR_CUDA;
    if (!rc && cudaEventCreateWithFlags(&B->fork_ev, cudaEventDisableTiming) != cudaSuccess) rc = FM_ERR_CUDA;
    for (int k = 0; k < fm_batch::kSideStreams && !rc; ++k)
        if (cudaStreamCreateWithFlags(&B->side[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&B->join_ev[k], cudaEventDisableTiming) != cudaSuccess)
            rc = FM_ERR_CUDA;
    if (rc) { fm_batch_destroy(B); return fail(FM_ERR_CUDA, "fm_batch_create: stream or event creation failed"); }
    {
        // lattices onto side streams: largest first, each to the least-loaded stream
        std::vector<int> order(B->lats.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return B->lats[a]->n > B->lats[b]->n; });
        long long load[fm_batch::kSideStreams] = {};
        B->side_of.assign(B->lats.size(), 0);
        for (int i : order) {
            int k = 0;
            for (int j = 1; j < fm_batch::kSideStreams; ++j)
                if (load[j] < load[k]) k = j;
            B->side_of[i] = k;
            load[k] += B->lats[i]->n;
        }
    }
    if (!rc) rc = batch_dispatch_items(B);
    if (!rc) rc = batch_work(B);
    if (rc) { fm_batch_destroy(B); return rc; }
    *out = B;
    return FM_OK;
}

int fm_batch_destroy(fm_batch* B)
{
    if (!B) return FM_OK;
    if (B->stream) cudaStreamSynchronize(B->stream);
    batch_drop_graph(B);
    dev_free(B->d_items[0], B->stream); dev_free(B->d_items[1], B->stream); dev_free(B->d_work, B->stream); dev_free(B->d_probes, B->stream); dev_free(B->d_off, B->stream);
    dev_free(B->d_counters, B->stream);
    if (B->ev) cudaEventDestroy(B->ev);
    if (B->fork_ev) cudaEventDestroy(B->fork_ev);
    for (int k = 0; k < fm_batch::kSideStreams; ++k) {
        if (B->side[k]) { cudaStreamSynchronize(B->side[k]); cudaStreamDestroy(B->side[k]); }
        if (B->join_ev[k]) cudaEventDestroy(B->join_ev[k]);
    }
    if (B->own_stream) cudaStreamDestroy(B->stream);
    for (fm_lattice* L : B->lats) --L->in_batch;
    delete B;
    return FM_OK;
}

long long fm_batch_cells(const fm_batch* B) { return B ? B->cells : -1; }

int fm_batch_set_config(fm_batch* B, int block, int cells_per_thread, int prefetch)
{
    return fm_batch_set_mode(B, B ? B->mode : 3, block, cells_per_thread, prefetch);
}

int fm_batch_set_mode(fm_batch* B, int mode, int block, int cells_per_thread, int prefetch)
{
    if (!B) return fail(FM_ERR_ARG, "null batch");
    if ((block != 128 && block != 256) || cells_per_thread < 1 || cells_per_thread > 8 || prefetch < 0 ||
        prefetch > 1024)
        return fail(FM_ERR_ARG, "fm_batch_set_config: block 128|256, cells_per_thread 1..8, prefetch 0..1024");
    if (mode < 0 || mode > 3) return fail(FM_ERR_ARG, "fm_batch_set_mode: mode 0, 1, 2 or 3");
    if ((mode == 1 || mode == 2) && !B->use_const)
        return fail(FM_ERR_UNSUPPORTED, "fm_batch_set_mode: argument tables exceed constant memory; mode 0 only");
    B->mode = mode;
    B->block = block;
    B->cpt = cells_per_thread;
    B->pf = prefetch;
    batch_drop_graph(B);
    return batch_work(B);
}

int fm_batch_step(fm_batch* B, int nsteps)
{
    if (!B) return fail(FM_ERR_ARG, "null batch");
    if (nsteps < 0) return fail(FM_ERR_ARG, "fm_batch_step: negative step count");
    if (nsteps == 0) return FM_OK;
    fm_lattice* L0 = B->lats[0];
    int rc = batch_ready(B);
    if (rc) return rc;
    const long long every = B->probe_every;
    rc = batch_probes(B, every > 0 ? (int)(nsteps / every + 1) : 0);
    if (rc) return rc;
    if (B->nprobes) {
        std::vector<int> cnt(B->nprobes);
        for (int i = 0; i < B->nprobes; ++i) cnt[i] = B->lats[B->probe_lat[i]]->bt_count;
        FM_CUDA(cudaMemcpyAsync(B->d_counters, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, B->stream));
        FM_CUDA(cudaStreamSynchronize(B->stream));   // cnt lives on this host stack frame
    }
    // a graph covers G steps, G = lcm(2, probe period), starting at a step
    // that is a multiple of G (so the parity and the probe phase repeat)
    const long long G = every > 0 ? 2 * every / gcd_ll(2, every) : 2;
    long long s = L0->step;
    int parity = L0->cur;
    int left = nsteps;
    // constant tables are shared by every batch of the process: load this
    // batch's before its launches (and again inside its graph)
    if ((rc = batch_dispatch_const(B))) return rc;
    auto single = [&]() -> int {
        int r = batch_one(B, s + 1, parity);
        ++s;
        parity ^= 1;
        --left;
        return r;
    };
    while (left > 0 && s % G != 0)
        if ((rc = single())) return rc;
    if (left >= G) {
        if (!B->graph || B->graph_steps != G) {
            batch_drop_graph(B);
            cudaGraph_t g = nullptr;
            FM_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
            int rc2 = batch_dispatch_const(B);
            for (long long i = 0; i < G && !rc2; ++i)
                rc2 = batch_one(B, i + 1, (int)((parity + i) & 1));
            cudaError_t e = cudaStreamEndCapture(B->stream, &g);
            if (rc2) { if (g) cudaGraphDestroy(g); return rc2; }
            if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&B->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) { B->graph = nullptr; return fail(FM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
            B->graph_steps = (int)G;
        }
        while (left >= G) {
            FM_CUDA(cudaGraphLaunch(B->graph, B->stream));
            s += G;
            left -= (int)G;
        }
    }
    while (left > 0)
        if ((rc = single())) return rc;
    // bookkeeping: every lattice advanced nsteps; later work on a lattice's
    // own stream waits for the batch
    FM_CUDA(cudaEventRecord(B->ev, B->stream));
    for (fm_lattice* L : B->lats) {
        L->step += nsteps;
        L->cur = (L->cur + nsteps) & 1;
        FM_CUDA(cudaStreamWaitEvent(L->stream, B->ev, 0));
    }
    if (B->nprobes) {
        std::vector<int> cnt(B->nprobes);
        FM_CUDA(cudaMemcpyAsync(cnt.data(), B->d_counters, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, B->stream));
        FM_CUDA(cudaStreamSynchronize(B->stream));
        for (int i = 0; i < B->nprobes; ++i) B->lats[B->probe_lat[i]]->bt_count = cnt[i];
    }
    return FM_OK;
}

int fm_batch_synchronize(fm_batch* B)
{
    if (!B) return fail(FM_ERR_ARG, "null batch");
    FM_CUDA(cudaStreamSynchronize(B->stream));
    return FM_OK;
}

int fm_batch_autotune(fm_batch* B, int trial_steps, int* mode, int* block, int* cells_per_thread, int* prefetch,
                      double* best_ms_per_step)
{
    if (!B) return fail(FM_ERR_ARG, "null batch");
    const int trials = std::max(2, (trial_steps + 1) / 2 * 2);
    {
        const int rr = batch_ready(B);
        if (rr) return rr;
    }
    FM_CUDA(cudaStreamSynchronize(B->stream));   // ordered after the lattices' own streams (batch_ready)
    // snapshot of everything a step writes: both population buffers are
    // rewritten, so the current one, phi, q and x0post are saved
    struct Snap { fm_lattice* L; void *f, *g, *phi, *q, *x0; long long step; int cur, bt, inlet; };
    std::vector<Snap> snaps;
    int rc = FM_OK;
    for (fm_lattice* L : B->lats) {
        Snap sn{L, nullptr, nullptr, nullptr, nullptr, nullptr, L->step, L->cur, L->bt_count, L->inlet_state};
        const size_t fb = (size_t)19 * L->ns * L->elt, gb = (size_t)7 * L->ns * L->elt;
        rc = dev_alloc((char**)&sn.f, fb, B->stream);
        if (!rc) rc = dev_alloc((char**)&sn.g, gb, B->stream);
        if (!rc) rc = dev_alloc((char**)&sn.phi, (size_t)L->ns * L->relt, B->stream);
        if (!rc) rc = dev_alloc((char**)&sn.q, (size_t)L->ns * L->qelt, B->stream);
        if (!rc && L->x0post) rc = dev_alloc((char**)&sn.x0, (size_t)19 * L->rows_stride * L->elt, B->stream);
        snaps.push_back(sn);
        if (rc) break;
        FM_CUDA(cudaMemcpyAsync(sn.f, L->f[L->cur], fb, cudaMemcpyDeviceToDevice, B->stream));
        FM_CUDA(cudaMemcpyAsync(sn.g, L->g[L->cur], gb, cudaMemcpyDeviceToDevice, B->stream));
        FM_CUDA(cudaMemcpyAsync(sn.phi, L->phi, (size_t)L->ns * L->relt, cudaMemcpyDeviceToDevice, B->stream));
        FM_CUDA(cudaMemcpyAsync(sn.q, L->q, (size_t)L->ns * L->qelt, cudaMemcpyDeviceToDevice, B->stream));
        if (L->x0post)
            FM_CUDA(cudaMemcpyAsync(sn.x0, L->x0post, (size_t)19 * L->rows_stride * L->elt, cudaMemcpyDeviceToDevice,
                                    B->stream));
    }
    // prefetch distances in work items: the persistent modes prefetch their own
    // next items; in the flat mode the next items run in neighbouring blocks,
    // so the useful distance is a fraction of a resident wave (as k_coupled_step)
    const int blocks[2] = {128, 256}, cpts[3] = {1, 2, 4};
    const int pfs_run[4] = {0, 1, 2, 2}, pfs_flat[4] = {0, 64, 192, 384};
    int bb = B->block, bc = B->cpt, bp = B->pf, bm = B->mode;
    const int modes[4] = {3, 0, 1, 2};
    const int nmodes = B->use_const ? 4 : 2;
    double best = 1e300;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = fail(FM_ERR_CUDA, "cudaEventCreate failed");
    for (int im = 0; im < nmodes && !rc; ++im)
    for (int ib = 0; ib < 2 && !rc; ++ib)
        for (int ic = 0; ic < 3 && !rc; ++ic)
            for (int ip = 0; ip < 4 && !rc; ++ip) {
                const int* pfs = modes[im] == 2 ? pfs_flat : pfs_run;
                if (ip > 0 && pfs[ip] == pfs[ip - 1]) continue;
                // mode 3 launches the single-lattice kernel: one shape (256 threads, the lattices' own prefetch)
                if (modes[im] == 3 && (ib != 1 || ic != 0 || ip != 0)) continue;
                rc = fm_batch_set_mode(B, modes[im], blocks[ib], cpts[ic], pfs[ip]);
                if (!rc) rc = batch_dispatch_const(B);
                if (rc) break;
                int parity = B->lats[0]->cur;
                for (int i = 0; i < 2 && !rc; ++i, parity ^= 1) rc = batch_dispatch_step(B, parity);
                if (rc) break;
                cudaEventRecord(e0, B->stream);
                for (int i = 0; i < trials && !rc; ++i, parity ^= 1) rc = batch_dispatch_step(B, parity);
                cudaEventRecord(e1, B->stream);
                if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(FM_ERR_CUDA, "autotune sync failed"); break; }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms / trials < best) { best = ms / trials; bm = modes[im]; bb = blocks[ib]; bc = cpts[ic]; bp = pfs[ip]; }
            }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    // restore the state (the trials left every lattice's buffers at the same parity)
    for (const Snap& sn : snaps) {
        fm_lattice* L = sn.L;
        if (!rc && sn.f) {
            L->cur = sn.cur;
            cudaMemcpyAsync(L->f[L->cur], sn.f, (size_t)19 * L->ns * L->elt, cudaMemcpyDeviceToDevice, B->stream);
            cudaMemcpyAsync(L->g[L->cur], sn.g, (size_t)7 * L->ns * L->elt, cudaMemcpyDeviceToDevice, B->stream);
            cudaMemcpyAsync(L->phi, sn.phi, (size_t)L->ns * L->relt, cudaMemcpyDeviceToDevice, B->stream);
            cudaMemcpyAsync(L->q, sn.q, (size_t)L->ns * L->qelt, cudaMemcpyDeviceToDevice, B->stream);
            if (sn.x0)
                cudaMemcpyAsync(L->x0post, sn.x0, (size_t)19 * L->rows_stride * L->elt, cudaMemcpyDeviceToDevice,
                                B->stream);
            L->step = sn.step;
            L->bt_count = sn.bt;
            L->inlet_state = sn.inlet;
        }
        dev_free(sn.f, B->stream); dev_free(sn.g, B->stream); dev_free(sn.phi, B->stream); dev_free(sn.q, B->stream); dev_free(sn.x0, B->stream);
    }
    // the restored state is in place before anything else reads the lattices
    if (cudaStreamSynchronize(B->stream) != cudaSuccess && !rc) rc = fail(FM_ERR_CUDA, "autotune: restore failed");
    if (rc) return rc;
    rc = fm_batch_set_mode(B, bm, bb, bc, bp);
    if (rc) return rc;
    if (mode) *mode = bm;
    if (block) *block = bb;
    if (cells_per_thread) *cells_per_thread = bc;
    if (prefetch) *prefetch = bp;
    if (best_ms_per_step) *best_ms_per_step = best;
    return FM_OK;
}

// ===========================================================================
// adjoint of the breakthrough-curve loss
// ===========================================================================
}  // extern "C"

namespace {

// one stored state X_s of a lattice (population storage T, q type QT)
struct AdjState {
    void *f = nullptr, *g = nullptr, *phi = nullptr, *q = nullptr;
};

struct AdjCtx {
    fm_lattice* L = nullptr;
    long long s0 = 0;
    int every = 0;
    std::vector<double> wl;        // loss weight per step index t - s0 (0 if not sampled)
    std::vector<AdjState> pool;    // free state buffers
    AdjState tmp;                  // ping-pong partner of advances over several steps
    long long forward_steps = 0;   // recomputed forward steps (statistics)
    void* x0scratch = nullptr;     // x0post of recomputed steps
    AdjState lam[2];               // adjoint state (R): f 19, g 7, phi, q
    void *lfi = nullptr, *lgi = nullptr;
    double *gpor = nullptr, *gpar = nullptr;
    int cur = 0;
};

// bump allocator over the lattice's adjoint arena (256-byte aligned pieces)
struct Carver {
    char* base = nullptr;
    size_t off = 0;
    void* take(size_t bytes)
    {
        void* p = base ? base + off : nullptr;
        off += (bytes + 255) / 256 * 256;
        return p;
    }
    void state(const fm_lattice* L, AdjState& S, size_t fe, size_t ge, size_t pe, size_t qe)
    {
        S.f = take((size_t)19 * L->ns * fe);
        S.g = take((size_t)7 * L->ns * ge);
        S.phi = take((size_t)L->ns * pe);
        S.q = take((size_t)L->ns * qe);
    }
};

int adj_copy_state(const fm_lattice* L, AdjState& dst, const void* f, const void* g, const void* phi, const void* q)
{
    FM_CUDA(cudaMemcpyAsync(dst.f, f, (size_t)19 * L->ns * L->elt, cudaMemcpyDeviceToDevice, L->stream));
    FM_CUDA(cudaMemcpyAsync(dst.g, g, (size_t)7 * L->ns * L->elt, cudaMemcpyDeviceToDevice, L->stream));
    FM_CUDA(cudaMemcpyAsync(dst.phi, phi, (size_t)L->ns * L->relt, cudaMemcpyDeviceToDevice, L->stream));
    FM_CUDA(cudaMemcpyAsync(dst.q, q, (size_t)L->ns * L->qelt, cudaMemcpyDeviceToDevice, L->stream));
    return FM_OK;
}

// X_out = step(X_in) with the fused forward kernel on the given buffers
template <typename T, typename QT>
int adj_forward(AdjCtx& X, const AdjState& in, AdjState& out)
{
    using R = typename fm::Pop<T>::R;
    fm_lattice* L = X.L;
    FM_CUDA(cudaMemcpyAsync(out.phi, in.phi, (size_t)L->ns * sizeof(R), cudaMemcpyDeviceToDevice, L->stream));
    FM_CUDA(cudaMemcpyAsync(out.q, in.q, (size_t)L->ns * sizeof(QT), cudaMemcpyDeviceToDevice, L->stream));
    fm::StepArgs<T, QT> a = make_args<T, QT>(L);
    a.fA = (const T*)in.f; a.gA = (const T*)in.g;
    a.fB = (T*)out.f; a.gB = (T*)out.g;
    a.phi = (R*)out.phi; a.q = (QT*)out.q;
    a.x0post = (T*)X.x0scratch;
    a.pf_dist = 0;
    ++X.forward_steps;
    if (L->collision == FM_COLL_BGK) fm::k_coupled_step<T, QT, false><<<grid_for(L->n), kBlock, 0, L->stream>>>(a);
    else fm::k_coupled_step<T, QT, true><<<grid_for(L->n), kBlock, 0, L->stream>>>(a);
    FM_CHECK_LAUNCH("adjoint forward");
    return FM_OK;
}

// backward step t (forward step t maps X_{t-1} -> X_t): lam[cur] = lambda_t -> lambda_{t-1}
template <typename T, typename QT>
int adj_backward(AdjCtx& X, long long t, const AdjState& xprev)
{
    using R = typename fm::Pop<T>::R;
    fm_lattice* L = X.L;
    fm::AdjArgs<T, QT> A{};
    A.a = make_args<T, QT>(L);
    A.a.fA = (const T*)xprev.f; A.a.gA = (const T*)xprev.g;
    A.a.fB = nullptr; A.a.gB = nullptr;
    A.a.phi = (R*)xprev.phi; A.a.q = (QT*)xprev.q;
    A.a.pf_dist = 0;
    AdjState& l1 = X.lam[X.cur];
    AdjState& l0 = X.lam[1 - X.cur];
    A.lf1 = (const R*)l1.f; A.lg1 = (const R*)l1.g; A.lphi1 = (const R*)l1.phi; A.lq1 = (const R*)l1.q;
    A.lfi = (R*)X.lfi; A.lgi = (R*)X.lgi;
    A.lphi0 = (R*)l0.phi; A.lq0 = (R*)l0.q;
    A.gpor = X.gpor; A.gpar = X.gpar;
    A.wl = (R)X.wl[(size_t)(t - X.s0)];
    if (L->collision == FM_COLL_BGK) {
        fm::k_adj_cell<T, QT, false><<<grid_for(L->n), kBlock, 0, L->stream>>>(A);
        fm::k_adj_stream<T, QT, false><<<grid_for(L->n), kBlock, 0, L->stream>>>(A, (R*)l0.f, (R*)l0.g);
    } else {
        fm::k_adj_cell<T, QT, true><<<grid_for(L->n), kBlock, 0, L->stream>>>(A);
        fm::k_adj_stream<T, QT, true><<<grid_for(L->n), kBlock, 0, L->stream>>>(A, (R*)l0.f, (R*)l0.g);
    }
    if (L->fuse_inlet)
        fm::k_adj_inlet<T, QT><<<grid_for((long long)L->p.ny * L->p.nz * 32), kBlock, 0, L->stream>>>(A, (R*)l0.f);
    FM_CHECK_LAUNCH("adjoint step");
    X.cur = 1 - X.cur;
    return FM_OK;
}

// Binomial checkpointing.  Reversing l steps from a held start state with c
// free state buffers costs at least
//     t(l, c) = r l - C(c + r, r - 1)  forward steps,
// r the smallest repetition number with C(c + r, c) >= l (Griewank's
// binomial bound; r = 1 stores every intermediate state).  The optimal first
// split j minimises j + t(l - j, c - 1) + t(j, c): advance j steps, keep that
// state in one buffer, reverse the upper part with one buffer fewer, then the
// lower part again from the start state.
double binom_sat(int n, int k)
{
    if (k < 0 || k > n) return 0.0;
    double v = 1.0;
    for (int i = 1; i <= k; ++i) {
        v = v * (double)(n - k + i) / (double)i;
        if (v > 1e18) return 1e18;
    }
    return v;
}
double revolve_cost(long long l, int c)
{
    if (l <= 1) return 0.0;
    if (c <= 0) return 1e30;
    if (c == 1) return 0.5 * (double)l * (double)(l - 1);
    int r = 1;
    while (binom_sat(c + r, c) < (double)l) ++r;
    return (double)r * (double)l - binom_sat(c + r, r - 1);
}

// advance X_a by k >= 1 steps into dst, ping-ponging through X.tmp
template <typename T, typename QT>
int adj_advance(AdjCtx& X, const AdjState& xa, long long k, AdjState& dst)
{
    const AdjState* src = &xa;
    for (long long i = 0; i < k; ++i) {
        AdjState& out = ((k - 1 - i) % 2 == 0) ? dst : X.tmp;
        int rc = adj_forward<T, QT>(X, *src, out);
        if (rc) return rc;
        src = &out;
    }
    return FM_OK;
}

// Reverse backward steps b, b-1, ..., a+1 given X_a (kept intact), drawing
// state buffers from X.pool (returned on exit).
template <typename T, typename QT>
int adj_reverse(AdjCtx& X, long long a, long long b, const AdjState& xa)
{
    const long long l = b - a;
    if (l <= 0) return FM_OK;
    if (l == 1) return adj_backward<T, QT>(X, b, xa);
    const int c = (int)X.pool.size();
    if (c <= 0) return fail(FM_ERR_NOMEM, "adjoint: no state buffer left");
    if (l - 1 <= c) {
        // store every intermediate state, then reverse
        std::vector<AdjState> st;
        st.push_back(xa);
        for (long long i = 0; i < l - 1; ++i) {
            AdjState o = X.pool.back();
            X.pool.pop_back();
            int rc = adj_forward<T, QT>(X, st.back(), o);
            if (rc) return rc;
            st.push_back(o);
        }
        int rc = FM_OK;
        for (long long t = b; t > a && !rc; --t) rc = adj_backward<T, QT>(X, t, st[(size_t)(t - 1 - a)]);
        for (size_t i = 1; i < st.size(); ++i) X.pool.push_back(st[i]);
        return rc;
    }
    AdjState hold = X.pool.back();
    X.pool.pop_back();
    int rc = FM_OK;
    if (c == 1) {
        // one buffer: recompute X_{t-1} from X_a for every step
        for (long long t = b; t > a + 1 && !rc; --t) {
            rc = adj_advance<T, QT>(X, xa, t - 1 - a, hold);
            if (!rc) rc = adj_backward<T, QT>(X, t, hold);
        }
        if (!rc) rc = adj_backward<T, QT>(X, a + 1, xa);
    } else {
        long long best = 1;
        double bc = 1e300;
        for (long long j = 1; j < l; ++j) {
            const double v = (double)j + revolve_cost(l - j, c - 1) + revolve_cost(j, c);
            if (v < bc) { bc = v; best = j; }
        }
        rc = adj_advance<T, QT>(X, xa, best, hold);
        if (!rc) rc = adj_reverse<T, QT>(X, a + best, b, hold);
        if (!rc) {
            X.pool.push_back(hold);
            hold = AdjState{};
            rc = adj_reverse<T, QT>(X, a, a + best, xa);
        }
    }
    if (hold.f) X.pool.push_back(hold);
    return rc;
}

template <typename T, typename QT>
int adjoint_run(fm_lattice* L, int nsteps, const double* target, int ntarget, int checkpoint_every, int max_states,
                double* loss, double* grad_params, double* grad_porosity)
{
    using R = typename fm::Pop<T>::R;
    AdjCtx X;
    X.L = L;
    X.s0 = L->step;
    X.every = L->probe_every;
    const int C = checkpoint_every > 0 ? std::min(checkpoint_every, nsteps) : nsteps;
    const int nseg = (nsteps + C - 1) / C;
    const int nstates = std::max(1, std::min(max_states > 0 ? max_states : C - 1, C - 1));
    std::vector<AdjState> snaps((size_t)nseg);
    // ---- workspace: one arena, carved (a dry run sizes it) ----
    auto carve = [&](Carver& cv) {
        for (auto& sn : snaps) cv.state(L, sn, L->elt, L->elt, L->relt, L->qelt);
        cv.state(L, X.tmp, L->elt, L->elt, L->relt, L->qelt);
        X.pool.assign((size_t)nstates, AdjState{});
        for (auto& st : X.pool) cv.state(L, st, L->elt, L->elt, L->relt, L->qelt);
        cv.state(L, X.lam[0], sizeof(R), sizeof(R), sizeof(R), sizeof(R));
        cv.state(L, X.lam[1], sizeof(R), sizeof(R), sizeof(R), sizeof(R));
        X.lfi = cv.take((size_t)19 * L->ns * sizeof(R));
        X.lgi = cv.take((size_t)7 * L->ns * sizeof(R));
        X.gpor = (double*)cv.take(sizeof(double) * L->ns);
        X.gpar = (double*)cv.take(sizeof(double) * 3);
        X.x0scratch = L->rows_stride ? cv.take((size_t)19 * L->rows_stride * L->elt) : nullptr;
    };
    Carver dry;
    carve(dry);
    if (dry.off > L->adj_bytes) {
        dev_free(L->adj_arena, L->stream);
        L->adj_arena = nullptr;
        L->adj_bytes = 0;
        int rc = dev_alloc(&L->adj_arena, dry.off, L->stream);
        if (rc) return rc;
        L->adj_bytes = dry.off;
    }
    Carver cv;
    cv.base = L->adj_arena;
    carve(cv);
    // ---- forward with checkpoints (the lattice ends at X_{s0+nsteps}) ----
    const int bt0 = L->bt_count;
    int rc = FM_OK;
    for (int k = 0; k < nseg && !rc; ++k) {
        rc = adj_copy_state(L, snaps[k], L->f[L->cur], L->g[L->cur], L->phi, L->q);
        if (!rc) rc = fm_step(L, std::min(C, nsteps - k * C));
    }
    if (rc) return rc;
    // ---- loss and its weights on the sampled outlet means ----
    const int have = L->bt_count - bt0;
    if (ntarget > have) return fail(FM_ERR_ARG, "adjoint: more targets than breakthrough samples");
    std::vector<double> series((size_t)std::max(have, 1));
    if (have) {
        FM_CUDA(cudaMemcpyAsync(series.data(), L->d_bt + bt0, sizeof(double) * have, cudaMemcpyDeviceToHost,
                                L->stream));
        FM_CUDA(cudaStreamSynchronize(L->stream));
    }
    X.wl.assign((size_t)nsteps + 1, 0.0);
    double Ls = 0.0;
    for (int i = 0; i < ntarget; ++i) {
        const long long t = X.s0 + (long long)(i + 1) * X.every;
        const double r = series[(size_t)i] - target[i];
        Ls += r * r;
        X.wl[(size_t)(t - X.s0)] = 2.0 * r / (double)L->nprobe;
    }
    // ---- reverse sweep, segment by segment ----
    for (int i = 0; i < 2; ++i) {
        FM_CUDA(cudaMemsetAsync(X.lam[i].f, 0, (size_t)19 * L->ns * sizeof(R), L->stream));
        FM_CUDA(cudaMemsetAsync(X.lam[i].g, 0, (size_t)7 * L->ns * sizeof(R), L->stream));
        FM_CUDA(cudaMemsetAsync(X.lam[i].phi, 0, (size_t)L->ns * sizeof(R), L->stream));
        FM_CUDA(cudaMemsetAsync(X.lam[i].q, 0, (size_t)L->ns * sizeof(R), L->stream));
    }
    FM_CUDA(cudaMemsetAsync(X.gpor, 0, sizeof(double) * L->ns, L->stream));
    FM_CUDA(cudaMemsetAsync(X.gpar, 0, sizeof(double) * 3, L->stream));
    for (int k = nseg - 1; k >= 0 && !rc; --k) {
        const long long a = X.s0 + (long long)k * C;
        const long long b = std::min(a + C, X.s0 + nsteps);
        rc = adj_reverse<T, QT>(X, a, b, snaps[k]);
    }
    if (rc) return rc;
    double gp[3] = {0, 0, 0};
    FM_CUDA(cudaMemcpyAsync(gp, X.gpar, sizeof(gp), cudaMemcpyDeviceToHost, L->stream));
    if (grad_porosity)
        FM_CUDA(cudaMemcpyAsync(grad_porosity, X.gpor, sizeof(double) * L->n, cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    if (loss) *loss = Ls;
    if (grad_params) for (int i = 0; i < 3; ++i) grad_params[i] = gp[i];
    L->adj_forward_steps = X.forward_steps;
    return FM_OK;
}

template <typename T, typename QT> struct AdjointOp {
    static int run(fm_lattice* L, int nsteps, const double* target, int ntarget, int ce, int ms, double* loss,
                   double* gp, double* gpor)
    {
        return adjoint_run<T, QT>(L, nsteps, target, ntarget, ce, ms, loss, gp, gpor);
    }
};

}  // namespace

extern "C" {

int fm_adjoint_breakthrough(fm_lattice* L, int nsteps, const double* target, int ntarget, int checkpoint_every,
                            int max_stored_states, double* loss, double* grad_params, double* grad_porosity)
{
    if (L) L->adj_forward_steps = 0;
    if (check_lattice(L)) return FM_ERR_ARG;
    if (nsteps <= 0 || ntarget < 0 || (ntarget && !target)) return fail(FM_ERR_ARG, "fm_adjoint_breakthrough: bad arguments");
    if (!L->initialised || !L->collision_set) return fail(FM_ERR_STATE, "fm_adjoint_breakthrough: lattice not initialised");
    // the adjoint kernels recompute each cell in the reference's FP32 / FP64
    // evaluation order; the 16-bit forms update in deviation form
    if (L->precision != FM_F32 && L->precision != FM_F64)
        return fail(FM_ERR_UNSUPPORTED, "fm_adjoint_breakthrough: FP32 or FP64 lattices only");
    int rc = prepare(L);
    if (rc) return rc;
    const int nx = L->p.nx;
    if (!L->nprobe || L->probe_every <= 0 || L->step % L->probe_every != 0)
        return fail(FM_ERR_STATE, "fm_adjoint_breakthrough: needs an outlet probe whose period divides the current step");
    if (L->nprobe != L->p.ny * L->p.nz)
        return fail(FM_ERR_UNSUPPORTED, "fm_adjoint_breakthrough: the outlet probe must be the x = nx-1 plane");
    {
        std::vector<int> h((size_t)L->nprobe);
        FM_CUDA(cudaMemcpyAsync(h.data(), L->probe, h.size() * sizeof(int), cudaMemcpyDeviceToHost, L->stream));
        FM_CUDA(cudaStreamSynchronize(L->stream));
        for (size_t i = 0; i < h.size(); ++i)
            if (h[i] != nx - 1 + nx * (int)i) return fail(FM_ERR_UNSUPPORTED, "fm_adjoint_breakthrough: the outlet probe must be the x = nx-1 plane");
    }
    if (fm_launches_per_step(L) != 1 || !L->ad_pre.empty())
        return fail(FM_ERR_UNSUPPORTED, "fm_adjoint_breakthrough: only fused full-plane boundaries (even nx, no pulse) are differentiated");
    if (!L->ns_pre.empty() && !L->fuse_inlet)
        return fail(FM_ERR_UNSUPPORTED, "fm_adjoint_breakthrough: NS inlet must be the fused NEQ plane");
    if (L->fuse_inlet && L->inlet_state == 0 && (rc = dispatch<InletFusedOp>(L))) return rc;
    return dispatch<AdjointOp>(L, nsteps, target, ntarget, checkpoint_every, max_stored_states, loss, grad_params,
                               grad_porosity);
}

int fm_adjoint_release(fm_lattice* L)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    FM_CUDA(cudaStreamSynchronize(L->stream));
    dev_free(L->adj_arena, L->stream);
    L->adj_arena = nullptr;
    L->adj_bytes = 0;
    return FM_OK;
}

int fm_adjoint_stats(const fm_lattice* L, long long* recomputed_steps, long long* workspace_bytes)
{
    if (!L) return fail(FM_ERR_ARG, "null lattice");
    if (recomputed_steps) *recomputed_steps = L->adj_forward_steps;
    if (workspace_bytes) *workspace_bytes = (long long)L->adj_bytes;
    return FM_OK;
}

int fm_launches_per_step(const fm_lattice* L)
{
    if (!L) return -1;
    if (prepare(const_cast<fm_lattice*>(L))) return -1;
    int k = 1;
    if (!L->fuse_inlet)
        for (const Bc& b : L->ns_pre) k += b.count > 0;
    for (const Bc& b : L->ad_pre) k += b.count > 0;
    if (!L->fuse_outlet)
        for (const Bc& b : L->ns_post) k += b.count > 0;
    for (const Bc& b : L->ad_post) {
        if (b.kind == BC_AD_DIRICHLET && L->fuse_dirichlet) continue;
        if (b.kind == BC_AD_NEUMANN && L->fuse_neumann) continue;
        k += b.count > 0;
    }
    k += L->ndeferred > 0;
    return k;
}

}  // extern "C"

// one z-plane's 26 stored populations <-> a contiguous buffer [26][nx*ny]
// (each population's plane is one contiguous run of nx*ny cells)
template <typename E>
__global__ void k_zplane(E* __restrict__ f, E* __restrict__ g, E* __restrict__ buf, long long ns, long long nxy,
                         int z, int pack)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= 26LL * nxy) return;
    const int k = (int)(i / nxy);
    const long long r = i - (long long)k * nxy;
    E* p = (k < 19 ? f + (long long)k * ns : g + (long long)(k - 19) * ns) + (long long)z * nxy + r;
    if (pack) buf[i] = *p;
    else *p = buf[i];
}

static int zplane_copy(fm_lattice* L, int z, void* buf, int pack)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!buf || z < 0 || z >= L->p.nz) return fail(FM_ERR_ARG, "fm_pack/unpack_zplane: z outside [0, nz) or null buffer");
    if (!L->initialised) return fail(FM_ERR_STATE, "fm_pack/unpack_zplane: lattice not initialised");
    const long long nxy = (long long)L->p.nx * L->p.ny;
    const int grid = grid_for(26LL * nxy);
    void* f = L->f[L->cur];
    void* g = L->g[L->cur];
    switch (L->elt) {
    case 2:
        k_zplane<uint16_t><<<grid, kBlock, 0, L->stream>>>((uint16_t*)f, (uint16_t*)g, (uint16_t*)buf, L->ns, nxy, z, pack);
        break;
    case 4:
        k_zplane<uint32_t><<<grid, kBlock, 0, L->stream>>>((uint32_t*)f, (uint32_t*)g, (uint32_t*)buf, L->ns, nxy, z, pack);
        break;
    default:
        k_zplane<uint64_t><<<grid, kBlock, 0, L->stream>>>((uint64_t*)f, (uint64_t*)g, (uint64_t*)buf, L->ns, nxy, z, pack);
    }
    FM_CHECK_LAUNCH("k_zplane");
    return FM_OK;
}

// the populations of one z-plane that cross a z-face in direction `dir` <-> a
// contiguous buffer [6][nx*ny]: dir = +1 the D3Q19 directions with c_z = +1
// (5, 11, 12, 15, 16) and D3Q7 direction 5 -- what the slab above pulls from
// this plane; dir = -1 those with c_z = -1 (6, 13, 14, 17, 18) and D3Q7 6
template <typename E>
__global__ void k_zhalo(E* __restrict__ f, E* __restrict__ g, E* __restrict__ buf, long long ns, long long nxy, int z,
                        int dir, int pack)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= 6LL * nxy) return;
    const int j = (int)(i / nxy);
    const long long r = i - (long long)j * nxy;
    constexpr int up[5] = {5, 11, 12, 15, 16}, down[5] = {6, 13, 14, 17, 18};
    E* p = j < 5 ? f + (long long)(dir > 0 ? up[j] : down[j]) * ns : g + (long long)(dir > 0 ? 5 : 6) * ns;
    p += (long long)z * nxy + r;
    if (pack) buf[i] = *p;
    else *p = buf[i];
}

// the buffer the halo calls act on: the one the open split step is writing,
// else the current one
static int zhalo_copy(fm_lattice* L, int z, int dir, void* buf, int pack)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!buf || z < 0 || z >= L->p.nz || (dir != 1 && dir != -1))
        return fail(FM_ERR_ARG, "fm_pack/unpack_zhalo: z outside [0, nz), dir not +1 / -1, or null buffer");
    if (!L->initialised) return fail(FM_ERR_STATE, "fm_pack/unpack_zhalo: lattice not initialised");
    const long long nxy = (long long)L->p.nx * L->p.ny;
    const int grid = grid_for(6LL * nxy);
    const int b = L->split_open ? 1 - L->cur : L->cur;
    void* f = L->f[b];
    void* g = L->g[b];
    switch (L->elt) {
    case 2:
        k_zhalo<uint16_t><<<grid, kBlock, 0, L->stream>>>((uint16_t*)f, (uint16_t*)g, (uint16_t*)buf, L->ns, nxy, z,
                                                          dir, pack);
        break;
    case 4:
        k_zhalo<uint32_t><<<grid, kBlock, 0, L->stream>>>((uint32_t*)f, (uint32_t*)g, (uint32_t*)buf, L->ns, nxy, z,
                                                          dir, pack);
        break;
    default:
        k_zhalo<uint64_t><<<grid, kBlock, 0, L->stream>>>((uint64_t*)f, (uint64_t*)g, (uint64_t*)buf, L->ns, nxy, z,
                                                          dir, pack);
    }
    FM_CHECK_LAUNCH("k_zhalo");
    return FM_OK;
}

extern "C" {

int fm_pack_zhalo(fm_lattice* L, int z, int dir, void* d_buf) { return zhalo_copy(L, z, dir, d_buf, 1); }
int fm_unpack_zhalo(fm_lattice* L, int z, int dir, const void* d_buf)
{
    return zhalo_copy(L, z, dir, const_cast<void*>(d_buf), 0);
}

int fm_step_planes(fm_lattice* L, int z0, int z1)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (z0 < 0 || z1 > L->p.nz || z0 >= z1) return fail(FM_ERR_ARG, "fm_step_planes: planes outside [0, nz)");
    if (!L->collision_set) return fail(FM_ERR_STATE, "NSLattice: collision operator not set, could not step()!");
    if (!L->initialised) return fail(FM_ERR_STATE, "fm_step_planes: fm_init_equilibrium not called");
    if (L->isotherm != FM_ISO_NONE && !L->region) return fail(FM_ERR_STATE, "isotherm without region mask");
    if (!L->split_open) {
        int rc = prepare(L);
        if (!rc) rc = ensure_layout(L);
        if (rc) return rc;
        if (fm_launches_per_step(L) != 1)
            return fail(FM_ERR_UNSUPPORTED, "fm_step_planes: the step needs boundary kernels besides the fused one");
        // launches over planes keep the warps of a whole-lattice launch:
        // plane starts at a multiple of 32 cells (and 32 words of the pair layout)
        if (((long long)L->p.nx * L->p.ny) % 64 != 0)
            return fail(FM_ERR_UNSUPPORTED, "fm_step_planes: nx * ny must be a multiple of 64");
        if (L->fuse_inlet && L->inlet_state == 0) rc = dispatch<InletFusedOp>(L);
        if (rc) return rc;
        L->split_open = true;
    }
    return dispatch<PlanesOp>(L, z0, z1);
}

int fm_step_finish(fm_lattice* L)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!L->split_open) return fail(FM_ERR_STATE, "fm_step_finish: no step begun by fm_step_planes");
    L->split_open = false;
    L->cur = 1 - L->cur;
    L->step += 1;
    if (L->nprobe && L->probe_every > 0 && L->step % L->probe_every == 0) return take_sample(L);
    return FM_OK;
}

int fm_reduce_zrange(fm_lattice* L, int z0, int z1, double out[3])
{
    if (check_lattice(L)) return FM_ERR_ARG;
    if (!out || z0 < 0 || z1 > L->p.nz || z0 > z1) return fail(FM_ERR_ARG, "fm_reduce_zrange: planes outside [0, nz)");
    if (L->split_open) return fail(FM_ERR_STATE, "fm_reduce_zrange: a step begun by fm_step_planes is not finished");
    int rc = ensure_plain(L);
    if (rc) return rc;
    rc = dispatch<RangeSumOp>(L, z0, z1);
    if (rc) return rc;
    FM_CUDA(cudaMemcpyAsync(out, L->d_acc, 3 * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return FM_OK;
}

int fm_pack_zplane(fm_lattice* L, int z, void* d_buf) { return zplane_copy(L, z, d_buf, 1); }
int fm_unpack_zplane(fm_lattice* L, int z, const void* d_buf) { return zplane_copy(L, z, const_cast<void*>(d_buf), 0); }

int fm_debug_layout(const fm_lattice* L, long long* plane_stride, int* precision)
{
    if (!L) return fail(FM_ERR_ARG, "null lattice");
    if (plane_stride) *plane_stride = L->ns;
    if (precision) *precision = L->precision;
    return FM_OK;
}

int fm_debug_set_status(fm_lattice* L, int status)
{
    if (check_lattice(L)) return FM_ERR_ARG;
    FM_CUDA(cudaMemcpyAsync(L->d_status, &status, sizeof(int), cudaMemcpyHostToDevice, L->stream));
    FM_CUDA(cudaStreamSynchronize(L->stream));
    return FM_OK;
}

}  // extern "C"
