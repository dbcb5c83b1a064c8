// fm_kernels.cuh -- sm_100a kernels of the coupled D3Q19 NS + D3Q7 AD + LDF step.
//
// Memory layout (HBM):
//   f[2][19][ns], g[2][7][ns]  population buffers, structure of arrays; plane
//                              stride ns = N rounded up to 32 cells so every
//                              plane starts 128-byte aligned.  Buffer A holds
//                              the post-step populations of step s-1, buffer B
//                              receives step s; the roles swap every step.
//   phi[ns]                    AD scalar of the previous step (the LDF source
//                              at step s reads phi(s-1), src/main.cpp:328-335)
//   q[ns]                      adsorbed loading
//   cellw[ns]                  per-cell flag word (obstacle, bounce-back links,
//                              region, deferred)
//
// Storage formats (template parameter T) and the arithmetic type R = Pop<T>::R:
//   float          FP32 storage, FP32 arithmetic (the reference's float build)
//   __half / bf16  FP16 / BF16 storage of (value - shift), FP32 arithmetic
//   hq             FP16 D3Q19 as __half, 16-bit fixed-point D3Q7 (PopG<hq>)
//   double         FP64 storage and arithmetic (the reference as shipped)
// In the FP32 and FP64 forms every expression keeps the evaluation order of
// the reference kernel it restates (the library is built without multiply-add
// contraction), so they reproduce the reference bit for bit.  The 16-bit
// forms update in deviation form with explicit multiply-adds
// (coupled_cell_dev), which the reference order does not constrain.
//
// One fused kernel per step (k_coupled_step) does, per cell: the NS pull +
// collision (BGK with obstacle bounce-back or porous BGK), the NS velocity of
// the post-collision populations (the coupling of Lattice::computeMacroscopicDevice),
// the LDF source from phi(s-1) and q, and the D3Q7 pull + collision with that
// source.  Full x-plane boundaries (NEQ inlet, pressure outlet, AD Dirichlet
// and Neumann) are handled inside it; other boundary masks run as small
// kernels over compacted cell lists:
//   pre-collision  : NS velocity inlets (on f_A), AD tanh pulse (on g_A)
//   post-stream NS : pressure outlet, bounce-back BC (on f_B); the AD update of
//                    those cells needs their post-BC velocity, so the fused
//                    kernel skips them ("deferred") and k_ad_deferred does it
//   post-stream AD : Dirichlet inlet, Neumann outlet (on g_B)
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

namespace fm {

// ---------------------------------------------------------------------------
// velocity sets in the reference's order (include/core/descriptors/D3Q19.hpp:14-49,
// include/core/descriptors/D3Q7.hpp:10-27)
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ constexpr int cx19(int k)
{
    constexpr int v[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return v[k];
}
__host__ __device__ __forceinline__ constexpr int cy19(int k)
{
    constexpr int v[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    return v[k];
}
__host__ __device__ __forceinline__ constexpr int cz19(int k)
{
    constexpr int v[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    return v[k];
}
__host__ __device__ __forceinline__ constexpr int opp19(int k)
{
    constexpr int v[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    return v[k];
}
// weights as the descriptors spell them: DATA_TYPE(1)/DATA_TYPE(k)
template <typename R>
__host__ __device__ __forceinline__ constexpr R w19(int k)
{
    return k == 0 ? R(1) / R(3) : (k < 7 ? R(1) / R(18) : R(1) / R(36));
}
__host__ __device__ __forceinline__ constexpr int cx7(int k)
{
    constexpr int v[7] = {0, 1, -1, 0, 0, 0, 0};
    return v[k];
}
__host__ __device__ __forceinline__ constexpr int cy7(int k)
{
    constexpr int v[7] = {0, 0, 0, 1, -1, 0, 0};
    return v[k];
}
__host__ __device__ __forceinline__ constexpr int cz7(int k)
{
    constexpr int v[7] = {0, 0, 0, 0, 0, 1, -1};
    return v[k];
}
template <typename R>
__host__ __device__ __forceinline__ constexpr R w7(int k)
{
    return k == 0 ? R(1) / R(4) : R(1) / R(8);
}

// c.u with only the nonzero velocity components (c_i in {-1,0,1}); equal in
// IEEE arithmetic to the reference's cx*ux + cy*uy + cz*uz.
template <int CX, int CY, int CZ, typename R>
__device__ __forceinline__ R cdot(R ux, R uy, R uz)
{
    R e = R(0);
    bool first = true;
    if (CX != 0) { e = CX > 0 ? ux : -ux; first = false; }
    if (CY != 0) { e = first ? (CY > 0 ? uy : -uy) : (CY > 0 ? e + uy : e - uy); first = false; }
    if (CZ != 0) { e = first ? (CZ > 0 ? uz : -uz) : (CZ > 0 ? e + uz : e - uz); }
    return e;
}

// ---------------------------------------------------------------------------
// population storage: FP32 / FP64 as is; FP16 / BF16 hold the value minus a
// shift (w_i rho0 for f, w_i c_shift for g) and compute in FP32.
// ---------------------------------------------------------------------------
template <typename T> struct Pop;
template <> struct Pop<float> {
    using R = float;
    static constexpr bool kShifted = false;
    __device__ static __forceinline__ R ld(const float* p, R) { return __ldg(p); }
    __device__ static __forceinline__ R ld_coherent(const float* p, R) { return *p; }
    __device__ static __forceinline__ void st(float* p, R v, R) { *p = v; }
    __device__ static __forceinline__ R ld_raw(const float* p) { return __ldg(p); }
    __device__ static __forceinline__ void st_raw(float* p, R v) { *p = v; }
};
template <> struct Pop<double> {
    using R = double;
    static constexpr bool kShifted = false;
    __device__ static __forceinline__ R ld(const double* p, R) { return __ldg(p); }
    __device__ static __forceinline__ R ld_coherent(const double* p, R) { return *p; }
    __device__ static __forceinline__ void st(double* p, R v, R) { *p = v; }
    __device__ static __forceinline__ R ld_raw(const double* p) { return __ldg(p); }
    __device__ static __forceinline__ void st_raw(double* p, R v) { *p = v; }
};
template <> struct Pop<__half> {
    using R = float;
    static constexpr bool kShifted = true;
    __device__ static __forceinline__ R ld(const __half* p, R sh) { return __half2float(__ldg(p)) + sh; }
    __device__ static __forceinline__ R ld_coherent(const __half* p, R sh) { return __half2float(*p) + sh; }
    __device__ static __forceinline__ void st(__half* p, R v, R sh) { *p = __float2half_rn(v - sh); }
    // the stored value itself (the deviation from the shift)
    __device__ static __forceinline__ R ld_raw(const __half* p) { return __half2float(__ldg(p)); }
    __device__ static __forceinline__ void st_raw(__half* p, R v) { *p = __float2half_rn(v); }
};
template <> struct Pop<__nv_bfloat16> {
    using R = float;
    static constexpr bool kShifted = true;
    __device__ static __forceinline__ R ld(const __nv_bfloat16* p, R sh) { return __bfloat162float(__ldg(p)) + sh; }
    __device__ static __forceinline__ R ld_coherent(const __nv_bfloat16* p, R sh)
    {
        return __bfloat162float(*p) + sh;
    }
    __device__ static __forceinline__ void st(__nv_bfloat16* p, R v, R sh) { *p = __float2bfloat16_rn(v - sh); }
    __device__ static __forceinline__ R ld_raw(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
    __device__ static __forceinline__ void st_raw(__nv_bfloat16* p, R v) { *p = __float2bfloat16_rn(v); }
};

// FP16-shifted D3Q19 with 16-bit fixed-point D3Q7 (PopG<hq> below): the
// D3Q19 planes hold FP16 bits exactly as Pop<__half> does
struct hq {
    unsigned short bits;
};
template <> struct Pop<hq> {
    using R = float;
    static constexpr bool kShifted = true;
    __device__ static __forceinline__ R ld(const hq* p, R sh)
    {
        return __half2float(__ushort_as_half(__ldg(&p->bits))) + sh;
    }
    __device__ static __forceinline__ R ld_coherent(const hq* p, R sh)
    {
        return __half2float(__ushort_as_half(p->bits)) + sh;
    }
    __device__ static __forceinline__ void st(hq* p, R v, R sh) { p->bits = __half_as_ushort(__float2half_rn(v - sh)); }
    __device__ static __forceinline__ R ld_raw(const hq* p) { return __half2float(__ushort_as_half(__ldg(&p->bits))); }
    __device__ static __forceinline__ void st_raw(hq* p, R v) { p->bits = __half_as_ushort(__float2half_rn(v)); }
};

// shift of direction k for storage T (0 for unshifted formats)
template <typename T>
__device__ __forceinline__ typename Pop<T>::R fshift(int k, typename Pop<T>::R s)
{
    using R = typename Pop<T>::R;
    return Pop<T>::kShifted ? w19<R>(k) * s : R(0);
}
template <typename T>
__device__ __forceinline__ typename Pop<T>::R gshift(int k, typename Pop<T>::R s)
{
    using R = typename Pop<T>::R;
    return Pop<T>::kShifted ? w7<R>(k) * s : R(0);
}

// D3Q7 population storage: Pop<T> with the D3Q7 shift, except for hq, whose
// D3Q7 planes are unsigned 16-bit fixed point over w_k [kGLo, kGLo + kGRange]
// (step 2.5 w_k / 65535 = 3.8e-5 w_k everywhere in the range, against up to
// 2^-12 w_k for FP16 shifted by w_k / 2); values outside the range saturate.
// Code b stands for (b - kGZero) * kGStep * w_k: one integer subtract and one
// product (w_k is a power of two, so kGStep * w_k is exact), which rounds the
// same wherever it is evaluated -- a multiply followed by an add could be
// fused into one FMA by the code generator in some kernels and not in others.
template <typename T> struct PopG {
    using R = typename Pop<T>::R;
    __device__ static __forceinline__ R ld(const T* p, int k, R gsh) { return Pop<T>::ld(p, gshift<T>(k, gsh)); }
    __device__ static __forceinline__ void st(T* p, R v, int k, R gsh, uint32_t) { Pop<T>::st(p, v, gshift<T>(k, gsh)); }
};
constexpr float kGLo = -0.5f;
constexpr float kGRange = 2.5f;
constexpr float kGStep = kGRange / 65535.0f;   // value step of one code, before w_k
constexpr int kGZero = 13107;                   // the code of 0: -kGLo * 65535 / kGRange
static_assert(kGZero * 5 == 65535, "kGZero is -kGLo / kGRange of the 16-bit range");
template <> struct PopG<hq> {
    using R = float;
    __device__ static __forceinline__ R ld(const hq* p, int k, R)
    {
        return (R)((int)__ldg(&p->bits) - kGZero) * (w7<R>(k) * kGStep);
    }
    // Stochastic rounding: floor(t + r) with r in [0, 1) from a hash of the
    // value's bits, the cell and the direction, so E[stored] = t and changes
    // smaller than one step are not lost (round-to-nearest would freeze the
    // slowly rising concentration ahead of a front).  The draw depends only on
    // (value, cell, direction): runs are reproducible and independent of the
    // buffer a state is stored in.
    __device__ static __forceinline__ void st(hq* p, R v, int k, R, uint32_t cell)
    {
        // v / w_k is exact (w_k = 1/4 or 1/8)
        const R t = (v * (k == 0 ? R(4) : R(8)) - kGLo) * (65535.0f / kGRange);
        uint32_t h = __float_as_uint(v) ^ (cell * 0x9E3779B1u) ^ ((uint32_t)k << 27);
        // one xor-shift and one multiply, the draw from the product's top 24 bits
        // (a two-round finaliser measured 1.8% slower with the same error)
        h ^= h >> 16;
        h *= 0x7FEB352Du;
        const R r = (R)(h >> 8) * (1.0f / 16777216.0f);
        const R u = fminf(fmaxf(floorf(t + r), 0.0f), 65535.0f);
        p->bits = (unsigned short)u;
    }
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint32_t bit_at(const uint32_t* __restrict__ m, int c)
{
    return (__ldg(m + (c >> 5)) >> (c & 31)) & 1u;
}

// ---------------------------------------------------------------------------
// per-cell flag word (built once per set-up by k_build_flags)
// ---------------------------------------------------------------------------
constexpr uint32_t kSolid = 1u << 0;      // obstacle cell: on-site reversal (BGK)
// bits 1..18: the pull source of direction k is an in-domain obstacle cell
constexpr uint32_t kRegion = 1u << 19;    // adsorption region
constexpr uint32_t kDeferred = 1u << 20;  // AD update runs after the post-stream NS lists
constexpr uint32_t kFaceYZ = 1u << 21;    // y = 0, y = ny-1, z = 0 or z = nz-1
constexpr uint32_t kXLo = 1u << 22;       // x = 0
constexpr uint32_t kXHi = 1u << 23;       // x = nx-1

// division by an invariant divisor d: q = floor(c * M / 2^64) with
// M = ceil(2^64 / d) is exact for every 32-bit c (M = 0 encodes d = 1)
__host__ __device__ __forceinline__ uint32_t fastdiv(uint32_t c, unsigned long long M)
{
#ifdef __CUDA_ARCH__
    return M ? (uint32_t)__umul64hi((unsigned long long)c, M) : c;
#else
    return M ? (uint32_t)(((unsigned __int128)c * M) >> 64) : c;
#endif
}
inline unsigned long long fastdiv_magic(uint32_t d) { return d <= 1 ? 0ull : ~0ull / d + 1ull; }

// Storage element of cell c in the population planes: c itself in the natural
// layout (h = 0); in the pair layout of the 16-bit kernel (fm_pair.cuh), with
// h = nx / 2, word w of an x-row holds the cells x = w and x = w + h, so
// element = row nx + (x < h ? 2x : 2(x - h) + 1).  div_nx: fastdiv magic of nx.
__host__ __device__ __forceinline__ uint32_t pair_element(uint32_t c, uint32_t h, unsigned long long div_nx)
{
    if (!h) return c;
    const uint32_t r = fastdiv(c, div_nx);
    const uint32_t x = c - r * 2u * h;
    return r * 2u * h + (x < h ? 2u * x : 2u * (x - h) + 1u);
}

// ---------------------------------------------------------------------------
// kernel arguments; R = arithmetic type of storage T, QT = type of q
// ---------------------------------------------------------------------------
template <typename T, typename QT>
struct StepArgs {
    using R = typename Pop<T>::R;
    const T* __restrict__ fA;
    T* __restrict__ fB;
    const T* __restrict__ gA;
    T* __restrict__ gB;
    R* __restrict__ phi;
    QT* __restrict__ q;
    const uint32_t* __restrict__ cellw;   // per-cell flag word
    const R* __restrict__ porosity;       // porous collision
    const R* __restrict__ tau_ad;         // null: omega_ad for all cells
    unsigned long long div_nx, div_nxy;   // fastdiv magics
    uint32_t ns;                          // plane stride (elements); 19*ns < 2^32
    int n, nx, ny, nz;
    int px, py, pz;
    R omega;                              // NS 1/max(tau, 0.5001)
    R rho0;                               // NS density fallback (rho <= 0)
    R omega_ad;
    R min_conc;
    R f_shift, g_shift;                   // shifted storage: rho0 and c_shift
    int coupling;
    int isotherm;                         // 0 none, 1 linear, 2 Langmuir
    R iso_a, iso_b, iso_k;                // linear: K, -, k ; Langmuir: q_max, b, k
    // boundary planes handled inside the fused kernel (full x = 0 / x = nx-1 planes)
    int fuse_outlet;                      // PressureDirichlet at x = nx-1
    R rho_out;
    int fuse_neumann;                     // ADNeumannOutlet at x = nx-1
    int fuse_dirichlet;                   // ADDirichlet at x = 0
    R c_in;
    int fuse_inlet;                       // VelocityDirichletNEQ on the full x = 0 plane
    R uin_x, uin_y, uin_z;
    T* __restrict__ x0post;               // [19][rows]: post-collision populations of the x = 0 cells
    uint32_t rows_stride;                 // plane stride of x0post (ny*nz rounded up to 32)
    uint32_t pf_dist;                     // L2 prefetch distance in blocks (0 = off)
    unsigned long long div_h;             // fastdiv magic of nx / 2 (pair layout, fm_pair.cuh)
    uint32_t c_first, c_end;              // the launch's range: cells [c_first, c_end) (pair kernel: words)
    double* __restrict__ mon;             // monitored launches: per-block partial sums [gridDim.x][kMonN]
    R neg_zero;                           // -0, a value the code generator cannot see (fm_pair.cuh)
    uint32_t st_rows;                     // staged pair kernel: x-rows per tile (fm_pair.cuh)
    int* __restrict__ status;             // device status word: bit 0 a shared-memory stage wait gave up
};

// The step monitor: FP64 sums over the cells of a launch of the post-step
// density (the domain mass), C, q, the outlet flux C u_x over the x = nx-1
// cells, and the number of cells whose density is not positive or whose rho
// or C is not finite (a status word for diverged runs).
constexpr int kMonN = 5;
struct MonAcc {
    double v[kMonN] = {0.0, 0.0, 0.0, 0.0, 0.0};
    __device__ __forceinline__ void add(double rho, double c, double q, double flux, bool bad)
    {
        v[0] += rho;
        v[1] += c;
        v[2] += q;
        v[3] += flux;
        v[4] += bad ? 1.0 : 0.0;
    }
};

// block reduction of the monitor sums (warp shuffles, then warp 0) into
// dst[0..kMonN); every thread of the block calls it
__device__ __forceinline__ void monitor_block_reduce(MonAcc& m, double* __restrict__ dst)
{
    __shared__ double part[32][kMonN];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < kMonN; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m.v[j] += __shfl_xor_sync(0xffffffffu, m.v[j], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < kMonN; ++j) part[wid][j] = m.v[j];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int j = 0; j < kMonN; ++j) {
            double s = lane < nw ? part[lane][j] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) dst[j] = s;
        }
    }
}

// the value a 16-bit form stores for the deviation v (FP32 forms: v itself)
template <typename T>
__device__ __forceinline__ float stored16(float v)
{
    if constexpr (sizeof(T) != 2) return v;
    else if constexpr (std::is_same<T, __nv_bfloat16>::value) return __bfloat162float(__float2bfloat16_rn(v));
    else return __half2float(__float2half_rn(v));
}

// TMA bulk prefetch of `bytes` (multiple of 16, 16-byte aligned) into L2
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// The first warp of a block prefetches into L2 everything the block
// `pf_dist` blocks ahead reads at its own cells: the 19 + 7 population planes
// of buffer A, the flag words, phi, q and the optional per-cell fields.  Pulls
// from neighbouring rows and planes then find their data prefetched by the
// blocks that own those rows.  Segments start at a multiple of 256 cells and
// end inside the plane (ns is a multiple of 32 cells), so every prefetch is
// 16-byte aligned and in bounds.
template <typename T, typename QT>
__device__ __forceinline__ void prefetch_ahead(const StepArgs<T, QT>& a)
{
    using R = typename Pop<T>::R;
    if (a.pf_dist == 0 || threadIdx.x >= 32) return;
    const uint32_t c0 = a.c_first + (blockIdx.x + a.pf_dist) * blockDim.x;
    if (c0 >= a.ns) return;
    const uint32_t cnt = min((uint32_t)blockDim.x, a.ns - c0);
    const int lane = threadIdx.x;
    if (lane < 19) l2_prefetch(a.fA + (uint32_t)lane * a.ns + c0, cnt * (uint32_t)sizeof(T));
    else if (lane < 26) l2_prefetch(a.gA + (uint32_t)(lane - 19) * a.ns + c0, cnt * (uint32_t)sizeof(T));
    else if (lane == 26) l2_prefetch(a.cellw + c0, cnt * 4u);
    else if (lane == 27) l2_prefetch(a.phi + c0, cnt * (uint32_t)sizeof(R));
    else if (lane == 28 && a.isotherm) l2_prefetch(a.q + c0, cnt * (uint32_t)sizeof(QT));
    else if (lane == 29 && a.porosity) l2_prefetch(a.porosity + c0, cnt * (uint32_t)sizeof(R));
    else if (lane == 30 && a.tau_ad) l2_prefetch(a.tau_ad + c0, cnt * (uint32_t)sizeof(R));
}

// neighbour coordinates of a cell with the reference's mapCoord rule
// (src/collision/BGKCollision.cu:26-41): periodic wrap, else "outside".
// Index d = 1 - c_i selects the source x - c_i.
struct Nbr {
    int xs[3], yr[3], zp[3];
    bool xo[3], yo[3], zo[3];
    __device__ __forceinline__ Nbr(int x, int y, int z, int nx, int ny, int nz, int px, int py, int pz)
    {
        const int nxy = nx * ny;
        xs[0] = x - 1; xs[1] = x; xs[2] = x + 1;
        xo[0] = xo[1] = xo[2] = true;
        if (x == 0) { if (px) xs[0] = nx - 1; else xo[0] = false; }
        if (x == nx - 1) { if (px) xs[2] = 0; else xo[2] = false; }
        int ym = y - 1, yp = y + 1;
        yo[0] = yo[1] = yo[2] = true;
        if (y == 0) { if (py) ym = ny - 1; else yo[0] = false; }
        if (y == ny - 1) { if (py) yp = 0; else yo[2] = false; }
        yr[0] = ym * nx; yr[1] = y * nx; yr[2] = yp * nx;
        int zm = z - 1, zq = z + 1;
        zo[0] = zo[1] = zo[2] = true;
        if (z == 0) { if (pz) zm = nz - 1; else zo[0] = false; }
        if (z == nz - 1) { if (pz) zq = 0; else zo[2] = false; }
        zp[0] = zm * nxy; zp[1] = z * nxy; zp[2] = zq * nxy;
    }
    template <int CX, int CY, int CZ>
    __device__ __forceinline__ bool inside() const { return xo[1 - CX] && yo[1 - CY] && zo[1 - CZ]; }
    template <int CX, int CY, int CZ>
    __device__ __forceinline__ int src() const { return xs[1 - CX] + yr[1 - CY] + zp[1 - CZ]; }
};

__device__ __forceinline__ void cell_xyz(uint32_t c, int nx, int ny, unsigned long long mnx,
                                         unsigned long long mnxy, int& x, int& y, int& z)
{
    const uint32_t zz = fastdiv(c, mnxy);
    const uint32_t r = c - zz * (uint32_t)(nx * ny);
    const uint32_t yy = fastdiv(r, mnx);
    z = (int)zz;
    y = (int)yy;
    x = (int)(r - yy * (uint32_t)nx);
}

// ---------------------------------------------------------------------------
// NS pull of direction K.  Obstacle cell: own opposite population (on-site
// reversal, src/collision/BGKCollision.cu:90-97).  Fluid cell: keep-local
// outside non-periodic faces, own opposite population when the source is an
// obstacle (src/collision/BGKCollision.cu:105-130); porous: no reflection
// (src/collision/PorousBGKCollision.cu:88-101).
// ---------------------------------------------------------------------------
template <typename T, int K, bool BB, bool RAW = false>
__device__ __forceinline__ typename Pop<T>::R pull19(const T* __restrict__ fA, uint32_t ns, uint32_t c, const Nbr& nb,
                                                     uint32_t w, typename Pop<T>::R shift)
{
    constexpr int CX = cx19(K), CY = cy19(K), CZ = cz19(K);
    uint32_t off;
    if (K == 0) {
        off = c;
    } else if (BB && (w & kSolid)) {
        off = (uint32_t)opp19(K) * ns + c;
    } else if (!nb.inside<CX, CY, CZ>()) {
        off = (uint32_t)K * ns + c;
    } else if (BB && ((w >> K) & 1u)) {
        off = (uint32_t)opp19(K) * ns + c;
    } else {
        off = (uint32_t)K * ns + (uint32_t)nb.src<CX, CY, CZ>();
    }
    if (RAW) return Pop<T>::ld_raw(fA + off);
    return Pop<T>::ld(fA + off, shift);
}

// RAW: the stored values (for shifted storage, the deviations f - w rho0)
template <typename T, bool BB, bool RAW = false, int... Ks>
__device__ __forceinline__ void pull19_all(typename Pop<T>::R* fi, const T* __restrict__ fA, uint32_t ns, uint32_t c,
                                           const Nbr& nb, uint32_t w, typename Pop<T>::R fsh,
                                           std::integer_sequence<int, Ks...>)
{
    // w_k = w_opp(k), so the shift of a reflected population is that of its own plane
    ((fi[Ks] = pull19<T, Ks, BB, RAW>(fA, ns, c, nb, w, fshift<T>(Ks, fsh))), ...);
}

// f_new = f + omega (feq - f) with feq = w rho (1 + 3eu + 4.5eu^2 - 1.5u^2)
// written as in src/collision/BGKCollision.cu:163-176.
template <int K, typename R>
__device__ __forceinline__ R bgk19(R fi, R rho, R ux, R uy, R uz, R u2, R omega)
{
    const R eu = cdot<cx19(K), cy19(K), cz19(K)>(ux, uy, uz);
    const R cu = R(3) * eu;
    const R feq = w19<R>(K) * rho * (R(1) + cu + R(0.5) * cu * cu - R(1.5) * u2);
    return fi + omega * (feq - fi);
}

template <typename R, int... Ks>
__device__ __forceinline__ void collide19(R* fi, R rho, R ux, R uy, R uz, R omega, std::integer_sequence<int, Ks...>)
{
    const R u2 = ux * ux + uy * uy + uz * uz;
    ((fi[Ks] = bgk19<Ks>(fi[Ks], rho, ux, uy, uz, u2, omega)), ...);
}

template <typename R, int... Ks>
__device__ __forceinline__ void moments19(const R* f, R& rho, R& jx, R& jy, R& jz, std::integer_sequence<int, Ks...>)
{
    rho = R(0); jx = R(0); jy = R(0); jz = R(0);
    ((rho += f[Ks]), ...);
    ((jx = cx19(Ks) == 0 ? jx : (cx19(Ks) > 0 ? jx + f[Ks] : jx - f[Ks])), ...);
    ((jy = cy19(Ks) == 0 ? jy : (cy19(Ks) > 0 ? jy + f[Ks] : jy - f[Ks])), ...);
    ((jz = cz19(Ks) == 0 ? jz : (cz19(Ks) > 0 ? jz + f[Ks] : jz - f[Ks])), ...);
}

using Seq19 = std::make_integer_sequence<int, 19>;
using Seq7 = std::make_integer_sequence<int, 7>;

// velocity of a population set as Lattice::computeMacroscopicDevice forms it
// (src/core/Macros.cu:40-60): u = j / rho, zero if rho <= 0.
template <typename R>
__device__ __forceinline__ void macro_velocity(const R* f, R& ux, R& uy, R& uz)
{
    R r, jx, jy, jz;
    moments19(f, r, jx, jy, jz, Seq19{});
    const R inv = (r > R(0)) ? (R(1) / r) : R(0);
    ux = jx * inv; uy = jy * inv; uz = jz * inv;
}

// PressureDirichlet's equilibrium (src/boundary/ns/PressureDirichlet.cu:76-95):
// feq(rho_out, u) in the 1 + 3eu + 4.5eu^2 - 1.5u^2 form.
template <int K, typename R>
__device__ __forceinline__ R feq_outlet(R rho_out, R ux, R uy, R uz, R u2)
{
    const R eu = cdot<cx19(K), cy19(K), cz19(K)>(ux, uy, uz);
    return w19<R>(K) * rho_out * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * u2);
}
template <typename R, int... Ks>
__device__ __forceinline__ void feq_outlet_all(R* f, R rho_out, R ux, R uy, R uz, std::integer_sequence<int, Ks...>)
{
    const R u2 = ux * ux + uy * uy + uz * uz;
    ((f[Ks] = feq_outlet<Ks>(rho_out, ux, uy, uz, u2)), ...);
}

// ---------------------------------------------------------------------------
// Pulls of a cell away from the y/z faces: the normal source of direction K
// is the lattice constant K*ns - (cx + cy*nx + cz*nx*ny) from the cell's own
// base pointer; an x-face source keeps the cell's own value (non-periodic
// x) or wraps by nx; with bounce-back, a link to an obstacle source (or an
// obstacle cell, all of whose bits 1..18 are passed set) reads the own
// opposite population.  The same sources as pull19 / pull7 with Nbr, chosen
// by selects on constants instead of a per-axis neighbour table.
// OFF is the offset type.  Unsigned 32-bit is exact for every lattice: such
// a cell has 1 <= z <= nz-2, so ns > nx*ny + nx + 1 exceeds every shift and
// each source lies in [0, 19 ns) past the cell, and the lattice size limit
// keeps 19 ns below 2^32.  Signed int is exact while 18 ns + nx*ny + 2 nx + 1
// < 2^31 (lattices up to ~119M cells) and lets the compiler fold the constant
// x shift into the load: measured 3-7% faster for the 16-bit forms, no
// difference for FP32.
// ---------------------------------------------------------------------------
template <typename T, int K, bool BB, bool RAW = false, bool XF = true, typename OFF>
__device__ __forceinline__ typename Pop<T>::R pull19_fast(const T* __restrict__ base, OFF ns, int nx, int nxy,
                                                          int px, bool xlo, bool xhi, uint32_t lk,
                                                          typename Pop<T>::R shift)
{
    constexpr int CX = cx19(K), CY = cy19(K), CZ = cz19(K);
    OFF off = (OFF)K * ns - (OFF)(CX + CY * nx + CZ * nxy);
    if (XF && CX > 0 && xlo) off = px ? off + (OFF)nx : (OFF)K * ns;
    if (XF && CX < 0 && xhi) off = px ? off - (OFF)nx : (OFF)K * ns;
    if (BB && K != 0 && ((lk >> K) & 1u)) off = (OFF)opp19(K) * ns;
    if (RAW) return Pop<T>::ld_raw(base + off);
    return Pop<T>::ld(base + off, shift);
}

template <typename T, bool BB, bool RAW = false, bool XF = true, typename OFF, int... Ks>
__device__ __forceinline__ void pull19_fast_all(typename Pop<T>::R* fi, const T* __restrict__ base, OFF ns, int nx,
                                                int nxy, int px, bool xlo, bool xhi, uint32_t lk,
                                                typename Pop<T>::R fsh, std::integer_sequence<int, Ks...>)
{
    ((fi[Ks] = pull19_fast<T, Ks, BB, RAW, XF, OFF>(base, ns, nx, nxy, px, xlo, xhi, lk, fshift<T>(Ks, fsh))), ...);
}

// One NS collision of the pulled fn[19] in place (post-collision, before
// post-stream boundaries).
template <typename T, typename QT, bool POROUS>
__device__ __forceinline__ void ns_collide(const StepArgs<T, QT>& a, uint32_t c, uint32_t w, typename Pop<T>::R* fn)
{
    using R = typename Pop<T>::R;
    if (!POROUS && (w & kSolid)) return;   // on-site reversal: no collision
    R rho, jx, jy, jz;
    moments19(fn, rho, jx, jy, jz, Seq19{});
    R ux, uy, uz;
    if (!POROUS) {
        // src/collision/BGKCollision.cu:148-158
        if (!(rho > R(0))) { rho = a.rho0; ux = uy = uz = R(0); }
        else { const R inv = R(1) / rho; ux = jx * inv; uy = jy * inv; uz = jz * inv; }
    } else {
        // src/collision/PorousBGKCollision.cu:118-136
        if (!(rho > R(0))) { rho = a.rho0; jx = jy = jz = R(0); }
        const R inv = R(1) / rho;
        ux = jx * inv; uy = jy * inv; uz = jz * inv;
        R ph = __ldg(a.porosity + c);
        if (ph < R(0)) ph = R(0);
        if (ph > R(1)) ph = R(1);
        ux *= ph; uy *= ph; uz *= ph;
    }
    collide19(fn, rho, ux, uy, uz, a.omega, Seq19{});
}

// One NS update into fn[19]: pull, then collide.
template <typename T, typename QT, bool POROUS>
__device__ __forceinline__ void ns_update(const StepArgs<T, QT>& a, uint32_t c, const Nbr& nb, uint32_t w,
                                          typename Pop<T>::R* fn)
{
    pull19_all<T, !POROUS>(fn, a.fA, a.ns, c, nb, w, a.f_shift, Seq19{});
    ns_collide<T, QT, POROUS>(a, c, w, fn);
}

template <typename T, typename QT>
__device__ __forceinline__ void store19(const StepArgs<T, QT>& a, uint32_t c, const typename Pop<T>::R* fn)
{
    // the cell's base pointer plus a lattice-uniform plane offset per store
    T* const p = a.fB + c;
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(p + (size_t)k * a.ns, fn[k], fshift<T>(k, a.f_shift));
}

// ---------------------------------------------------------------------------
// D3Q7 pull with keep-local outside non-periodic faces
// (src/collision/ADBGKCollision.cu:74-93)
// ---------------------------------------------------------------------------
template <typename T, typename QT>
__device__ __forceinline__ void pull7(const StepArgs<T, QT>& a, uint32_t c, const Nbr& nb, typename Pop<T>::R* gi)
{
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        const int cx = cx7(k), cy = cy7(k), cz = cz7(k);
        const bool in = nb.xo[1 - cx] && nb.yo[1 - cy] && nb.zo[1 - cz];
        const uint32_t s = (uint32_t)(nb.xs[1 - cx] + nb.yr[1 - cy] + nb.zp[1 - cz]);
        gi[k] = PopG<T>::ld(a.gA + (uint32_t)k * a.ns + (in ? s : c), k, a.g_shift);
    }
}

// D3Q7 pulls of a cell away from the y/z faces (see pull19_fast)
template <typename T, int K, bool XF = true, typename OFF>
__device__ __forceinline__ typename Pop<T>::R pull7_fast(const T* __restrict__ base, OFF ns, int nx, int nxy, int px,
                                                         bool xlo, bool xhi, typename Pop<T>::R gsh)
{
    constexpr int CX = cx7(K), CY = cy7(K), CZ = cz7(K);
    OFF off = (OFF)K * ns - (OFF)(CX + CY * nx + CZ * nxy);
    if (XF && CX > 0 && xlo) off = px ? off + (OFF)nx : (OFF)K * ns;
    if (XF && CX < 0 && xhi) off = px ? off - (OFF)nx : (OFF)K * ns;
    return PopG<T>::ld(base + off, K, gsh);
}

template <typename T, bool XF = true, typename OFF, int... Ks>
__device__ __forceinline__ void pull7_fast_all(typename Pop<T>::R* gi, const T* __restrict__ base, OFF ns, int nx,
                                               int nxy, int px, bool xlo, bool xhi, typename Pop<T>::R gsh,
                                               std::integer_sequence<int, Ks...>)
{
    ((gi[Ks] = pull7_fast<T, Ks, XF, OFF>(base, ns, nx, nxy, px, xlo, xhi, gsh)), ...);
}

// LDF source of a cell (src/reaction/LinearLDF.cu:13-48, src/reaction/LangmuirLDF.cu:7-41)
// from its C(s-1) `cphi` and loading `qi`: S = -dq with dq = k (q_eq(C) - q);
// `commit` stores q + dq to a.q[c]; `qn` receives the cell's loading after
// the call.  Cells outside the region (or no isotherm) have S = 0.
template <typename T, typename QT>
__device__ __forceinline__ typename Pop<T>::R ldf_source_of(const StepArgs<T, QT>& a, uint32_t c, uint32_t w, bool commit,
                                                            typename Pop<T>::R cphi, QT qi, QT& qn)
{
    using R = typename Pop<T>::R;
    R S = R(0);
    qn = qi;
    if (a.isotherm != 0 && (w & kRegion)) {
        R cc = cphi;
        if (cc < a.min_conc) cc = a.min_conc;
        const R ce = cc - a.min_conc;
        QT qeq;
        if (a.isotherm == 1) {
            qeq = (QT)(a.iso_a * ce);
        } else {
            const R bc = a.iso_b * ce;
            qeq = (QT)(a.iso_a * (bc / (R(1) + bc)));
        }
        const QT dq = (QT)a.iso_k * (qeq - qi);
        if (commit) {
            qn = qi + dq;
            a.q[c] = qn;
        }
        S = (R)(-dq);
    }
    return S;
}
// the same with C(s-1) and q read from the lattice's arrays
template <typename T, typename QT>
__device__ __forceinline__ typename Pop<T>::R ldf_source(const StepArgs<T, QT>& a, uint32_t c, uint32_t w, bool commit)
{
    using R = typename Pop<T>::R;
    if (a.isotherm == 0 || !(w & kRegion)) return R(0);
    QT qn;
    return ldf_source_of(a, c, w, commit, a.phi[c], a.q[c], qn);
}

// the LDF source then the D3Q7 collision with that source (src/collision/ADBGKCollision.cu:95-124)
// of the pulled gi[7] into gn[7]; returns phi.  `commit` false: q is not updated.
template <typename T, typename QT>
__device__ __forceinline__ typename Pop<T>::R ad_collide(const StepArgs<T, QT>& a, uint32_t c, uint32_t w,
                                                         const typename Pop<T>::R* gi, typename Pop<T>::R ux,
                                                         typename Pop<T>::R uy, typename Pop<T>::R uz, bool commit,
                                                         typename Pop<T>::R* gn)
{
    using R = typename Pop<T>::R;
    const R S = ldf_source(a, c, w, commit);
    R ph = gi[0];
#pragma unroll
    for (int k = 1; k < 7; ++k) ph += gi[k];
    if (ph < a.min_conc) ph = a.min_conc;
    const R om = a.tau_ad ? R(1) / __ldg(a.tau_ad + c) : a.omega_ad;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        R eu;
        if (k == 0) eu = R(0);
        else if (k == 1) eu = ux;
        else if (k == 2) eu = -ux;
        else if (k == 3) eu = uy;
        else if (k == 4) eu = -uy;
        else if (k == 5) eu = uz;
        else eu = -uz;
        const R geq = w7<R>(k) * ph * (R(1) + R(4) * eu);
        gn[k] = gi[k] + om * (geq - gi[k]) + w7<R>(k) * S;
    }
    return ph;
}

template <typename T, typename QT>
__device__ __forceinline__ void store7(const StepArgs<T, QT>& a, uint32_t c, const typename Pop<T>::R* gn)
{
    T* const p = a.gB + c;
#pragma unroll
    for (int k = 0; k < 7; ++k) PopG<T>::st(p + (size_t)k * a.ns, gn[k], k, a.g_shift, c);
}

// direction sets as bit masks, for per-lane (runtime) direction indices
constexpr uint32_t kPX = (1u << 1) | (1u << 7) | (1u << 9) | (1u << 11) | (1u << 13);
constexpr uint32_t kMX = (1u << 2) | (1u << 8) | (1u << 10) | (1u << 12) | (1u << 14);
constexpr uint32_t kPY = (1u << 3) | (1u << 7) | (1u << 8) | (1u << 15) | (1u << 17);
constexpr uint32_t kMY = (1u << 4) | (1u << 9) | (1u << 10) | (1u << 16) | (1u << 18);
constexpr uint32_t kPZ = (1u << 5) | (1u << 11) | (1u << 12) | (1u << 15) | (1u << 16);
constexpr uint32_t kMZ = (1u << 6) | (1u << 13) | (1u << 14) | (1u << 17) | (1u << 18);

// feq of direction j (runtime), as feq_d3q19 of src/boundary/ns/VelocityDirichletNEQ.cu:35-46
// writes it: eu = cx*ux + cy*uy + cz*uz with R(c) factors, then
// w rho (1 + cu + 0.5 cu^2 - 1.5 u^2), cu = 3 eu.
template <typename R>
__device__ __forceinline__ R feq19_dyn(int j, R rho, R ux, R uy, R uz)
{
    const R cx = (R)((int)((kPX >> j) & 1u) - (int)((kMX >> j) & 1u));
    const R cy = (R)((int)((kPY >> j) & 1u) - (int)((kMY >> j) & 1u));
    const R cz = (R)((int)((kPZ >> j) & 1u) - (int)((kMZ >> j) & 1u));
    const R w = j == 0 ? R(1) / R(3) : (j < 7 ? R(1) / R(18) : R(1) / R(36));
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R eu = cx * ux + cy * uy + cz * uz;
    const R cu = R(3) * eu;
    return w * rho * (R(1) + cu + R(0.5) * cu * cu - R(1.5) * u2);
}

// feq_outlet of a runtime direction k (c.u as cx ux + cy uy + cz uz, equal in
// IEEE arithmetic to cdot's form)
template <typename R>
__device__ __forceinline__ R feq_outlet_dyn(int k, R rho_out, R ux, R uy, R uz)
{
    const R cx = (R)((int)((kPX >> k) & 1u) - (int)((kMX >> k) & 1u));
    const R cy = (R)((int)((kPY >> k) & 1u) - (int)((kMY >> k) & 1u));
    const R cz = (R)((int)((kPZ >> k) & 1u) - (int)((kMZ >> k) & 1u));
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R eu = cx * ux + cy * uy + cz * uz;
    return w19<R>(k) * rho_out * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * u2);
}

// VelocityDirichletNEQ of the next step, fused (src/boundary/ns/VelocityDirichletNEQ.cu:49-96).
// Runs at the end of the step kernel, after every store, when little else is
// live.  Per x = 1 lane of the warp (one per x-row the warp holds):
//   - that lane reloads the 19 populations it stored and sums rho and j in the
//     order of src/core/Macros.cu:40-60, then broadcasts the four sums;
//   - lane k < 19 reloads direction k of the x = 0 cell (the previous lane's
//     stored value) into the x0post side plane, reloads direction k of the
//     x = 1 cell, forms f_k(0) = feq_k(rho_N, u_BC) + f_k,N - feq_k(rho_N, u_N)
//     and stores it over the x = 0 cell's population k.
// The reloads read other lanes' stores of this kernel (ordinary coherent loads
// after __syncwarp); one load and one store per lane replace a broadcast and a
// gather of 19 values per row.
// `e` is the storage element of cell c in the population planes (c itself in
// the natural layout; see the pair layout of fm_pair.cuh).
template <typename T, typename QT>
__device__ __forceinline__ void fused_inlet(const StepArgs<T, QT>& a, uint32_t c, uint32_t e, int x, bool active)
{
    using R = typename Pop<T>::R;
    const uint32_t m0 = __ballot_sync(0xffffffffu, active && x == 1);
    if (!m0) return;
    __syncwarp();   // the x = 0 and x = 1 lanes' stores are visible to the whole warp
    const int lane = threadIdx.x & 31;
    R r = R(0), jx = R(0), jy = R(0), jz = R(0);
    if (active && x == 1) {
#pragma unroll
        for (int k = 0; k < 19; ++k) {
            const R t = Pop<T>::ld_coherent(a.fB + (uint32_t)k * a.ns + e, fshift<T>(k, a.f_shift));
            r += t;
            if (cx19(k) != 0) jx = cx19(k) > 0 ? jx + t : jx - t;
            if (cy19(k) != 0) jy = cy19(k) > 0 ? jy + t : jy - t;
            if (cz19(k) != 0) jz = cz19(k) > 0 ? jz + t : jz - t;
        }
    }
    const uint32_t row = fastdiv(c, a.div_nx);   // the x-row of this lane's cell (x0post index)
    uint32_t m = m0;
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1u;
        const int dst = src - 1;   // the x = 0 cell of the same row
        const R rs = __shfl_sync(0xffffffffu, r, src);
        const R js_x = __shfl_sync(0xffffffffu, jx, src);
        const R js_y = __shfl_sync(0xffffffffu, jy, src);
        const R js_z = __shfl_sync(0xffffffffu, jz, src);
        const uint32_t e1 = __shfl_sync(0xffffffffu, e, src);
        const uint32_t e0 = __shfl_sync(0xffffffffu, e, dst);
        const uint32_t row0 = __shfl_sync(0xffffffffu, row, dst);
        if (lane < 19) {
            const R sh = fshift<T>(lane, a.f_shift);
            const R post = Pop<T>::ld_coherent(a.fB + (uint32_t)lane * a.ns + e0, sh);
            Pop<T>::st(a.x0post + (uint32_t)lane * a.rows_stride + row0, post, sh);
            const R mine = Pop<T>::ld_coherent(a.fB + (uint32_t)lane * a.ns + e1, sh);
            const R inv = (rs > R(0)) ? (R(1) / rs) : R(0);
            const R feqN = feq19_dyn(lane, rs, js_x * inv, js_y * inv, js_z * inv);
            const R feqB = feq19_dyn(lane, rs, a.uin_x, a.uin_y, a.uin_z);
            Pop<T>::st(a.fB + (uint32_t)lane * a.ns + e0, feqB + (mine - feqN), sh);
        }
    }
}

// ---------------------------------------------------------------------------
// The coupled update for shifted 16-bit storage (FP16 / BF16 / FP16 with
// fixed-point D3Q7), in deviation form.  The NS populations stay the stored
// deviations h_k = f_k - w_k rho0 (no shift added on load or removed on
// store); rho = rho0 + sum h, j = sum c h (the shifts' moments are rho0 and 0).
// The BGK equilibrium deviation is
//   feq_k - w_k rho0 = w_k (drho + rho t_k),  t_k = e (3 + 4.5 e) - 1.5 u^2,
// e = c_k.u, evaluated with multiply-adds over the three weight classes.  The
// velocity of the post-collision populations follows from the conservation
// of the collision (BGK: u; porous: u_bar (1 - omega (1 - phi)); an obstacle:
// its pulled velocity; the outlet plane: the velocity it was set to) instead
// of re-summing 19 moments.  These forms round differently from the FP32
// reference order, which the 16-bit forms do not keep anyway; the storage
// format is that of Pop<T>, so every other kernel reads and writes it as is.
// Every product that feeds a sum is written as an explicit FMA (u^2, the
// porous factor 1 - omega (1 - phi)), so the pair kernel (fm_pair.cuh), whose
// packed multiplies the code generator may fuse into a following add, rounds
// exactly as this one-cell update.
// ---------------------------------------------------------------------------
template <int CX, int CY, int CZ>
__device__ __forceinline__ float dev_eq(float h, float wr, float wd, float ux, float uy, float uz, float m15u2,
                                        float omega)
{
    const float e = cdot<CX, CY, CZ>(ux, uy, uz);
    const float t = fmaf(e, fmaf(4.5f, e, 3.0f), m15u2);
    const float heq = fmaf(wr, t, wd);
    return fmaf(omega, heq - h, h);
}
template <int... Ks>
__device__ __forceinline__ void dev_collide(float* h, float rho, float drho, float ux, float uy, float uz, float omega,
                                            std::integer_sequence<int, Ks...>)
{
    const float m15u2 = -1.5f * fmaf(ux, ux, fmaf(uy, uy, uz * uz));
    const float wr0 = rho * (1.0f / 3.0f), wr1 = rho * (1.0f / 18.0f), wr2 = rho * (1.0f / 36.0f);
    const float wd0 = drho * (1.0f / 3.0f), wd1 = drho * (1.0f / 18.0f), wd2 = drho * (1.0f / 36.0f);
    ((h[Ks] = dev_eq<cx19(Ks), cy19(Ks), cz19(Ks)>(h[Ks], Ks == 0 ? wr0 : (Ks < 7 ? wr1 : wr2),
                                                   Ks == 0 ? wd0 : (Ks < 7 ? wd1 : wd2), ux, uy, uz, m15u2, omega)),
     ...);
}
// the outlet plane: h_k = w_k (rho_out - rho0) + w_k rho_out t_k(u_N)
template <int... Ks>
__device__ __forceinline__ void dev_outlet(float* h, float rho_out, float drho_out, float ux, float uy, float uz,
                                           std::integer_sequence<int, Ks...>)
{
    const float m15u2 = -1.5f * fmaf(ux, ux, fmaf(uy, uy, uz * uz));
    ((h[Ks] = fmaf(rho_out * w19<float>(Ks),
                   fmaf(cdot<cx19(Ks), cy19(Ks), cz19(Ks)>(ux, uy, uz),
                        fmaf(4.5f, cdot<cx19(Ks), cy19(Ks), cz19(Ks)>(ux, uy, uz), 3.0f), m15u2),
                   drho_out * w19<float>(Ks))),
     ...);
}

// The NS collision of one cell in deviation form, in place on h[19]; returns
// the velocity of the post-collision populations.  Shared by the one-cell
// kernel and the rare (rho <= 0) path of the pair kernel (fm_pair.cuh).
template <typename T, typename QT, bool POROUS>
__device__ __forceinline__ void dev_ns_collide_por(const StepArgs<T, QT>& a, uint32_t w, float por, float* h, float& vx,
                                                   float& vy, float& vz)
{
    float drho, jx, jy, jz;
    moments19(h, drho, jx, jy, jz, Seq19{});
    const float rho = a.rho0 + drho;
    const bool ok = rho > 0.0f;
    if (!POROUS && (w & kSolid)) {
        const float inv = ok ? __frcp_rn(rho) : 0.0f;   // on-site reversal: no collision
        vx = jx * inv; vy = jy * inv; vz = jz * inv;
    } else if (!POROUS) {
        if (ok) {
            const float inv = __frcp_rn(rho);
            vx = jx * inv; vy = jy * inv; vz = jz * inv;
            dev_collide(h, rho, drho, vx, vy, vz, a.omega, Seq19{});
        } else {
            // rho <= 0: relax to feq(rho0, 0); rho' = (1-w) rho + w rho0, j' = (1-w) j
            dev_collide(h, a.rho0, 0.0f, 0.0f, 0.0f, 0.0f, a.omega, Seq19{});
            const float rp = (1.0f - a.omega) * rho + a.omega * a.rho0;
            const float inv = rp > 0.0f ? (1.0f - a.omega) / rp : 0.0f;
            vx = jx * inv; vy = jy * inv; vz = jz * inv;
        }
    } else {
        const float ph = fminf(fmaxf(por, 0.0f), 1.0f);
        const float rr = ok ? rho : a.rho0, dr = ok ? drho : 0.0f;
        const float inv = ok ? __frcp_rn(rho) : 0.0f;   // j = 0 when rho <= 0
        const float bx = jx * inv, by = jy * inv, bz = jz * inv;
        dev_collide(h, rr, dr, bx * ph, by * ph, bz * ph, a.omega, Seq19{});
        if (ok) {
            const float s = fmaf(-a.omega, 1.0f - ph, 1.0f);
            vx = bx * s; vy = by * s; vz = bz * s;
        } else {
            // the populations keep their momentum: j' = (1-w) j, rho' = (1-w) rho + w rho0
            const float rp = (1.0f - a.omega) * rho + a.omega * a.rho0;
            const float iv = rp > 0.0f ? (1.0f - a.omega) / rp : 0.0f;
            vx = jx * iv; vy = jy * iv; vz = jz * iv;
        }
    }
}

// the same with the porosity of cell c read from the lattice
template <typename T, typename QT, bool POROUS>
__device__ __forceinline__ void dev_ns_collide(const StepArgs<T, QT>& a, uint32_t c, uint32_t w, float* h, float& vx,
                                               float& vy, float& vz)
{
    dev_ns_collide_por<T, QT, POROUS>(a, w, POROUS ? __ldg(a.porosity + c) : 0.0f, h, vx, vy, vz);
}

template <typename T, typename QT, bool POROUS, bool MON = false, bool WIDE = false>
__device__ __forceinline__ void coupled_cell_dev(const StepArgs<T, QT>& a, uint32_t cg, MonAcc* mon = nullptr)
{
    static_assert(Pop<T>::kShifted, "deviation form: shifted storage only");
    const bool active = cg < a.c_end;
    const uint32_t c = active ? cg : a.c_end - 1u;
    int x, y, z;
    cell_xyz(c, a.nx, a.ny, a.div_nx, a.div_nxy, x, y, z);
    const uint32_t w = __ldg(a.cellw + c);
    float gi[7], h[19];
    const bool yz_face = y == 0 || y == a.ny - 1 || z == 0 || z == a.nz - 1;
    // warps with no cell at x = 0, 1 or nx-1 (rows start at even cells when
    // planes are fused, so x = 1 shares its warp with x = 0) skip the x-face
    // selects and the fused-plane work (measured: for the 16-bit forms the
    // coordinates cost less than the flag-word face bits the FP32 path tests)
    bool xedge = true;
    if (__any_sync(0xffffffffu, yz_face)) {
        const Nbr nb(x, y, z, a.nx, a.ny, a.nz, a.px, a.py, a.pz);
        pull7(a, c, nb, gi);
        pull19_all<T, !POROUS, true>(h, a.fA, a.ns, c, nb, w, 0.0f, Seq19{});
    } else {
        using Off = std::conditional_t<WIDE, uint32_t, int>;   // signed unless too large (pull19_fast)
        const Off ns = (Off)a.ns;
        const int nxy = a.nx * a.ny;
        const bool xlo = x == 0, xhi = x == a.nx - 1;
        const uint32_t lk = (!POROUS && (w & kSolid)) ? 0x7fffeu : w;
        xedge = __any_sync(0xffffffffu, xlo || xhi);
        if (xedge) {
            pull7_fast_all<T>(gi, a.gA + c, ns, a.nx, nxy, a.px, xlo, xhi, a.g_shift, Seq7{});
            pull19_fast_all<T, !POROUS, true>(h, a.fA + c, ns, a.nx, nxy, a.px, xlo, xhi, lk, 0.0f, Seq19{});
        } else {   // x-face selects compiled out
            pull7_fast_all<T, false>(gi, a.gA + c, ns, a.nx, nxy, a.px, false, false, a.g_shift, Seq7{});
            pull19_fast_all<T, !POROUS, true, false>(h, a.fA + c, ns, a.nx, nxy, a.px, false, false, lk, 0.0f,
                                                     Seq19{});
        }
    }

    // ---- NS collision (src/collision/BGKCollision.cu:140-176, PorousBGKCollision.cu:110-152) ----
    float vx, vy, vz;   // velocity of the post-collision populations
    dev_ns_collide<T, QT, POROUS>(a, c, w, h, vx, vy, vz);
    if (a.fuse_outlet && xedge) {
        const float lx = __shfl_up_sync(0xffffffffu, vx, 1);
        const float ly = __shfl_up_sync(0xffffffffu, vy, 1);
        const float lz = __shfl_up_sync(0xffffffffu, vz, 1);
        if (x == a.nx - 1) {
            dev_outlet(h, a.rho_out, a.rho_out - a.rho0, lx, ly, lz, Seq19{});
            vx = lx; vy = ly; vz = lz;
        }
    }
    if (active) {
#pragma unroll
        for (int k = 0; k < 19; ++k) Pop<T>::st_raw(a.fB + c + (size_t)k * a.ns, h[k]);
    }
    float mrho = 0.0f;
    const float mux = vx;
    if (MON) {
        // the density of the stored (rounded) populations
#pragma unroll
        for (int k = 0; k < 19; ++k) mrho += stored16<T>(h[k]);
        mrho += a.rho0;
    }
    if (!a.coupling) vx = vy = vz = 0.0f;

    // ---- LDF source and D3Q7 collision (src/collision/ADBGKCollision.cu:95-124) ----
    const bool do_ad = active && !(w & kDeferred);
    const float S = ldf_source(a, c, w, do_ad);
    float ph = gi[0];
#pragma unroll
    for (int k = 1; k < 7; ++k) ph += gi[k];
    ph = fmaxf(ph, a.min_conc);
    const float om = a.tau_ad ? __frcp_rn(__ldg(a.tau_ad + c)) : a.omega_ad;
    const float wp0 = 0.25f * ph, wp1 = 0.125f * ph, ws0 = 0.25f * S, ws1 = 0.125f * S;
    float gn[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        float eu;
        if (k == 0) eu = 0.0f;
        else if (k == 1) eu = vx;
        else if (k == 2) eu = -vx;
        else if (k == 3) eu = vy;
        else if (k == 4) eu = -vy;
        else if (k == 5) eu = vz;
        else eu = -vz;
        const float wp = k == 0 ? wp0 : wp1;
        const float geq = fmaf(4.0f * wp, eu, wp);
        gn[k] = fmaf(om, geq - gi[k], gi[k] + (k == 0 ? ws0 : ws1));
    }
    if (a.fuse_neumann && xedge) {
        float left[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) left[k] = __shfl_up_sync(0xffffffffu, gn[k], 1);
        if (x == a.nx - 1) {
#pragma unroll
            for (int k = 0; k < 7; ++k) gn[k] = left[k];
        }
    }
    if (a.fuse_dirichlet && x == 0) {
#pragma unroll
        for (int k = 0; k < 7; ++k) gn[k] = a.c_in * w7<float>(k);
    }
    if (do_ad) {
        store7(a, c, gn);
        a.phi[c] = ph;
    }
    if (MON && active) {
        mon->add((double)mrho, (double)ph, (double)a.q[c], (w & kXHi) ? (double)ph * (double)mux : 0.0,
                 !(mrho > 0.0f) || !isfinite(mrho) || !isfinite(ph));
    }
    if (a.fuse_inlet && xedge) fused_inlet(a, c, c, x, active);
}

// ---------------------------------------------------------------------------
// the fused step: one thread per cell, linear cell order (a warp covers 32
// consecutive cells, so x-neighbours in one row are adjacent lanes).  Lanes
// past the last cell stay alive for the warp shuffles but store nothing.  A
// launch covers cells [c_first, c_end); c_first is a multiple of 32, so the
// warps are those of a launch over the whole lattice.
// ---------------------------------------------------------------------------
template <typename T, typename QT, bool POROUS, bool MON = false, bool WIDE = false>
__device__ __forceinline__ void coupled_cell(const StepArgs<T, QT>& a, uint32_t cg, MonAcc* mon = nullptr)
{
    if constexpr (Pop<T>::kShifted) {
        coupled_cell_dev<T, QT, POROUS, MON, WIDE>(a, cg, mon);
        return;
    }
    using R = typename Pop<T>::R;
    const bool active = cg < a.c_end;
    const uint32_t c = active ? cg : a.c_end - 1u;
    const uint32_t w = __ldg(a.cellw + c);
    // the D3Q7 pull does not depend on the NS update: issue it first so its
    // loads are in flight together with the D3Q19 pull
    R gi[7], fn[19];
    // warps with no cell at x = 0, 1 or nx-1 (rows start at even cells when
    // planes are fused, so x = 1 shares its warp with x = 0) skip the x-face
    // selects and the fused-plane work, and never form x (-1 there)
    bool xedge = true;
    int x = -1;
    if (__any_sync(0xffffffffu, w & kFaceYZ)) {
        int y, z;
        cell_xyz(c, a.nx, a.ny, a.div_nx, a.div_nxy, x, y, z);
        const Nbr nb(x, y, z, a.nx, a.ny, a.nz, a.px, a.py, a.pz);
        pull7(a, c, nb, gi);
        pull19_all<T, !POROUS>(fn, a.fA, a.ns, c, nb, w, a.f_shift, Seq19{});
    } else {
        const uint32_t ns = a.ns;
        const int nxy = a.nx * a.ny;
        const bool xlo = (w & kXLo) != 0u, xhi = (w & kXHi) != 0u;
        const uint32_t lk = (!POROUS && (w & kSolid)) ? 0x7fffeu : w;
        xedge = __any_sync(0xffffffffu, xlo || xhi);
        if (xedge) {
            x = (int)(c - fastdiv(c, a.div_nx) * (uint32_t)a.nx);
            pull7_fast_all<T>(gi, a.gA + c, ns, a.nx, nxy, a.px, xlo, xhi, a.g_shift, Seq7{});
            pull19_fast_all<T, !POROUS>(fn, a.fA + c, ns, a.nx, nxy, a.px, xlo, xhi, lk, a.f_shift, Seq19{});
        } else {   // x-face selects compiled out
            pull7_fast_all<T, false>(gi, a.gA + c, ns, a.nx, nxy, a.px, false, false, a.g_shift, Seq7{});
            pull19_fast_all<T, !POROUS, false, false>(fn, a.fA + c, ns, a.nx, nxy, a.px, false, false, lk, a.f_shift,
                                                      Seq19{});
        }
    }
    ns_collide<T, QT, POROUS>(a, c, w, fn);
    R ux = R(0), uy = R(0), uz = R(0);
    if (a.coupling || a.fuse_outlet) macro_velocity(fn, ux, uy, uz);
    if (a.fuse_outlet && xedge) {
        // PressureDirichlet on the x = nx-1 plane: feq(rho_out, u of the
        // post-collision x-1 neighbour, which is the previous lane)
        const R lx = __shfl_up_sync(0xffffffffu, ux, 1);
        const R ly = __shfl_up_sync(0xffffffffu, uy, 1);
        const R lz = __shfl_up_sync(0xffffffffu, uz, 1);
        if constexpr (sizeof(R) == 4) {
            // FP32: the 19 equilibria of each outlet cell of the warp, one
            // direction per lane, gathered into the outlet lane (in place of 19
            // in that lane alone; FP64 keeps the one-lane form, whose registers
            // fit without spills)
            const int lane = threadIdx.x & 31;
            for (uint32_t m = __ballot_sync(0xffffffffu, x == a.nx - 1); m; m &= m - 1u) {
                const int o = __ffs(m) - 1;
                const R ox = __shfl_sync(0xffffffffu, lx, o);
                const R oy = __shfl_sync(0xffffffffu, ly, o);
                const R oz = __shfl_sync(0xffffffffu, lz, o);
                const R v = lane < 19 ? feq_outlet_dyn(lane, a.rho_out, ox, oy, oz) : R(0);
#pragma unroll
                for (int k = 0; k < 19; ++k) {
                    const R t = __shfl_sync(0xffffffffu, v, k);
                    if (lane == o) fn[k] = t;
                }
            }
        } else {
            if (x == a.nx - 1) feq_outlet_all(fn, a.rho_out, lx, ly, lz, Seq19{});
        }
        if (x == a.nx - 1) macro_velocity(fn, ux, uy, uz);
    }
    if (active) store19(a, c, fn);
    R mrho = R(0), mux = ux;
    if (MON) {
        // the density of the stored populations, summed as k_domain_sums sums them
#pragma unroll
        for (int k = 0; k < 19; ++k) mrho += fn[k];
        if (!(a.coupling || a.fuse_outlet)) {   // the velocity was not formed for the step itself
            R vy, vz;
            macro_velocity(fn, mux, vy, vz);
        }
    }
    if (!a.coupling) ux = uy = uz = R(0);

    const bool do_ad = active && !(w & kDeferred);
    R gn[7];
    const R ph = ad_collide(a, c, w, gi, ux, uy, uz, do_ad, gn);
    if (a.fuse_neumann && xedge) {
        // ADNeumannOutlet: x = nx-1 copies the post-collision x-1 neighbour
        R left[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) left[k] = __shfl_up_sync(0xffffffffu, gn[k], 1);
        if (x == a.nx - 1) {
#pragma unroll
            for (int k = 0; k < 7; ++k) gn[k] = left[k];
        }
    }
    if (a.fuse_dirichlet && x == 0) {
#pragma unroll
        for (int k = 0; k < 7; ++k) gn[k] = a.c_in * w7<R>(k);
    }
    if (do_ad) {
        store7(a, c, gn);
        a.phi[c] = ph;
    }
    if (MON && active) {
        mon->add((double)mrho, (double)ph, (double)a.q[c], (w & kXHi) ? (double)ph * (double)mux : 0.0,
                 !(mrho > R(0)) || !isfinite(mrho) || !isfinite(ph));
    }
    if (a.fuse_inlet && xedge) fused_inlet(a, c, c, x, active);
}

// resident 256-thread blocks per SM the step kernel is compiled for: 5 (at
// most 51 registers) for 4- and 2-byte populations; FP64 needs its 80
template <typename T>
constexpr int kStepBlocks = sizeof(T) == 8 ? 3 : 5;

// WIDE: unsigned pull offsets in the 16-bit cell update, for lattices too
// large for signed ones (FP32 and FP64 always use unsigned offsets)
template <typename T, typename QT, bool POROUS, bool MON = false, bool WIDE = false>
__global__ void __launch_bounds__(256, kStepBlocks<T>) k_coupled_step(const StepArgs<T, QT> a)
{
    prefetch_ahead(a);
    if constexpr (MON) {
        MonAcc m;
        coupled_cell<T, QT, POROUS, true, WIDE>(a, a.c_first + blockIdx.x * blockDim.x + threadIdx.x, &m);
        monitor_block_reduce(m, a.mon + (size_t)blockIdx.x * kMonN);
    } else {
        coupled_cell<T, QT, POROUS, false, WIDE>(a, a.c_first + blockIdx.x * blockDim.x + threadIdx.x);
    }
}

// the monitor's per-block partials of one launch, summed in a fixed order by
// one block, into out[0..kMonN)
__global__ void __launch_bounds__(256) k_monitor_fold(const double* __restrict__ part, int nblocks,
                                                      double* __restrict__ out)
{
    MonAcc m;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
        for (int j = 0; j < kMonN; ++j) m.v[j] += part[(size_t)b * kMonN + j];
    }
    monitor_block_reduce(m, out);
}

// ---------------------------------------------------------------------------
// The memory ceiling of the step's access pattern (a measurement aid): each
// cell reads the 19 + 7 pull sources of the fast path (plane k at
// cell - (c_x + c_y nx + c_z nx ny)) and writes them to its own slots of the B
// buffers, with no arithmetic, flag word, phi or q.  Only cells [c_lo, c_hi)
// run; the host picks them so that every source lies inside the lattice.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_pull_copy(const T* __restrict__ fA, T* __restrict__ fB,
                                                   const T* __restrict__ gA, T* __restrict__ gB, uint32_t ns, int nx,
                                                   int nxy, uint32_t c_lo, uint32_t c_hi)
{
    const uint32_t c = c_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c_hi) return;
    T v[19], u[7];
#pragma unroll
    for (int k = 0; k < 19; ++k)
        v[k] = fA[(size_t)k * ns + (c - (uint32_t)(cx19(k) + cy19(k) * nx + cz19(k) * nxy))];
#pragma unroll
    for (int k = 0; k < 7; ++k)
        u[k] = gA[(size_t)k * ns + (c - (uint32_t)(cx7(k) + cy7(k) * nx + cz7(k) * nxy))];
#pragma unroll
    for (int k = 0; k < 19; ++k) fB[(size_t)k * ns + c] = v[k];
#pragma unroll
    for (int k = 0; k < 7; ++k) gB[(size_t)k * ns + c] = u[k];
}

// ---------------------------------------------------------------------------
// batched step: many lattices (samples) in one persistent launch
// ---------------------------------------------------------------------------
// One work item is a chunk of `blockDim.x * cpt` consecutive cells of one
// lattice (a multiple of 32, so warps never straddle lattices or break the
// row/lane alignment the fused planes rely on).
struct WorkItem {
    int lattice;
    uint32_t first;
};

// L2 prefetch of a work item's own segments (as prefetch_ahead, for a chunk)
template <typename T, typename QT>
__device__ __forceinline__ void prefetch_chunk(const StepArgs<T, QT>& a, uint32_t c0, uint32_t len)
{
    using R = typename Pop<T>::R;
    if (threadIdx.x >= 32 || c0 >= a.ns) return;
    const uint32_t cnt = min(len, a.ns - c0);
    const int lane = threadIdx.x;
    if (lane < 19) l2_prefetch(a.fA + (uint32_t)lane * a.ns + c0, cnt * (uint32_t)sizeof(T));
    else if (lane < 26) l2_prefetch(a.gA + (uint32_t)(lane - 19) * a.ns + c0, cnt * (uint32_t)sizeof(T));
    else if (lane == 26) l2_prefetch(a.cellw + c0, cnt * 4u);
    else if (lane == 27) l2_prefetch(a.phi + c0, cnt * (uint32_t)sizeof(R));
    else if (lane == 28 && a.isotherm) l2_prefetch(a.q + c0, cnt * (uint32_t)sizeof(QT));
}

// Persistent kernel: block b takes a contiguous share of the work list, so
// consecutive items are neighbouring chunks of one lattice.  The lattice's
// arguments are staged in shared memory (all threads read them from there) and
// re-staged only when the lattice changes.  With pf > 0 the block prefetches,
// into L2, its item pf positions ahead.
template <typename T, typename QT, bool POROUS>
__global__ void __launch_bounds__(256, 5) k_coupled_batch(const StepArgs<T, QT>* __restrict__ items,
                                                          const WorkItem* __restrict__ work, int nwork, int cpt, int pf)
{
    __shared__ StepArgs<T, QT> sa;
    const uint32_t chunk = blockDim.x * (uint32_t)cpt;
    // items round-robin over the resident blocks: the items in flight form one
    // compact front, so the z-neighbour rows they pull are still in L2
    // (contiguous runs per block spread the blocks over the whole batch: 9.8
    // against 6.9 ms per step on the 64-sample batch)
    const int w1 = nwork;
    int staged = -1;
    for (int wi = (int)blockIdx.x; wi < w1; wi += (int)gridDim.x) {
        const WorkItem it = work[wi];
        if (it.lattice != staged) {   // uniform across the block
            __syncthreads();          // every thread is done with the previous arguments
            const uint32_t* src = reinterpret_cast<const uint32_t*>(items + it.lattice);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
            for (uint32_t i = threadIdx.x; i < sizeof(StepArgs<T, QT>) / 4; i += blockDim.x) dst[i] = src[i];
            __syncthreads();
            staged = it.lattice;
        }
        if (pf > 0 && wi + pf * (int)gridDim.x < w1) {
            const WorkItem nx = work[wi + pf * (int)gridDim.x];
            prefetch_chunk(items[nx.lattice], nx.first, chunk);
        }
        for (int j = 0; j < cpt; ++j) coupled_cell<T, QT, POROUS>(sa, it.first + (uint32_t)j * blockDim.x + threadIdx.x);
    }
}

// The batch's lattice arguments and its cell-range work list in constant
// memory: c_batch_args holds StepArgs[2][nlat] (buffer parity 0 and 1), and
// lattice l owns work items (chunks of blockDim*cpt cells) c_batch_off[l] ..
// c_batch_off[l+1]-1.  Reads use a block-uniform index, served by the
// constant cache like kernel parameters.
constexpr int kBatchConstBytes = 48 * 1024;
constexpr int kBatchMaxLattices = 255;
__constant__ __align__(16) unsigned char c_batch_args[kBatchConstBytes];
__constant__ uint32_t c_batch_off[kBatchMaxLattices + 1];

__device__ __forceinline__ int batch_lattice_of(uint32_t item, int nlat)
{
    int lo = 0, hi = nlat;   // c_batch_off[lo] <= item < c_batch_off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (c_batch_off[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <typename T, typename QT>
__device__ __forceinline__ const StepArgs<T, QT>& batch_args(int parity, int nlat, int l)
{
    return reinterpret_cast<const StepArgs<T, QT>*>(c_batch_args)[parity * nlat + l];
}

// One launch per step over every lattice.  persistent != 0: a grid of resident
// blocks taking the work items round-robin; otherwise one block per work item.
// pf > 0: L2 prefetch of the item pf positions ahead in this block's sequence
// (same lattice).
template <typename T, typename QT, bool POROUS>
__global__ void __launch_bounds__(256, 5) k_coupled_batch_c(int nlat, int parity, int cpt, int pf, int persistent)
{
    const uint32_t chunk = blockDim.x * (uint32_t)cpt;
    const uint32_t nitems = c_batch_off[nlat];
    // persistent: items round-robin over the resident blocks (one compact front
    // of items in flight, as in k_coupled_batch); otherwise one block per item
    const uint32_t stride = persistent ? gridDim.x : nitems;
    const uint32_t w0 = blockIdx.x, w1 = nitems;
    if (w0 >= w1) return;
    int l = batch_lattice_of(w0, nlat);
    for (uint32_t wi = w0; wi < w1; wi += stride) {
        while (wi >= c_batch_off[l + 1]) ++l;
        const StepArgs<T, QT>& a = batch_args<T, QT>(parity, nlat, l);
        const uint32_t first = (wi - c_batch_off[l]) * chunk;
        const uint32_t pstep = persistent ? gridDim.x : 1u;   // the item this block (or its neighbour) takes pf items on
        if (pf > 0 && wi + (uint32_t)pf * pstep < c_batch_off[l + 1])
            prefetch_chunk(a, first + (uint32_t)pf * pstep * chunk, chunk);
        for (int j = 0; j < cpt; ++j) coupled_cell<T, QT, POROUS>(a, first + (uint32_t)j * blockDim.x + threadIdx.x);
    }
}

// Breakthrough samples of many lattices: block i averages phi over probe i's
// cells and appends the mean at the device-side sample counter (graph-safe).
struct ProbeItem {
    const void* phi;     // R per cell
    const int* cells;
    int count;
    double* series;      // samples of this lattice
    int* counter;        // next sample slot
    int capacity;
};

template <typename R>
__global__ void k_probe_batch(const ProbeItem* __restrict__ probes)
{
    const ProbeItem p = probes[blockIdx.x];
    const R* phi = static_cast<const R*>(p.phi);
    double v = 0.0;
    for (int i = threadIdx.x; i < p.count; i += blockDim.x) v += (double)phi[p.cells[i]];
    __shared__ double part[32];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double s = threadIdx.x < (blockDim.x + 31) / 32 ? part[threadIdx.x] : 0.0;
        s = warp_sum(s);
        if (threadIdx.x == 0) {
            const int slot = *p.counter;
            if (slot < p.capacity) p.series[slot] = s / (double)p.count;
            *p.counter = slot + 1;
        }
    }
}

// AD update of cells whose NS populations a post-stream NS boundary of the
// general (list) path rewrote: their advection velocity is that of the
// post-boundary f_B.
template <typename T, typename QT>
__global__ void __launch_bounds__(256) k_ad_deferred(const StepArgs<T, QT> a, const int* __restrict__ cells,
                                                     int count)
{
    using R = typename Pop<T>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t c = (uint32_t)cells[i];
    int x, y, z;
    cell_xyz(c, a.nx, a.ny, a.div_nx, a.div_nxy, x, y, z);
    const Nbr nb(x, y, z, a.nx, a.ny, a.nz, a.px, a.py, a.pz);
    const uint32_t w = __ldg(a.cellw + c);
    R ux = R(0), uy = R(0), uz = R(0);
    if (a.coupling) {
        R f[19];
#pragma unroll
        for (int k = 0; k < 19; ++k) f[k] = Pop<T>::ld(a.fB + (uint32_t)k * a.ns + c, fshift<T>(k, a.f_shift));
        macro_velocity(f, ux, uy, uz);
    }
    R gi[7], gn[7];
    pull7(a, c, nb, gi);
    const R ph = ad_collide(a, c, w, gi, ux, uy, uz, true, gn);
    store7(a, c, gn);
    a.phi[c] = ph;
}

// Per-cell flag word from the bit-packed obstacle / region / deferred masks.
// Link bit k is set when direction k pulls from an in-domain obstacle cell
// (periodic wrap applied), which is the reference's half-way bounce-back test.
__global__ void k_build_flags(uint32_t* __restrict__ cellw, const uint32_t* __restrict__ solid,
                              const uint32_t* __restrict__ region, const uint32_t* __restrict__ defer, int n, int nx,
                              int ny, int nz, int px, int py, int pz, unsigned long long mnx, unsigned long long mnxy,
                              int links)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (uint32_t)n) return;
    int x, y, z;
    cell_xyz(c, nx, ny, mnx, mnxy, x, y, z);
    const Nbr nb(x, y, z, nx, ny, nz, px, py, pz);
    uint32_t w = 0u;
    if (bit_at(solid, (int)c)) w |= kSolid;
    if (links) {
#pragma unroll
        for (int k = 1; k < 19; ++k) {
            const int cx = cx19(k), cy = cy19(k), cz = cz19(k);
            const bool in = nb.xo[1 - cx] && nb.yo[1 - cy] && nb.zo[1 - cz];
            if (in && bit_at(solid, nb.xs[1 - cx] + nb.yr[1 - cy] + nb.zp[1 - cz])) w |= 1u << k;
        }
    }
    if (region && bit_at(region, (int)c)) w |= kRegion;
    if (defer && bit_at(defer, (int)c)) w |= kDeferred;
    if (y == 0 || y == ny - 1 || z == 0 || z == nz - 1) w |= kFaceYZ;
    if (x == 0) w |= kXLo;
    if (x == nx - 1) w |= kXHi;
    cellw[c] = w;
}

// ---------------------------------------------------------------------------
// boundary kernels over compacted cell lists
// ---------------------------------------------------------------------------
template <int K, typename R>
__device__ __forceinline__ R feq19(R rho, R ux, R uy, R uz, R u2)
{
    // src/boundary/ns/VelocityDirichletNEQ.cu:35-46 and VelocityDirichlet.cu:76-80
    const R eu = cdot<cx19(K), cy19(K), cz19(K)>(ux, uy, uz);
    const R cu = R(3) * eu;
    return w19<R>(K) * rho * (R(1) + cu + R(0.5) * cu * cu - R(1.5) * u2);
}

template <typename R, int... Ks>
__device__ __forceinline__ void feq19_all(R* out, R rho, R ux, R uy, R uz, std::integer_sequence<int, Ks...>)
{
    const R u2 = ux * ux + uy * uy + uz * uz;
    ((out[Ks] = feq19<Ks>(rho, ux, uy, uz, u2)), ...);
}

// VelocityDirichletEq, pre-collision on f_A (src/boundary/ns/VelocityDirichlet.cu:54-84)
template <typename T>
__global__ void k_ns_velocity_eq(T* __restrict__ f, long long ns, const int* __restrict__ cells, int count,
                                 typename Pop<T>::R rho0, typename Pop<T>::R ux, typename Pop<T>::R uy,
                                 typename Pop<T>::R uz, typename Pop<T>::R fsh)
{
    using R = typename Pop<T>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i];
    R fe[19];
    feq19_all(fe, rho0, ux, uy, uz, Seq19{});
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(f + (long long)k * ns + c, fe[k], fshift<T>(k, fsh));
}

// VelocityDirichletNEQ, pre-collision on f_A (src/boundary/ns/VelocityDirichletNEQ.cu:49-96)
template <typename T>
__global__ void k_ns_velocity_neq(T* __restrict__ f, long long ns, const int* __restrict__ cells,
                                  const int* __restrict__ nei, int count, typename Pop<T>::R ux, typename Pop<T>::R uy,
                                  typename Pop<T>::R uz, typename Pop<T>::R fsh)
{
    using R = typename Pop<T>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int cb = cells[i], cn = nei[i];
    R fN[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) fN[k] = Pop<T>::ld(f + (long long)k * ns + cn, fshift<T>(k, fsh));
    R r, jx, jy, jz;
    moments19(fN, r, jx, jy, jz, Seq19{});
    const R inv = (r > R(0)) ? (R(1) / r) : R(0);
    R eqN[19], eqB[19];
    feq19_all(eqN, r, jx * inv, jy * inv, jz * inv, Seq19{});
    feq19_all(eqB, r, ux, uy, uz, Seq19{});
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(f + (long long)k * ns + cb, eqB[k] + (fN[k] - eqN[k]), fshift<T>(k, fsh));
}

// PressureDirichlet, post-stream on f_B (src/boundary/ns/PressureDirichlet.cu:26-96):
// feq(rho_out, u of the x-1 neighbour) in the 1 + 3eu + 4.5eu^2 - 1.5u^2 form.
template <typename T>
__global__ void k_ns_pressure(T* __restrict__ f, long long ns, const int* __restrict__ cells, int count,
                              typename Pop<T>::R rho_out, typename Pop<T>::R fsh)
{
    using R = typename Pop<T>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i], cn = c - 1;
    R fN[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) fN[k] = Pop<T>::ld(f + (long long)k * ns + cn, fshift<T>(k, fsh));
    R r, ux, uy, uz;
    moments19(fN, r, ux, uy, uz, Seq19{});
    if (r > R(0)) { const R inv = R(1) / r; ux *= inv; uy *= inv; uz *= inv; }
    else { ux = uy = uz = R(0); }
    R fe[19];
    feq_outlet_all(fe, rho_out, ux, uy, uz, Seq19{});
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(f + (long long)k * ns + c, fe[k], fshift<T>(k, fsh));
}

// BounceBack BC, post-stream on f_B, as the reference kernel behaves
// (src/boundary/ns/BounceBack.cu:12-31): the in-place f[k] = f[opp k] loop
// leaves both members of each pair equal to the higher-index direction.
template <typename T>
__global__ void k_ns_bounceback(T* __restrict__ f, long long ns, const int* __restrict__ cells, int count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i];
#pragma unroll
    for (int k = 1; k < 19; ++k) {
        const int hi = k > opp19(k) ? k : opp19(k);
        if (hi != k) f[(long long)k * ns + c] = f[(long long)hi * ns + c];
    }
}

// ADDirichlet (post-stream, g_B) and ADDirichletTanhPulse (pre-collision, g_A):
// g = value * w on the listed cells (src/boundary/ad/ADDirichlet.cu:11-30,
// src/boundary/ad/ADDirichletTanhPulse.cu:11-31).
template <typename T>
__global__ void k_ad_fill(T* __restrict__ g, long long ns, const int* __restrict__ cells, int count,
                          typename Pop<T>::R value, typename Pop<T>::R gsh)
{
    using R = typename Pop<T>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i];
#pragma unroll
    for (int k = 0; k < 7; ++k) PopG<T>::st(g + (long long)k * ns + c, value * w7<R>(k), k, gsh, (uint32_t)c);
}

// ADNeumannOutlet, post-stream on g_B (src/boundary/ad/ADNeumannOutlet.cu:5-31)
template <typename T>
__global__ void k_ad_neumann(T* __restrict__ g, long long ns, const int* __restrict__ cells, int count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i];
#pragma unroll
    for (int k = 0; k < 7; ++k) g[(long long)k * ns + c] = g[(long long)k * ns + c - 1];
}

// ---------------------------------------------------------------------------
// initial state (k_init_eq_d3q19_1d / k_init_eq_d3q19 / k_ad_init_eq_d3q7)
// ---------------------------------------------------------------------------
template <typename T, typename QT>
__global__ void k_init(T* __restrict__ f, T* __restrict__ g, typename Pop<T>::R* __restrict__ phi,
                       QT* __restrict__ q, long long ns, int n, typename Pop<T>::R rho0, typename Pop<T>::R phi0,
                       typename Pop<T>::R fsh, typename Pop<T>::R gsh)
{
    using R = typename Pop<T>::R;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(f + (long long)k * ns + c, w19<R>(k) * rho0, fshift<T>(k, fsh));
#pragma unroll
    for (int k = 0; k < 7; ++k) PopG<T>::st(g + (long long)k * ns + c, phi0 * w7<R>(k), k, gsh, (uint32_t)c);
    phi[c] = R(0);
    q[c] = (QT)0;
}

// Switch a full x = 0 NEQ inlet plane into the fused representation: save the
// x = 0 populations to x0post and write the NEQ values (from the x = 1 cells)
// in their place -- what k_ns_velocity_neq does at the start of the next step.
// (pair_h, div_nx: the storage layout, as pair_element)
template <typename T>
__global__ void k_inlet_prime(T* __restrict__ f, long long ns, const int* __restrict__ cells,
                              const int* __restrict__ nei, int count, typename Pop<T>::R ux, typename Pop<T>::R uy,
                              typename Pop<T>::R uz, typename Pop<T>::R fsh, T* __restrict__ x0post,
                              uint32_t rows_stride, uint32_t pair_h, unsigned long long div_nx)
{
    using R = typename Pop<T>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int cb = (int)pair_element((uint32_t)cells[i], pair_h, div_nx);
    const int cn = (int)pair_element((uint32_t)nei[i], pair_h, div_nx);
#pragma unroll
    for (int k = 0; k < 19; ++k) x0post[(uint32_t)k * rows_stride + i] = f[(long long)k * ns + cb];
    R fN[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) fN[k] = Pop<T>::ld(f + (long long)k * ns + cn, fshift<T>(k, fsh));
    R r, jx, jy, jz;
    moments19(fN, r, jx, jy, jz, Seq19{});
    const R inv = (r > R(0)) ? (R(1) / r) : R(0);
    R eqN[19], eqB[19];
    feq19_all(eqN, r, jx * inv, jy * inv, jz * inv, Seq19{});
    feq19_all(eqB, r, ux, uy, uz, Seq19{});
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(f + (long long)k * ns + cb, eqB[k] + (fN[k] - eqN[k]), fshift<T>(k, fsh));
}

// Back to the plain representation: the x = 0 populations from x0post.
template <typename T>
__global__ void k_inlet_restore(T* __restrict__ f, long long ns, const int* __restrict__ cells, int count,
                                const T* __restrict__ x0post, uint32_t rows_stride, uint32_t pair_h,
                                unsigned long long div_nx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t e = pair_element((uint32_t)cells[i], pair_h, div_nx);
#pragma unroll
    for (int k = 0; k < 19; ++k) f[(long long)k * ns + e] = x0post[(uint32_t)k * rows_stride + i];
}

// ---------------------------------------------------------------------------
// macroscopic fields and FP64 reductions
// ---------------------------------------------------------------------------
// rho, u of the current f (src/core/Macros.cu:20-61) into planes of type R.
template <typename T>
__global__ void k_macros(const T* __restrict__ f, long long ns, int n, typename Pop<T>::R fsh,
                         typename Pop<T>::R* __restrict__ rho, typename Pop<T>::R* __restrict__ ux,
                         typename Pop<T>::R* __restrict__ uy, typename Pop<T>::R* __restrict__ uz, uint32_t pair_h,
                         unsigned long long div_nx)
{
    using R = typename Pop<T>::R;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const uint32_t e = pair_element((uint32_t)c, pair_h, div_nx);
    R v[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) v[k] = Pop<T>::ld(f + (long long)k * ns + e, fshift<T>(k, fsh));
    R r, jx, jy, jz;
    moments19(v, r, jx, jy, jz, Seq19{});
    const R inv = (r > R(0)) ? (R(1) / r) : R(0);
    rho[c] = r;
    ux[c] = jx * inv;
    uy[c] = jy * inv;
    uz[c] = jz * inv;
}

// Block-reduce NV values per thread and add them to acc[0..NV) in FP64.
template <int NV>
__device__ __forceinline__ void block_accumulate(double (&v)[NV], double* __restrict__ acc)
{
    __shared__ double part[32][NV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) part[wid][j] = v[j];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double s = lane < nw ? part[lane][j] : 0.0;
            s = warp_sum(s);
            if (lane == 0) atomicAdd(acc + j, s);
        }
    }
}

// acc[0] += sum rho, acc[1] += sum phi, acc[2] += sum q over all cells.
template <typename T, typename QT>
__global__ void k_domain_sums(const T* __restrict__ f, const typename Pop<T>::R* __restrict__ phi,
                              const QT* __restrict__ q, long long ns, int n, typename Pop<T>::R fsh,
                              double* __restrict__ acc)
{
    using R = typename Pop<T>::R;
    double v[3] = {0.0, 0.0, 0.0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        R r = R(0);
#pragma unroll
        for (int k = 0; k < 19; ++k) r += Pop<T>::ld(f + (long long)k * ns + c, fshift<T>(k, fsh));
        v[0] += (double)r;
        v[1] += (double)phi[c];
        v[2] += (double)q[c];
    }
    block_accumulate<3>(v, acc);
}

// acc[slot] += mean of phi over the listed probe cells (OutletCSV::log).
template <typename R>
__global__ void k_probe_mean(const R* __restrict__ phi, const int* __restrict__ cells, int count,
                             double* __restrict__ acc)
{
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        v[0] += (double)phi[cells[i]];
    v[0] /= (double)count;
    block_accumulate<1>(v, acc);
}

// mean, min and max of phi over the probe cells (one block; deterministic)
template <typename R>
__global__ void __launch_bounds__(1024) k_probe_stats(const R* __restrict__ phi, const int* __restrict__ cells, int count,
                                                      double* __restrict__ out)
{
    __shared__ double ssum[32], smin[32], smax[32];
    double s = 0.0, lo = INFINITY, hi = -INFINITY;
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const double v = (double)phi[cells[i]];
        s += v;
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) { ssum[threadIdx.x >> 5] = s; smin[threadIdx.x >> 5] = lo; smax[threadIdx.x >> 5] = hi; }
    __syncthreads();
    if (threadIdx.x < 32) {
        const bool has = threadIdx.x < (blockDim.x + 31) / 32;
        s = has ? ssum[threadIdx.x] : 0.0;
        lo = has ? smin[threadIdx.x] : INFINITY;
        hi = has ? smax[threadIdx.x] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (threadIdx.x == 0) {
            out[0] = count > 0 ? s / (double)count : 0.0;
            out[1] = count > 0 ? lo : 0.0;
            out[2] = count > 0 ? hi : 0.0;
        }
    }
}

}  // namespace fm
