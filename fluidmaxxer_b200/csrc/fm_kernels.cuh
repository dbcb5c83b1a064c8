// fm_kernels.cuh -- sm_100a kernels of the coupled D3Q19 NS + D3Q7 AD + LDF step.
//
// Memory layout (HBM):
//   f[2][19][ns], g[2][7][ns]  population buffers, structure of arrays; plane
//                              stride ns = N rounded up to 32 cells so every
//                              plane starts 128-byte aligned.  Buffer A holds
//                              the post-step populations of step s-1, buffer B
//                              receives step s; the roles swap every step.
//   phi[ns] (float)            AD scalar of the previous step (the LDF source
//                              at step s reads phi(s-1), src/main.cpp:328-335)
//   q[ns] (float or double)    adsorbed loading
//   solid/region/defer bits    one bit per cell, word c>>5, bit c&31
//
// One fused kernel per step (k_coupled_step) does, per cell: the NS pull +
// collision (BGK with obstacle bounce-back or porous BGK), the NS velocity of
// the post-collision populations (the coupling of Lattice::computeMacroscopicDevice),
// the LDF source from phi(s-1) and q, and the D3Q7 pull + collision with that
// source.  Boundary conditions that the reference applies to whole-grid masks
// run as small kernels over compacted cell lists:
//   pre-collision  : NS velocity inlets (on f_A), AD tanh pulse (on g_A)
//   post-stream NS : pressure outlet, bounce-back BC (on f_B); the AD update of
//                    those cells needs their post-BC velocity, so the fused
//                    kernel skips them ("defer" bit) and k_ad_deferred does it
//   post-stream AD : Dirichlet inlet, Neumann outlet (on g_B)
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

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
__host__ __device__ __forceinline__ constexpr float w19(int k)
{
    return k == 0 ? 1.0f / 3.0f : (k < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
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
__host__ __device__ __forceinline__ constexpr float w7(int k) { return k == 0 ? 0.25f : 0.125f; }

// c.u with only the nonzero velocity components (c_i in {-1,0,1}); equal in
// IEEE arithmetic to the reference's cx*ux + cy*uy + cz*uz.
template <int CX, int CY, int CZ>
__device__ __forceinline__ float cdot(float ux, float uy, float uz)
{
    float e = 0.0f;
    bool first = true;
    if (CX != 0) { e = CX > 0 ? ux : -ux; first = false; }
    if (CY != 0) { e = first ? (CY > 0 ? uy : -uy) : (CY > 0 ? e + uy : e - uy); first = false; }
    if (CZ != 0) { e = first ? (CZ > 0 ? uz : -uz) : (CZ > 0 ? e + uz : e - uz); }
    return e;
}

// ---------------------------------------------------------------------------
// population storage: FP32 as is; FP16 / BF16 hold the value minus a shift
// (w_i rho0 for f, w_i c_shift for g) and all arithmetic is FP32.
// ---------------------------------------------------------------------------
template <typename T> struct Pop;
template <> struct Pop<float> {
    static constexpr bool kShifted = false;
    __device__ static __forceinline__ float ld(const float* p, float) { return __ldg(p); }
    __device__ static __forceinline__ void st(float* p, float v, float) { *p = v; }
};
template <> struct Pop<__half> {
    static constexpr bool kShifted = true;
    __device__ static __forceinline__ float ld(const __half* p, float sh) { return __half2float(__ldg(p)) + sh; }
    __device__ static __forceinline__ void st(__half* p, float v, float sh) { *p = __float2half_rn(v - sh); }
};
template <> struct Pop<__nv_bfloat16> {
    static constexpr bool kShifted = true;
    __device__ static __forceinline__ float ld(const __nv_bfloat16* p, float sh)
    {
        return __bfloat162float(__ldg(p)) + sh;
    }
    __device__ static __forceinline__ void st(__nv_bfloat16* p, float v, float sh)
    {
        *p = __float2bfloat16_rn(v - sh);
    }
};

// q loading: FP32 in the plain form, FP64 accumulator in the reduced-precision forms
template <typename QT> __device__ __forceinline__ QT qload(const QT* p) { return *p; }

__device__ __forceinline__ uint32_t bit_at(const uint32_t* __restrict__ m, int c)
{
    return (__ldg(m + (c >> 5)) >> (c & 31)) & 1u;
}

// ---------------------------------------------------------------------------
// kernel arguments
// ---------------------------------------------------------------------------
template <typename T, typename QT>
struct StepArgs {
    const T* __restrict__ fA;
    T* __restrict__ fB;
    const T* __restrict__ gA;
    T* __restrict__ gB;
    float* __restrict__ phi;
    QT* __restrict__ q;
    const uint32_t* __restrict__ solid;
    const uint32_t* __restrict__ region;
    const uint32_t* __restrict__ defer;   // may be null
    const float* __restrict__ porosity;   // porous collision
    const float* __restrict__ tau_ad;     // null: omega_ad for all cells
    long long ns;                         // plane stride (elements)
    int n, nx, ny, nz;
    int px, py, pz;
    float omega;                          // NS 1/max(tau, 0.5001)
    float rho0;                           // NS density fallback (rho <= 0)
    float omega_ad;
    float min_conc;
    float f_shift, g_shift;               // shifted storage: rho0 and c_shift
    int coupling;
    int isotherm;                         // 0 none, 1 linear, 2 Langmuir
    float iso_a, iso_b, iso_k;            // linear: K, -, k ; Langmuir: q_max, b, k
};

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

__device__ __forceinline__ void cell_xyz(int c, int nx, int ny, int& x, int& y, int& z)
{
    const int nxy = nx * ny;
    z = c / nxy;
    const int r = c - z * nxy;
    y = r / nx;
    x = r - y * nx;
}

// ---------------------------------------------------------------------------
// NS pull + collision of one fluid cell.  BGK: keep-local outside
// non-periodic faces, own opposite population when the source is solid
// (src/collision/BGKCollision.cu:105-130); porous: no reflection
// (src/collision/PorousBGKCollision.cu:88-101).
// ---------------------------------------------------------------------------
template <typename T, int K, bool BB>
__device__ __forceinline__ float pull19(const T* __restrict__ fA, long long ns, int c, const Nbr& nb,
                                        const uint32_t* __restrict__ solid, float shift)
{
    constexpr int CX = cx19(K), CY = cy19(K), CZ = cz19(K);
    long long off;
    if (K == 0) {
        off = c;
    } else if (!nb.inside<CX, CY, CZ>()) {
        off = (long long)K * ns + c;
    } else {
        const int s = nb.src<CX, CY, CZ>();
        off = (BB && bit_at(solid, s)) ? (long long)opp19(K) * ns + c : (long long)K * ns + s;
    }
    return Pop<T>::ld(fA + off, shift);
}

template <typename T, bool BB, int... Ks>
__device__ __forceinline__ void pull19_all(float* fi, const T* __restrict__ fA, long long ns, int c,
                                           const Nbr& nb, const uint32_t* __restrict__ solid, float fsh,
                                           std::integer_sequence<int, Ks...>)
{
    ((fi[Ks] = pull19<T, Ks, BB>(fA, ns, c, nb, solid, Pop<T>::kShifted ? w19(Ks) * fsh : 0.0f)), ...);
}

// f_new = f + omega (feq - f) with feq = w rho (1 + 3eu + 4.5eu^2 - 1.5u^2)
// written as in src/collision/BGKCollision.cu:163-176.
template <int K>
__device__ __forceinline__ float bgk19(float fi, float rho, float ux, float uy, float uz, float u2, float omega)
{
    const float eu = cdot<cx19(K), cy19(K), cz19(K)>(ux, uy, uz);
    const float cu = 3.0f * eu;
    const float feq = w19(K) * rho * (1.0f + cu + 0.5f * cu * cu - 1.5f * u2);
    return fi + omega * (feq - fi);
}

template <int... Ks>
__device__ __forceinline__ void collide19(float* fi, float rho, float ux, float uy, float uz, float omega,
                                          std::integer_sequence<int, Ks...>)
{
    const float u2 = ux * ux + uy * uy + uz * uz;
    ((fi[Ks] = bgk19<Ks>(fi[Ks], rho, ux, uy, uz, u2, omega)), ...);
}

template <int... Ks>
__device__ __forceinline__ void moments19(const float* f, float& rho, float& jx, float& jy, float& jz,
                                          std::integer_sequence<int, Ks...>)
{
    rho = 0.0f; jx = 0.0f; jy = 0.0f; jz = 0.0f;
    ((rho += f[Ks]), ...);
    ((jx = cx19(Ks) == 0 ? jx : (cx19(Ks) > 0 ? jx + f[Ks] : jx - f[Ks])), ...);
    ((jy = cy19(Ks) == 0 ? jy : (cy19(Ks) > 0 ? jy + f[Ks] : jy - f[Ks])), ...);
    ((jz = cz19(Ks) == 0 ? jz : (cz19(Ks) > 0 ? jz + f[Ks] : jz - f[Ks])), ...);
}

using Seq19 = std::make_integer_sequence<int, 19>;
using Seq7 = std::make_integer_sequence<int, 7>;

// velocity of a population set as Lattice::computeMacroscopicDevice forms it
// (src/core/Macros.cu:40-60): u = j / rho, zero if rho <= 0.
__device__ __forceinline__ void macro_velocity(const float* f, float& ux, float& uy, float& uz)
{
    float r, jx, jy, jz;
    moments19(f, r, jx, jy, jz, Seq19{});
    const float inv = (r > 0.0f) ? (1.0f / r) : 0.0f;
    ux = jx * inv; uy = jy * inv; uz = jz * inv;
}

// One NS update into fn[19] (post-collision, pre post-stream BC).
template <typename T, typename QT, bool POROUS>
__device__ __forceinline__ void ns_update(const StepArgs<T, QT>& a, int c, const Nbr& nb, float* fn)
{
    const float fsh = a.f_shift;
    if (!POROUS && bit_at(a.solid, c)) {
        // on-site reversal in an obstacle cell (src/collision/BGKCollision.cu:90-97)
#pragma unroll
        for (int k = 0; k < 19; ++k)
            fn[k] = Pop<T>::ld(a.fA + (long long)opp19(k) * a.ns + c, Pop<T>::kShifted ? w19(opp19(k)) * fsh : 0.0f);
        return;
    }
    pull19_all<T, !POROUS>(fn, a.fA, a.ns, c, nb, a.solid, fsh, Seq19{});
    float rho, jx, jy, jz;
    moments19(fn, rho, jx, jy, jz, Seq19{});
    float ux, uy, uz;
    if (!POROUS) {
        // src/collision/BGKCollision.cu:148-158
        if (!(rho > 0.0f)) { rho = a.rho0; ux = uy = uz = 0.0f; }
        else { const float inv = 1.0f / rho; ux = jx * inv; uy = jy * inv; uz = jz * inv; }
    } else {
        // src/collision/PorousBGKCollision.cu:118-136
        if (!(rho > 0.0f)) { rho = a.rho0; jx = jy = jz = 0.0f; }
        const float inv = 1.0f / rho;
        ux = jx * inv; uy = jy * inv; uz = jz * inv;
        float ph = __ldg(a.porosity + c);
        if (ph < 0.0f) ph = 0.0f;
        if (ph > 1.0f) ph = 1.0f;
        ux *= ph; uy *= ph; uz *= ph;
    }
    collide19(fn, rho, ux, uy, uz, a.omega, Seq19{});
}

template <typename T, typename QT>
__device__ __forceinline__ void store19(const StepArgs<T, QT>& a, int c, const float* fn)
{
#pragma unroll
    for (int k = 0; k < 19; ++k)
        Pop<T>::st(a.fB + (long long)k * a.ns + c, fn[k], Pop<T>::kShifted ? w19(k) * a.f_shift : 0.0f);
}

// ---------------------------------------------------------------------------
// LDF source (src/reaction/LinearLDF.cu:13-48, src/reaction/LangmuirLDF.cu:7-41)
// then the D3Q7 pull + collision with that source
// (src/collision/ADBGKCollision.cu:41-128).
// ---------------------------------------------------------------------------
template <typename T, typename QT>
__device__ __forceinline__ void ad_update(const StepArgs<T, QT>& a, int c, const Nbr& nb, float ux, float uy,
                                          float uz, float* c_out)
{
    float S = 0.0f;
    if (a.isotherm != 0 && bit_at(a.region, c)) {
        float cc = a.phi[c];
        if (cc < a.min_conc) cc = a.min_conc;
        const float ce = cc - a.min_conc;
        QT qeq;
        if (a.isotherm == 1) {
            qeq = (QT)(a.iso_a * ce);
        } else {
            const float bc = a.iso_b * ce;
            qeq = (QT)(a.iso_a * (bc / (1.0f + bc)));
        }
        const QT qi = a.q[c];
        const QT dq = (QT)a.iso_k * (qeq - qi);
        a.q[c] = qi + dq;
        S = (float)(-dq);
    }
    const float gsh = a.g_shift;
    float gi[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        const float sh = Pop<T>::kShifted ? w7(k) * gsh : 0.0f;
        const int cx = cx7(k), cy = cy7(k), cz = cz7(k);
        const bool in = nb.xo[1 - cx] && nb.yo[1 - cy] && nb.zo[1 - cz];
        const int s = nb.xs[1 - cx] + nb.yr[1 - cy] + nb.zp[1 - cz];
        gi[k] = Pop<T>::ld(a.gA + (long long)k * a.ns + (in ? s : c), sh);
    }
    float ph = gi[0];
#pragma unroll
    for (int k = 1; k < 7; ++k) ph += gi[k];
    if (ph < a.min_conc) ph = a.min_conc;
    const float om = a.tau_ad ? 1.0f / __ldg(a.tau_ad + c) : a.omega_ad;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        float eu;
        if (k == 0) eu = 0.0f;
        else if (k == 1) eu = ux;
        else if (k == 2) eu = -ux;
        else if (k == 3) eu = uy;
        else if (k == 4) eu = -uy;
        else if (k == 5) eu = uz;
        else eu = -uz;
        const float geq = w7(k) * ph * (1.0f + 4.0f * eu);
        const float gn = gi[k] + om * (geq - gi[k]) + w7(k) * S;
        Pop<T>::st(a.gB + (long long)k * a.ns + c, gn, Pop<T>::kShifted ? w7(k) * gsh : 0.0f);
    }
    a.phi[c] = ph;
    if (c_out) *c_out = ph;
}

// ---------------------------------------------------------------------------
// the fused step: one thread per cell
// ---------------------------------------------------------------------------
template <typename T, typename QT, bool POROUS>
__global__ void __launch_bounds__(256) k_coupled_step(const StepArgs<T, QT> a)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    int x, y, z;
    cell_xyz(c, a.nx, a.ny, x, y, z);
    const Nbr nb(x, y, z, a.nx, a.ny, a.nz, a.px, a.py, a.pz);
    float fn[19];
    ns_update<T, QT, POROUS>(a, c, nb, fn);
    store19(a, c, fn);
    if (a.defer && bit_at(a.defer, c)) return;
    float ux = 0.0f, uy = 0.0f, uz = 0.0f;
    if (a.coupling) macro_velocity(fn, ux, uy, uz);
    ad_update(a, c, nb, ux, uy, uz, nullptr);
}

// AD update of cells whose NS populations a post-stream NS boundary rewrote:
// their advection velocity is that of the post-BC f_B.
template <typename T, typename QT>
__global__ void __launch_bounds__(256) k_ad_deferred(const StepArgs<T, QT> a, const int* __restrict__ cells,
                                                     int count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i];
    int x, y, z;
    cell_xyz(c, a.nx, a.ny, x, y, z);
    const Nbr nb(x, y, z, a.nx, a.ny, a.nz, a.px, a.py, a.pz);
    float ux = 0.0f, uy = 0.0f, uz = 0.0f;
    if (a.coupling) {
        float f[19];
#pragma unroll
        for (int k = 0; k < 19; ++k)
            f[k] = Pop<T>::ld(a.fB + (long long)k * a.ns + c, Pop<T>::kShifted ? w19(k) * a.f_shift : 0.0f);
        macro_velocity(f, ux, uy, uz);
    }
    ad_update(a, c, nb, ux, uy, uz, nullptr);
}

// ---------------------------------------------------------------------------
// boundary kernels over compacted cell lists
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ float feq19(float rho, float ux, float uy, float uz, float u2)
{
    // src/boundary/ns/VelocityDirichletNEQ.cu:35-46 and VelocityDirichlet.cu:76-80
    const float eu = cdot<cx19(K), cy19(K), cz19(K)>(ux, uy, uz);
    const float cu = 3.0f * eu;
    return w19(K) * rho * (1.0f + cu + 0.5f * cu * cu - 1.5f * u2);
}

template <int... Ks>
__device__ __forceinline__ void feq19_all(float* out, float rho, float ux, float uy, float uz,
                                          std::integer_sequence<int, Ks...>)
{
    const float u2 = ux * ux + uy * uy + uz * uz;
    ((out[Ks] = feq19<Ks>(rho, ux, uy, uz, u2)), ...);
}

// VelocityDirichletEq, pre-collision on f_A (src/boundary/ns/VelocityDirichlet.cu:54-84)
template <typename T>
__global__ void k_ns_velocity_eq(T* __restrict__ f, long long ns, const int* __restrict__ cells, int count,
                                 float rho0, float ux, float uy, float uz, float fsh)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i];
    float fe[19];
    feq19_all(fe, rho0, ux, uy, uz, Seq19{});
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(f + (long long)k * ns + c, fe[k], Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
}

// VelocityDirichletNEQ, pre-collision on f_A (src/boundary/ns/VelocityDirichletNEQ.cu:49-96)
template <typename T>
__global__ void k_ns_velocity_neq(T* __restrict__ f, long long ns, const int* __restrict__ cells,
                                  const int* __restrict__ nei, int count, float ux, float uy, float uz, float fsh)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int cb = cells[i], cn = nei[i];
    float fN[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) fN[k] = Pop<T>::ld(f + (long long)k * ns + cn, Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
    float r, jx, jy, jz;
    moments19(fN, r, jx, jy, jz, Seq19{});
    const float inv = (r > 0.0f) ? (1.0f / r) : 0.0f;
    float eqN[19], eqB[19];
    feq19_all(eqN, r, jx * inv, jy * inv, jz * inv, Seq19{});
    feq19_all(eqB, r, ux, uy, uz, Seq19{});
#pragma unroll
    for (int k = 0; k < 19; ++k)
        Pop<T>::st(f + (long long)k * ns + cb, eqB[k] + (fN[k] - eqN[k]), Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
}

// PressureDirichlet, post-stream on f_B (src/boundary/ns/PressureDirichlet.cu:26-96):
// feq(rho_out, u of the x-1 neighbour) in the 1 + 3eu + 4.5eu^2 - 1.5u^2 form.
template <typename T>
__global__ void k_ns_pressure(T* __restrict__ f, long long ns, const int* __restrict__ cells, int count,
                              float rho_out, float fsh)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i], cn = c - 1;
    float fN[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) fN[k] = Pop<T>::ld(f + (long long)k * ns + cn, Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
    float r, ux, uy, uz;
    moments19(fN, r, ux, uy, uz, Seq19{});
    if (r > 0.0f) { const float inv = 1.0f / r; ux *= inv; uy *= inv; uz *= inv; }
    else { ux = uy = uz = 0.0f; }
    const float u2 = ux * ux + uy * uy + uz * uz;
#pragma unroll
    for (int k = 0; k < 19; ++k) {
        float eu;
        switch (k) {
            case 0: eu = 0.0f; break;
            case 1: eu = ux; break;   case 2: eu = -ux; break;
            case 3: eu = uy; break;   case 4: eu = -uy; break;
            case 5: eu = uz; break;   case 6: eu = -uz; break;
            case 7: eu = ux + uy; break;  case 8: eu = -ux + uy; break;
            case 9: eu = ux - uy; break;  case 10: eu = -ux - uy; break;
            case 11: eu = ux + uz; break; case 12: eu = -ux + uz; break;
            case 13: eu = ux - uz; break; case 14: eu = -ux - uz; break;
            case 15: eu = uy + uz; break; case 16: eu = -uy + uz; break;
            case 17: eu = uy - uz; break; default: eu = -uy - uz; break;
        }
        const float fe = w19(k) * rho_out * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * u2);
        Pop<T>::st(f + (long long)k * ns + c, fe, Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
    }
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
__global__ void k_ad_fill(T* __restrict__ g, long long ns, const int* __restrict__ cells, int count, float value,
                          float gsh)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int c = cells[i];
#pragma unroll
    for (int k = 0; k < 7; ++k) Pop<T>::st(g + (long long)k * ns + c, value * w7(k), Pop<T>::kShifted ? w7(k) * gsh : 0.0f);
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
__global__ void k_init(T* __restrict__ f, T* __restrict__ g, float* __restrict__ phi, QT* __restrict__ q,
                       long long ns, int n, float rho0, float phi0, float fsh, float gsh)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
#pragma unroll
    for (int k = 0; k < 19; ++k) Pop<T>::st(f + (long long)k * ns + c, w19(k) * rho0, Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
#pragma unroll
    for (int k = 0; k < 7; ++k) Pop<T>::st(g + (long long)k * ns + c, phi0 * w7(k), Pop<T>::kShifted ? w7(k) * gsh : 0.0f);
    phi[c] = 0.0f;
    q[c] = (QT)0;
}

// ---------------------------------------------------------------------------
// macroscopic fields and FP64 reductions
// ---------------------------------------------------------------------------
// rho, u of the current f (src/core/Macros.cu:20-61) into float planes.
template <typename T>
__global__ void k_macros(const T* __restrict__ f, long long ns, int n, float fsh, float* __restrict__ rho,
                         float* __restrict__ ux, float* __restrict__ uy, float* __restrict__ uz)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float v[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) v[k] = Pop<T>::ld(f + (long long)k * ns + c, Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
    float r, jx, jy, jz;
    moments19(v, r, jx, jy, jz, Seq19{});
    const float inv = (r > 0.0f) ? (1.0f / r) : 0.0f;
    rho[c] = r;
    ux[c] = jx * inv;
    uy[c] = jy * inv;
    uz[c] = jz * inv;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
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
__global__ void k_domain_sums(const T* __restrict__ f, const float* __restrict__ phi, const QT* __restrict__ q,
                              long long ns, int n, float fsh, double* __restrict__ acc)
{
    double v[3] = {0.0, 0.0, 0.0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        float r = 0.0f;
#pragma unroll
        for (int k = 0; k < 19; ++k) r += Pop<T>::ld(f + (long long)k * ns + c, Pop<T>::kShifted ? w19(k) * fsh : 0.0f);
        v[0] += (double)r;
        v[1] += (double)phi[c];
        v[2] += (double)q[c];
    }
    block_accumulate<3>(v, acc);
}

// acc[slot] += mean of phi over the listed probe cells (OutletCSV::log).
__global__ void k_probe_mean(const float* __restrict__ phi, const int* __restrict__ cells, int count,
                             double* __restrict__ acc)
{
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        v[0] += (double)phi[cells[i]];
    v[0] /= (double)count;
    block_accumulate<1>(v, acc);
}

}  // namespace fm
