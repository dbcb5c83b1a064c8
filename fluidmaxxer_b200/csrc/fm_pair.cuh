// fm_pair.cuh -- the coupled step of the 16-bit storage forms over the pair
// layout: two cells per thread, one 32-bit word per population and pair.
//
// Pair layout.  The population planes of a lattice with nx divisible by 4
// hold each x-row of nx cells as h = nx/2 32-bit words; word w of a row keeps
// the cells x = w (low half) and x = w + h (high half):
//
//     storage element of (x, y, z) = nx (y + ny z) + (x < h ? 2x : 2(x - h) + 1)
//
// A thread takes one word W = h (y + ny z) + w, i.e. the cell pair
// (w, w + h) of one row.  The pull source of both cells of a pair in
// direction k is then one aligned word, the pair (w - c_x, w + h - c_x) of the
// source row, for every 0 < w < h - 1; only the words at the two fold points
// (w = 0 and w = h - 1) assemble their halves from two words.  So every
// population load and store of the step is one coalesced 32-bit access per
// two cells (128 bytes per warp), where the one-cell kernel issues a 2-byte
// access per cell (64 bytes per warp, the x-shifted ones misaligned).  Both
// cells are updated together with Blackwell's packed FP32 pair arithmetic
// (FFMA2 / FADD2), one instruction for the two cells.
//
// The arithmetic is exactly that of the one-cell deviation-form update
// (coupled_cell_dev in fm_kernels.cuh): the same operations in the same order
// on each half, so the two kernels give bit-identical populations.  The cell
// arrays (flag words, phi, q, porosity, tau) keep the natural cell order.
//
// Which lattices use it: a 16-bit form, nx % 4 == 0 and nx >= 8 (so h is even
// and x = 0, 1 and x = nx-2, nx-1 sit in neighbouring lanes of one warp, as
// the fused boundary planes need), every boundary fused into the step (no
// list-path boundary kernels), and not inside a batch.  The host converts the
// stored populations between the layouts when that choice changes.
#pragma once

#include "fm_kernels.cuh"

namespace fm {

// ---------------------------------------------------------------------------
// packed FP32 pair arithmetic
// ---------------------------------------------------------------------------
// The pair update must round exactly as the one-cell update, which is built
// without multiply-add contraction.  The code generator may still fuse a
// packed multiply into a packed add that consumes it (measured on sm_100a for
// the __fmul2_rn intrinsic, an explicit mul.rn.f32x2 and fma(a, b, -0) alike),
// which rounds once where the scalar code rounds twice.  So no product of the
// deviation-form update feeds a sum: the sums of products are explicit FMAs in
// both kernels (u^2, the porous factor, the fixed-point decode is a single
// product), the velocities are j * (1/rho) + (-0) with a runtime -0, and the
// remaining products are exact (powers of two) or feed FMAs.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// ---------------------------------------------------------------------------
// packed pairs of stored 16-bit values
// ---------------------------------------------------------------------------
template <typename T> struct Pair;
// unpack() is an opaque (volatile) conversion so that the compiler converts a
// word again where it is used instead of keeping both the packed word and its
// two floats live across the update (which spills at the 64-register budget)
template <> struct Pair<__half> {
    __device__ static __forceinline__ float2 unpack(uint32_t v)
    {
        float lo, hi;
        asm volatile("{.reg .b16 l, h;\n mov.b32 {l, h}, %2;\n cvt.f32.f16 %0, l;\n cvt.f32.f16 %1, h;}"
                     : "=f"(lo), "=f"(hi) : "r"(v));
        return make_float2(lo, hi);
    }
    __device__ static __forceinline__ uint32_t pack(float2 v)
    {
        const __half2 h = __float22half2_rn(v);
        return *reinterpret_cast<const uint32_t*>(&h);
    }
};
template <> struct Pair<__nv_bfloat16> {
    __device__ static __forceinline__ float2 unpack(uint32_t v)
    {
        uint32_t lo, hi;   // a BF16 value is the high half of its FP32 bits
        asm volatile("{\n shl.b32 %0, %2, 16;\n and.b32 %1, %2, 0xffff0000;\n}" : "=r"(lo), "=r"(hi) : "r"(v));
        return make_float2(__uint_as_float(lo), __uint_as_float(hi));
    }
    __device__ static __forceinline__ uint32_t pack(float2 v)
    {
        const __nv_bfloat162 h = __float22bfloat162_rn(v);
        return *reinterpret_cast<const uint32_t*>(&h);
    }
};
// the D3Q19 planes of the fixed-point form hold FP16 bits
template <> struct Pair<hq> : Pair<__half> {};

// D3Q7 pairs: the stored value plus its shift (as PopG<T>::ld), and back
template <typename T> struct PairG {
    __device__ static __forceinline__ float2 ld(uint32_t v, int k, float gsh)
    {
        const float s = w7<float>(k) * gsh;
        return add2(Pair<T>::unpack(v), f2(s));
    }
    __device__ static __forceinline__ uint32_t st(float2 v, int k, float gsh, uint32_t, uint32_t)
    {
        const float s = -(w7<float>(k) * gsh);
        return Pair<T>::pack(add2(v, f2(s)));
    }
};
template <> struct PairG<hq> {
    __device__ static __forceinline__ float2 ld(uint32_t v, int k, float)
    {
        // PopG<hq>::ld on each half: (code - kGZero) * (w_k kGStep), one product
        const float2 u = make_float2((float)((int)(v & 0xffffu) - kGZero), (float)((int)(v >> 16) - kGZero));
        return mul2(u, f2(w7<float>(k) * kGStep));
    }
    __device__ static __forceinline__ uint32_t st(float2 v, int k, float, uint32_t clo, uint32_t chi)
    {
        hq lo, hi;
        PopG<hq>::st(&lo, v.x, k, 0.0f, clo);
        PopG<hq>::st(&hi, v.y, k, 0.0f, chi);
        return (uint32_t)lo.bits | ((uint32_t)hi.bits << 16);
    }
};


// byte_perm selector keeping the halves of x, except those flagged, which come from y
__device__ __forceinline__ uint32_t half_sel(uint32_t lo_from_y, uint32_t hi_from_y)
{
    return 0x3210u + lo_from_y * 0x44u + hi_from_y * 0x4400u;
}

// ---------------------------------------------------------------------------
// pulls of one pair
// ---------------------------------------------------------------------------
// The source word of direction K for a pair off the fold points is
// pk + row + w - c_x, `row` the word index of the source row.  At w = 0 the +x
// pull takes its high half from the low half of the source row's last word
// (x = h - 1) and its low half from that word's high half (periodic x:
// x = nx - 1) or from the cell itself (keep-local); at w = h - 1 the -x pull
// mirrors it with the row's first word.
template <int CX>
__device__ __forceinline__ uint32_t pull_x(const uint32_t* __restrict__ pk, uint32_t row, int w, int h, uint32_t W,
                                           int px, bool fold)
{
    if (CX == 0 || !fold) return __ldg(pk + (row + (uint32_t)(w - CX)));
    if (CX > 0) {   // w == 0
        const uint32_t t = __ldg(pk + row + (uint32_t)(h - 1));
        const uint32_t own = px ? t : __ldg(pk + W);
        // low half <- (px ? high half of t : low half of own), high half <- low half of t
        return __byte_perm(own, t, px ? 0x5476u : 0x5410u);
    } else {        // w == h - 1
        const uint32_t t = __ldg(pk + row);
        const uint32_t own = px ? t : __ldg(pk + W);
        // low half <- high half of t, high half <- (px ? low half of t : high half of own)
        return __byte_perm(t, own, px ? 0x5432u : 0x7632u);
    }
}

// with bounce-back: halves whose link bit K is set read the pair's own
// opposite population instead (an obstacle cell has every link set)
template <int K, bool BB>
__device__ __forceinline__ uint32_t link_select(uint32_t v, const uint32_t* __restrict__ fA, uint32_t ns2, uint32_t W,
                                                uint32_t lk_lo, uint32_t lk_hi)
{
    if (!BB || K == 0) return v;
    const uint32_t bl = (lk_lo >> K) & 1u, bh = (lk_hi >> K) & 1u;
    if (bl | bh) v = __byte_perm(v, __ldg(fA + (uint32_t)opp19(K) * ns2 + W), half_sel(bl, bh));
    return v;
}

// source row (word index of its first word) of a pair with y/z neighbours
// looked up per axis; `inside` false: the source lies outside a non-periodic
// y or z face and both cells keep their own value
struct RowNbr {
    uint32_t rb[3][3];
    bool in[3][3];
    __device__ __forceinline__ RowNbr(int y, int z, int ny, int nz, int h, int py, int pz)
    {
        int ys[3] = {y - 1, y, y + 1}, zs[3] = {z - 1, z, z + 1};
        bool yo[3] = {true, true, true}, zo[3] = {true, true, true};
        if (y == 0) { if (py) ys[0] = ny - 1; else yo[0] = false; }
        if (y == ny - 1) { if (py) ys[2] = 0; else yo[2] = false; }
        if (z == 0) { if (pz) zs[0] = nz - 1; else zo[0] = false; }
        if (z == nz - 1) { if (pz) zs[2] = 0; else zo[2] = false; }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                in[i][j] = yo[i] && zo[j];
                rb[i][j] = (uint32_t)(ys[i] + ny * zs[j]) * (uint32_t)h;
            }
    }
};

template <typename T, int K, bool BB>
__device__ __forceinline__ uint32_t pull19_pair_nbr(const uint32_t* __restrict__ fA, uint32_t ns2, uint32_t W, int w,
                                                    int h, const RowNbr& nr, int px, uint32_t lk_lo, uint32_t lk_hi)
{
    constexpr int CX = cx19(K), CY = cy19(K), CZ = cz19(K);
    const uint32_t* pk = fA + (uint32_t)K * ns2;
    const uint32_t bl = (lk_lo >> K) & 1u, bh = (lk_hi >> K) & 1u;
    uint32_t v = 0u;
    if (K == 0 || !nr.in[1 - CY][1 - CZ]) {
        v = __ldg(pk + W);   // own value (keep-local across a y/z face)
    } else if (!(BB && (bl & bh))) {
        const bool fold = (CX > 0 && w == 0) || (CX < 0 && w == h - 1);
        v = pull_x<CX>(pk, nr.rb[1 - CY][1 - CZ], w, h, W, px, fold);
    }
    return link_select<K, BB>(v, fA, ns2, W, lk_lo, lk_hi);
}

template <typename T, bool BB, int... Ks>
__device__ __forceinline__ void pull19_pair_nbr_all(uint32_t* v, const uint32_t* __restrict__ fA, uint32_t ns2,
                                                    uint32_t W, int w, int h, const RowNbr& nr, int px,
                                                    uint32_t lk_lo, uint32_t lk_hi, std::integer_sequence<int, Ks...>)
{
    ((v[Ks] = pull19_pair_nbr<T, Ks, BB>(fA, ns2, W, w, h, nr, px, lk_lo, lk_hi)), ...);
}

// off the y/z faces: the source row is the pair's own row shifted by
// -(c_y + c_z ny) rows, a lattice constant
template <typename T, int K, bool BB, bool XF>
__device__ __forceinline__ uint32_t pull19_pair_fast(const uint32_t* __restrict__ fA, uint32_t ns2, uint32_t W,
                                                     uint32_t row0, int w, int h, int hny, int px, uint32_t lk_lo,
                                                     uint32_t lk_hi)
{
    constexpr int CX = cx19(K), CY = cy19(K), CZ = cz19(K);
    const uint32_t* pk = fA + (uint32_t)K * ns2;
    const uint32_t bl = (lk_lo >> K) & 1u, bh = (lk_hi >> K) & 1u;
    uint32_t v = 0u;
    if (K == 0) {
        v = __ldg(pk + W);
    } else if (!(BB && (bl & bh))) {
        const uint32_t row = row0 - (uint32_t)(CY * h + CZ * hny);
        const bool fold = XF && ((CX > 0 && w == 0) || (CX < 0 && w == h - 1));
        v = pull_x<CX>(pk, row, w, h, W, px, fold);
    }
    return link_select<K, BB>(v, fA, ns2, W, lk_lo, lk_hi);
}

template <typename T, bool BB, bool XF, int... Ks>
__device__ __forceinline__ void pull19_pair_fast_all(uint32_t* v, const uint32_t* __restrict__ fA, uint32_t ns2,
                                                     uint32_t W, uint32_t row0, int w, int h, int hny, int px,
                                                     uint32_t lk_lo, uint32_t lk_hi,
                                                     std::integer_sequence<int, Ks...>)
{
    ((v[Ks] = pull19_pair_fast<T, Ks, BB, XF>(fA, ns2, W, row0, w, h, hny, px, lk_lo, lk_hi)), ...);
}

// D3Q7: no bounce-back, keep-local outside non-periodic faces
template <int K>
__device__ __forceinline__ uint32_t pull7_pair_nbr(const uint32_t* __restrict__ gA, uint32_t ns2, uint32_t W, int w,
                                                   int h, const RowNbr& nr, int px)
{
    constexpr int CX = cx7(K), CY = cy7(K), CZ = cz7(K);
    const uint32_t* pk = gA + (uint32_t)K * ns2;
    if (K == 0 || !nr.in[1 - CY][1 - CZ]) return __ldg(pk + W);
    const bool fold = (CX > 0 && w == 0) || (CX < 0 && w == h - 1);
    return pull_x<CX>(pk, nr.rb[1 - CY][1 - CZ], w, h, W, px, fold);
}
template <int K, bool XF>
__device__ __forceinline__ uint32_t pull7_pair_fast(const uint32_t* __restrict__ gA, uint32_t ns2, uint32_t W,
                                                    uint32_t row0, int w, int h, int hny, int px)
{
    constexpr int CX = cx7(K), CY = cy7(K), CZ = cz7(K);
    const uint32_t* pk = gA + (uint32_t)K * ns2;
    if (K == 0) return __ldg(pk + W);
    const bool fold = XF && ((CX > 0 && w == 0) || (CX < 0 && w == h - 1));
    return pull_x<CX>(pk, row0 - (uint32_t)(CY * h + CZ * hny), w, h, W, px, fold);
}
template <int... Ks>
__device__ __forceinline__ void pull7_pair_nbr_all(uint32_t* v, const uint32_t* __restrict__ gA, uint32_t ns2,
                                                   uint32_t W, int w, int h, const RowNbr& nr, int px,
                                                   std::integer_sequence<int, Ks...>)
{
    ((v[Ks] = pull7_pair_nbr<Ks>(gA, ns2, W, w, h, nr, px)), ...);
}
template <bool XF, int... Ks>
__device__ __forceinline__ void pull7_pair_fast_all(uint32_t* v, const uint32_t* __restrict__ gA, uint32_t ns2,
                                                    uint32_t W, uint32_t row0, int w, int h, int hny, int px,
                                                    std::integer_sequence<int, Ks...>)
{
    ((v[Ks] = pull7_pair_fast<Ks, XF>(gA, ns2, W, row0, w, h, hny, px)), ...);
}

// ---------------------------------------------------------------------------
// the deviation-form update on pairs (dev_collide / dev_outlet per half)
// ---------------------------------------------------------------------------
template <int CX, int CY, int CZ>
__device__ __forceinline__ float2 cdot2(float2 ux, float2 uy, float2 uz)
{
    float2 e = f2(0.0f);
    bool first = true;
    if (CX != 0) { e = CX > 0 ? ux : neg2(ux); first = false; }
    if (CY != 0) { e = first ? (CY > 0 ? uy : neg2(uy)) : (CY > 0 ? add2(e, uy) : sub2(e, uy)); first = false; }
    if (CZ != 0) { e = first ? (CZ > 0 ? uz : neg2(uz)) : (CZ > 0 ? add2(e, uz) : sub2(e, uz)); }
    return e;
}

template <int CX, int CY, int CZ>
__device__ __forceinline__ float2 dev_eq2(float2 h, float2 wr, float2 wd, float2 ux, float2 uy, float2 uz, float2 m15u2,
                                          float2 omega)
{
    const float2 e = cdot2<CX, CY, CZ>(ux, uy, uz);
    const float2 t = fma2(e, fma2(f2(4.5f), e, f2(3.0f)), m15u2);
    const float2 heq = fma2(wr, t, wd);
    return fma2(omega, sub2(heq, h), h);
}

__device__ __forceinline__ float2 m15u2_of(float2 ux, float2 uy, float2 uz)
{
    return mul2(f2(-1.5f), fma2(ux, ux, fma2(uy, uy, mul2(uz, uz))));
}

// BGK in deviation form on both halves of the packed words h[19], in place:
// each direction is unpacked, collided, packed and then merged with the
// pulled word by the byte_perm selector `keep` (half_sel: halves taken from
// the pulled word are not collided -- an obstacle cell's on-site reversal).
template <typename T, int K>
__device__ __forceinline__ uint32_t dev_eq_packed(uint32_t v, float2 wr, float2 wd, float2 ux, float2 uy, float2 uz,
                                                  float2 m15u2, float2 omega, uint32_t keep)
{
    const float2 hn = dev_eq2<cx19(K), cy19(K), cz19(K)>(Pair<T>::unpack(v), wr, wd, ux, uy, uz, m15u2, omega);
    return __byte_perm(Pair<T>::pack(hn), v, keep);
}
template <typename T, int... Ks>
__device__ __forceinline__ void dev_collide_packed(uint32_t* h, float2 rho, float2 drho, float2 ux, float2 uy,
                                                   float2 uz, float2 omega, uint32_t keep,
                                                   std::integer_sequence<int, Ks...>)
{
    const float2 m15u2 = m15u2_of(ux, uy, uz);
    const float2 wr0 = mul2(rho, f2(1.0f / 3.0f)), wr1 = mul2(rho, f2(1.0f / 18.0f)), wr2 = mul2(rho, f2(1.0f / 36.0f));
    const float2 wd0 = mul2(drho, f2(1.0f / 3.0f)), wd1 = mul2(drho, f2(1.0f / 18.0f)),
                 wd2 = mul2(drho, f2(1.0f / 36.0f));
    ((h[Ks] = dev_eq_packed<T, Ks>(h[Ks], Ks == 0 ? wr0 : (Ks < 7 ? wr1 : wr2), Ks == 0 ? wd0 : (Ks < 7 ? wd1 : wd2),
                                   ux, uy, uz, m15u2, omega, keep)),
     ...);
}

// the outlet plane (dev_outlet) on the high halves of the packed words
template <typename T, int... Ks>
__device__ __forceinline__ void dev_outlet_hi_packed(uint32_t* h, float rho_out, float drho_out, float ux, float uy,
                                                     float uz, std::integer_sequence<int, Ks...>)
{
    const float m15u2 = -1.5f * fmaf(ux, ux, fmaf(uy, uy, uz * uz));
    ((h[Ks] = __byte_perm(h[Ks],
                          Pair<T>::pack(f2(fmaf(rho_out * w19<float>(Ks),
                                                fmaf(cdot<cx19(Ks), cy19(Ks), cz19(Ks)>(ux, uy, uz),
                                                     fmaf(4.5f, cdot<cx19(Ks), cy19(Ks), cz19(Ks)>(ux, uy, uz), 3.0f),
                                                     m15u2),
                                                drho_out * w19<float>(Ks)))),
                          0x7610u)),
     ...);
}

// j of the packed words, in moments19's order on each half
template <typename T, int... Ks>
__device__ __forceinline__ void moments_j2(const uint32_t* f, float2& jx, float2& jy, float2& jz,
                                           std::integer_sequence<int, Ks...>)
{
    ((jx = cx19(Ks) == 0 ? jx : (cx19(Ks) > 0 ? add2(jx, Pair<T>::unpack(f[Ks])) : sub2(jx, Pair<T>::unpack(f[Ks])))),
     ...);
    ((jy = cy19(Ks) == 0 ? jy : (cy19(Ks) > 0 ? add2(jy, Pair<T>::unpack(f[Ks])) : sub2(jy, Pair<T>::unpack(f[Ks])))),
     ...);
    ((jz = cz19(Ks) == 0 ? jz : (cz19(Ks) > 0 ? add2(jz, Pair<T>::unpack(f[Ks])) : sub2(jz, Pair<T>::unpack(f[Ks])))),
     ...);
}

__device__ __forceinline__ float2 rcp2(float2 v) { return make_float2(__frcp_rn(v.x), __frcp_rn(v.y)); }

// ---------------------------------------------------------------------------
// one pair of cells: pull, NS collision, fused outlet, LDF source, D3Q7
// collision, fused AD planes, stores, fused NEQ inlet
// ---------------------------------------------------------------------------
// The cell arrays of a pair (flag words, porosity, tau, C(s-1), q) come
// through a `Cells` policy -- global memory for k_coupled_pair, the staged
// tile for k_pair_staged -- and the D3Q7 pull through `pull7(gv)`; the update
// itself is one function for both kernels.
template <typename T, typename QT>
struct PairCellsGlobal {
    using R = typename Pop<T>::R;
    const StepArgs<T, QT>& a;
    uint32_t clo, chi;
    __device__ __forceinline__ uint32_t cell(int hi) const { return hi ? chi : clo; }
    __device__ __forceinline__ uint32_t flag(int hi) const { return __ldg(a.cellw + cell(hi)); }
    __device__ __forceinline__ R por(int hi) const { return __ldg(a.porosity + cell(hi)); }
    __device__ __forceinline__ R tau(int hi) const { return __ldg(a.tau_ad + cell(hi)); }
    __device__ __forceinline__ R source(int hi, uint32_t w, bool commit) const { return ldf_source(a, cell(hi), w, commit); }
};

template <typename T, typename QT, bool POROUS, bool MON, class Cells, class Pull7>
__device__ __forceinline__ void pair_update(const StepArgs<T, QT>& a, uint32_t W, int w, int h, uint32_t clo, bool active,
                                            bool xedge, uint32_t wlo, uint32_t whi, uint32_t* fv, const Cells& cells,
                                            const Pull7& pull7, MonAcc* mon)
{
    const uint32_t chi = clo + (uint32_t)h;
    const uint32_t ns2 = a.ns >> 1;
    uint32_t gv[7];
    // ---- NS collision, deviation form (dev_ns_collide on each half) ----
    // Only the packed words stay live: the moments and the collision unpack
    // each word as they use it, and every direction is collided, packed and
    // held packed in turn.
    float2 drho = f2(0.0f), jx = f2(0.0f), jy = f2(0.0f), jz = f2(0.0f);
#pragma unroll
    for (int k = 0; k < 19; ++k) drho = add2(drho, Pair<T>::unpack(fv[k]));
    moments_j2<T>(fv, jx, jy, jz, Seq19{});
    const float2 rho = add2(f2(a.rho0), drho);
    // the velocities enter the sums c.u of the collision: formed as j * (1/rho)
    // + (-0) with a -0 the code generator cannot fold, so no sum absorbs the product
    const float2 nz = f2(a.neg_zero);
    float2 vx, vy, vz;   // velocity of the post-collision populations
    if (__all_sync(0xffffffffu, rho.x > 0.0f && rho.y > 0.0f)) {
        const float2 inv = rcp2(rho);
        if (!POROUS) {
            vx = fma2(jx, inv, nz); vy = fma2(jy, inv, nz); vz = fma2(jz, inv, nz);
            // an obstacle cell keeps its pulled (reversed) populations: the
            // packed result takes those halves from the pulled word
            const uint32_t keep = half_sel((wlo & kSolid) ? 1u : 0u, (whi & kSolid) ? 1u : 0u);
            dev_collide_packed<T>(fv, rho, drho, vx, vy, vz, f2(a.omega), keep, Seq19{});
        } else {
            float2 ph = make_float2(cells.por(0), cells.por(1));
            ph = make_float2(fminf(fmaxf(ph.x, 0.0f), 1.0f), fminf(fmaxf(ph.y, 0.0f), 1.0f));
            const float2 bx = mul2(jx, inv), by = mul2(jy, inv), bz = mul2(jz, inv);
            dev_collide_packed<T>(fv, rho, drho, fma2(bx, ph, nz), fma2(by, ph, nz), fma2(bz, ph, nz), f2(a.omega),
                                  0x3210u, Seq19{});
            const float2 s = fma2(f2(-a.omega), sub2(f2(1.0f), ph), f2(1.0f));
            vx = mul2(bx, s); vy = mul2(by, s); vz = mul2(bz, s);
        }
    } else {
        // a warp with a cell of rho <= 0: the one-cell update on each half
        float hl[19], hh[19];
#pragma unroll
        for (int k = 0; k < 19; ++k) {
            const float2 t = Pair<T>::unpack(fv[k]);
            hl[k] = t.x;
            hh[k] = t.y;
        }
        dev_ns_collide_por<T, QT, POROUS>(a, wlo, POROUS ? cells.por(0) : 0.0f, hl, vx.x, vy.x, vz.x);
        dev_ns_collide_por<T, QT, POROUS>(a, whi, POROUS ? cells.por(1) : 0.0f, hh, vx.y, vy.y, vz.y);
#pragma unroll
        for (int k = 0; k < 19; ++k) fv[k] = Pair<T>::pack(make_float2(hl[k], hh[k]));
    }
    // PressureDirichlet at x = nx-1: the high half of w = h-1, whose x-1
    // neighbour is the high half of the previous lane
    if (a.fuse_outlet && xedge) {
        const float lx = __shfl_up_sync(0xffffffffu, vx.y, 1);
        const float ly = __shfl_up_sync(0xffffffffu, vy.y, 1);
        const float lz = __shfl_up_sync(0xffffffffu, vz.y, 1);
        if (w == h - 1) {
            dev_outlet_hi_packed<T>(fv, a.rho_out, a.rho_out - a.rho0, lx, ly, lz, Seq19{});
            vx.y = lx; vy.y = ly; vz.y = lz;
        }
    }
    uint32_t* fB = reinterpret_cast<uint32_t*>(a.fB);
    if (active) {
#pragma unroll
        for (int k = 0; k < 19; ++k) fB[(uint32_t)k * ns2 + W] = fv[k];
    }
    float2 mrho = f2(0.0f);
    const float mux = vx.y;   // the high half holds the pair's outlet cell, if any
    if (MON) {
        // the density of the stored populations
#pragma unroll
        for (int k = 0; k < 19; ++k) mrho = add2(mrho, Pair<T>::unpack(fv[k]));
        mrho = add2(mrho, f2(a.rho0));
    }
    if (!a.coupling) vx = vy = vz = f2(0.0f);

    // ---- the D3Q7 pull, after the D3Q19 stores (fewer live registers) ----
    pull7(gv);
    // ---- LDF source and D3Q7 collision ----
    const float2 S = make_float2(cells.source(0, wlo, active), cells.source(1, whi, active));
    float2 ph = PairG<T>::ld(gv[0], 0, a.g_shift);
#pragma unroll
    for (int k = 1; k < 7; ++k) ph = add2(ph, PairG<T>::ld(gv[k], k, a.g_shift));
    ph = make_float2(fmaxf(ph.x, a.min_conc), fmaxf(ph.y, a.min_conc));
    const float2 om = a.tau_ad ? make_float2(__frcp_rn(cells.tau(0)), __frcp_rn(cells.tau(1))) : f2(a.omega_ad);
    const float2 wp0 = mul2(f2(0.25f), ph), wp1 = mul2(f2(0.125f), ph);
    const float2 ws0 = mul2(f2(0.25f), S), ws1 = mul2(f2(0.125f), S);
    const bool neumann = a.fuse_neumann && xedge;
    uint32_t* gB = reinterpret_cast<uint32_t*>(a.gB);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        float2 eu;
        if (k == 0) eu = f2(0.0f);
        else if (k == 1) eu = vx;
        else if (k == 2) eu = neg2(vx);
        else if (k == 3) eu = vy;
        else if (k == 4) eu = neg2(vy);
        else if (k == 5) eu = vz;
        else eu = neg2(vz);
        const float2 wp = k == 0 ? wp0 : wp1;
        const float2 gi = PairG<T>::ld(gv[k], k, a.g_shift);
        const float2 geq = fma2(mul2(f2(4.0f), wp), eu, wp);
        float2 gn = fma2(om, sub2(geq, gi), add2(gi, k == 0 ? ws0 : ws1));
        if (neumann) {
            // ADNeumannOutlet: x = nx-1 copies x = nx-2, the previous lane's high half
            const float left = __shfl_up_sync(0xffffffffu, gn.y, 1);
            if (w == h - 1) gn.y = left;
        }
        if (a.fuse_dirichlet && w == 0) gn.x = a.c_in * w7<float>(k);
        if (active) gB[(uint32_t)k * ns2 + W] = PairG<T>::st(gn, k, a.g_shift, clo, chi);
    }
    if (active) {
        a.phi[clo] = ph.x;
        a.phi[chi] = ph.y;
    }
    if (MON && active) {
        mon->add((double)mrho.x, (double)ph.x, (double)a.q[clo], 0.0,
                 !(mrho.x > 0.0f) || !isfinite(mrho.x) || !isfinite(ph.x));
        mon->add((double)mrho.y, (double)ph.y, (double)a.q[chi], (whi & kXHi) ? (double)ph.y * (double)mux : 0.0,
                 !(mrho.y > 0.0f) || !isfinite(mrho.y) || !isfinite(ph.y));
    }
    // the NEQ inlet of the next step on the low halves: x = 0 is the low half
    // of w = 0 (storage element 2W), x = 1 that of the next lane
    if (a.fuse_inlet && xedge) fused_inlet(a, clo, 2u * W, w, active);
}

template <typename T, typename QT, bool POROUS, bool MON = false>
__device__ __forceinline__ void coupled_pair(const StepArgs<T, QT>& a, uint32_t Wg, MonAcc* mon = nullptr)
{
    static_assert(Pop<T>::kShifted, "pair layout: 16-bit shifted storage only");
    constexpr bool BB = !POROUS;
    const bool active = Wg < a.c_end;
    const uint32_t W = active ? Wg : a.c_end - 1u;
    const int h = a.nx >> 1;
    const uint32_t row = fastdiv(W, a.div_h);
    const int w = (int)(W - row * (uint32_t)h);
    const uint32_t clo = row * (uint32_t)a.nx + (uint32_t)w, chi = clo + (uint32_t)h;
    const PairCellsGlobal<T, QT> cells{a, clo, chi};
    const uint32_t wlo = cells.flag(0), whi = cells.flag(1);
    const uint32_t ns2 = a.ns >> 1;
    const uint32_t* fA = reinterpret_cast<const uint32_t*>(a.fA);
    const uint32_t* gA = reinterpret_cast<const uint32_t*>(a.gA);
    const uint32_t lk_lo = (BB && (wlo & kSolid)) ? 0x7fffeu : wlo;
    const uint32_t lk_hi = (BB && (whi & kSolid)) ? 0x7fffeu : whi;
    uint32_t fv[19];
    // both cells of a pair share y and z, so the y/z-face test is the pair's
    bool xedge = true;
    const bool face = __any_sync(0xffffffffu, (wlo & kFaceYZ) != 0u);
    if (face) {
        int x, y, z;
        cell_xyz(clo, a.nx, a.ny, a.div_nx, a.div_nxy, x, y, z);
        const RowNbr nr(y, z, a.ny, a.nz, h, a.py, a.pz);
        pull19_pair_nbr_all<T, BB>(fv, fA, ns2, W, w, h, nr, a.px, lk_lo, lk_hi, Seq19{});
    } else {
        const int hny = h * a.ny;
        const uint32_t row0 = W - (uint32_t)w;
        xedge = __any_sync(0xffffffffu, w == 0 || w == h - 1);
        if (xedge) {
            pull19_pair_fast_all<T, BB, true>(fv, fA, ns2, W, row0, w, h, hny, a.px, lk_lo, lk_hi, Seq19{});
        } else {
            pull19_pair_fast_all<T, BB, false>(fv, fA, ns2, W, row0, w, h, hny, a.px, lk_lo, lk_hi, Seq19{});
        }
    }
    const auto pull7 = [&](uint32_t* gv) {
        if (face) {
            int x, y, z;
            cell_xyz(clo, a.nx, a.ny, a.div_nx, a.div_nxy, x, y, z);
            const RowNbr nr(y, z, a.ny, a.nz, h, a.py, a.pz);
            pull7_pair_nbr_all(gv, gA, ns2, W, w, h, nr, a.px, Seq7{});
        } else if (xedge) {
            pull7_pair_fast_all<true>(gv, gA, ns2, W, W - (uint32_t)w, w, h, h * a.ny, a.px, Seq7{});
        } else {
            pull7_pair_fast_all<false>(gv, gA, ns2, W, W - (uint32_t)w, w, h, h * a.ny, a.px, Seq7{});
        }
    };
    pair_update<T, QT, POROUS, MON>(a, W, w, h, clo, active, xedge, wlo, whi, fv, cells, pull7, mon);
}

// one pair per thread, words [c_first, c_end) (c_first a multiple of 32); the
// first warp of a block prefetches into L2 what the
// block pf_dist blocks ahead reads at its own words and cells
template <typename T, typename QT>
__device__ __forceinline__ void prefetch_pairs_ahead(const StepArgs<T, QT>& a)
{
    using R = typename Pop<T>::R;
    if (a.pf_dist == 0 || threadIdx.x >= 32) return;
    const uint32_t ns2 = a.ns >> 1;
    const uint32_t w0 = a.c_first + (blockIdx.x + a.pf_dist) * blockDim.x;
    if (w0 >= ns2) return;
    // within the padded planes: a multiple of 16 words from a multiple of 256
    const uint32_t wcnt = min((uint32_t)blockDim.x, ns2 - w0);
    const int lane = threadIdx.x;
    // population words: a 16-byte aligned run (blockDim.x and ns2 are multiples of 4 words)
    if (lane < 19) l2_prefetch(reinterpret_cast<const uint32_t*>(a.fA) + (uint32_t)lane * ns2 + w0, wcnt * 4u);
    else if (lane < 26)
        l2_prefetch(reinterpret_cast<const uint32_t*>(a.gA) + (uint32_t)(lane - 19) * ns2 + w0, wcnt * 4u);
    else {
        // the cells of those words lie within their rows: [row(w0) nx, (row(last) + 1) nx)
        const uint32_t h = (uint32_t)a.nx >> 1;
        const uint32_t r0 = fastdiv(w0, a.div_h), r1 = fastdiv(w0 + wcnt - 1u, a.div_h);
        const uint32_t c0 = (r0 * (uint32_t)a.nx) & ~31u;
        const uint32_t c1 = min((r1 + 1u) * 2u * h, (uint32_t)a.ns);
        const uint32_t cnt = c1 - c0;
        if (lane == 26) l2_prefetch(a.cellw + c0, cnt * 4u);
        else if (lane == 27) l2_prefetch(a.phi + c0, cnt * (uint32_t)sizeof(R));
        else if (lane == 28 && a.isotherm) l2_prefetch(a.q + c0, cnt * (uint32_t)sizeof(QT));
        else if (lane == 29 && a.porosity) l2_prefetch(a.porosity + c0, cnt * (uint32_t)sizeof(R));
        else if (lane == 30 && a.tau_ad) l2_prefetch(a.tau_ad + c0, cnt * (uint32_t)sizeof(R));
    }
}

// resident 256-thread blocks per SM the pair kernel is compiled for: 4 (64
// registers) for BGK; porous BGK carries the porosity and a second velocity
// through the collision and gets 3 (80 registers)
template <bool POROUS>
constexpr int kPairBlocks = POROUS ? 3 : 4;

template <typename T, typename QT, bool POROUS, bool MON = false>
__global__ void __launch_bounds__(256, kPairBlocks<POROUS>) k_coupled_pair(const StepArgs<T, QT> a)
{
    prefetch_pairs_ahead(a);
    if constexpr (MON) {
        MonAcc m;
        coupled_pair<T, QT, POROUS, true>(a, a.c_first + blockIdx.x * blockDim.x + threadIdx.x, &m);
        monitor_block_reduce(m, a.mon + (size_t)blockIdx.x * kMonN);
    } else {
        coupled_pair<T, QT, POROUS>(a, a.c_first + blockIdx.x * blockDim.x + threadIdx.x);
    }
}

// ---------------------------------------------------------------------------
// the staged pair kernel: source rows by bulk copy into shared memory
// ---------------------------------------------------------------------------
// k_coupled_pair loads its 26 pulled words per pair straight from global
// memory; at 64-80 registers per thread few warps fit on an SM and each warp
// waits for its loads before it can compute (measured: long-scoreboard stalls,
// about half of HBM bandwidth).  k_pair_staged instead runs a persistent grid
// over tiles of whole x-rows: for every tile the copy engine brings, by 1D
// bulk copies (cp.async.bulk, completion counted on an mbarrier), the 26
// source rows the tile pulls from -- direction k's row of each tile row is the
// row at (y - c_y, z - c_z), wrapped on periodic faces and the row itself
// across a closed face -- plus the tile's flag words, C(s-1), q, porosity and
// tau.  Two stages alternate: while the block updates tile i from one stage,
// the copies of its next tile fill the other, so the loads of a tile overlap
// the arithmetic of the one before and no thread holds a load in flight.
//
// Within a staged row the x shift is an index: word w pulls word w - c_x of
// the source row; the fold words (w = 0 with c_x = +1, w = h-1 with c_x = -1)
// assemble their halves from the row's other end exactly as pull_x does.
// The few words that are not in a staged row -- the pair's own word of a
// direction with c_y or c_z != 0, which a closed x face keeps and bounce-back
// reads -- come from global memory as in k_coupled_pair.
//
// Tiles: R = 256 / h rows (h = nx/2 <= 256 words, nx % 8 == 0 so every row
// starts on a 16-byte boundary), one thread per word.  Each wait on a stage is
// bounded (kStageWaitLimit polls); a wait that gives up sets bit 0 of
// a.status, and the block waits (bounded again) for its copies in flight and
// leaves the grid.
constexpr int kStageThreads = 256;
constexpr uint32_t kStageHeader = 128;          // the two mbarriers, 128-byte aligned stages after them
constexpr uint32_t kStageWaitLimit = 1u << 22;  // try_wait polls before a wait gives up

struct StageGeom {
    uint32_t rows, words, cells;   // x-rows, words (rows h) and cells (rows nx) of a tile
    uint32_t off_q, off_pop, off_flag, off_phi, off_por, off_tau, bytes;
};
// the layout of one stage: [q][26 population rows][flag][C][porosity][tau],
// each part a multiple of 16 bytes (nx % 8 == 0)
__host__ __device__ inline StageGeom stage_geom(int nx, uint32_t rows, bool has_q, bool has_por, bool has_tau,
                                                uint32_t q_bytes, uint32_t r_bytes)
{
    StageGeom g;
    g.rows = rows;
    g.words = rows * (uint32_t)(nx / 2);
    g.cells = rows * (uint32_t)nx;
    uint32_t o = 0;
    g.off_q = o;
    o += has_q ? g.cells * q_bytes : 0u;
    g.off_pop = o;
    o += 26u * g.words * 4u;
    g.off_flag = o;
    o += g.cells * 4u;
    g.off_phi = o;
    o += g.cells * r_bytes;
    g.off_por = o;
    o += has_por ? g.cells * r_bytes : 0u;
    g.off_tau = o;
    o += has_tau ? g.cells * r_bytes : 0u;
    g.bytes = o;
    return g;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0u;
}
// bounded wait for the phase of `parity` of *bar; false: gave up
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kStageWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// global -> shared bulk copy of `bytes` (16-byte aligned, a multiple of 16),
// completion counted on *bar; into this CTA's own shared memory only, from
// this GPU's own memory
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// the source row of `row` (= y + ny z) in a direction with velocity (cy, cz):
// the neighbour row, wrapped on periodic faces, or the row itself across a
// closed face (keep-local)
__device__ __forceinline__ uint32_t stage_source_row(uint32_t row, int cy, int cz, int ny, int nz, int py, int pz)
{
    const int z = (int)(row / (uint32_t)ny), y = (int)row - z * ny;
    int ys = y - cy, zs = z - cz;
    bool in = true;
    if (ys < 0) { if (py) ys += ny; else in = false; }
    if (ys >= ny) { if (py) ys -= ny; else in = false; }
    if (zs < 0) { if (pz) zs += nz; else in = false; }
    if (zs >= nz) { if (pz) zs -= nz; else in = false; }
    return in ? (uint32_t)(ys + ny * zs) : row;
}
// c_y and c_z of direction k (D3Q19 k < 19, D3Q7 k - 19 otherwise) for a
// runtime k, from bit masks (a runtime index into the constexpr tables would
// put them in local memory)
__device__ __forceinline__ int stage_cy(int k)
{
    if (k < 19) return (int)((kPY >> k) & 1u) - (int)((kMY >> k) & 1u);
    return (int)(k == 19 + 3) - (int)(k == 19 + 4);
}
__device__ __forceinline__ int stage_cz(int k)
{
    if (k < 19) return (int)((kPZ >> k) & 1u) - (int)((kMZ >> k) & 1u);
    return (int)(k == 19 + 5) - (int)(k == 19 + 6);
}

// warp 0 queues the copies of the tile of rows [r0, r0 + nrows) into stage `st`
template <typename T, typename QT>
__device__ __forceinline__ void stage_issue(const StepArgs<T, QT>& a, const StageGeom& g, unsigned char* st,
                                            uint64_t* bar, uint32_t r0, uint32_t nrows)
{
    using R = typename Pop<T>::R;
    const int lane = threadIdx.x & 31;
    const uint32_t h = (uint32_t)a.nx >> 1, ns2 = a.ns >> 1;
    const uint32_t cells = nrows * (uint32_t)a.nx;
    uint32_t bytes = 26u * nrows * h * 4u + cells * (4u + (uint32_t)sizeof(R));
    if (a.isotherm) bytes += cells * (uint32_t)sizeof(QT);
    if (a.porosity) bytes += cells * (uint32_t)sizeof(R);
    if (a.tau_ad) bytes += cells * (uint32_t)sizeof(R);
    // shared memory this block read through the generic proxy is rewritten by
    // the copy engine: order the two proxies, then count the bytes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane == 0) mbar_expect_tx(bar, bytes);
    __syncwarp();
    if (lane < 26) {
        const int k = lane;
        const uint32_t* base = k < 19 ? reinterpret_cast<const uint32_t*>(a.fA) + (uint32_t)k * ns2
                                      : reinterpret_cast<const uint32_t*>(a.gA) + (uint32_t)(k - 19) * ns2;
        uint32_t* dst = reinterpret_cast<uint32_t*>(st + g.off_pop) + (uint32_t)k * g.rows * h;
        const int cy = stage_cy(k), cz = stage_cz(k);
        // consecutive tile rows whose sources are consecutive rows go in one copy
        uint32_t run_src = 0, run_dst = 0, run_len = 0;
        for (uint32_t rr = 0; rr < nrows; ++rr) {
            const uint32_t src = stage_source_row(r0 + rr, cy, cz, a.ny, a.nz, a.py, a.pz);
            if (run_len && src == run_src + run_len) {
                ++run_len;
                continue;
            }
            if (run_len) bulk_to_smem(dst + run_dst * h, base + run_src * h, run_len * h * 4u, bar);
            run_src = src;
            run_dst = rr;
            run_len = 1;
        }
        if (run_len) bulk_to_smem(dst + run_dst * h, base + run_src * h, run_len * h * 4u, bar);
    } else {
        const size_t c0 = (size_t)r0 * (size_t)a.nx;
        if (lane == 26) bulk_to_smem(st + g.off_flag, a.cellw + c0, cells * 4u, bar);
        else if (lane == 27) bulk_to_smem(st + g.off_phi, a.phi + c0, cells * (uint32_t)sizeof(R), bar);
        else if (lane == 28 && a.isotherm) bulk_to_smem(st + g.off_q, a.q + c0, cells * (uint32_t)sizeof(QT), bar);
        else if (lane == 29 && a.porosity) bulk_to_smem(st + g.off_por, a.porosity + c0, cells * (uint32_t)sizeof(R), bar);
        else if (lane == 30 && a.tau_ad) bulk_to_smem(st + g.off_tau, a.tau_ad + c0, cells * (uint32_t)sizeof(R), bar);
    }
}

// the cell arrays of a pair from the staged tile (il, ih: the pair's cells
// within the tile); q is written back to global memory by ldf_source_of
template <typename T, typename QT>
struct PairCellsStaged {
    using R = typename Pop<T>::R;
    const StepArgs<T, QT>& a;
    const unsigned char* st;
    StageGeom g;
    uint32_t il, ih, clo, chi;
    __device__ __forceinline__ uint32_t at(int hi) const { return hi ? ih : il; }
    __device__ __forceinline__ uint32_t flag(int hi) const
    {
        return reinterpret_cast<const uint32_t*>(st + g.off_flag)[at(hi)];
    }
    __device__ __forceinline__ R por(int hi) const { return reinterpret_cast<const R*>(st + g.off_por)[at(hi)]; }
    __device__ __forceinline__ R tau(int hi) const { return reinterpret_cast<const R*>(st + g.off_tau)[at(hi)]; }
    __device__ __forceinline__ R source(int hi, uint32_t w, bool commit) const
    {
        if (a.isotherm == 0 || !(w & kRegion)) return R(0);
        QT qn;
        return ldf_source_of(a, hi ? chi : clo, w, commit, reinterpret_cast<const R*>(st + g.off_phi)[at(hi)],
                             reinterpret_cast<const QT*>(st + g.off_q)[at(hi)], qn);
    }
};

// pulls of one pair from the staged rows.  `keep`: bit k set when the pair's
// row keeps direction k (a closed y/z face; bit 19 + k for D3Q7); XF: fold
// words possible in this warp.  own(k) is the pair's own word of direction k:
// the staged row itself when c_y = c_z = 0, else a global load.
template <int K, bool XF>
__device__ __forceinline__ uint32_t stage_pull(const uint32_t* row, int w, int h, bool kp, int px,
                                               const uint32_t* __restrict__ own_k)
{
    constexpr int CX = K < 19 ? cx19(K) : cx7(K - 19);
    constexpr int CY = K < 19 ? cy19(K) : cy7(K - 19);
    constexpr int CZ = K < 19 ? cz19(K) : cz7(K - 19);
    if (CX == 0 || kp) return row[w];
    if (XF && CX > 0 && w == 0) {
        const uint32_t t = row[h - 1];
        const uint32_t own = px ? t : ((CY == 0 && CZ == 0) ? row[0] : __ldg(own_k));
        return __byte_perm(own, t, px ? 0x5476u : 0x5410u);
    }
    if (XF && CX < 0 && w == h - 1) {
        const uint32_t t = row[0];
        const uint32_t own = px ? t : ((CY == 0 && CZ == 0) ? row[h - 1] : __ldg(own_k));
        return __byte_perm(t, own, px ? 0x5432u : 0x7632u);
    }
    return row[w - CX];
}

// bounce-back on a staged pull: halves whose link bit K is set take the
// pair's own opposite word (staged when the opposite direction has c_y = c_z = 0)
template <int K, bool BB>
__device__ __forceinline__ uint32_t stage_link(uint32_t v, const uint32_t* spop, uint32_t rows, uint32_t rr, int w, int h,
                                               const uint32_t* __restrict__ fA, uint32_t ns2, uint32_t W, uint32_t lk_lo,
                                               uint32_t lk_hi)
{
    if (!BB || K == 0) return v;
    constexpr int O = opp19(K);
    const uint32_t bl = (lk_lo >> K) & 1u, bh = (lk_hi >> K) & 1u;
    if (bl | bh) {
        const uint32_t o = (cy19(O) == 0 && cz19(O) == 0) ? spop[((uint32_t)O * rows + rr) * (uint32_t)h + (uint32_t)w]
                                                          : __ldg(fA + (uint32_t)O * ns2 + W);
        v = __byte_perm(v, o, half_sel(bl, bh));
    }
    return v;
}

template <bool BB, bool XF, int... Ks>
__device__ __forceinline__ void stage_pull19_all(uint32_t* fv, const uint32_t* spop, uint32_t rows, uint32_t rr, int w,
                                                 int h, uint32_t keep, int px, const uint32_t* __restrict__ fA,
                                                 uint32_t ns2, uint32_t W, uint32_t lk_lo, uint32_t lk_hi,
                                                 std::integer_sequence<int, Ks...>)
{
    ((fv[Ks] = stage_link<Ks, BB>(
          stage_pull<Ks, XF>(spop + ((uint32_t)Ks * rows + rr) * (uint32_t)h, w, h, (keep >> Ks) & 1u, px,
                             fA + (uint32_t)Ks * ns2 + W),
          spop, rows, rr, w, h, fA, ns2, W, lk_lo, lk_hi)),
     ...);
}
template <bool XF, int... Ks>
__device__ __forceinline__ void stage_pull7_all(uint32_t* gv, const uint32_t* spop, uint32_t rows, uint32_t rr, int w,
                                                int h, uint32_t keep, int px, const uint32_t* __restrict__ gA,
                                                uint32_t ns2, uint32_t W, std::integer_sequence<int, Ks...>)
{
    ((gv[Ks] = stage_pull<19 + Ks, XF>(spop + ((uint32_t)(19 + Ks) * rows + rr) * (uint32_t)h, w, h,
                                       (keep >> (19 + Ks)) & 1u, px, gA + (uint32_t)Ks * ns2 + W)),
     ...);
}

// keep bits of a row at (y, z): directions whose source row lies across a closed y/z face
__device__ __forceinline__ uint32_t stage_keep_bits(uint32_t row, int ny, int nz, int py, int pz)
{
    const int z = (int)(row / (uint32_t)ny), y = (int)row - z * ny;
    uint32_t keep = 0;
#pragma unroll
    for (int k = 1; k < 26; ++k) {
        const int ys = y - stage_cy(k), zs = z - stage_cz(k);
        const bool out = (!py && (ys < 0 || ys >= ny)) || (!pz && (zs < 0 || zs >= nz));
        keep |= out ? (1u << k) : 0u;
    }
    return keep;
}

template <typename T, typename QT, bool POROUS, bool MON>
__global__ void __launch_bounds__(kStageThreads, 3) k_pair_staged(const StepArgs<T, QT> a)
{
    static_assert(Pop<T>::kShifted, "pair layout: 16-bit shifted storage only");
    using R = typename Pop<T>::R;
    constexpr bool BB = !POROUS;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
    const int h = a.nx >> 1;
    const StageGeom g = stage_geom(a.nx, a.st_rows, a.isotherm != 0, a.porosity != nullptr, a.tau_ad != nullptr,
                                   (uint32_t)sizeof(QT), (uint32_t)sizeof(R));
    unsigned char* const stage0 = smem + kStageHeader;   // stage s at stage0 + s * g.bytes
    const uint32_t row_begin = a.c_first / (uint32_t)h, row_end = a.c_end / (uint32_t)h;
    const uint32_t ntiles = (row_end - row_begin + g.rows - 1u) / g.rows;
    const uint32_t ns2 = a.ns >> 1;
    const uint32_t* fA = reinterpret_cast<const uint32_t*>(a.fA);
    const uint32_t* gA = reinterpret_cast<const uint32_t*>(a.gA);
    const int t = threadIdx.x;
    const uint32_t rr_t = (uint32_t)t / (uint32_t)h;   // this thread's row within a tile
    const int w = t - (int)rr_t * h;                     // and its word within the row
    const bool in_tile = rr_t < g.rows;
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    MonAcc m;
    uint32_t tile = blockIdx.x;
    if (tile < ntiles && t < 32) {
        const uint32_t r0 = row_begin + tile * g.rows;
        stage_issue(a, g, stage0, &bars[0], r0, min(g.rows, row_end - r0));
    }
    for (uint32_t it = 0; tile < ntiles; tile += gridDim.x, ++it) {
        const uint32_t s = it & 1u;
        const bool arrived = mbar_wait_bounded(&bars[s], (it >> 1) & 1u);
        if (__syncthreads_or(!arrived)) {
            // a copy that never completes: report it and leave once the
            // copies in flight have landed (or that wait gives up too)
            if (t == 0) atomicOr(a.status, 1);
            mbar_wait_bounded(&bars[s], (it >> 1) & 1u);
            return;
        }
        // every thread is past the previous tile, so the other stage is free:
        // queue the next tile's copies before updating this one
        const uint32_t next = tile + gridDim.x;
        if (next < ntiles && t < 32) {
            const uint32_t r0n = row_begin + next * g.rows;
            stage_issue(a, g, stage0 + (s ^ 1u) * g.bytes, &bars[s ^ 1u], r0n, min(g.rows, row_end - r0n));
        }
        const uint32_t r0 = row_begin + tile * g.rows;
        const uint32_t nrows = min(g.rows, row_end - r0);
        const bool active = in_tile && rr_t < nrows;
        const uint32_t rr = active ? rr_t : 0u;       // idle threads recompute row 0 and store nothing
        const uint32_t row = r0 + rr;
        const uint32_t W = row * (uint32_t)h + (uint32_t)w;
        const uint32_t clo = row * (uint32_t)a.nx + (uint32_t)w;
        const unsigned char* st = stage0 + s * g.bytes;
        const uint32_t il = rr * (uint32_t)a.nx + (uint32_t)w;
        const PairCellsStaged<T, QT> cells{a, st, g, il, il + (uint32_t)h, clo, clo + (uint32_t)h};
        const uint32_t wlo = cells.flag(0), whi = cells.flag(1);
        const uint32_t lk_lo = (BB && (wlo & kSolid)) ? 0x7fffeu : wlo;
        const uint32_t lk_hi = (BB && (whi & kSolid)) ? 0x7fffeu : whi;
        const uint32_t* spop = reinterpret_cast<const uint32_t*>(st + g.off_pop);
        uint32_t keep = 0;
        if (__any_sync(0xffffffffu, (wlo & kFaceYZ) != 0u)) keep = stage_keep_bits(row, a.ny, a.nz, a.py, a.pz);
        const bool xedge = __any_sync(0xffffffffu, w == 0 || w == h - 1);
        uint32_t fv[19];
        if (xedge)
            stage_pull19_all<BB, true>(fv, spop, g.rows, rr, w, h, keep, a.px, fA, ns2, W, lk_lo, lk_hi, Seq19{});
        else
            stage_pull19_all<BB, false>(fv, spop, g.rows, rr, w, h, keep, a.px, fA, ns2, W, lk_lo, lk_hi, Seq19{});
        const auto pull7 = [&](uint32_t* gv) {
            if (xedge) stage_pull7_all<true>(gv, spop, g.rows, rr, w, h, keep, a.px, gA, ns2, W, Seq7{});
            else stage_pull7_all<false>(gv, spop, g.rows, rr, w, h, keep, a.px, gA, ns2, W, Seq7{});
        };
        if constexpr (MON) pair_update<T, QT, POROUS, true>(a, W, w, h, clo, active, xedge, wlo, whi, fv, cells, pull7, &m);
        else pair_update<T, QT, POROUS, false>(a, W, w, h, clo, active, xedge, wlo, whi, fv, cells, pull7, nullptr);
    }
    if constexpr (MON) monitor_block_reduce(m, a.mon + (size_t)blockIdx.x * kMonN);
}

// ---------------------------------------------------------------------------
// layout conversion and element mapping
// ---------------------------------------------------------------------------
// dst[k][e(c)] = src[k][c] (to_pair) or dst[k][c] = src[k][e(c)], over nq planes of n cells
template <typename E>
__global__ void k_pair_permute(const E* __restrict__ src, E* __restrict__ dst, long long ns, int n, int nq,
                               uint32_t h, unsigned long long div_nx, int to_pair)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)nq * n) return;
    const int k = (int)(i / n);
    const uint32_t c = (uint32_t)(i - (long long)k * n);
    const uint32_t e = pair_element(c, h, div_nx);
    if (to_pair) dst[(long long)k * ns + e] = src[(long long)k * ns + c];
    else dst[(long long)k * ns + c] = src[(long long)k * ns + e];
}

// The access pattern of the pair kernel as a pure copy (measurement aid):
// every word reads its 19 + 7 pull sources off the fold points and writes them
// to its own words, no arithmetic.  Words [w_lo, w_hi) run; the host picks
// them so every source lies inside the lattice.
__global__ void __launch_bounds__(256) k_pull_copy_pair(const uint32_t* __restrict__ fA, uint32_t* __restrict__ fB,
                                                        const uint32_t* __restrict__ gA, uint32_t* __restrict__ gB,
                                                        uint32_t ns2, int h, int hny, uint32_t w_lo, uint32_t w_hi)
{
    const uint32_t W = w_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (W >= w_hi) return;
    uint32_t v[19], u[7];
#pragma unroll
    for (int k = 0; k < 19; ++k)
        v[k] = fA[(size_t)k * ns2 + (W - (uint32_t)(cx19(k) + cy19(k) * h + cz19(k) * hny))];
#pragma unroll
    for (int k = 0; k < 7; ++k) u[k] = gA[(size_t)k * ns2 + (W - (uint32_t)(cx7(k) + cy7(k) * h + cz7(k) * hny))];
#pragma unroll
    for (int k = 0; k < 19; ++k) fB[(size_t)k * ns2 + W] = v[k];
#pragma unroll
    for (int k = 0; k < 7; ++k) gB[(size_t)k * ns2 + W] = u[k];
}

}  // namespace fm
