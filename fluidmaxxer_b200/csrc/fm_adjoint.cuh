// fm_adjoint.cuh -- reverse-mode (adjoint) kernels of the coupled step.
//
// Forward step s+1 maps the state X_s = (f_s, g_s, phi_s, q_s) to X_{s+1};
// phi_s is the AD scalar computed during step s (the LDF source of step s+1
// reads it).  f_s is held as the fused kernel holds it: at x = 0 the
// VelocityDirichletNEQ values the next pull reads, derived from f_s at x = 1.
// Given the adjoint lambda_{s+1} = dL/dX_{s+1}, two kernels produce lambda_s:
//
//   k_adj_cell    per cell: recompute the forward step at the cell (the same
//                 device functions as k_coupled_step), then apply in reverse
//                 the AD boundaries, the D3Q7 collision, the LDF source, the
//                 coupling velocity, the pressure outlet and the NS collision.
//                 Writes the adjoints of the pulled populations (lfi, lgi),
//                 lambda(phi_s), lambda(q_s) and accumulates the gradients of
//                 the isotherm parameters and of the porosity field.
//   k_adj_stream  per cell: the transposed pull (a gather of lfi / lgi from
//                 the cells that read each population: neighbour pull,
//                 keep-local, own-opposite bounce-back, obstacle reversal);
//   k_adj_inlet   per inlet row: the NEQ inlet's adjoint from x = 0 into x = 1.
//
// Non-smooth points take the derivative of the branch the forward took (the
// phi clamp, max(c, eps), the porosity clamp).  Supported set-up: BGK or
// porous collision, NEQ inlet on the full x = 0 plane (or none), pressure
// outlet on the full x = nx-1 plane (or none), AD Dirichlet / Neumann on the
// full planes (or none), linear or Langmuir isotherm, the outlet probe on the
// x = nx-1 plane, even nx.
#pragma once

#include "fm_kernels.cuh"

namespace fm {

template <typename T, typename QT>
struct AdjArgs {
    using R = typename Pop<T>::R;
    StepArgs<T, QT> a;              // forward step from X_s (fA = f_s, gA = g_s, phi = phi_s, q = q_s)
    const R* __restrict__ lf1;      // lambda f_{s+1}   [19][ns]
    const R* __restrict__ lg1;      // lambda g_{s+1}   [7][ns]
    const R* __restrict__ lphi1;    // lambda phi_{s+1}
    const R* __restrict__ lq1;      // lambda q_{s+1}
    R* __restrict__ lfi;            // out: lambda of the pulled D3Q19 populations
    R* __restrict__ lgi;            // out: lambda of the pulled D3Q7 populations
    R* __restrict__ lphi0;          // out: lambda phi_s
    R* __restrict__ lq0;            // out: lambda q_s
    double* __restrict__ gpor;      // += dL/d porosity per cell (porous collision)
    double* __restrict__ gpar;      // += dL/d (isotherm a, b, k)
    R wl;                           // loss weight on phi_{s+1} of the outlet plane (0: not sampled)
};

// d feq_k / du of the second-order equilibrium: w rho (3 c + 9 (c.u) c - 3 u)
template <typename R>
__device__ __forceinline__ void dfeq_du(int k, R w, R rho, R ux, R uy, R uz, R& gx, R& gy, R& gz)
{
    const R cx = (R)cx19(k), cy = (R)cy19(k), cz = (R)cz19(k);
    const R e = cx * ux + cy * uy + cz * uz;
    gx = w * rho * (R(3) * cx + R(9) * e * cx - R(3) * ux);
    gy = w * rho * (R(3) * cy + R(9) * e * cy - R(3) * uy);
    gz = w * rho * (R(3) * cz + R(9) * e * cz - R(3) * uz);
}

template <typename R>
__device__ __forceinline__ R poly19(int k, R ux, R uy, R uz)
{
    const R e = (R)cx19(k) * ux + (R)cy19(k) * uy + (R)cz19(k) * uz;
    return R(1) + R(3) * e + R(4.5) * e * e - R(1.5) * (ux * ux + uy * uy + uz * uz);
}

// resident 256-thread blocks per SM k_adj_cell is compiled for (FP64 needs its
// registers: the recomputed forward and the adjoint are both live)
template <typename T>
constexpr int kAdjBlocks = sizeof(T) == 8 ? 1 : 3;

template <typename T, typename QT, bool POROUS>
__global__ void __launch_bounds__(256, kAdjBlocks<T>) k_adj_cell(const AdjArgs<T, QT> A)
{
    using R = typename Pop<T>::R;
    const StepArgs<T, QT>& a = A.a;
    const uint32_t cg = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = cg < (uint32_t)a.n;
    const uint32_t c = active ? cg : (uint32_t)a.n - 1u;
    int x, y, z;
    cell_xyz(c, a.nx, a.ny, a.div_nx, a.div_nxy, x, y, z);
    const Nbr nb(x, y, z, a.nx, a.ny, a.nz, a.px, a.py, a.pz);
    const uint32_t w = __ldg(a.cellw + c);
    const bool solid = !POROUS && (w & kSolid);
    const uint32_t ns = a.ns;

    // ---- forward recompute of the NS part ----
    R fi[19];
    pull19_all<T, !POROUS>(fi, a.fA, ns, c, nb, w, a.f_shift, Seq19{});
    R rho = R(0), ubx = R(0), uby = R(0), ubz = R(0), ux = R(0), uy = R(0), uz = R(0), por = R(1);
    bool por_free = false;   // porosity strictly inside [0,1]: the clamp passes the derivative
    if (!solid) {
        R jx, jy, jz;
        moments19(fi, rho, jx, jy, jz, Seq19{});
        if (!(rho > R(0))) { rho = a.rho0; jx = jy = jz = R(0); }
        const R inv = R(1) / rho;
        ubx = jx * inv; uby = jy * inv; ubz = jz * inv;
        ux = ubx; uy = uby; uz = ubz;
        if (POROUS) {
            R ph = __ldg(a.porosity + c);
            por_free = ph > R(0) && ph < R(1);
            if (ph < R(0)) ph = R(0);
            if (ph > R(1)) ph = R(1);
            por = ph;
            ux *= ph; uy *= ph; uz *= ph;
        }
    }
    // post-collision populations fh (BGK: fi + omega (feq - fi); obstacle: fi)
    R fh[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) {
        if (solid) { fh[k] = fi[k]; continue; }
        const R feq = w19<R>(k) * rho * poly19(k, ux, uy, uz);
        fh[k] = fi[k] + a.omega * (feq - fi[k]);
    }
    // moments of fh (the x-1 neighbour's velocity for the outlet)
    R rh, hx, hy, hz;
    moments19(fh, rh, hx, hy, hz, Seq19{});
    const R ih = (rh > R(0)) ? (R(1) / rh) : R(0);
    const R uhx = hx * ih, uhy = hy * ih, uhz = hz * ih;
    const bool outlet = a.fuse_outlet && x == a.nx - 1;
    const R uNx = __shfl_up_sync(0xffffffffu, uhx, 1);
    const R uNy = __shfl_up_sync(0xffffffffu, uhy, 1);
    const R uNz = __shfl_up_sync(0xffffffffu, uhz, 1);
    // post-boundary populations and the coupling velocity of them
    R fp[19];
#pragma unroll
    for (int k = 0; k < 19; ++k)
        fp[k] = outlet ? w19<R>(k) * a.rho_out * poly19(k, uNx, uNy, uNz) : fh[k];
    R rp, px, py, pz;
    moments19(fp, rp, px, py, pz, Seq19{});
    const R ip = (rp > R(0)) ? (R(1) / rp) : R(0);
    const R uax = a.coupling ? px * ip : R(0), uay = a.coupling ? py * ip : R(0), uaz = a.coupling ? pz * ip : R(0);

    // ---- forward recompute of the AD part ----
    R gi[7];
    pull7(a, c, nb, gi);
    R gs = gi[0];
#pragma unroll
    for (int k = 1; k < 7; ++k) gs += gi[k];
    const bool phi_free = !(gs < a.min_conc);
    const R phi = phi_free ? gs : a.min_conc;
    const R om = a.tau_ad ? R(1) / __ldg(a.tau_ad + c) : a.omega_ad;
    const bool region = a.isotherm != 0 && (w & kRegion);

    // ---- adjoint of the AD boundaries and collision ----
    R lg[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) lg[k] = A.lg1[(uint32_t)k * ns + c];
    if (a.fuse_dirichlet && x == 0) {
#pragma unroll
        for (int k = 0; k < 7; ++k) lg[k] = R(0);
    }
    if (a.fuse_neumann) {
        if (x == a.nx - 1) {
#pragma unroll
            for (int k = 0; k < 7; ++k) lg[k] = R(0);
        } else if (x == a.nx - 2) {
#pragma unroll
            for (int k = 0; k < 7; ++k) lg[k] += A.lg1[(uint32_t)k * ns + c + 1];
        }
    }
    R lphi = A.lphi1[c] + (x == a.nx - 1 ? A.wl : R(0));
    R lS = R(0), lux = R(0), luy = R(0), luz = R(0);
    R bsum = lphi;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        R eu;
        if (k == 0) eu = R(0);
        else if (k == 1) eu = uax;
        else if (k == 2) eu = -uax;
        else if (k == 3) eu = uay;
        else if (k == 4) eu = -uay;
        else if (k == 5) eu = uaz;
        else eu = -uaz;
        bsum += lg[k] * om * w7<R>(k) * (R(1) + R(4) * eu);
        lS += lg[k] * w7<R>(k);
        const R t = lg[k] * om * w7<R>(k) * phi * R(4);
        if (k == 1) lux += t;
        else if (k == 2) lux -= t;
        else if (k == 3) luy += t;
        else if (k == 4) luy -= t;
        else if (k == 5) luz += t;
        else if (k == 6) luz -= t;
    }
    R lgo[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) lgo[k] = (R(1) - om) * lg[k] + (phi_free ? bsum : R(0));

    // ---- adjoint of the LDF source ----
    R lq = A.lq1[c];
    R lphi0 = R(0);
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    if (region) {
        const R p0 = a.phi[c];
        const bool cfree = !(p0 < a.min_conc);
        const R ce = (cfree ? p0 : a.min_conc) - a.min_conc;
        const R qi = (R)a.q[c];
        R qeq, dqeq_dce, g_a, g_b;
        if (a.isotherm == 1) {
            qeq = a.iso_a * ce;
            dqeq_dce = a.iso_a;
            g_a = ce;
            g_b = R(0);
        } else {
            const R bc = a.iso_b * ce;
            const R den = R(1) + bc;
            qeq = a.iso_a * (bc / den);
            dqeq_dce = a.iso_a * a.iso_b / (den * den);
            g_a = bc / den;
            g_b = a.iso_a * ce / (den * den);
        }
        const R ldq = lq - lS;              // q' = q + dq, S = -dq
        const R lqeq = a.iso_k * ldq;
        g0 = (double)(lqeq * g_a);
        g1 = (double)(lqeq * g_b);
        g2 = (double)(ldq * (qeq - qi));
        lq = lq - a.iso_k * ldq;
        lphi0 = cfree ? lqeq * dqeq_dce : R(0);
    }

    // ---- adjoint of the NS part ----
    R lf[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) lf[k] = A.lf1[(uint32_t)k * ns + c];
    if (a.coupling && rp > R(0)) {
        // u_adv = j(fp) / rho(fp)
#pragma unroll
        for (int k = 0; k < 19; ++k)
            lf[k] += (((R)cx19(k) - uax) * lux + ((R)cy19(k) - uay) * luy + ((R)cz19(k) - uaz) * luz) * ip;
    }
    // pressure outlet: fp(nx-1) = feq_out(rho_out, u of fh(nx-2))
    R lNx = R(0), lNy = R(0), lNz = R(0);
    if (outlet) {
#pragma unroll
        for (int k = 0; k < 19; ++k) {
            R gx, gy, gz;
            dfeq_du(k, w19<R>(k), a.rho_out, uNx, uNy, uNz, gx, gy, gz);
            lNx += lf[k] * gx; lNy += lf[k] * gy; lNz += lf[k] * gz;
            lf[k] = R(0);
        }
    }
    if (a.fuse_outlet) {
        const R rx = __shfl_down_sync(0xffffffffu, lNx, 1);
        const R ry = __shfl_down_sync(0xffffffffu, lNy, 1);
        const R rz = __shfl_down_sync(0xffffffffu, lNz, 1);
        if (x == a.nx - 2 && rh > R(0)) {
#pragma unroll
            for (int k = 0; k < 19; ++k)
                lf[k] += (((R)cx19(k) - uhx) * rx + ((R)cy19(k) - uhy) * ry + ((R)cz19(k) - uhz) * rz) * ih;
        }
    }
    // collision: fh = fi + omega (feq(rho, u) - fi), u = por * j / rho
    if (!solid) {
        R As = R(0), Vx = R(0), Vy = R(0), Vz = R(0);
#pragma unroll
        for (int k = 0; k < 19; ++k) {
            As += lf[k] * w19<R>(k) * poly19(k, ux, uy, uz);
            R gx, gy, gz;
            dfeq_du(k, w19<R>(k), rho, ux, uy, uz, gx, gy, gz);
            Vx += lf[k] * gx; Vy += lf[k] * gy; Vz += lf[k] * gz;
        }
        const R sc = a.omega * por / rho;
#pragma unroll
        for (int k = 0; k < 19; ++k)
            lf[k] = (R(1) - a.omega) * lf[k] + a.omega * As +
                    sc * (((R)cx19(k) - ubx) * Vx + ((R)cy19(k) - uby) * Vy + ((R)cz19(k) - ubz) * Vz);
        if (POROUS && active && por_free)
            A.gpor[c] += (double)(a.omega * (Vx * ubx + Vy * uby + Vz * ubz));
    }
    if (active) {
#pragma unroll
        for (int k = 0; k < 19; ++k) A.lfi[(uint32_t)k * ns + c] = lf[k];
#pragma unroll
        for (int k = 0; k < 7; ++k) A.lgi[(uint32_t)k * ns + c] = lgo[k];
        A.lphi0[c] = lphi0;
        A.lq0[c] = lq;
    }
    if (!active) { g0 = g1 = g2 = 0.0; }
    double v[3] = {g0, g1, g2};
    block_accumulate<3>(v, A.gpar);
}

// Transposed pull: lambda of every stored population of X_s from the
// adjoints of the pulled values, then the NEQ inlet (x = 0 values derived
// from x = 1 in the fused representation).
template <typename T, typename QT, bool POROUS>
__global__ void __launch_bounds__(256) k_adj_stream(const AdjArgs<T, QT> A, typename Pop<T>::R* __restrict__ lf0,
                                                    typename Pop<T>::R* __restrict__ lg0)
{
    using R = typename Pop<T>::R;
    const StepArgs<T, QT>& a = A.a;
    const uint32_t cg = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = cg < (uint32_t)a.n;
    const uint32_t c = active ? cg : (uint32_t)a.n - 1u;
    int x, y, z;
    cell_xyz(c, a.nx, a.ny, a.div_nx, a.div_nxy, x, y, z);
    const Nbr nb(x, y, z, a.nx, a.ny, a.nz, a.px, a.py, a.pz);
    const uint32_t w = __ldg(a.cellw + c);
    const bool solid = !POROUS && (w & kSolid);
    const uint32_t ns = a.ns;
#pragma unroll
    for (int j = 0; j < 19; ++j) {
        const int o = opp19(j);
        const int ox = cx19(o), oy = cy19(o), oz = cz19(o);
        // the cell d = c + c_j pulls direction j from c (its direction-j source)
        const bool in_o = nb.xo[1 - ox] && nb.yo[1 - oy] && nb.zo[1 - oz];
        const uint32_t d = (uint32_t)(nb.xs[1 - ox] + nb.yr[1 - oy] + nb.zp[1 - oz]);
        const bool link_o = !POROUS && ((w >> o) & 1u);
        const int jx = cx19(j), jy = cy19(j), jz = cz19(j);
        const bool in_j = nb.xo[1 - jx] && nb.yo[1 - jy] && nb.zo[1 - jz];
        R v = R(0);
        if (j == 0) {
            v = A.lfi[c];
        } else {
            if (in_o && !link_o && !solid) v += A.lfi[(uint32_t)j * ns + d];
            if (!in_j && !solid) v += A.lfi[(uint32_t)j * ns + c];
            if (solid || (in_o && link_o)) v += A.lfi[(uint32_t)o * ns + c];
        }
        if (active) lf0[(uint32_t)j * ns + c] = v;
    }
    R lg[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        const int jx = cx7(j), jy = cy7(j), jz = cz7(j);
        const bool in_o = nb.xo[1 + jx] && nb.yo[1 + jy] && nb.zo[1 + jz];
        const uint32_t d = (uint32_t)(nb.xs[1 + jx] + nb.yr[1 + jy] + nb.zp[1 + jz]);
        const bool in_j = nb.xo[1 - jx] && nb.yo[1 - jy] && nb.zo[1 - jz];
        R v = R(0);
        if (j == 0) v = A.lgi[c];
        else {
            if (in_o) v += A.lgi[(uint32_t)j * ns + d];
            if (!in_j) v += A.lgi[(uint32_t)j * ns + c];
        }
        lg[j] = v;
    }
    if (active) {
#pragma unroll
        for (int k = 0; k < 7; ++k) lg0[(uint32_t)k * ns + c] = lg[k];
    }
}

// The NEQ inlet in the fused representation: the stored x = 0 populations of
// X_s are NEQ(f_s at x = 1) (src/boundary/ns/VelocityDirichletNEQ.cu:49-96),
// f_B = feq(rho_N, u_BC) + f_N - feq(rho_N, u_N).  After the gather, one warp
// per inlet row (lane k = direction k) moves the x = 0 adjoint into the x = 1
// cell through the transposed Jacobian (identity, the rho_N derivative of the
// two equilibria, the u_N derivative of feq(rho_N, u_N)) and clears x = 0.
template <typename R>
__device__ __forceinline__ R warp_sum_r(R v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T, typename QT>
__global__ void __launch_bounds__(256) k_adj_inlet(const AdjArgs<T, QT> A, typename Pop<T>::R* __restrict__ lf0)
{
    using R = typename Pop<T>::R;
    const StepArgs<T, QT>& a = A.a;
    const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);   // warp-uniform
    if (row >= a.ny * a.nz) return;
    const int lane = threadIdx.x & 31;
    const bool on = lane < 19;
    const int k = on ? lane : 0;
    const uint32_t ns = a.ns;
    const uint32_t c0 = (uint32_t)row * (uint32_t)a.nx, c1 = c0 + 1u;
    const R cx = (R)((int)((kPX >> k) & 1u) - (int)((kMX >> k) & 1u));
    const R cy = (R)((int)((kPY >> k) & 1u) - (int)((kMY >> k) & 1u));
    const R cz = (R)((int)((kPZ >> k) & 1u) - (int)((kMZ >> k) & 1u));
    const R wk = k == 0 ? R(1) / R(3) : (k < 7 ? R(1) / R(18) : R(1) / R(36));
    const R fN = on ? Pop<T>::ld(a.fA + (uint32_t)k * ns + c1, fshift<T>(k, a.f_shift)) : R(0);
    const R lB = on ? lf0[(uint32_t)k * ns + c0] : R(0);
    const R r = warp_sum_r(fN);
    const R jx = warp_sum_r(cx * fN), jy = warp_sum_r(cy * fN), jz = warp_sum_r(cz * fN);
    const R inv = (r > R(0)) ? (R(1) / r) : R(0);
    const R unx = jx * inv, uny = jy * inv, unz = jz * inv;
    const R cuB = R(3) * (cx * a.uin_x + cy * a.uin_y + cz * a.uin_z);
    const R cuN = R(3) * (cx * unx + cy * uny + cz * unz);
    const R pB = R(1) + cuB + R(0.5) * cuB * cuB - R(1.5) * (a.uin_x * a.uin_x + a.uin_y * a.uin_y + a.uin_z * a.uin_z);
    const R pN = R(1) + cuN + R(0.5) * cuN * cuN - R(1.5) * (unx * unx + uny * uny + unz * unz);
    // d feq_k(r, u_N) / d u_N = w r (3 c + 9 (c.u) c - 3 u)
    const R e = cx * unx + cy * uny + cz * unz;
    const R gx = wk * r * (R(3) * cx + R(9) * e * cx - R(3) * unx);
    const R gy = wk * r * (R(3) * cy + R(9) * e * cy - R(3) * uny);
    const R gz = wk * r * (R(3) * cz + R(9) * e * cz - R(3) * unz);
    const R s1 = warp_sum_r(lB * wk * (pB - pN));
    const R Vx = warp_sum_r(lB * gx), Vy = warp_sum_r(lB * gy), Vz = warp_sum_r(lB * gz);
    if (on) {
        R* p1 = lf0 + (uint32_t)k * ns + c1;
        *p1 += lB + s1 - ((cx - unx) * Vx + (cy - uny) * Vy + (cz - unz) * Vz) * inv;
        lf0[(uint32_t)k * ns + c0] = R(0);
    }
}

}  // namespace fm
