/*
 * fm_oracle.c -- CPU restatement of FluidMaxxer's coupled time step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline arm load the library
 * built from this file (oracle/build_oracle.py).  The product path never links
 * it and has no CPU fallback.
 *
 * Plain C (C11) + OpenMP over cells.  The arithmetic type is FMO_REAL (double
 * or float, set by the build); every expression keeps the evaluation order of
 * the reference kernel it restates, so that built with -ffp-contract=off it
 * agrees bit for bit with the reference kernels compiled for the host
 * (oracle/_ref, see test_oracle_pins.py).  Storage here is SoA, f[q*N + c].
 *
 * Parity pin: the reference ships no tests, fixtures or golden vectors.  This
 * restatement is pinned against the reference's own kernel bodies executed on
 * the host (oracle/_ref), and against the golden fixtures generated from them
 * (tests/golden/make_golden.py).
 */
#include "fm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef FMO_REAL
#define FMO_REAL double
#endif
typedef FMO_REAL real;

/* D3Q19 / D3Q7 velocity sets in the reference's order
 * (include/core/descriptors/D3Q19.hpp:14-49, include/core/descriptors/D3Q7.hpp:10-27) */
static const int CX19[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int CY19[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int CZ19[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
static const int OPP19[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
static const int CX7[7] = {0, 1, -1, 0, 0, 0, 0};
static const int CY7[7] = {0, 0, 0, 1, -1, 0, 0};
static const int CZ7[7] = {0, 0, 0, 0, 0, 1, -1};

typedef struct fmo_state {
    fmo_config cfg;
    long n;
    int nx, ny, nz, px, py, pz;
    real w19[19], w7[7];
    real *f, *fn, *g, *gn;
    real *phi, *sphi, *uxa, *uya, *uza, *tau, *q, *por;
    real *rho, *ux, *uy, *uz;
    uint8_t *solid, *region, *inlet, *outlet;
    int *bnd, *nei;
    int nbnd;
    double* c_out;
    int n_out, cap_out;
    long step;
} fmo_state;

/* Periodic wrap or out-of-domain test (src/collision/BGKCollision.cu:26-41). */
static inline int map_coord(const fmo_state* S, int* x, int* y, int* z)
{
    if (S->px) *x = (*x % S->nx + S->nx) % S->nx;
    else if (*x < 0 || *x >= S->nx) return 0;
    if (S->py) *y = (*y % S->ny + S->ny) % S->ny;
    else if (*y < 0 || *y >= S->ny) return 0;
    if (S->pz) *z = (*z % S->nz + S->nz) % S->nz;
    else if (*z < 0 || *z >= S->nz) return 0;
    return 1;
}

static inline long cell_of(const fmo_state* S, int x, int y, int z)
{
    return (long)x + (long)S->nx * ((long)y + (long)S->ny * z);
}

/* Second-order D3Q19 equilibrium as the collision kernels form it
 * (src/collision/BGKCollision.cu:166-173). */
static inline real feq19(const fmo_state* S, int k, real rho, real ux, real uy, real uz, real u2)
{
    const real eu = (real)CX19[k] * ux + (real)CY19[k] * uy + (real)CZ19[k] * uz;
    const real cu = (real)3 * eu;
    return S->w19[k] * rho * ((real)1 + cu + (real)0.5 * cu * cu - (real)1.5 * u2);
}

/* ---------------- NS collide + stream (pull) ---------------- */

/* k_bgk_stream_pull_d3q19 (src/collision/BGKCollision.cu:74-177): on-site
 * reversal in solids; pull with "keep local" outside non-periodic faces and
 * half-way bounce-back (own opposite population) when pulling from a solid. */
static void ns_bgk(fmo_state* S, real omega)
{
    const long n = S->n;
    const real* f = S->f;
    real* fn = S->fn;
    const real rho0 = (real)S->cfg.rho0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        if (S->solid[c]) {
            for (int k = 0; k < 19; ++k) fn[k * n + c] = f[OPP19[k] * n + c];
            continue;
        }
        const int z = (int)(c / ((long)S->nx * S->ny));
        const long rem = c - (long)z * S->nx * S->ny;
        const int y = (int)(rem / S->nx);
        const int x = (int)(rem - (long)y * S->nx);
        real fi[19];
        for (int k = 0; k < 19; ++k) {
            int xs = x - CX19[k], ys = y - CY19[k], zs = z - CZ19[k];
            if (!map_coord(S, &xs, &ys, &zs)) {
                fi[k] = f[k * n + c];
            } else {
                const long src = cell_of(S, xs, ys, zs);
                fi[k] = S->solid[src] ? f[OPP19[k] * n + c] : f[k * n + src];
            }
        }
        real rho = 0, ux = 0, uy = 0, uz = 0;
        for (int k = 0; k < 19; ++k) {
            const real v = fi[k];
            rho += v;
            ux += v * (real)CX19[k];
            uy += v * (real)CY19[k];
            uz += v * (real)CZ19[k];
        }
        if (!(rho > (real)0)) {
            rho = rho0;
            ux = uy = uz = (real)0;
        } else {
            const real inv = (real)1 / rho;
            ux *= inv; uy *= inv; uz *= inv;
        }
        const real u2 = ux * ux + uy * uy + uz * uz;
        for (int k = 0; k < 19; ++k) {
            const real fe = feq19(S, k, rho, ux, uy, uz, u2);
            fn[k * n + c] = fi[k] + omega * (fe - fi[k]);
        }
    }
}

/* k_porous_bgk_stream_pull_d3q19 (src/collision/PorousBGKCollision.cu:64-155):
 * pull without obstacle reflection, u = j/rho scaled by clamp(porosity,0,1). */
static void ns_porous(fmo_state* S, real omega)
{
    const long n = S->n;
    const real* f = S->f;
    real* fn = S->fn;
    const real rho0 = (real)S->cfg.rho0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        const int z = (int)(c / ((long)S->nx * S->ny));
        const long rem = c - (long)z * S->nx * S->ny;
        const int y = (int)(rem / S->nx);
        const int x = (int)(rem - (long)y * S->nx);
        real fi[19];
        for (int k = 0; k < 19; ++k) {
            int xs = x - CX19[k], ys = y - CY19[k], zs = z - CZ19[k];
            fi[k] = map_coord(S, &xs, &ys, &zs) ? f[k * n + cell_of(S, xs, ys, zs)] : f[k * n + c];
        }
        real rho = 0, jx = 0, jy = 0, jz = 0;
        for (int k = 0; k < 19; ++k) {
            const real v = fi[k];
            rho += v;
            jx += v * (real)CX19[k];
            jy += v * (real)CY19[k];
            jz += v * (real)CZ19[k];
        }
        if (!(rho > (real)0)) {
            rho = rho0;
            jx = jy = jz = (real)0;
        }
        const real inv = (real)1 / rho;
        real ux = jx * inv, uy = jy * inv, uz = jz * inv;
        real ph = S->por[c];
        if (ph < (real)0) ph = (real)0;
        if (ph > (real)1) ph = (real)1;
        ux *= ph; uy *= ph; uz *= ph;
        const real u2 = ux * ux + uy * uy + uz * uz;
        for (int k = 0; k < 19; ++k) {
            const real fe = feq19(S, k, rho, ux, uy, uz, u2);
            fn[k * n + c] = fi[k] + omega * (fe - fi[k]);
        }
    }
}

/* ---------------- NS boundaries ---------------- */

/* rho and u of one cell as the NEQ inlet forms them
 * (src/boundary/ns/VelocityDirichletNEQ.cu:13-33). */
static void moments_guarded(const real* f, long n, long c, real* rho, real* ux, real* uy, real* uz)
{
    real r = 0, jx = 0, jy = 0, jz = 0;
    for (int k = 0; k < 19; ++k) {
        const real v = f[k * n + c];
        r += v;
        jx += v * (real)CX19[k];
        jy += v * (real)CY19[k];
        jz += v * (real)CZ19[k];
    }
    *rho = r;
    const real inv = (r > (real)0) ? ((real)1 / r) : (real)0;
    *ux = jx * inv; *uy = jy * inv; *uz = jz * inv;
}

/* k_velocity_dirichlet_eq_pre_d3q19 (src/boundary/ns/VelocityDirichlet.cu:54-84). */
static void ns_inlet_eq(fmo_state* S)
{
    const long n = S->n;
    const real ux = (real)S->cfg.u_in[0], uy = (real)S->cfg.u_in[1], uz = (real)S->cfg.u_in[2];
    const real rho0 = (real)S->cfg.rho0;
    const real u2 = ux * ux + uy * uy + uz * uz;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        if (!S->inlet[c]) continue;
        for (int k = 0; k < 19; ++k) S->f[k * n + c] = feq19(S, k, rho0, ux, uy, uz, u2);
    }
}

/* k_velocity_dirichlet_neq_pre_d3q19 (src/boundary/ns/VelocityDirichletNEQ.cu:49-96):
 * f_B = feq(rho_N, u_BC) + (f_N - feq(rho_N, u_N)). */
static void ns_inlet_neq(fmo_state* S)
{
    const long n = S->n;
    const real bx = (real)S->cfg.u_in[0], by = (real)S->cfg.u_in[1], bz = (real)S->cfg.u_in[2];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < S->nbnd; ++i) {
        const long cb = S->bnd[i], cn = S->nei[i];
        real rn, ux, uy, uz;
        moments_guarded(S->f, n, cn, &rn, &ux, &uy, &uz);
        const real u2n = ux * ux + uy * uy + uz * uz;
        const real u2b = bx * bx + by * by + bz * bz;
        for (int k = 0; k < 19; ++k) {
            const real fN = S->f[k * n + cn];
            const real feqN = feq19(S, k, rn, ux, uy, uz, u2n);
            const real feqB = feq19(S, k, rn, bx, by, bz, u2b);
            S->f[k * n + cb] = feqB + (fN - feqN);
        }
    }
}

/* k_pressure_dirichlet_outlet_d3q19 (src/boundary/ns/PressureDirichlet.cu:26-96):
 * f(x) = feq(rho_out, u of f(x-1)) with the 1 + 3eu + 4.5eu^2 - 1.5u^2 form. */
static void ns_outlet_pressure(fmo_state* S)
{
    const long n = S->n;
    real* f = S->fn;
    const real ro = (real)S->cfg.rho_out;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        if (!S->outlet[c]) continue;
        const long x = c % S->nx;
        if (x <= 0) continue;
        const long cn = c - 1;
        real r = 0, ux = 0, uy = 0, uz = 0;
        for (int k = 0; k < 19; ++k) {
            const real v = f[k * n + cn];
            r += v;
            ux += v * (real)CX19[k];
            uy += v * (real)CY19[k];
            uz += v * (real)CZ19[k];
        }
        if (r > (real)0) {
            const real inv = (real)1 / r;
            ux *= inv; uy *= inv; uz *= inv;
        } else {
            ux = uy = uz = (real)0;
        }
        const real u2 = ux * ux + uy * uy + uz * uz;
        for (int k = 0; k < 19; ++k) {
            const real eu = (real)CX19[k] * ux + (real)CY19[k] * uy + (real)CZ19[k] * uz;
            f[k * n + c] = S->w19[k] * ro * ((real)1 + (real)3 * eu + (real)4.5 * eu * eu - (real)1.5 * u2);
        }
    }
}

/* k_bounceback_post_d3q19 (src/boundary/ns/BounceBack.cu:12-31): the in-place
 * loop f[k] = f[opp k] without a temporary, so both members of each pair end
 * as the value of the higher-index direction.  Restated as it behaves. */
static void ns_bounceback(fmo_state* S)
{
    const long n = S->n;
    real* f = S->fn;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        if (!S->solid[c]) continue;
        for (int k = 0; k < 19; ++k) f[k * n + c] = f[OPP19[k] * n + c];
    }
}

/* k_compute_macros_d3q19 (src/core/Macros.cu:20-61) on the current f. */
static void macros(fmo_state* S)
{
    const long n = S->n;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        real r = 0, vx = 0, vy = 0, vz = 0;
        for (int k = 0; k < 19; ++k) {
            const real v = S->f[k * n + c];
            r += v;
            vx += v * (real)CX19[k];
            vy += v * (real)CY19[k];
            vz += v * (real)CZ19[k];
        }
        const real inv = (r > (real)0) ? ((real)1 / r) : (real)0;
        S->rho[c] = r;
        S->ux[c] = vx * inv;
        S->uy[c] = vy * inv;
        S->uz[c] = vz * inv;
    }
}

/* ---------------- reaction ---------------- */

/* k_henry_ldf_source / k_langmuir_ldf_source (src/reaction/LinearLDF.cu:13-48,
 * src/reaction/LangmuirLDF.cu:7-41): c = max(phi,eps) - eps, LDF step on q,
 * S = -dq inside the region, S = 0 outside. */
static void reaction(fmo_state* S)
{
    const long n = S->n;
    const real eps = (real)S->cfg.min_conc;
    const int lin = S->cfg.isotherm == FMO_LINEAR;
    const real K = (real)S->cfg.k_henry, kA = (real)S->cfg.k_a;
    const real qm = (real)S->cfg.q_max, b = (real)S->cfg.b_langmuir, kL = (real)S->cfg.k_ldf;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        if (!S->region[c]) {
            S->sphi[c] = (real)0;
            continue;
        }
        real cc = S->phi[c];
        if (cc < eps) cc = eps;
        const real ce = cc - eps;
        real qeq, k;
        if (lin) {
            qeq = K * ce;
            k = kA;
        } else {
            const real bc = b * ce;
            qeq = qm * (bc / ((real)1 + bc));
            k = kL;
        }
        const real qi = S->q[c];
        const real dq = k * (qeq - qi);
        S->q[c] = qi + dq;
        S->sphi[c] = -dq;
    }
}

/* ---------------- AD collide + stream ---------------- */

/* k_ad_bgk_stream_pull_d3q7_source (src/collision/ADBGKCollision.cu:41-128):
 * pull with keep-local, phi = sum clamped below, geq = w phi (1 + 4 c.u),
 * g' = g + omega (geq - g) + w S, phi written back. */
static void ad_collide(fmo_state* S)
{
    const long n = S->n;
    const real* g = S->g;
    real* gn = S->gn;
    const real eps = (real)S->cfg.min_conc;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; ++c) {
        const int z = (int)(c / ((long)S->nx * S->ny));
        const long rem = c - (long)z * S->nx * S->ny;
        const int y = (int)(rem / S->nx);
        const int x = (int)(rem - (long)y * S->nx);
        const real omega = (real)1 / S->tau[c];
        const real ux = S->uxa[c], uy = S->uya[c], uz = S->uza[c];
        real gi[7];
        for (int k = 0; k < 7; ++k) {
            int xs = x - CX7[k], ys = y - CY7[k], zs = z - CZ7[k];
            gi[k] = map_coord(S, &xs, &ys, &zs) ? g[k * n + cell_of(S, xs, ys, zs)] : g[k * n + c];
        }
        real ph = 0;
        for (int k = 0; k < 7; ++k) ph += gi[k];
        if (ph < eps) ph = eps;
        const real src = S->sphi[c];
        for (int k = 0; k < 7; ++k) {
            const real eu = (real)CX7[k] * ux + (real)CY7[k] * uy + (real)CZ7[k] * uz;
            const real ge = S->w7[k] * ph * ((real)1 + (real)4 * eu);
            gn[k * n + c] = gi[k] + omega * (ge - gi[k]) + S->w7[k] * src;
        }
        S->phi[c] = ph;
    }
}

/* ---------------- AD boundaries ---------------- */

/* k_ad_dirichlet / k_ad_dirichlet_tanh_pulse_d3q7 (src/boundary/ad/ADDirichlet.cu:11-30,
 * src/boundary/ad/ADDirichletTanhPulse.cu:11-31): g = value * w on the mask. */
static void ad_fill(fmo_state* S, real* g, real value)
{
    const long n = S->n;
    for (long c = 0; c < n; ++c) {
        if (!S->inlet[c]) continue;
        for (int k = 0; k < 7; ++k) g[k * n + c] = value * S->w7[k];
    }
}

/* k_ad_neumann (src/boundary/ad/ADNeumannOutlet.cu:5-31): outlet-mask cells on
 * x = Nx-1 copy all populations from x = Nx-2.  With Nx = 1 there is no x = -1
 * neighbour (the reference reads before the array for the first row): no copy. */
static void ad_neumann(fmo_state* S)
{
    const long n = S->n;
    real* g = S->gn;
    if (S->nx < 2) return;
    for (long c = 0; c < n; ++c) {
        if (!S->outlet[c]) continue;
        if (c % S->nx != S->nx - 1) continue;
        for (int k = 0; k < 7; ++k) g[k * n + c] = g[k * n + c - 1];
    }
}

static void sample_outlet(fmo_state* S)
{
    /* OutletCSV::log (include/core/io/OutletCSV.hpp:29-58) */
    double sum = 0.0;
    long cnt = 0;
    for (long c = 0; c < S->n; ++c)
        if (S->outlet[c]) { sum += (double)S->phi[c]; ++cnt; }
    if (S->n_out == S->cap_out) {
        const int cap = S->cap_out ? 2 * S->cap_out : 256;
        double* p = (double*)realloc(S->c_out, sizeof(double) * (size_t)cap);
        if (!p) return;
        S->c_out = p;
        S->cap_out = cap;
    }
    S->c_out[S->n_out++] = cnt ? sum / (double)cnt : 0.0;
}

/* One coupled step in the order of src/main.cpp:319-357 with
 * Lattice::step (include/core/lattice/NSLattice.hpp:188-209) and
 * ADLattice::step (include/core/lattice/ADLattice.hpp:144-162). */
static void one_step(fmo_state* S)
{
    const fmo_config* c = &S->cfg;
    const long s = S->step + 1;
    real* t;

    if (c->ns_inlet == FMO_VEL_EQ) ns_inlet_eq(S);
    else if (c->ns_inlet == FMO_VEL_NEQ && S->nbnd > 0) ns_inlet_neq(S);
    {
        real tau = (real)c->tau;
        if (tau < (real)0.5001) tau = (real)0.5001;
        const real omega = (real)1 / tau;
        if (c->collision == FMO_BGK) ns_bgk(S, omega);
        else ns_porous(S, omega);
    }
    if (c->ns_outlet == FMO_PRESSURE) ns_outlet_pressure(S);
    if (c->ns_bounceback) ns_bounceback(S);
    t = S->f; S->f = S->fn; S->fn = t;

    if (c->coupling) {
        macros(S);
        memcpy(S->uxa, S->ux, sizeof(real) * (size_t)S->n);
        memcpy(S->uya, S->uy, sizeof(real) * (size_t)S->n);
        memcpy(S->uza, S->uz, sizeof(real) * (size_t)S->n);
    }
    if (c->isotherm != FMO_NONE) reaction(S);

    if (c->ad_inlet == FMO_AD_PULSE) {
        const double kk = (double)(real)c->pulse_k;
        const double pulse = 0.5 * (tanh(((double)s - (double)c->pulse_on) / kk) -
                                     tanh(((double)s - (double)c->pulse_off) / kk));
        ad_fill(S, S->g, (real)c->pulse_base + (real)pulse * (real)c->pulse_amp);
    }
    ad_collide(S);
    if (c->ad_inlet == FMO_AD_DIRICHLET) ad_fill(S, S->gn, (real)c->c_in);
    if (c->ad_outlet == FMO_AD_NEUMANN) ad_neumann(S);
    t = S->g; S->g = S->gn; S->gn = t;

    S->step = s;
    if (c->sample_every > 0 && s % c->sample_every == 0) sample_outlet(S);
}

/* VelocityDirichletNEQ's boundary list and inward neighbours
 * (include/boundary/ns/VelocityDirichletNEQ.hpp:26-107). */
static int build_neq(fmo_state* S)
{
    int minx = S->nx - 1, maxx = 0, miny = S->ny - 1, maxy = 0, minz = S->nz - 1, maxz = 0;
    int nb = 0;
    for (long c = 0; c < S->n; ++c) nb += S->inlet[c] != 0;
    S->nbnd = nb;
    if (nb == 0) return 0;
    S->bnd = (int*)malloc(sizeof(int) * (size_t)nb);
    S->nei = (int*)malloc(sizeof(int) * (size_t)nb);
    if (!S->bnd || !S->nei) return 1;
    nb = 0;
    for (long c = 0; c < S->n; ++c) {
        if (!S->inlet[c]) continue;
        S->bnd[nb++] = (int)c;
        const int x = (int)(c % S->nx), y = (int)((c / S->nx) % S->ny), z = (int)(c / ((long)S->nx * S->ny));
        if (x < minx) minx = x;
        if (x > maxx) maxx = x;
        if (y < miny) miny = y;
        if (y > maxy) maxy = y;
        if (z < minz) minz = z;
        if (z > maxz) maxz = z;
    }
    const int isx = minx == maxx, isy = miny == maxy, isz = minz == maxz;
    if (isx + isy + isz != 1) return 1;
    int dx = 0, dy = 0, dz = 0;
    if (isx) dx = minx == 0 ? 1 : (minx == S->nx - 1 ? -1 : 0);
    if (isy) dy = miny == 0 ? 1 : (miny == S->ny - 1 ? -1 : 0);
    if (isz) dz = minz == 0 ? 1 : (minz == S->nz - 1 ? -1 : 0);
    if (!dx && !dy && !dz) return 1;
    for (int i = 0; i < nb; ++i) {
        const long c = S->bnd[i];
        const int x = (int)(c % S->nx) + dx, y = (int)((c / S->nx) % S->ny) + dy;
        const int z = (int)(c / ((long)S->nx * S->ny)) + dz;
        if (x < 0 || x >= S->nx || y < 0 || y >= S->ny || z < 0 || z >= S->nz) return 1;
        S->nei[i] = (int)cell_of(S, x, y, z);
    }
    return 0;
}

static void free_state(fmo_state* S)
{
    if (!S) return;
    real* bufs[] = {S->f, S->fn, S->g, S->gn, S->phi, S->sphi, S->uxa, S->uya, S->uza,
                    S->tau, S->q, S->por, S->rho, S->ux, S->uy, S->uz};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); ++i) free(bufs[i]);
    free(S->solid); free(S->region); free(S->inlet); free(S->outlet);
    free(S->bnd); free(S->nei); free(S->c_out);
    free(S);
}

void* fmo_create(const fmo_config* cfg, const fmo_inputs* in)
{
    if (!cfg || !in || cfg->nx <= 0 || cfg->ny <= 0 || cfg->nz <= 0) return NULL;
    fmo_state* S = (fmo_state*)calloc(1, sizeof(fmo_state));
    if (!S) return NULL;
    S->cfg = *cfg;
    S->nx = cfg->nx; S->ny = cfg->ny; S->nz = cfg->nz;
    S->px = cfg->periodic_x != 0; S->py = cfg->periodic_y != 0; S->pz = cfg->periodic_z != 0;
    const long n = (long)cfg->nx * cfg->ny * cfg->nz;
    S->n = n;
    /* weights as the descriptors spell them: DATA_TYPE(1)/DATA_TYPE(k) */
    for (int k = 0; k < 19; ++k)
        S->w19[k] = k == 0 ? (real)1 / (real)3 : (k < 7 ? (real)1 / (real)18 : (real)1 / (real)36);
    for (int k = 0; k < 7; ++k) S->w7[k] = k == 0 ? (real)1 / (real)4 : (real)1 / (real)8;

    S->f = (real*)calloc((size_t)(19 * n), sizeof(real));
    S->fn = (real*)calloc((size_t)(19 * n), sizeof(real));
    S->g = (real*)calloc((size_t)(7 * n), sizeof(real));
    S->gn = (real*)calloc((size_t)(7 * n), sizeof(real));
    real** fields[] = {&S->phi, &S->sphi, &S->uxa, &S->uya, &S->uza, &S->tau, &S->q,
                       &S->por, &S->rho, &S->ux, &S->uy, &S->uz};
    int ok = S->f && S->fn && S->g && S->gn;
    for (size_t i = 0; i < sizeof(fields) / sizeof(fields[0]); ++i) {
        *fields[i] = (real*)calloc((size_t)n, sizeof(real));
        ok = ok && *fields[i];
    }
    uint8_t** masks[] = {&S->solid, &S->region, &S->inlet, &S->outlet};
    const uint8_t* src[] = {in->solid, in->region, in->inlet, in->outlet};
    for (int i = 0; i < 4; ++i) {
        *masks[i] = (uint8_t*)calloc((size_t)n, 1);
        ok = ok && *masks[i];
        if (*masks[i] && src[i]) memcpy(*masks[i], src[i], (size_t)n);
    }
    if (!ok) { free_state(S); return NULL; }
    for (long c = 0; c < n; ++c) {
        if (in->porosity) S->por[c] = (real)in->porosity[c];
        if (in->tau_ad) S->tau[c] = (real)in->tau_ad[c];
    }
    if (cfg->ns_inlet == FMO_VEL_NEQ && build_neq(S)) { free_state(S); return NULL; }

    /* initEq: k_init_eq_d3q19_1d / k_init_eq_d3q19 (f = w rho0 at u = 0) and
     * k_ad_init_eq_d3q7 (g = phi0 w); phi and S start at zero
     * (include/core/lattice/ADLattice.hpp:49-52). */
    for (int k = 0; k < 19; ++k) {
        const real v = cfg->collision == FMO_BGK
                           ? S->w19[k] * (real)cfg->rho0 * ((real)1 + (real)0 + (real)0.5 * (real)0 * (real)0 - (real)1.5 * (real)0)
                           : S->w19[k] * (real)cfg->rho0;
        for (long c = 0; c < n; ++c) S->f[k * n + c] = v;
    }
    for (int k = 0; k < 7; ++k)
        for (long c = 0; c < n; ++c) S->g[k * n + c] = (real)cfg->phi0 * S->w7[k];
    if (cfg->sample_every > 0) sample_outlet(S);
    return S;
}

int fmo_set_state(void* h, const double* f, const double* g, const double* phi, const double* q)
{
    fmo_state* S = (fmo_state*)h;
    if (!S) return 1;
    const long n = S->n;
    for (long i = 0; i < 19 * n && f; ++i) S->f[i] = (real)f[i];
    for (long i = 0; i < 7 * n && g; ++i) S->g[i] = (real)g[i];
    for (long i = 0; i < n; ++i) {
        if (phi) S->phi[i] = (real)phi[i];
        if (q) S->q[i] = (real)q[i];
    }
    return 0;
}

int fmo_step(void* h, int nsteps)
{
    fmo_state* S = (fmo_state*)h;
    if (!S || nsteps < 0) return 1;
    for (int i = 0; i < nsteps; ++i) one_step(S);
    return 0;
}

int fmo_get(void* h, fmo_outputs* o)
{
    fmo_state* S = (fmo_state*)h;
    if (!S || !o) return 1;
    const long n = S->n;
    macros(S);
    double srho = 0, sphi = 0, sq = 0, sout = 0;
    long nout = 0;
    for (long c = 0; c < n; ++c) {
        if (o->rho) o->rho[c] = (double)S->rho[c];
        if (o->ux) o->ux[c] = (double)S->ux[c];
        if (o->uy) o->uy[c] = (double)S->uy[c];
        if (o->uz) o->uz[c] = (double)S->uz[c];
        if (o->phi) o->phi[c] = (double)S->phi[c];
        if (o->q) o->q[c] = (double)S->q[c];
        if (o->sphi) o->sphi[c] = (double)S->sphi[c];
        srho += (double)S->rho[c];
        sphi += (double)S->phi[c];
        sq += (double)S->q[c];
        if (S->outlet[c]) { sout += (double)S->phi[c]; ++nout; }
    }
    for (long i = 0; i < 19 * n && o->f; ++i) o->f[i] = (double)S->f[i];
    for (long i = 0; i < 7 * n && o->g; ++i) o->g[i] = (double)S->g[i];
    o->sums[0] = srho; o->sums[1] = sphi; o->sums[2] = sq;
    o->sums[3] = nout ? sout / (double)nout : 0.0;
    o->n_samples = S->n_out;
    if (o->c_out)
        for (int i = 0; i < S->n_out && i < o->c_out_cap; ++i) o->c_out[i] = S->c_out[i];
    return 0;
}

int fmo_precision_bytes(void) { return (int)sizeof(real); }

void fmo_destroy(void* h) { free_state((fmo_state*)h); }
