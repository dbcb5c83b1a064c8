/*
 * Host driver for the reference's OWN kernel bodies (TEST INFRASTRUCTURE ONLY).
 *
 * oracle/build_oracle.py compiles each reference kernel file, cut before its
 * class glue, through oracle/shim/fm_ref_shim.h and links the objects with this
 * file into oracle/_ref/libfmref_{f64,f32}.so.  This file is project code: it
 * replays, with OpenMP over cells in place of a CUDA grid, the glue the
 * reference wraps around those kernels:
 *   - the lattice set-up and initEquilibrium of
 *     include/core/lattice/NSLattice.hpp:18-55,177-185 and
 *     include/core/lattice/ADLattice.hpp:17-56,134-141;
 *   - the NS step of include/core/lattice/NSLattice.hpp:188-209 and the AD step
 *     of include/core/lattice/ADLattice.hpp:144-162;
 *   - the coupled time loop of src/main.cpp:319-357 (coupling, zeroSource,
 *     computeSource with region mask, AD step, OutletCSV sample);
 *   - the boundary-list set-up of include/boundary/ns/VelocityDirichletNEQ.hpp:26-107
 *     and the pulse value of src/boundary/ad/ADDirichletTanhPulse.cu:66-100.
 * Every launch is 256 threads per block, as in the reference glue, with one
 * host iteration per in-range CUDA thread.
 */
#include "fm_oracle.h"
#include "shim/fm_ref_shim.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <stdexcept>
#include <vector>

#ifndef FM_REF_REAL
#define FM_REF_REAL double
#endif
typedef FM_REF_REAL real;

thread_local fm_shim_dim3 fm_shim_blockIdx;
thread_local fm_shim_dim3 fm_shim_blockDim;
thread_local fm_shim_dim3 fm_shim_threadIdx;

/* ---- the reference kernels (signatures as declared in their .cu files) ---- */
void uploadD3Q19Constants();
void uploadD3Q7Constants();
void k_init_eq_d3q19_1d(real* f, int nCells, real rho0);
void k_bgk_stream_pull_d3q19(const real* f, real* f_new, const std::uint8_t* obstacle,
                             int Nx, int Ny, int Nz, bool px, bool py, bool pz,
                             real omega, real rho0_fallback);
void k_init_eq_d3q19(real* f, int nCells, real rho0);
void k_porous_bgk_stream_pull_d3q19(const real* f, real* f_new, const real* porosity,
                                    int Nx, int Ny, int Nz, bool px, bool py, bool pz,
                                    real omega, real rho0_fallback);
void k_ad_init_eq_d3q7(real* g, int nCells, real phi0);
void k_ad_bgk_stream_pull_d3q7_source(const real* g, real* g_new, real* phi_out,
                                      const real* tauField, const real* ux_adv,
                                      const real* uy_adv, const real* uz_adv,
                                      const real* Sphi, int Nx, int Ny, int Nz,
                                      bool px, bool py, bool pz, real phiMinClamp);
void k_compute_macros_d3q19(const real* f, real* rho, real* ux, real* uy, real* uz,
                            int Nx, int Ny, int Nz);
void k_pressure_dirichlet_outlet_d3q19(real* f, const std::uint8_t* mask,
                                       int Nx, int Ny, int Nz, real rho_out);
void k_velocity_dirichlet_neq_pre_d3q19(real* f, const int* bndIdx, const int* neiIdx,
                                        int nBnd, real ux, real uy, real uz);
void k_velocity_dirichlet_eq_pre_d3q19(real* f, const std::uint8_t* mask, int nCells,
                                       real rho0, real ux, real uy, real uz);
void k_bounceback_post_d3q19(real* f_new, const std::uint8_t* mask, int nCells);
void k_ad_dirichlet(real* g_new, const std::uint8_t* mask, int n, real phi);
void k_ad_neumann(real* g_new, int Nx, int Ny, int Nz, const std::uint8_t* mask);
void k_ad_dirichlet_tanh_pulse_d3q7(real* g, const std::uint8_t* mask, int nCells, real phiIn);
void k_henry_ldf_source(int nCells, const std::uint8_t* region, const real* phi,
                        real* Sphi, real* q, real K, real kLDF, real phiMinClamp);
void k_langmuir_ldf_source(int nCells, const std::uint8_t* region, const real* phi,
                           real* Sphi, real* q, real qMax, real b, real kLDF,
                           real phiMinClamp);

namespace {

/* one host iteration per in-range thread of a <<<ceil(n/256), 256>>> launch */
template <class Body>
void launch1d(long n, Body body)
{
#pragma omp parallel for schedule(static)
    for (long t = 0; t < n; ++t) {
        fm_shim_blockDim = {256u, 1u, 1u};
        fm_shim_blockIdx = {unsigned(t / 256), 0u, 0u};
        fm_shim_threadIdx = {unsigned(t % 256), 0u, 0u};
        body();
    }
}

struct RefLattice {
    fmo_config cfg{};
    long n = 0;
    int nx = 0, ny = 0, nz = 0;
    bool px = false, py = false, pz = false;
    std::vector<real> f, fnew, g, gnew;
    std::vector<real> phi, sphi, uxa, uya, uza, tau, q, porosity;
    std::vector<real> rho, ux, uy, uz;
    std::vector<std::uint8_t> solid, region, inlet, outlet;
    std::vector<int> bnd, nei;
    std::vector<double> c_out;
    long step = 0;
};

/* VelocityDirichletNEQ's host set-up: compress the mask, infer the single
 * axis-aligned boundary plane and the inward neighbour of each boundary cell
 * (include/boundary/ns/VelocityDirichletNEQ.hpp:26-107). */
void build_neq_lists(RefLattice& L)
{
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    for (long i = 0; i < L.n; ++i)
        if (L.inlet[i]) L.bnd.push_back(int(i));
    if (L.bnd.empty()) return;
    int minx = nx - 1, maxx = 0, miny = ny - 1, maxy = 0, minz = nz - 1, maxz = 0;
    for (int c : L.bnd) {
        const int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        minx = std::min(minx, x); maxx = std::max(maxx, x);
        miny = std::min(miny, y); maxy = std::max(maxy, y);
        minz = std::min(minz, z); maxz = std::max(maxz, z);
    }
    const bool isx = minx == maxx, isy = miny == maxy, isz = minz == maxz;
    if (int(isx) + int(isy) + int(isz) != 1)
        throw std::runtime_error("NEQ inlet mask is not exactly one axis-aligned plane");
    int dx = 0, dy = 0, dz = 0;
    if (isx) dx = (minx == 0) ? 1 : (minx == nx - 1 ? -1 : 0);
    if (isy) dy = (miny == 0) ? 1 : (miny == ny - 1 ? -1 : 0);
    if (isz) dz = (minz == 0) ? 1 : (minz == nz - 1 ? -1 : 0);
    if (dx == 0 && dy == 0 && dz == 0)
        throw std::runtime_error("NEQ inlet plane is not on the domain boundary");
    for (int c : L.bnd) {
        const int x = c % nx + dx, y = (c / nx) % ny + dy, z = c / (nx * ny) + dz;
        if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz)
            throw std::runtime_error("NEQ inferred neighbour out of domain");
        L.nei.push_back(x + y * nx + z * nx * ny);
    }
}

void compute_macros(RefLattice& L)
{
    const int nx = L.nx, ny = L.ny, nz = L.nz;
#pragma omp parallel for schedule(static) collapse(2)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                fm_shim_blockDim = {1u, 1u, 1u};
                fm_shim_threadIdx = {0u, 0u, 0u};
                fm_shim_blockIdx = {unsigned(x), unsigned(y), unsigned(z)};
                k_compute_macros_d3q19(L.f.data(), L.rho.data(), L.ux.data(), L.uy.data(),
                                       L.uz.data(), nx, ny, nz);
            }
}

void sample_outlet(RefLattice& L)
{
    /* OutletCSV::log: mean of phi over the outlet mask (include/core/io/OutletCSV.hpp:29-58) */
    double sum = 0.0;
    long cnt = 0;
    for (long i = 0; i < L.n; ++i)
        if (L.outlet[i]) { sum += double(L.phi[i]); ++cnt; }
    L.c_out.push_back(cnt ? sum / double(cnt) : 0.0);
}

void one_step(RefLattice& L)
{
    const fmo_config& c = L.cfg;
    const int n = int(L.n);
    const long s = L.step + 1;
    const real u0x = real(c.u_in[0]), u0y = real(c.u_in[1]), u0z = real(c.u_in[2]);

    /* ---- Lattice<D3Q19>::step (NSLattice.hpp:188-209) ---- */
    if (c.ns_inlet == FMO_VEL_EQ) {
        real* f = L.f.data();
        const std::uint8_t* m = L.inlet.data();
        const real rho0 = real(c.rho0);
        launch1d(n, [&] { k_velocity_dirichlet_eq_pre_d3q19(f, m, n, rho0, u0x, u0y, u0z); });
    } else if (c.ns_inlet == FMO_VEL_NEQ && !L.bnd.empty()) {
        real* f = L.f.data();
        const int nb = int(L.bnd.size());
        const int* b = L.bnd.data();
        const int* e = L.nei.data();
        launch1d(nb, [&] { k_velocity_dirichlet_neq_pre_d3q19(f, b, e, nb, u0x, u0y, u0z); });
    }
    std::memcpy(L.fnew.data(), L.f.data(), L.f.size() * sizeof(real)); /* NSLattice.hpp:198 */
    {
        real tau = real(c.tau);
        if (tau < real(0.5001)) tau = real(0.5001);
        const real omega = real(1) / tau;
        const real* f = L.f.data();
        real* fn = L.fnew.data();
        const real rho0 = real(c.rho0);
        if (c.collision == FMO_BGK) {
            const std::uint8_t* ob = L.solid.data();
            launch1d(n, [&] {
                k_bgk_stream_pull_d3q19(f, fn, ob, L.nx, L.ny, L.nz, L.px, L.py, L.pz, omega, rho0);
            });
        } else {
            const real* por = L.porosity.data();
            launch1d(n, [&] {
                k_porous_bgk_stream_pull_d3q19(f, fn, por, L.nx, L.ny, L.nz, L.px, L.py, L.pz,
                                               omega, rho0);
            });
        }
    }
    if (c.ns_outlet == FMO_PRESSURE) {
        real* fn = L.fnew.data();
        const std::uint8_t* m = L.outlet.data();
        const real ro = real(c.rho_out);
        launch1d(n, [&] { k_pressure_dirichlet_outlet_d3q19(fn, m, L.nx, L.ny, L.nz, ro); });
    }
    if (c.ns_bounceback) {
        real* fn = L.fnew.data();
        const std::uint8_t* m = L.solid.data();
        launch1d(n, [&] { k_bounceback_post_d3q19(fn, m, n); });
    }
    std::swap(L.f, L.fnew);

    /* ---- coupling (main.cpp:322-326) ---- */
    if (c.coupling) {
        compute_macros(L);
        L.uxa = L.ux; L.uya = L.uy; L.uza = L.uz;
    }

    /* ---- adsorption source (main.cpp:328-335) ---- */
    if (c.isotherm != FMO_NONE) {
        std::fill(L.sphi.begin(), L.sphi.end(), real(0));
        const std::uint8_t* rg = L.region.data();
        const real* ph = L.phi.data();
        real* sp = L.sphi.data();
        real* qq = L.q.data();
        const real mc = real(c.min_conc);
        if (c.isotherm == FMO_LINEAR) {
            const real K = real(c.k_henry), k = real(c.k_a);
            launch1d(n, [&] { k_henry_ldf_source(n, rg, ph, sp, qq, K, k, mc); });
        } else {
            const real qm = real(c.q_max), b = real(c.b_langmuir), k = real(c.k_ldf);
            launch1d(n, [&] { k_langmuir_ldf_source(n, rg, ph, sp, qq, qm, b, k, mc); });
        }
    }

    /* ---- ADLattice<D3Q7>::step (ADLattice.hpp:144-162) ---- */
    if (c.ad_inlet == FMO_AD_PULSE) {
        const double tt = double(s), ton = double(c.pulse_on), toff = double(c.pulse_off);
        const double kk = double(real(c.pulse_k));
        const double pulse = 0.5 * (std::tanh((tt - ton) / kk) - std::tanh((tt - toff) / kk));
        const real phiIn = real(c.pulse_base) + static_cast<real>(pulse) * real(c.pulse_amp);
        real* g = L.g.data();
        const std::uint8_t* m = L.inlet.data();
        launch1d(n, [&] { k_ad_dirichlet_tanh_pulse_d3q7(g, m, n, phiIn); });
    }
    {
        const real* g = L.g.data();
        real* gn = L.gnew.data();
        real* ph = L.phi.data();
        const real* ta = L.tau.data();
        const real *ax = L.uxa.data(), *ay = L.uya.data(), *az = L.uza.data();
        const real* sp = L.sphi.data();
        const real mc = real(c.min_conc);
        launch1d(n, [&] {
            k_ad_bgk_stream_pull_d3q7_source(g, gn, ph, ta, ax, ay, az, sp, L.nx, L.ny, L.nz,
                                             L.px, L.py, L.pz, mc);
        });
    }
    if (c.ad_inlet == FMO_AD_DIRICHLET) {
        real* gn = L.gnew.data();
        const std::uint8_t* m = L.inlet.data();
        const real ci = real(c.c_in);
        launch1d(n, [&] { k_ad_dirichlet(gn, m, n, ci); });
    }
    if (c.ad_outlet == FMO_AD_NEUMANN) {
        real* gn = L.gnew.data();
        const std::uint8_t* m = L.outlet.data();
        launch1d(n, [&] { k_ad_neumann(gn, L.nx, L.ny, L.nz, m); });
    }
    std::swap(L.g, L.gnew);

    L.step = s;
    if (c.sample_every > 0 && s % c.sample_every == 0) sample_outlet(L);
}

}  // namespace

extern "C" {

void* fmo_ref_create(const fmo_config* cfg, const fmo_inputs* in)
{
    if (!cfg || !in || cfg->nx <= 0 || cfg->ny <= 0 || cfg->nz <= 0) return nullptr;
    RefLattice* L = new (std::nothrow) RefLattice();
    if (!L) return nullptr;
    try {
        L->cfg = *cfg;
        L->nx = cfg->nx; L->ny = cfg->ny; L->nz = cfg->nz;
        L->px = cfg->periodic_x != 0; L->py = cfg->periodic_y != 0; L->pz = cfg->periodic_z != 0;
        L->n = long(cfg->nx) * cfg->ny * cfg->nz;
        const long n = L->n;
        uploadD3Q19Constants();
        uploadD3Q7Constants();
        L->f.assign(19 * n, real(0)); L->fnew.assign(19 * n, real(0));
        L->g.assign(7 * n, real(0)); L->gnew.assign(7 * n, real(0));
        L->phi.assign(n, real(0)); L->sphi.assign(n, real(0));
        L->uxa.assign(n, real(0)); L->uya.assign(n, real(0)); L->uza.assign(n, real(0));
        L->q.assign(n, real(0)); L->porosity.assign(n, real(0)); L->tau.assign(n, real(0));
        L->rho.assign(n, real(0)); L->ux.assign(n, real(0)); L->uy.assign(n, real(0));
        L->uz.assign(n, real(0));
        L->solid.assign(n, 0); L->region.assign(n, 0); L->inlet.assign(n, 0); L->outlet.assign(n, 0);
        for (long i = 0; i < n; ++i) {
            if (in->solid) L->solid[i] = in->solid[i];
            if (in->region) L->region[i] = in->region[i];
            if (in->inlet) L->inlet[i] = in->inlet[i];
            if (in->outlet) L->outlet[i] = in->outlet[i];
            if (in->porosity) L->porosity[i] = real(in->porosity[i]);
            if (in->tau_ad) L->tau[i] = real(in->tau_ad[i]);
        }
        if (cfg->ns_inlet == FMO_VEL_NEQ) build_neq_lists(*L);

        /* initEquilibrium of both lattices */
        real* f = L->f.data();
        const int ni = int(n);
        const real rho0 = real(cfg->rho0);
        if (cfg->collision == FMO_BGK)
            launch1d(n, [&] { k_init_eq_d3q19_1d(f, ni, rho0); });
        else
            launch1d(n, [&] { k_init_eq_d3q19(f, ni, rho0); });
        L->fnew = L->f;
        real* g = L->g.data();
        const real phi0 = real(cfg->phi0);
        launch1d(n, [&] { k_ad_init_eq_d3q7(g, ni, phi0); });
        L->gnew = L->g;
        if (cfg->sample_every > 0) sample_outlet(*L);
    } catch (...) {
        delete L;
        return nullptr;
    }
    return L;
}

int fmo_ref_set_state(void* h, const double* f, const double* g, const double* phi,
                      const double* q)
{
    RefLattice* L = static_cast<RefLattice*>(h);
    if (!L) return 1;
    const long n = L->n;
    for (long c = 0; c < n; ++c) {
        if (f) for (int k = 0; k < 19; ++k) L->f[c * 19 + k] = real(f[k * n + c]);
        if (g) for (int k = 0; k < 7; ++k) L->g[c * 7 + k] = real(g[k * n + c]);
        if (phi) L->phi[c] = real(phi[c]);
        if (q) L->q[c] = real(q[c]);
    }
    return 0;
}

int fmo_ref_step(void* h, int nsteps)
{
    RefLattice* L = static_cast<RefLattice*>(h);
    if (!L || nsteps < 0) return 1;
    try {
        for (int i = 0; i < nsteps; ++i) one_step(*L);
    } catch (...) {
        return 2;
    }
    return 0;
}

int fmo_ref_get(void* h, fmo_outputs* o)
{
    RefLattice* L = static_cast<RefLattice*>(h);
    if (!L || !o) return 1;
    const long n = L->n;
    compute_macros(*L);
    double srho = 0, sphi = 0, sq = 0, sout = 0;
    long nout = 0;
    for (long c = 0; c < n; ++c) {
        if (o->rho) o->rho[c] = double(L->rho[c]);
        if (o->ux) o->ux[c] = double(L->ux[c]);
        if (o->uy) o->uy[c] = double(L->uy[c]);
        if (o->uz) o->uz[c] = double(L->uz[c]);
        if (o->phi) o->phi[c] = double(L->phi[c]);
        if (o->q) o->q[c] = double(L->q[c]);
        if (o->sphi) o->sphi[c] = double(L->sphi[c]);
        if (o->f) for (int k = 0; k < 19; ++k) o->f[k * n + c] = double(L->f[c * 19 + k]);
        if (o->g) for (int k = 0; k < 7; ++k) o->g[k * n + c] = double(L->g[c * 7 + k]);
        srho += double(L->rho[c]);
        sphi += double(L->phi[c]);
        sq += double(L->q[c]);
        if (L->outlet[c]) { sout += double(L->phi[c]); ++nout; }
    }
    o->sums[0] = srho; o->sums[1] = sphi; o->sums[2] = sq;
    o->sums[3] = nout ? sout / double(nout) : 0.0;
    const int ns = int(L->c_out.size());
    o->n_samples = ns;
    if (o->c_out)
        for (int i = 0; i < ns && i < o->c_out_cap; ++i) o->c_out[i] = L->c_out[i];
    return 0;
}

int fmo_ref_precision_bytes(void) { return int(sizeof(real)); }
int fmo_ref_threads(void) { return omp_get_max_threads(); }
void fmo_ref_destroy(void* h) { delete static_cast<RefLattice*>(h); }

}  // extern "C"
