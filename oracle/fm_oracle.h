/*
 * Oracle interface (TEST INFRASTRUCTURE ONLY -- never on the product path).
 *
 * Two CPU implementations of FluidMaxxer's coupled time step share this
 * interface:
 *   fmo_*      oracle/fm_oracle.c: a plain-C restatement of the reference
 *              algorithm (FP64 or FP32 by build), each function citing the
 *              reference file:line it follows;
 *   fmo_ref_*  oracle/ref_driver.cpp linked with the reference's OWN kernel
 *              bodies compiled for the host (oracle/build_oracle.py), replaying
 *              the reference loop order of src/main.cpp:319-357.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm may load
 * the libraries built from these files.
 *
 * Cell index c = x + nx*(y + ny*z) (include/core/lattice/NSLattice.hpp:83-86).
 * Population arrays exchanged through this interface are SoA: f[q*N + c],
 * g[q*N + c]; the D3Q19/D3Q7 direction order is the reference's
 * (include/core/descriptors/D3Q19.hpp:14-49, D3Q7.hpp:10-27).
 */
#ifndef FM_ORACLE_H
#define FM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { FMO_NONE = 0 };
/* NS collision operator (src/collision/BGKCollision.cu, PorousBGKCollision.cu) */
enum { FMO_BGK = 0, FMO_POROUS = 1 };
/* NS pre-collision inlet (src/boundary/ns/VelocityDirichlet.cu:54-84,
 * src/boundary/ns/VelocityDirichletNEQ.cu:49-96) */
enum { FMO_VEL_EQ = 1, FMO_VEL_NEQ = 2 };
/* NS post-stream outlet (src/boundary/ns/PressureDirichlet.cu:26-96) */
enum { FMO_PRESSURE = 1 };
/* AD inlet: post-stream Dirichlet (src/boundary/ad/ADDirichlet.cu:11-30) or the
 * pre-collision tanh pulse (src/boundary/ad/ADDirichletTanhPulse.cu:11-31) */
enum { FMO_AD_DIRICHLET = 1, FMO_AD_PULSE = 2 };
/* AD outlet (src/boundary/ad/ADNeumannOutlet.cu:5-31) */
enum { FMO_AD_NEUMANN = 1 };
/* isotherm (src/reaction/LinearLDF.cu:13-48, src/reaction/LangmuirLDF.cu:7-41) */
enum { FMO_LINEAR = 1, FMO_LANGMUIR = 2 };

typedef struct fmo_config {
    int nx, ny, nz;
    int periodic_x, periodic_y, periodic_z;
    int collision;            /* FMO_BGK | FMO_POROUS */
    double rho0, tau;         /* LBMParams::rho0, tau */
    double phi0, min_conc;    /* LBMParams::phi0, minConcentration */
    int ns_inlet;             /* FMO_NONE | FMO_VEL_EQ | FMO_VEL_NEQ */
    double u_in[3];
    int ns_outlet;            /* FMO_NONE | FMO_PRESSURE */
    double rho_out;
    int ns_bounceback;        /* 1: BounceBack BC on the solid mask, post-stream */
    int ad_inlet;             /* FMO_NONE | FMO_AD_DIRICHLET | FMO_AD_PULSE */
    double c_in;              /* ADDirichlet phi */
    double pulse_base, pulse_amp, pulse_k;
    int pulse_on, pulse_off;
    int ad_outlet;            /* FMO_NONE | FMO_AD_NEUMANN */
    int coupling;             /* 1: u_adv = NS velocity every step (--coupling) */
    int isotherm;             /* FMO_NONE | FMO_LINEAR | FMO_LANGMUIR (--adsorb) */
    double k_henry, k_a;      /* LinearLDF: KHenry, kA */
    double q_max, b_langmuir, k_ldf; /* LangmuirLDF: qMax, bLangmuir, kLDF */
    int sample_every;         /* breakthrough sample period (OutletCSV::log), 0 = off */
} fmo_config;

typedef struct fmo_inputs {
    const uint8_t* solid;     /* N: obstacle mask (NSLattice::setObstacleMask) */
    const double* porosity;   /* N or NULL: porosity field (FMO_POROUS) */
    const double* tau_ad;     /* N: AD relaxation time field (ADLattice::setTauField) */
    const uint8_t* region;    /* N: adsorption region mask (computeSource's region) */
    const uint8_t* inlet;     /* N: inlet mask (buildXPlaneMask(...,0)) */
    const uint8_t* outlet;    /* N: outlet mask (buildXPlaneMask(...,Nx-1)) */
} fmo_inputs;

/* Final-state view; any pointer may be NULL.  rho/u are the moments of the
 * current f exactly as Lattice::computeMacroscopicDevice forms them
 * (src/core/Macros.cu:20-61). */
typedef struct fmo_outputs {
    double *rho, *ux, *uy, *uz;
    double *phi, *q, *sphi;
    double *f, *g;            /* SoA 19N / 7N */
    double *c_out;            /* breakthrough samples (capacity c_out_cap) */
    int c_out_cap;
    int n_samples;            /* written: samples taken so far */
    double sums[4];           /* written: sum rho, sum phi, sum q, outlet mean phi */
} fmo_outputs;

/* restatement (fm_oracle.c) */
void* fmo_create(const fmo_config* cfg, const fmo_inputs* in);
int   fmo_set_state(void* h, const double* f, const double* g, const double* phi,
                    const double* q);
int   fmo_step(void* h, int nsteps);
int   fmo_get(void* h, fmo_outputs* out);
int   fmo_precision_bytes(void);
void  fmo_destroy(void* h);

/* reference kernels on the host (ref_driver.cpp + oracle/_ref) */
void* fmo_ref_create(const fmo_config* cfg, const fmo_inputs* in);
int   fmo_ref_set_state(void* h, const double* f, const double* g,
                        const double* phi, const double* q);
int   fmo_ref_step(void* h, int nsteps);
int   fmo_ref_get(void* h, fmo_outputs* out);
int   fmo_ref_precision_bytes(void);
int   fmo_ref_threads(void);
void  fmo_ref_destroy(void* h);

#ifdef __cplusplus
}
#endif
#endif
