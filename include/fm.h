/*
 * fm.h -- C ABI of the B200 coupled lattice-Boltzmann step (libfm.so).
 *
 * One fm_lattice is the reference's pair of lattices -- Lattice<D3Q19>
 * (include/core/lattice/NSLattice.hpp:14-264) and ADLattice<D3Q7>
 * (include/core/lattice/ADLattice.hpp:17-189) -- together with the operators,
 * boundary conditions, adsorbed field and isotherm that src/main.cpp:101-303
 * attaches to them.  fm_step advances the coupled time step of
 * src/main.cpp:319-357 (NS step, velocity coupling, LDF source, AD step) on
 * one B200 with fused sm_100a kernels.
 *
 * Conventions
 *   - Every function returns FM_OK (0) or a negative FM_ERR_* code; the
 *     message is available from fm_last_error() on the calling thread.  The
 *     reference throws std::runtime_error at the same points.
 *   - Cell index c = x + nx*(y + ny*z) (NSLattice.hpp:83-86).  Byte masks are
 *     uint8 per cell, nonzero = set.  Host arrays are passed as plain pointers
 *     with their element count.
 *   - Work is queued on the lattice's CUDA stream and is asynchronous;
 *     getters synchronise that stream.
 *   - A lattice is not thread-safe (as the reference: one host thread).
 */
#ifndef FM_H
#define FM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FM_ABI_VERSION 1

enum fm_status {
    FM_OK = 0,
    FM_ERR_ARG = -1,        /* invalid argument / size mismatch           */
    FM_ERR_STATE = -2,      /* call out of order (e.g. no collision set)  */
    FM_ERR_CUDA = -3,       /* CUDA runtime error                         */
    FM_ERR_UNSUPPORTED = -4,/* valid for the reference, not supported here */
    FM_ERR_NOMEM = -5,
    FM_ERR_DEVICE = -6      /* a device-side wait gave up (see fm_step_status) */
};

/* population storage formats */
enum fm_precision {
    FM_F32 = 0,             /* FP32 populations                              */
    FM_F16_SHIFTED = 1,     /* FP16 storage of f_i - w_i rho0, g_i - w_i c_s */
    FM_BF16_SHIFTED = 2,    /* BF16 storage of the same shifted values       */
    FM_F64 = 3,             /* FP64 populations and arithmetic (the reference's
                               DATA_TYPE as shipped)                          */
    FM_F16_FIXED_AD = 4     /* D3Q19 as FM_F16_SHIFTED; D3Q7 as unsigned 16-bit
                               fixed point over w_i [-0.5, 2.0] (step 3.8e-5 w_i) */
};

enum fm_collision { FM_COLL_BGK = 0, FM_COLL_POROUS = 1 };
enum fm_isotherm { FM_ISO_NONE = 0, FM_ISO_LINEAR = 1, FM_ISO_LANGMUIR = 2 };
enum fm_field {
    FM_FIELD_RHO = 0, FM_FIELD_UX = 1, FM_FIELD_UY = 2, FM_FIELD_UZ = 3,
    FM_FIELD_C = 4,   /* AD scalar phi (ADLattice d_phi) */
    FM_FIELD_Q = 5    /* adsorbed loading (AdsorbedField d_q) */
};

/* LBMParams (include/core/Params.hpp:6-37). */
typedef struct fm_params {
    int nx, ny, nz;
    double rho0;
    double tau;
    double tau_ad;            /* AD relaxation time used until fm_set_tau_field */
    double phi0;
    double min_concentration; /* reference default 1e-8 */
    int periodic_x, periodic_y, periodic_z;
} fm_params;

typedef struct fm_lattice fm_lattice;

/* ---- errors / version ---------------------------------------------------- */
const char* fm_last_error(void);
int fm_abi_version(void);

/* ---- lattice lifetime ----------------------------------------------------
 * fm_lattice_create replaces the constructors Lattice<D3Q19>(p)
 * (NSLattice.hpp:18-55), ADLattice<D3Q7>(p) (ADLattice.hpp:20-56) and
 * AdsorbedField(p) (include/reaction/AdsorbedField.hpp:10-21): device
 * buffers are allocated and zeroed (phi = S = u_adv = q = 0).  `stream` is a
 * cudaStream_t, or NULL for a stream owned by the lattice.  Device memory
 * comes from the library's own stream-ordered pool (see fm_trim_memory);
 * fm_lattice_destroy frees it in the order of the lattice's stream.  A lattice
 * that a batch holds cannot be destroyed (FM_ERR_STATE): destroy the batch
 * first. */
int fm_lattice_create(const fm_params* p, int precision, void* stream, fm_lattice** out);
int fm_lattice_destroy(fm_lattice* lat);

/* ---- geometry and fields -------------------------------------------------- */
/* Lattice::setObstacleMask (NSLattice.hpp:151-156); n must equal nx*ny*nz. */
int fm_set_obstacle_mask(fm_lattice* lat, const uint8_t* mask, size_t n);
/* Same, bit-packed: bit (c & 31) of word c >> 5, nwords = ceil(n/32). */
int fm_set_obstacle_bits(fm_lattice* lat, const uint32_t* bits, size_t nwords);
/* Lattice::setPorosityFromMask (NSLattice.hpp:88-114). */
int fm_set_porosity_from_mask(fm_lattice* lat, const uint8_t* mask, size_t n,
                              double phi_masked, double phi_else);
/* Direct upload of the porosity field (Lattice::d_porosity_ptr, NSLattice.hpp:144). */
int fm_set_porosity(fm_lattice* lat, const double* porosity, size_t n);
/* ADLattice::setTauField (ADLattice.hpp:95-100). */
int fm_set_tau_field(fm_lattice* lat, const double* tau, size_t n);
/* ADUnitConverter<D3Q7>::buildTauField (include/core/io/ADUnitConverter.hpp:30-104),
 * host only, no lattice needed: tau = D dt / dx^2 / cs2 + 1/2 (cs2 = 1/4) for the
 * fluid and the solid diffusivity, tau_out[c] = mask[c] ? tau(D_solid) : tau(D_fluid),
 * n = nx*ny*nz values in double (fm_set_tau_field rounds them to the storage's
 * arithmetic type, as the reference's static_cast<DATA_TYPE> does).  Errors as the
 * reference's constructor and builder throw them: nx < 2, dx_phys <= 0,
 * dt_phys <= 0, a tau <= 1/2 ("unstable") and a mask of the wrong size. */
int fm_build_tau_field(int nx, int ny, int nz, double dx_phys, double dt_phys, const uint8_t* mask, size_t n,
                       double d_fluid_phys, double d_solid_phys, double* tau_out);

/* ---- operators -------------------------------------------------------------
 * Lattice::setCollisionOperator (NSLattice.hpp:159-162) with BGKCollision
 * (include/collision/BGKCollision.hpp) or PorousBGKCollision
 * (include/collision/PorousBGKCollision.hpp).  The AD operator is always
 * ADBGKCollision<D3Q7> (include/collision/ADBGKCollision.hpp). */
int fm_set_collision(fm_lattice* lat, int collision);
/* main.cpp's --coupling: u_adv <- NS velocity after every NS step
 * (Lattice::computeMacroscopicDevice + ADLattice::setAdvectionFromFluidDevice,
 * src/main.cpp:322-326).  Default on. */
int fm_set_coupling(fm_lattice* lat, int enabled);
/* LinearLDF<D3Q7>::computeSource (include/reaction/LinearLDF.hpp:20-49):
 * Henry constant K and LDF rate k per step; region = adsorption mask. */
int fm_set_isotherm_linear(fm_lattice* lat, const uint8_t* region, size_t n,
                           double k_henry, double k_ldf);
/* LangmuirLDF<D3Q7>::computeSource (include/reaction/LangmuirLDF.hpp:16-37). */
int fm_set_isotherm_langmuir(fm_lattice* lat, const uint8_t* region, size_t n,
                             double q_max, double b, double k_ldf);
int fm_clear_isotherm(fm_lattice* lat);

/* ---- boundary conditions (applied in the order added, per lattice) ------- */
/* VelocityDirichletEq (include/boundary/ns/VelocityDirichlet.hpp:12-36). */
int fm_add_ns_velocity_eq(fm_lattice* lat, const uint8_t* mask, size_t n,
                          double ux, double uy, double uz);
/* VelocityDirichletNEQ (include/boundary/ns/VelocityDirichletNEQ.hpp:17-107);
 * the mask must be one axis-aligned plane on the domain boundary. */
int fm_add_ns_velocity_neq(fm_lattice* lat, const uint8_t* mask, size_t n,
                           double ux, double uy, double uz);
/* PressureDirichlet (include/boundary/ns/PressureDirichlet.hpp:13-28). */
int fm_add_ns_pressure(fm_lattice* lat, const uint8_t* mask, size_t n, double rho_out);
/* BounceBack (include/boundary/ns/BounceBack.hpp:11-44), as the reference
 * kernel behaves (src/boundary/ns/BounceBack.cu:12-31). */
int fm_add_ns_bounceback(fm_lattice* lat, const uint8_t* mask, size_t n);
/* ADDirichlet (include/boundary/ad/ADDirichlet.hpp:11-42). */
int fm_add_ad_dirichlet(fm_lattice* lat, const uint8_t* mask, size_t n, double phi);
/* ADDirichletTanhPulse (include/boundary/ad/ADDirichletTanhPulse.hpp:10-38). */
int fm_add_ad_tanh_pulse(fm_lattice* lat, const uint8_t* mask, size_t n, double phi_base,
                         double phi_amp, int t_on_step, int t_off_step, double k_step);
/* ADNeumannOutlet (include/boundary/ad/ADNeumannOutlet.hpp:11-38). */
int fm_add_ad_neumann(fm_lattice* lat, const uint8_t* mask, size_t n);

/* ---- time stepping ---------------------------------------------------------
 * Lattice::initEquilibrium + ADLattice::initEquilibrium
 * (NSLattice.hpp:177-185, ADLattice.hpp:134-141); resets the step counter. */
int fm_init_equilibrium(fm_lattice* lat);
/* nsteps iterations of the loop body of src/main.cpp:319-357 (queued, async). */
int fm_step(fm_lattice* lat, int nsteps);
/* Wait for queued work; a failed launch or kernel returns FM_ERR_CUDA. */
int fm_synchronize(fm_lattice* lat);
long long fm_step_count(const fm_lattice* lat);

/* ---- outputs ---------------------------------------------------------------
 * Field download to host doubles (n = nx*ny*nz): rho and u are the moments of
 * the current f as Lattice::computeMacroscopicDevice forms them
 * (src/core/Macros.cu:20-61); C is ADLattice::downloadPhi
 * (ADLattice.hpp:167-170); Q is AdsorbedField::download
 * (include/reaction/AdsorbedField.hpp:30-34). */
int fm_get_field(fm_lattice* lat, int field, double* out, size_t n);
/* The same field as FP32 values (the arithmetic type of every form but FM_F64):
 * copied straight from the device for FP32 planes, narrowed on the device for
 * FP64 ones (FM_F64 fields, the FP64 q of the 16-bit forms).  Half the bytes
 * of fm_get_field.  No reference counterpart (the reference's FP32 build
 * downloads its DATA_TYPE = float fields the same way). */
int fm_get_field_f32(fm_lattice* lat, int field, float* out, size_t n);
/* All six fields in one call: out[0..5] receive rho, ux, uy, uz, C, q (FP64 or
 * FP32; a null pointer skips that field).  One macroscopic pass and one
 * synchronisation for all of them; the copies run back to back on the
 * lattice's stream, so page-locked outputs receive them at the host link's
 * rate.  Same values as six fm_get_field / fm_get_field_f32 calls. */
int fm_get_fields(fm_lattice* lat, double* const out[6], size_t n);
int fm_get_fields_f32(fm_lattice* lat, float* const out[6], size_t n);
/* OutletCSV (include/core/io/OutletCSV.hpp:11-67): mean of C over `mask`
 * sampled at step 0 and every `every` steps thereafter. */
int fm_set_outlet_probe(fm_lattice* lat, const uint8_t* mask, size_t n, int every);
int fm_get_breakthrough(fm_lattice* lat, double* out, int capacity, int* count);
/* Domain sums in FP64 on the device: out[0] = sum rho, out[1] = sum C,
 * out[2] = sum q, out[3] = mean C over the outlet probe (0 if none). */
int fm_reduce(fm_lattice* lat, double out[4]);

/* ---- state I/O (checkpoints, tests) ----------------------------------------
 * Populations as FP64 SoA on the host: f[k*n + c] (19 n), g[k*n + c] (7 n);
 * phi/q per cell; any pointer may be NULL. */
int fm_get_state(fm_lattice* lat, double* f, double* g, double* phi, double* q);
int fm_set_state(fm_lattice* lat, const double* f, const double* g, const double* phi,
                 const double* q);

/* ---- the reference's free reaction launchers, on device pointers ----------
 * launch_henry_ldf_source_d3q7 (include/reaction/LinearLDF.hpp:8-17) and
 * launch_langmuir_ldf_source_d3q7 (include/reaction/LangmuirLDF.hpp:7-14)
 * with DATA_TYPE = float; `stream` is a cudaStream_t or NULL (default
 * stream).  These do not synchronise. */
int fm_launch_henry_ldf_source_d3q7(int n_cells, const uint8_t* d_region, const float* d_phi,
                                    float* d_sphi, float* d_q, float k_henry, float k_ldf,
                                    float phi_min_clamp, void* stream);
int fm_launch_langmuir_ldf_source_d3q7(int n_cells, const uint8_t* d_region, const float* d_phi,
                                       float* d_sphi, float* d_q, float q_max, float b,
                                       float k_ldf, float phi_min_clamp, void* stream);

/* ---- batching (no reference counterpart) ----------------------------------------
 * Many lattices -- porous samples with their own sizes, masks, boundaries and
 * isotherm parameters -- advanced together: one persistent kernel launch per
 * time step walks a work list of cell chunks over all of them, and the step
 * loop is replayed from a captured CUDA graph.  Requirements, checked by
 * fm_batch_create: the lattices share precision and collision operator, are
 * initialised and at the same step, and run one launch per step each
 * (fm_launches_per_step == 1: full x-plane boundaries, even Nx); their outlet
 * probes share one period (or are off).  fm_batch_create snapshots each
 * lattice's parameters and boundaries; set lattices up completely first.  The
 * lattices remain the caller's: fields, breakthrough series and state are read
 * per lattice; fm_batch_step orders each lattice's stream after the batch. */
typedef struct fm_batch fm_batch;
int fm_batch_create(fm_lattice* const* lattices, int count, void* stream, fm_batch** out);
int fm_batch_destroy(fm_batch* batch);
/* nsteps coupled time steps of every lattice (queued, async). */
int fm_batch_step(fm_batch* batch, int nsteps);
int fm_batch_synchronize(fm_batch* batch);
long long fm_batch_cells(const fm_batch* batch);
/* Launch shape: threads per block (128 or 256), cells per thread per work
 * item (1..8), L2 prefetch distance in work items (0..1024; the persistent
 * modes prefetch their own next items, the flat mode a fraction of a resident
 * wave ahead), and the launch mode:
 * 0 = persistent kernel reading the lattice arguments from global memory
 * (any batch size), 1 = persistent kernel and 2 = one block per work item,
 * both with the arguments and the work list in constant memory (batches of up
 * to ~96 lattices), 3 = one single-lattice step launch per lattice with its
 * arguments as kernel parameters, spread over four streams forked from the
 * batch's stream and joined each step, so independent lattices overlap (any
 * batch size; the shape arguments are not used).  All modes run inside the
 * batch's captured step graph.  A new batch starts in mode 3;
 * fm_batch_set_config keeps the current mode. */
int fm_batch_set_config(fm_batch* batch, int block, int cells_per_thread, int prefetch);
int fm_batch_set_mode(fm_batch* batch, int mode, int block, int cells_per_thread, int prefetch);
/* Project autotuner: times `trial_steps` steps (rounded up to even) of every
 * candidate launch shape and mode, keeps the fastest and restores the
 * lattices' state afterwards; writes the choice to the optional outputs.  The
 * constant-memory tables are shared by all batches of a process: only one
 * batch may have work in flight at a time. */
int fm_batch_autotune(fm_batch* batch, int trial_steps, int* mode, int* block, int* cells_per_thread,
                      int* prefetch, double* best_ms_per_step);

/* ---- outlet statistics (OutletCSV::log, include/core/io/OutletCSV.hpp:29-57) -------
 * Mean, min and max of C over the outlet probe cells (fm_set_outlet_probe; a
 * period of 0 sets the cells without automatic sampling), reduced on the
 * device in FP64 from the current state; all three are 0 without probe cells. */
int fm_outlet_stats(fm_lattice* lat, double out[3]);

/* ---- VTI geometry (readVTI, include/vti/VTIReader.hpp:35-160) -------------------------
 * fm_vti_info: Nx, Ny, Nz from WholeExtent (else Extent) and the number of
 * values in the first DataArray.  fm_vti_read: n = Nx*Ny*Nz outputs; mask[i]
 * = value > threshold (3 components: their magnitude; any other count: the
 * first min(count, n) values, with the reference's warning); values (optional)
 * receives the per-cell value or magnitude.  ASCII DataArrays as the
 * reference reads them, plus format="binary" (base64) and format="appended"
 * (raw or base64), uncompressed, of any VTK scalar type.  Errors carry the
 * reference's messages.  fm_vti_write writes n*components Float64 values as
 * CellData (binary != 0: appended raw; else ASCII) that fm_vti_read and
 * readVTI both read. */
int fm_vti_info(const char* path, int* nx, int* ny, int* nz, long long* nvalues);
int fm_vti_read(const char* path, double threshold, uint8_t* mask, double* values, size_t n);
int fm_vti_write(const char* path, int nx, int ny, int nz, const double* values, int components, const char* name,
                 int binary);

/* ---- adjoint (no reference counterpart) -------------------------------------------
 * Gradients of the breakthrough-curve loss
 *     L = sum_i (C_out(s0 + i*P) - target[i])^2,  i = 1..ntarget,
 * where C_out is the mean AD scalar over the outlet probe (the x = nx-1
 * plane), P its period and s0 the current step (a multiple of P).  Runs
 * nsteps forward from the current state (the lattice ends there, with its
 * breakthrough series extended), keeping a snapshot every checkpoint_every
 * steps, then the hand-written adjoint kernels backwards, recomputing each
 * segment from its snapshot: with at least checkpoint_every stored states the
 * segment is recomputed once, otherwise by binomial checkpointing within
 * max_stored_states state buffers (plus one scratch state).
 * Outputs: *loss; grad_params[3] = dL/d(q_max, b, k_ldf) for Langmuir or
 * dL/d(K_henry, 0, k_ldf) for linear; grad_porosity (NULL or n values) =
 * dL/d porosity per cell (porous collision; zero otherwise).  Differentiated
 * set-up: BGK or porous collision, fused full-plane NEQ inlet, pressure
 * outlet, AD Dirichlet / Neumann (each optional), linear or Langmuir LDF;
 * FM_F32 or FM_F64 storage. */
int fm_adjoint_breakthrough(fm_lattice* lat, int nsteps, const double* target, int ntarget, int checkpoint_every,
                            int max_stored_states, double* loss, double* grad_params, double* grad_porosity);

/* The workspace of fm_adjoint_breakthrough (one device allocation holding the
 * segment snapshots, the state buffers and the adjoint fields) stays with the
 * lattice for the next call; fm_adjoint_release frees it (fm_lattice_destroy
 * does too).  fm_adjoint_stats reports the forward steps the last call
 * recomputed in its reverse sweep and the workspace size in bytes. */
int fm_adjoint_release(fm_lattice* lat);
int fm_adjoint_stats(const fm_lattice* lat, long long* recomputed_steps, long long* workspace_bytes);

/* ---- allocation-free reduction ------------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc --
 * a host application that reserved its device memory up front in its own pool,
 * or code running where an allocation would stall the device or break an
 * asynchronous pipeline.  Sums over n_cells cells of FP32 buffers the caller
 * owns: out[0] = sum of rho (the FP32 sum of the 19 populations of each cell,
 * read from d_f[k*plane_stride + c]), out[1] = sum of d_phi, out[2] = sum of
 * d_q -- the first three values of fm_reduce, in a fixed (run-to-run
 * deterministic) order.  Allocates nothing: intermediate sums live in a
 * 128 KiB array in static device memory that every GPU loading the library
 * holds until the process exits.  Limit: n_cells <= 134,217,728, else
 * FM_ERR_ARG.  The first call on each device (with that device current) looks
 * up the array's device address, so make it before any stream capture; the
 * address is cached per device and looked up again when the device's context
 * has changed (after cudaDeviceReset), so the call after a reset must also
 * come before any capture.  All
 * calls share the array: calls that overlap on the GPU (other streams or
 * threads) race.  Queued on `stream` (NULL = default stream); returns after
 * the result has reached `out` on the host. */
int fm_reduce_static(const float* d_f, const float* d_phi, const float* d_q, long long plane_stride,
                     long long n_cells, double out[3], void* stream);

/* ---- measurement -------------------------------------------------------------
 * When enabled, fm_step brackets every launch of the fused step kernel with a
 * pair of CUDA events on the lattice's stream.  fm_profile_read synchronises,
 * returns the summed kernel time (ms) and launch count since the last
 * enable/read, and resets them.  No reference counterpart (measurement aid). */
int fm_profile_enable(fm_lattice* lat, int enabled);
int fm_profile_read(fm_lattice* lat, double* kernel_ms, long long* launches);
/* The memory ceiling of the step's access pattern: `reps` launches of a pure
 * copy that reads, for every cell off the first and last z-plane, the 19 + 7
 * pull sources the step reads and writes them to the cell's own slots, with
 * no arithmetic.  Writes the mean time per launch (ms) and the bytes moved per
 * launch.  Overwrites the lattice's write buffers (the next step rewrites
 * them); the state is unchanged.  No reference counterpart (measurement aid). */
int fm_bench_pull_copy(fm_lattice* lat, int reps, double* ms_per_rep, double* bytes_per_rep);

/* ---- step monitor ----------------------------------------------------------------
 * No reference counterpart (the reference reduces nothing on the device;
 * main.cpp downloads phi for its outlet log).  With fm_set_monitor(lat,
 * every > 0), each step whose number is a multiple of `every` runs a variant of
 * the fused kernel that also reduces, in FP64 by warp shuffles with one
 * partial per block and one small fold launch, over all cells: the domain mass
 * sum(rho) of the stored populations, sum(C), sum(q), the outlet flux
 * sum(C u_x) over the x = nx-1 cells, and the number of cells whose rho is not
 * positive or whose rho or C is not finite (a divergence status).  Needs
 * every boundary inside the fused step (fm_launches_per_step == 1), else
 * fm_step returns FM_ERR_UNSUPPORTED.  fm_get_monitor copies up to `capacity`
 * rows of 6 doubles (step, mass, C, q, outlet flux, bad cells) and writes the
 * number of rows; fm_init_equilibrium and fm_set_monitor restart the rows.
 * every = 0 turns the monitor off. */
int fm_set_monitor(fm_lattice* lat, int every);
int fm_get_monitor(fm_lattice* lat, double* out, int capacity, int* count);

/* ---- device memory ---------------------------------------------------------------
 * No reference counterpart.  The library allocates device memory from a
 * stream-ordered pool of its own on each device (the device's default pool and
 * its settings are left to the host application) and frees it in the order of
 * the owning lattice's or batch's stream, without synchronising the device.
 * Freed memory stays mapped in the pool, up to half of the device memory, so
 * the next lattice reuses it without mapping it again; fm_trim_memory hands
 * all but `keep_bytes` of it back to the device (current device). */
int fm_trim_memory(size_t keep_bytes);

/* ---- storage layout of the 16-bit forms ----------------------------------------
 * No reference counterpart.  fm_set_pair_layout(lat, 1) lets a lattice of a
 * 16-bit form (FM_F16_SHIFTED, FM_BF16_SHIFTED, FM_F16_FIXED_AD) with
 * nx % 4 == 0 and nx >= 8, whose boundaries all run inside the fused step
 * (fm_launches_per_step == 1), and that no batch holds, store its populations
 * in the pair layout: word w of an x-row holds the cells x = w and
 * x = w + nx/2, and one thread updates both (32-bit loads and stores, packed
 * FP32 pair arithmetic); the results are the same, bit for bit, as the one-cell
 * kernel's.  It is off by default (0): on B200 the one-cell kernel on the
 * natural layout measured faster.  The getters, fm_get_state / fm_set_state and
 * the z-plane halo calls see cells in the natural order whatever the layout.
 * fm_storage_layout returns the layout the next step runs on (0 natural,
 * 1 pair; converting the stored populations if that changed) or a negative
 * status. */
int fm_set_pair_layout(fm_lattice* lat, int enabled);
int fm_storage_layout(fm_lattice* lat);

/* The pair layout has two step kernels with the same results bit for bit.
 * The staged kernel (the default where it applies: nx % 8 == 0 and
 * nx <= 512, and the two stages of a block fit its shared memory) runs a
 * persistent grid over tiles of whole x-rows; the copy engine brings each
 * tile's 26 source rows and cell arrays into shared memory by bulk copies
 * while the block updates the previous tile.  fm_set_pair_kernel(lat, 0)
 * selects k_coupled_pair, which loads its pulls straight from global memory.
 * fm_step_kernel returns the kernel the next step runs: 0 the one-cell
 * kernel (natural layout), 1 k_coupled_pair, 2 the staged kernel, 3 the
 * one-cell kernel with unsigned pull offsets (a 16-bit lattice too large for
 * the faster signed ones: 18*ns + nx*ny + 2*nx + 1 >= 2^31, ns the cell count
 * rounded up to 32; about 119M cells); or a negative status. */
int fm_set_pair_kernel(fm_lattice* lat, int staged);
int fm_step_kernel(fm_lattice* lat);

/* The step kernels' device status word since the last call, then cleared:
 * 0, or bit 0 when a wait of the staged kernel for its shared-memory copies
 * gave up after its poll limit (the block then left the step unfinished;
 * the state of that step is not valid).  No reference counterpart. */
int fm_step_status(fm_lattice* lat, int* status);

/* ---- tuning ------------------------------------------------------------------
 * L2 prefetch distance of the fused step kernel, in 256-cell blocks
 * (0 disables the prefetch; negative restores the automatic choice: about
 * half a resident wave for FM_F32, none for FM_F64 and the 16-bit forms, for
 * which a prefetch measured slower on large lattices).  No reference
 * counterpart. */
int fm_set_prefetch_distance(fm_lattice* lat, int blocks);

/* ---- introspection (bench / tests) ---------------------------------------- */
/* Number of kernel launches fm_step queues per time step for this set-up. */
int fm_launches_per_step(const fm_lattice* lat);
/* ---- z-slab decomposition (no reference counterpart) ---------------------------
 * A lattice split into z-slabs keeps one ghost plane per inner face; after
 * every step each slab sends the stored populations of the plane next to a
 * face to its neighbour's ghost plane.  fm_pack_zplane copies the stored
 * populations of plane z (the 19 D3Q19 then the 7 D3Q7 directions, nx*ny cells
 * each, x fastest) into a contiguous device buffer of 26*nx*ny elements of the
 * storage type (2 bytes for the 16-bit forms, 4 for FM_F32, 8 for FM_F64);
 * fm_unpack_zplane writes such a buffer into plane z.  Both are queued on the
 * lattice's stream. */
int fm_pack_zplane(fm_lattice* lat, int z, void* d_buf);
int fm_unpack_zplane(fm_lattice* lat, int z, const void* d_buf);
/* The halo proper: only the populations of plane z that cross a z-face in
 * direction dir, 6 of the 26 -- dir = +1 the D3Q19 directions with c_z = +1
 * (5, 11, 12, 15, 16) then D3Q7 direction 5 (what the neighbour above pulls
 * from this plane), dir = -1 those with c_z = -1 (6, 13, 14, 17, 18) then
 * D3Q7 6 -- to / from a buffer of 6*nx*ny elements of the storage type.  They
 * act on the populations being written by a step begun with fm_step_planes,
 * else on the current ones.  Queued on the lattice's stream. */
int fm_pack_zhalo(fm_lattice* lat, int z, int dir, void* d_buf);
int fm_unpack_zhalo(fm_lattice* lat, int z, int dir, const void* d_buf);
/* A time step in parts, so that a halo exchange overlaps the interior update:
 * fm_step_planes runs the fused step of the next step for the z-planes
 * [z0, z1) only (any number of calls, each queued on the lattice's stream, for
 * disjoint plane ranges); fm_step_finish completes the step (buffer swap, step
 * count, outlet sample).  Planes not stepped keep stale populations in the
 * buffer being written (ghost planes, whose crossing populations the halo
 * unpack then supplies).  Requires a lattice whose step is one launch
 * (fm_launches_per_step == 1) and nx*ny a multiple of 64; FM_ERR_UNSUPPORTED
 * otherwise.  fm_step and fm_reduce_zrange refuse while a step is open. */
int fm_step_planes(fm_lattice* lat, int z0, int z1);
int fm_step_finish(fm_lattice* lat);
/* Sums of rho, C and q over the z-planes [z0, z1) (the interior of a slab),
 * FP64, as the first three values of fm_reduce. */
int fm_reduce_zrange(fm_lattice* lat, int z0, int z1, double out[3]);

/* Device pointer of the current NS population buffer and its plane stride
 * (elements between f_k and f_{k+1}); for tests of the layout. */
int fm_debug_layout(const fm_lattice* lat, long long* plane_stride, int* precision);
/* Test aid: writes the device status word (fm_step_status) from the host, so
 * the host-side detection of a device wait that gave up can be tested without
 * making a kernel wait run out. */
int fm_debug_set_status(fm_lattice* lat, int status);

#ifdef __cplusplus
}
#endif
#endif /* FM_H */
