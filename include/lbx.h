/*
 * lbx.h — C ABI of the B200-native LBcuda hot path.
 *
 * The reference (LBcuda, CUDA Fortran) drives its kernels from `program TestLB`
 * (main.CUF:1-316) on module-global device arrays (kernels_fluid.CUF:9-48)
 * with parameters in Fortran `parameter`s and `constant` memory
 * (dimensions_m.CUF:1-365, main.CUF:1043-1162).  This header replaces that
 * surface with an opaque context and plain-pointer entry points that a
 * Fortran host can bind with ISO_C_BINDING (`bind(C)`, `type(c_ptr)`,
 * `integer(c_int), value`).  No entry point takes or returns a torch or CUDA
 * type.
 *
 * Conventions
 *  - Every function returns an int status: 0 = ok, <0 = CUDA/runtime error
 *    (LBX_ERR_*), >0 = device range-check error raised by a kernel (the
 *    reference's `stop_d = __LINE__` protocol, main.CUF:2410-2442).  No entry
 *    point aborts the process.
 *  - Host field buffers are x-fastest, interior cells only, nx*ny*nz values
 *    (Fortran order `a(1:nx,1:ny,1:nz)`); vector fields are (3, nx, ny, nz).
 *  - Population buffers are (nx, ny, nz, Q) x-fastest, Q = 19 (D3Q19, the
 *    reference default `noD3Q27`, defines.h:8) in the reference lattice order
 *    (dimensions_m.CUF:211-218).
 *  - Particle arrays are FP64, (3, n) or (4, n) column-major like the
 *    reference's pos_d(13,N,2) slices (dimensions_m.CUF:352-360).
 *  - One context per CUDA stream; calls on one context are not thread-safe.
 *    lbx_step only enqueues work; lbx_get_*, lbx_sync and lbx_status
 *    synchronise.
 */
#ifndef LBX_H
#define LBX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enumerations ------------------------------------------------------ */
#define LBX_MODEL_BGK 0 /* single-component BGK (kernels_fluid_BGK.CUF)        */
#define LBX_MODEL_CG 1  /* two-component colour gradient (kernels_fluid_CG.CUF) */
#define LBX_MODEL_CG_DIFFDENS 2 /* colour gradient with two fluid densities (the DIFFDENS build,
                                 kernels_fluid_CG.CUF:40-49,163-177,539-819): two-pass schedule */
#define LBX_MODEL_CG_D3Q27 3    /* colour gradient on the D3Q27 lattice (the D3Q27 build,
                                   dimensions_m.CUF:117-198): 27 populations per component,
                                   two-pass schedule, no spheres (the reference's bounce-back is
                                   D3Q19 only, kernels_fluid_PART.CUF:1929-1941) */
#define LBX_MODEL_CG_DIFFDENS_D3Q27 4 /* both builds together */

#define LBX_STORE_F32 0  /* FP32 populations (reference storage)            */
#define LBX_STORE_F16 1  /* FP16 populations shifted by w_l * rho0           */
#define LBX_STORE_BF16 2 /* BF16 populations shifted by w_l * rho0           */
#define LBX_STORE_F64 3  /* FP64 populations and FP64 arithmetic (error runs) */
/* 16-bit sum / difference pairs (no counterpart in the reference): per
 * direction and cell the pair (f_R + f_B - w_l (rho0R + rho0B),
 * f_R - f_B - w_l (rho0R - rho0B)) instead of (f_R - w_l rho0R,
 * f_B - w_l rho0B).  The total population carries the momentum and sits near
 * w_l rho, so its shifted value is small and keeps more bits; rounding then
 * moves the velocity far less.  FP32 arithmetic as for LBX_STORE_F16.
 * Colour-gradient model (LBX_MODEL_CG) on the single-pass schedule (one box
 * or the ensemble), with or without spheres; lbx_create rejects it with
 * another model, lbx_set_schedule on the other schedules.
 * lbx_set_pops / lbx_get_pops and the field calls convert, so callers still
 * see f_R and f_B. */
#define LBX_STORE_F16_SD 4
#define LBX_STORE_BF16_SD 5
/* 16-bit sum / predicted-split pairs (no counterpart in the reference): the
 * total as in LBX_STORE_F16_SD, and in place of the colour difference
 * D = f_R - f_B its deviation from the split the receiving cell predicts,
 * E = D - phi_y (f_R + f_B), phi_y the phase field of the cell y that will
 * pull the pair, from the step in which the pair was written (an FP32 value
 * per cell, kept beside each population buffer).  In the bulk of either
 * fluid E is only the small recolouring term, so its rounding no longer
 * stirs the flow.  Colour-gradient model on the single-pass schedule without
 * spheres (lbx_create rejects max_particles > 0, the ensemble rejects it);
 * the population and field calls convert as for the other formats. */
#define LBX_STORE_F16_SDP 6
#define LBX_STORE_BF16_SDP 7

#define LBX_WET_JANUS 0   /* compute_virtual_rho, kernels_fluid_PART.CUF:299-352 */
#define LBX_WET_NEUTRAL 1 /* compute_densities_wall, kernels_fluid_PART.CUF:267-297 */

/* cell flags, dimensions_m.CUF:306-310 */
#define LBX_FLUID_WALL 0
#define LBX_FLUID_FLUID 1
#define LBX_FLUID_SPHERELIST 2
#define LBX_FLUID_SPHEREDEAD 4
#define LBX_FLUID_PARTICLECM 5

/* host-side error codes (negative) */
#define LBX_ERR_CUDA (-1)
#define LBX_ERR_ARG (-2)
#define LBX_ERR_ALLOC (-3)
#define LBX_ERR_STATE (-4)
#define LBX_ERR_TIMEOUT (-5)
#define LBX_ERR_NOSYM (-6)

/* device error codes (positive, first one wins), each tied to the reference
 * check it restates */
#define LBX_DEV_RHO_RANGE 1       /* init_rhoR_CG/init_rhoB_CG, kernels_fluid_CG.CUF:438-441,496-499 */
#define LBX_DEV_BIG_FORCE 2       /* nve_lf, kernels_fluid_PART.CUF:1532-1537 */
#define LBX_DEV_EXTREME_VEL 3     /* nve_lf, kernels_fluid_PART.CUF:1545-1549 */
#define LBX_DEV_POSITION 4        /* nve_lf, kernels_fluid_PART.CUF:1581-1598 */
#define LBX_DEV_LIST_OVERFLOW 5   /* makeListAtomsGPU, kernels_fluid_PART.CUF:2436-2439 */
#define LBX_DEV_BELT_RANGE 6      /* compute_onebelt_*, kernels_fluid_PART.CUF:800-803 */
#define LBX_DEV_WAIT_TIMEOUT 7    /* a bounded in-kernel wait gave up (no counterpart in the reference) */

/* ---- parameters -------------------------------------------------------- */
/* The reference keeps these as compile-time `parameter`s (dimensions_m.CUF:
 * 50-84) plus the runtime input.dat values (main.CUF:409-496).  Here they are
 * one runtime struct; lbx_default_params fills the reference values. */
typedef struct lbx_params {
  int32_t nx, ny, nz;     /* interior lattice (glx, gly, glz) */
  int32_t model;          /* LBX_MODEL_* */
  int32_t storage;        /* LBX_STORE_* */
  int32_t wetting;        /* LBX_WET_* */
  int32_t lrotate;        /* particle rotation (input.dat line 9) */
  int32_t max_particles;  /* capacity of the particle arrays */
  float tau;              /* BGK relaxation time, omega = 1/tau */
  float tauR, tauB;       /* CG relaxation times (dimensions_m.CUF:98-99) */
  float sigma, beta;      /* sigma_CG, beta_CG (dimensions_m.CUF:50) */
  float rho0R, rho0B;     /* shift densities of the 16-bit storage */
  float radius;           /* rdim (dimensions_m.CUF:59) */
  float rmass;            /* 1/mass (dimensions_m.CUF:60) */
  float max_vel;          /* MAX_PARTICLE_VEL (input.dat line 8) */
  float ext_force[3];     /* ext_fxx, ext_fyy, ext_fzz */
  float ext_torque[3];    /* ext_tqx, ext_tqy, ext_tqz */
  float hz_k, hz_rmin, hz_rcap;             /* Hertz (dimensions_m.CUF:77-80) */
  int32_t lubrication;                      /* llubrication (dimensions_m.CUF:81) */
  float lubric_k, lubric_rmin, lubric_rcap; /* dimensions_m.CUF:82-84 */
  int32_t kinematic;      /* force probes, no counterpart in the reference.  1: prescribed
                             motion: centres move with the set velocity; velocity, angular
                             velocity, orientation kept.  2: frozen geometry: centres stay,
                             the bounce-back walls move with the set velocities */
  int32_t closure;        /* 1: learned pair closure with analytic fallback (lbx_closure_*) */
  float closure_gap_min;  /* training envelope of the closure: gap / R in [min, max] */
  float closure_gap_max;
  float closure_vmax;     /* and |relative velocity| components <= vmax */
  int32_t exact_tiles;    /* 1 (default): a sphere acts on a cell only where the reference's 8x4x4
                             tile lists (makeListAtomsGPU) reach it; for integer radii those lists
                             miss template cells.  0: every cell of the sphere's template box */
  float densR, densB;     /* densities of the two fluids for LBX_MODEL_CG_DIFFDENS (namelist
                             &fluid, main.CUF:343; SetConstants 1047-1083): both > 0, at least
                             one equal to 1; ignored by the other models (default 1, 1) */
} lbx_params;

/* Fill the reference defaults for an nx*ny*nz periodic box: CG model, FP32
 * storage, Janus wetting, tau = 1, sigma = 0.1, beta = 0.999, r = 5.5,
 * rmass = 1/1500, Hertz k = 10, rmin = 10.5, rcap = 9. */
void lbx_default_params(lbx_params* p, int32_t nx, int32_t ny, int32_t nz);

/* ---- lifetime ---------------------------------------------------------- */
/* Replaces setupGPUgridAndAlloc + SetConstants (main.CUF:2133-2407,
 * 1043-1162): allocates every device array of the path and uploads the
 * lattice tables.  The library owns all device memory. */
int lbx_create(const lbx_params* p, void** ctx);
int lbx_destroy(void* ctx);

/* ---- initial conditions ------------------------------------------------ */
/* setupPops (kernels_fluid_CG.CUF:313-346): equilibrium populations at
 * density rhoR/rhoB and uniform velocity (vx,vy,vz); all flags fluid.  For
 * the BGK model rhoB is ignored (may be NULL).  Covers initType 1,2,3,5,6
 * once the host has built the density fields (main.CUF:2531-2608). */
int lbx_set_fields(void* ctx, const float* rhoR, const float* rhoB, float vx, float vy, float vz);
/* initType 4 (read_and_setPops, main.CUF:2489-2529): raw populations,
 * q planes of nx*ny*nz per component (q = 19; 27 for the D3Q27 models). */
int lbx_set_pops(void* ctx, const float* popsR, const float* popsB);

/* ---- particles --------------------------------------------------------- */
/* read_input_atom (main.CUF:1230-1350) + the step-0 flags of setupRho_Pops
 * (main.CUF:2586-2600): n spheres of radius p->radius at xyz (3,n), with
 * velocities vel (3,n), body-frame angular velocities omega (3,n, may be
 * NULL) and quaternions q (4,n, may be NULL = identity).  Needs a CG context
 * created with max_particles >= n and nx % 8 == ny % 4 == nz % 4 == 0 (the
 * reference's tile grid).  Call after lbx_set_fields. */
int lbx_set_particles(void* ctx, int32_t n, const double* xyz, const double* vel, const double* omega,
                      const double* q);
/* Particle state after the last step and the total force / torque its
 * integrator used (forceAtoms_d(1:3) and (7:9), kernels_fluid_PART.CUF:
 * 1266-1382); any pointer may be NULL. */
int lbx_get_particles(void* ctx, double* xyz, double* vel, double* omega, double* q, double* force, double* torque);

/* ---- the time step ----------------------------------------------------- */
/* One or more full steps in the order of main.CUF:125-308 (fluid: moments,
 * collision, streaming; with particles also flags, fill/drain, wetting,
 * bounce-back, pair forces and the particle integrator). */
int lbx_step(void* ctx, int32_t nsteps);
/* Kernel-level entries of the same step, for callers that drive the order
 * themselves (the reference's host does, main.CUF:130-271).  Fluid only:
 * lbx_init_rho, lbx_time_step_cg (each lbx_time_step_cg completes a step).
 * With spheres, one step is the sequence below, in this order, and gives
 * the same state as lbx_step(ctx, 1); the step ends (every ping-pong index
 * flips) in lbx_time_step_force_particles.  Streaming has no entry of its
 * own: it is the periodic pull inside lbx_time_step_cg (the reference's
 * flipflop*Pop0_CG, stream*_CG, stream_CG_x/_y/_z and halo copies,
 * main.CUF:206-221).  The particle entries return LBX_ERR_STATE before
 * lbx_set_particles. */
int lbx_make_list_atoms(void* ctx);   /* makeListAtomsGPU (main.CUF:240, previous step's end) */
int lbx_init_isfluid(void* ctx);      /* init_isfluid_CG + fixPeriodic_isfluid (main.CUF:130-131) */
int lbx_del_fluid(void* ctx);         /* del_fluid_CG (main.CUF:132) */
int lbx_init_rho(void* ctx);          /* init_rhoR_CG + init_rhoB_CG (+ periodic rho halo) (main.CUF:143-149) */
int lbx_make_fluid(void* ctx);        /* make_fluid_CG (main.CUF:154) */
int lbx_virtual_rho(void* ctx);       /* compute_virtual_rho / compute_densities_wall (main.CUF:164-165) */
int lbx_time_step_cg(void* ctx);      /* time_step_CG + flipflop*Pop0 + stream*_CG (+ halos) (main.CUF:172-221) */
int lbx_partbb(void* ctx);            /* partBB_CG: node -> particle momentum (main.CUF:179) */
int lbx_partbb_p2n(void* ctx);        /* partBB_CG_p2n: bounce-back copy (main.CUF:184) */
int lbx_partbb_p2n2(void* ctx);       /* partBB_CG_p2n2: moving-wall term (main.CUF:187) */
int lbx_inter_force_particles(void* ctx);      /* inter_force_particles (+ closure) (main.CUF:224) */
int lbx_time_step_force_particles(void* ctx);  /* time_step_force_particles + flips (main.CUF:230) */
int lbx_time_step_bgk(void* ctx);     /* init_rho_isfluid_BGK + time_step_BGK + stream_BGK */

/* ---- readback ---------------------------------------------------------- */
/* moments2Fl (write_output.f90:975-1041) of the populations the reference
 * holds after the last step: rhoR, rhoB (nx*ny*nz), vel (3*nx*ny*nz),
 * phase (nx*ny*nz); zero on non-fluid cells.  Any pointer may be NULL. */
int lbx_get_fields(void* ctx, float* rhoR, float* rhoB, float* vel, float* phase);
/* The same in FP64 (exact moments of the stored populations). */
int lbx_get_fields_f64(void* ctx, double* rhoR, double* rhoB, double* vel, double* phase);
/* Post-streaming populations (the reference's `flip` buffer after a step),
 * q planes of nx*ny*nz per component as for lbx_set_pops. */
int lbx_get_pops(void* ctx, float* popsR, float* popsB);
/* Cell flags of the last step (myfluid_d(:,:,:,flip)), int8 nx*ny*nz. */
int lbx_get_flags(void* ctx, int8_t* flags);
/* The boundary links of the particle bounce-back at the flags lbx_get_flags
 * returns (those of the last step; before the first step, those of
 * lbx_set_particles), at the sphere positions that stamped them: every
 * (sphere, surface cell, direction) for which node_to_particle_bounce_back_bc2
 * (kernels_fluid_PART.CUF:1874-2113, pair loop 1929-1941) exchanges momentum:
 * a spherelist cell within the sphere's reach (d^2 < rmax^2, on the sphere's
 * tile list) and an opposite pair (2i-1, 2i) with exactly one fluid end.
 * cell = x + nx*(y + ny*z) of the surface cell, dir = the direction (1..18,
 * reference order) from it towards the fluid end, sphere = 0-based index.
 * Sorted by (sphere, cell, dir).  *n receives the total; at most cap entries
 * are written (cap = 0 queries the count).  LBX_ERR_STATE without spheres. */
int lbx_get_links(void* ctx, int32_t* cell, int8_t* dir, int32_t* sphere, int64_t cap, int64_t* n);
/* FP64 global sums: mass[2] (red, blue) and momentum[3], over fluid cells. */
int lbx_get_sums(void* ctx, double* mass, double* momentum);

/* ---- status ------------------------------------------------------------ */
int lbx_sync(void* ctx);
/* First device error since the last call: code (LBX_DEV_*), step, and the
 * cell (x + nx*(y + ny*z)) or particle index it concerns.  Clears it. */
int lbx_status(void* ctx, int32_t* code, int32_t* step, int64_t* where);
const char* lbx_error_string(int code);
/* Steps taken so far (the reference's `step`). */
int lbx_get_step(void* ctx, int64_t* step);

/* ---- learned pair closure (no counterpart in the reference) ------------ */
/* MLP 13 -> 64 -> 64 -> 64 -> 12 (SiLU, FP32) correcting the pair force and
 * torque of near-contact spheres; the reference's analytic lubrication
 * (addHertzian, kernels_fluid_PART.CUF:1463-1501) is the fallback outside
 * the training envelope.  Inputs per pair i < j, in the lattice-fixed pair
 * frame E (first axis n = (x_j - x_i)/|x_j - x_i|, transverse axes fixed by
 * the cubic symmetry class of n, s = +-1 the sign of that class map):
 * gap/R, E(v_j - v_i), s E omega_i, s E omega_j, R, nc_1, nc_2 (nc: |n|
 * sorted descending).  Outputs: force and torque on i, then on j, in E
 * (torques times s).  The weights travel as one flat blob of
 * LBX_CLOSURE_NWEIGHTS floats: W0[64][13] b0 W1[64][64] b1 W2[64][64] b2
 * W3[12][64] b3, then the input mean[13], std[13] and output mean[12],
 * std[12] used to standardise. */
#define LBX_CLOSURE_NWEIGHTS 10046
/* Glorot-uniform initial weights, identity standardisation. */
int lbx_closure_init(float* weights, int32_t seed);
/* Train on the GPU (one fused forward/backward/Adam kernel for all epochs):
 * X (n,13), T (n,12) raw features and targets, standardised with the
 * statistics in the blob; weights updated in place; loss[epochs] optional.
 * Minibatches of 64, Adam with the step size decaying from lr to 0 as a half
 * cosine over all epochs. */
int lbx_closure_train(float* weights, const float* X, const float* T, int32_t n, int32_t epochs, float lr,
                      int32_t seed, float* loss);
/* Gradient of the mean-squared error over the first min(n,128) standardised
 * samples (no update), for checking the backward pass. */
int lbx_closure_grad(const float* weights, const float* Xs, const float* Ts, int32_t n, float* grad);
/* Batched inference on raw features: Y (n,12). */
int lbx_closure_infer(const float* weights, const float* X, int32_t n, float* Y);
/* lbx_closure_infer without any device allocation (no counterpart in the
 * reference), for callers that must not allocate or free device memory:
 * inputs and outputs go through one fixed device array per device
 * (449,792 bytes).  n <= LBX_CLOSURE_NOALLOC_MAX, else LBX_ERR_ARG.  The
 * first call on a device (that device current) looks the array up; with lazy
 * module loading that is also when the array gets its device memory, so make
 * the first call before reserving device memory up front and before any
 * stream capture.  Not valid after cudaDeviceReset in the same process.
 * Calls that overlap in time on one device share the array and race:
 * serialise them.  Same results as lbx_closure_infer. */
#define LBX_CLOSURE_NOALLOC_MAX 4096
int lbx_closure_infer_noalloc(const float* weights, const float* X, int32_t n, float* Y);
/* Attach trained weights to a particle context; with p->closure = 1 each
 * step then corrects every close pair inside the envelope (closure_gap_min
 * <= gap/R <= closure_gap_max, relative velocity and angular velocity
 * components <= closure_vmax) and applies the analytic lubrication
 * (p->lubrication) to the pairs outside it.  Without weights every pair
 * takes the fallback. */
int lbx_closure_set(void* ctx, const float* weights);

/* ---- ensemble of boxes (no counterpart in the reference) ---------------- */
/* nbox independent colour-gradient boxes (params[i]: sizes and spheres may
 * differ; storage, tau, sigma, beta, rho0 must agree) advanced together:
 * one persistent fluid kernel for all boxes per step, the sphere kernels of
 * each box around it, two steps captured into one CUDA graph. */
int lbx_ensemble_create(int32_t nbox, const lbx_params* params, void** ens);
int lbx_ensemble_destroy(void* ens);
/* Context of box i, for lbx_set_fields / lbx_set_particles / lbx_get_* /
 * lbx_closure_set; owned by the ensemble (do not destroy). */
int lbx_ensemble_box(void* ens, int32_t i, void** ctx);
int lbx_ensemble_step(void* ens, int32_t nsteps);
int lbx_ensemble_time(void* ens, int32_t nsteps, double* ms);
/* Autotuner: times the fused fluid kernel of every (CTA shape, z-segment
 * length) candidate over `trial` steps on the boxes themselves (this
 * advances them) and keeps the fastest; chosen = {shape, zlen}, best_ms =
 * that kernel's time per step. */
int lbx_ensemble_tune(void* ens, int32_t trial, int32_t* chosen, double* best_ms);

/* ---- z-slab decomposition --------------------------------------------- */
/* Replaces the reference's MPI z-slab split (main.CUF:504-1000 halo swaps,
 * setupMPI.CUF:26-30 rank layout): one context per slab holds its own planes
 * [zlo, zhi) plus at least two halo planes on each side; lbx_step then
 * computes and writes the own planes only.  zlo = zhi = 0 restores the
 * whole periodic box.  Colour-gradient model on the lean kernel, no spheres
 * (else LBX_ERR_STATE); zlo >= 2, zhi <= nz - 2 (else LBX_ERR_ARG). */
int lbx_set_zrange(void* ctx, int32_t zlo, int32_t zhi);
/* Bytes of a packed buffer of nplanes planes (lbx_pack_planes). */
int lbx_plane_bytes(void* ctx, int32_t nplanes, int64_t* bytes);
/* Planes [z0, z0 + nplanes) of the current populations (stored form; with
 * sum / predicted-split pairs followed by their split field) to / from a
 * packed DEVICE buffer: the halo exchange of a slab.  Enqueued on the
 * context's stream: lbx_sync before the buffer is used elsewhere. */
int lbx_pack_planes(void* ctx, int32_t z0, int32_t nplanes, void* dev_buf);
int lbx_unpack_planes(void* ctx, int32_t z0, int32_t nplanes, const void* dev_buf);
/* The context's CUDA stream (a cudaStream_t): a host that moves the packed
 * planes itself (NCCL, CUDA-aware MPI) orders its transfers after the pack
 * and before the unpack on it, without waiting on the host. */
int lbx_get_stream(void* ctx, void** stream);

/* ---- measurement ------------------------------------------------------- */
/* Colour-gradient schedule: 2 = lean single-pass kernel (default), 1 = the
 * first single-pass kernel, 0 = two passes (phase field, then collision).
 * LBX_MODEL_CG_DIFFDENS runs on 0 only (other values: LBX_ERR_ARG).
 * The reference prints Mlup/s from CUDA events around the step loop
 * (main.CUF:274-292); these are the hooks the benchmark uses for the same. */
int lbx_set_schedule(void* ctx, int32_t fused);
/* Lean single-pass kernel shape: 0 = 32x8 cells per CTA, 1 = 32x16; zlen =
 * lattice planes per z-segment (0 = automatic). */
int lbx_set_lean_shape(void* ctx, int32_t shape, int32_t zlen);
/* How the lean kernel stages 16-bit pulls in shared memory: 1 = 16-byte
 * granules of a box of rows per direction (default; used when nx is a
 * multiple of 4), 0 = one 4-byte copy per pull.  Both give the same bits. */
int lbx_set_lean_copies(void* ctx, int32_t mode);
/* Enqueue nsteps steps bracketed by CUDA events on the context stream and
 * wait: total device ms, and the summed duration / launch count of the
 * step's dominant kernel (NULL kernel_ms disables per-kernel events). */
int lbx_time_steps(void* ctx, int32_t nsteps, double* total_ms, double* kernel_ms, int64_t* kernel_launches);

#ifdef __cplusplus
}
#endif
#endif /* LBX_H */
