/*
 * matter_gpu.h — C ABI of the B200 MPM time step (libmatter_gpu.so).
 *
 * The reference (Matter, C++17/OpenMP) has no FFI: its setup code calls the
 * member functions of class Simulation directly.  Each entry point below
 * replaces one such call (or the part of it that moves data), and the host
 * drop-in (matter_tests_b200/host/) binds them behind the unchanged
 * Simulation surface.  All functions return MTR_OK (0) or a negative
 * MTR_ERR_* code; no C++ exception crosses this boundary.  Pointers are plain
 * host pointers; sizes are element counts.  A context is not thread-safe.
 *
 * Layout conventions shared by every entry point:
 *   - vectors are AoS doubles, `dim` per particle (x[p*dim + d]);
 *   - matrices are per particle, column-major, dim*dim doubles
 *     (F[p*dim*dim + c*dim + r]) — the storage order of the reference's
 *     Eigen TM in std::vector<TM> (data_structures.hpp:29-45);
 *   - particle scalars are six doubles per particle in the order
 *     MTR_SCALAR_* below.
 */
#ifndef MATTER_GPU_H
#define MATTER_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------- */
#define MTR_OK                    0
#define MTR_ERR_INVALID          -1  /* bad argument or unsupported option   */
#define MTR_ERR_CUDA             -2  /* a CUDA runtime call failed           */
#define MTR_ERR_OOM              -3  /* device allocation failed             */
#define MTR_ERR_DEVICE_STATUS    -4  /* the step raised a status flag; see mtr_status */
#define MTR_ERR_TIMEOUT          -5  /* bounded wait for the device expired  */
#define MTR_ERR_NO_DEVICE        -6  /* no CUDA device is visible            */
#define MTR_ERR_STATE            -7  /* call out of order (e.g. step before upload) */
#define MTR_ERR_TOO_LARGE        -8  /* request exceeds a fixed capacity (mtr_p2g_noalloc) */

/* ---- device status flags (mtr_status) ----------------------------------- */
#define MTR_STATUS_GRID_OVERFLOW   0x0001u /* grid outgrew capacity; host regrows and retries */
#define MTR_STATUS_STENCIL_OOB     0x0002u /* a particle stencil left the grid (skipped)     */
#define MTR_STATUS_BAD_BC          0x0004u /* invalid BC enum (boundary_collision.cpp:66-70) */
#define MTR_STATUS_RMA_NOCONV      0x0008u /* Newton loop hit its cap where the reference sets exit=1 */
#define MTR_STATUS_RMA_NOSTEP      0x0010u /* limited search found no admissible step        */
#define MTR_STATUS_NEG_DGAMMA      0x0020u /* Perzyna delta_gamma < 0 (plasticity.cpp:286-289) */
#define MTR_STATUS_NONFINITE       0x0040u /* NaN/Inf in particle state                       */
#define MTR_STATUS_BAD_MODEL       0x0080u /* invalid plastic/hardening model                 */
#define MTR_STATUS_RESID_DIFF      0x0100u /* Perzyna Newton derivative ~ 0                   */

/* ---- enums: numbering identical to tools.hpp:53-57 ---------------------- */
enum mtr_plate_type { MTR_PLATE_TOP = 0, MTR_PLATE_BOTTOM, MTR_PLATE_LEFT, MTR_PLATE_RIGHT,
                      MTR_PLATE_FRONT, MTR_PLATE_BACK };
enum mtr_elastic_model { MTR_EL_HENCKY = 0, MTR_EL_NEOHOOKEAN };
enum mtr_plastic_model { MTR_PM_NOPLASTICITY = 0, MTR_PM_VM, MTR_PM_DP, MTR_PM_DPSOFT, MTR_PM_MCC,
                         MTR_PM_VMVISC, MTR_PM_DPVISC, MTR_PM_MCCVISC, MTR_PM_DPMUI, MTR_PM_MCCMUI,
                         MTR_PM_SNOW };
enum mtr_hardening_law { MTR_HL_NOHARD = 0, MTR_HL_EXPOEXPL, MTR_HL_EXPOIMPL, MTR_HL_SINHEXPL,
                         MTR_HL_SINHIMPL };
enum mtr_bc { MTR_BC_NOSLIP = 0, MTR_BC_SLIPSTICK, MTR_BC_SLIPFREE };

/* analytic level-set objects (objects/object_*.hpp); prm[] meaning per kind */
enum mtr_object_kind {
  MTR_OBJ_BUMP = 0,        /* object_bump.hpp:15-41     no parameters                         */
  MTR_OBJ_GROUND = 1,      /* object_ground.hpp:16-36   prm[0] = y_ground                     */
  MTR_OBJ_RAMP = 2,        /* object_ramp.hpp:15-40     no parameters                         */
  MTR_OBJ_CURVE = 3,       /* object_curve.hpp:15-37    no parameters                         */
  MTR_OBJ_GATE = 4,        /* object_gate.hpp:16-41     prm[0] = height                       */
  MTR_OBJ_SILO = 5,        /* object_silo.hpp:16-54     prm[0] = cut (3D only)                */
  MTR_OBJ_BOX_ROTATED = 6, /* object_box.hpp:18-43       prm[0..2] center, prm[3..5] half
                              extents, prm[6..14] rotation, column-major (dim-sized in 2D)    */
  MTR_OBJ_TERRAIN_GAUSS = 7, /* no reference counterpart: surface y = prm[0] + sum_k h_k *
                              exp(-r_k^2 / (2 sigma_k^2)), prm[1] = nbumps (<= 4), bump k at
                              prm[2+4k..5+4k] = (x_k, z_k, h_k, sigma_k); 2D ignores z_k      */
  MTR_OBJ_LEVELSET = 8      /* object_vdb.hpp:17-94 on a dense lattice: prm[0] = level-set
                              slot (mtr_set_levelset).  Inside where the trilinear sample of
                              the signed distance phi is <= 0; normal = the trilinear sample
                              of its gradient (second-order central differences, or the
                              normals given at upload), normalised, zero where that is zero */
};
#define MTR_MAX_LEVELSETS 4

/* scalar slots per particle (data_structures.hpp:16-21) */
enum { MTR_SCALAR_EPS_PL_DEV = 0, MTR_SCALAR_EPS_PL_VOL, MTR_SCALAR_EPS_PL_VOL_PRADHANA,
       MTR_SCALAR_DELTA_GAMMA, MTR_SCALAR_VISCOSITY, MTR_SCALAR_MUI, MTR_NUM_SCALARS };

/* MTR_PREC_FP64: the reference's double precision throughout.
 * MTR_PREC_MIXED: particle velocity, deformation gradient (kept as F - I),
 * affine matrix, stress and plastic scalars, the grid channels and the
 * transfers in FP32; positions, the clock, the deformation update, the SVD,
 * the Hencky log/exp, the return mapping and the balances in FP64.  The ABI
 * is FP64 on both paths. */
enum mtr_precision { MTR_PREC_FP64 = 0, MTR_PREC_MIXED = 1 };

/* Public fields of Simulation (simulation.hpp:28-106) that the step reads,
 * plus the compile-time choices of tools.hpp:19-21 (dim, spline degree) that
 * become run-time fields here. */
typedef struct mtr_params {
  int32_t dim;              /* 2 or 3 (tools.hpp:20 THREEDIM)                    */
  int32_t spline_deg;       /* 2 or 3 (tools.hpp:21 SPLINEDEG)                   */
  int32_t precision;        /* enum mtr_precision                                */
  int32_t elastic_model;    /* enum mtr_elastic_model                            */
  int32_t plastic_model;    /* enum mtr_plastic_model                            */
  int32_t hardening_law;    /* enum mtr_hardening_law                            */
  int32_t use_pradhana, use_mises_q, use_mibf, use_musl;
  int32_t gravity_special;
  int32_t pbc;              /* periodic in x over [0, L[0]] (pbc.cpp, remesh.cpp:14-36) */
  uint32_t end_frame;
  int32_t change_particle_positions; /* hard-coded teleport hook, position_update.cpp:35-41 */
  double fps, cfl, cfl_elastic, flip_ratio, rho, gravity_time;
  double gravity[3];
  double grid_reference_point[3];
  double dx, particle_mass, particle_volume;
  double E, nu, stress_tolerance, xi;
  double q_max, q_min, p_min;
  double M, q_cohesion;
  double perzyna_exp, perzyna_visc;
  double beta, p0;
  double rho_s, grain_diameter, I_ref, mu_1, mu_2;
  double L[3];              /* Lx, Ly, Lz: the periodic box of pbc (simulation.hpp:60-66) */
} mtr_params;

/* ObjectPlate state (object_plate.hpp:13-24, 136-190). v_object[2] unused in 2D. */
typedef struct mtr_plate {
  int32_t plate_type;       /* enum mtr_plate_type */
  int32_t bc;               /* enum mtr_bc         */
  double friction;
  double pos_object, pos_lower, pos_upper;
  double v_object[3];
  double v_object_original[3];
  double vmin_factor, load_factor;
} mtr_plate;

typedef struct mtr_object {
  int32_t kind;             /* enum mtr_object_kind */
  int32_t bc;               /* enum mtr_bc          */
  double friction;
  double prm[24];
} mtr_object;

typedef struct mtr_clock {
  double time;              /* simulated time after the last completed step      */
  double dt;                /* dt of the last completed step                      */
  uint32_t step;            /* current_time_step                                  */
  uint32_t frame;
  int32_t done;             /* 1 once final_time is reached (simulation.cpp:191)  */
  int32_t reserved;
} mtr_clock;

typedef struct mtr_ctx mtr_ctx;
typedef struct mtr_batch mtr_batch;

/* Validates the parameters and derives the constants of Simulation::simulate
 * (simulation.cpp:94-136: Lame constants, dt_max, prefactors, apicDinverse,
 * fac_Q).  Replaces the constant block at the top of simulate(). */
int mtr_ctx_create(const mtr_params* params, int device, mtr_ctx** out);

/* Copies the particle state in (replaces the host-side Particles arrays the
 * reference mutates in place, data_structures.hpp:8-47).  Any of v, F, B,
 * scalars may be NULL (zero velocity, identity F, zero B, zero scalars; filled
 * on the device, nothing is copied for them).  With use_mibf the muI slot is
 * initialised as simulate() does (simulation.cpp:138-145).  Pinned host arrays
 * are copied directly; pageable ones through two pinned 8 MB staging chunks
 * per device, so that a long copy leaves the driver and the copy engine free
 * between chunks for other threads' work (a batch stepping beside it).
 * mtr_download copies back the same way. */
int mtr_upload(mtr_ctx* ctx, const double* x, const double* v, const double* F, const double* B,
               const double* scalars, uint32_t Np);

/* Replaces the plate and object lists (simulation.hpp:109-110). */
int mtr_set_objects(mtr_ctx* ctx, const mtr_plate* plates, int n_plates,
                    const mtr_object* objects, int n_objects);

/* Dense level set for MTR_OBJ_LEVELSET objects (the grid an ObjectVdb samples,
 * object_vdb.hpp:17-94, baked to a dense lattice; OpenVDB itself is not
 * used).  phi: signed distance (negative inside) at origin + (i, j, k) *
 * spacing, dims[0] x dims[1] x dims[2] samples (dims[2] = 1 in 2D), stored
 * like grid nodes: index (i * dims[1] + j) * dims[2] + k.  normals: NULL to
 * use the central-difference gradient of phi, or 3 floats per sample (a
 * baked normal field).  Samples outside the lattice read phi = 3 * spacing
 * (an OpenVDB narrow-band background) and a zero gradient.  Slots
 * 0..MTR_MAX_LEVELSETS-1; a slot may be replaced at any time between steps. */
int mtr_set_levelset(mtr_ctx* ctx, int slot, const float* phi, const float* normals, const uint32_t dims[3],
                     const double origin[3], double spacing);

/* Advances up to nsteps calls of Simulation::advanceStep (simulation.cpp:219-273)
 * including the time/frame bookkeeping of simulate() (simulation.cpp:176-200);
 * stops early once the final time is reached.  Asynchronous on the context's
 * stream except for a status read every `nsteps` steps. */
int mtr_step(mtr_ctx* ctx, int nsteps);

/* Runs Simulation::simulate's loop (simulation.cpp:168-201) to the end. */
int mtr_run(mtr_ctx* ctx);

/* Runs steps until the frame counter advances (the point where simulate()
 * saves a frame, simulation.cpp:180-190) or the simulation ends;
 * *frame_done = 1 when a frame was completed. */
int mtr_run_frame(mtr_ctx* ctx, int* frame_done);

/* Copies the particle state back in the original particle order (any pointer
 * may be NULL).  Also returns pic and flip of the last step if requested. */
int mtr_download(mtr_ctx* ctx, double* x, double* v, double* F, double* B, double* scalars);
int mtr_download_pic_flip(mtr_ctx* ctx, double* pic, double* flip);

/* Grid of the last completed step (Simulation::grid, data_structures.hpp:49-66):
 * dims[0..2] = Nx, Ny, Nz (Nz = 1 in 2D); axis coordinates; mass, v, flip in
 * the reference's node order ind = (i*Ny + j)*Nz + k (simulation.hpp:196-204).
 * Pass NULL for arrays to query dims only. */
int mtr_get_grid(mtr_ctx* ctx, uint32_t dims[3], double* gx, double* gy, double* gz,
                 double* mass, double* v, double* flip);

/* Cell keys and stable sort order of the last step's particle sort, both in
 * the particle order of the sort's input, for bit-exact checks. */
int mtr_get_sort(mtr_ctx* ctx, uint32_t* keys_in_input_order, uint32_t* sorted_input_index,
                 uint32_t* input_particle_id);

int mtr_get_plates(mtr_ctx* ctx, mtr_plate* plates, int n_plates);
int mtr_get_clock(mtr_ctx* ctx, mtr_clock* clock);

/* Device status word (bit flags MTR_STATUS_*) and the first particle (original
 * id) that raised one.  The reference's analogue is the int exit flag
 * (simulation.hpp:28) polled once per step (simulation.cpp:176-177). */
int mtr_status(mtr_ctx* ctx, uint32_t* flags, uint32_t* first_bad);
int mtr_clear_status(mtr_ctx* ctx);

/* Bounded wait for the context's stream (polls cudaEventQuery). */
int mtr_sync(mtr_ctx* ctx, double timeout_seconds);

/* The context's CUDA stream (cudaStream_t as an opaque pointer) for timing. */
void* mtr_stream(mtr_ctx* ctx);

/* Number of kernel launches issued by the last mtr_step call. */
int64_t mtr_launch_count(mtr_ctx* ctx);

/* Test and timing controls (no counterpart in the reference):
 * mtr_keep_pic_flip makes the step keep each particle's pic and flip vectors
 * (Particles::pic/flip, data_structures.hpp:12-13) for mtr_download_pic_flip;
 * mtr_use_graphs turns CUDA-graph replay of the step on (default) or off. */
int mtr_keep_pic_flip(mtr_ctx* ctx, int on);
int mtr_use_graphs(mtr_ctx* ctx, int on);

/* Timing support (no counterpart in the reference, whose per-phase timers are
 * timer.hpp:6-29 around simulation.cpp:240-267): runs nsteps steps with direct
 * launches and a CUDA event after every launch, and returns the mean device
 * time of each launch slot of a step (slot_ms, slot_names; up to max_slots;
 * *nslots = slots per step).  mtr_active_nodes counts grid nodes with mass
 * in the last step. */
int mtr_profile(mtr_ctx* ctx, int nsteps, double* slot_ms, const char** slot_names, int max_slots, int* nslots);
int mtr_active_nodes(mtr_ctx* ctx, uint64_t* active, uint64_t* total);

/* Mass and momentum balance of the last step, in FP64 on both paths
 * (Simulation::checkMassConservation / checkMomentumConservation,
 * simulation.cpp:292-333): total grid mass and momentum right after P2G, and
 * the particles' total mass and momentum (particle_mass * sum of v) before
 * it.  Momenta are dim values. */
int mtr_balance(mtr_ctx* ctx, double* grid_mass, double* grid_momentum, double* particle_mass,
                double* particle_momentum);

/* Batched stepping — no counterpart in the reference, which runs one
 * Simulation per process.  A batch advances several uploaded contexts on one
 * GPU together: contexts with the same dim, spline degree, precision and
 * USL/MUSL choice form a group, and every phase of a step is one kernel launch
 * for the whole group over a device table of the members' buffers, captured
 * in a CUDA graph.  Each member keeps its own clock, grid, regrowth and end of
 * simulation; mtr_batch_step(batch, n) advances every member by n steps (or to
 * its end) and returns when all are there.  Members stay ordinary contexts
 * (mtr_download, mtr_get_clock, mtr_status ... work as before), but must not
 * be stepped on their own while the batch exists.  mtr_batch_destroy leaves
 * the members alive.
 *
 * mtr_footprint estimates the device bytes mtr_upload will allocate for Np
 * particles at positions x (AoS) with these parameters, for admission by
 * memory budget; the grid may later grow with the scene. */
/* mtr_set_step_limit: the context takes no step past step number last_step
 * (steps counted from mtr_upload; 0xffffffff = no limit, the default).  Both
 * mtr_step and mtr_batch_step stop there, so a batch member that needs fewer
 * steps than the others ends exactly on time. */
int mtr_set_step_limit(mtr_ctx* ctx, uint32_t last_step);
int mtr_batch_create(mtr_ctx* const* ctxs, int n, mtr_batch** out);
/* Replaces the members of a batch (no counterpart in the reference): the
 * batch keeps its stream, the block shapes of every group whose key stays in
 * use and its instantiated step graph, which the next mtr_batch_step updates
 * in place when the launch sequence is unchanged (same groups and radix
 * passes) instead of instantiating it again.  A serving loop calls it when
 * scenes join or leave.  Members that leave stay alive. */
int mtr_batch_set_members(mtr_batch* batch, mtr_ctx* const* ctxs, int n);
/* How many batch rebuilds updated the instantiated graph in place. */
int mtr_batch_graph_updates(mtr_batch* batch);
int mtr_batch_step(mtr_batch* batch, int nsteps);
int64_t mtr_batch_launch_count(mtr_batch* batch);
/* Host-side bookkeeping of mtr_batch_step since mtr_batch_create: members'
 * grid regrowths and the wall milliseconds they took, and batch rebuilds
 * (device tables and graph capture) and theirs.  Any pointer may be NULL. */
int mtr_batch_stats(mtr_batch* batch, int64_t* regrowths, double* regrow_ms, int64_t* rebuilds, double* rebuild_ms);
void* mtr_batch_stream(mtr_batch* batch);
void mtr_batch_destroy(mtr_batch* batch);
int mtr_footprint(const mtr_params* params, uint32_t Np, const double* x, uint64_t* bytes);

/* Frame output (Simulation::saveParticleData, save_data.cpp:7-171).
 * mtr_frame_begin enqueues, behind the steps already issued, a kernel that
 * writes one row of FP64 columns per particle in the original particle order
 * — the columns of the reference's particle file, in its order:
 *   x y [z] vx vy [vz] p q Je [eps_pl_vol eps_pl_dev delta_gamma] [muI] [viscosity]
 * (p = -tr(tau)/dim, q = sqrt(c tau_dev:tau_dev), c = 3/2 with use_mises_q
 * else 1/2, Je = det F; the plastic triple with any plastic model, muI with
 * DPVisc/MCCVisc and use_mibf or a mu(I) model, viscosity with a mu(I)
 * model) — and copies them to pinned host memory on a second stream.  It
 * returns at once: the context can go on stepping while the copy runs and the
 * caller writes the previous file.  mtr_frame_wait waits (bounded) for that
 * copy and returns the rows (valid until the next mtr_frame_begin), their
 * count and width, and the clock of the snapshot.  mtr_frame_columns writes
 * the column names (static strings) and returns their number.
 * mtr_get_grid_friction: the grid friction of the last step (Grid::friction,
 * use_mibf only; the grid file's `friction` column, save_data.cpp:247-255). */
int mtr_frame_columns(mtr_ctx* ctx, const char** names, int max_names);
int mtr_frame_begin(mtr_ctx* ctx);
int mtr_frame_wait(mtr_ctx* ctx, double timeout_seconds, const double** rows, uint32_t* n, int* ncols,
                   mtr_clock* clock);
int mtr_get_grid_friction(mtr_ctx* ctx, double* friction);

/* Block shapes of the tile kernels — no counterpart in the reference, whose
 * loops are OpenMP-scheduled over particles.  Each step phase that walks the
 * particles of a grid tile runs one thread block per tile; its size is chosen
 * per context (or per batch group) among 64, 128 and 256 threads, by slot:
 *   threads[MTR_TILE_P2G]     P2G with the stress force (default 128)
 *   threads[MTR_TILE_MUSL]    MUSL G2P and re-scatter (default 128)
 *   threads[MTR_TILE_G2P]     USL G2P, deformation update, return mapping (64..128)
 *   threads[MTR_TILE_DEFGRAD] MUSL deformation update, return mapping (default 128)
 * Results do not depend on the shapes beyond the order of floating-point
 * atomic sums.  mtr_autotune times `reps` rounds of trial steps of the
 * context's current state with each candidate shape and keeps the fastest
 * per slot (a slot keeps its shape unless another is more than 2% faster).
 * A trial step runs every kernel of a step except the commit, so the particle
 * state, the clock, the plates and the counters are the same afterwards; a
 * grid that must grow is grown as the next step would.  A context that has
 * ended keeps its shapes.  mtr_batch_autotune does the same for every group of
 * a batch at once; mtr_batch_get_group reports a group's key, size and shapes.
 * Groups start with the shapes of their first member. */
#define MTR_TILE_P2G 0
#define MTR_TILE_MUSL 1
#define MTR_TILE_G2P 2
#define MTR_TILE_DEFGRAD 3
typedef struct mtr_group_info {
  int32_t dim, spline_deg, fp32, musl;
  int32_t plastic_model_kernel; /* model the return mapping is compiled for, -1: any */
  int32_t members;
  int32_t tile_threads[4];
  int32_t tile_lanes[2];        /* lanes per particle of the P2G and MUSL scatters */
} mtr_group_info;
int mtr_autotune(mtr_ctx* ctx, int reps, int* threads /* [4] out, may be NULL */);
int mtr_set_tile_threads(mtr_ctx* ctx, const int* threads /* [4] */);
int mtr_get_tile_threads(mtr_ctx* ctx, int* threads /* [4] */);
/* Lanes per particle of the two scatters, lanes[0] P2G and lanes[1] MUSL: the
 * warp lanes that share one particle's stencil (3D: 16, each lane one (y, z)
 * column of 4 x nodes, or 32, each lane 2 of a column's x nodes; 2D: 4 or 8).
 * A warp scatters 32 / lanes particles at a time.  mtr_autotune tunes them
 * with the block sizes (candidates 64/128/256 threads x both lane counts). */
int mtr_set_tile_lanes(mtr_ctx* ctx, const int* lanes /* [2] */);
int mtr_get_tile_lanes(mtr_ctx* ctx, int* lanes /* [2] */);
int mtr_batch_set_tile_lanes(mtr_batch* batch, int group, const int* lanes /* [2] */);
int mtr_batch_autotune(mtr_batch* batch, int reps);
/* Re-tuning as scenes spread: with reps > 0, mtr_batch_step tunes the batch
 * again (mtr_batch_autotune with reps repetitions, inside the call) when a
 * group's members together hold more than twice the grid nodes they held at
 * the last tune; reps = 0 (the default) turns it off.  A membership change
 * (mtr_batch_set_members) takes the next step's grid size as the new
 * baseline.  A re-tune costs about as many batched steps as a tune, so a
 * latency-bound caller (a serving loop with cached shapes) leaves it off.
 * mtr_batch_retunes counts the re-tunes so far. */
int mtr_batch_set_retune(mtr_batch* batch, int reps);
int mtr_batch_retunes(mtr_batch* batch);
/* The clocks of the members (in mtr_batch_create order) as of the end of the
 * last mtr_batch_step, without a device round trip; returns the member count. */
int mtr_batch_clocks(mtr_batch* batch, mtr_clock* clocks, int n);
int mtr_batch_groups(mtr_batch* batch);
int mtr_batch_get_group(mtr_batch* batch, int group, mtr_group_info* info);
int mtr_batch_set_tile_threads(mtr_batch* batch, int group, const int* threads /* [4] */);

/* mtr_p2g_noalloc — no counterpart in the reference.  The particle-to-grid
 * transfer (the P2G of p2g.cpp: grid mass = particle mass * sum of weights,
 * grid velocity = sum of w (v_p + B_p D^-1 (x_i - x_p)) / sum of w) of one
 * particle set onto a grid the caller describes, for callers that cannot
 * allocate device memory where they call it: code being captured into a CUDA
 * graph, solvers living inside a framework that owns all device memory
 * through its own pool, real-time loops that must not risk an allocation.
 * Nothing is allocated: the sort, tile and accumulator scratch lives in one
 * fixed device array (~10 MB, held by every GPU that loads the library until
 * exit).  Inputs and outputs are device pointers the caller owns:
 *   x, v  [dim][Np] component-major; B [dim*dim][Np], entry (r,c) at r*dim+c
 *         (read only when params->flip_ratio < 0); gx, gy, gz the node
 *         coordinates per axis (gz unused in 2D), uniformly spaced at
 *         params->dx (tiles and stencils are located from gx[0], gy[0],
 *         gz[0] and 1/dx; other spacings deposit wrongly);
 *         dims = nodes per axis (host);
 *   grid_mass [G], grid_v [dim][G] with G = dims product, node order
 *         (i*Ny + j)*Nz + k;
 *   status  optional (NULL: not written): one device uint32_t that receives
 *         this call's MTR_STATUS_* word, written in stream order after the
 *         transfer (no host synchronisation needed, readable by later work
 *         on the stream).  MTR_STATUS_STENCIL_OOB means some particles were
 *         dropped: those whose cell lies outside the grid, whose position is
 *         not finite, or whose stencil reaches past the last node.  The
 *         remaining particles are deposited exactly as if the dropped ones
 *         were absent.
 * Uses params->dim, spline_deg, dx, flip_ratio, particle_mass.  Runs on
 * `stream` (cudaStream_t; NULL = legacy default stream) and returns without
 * synchronising.  More than MTR_NOALLOC_MAX_PARTICLES particles or
 * MTR_NOALLOC_MAX_NODES nodes returns MTR_ERR_TOO_LARGE.  All calls share the
 * scratch array: calls that overlap on the GPU race.  The first call on each
 * device looks the array up (cudaGetSymbolAddress) and must not be inside a
 * stream capture. */
#define MTR_NOALLOC_MAX_PARTICLES (1u << 18)
#define MTR_NOALLOC_MAX_NODES (1u << 17)
int mtr_p2g_noalloc(const mtr_params* params, const double* x, const double* v, const double* B, uint32_t Np,
                    const double* gx, const double* gy, const double* gz, const uint32_t dims[3], double* grid_mass,
                    double* grid_v, uint32_t* status, void* stream);

void mtr_ctx_destroy(mtr_ctx* ctx);

/* Last error message of this thread (static storage). */
const char* mtr_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* MATTER_GPU_H */
