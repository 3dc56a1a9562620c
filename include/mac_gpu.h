/* C-ABI of the B200 implementation of Mac's per-timestep fluid hot path.
 *
 * Plain C types only: a host program (or the C++ policy wrappers in
 * include/mac_gpu/) hands the world over through mac_host_state, runs the
 * reference's algorithms on the device, and reads the world back. Each entry
 * point replaces one reference algorithm or policy; the comment above it names
 * the reference interface (file:line, relative to the reference repository).
 *
 * Every function returns MAC_OK (0) or a negative MAC_ERR_* status; nothing
 * aborts. A context owns one CUDA stream and its device memory; calls on one
 * context must not overlap (not thread-safe per context).
 */
#ifndef MAC_GPU_H
#define MAC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  MAC_OK = 0,
  MAC_ERR_INVALID = -1,       /* bad argument or state */
  MAC_ERR_CUDA = -2,          /* a CUDA call failed */
  MAC_ERR_CAPACITY = -3,      /* brick pool, particle array or hash table full */
  MAC_ERR_NOT_CONVERGED = -4, /* iterative solve hit max_iters */
  MAC_ERR_NO_DEVICE = -5,     /* no CUDA device */
  MAC_ERR_OUT_OF_MEMORY = -6,
  MAC_ERR_TIMEOUT = -7,
  MAC_ERR_MATRIX = -8         /* matrix not of the form the solver handles */
};

/* Pressure solver of the projection. */
enum {
  MAC_SOLVER_MGPCG_FP64 = 0,  /* plain form: FP64 multigrid-preconditioned CG */
  MAC_SOLVER_MGPCG_MIXED = 1, /* FP32 multigrid inside FP64 CG */
  MAC_SOLVER_CG_FP64 = 2,     /* Jacobi-preconditioned CG (reference for the others) */
  MAC_SOLVER_LEARNED = 3,     /* flexible CG with the learned preconditioner (mac_set_preconditioner_net);
                                 FP64 MG-PCG takes over when it stalls */
  MAC_SOLVER_LEARNED_MIXED = 4 /* the same, with the FP32 multigrid as the fall-back */
};

/* Cell materials, as Data_CellType_Fluid_Air_Solid_Inflow::MaterialToInt
 * (src/Data_CellType_Fluid_Air_Solid_Inflow.tpp:3-18); interior is the fifth
 * material of Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres
 * (src/Data_CellType_Fluid_Air_Solid_Inflow_Interior_0_Pres.tpp:3-22), used
 * by the depth composition only. */
enum { MAC_CELL_AIR = 0, MAC_CELL_FLUID = 1, MAC_CELL_SOLID = 2, MAC_CELL_INFLOW = 3, MAC_CELL_INTERIOR = 4 };
/* Per-cell flag bits: const faces x/y/z (src/Data_Grid_Speed.h:54-59) and the
 * no-delete mark (src/Data_CellType_Fluid_Air_Solid_Inflow.h:331-338). */
enum { MAC_FLAG_CONST_X = 1, MAC_FLAG_CONST_Y = 2, MAC_FLAG_CONST_Z = 4, MAC_FLAG_NODELETE = 8 };

#define MAC_BRICK_EDGE 8
#define MAC_BRICK_CELLS 512

typedef struct {
  double h[3];          /* cell spacing (Data_Grid_Base_Spacing::m_h) */
  double cfl_factor;    /* Data_Timing_Time::m_factor */
  double dt_min, dt_max;/* Policy_CheckDT(min, max) */
  double gravity;       /* Policy_Gravity(g, axis) */
  int32_t gravity_axis; /* 1..3 */
  int32_t layer_max;    /* Policy_Layer_Max */
  int32_t interp_symmetric; /* 1: Policy_Speed_Interpolation_Linear_Symmetric, 0: _Linear */
  int32_t solver;       /* MAC_SOLVER_* */
  double rtol;          /* relative residual target of the projection solve */
  int32_t max_iters;
  int32_t warm_start;   /* 1: start the solve from the last pressure */
  int64_t max_bricks;   /* device brick pool capacity (8^3 cells each) */
  int64_t max_particles;
  int32_t device;
  int32_t div_check;    /* 1: compute max |div| after each projection */
  /* Kinematic viscosity (Data_Grid_Base::m_viscosity). 0 runs the inviscid
   * composition (Algorithms_Gravity + Algorithms_Convection, Algorithms_Solve_Pressure);
   * > 0 adds Algorithms_Viscosity with Policy_Laplacian_Speed and
   * Policy_Viscosity_Apply_If to the forces and projects with
   * Algorithms_Solve_Pressure_Dirichlet + Policy_Dirichlet_Boundary
   * (src/Algorithms_Viscosity.h:24-30, src/Algorithms_Solve_Pressure_Dirichlet.h:171-233). */
  double viscosity;
  /* 1: the depth composition of the topology (test/Jet3.cpp:519-549):
   * Algorithms_Initialize_Layer_And_Depth, _Layer_Initial_With_Particle_Depth,
   * _Create_Fluid_Particle_Depth and _Update_CellType_Layer_Depth with
   * Policy_Depth(depth_max, depth_interior, depth_remove) in place of the four
   * pipeline-A topology passes; cells get a depth and the interior material. */
  int32_t depth_mode;
  int32_t depth_max, depth_interior, depth_remove;
  /* inflow (and interior) refill: 0 = 8 jittered particles per cell,
   * n >= 1 = Policy_Add_Particle_Cube(n), (2n+1)^3 particles per cell */
  int32_t refill_cube;
  /* 0: pipeline A, the step of test/TestJetDEau_Basic.cpp:434-441 (RK2-TVD,
   * extrapolation, particle RK4); 1: pipeline B, the step of test/Jet3.cpp:713-726
   * (per-step init with the extrapolation, then Algorithms_RungeKutta_all over
   * grid and particles with the topology re-run, the force projection and the
   * extrapolation of the acceleration at every stage); needs depth_mode. */
  int32_t pipeline;
} mac_params;

/* Host view of a world, arrays owned by the caller. Brick b holds cells
 * key = 8*keys[b] + (x, y, z), slot x + 8y + 64z (src/Offset.h:14-24). All 512
 * slots of a live brick are carried, existing or not: the reference keeps the
 * data of erased cells of a live chunk (src/ChunkHashTable.tpp:62-87,132-147). */
typedef struct {
  int64_t nbricks, nparticles;
  int32_t* keys;        /* [nbricks][3] */
  uint8_t* exists;      /* [nbricks*512] */
  double* u[2][3];      /* two speed buffers (src/Data_Chunk_Speed.h:13) */
  double* acc[3];       /* acceleration buffer */
  double* p;            /* pressure */
  /* Any of u[1][*], acc[*] and p may be NULL: that field is left out of the
   * transfer (upload zeroes it on the device, download skips it). Pipeline A's
   * step writes speed buffer 1 and the acceleration before it reads them
   * (RK2-TVD's stage buffers, src/Algorithms_RungeKutta_RK2_TVD.h:25-55) and
   * the pressure of every existing cell (read first only with warm_start), so
   * a caller that does not look at them need not move them. */
  uint8_t* flags;       /* MAC_FLAG_* */
  uint8_t* type;        /* MAC_CELL_* */
  int32_t* layer;       /* -1 empty */
  double* pos;          /* [nparticles][3] */
  double t, dt;
  uint64_t step;        /* refill seed counter */
  int32_t* depth;       /* [nbricks*512] distance to the surface, -1 empty
                           (src/Data_Grid_Depth_Empty.h:6-14); NULL: not carried */
} mac_host_state;

typedef struct {
  int32_t iterations;   /* CG iterations of the last solve */
  int32_t solves;
  double relres;        /* final relative residual of the last solve */
  double max_div;       /* max |div u| over domain cells after the last projection */
  int64_t fluid_cells;  /* fluid + inflow (+ interior) cells after the last topology rebuild */
  int64_t unknowns;     /* in-domain cells of the last system */
  int64_t live_bricks;
  int64_t particles;
  int64_t total_iterations; /* accumulated over the context's life */
  int32_t learned_iterations; /* iterations of the last solve with the learned preconditioner */
  int32_t fallbacks;          /* solves (over the context's life) where MG-PCG took over */
} mac_stats;

/* ---- context ---- */
void mac_default_params(mac_params* p);
int mac_ctx_create(const mac_params* p, void** ctx);
int mac_ctx_destroy(void* ctx);
int mac_get_stats(void* ctx, mac_stats* out);
const char* mac_error_string(int code);

/* ---- state transfer (host <-> device), cf. the chunk grid src/ChunkHashTable.h:22-160 ---- */
int mac_upload_state(void* ctx, const mac_host_state* s);
int mac_query_sizes(void* ctx, int64_t* nbricks, int64_t* nparticles);
int mac_download_state(void* ctx, mac_host_state* s);
/* One FP64 cell field of every live brick, [nbricks][512] in the brick order of
 * mac_download_state (the order of the last mac_upload_state until a topology pass
 * runs): for host integrators that keep the world on the host and project on the
 * device (Algorithms_Solve_Pressure_GPU in include/mac_gpu/Mac_GPU.h). */
enum { MAC_FIELD_U0X = 0, MAC_FIELD_U0Y, MAC_FIELD_U0Z, MAC_FIELD_U1X, MAC_FIELD_U1Y, MAC_FIELD_U1Z,
       MAC_FIELD_AX, MAC_FIELD_AY, MAC_FIELD_AZ, MAC_FIELD_P };
int mac_upload_field(void* ctx, int field, const double* data);
int mac_download_field(void* ctx, int field, double* data);

/* ---- topology rebuild: Algorithms<Initialize_MacCell, Layer_Initial_With_Particle,
 *      Create_Fluid_Particle, Update_CellType_Layer, Delete_MacCell, Calculate_Time_Step>
 *      (test/TestJetDEau_Basic.cpp:325-326) ---- */
/* src/Algorithms_Initialize_MacCell.h:15-21; depth_mode: src/Algorithms_Initialize_Layer_And_Depth.h:16-33 */
int mac_initialize_maccell(void* ctx);
/* src/Algorithms_Layer_Initial_With_Particle.h:20-34 + Policy_Particle_To_Key (src/Policy_Particle_To_Key.h:24-35);
 * depth_mode: src/Algorithms_Layer_Initial_With_Particle_Depth.h:26-47 (removes particles of deep interior cells) */
int mac_layer_initial_with_particle(void* ctx);
/* src/Algorithms_Create_Fluid_Particle.h:19-33 (refill: 8 jittered particles, or
 * Policy_Add_Particle_Cube(refill_cube)); depth_mode: src/Algorithms_Create_Fluid_Particle_Depth.h:21-43 */
int mac_create_fluid_particle(void* ctx);
/* src/Algorithms_Update_CellType_Layer.h:22-89; depth_mode: src/Algorithms_Update_CellType_Layer_Depth.h:24-138
 * with Policy_Depth (src/Policy_Depth.h:12-26) */
int mac_update_celltype_layer(void* ctx);
/* src/Algorithms_Delete_MacCell.h:22-44 */
int mac_delete_maccell(void* ctx);
/* src/Algorithms_Calculate_Time_Step.h:35-66 + Policy_CheckDT (src/Policy_CheckDT.h:16-29) */
int mac_calculate_time_step(void* ctx, double* dt);
/* The whole init sequence above, in the reference's order. Increments the refill seed first. */
int mac_topology_rebuild(void* ctx);

/* ---- advection and projection ---- */
/* acc = 0; Algorithms_Gravity + Algorithms_Convection with Policy_Upwind_1_Order on speed buffer
 * ispeed (src/Algorithms_Gravity.h:15-28, src/Algorithms_Convection.h:18-37) */
int mac_forces(void* ctx, int ispeed);
/* Algorithms_Do_Pressure::Do on speed buffer ispeed: Init_Iteration + Divergence_Projection +
 * End_Iteration of Algorithms_Solve_Pressure (src/Algorithms_Do_Pressure.h:16-21,
 * src/Algorithms_Solve_Pressure.h:44-222) */
int mac_pressure_project(void* ctx, int ispeed);
/* Algorithms_Solve_Pressure at its composable interface, the three member
 * functions the reference's integrators call through Policy::
 * (src/Algorithms_Solve_Pressure.h:44,158,168; src/Algorithms_RungeKutta_RK2_TVD.h:29,50,60-61;
 * src/Algorithms_Do_Pressure.h:16-21):
 * - mac_pressure_init = Init_Iteration: numbers the domain cells' system from the
 *   current cell types, existence and const faces (face classes, multigrid set-up);
 * - mac_pressure_divergence_projection = Divergence_Projection on the system of the
 *   last init: divergence of speed buffer ispeed (accel = 1: of the acceleration,
 *   Speed_GetRef() with SetAccel_Instead_Speed(true), src/Data_Chunk_Speed.h:164-171,
 *   with the viscous Dirichlet pressures read from speed buffer ispeed), solve,
 *   pressure write-back, gradient correction; MAC_ERR_INVALID without an init;
 * - mac_pressure_end = End_Iteration: drops the system.
 * A topology pass between init and end invalidates the system (re-init). */
int mac_pressure_init(void* ctx);
int mac_pressure_divergence_projection(void* ctx, int ispeed, int accel);
int mac_pressure_end(void* ctx);
/* Algorithms_RungeKutta_RK2_TVD::Do with Policy = Algorithms<Gravity, Convection> +
 * Algorithms_Solve_Pressure (src/Algorithms_RungeKutta_RK2_TVD.h:20-66) */
int mac_rk2tvd(void* ctx);
/* src/Algorithms_RungeKutta_all.h:35-156 with the policy of test/Jet3.cpp:642-675
 * (pipeline B only: mac_params.pipeline = 1): four stages of topology, forces,
 * force projection and extrapolation, moving grid speeds and particles */
int mac_rungekutta_all(void* ctx);
/* src/Algorithms_Extrapolate.h:25-233 */
int mac_extrapolate(void* ctx);
/* Algorithm_Extrapolate_Boundary_Condition, 3D form, with Policy_Is_In_Domain_Speed
 * (src/Algorithm_Extrapolate_Boundary_Condition.h:454-975, src/Policy_Is_In_Domain_Speed.h:15-48)
 * on speed buffer ispeed: the reference's output-time stage (test/Lateral_jet_3.cpp:706-711).
 * The reference visits its hash map's order, on which its result depends; the device
 * visits the boundary cells by colour (key x, y, z mod 5), one colour at a time, the
 * three-face corners last in reverse colour order: a fixed order whose result the oracle
 * reproduces bit for bit. */
int mac_extrapolate_boundary_condition(void* ctx, int ispeed);
/* Algorithms_Move_Particles + Policy_Advance_Ode_RungeKutta + Get_Speed
 * (src/Algorithms_Move_Particles.h:22-36, src/Policy_Advance_ODE_RungeKutta.h:14-27,
 * src/Policy_Speed_Interpolation_Linear_Symmetric.h:79-119 or src/Policy_Speed_Interpolation_Linear.h:64-106) */
int mac_move_particles(void* ctx);
/* One full step of test/TestJetDEau_Basic.cpp:434-441: topology rebuild, RK2-TVD,
 * extrapolation, particle move, t += dt. */
int mac_step(void* ctx);
/* Synchronises the context's stream. */
int mac_sync(void* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work on it. */
int mac_stream(void* ctx, void** stream);
/* Number of kernels the context has launched so far. */
int mac_launch_count(void* ctx, int64_t* count);

/* Per-phase device timing with CUDA events on the context's stream (the
 * reference's per-algorithm times() prints, e.g. src/Algorithms_Convection.h:20-36).
 * mac_get_profile returns and resets the accumulated milliseconds and the
 * number of timed regions per phase. */
enum {
  MAC_PHASE_TOPOLOGY = 0, MAC_PHASE_FORCES, MAC_PHASE_SETUP, MAC_PHASE_DIVERGENCE, MAC_PHASE_SPMV,
  MAC_PHASE_CGVEC, MAC_PHASE_VCYCLE, MAC_PHASE_GRADIENT, MAC_PHASE_EXTRAPOLATE, MAC_PHASE_MOVE, MAC_NPHASES
};
int mac_set_profiling(void* ctx, int on);
int mac_get_profile(void* ctx, double* ms, int64_t* count, int nphase);

/* ---- drop-in linear solver: the Policy_Solve_Linear_Umfpack member functions
 * (src/Policy_Solve_Linear_Umfpack.h:28-70) over the CSC arrays the reference assembles
 * in Algorithms_Solve_Pressure::Init_Iteration (src/Algorithms_Solve_Pressure.h:52-152).
 * mac_csc_factorize checks the arrays (MAC_ERR_INVALID: offsets not starting at 0 or
 * decreasing, a row index outside [0, n)) and the matrix's form: the symmetric matrix
 * with a negative diagonal the reference assembles is solved by FP64 Jacobi-PCG on the
 * device; any other matrix (the general LU of Umfpack takes any non-singular one) by
 * FP64 Jacobi-preconditioned BiCGStab on a row-major copy. Both stop at
 * ||b - A x|| <= rtol ||b|| (mac_params.rtol) or return MAC_ERR_NOT_CONVERGED after
 * max_iters or on a breakdown, with x the last finite iterate. ---- */
int mac_csc_factorize(void* ctx, int n, const int* offset, const int* indice, const double* value);
int mac_csc_solve(void* ctx, int n, const double* b, double* x);
int mac_csc_clean(void* ctx);

/* ---- learned preconditioner (no counterpart in the reference) ----
 * A 3-level 3D U-Net (16/32/64 channels, 3x3x3 convolutions, ReLU; BF16
 * weights and activations, FP32 accumulation) mapping a residual and a cell
 * mask (1 fluid, 0 air, -1 solid) on a dense grid to a correction, for the
 * unit-spacing operator; trained on (residual, error) pairs from plain FP64
 * CG iterates. Grids are [n][d][h][w] with x fastest, d, h, w multiples of 4.
 * Parameters are FP32 [layer][tap][cout][cin] + bias, the layout of
 * mac_unet_get_params; tscale is the fixed output scale of the network. */
int mac_unet_create(int device, void** net);
int mac_unet_destroy(void* net);
int mac_unet_nparams(void* net, int64_t* n);
int mac_unet_init(void* net, uint64_t seed);
int mac_unet_get_params(void* net, float* params, float* tscale);
int mac_unet_set_params(void* net, const float* params, float tscale);
/* out = net(r / rms(r), mask) * rms(r) * tscale on fluid cells, 0 elsewhere (host arrays). */
int mac_unet_forward(void* net, int n, int d, int h, int w, const float* r, const int8_t* mask, float* out);
/* loss = mean over fluid cells of (net(r / rms(r), mask) - e / (rms(r) tscale))^2 and its
 * gradient with respect to every parameter (host arrays). */
int mac_unet_loss_grad(void* net, int n, int d, int h, int w, const float* r, const int8_t* mask, const float* e,
                       double* loss, float* grad);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) with the given gradient. */
int mac_unet_adam_step(void* net, const float* grad, float lr);
/* Training set on the device: nmasks random pool + 12 sphere masks on a size^3 grid,
 * each solved by plain FP64 CG for niter iterations from 0; pairs at iterations
 * 1, 2, 4, ... (nsnap). stats[0]: worst final relative residual, stats[1]: tscale. */
int mac_unet_make_dataset(void* net, int nmasks, int size, int nsnap, int niter, uint64_t seed, double* stats);
/* The same with the first nmasks_given masks supplied by the caller (host,
 * nmasks_given x size^3 int8: 1 fluid, 0 air or missing, -1 solid), e.g. patches
 * of jet states; the remaining nmasks - nmasks_given are random as above. */
int mac_unet_make_dataset_ext(void* net, int nmasks, int size, int nsnap, int niter, uint64_t seed,
                              const int8_t* masks, int nmasks_given, double* stats);
int mac_unet_get_sample(void* net, int index, float* r, float* e, int8_t* mask);
/* steps Adam steps on random batches of the training set; losses[steps] (may be NULL). */
int mac_unet_train(void* net, int steps, int batch, float lr, uint64_t seed, float* losses);
/* Training loss: 0 = mean squared error of the correction (default), 1 = its
 * energy norm sum d (M d) / count, d = correction - target, M the unit operator. */
int mac_unet_set_loss(void* net, int kind);
int mac_unet_launch_count(void* net, int64_t* count);
/* Device time of one forward pass (mean over reps, CUDA events) on an n x d x h x w
 * grid and its algorithmic FLOPs (2 taps cin cout per output cell, unpadded channels). */
int mac_unet_time_forward(void* net, int n, int d, int h, int w, int reps, double* ms, double* flops);
/* Kernel of the forward 3x3x3 convolutions: 1 (default) stages each tile's input
 * box with its halo in shared memory once and runs the 27 taps from it; 0 gathers
 * every tap's operand separately (the kernel the backward pass shares). Both
 * accumulate in the same order. */
int mac_unet_set_conv(void* net, int staged);

/* Attaches a network (mac_unet_create) as the preconditioner of the
 * MAC_SOLVER_LEARNED* solvers; NULL detaches it. The context does not own it. */
int mac_set_preconditioner_net(void* ctx, void* net);
/* Weight of the Jacobi step applied after the network (z += omega D^-1 (r - M z));
 * 0 turns it off. Default 0.8. */
int mac_set_learned_smoothing(void* ctx, double omega);

/* Multigrid preconditioner of the MG-PCG solvers (no counterpart in the
 * reference, which factorises with Umfpack): weighted-Jacobi sweeps before and
 * after the coarse correction on the finest level, 1 or 2 (default 2). One
 * sweep fuses the pre-sweep with the residual's restriction, so a V-cycle
 * reads the fine grid twice instead of four times; the CG iteration count may
 * rise. The preconditioner stays symmetric either way. prefetch = 1 runs the
 * V-cycle's first kernel as resident blocks that prefetch each next brick's CG
 * vectors with asynchronous bulk copies; 0 (default, measured faster on the
 * 256^3 pool and the 256x256x512 jet) runs one block per brick. */
int mac_set_multigrid(void* ctx, int sweeps0, int prefetch);
/* Launch of the pressure solve's CG-loop kernels (the V-cycle, SpMV, vector
 * updates and scalar finishers): on = 1 (default) launches each with
 * programmatic stream serialisation, so its blocks are scheduled while the
 * previous kernel drains and wait on the device for its completion; 0 uses
 * plain stream order. The results are bit-identical either way. */
int mac_set_dependent_launch(void* ctx, int on);
/* mac_step (pipeline A): on = 1 bins the particles by brick and cell on a
 * second stream of the context, started when the first projection's CG loop
 * begins and overlapping the rest of RK2-TVD and the extrapolation (the
 * particles do not move in between); 0 (default) bins them in the move
 * itself. The results are bit-identical either way. On the 256x256x512 jet
 * the binning's memory traffic slows the solve by about what it saves, so the
 * default keeps one stream. With 1, the "move" phase of mac_get_profile holds
 * the RK4 move alone. */
int mac_set_concurrent_binning(void* ctx, int on);
/* The multigrid's dense levels (level 3, one cell per brick, and its
 * coarsenings): levels of more than max_cells cells (at least 64) run as
 * device-wide sweep kernels, the rest in one 1024-thread block that solves the
 * coarsest exactly. Default 1024. */
int mac_set_coarse_block(void* ctx, int max_cells);
/* The multigrid's smoother and coarse operators: weights w1, w2 of the two
 * Jacobi sweeps before and after each coarse correction (on every level), the
 * weight of the single finest-level sweep (mac_set_multigrid(ctx, 1, .)), and
 * the scale of the Galerkin coarse operators (piecewise-constant transfer
 * over-weights them). Two sweeps damp an error component of eigenvalue lambda
 * of D^-1 A (in (0, 2]) by (1 - w1 lambda)(1 - w2 lambda); weights outside
 * (0, 4), or for which that leaves (-1, 1) anywhere on (0, 2], are refused
 * (MAC_ERR_INVALID), as they would break the preconditioner's definiteness. Defaults 0.5711, 1.8216 (the
 * reciprocals of the degree-2 Chebyshev roots on [0.3, 2]), 0.9, 0.6. */
int mac_set_smoother(void* ctx, double w1, double w2, double w_single, double coarse_scale);

/* ---- allocation-free CSC solve (no counterpart in the reference) ----
 * The same FP64 Jacobi-PCG as mac_csc_factorize + mac_csc_solve, for callers
 * that must not allocate device memory: a host program whose device memory is
 * already handed out by its own allocator (a caching allocator that keeps HBM
 * reserved), or a per-step loop that cannot pay for the device-wide
 * synchronisation a cudaMalloc/cudaFree pair can cause. No context is needed.
 *
 * - offset/indice/value (CSC, as mac_csc_factorize), b and x are DEVICE
 *   pointers owned by the caller; x is overwritten (the solve starts from 0).
 * - The matrix must be the symmetric matrix with a negative diagonal that the
 *   reference assembles (the solve is CG); the call checks this on the device
 *   first and returns MAC_ERR_MATRIX otherwise (use mac_csc_factorize for other
 *   matrices). The arrays must form a valid CSC matrix of n columns.
 * - Work vectors live in one fixed device array of MAC_NOALLOC_MAX_N rows per
 *   device; n > MAC_NOALLOC_MAX_N returns MAC_ERR_CAPACITY and touches nothing.
 *   Its reduction slots must be zero before each reduction, and the call clears
 *   them itself, so the caller prepares nothing.
 * - Runs on `stream` (a cudaStream_t, 0 for the legacy stream) on the current
 *   device and returns after the solve has finished (it reads the CG scalars
 *   on the host every iteration).
 * - The first call on a device looks up the array's address with
 *   cudaGetSymbolAddress; the driver then places the array (2.5 MiB) in device
 *   memory, so that first call needs that much free. A call with n = 0 does
 *   only this set-up: make it on each device before handing its memory to
 *   another allocator, and before any stream capture begins on that device.
 * - All calls on one device share the array: two calls in flight at the same
 *   time on one device (other streams or host threads) race and corrupt each
 *   other's result. Serialise them.
 * Stops when ||b - A x|| <= rtol ||b|| (MAC_OK) or after max_iters iterations
 * (MAC_ERR_NOT_CONVERGED); iterations and relres may be NULL. */
#define MAC_NOALLOC_MAX_N 65536
int mac_csc_solve_noalloc(void* stream, int n, const int* offset, const int* indice, const double* value,
                          const double* b, double* x, double rtol, int max_iters, int* iterations,
                          double* relres);

#ifdef __cplusplus
}
#endif
#endif
