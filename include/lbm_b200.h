/*
 * lbm_b200.h -- C ABI of the B200 (sm_100a) lattice-Boltzmann node step.
 *
 * The library replaces the arithmetic of MADDENING's LBMNode
 * (src/maddening/nodes/lbm.py, class LBMNode at lbm.py:531-1036).  It is the
 * surface that an XLA FFI handler (jax.ffi), a torch extension or a ctypes
 * binding calls: POD arguments, device pointers, a CUDA stream, an int status.
 *
 * Conventions
 *  - Every function returns LBM_OK (0) or a negative lbm_status.  The message
 *    of the last failure on the calling thread is read with lbm_last_error().
 *  - No entry point allocates device memory.  Buffers are owned by the caller;
 *    scratch ("workspace") sizes are queried up front.
 *  - Layouts are the reference's: a grid_shape (n0, n1[, n2]) C-ordered array
 *    of cells, populations innermost: f is (*grid_shape, Q), velocity and
 *    force fields are (*grid_shape, D), density/pressure/wall are grid_shape.
 *  - Direction order is the reference's (d3q19 at lbm.py:92-135, d2q9 at
 *    lbm.py:144-169).
 *  - Floating-point buffers are float32, except for plans with storage
 *    LBM_STORE_F64, whose f/force/moment buffers are all float64.
 *  - A plan is immutable after creation; it may be used concurrently from
 *    several threads on different streams.
 */
#ifndef LBM_B200_H_
#define LBM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

typedef struct CUstream_st* lbm_stream_t; /* == cudaStream_t */

typedef enum {
  LBM_OK = 0,
  LBM_ERR_INVALID = -1,     /* bad argument (shape, tau <= 0.5, null ...) */
  LBM_ERR_UNSUPPORTED = -2, /* valid but not implemented for this plan   */
  LBM_ERR_CUDA = -3,        /* a CUDA runtime call failed                 */
  LBM_ERR_WORKSPACE = -4,   /* workspace missing or too small             */
  LBM_ERR_TIMEOUT = -5      /* a bounded device-side wait gave up         */
} lbm_status;

typedef enum { LBM_D2Q9 = 9, LBM_D3Q19 = 19 } lbm_lattice;

/* How populations are kept on the device between steps.  All forms store the
 * normalised offsets d_q = (f_q - w_q) / w_q and do the collide arithmetic in
 * FP32 (FP64 for LBM_STORE_F64). */
typedef enum {
  LBM_STORE_F32 = 0,
  LBM_STORE_F16 = 1,
  LBM_STORE_BF16 = 2,
  LBM_STORE_F64 = 3
} lbm_storage;

typedef enum { LBM_FORCE_NONE = 0, LBM_FORCE_UNIFORM = 1, LBM_FORCE_FIELD = 2 } lbm_force_mode;

/* Faces in the order of the reference's _FACE_MAP (lbm.py:517-524). */
typedef enum {
  LBM_FACE_X_MIN = 0, LBM_FACE_X_MAX = 1,
  LBM_FACE_Y_MIN = 2, LBM_FACE_Y_MAX = 3,
  LBM_FACE_Z_MIN = 4, LBM_FACE_Z_MAX = 5
} lbm_face;

typedef enum {
  LBM_BC_NONE = 0,
  LBM_BC_PRESSURE = 1,      /* reference Zou-He pressure face (lbm.py:425-510);
                               value[0] = prescribed density rho_p = P / cs2 */
  LBM_BC_VELOCITY = 2,      /* extension: velocity face, value[0..D-1] = u   */
  LBM_BC_ZERO_GRADIENT = 3  /* extension: unknown populations copied from the
                               plane one cell inwards (outlet only)          */
} lbm_bc_kind;

typedef struct {
  int32_t kind;     /* lbm_bc_kind */
  int32_t face;     /* lbm_face    */
  double value[3];
} lbm_face_bc;

/* lbm_desc.flags */
/* bit 1u is reserved (an earlier row-staged rollout step, slower than the
   default gather, was removed) and rejected by lbm_plan_create; so is every
   bit not defined below */
#define LBM_PLAN_SINGLE_CELLS 2u /* rollout steps update one cell per thread
                                   (FP16/BF16 storage otherwise takes the
                                   four-cell step on rows of a multiple of 256
                                   cells for D3Q19 / 128 for D2Q9, else the
                                   paired two-cell step when the contiguous
                                   extent is even) */
#define LBM_PLAN_PAIRED_CELLS 4u /* also use the paired two-cell step for FP32
                                   storage (same conditions) */
#define LBM_PLAN_TWO_PASS 8u /* lbm_update and the first step of lbm_rollout run
                                as two passes (collide into the workspace, then
                                the pull step) instead of the one-pass tiled
                                kernel; same results bit for bit */
#define LBM_PLAN_TEST_WAIT_TIMEOUT 16u /* test hook: the one-pass tiled kernel arms
                                its barriers but issues no copies and gives up a
                                wait after 0.2 ms (instead of 2 s), so its waits
                                run out: it sets the status word and returns
                                early with the outputs incomplete.  Only for
                                testing the timeout path */

typedef struct {
  int32_t lattice;  /* lbm_lattice: 19 (D3Q19) or 9 (D2Q9)                */
  int32_t storage;  /* lbm_storage                                        */
  int64_t shape[3]; /* grid_shape; shape[2] is ignored for D2Q9           */
  double tau;       /* BGK relaxation time, tau = 0.5 + viscosity / cs2    */
  uint32_t flags;   /* LBM_PLAN_* bits, 0 = defaults                       */
} lbm_desc;

/* Per-call inputs of one step (the reference's boundary_inputs). */
typedef struct {
  int32_t force_mode;        /* lbm_force_mode                                   */
  double force[3];           /* uniform body force (D components)                */
  const void* force_field;   /* device (*grid_shape, D) when LBM_FORCE_FIELD      */
  const uint8_t* wall;       /* device grid_shape, nonzero = wall; NULL = none    */
  lbm_face_bc inlet;         /* applied first  (lbm.py:954-960)                  */
  lbm_face_bc outlet;        /* applied second (lbm.py:962-968)                  */
  const float* dev_values;   /* optional device float[9] overriding, in order,
                                inlet.value[0..2], outlet.value[0..2], force[0..2]
                                (for values that live on the device, e.g. traced
                                JAX scalars); NULL = use the host values          */
} lbm_step_args;

#define LBM_MOMENTS_DENSITY_DEVIATION 1u /* write rho - 1 instead of rho */

/* Outputs of the macroscopic fields (lbm.py:970-976); NULL = not written. */
typedef struct {
  void* density;   /* grid_shape                   */
  void* velocity;  /* (*grid_shape, D), 0 in walls */
  void* pressure;  /* grid_shape, rho * cs2        */
  uint32_t flags;
} lbm_moments;

typedef struct lbm_plan lbm_plan;

int lbm_abi_version(void);

/* Copies the last error message of the calling thread (NUL-terminated). */
int lbm_last_error(char* buf, size_t len);

/* Validates the lattice/shape/tau like LBMNode.__init__ (lbm.py:604-688). */
int lbm_plan_create(const lbm_desc* desc, lbm_plan** plan);
int lbm_plan_destroy(lbm_plan* plan);

/* Bytes of one device copy of the populations in the plan's storage form. */
int lbm_state_bytes(const lbm_plan* plan, size_t* bytes);

/* Scratch bytes that lbm_update / lbm_rollout need (two population copies). */
int lbm_workspace_bytes(const lbm_plan* plan, size_t* bytes);

/* f = f_eq(rho, u) (lbm.py:180-206), as initial_state does (lbm.py:719-745).
 * rho: grid_shape or NULL (= 1); u: (*grid_shape, D) or NULL (= 0). */
int lbm_equilibrium(const lbm_plan* plan, lbm_stream_t stream, const void* rho,
                    const void* u, void* f_out);

/* One reference step, LBMNode.update (lbm.py:899-986): macroscopic with F/2,
 * BGK + Guo collide on every cell, periodic stream on every axis, wall-node
 * swap, inlet then outlet face, output moments (u = 0 in walls). */
int lbm_update(const lbm_plan* plan, lbm_stream_t stream, const void* f_in,
               void* f_out, const lbm_step_args* args, const lbm_moments* out,
               void* workspace, size_t workspace_bytes);

/* The halo-padded step, LBMNode.update_padded (lbm.py:747-897), used under
 * spatial sharding: the plan's shape is the PADDED block, one halo cell on each
 * side of every spatial axis (extents >= 3).  The whole block is collided, the
 * interior is streamed across the halo without wrapping (lbm.py:270-304), the
 * wall swap (args->wall is the padded mask) and the faces act on the interior
 * (face planes one cell inside the block), and the interior moments are
 * written; halo cells of f_out_pad are copied from f_pad and halo entries of
 * the moment buffers are left untouched (the reference keeps the input's halo
 * values).  A body-force field is padded too (the node zero-pads an
 * interior-shaped field, as lbm.py:826-832 does).  Workspace: one population
 * copy (lbm_state_bytes). */
int lbm_update_padded(const lbm_plan* plan, lbm_stream_t stream, const void* f_pad,
                      void* f_out_pad, const lbm_step_args* args, const lbm_moments* out,
                      void* workspace, size_t workspace_bytes);

/* n_steps >= 1 successive reference steps with the same inputs (the loop body
 * of GraphManager.run_scan, graph_manager.py:2697-2751).  Between steps the
 * populations stay on the device as offsets in the plan's storage form; the
 * moments are those of the last step.  f_in may equal f_out. */
int lbm_rollout(const lbm_plan* plan, lbm_stream_t stream, const void* f_in,
                void* f_out, int64_t n_steps, const lbm_step_args* args,
                const lbm_moments* out, void* workspace, size_t workspace_bytes);

/* History of a rollout, GraphManager.run_scan_with_history
 * (graph_manager.py:2753-2805), which stacks the whole state after every step.
 * Record r holds the reference state after step (r + 1) * every, for
 * r < n_steps / every; each pointer (NULL = field not recorded) points at
 * n_steps / every consecutive arrays: f (*grid_shape, Q), density grid_shape,
 * velocity (*grid_shape, D) (0 in walls), pressure grid_shape. */
typedef struct {
  void* f;
  void* density;
  void* velocity;
  void* pressure;
} lbm_history;

/* lbm_rollout that also fills `history`; recorded steps write their outputs
 * while they collide, the others run as in lbm_rollout (same results bit for
 * bit).  Workspace: lbm_workspace_bytes. */
int lbm_rollout_history(const lbm_plan* plan, lbm_stream_t stream, const void* f_in,
                        void* f_out, int64_t n_steps, int64_t every,
                        const lbm_step_args* args, const lbm_moments* out,
                        const lbm_history* history, void* workspace, size_t workspace_bytes);

/* ---- Stepping the device state directly ------------------------------------
 * For runners that step a block of a larger lattice themselves and exchange
 * halo planes between steps (the slab-sharded runner; the reference's
 * ShardedStencilNode around update_padded, cloud/multigpu/sharded_node.py:
 * 345-413).  The state is what lbm_rollout keeps between steps: Q planes of
 * the plan's cells (plane q holds population q of every cell, cells in the
 * grid's C order) of post-collision normalised offsets in the plan's storage
 * type, lbm_state_bytes bytes.  A "slice" is one index of reference axis 0
 * (n1 n2 cells for D3Q19, ny for D2Q9).  Every axis is periodic in the
 * pull, so a block padded by one slice on each side of axis 0 steps its
 * interior correctly once its pad slices hold the neighbours' populations
 * that cross into it (the 5 of D3Q19 / 3 of D2Q9 whose axis-0 component
 * points inwards).  index_offset: the index of the block's first cell in the
 * whole lattice (it seeds the stochastic rounding of 16-bit storage, so a
 * block rounds as the whole lattice would); 0 for a whole lattice.
 *
 * lbm_state_from_f: state = C(f) of a reference-layout f (the first pass of a
 *   rollout).
 * lbm_state_step: one step (pull, wall swap, faces, collide) of the slices
 *   [first, first + count), state_in -> state_out (not aliased); one cell per
 *   thread for every storage form, bit-identical to the rollout's forms.
 * lbm_state_to_f: the reference f_bc and moments of the step that pulls from
 *   state (the last pass of a rollout). */
int lbm_state_from_f(const lbm_plan* plan, lbm_stream_t stream, const void* f_in,
                     void* state_out, const lbm_step_args* args, int64_t index_offset);
int lbm_state_step(const lbm_plan* plan, lbm_stream_t stream, const void* state_in,
                   void* state_out, const lbm_step_args* args, int64_t first, int64_t count,
                   int64_t index_offset);
int lbm_state_to_f(const lbm_plan* plan, lbm_stream_t stream, const void* state_in,
                   void* f_out, const lbm_step_args* args, const lbm_moments* out);

/* ---- Pipe node -----------------------------------------------------------
 * MADDENING's LBMPipeNode (src/maddening/nodes/lbm_pipe.py:393-879).
 * Single phase (G == 0): D3Q19 BGK with the Guo source of an actuator-disc
 * propeller (x force on the disc cells of plane propeller_x) and gravity (z
 * force on every non-wall cell), moments without the half-force step,
 * periodic stream, wall-node swap; then the D3Q7 passive tracer collided with
 * the step's new velocity (not in walls), streamed and wall-swapped.
 * Multiphase (G != 0, lbm_pipe.py:775-864): the Shan-Chen force of the
 * Yuan-Schaefer pseudopotential psi = rho_0 (1 - exp(-rho / rho_0)) (walls at
 * psi(rho_wall), force 0 in walls) added to the propeller and gravity, exact-
 * difference forcing with the shifted velocity clamped to |u| <= 0.25, the
 * density floor 0.01 after the stream, tracer = clip((rho - rho_gas) /
 * (rho_liquid - rho_gas), 0, 1); tracer_f is copied through unchanged.
 * The plan is D3Q19 with FP32 or FP64 storage. */
typedef struct {
  const uint8_t* wall;       /* grid, nonzero = wall                                */
  const uint8_t* propeller;  /* (ny, nz) disc mask of the propeller plane, or NULL */
  int32_t propeller_x;       /* the propeller plane (x index)                      */
  double propeller_force;    /* x force on the disc cells                          */
  double gravity;            /* z force on the non-wall cells                      */
  double tau_tracer;         /* tracer relaxation time, > 0.5                      */
  double G;                  /* Shan-Chen interaction strength; 0 = single phase   */
  double rho_liquid, rho_gas;/* multiphase: rho_liquid > rho_gas > 0               */
  double rho_0;              /* multiphase: pseudopotential density, > 0           */
  double rho_wall;           /* multiphase: density that sets psi in wall cells    */
} lbm_pipe_args;

int lbm_pipe_workspace_bytes(const lbm_plan* plan, size_t* bytes);

/* n_steps pipe-node steps.  f: (*grid, 19); tracer_f: (*grid, 7); outputs of
 * the last step: f_out, tracer_f_out, out->density / out->velocity (0 in
 * walls; out->pressure is not written), tracer_out (grid, 0 in walls; NULL =
 * not written).  Inputs may not alias outputs. */
int lbm_pipe_rollout(const lbm_plan* plan, lbm_stream_t stream, const void* f_in, void* f_out,
                     const void* tracer_f_in, void* tracer_f_out, int64_t n_steps,
                     const lbm_pipe_args* args, const lbm_moments* out, void* tracer_out,
                     void* workspace, size_t workspace_bytes);

/* ---- Differentiated rollout --------------------------------------------
 * Reverse mode of lbm_rollout for walls and body forces (no face conditions),
 * FP32 or FP64 storage.  The reference differentiates LBMNode.update with
 * jax.grad through lax.scan (graph_manager.py:2697-2805); here the forward keeps
 * a checkpoint of the populations every `checkpoint_every` steps (<= 0: the
 * ceiling of sqrt(n_steps)) in the workspace, and the backward recomputes each
 * segment storing only (rho, u) per step, then runs the hand-written adjoint
 * step.  The workspace must stay untouched between the two calls. */
int lbm_adjoint_workspace_bytes(const lbm_plan* plan, int64_t n_steps, int64_t checkpoint_every,
                                size_t* bytes);

/* Same result as lbm_rollout (f_out, moments of the last step), plus the
 * checkpoints the backward needs.  f_in must not alias f_out. */
int lbm_rollout_forward(const lbm_plan* plan, lbm_stream_t stream, const void* f_in, void* f_out,
                        int64_t n_steps, int64_t checkpoint_every, const lbm_step_args* args,
                        const lbm_moments* out, void* workspace, size_t workspace_bytes);

/* Gradients of a loss L given dL/d(outputs of the last step): grad_density
 * (grid), grad_velocity ((grid, D); velocity is 0 in walls), grad_f ((grid, Q));
 * any may be NULL (= 0).  Outputs (NULL = not wanted): grad_force in FP64 --
 * (grid, D) for LBM_FORCE_FIELD and LBM_FORCE_NONE (the gradient with respect
 * to a body-force field, at its value), D values for LBM_FORCE_UNIFORM -- and
 * grad_f_in = dL/df_in ((grid, Q), the plan's IO type).  f_in, n_steps,
 * checkpoint_every and args must be the forward's. */
int lbm_rollout_backward(const lbm_plan* plan, lbm_stream_t stream, const void* f_in,
                         int64_t n_steps, int64_t checkpoint_every, const lbm_step_args* args,
                         const void* grad_density, const void* grad_velocity, const void* grad_f,
                         double* grad_force, void* grad_f_in, void* workspace,
                         size_t workspace_bytes);

/* ---- Batched ensemble ------------------------------------------------------
 * Many independent lattices (own shape, tau, walls, force, faces; one lattice
 * type and storage form) advanced together: every step is ONE persistent
 * launch over a tile list of all instances (the reference runs a batch as
 * jax.vmap over lax.scan, graph_manager.py:2807-2881, which needs equal shapes).
 * Instance i behaves exactly like lbm_rollout with plans[i] and args[i]. */
typedef struct lbm_batch lbm_batch;

typedef struct {
  int32_t blocks_per_sm; /* persistent grid = blocks_per_sm x SMs; 0 = one block per tile */
  int32_t tile_order;    /* 0: instance after instance; 1: round-robin across instances;
                            2: instance after instance, smallest first.  In orders 0
                            and 2 the members whose state steps run paired (FP16/BF16
                            storage, even contiguous extent) come first and step
                            with the paired kernel                                  */
  int32_t use_graph;     /* 1: record the step sequence as a CUDA graph and replay it */
  int32_t group_mib;     /* 0: every launch covers all instances.  > 0: consecutive
                            instances of the tile order (0 or 2) whose two population
                            copies fit in group_mib MiB form a group that runs all
                            its steps before the next group starts, so a group that
                            fits in L2 is stepped from L2 */
} lbm_batch_config;

/* plans[0..n-1] must outlive the batch and share lattice and storage. */
int lbm_batch_create(const lbm_plan* const* plans, int32_t n, lbm_batch** batch);
int lbm_batch_destroy(lbm_batch* batch);
int lbm_batch_workspace_bytes(const lbm_batch* batch, size_t* bytes);

/* n_steps reference steps of every instance.  f_in[i] / f_out[i] / args[i] /
 * out[i] (out may be NULL) are instance i's; cfg may be NULL (defaults). */
int lbm_batch_rollout(const lbm_batch* batch, lbm_stream_t stream, const void* const* f_in,
                      void* const* f_out, int64_t n_steps, const lbm_step_args* args,
                      const lbm_moments* out, const lbm_batch_config* cfg, void* workspace,
                      size_t workspace_bytes);

/* Scratch capacity of lbm_update_noalloc: one population copy of at most
 * 24 MiB.  D3Q19: up to 331,129 cells with FP32 storage (e.g. 64^3), 662,258
 * with FP16/BF16, 165,564 with FP64; D2Q9: up to 699,050 cells with FP32. */
#define LBM_NOALLOC_SCRATCH_BYTES (24u << 20)

/* lbm_update for callers that cannot allocate device memory.  No counterpart in
 * the reference.  Some callers cannot call cudaMalloc or hand over a workspace:
 * a custom-call handler whose runtime gives it no scratch allocator, an
 * embedded or real-time loop where device allocation is not allowed, a plugin
 * that must not grow its host process's device memory per call.  This entry
 * point takes no workspace: its
 * scratch is a static device array of LBM_NOALLOC_SCRATCH_BYTES inside the
 * library, which every GPU that loads the library holds until the process
 * exits.  It allocates nothing (no cudaMalloc / cudaFree / allocating library
 * call).  Every call looks up that array's device address in the current
 * context and keeps none between calls, so a device reset or another context
 * on the same device never leaves it a stale address; the first lookup on a
 * device also loads the library's code there, so make the first call on each
 * device before any stream capture.  Lattices whose populations need more than the array are rejected
 * with LBM_ERR_WORKSPACE.  All calls share the one array: calls that overlap on
 * the GPU (different streams, or different threads without ordering) race and
 * corrupt each other; order them on one stream.  The array keeps the last
 * call's contents; nothing in it needs to start at zero (every byte read is
 * written first in the same call).  Results equal lbm_update's. */
int lbm_update_noalloc(const lbm_plan* plan, lbm_stream_t stream, const void* f_in,
                       void* f_out, const lbm_step_args* args, const lbm_moments* out);

/* Scratch bytes of lbm_mass_momentum. */
int lbm_reduce_workspace_bytes(const lbm_plan* plan, size_t* bytes);

/* FP64 conservation diagnostics of a state f (*grid_shape, Q):
 * out_dev[0] = sum rho, out_dev[1..D] = sum_x sum_q f e (device double[4]).
 * Deterministic (fixed two-pass order). */
int lbm_mass_momentum(const lbm_plan* plan, lbm_stream_t stream, const void* f,
                      double* out_dev, void* workspace, size_t workspace_bytes);

/* ---- Streaming frames ------------------------------------------------------
 * The float payload of a streaming frame, MADDENING BinaryStateEncoder.encode
 * (src/maddening/api/binary_encoder.py:151-205): each field (a contiguous
 * device array) converted to float32, round to nearest, and written to
 * out[offset .. offset + count), all fields in one launch.  The frame header
 * (sim_time, 8 bytes) and any host-side fields are the caller's. */
#define LBM_DTYPE_F32 0
#define LBM_DTYPE_F16 1
#define LBM_DTYPE_BF16 2
#define LBM_DTYPE_F64 3
#define LBM_DTYPE_U8 4  /* also bool */
#define LBM_DTYPE_I32 5
#define LBM_DTYPE_I64 6

typedef struct {
  const void* data; /* device pointer                         */
  int64_t count;    /* elements                               */
  int64_t offset;   /* first payload element written          */
  int32_t dtype;    /* LBM_DTYPE_*                            */
} lbm_pack_field;

int lbm_pack_f32(lbm_stream_t stream, const lbm_pack_field* fields, int32_t n_fields,
                 float* out, int64_t out_count);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H_ */
