/*
 * gfb.h -- C ABI of the B200 (sm_100a) CG-SEM elastic time loop.
 *
 * Drop-in boundary for the path that `gf_solver_elastic_cuda --direction
 * {x,y,z}` runs in changguo1998/GF-only-SEM.  The reference binds this path
 * through C++ only: `int gf::run_forward(const std::string&, bool, int)`
 * (forward/share/include/gf/solver.hpp:21) over the device API of
 * forward/share/include/gf/cuda_step.hpp:70-129 and the element kernel
 * entry `compute_element_residual<BackendCUDA>` (forward/share/include/gf/
 * element.hpp:39-42).  Each entry point below names the reference interface
 * it replaces.
 *
 * Conventions
 *  - Plain pointers and sizes; no C++ or torch types cross the boundary.
 *  - Every function returns a gfb_status; GFB_OK == 0.  A failing call
 *    leaves a message retrievable with gfb_last_error() (per thread).
 *    Nothing aborts the process (the reference aborts in GF_CUDA_CHECK,
 *    forward/share/include/gf/cuda_check.h:16-24).
 *  - Host arrays passed to gfb_create are read during the call only.
 *  - Array layouts are the reference's (RankData, forward/share/include/gf/
 *    types.hpp:27-140): element-major, GLL node (i*ngll + j)*ngll + k,
 *    components last.
 */
#ifndef GFB_H
#define GFB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GFB_ABI_VERSION 1

typedef enum gfb_status {
    GFB_OK = 0,
    GFB_ERR_INVALID = 1,    /* bad argument or inconsistent mesh            */
    GFB_ERR_CUDA = 2,       /* CUDA runtime error (message has the detail)  */
    GFB_ERR_NOMEM = 3,      /* device or host allocation failed             */
    GFB_ERR_STATE = 4,      /* call not valid in the solver's current state */
    GFB_ERR_UNSUPPORTED = 5,/* e.g. polynomial order outside 2..5           */
    GFB_ERR_NO_DEVICE = 6,  /* no CUDA device (reference main.cpp:51-58)    */
    GFB_ERR_IO = 7          /* file input/output failure                    */
} gfb_status;

typedef enum gfb_precision {
    GFB_FP64 = 0, /* all arithmetic in FP64 (parity path, 1e-10 vs oracle)         */
    GFB_FP32 = 1  /* FP32 element/C-PML arithmetic, FP64 displacement & velocity  */
} gfb_precision;

/*
 * Merged partition set (the result of read_partition_all,
 * forward/share/src/io.cpp:319-450).  n_node is n_rank_node.
 */
typedef struct gfb_mesh {
    int32_t n_cell;            /* number of hexahedral cells                   */
    int32_t ngll;              /* N+1, 3..6 supported                          */
    int32_t n_node;            /* unique GLL nodes (max(ibool)+1)              */
    const int32_t* ibool;      /* [n_cell*ngll^3] local_cell2rank_node         */
    const int64_t* cell_ids;   /* [n_cell] local_cell_ids; NULL -> 0..n-1      */
    const double* dxi_dx;      /* [n_cell*ngll^3*9]                            */
    const double* jacobian;    /* [n_cell*ngll^3] det J                        */
    const double* lambda_;     /* [n_cell*ngll^3]                              */
    const double* mu;          /* [n_cell*ngll^3]                              */
    const double* density;     /* [n_cell*ngll^3] (read only with C-PML)       */
    const double* mass;        /* [n_cell*ngll^3] element-local lumped mass    */
    const double* damping;     /* [n_cell*ngll^3] legacy ramp; NULL -> none    */
    const int32_t* pml_region; /* [n_cell] 0 interior, 1..7 C-PML region       */
    const double* pml_coef_alpha; /* [n_cell*ngll^3*9]                         */
    const double* pml_coef_abar;  /* [n_cell*ngll^3*5]; NULL -> no C-PML       */
    int32_t n_rec_cell;        /* recording cells (0 -> no snapshots)          */
    const int32_t* rec_cell_local; /* [n_rec_cell] merged local cell index     */
} gfb_mesh;

/* Time-loop configuration (ConfigData, types.hpp:128-140, subset). */
typedef struct gfb_config {
    double dt;                 /* solver_dt                                    */
    int32_t snapshot_stride;   /* record when step % stride == 0; <=0 never    */
    int32_t precision;         /* gfb_precision                                */
    int32_t n_field;           /* wavefields advanced together, 1..3           */
    int32_t field_dir[3];      /* force direction per wavefield, 0=x 1=y 2=z   */
    int32_t device;            /* CUDA device ordinal                          */
    int32_t record_slots;      /* snapshot slots kept on the device (>=1)      */
    int32_t flags;             /* GFB_FLAG_* bits, 0 for defaults              */
} gfb_config;

/* Keep C-PML memory per cell and GLL node, as the reference does
 * (pml.cpp:112-149), also on the FP32 path.  Without it the FP32 path keeps
 * one memory per global node and axis when the cells' axis coefficients
 * agree at every shared node (they are functions of the node position). */
#define GFB_FLAG_CELL_PML 1
/* Store snapshots as float on the device and in the pinned host ring (the
 * reference's snapshot_precision = "float32", record.cpp:91-98, 132-139);
 * gfb_read_record still returns doubles, gfb_read_record_f32 floats. */
#define GFB_FLAG_RECORD_F32 2
/* Update each node in the epilogue of the element kernel of the highest
 * colour touching it instead of in a separate node pass (same results).
 * Slower on B200 as laid out today: the epilogue's scattered per-node
 * accesses cost far more L1 transactions than the contiguous node pass. */
#define GFB_FLAG_FUSED_NODE 4
/* Run the FP32 path with the thread-per-GLL-point element kernel instead of
 * the thread-per-xi-line kernel (same arithmetic, different summation order;
 * for comparisons). */
#define GFB_FLAG_POINT_KERNEL 8
/* Launch each step's kernels one by one instead of replaying the step as a
 * captured CUDA graph. */
#define GFB_FLAG_NO_GRAPH 16
/* At the end of gfb_create(_batch), time full colour sweeps of each FP32
 * element-kernel candidate (the line kernel with each cells-per-group count
 * it is built with, and the thread-per-point kernel) on this mesh and keep
 * the fastest; gfb_get_info reports the choice.  Tuning leaves the state
 * unchanged. */
#define GFB_FLAG_AUTOTUNE 32
/* FP32 path: evaluate the element force from the full predicted
 * displacement at every step.  By default most steps add the force of the
 * predicted displacement's increment over the previous step to the stored
 * force, with a full evaluation every 800 steps (and after the state is
 * overwritten; gfb_set_force_refresh changes the period): the float rounding of the full predicted displacement,
 * amplified by the stiffness into the highest modes, is what bounds the
 * FP32 path's accuracy (recorded acceleration ~1.5e-4 relative L2 after
 * 2000 steps in full, ~3e-5 by increments).  Applies only where the C-PML
 * term is added at the nodes or there is none, and without a learned layer
 * or GFB_FLAG_FUSED_NODE (those evaluate in full every step). */
#define GFB_FLAG_DIRECT_FORCE 64

/* Point-force source (config.h5 /source, io.cpp:681-707). */
typedef struct gfb_source {
    int32_t n_src_cell;        /* containing cells                             */
    const int64_t* cell_ids;   /* [n_src_cell] matched against mesh cell_ids   */
    const double* weights;     /* [n_src_cell*ngll^3] Lagrange weights         */
    int32_t n_stf;             /* samples of the source time function          */
    const double* stf;         /* [n_stf] stf_values; step s uses stf[s]       */
} gfb_source;

typedef struct gfb_solver gfb_solver;

/* ABI version of the loaded library (compare with GFB_ABI_VERSION). */
int32_t gfb_abi_version(void);

/* Architecture the library's device code was built for, as the CUDA runtime
 * reports it for one of its kernels on `device` (cudaFuncGetAttributes):
 * binary_version 100 is sm_100 (sm_100a).  No counterpart in the reference. */
gfb_status gfb_kernel_arch(int32_t device, int32_t* binary_version, int32_t* ptx_version);

/* Message of the last failing call on this thread ("" if none). */
const char* gfb_last_error(void);

/*
 * Build a solver on the GPU: validate the mesh, assemble the global lumped
 * mass / damping (solver.cpp:188-217), initialise C-PML memory
 * (pml.cpp:41-53), map source cells (solver.cpp:247-261), colour the cells
 * for atomic-free assembly and upload everything.
 * Replaces cuda_allocate_state (cuda_step.hpp:70-78) and the set-up part of
 * run_forward (solver.cpp:100-276).
 */
gfb_status gfb_create(const gfb_mesh* mesh, const gfb_config* config, const gfb_source* source,
                      gfb_solver** out);

/*
 * One of several independent models held by one solver (no counterpart in
 * the reference, which runs one model per process).  The batch mesh passed to
 * gfb_create_batch is the models' meshes one after the other: model k owns
 * cells [cell_begin, cell_end) and nodes [node_begin, node_end), and its
 * cells use only its nodes.  Source cells are found by cell_ids over the
 * whole batch mesh; each model has its own time step and source time
 * function.  A model takes n_steps steps; after that gfb_advance leaves its
 * state as it is while the other models go on.
 */
typedef struct gfb_model {
    int32_t cell_begin, cell_end;
    int32_t node_begin, node_end;
    double dt;
    int32_t n_steps;
    int32_t n_stf;
    const double* stf;         /* [n_stf] this model's stf_values              */
} gfb_model;

/*
 * gfb_create for n_model (1..255) models advanced together: one element
 * launch per colour covers the cells of every model, so many small models
 * fill the GPU as one large one does.  config->dt is not used (each model's
 * dt is); the snapshot stride, precision and wavefield directions are shared.
 * gfb_get_state / gfb_read_record return the batch's node and recording-cell
 * arrays, model after model.
 */
gfb_status gfb_create_batch(const gfb_mesh* mesh, const gfb_config* config, const gfb_source* source,
                            int32_t n_model, const gfb_model* models, gfb_solver** out);

/*
 * One solver for several source positions (no counterpart in the
 * reference, which runs one source and one direction per process): the
 * geometry and materials are read once per step for all wavefields.
 * sources[0..n_source) are point sources as gfb_source (cells, weights,
 * stf); wavefield f is driven by source field_source[f] in direction
 * field_dir[f] (0=x 1=y 2=z).  n_field: 1..3 at any ngll, or 6, 9 or 12 at
 * ngll 5 (two to four positions times x/y/z); the FP64 path takes at most 6.
 * config->n_field and config->field_dir are not used.  Records, state and
 * Green's functions are per wavefield as for gfb_create.
 */
#define GFB_MAX_FIELDS 12
gfb_status gfb_create_sources(const gfb_mesh* mesh, const gfb_config* config, int32_t n_source,
                              const gfb_source* sources, int32_t n_field, const int32_t* field_dir,
                              const int32_t* field_source, gfb_solver** out);

/* Release all device and host memory.  Replaces cuda_free_state
 * (cuda_step.hpp:80-81). */
gfb_status gfb_destroy(gfb_solver* solver);

/*
 * Advance n_steps solver steps for all wavefields.  One step is the sequence
 * of run_forward's loop body (solver.cpp:389-444 on the GPU, 510-622 on the
 * CPU): Newmark predictor, gather, element internal force, C-PML or legacy
 * damping, source injection, assembly, corrector, C-PML memory update; at
 * steps with step % stride == 0 a snapshot of the recording cells is stored
 * in the device ring (solver.cpp:454-507).
 * Replaces cuda_newmark_predict, cuda_gather_predicted, cuda_zero_residual,
 * cuda_launch_element_residual, cuda_pml_damping, cuda_source_injection,
 * cuda_scatter_to_rank and cuda_newmark_correct (cuda_step.hpp:87-117).
 * Snapshots are copied to pinned host memory on a second stream while the
 * following steps run; when all record_slots hold unread snapshots, the
 * oldest is moved to ordinary host memory, so none is lost.
 */
gfb_status gfb_advance(gfb_solver* solver, int32_t n_steps);

/*
 * gfb_advance with one pair of CUDA events on the solver's stream around the
 * n_steps steps; adds their device milliseconds to *ms and synchronises.
 */
gfb_status gfb_advance_timed(gfb_solver* solver, int32_t n_steps, double* ms);

/*
 * gfb_advance with CUDA events on the solver's stream around each phase of
 * every step; adds the device milliseconds spent in the element/assembly
 * launches, the node update and the snapshot kernel to the three outputs
 * (any may be NULL).  Synchronises before returning.  The reference times
 * its loop with std::chrono only (solver.cpp:342-348, 729-732).
 */
gfb_status gfb_advance_profiled(gfb_solver* solver, int32_t n_steps, double* ms_element,
                                double* ms_node, double* ms_record);

/* Static description of a solver and its cumulative kernel-launch count. */
typedef struct gfb_info {
    int32_t n_colour;        /* assembly colours (launches of the element kernel per step) */
    int32_t n_pml_cell;      /* cells with C-PML state                                      */
    int32_t n_rec_cell;
    int32_t n_field;
    int32_t precision;
    int32_t n_cell;
    int32_t n_node;
    int32_t ngll;
    int64_t device_bytes;    /* device memory held                                         */
    int64_t upload_bytes;    /* bytes copied host->device by gfb_create                    */
    int64_t kernel_launches; /* kernels launched by this solver so far                     */
    int32_t n_pml_node;      /* global nodes carrying C-PML state (0: per-cell form)        */
    int32_t elem_blocks;     /* blocks in the persistent grid of the element kernel in use  */
    int32_t elem_kernel;     /* 1: thread-per-xi-line kernel, 0: thread-per-point kernel    */
    int32_t cells_per_group; /* cells per block iteration of the line kernel (0 otherwise)  */
    int32_t force_refresh;   /* steps between full element-force evaluations (1: every step) */
    int32_t half_v;          /* 1: plain nodes keep the half-step velocity, no acceleration */
    int32_t elem_variant;    /* FP32 element kernel in use: -1 thread-per-point; line kernel
                                0 the default (at ngll 5 with <= 3 wavefields: eta/zeta
                                contractions by line owners); there also 1 one fewer cell
                                per group, 2 one more, 3 the default count, the exchange
                                done by every thread                                         */
    int32_t n_elem_variants; /* line-kernel variants built for this ngll / field count
                                (0: the solver has one element kernel)                        */
} gfb_info;

gfb_status gfb_get_info(const gfb_solver* solver, gfb_info* info);

/* FP32 path: steps between full evaluations of the element force (the steps
 * between add the force of the predicted displacement's increment; 800 by
 * default, 1 = in full every step).  The next step evaluates in full.
 * GFB_ERR_UNSUPPORTED for a period > 1 on a solver that evaluates in full
 * every step (FP64, per-cell C-PML, fused node update, GFB_FLAG_DIRECT_FORCE,
 * a learned layer attached). */
gfb_status gfb_set_force_refresh(gfb_solver* solver, int32_t steps);

/* Use element-kernel variant `variant` (as in gfb_info.elem_variant) from
 * the next step on, in place of the autotuner's or the default choice; the
 * next step evaluates the element force in full.  GFB_ERR_UNSUPPORTED when
 * the solver has one element kernel (FP64, per-cell C-PML, fused node
 * update); GFB_ERR_INVALID for a variant outside [-1, n_elem_variants). */
gfb_status gfb_select_element_kernel(gfb_solver* solver, int32_t variant);

/* Wait for all queued work. */
gfb_status gfb_synchronize(gfb_solver* solver);

/* Next solver step index (number of steps taken since step 0). */
gfb_status gfb_current_step(const gfb_solver* solver, int32_t* step);

/*
 * Copy the global state of wavefield `field` to host arrays of n_node*3
 * doubles (any may be NULL).  Replaces cuda_copy_state_to_host
 * (cuda_step.hpp:103-105).
 */
gfb_status gfb_get_state(gfb_solver* solver, int32_t field, double* u, double* v, double* a);

/*
 * Overwrite the global state of wavefield `field` and set the step counter
 * (resume from a restart file, solver.cpp:369-388).  C-PML memory is reset
 * to zero, as the reference restart does not store it (restart.cpp:120-152).
 */
gfb_status gfb_set_state(gfb_solver* solver, int32_t field, int32_t step, const double* u,
                         const double* v, const double* a);

/*
 * Strain Green's functions at the recording nodes.  Recording cells share
 * GLL nodes; each snapshot also holds its values merged per node, as the
 * reference's post-processing does (postprocess/cpp/main.cpp:300-425):
 * strain weighted by the lumped mass of each (cell, point) occurrence
 * (sum m e / sum m), u, v, a averaged over the occurrences.  The reference
 * divides its accumulated displacement by the mass sum too (main.cpp:419-423,
 * a unit mismatch unless the masses are 1); here displacement is the plain
 * average.  gfb_rec_nodes gives the node count and ids (ascending: the
 * recording map's gll_node_ids); gfb_read_green reads the oldest pending
 * snapshot for every wavefield at once: strain [node][field][6] (with
 * field_dir = {x, y, z} this is the 3 x 6 Green's tensor of main.cpp:540-560
 * per node), u, v, a [node][field][3]; release != 0 consumes the snapshot.
 */
gfb_status gfb_rec_nodes(gfb_solver* solver, int32_t* n_node, int64_t* node_ids);
gfb_status gfb_read_green(gfb_solver* solver, int32_t* step, double* strain, double* u, double* v, double* a,
                          int32_t release);

/*
 * Exact checkpoint of the time loop: u, v, a, the predicted displacement,
 * the C-PML memory and previous fields (per cell or per node) and the step
 * counters, in the device layout.  The reference's restart file keeps u, v,
 * a only (restart.cpp:120-152), so its resume restarts C-PML memory from
 * zero; loading a checkpoint continues bit for bit.  A checkpoint loads
 * into a solver built from the same inputs and flags (checked); snapshots
 * pending in the ring and a learned layer's history are not part of it.
 */
gfb_status gfb_checkpoint_size(gfb_solver* solver, int64_t* bytes);
gfb_status gfb_checkpoint_save(gfb_solver* solver, void* buffer, int64_t bytes);
gfb_status gfb_checkpoint_load(gfb_solver* solver, const void* buffer, int64_t bytes);

/* Number of snapshots waiting to be read.  gfb_records_pending and
 * gfb_read_record may be called from another host thread while
 * gfb_advance runs (a writer thread draining records); all other calls on a
 * solver must come from one thread at a time. */
gfb_status gfb_records_pending(gfb_solver* solver, int32_t* n);

/*
 * Pop the oldest snapshot of wavefield `field` into host buffers laid out as
 * the record datasets of RecordWriter::write_step (record.cpp:175-257)
 * without the leading unit axis:
 *   strain [n_rec_cell, ngll^3, 6] (xx,yy,zz,xy,xz,yz)
 *   u, v, a [n_rec_cell, ngll^3, 3]
 * Any buffer may be NULL (with all four NULL nothing is copied: the call
 * only waits for the snapshot to reach host memory and can release it).
 * The snapshot is released once every wavefield has been read (or
 * immediately when release != 0).
 */
gfb_status gfb_read_record(gfb_solver* solver, int32_t field, int32_t* step, double* strain,
                           double* u, double* v, double* a, int32_t release);

/* The same into float32 buffers: the record datasets as RecordWriter writes
 * them with snapshot_precision = "float32" (record.cpp:91-98).  Values
 * recorded in float (GFB_FLAG_RECORD_F32) come out unchanged; values
 * recorded in double are rounded. */
gfb_status gfb_read_record_f32(gfb_solver* solver, int32_t field, int32_t* step, float* strain, float* u,
                               float* v, float* a, int32_t release);

/*
 * Element internal force for n_elem independent elements, host arrays in
 * and out (r is overwritten with K_e u).  Replaces
 * compute_element_residual<BackendCUDA> (element.hpp:39-42,
 * element_cuda.cu:195-252).  D [ngll*ngll] (D[i*ngll+j] = l_j'(x_i)) and
 * weights [ngll] are used as given, as the reference uses the tables it is
 * passed; either may be NULL to use the GLL tables of ngll.
 * precision selects the FP64 or FP32 kernel.
 */
gfb_status gfb_element_residual(int32_t n_elem, const double* dxi_dx, const double* jacobian,
                                const double* lambda_, const double* mu, const double* D,
                                const double* weights, int32_t ngll, const double* u, double* r,
                                int32_t precision, int32_t device);

/*
 * Element internal force that allocates nothing.  No counterpart in the
 * reference.
 *
 * For callers that cannot call cudaMalloc: code whose device memory is all
 * owned by a caching pool or a host framework (allocating behind it
 * fragments the pool and can fail under memory pressure), code that cannot
 * afford the implicit device synchronisation of cudaMalloc/cudaFree inside
 * its loop, and code running where the allocator is intercepted.  The
 * caller passes DEVICE pointers, in the layouts of gfb_element_residual:
 * dxi_dx [n_elem*ngll^3*9], jacobian, lambda_, mu [n_elem*ngll^3],
 * u [n_elem*ngll^3*3] in, r [n_elem*ngll^3*3] out (overwritten with K_e u).
 * Work is queued on `stream` (a cudaStream_t; NULL = legacy default stream)
 * of the current device; the call does not wait for it.
 *
 * The kernel's scratch (cell geometry repacked for the kernel, the node
 * table and the derivative table) lives in one fixed 8 MiB device array
 * inside the library; every GPU that loads the library holds it until the
 * process exits.  n_elem is limited to what fits: 3106 cells at ngll=3,
 * 1310 at ngll=4, 671 at ngll=5, 388 at ngll=6; larger calls are rejected
 * with GFB_ERR_INVALID and a message giving the maximum (split the call).
 * The first call on a device looks up the array's device address, and so
 * does the first call after a device reset (cudaDeviceReset, or the
 * primary context released and created again), where the array can move;
 * make those calls before any CUDA stream capture.  All calls on a device
 * share the one array and each call rewrites the part it reads, so calls
 * that may overlap on the GPU (different streams, or host threads without
 * ordering) race; serialise them on one stream.  FP64 only.
 */
gfb_status gfb_element_residual_noalloc(int32_t n_elem, const double* dxi_dx, const double* jacobian,
                                        const double* lambda_, const double* mu, int32_t ngll,
                                        const double* u, double* r, void* stream);

/* ------------------------------------------------------------------------
 * Learned absorbing layer (no counterpart in the reference, which truncates
 * the domain with C-PML, pml.cpp, or the legacy damping layer).
 *
 * A thin domain (the model plus a one-element C-PML layer) gets a force
 * correction at the nodes of its layer cells from a small network per node
 * class ("net"): inputs are u, v, a of the node (in the node's face frame,
 * each channel divided by its scale) over the last 4 steps, 36 values,
 * normalised to unit length (xh); hidden layers relu(+-W1 xh) and
 * relu(W2 h) of 64; output W3 h; damping sigma_j = softplus of the mean of
 * the +xh and -xh outputs; correction_j = -(s_c / s_v) sigma_j v_j in the
 * face frame (a learned dashpot, at most m/dt), which only takes energy out
 * and scales with the wavefield.  Weights are BF16 and inference runs on the
 * tensor cores with FP32 accumulation, between the element and node phases
 * of every step.  The networks are trained on the GPU from replays of a
 * thick-C-PML run of the enlarged domain: the thick run's state is copied
 * into the thin solver each step and the target is m (a_thick - a_thin).
 * A monitor tracks, per step, the work done by the correction relative to
 * the kinetic energy of the layer nodes: three steps in a row above the
 * threshold, a value 100 times the threshold, or a non-finite value switch
 * the correction off for good and the layer is plain one-element C-PML (the
 * fallback).
 * ------------------------------------------------------------------------ */
#define GFB_LAYER_NIN 36
#define GFB_LAYER_NHID 64
#define GFB_LAYER_NOUT 3
/* FP32 parameters of one network: W1 [64][36], W2 [64][64], W3 [3][64] */
#define GFB_LAYER_PARAMS 6592
/* BF16 values of one network in the inference layout (gfb_layer_pack) */
#define GFB_LAYER_WEIGHTS 8768

typedef struct gfb_layer {
    int32_t n_node;          /* layer nodes carrying a correction            */
    const int32_t* node;     /* [n_node] node ids of the solver's mesh       */
    const int8_t* frame;     /* [n_node][3]: local axis j is global axis
                                |frame[j]|-1 taken with the sign of frame[j]
                                (local axis 0 = outward normal)              */
    const uint8_t* net;      /* [n_node] network of the node, < n_net        */
    int32_t n_net;           /* 1..64                                        */
} gfb_layer;

/* BF16 inference layout [n_net][GFB_LAYER_WEIGHTS] from FP32 parameters
 * [n_net][GFB_LAYER_PARAMS] (round to nearest even). */
gfb_status gfb_layer_pack(int32_t n_net, const float* params, uint16_t* weights);

/* Attach a trained layer to an FP32 single-model solver (replaces any
 * previous one).  scales = {u, v, a channel scales, output scale};
 * threshold = fallback limit of the monitored residual. */
gfb_status gfb_layer_attach(gfb_solver* solver, const gfb_layer* layer, const uint16_t* weights,
                            const float* scales, double threshold);

/* Damping gains [n_net][3] (network, face axis; >= 0, all 1 at attach): the
 * dashpot coefficient of axis j at a node of network k is
 * gains[k][j] * (s_c / s_v) * sigma_j.  The closed-loop stage of training
 * fits them to the reflection error of whole runs. */
gfb_status gfb_layer_set_gains(gfb_solver* solver, int32_t n_net, const float* gains);

/* Whether the correction is still applied, and the monitored residual. */
gfb_status gfb_layer_status(gfb_solver* solver, int32_t* active, double* residual);

typedef struct gfb_trainer gfb_trainer;

/* Trainer with room for `capacity` samples per network on `device`; seeded
 * He initialisation of the FP32 parameters. */
gfb_status gfb_trainer_create(int32_t n_net, int64_t capacity, int32_t device, uint64_t seed,
                              gfb_trainer** out);
gfb_status gfb_trainer_destroy(gfb_trainer* trainer);

/* Replay n_steps steps: before each step the thin solver's state is set to
 * the thick solver's on the shared nodes (thin_to_thick maps thin node ids
 * to thick node ids), both solvers step, and every sample_stride-th step
 * the (features, target) pairs of every node_stride-th layer node are added
 * to the data set.  Both solvers: FP32, same wavefields, same step, no layer
 * attached to the thin one. */
gfb_status gfb_trainer_collect(gfb_trainer* trainer, gfb_solver* thin, gfb_solver* thick,
                               const int32_t* thin_to_thick, const gfb_layer* layer, int32_t n_steps,
                               int32_t sample_stride, int32_t node_stride);

/* Samples held per network [n_net]. */
gfb_status gfb_trainer_samples(gfb_trainer* trainer, int64_t* counts);

/* Channel scales (set before fitting; otherwise the RMS of the collected
 * u, v, a features and targets). */
gfb_status gfb_trainer_set_scales(gfb_trainer* trainer, const float* scales);

/* Adam on the mean squared error of per-sample normalised (features,
 * targets); loss[epochs] receives the mean loss of each epoch. */
gfb_status gfb_trainer_fit(gfb_trainer* trainer, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                           double* loss);

/* Mean loss over every collected sample at the current parameters. */
gfb_status gfb_trainer_evaluate(gfb_trainer* trainer, double* loss);

/* Gradient of the summed loss over n given samples (raw face-frame features
 * [n][36], targets [n][3]) for network `net` at the current parameters. */
gfb_status gfb_trainer_gradient(gfb_trainer* trainer, int32_t net, int32_t n, const float* x, const float* y,
                                float* grad, double* loss);

/* FP32 parameters [n_net][GFB_LAYER_PARAMS] and scales [4]. */
gfb_status gfb_trainer_get_params(gfb_trainer* trainer, float* params, float* scales);
gfb_status gfb_trainer_set_params(gfb_trainer* trainer, const float* params);

/*
 * Mesh inputs computed on the device.  The reference computes them on the
 * host in its Python preprocessor; these produce the same arrays (host
 * pointers in and out, float64/int32 in the reference layouts) with one GPU
 * thread per GLL point, processing the cells in bounded chunks.
 *
 * gfb_prep_geometry replaces preprocess/gll_geometry.py:132-186 (trilinear
 * hexes): corners [n_cell][8][3] in GMSH order, GLL points and weights
 * [ngll] -> coords [n_cell][ngll^3][3], jacobian (det J) [n_cell][ngll^3],
 * dxi_dx (inv(J) raveled) [n_cell][ngll^3][9], geometric mass
 * det J w_i w_j w_k [n_cell][ngll^3].
 */
gfb_status gfb_prep_geometry(int32_t device, int64_t n_cell, int32_t ngll, const double* gll_x, const double* gll_w,
                             const double* corners, double* coords, double* jacobian, double* dxi_dx,
                             double* mass_geo);

/*
 * Global node numbering, replacing preprocess/partition.py:192-254: points
 * [n_point][3] quantised to rint(x / (1e-12 extent)), numbered by the
 * lexicographic (x, y, z) order of the distinct quantised points.
 * ibool [n_point], n_node = number of distinct points.
 */
gfb_status gfb_prep_numbering(int32_t device, int64_t n_point, const double* coords, int32_t* ibool,
                              int32_t* n_node);

/*
 * C-PML inputs, replacing preprocess/pml_cpml.py:42-147, 174-253, 261-345,
 * 353-515: region per cell (0 outside the layer), coef_alpha
 * [n_cell][ngll^3][9] and A1..A5 abar [n_cell][ngll^3][5] from the points
 * coords, the cells' PML flags is_pml [n_cell], vp [n_cell][ngll^3], domain
 * bounds and layer widths (xmin xmax ymin ymax zmin zmax; width 0 = no
 * layer), the frequency f0 of the alpha profile, dt and log_r = ln R of the
 * reflection coefficient.
 */
gfb_status gfb_prep_cpml(int32_t device, int64_t n_cell, int32_t ngll, const double* coords, const uint8_t* is_pml,
                         const double* vp, const double* bounds, const double* widths, double f0, double dt,
                         double log_r, int32_t* region, double* coef_alpha, double* abar);

/*
 * File-level driver: the forward solve of one direction with the
 * reference's working-directory file contract (run_forward,
 * forward/share/src/solver.cpp:73-739; the CLI of main.cpp:32-137 is the
 * gf_solver_elastic_cuda executable over this call).  Reads config.<ext>
 * and every partitions/partition_{r}.<ext> (merged onto one GPU as
 * read_partition_all does, io.cpp:319-450), writes
 * wavefields/{dir}/record_0_{step}.<ext> per snapshot with the datasets
 * and attributes of RecordWriter::write_step (record.cpp:175-257),
 * wavefields/{dir}/restart_0.<ext> (restart.cpp:87-139) and
 * log/forward_{dir}_0.log (logger.hpp:23-30).  <ext> is h5 in a build with
 * HDF5 when config.h5 exists, else gfr: a raw container holding the same
 * dataset and attribute names (layout in csrc/gfb_files.h).  With resume,
 * the state of wavefields/{dir}/restart_0.<ext> is loaded before the file
 * is recreated.  The environment variable GFB_PRECISION=fp32 selects the
 * FP32 path (FP64 otherwise).  Returns 0 on success, 1 on failure (message
 * in the log, on stderr and in gfb_last_error), like run_forward.
 */
int32_t gfb_run_forward(const char* direction, int32_t resume, int32_t effective_nprocs);

/*
 * The partition merge of gfb_run_forward on its own, for checking and for
 * merging once ahead of runs: reads partition_dir/partition_{r}.<extension>
 * for r = 0, 1, ... and writes the merged set (read_partition_all,
 * io.cpp:319-450) to out_path (.gfr or .h5): attributes n_partitions,
 * n_cell, ngll, n_rank_node; datasets local_cell_ids, local_cell2rank_node
 * [n_cell, ngll^3] (the concatenated local_cell2global_node), the per-point
 * fields, pml_region and recording/{gll_node_ids, gll_node_coords,
 * rec_cell_local, rec_cell_global_ids, cell_gll_node_index}.  Needs no GPU.
 */
gfb_status gfb_merge_partitions(const char* partition_dir, const char* extension, const char* out_path);

/* Number of CUDA devices visible to the process (0 when there is none or the
 * driver cannot be reached); main.cpp:43-58 exits 1 when it is 0. */
gfb_status gfb_device_count(int32_t* n);

#ifdef __cplusplus
}
#endif
#endif /* GFB_H */
