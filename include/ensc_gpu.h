/* EnSCDynamics-B200: C ABI of the GPU explicit central-difference stepper.
 *
 * This is the drop-in boundary for the reference solver's time-step loop
 * (EnSC::exDyna3D::run, Explicit3D/source/exDyna3D.cpp:54-102).  A host
 * program that has read a deck with the reference reader hands the mesh,
 * material, controls and boundary conditions to ensc_create/ensc_set_bcs and
 * advances the solution with ensc_step; ensc_download copies the state back
 * into the reference's own arrays.  All entry points use plain pointers and
 * sizes; no C++ or torch types cross the boundary.
 *
 * Conventions
 *   - Nodal vectors are interleaved xyz per node, float64, as the reference's
 *     solution_u / solution_v (exDyna3D.h:159-160) and vertices
 *     (exDyna3D.h:141, std::array<double,3> per node).
 *   - Connectivity is 8 x uint32 per element, 0-based, in the reference's
 *     local node order (Element_HexN8.cpp:49-91; ElementBase.h:110).
 *   - Stress is [xx, yy, zz, xy, xz, yz] per element (all_sigma,
 *     exDyna3D.h:146); hourglass history is 12 doubles per element (all_QIA,
 *     exDyna3D.h:148).
 *   - Every call returns 0 on success or a negative ENSC_ERR_* code; the
 *     library never calls exit() and throws nothing across the ABI.
 *   - There is no global mutable state: one handle per solve, each on its own
 *     CUDA stream.  Calls on one handle are not thread-safe; separate handles
 *     are independent.
 *   - The caller owns all host arrays; the library copies them and keeps no
 *     host pointer after a call returns.
 */
#ifndef ENSC_GPU_H
#define ENSC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ENSC_ABI_VERSION 2

/* return codes */
#define ENSC_OK 0
#define ENSC_ERR_ARG (-1)          /* invalid argument / size */
#define ENSC_ERR_OOM (-2)          /* device allocation failed or budget exceeded */
#define ENSC_ERR_CUDA (-3)         /* CUDA runtime error */
#define ENSC_ERR_NONFINITE (-4)    /* non-finite nodal state detected */
#define ENSC_ERR_INVERTED (-5)     /* element with J <= 0 detected */
#define ENSC_ERR_TIMEOUT (-6)      /* a bounded device wait expired */
#define ENSC_ERR_NODEVICE (-7)     /* no usable CUDA device */

/* precision of the stepper */
#define ENSC_FP64 0     /* plain FP64, operation order of the reference */
#define ENSC_MIXED 1    /* FP32 element work and gather; FP64 x, u (= x - x_ref), time, dt, energy */

/* Force assembly (ensc_params.assembly).  SLOT: every element writes its 8
 * nodal forces to the reference's per-local-slot nodal vectors and the node
 * pass adds the 8 slots in order, ((a0 + a1) + ...) + a7, as the reference
 * does (exDyna3D.cpp:589-639).  PATCH (mixed precision, meshes where no node
 * repeats a local slot): elements are stored in spatially compact patches
 * of 64 (Morton order of their centroids); the element pass sums each
 * patch's forces per patch node in shared memory and the node pass adds the
 * ~1.5-1.8 patch partials of each node in patch order -- 30% fewer bytes per
 * cycle, different FP32 rounding, but on B200 a slower element pass (the
 * per-patch sums serialise each tile behind two more block barriers and
 * dependent table reads).  AUTO: SLOT. */
#define ENSC_ASSEMBLY_AUTO 0
#define ENSC_ASSEMBLY_SLOT 1
#define ENSC_ASSEMBLY_PATCH 2

/* BC code bits per DOF, as resolved by apply_boundary_condition_vec /
 * apply_boundary_condition_a (exDyna3D.cpp:379-490, 2029-2145) */
#define ENSC_BC_FIXED 1      /* SPC: v := 0, a := 0, reaction recorded */
#define ENSC_BC_VELOCITY 2   /* prescribed velocity: v := value, a := 0 */

typedef struct ensc_handle ensc_handle;

/* Mesh and initial state.  Replaces the reference's vertices,
 * hexahedron_elements and solution_v after apply_initial_condition
 * (exDyna3D.h:141-142,160; exDyna3D.cpp:338-377). */
typedef struct {
    int64_t n_nodes;
    int64_t n_elements;
    const uint32_t* conn;   /* [n_elements*8] */
    const double* x0;       /* [n_nodes*3] reference coordinates */
    const double* v0;       /* [n_nodes*3] initial velocity, or NULL for zero */
    /* Optional precomputed element constants.  When NULL they are computed
     * as compute_invMassMatrix does (exDyna3D.cpp:492-515); a drop-in caller
     * that already ran the reference's init() passes its all_BT (row-major
     * 8x3 per element), all_Volume and inv_mass_matrix (per DOF). */
    const double* bt;       /* [n_elements*24] or NULL */
    const double* vol0;     /* [n_elements] or NULL */
    const double* inv_mass; /* [n_nodes*3] or NULL */
} ensc_mesh_desc;

/* Material_elastic (Material_elastic.h:8-21) plus J2 plasticity, which the
 * reference does not have: yield_stress <= 0 selects the reference's
 * hypoelastic update unchanged. */
typedef struct {
    double E, nu, rho;
    double yield_stress;       /* initial yield stress; <= 0: elastic */
    double hardening_modulus;  /* linear isotropic hardening H = E*Et/(E-Et) */
} ensc_material;

/* Solver controls: exDyna3D members c_dr, c_cr, factor_timeStep, Cvisl,
 * Cvisq, totalTime (exDyna3D.h:176-185) and the current step's gravity
 * (StepData::gravity, StepData.h:22; its amplitude is set with
 * ensc_set_gravity_amplitude). */
typedef struct {
    double c_dr, c_cr, factor_timestep, cvisl, cvisq;
    double total_time;
    int32_t gravity_on;
    double gravity_value;
    double gravity_dir[3];
    int32_t precision;      /* ENSC_FP64 or ENSC_MIXED */
    int32_t device;         /* CUDA device ordinal */
    void* stream;           /* cudaStream_t to run on, or NULL for a private stream */
    int32_t graph_chunk;    /* cycles per captured CUDA graph; 0 = default */
    int32_t assembly;       /* ENSC_ASSEMBLY_*; 0 = AUTO */
} ensc_params;

typedef struct {
    double time;            /* exDyna3D::time */
    double dt_i;            /* exDyna3D::dt_i */
    double dt_i_1;          /* exDyna3D::dt_i_1 */
    int64_t cycles;         /* cycles run by this call */
    int64_t total_cycles;   /* cycles since ensc_create */
    int32_t status;         /* 0 or the ENSC_ERR_* that stopped stepping */
    int32_t done;           /* 1 when time reached step_end */
    double dt_stable_min;   /* min of dtStable (exDyna3D.h:206) over the last
                               force pass; seeds the next cycle's dt */
} ensc_step_report;

typedef struct {
    double kinetic;         /* 1/2 sum m v^2 at the last half step */
    double internal;        /* accumulated stress work */
    double hourglass;       /* accumulated hourglass work */
    double viscous;         /* accumulated bulk-viscosity work */
    double external;        /* accumulated work of gravity and reactions */
    double kinetic0;        /* kinetic energy after the first ensc_set_bcs */
} ensc_energy_report;

int ensc_abi_version(void);

/* Creates a solver instance: exDyna3D::init() (exDyna3D.cpp:105-142) --
 * element constants and lumped mass, then the init force pass with dt = 0
 * that seeds the stable time step -- on the device.  No boundary condition
 * is active until ensc_set_bcs. */
int ensc_create(const ensc_mesh_desc* mesh, const ensc_material* mat, const ensc_params* params,
                ensc_handle** out);

/* Activates a step's resolved boundary conditions (setCurrentStep,
 * exDyna3D.cpp:1760-1940) and applies them to the velocity field at once, as
 * setCurrentStep's call to apply_boundary_condition_vec does (:1911).
 * dof_code/dof_value: [n_nodes*3]; dof_value is read where the code has
 * ENSC_BC_VELOCITY.  NULL code clears all conditions. */
int ensc_set_bcs(ensc_handle* h, const int8_t* dof_code, const double* dof_value);

/* Changes the gravity load of the current step (apply_gravity,
 * exDyna3D.cpp:800-826). */
int ensc_set_gravity(ensc_handle* h, int32_t on, double value, const double dir[3]);

/* Gravity amplitude of the current step (the *Amplitude named by the step's
 * *Dload, map_amp_list / deal_amp, exDyna3D.cpp:809-813, 1222-1278): n_points
 * (time, value) pairs interleaved in time_value; each cycle scales gravity by
 * the factor deal_amp gives for the cycle's time and dt.  n_points = 0
 * removes the amplitude (factor 1). */
#define ENSC_MAX_AMPLITUDE_POINTS 4096
int ensc_set_gravity_amplitude(ensc_handle* h, int32_t n_points, const double* time_value);

/* Runs the body of run()'s step loop (exDyna3D.cpp:86-100) -- stable dt,
 * last-step clamp, computeSate -- while time < step_end_time, at most
 * max_cycles cycles.  Blocks until done; report may be NULL. */
int ensc_step(ensc_handle* h, int64_t max_cycles, double step_end_time, ensc_step_report* report);

/* ensc_step that also stops after the cycle in which time first reaches
 * pause_time, without shortening any dt: the reference writes results from
 * inside the cycle in which time reaches the next output time
 * (output_results, exDyna3D.cpp:207-219, called from computeSate :788), so
 * a caller that writes output pauses there and continues with the same
 * trajectory. */
int ensc_step_until(ensc_handle* h, int64_t max_cycles, double step_end_time, double pause_time,
                    ensc_step_report* report);

/* Enqueues the same work without waiting (for callers that time the stream
 * themselves); finish with ensc_sync. */
int ensc_step_async(ensc_handle* h, int64_t max_cycles, double step_end_time);
int ensc_sync(ensc_handle* h, ensc_step_report* report);

/* ensc_step_until without waiting: enqueues up to max_cycles cycles (at most
 * 2^24) that stop after the cycle in which time reaches pause_time, and
 * returns at once, so the host can write output while the device steps.
 * Cycles past the stop are no-ops; ensc_sync (or a later ensc_step_until
 * with the same limits) completes the call and reports. */
int ensc_step_until_async(ensc_handle* h, int64_t max_cycles, double step_end_time, double pause_time);

/* ---- output snapshots ----------------------------------------------------
 * The fields output_results writes at an output time (exDyna3D.cpp:207-336):
 * vertices, solution_u, solution_v and solution_a (the last cycle's
 * acceleration, compute_a :642-644: assembled force and gravity with the
 * acceleration conditions applied, times the inverse mass), the reactions
 * solution_rf and all_sigma, plus the clock.  ensc_snapshot_begin captures
 * them on the device in stream order (after the cycles already enqueued)
 * and copies them to pinned host memory on a second stream, without
 * waiting: stepping can continue while the copy runs.  ensc_snapshot_wait
 * waits for the last snapshot begun and points `out` at its host copy, which
 * stays valid until the second ensc_snapshot_begin after it (two host
 * buffers are used in turn).  The acceleration is evaluated from the last
 * force pass's element forces, which ensc_download and ensc_upload_state
 * overwrite: begin fails with ENSC_ERR_ARG when no cycle ran since them.
 * (The reference also writes a "force" field, solution_f, which it never
 * fills, exDyna3D.cpp:157,179,232: it is zero there.) */
typedef struct {
    const double* x;        /* [n_nodes*3] vertices */
    const double* u;        /* [n_nodes*3] solution_u */
    const double* v;        /* [n_nodes*3] solution_v */
    const double* a;        /* [n_nodes*3] solution_a of the last cycle */
    const double* rf;       /* [n_nodes*3] solution_rf */
    const double* sigma;    /* [n_elements*6] all_sigma */
    double time, dt_i, dt_i_1;
    int64_t total_cycles;
    int32_t status;         /* 0 or the ENSC_ERR_* the device had raised */
} ensc_snapshot;
int ensc_snapshot_begin(ensc_handle* h);
int ensc_snapshot_wait(ensc_handle* h, ensc_snapshot* out);

/* Copies state to host arrays (any pointer may be NULL): x = vertices,
 * u = solution_u, v = solution_v ([n_nodes*3]), sigma = all_sigma
 * ([n_elements*6]), qia = all_QIA ([n_elements*12]), eps_p = equivalent
 * plastic strain ([n_elements]). */
int ensc_download(ensc_handle* h, double* x, double* u, double* v, double* sigma, double* qia,
                  double* eps_p);

/* Replaces the evolving state from host arrays (all [..] as in
 * ensc_download; NULL leaves a field unchanged) and the clock.  Used to
 * restart from a checkpoint: time, dt_i, dt_i_1 and dt_stable_min as reported
 * by ensc_step at the checkpoint (dt_stable_min <= 0 keeps the current
 * value). */
int ensc_upload_state(ensc_handle* h, const double* x, const double* u, const double* v,
                      const double* sigma, const double* qia, const double* eps_p, double time,
                      double dt_i, double dt_i_1, double dt_stable_min);

/* Energy sums (no counterpart in the reference). */
int ensc_energy(ensc_handle* h, ensc_energy_report* out);

/* Reaction forces at fixed DOFs of the last cycle (solution_rf,
 * exDyna3D.h:164), [n_nodes*3]. */
int ensc_download_reactions(ensc_handle* h, double* rf);

/* Runs up to max_cycles cycles (same work as ensc_step, launched kernel by
 * kernel instead of as a graph) with CUDA events around every kernel on the
 * handle's stream, and returns each kernel's summed duration in milliseconds
 * and launch count.  Kernel order: [0] cycle begin, [1] edge prepass,
 * [2] exact-dt begin, [3] element pass, [4] node pass.  For measurement. */
int ensc_profile(ensc_handle* h, int64_t max_cycles, double step_end_time, double ms[5], int64_t launches[5]);

/* Device bytes held by the handle. */
int64_t ensc_device_bytes(const ensc_handle* h);

/* Number of kernel launches one cycle issues (for launch accounting). */
int32_t ensc_kernels_per_cycle(const ensc_handle* h);

/* The force assembly the instance uses (ENSC_ASSEMBLY_SLOT or _PATCH), and
 * for PATCH its number of patches and of (patch, node) partials; any
 * pointer may be NULL. */
int ensc_assembly(const ensc_handle* h, int32_t* assembly, int64_t* patches, int64_t* partials);

void ensc_destroy(ensc_handle* h);

/* ---- batches of independent solves --------------------------------------
 * No counterpart in the reference, which runs one exDyna3D per process
 * (main.cpp).  A batch steps many independent instances -- each its own
 * mesh, material, controls, boundary conditions and clock, exactly what
 * ensc_create/ensc_set_bcs/ensc_step would do for it alone -- with one
 * launch per cycle phase for all of them.  Instances are sub-allocated from
 * a device memory pool bounded by budget_bytes and can be added and removed
 * between runs.  An armed instance advances until its own cycle budget or
 * step end, then idles while the others continue.  All instances of a batch
 * share its precision and stream.  Results of an instance do not depend on
 * the other instances in the batch: its state and energies are those of the
 * same solve with ensc_create (state bit-identical; energy sums may differ in
 * the last bits, being summed per 32-element tile). */
typedef struct ensc_batch ensc_batch;

/* params: precision, device, stream (NULL: own stream) and graph_chunk
 * (cycles per graph launch, 0: tuned) are used; the solve controls come per
 * instance.  Capacities bound the instances and their total elements and
 * nodes; budget_bytes bounds the instances' device memory. */
int ensc_batch_create(const ensc_params* params, int32_t max_instances, int64_t max_elements, int64_t max_nodes,
                      int64_t budget_bytes, ensc_batch** out);

/* Adds an instance (ensc_create's work for it, controls from `controls`);
 * *slot receives its index.  ENSC_ERR_OOM when the budget, the slots or the
 * tile capacity would be exceeded.  The device work of adding an instance,
 * and of its ensc_batch_set_bcs and ensc_batch_arm until the batch next
 * runs, syncs, downloads or removes, goes on the batch's own admission
 * stream: it overlaps cycles already enqueued by ensc_batch_run, which the
 * new instance does not take part in; the next ensc_batch_run includes it. */
int ensc_batch_add(ensc_batch* b, const ensc_mesh_desc* mesh, const ensc_material* mat, const ensc_params* controls,
                   int32_t* slot);

/* ensc_batch_add in two parts, so that the host work of an arriving solve
 * can overlap the batch's running cycles.  ensc_batch_prepare does the host
 * part -- checks the mesh and material and computes the element constants,
 * lumped mass and node tables for params->precision and params->assembly
 * (the other fields are not read) -- on the calling thread and
 * makes no CUDA call, so it may run on any thread while a batch steps;
 * errors are reported through ensc_last_error(NULL) of that thread.  It
 * also forms the rows the device part copies as they are, and keeps no
 * pointer into the mesh: its arrays may be freed when it returns.
 * ensc_batch_add_prepared does the device part
 * (ENSC_ERR_OOM as ensc_batch_add; ENSC_ERR_ARG when the precision is not the
 * batch's) and leaves `prep` to the caller, who frees it with
 * ensc_prepared_destroy; the instance is the one ensc_batch_add would add. */
typedef struct ensc_prepared ensc_prepared;
int ensc_batch_prepare(const ensc_mesh_desc* mesh, const ensc_material* mat, const ensc_params* params,
                       ensc_prepared** out);
int ensc_batch_add_prepared(ensc_batch* b, const ensc_prepared* prep, const ensc_params* controls, int32_t* slot);
int64_t ensc_prepared_bytes(const ensc_prepared* prep);  /* device bytes the instance will take */
/* The force assembly the instance uses (ENSC_ASSEMBLY_SLOT or _PATCH), and
 * for PATCH its number of patches and of (patch, node) partials; any
 * pointer may be NULL. */
int ensc_prepared_assembly(const ensc_prepared* prep, int32_t* assembly, int64_t* patches, int64_t* partials);

/* The host tables of a PATCH instance, for inspection; the pointers stay
 * valid until ensc_prepared_destroy.  Patch p holds the elements stored at
 * positions 64 p .. 64 p + 63 and the partials patch_first[p] ..
 * patch_first[p + 1] - 1; partial q sums the incidences inc[inc_first[q] ..
 * inc_first[q + 1]), each (element position in the patch << 3 | local slot);
 * node n adds the partials node_partials[node_first[n] .. node_first[n + 1]).
 * ENSC_ERR_ARG for a SLOT instance. */
typedef struct {
    int64_t n_elements, n_nodes, n_patches, n_partials;
    const int32_t* stored;          /* [n_elements] element of the caller's numbering -> stored position */
    const uint32_t* patch_first;    /* [n_patches + 1] */
    const uint32_t* inc_first;      /* [n_partials + 1] */
    const uint16_t* inc;            /* [8 n_elements] */
    const uint32_t* node_first;     /* [n_nodes + 1] */
    const uint32_t* node_partials;  /* [n_partials] */
} ensc_patch_tables;
int ensc_prepared_patch_tables(const ensc_prepared* prep, ensc_patch_tables* out);
void ensc_prepared_destroy(ensc_prepared* prep);

/* ensc_set_bcs for one instance. */
int ensc_batch_set_bcs(ensc_batch* b, int32_t slot, const int8_t* dof_code, const double* dof_value);

/* ensc_set_gravity_amplitude for one instance. */
int ensc_batch_set_gravity_amplitude(ensc_batch* b, int32_t slot, int32_t n_points, const double* time_value);

/* Lets the instance run up to max_cycles more cycles while its time is below
 * step_end_time (ensc_step's limits), starting with the next run. */
int ensc_batch_arm(ensc_batch* b, int32_t slot, int64_t max_cycles, double step_end_time);

/* Enqueues `cycles` cycles of the whole batch (instances that are done skip
 * them) on the batch's stream and returns without waiting. */
int ensc_batch_run(ensc_batch* b, int64_t cycles);

/* Waits for the batch's stream and refreshes every instance's report;
 * *n_running (may be NULL) receives the number of armed instances not done. */
int ensc_batch_sync(ensc_batch* b, int32_t* n_running);

/* Report and energies of an instance as of the last ensc_batch_sync. */
int ensc_batch_report(ensc_batch* b, int32_t slot, ensc_step_report* report);
int ensc_batch_energy(ensc_batch* b, int32_t slot, ensc_energy_report* out);

/* ensc_download for one instance (waits for the batch's stream). */
int ensc_batch_download(ensc_batch* b, int32_t slot, double* x, double* u, double* v, double* sigma, double* qia,
                        double* eps_p);

/* Removes an instance; its memory returns to the batch's pool. */
int ensc_batch_remove(ensc_batch* b, int32_t slot);

/* Device bytes held by the batch's instances, and their number. */
int64_t ensc_batch_device_bytes(const ensc_batch* b);
int32_t ensc_batch_instances(const ensc_batch* b);

/* The launch choices of the batch's autotuner (no reference counterpart:
 * the reference has no batched stepper): grid multipliers over one wave of
 * resident blocks of the element and node passes, cycles per graph launch,
 * threads per block of the node pass and elements per thread of the element
 * pass -- zero until the first tuning completes; the autotuner spreads its
 * candidates over the first runs and tunes again when the batch's element
 * count changes four-fold -- and the force assembly of the batch's
 * instances (ENSC_ASSEMBLY_SLOT or _PATCH, fixed at ensc_batch_create:
 * the assemblies round differently, so they are not timed against each
 * other mid-solve).  Any pointer may be NULL. */
int ensc_batch_tuning(const ensc_batch* b, int32_t* mult_element, int32_t* mult_node, int32_t* graph_cycles,
                      int32_t* node_threads, int32_t* elements_per_thread, int32_t* assembly);

void ensc_batch_destroy(ensc_batch* b);

/* Message of the last error on b (NULL: as ensc_last_error(NULL)). */
const char* ensc_batch_last_error(const ensc_batch* b);

/* ---- stepping without device allocation --------------------------------
 * No counterpart in the reference: the reference stepper never allocates on
 * a GPU.  For callers that may not call cudaMalloc -- plug-ins inside a host
 * application that owns and budgets all device memory through its own pool,
 * solver loops whose device memory is fixed at start-up (an allocation can
 * synchronise the device, and its failure mid-run has no recovery there) --
 * ensc_step_noalloc runs the FP64 cycle on device arrays the caller already
 * owns and keeps its scratch (element-force hand-off, energy partials,
 * control block) in one fixed file-scope device array of about 6.3 MiB that
 * every GPU loading this library holds until exit.  It allocates nothing.
 * Meshes above the limits below are rejected with ENSC_ERR_ARG; meshes where
 * a node sits in the same local slot of two elements are not supported
 * (node_elem holds one element per slot; build it with a check for such
 * clashes, as capi.noalloc_node_elem does).  All calls share the scratch and
 * it keeps the last call's contents: each call re-initialises it, but calls
 * that overlap on the GPU race on it.  The first call on a device looks up
 * the scratch address (once per device); make it before any stream capture.
 * Messages: ensc_last_error(NULL). */
#define ENSC_NOALLOC_MAX_ELEMENTS 32768
#define ENSC_NOALLOC_MAX_NODES 262144

/* Caller-owned device arrays, structure of arrays with component stride
 * n_elements (element arrays) or n_nodes (node arrays), no padding. */
typedef struct {
    int64_t n_nodes, n_elements;
    const uint32_t* conn;       /* [8][n_elements] local node k of element e */
    const double* bt;           /* [24][n_elements] component 3k+c = B0^T(k, c) */
    const double* vol0;         /* [n_elements] V0 */
    const double* cbrt_v0;      /* [n_elements] cbrt(V0) */
    const double* cbrt_v0sq;    /* [n_elements] cbrt(V0 * V0) */
    const double* inv_mass;     /* [n_nodes] inverse lumped mass */
    const uint8_t* bc;          /* [n_nodes] bits 2c / 2c+1: DOF c fixed / velocity */
    const double* bc_value;     /* [3][n_nodes] prescribed velocities */
    const uint32_t* node_elem;  /* [8][n_nodes] element holding node n in slot k, or 0xFFFFFFFF */
    double* x;                  /* [3][n_nodes] current coordinates, in/out */
    double* u;                  /* [3][n_nodes] displacement, in/out */
    double* v;                  /* [3][n_nodes] velocity, in/out */
    double* sigma;              /* [6][n_elements] in/out */
    double* qia;                /* [12][n_elements] in/out */
    double* eps_p;              /* [n_elements] in/out */
    double* rf;                 /* [3][n_nodes] reactions, out */
    /* gravity amplitude of the step (as ensc_set_gravity_amplitude): in
     * device memory, gravity_amp_n (time, value) pairs interleaved, or NULL
     * with gravity_amp_n = 0 for none (factor 1) */
    const double* gravity_amp;
    int32_t gravity_amp_n;
} ensc_device_model;

/* Clock carried between calls (in/out). */
typedef struct {
    double time, dt_i, dt_i_1;
    double dt_stable_min;       /* min element dt of the last force pass */
    int32_t init_pass;          /* 1 on the first call: run init()'s dt = 0 pass */
    int64_t cycles;             /* out: cycles run by the call */
} ensc_noalloc_clock;

/* Runs up to max_cycles FP64 cycles while time < step_end_time, on
 * params->stream (NULL: the legacy default stream) of params->device, and
 * waits for them: cycles are launched in batches of 32 and the call returns
 * after the batch in which the step end is reached or a status stops the run
 * (so max_cycles may be INT64_MAX with a finite step_end_time).
 * params->precision must be ENSC_FP64; gravity comes from params and the
 * model's amplitude table. */
int ensc_step_noalloc(const ensc_device_model* m, const ensc_material* mat, const ensc_params* params,
                      ensc_noalloc_clock* clk, int64_t max_cycles, double step_end_time);

/* Message of the last error on h (or of the last failed ensc_create on this
 * thread when h is NULL). */
const char* ensc_last_error(const ensc_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* ENSC_GPU_H */
