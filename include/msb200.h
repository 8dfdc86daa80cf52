/*
 * msb200.h - C-ABI of the B200 capsule contact-mechanics backend.
 *
 * Every entry point takes plain pointers, sizes and POD structs and returns an
 * int status (MSB_OK = 0).  Nothing here mentions a C++ or torch type, so the
 * engine's C++ ComputeBackend, a Python ctypes binding or any other FFI can
 * bind it directly.  Each function names the reference interface it replaces
 * (paths are relative to the MicroSimulator source tree).
 *
 * Error mapping (reference exceptions -> status):
 *   std::invalid_argument -> MSB_ERR_INVALID_ARGUMENT
 *   std::overflow_error   -> MSB_ERR_OVERFLOW
 *   std::runtime_error    -> MSB_ERR_RUNTIME   (e.g. a step that cannot
 *                            resolve its contacts, cpp/core/contact_dynamics.cpp:745-748)
 *   CUDA errors           -> MSB_ERR_CUDA      (cpp/cuda/cuda_backend.cu:33-37 throws
 *                            std::runtime_error with the CUDA text)
 * msb_last_error() returns the message of the last failure on a context.
 * Solver non-convergence is not an error: it is msb_contact_solve_report.status,
 * as ContactSolveReport.status is (cpp/include/microsimulator/contact_dynamics.hpp:244-255).
 */
#ifndef MSB200_H
#define MSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum msb_status {
  MSB_OK = 0,
  MSB_ERR_INVALID_ARGUMENT = 1,
  MSB_ERR_OVERFLOW = 2,
  MSB_ERR_RUNTIME = 3,
  MSB_ERR_CUDA = 4,
  /* The output array was too small; *count holds the size that is needed and
   * nothing was written.  Call again with a larger array. */
  MSB_ERR_CAPACITY = 5,
  /* A device-side check failed (index out of range, iteration cap of a
   * device loop); the kernel skipped the access and reported it. */
  MSB_ERR_DEVICE_CHECK = 6,
  MSB_ERR_NO_DEVICE = 7
};

/* Solver outcome, ContactSolveStatus (contact_dynamics.hpp:244-248). */
enum msb_solve_status {
  MSB_SOLVE_CONVERGED = 0,
  MSB_SOLVE_ITERATION_LIMIT = 1,
  MSB_SOLVE_BREAKDOWN = 2
};

/* GrowthLoadLaw (contact_dynamics.hpp:151-159). */
enum msb_growth_load_law {
  MSB_GROWTH_LAW_NONE = 0,
  MSB_GROWTH_LAW_EXPONENTIAL = 1,
  MSB_GROWTH_LAW_LINEAR = 2
};

/* ExternalConstraintKind / ConstraintRegion / RodContactLocation
 * (cpp/include/microsimulator/constraints.hpp:16-36). */
enum msb_constraint_kind {
  MSB_CONSTRAINT_PLANE = 0,
  MSB_CONSTRAINT_SPHERE = 1,
  MSB_CONSTRAINT_BOX = 2,
  MSB_CONSTRAINT_CYLINDER = 3
};
enum msb_constraint_region { MSB_REGION_OUTSIDE = 0, MSB_REGION_INSIDE = 1 };
enum msb_rod_location { MSB_ROD_NEGATIVE = 0, MSB_ROD_POSITIVE = 1, MSB_ROD_INTERIOR = 2 };

/* ------------------------------------------------------------------- types */
typedef struct msb_vec3 {
  float x, y, z;
} msb_vec3;

/* The cells of a WorldState as structure-of-arrays views, by slot
 * (CellGeometryView + CellAttributeView, world_state.hpp:58-78).  Positions,
 * directions and lengths are written back by the stepping calls; the other
 * arrays are only read.  `fixed` holds 0 or 1 per cell. */
typedef struct msb_cell_arrays {
  uint64_t count;
  const uint64_t* ids;
  float* position_x;
  float* position_y;
  float* position_z;
  float* direction_x;
  float* direction_y;
  float* direction_z;
  float* lengths;
  const float* radii;
  const float* growth_rates;
  const uint8_t* fixed;
} msb_cell_arrays;

/* ContactParameters (contact_graph.hpp:13-17). */
typedef struct msb_contact_parameters {
  float activation_margin;
  float parallel_sine_threshold;
  float degeneracy_epsilon;
} msb_contact_parameters;

/* CellContact (contact_graph.hpp:19-29).  64 bytes. */
typedef struct msb_cell_contact {
  uint64_t first_id;
  uint64_t second_id;
  uint32_t first_slot;
  uint32_t second_slot;
  uint32_t ordinal;
  msb_vec3 point_on_first;
  msb_vec3 normal;
  float signed_separation;
  float weight;
  uint32_t reserved;
} msb_cell_contact;

/* One constraint of a ConstraintSet (constraints.hpp:66-96), flattened.
 *   plane:    a = point,  b = inward normal
 *   sphere:   a = center, radius
 *   box:      a = center, b = half extents
 *   cylinder: a = center, radius, half_height (axis along z) */
typedef struct msb_constraint {
  uint64_t id;
  uint32_t kind;           /* msb_constraint_kind */
  uint32_t allowed_region; /* msb_constraint_region */
  msb_vec3 a;
  msb_vec3 b;
  float radius;
  float half_height;
  float coefficient;
  uint32_t reserved;
} msb_constraint;

/* ConstraintContactParameters (constraints.hpp:141-144). */
typedef struct msb_constraint_contact_parameters {
  float activation_margin;
  float degeneracy_epsilon;
} msb_constraint_contact_parameters;

/* ExternalContact (constraints.hpp:146-156).  56 bytes. */
typedef struct msb_external_contact {
  uint64_t cell_id;
  uint64_t constraint_id;
  uint32_t cell_slot;
  uint32_t constraint_kind; /* msb_constraint_kind */
  uint32_t location;        /* msb_rod_location */
  msb_vec3 point_on_cell;
  msb_vec3 normal;
  float signed_separation;
  float weight;
  uint32_t reserved;
} msb_external_contact;

/* GrowthLoadResponse (contact_dynamics.hpp:161-166). */
typedef struct msb_growth_load_response {
  uint32_t law; /* msb_growth_load_law */
  float sensitivity;
  float free_load;
  float stall_load;
} msb_growth_load_response;

/* ContactRow (contact_dynamics.hpp:210-219).  72 bytes; a row against a
 * constraint has second_slot = 0xFFFFFFFF (invalid_slot). */
typedef struct msb_contact_row {
  uint32_t first_slot;
  uint32_t second_slot;
  float first_jacobian[6];
  float second_jacobian[6];
  float first_length_lever;
  float second_length_lever;
  float offset;
  float compliance;
} msb_contact_row;

/* ContactBody (contact_dynamics.hpp:224-231).  52 bytes. */
typedef struct msb_contact_body {
  msb_vec3 axis;
  float translational_mobility;
  float transverse_mobility;
  float axial_mobility;
  float length_rate;
  float drift[6];
} msb_contact_body;

/* ContactSystem (contact_dynamics.hpp:237-242). */
typedef struct msb_contact_system {
  const msb_contact_row* rows;
  uint64_t row_count;
  const msb_contact_body* bodies;
  uint64_t body_count;
  float dt;
  msb_growth_load_response growth;
} msb_contact_system;

/* ContactSolveParameters / ContactSolveReport (contact_dynamics.hpp:250-260). */
typedef struct msb_contact_solve_parameters {
  float tolerance;
  uint32_t max_iterations;
} msb_contact_solve_parameters;

typedef struct msb_contact_solve_report {
  uint32_t status; /* msb_solve_status */
  uint32_t iterations;
  float residual;
} msb_contact_solve_report;

/* ContactDynamicsParameters (contact_dynamics.hpp:173-201). */
typedef struct msb_contact_dynamics_parameters {
  float drag;
  float contact_stiffness;
  float wall_stiffness;
  float overlap_tolerance;
  float candidate_margin;
  float max_overlap_recovery;
  float max_growth_fraction;
  uint32_t max_iterations;
  uint32_t max_refinements;
  uint32_t max_step_halvings;
  uint32_t flow_drift; /* 1: cells drift with the flow field of msb_set_flow_field (the batch call takes 0) */
  msb_growth_load_response growth;
} msb_contact_dynamics_parameters;

/* ContactDynamicsReport (contact_dynamics.hpp:291-299). */
typedef struct msb_contact_dynamics_report {
  uint32_t substeps;
  uint32_t halvings;
  uint32_t refinements;
  uint32_t reserved;
  uint64_t iterations;
  uint64_t max_rows;
  float max_overlap;
  uint32_t reserved2;
} msb_contact_dynamics_report;

/* ContactDynamicsResult arrays (contact_dynamics.hpp:301-309), by slot.
 * Any pointer may be NULL when the caller does not want that output.
 * center_velocities holds x, y, z per cell (3 * count floats). */
typedef struct msb_contact_dynamics_outputs {
  float* center_velocities;
  float* axial_loads;
  float* length_increments;
} msb_contact_dynamics_outputs;

typedef struct msb_context msb_context;

/* ---------------------------------------------------------- backend handle */

/* cuda_backend_device_count() (cpp/include/microsimulator/backend.hpp:62). */
size_t msb_device_count(void);

/* make_cuda_backend(device_index) (backend.hpp:60; cpp/cuda/cuda_backend.cu:1529-1541).
 * The context owns its device buffers (grown on demand) and one non-blocking
 * stream.  Calls on one context must not overlap; separate contexts may run
 * from separate threads. */
int msb_context_create(uint32_t device_index, msb_context** out);
void msb_context_destroy(msb_context* context);

/* Text of the last failure on `context` (empty if none). */
const char* msb_last_error(const msb_context* context);

/* BackendInfo (types.hpp:88-94): the device name, e.g. "NVIDIA B200". */
int msb_backend_info(const msb_context* context, char* device_name, size_t capacity);

/* ------------------------------------------------------ contact detection */

/* ComputeBackend::find_cell_contacts (backend.hpp:35-36), with the behaviour of
 * find_cell_contacts_cpu (cpp/cpu/cpu_contacts.cpp:216-219): every capsule pair
 * whose padded boxes overlap and whose signed separation is below the
 * activation margin, one or two contacts per pair, sorted by
 * (first_id, second_id, ordinal).  `cells` are host arrays.  Writes at most
 * `capacity` contacts; *count receives the total. */
int msb_find_cell_contacts(msb_context* context, const msb_cell_arrays* cells,
                           const msb_contact_parameters* parameters, msb_cell_contact* contacts,
                           uint64_t capacity, uint64_t* count);

/* ComputeBackend::find_external_contacts (backend.hpp:37-39) when every_face is
 * 0 (find_external_contacts_cpu, cpp/cpu/cpu_constraints.cpp:602-606), and
 * find_external_contact_faces (constraints.hpp:190-192, cpu_constraints.cpp:608-612)
 * when every_face is 1.  Sorted by (cell_id, constraint_id, location). */
int msb_find_external_contacts(msb_context* context, const msb_cell_arrays* cells,
                               const msb_constraint* constraints, uint64_t constraint_count,
                               const msb_constraint_contact_parameters* parameters,
                               uint32_t every_face, msb_external_contact* contacts,
                               uint64_t capacity, uint64_t* count);

/* ----------------------------------------------------- contact graph index */

/* The index arrays of a ContactGraph (contact_graph.hpp:40-63): per slot the
 * indices of its contacts in contact order (incident_contact_indices,
 * contact_graph.cpp:376-384) and its distinct partner ids in ascending order
 * (neighbor_ids, contact_graph.cpp:386-394), each as cell_count + 1 offsets
 * into one packed array, as the constructor lays them out
 * (contact_graph.cpp:302-349).  All arrays are host or device memory as the
 * call's device_pointers says. */
typedef struct msb_contact_graph_index {
  uint64_t* incidence_offsets;  /* cell_count + 1 */
  uint64_t* incidence_contacts; /* 2 * contact count */
  uint64_t* neighbor_offsets;   /* cell_count + 1; null with neighbor_ids: no neighbour index */
  uint64_t* neighbor_ids;       /* neighbor_capacity ids; 2 * contact count always suffices */
  uint64_t neighbor_capacity;
  uint64_t neighbor_count;      /* out: the packed neighbour ids' count */
} msb_contact_graph_index;

/* ContactGraph(cell_count, contacts) (contact_graph.cpp:302-349) for a
 * caller's contact list: validates every contact as the constructor does
 * (contact_graph.cpp:217-237; the lowest failing contact's reason is the
 * error text, MSB_ERR_INVALID_ARGUMENT) and builds the index on the device.
 * MSB_ERR_OVERFLOW beyond the slot index space (cell_count >= 2^32 - 1) or
 * 2^31 - 1 contacts; MSB_ERR_CAPACITY (neighbor_count set) when the
 * neighbour ids do not fit. */
int msb_build_contact_graph(msb_context* context, const msb_cell_contact* contacts, uint64_t count,
                            uint64_t cell_count, uint32_t device_pointers, msb_contact_graph_index* index);

/* ExternalContactGraph(cell_count, contacts) (cpp/core/constraints.cpp:288-307):
 * validation (constraints.cpp:126-145) and the per-slot incidence
 * (incident_contact_indices): cell_count + 1 offsets and `count` indices. */
int msb_build_external_contact_graph(msb_context* context, const msb_external_contact* contacts, uint64_t count,
                                     uint64_t cell_count, uint32_t device_pointers, uint64_t* incidence_offsets,
                                     uint64_t* incidence_contacts);

/* ComputeBackend::find_external_contacts returning its whole
 * ExternalContactGraph (backend.hpp:37-39, cpu_constraints.cpp:597): the
 * contacts of msb_find_external_contacts and, from the same device-resident
 * list, the incidence of msb_build_external_contact_graph (host arrays:
 * cells->count + 1 offsets and one index per contact; null offsets: none). */
int msb_find_external_contact_graph(msb_context* context, const msb_cell_arrays* cells,
                                    const msb_constraint* constraints, uint64_t constraint_count,
                                    const msb_constraint_contact_parameters* parameters, uint32_t every_face,
                                    msb_external_contact* contacts, uint64_t capacity, uint64_t* count,
                                    uint64_t* incidence_offsets, uint64_t* incidence_contacts);

/* ComputeBackend::find_cell_contacts returning its whole ContactGraph
 * (backend.hpp:35-36, cpu_contacts.cpp:211): the contacts of
 * msb_find_cell_contacts and, from the same device-resident list, the index
 * of msb_build_contact_graph (host arrays; cell_count = cells->count).
 * `index` may be null (contacts only). */
int msb_find_cell_contact_graph(msb_context* context, const msb_cell_arrays* cells,
                                const msb_contact_parameters* parameters, msb_cell_contact* contacts,
                                uint64_t capacity, uint64_t* count, msb_contact_graph_index* index);

/* --------------------------------------------------------- contact solve */

/* ComputeBackend::solve_contact_forces (backend.hpp:41-43): Barzilai-Borwein
 * projected gradient from `initial_multipliers` (cpp/core/contact_solver.hpp:86-120,
 * cpp/cpu/cpu_contact_dynamics.cpp:262-338), run to convergence on the device.
 * Host arrays; `multipliers` receives row_count values. */
int msb_solve_contact_forces(msb_context* context, const msb_contact_system* system,
                             const float* initial_multipliers,
                             const msb_contact_solve_parameters* parameters, float* multipliers,
                             msb_contact_solve_report* report);

/* evaluate_contact_response (contact_dynamics.hpp:277-278): per body the
 * velocity then angular velocity (6 floats), the axial load and the loaded
 * elongation rate.  Any output may be NULL. */
int msb_evaluate_contact_response(msb_context* context, const msb_contact_system* system,
                                  const float* multipliers, float* velocities, float* loads,
                                  float* length_rates);

/* evaluate_contact_gaps (contact_dynamics.hpp:280-281). */
int msb_evaluate_contact_gaps(msb_context* context, const msb_contact_system* system,
                              const float* multipliers, float* gaps);

/* contact_system_diagonal_bound (contact_dynamics.hpp:285). */
int msb_contact_system_diagonal_bound(msb_context* context, const msb_contact_system* system,
                                      float* bound);

/* No counterpart in the reference.  The contact solve of
 * msb_solve_contact_forces for callers that cannot allocate device memory:
 * code under an allocator policy that forbids new device allocations after
 * start-up (a pool sized once, a memory budget fixed by a host framework), or
 * a real-time loop that must not wait on the driver's allocator.  It needs no
 * context and calls no cudaMalloc, cudaFree or allocating library routine:
 * every buffer lives in one static 8 MiB device array that each GPU loading
 * this library holds until the process exits.  Limits: at most 16,384 rows
 * and 8,192 bodies; a larger system returns MSB_ERR_CAPACITY.  Inputs and
 * outputs are host arrays, as in msb_solve_contact_forces; work runs on
 * `stream` (a cudaStream_t, NULL for the default stream) of the current
 * device, and the call synchronises that stream before it returns, so it
 * does not serve code inside a stream capture or a host callback.  All calls
 * share the static array: calls that overlap on the GPU race, so serialize
 * them.  The first call on a device looks up the array's device address.
 * On MSB_ERR_CUDA, *report is left as it was and `multipliers` may hold part
 * of the result.  The result agrees with msb_solve_contact_forces to the
 * solve tolerance (the BB products are reduced in a different fixed order). */
int msb_solve_contact_forces_no_alloc(const msb_contact_system* system, const float* initial_multipliers,
                                      const msb_contact_solve_parameters* parameters, float* multipliers,
                                      msb_contact_solve_report* report, void* stream);

/* ------------------------------------------------------------ whole step */

/* The contact-dynamics step of Simulation::step(dt, dynamics, contacts,
 * constraints) (cpp/core/simulation.cpp:387-397): detail::advance_contact_dynamics
 * (cpp/core/contact_stepper.hpp:32-35, cpp/core/contact_dynamics.cpp:676-782) with
 * every per-cell, per-row and per-contact pass on the device and the substep
 * controller on the host.  `cells` are host arrays; positions, directions and
 * lengths are updated in place.  On failure the arrays are left unchanged. */
int msb_advance_contact_dynamics(msb_context* context, msb_cell_arrays* cells,
                                 const msb_constraint* constraints, uint64_t constraint_count,
                                 float dt, const msb_contact_dynamics_parameters* dynamics,
                                 const msb_contact_parameters* contacts,
                                 const msb_constraint_contact_parameters* constraint_parameters,
                                 msb_contact_dynamics_report* report,
                                 msb_contact_dynamics_outputs* outputs);

/* The same step with every array of `cells` and `outputs` in device memory of
 * the context's GPU (for callers that keep the world resident in HBM). */
int msb_advance_contact_dynamics_device(
    msb_context* context, msb_cell_arrays* cells, const msb_constraint* constraints,
    uint64_t constraint_count, float dt, const msb_contact_dynamics_parameters* dynamics,
    const msb_contact_parameters* contacts,
    const msb_constraint_contact_parameters* constraint_parameters,
    msb_contact_dynamics_report* report, msb_contact_dynamics_outputs* outputs);

/* Measurement hook, no counterpart in the reference: runs `iterations` more
 * projected iterations of the last system this context solved, timing each
 * pass with CUDA events on the context's stream; returns the mean duration
 * of the body pass and of the row pass and the system's rows and bodies. */
int msb_profile_iterations(msb_context* context, uint32_t iterations, float* body_ms, float* row_ms,
                           uint64_t* rows, uint64_t* bodies);

/* One solve of the stepper: rows, iterations, final status and residual. */
typedef struct msb_solve_record {
  uint32_t rows;
  uint32_t iterations;
  uint32_t status;
  float residual;
} msb_solve_record;

/* The solves of the last msb_advance_contact_dynamics(_device) call in the
 * order they ran (probe, full solve, refinement re-solves, and those of
 * rejected substeps).  *count receives their number; MSB_ERR_CAPACITY when
 * it exceeds capacity (the first capacity records are written).  A
 * diagnostic with no counterpart in the reference. */
int msb_last_step_solves(const msb_context* context, msb_solve_record* records, uint32_t capacity,
                         uint32_t* count);

/* The overlap re-checks of the last msb_advance_contact_dynamics(_device)
 * or batch call by how their pair candidates were found: a full contact
 * search, the substep's kept candidates (no cell moved further than their
 * padding allows), or the kept candidates of the cells that did not merged
 * with a search of the cells that did (a partial re-search).  Every kind
 * gives the touches of a full search in its order.  A diagnostic with no
 * counterpart in the reference. */
int msb_last_step_searches(const msb_context* context, uint32_t* full, uint32_t* kept, uint32_t* partial);

/* Which re-check kinds the stepper may use (a diagnostic with no
 * counterpart in the reference): 0 all (the default), 1 no partial
 * re-search, 2 a full search for every re-check. */
int msb_set_search_reuse(msb_context* context, uint32_t mode);

/* The form of the BB relaxation on the device (no counterpart in the
 * reference, whose CUDA backend synchronises with the host every iteration,
 * cpp/cuda/cuda_backend.cu:1397-1400):
 *   0  automatic (the default): 1, which measures faster at every size;
 *   1  a CUDA graph: bound, initial gaps, then a WHILE node repeating a body
 *      pass and a row pass kernel, whose last block sets the condition;
 *   2  fused: one persistent cooperative kernel runs the whole solve, with
 *      two grid barriers per iteration (bounded waits; a wait that runs out
 *      fails the call with MSB_ERR_DEVICE_CHECK).
 * Both run the same arithmetic per pass and converge to the same tolerance;
 * the block count they reduce the BB products over can differ, so step
 * lengths can differ in the last bits. */
int msb_set_relaxation(msb_context* context, uint32_t form);

/* Warm starts of the stepper, extensions with no counterpart in the
 * reference (whose stepper starts every step from zero multipliers and keeps
 * no state between steps, contact_dynamics.cpp:725).  `mode` ORs flags:
 *   0  none: the reference's semantics (the default);
 *   1  carry: each step's first solve starts from the final contact forces of
 *      the context's previous step, matched by the reference's substep keys
 *      (first cell, partner, occurrence) and checked against cell ids, so a
 *      divided cell's daughters start from zero;
 *   2  guess: with a motion guess set for the step (msb_set_motion_guess),
 *      the first solve of each substep starts from multipliers moved toward
 *      the forces the guessed motion asks of each body (a least-squares step
 *      along each body's rows);
 *   4  learned: the warm-start network (msb_set_warm_start_network) makes
 *      the motion guess of every step from the cells' neighbour features,
 *      used as flag 2 uses a guess.
 * Only the multipliers a solve starts from change: the rows, the tolerance
 * and the stepper's acceptance test are the reference's, and every solve
 * converges to the same tolerance. */
int msb_set_warm_start(msb_context* context, uint32_t mode);

/* A motion guess for the next step of `context` only: guess[3 s + 0..2] =
 * (dx, dy, dtheta) of cell slot s over `dt`, the displacement in the
 * xy-plane and the turn about z (a monolayer).  Host memory; copied.  The
 * next step fails with MSB_ERR_INVALID_ARGUMENT when its cell count differs
 * from cell_count.  A null guess clears it. */
int msb_set_motion_guess(msb_context* context, const float* guess, uint64_t cell_count, float dt);

/* ---- The warm-start network (no counterpart in the reference) ----------
 *
 * A per-cell MLP that guesses each cell's displacement over a step from its
 * neighbourhood: 81 features (for each of the 16 nearest centres, the offset
 * in the cell's frame along and across its axis over 5 um, the cosine and
 * sine of the neighbour's orientation relative to the cell's with axis signs
 * aligned, and the neighbour's length over 3 um; then the cell's own length
 * over 3 um), zero-padded to 96; three hidden layers of 128 with GELU
 * (the error-function form); 3 outputs, the normalized displacement along
 * the axis, across it, and the turn.  Weights and activations are bf16, sums
 * fp32, on the tensor cores.  All pointers below are device memory. */
enum {
  MSB_MLP_INPUT = 96,
  MSB_MLP_HIDDEN = 128,
  MSB_MLP_OUTPUTS = 3,
  /* bf16 weights, row-major (out, in): W0 128x96 | W1 128x128 | W2 128x128 | W3 8x128 (rows 3..7 zero) */
  MSB_MLP_WEIGHTS = 45056,
  /* fp32 biases: b0 128 | b1 128 | b2 128 | b3 8 */
  MSB_MLP_BIASES = 392,
  /* fp32 parameters for training: the weights' layout followed by the biases' */
  MSB_MLP_PARAMETERS = 45448
};

/* Features of the cells (device arrays in msb_cell_arrays) into `features`,
 * count x MSB_MLP_INPUT bf16 (uint16 bits).  The 16 nearest centres are
 * searched in the 3 x 3 bins of 6 um around each cell (exact whenever the
 * 16th lies within 6 um); missing neighbours give zero features. */
int msb_cell_features(msb_context* context, const msb_cell_arrays* cells, uint16_t* features);
/* Bytes of the activations msb_mlp_forward keeps for msb_mlp_backward, and
 * of msb_mlp_backward's scratch, for `rows` rows. */
uint64_t msb_mlp_activation_bytes(uint64_t rows);
uint64_t msb_mlp_backward_scratch_bytes(uint64_t rows);
/* outputs (rows x 3 fp32) of the network on `features`; with a non-null
 * `activations` buffer, keeps what msb_mlp_backward needs.  `stream` is a
 * cudaStream_t (null: the default stream).  Without activations (inference)
 * the pass runs on tcgen05 with TMEM accumulators; with them (training),
 * on mma.sync keeping each layer's activations. */
int msb_mlp_forward(const uint16_t* weights, const float* biases, const uint16_t* features, uint64_t rows,
                    float* outputs, void* activations, void* stream);
/* Gradients (MSB_MLP_PARAMETERS fp32, the parameters' layout) of a loss
 * whose gradient with respect to the outputs is output_grad (rows x 3). */
int msb_mlp_backward(const uint16_t* weights, const uint16_t* features, uint64_t rows, const void* activations,
                     const float* output_grad, float* grads, void* scratch, void* stream);
/* One Adam step (bias-corrected, step >= 1) on the fp32 parameters; writes
 * the bf16 weights and fp32 biases the network reads. */
int msb_mlp_adam(float* params, const float* grads, float* m, float* v, uint32_t step, float lr, float beta1,
                 float beta2, float epsilon, uint16_t* weights, float* biases, void* stream);
/* Gives the context a network (weights and biases copied; host or device
 * memory) and the scales of its three outputs (um, um, rad), for warm-start
 * flag 4.  A null `weights` removes it. */
int msb_set_warm_start_network(msb_context* context, const uint16_t* weights, const float* biases,
                               const float* scale);

/* ---- Flow drift inside the stepper ----------------------------------------
 *
 * A fluid velocity field on a regular lattice of sites (the signal grid's
 * SignalGridSpec shape/origin/spacing/obstacles with its
 * SignalGridVelocityField, signals.hpp:116-156) that carries the cells:
 * with ContactDynamicsParameters.flow_drift the stepper gives every body the
 * drift of Simulation::flow_drift_rates (simulation.cpp:159-186) for each
 * substep, an equivalent-spheroid Jeffery closure of the face velocities
 * sampled with SignalGrid::sample_velocity (signals.cpp:923-955, clamped to
 * the lattice, fluid sites only), and limits substeps so that no cell drifts
 * more than a quarter of the smallest spacing (contact_dynamics.cpp:708-714).
 * Face arrays: x_faces (shape_x + 1) * shape_y * shape_z, y_faces
 * shape_x * (shape_y + 1) * shape_z, z_faces shape_x * shape_y * (shape_z + 1),
 * x-major as signals.cpp:134-152; obstacles (optional) one byte per site,
 * nonzero for solid. */
typedef struct msb_flow_field {
  uint32_t shape_x, shape_y, shape_z;
  uint32_t reserved;
  msb_vec3 origin;
  msb_vec3 spacing;
  const float* x_faces;
  const float* y_faces;
  const float* z_faces;
  const uint8_t* obstacles;
} msb_flow_field;

/* Gives the context a flow field (copied from host memory) for steps with
 * flow_drift = 1; a null field removes it (such steps then fail). */
int msb_set_flow_field(msb_context* context, const msb_flow_field* field);

/* ---- Batches of independent colonies (no counterpart in the reference) --
 *
 * One contact-dynamics step of many independent colonies at once, as a
 * parameter sweep runs them.  The cells of all colonies are passed colony
 * after colony in one msb_cell_arrays (ids unique across the batch); each
 * colony has its own drag and contact stiffness (replacing those of
 * `dynamics`, whose other parameters all colonies share).  Colonies never
 * touch one another, wherever their cells lie: the contact search's grid
 * gives each colony its own range of boxes.
 *
 * Each colony's contacts and rows are those it would have alone.  Each
 * colony's solves run their own Barzilai-Borwein iteration (own step length,
 * residual, tolerance and iteration count) to its own tolerance, all colonies
 * in one persistent launch of thread-block clusters.  The substep plan is the
 * batch's: a colony whose substep fails the rotation or overlap checks makes
 * the whole batch halve, and growth bounds are the batch's largest.
 * Constraints (walls) are not taken.  Warm-start flags other than carry are
 * rejected.
 *
 * The first call on a context tunes the launch shape of the batched solve
 * (CTAs per cluster, threads per CTA, register form) and the box scale of the contact search
 * by timing each candidate on that call's system; msb_tune_batch asks for a
 * new tuning at the next call and msb_batch_tuning reads the choice. */
typedef struct msb_colony_parameters {
  float drag;
  float contact_stiffness;
} msb_colony_parameters;

typedef struct msb_colony_report {
  uint64_t iterations; /* BB iterations of this colony's solves over the step */
  float max_overlap;   /* deepest overlap at the accepted geometry */
  uint32_t rows;       /* rows of the colony's last solved system */
  uint32_t cells;
  uint32_t status;     /* msb_solve_status of the colony's last solve */
} msb_colony_report;

int msb_advance_contact_dynamics_batch(msb_context* context, msb_cell_arrays* cells, const uint32_t* colony_cells,
                                       uint32_t colony_count, const msb_colony_parameters* colony_parameters,
                                       float dt, const msb_contact_dynamics_parameters* dynamics,
                                       const msb_contact_parameters* contacts, msb_contact_dynamics_report* report,
                                       msb_colony_report* colony_reports, msb_contact_dynamics_outputs* outputs,
                                       int device_pointers);
int msb_tune_batch(msb_context* context);
/* The tuned launch: CTAs per cluster, threads per CTA, lean (1: the
 * 64-register form of the solve kernel, one gather in flight per thread;
 * 0: four in flight, 128 registers) and the contact search's box scale. */
int msb_batch_tuning(const msb_context* context, uint32_t* cluster, uint32_t* threads, uint32_t* lean,
                     float* box_scale);

/* Device time of the last msb_advance_contact_dynamics(_device) call by
 * phase, measured with CUDA events on the context's stream, in
 * milliseconds: [0] upload, validation and id order; [1] contact searches;
 * [2] bodies, rows, keys and warm start; [3] incidence builds; [4] BB solves;
 * [5] moves and overlap re-checks; [6] outputs and download; [7] the
 * learned warm start's features and network.  Writes min(capacity, 8)
 * values.  A measurement aid with no counterpart in the
 * reference. */
int msb_last_step_phases(const msb_context* context, double* milliseconds, uint32_t capacity);

/* Kernel launches issued by this context since it was created (for the
 * launch counts that benchmarks report). */
uint64_t msb_launch_count(const msb_context* context);

#ifdef __cplusplus
}
#endif

#endif /* MSB200_H */
