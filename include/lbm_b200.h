/*
 * lbm_b200.h — C ABI of the B200 lattice-Boltzmann engine.
 *
 * The engine replaces the per-time-step loop of the reference solver
 * (Simulation::Iterate, Simulation.cpp:538-618) on one GPU. A caller that
 * holds the reference's SubDomain (its node list Involved_Lat_, the inlet /
 * outlet / wall lists and the near-wall list with normals) flattens it once
 * into an lbm_desc, creates an engine, and then drives time steps and reads
 * results through these functions. Plain C types only; no exceptions cross
 * the ABI; every function returns 0 on success or a negative lbm_status, and
 * lbm_last_error() describes the last failure of a handle.
 *
 * Node order: every per-node array the caller passes or receives uses the
 * caller's node order (for the reference, the order of Involved_Lat_,
 * Subdomain.cpp:598-611); per-near-wall-node arrays use the order of the
 * caller's near-wall list (SubDomain::nextToTheWall). Populations are in the
 * reference's direction order (LatticeModel.cpp:92-192 for D3Q19), laid out
 * [node][direction].
 *
 * Threading: one host thread per handle at a time. All device work of a
 * handle runs on one CUDA stream (its own, or the one set with
 * lbm_set_stream).
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbm_engine lbm_engine;

typedef enum {
    LBM_OK = 0,
    LBM_ERR_ARGUMENT = -1,    /* invalid argument or descriptor */
    LBM_ERR_CUDA = -2,        /* a CUDA call failed */
    LBM_ERR_NO_DEVICE = -3,   /* no CUDA device, or the kernels were not built for it */
    LBM_ERR_STATE = -4,       /* call not valid in the engine's current state */
    LBM_ERR_NUMERIC = -5      /* the device reported non-finite densities */
} lbm_status;

typedef enum { LBM_D3Q19 = 19, LBM_D3Q27 = 27 } lbm_lattice;

/* Storage type of the populations. FP64 stores f and computes in FP64 with
 * the reference's operand order; the others store f - w_q and compute in
 * FP32. */
typedef enum { LBM_STORE_F64 = 0, LBM_STORE_F32 = 1, LBM_STORE_F16 = 2, LBM_STORE_BF16 = 3 } lbm_storage;

/* Boundary semantics.
 * LBM_BC_REFERENCE: the reference's own rules — Zou-He plug inlet
 *   (Boundary.cpp:111-289), zero-gradient outlet copy (Simulation.cpp:650-741),
 *   wall-node fix-up (Simulation.cpp:746-763), wall nodes at rest in the
 *   collision (Simulation.cpp:92-95). D3Q19 only.
 * LBM_BC_PHYSICS: halfway bounce-back walls, velocity bounce-back inlet with a
 *   per-node profile times a waveform factor, anti-bounce-back pressure outlet. */
typedef enum { LBM_BC_REFERENCE = 0, LBM_BC_PHYSICS = 1 } lbm_bc_mode;

/* Node kinds (Node::NodeType_ / Node::BoundaryType_, Struct.h:49-63). */
typedef enum { LBM_NODE_FLUID = 0, LBM_NODE_INLET = 1, LBM_NODE_OUTLET = 2, LBM_NODE_WALL = 3 } lbm_node_kind;

/* Flattened SubDomain. Replaces SubDomain's node graph (Subdomain.h:58-125):
 * coordinates instead of neighbour pointers (the engine derives neighbours as
 * SubDomain::Connectivity does, Subdomain.cpp:447-471), node kinds, and the
 * boundary lists. Indices in the lists refer to the caller's node order. */
typedef struct {
    int32_t lattice;               /* lbm_lattice */
    int32_t storage;               /* lbm_storage */
    int32_t bc_mode;               /* lbm_bc_mode */
    int32_t device;                /* CUDA device ordinal */
    int64_t n_nodes;
    const int32_t* coords;         /* [n_nodes][3] lattice coordinates (x_position...) */
    const uint8_t* kind;           /* [n_nodes] lbm_node_kind */
    int64_t n_inlet;
    const int64_t* inlet;          /* InletBoundaryNode_.first */
    double inlet_normal[3];        /* InletBoundaryNode_.second */
    int32_t n_outlets;
    const int64_t* outlet_offsets; /* [n_outlets + 1] into outlet_nodes */
    const int64_t* outlet_nodes;   /* OutletBoundaryNodes_[k].first, concatenated */
    const double* outlet_normals;  /* [n_outlets][3] OutletBoundaryNodes_[k].second */
    int64_t n_wall;
    const int64_t* wall;           /* WallBoundaryNode_ */
    int64_t n_nearwall;
    const int64_t* nearwall;       /* nextToTheWall */
    const double* nearwall_normals;/* [n_nearwall][3] Node::normal */
    double tau;                    /* relaxation time, Simulation::m_relaxation */
    double dt;                     /* time step, Simulation::m_dt */
    double spacing;                /* Geometry::spacing (mm), for the WSS scale */
} lbm_desc;

/* Flow types: the two of Simulation::Iterate (Simulation.cpp:549-562), and a
 * harmonic waveform (lbm_set_waveform) for physics-mode inflow. */
typedef enum { LBM_FLOW_CONSTANT = 0, LBM_FLOW_PULSATILE = 1, LBM_FLOW_HARMONIC = 2 } lbm_flow;

/* Replaces Simulation(SubDomain&, SimulationParameters&) up to Iterate():
 * flattens the node graph to device arrays and sets f = w (Node::Initialize,
 * Node.cpp:71-78) and zero WSS accumulators (Simulation.cpp:66-71). */
int lbm_create(const lbm_desc* desc, lbm_engine** out);
int lbm_destroy(lbm_engine* e);

/* Uses the given cudaStream_t (as void*) for all later device work. */
int lbm_set_stream(lbm_engine* e, void* stream);

/* Inlet velocity per step, as Iterate sets InletVelocity_ (Simulation.cpp:558-562):
 * constant CteVel, or the pulsatile waveform of Simulation::getInletVelocity
 * (:519-534) evaluated at the engine's flow clock, which starts at 0 and
 * advances by dt per pulsatile step. */
int lbm_set_flow(lbm_engine* e, int32_t flow, double cte_vel);

/* Physics mode: inlet velocity per inlet node [n_inlet][3] (lattice units,
 * caller's inlet list order), multiplied each step by the waveform factor: 1
 * for constant flow, the reference waveform value for pulsatile flow, the
 * harmonic factor for harmonic flow. */
int lbm_set_inlet_profile(lbm_engine* e, const double* velocity);

/* Harmonic waveform (no counterpart in the reference, whose waveform is the
 * fixed polynomial of pulsatile.h): factor(t) = 1 + sum_k amplitude[k]
 * cos(2 pi (k+1) t / period_steps + phase[k]), t = index of the step (0 for
 * the first). With LBM_FLOW_HARMONIC the reference-mode inlet velocity is
 * cte_vel * factor and the physics-mode profile is scaled by factor. */
int lbm_set_waveform(lbm_engine* e, double period_steps, int32_t n_harmonics, const double* amplitude,
                     const double* phase);

/* Physics mode: outlet density (default 1). */
int lbm_set_outlet_density(lbm_engine* e, double rho);

/* Runs n_steps time steps: for each, the work of Collision, Streaming,
 * ApplyZouHeBc, ApplyOutletBc, ApplyWallBc, ComputeWallShearStress
 * (Simulation.cpp:553-568). Asynchronous on the engine's stream; results
 * below synchronise.
 * Numeric faults: behind every 256 steps (and at the end of the call) the
 * device flags are copied to the host without waiting for them. With the
 * numeric check on (the default), once such a copy has arrived showing a
 * non-finite density (lbm_get_flags bit 2), lbm_step runs no further steps and
 * returns LBM_ERR_NUMERIC; the steps taken before stay taken (lbm_get_time).
 * The reference has no such check (it runs on with NaN and inf values). */
int lbm_step(lbm_engine* e, int64_t n_steps);

/* Numeric check of lbm_step (default 1): 0 runs on through non-finite values,
 * as the reference does. */
int lbm_set_numeric_check(lbm_engine* e, int32_t enabled);

/* Observation policy (default 1). With 1, the last two steps of every
 * lbm_step call also store the state the getters read (populations, density
 * and velocity); with 0 they do not, which saves that traffic when a caller
 * steps many times between outputs (the reference reads state only at its
 * output steps, Simulation.cpp:575-603). Population and moment getters fail
 * with LBM_ERR_STATE after unobserved steps; WSS getters are always valid. */
int lbm_set_observation(lbm_engine* e, int32_t enabled);

/* Steps taken so far, and the flow clock (total_runtime). */
int lbm_get_time(lbm_engine* e, int64_t* steps, double* runtime);

/* Restart support. The reference writes no restart files, so these three have
 * no counterpart in it. The state the next step reads is copied as one host
 * blob of lbm_state_size bytes. It holds the stored populations (storage type,
 * internal layout), the near-wall moments the next wall shear stress uses, the
 * WSS with its FP64 accumulators, the step count, the flow clock and the AA
 * phase. lbm_get_state copies it out; a whole step must have been taken
 * (always the case between calls). lbm_set_state puts it into an engine built
 * from the same node set with the same lattice, storage type and boundary
 * mode; other blobs are refused with LBM_ERR_ARGUMENT. With the caller's flow
 * settings set again, the steps then continue bit for bit. Populations,
 * moments and fluxes are readable again after the next step (LBM_ERR_STATE
 * before it); WSS and OSI/TAWSS at once. */
int lbm_state_size(lbm_engine* e, int64_t* bytes);
int lbm_get_state(lbm_engine* e, void* dst, int64_t dst_bytes);   /* dst_bytes >= the size */
int lbm_set_state(lbm_engine* e, const void* src, int64_t src_bytes);  /* src_bytes == the size */

/* Node::m_distributions after the last step (post-boundary populations),
 * [n_nodes][q] in the caller's node order. */
int lbm_get_populations(lbm_engine* e, double* f);

/* Replaces the populations (the state after the current step); the next
 * step collides them. Clears the device flags and the numeric-fault state. */
int lbm_set_populations(lbm_engine* e, const double* f);

/* Node::density and Node::velocity after the last step: the moments the
 * last step's collision used (Simulation.cpp:85-134). rho [n_nodes],
 * u [n_nodes][3]; either may be NULL. */
int lbm_get_macros(lbm_engine* e, double* rho, double* u);

/* Near-wall outputs after the last step, in the caller's near-wall order:
 * Node::wall_shear_stress, accumulated_shear_stress [3],
 * accumulated_shear_stress_magnitude (Simulation.cpp:792-797). Any may be NULL. */
int lbm_get_wss(lbm_engine* e, double* wss, double* acc, double* accmag);

/* OSI and TAWSS from the accumulators (Simulation::ComputeOSIAndTAWSS,
 * Simulation.cpp:804-826). Either may be NULL. */
int lbm_get_osi_tawss(lbm_engine* e, double* osi, double* tawss);

/* Mass flux through the inlet and each outlet for the populations after the
 * last observed step, in FP64: over each list, the sum of (sum_q c_q f_q) .
 * normal with that list's normal (InletBoundaryNode_.second,
 * OutletBoundaryNodes_[k].second), so with outward normals inflow is negative
 * and a balanced flow gives inlet + sum(outlets) = 0. outlets has n_outlets
 * entries. Either may be NULL. */
int lbm_get_flux(lbm_engine* e, double* inlet, double* outlets);

/* Longest node list lbm_flux_noalloc accepts. */
#define LBM_FLUX_NOALLOC_MAX_NODES 1048576

/* Allocation-free mass flux. No counterpart in the reference. For callers
 * that cannot allocate device memory: a framework that owns all device memory
 * through its own pool and hands out only pointers into it, a process that may
 * not allocate after start-up, or post-processing of populations held in
 * another program's buffers without creating an engine (lbm_create allocates
 * the whole lattice). Computes in FP64, on the device, the same quantity as
 * lbm_get_flux: the sum over nodes[0 .. n_list) of (sum_q c_q f[node][q]) .
 * normal, from populations f laid out [n_nodes][q] (q = 19 or 27, the
 * reference's direction order). f, nodes and flux are device pointers; *flux
 * receives the sum; normal is a host array. It allocates nothing: the block
 * partial sums go to a fixed 32 KiB device array inside the library, so
 * n_list may not exceed LBM_FLUX_NOALLOC_MAX_NODES (longer lists are rejected
 * with LBM_ERR_ARGUMENT). Runs asynchronously on `stream` (a cudaStream_t, NULL
 * for the default stream) of the current device. The array belongs to the
 * library's device code, which CUDA loads (by default lazily) on the first
 * call on each device: that call is where the driver allocates the array, so
 * a caller that may not allocate later makes a first call at start-up (n_list
 * = 0 is enough; it writes 0 to *flux), outside any stream capture. Every call
 * on a device shares the array, so calls that overlap on the GPU race. List
 * entries outside [0, n_nodes) contribute nothing. Errors:
 * lbm_last_error(NULL). */
int lbm_flux_noalloc(const double* f, int64_t n_nodes, int32_t q, const int64_t* nodes, int64_t n_list,
                     const double normal[3], double* flux, void* stream);

/* Device status bits since creation or the last lbm_set_populations: 1 = a
 * streamed population was exactly zero (the reference would not have streamed
 * it), 2 = non-finite density. */
int lbm_get_flags(lbm_engine* e, uint32_t* flags);

/* Runs n_steps steps like lbm_step and returns their device time per kernel
 * class (milliseconds, summed over the steps, CUDA events on the engine's
 * stream): the stream+collide kernel, and the boundary work around it — the
 * pre-pass (wall shear stress, outlet copy sources) in reference mode, the
 * post-pass (wall shear stress, open-boundary corrections) in physics mode.
 * The events are recorded around a sample of the steps (the two that begin
 * every 32 steps, one of each phase), and the sums are the sampled averages
 * times n_steps: an event between every pair of kernels would add about 10 us
 * of device time to each step. In physics mode a step's kernels overlap the
 * previous kernel's tail (programmatic dependent launch), except around the
 * sampled steps, so the two sums can exceed the call's device time: time the
 * call itself for throughput. */
int lbm_step_timed(lbm_engine* e, int64_t n_steps, double* step_kernel_ms, double* boundary_kernel_ms);

/* Sizes: nodes, padded leading dimension, segments, near-wall nodes, outlet
 * nodes, bytes of device memory held. Any may be NULL. */
int lbm_get_info(lbm_engine* e, int64_t* n_nodes, int64_t* ld, int64_t* n_segments, int64_t* n_nearwall,
                 int64_t* n_outlet_nodes, int64_t* device_bytes);

/* Adjoint sensitivities of a time-averaged wall-shear objective. No
 * counterpart in the reference (whose WSS, Simulation.cpp:767-799, is only
 * evaluated). Physics mode only (D3Q19 or D3Q27).
 *
 * Starting from the engine's current populations (those of its last step,
 * which must have been observed), the run integrates n_steps physics-mode
 * steps with its own copy of the state, leaving the engine unchanged:
 * halfway bounce-back walls, the anti-bounce-back outlet at the engine's
 * outlet density, and an inlet whose speed along -inlet_normal at inlet node
 * i is v_i = sum_j coeffs[j] basis[j][i] (the engine's own inlet profile is
 * not used), times the engine's waveform factor of each step. Objective
 * (desc->objective):
 *   LBM_ADJOINT_WSS2: J = (1/T) sum_{t=1..T} sum_{k in target} |tau_k^t|^2,
 *   LBM_ADJOINT_OSI:  J = mean over the targets of their OSI over the T steps,
 * tau_k^t the wall-shear traction vector of near-wall entry k at step t, with
 * the definition and scale of lbm_get_wss. With gradient = 1 it also returns
 * dJ/dcoeffs, dJ/dtau and dJ/dv_i from a hand-written discrete adjoint: the
 * state is checkpointed every checkpoint_every steps, and the reverse sweep
 * recomputes each segment from its checkpoint, overlapped with the reverse
 * steps of the later segment (memory ~ (T/K + 2K) states). */
/* Objectives of lbm_adjoint_run. LBM_ADJOINT_OSI is the mean over the
 * targets of OSI_k = (1 - |A_k| / M_k) / 2 with A_k = sum_t tau_k^t and
 * M_k = sum_t |tau_k^t| (the accumulators of lbm_get_wss, taken over the
 * run's T steps; a target whose M_k is 0 contributes 0). */
typedef enum { LBM_ADJOINT_WSS2 = 0, LBM_ADJOINT_OSI = 1 } lbm_adjoint_objective;

typedef struct {
    int64_t n_steps;            /* T >= 1 */
    int64_t checkpoint_every;   /* K >= 1; ignored without gradient */
    int32_t precision;          /* LBM_STORE_F64 or LBM_STORE_F32: type of the state and adjoint */
    int32_t n_target;
    const int64_t* target;      /* [n_target] distinct entries of the near-wall list */
    int32_t n_coeffs;
    const double* basis;        /* [n_coeffs][n_inlet], caller's inlet order */
    const double* coeffs;       /* [n_coeffs] */
    int32_t objective;          /* lbm_adjoint_objective */
} lbm_adjoint_desc;

typedef struct {
    double objective;           /* J */
    double dJ_dtau;             /* with gradient */
    double* grad_coeffs;        /* caller-owned [n_coeffs], or NULL */
    double* grad_inlet;         /* caller-owned [n_inlet] dJ/dv_i, or NULL */
    double* final_populations;  /* caller-owned [n_nodes][q], f after the T steps, or NULL */
    double forward_ms;          /* device time of the forward sweep */
    double reverse_ms;          /* device time of recomputation and reverse sweep */
    int64_t steps_recomputed;
    int64_t device_bytes;       /* device memory the run allocated (freed on return) */
} lbm_adjoint_result;

int lbm_adjoint_run(lbm_engine* e, const lbm_adjoint_desc* desc, int32_t gradient, lbm_adjoint_result* result);

/* ---------------------------------------------------- geometry pipeline ---
 * Builds the node set of an lbm_desc from STL triangles on the GPU, with the
 * results of the reference's setup chain: Reader::readSTLASCII
 * (GeometryReader.cpp:74-158), Geometry (ComplexGeometry.cpp:83-662: bounding
 * box, grid at spacing 2 x grid_size, +z ray-parity labelling, boundary
 * points, inlet / outlet planes, wall points) and SubDomain::CreateNodes,
 * IdentifyNextToWallLattices, calculateBoundaryNormals (Subdomain.cpp:364-572).
 * Node coordinates are grid indices; nodes are in the reference's
 * Involved_Lat_ order (x-major, z-fastest). Errors: lbm_last_error(NULL). */

/* An inlet or outlet plane of the reference's config.txt (LBM.h:129-168):
 * boundary points within 2.5e-2 of `coordinate` on `axis` and inside the
 * ranges of the other two axes (+-infinity when the config gives none). */
typedef struct {
    int32_t outlet;            /* 0: inlet, 1: outlet */
    int32_t axis;              /* plane: 0 x, 1 y, 2 z */
    double coordinate;
    double normal[3];
    double range[3][2];        /* [axis][lo, hi] */
} lbm_opening;

typedef struct {
    int64_t n_triangles;
    const double* triangles;   /* [n_triangles][12]: vertex 1, 2, 3 (x, y, z), then the file's facet normal */
    double grid_size;          /* config grid_size (SimulationParameters::dx); grid spacing = 2 x grid_size */
    int32_t n_openings;
    const lbm_opening* openings; /* inlets and outlets in config order; outlets are numbered in this order */
    int32_t device;
} lbm_voxel_desc;

typedef struct lbm_voxel lbm_voxel;

/* Reads an ASCII STL with the line grammar of Reader::readSTLASCII into a
 * malloc'd [n][12] array (layout of lbm_voxel_desc.triangles); release it
 * with lbm_free. Where the reference silently skips a malformed facet (or
 * reuses the previous facet's vertices), this returns LBM_ERR_ARGUMENT with
 * the file and line: a facet that breaks the grammar, a file that ends inside
 * a facet, a file without facets. */
int lbm_stl_read_ascii(const char* path, int64_t* n_triangles, double** triangles);
void lbm_free(void* p);

/* LBM_ERR_ARGUMENT where the reference only warns (ComplexGeometry.cpp:
 * 664-692) and goes on to a simulation nothing drives: no inlet opening, or
 * inlet openings that match no grid point. */
int lbm_voxelise(const lbm_voxel_desc* desc, lbm_voxel** out);
/* Grid points per axis, grid origin (bounding-box minimum), spacing, node and
 * near-wall counts, wall-clock build time (ms). Any may be NULL. */
int lbm_voxel_info(const lbm_voxel* v, int32_t dims[3], double origin[3], double* spacing, int64_t* n_nodes,
                   int64_t* n_nearwall, double* build_ms);
/* Points the node and boundary fields of desc (n_nodes ... nearwall_normals,
 * and spacing) at v's arrays, valid until lbm_voxel_destroy; the caller sets
 * lattice, storage, bc_mode, device, tau and dt. */
int lbm_voxel_describe(const lbm_voxel* v, lbm_desc* desc);
int lbm_voxel_destroy(lbm_voxel* v);

/* ------------------------------------------------------- result files ---
 * The files of Simulation::WriteOutput (Simulation.cpp:835-856) without VTK.
 * Errors: lbm_last_error(NULL) for file problems, lbm_last_error(e) for an
 * engine state problem (state of the last step not observed). */

/* OutputFile::WriteSurfaceAttribute (OutputFile.cpp:234-316): one row per
 * near-wall node, in the near-wall list's order: X,Y,Z (origin + index x
 * spacing, as Geometry::pointsBox), WSS, with pulsatile != 0 also OSI and
 * TAWSS, and |u|; the reference's header line and ostream number format. */
int lbm_write_surface_csv(lbm_engine* e, const char* path, const double origin[3], double spacing,
                          int32_t pulsatile);

/* OutputFile::processFlowData (OutputFile.cpp:395-483): reads such a file and
 * writes it with WSS (and OSI, TAWSS) replaced by the mean over the other
 * rows within `radius` (the row's own value when there is none). The
 * neighbour search runs on `device`; neighbour sets and summation order are
 * the reference's, so the numbers written are the same. */
int lbm_smooth_surface_csv(const char* in_path, const char* out_path, double radius, int32_t pulsatile,
                           int32_t device);

/* OutputFile::WriteVTK_Collective (OutputFile.cpp:60-230) as VTK XML with raw
 * appended data: every node (order: z, then y, x fastest) with Velocity,
 * Density, VelocityMagnitude, and a hexahedron for each lattice cell (x, y, z)
 * with x < cells[0] - 1, y < cells[1] - 1, z < cells[2] - 1 whose eight
 * corners are nodes; cells = the reference's Geometry nx, ny, nz. */
int lbm_write_vtu(lbm_engine* e, const char* path, const int32_t cells[3]);

/* ------------------------------------------------- pulsatile waveform ---
 * The inlet waveform of Simulation::getInletVelocity (Simulation.cpp:519-534)
 * with its polynomials given instead of fixed (pulsatile.h:55-69 hard-codes
 * the three pieces that config.txt's equations: section lists, and the
 * reference never reads that section). With x = fmod(t, period), piece k
 * applies where bounds[k] * period <= x < bounds[k + 1] * period, and its value
 * is c_0 x^d + c_1 x^(d-1) + ... + c_d, summed left to right with the
 * reference's powers (pow, x * x for the square, x, 1); outside every piece
 * the value is 0. The reference's pieces (bounds 0, 0.1, 0.3, 0.9 of a 0.9 s
 * period with its coefficients) give its waveform bit for bit. */
typedef struct {
    double period;            /* Pulsatile::period */
    int32_t n_pieces;
    const double* bounds;     /* [n_pieces + 1], fractions of the period, ascending */
    const int32_t* n_coeffs;  /* [n_pieces], 1..LBM_PULSE_MAX_COEFFS */
    const double* coeffs;     /* concatenated, highest power first (the equations: order) */
} lbm_pulse_desc;

#define LBM_PULSE_MAX_COEFFS 16

/* Uses w for pulsatile flow from the next step on; NULL restores the
 * reference's built-in waveform. */
int lbm_set_pulsatile(lbm_engine* e, const lbm_pulse_desc* w);

/* The waveform value at time t (host only; w NULL: the reference's).
 * Errors: lbm_last_error(NULL). */
int lbm_pulse_eval(const lbm_pulse_desc* w, double t, double* value);

/* ------------------------------------------------------------ config.txt ---
 * parseInputFile (LBM.h:81-188) with its line grammar: " \t"-trimmed lines,
 * '#' lines skipped, "name:" opens a section; in parameters: key: value
 * (numbers through std::stod / std::stoi, quotes removed from FlowType and
 * stl_file); in inlets / outlets: blocks of plane, coordinate, range_x/y/z
 * and normal lines ended by an empty line (missing ranges are unbounded); in
 * equations: "name: [c0, c1, ...]". Where the reference reads an
 * uninitialised value or indexes past a vector (a block without coordinate
 * or normal, a range with fewer than two values), or a plane other than x,
 * y, z, this parser returns LBM_ERR_ARGUMENT instead.
 *
 * Extension keys in parameters: (the reference's parser skips unknown keys,
 * so a file carrying them still runs there): lattice (D3Q19 | D3Q27, the
 * compile-time choice of Macro.h:49), storage (f64 | f32 | f16 | bf16),
 * boundary (reference | physics), period (of the pulsatile waveform; the
 * reference's file carries it but its parser ignores it and uses 0.9),
 * equation_bounds ([fractions of the period], one more than equations),
 * outlet_density, harmonic_period_steps, harmonic_amplitudes [...],
 * harmonic_phases [...] (FlowType "Harmonic"), device. */
#define LBM_CONFIG_MAX_OPENINGS 64
#define LBM_CONFIG_MAX_EQUATIONS 16
#define LBM_CONFIG_MAX_HARMONICS 16

typedef struct {
    char name[64];
    int32_t n_coeffs;
    double coeffs[LBM_PULSE_MAX_COEFFS];
} lbm_equation;

typedef struct {
    /* SimulationParameters (SimulationParameters.h:51-67) */
    char stl_file[1024];
    char flow_type[64];
    double dt, rho, nu_blood, tau, grid_size, pressure, cte_vel, reynolds_number, systole, diastole;
    int32_t number_of_outlets, max_iter, iter_to_write, num_cycle;
    int32_t n_inlets, n_outlets;
    lbm_opening openings[LBM_CONFIG_MAX_OPENINGS]; /* inlets, then outlets, each in file order */
    int32_t n_equations;
    lbm_equation equations[LBM_CONFIG_MAX_EQUATIONS];
    /* extensions and what follows from them */
    int32_t flow;             /* lbm_flow of FlowType (Constant, Pulsatile, Harmonic), -1 for others */
    int32_t lattice;          /* lbm_lattice, default D3Q19 */
    int32_t storage;          /* lbm_storage, default F64 */
    int32_t bc_mode;          /* lbm_bc_mode, default REFERENCE */
    int32_t device;           /* default 0 */
    double period;            /* default 0.9 */
    int32_t n_bounds;         /* 0: the reference's 0, 0.1, 0.3, 0.9 for three equations */
    double equation_bounds[LBM_CONFIG_MAX_EQUATIONS + 1];
    double outlet_density;    /* default 1 */
    double harmonic_period_steps;
    int32_t n_harmonics;
    double harmonic_amplitudes[LBM_CONFIG_MAX_HARMONICS];
    double harmonic_phases[LBM_CONFIG_MAX_HARMONICS];
} lbm_config;

/* Errors: lbm_last_error(NULL). */
int lbm_config_parse(const char* path, lbm_config* out);

/* ----------------------------------------------------- slab halo exchange ---
 * Replaces the reference's six-face halo exchange of Simulation::Communicate
 * (Simulation.cpp:270-516) over the Cartesian split of SubDomain
 * (Subdomain.cpp:96-245) for a domain cut into slabs, one engine per slab
 * (physics mode). A slab's engine holds its own nodes and, as plain fluid
 * nodes in no list, the ghost copies of the other slabs' nodes next to them.
 * Only the populations that cross a cut move: for the link set L of a pair of
 * slabs A, B (node b of A, direction p, with b - c_p a node of B), the store
 * that precedes a phase-1 step (the initialisation's or a phase-0 step's)
 * leaves in slot p of b the value B's node pulls, and a phase-1 step leaves in
 * B's ghost copy of b, slot p, the value b must receive. So after every step
 * (and once before the first), by lbm_get_phase:
 *   next_phase 1: A packs its list of (b, p) over its own nodes and sends it;
 *                 B unpacks it into the same (b, p) of its ghosts;
 *   next_phase 0: B packs that list over its ghosts and sends it back; A
 *                 unpacks it into its own nodes.
 * Both sides must define the list with the same entries in the same order.
 *
 * lbm_halo_define: list `id` (0..63) of n entries, node (caller index of this
 * engine) and dir (0..Q-1); a list may be defined once. */
int lbm_halo_define(lbm_engine* e, int32_t id, int64_t n, const int64_t* node, const int32_t* dir);

/* Copies list `id`'s slots into dst / from src (device memory, n elements
 * of the storage type: 8, 4 or 2 bytes), on the engine's stream. */
int lbm_halo_pack(lbm_engine* e, int32_t id, void* dst);
int lbm_halo_unpack(lbm_engine* e, int32_t id, const void* src);

/* The phase of the next step: 1 after the initialisation and after a phase-0
 * step, 0 after a phase-1 step. */
int lbm_get_phase(lbm_engine* e, int32_t* next_phase);

/* Message of the last failed call on e (or of the last failed lbm_create when
 * e is NULL). Never NULL. */
const char* lbm_last_error(const lbm_engine* e);

#ifdef __cplusplus
}
#endif

#endif
