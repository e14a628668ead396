/*
 * tfiga.h -- C ABI of the B200 body-fitted IGA Navier-Stokes hot path.
 *
 * This is the drop-in boundary for the solve behind the reference's
 * `iga_cuda navier-stokes` command (solvers/cuda/src/iga_cuda.cu:734-1153).
 * The reference has no FFI of its own: its host loop includes CUDA templates
 * directly.  Each entry point below replaces one of those in-process
 * interfaces; the reference file:line it stands in for is given beside it.
 *
 * Conventions
 *  - Every call returns an int status: 0 on success, a negative TFIGA_E_*
 *    code on failure; tfiga_last_error() gives the message of the calling
 *    thread's last failure.  No C++ exception crosses this boundary.
 *  - Arrays are plain caller-owned host pointers unless the name says
 *    "device"; sizes are explicit.  Nodal vectors are node-major with 4
 *    fields (u, v, w, p): value[4*node + field].
 *  - A tfiga_ns handle owns device state on the current CUDA device and its
 *    own stream; a handle is not thread-safe, use one per host thread.
 *  - Every device-side wait is bounded and reports a status.
 *  - There is no CPU fallback: without a usable sm_100 device the create
 *    calls fail with TFIGA_E_CUDA.
 */
#ifndef TFIGA_H
#define TFIGA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TFIGA_OK 0
#define TFIGA_E_INVALID (-1)       /* bad argument or inconsistent sizes */
#define TFIGA_E_CUDA (-2)          /* CUDA runtime / device failure */
#define TFIGA_E_IO (-3)            /* file could not be read or written */
#define TFIGA_E_FORMAT (-4)        /* malformed .ntiga / case input */
#define TFIGA_E_GEOMETRY (-5)      /* non-positive element Jacobian */
#define TFIGA_E_NOT_CONVERGED (-6) /* linear or nonlinear solve did not converge */
#define TFIGA_E_UNSUPPORTED (-7)   /* valid input outside what this build supports */
#define TFIGA_E_MEMORY (-8)        /* device or host allocation failed */

typedef struct tfiga_mesh tfiga_mesh;
typedef struct tfiga_ns tfiga_ns;
typedef struct tfiga_learned tfiga_learned;
typedef struct tfiga_transport tfiga_transport;

/* Flattened mesh, the layout of iga::cuda::FlatMesh
 * (solvers/cuda/include/DeviceMesh.hpp:16-57). */
typedef struct tfiga_mesh_desc {
	int64_t nodes;
	int64_t elements;
	const int32_t* element_offsets;    /* [elements+1] */
	const int32_t* connectivity;       /* [element_offsets[elements]] */
	const int32_t* extraction_offsets; /* [element_offsets[elements]+1] */
	const uint8_t* extraction_columns; /* [nnz] Bernstein index i+4j+16k */
	const double* extraction_values;   /* [nnz] */
	const double* bezier_points;       /* [elements*64*3] */
	const int32_t* boundary_labels;    /* [elements*6] face labels, -1 = none; may be NULL */
} tfiga_mesh_desc;

typedef struct tfiga_mesh_info {
	int64_t nodes;
	int64_t elements;
	int32_t max_basis;
	int64_t basis_entries;
	int64_t extraction_nonzeros;
	int64_t block_nonzeros;       /* 4x4 blocks of the node-graph pattern */
	int32_t max_block_row;
	double min_detj;              /* min 0.125 det(dx/dxi) over the 4x4x4 Gauss points */
	int64_t bad_samples;          /* Gauss points with det <= 0 or non-finite */
	int64_t device_bytes;         /* resident mesh + pattern + basis tables */
} tfiga_mesh_info;

/* Solver parameters (the options of iga_cuda.cu:402-417 and the fixed
 * GMRES settings of :858 and :1015). */
typedef struct tfiga_ns_params {
	double density;
	double viscosity;              /* dynamic viscosity */
	double dt;                     /* backward-Euler step; 0 = steady */
	int32_t max_newton;            /* default 12 */
	double nonlinear_rtol;         /* default 1e-5 */
	double nonlinear_atol;         /* default 1e-10 (scaled by sqrt(4n)) */
	double mass_rtol;              /* default 1e-3 */
	int32_t gmres_restart;         /* default 200 */
	int32_t gmres_max_iterations;  /* default 5000 */
	double gmres_rtol;             /* default 1e-8 */
	/* TFIGA_PRECONDITIONER_BLOCK_JACOBI: left-preconditioned GMRES with the
	 * reference's tolerance on the preconditioned residual (Gmres.hpp:192-336);
	 * TFIGA_PRECONDITIONER_AMG: flexible GMRES right-preconditioned by one
	 * point-block aggregation AMG V-cycle, tolerance on the true residual. */
	int32_t preconditioner;        /* default TFIGA_PRECONDITIONER_BLOCK_JACOBI */
	/* TFIGA_PRECISION_FP64: every array and operation in FP64 (the reference's precision).
	 * TFIGA_PRECISION_MIXED: FP64 nonlinear residual, Newton update and Krylov vectors;
	 * the element tangent is contracted on the tensor cores (BF16 operands, FP32
	 * accumulation) and the Jacobian is stored in FP32 for SpMV and the preconditioner,
	 * with FGMRES true-residual restarts acting as FP64 iterative refinement.
	 * TFIGA_PRECISION_FP32_JACOBIAN: as MIXED, but the tangent is assembled in FP64 and
	 * rounded once to FP32 for storage.
	 * TFIGA_PRECISION_MIXED_BF16X3: as MIXED, with every tensor-core operand split into
	 * two BF16 terms (x = hi + lo) and three products per tile (hi hi + hi lo + lo hi):
	 * a tangent accurate to about 1e-5 instead of 2e-3, so that Newton converges as with
	 * the FP64 tangent.
	 * TFIGA_PRECISION_MIXED_TF32: as MIXED, with TF32 tensor-core operands (FP32 values
	 * rounded to 10 fraction bits, one product per tile): a tangent accurate to about
	 * 5e-4 with no splitting of the operands.
	 * The reduced modes require TFIGA_PRECONDITIONER_AMG. */
	int32_t precision;             /* default TFIGA_PRECISION_FP64 */
	/* AMG: aggregate until at most this many coarse nodes remain (dense
	 * coarse solve of 4x that order; at most 2048). */
	int32_t amg_coarse_nodes;      /* default 300 */
	/* AMG: rebuild the Galerkin coarse operator and its dense inverse on every
	 * amg_coarse_period-th linear solve only (the fine-level data, A P and the
	 * block-Jacobi inverses, are refreshed on every solve). */
	int32_t amg_coarse_period;     /* default 1 */
	/* Reduced-precision modes: keep the flexible GMRES Krylov basis in FP64 instead
	 * of FP32 (twice the basis traffic; no loss of orthogonality from FP32 storage
	 * over long Arnoldi cycles).  Ignored in TFIGA_PRECISION_FP64. */
	int32_t krylov_fp64_basis;     /* default 0 */
	/* Inexact Newton: 1 solves each Newton system to an Eisenstat-Walker forcing
	 * tolerance eta_k = 0.9 (|r_k| / |r_{k-1}|)^2 (safeguarded, at most 1e-3, at least
	 * gmres_rtol and at least half of what the Newton tolerance still asks for)
	 * instead of gmres_rtol.  The step (tfiga_ns_step and the outlet steps) first sets
	 * the constrained entries of the state to their prescribed values, so the residual
	 * of the first Newton iteration -- the reference of the relative Newton test -- is
	 * that of the PDE rows at the lifted state.  0 (default): every system to
	 * gmres_rtol and no lifting, as the reference. */
	int32_t newton_forcing;        /* default 0 */
	/* Every precision mode: a factor c > 0 keeps the previous Newton iteration's
	 * tangent (and its Dirichlet rows) while that iteration reached what its linear
	 * tolerance allowed, |r_k| <= c eta_{k-1} |r_{k-1}| (eta the relative tolerance
	 * of the previous linear solve): a tangent that still gives the contraction the
	 * linear solve asked for is good enough.  The tangent is assembled afresh at the
	 * first iteration of every step and whenever the contraction falls short.  The
	 * residual is always evaluated in FP64 at the current state (by its own kernel,
	 * before the tangent, so a converged check assembles no tangent), so only the
	 * Newton convergence rate can change.  Default 0 (off). */
	double tangent_reuse_factor;   /* default 0 */
	/* Tensor-core modes: how the tangent's operands reach the tensor cores.
	 * TFIGA_TANGENT_COEFFICIENTS: the point kernel stores every element's point
	 * coefficients (80 KiB per element) and an FP32 copy of the basis tables is kept;
	 * TFIGA_TANGENT_FUSED: the point kernel stores the FP64 point state (11 KiB per
	 * element) and the tensor-core kernel makes the coefficients itself and stages
	 * the basis from the FP64 tables (about 96 KiB per element less);
	 * TFIGA_TANGENT_ELEMENT: the arrays of TFIGA_TANGENT_COEFFICIENTS contracted by one
	 * persistent CTA per SM that takes whole elements (all four row fields at once, the
	 * basis staged once per element);
	 * TFIGA_TANGENT_AUTO: the first tangent assembly times the three (the two
	 * coefficient-array ones when their memory is free) and keeps the fastest; the
	 * fused one otherwise.
	 * All give the same tangent up to the order of the FP32 additions. */
	int32_t tangent_kernel;        /* default TFIGA_TANGENT_AUTO */
} tfiga_ns_params;

#define TFIGA_PRECISION_FP64 0
#define TFIGA_PRECISION_MIXED 1
#define TFIGA_PRECISION_FP32_JACOBIAN 2
#define TFIGA_PRECISION_MIXED_BF16X3 3
#define TFIGA_PRECISION_MIXED_TF32 4
#define TFIGA_LEARNED_RESIDUAL_LOSS 0
#define TFIGA_LEARNED_ERROR_LOSS 1
#define TFIGA_TANGENT_AUTO 0
#define TFIGA_TANGENT_COEFFICIENTS 1
#define TFIGA_TANGENT_FUSED 2
#define TFIGA_TANGENT_ELEMENT 3

#define TFIGA_PRECONDITIONER_BLOCK_JACOBI 0
#define TFIGA_PRECONDITIONER_AMG 1

/* One Newton iteration's log record (iga_cuda.cu:1000-1009, 1034-1045). */
typedef struct tfiga_newton_report {
	int32_t converged;             /* 1 when the convergence test passed before solving */
	int32_t linear_iterations;
	int32_t singular_diagonal_blocks;
	double residual_l2;            /* ||rhs|| after the Dirichlet rows */
	double tolerance;
	double continuity_l2;          /* from the raw rhs before Dirichlet rows */
	double continuity_sum;
	double net_boundary_flow;
	double absolute_boundary_flow;
	double relative_mass_imbalance;
	double update_l2;
	double linear_residual;
	double assembly_ms;
	double linear_ms;
} tfiga_newton_report;

/* Multigrid hierarchy of the AMG preconditioner (after the first solve). */
typedef struct tfiga_amg_info {
	int32_t levels;
	int32_t nodes[8];
	int64_t blocks[8];
	int64_t transfer_blocks;      /* 4x4 blocks of A P (fine operator times prolongation) */
} tfiga_amg_info;

/* One physical step (the Newton loop of iga_cuda.cu:956-1054). */
typedef struct tfiga_step_report {
	int32_t converged;
	int32_t newton_iterations;
	int32_t linear_iterations;
	double residual_l2;
	double initial_residual_l2;
	double relative_mass_imbalance;
	double assembly_ms;
	double linear_ms;
} tfiga_step_report;

/* Outlet model of one labelled outlet (OutletModelState, include/OutletModel.hpp:15-26;
 * EvaluateOutletModel :70-90): resistance P = Pref + R Q; RC / RCR capacitor
 * Pc = (C Pc_prev / dt + Q + Pref / R_d) / (C / dt + 1 / R_d), P = Pc (+ R_p Q for RCR). */
enum { TFIGA_OUTLET_RESISTANCE = 0, TFIGA_OUTLET_RC = 1, TFIGA_OUTLET_RCR = 2 };
typedef struct tfiga_outlet {
	int32_t label;
	int32_t kind;                 /* TFIGA_OUTLET_* */
	double resistance;            /* resistance and RC models */
	double proximal_resistance;   /* RCR R_p */
	double distal_resistance;     /* RCR R_d */
	double capacitance;
	double reference_pressure;
	double capacitor_pressure;    /* in: committed value of the previous step; out: this step's */
	double flow;                  /* out: outward flow of the accepted iterate */
	double pressure;              /* in: first traction; out: accepted pressure */
} tfiga_outlet;

/* ---- errors ------------------------------------------------------------ */
/* Copies the calling thread's last error message; returns its full length. */
size_t tfiga_last_error(char* buffer, size_t capacity);
/* Library build string (arch, version). */
const char* tfiga_version(void);

/* ---- mesh -------------------------------------------------------------- */
/* Replaces FlatMesh + DeviceMesh + BlockPattern + DevicePattern + ReferenceData
 * + GeometryData (iga_cuda.cu:820-851; DeviceMesh.hpp:27-114; BlockCsr.hpp:15-55;
 * iga_cuda.cu:73-220): uploads the mesh, builds the block pattern and the
 * per-element basis tables on the device, and checks the geometry. */
int tfiga_mesh_create(const tfiga_mesh_desc* desc, tfiga_mesh** out);
/* Batched tubes: the disjoint union of `count` meshes as one mesh, solved by one
 * tfiga_ns handle (the tubes' unknowns form independent diagonal blocks of one
 * system; connectivity of tube k is offset by the nodes of tubes 0..k-1, the
 * geometry is used as given).  node_offsets / element_offsets [count+1] (either
 * may be NULL) receive where each tube's nodes and elements start; they are
 * filled before the device mesh is built.  No counterpart in the reference
 * (its C5-like runs solve one tube per process). */
int tfiga_batch_mesh_create(const tfiga_mesh_desc* tubes, int32_t count, tfiga_mesh** out, int64_t* node_offsets,
	int64_t* element_offsets);
/* Same from a packed .ntiga file (iga::Database, IgaDatabase.hpp:95-161). */
int tfiga_mesh_load_ntiga(const char* path, tfiga_mesh** out);
int tfiga_mesh_destroy(tfiga_mesh* mesh);
/* mesh-check numbers (iga_cuda.cu:604-617). */
int tfiga_mesh_info_get(const tfiga_mesh* mesh, tfiga_mesh_info* info);
/* Block-CSR pattern (BlockPattern, BlockCsr.hpp:15-55): row_offsets[nodes+1],
 * columns[blocks], diagonal[nodes]; any pointer may be NULL. */
int tfiga_mesh_pattern(const tfiga_mesh* mesh, int32_t* row_offsets, int32_t* columns, int32_t* diagonal);

/* ---- Navier-Stokes solver -------------------------------------------- */
void tfiga_ns_default_params(tfiga_ns_params* params);
/* Allocates matrix, vectors and the GMRES workspace (iga_cuda.cu:858-865, 899). */
int tfiga_ns_create(tfiga_mesh* mesh, const tfiga_ns_params* params, tfiga_ns** out);
int tfiga_ns_destroy(tfiga_ns* ns);
/* Dirichlet masks and values (ResolvedBoundaryConditions after the wall trace,
 * iga_cuda.cu:750-797 and :854-857): masks [nodes] (nonzero = constrained),
 * velocity [3*nodes], pressure [nodes]; pressure may be NULL (all zero). */
int tfiga_ns_set_dirichlet(tfiga_ns* ns, const int32_t* velocity_mask, const int32_t* pressure_mask,
	const double* velocity, const double* pressure);
/* Dirichlet values only (per-step waveform update, iga_cuda.cu:944-946). */
int tfiga_ns_set_dirichlet_values(tfiga_ns* ns, const double* velocity, const double* pressure);
/* Natural pressure traction on labelled faces (IntegratePressureTractionForces,
 * PressureTractionFlow.hpp:41-64; iga_cuda.cu:948-951), computed on the device. */
int tfiga_ns_set_tractions(tfiga_ns* ns, const int32_t* labels, const double* pressures, int32_t count);
/* State and previous state [4*nodes]; previous may be NULL (= state). */
int tfiga_ns_set_state(tfiga_ns* ns, const double* state, const double* previous);
int tfiga_ns_get_state(tfiga_ns* ns, double* state);
/* previous <- state (start of a physical step, iga_cuda.cu:918-920). */
int tfiga_ns_commit_step(tfiga_ns* ns);
/* Raw assembly for parity tests: Jacobian values [blocks*16] (row-major 4x4
 * blocks) and rhs = -r + traction [4*nodes], before the Dirichlet rows;
 * either output may be NULL (AssembleNavierStokesKernel + the traction axpy,
 * iga_cuda.cu:959-969, with the exact tangent of NavierStokesElement.hpp:244-312). */
int tfiga_ns_assemble(tfiga_ns* ns, double* values, double* rhs);
/* Dirichlet rows applied to the last assembly (IgaCudaKernels.cuh:436-463):
 * copies back values/rhs after the rows were applied; either may be NULL. */
int tfiga_ns_apply_dirichlet(tfiga_ns* ns, double* values, double* rhs);
/* Block-Jacobi GMRES on the current (Dirichlet-applied) system
 * (SolveGmres, Gmres.hpp:192-336): update = A^{-1} rhs. */
int tfiga_ns_solve_linear(tfiga_ns* ns, double rtol, int32_t max_iterations, double* update,
	int32_t* iterations, double* residual);
/* One full Newton iteration: assemble, diagnostics, Dirichlet rows, norm and
 * convergence test, GMRES, state += update (iga_cuda.cu:956-1046).
 * initial_residual is the step's first residual norm (<0 on the first iteration). */
int tfiga_ns_newton_iteration(tfiga_ns* ns, double initial_residual, tfiga_newton_report* report);
/* One physical step: the Newton loop to convergence (iga_cuda.cu:952-1054). */
int tfiga_ns_step(tfiga_ns* ns, tfiga_step_report* report);
/* One physical step coupled to outlet models by the relaxed fixed point of
 * iga_cuda.cu:927-1086 (EvaluateOutletCoupling / OutletCouplingTolerance /
 * RelaxOutletCoupling / CommitOutletCoupling, OutletModel.hpp:92-150): the Newton
 * loop runs with each outlet's pressure as its traction (other labels keep the
 * tractions of tfiga_ns_set_tractions), the outward flows are evaluated, and the
 * iteration stops when max |P_eval - P| <= 1e-8 + 1e-6 max(1, |P_eval|); otherwise
 * P <- (1 - relaxation) P + relaxation P_eval.  The reference uses relaxation 0.5
 * and 12 iterations; with rigid walls and a Dirichlet inflow the total outlet flow
 * does not depend on the outlet pressures, so relaxation 1 reaches the same fixed
 * point in two iterations.  report sums the Newton and linear counts over all
 * outlet iterations; *outlet_iterations (may be NULL) is the number of Newton
 * loops.  TFIGA_E_NOT_CONVERGED after max_iterations. */
int tfiga_ns_step_outlets(tfiga_ns* ns, tfiga_outlet* outlets, int32_t count, double relaxation,
	int32_t max_iterations, tfiga_step_report* report, int32_t* outlet_iterations);
/* One physical step with the outlet models coupled inside a single Newton loop
 * (no reference counterpart; same fixed point and acceptance tests as
 * tfiga_ns_step_outlets): after every Newton update the outward flows are
 * evaluated and each outlet pressure P moves to (1 - relaxation) P + relaxation
 * P_eval; the step is accepted when the Newton residual test holds (relative to
 * the step's first residual) and max |P_eval - P| <= 1e-8 + 1e-6 max(1, |P_eval|).
 * The reference's outer loop restarts Newton for every outlet iteration and
 * tightens the residual test to the new, small initial residual; this form
 * needs about as many Newton solves as a step without outlets.  report counts
 * the solves; *pressure_updates (may be NULL) the pressure changes.
 * TFIGA_E_NOT_CONVERGED after max_newton Newton iterations. */
int tfiga_ns_step_outlets_coupled(tfiga_ns* ns, tfiga_outlet* outlets, int32_t count, double relaxation,
	int32_t max_newton, tfiga_step_report* report, int32_t* pressure_updates);
/* AMG hierarchy sizes (levels = 0 before the hierarchy is built). */
int tfiga_ns_amg_info(tfiga_ns* ns, tfiga_amg_info* info);
/* Batched tubes (a batching form with no counterpart in the reference, which solves one mesh): the
 * node ranges [node_offsets[k], node_offsets[k+1]) of count independent tubes (node_offsets increasing
 * from 0 to nodes, e.g. tfiga_batch_mesh_create's node offsets); count 0 removes them.  The Newton
 * test is then taken per tube, relative to the tube's own first residual of the step, and a tube that
 * passes is frozen for the rest of the step (its rows of the linear system carry a zero rhs); the
 * linear solves run one FGMRES per tube over shared launches (each tube its own Arnoldi process,
 * Hessenberg matrix and tolerance, stopping on its own; the AMG preconditioner only; each Arnoldi step
 * replayed from a CUDA graph captured on its first use, except while profiling), each open
 * tube's rhs scaled to unit norm and its update scaled back; the step converges when every tube has
 * passed. */
int tfiga_ns_set_segments(tfiga_ns* ns, const int64_t* node_offsets, int32_t count);
/* Per tube, after a Newton iteration: done[k] 1 when tube k has passed its test in this step, and its
 * residual norm (either output may be NULL). */
int tfiga_ns_segment_status(tfiga_ns* ns, int32_t* done, double* residuals);
/* Tensor-core modes: the tangent organisation in use (*kernel: TFIGA_TANGENT_*, AUTO before the
 * first tangent) and the autotuner's times of the coefficient-array (row-field-pair kernel) and fused
 * organisations (ms, 0 when not timed).  No counterpart in the reference.  Any output may be NULL. */
int tfiga_ns_tangent_kernel(tfiga_ns* ns, int32_t* kernel, double* coefficients_ms, double* fused_ms);
/* The autotuner's time of the element kernel (TFIGA_TANGENT_ELEMENT) on the coefficient arrays (ms, 0
 * when not timed). */
int tfiga_ns_tangent_element_ms(tfiga_ns* ns, double* element_ms);
/* Outward flow through each labelled boundary (IntegrateBoundaryFlow,
 * BoundaryFlow.hpp:165-200; MeasureFlowConvergence iga_cuda.cu:520-557). */
int tfiga_ns_boundary_flows(tfiga_ns* ns, const int32_t* labels, int32_t count, double* flows);

/* ---- raw kernels on device pointers (measurement and integration) ------ */
/* y = A x over the mesh pattern with the active Jacobian (FP32 storage in the
 * reduced-precision modes) (BlockSpmvKernel<4>, SparseKernels.cuh:25-40). */
int tfiga_ns_spmv_device(tfiga_ns* ns, const double* x_device, double* y_device);
/* Device pointers of the handle's FP64 matrix values (NULL in
 * TFIGA_PRECISION_MIXED, which keeps no FP64 Jacobian), state and rhs. */
int tfiga_ns_device_buffers(tfiga_ns* ns, double** values, double** state, double** rhs);
/* Counters of kernel launches issued by this handle (for launch accounting). */
int64_t tfiga_ns_launch_count(const tfiga_ns* ns);
/* Waits for the handle's stream (bounded by the driver). */
int tfiga_ns_synchronize(tfiga_ns* ns);
/* The handle's CUDA stream (a cudaStream_t), for callers that time with
 * CUDA events on the launching stream. */
int tfiga_ns_stream(tfiga_ns* ns, void** stream);
/* Per-kernel-family device timing with CUDA events recorded around each
 * launch on the handle's stream (the reference's PhaseProfile,
 * include/PhaseProfile.hpp:14-138, at kernel granularity).  Families:
 * 0 assembly (the tangent; in the tensor-core modes the tcgen05 kernel),
 * 1 SpMV (fused with the block-Jacobi apply in that mode), 2 Krylov
 * orthogonalisation, 3 AMG V-cycle, 4 the FP64 residual and point
 * coefficients of the tensor-core modes (0 elsewhere: the FP64 kernel does
 * both in family 0), 5 AMG set-up for a new Jacobian (point-block inverses,
 * Galerkin coarse operator, dense coarse inverse), 6 the Newton loop's own
 * vector work (residual and Jacobian zeroing, traction, convergence
 * diagnostics, Dirichlet rows, norms, the state update, device outlet
 * coupling, per-segment tests). */
#define TFIGA_PROFILE_FAMILIES 7
int tfiga_ns_set_profiling(tfiga_ns* ns, int enable);
/* Totals since the last reset: milliseconds and launch counts per family. */
int tfiga_ns_profile(tfiga_ns* ns, double* milliseconds, int64_t* launches, int32_t reset);
/* Bytes per family since the last reset, as the solver accounts them while
 * profiling is on: bytes[0..6] algorithmic, bytes[7..13] actually moved
 * (2 * TFIGA_PROFILE_FAMILIES entries).  Family 2, Krylov orthogonalisation:
 * algorithmic s_v n (2j + 7) per Arnoldi step j (+ 8 n for the stored
 * FGMRES vector), s_v the basis entry size; moved: both classical
 * Gram-Schmidt passes.  The other families report 0. */
int tfiga_ns_profile_bytes(tfiga_ns* ns, double* bytes);

/* ---- learned FGMRES preconditioner stage ------------------------------ */
/* A message-passing network over the element face-adjacency graph (hidden
 * width 64, `layers` message-passing layers) that adds N(D^{-1} r) to the AMG
 * application inside the flexible GMRES: z = M_AMG(r) + N(D^{-1} r).  FGMRES
 * still drives the FP64 true residual to the same tolerance, so the network
 * changes only the iteration count.  Training pairs come from the solver
 * itself: with `collect` on, every solved Newton system J delta = b adds
 * (D^{-1} b / |b|, (delta - M_AMG(b)) / |b|).  Inference reads BF16 weights
 * with FP32 accumulation; training (hand-written backward kernels, Adam)
 * keeps FP32 master weights.  The parameter vector layout and the network
 * definition are those of the CPU oracle (oracle/learned_oracle.py).  No
 * counterpart in the reference.  Needs TFIGA_PRECONDITIONER_AMG.  Destroying
 * the ns handle detaches it. */
/* linear != 0: identity activation and zero biases (the stage is then a fixed linear operator). */
int tfiga_learned_create(tfiga_ns* ns, int32_t layers, uint64_t seed, int32_t linear, tfiga_learned** out);
int tfiga_learned_destroy(tfiga_learned* learned);
int tfiga_learned_info(const tfiga_learned* learned, int64_t* parameters, int64_t* elements, int32_t* pairs);
/* learned = NULL detaches; use: apply in the FGMRES; collect: store a pair per Newton solve. */
int tfiga_ns_set_learned(tfiga_ns* ns, tfiga_learned* learned, int32_t use, int32_t collect);
/* Linear solves that did not converge with the learned stage and were redone with the AMG alone. */
int tfiga_ns_learned_fallbacks(const tfiga_ns* ns, int64_t* count);
/* Training loss: TFIGA_LEARNED_RESIDUAL_LOSS (default) fits A N(x) to the residual the AMG leaves,
 * through the current Jacobian; TFIGA_LEARNED_ERROR_LOSS fits N(x) to the FP64 error of the AMG,
 * delta - M_AMG(b), of the solver's own (residual, FP64 solution) pairs. */
int tfiga_learned_set_loss(tfiga_learned* learned, int32_t loss);
/* Pair store size (default 128; before the first pair is stored): 3 vectors of 4n doubles each. */
int tfiga_learned_set_capacity(tfiga_learned* learned, int32_t capacity);
/* Per-field input/output scales and loss weights from the stored pairs. */
int tfiga_learned_fit_scales(tfiga_learned* learned);
/* `steps` Adam steps over the stored pairs; *loss = mean loss of the last pass. */
int tfiga_learned_train(tfiga_learned* learned, int32_t steps, double learning_rate, double* loss);
int tfiga_learned_evaluate(tfiga_learned* learned, double* loss);
/* Least-squares output gain over the stored pairs, folded into the output scales (clamped at 0, so
 * a stage that learned nothing adds nothing); *gain receives it. */
int tfiga_learned_fit_gain(tfiga_learned* learned, double* gain);
int tfiga_learned_get_parameters(const tfiga_learned* learned, float* parameters);
int tfiga_learned_set_parameters(tfiga_learned* learned, const float* parameters);
/* scales[0..3] input, [4..7] output, [8..11] loss weights. */
int tfiga_learned_get_scales(const tfiga_learned* learned, double* scales);
int tfiga_learned_set_scales(tfiga_learned* learned, const double* scales);
/* Face neighbours [6 * elements], -1 = none. */
int tfiga_learned_neighbours(const tfiga_learned* learned, int32_t* neighbours);
/* FP32 forward o = N(x) and loss/gradient against a target (device vectors of 4n doubles). */
int tfiga_learned_forward_device(tfiga_learned* learned, const double* x_device, double* o_device);
/* The inference path used inside the FGMRES (BF16 weights): z_device += N(x_device). */
int tfiga_learned_apply_device(tfiga_learned* learned, const double* x_device, double* z_device);
int tfiga_learned_loss_gradient_device(tfiga_learned* learned, const double* x_device, const double* target_device,
	double* loss, float* gradient);
int tfiga_learned_save(const tfiga_learned* learned, const char* path);
int tfiga_learned_load(tfiga_learned* learned, const char* path);

/* ---- case inputs (host only) ------------------------------------------ */
/* The flow boundary set-up of the navier-stokes command for a simulation_config.json case at
 * physical time `time` with the outlet models at their initial state (iga_cuda.cu:766-790:
 * ReadSimulationConfiguration, FindNavierStokesSystem, InitializeOutletModels,
 * MaterializeBoundaryWaveforms, MaterializeOutletPressures, ExtractPressureTractions,
 * ResolveFlowBoundaries), before the wall trace.  system may be NULL or "" (the first
 * Navier-Stokes system).  Outputs [nodes] ([3*nodes] for velocity; any may be NULL);
 * counts[2] = velocity, pressure nodes; traction_labels / traction_values receive up to
 * *traction_count entries (in: capacity, out: the number of labelled pressure tractions);
 * physics[5] = viscosity, density, dt, steps, transient (1 or 0). */
int tfiga_resolve_flow_boundaries(const char* config_path, const char* system, double time, int64_t nodes,
	const int32_t* labels, const double* reference_velocity, int32_t* velocity_mask, double* velocity,
	int32_t* pressure_mask, double* pressure, int64_t* counts, int32_t* traction_labels, double* traction_values,
	int32_t* traction_count, double* physics);

/* The navier-stokes command's VTU snapshot (WriteNavierStokesVtu, iga_cuda.cu:366-388; WriteVtu,
 * include/VtkOutput.hpp:107-155): the control mesh of the legacy ASCII mesh_vtk with `velocity` (3)
 * and `pressure` (1) point arrays from state [4*nodes] and TimeValue = time.  Host only. */
int tfiga_write_vtu(const char* mesh_vtk, const char* output, const double* state, int64_t nodes, double time);

/* The bases the navier-stokes command holds at no slip (WallTraceBasis,
 * solvers/cpu/include/BoundarySupport.hpp:82-150): every basis with a nonzero trace on a face of
 * controlmesh.vtk's wall (label 0) hexes, from the database read by this library's .ntiga reader.
 * Sorted node indices, up to `capacity` written; *count = their number.  Host only. */
int tfiga_wall_trace_basis(const char* database, const char* controlmesh_vtk, int32_t* nodes, int64_t capacity,
	int64_t* count);

/* The navier-stokes command's checkpoint (WriteCudaFlowCheckpoint, iga_cuda.cu:584-602):
 * PREFIX.state (raw float64 [4*nodes]) and PREFIX.json (schema 1: nodes, fields, completed step,
 * time, dt, density, viscosity, state file and format, outlet states).  Host only. */
int tfiga_write_flow_checkpoint(const char* prefix, int64_t nodes, int32_t completed_step, double physical_time,
	double dt, double density, double viscosity, const tfiga_outlet* outlets, int32_t count, const double* state);
/* Restart from it (ReadFlowCheckpointMetadata + ValidateFlowCheckpoint + ReadCudaFlowCheckpoint,
 * include/FlowCheckpoint.hpp:186-211, iga_cuda.cu:566-582): checks nodes, dt, density, viscosity
 * and the state size; outlets whose labels appear take the stored flow, pressure and capacitor
 * pressure.  Host only. */
int tfiga_read_flow_checkpoint(const char* prefix, int64_t nodes, double dt, double density, double viscosity,
	tfiga_outlet* outlets, int32_t count, double* state, int32_t* completed_step, double* physical_time);

/* ---- two-species transport ------------------------------------------ */
/* The `iga_cuda transport` path (Transport, solvers/cuda/src/iga_cuda.cu:621-732):
 * N0 (attached: diffusion and exchange) and N+ (advected by a prescribed nodal
 * velocity, SUPG-stabilised) on the mesh of a tfiga_mesh, 2 unknowns per node
 * stored value[2*node + field] (field 0 = N0, 1 = N+), 2x2 blocks
 * values[block*4 + 2*i + j] on the mesh's block pattern.  Backward Euler with
 * a constant left matrix L and previous-state matrix P assembled once
 * (AssembleTransportKernel, IgaCudaKernels.cuh:155-237; the CPU element is
 * BuildTransportElement, solvers/cpu/include/TransportElement.hpp:213-253);
 * constrained rows zeroed with an identity diagonal block in L
 * (ApplyTransportBoundaryKernel, IgaCudaKernels.cuh:411-424).  A step is
 * rhs = P c, the boundary values written into rhs
 * (SetTransportBoundaryVectorKernel :426-434), then L c' = rhs by block-Jacobi
 * GMRES(restart) to gmres_rtol of the preconditioned residual, started from 0
 * on the first step and from c afterwards, the block inverse built once. */

/* iga::TransportParameters (solvers/cpu/include/CaseInput.hpp:19-33) plus the
 * solver settings the reference fixes in Transport (restart 50, rtol 1e-8,
 * at most 10000 iterations: iga_cuda.cu:660, 691). */
typedef struct tfiga_transport_params {
	double diffusion;            /* D: N0 diffusion */
	double vplus;                /* inlet velocity scale; weights the artificial diffusion */
	double vminus;               /* read, unused by the two-species model */
	double kplus;                /* N0 -> N+ exchange rate */
	double kminus;               /* N0 loss rate */
	double detach_plus;          /* k'plus: N+ -> N0 detachment rate */
	double detach_minus;         /* k'minus: read, unused */
	double dt;
	int32_t steps;               /* nstep */
	int32_t restart;             /* GMRES restart */
	double n0_bc;                /* N0bc: legacy inlet value of N0 */
	double nplus_bc;             /* Nplusbc: legacy inlet value of N+ */
	double nminus_bc;            /* Nminusbc: read, unused */
	double artificial_diffusion; /* SUPG-weighted artificial diffusion coefficient */
	double gmres_rtol;
	int32_t gmres_max_iterations;
	/* TFIGA_PRECISION_FP64 (the reference's arithmetic) or TFIGA_PRECISION_MIXED:
	 * L also kept in FP32 for the SpMV inside the Arnoldi process, while the
	 * block inverse, the vectors and the true residual of every restart (the
	 * stopping test) stay FP64. */
	int32_t precision;
	/* TFIGA_TRANSPORT_BLOCK_JACOBI (the reference's) or TFIGA_TRANSPORT_FLOW_LINES: exact solves
	 * along flow lines read from L (tfiga_transport_flow_lines), factored once per handle. */
	int32_t preconditioner;
	int32_t reserved;
} tfiga_transport_params;

#define TFIGA_TRANSPORT_BLOCK_JACOBI 0
#define TFIGA_TRANSPORT_FLOW_LINES 1

/* Totals of one tfiga_transport_step call (the `transport step=` and
 * `transport_cuda` log lines, iga_cuda.cu:702-731). */
typedef struct tfiga_transport_report {
	int32_t steps;               /* steps taken by the call */
	int32_t last_iterations;     /* GMRES iterations of the last step */
	int64_t total_iterations;    /* over the call's steps */
	double last_residual;        /* final preconditioned residual of the last step */
	double final_l2;             /* ||c||_2 after the last step (cublasDnrm2, iga_cuda.cu:711-713) */
	uint32_t singular_blocks;    /* singular diagonal blocks of the block-Jacobi build */
	uint32_t reserved;
} tfiga_transport_report;

/* Zeros, restart 50, gmres_rtol 1e-8, gmres_max_iterations 10000, FP64. */
void tfiga_transport_default_params(tfiga_transport_params* params);
/* simulation_parameter.txt (ReadTransportParameters, CaseInput.hpp:85-118) into
 * the physical fields of *params (solver fields untouched).  Errors:
 * TFIGA_E_IO (unreadable), TFIGA_E_FORMAT (missing key, dt <= 0, nstep < 0). */
int tfiga_transport_read_params(const char* path, tfiga_transport_params* params);
/* Boundary resolution of a legacy case (ResolveBoundaryConditions,
 * CaseInput.hpp:162-258): labels[nodes] of controlmesh.vtk, the reference
 * velocity [3*nodes] and, when case_config_path names an existing file, its
 * schema-1 rules (ReadCaseConfiguration, include/CaseConfig.hpp:280-387).
 * Writes the transport mask and values [nodes] (any may be NULL) and returns
 * the constrained count in *transport_nodes. */
int tfiga_transport_resolve_boundaries(int64_t nodes, const int32_t* labels, const double* reference_velocity,
	const tfiga_transport_params* params, const char* case_config_path, int32_t* constrained, double* n0,
	double* nplus, int64_t* transport_nodes);
/* The whole resolution of a legacy case (ResolveBoundaryConditions, CaseInput.hpp:162-258), as the
 * navier-stokes command uses it without simulation_config.json: velocity mask and values [nodes],
 * [3*nodes], pressure mask and values, transport mask and values [nodes] (any output may be NULL);
 * counts[3] = velocity, pressure and transport nodes (may be NULL).  Host only. */
int tfiga_resolve_legacy_boundaries(int64_t nodes, const int32_t* labels, const double* reference_velocity,
	const tfiga_transport_params* params, const char* case_config_path, int32_t* velocity_mask, double* velocity,
	int32_t* pressure_mask, double* pressure, int32_t* transport_mask, double* n0, double* nplus, int64_t* counts);
/* The flow-line preconditioner's host construction for a 2x2 block system given by host arrays
 * (row_offsets [nodes+1], sorted columns, values [4*blocks]): lines chained along the largest
 * antisymmetric coupling of the second field (a_ij = L++_ji - L++_ij > 0), then the banded 2x2-block
 * LU (no pivoting) of every line's system.  Outputs (any may be NULL): line_offsets [lines+1],
 * line_nodes [nodes], band_width and band_offsets [lines], factors [*factor_count]; *lines and
 * *factor_count give the sizes (call once with NULL arrays to size them).  No counterpart in the
 * reference (it preconditions with block-Jacobi).  Host only. */
int tfiga_transport_flow_lines(int64_t nodes, const int32_t* row_offsets, const int32_t* columns,
	const double* values, int32_t* line_offsets, int32_t* line_nodes, int32_t* band_width, int64_t* band_offsets,
	double* factors, int32_t* lines, int64_t* factor_count);
/* Assembles L and P from the nodal velocity [3*nodes], applies the boundary
 * rows of the constrained[nodes] mask and sets the boundary values n0/nplus
 * [nodes] into the zero initial state (iga_cuda.cu:664-679).  Host or device
 * pointers.  The handle keeps a reference to the mesh. */
int tfiga_transport_create(tfiga_mesh* mesh, const tfiga_transport_params* params, const double* velocity,
	const int32_t* constrained, const double* n0, const double* nplus, tfiga_transport** out);
int tfiga_transport_destroy(tfiga_transport* transport);
/* `steps` backward-Euler steps (the loop of iga_cuda.cu:683-707); report may
 * be NULL.  TFIGA_E_NOT_CONVERGED when a step's GMRES stops above tolerance. */
int tfiga_transport_step(tfiga_transport* transport, int32_t steps, tfiga_transport_report* report);
/* State c [2*nodes], host or device. */
int tfiga_transport_set_state(tfiga_transport* transport, const double* state);
int tfiga_transport_get_state(tfiga_transport* transport, double* state);
/* L and P after the boundary rows, [4*blocks] each (either may be NULL). */
int tfiga_transport_matrices(tfiga_transport* transport, double* left, double* previous);
/* y = M^{-1} x [2*nodes] (host or device) with the handle's flow-line factors
 * (params.preconditioner TFIGA_TRANSPORT_FLOW_LINES; TFIGA_E_INVALID otherwise): the
 * device application the GMRES uses, exposed to check it.  No counterpart in the
 * reference (it preconditions with block-Jacobi). */
int tfiga_transport_apply_preconditioner(tfiga_transport* transport, const double* x, double* y);
/* Device time of the assembly launch sequence (ms), steps taken, kernel launches issued. */
int tfiga_transport_info(const tfiga_transport* transport, double* assembly_ms, int32_t* steps, int64_t* launches);
/* The handle's CUDA stream (a cudaStream_t). */
int tfiga_transport_stream(tfiga_transport* transport, void** stream);
/* Per-family device timing as tfiga_ns_set_profiling / tfiga_ns_profile:
 * family 1 SpMV (P c and the block-Jacobi SpMV of GMRES), 2 Krylov
 * orthogonalisation; the others stay 0. */
int tfiga_transport_set_profiling(tfiga_transport* transport, int enable);
int tfiga_transport_profile(tfiga_transport* transport, double* milliseconds, int64_t* launches, int32_t reset);

/* ---- allocation-free kernel ------------------------------------------- */
/* *norm_device = ||b - A x||_2 for a 4x4 block-CSR matrix given entirely by
 * device pointers (row_offsets [nodes+1], columns and values [blocks*16]
 * FP64, x and b [4*nodes]), enqueued on `stream` (a cudaStream_t; NULL is
 * the legacy default stream).  No counterpart in the reference: it exists for
 * callers that may not allocate device memory at call time.  It allocates
 * nothing: its scratch is a static device array of 32768 partial sums, so
 * nodes <= 262144 (larger -> TFIGA_E_UNSUPPORTED, nothing launched).  No
 * scratch has to start at zero.  Calls share that scratch, so calls whose
 * kernels could overlap must be serialized.  The first call on a device looks
 * up the scratch address; make it before any stream capture begins.  The
 * address is kept with the id of the context it was looked up in: after
 * cudaDeviceReset the next call looks it up again (so, again, outside any
 * capture). */
int tfiga_block_residual_norm_static(int64_t nodes, const int32_t* row_offsets_device,
	const int32_t* columns_device, const double* values_device, const double* x_device, const double* b_device,
	double* norm_device, void* stream);

/* ---- drop-in command ------------------------------------------------- */
/* `navier-stokes DATABASE CASE_DIR [MAX_NEWTON] [OUTPUT] [options]`, the argv of
 * iga_cuda's navier-stokes command (ParseCudaFlowOptions iga_cuda.cu:447-498,
 * NavierStokes :734-1153), or `transport DATABASE CASE_DIR [STEPS] [OUTPUT]
 * [VELOCITY]` (Transport :621-732).  argv[0] is the program name, argv[1] the
 * command ("navier-stokes", "transport", "mesh-check" or "device-info").  Prints the reference's
 * key=value lines to stdout; returns the process exit code (0 or 1). */
int tfiga_main(int argc, char** argv);

#ifdef __cplusplus
}
#endif

#endif
