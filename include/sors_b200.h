/*
 * sors_b200.h -- C ABI of the B200 implicit-Euler FEM step (libsors_b200.so).
 *
 * Plain C: opaque handle, caller-owned buffers, int32 status codes.  All
 * vectors are FP64, 3*N long, in the reference's DOF order (3*vertex +
 * component, cpp/src/energy.cpp:217-222).  Host pointers unless a name says
 * "_device".
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the SORS project root).  The reference's Python module py_sors
 * (cpp/py_sors.cpp) binds the C++ classes Energy<3,E> and Solver<3,E>; a
 * maintainer binds these functions instead.
 */
#ifndef SORS_B200_H
#define SORS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference throws std::runtime_error; the shim above this
 * ABI rethrows with the same messages (see sors_last_error). */
#define SORS_OK 0
#define SORS_ERR_ARG 1            /* bad argument / unknown option            */
#define SORS_ERR_INVERTED 2       /* "Inverted Elements" neoHookean.cpp:98-101 */
#define SORS_ERR_NOT_CONVERGED 3  /* "Newton's method did not converge" solver.cpp:100-103 */
#define SORS_ERR_PCG_BREAKDOWN 4  /* non-positive curvature in the linear solve */
#define SORS_ERR_CUDA 5           /* CUDA runtime error                        */
#define SORS_ERR_OOM 6            /* device allocation failed                  */
#define SORS_ERR_LINESEARCH 7     /* Armijo backtracking exhausted             */
#define SORS_ERR_UNSUPPORTED 8    /* option not built for this mesh type       */

/* SimulationSettings (cpp/headers/simulationSettings.h:18-71) plus the
 * device-solver options that have no reference counterpart. */
typedef struct SorsSettings {
    int32_t time_stepping;   /* 0 "backward_euler", 1 "crank_nicolson"           */
    int32_t solver_method;   /* 0 "minimize_newton", 1 "minimize_newton_linesearch",
                                2 "minimize_frozenhessian", 3 "minimize_SQP"      */
    double dt;               /* settings.dt, used when a call passes dt == 0      */
    int32_t substeps;        /* settings.substeps                                */
    int32_t cfl;             /* settings.CFLtimeSteppingFlag                     */
    double grav[3];          /* gravAcceleration                                 */
    double damping_alpha;    /* dampingAlpha                                     */
    int32_t precision;       /* 0: FP64 everywhere; 1: FP32 Hessian + PCG, FP64
                                residual, energy, dots and log(J)                */
    int32_t project_spd;     /* 1: clamp negative eigenvalues of dP/dF per
                                quadrature point before assembly; 0: exact
                                Hessian; 2 (default): exact, and projected for
                                an iteration whose PCG met negative curvature    */
    int32_t material;        /* 0 "neohookean"; 1 the reference's quartic test
                                element (cpp/src/_test.cpp:8-66)                 */
    double newton_dx_tol;    /* ||dx|| stop, reference DX_TOL = 1e-9              */
    double newton_res_tol;   /* ||gradient|| stop (absolute); <= 0 disables       */
    int32_t newton_max_iter; /* reference MAX_ITER = 100                          */
    double pcg_rel_tol;      /* smallest PCG forcing term                         */
    int32_t pcg_max_iter;
    int32_t device;          /* CUDA device ordinal                              */
    int32_t newton_predictor;/* 1: start each Newton solve from q + dt v_prev
                                (falls back to q if that inverts an element);
                                changes only the iterates, not the solution      */
    int32_t max_blocks;      /* largest grid of any kernel of this handle; 0 = the
                                whole GPU (148 x 8 blocks).  Smaller grids let the
                                kernels of several handles run side by side     */
    int32_t newton_safeguard;/* 1 (with project_spd 2, "minimize_newton"): halve a
                                Newton step that does not reduce ||g|| (no
                                reference counterpart; off by default)            */
    int32_t two_level;       /* 1: precondition the Newton PCG with block Jacobi
                                plus an exact coarse correction on per-aggregate
                                rigid-body modes (no reference counterpart);
                                0: block Jacobi; 2 (default): 1 for meshes of
                                20,000 nodes or more                              */
    int32_t linear_solver;   /* Newton systems of "minimize_newton": 0 (default)
                                PCG; 1 MINRES, which takes the Newton step of an
                                indefinite exact Hessian as the reference's LDL^T
                                does (cpp/src/solver.cpp:65-84), preconditioned
                                by block Jacobi on |D_ii| and the coarse
                                correction of the projected Hessian.  Contact
                                QPs, adjoints and unions use PCG.              */
    int32_t pressure_jac_exact; /* 1: the Newton matrix takes the exact follower
                                load coefficient for quads (p/8, the derivative of
                                the quad force -p A / 4) instead of the reference's
                                p/6 (pressureForce.cpp:105,174); the solution is
                                the same, only the Newton iterates change.
                                0 (default): the reference's                   */
} SorsSettings;

typedef struct SorsStepStats {
    int32_t newton_iters;    /* summed over substeps                             */
    int32_t pcg_iters;       /* summed over Newton iterations                    */
    int32_t substeps;
    double residual_norm;    /* ||gradient|| at the last evaluation              */
    double dx_norm;          /* ||dx|| of the last Newton update                 */
} SorsStepStats;

typedef struct SorsHandle SorsHandle;

/* Fills the defaults listed above. */
void sors_default_settings(SorsSettings* s);

/* Replaces Energy<3,E>::Energy (cpp/src/energy.cpp:4-204) for Neo-Hookean
 * elements and the py_sors factory Energy(...) (cpp/py_sors.cpp:30-62).
 * X: N x 3 undeformed vertices; conn: E x nodes_per_elem (4 tets, 8 hexes);
 * density/youngs/poisson: per element.  Copies everything to the device,
 * builds the fixed block-CSR Hessian pattern and the row-owner slot maps. */
int sors_create(const double* X, int32_t n_nodes, const int32_t* conn, int32_t n_elems,
                int32_t nodes_per_elem, const double* density, const double* youngs,
                const double* poisson, const SorsSettings* settings, SorsHandle** out);

/* Frees the handle and all its device memory. */
void sors_destroy(SorsHandle* h);

/* Message of the last failed call on this thread (reference exception text). */
int sors_last_error(char* buf, size_t n);

/* NeumannBC constraint parameters neumannBCmask / neumannBCvalue
 * (cpp/src/energy.cpp:61-68, cpp/src/constraints/neumannBC.cpp). 3N each. */
int sors_set_neumann(SorsHandle* h, const int32_t* mask, const double* value);

/* PressureForce(surfaceVertexIdx, surfaceGroups)
 * (cpp/src/forces/pressureForce.cpp:4-10): faces F x {3|4}, group per face. */
int sors_set_pressure_faces(SorsHandle* h, const int32_t* faces, int32_t n_faces,
                            int32_t verts_per_face, const int32_t* groups, int32_t n_groups);

/* VertexForce (cpp/src/forces/vertexForce.cpp): enables the "vertexForce" actuation. */
int sors_enable_vertex_force(SorsHandle* h, int32_t enable);

/* SoftCon fibre terms, replacing the per-element "softconMuscle" energy and its
 * Params muscleGroup / softconStiffness / softconDirection
 * (cpp/src/geometries/tetrahedron.cpp:82-88, hexahedron.cpp:51-57,
 * cpp/src/energies/softconMuscle.cpp).  group: E entries, -1 = no fibre term;
 * stiffness: E; direction: E x 3 row-major.  Activations start at 0 and are set
 * with the "softconMuscle" actuation.  Energy k/2 (|F m| - (1 - e))^2, whose
 * gradient is the reference's; its exact Hessian (projected when project_spd). */
int sors_set_muscles(SorsHandle* h, const int32_t* group, const double* stiffness, const double* direction,
                     int32_t n_groups);

/* Replaces every element's Young's modulus and Poisson ratio (E entries each),
 * as constructing Energy<3,E> again with new Params would (mass unchanged). */
int sors_set_material(SorsHandle* h, const double* youngs, const double* poisson);

/* PlaneContact (cpp/src/constraints/planeContact.cpp, energy.cpp:69-84): planes
 * given by a point and a normal (n_planes x 3 each, row-major) and the surface
 * vertices that may touch them ("surfaceVerticesIdx").  Used by solver_method 3
 * ("minimize_SQP"): a surface vertex whose signed distance to its closest plane
 * is below 0.01 at the start of a step gets the constraint n . (x - p) >= 0. */
int sors_set_plane_contact(SorsHandle* h, const double* points, const double* normals, int32_t n_planes,
                           const int32_t* surface_vertices, int32_t n_surface);

/* DiskContact (cpp/src/constraints/diskContact.cpp, energy.cpp:85-108): disks
 * (centers, normals n_disks x 3, radii n_disks) and candidate surface vertices.
 * The captured footprint stays frozen until all of it is 3 x 0.01 above its
 * disk (diskContact.cpp:94-205).  Normals are normalised. */
int sors_set_disk_contact(SorsHandle* h, const double* centers, const double* normals, const double* radii,
                          int32_t n_disks, const int32_t* surface_vertices, int32_t n_surface);

/* Disks that act as independent DiskContact constraints (no reference
 * counterpart as one call): disk k may touch only surface_vertices
 * [surface_ptr[k], surface_ptr[k+1]) and keeps its own frozen footprint, as if
 * each disk were a separate diskContact entry.  Used to step several meshes in
 * one handle (serving), each with its own indenter. */
int sors_set_disk_contact_groups(SorsHandle* h, const double* centers, const double* normals, const double* radii,
                                 int32_t n_disks, const int32_t* surface_vertices, const int32_t* surface_ptr);

/* DiskContact::set_disk (cpp/py_sors.cpp:231-245): moves disk disk_idx. */
int sors_set_disk(SorsHandle* h, int32_t disk_idx, const double* center, const double* normal, double radius);

/* maxDistance constraint (cpp/src/energy.cpp:109-120, constraints/
 * maxDistance.cpp:4-80): |q_vertex1[k] - q_vertex2[k]| <= max_distance[k] for
 * every pair, always active, an inequality row of the SQP subproblem
 * (solver_method 3).  n_pairs == 0 removes the constraint. */
int sors_set_max_distance(SorsHandle* h, const int32_t* vertex1, const int32_t* vertex2, const double* max_distance,
                          int32_t n_pairs);

/* Max-distance pairs held (at their bound) when the last SQP step converged:
 * indices into the sors_set_max_distance list and their multipliers (>= 0;
 * grad E = sum mu_k grad g_k at the solution).  Writes min(count, cap) entries
 * of either array (may be NULL); returns the count. */
int32_t sors_held_pairs(SorsHandle* h, int32_t* pairs, double* multipliers, int32_t cap);

/* Held max-distance pairs (indices and multipliers, as sors_held_pairs gave
 * them right after the step) for the following sors_adjoint_step calls, until
 * set again; n == 0 clears.  No reference counterpart. */
int sors_adjoint_set_pairs(SorsHandle* h, const int32_t* pairs, const double* multipliers, int32_t n);

/* Number of contact constraints active in the last SQP step. */
int32_t sors_active_contacts(SorsHandle* h);

/* Contacts held (at their bound) when the last SQP step converged: nodes and
 * normals (3 per node).  Writes min(count, cap) entries; returns the count. */
int32_t sors_held_contacts(SorsHandle* h, int32_t* nodes, double* normals, int32_t cap);

/* The disk contacts' state between steps (per DiskContact: frozen flag and
 * captured footprint), for restarting a rollout from a saved step.  get returns
 * the length and fills state when cap is large enough; set takes that many. */
int32_t sors_get_contact_state(SorsHandle* h, int32_t* state, int32_t cap);
int sors_set_contact_state(SorsHandle* h, const int32_t* state, int32_t n);

/* Params actuation entries (cpp/headers/params.h): "pressure" (n_groups values),
 * "vertexForce" (3N values, row-major N x 3) or "softconMuscle" (one activation
 * per muscle group). */
int sors_set_actuation(SorsHandle* h, const char* name, const double* values, int64_t n);

/* Energy::set_initial_deformation / set_initial_velocity (cpp/headers/energy.h:203-204). */
int sors_set_initial_deformation(SorsHandle* h, const double* q);
int sors_set_initial_velocity(SorsHandle* h, const double* v);

/* TimeIntegrator::get_qPrev / get_vPrev (cpp/headers/integrator.h:100-101). */
int sors_get_state(SorsHandle* h, double* q_prev, double* v_prev);

/* The Crank-Nicolson state's previous-step force gPrev_ (3N; cpp/headers/
 * integrator.h:82, zero at construction), read and restored with q_prev and
 * v_prev when a rollout is checkpointed. */
int sors_get_prev_force(SorsHandle* h, double* g_prev);
int sors_set_prev_force(SorsHandle* h, const double* g_prev);

/* Energy::compute_energy (cpp/src/energy.cpp:208-248). */
int sors_energy(SorsHandle* h, const double* q, double dt, double* out);

/* Energy::compute_gradient (cpp/src/energy.cpp:252-308). */
int sors_gradient(SorsHandle* h, const double* q, double dt, double* g);

/* Energy::compute_hessian (cpp/src/energy.cpp:312-390) as 3x3 block CSR.
 * Call with NULL outputs to get nnzb; row_ptr has N+1 entries, val 9*nnzb
 * (row-major blocks).  The pattern is fixed at sors_create. */
int sors_hessian_bsr(SorsHandle* h, const double* q, double dt, int32_t* row_ptr, int32_t* col,
                     double* val, int64_t* nnzb);

/* Per-element Tetrahedron/Hexahedron::compute_{energy,gradient,hessian}
 * (cpp/src/geometries/tetrahedron.cpp:99-134, hexahedron.cpp:68-103),
 * scaled by the undeformed volume.  psi: E; grad: E x 3nv; hess: E x (3nv)^2.
 * Any output may be NULL. */
int sors_elem_eval(SorsHandle* h, const double* q, int32_t project, double* psi, double* grad,
                   double* hess);

/* Solver<3,E>::step (cpp/src/solver.cpp:5-44): substeps of the configured
 * minimiser followed by Energy::update_state.  dt == 0 / substeps == 0 take
 * the settings.  q_in and q_out may alias. */
int sors_step(SorsHandle* h, const double* q_in, double* q_out, double dt, int32_t substeps,
              SorsStepStats* stats);

/* Adjoint of one backward-Euler step (no reference counterpart: SORS has no
 * differentiation).  A step took the state (q_n, v_n) to q_next with this
 * handle's materials and the activations set at the time; call this with the
 * same activations set.  held_nodes / held_normals (n_held, may be 0) are the
 * contacts the step held (sors_held_contacts right after it); held
 * max-distance pairs come from sors_adjoint_set_pairs.  Given dL/dq_next (3N)
 * it solves the transpose system of the step's residual at q_next (exact,
 * unprojected Hessian, plus the held pairs' constraint curvature mu_k / L_k
 * (I - u u^T)) on the subspace the Neumann DOFs, the held contacts and the held
 * pairs leave free, and writes (any output may be NULL):
 *   dL/dq_n (3N), dL/dv_n (3N)  through the residual's old-state terms and the
 *                                Neumann targets q_n + dt val,
 *   dL/dyoungs (E)               per element,
 *   dL/dact (one per muscle group, "softconMuscle" activations),
 *   dL/dneumann (3N)             the Neumann velocities, nonzero on fixed DOFs.
 * Any dependence of the loss on v_next = (q_next - q_n)/dt is the caller's to
 * add to dL/dq_next (and subtract from dL/dq_n).  With pressure loads the
 * transpose system uses the exact derivative of the follower load (not the
 * Newton matrix's symmetrised one; see sors_adjoint_pressure_grad); pressure
 * loads with held max-distance pairs return SORS_ERR_UNSUPPORTED, and
 * Crank-Nicolson steps are differentiated by sors_adjoint_step_cn.  dt = 0
 * takes settings.dt. */
int sors_adjoint_step(SorsHandle* h, const double* q_next, double dt, const double* dL_dq_next,
                      const int32_t* held_nodes, const double* held_normals, int32_t n_held, double* dL_dq_prev,
                      double* dL_dv_prev, double* dL_dyoungs, double* dL_dact, double* dL_dneumann,
                      SorsStepStats* stats);

/* dL/d(pressure of each group) of the last sors_adjoint_step on this handle
 * (no reference counterpart), for PressureForce's per-group "pressure"
 * actuation (cpp/src/forces/pressureForce.cpp:12-56): lam . f_g with lam the
 * step's adjoint and f_g the follower load of group g at unit pressure on
 * q_next.  n_groups must equal the groups given to sors_set_pressure_faces. */
int sors_adjoint_pressure_grad(SorsHandle* h, double* dL_dpressure, int32_t n_groups);

/* Adjoint of one Crank-Nicolson step (no reference counterpart; the residual
 * of cpp/src/integrator.cpp:72-78).  As sors_adjoint_step, plus the state's
 * previous-step force: the step's residual holds 0.5 gPrev, and the next
 * step's gPrev is this step's internal force at q_next.  dL_dgprev_next (3N,
 * NULL = zero) is the cotangent of the next step's gPrev (the
 * dL_dgprev_prev that the next step's call wrote); dL_dgprev_prev receives
 * this step's.  The velocity of the state is v_next = 2 (q_next - q_n) / dt
 * - v_n; the caller chains it as it chains v for backward Euler.  Pressure
 * loads and held max-distance pairs return SORS_ERR_UNSUPPORTED. */
int sors_adjoint_step_cn(SorsHandle* h, const double* q_next, double dt, const double* dL_dq_next,
                         const double* dL_dgprev_next, const int32_t* held_nodes, const double* held_normals,
                         int32_t n_held, double* dL_dq_prev, double* dL_dv_prev, double* dL_dgprev_prev,
                         double* dL_dyoungs, double* dL_dact, double* dL_dneumann, SorsStepStats* stats);

/* Same step on a device-resident FP64 solution vector (in place). */
int sors_step_device(SorsHandle* h, double* q_device, double dt, int32_t substeps,
                     SorsStepStats* stats);

/* Energy::update_state (cpp/src/energy.cpp:539-557). */
int sors_update_state(SorsHandle* h, const double* q, double dt);

/* Device memory held by the handle, in bytes (admission by HBM footprint). */
int64_t sors_device_bytes(const SorsHandle* h);

/* Sizes of the fixed pattern: N, E, nnz blocks. */
int sors_sizes(const SorsHandle* h, int64_t* n_nodes, int64_t* n_elems, int64_t* nnzb);

/* Per-launch device time (CUDA events on the handle's stream, averaged over
 * `iters` back-to-back launches on the current assembled system) and the
 * algorithmic bytes each launch must move: every input and output counted
 * once.  Diagnostic only; no reference counterpart. */
typedef struct SorsKernelProfile {
    double assemble_ms, spmv_ms, pcg_update_ms, energy_ms;
    double assemble_bytes, spmv_bytes, pcg_update_bytes, energy_bytes;
    /* two-level PCG iteration kernels (0 without the two-level preconditioner):
     * the x / r update fused with the restriction, and the coarse solve fused
     * with the prolongation and z = Minv r */
    double tl_restrict_ms, tl_coarse_z_ms, tl_restrict_bytes, tl_coarse_z_bytes;
    /* p = z + beta p_old, formed before the SpMV (padded, 4 values per node) */
    double form_p_ms, form_p_bytes;
    /* the assembly launch without the Hessian (gradient rows only) */
    double assemble_grad_ms;
} SorsKernelProfile;
int sors_profile_kernels(SorsHandle* h, int32_t iters, SorsKernelProfile* out);

/* Number of kernels this library has launched in this process (graph
 * launches count every kernel node).  Diagnostic only. */
int64_t sors_kernel_launch_count(void);

/* Number of system evaluations (gradient rows, and the Hessian when
 * with_hessian != 0) this handle has made since it was created; with_hessian
 * == 0 counts the gradient-only ones.  Diagnostic only. */
int64_t sors_evaluation_count(SorsHandle* h, int32_t with_hessian);

/* Assembly kernel of the handle's tet Hessian and gradient evaluations:
 * 0 (default) the element-owner kernel over node chunks wherever it applies
 * (exact Neo-Hookean or stable Neo-Hookean tets without fibre terms; the
 * projected Hessian, fibres, the quartic test element and hexes always use
 * the row-owner kernel), 1 the row-owner kernel everywhere, 2 the chunked
 * kernel in two passes (every element evaluated once into records in device
 * memory, which the chunks then load; allocates those records on first use).
 * All give the same Hessian values to rounding; no counterpart in the
 * reference.  Diagnostic only. */
int sors_set_assembly_variant(SorsHandle* h, int32_t variant);

/* Node chunks of the element-owner assembly (0: the mesh uses the row-owner
 * kernel only).  Diagnostic only. */
int64_t sors_assembly_chunks(SorsHandle* h);

/* Declares the handle's mesh to be n_members independent meshes: member k
 * owns nodes [node_offsets[k], node_offsets[k+1]) (node_offsets[0] = 0,
 * node_offsets[n_members] = the node count) and no element joins two members,
 * which is checked.  Every linear solve then runs one preconditioned CG per
 * member, with its own step lengths, tolerance and convergence, in the same
 * kernel launches (the block-Jacobi preconditioner; the two-level one is not
 * used).  A rollout server packs small meshes into one handle this way.
 * n_members <= 1 returns to one CG over the whole system.  No counterpart in
 * the reference (it steps one mesh per Energy). */
int sors_set_members(SorsHandle* h, const int32_t* node_offsets, int32_t n_members);

/* Linear solves of the last sors_step / sors_step_device whose PCG met a
 * direction p of non-positive curvature, on the subspace the step's
 * constraints leave free (the exact Hessian is indefinite there), and the most
 * negative Rayleigh quotient p'Hp / p'p among them (+inf when none).  The
 * reference's OSQP rejects a QP as non-convex when H + sigma I + A' rho A has a
 * negative pivot (sigma = 1e-6, rho = 0.1 on contact rows), which a quotient
 * below -(sigma + rho) certifies.  Diagnostic; no counterpart in the reference. */
int sors_last_step_curvature(SorsHandle* h, double* min_rayleigh, int32_t* indefinite_solves);

/* Sum of the Neo-Hookean element energies (volume x Psi, the element part of
 * sors_energy) of a tet (nodes_per_elem = 4) or hex (8) mesh, computed from
 * caller-owned DEVICE arrays, without any device allocation.  No counterpart
 * in the reference: it exists for callers that cannot let a library call
 * cudaMalloc (memory owned by their own pool or arena, or real-time loops that
 * must not allocate after start-up).  X_device, q_device: 3N doubles;
 * conn_device: n_elems x nodes_per_elem; youngs_device, poisson_device:
 * n_elems; out_device: one double.  Launched on `stream` (NULL = default
 * stream) and asynchronous to the host.  The kernel's scratch is a fixed
 * 64 KiB array inside the library, shared by all calls: n_elems above
 * 8,388,608 is rejected (SORS_ERR_ARG), and calls that overlap on the GPU
 * race and must be serialised by the caller.  A call on a stream that is not
 * capturing looks up the array's device address and remembers it; a call on a
 * capturing stream uses the remembered one.  So make the first call on each
 * device before any stream capture, and after a device reset (which may move
 * the array) make one uncaptured call before the next capture. */
int sors_elem_energy_noalloc(const double* X_device, const double* q_device, const int32_t* conn_device,
                             int32_t n_elems, int32_t nodes_per_elem, const double* youngs_device,
                             const double* poisson_device, double* out_device, void* stream);

/* CUDA stream of the handle (cudaStream_t as void*), for callers that order
 * their own work after a step. */
void* sors_stream(SorsHandle* h);

#ifdef __cplusplus
}
#endif

#endif /* SORS_B200_H */
