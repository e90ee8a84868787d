/*
 * b200fem.h -- C ABI of the B200 (sm_100a) FEM force/stiffness assembly and
 * BackwardEuler step engine (libb200fem.so).
 *
 * The entry points mirror the operations of ArtiSynth's hot path and of the
 * JNI bridge the reference already ships for its cuDSS solver:
 *
 *   handle lifecycle / errors  CuDssJNI.cc:15-747 (doInit, doDispose,
 *                              doGetLastError), cudssBridge.h:39-52,187-189
 *   pattern + CRS slot map     SparseNumberedBlockMatrix.createCrsBlockSlotMap
 *                              (SparseNumberedBlockMatrix.java:389-498),
 *                              SparseBlockMatrix.getCRSIndices (:1511-1532)
 *   force/stiffness update     FemModel3d.updateStressAndStiffness
 *                              (FemModel3d.java:2894-3051)
 *   BackwardEuler step         MechSystemSolver.backwardEuler
 *                              (MechSystemSolver.java:2171-2476)
 *   SpMV / iterative solve     CuDssBridge::multiply / iterativeSolveBiCGStab
 *                              (cudssBridge.cc:1419-1452,1705-2006)
 *
 * Conventions (same as the reference bridge): every function returns an int
 * status, 0 on success and a negative B200FEM_ERR_* code on failure; the
 * message of the last failure is available from b200fem_last_error().  The
 * handle owns all device memory; caller arrays are borrowed for the duration
 * of the call only.  Calls on one handle are synchronous and must not be
 * made concurrently from several threads.  There is no CPU fallback: a
 * handle cannot be created without a CUDA device.
 *
 * Array conventions: node positions/velocities/forces are (3*n_nodes)
 * doubles in node order; connectivity is (nen*n_elems) int32 in the
 * reference's local node order (TetElement, HexElement); stiffness blocks
 * are 3x3 row-major, stored in block-CSR order over active nodes (block row
 * = solve index), 9 doubles per block.
 */
#ifndef B200FEM_H
#define B200FEM_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (cf. CUDSS_BRIDGE_ERR_*, cudssBridge.h:39-52) */
#define B200FEM_OK 0
#define B200FEM_ERR_INVALID_ARG (-1)
#define B200FEM_ERR_CUDA (-2)
#define B200FEM_ERR_STATE (-3)
#define B200FEM_ERR_UNSUPPORTED (-4)
#define B200FEM_ERR_INVERTED (-5)
#define B200FEM_ERR_BUDGET (-6)
#define B200FEM_ERR_TIMEOUT (-7)
#define B200FEM_ERR_NO_CONVERGE (-13)

/* element types */
#define B200FEM_ELEM_TET 0 /* TetElement, 4 nodes, 1 integration point */
#define B200FEM_ELEM_HEX 1 /* HexElement, 8 nodes, 8 Gauss points */
#define B200FEM_ELEM_WEDGE 2   /* WedgeElement, 6 nodes, 6 integration points */
#define B200FEM_ELEM_PYRAMID 3 /* PyramidElement, 5 nodes, 5 integration points */
#define B200FEM_ELEM_QUADTET 4 /* QuadtetElement, 10 nodes (corners 0-3, then the midpoints
                                  of edges 01, 12, 02, 03, 13, 23), 4 integration points;
                                  soft incompressibility resolves to ELEMENT */
#define B200FEM_ELEM_QUADHEX 5 /* QuadhexElement, 20 nodes (corners 0-7, then the midpoints of
                                  edges 01 12 23 30, 45 56 67 74, 04 15 26 37), 14 points;
                                  soft incompressibility resolves to ELEMENT with four pressure
                                  values per element */
#define B200FEM_ELEM_QUADWEDGE 6   /* QuadwedgeElement, 15 nodes (edges 01 12 20, 34 45 53, 03 14
                                      25), 9 points; ELEMENT with two pressure values */
#define B200FEM_ELEM_QUADPYRAMID 7 /* QuadpyramidElement, 13 nodes (edges 01 12 23 30, 04 14 24
                                      34), 5 points; soft incompressibility resolves to ELEMENT */

/* materials (parameter layout of b200fem_set_material) */
#define B200FEM_MAT_LINEAR 0       /* {E, nu, corotated(0/1)}: LinearMaterial */
#define B200FEM_MAT_NEOHOOKEAN 1   /* {E, nu}: NeoHookeanMaterial */
#define B200FEM_MAT_STVK 3         /* {E, nu}: StVenantKirchoffMaterial (the reference's FEBio
                                       form, StVenantKirchoffMaterial.java:136-164) */
#define B200FEM_MAT_MOONEYRIVLIN 2 /* {c10, c01, c11, c20, c02, kappa, jlimit,
                                      bulk_potential(0 quadratic, 1 log)} */
#define B200FEM_MAT_MODEL (-1)     /* b200fem_set_element_materials: the model's material */

/* soft incompressibility (FemModel3d.IncompMethod) */
#define B200FEM_INCOMP_OFF 0
#define B200FEM_INCOMP_NODAL 1
#define B200FEM_INCOMP_AUTO 2
#define B200FEM_INCOMP_ELEMENT 3 /* one pressure value per element: p = effective pressure of
                                    V/V0, dilational stiffness Rinv c_i c_j^T (FemModel3d.java:
                                    2517-2591, 3650-3663); AUTO picks it when #elements <=
                                    #active nodes */

/* precision of the engine */
#define B200FEM_PREC_FP64 0  /* plain FP64 drop-in */
#define B200FEM_PREC_MIXED 1 /* FP32 element/SpMV, FP64 residual/dots/update */

/* scalar CRS partitions (Matrix.Partition) */
#define B200FEM_PART_FULL 0
#define B200FEM_PART_UPPER 1

typedef struct b200fem_engine* b200fem_handle;

typedef struct {
  int device;    /* CUDA device ordinal */
  int precision; /* B200FEM_PREC_* */
  int reserved[6];
} b200fem_config;

/* BackwardEuler parameters: FemModel.massDamping (default 2),
   FemModel.stiffnessDamping (default 0), MechModel gravity, PCG controls. */
typedef struct {
  double h;          /* step size */
  double alpha_m;    /* mass damping */
  double beta_k;     /* stiffness damping */
  double gravity[3]; /* gravity acceleration */
  double tol;        /* PCG relative residual ||b - S v|| / ||b|| */
  int max_iter;      /* PCG iteration cap (ERR_NO_CONVERGE beyond it) */
  int abort_on_inverted; /* FemModel3d.abortOnInvertedElems */
  int pcg_variant;   /* 0 auto: pipelined CG (one grid barrier per iteration),
                        switching to classic PCG after a residual replacement;
                        1 classic PCG (two barriers, better attainable accuracy);
                        2 pipelined only */
  int integrator;    /* B200FEM_INTEGRATOR_*: BackwardEuler ignores constraints;
                        ConstrainedBackwardEuler enforces the plane constraints */
} b200fem_step_params;

/* MechSystemSolver.Integrator */
#define B200FEM_INTEGRATOR_BACKWARD_EULER 0
#define B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER 1

typedef struct {
  int iterations;      /* PCG iterations of the last solve */
  int num_inverted;    /* elements with detJ <= 0 at the last update */
  double rel_residual; /* true relative residual of the last solve */
  double min_detJ;     /* smallest Jacobian determinant seen */
  int refinements;     /* iterative-refinement sweeps (mixed precision) */
  int reserved[3];
} b200fem_stats;

/* ---- library / handle ---------------------------------------------------- */
int b200fem_version(void);
/* CuDssJNI doInit: returns NULL on failure (message via b200fem_last_error(NULL)) */
b200fem_handle b200fem_create(const b200fem_config* cfg);
/* CuDssJNI doDispose: idempotent; NULL is accepted */
int b200fem_destroy(b200fem_handle h);
/* CuDssJNI doGetLastError; h may be NULL for create failures */
const char* b200fem_last_error(b200fem_handle h);

/* ---- mesh factory (FemFactory.createTetGrid/createHexGrid, host only) ---- */
int b200fem_grid_dims(int elem_type, int nx, int ny, int nz, int* n_nodes, int* n_elems);
int b200fem_create_grid(int elem_type, double wx, double wy, double wz, int nx, int ny, int nz,
                        double* xyz, int* conn);
/* FemFactory.createQuadraticModel for a tet mesh: the n_nodes linear nodes
   keep their indices, edge midpoints follow in element order (shared edges
   once); conn_out holds 10 nodes per tet (B200FEM_ELEM_QUADTET order).
   xyz_out / conn_out may be NULL to query *n_nodes_out first. */
int b200fem_quadratic_tet_mesh(int n_nodes, const double* xyz, int n_tets, const int* conn, int* n_nodes_out,
                               double* xyz_out, int* conn_out);
/* seeded interior-node jitter: (2u-1)*frac*spacing per axis, u from
   splitmix64(seed) drawn in node order; boundary nodes stay put */
int b200fem_jitter_grid(int nx, int ny, int nz, double wx, double wy, double wz, double frac,
                        unsigned long long seed, double* xyz);

/* ---- model definition (FemModel3d nodes/elements/material) -------------- */
/* fixed[n] != 0 marks a non-dynamic node (no solve index) */
int b200fem_set_mesh(b200fem_handle h, int elem_type, int n_nodes, const double* rest_xyz,
                     int n_elems, const int* conn, const int* fixed);
/* A mesh whose elements are of several types (FemModel3d holds any mix of
   FemElement3d subclasses; computeStressAndStiffness, FemModel3d.java:3333,
   runs over each element by its own type): elem_types[e] is element e's
   B200FEM_ELEM_* type and conn holds every element's nodes concatenated in
   element order (elem_nen(type) entries each).  Pattern, masses, forces,
   stiffness and steps are those of the same elements in this order; soft
   incompressibility AUTO resolves over all elements (NODAL only when every
   element is a tet, hex, wedge or pyramid). */
int b200fem_set_mesh_mixed(b200fem_handle h, int n_nodes, const double* rest_xyz, int n_elems,
                           const int* elem_types, const int* conn, const int* fixed);
int b200fem_set_material(b200fem_handle h, int mat_kind, const double* params, double density,
                         int incomp_method);
/* Per-element materials (FemElement.setMaterial; FemModel3d.getElementMaterial,
   FemModel3d.java:608-614, returns the element's own material when it has
   one, else the model's): mat_kinds[e] is element e's B200FEM_MAT_* kind, or
   B200FEM_MAT_MODEL for the model's material, and params holds 8 values per
   element in b200fem_set_material's layout (read only where mat_kinds[e] is
   a kind).  Elements of a compressible kind run without soft
   incompressibility (FemModel3d.java:3346-3348); ELEMENT uses each element's
   own kappa; NODAL (which needs the model's material to be MooneyRivlin)
   uses the model's kappa and is refused with B200FEM_ERR_UNSUPPORTED at the
   build when any element's material is compressible (the reference divides
   by a zero nodal rest volume at a node only such elements touch).  model is
   the pack index (0 for a single model); n_elems must equal its element
   count; mat_kinds == NULL gives every element the model's material again.
   b200fem_set_mesh / _set_mesh_mixed clear them. */
int b200fem_set_element_materials(b200fem_handle h, int model, int n_elems, const int* mat_kinds,
                                  const double* params);
/* builds rest data, the block pattern, the element-to-block scatter map and
   uploads everything (the reference's structure build + analyze) */
int b200fem_build(b200fem_handle h);

/* ---- pattern queries (bit-exact with the reference) ---------------------- */
int b200fem_get_sizes(b200fem_handle h, int* n_active, int* nnzb, int* crs_nnz_full,
                      int* crs_nnz_upper);
/* solve index per node (-1 for fixed nodes), MechSystemBase numbering */
int b200fem_get_solve_index(b200fem_handle h, int* sidx);
int b200fem_get_pattern(b200fem_handle h, int* blk_rowptr, int* blk_col);
/* 0-based scalar CRS row offsets (3*n_active+1) and column indices */
int b200fem_get_crs_indices(b200fem_handle h, int partition, int* row_offs, int* col_idx);
/* CrsBlockSlotMap: 9 slots per block in BSR order, -1 when excluded */
int b200fem_get_slot_map(b200fem_handle h, int partition, int* slots);
/* element-to-block scatter map: for every element and every local node pair
   (i, j) (nen*nen per element, concatenated in element order) the BSR block
   index receiving K_ij, or -1 */
int b200fem_get_scatter_map(b200fem_handle h, int* map);
int b200fem_get_masses(b200fem_handle h, double* mass);
int b200fem_get_incomp_method(b200fem_handle h, int* method);

/* ---- state -------------------------------------------------------------- */
int b200fem_set_state(b200fem_handle h, const double* x, const double* v);
int b200fem_get_state(b200fem_handle h, double* x, double* v);
int b200fem_set_external_forces(b200fem_handle h, const double* fext);

/* ---- hot path ------------------------------------------------------------ */
/* FemModel3d.updateStressAndStiffness at positions x (host, 3N): returns the
   internal elastic force per node (3N; may be NULL), the stiffness blocks in
   BSR order (9*nnzb; may be NULL) and/or the full-partition scalar CRS
   values in the reference slot order (crs_nnz_full; may be NULL). */
int b200fem_update_stress_stiffness(b200fem_handle h, const double* x, double* f_int,
                                    double* k_blocks, double* crs_vals);
/* ParticlePlaneConstraint (ParticlePlaneConstraint.java:144-160) on single
   nodes: node nodes[i] (not fixed, at most one constraint each) is held on the
   plane normals[i] . x = offsets[i] (normals need not be unit length).  The
   ConstrainedBackwardEuler integrator solves the KKT velocity system
   [S G^T; G 0] (MechSystemSolver.KKTFactorAndSolve) by PCG on the constrained
   velocities (every row's search directions projected onto its plane) and
   then moves each constrained node onto its plane (the GlobalMass position
   correction of a single-particle constraint).  n = 0 removes them. */
int b200fem_set_plane_constraints(b200fem_handle h, int n, const int* nodes, const double* normals,
                                  const double* offsets);
/* LinearPointConstraint (LinearPointConstraint.java), constraints that
   couple several nodes: constraint c holds sum_q weights[q] x[nodes[q]] at
   targets[3c .. 3c+2] over q in [ptr[c], ptr[c+1]) (n + 1 offsets from 0; at
   most 32 constraints; fixed points count in the position but have no
   velocity rows).  The ConstrainedBackwardEuler integrator solves the KKT
   velocity system [S G^T; G 0][v; lam] = [b; 0] (zero compliance) by its
   Schur complement on the device PCG -- 3n + 1 PCG solves per step -- and
   then applies the GlobalMass position correction (dx = M^-1 G^T mu,
   (G M^-1 G^T) mu = -(G x - target)); BackwardEuler ignores them.  Not
   combined with plane constraints in one step.  n = 0 removes them.  Node
   indices are the handle's (concatenated for a pack). */
int b200fem_set_point_constraints(b200fem_handle h, int n, const int* ptr, const int* nodes, const double* weights,
                                  const double* targets);
/* PointFrameAttachment with an active master frame (FemModel3d.
   getGpuNodeReduction, FemModel3d.java:4356-4387): node nodes[i] of the model
   (set by b200fem_set_mesh first; not fixed; at most one attachment each)
   follows frame frames[i] (0 .. n_frames - 1), its velocity v = H_i^T
   [v_F; w_F] with H_i the attachment's 6x3 master block (18 doubles per
   attachment, row-major; H = -PointFrameAttachment.getGT(0)).  Attached
   nodes leave the solve: the stiffness of b200fem_update_stress_stiffness
   is the reduced P^T K P -- each element block K_ij goes to T_i K_ij T_j^T,
   T = I for a free node and H for an attached one (the reference's
   scatterReduced3Block, cudssBridgeKernels.cu:325-365) -- over the free
   active nodes in node order followed by two 3x3 block rows per frame
   (translation, rotation: the frame's 6 scalar rows), and the pattern, CRS
   and solve-index queries describe that reduced system (attached nodes have
   solve index -1; frame f has block rows n_free + 2f and n_free + 2f + 1).
   Every frame needs at least one attached node; single-model handles only.
   The frames' own rigid-body dynamics are not part of the engine, so
   BackwardEuler steps of a model with attachments return
   B200FEM_ERR_UNSUPPORTED.  Takes effect at the next b200fem_build;
   n_frames = n_att = 0 removes them; b200fem_set_mesh clears them. */
int b200fem_set_frame_attachments(b200fem_handle h, int n_frames, int n_att, const int* nodes, const int* frames,
                                  const double* H);
/* nsteps BackwardEuler steps on the device-resident state */
int b200fem_backward_euler_step(b200fem_handle h, const b200fem_step_params* p, int nsteps,
                                b200fem_stats* stats);
/* MechSystemSolver.backwardEuler (MechSystemSolver.java:2171-2476) for a host
   that keeps the state: x, v (3N each, host memory, in/out) are copied in,
   nsteps steps run, and the new x, v are copied back, with one
   synchronisation for the whole call.  The PCG's initial guess extrapolates
   the engine's own last two velocities (the warm start); when the host hands
   back the state it received, the result equals b200fem_backward_euler_step
   on the device-resident state bit for bit. */
int b200fem_backward_euler_step_host(b200fem_handle h, const b200fem_step_params* p, int nsteps,
                                     double* x, double* v, b200fem_stats* stats);
/* y = S x with the solve matrix of the last step (host vectors, 3*n_active) */
int b200fem_spmv(b200fem_handle h, const double* x, double* y);
/* block-Jacobi PCG on the solve matrix of the last step (host vectors) */
int b200fem_pcg_solve(b200fem_handle h, const double* b, double* x, double tol, int max_iter,
                      b200fem_stats* stats);
/* synchronise and report the device time of the last step/update call */
int b200fem_last_timing(b200fem_handle h, double* assemble_ms, double* solve_ms);

/* ---- batched form: several independent models in one handle ------------- */
/* The handle's models form one "pack": any mix of element types and
   materials; kernels run over all models at once (each PCG launch solves
   every model, each with its own scalars and convergence test).
   b200fem_set_mesh/_set_material define model 0; b200fem_add_model appends
   (or fills model 0 while it is empty).  State arrays of set_state,
   get_state and set_external_forces are the models' node arrays
   concatenated in model order; b200fem_model_range gives each slice. */
int b200fem_add_model(b200fem_handle h, int elem_type, int n_nodes, const double* rest_xyz,
                      int n_elems, const int* conn, const int* fixed, int mat_kind,
                      const double* params, double density, int incomp_method, int* model_index);
int b200fem_clear_models(b200fem_handle h);
int b200fem_num_models(b200fem_handle h, int* n_models);
/* node offset and count of one model in the concatenated state arrays, and
   its active block rows (DOF / 3) */
int b200fem_model_range(b200fem_handle h, int model, int* node_offset, int* n_nodes, int* n_active);
/* per-model PCG iterations and true relative residuals of the last solve */
int b200fem_get_model_stats(b200fem_handle h, int* iterations, double* rel_residual);
/* Which models the following calls work on (continuous batching: one pack
   step advances only the models that have work).  active[m] == 0 leaves
   model m out of assembly, RHS, PCG and the state update: its positions and
   velocities stay as they are and its stats read 0 iterations.  NULL makes
   every model active again (the default after b200fem_build).  No
   counterpart in the reference, which steps one model per MechModel. */
int b200fem_set_active_models(b200fem_handle h, const int* active);
/* device memory the handle's pack holds (bytes), for admission against a
   device-memory budget */
int b200fem_memory_usage(b200fem_handle h, unsigned long long* bytes);

/* ---- tuning options ------------------------------------------------------
   No counterpart in the reference (its solves are a direct PARDISO/cuDSS
   factorisation or an unpreconditioned CGSolver).  They choose how the
   persistent PCG kernel lays the pack's rows over the GPU; results agree
   across settings to rounding (each setting is bit-reproducible by itself).
   SPLIT, CTAS and PIECE_ROWS take effect at b200fem_build; ROW_LANES,
   WARM_START and ELEM_TILE also afterwards (the step graphs are re-captured). */
#define B200FEM_OPT_PCG_SPLIT 1  /* 0 auto; 1 contiguous rows per CTA (shared-memory
                                    resident when they fit); 2 strided: every model cut
                                    into short pieces dealt over all CTAs; 3 cluster: one
                                    thread-block cluster per model, models taken from a
                                    queue largest first.  Auto: contiguous when the rows fit
                                    shared-memory residency or the handle has one model,
                                    else strided (on the 256-beam pack the strided split
                                    measured 10.1 ms per step against the cluster split's
                                    14.2: the slowest model is held to one cluster) */
#define B200FEM_OPT_ROW_LANES 2  /* lanes per block row in the iteration SpMV: 0 auto, 4, 8, 16, 32 */
#define B200FEM_OPT_PCG_CTAS 3   /* CTAs of the persistent PCG kernel: 0 auto (one per SM) */
#define B200FEM_OPT_PIECE_ROWS 4 /* block rows per piece in the strided split: 0 auto (64) */
#define B200FEM_OPT_WARM_START 5 /* PCG start: the velocity extrapolated by a polynomial of
                                    order 0..4 through the last 1..5 velocities: 0 v_n; 1
                                    2 v_n - v_(n-1); 2 3 (v_n - v_(n-1)) + v_(n-2); 3
                                    4 (v_n + v_(n-2)) - 6 v_(n-1) - v_(n-3); 4 (default)
                                    5 (v_n - v_(n-3)) + 10 (v_(n-2) - v_(n-1)) + v_(n-4).
                                    Only the iteration count depends on it (may be changed
                                    after the build) */
#define B200FEM_OPT_ELEM_TILE 6  /* non-linear element kernels: 0 (default) tets one thread per
                                    element in registers, hexes the staged kernel's large tile;
                                    1 the shared-memory staged kernel with its large tile (tet 256 /
                                    hex 32 NeoHookean, 128 / 16 MooneyRivlin); 2 with half of it
                                    (may be changed after the build) */
#define B200FEM_OPT_REFINE 8     /* refinement sweeps of the mixed form (0..4, default 0): each
                                    forms the FP64 residual b - S64 v matrix-free from the
                                    elements' FP64 tangents, solves the correction with the FP32
                                    matrix to 1e-3 and adds it (one NeoHookean/MooneyRivlin
                                    group without NODAL incompressibility; may be changed after
                                    the build) */
#define B200FEM_OPT_FUSED_ASSEMBLY 7 /* BackwardEuler assembly: 0 (default) element kernel +
                                        block gather; 1 fused row-chunk assembly for NeoHookean /
                                        MooneyRivlin packs without NODAL incompressibility (after
                                        the build: 1 when the fused path is in force).  The fused
                                        path avoids the element blocks' HBM round trip but
                                        recomputes boundary elements; it measured slower on the
                                        benchmark meshes and is kept for larger chunks later. */
#define B200FEM_OPT_BARRIER_TIMEOUT_MS 9 /* bound of every wait at the PCG's grid barriers, in ms
                                          (1..60000, default 5000): a wait that runs out ends
                                          the solve with B200FEM_ERR_TIMEOUT and the device
                                          context stays usable (may be changed after the build) */
#define B200FEM_OPT_TEST_SKIP_ARRIVAL 10 /* failure-detection tests only: CTA index + 1 of the PCG
                                           kernel that does not arrive at its first grid barrier,
                                           so every wait there runs out after
                                           B200FEM_OPT_BARRIER_TIMEOUT_MS; 0 (default) off */
#define B200FEM_OPT_TET_ASSEMBLY 11 /* BackwardEuler assembly of tetrahedral packs with non-linear
                                       materials: 0 node-row kernel -- a warp per few block rows
                                       recomputes each incident tetrahedron and sums the rows'
                                       blocks, forces and right-hand side, with no element data in
                                       HBM; 1 (default) element kernel + block gather.  S and b
                                       agree to rounding.  The node-row kernel evaluates every
                                       tetrahedron four times and is compute-bound: 1.10 ms per
                                       step on the 256-beam pack against 0.59 for the element
                                       path.  Set before b200fem_build; after it, 0 reads back
                                       as 1 where the node-row path does not apply */
#define B200FEM_OPT_PCG_RESIDENT 12 /* row state of the contiguous split's PCG: 2 in shared memory
                                       when the CTA's rows fit (512-thread CTAs, one per SM); 1
                                       never (1024-thread CTAs, global vectors: twice the warps
                                       for the SpMV's loads); 0 (auto) as 2 while the solve
                                       matrix is at most 64 MB (it stays in L2), else as 1.  Set
                                       before b200fem_build; after it, 2 or 1 as in force */
#define B200FEM_OPT_NODAL_FACTORED 13 /* BackwardEuler solve matrix of NODAL models: 2 factored
                                         -- the element blocks of direct neighbours assembled
                                         (S1), the dilational term (h^2 + h beta) sum_n kp_n
                                         d_n d_n^T (computeNodalIncompressibility,
                                         FemModel3d.java:2632-2669) applied from the divBlk
                                         rows d_n inside every SpMV, so the PCG streams the
                                         1-ring blocks instead of the 2-ring pattern; 1
                                         assembled (the 2-ring blocks, as the reference
                                         builds them); 0 (auto) as 2 wherever it applies
                                         (element-path assembly, grid-wide PCG, no frame
                                         attachments).  The step results agree to the PCG
                                         tolerance.  After a b200fem_update_stress_stiffness
                                         call the factored solve matrix is stale:
                                         b200fem_spmv and b200fem_pcg_solve then need another
                                         step.  Set before b200fem_build; after it, 2 or 1 as
                                         in force */
int b200fem_set_option(b200fem_handle h, int key, int value);
/* the value in force (after b200fem_build: the resolved one, e.g. the split chosen by auto) */
int b200fem_get_option(b200fem_handle h, int key, int* value);

/* ---- served form: continuous-batching request server ---------------------
   No counterpart in the reference (ArtiSynth steps one MechModel at a time).
   The server keeps admitted models resident on the device in packs and
   advances them in ticks: one tick is one BackwardEuler step of every
   resident model with a pending request, all models of a pack in the same
   launches; requests that arrive between ticks join at the next one, and a
   model's requests run FIFO.  Admission is against budget_bytes of device
   memory: idle packs are evicted (least recently used, states kept on the
   host) to make room, and a model larger than the budget fails its requests.
   Every pack steps with the parameters given at creation and the options set
   with b200fem_server_set_option.  Times are seconds on the server's clock
   (b200fem_server_clock).  Calls on one server are serialised. */
typedef struct b200fem_server* b200fem_server_handle;
typedef struct {
  long long ticks, model_steps, slot_steps, builds, evictions, completed, failed;
  unsigned long long resident_bytes, peak_bytes;
  int pending;          /* requests not yet done */
  int resident_models;
} b200fem_server_stats;
/* NULL on invalid arguments */
b200fem_server_handle b200fem_server_create(const b200fem_config* cfg, double budget_bytes, int pack_models,
                                            const b200fem_step_params* step);
int b200fem_server_destroy(b200fem_server_handle s);
const char* b200fem_server_last_error(b200fem_server_handle s);
double b200fem_server_clock(b200fem_server_handle s);
/* a B200FEM_OPT_* option for every pack the server builds */
int b200fem_server_set_option(b200fem_server_handle s, int key, int value);
/* a model of the pool (host copy; admitted on its first request or by preload);
   params as b200fem_set_material (8 values), fext may be NULL */
int b200fem_server_add_model(b200fem_server_handle s, int elem_type, int n_nodes, const double* rest_xyz,
                             int n_elems, const int* conn, const int* fixed, int mat_kind,
                             const double* params, double density, int incomp_method, const double* fext,
                             int* model_id);
/* a request of `steps` BackwardEuler steps of one model; t_arrive on the
   server clock (a negative value: now) -- a caller replaying an arrival
   stream passes the scheduled time so that queueing before the call counts */
int b200fem_server_submit(b200fem_server_handle s, int model, int steps, double t_arrive, int* request_id);
/* admit every pool model that fits the budget before any request */
int b200fem_server_preload(b200fem_server_handle s);
/* admission, then one step of every resident model with work */
int b200fem_server_tick(b200fem_server_handle s, int* model_steps);
/* state: 0 queued, 1 running, 2 done (latency = completion - arrival), -1 failed */
int b200fem_server_poll(b200fem_server_handle s, int request_id, int* state, double* latency_s);
int b200fem_server_get_state(b200fem_server_handle s, int model, double* x, double* v);
int b200fem_server_get_stats(b200fem_server_handle s, b200fem_server_stats* out);

/* ---- allocation-free solve ---------------------------------------------- */
/* Size limits of b200fem_pcg_solve_noalloc: its scratch is one fixed device
   array (about 2.6 MB) sized for these limits. */
#define B200FEM_NOALLOC_MAX_ROWS 8192  /* 3x3 block rows (24,576 unknowns) */
#define B200FEM_NOALLOC_MAX_ITER 16384

/* No counterpart in the reference.  Block-Jacobi PCG on S x = b that
   allocates nothing, for callers that cannot allocate device memory (their
   device memory belongs to another allocator or pool, or they forbid
   allocation after start-up).  All arrays are caller-owned DEVICE memory on
   the current device: the block-CSR matrix (rowptr n_rows+1, col nnzb, vals
   9*nnzb row-major 3x3 blocks, every row holding its diagonal block), b and
   x (3*n_rows; x is the initial guess on entry and the solution on exit).
   Every other buffer comes from a static device array that each device
   which loads the library holds until the process exits.  Sizes beyond
   B200FEM_NOALLOC_MAX_ROWS / _MAX_ITER are rejected with
   B200FEM_ERR_BUDGET; n_rows or max_iter below 1, and a matrix with a row
   that holds no diagonal block (checked before the solve reads any block),
   with B200FEM_ERR_INVALID_ARG.  Running out of iterations returns
   B200FEM_ERR_NO_CONVERGE with x holding the last iterate.  The first call on a device looks up the array's
   device address (cudaGetSymbolAddress); make that first call before any
   stream capture.  The call runs on `stream` (a cudaStream_t, NULL for the
   legacy default stream) and returns after it completes; all calls share
   the one array, so calls that overlap on the GPU (other threads, other
   streams) race and must be serialised by the caller.  Messages go to
   b200fem_last_error(NULL). */
int b200fem_pcg_solve_noalloc(int n_rows, const int* rowptr, const int* col, const double* vals,
                              const double* b, double* x, double tol, int max_iter, void* stream,
                              int* iterations, double* rel_residual);

#ifdef __cplusplus
}
#endif
#endif /* B200FEM_H */
