// engine.h -- internal data structures of the B200 FEM engine.
//
// One engine ("Pack") holds one or more independent FEM models packed into
// flat arrays: node, element, block-row and block indices are global across
// the pack, and per-model tables give each model's ranges and parameters.  A
// single-model handle is a pack of one; the batched and served forms use the
// same arrays with many models, so every kernel below is written once.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/b200fem.h"

namespace b200fem {

constexpr int kMaxNen = 20;
constexpr int kMaxIp = 8;
constexpr int kMatParams = 8;

// nodes and integration points per element type (0 for an unknown type);
// wedges and pyramids, like hexes, have one integration point per node
__host__ __device__ constexpr int elem_nen(int type) {
  return type == B200FEM_ELEM_TET ? 4 : type == B200FEM_ELEM_HEX ? 8 : type == B200FEM_ELEM_WEDGE ? 6
         : type == B200FEM_ELEM_PYRAMID ? 5 : type == B200FEM_ELEM_QUADTET ? 10 : type == B200FEM_ELEM_QUADHEX ? 20
         : type == B200FEM_ELEM_QUADWEDGE ? 15 : type == B200FEM_ELEM_QUADPYRAMID ? 13 : 0;
}
__host__ __device__ constexpr int elem_nip(int type) {
  return type == B200FEM_ELEM_TET ? 1 : type == B200FEM_ELEM_QUADTET ? 4 : type == B200FEM_ELEM_QUADHEX ? 14
         : type == B200FEM_ELEM_QUADWEDGE ? 9 : type == B200FEM_ELEM_QUADPYRAMID ? 5 : elem_nen(type);
}
// the linear type a quadratic type is built from (createQuadraticModel)
__host__ __device__ constexpr int elem_linear_base(int type) {
  return type == B200FEM_ELEM_QUADTET ? B200FEM_ELEM_TET : type == B200FEM_ELEM_QUADHEX ? B200FEM_ELEM_HEX
         : type == B200FEM_ELEM_QUADWEDGE ? B200FEM_ELEM_WEDGE : type == B200FEM_ELEM_QUADPYRAMID ? B200FEM_ELEM_PYRAMID
         : -1;
}
// pressure values per element of ELEMENT soft incompressibility
// (FemElement3d.numPressureVals: QuadhexElement 4, QuadwedgeElement 2)
__host__ __device__ constexpr int elem_npv(int type) {
  return type == B200FEM_ELEM_QUADHEX ? 4 : type == B200FEM_ELEM_QUADWEDGE ? 2 : 1;
}
// integration point k lies at node k (FemElement3d.integrationPointsMapToNodes)
__host__ __device__ constexpr bool elem_ip_at_nodes(int type) {
  return type == B200FEM_ELEM_HEX || type == B200FEM_ELEM_WEDGE || type == B200FEM_ELEM_PYRAMID;
}

// element type of a model or pack whose elements are not all of one type
constexpr int kElemMixed = -1;

// Model as given by the caller (host, FP64).
struct ModelDesc {
  int elem_type = B200FEM_ELEM_TET;  // kElemMixed: per element in etypes
  int n_nodes = 0, n_elems = 0;
  std::vector<double> rest;  // 3N
  std::vector<int> conn;     // every element's nodes, concatenated in element order
  std::vector<int> etypes;   // per element (mixed meshes only)
  std::vector<int> fixed;    // N
  int mat_kind = B200FEM_MAT_LINEAR;
  double mat_params[kMatParams] = {0};
  double density = 1000;
  int incomp_request = B200FEM_INCOMP_AUTO;
  bool has_material = false;
  // per-element materials (FemElement.setMaterial; FemModel3d.getElementMaterial,
  // FemModel3d.java:608-614): per caller element -1 (the model's material) or
  // an index into the distinct element materials emat_kind / emat_params
  std::vector<int> emat;
  std::vector<int> emat_kind;
  std::vector<double> emat_params;  // kMatParams each
};

// Host-side derived data of one model (setup only).
//
// Element data are held in storage order: the caller's elements sorted by
// type, then material kind and corotation (stable), so that each such class
// forms one contiguous section that the specialised kernels run over.  A
// mesh of one type and one material keeps the caller's order.  Per storage
// element s, coff/ipoff/sqoff give the offsets of its nodes (and force
// slots), integration points and nen x nen entries.
struct ModelHost {
  int incomp = B200FEM_INCOMP_OFF;  // resolved method
  int n_active = 0;
  std::vector<int> sidx;      // per node, -1 when fixed
  std::vector<int> act_node;  // per active row -> node
  std::vector<int> stype;     // per storage element: its type
  std::vector<int> perm;      // storage element -> caller's element
  std::vector<int> iperm;     // caller's element -> storage element
  std::vector<int> smat;      // per storage element: 0 the model's material, k + 1 element material k
  std::vector<int> skind;     // per storage element: its material kind
  std::vector<char> scorot;   // per storage element: corotated linear material
  std::vector<int> sec;       // section bounds in storage order (runs of one type, kind and
                              // corotation), sec.size() = runs + 1
  std::vector<long long> coff, ipoff, sqoff;  // E+1 each
  std::vector<int> sconn;     // nodes in storage order (coff)
  std::vector<double> invJ0;  // ipoff[E]*9
  std::vector<double> detJ0;  // ipoff[E]
  std::vector<double> winvJ0; // E*9 (warping point)
  std::vector<double> rest_vol;
  std::vector<double> mass;   // N
  std::vector<double> K0, f0; // linear materials: sqoff[E]*9, coff[E]*3
  std::vector<double> node_rest_vol;  // NODAL
  // block pattern over active nodes
  std::vector<int> rowptr, col;
  // direct node neighbours (sorted) for NODAL
  std::vector<std::vector<int>> nbr;
};

// Device arrays for the whole pack.  Precision-dependent value arrays are
// allocated in both FP64 and (for the mixed form) FP32.
struct DevPack {
  int n_models = 0;
  int n_nodes = 0, n_elems = 0, n_rows = 0;
  long long nnzb = 0;
  // node data (FP64)
  double* x = nullptr;       // 3N positions
  double* v = nullptr;       // 3N velocities
  double* fext = nullptr;    // 3N external forces
  double* mass = nullptr;    // N
  int* node_model = nullptr; // N
  int* sidx = nullptr;       // N global row or -1
  int* act_node = nullptr;   // rows -> node
  int* row_model = nullptr;  // rows -> model
  // elements
  int* conn = nullptr;       // node slots (nen per element, storage order): global node indices
  int* elem_model = nullptr; // E
  int* elem_mat = nullptr;   // E: row of mat (the model's row unless the element has its own
                             // material); aliases elem_model when no element has one
  double* invJ0 = nullptr;   // 9 per integration point
  double* winvJ0 = nullptr;  // E*9
  double* K0 = nullptr;      // linear: nen*nen*9 per element
  double* f0 = nullptr;      // linear: 3 per node slot
  float* invJ0_f = nullptr;  // mixed form copy
  // assembly maps
  int* blk_rowptr = nullptr; // n_rows+1 (global block index)
  int* blk_col = nullptr;    // nnzb (global row index)
  int* blk_diag = nullptr;   // n_rows
  int* blk_row = nullptr;    // nnzb -> row
  int* contrib_ptr = nullptr;  // nnzb+1
  int* contrib_idx = nullptr;  // (elem*npair + pair) << 1 | transpose
  int* inc_ptr = nullptr;      // N+1 node -> element incidences
  int* inc_idx = nullptr;      // node slot of the incidence (element's first slot + local node)
  // element outputs
  double* elemK = nullptr;     // 9 per upper-triangle node pair of each element
  double* elemF = nullptr;     // 3 per node slot
  float* elemK_f = nullptr;
  // assembled values
  double* K = nullptr;         // nnzb*9 stiffness (drop-in output)
  double* S = nullptr;         // nnzb*9 solve matrix
  float* S_f = nullptr;        // FP32 copy (mixed form)
  double* Dinv = nullptr;      // n_rows*9 block-Jacobi inverse
  double* fint = nullptr;      // 3N internal force
  // solve vectors (3*n_rows)
  double* b = nullptr;
  double* sol = nullptr;
  double* r = nullptr;
  double* z = nullptr;
  double* p = nullptr;
  double* q = nullptr;
  double* w = nullptr;
  double* u = nullptr;
  double* s = nullptr;
  double* m0 = nullptr;
  double* m1 = nullptr;
  // per model tables
  double* mat = nullptr;       // kMatParams per row: the models' materials, then element materials
  double* step = nullptr;      // n_models*8: h, alpha, beta, gx, gy, gz, tol, -
  // NODAL incompressibility (FemModel3d.java:2471-2669)
  double* node_rest_vol = nullptr;
  double* node_vol = nullptr;
  double* node_p = nullptr;    // nodal pressure
  double* node_kp = nullptr;   // dilational modulus / rest volume
  double* mat_node = nullptr;  // per node: kappa, bulk potential of its model
  int* nbr_ptr = nullptr;      // N+1 direct neighbours (sorted node ids)
  int* inc_slot = nullptr;     // per incidence (inc_idx order): nen_max slots in nbr(n)
  int* inc_tl = nullptr;       // mixed packs: per incidence (element type << 8) | local node
  double* divblk = nullptr;    // nbr_ptr[N] x 3: d V_n / d x_m
  int* dil_ptr = nullptr;      // nnzb+1 dilational contributions per block
  int* dil_idx = nullptr;      // (divblk row i, divblk row j, node n) triples
  int has_nodal = 0;
  // NODAL solve matrix in factored form (B200FEM_OPT_NODAL_FACTORED): the
  // direct-neighbour blocks S1 (the element terms) assembled, the dilational
  // term c_m sum_n kp_n d_n d_n^T applied from divBlk inside every SpMV
  int* s1_rowptr = nullptr;    // n_rows+1
  int* s1_col = nullptr;       // s1_nnzb
  int* s1_diag = nullptr;      // n_rows
  long long s1_nnzb = 0;
  double* S1 = nullptr;        // s1_nnzb*9 (FP64 form)
  float* S1_f = nullptr;       // s1_nnzb*9 (mixed form)
  int* up1_dst = nullptr;      // n_up1: S1 position of each upper direct block (up1 lists them)
  int* up1_mdst = nullptr;     // n_up1: S1 position of its transpose
  int* up1 = nullptr;          // n_up1: block index in the full pattern
  long long n_up1 = 0;
  int* dil_rptr = nullptr;     // n_rows+1: per row its (node n, divBlk slot of the row's node in nbr(n))
  int* dil_node = nullptr;
  int* dil_slot = nullptr;
  int* nbr_row = nullptr;      // nbr_ptr[N]: block row of each neighbour slot (-1 fixed)
  int* dil_nodes = nullptr;    // the active nodes of NODAL models (the dilational terms' nodes)
  int n_dil_nodes = 0;
  double* dil_t = nullptr;     // N: c_m kp_n (d_n . v) of the SpMV in progress
  // ELEMENT soft incompressibility: per element rest volume, pressure and
  // Rinv (effective modulus / rest volume)
  double* elem_rest_vol = nullptr;
  double* elem_p = nullptr;    // npv pressure values per element
  double* elem_r = nullptr;    // npv * npv per element: Rinv
  double* detJ0 = nullptr;     // per integration point: rest Jacobian determinant (several pressure values)
  // reductions / PCG control
  double* partials = nullptr;  // [2][n_pieces][4] (double-buffered by phase)
  int* piece_row = nullptr;    // n_pieces+1
  int* piece_model = nullptr;  // n_pieces
  int* model_piece = nullptr;  // n_models+1
  int* cta_piece = nullptr;    // pcg_grid+1
  int* cta_plist = nullptr;    // n_pieces: global piece indices, CTA-major
  int* model_active = nullptr; // n_models: 0 = left out of assembly and steps
  double* vprev = nullptr;     // 3N: velocity before the last step (warm-start extrapolation)
  double* vprev2 = nullptr;    // 3N: velocity before that (quadratic extrapolation)
  double* vprev3 = nullptr;    // 3N: and before that (cubic extrapolation)
  double* vprev4 = nullptr;    // 3N: and before that (quartic extrapolation)
  // fused assembly: block-row chunks, their incident elements, and the
  // contribution lists re-indexed to chunk-local elements
  int* chunk_row = nullptr;    // chunks+1
  int* chunk_eptr = nullptr;   // chunks+1
  int* chunk_elem = nullptr;
  int* contrib_loc = nullptr;  // parallel to contrib_idx
  int* blk_mirror = nullptr;   // nnzb: the block at the transposed position
  int* up_blocks = nullptr;    // the upper blocks (column >= row), in BSR order
  long long n_up = 0;
  // node-row tet assembly (tet_rows.cu): tasks of block rows, the rows'
  // element incidences, and per contribution the stage entry it reads
  int* task_row = nullptr;     // tasks+1
  int* row_incptr = nullptr;   // rows+1
  int* row_inc = nullptr;      // (element << 3) | (local node << 1) | records the element's statistics
  unsigned char* contrib_byte = nullptr;  // parallel to contrib_idx
  // cluster PCG split (pcg_cluster.cu)
  int* model_row = nullptr;    // models+1: first block row of each model
  int* cl_order = nullptr;     // models in queue order
  int* cl_queue = nullptr;     // next queue position (cleared per solve)
  double* row_nrm = nullptr;   // 3 per row: unit normal of the row's plane constraint (zero: none)
  // frame attachments (attach.cu): attachment of every extended row (-1
  // free), the attachments' H, the reduced blocks' rows, row offsets and
  // contribution lists (extended block, parts of T), the reduced K and its
  // scalar CRS export
  int* att_row = nullptr;
  double* att_H = nullptr;
  // LinearPointConstraints: constraint offsets, points, their solve rows
  // (-1 fixed), weights, targets; the Schur-complement solves Y (3 rows per
  // constraint x 3R), their right-hand side, the dense matrix and vector
  int* pc_ptr = nullptr;
  int* pc_node = nullptr;
  int* pc_row = nullptr;
  double* pc_w = nullptr;
  double* pc_target = nullptr;
  double* pc_Y = nullptr;
  double* pc_rhs = nullptr;
  double* pc_A = nullptr;
  double* pc_lam = nullptr;
  int pc_cap = 0;  // constraints the device arrays hold
  int* red_row = nullptr;
  int* red_rowptr = nullptr;
  int* red_eptr = nullptr;
  int* red_ep = nullptr;
  unsigned char* red_esel = nullptr;
  double* K_red = nullptr;
  double* crs_red = nullptr;
  double* row_off = nullptr;   // per row: the plane's offset
  // refinement sweeps: FP64 residual, correction, its PCG results
  double* rref = nullptr;
  double* dsol = nullptr;
  double* model_scal2 = nullptr;
  int* unconv = nullptr;       // PCG per-iteration 'some model unconverged' words
  int unconv_cap = 0;
  int n_pieces = 0;
  double* model_scal = nullptr;  // n_models*8: rho, rr, bb, pq, conv, iters...
  // mapped pinned host memory the status kernel fills after a step: flags[4]
  // (as doubles), the smallest detJ's ordered bits, model_scal (n_models * 4)
  double* status_host = nullptr;
  double* status_dev = nullptr;
  unsigned* barrier = nullptr;   // [count, generation]
  int* flags = nullptr;          // [error, inverted count, ...]
  double* dmin = nullptr;        // min detJ (atomically reduced as ordered bits)
};

// FEM nodes attached to frames (PointFrameAttachment with an active master
// frame): set by b200fem_set_frame_attachments, reduced by attach.cu
struct FrameAttach {
  int n_frames = 0;
  std::vector<int> node, frame;  // per attachment: the node (model 0) and its frame
  std::vector<double> H;         // per attachment: the 6x3 master block, row-major
  bool active() const { return n_frames > 0; }
  // the reduced system (built with the pack): free active nodes, then two
  // block rows per frame
  int n_free = 0, n_red = 0;
  long long nnzb = 0;
  std::vector<int> rowptr, col, sidx;
};

// LinearPointConstraints (b200fem_set_point_constraints): constraint c holds
// sum over q in [ptr[c], ptr[c+1]) of w[q] x[node[q]] at target[3c..3c+2]
struct PointCons {
  int n = 0;
  std::vector<int> ptr, node;
  std::vector<double> w, target;
  bool active() const { return n > 0; }
};

// One element group: contiguous element range with one element type and
// material kind (kernels are specialised on both).
//
// Kernels see a group's elements as 0 .. e1-e0-1: their per-element arrays
// are offset to the group's first element (c0 node slots, ip0 integration
// points, pr0 upper-triangle pairs, sq0 nen x nen entries, pv0 pressure
// values, pv20 npv x npv entries), so one layout serves every element type.
struct ElemGroup {
  int e0 = 0, e1 = 0;
  long long c0 = 0, ip0 = 0, pr0 = 0, sq0 = 0, pv0 = 0, pv20 = 0;
  int elem_type = B200FEM_ELEM_TET;
  int mat_kind = B200FEM_MAT_LINEAR;
  int corotated = 1;
  int nodal = 0;
  int elem_inc = 0;  // ELEMENT soft incompressibility (one pressure per element)
};

struct Engine {
  int device = 0;
  int precision = B200FEM_PREC_FP64;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> ev_pool;  // 3 per step of a multi-step call
  std::string last_error;
  std::vector<ModelDesc> models;
  std::vector<ModelHost> hosts;
  std::vector<ElemGroup> groups;
  std::vector<int> node_off, elem_off, row_off;
  std::vector<long long> blk_off;
  DevPack d;
  bool built = false;
  bool have_matrix = false;
  int elem_type = B200FEM_ELEM_TET;  // pack-wide element type (kElemMixed: several)
  int nen_max = 4;                   // largest element of the pack
  bool divblk_smem = false;          // NODAL divBlk sums in shared memory (every node <= 32 neighbours)
  // host copies for queries
  std::vector<int> h_rowptr, h_col;
  std::vector<int> h_scatter;  // E*nen*nen
  std::vector<int> h_sidx;
  std::vector<double> h_mass;
  // pcg launch geometry
  int pcg_grid = 0, pcg_block = 256;
  int pcg_resident = 0, pcg_cached = 0, pcg_nloc_max = 0, pcg_nb_max = 0;
  int pcg_strided = 0;  // pieces dealt to CTAs across models (large packs)
  bool pcg_cluster = false;  // one thread-block cluster per model (pcg_cluster.cu)
  int cl_clusters = 0;       // clusters resident at once
  int pcg_every_cta_rows = 0;  // every CTA of the PCG split holds at least one piece
  // plane constraints (b200fem_set_plane_constraints): per constrained node
  // its unit normal and offset; enforced by the ConstrainedBackwardEuler step
  FrameAttach att;  // frame attachments of model 0
  PointCons pcons;  // LinearPointConstraints (ConstrainedBackwardEuler)
  std::vector<int> cons_node;
  std::vector<double> cons_nrm, cons_off;
  int integrator = 0;  // of the captured step graph
  bool any_inactive = false;  // some model_active entry is 0 (kernels get the mask)
  // tuning options (B200FEM_OPT_*): 0 = automatic
  int opt_split = 0, opt_row_lanes = 0, opt_ctas = 0, opt_piece_rows = 0;
  // PCG initial guess: the velocity extrapolated by a polynomial of this
  // order through the last opt_warm_start + 1 velocities (0: v itself)
  int opt_warm_start = 4;
  bool elem_tile_small = false;  // element kernels: the small tile of each material
  bool elem_staged = false;      // tets: the shared-memory staged kernel instead of one thread per element
  bool fused = false;            // BackwardEuler assembly on the fused row-chunk path
  // BackwardEuler assembly of tet packs on the node-row path (tet_rows.cu):
  // B200FEM_OPT_TET_ASSEMBLY 0 (default) where supported, 1 element kernel + gather
  int opt_tet_assembly = 1;  // element path (B200FEM_OPT_TET_ASSEMBLY)
  int opt_resident = 0;      // B200FEM_OPT_PCG_RESIDENT
  int opt_nodal_factored = 0;  // B200FEM_OPT_NODAL_FACTORED: 0 auto, 1 assembled, 2 factored
  bool factored = false;       // the step's NODAL solve matrix in factored form
  bool tet_rows = false;
  int rows_cap = 32;                   // incidences per task (32 or 64)
  std::vector<int> rows_task_off;      // per element group: its task range
  int fused_chunks = 0, fused_emax = 0;
  int opt_fused = 0;             // 1: fused assembly where supported
  int opt_refine = 0;            // refinement sweeps of the mixed form
  bool refine_ok = false;        // supported by the pack (mixed, one NeoHookean/MooneyRivlin group, no NODAL)
  double refine_tol = 1e-3;      // relative tolerance of a correction solve
  // bound of every PCG grid-barrier wait (B200FEM_OPT_BARRIER_TIMEOUT_MS)
  int barrier_timeout_ms = 5000;
  // B200FEM_OPT_TEST_SKIP_ARRIVAL: CTA index + 1 that skips its first
  // barrier arrival (failure-detection tests; 0 off)
  int test_skip_arrival = 0;
  int pcg_attr_smem = -1;
  int pcg_variant = 0;
  int pcg_row_lanes = 16;  // lanes per block row in the PCG SpMV (tunable)
  // captured BackwardEuler step (element, gather, RHS, PCG) and its events
  cudaGraphExec_t asm_exec = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  int step_exec_max_iter = -1;
  // one step from page-locked host state as one graph (the buffers it holds)
  cudaGraphExec_t host_exec = nullptr;
  const double* host_x = nullptr;
  const double* host_v = nullptr;
  bool use_graphs = true;
  // last timing
  float last_asm_ms = 0, last_solve_ms = 0, last_call_ms = 0;
  std::vector<double> last_step_params;
  b200fem_stats last_stats{};
  std::vector<void*> allocations;
  size_t device_bytes = 0;  // sum of the allocations above
};

// setup.cpp
int setup_model_host(const ModelDesc& m, ModelHost& h, std::string& err);
int build_pack(Engine& eng);
void free_pack(Engine& eng);
cudaError_t launch_status_pack(Engine& eng);
int grid_dims(int type, int nx, int ny, int nz, int* nn, int* ne);
// linear -> quadratic elements with shared edge nodes (createQuadraticModel);
// lin_type tet, hex, wedge or pyramid
void quadratic_mesh(int lin_type, int nn, const double* xyz, int ne, const int* conn, std::vector<double>& out_xyz,
                    std::vector<int>& out_conn);
// dN/ds of the element's nodes at integration point k (k = -1: the warping
// point) and the point's weight
void shape_grads(int type, int k, double* g /* nen * 3 */, double* w);
// pressure weights H of every integration point (nip * npv) and the weight
// matrix W = (sum_k H H^T)^-1 (npv * npv) of a multi-pressure element type
void pressure_tables(int type, double* H, double* W);
void create_grid(int type, double wx, double wy, double wz, int nx, int ny, int nz, double* xyz,
                 int* conn);
void jitter_grid(int nx, int ny, int nz, double wx, double wy, double wz, double frac,
                 unsigned long long seed, double* xyz);

// tet_rows.cu
cudaError_t launch_tet_rows(Engine& eng, bool attr_only);

// point_cons.cu
cudaError_t launch_solve_points(Engine& eng, int max_iter);
// kernels.cu: x += h v, v and its history shifted, for the active rows
cudaError_t launch_state_update(Engine& eng, const double* vsol);

// attach.cu
int build_attachment_reduction(Engine& eng, std::string& err);
cudaError_t launch_attach_reduce(Engine& eng);

// pcg_cluster.cu
int pcg_cluster_capacity(bool fp32);
cudaError_t launch_pcg_cluster(Engine& eng, int max_iter, bool update_state, const double* rhs, double* xsol,
                               double tol_override, double* model_out);

// kernels.cu
cudaError_t launch_assemble(Engine& eng, double cK, double cM, bool want_K);
cudaError_t launch_rhs(Engine& eng);
cudaError_t launch_reset_status(Engine& eng);
cudaError_t launch_pcg(Engine& eng, int max_iter, bool update_state, int init_zero);
cudaError_t launch_pcg_on(Engine& eng, int max_iter, bool update_state, const double* rhs, double* xsol,
                          double tol_override, double* model_out);
cudaError_t launch_solve(Engine& eng, int max_iter);
cudaError_t launch_spmv(Engine& eng, const double* x, double* y);
cudaError_t launch_crs_export(Engine& eng, const double* vals, double* crs);
void crs_export_kernel_launch(Engine& eng, long long nnzb, const int* blk_row, const int* rowptr, const double* vals,
                              double* crs);
int read_pcg_result(Engine& eng, b200fem_stats* st);

}  // namespace b200fem
