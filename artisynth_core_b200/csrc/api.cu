// api.cu -- C ABI of libb200fem.so (declared in include/b200fem.h) and the
// pack builder that turns host models into device-resident arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>

#include "engine.h"

namespace b200fem {

cudaError_t launch_forces_only(Engine& eng);
int pcg_max_grid(int device);
int pcg_max_cta_pieces();
size_t fused_elem_bytes(int elem_type, int mat_kind, bool fp32);
size_t fused_smem_budget(int elem_type);
void pcg_plan_smem(int device, int nloc_max, int nb_max, int* resident, int* cached, bool fp32);
cudaError_t prepare_pcg(Engine& eng);
cudaError_t prepare_kernels(Engine& eng);
int pcg_solve_noalloc(int n_rows, const int* rowptr, const int* col, const double* vals, const double* b, double* x,
                      double tol, int max_iter, void* stream, int* iterations, double* rel_residual, const char** err);

namespace {

std::mutex g_err_mu;
std::string g_global_err;

void set_global_error(const std::string& s) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_global_err = s;
}

int fail(Engine* e, int code, const std::string& msg) {
  if (e) e->last_error = msg;
  else set_global_error(msg);
  return code;
}

int cuda_fail(Engine* e, cudaError_t err, const char* where) {
  return fail(e, B200FEM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(err));
}

#define CK(call)                                             \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return cuda_fail(&eng, _e, #call); \
  } while (0)

template <typename T>
cudaError_t dalloc(Engine& eng, T** ptr, size_t count) {
  *ptr = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)ptr, count * sizeof(T));
  if (e == cudaSuccess) {
    eng.allocations.push_back((void*)*ptr);
    eng.device_bytes += count * sizeof(T);
  }
  return e;
}

template <typename T>
cudaError_t upload(Engine& eng, T** ptr, const std::vector<T>& v) {
  cudaError_t e = dalloc(eng, ptr, v.size());
  if (e != cudaSuccess) return e;
  if (!v.empty()) e = cudaMemcpy(*ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

void free_pack(Engine& eng) {
  for (cudaGraphExec_t* ex : {&eng.asm_exec, &eng.step_exec, &eng.host_exec})
    if (*ex) {
      cudaGraphExecDestroy(*ex);
      *ex = nullptr;
    }
  eng.step_exec_max_iter = -1;
  eng.last_step_params.clear();
  for (void* p : eng.allocations) cudaFree(p);
  eng.allocations.clear();
  if (eng.d.status_host) cudaFreeHost(eng.d.status_host);
  eng.device_bytes = 0;
  eng.d = DevPack();
  eng.built = false;
  eng.have_matrix = false;
}

int build_pack(Engine& eng) {
  free_pack(eng);
  const int M = (int)eng.models.size();
  if (M == 0) return fail(&eng, B200FEM_ERR_STATE, "no model defined");
  for (auto& m : eng.models) {
    if (!m.has_material) return fail(&eng, B200FEM_ERR_STATE, "material not set");
    if (m.n_nodes <= 0 || m.n_elems <= 0) return fail(&eng, B200FEM_ERR_STATE, "mesh not set");
  }
  eng.hosts.assign(M, ModelHost());
  for (int m = 0; m < M; m++) {
    std::string err;
    int st = setup_model_host(eng.models[m], eng.hosts[m], err);
    if (st != B200FEM_OK) return fail(&eng, st, "model " + std::to_string(m) + ": " + err);
  }
  // pack-wide element type: one type, or kElemMixed
  eng.elem_type = eng.hosts[0].stype.empty() ? B200FEM_ELEM_TET : eng.hosts[0].stype[0];
  eng.nen_max = 0;
  for (auto& h : eng.hosts)
    for (int t : h.stype) {
      if (t != eng.elem_type) eng.elem_type = kElemMixed;
      eng.nen_max = std::max(eng.nen_max, elem_nen(t));
    }
  const bool mixed = eng.elem_type == kElemMixed;
  const int nen = mixed ? 0 : elem_nen(eng.elem_type), nip = mixed ? 0 : elem_nip(eng.elem_type);
  const int npair = nen * (nen + 1) / 2;
  // offsets
  eng.node_off.assign(M + 1, 0);
  eng.elem_off.assign(M + 1, 0);
  eng.row_off.assign(M + 1, 0);
  eng.blk_off.assign(M + 1, 0);
  for (int m = 0; m < M; m++) {
    eng.node_off[m + 1] = eng.node_off[m] + eng.models[m].n_nodes;
    eng.elem_off[m + 1] = eng.elem_off[m] + eng.models[m].n_elems;
    eng.row_off[m + 1] = eng.row_off[m] + eng.hosts[m].n_active;
    eng.blk_off[m + 1] = eng.blk_off[m] + (long long)eng.hosts[m].col.size();
  }
  const int N = eng.node_off[M], E = eng.elem_off[M], R = eng.row_off[M];
  const long long NB = eng.blk_off[M];
  // element layout of the pack in storage order (each model's elements
  // sorted by type): per element its type and the offsets of its node
  // slots, integration points, upper-triangle pairs, nen x nen entries and
  // pressure values; st_of maps the callers' element order to storage order
  std::vector<int> etype(E), st_of(E);
  std::vector<long long> coff(E + 1, 0), ipoff(E + 1, 0), proff(E + 1, 0), sqoff(E + 1, 0), pvoff(E + 1, 0),
      pv2off(E + 1, 0);
  for (int m = 0; m < M; m++) {
    const ModelHost& h = eng.hosts[m];
    const int eo = eng.elem_off[m];
    for (int s = 0; s < eng.models[m].n_elems; s++) {
      etype[eo + s] = h.stype[s];
      st_of[eo + h.perm[s]] = eo + s;
    }
  }
  for (int e = 0; e < E; e++) {
    const int t = etype[e], k = elem_nen(t), v = elem_npv(t);
    coff[e + 1] = coff[e] + k;
    ipoff[e + 1] = ipoff[e] + elem_nip(t);
    proff[e + 1] = proff[e] + k * (k + 1) / 2;
    sqoff[e + 1] = sqoff[e] + (long long)k * k;
    pvoff[e + 1] = pvoff[e] + v;
    pv2off[e + 1] = pv2off[e] + v * v;
  }
  if (NB >= (1ll << 31) || proff[E] * 2 >= (1ll << 31) || coff[E] >= (1ll << 31))
    return fail(&eng, B200FEM_ERR_UNSUPPORTED, "pack too large for 32-bit block indices");
  DevPack& d = eng.d;
  d.n_models = M;
  d.n_nodes = N;
  d.n_elems = E;
  d.n_rows = R;
  d.nnzb = NB;

  // ---- host arrays
  // material table: one row per model, then the models' element materials
  std::vector<int> mat_row(M + 1, M);
  for (int m = 0; m < M; m++) mat_row[m + 1] = mat_row[m] + (int)eng.models[m].emat_kind.size();
  const bool own_mats = mat_row[M] > M;
  std::vector<double> x(3 * (size_t)N), mass(N), mat((size_t)mat_row[M] * kMatParams, 0.0),
      step((size_t)M * 8, 0.0);
  std::vector<int> node_model(N), sidx(N), act_node(R), row_model(R);
  std::vector<int> conn((size_t)coff[E]), elem_model(E), elem_mat(own_mats ? E : 0);
  std::vector<double> invJ0((size_t)ipoff[E] * 9), winvJ0((size_t)E * 9);
  bool any_linear = false, any_nodal = false, permuted = false;
  for (auto& h : eng.hosts) any_linear |= !h.K0.empty();
  for (auto& h : eng.hosts) any_nodal |= (h.incomp == B200FEM_INCOMP_NODAL);
  std::vector<double> K0, f0, node_rest_vol;
  if (any_linear) {
    K0.assign((size_t)sqoff[E] * 9, 0.0);
    f0.assign((size_t)coff[E] * 3, 0.0);
  }
  if (any_nodal) node_rest_vol.assign(N, 1.0);
  std::vector<int> rowptr(R + 1, 0), col(NB), blk_diag(R), blk_row(NB);
  for (int m = 0; m < M; m++) {
    const ModelDesc& md = eng.models[m];
    const ModelHost& h = eng.hosts[m];
    const int no = eng.node_off[m], eo = eng.elem_off[m], ro = eng.row_off[m];
    const long long bo = eng.blk_off[m];
    std::copy(md.rest.begin(), md.rest.end(), x.begin() + 3 * (size_t)no);
    std::copy(h.mass.begin(), h.mass.end(), mass.begin() + no);
    for (int n = 0; n < md.n_nodes; n++) {
      node_model[no + n] = m;
      sidx[no + n] = h.sidx[n] >= 0 ? ro + h.sidx[n] : -1;
    }
    for (int r = 0; r < h.n_active; r++) {
      act_node[ro + r] = no + h.act_node[r];
      row_model[ro + r] = m;
      rowptr[ro + r + 1] = (int)(bo + h.rowptr[r + 1]);
      for (int p = h.rowptr[r]; p < h.rowptr[r + 1]; p++) {
        col[bo + p] = ro + h.col[p];
        blk_row[bo + p] = ro + r;
        if (h.col[p] == r) blk_diag[ro + r] = (int)(bo + p);
      }
    }
    for (size_t q = 0; q < h.sconn.size(); q++) conn[(size_t)coff[eo] + q] = no + h.sconn[q];
    for (int e = 0; e < md.n_elems; e++) {
      elem_model[eo + e] = m;
      if (own_mats) elem_mat[eo + e] = h.smat[e] == 0 ? m : mat_row[m] + h.smat[e] - 1;
      permuted |= h.perm[e] != e;
    }
    std::copy(h.invJ0.begin(), h.invJ0.end(), invJ0.begin() + (size_t)ipoff[eo] * 9);
    std::copy(h.winvJ0.begin(), h.winvJ0.end(), winvJ0.begin() + (size_t)eo * 9);
    if (!h.K0.empty()) {
      std::copy(h.K0.begin(), h.K0.end(), K0.begin() + (size_t)sqoff[eo] * 9);
      std::copy(h.f0.begin(), h.f0.end(), f0.begin() + (size_t)coff[eo] * 3);
    }
    if (!h.node_rest_vol.empty())
      std::copy(h.node_rest_vol.begin(), h.node_rest_vol.end(), node_rest_vol.begin() + no);
    std::copy(md.mat_params, md.mat_params + kMatParams, mat.begin() + (size_t)m * kMatParams);
    std::copy(md.emat_params.begin(), md.emat_params.end(), mat.begin() + (size_t)mat_row[m] * kMatParams);
    step[(size_t)m * 8 + 0] = 0.01;
    step[(size_t)m * 8 + 1] = 2.0;
    step[(size_t)m * 8 + 6] = 1e-10;
  }
  // ---- element-to-block scatter map (storage order, sqoff) and per-block
  // contribution lists; the lists follow the callers' element order, the
  // order in which the reference accumulates the element blocks
  auto block_of = [&](int r, int c) -> int {
    auto b = col.begin() + rowptr[r], e = col.begin() + rowptr[r + 1];
    auto it = std::lower_bound(b, e, c);
    return (it != e && *it == c) ? (int)(it - col.begin()) : -1;
  };
  std::vector<int> scat((size_t)sqoff[E], -1);
  std::vector<int> cptr(NB + 1, 0);
  for (int e = 0; e < E; e++) {
    const int* nodes = &conn[(size_t)coff[e]];
    const int k = elem_nen(etype[e]);
    for (int a = 0; a < k; a++)
      for (int b = 0; b < k; b++) {
        int ra = sidx[nodes[a]], rb = sidx[nodes[b]];
        if (ra < 0 || rb < 0) continue;
        int p = block_of(ra, rb);
        if (p < 0) return fail(&eng, B200FEM_ERR_STATE, "internal: element pair outside the pattern");
        scat[(size_t)sqoff[e] + a * k + b] = p;
        cptr[p + 1]++;
      }
  }
  for (long long p = 0; p < NB; p++) cptr[p + 1] += cptr[p];
  std::vector<int> cidx(cptr[NB]);
  {
    std::vector<int> fill(cptr.begin(), cptr.end() - 1);
    for (int o = 0; o < E; o++) {
      const int e = st_of[o], k = elem_nen(etype[e]);
      int w = 0;
      for (int a = 0; a < k; a++)
        for (int b = a; b < k; b++, w++) {
          int pab = scat[(size_t)sqoff[e] + a * k + b];
          if (pab < 0) continue;
          int code = (int)((proff[e] + w) << 1);
          cidx[fill[pab]++] = code;  // K_ab at (a, b)
          if (a != b) {
            int pba = scat[(size_t)sqoff[e] + b * k + a];
            cidx[fill[pba]++] = code | 1;  // K_ab^T at (b, a)
          }
        }
    }
  }
  // the scatter map in the callers' element order (b200fem_get_scatter_map)
  if (!permuted) {
    eng.h_scatter.swap(scat);
  } else {
    eng.h_scatter.clear();
    eng.h_scatter.reserve(scat.size());
    for (int o = 0; o < E; o++) {
      const int e = st_of[o];
      eng.h_scatter.insert(eng.h_scatter.end(), scat.begin() + sqoff[e], scat.begin() + sqoff[e + 1]);
    }
    std::vector<int>().swap(scat);
  }
  // node -> element incidences in the callers' element order: the node slot
  // (inc_idx), the storage element, and for mixed packs (type << 8) | local node
  std::vector<int> iptr(N + 1, 0);
  for (size_t q = 0; q < conn.size(); q++) iptr[conn[q] + 1]++;
  for (int n = 0; n < N; n++) iptr[n + 1] += iptr[n];
  std::vector<int> iidx(conn.size()), ielem(conn.size()), itl;
  if (mixed) itl.resize(conn.size());
  {
    std::vector<int> fill(iptr.begin(), iptr.end() - 1);
    for (int o = 0; o < E; o++) {
      const int e = st_of[o], k = elem_nen(etype[e]);
      for (int a = 0; a < k; a++) {
        const int q = fill[conn[(size_t)coff[e] + a]]++;
        iidx[q] = (int)coff[e] + a;
        ielem[q] = e;
        if (mixed) itl[q] = (etype[e] << 8) | a;
      }
    }
  }
  // ---- element groups: runs of one element type, material kind, corotation
  // and soft incompressibility (a model of several types or element materials
  // gives one run per section)
  eng.groups.clear();
  for (int m = 0; m < M; m++) {
    const ModelHost& h = eng.hosts[m];
    for (size_t k = 0; k + 1 < h.sec.size(); k++) {
      ElemGroup g;
      g.e0 = eng.elem_off[m] + h.sec[k];
      g.e1 = eng.elem_off[m] + h.sec[k + 1];
      if (g.e1 <= g.e0) continue;
      g.elem_type = etype[g.e0];
      g.mat_kind = h.skind[h.sec[k]];
      g.corotated = h.scorot[h.sec[k]];
      // elements of compressible materials run with OFF (FemModel3d.java:3346-3348)
      const bool inc = g.mat_kind == B200FEM_MAT_MOONEYRIVLIN;
      g.nodal = inc && h.incomp == B200FEM_INCOMP_NODAL;
      g.elem_inc = inc && h.incomp == B200FEM_INCOMP_ELEMENT;
      if (!eng.groups.empty()) {
        ElemGroup& last = eng.groups.back();
        if (last.elem_type == g.elem_type && last.mat_kind == g.mat_kind && last.corotated == g.corotated &&
            last.nodal == g.nodal && last.elem_inc == g.elem_inc && last.e1 == g.e0) {
          last.e1 = g.e1;
          continue;
        }
      }
      eng.groups.push_back(g);
    }
  }
  for (ElemGroup& g : eng.groups) {
    g.c0 = coff[g.e0];
    g.ip0 = ipoff[g.e0];
    g.pr0 = proff[g.e0];
    g.sq0 = sqoff[g.e0];
    g.pv0 = pvoff[g.e0];
    g.pv20 = pv2off[g.e0];
  }
  // ---- node-row tet assembly: tasks of consecutive block rows of one model
  // whose node incidences fit rows_cap lanes, the rows' incidences (element
  // order, the element's first active node records its statistics), and
  // per contribution the stage entry (incidence in task * 4 + column node)
  eng.tet_rows = false;
  eng.rows_task_off.clear();
  std::vector<int> task_row, row_incptr, row_inc;
  std::vector<unsigned char> cbyte;
  if (eng.opt_tet_assembly == 0 && eng.elem_type == B200FEM_ELEM_TET && eng.opt_fused == 0 && R > 0) {
    bool ok = true;
    // (its tasks are runs of one model's rows: every group must cover whole models)
    for (const ElemGroup& g : eng.groups)
      ok &= g.mat_kind != B200FEM_MAT_LINEAR &&
            std::binary_search(eng.elem_off.begin(), eng.elem_off.end(), g.e0) &&
            std::binary_search(eng.elem_off.begin(), eng.elem_off.end(), g.e1);
    std::vector<int> first_active(E, -1);
    for (int e = 0; ok && e < E; e++) {
      for (int a = 0; a < nen && first_active[e] < 0; a++)
        if (sidx[conn[(size_t)e * nen + a]] >= 0) first_active[e] = a;
      ok &= first_active[e] >= 0;  // an element without an active node keeps the element path
    }
    int maxinc = 0;
    for (int r = 0; ok && r < R; r++) maxinc = std::max(maxinc, iptr[act_node[r] + 1] - iptr[act_node[r]]);
    ok &= maxinc <= 64;
    if (ok) {
      const int cap = maxinc <= 32 ? 32 : 64;
      row_incptr.assign(R + 1, 0);
      for (int r = 0; r < R; r++) row_incptr[r + 1] = row_incptr[r] + iptr[act_node[r] + 1] - iptr[act_node[r]];
      row_inc.resize(row_incptr[R]);
      for (int r = 0, k = 0; r < R; r++) {
        const int n = act_node[r];
        for (int i = iptr[n]; i < iptr[n + 1]; i++) {
          const int e = iidx[i] / nen, a = iidx[i] % nen;
          row_inc[k++] = (e << 3) | (a << 1) | (first_active[e] == a ? 1 : 0);
        }
      }
      std::vector<int> task_of_row(R), model_task(M + 1, 0);
      for (int m = 0; m < M; m++) {
        model_task[m] = (int)task_row.size();
        int r = eng.row_off[m];
        while (r < eng.row_off[m + 1]) {
          const int t = (int)task_row.size();
          task_row.push_back(r);
          int cnt = 0;
          while (r < eng.row_off[m + 1] && cnt + (row_incptr[r + 1] - row_incptr[r]) <= cap) {
            cnt += row_incptr[r + 1] - row_incptr[r];
            task_of_row[r++] = t;
          }
        }
      }
      model_task[M] = (int)task_row.size();
      task_row.push_back(R);
      for (const ElemGroup& g : eng.groups) {
        const int m0 = (int)(std::lower_bound(eng.elem_off.begin(), eng.elem_off.end(), g.e0) - eng.elem_off.begin());
        const int m1 = (int)(std::lower_bound(eng.elem_off.begin(), eng.elem_off.end(), g.e1) - eng.elem_off.begin());
        if (eng.rows_task_off.empty()) eng.rows_task_off.push_back(model_task[m0]);
        eng.rows_task_off.push_back(model_task[m1]);
      }
      std::vector<int> pa, pb;
      for (int x0 = 0; x0 < nen; x0++)
        for (int x1 = x0; x1 < nen; x1++) {
          pa.push_back(x0);
          pb.push_back(x1);
        }
      cbyte.resize(cptr[NB]);
      for (long long p = 0; p < NB; p++) {
        const int r = blk_row[p];
        const int rowpos = row_incptr[r] - row_incptr[task_row[task_of_row[r]]];
        const int* rb = row_inc.data() + row_incptr[r];
        const int rn = row_incptr[r + 1] - row_incptr[r];
        for (int c = cptr[p]; c < cptr[p + 1]; c++) {
          const int code = cidx[c];
          const int e = (code >> 1) / npair, w = (code >> 1) % npair;
          const int am = (code & 1) ? pb[w] : pa[w], bl = (code & 1) ? pa[w] : pb[w];
          int lo = 0, hi = rn;
          while (lo < hi) {
            const int mid = (lo + hi) / 2;
            if ((rb[mid] >> 3) < e) lo = mid + 1;
            else hi = mid;
          }
          if (lo >= rn || (rb[lo] >> 3) != e || ((rb[lo] >> 1) & 3) != am)
            return fail(&eng, B200FEM_ERR_STATE, "internal: contribution without its row incidence");
          const int q = rowpos + lo;
          if (q >= cap) return fail(&eng, B200FEM_ERR_STATE, "internal: task incidence beyond its capacity");
          cbyte[c] = (unsigned char)(q * 4 + bl);
        }
      }
      eng.tet_rows = true;
      eng.rows_cap = cap;
    }
  }
  // ---- fused assembly: block-row chunks whose incident elements fit the
  // chunk's shared memory, and the contribution lists re-indexed to them
  std::vector<int> chunk_row, chunk_eptr, chunk_elem, contrib_loc;
  eng.fused = false;
  // (tets and hexes: the fused kernel is instantiated for those two)
  if (eng.opt_fused == 1 && eng.groups.size() == 1 && !eng.groups[0].nodal && !eng.groups[0].elem_inc &&
      (eng.elem_type == B200FEM_ELEM_TET || eng.elem_type == B200FEM_ELEM_HEX) &&
      (eng.groups[0].mat_kind == B200FEM_MAT_NEOHOOKEAN || eng.groups[0].mat_kind == B200FEM_MAT_MOONEYRIVLIN)) {
    const size_t per = fused_elem_bytes(eng.elem_type, eng.groups[0].mat_kind, eng.precision == B200FEM_PREC_MIXED);
    const int emax = (int)(fused_smem_budget(eng.elem_type) / per);
    std::vector<int> stamp(E, -1), loc(E, 0);
    contrib_loc.assign(cidx.size(), 0);
    bool ok = true;
    int cur = 0, nin = 0, rstart = 0;
    chunk_row.push_back(0);
    chunk_eptr.push_back(0);
    auto close = [&](int rend) {
      for (int p = rowptr[rstart]; p < rowptr[rend]; p++)
        for (int q = cptr[p]; q < cptr[p + 1]; q++) {
          const int code = cidx[q];
          const int e = (code >> 1) / npair, w = (code >> 1) % npair;
          contrib_loc[q] = ((loc[e] * npair + w) << 1) | (code & 1);
        }
      chunk_row.push_back(rend);
      chunk_eptr.push_back((int)chunk_elem.size());
      cur++;
      nin = 0;
      rstart = rend;
    };
    for (int r = 0; r < R && ok; r++) {
      const int n = act_node[r];
      int fresh = 0;
      for (int i = iptr[n]; i < iptr[n + 1]; i++) fresh += stamp[iidx[i] / nen] != cur;
      if (fresh > emax) ok = false;  // one row alone does not fit
      if (nin + fresh > emax && r > rstart) {
        close(r);
        fresh = iptr[n + 1] - iptr[n];
      }
      for (int i = iptr[n]; i < iptr[n + 1]; i++) {
        const int e = iidx[i] / nen;
        if (stamp[e] == cur) continue;
        stamp[e] = cur;
        loc[e] = nin++;
        chunk_elem.push_back(e);
      }
    }
    if (ok && R > 0) close(R);
    if (ok) {
      eng.fused = true;
      eng.fused_chunks = (int)chunk_row.size() - 1;
      eng.fused_emax = emax;
    }
  }

  // ---- NODAL soft incompressibility: direct-neighbour lists, incidence
  // slots, and per block the (divBlk i, divBlk j, node) triples of the
  // dilational term, node-ascending
  std::vector<int> nbr_ptr, nbr_idx, inc_slot, dptr, didx;
  std::vector<double> mat_node;
  if (any_nodal) {
    nbr_ptr.assign(N + 1, 0);
    mat_node.assign(2 * (size_t)N, 0.0);
    for (int m = 0; m < M; m++) {
      const int no = eng.node_off[m];
      for (int n = 0; n < eng.models[m].n_nodes; n++) {
        nbr_ptr[no + n + 1] = (int)eng.hosts[m].nbr[n].size();
        mat_node[2 * (size_t)(no + n)] = eng.models[m].mat_params[5];
        mat_node[2 * (size_t)(no + n) + 1] = eng.models[m].mat_params[7];
      }
    }
    int max_nbr = 0;
    for (int n = 0; n < N; n++) max_nbr = std::max(max_nbr, nbr_ptr[n + 1]);
    eng.divblk_smem = max_nbr <= 32;  // kDivSmemSlots
    for (int n = 0; n < N; n++) nbr_ptr[n + 1] += nbr_ptr[n];
    nbr_idx.resize(nbr_ptr[N]);
    for (int m = 0; m < M; m++) {
      const int no = eng.node_off[m];
      for (int n = 0; n < eng.models[m].n_nodes; n++) {
        const auto& v = eng.hosts[m].nbr[n];
        for (size_t k = 0; k < v.size(); k++) nbr_idx[nbr_ptr[no + n] + k] = no + v[k];
      }
    }
    auto slot_of = [&](int n, int node) -> int {
      auto b = nbr_idx.begin() + nbr_ptr[n], e = nbr_idx.begin() + nbr_ptr[n + 1];
      return (int)(std::lower_bound(b, e, node) - b);
    };
    // nen_max entries per incidence (the element's nen used)
    const int nm = eng.nen_max;
    inc_slot.assign(iidx.size() * nm, 0);
    for (int n = 0; n < N; n++)
      for (int i = iptr[n]; i < iptr[n + 1]; i++) {
        const int e = ielem[i], k = elem_nen(etype[e]);
        for (int j = 0; j < k; j++) inc_slot[(size_t)i * nm + j] = slot_of(n, conn[(size_t)coff[e] + j]);
      }
    dptr.assign(NB + 1, 0);
    for (int pass = 0; pass < 2; pass++) {
      std::vector<int> fill;
      if (pass == 1) {
        for (long long p = 0; p < NB; p++) dptr[p + 1] += dptr[p];
        didx.resize(3 * (size_t)dptr[NB]);
        fill.assign(dptr.begin(), dptr.end() - 1);
      }
      for (int m = 0; m < M; m++) {
        if (eng.hosts[m].incomp != B200FEM_INCOMP_NODAL) continue;
        for (int n = eng.node_off[m]; n < eng.node_off[m + 1]; n++) {
          if (sidx[n] < 0) continue;  // volumeIsControllable: active nodes only
          for (int a = nbr_ptr[n]; a < nbr_ptr[n + 1]; a++) {
            const int ra = sidx[nbr_idx[a]];
            if (ra < 0) continue;
            for (int b = nbr_ptr[n]; b < nbr_ptr[n + 1]; b++) {
              const int rb = sidx[nbr_idx[b]];
              if (rb < 0) continue;
              const int p = block_of(ra, rb);
              if (p < 0) return fail(&eng, B200FEM_ERR_STATE, "internal: dilational pair outside the pattern");
              if (pass == 0) {
                dptr[p + 1]++;
              } else {
                int* t = &didx[3 * (size_t)fill[p]++];
                t[0] = a;
                t[1] = b;
                t[2] = n;
              }
            }
          }
        }
      }
    }
  }

  // ---- NODAL solve matrix in factored form: S1 holds the blocks of direct
  // neighbours (those with element contributions), the dilational term is
  // applied in the SpMV as sum_n c kp_n d_n (d_n . v) over the active nodes
  // n of NODAL models (the gather's dilational triples regrouped by node)
  eng.factored = any_nodal && eng.opt_nodal_factored != 1 && !eng.tet_rows && !eng.fused && eng.opt_split != 3 &&
                 !eng.att.active();
  std::vector<int> s1_rowptr, s1_col, s1_diag, s1_of, dil_rptr, dil_node, dil_slot, nbr_row, dil_nodes;
  if (eng.factored) {
    s1_of.assign(NB, -1);
    s1_rowptr.assign(R + 1, 0);
    s1_diag.assign(R, 0);
    int cnt = 0;
    for (int r = 0; r < R; r++) {
      for (int p = rowptr[r]; p < rowptr[r + 1]; p++)
        if (cptr[p + 1] > cptr[p]) {
          s1_of[p] = cnt++;
          s1_col.push_back(col[p]);
        }
      s1_rowptr[r + 1] = cnt;
      // (a row without blocks -- an active node in no element -- points at
      // block 0, as its diagonal does in the full pattern)
      s1_diag[r] = s1_of[blk_diag[r]] >= 0 ? s1_of[blk_diag[r]] : 0;
    }
    nbr_row.resize(nbr_ptr[N]);
    for (int a = 0; a < nbr_ptr[N]; a++) nbr_row[a] = sidx[nbr_idx[a]];
    dil_rptr.assign(R + 1, 0);
    for (int r = 0; r < R; r++) {
      const int i = act_node[r];
      if (eng.hosts[row_model[r]].incomp == B200FEM_INCOMP_NODAL) {
        // nbr(i) ascending: the nodes n whose divBlk row holds a slot for i
        for (int a = nbr_ptr[i]; a < nbr_ptr[i + 1]; a++) {
          const int n = nbr_idx[a];
          if (sidx[n] < 0) continue;  // volumeIsControllable: active nodes only
          auto b = nbr_idx.begin() + nbr_ptr[n], e = nbr_idx.begin() + nbr_ptr[n + 1];
          dil_node.push_back(n);
          dil_slot.push_back((int)(std::lower_bound(b, e, i) - nbr_idx.begin()));
        }
      }
      dil_rptr[r + 1] = (int)dil_node.size();
    }
    for (int m = 0; m < M; m++)
      if (eng.hosts[m].incomp == B200FEM_INCOMP_NODAL)
        for (int n = eng.node_off[m]; n < eng.node_off[m + 1]; n++)
          if (sidx[n] >= 0) dil_nodes.push_back(n);
  }
  // PCG work per row: its blocks, plus (factored) half a block per
  // dilational entry (32 against 76 bytes)
  const std::vector<int>& prow = eng.factored ? s1_rowptr : rowptr;
  std::vector<long long> wrow(R + 1, 0);
  for (int r = 0; r <= R; r++) wrow[r] = prow[r] + (eng.factored ? dil_rptr[r] / 2 : 0);
  const long long WB = wrow[R];

  // ---- PCG work split.  Contiguous: CTAs own contiguous row ranges
  // balanced by blocks, cut into pieces at model boundaries.
  // One 1024-thread CTA per SM at most, >= 32 rows (one per warp) each.
  int gmax = std::min(pcg_max_grid(eng.device), eng.num_sms);
  if (eng.opt_ctas > 0) gmax = std::min(gmax, eng.opt_ctas);
  int G = std::max(1, std::min(gmax, (R + 31) / 32));
  std::vector<int> piece_row, piece_model, cta_piece, model_piece(M + 1, 0);
  bool contiguous_ok = true;
  for (;;) {
    piece_row.clear();
    piece_model.clear();
    cta_piece.assign(G + 1, 0);
    std::vector<int> cut(G + 1, R);
    cut[0] = 0;
    int r = 0;
    for (int c = 1; c < G; c++) {
      long long target = WB * c / G;
      while (r < R && wrow[r] < target) r++;
      cut[c] = std::max(r, cut[c - 1]);
    }
    int maxp = 0;
    for (int c = 0; c < G; c++) {
      cta_piece[c] = (int)piece_model.size();
      int a = cut[c], b = cut[c + 1];
      while (a < b) {
        int m = row_model[a];
        int e = std::min(b, eng.row_off[m + 1]);
        piece_row.push_back(a);
        piece_model.push_back(m);
        a = e;
      }
      maxp = std::max(maxp, (int)piece_model.size() - cta_piece[c]);
    }
    cta_piece[G] = (int)piece_model.size();
    piece_row.push_back(R);
    if (maxp <= pcg_max_cta_pieces()) break;
    if (G >= gmax) {
      // no contiguous split fits: the strided split below takes over
      if (M <= 1) return fail(&eng, B200FEM_ERR_UNSUPPORTED, "too many pieces for one PCG launch");
      contiguous_ok = false;
      break;
    }
    G = std::min(gmax, G * 2);
  }
  std::vector<int> cta_plist(piece_model.size());
  for (size_t k = 0; k < cta_plist.size(); k++) cta_plist[k] = (int)k;
  eng.pcg_nloc_max = 0;
  eng.pcg_nb_max = 0;
  for (int c = 0; c < G; c++) {
    int ra = piece_row[cta_piece[c]], rb = piece_row[cta_piece[c + 1]];
    eng.pcg_nloc_max = std::max(eng.pcg_nloc_max, rb - ra);
    eng.pcg_nb_max = std::max(eng.pcg_nb_max, prow[rb] - prow[ra]);
  }
  pcg_plan_smem(eng.device, eng.pcg_nloc_max, eng.pcg_nb_max, &eng.pcg_resident, &eng.pcg_cached,
                eng.precision == B200FEM_PREC_MIXED);
  // Shared-memory row state pays off while the solve matrix stays in L2
  // (the 40x10x10 hex beam, 8 MB: 5.6 us per iteration resident, 9.6 with
  // global vectors); a matrix streamed from HBM needs the non-resident
  // form's 1024-thread CTAs, twice the warps for its loads (the 60x30x30
  // MooneyRivlin block, 142 MB FP32: 60 us per iteration against 78
  // resident).  Auto: resident up to 64 MB of S; the factored NODAL matrix
  // (S1, divBlk rows and their indices; gathered, latency-bound) up to 32 MB
  // (the same block factored: 35.3 us per iteration mixed with global
  // vectors against 36.9 resident, 48 MB; FP64 41.8 against 41.6, 79 MB)
  double s_bytes = 9.0 * (eng.precision == B200FEM_PREC_MIXED ? 4 : 8) * (double)prow[R];
  if (eng.factored) s_bytes += 24.0 * nbr_ptr[N] + 8.0 * dil_rptr[R];
  const double res_max = eng.factored ? 32e6 : 64e6;
  if (eng.opt_resident == 1 || (eng.opt_resident == 0 && s_bytes > res_max)) eng.pcg_resident = eng.pcg_cached = 0;
  eng.pcg_strided = 0;
  if (!contiguous_ok) {
    if (eng.opt_split == 1) return fail(&eng, B200FEM_ERR_UNSUPPORTED, "too many models for a contiguous PCG split");
    eng.pcg_resident = eng.pcg_cached = 0;
  }
  // cluster split (on request): one thread-block cluster per model, models
  // taken from a queue largest first (pcg_cluster.cu)
  eng.pcg_cluster = false;
  if (eng.opt_split == 3) {
    eng.cl_clusters = pcg_cluster_capacity(eng.precision == B200FEM_PREC_MIXED);
    if (eng.cl_clusters > 0) eng.pcg_cluster = true;
    else return fail(&eng, B200FEM_ERR_UNSUPPORTED, "thread-block clusters unavailable");
  }
  if (eng.opt_split == 2 || (eng.opt_split == 0 && !eng.pcg_resident && M > 1)) {
    // Strided split for packs too large for shared-memory residency: every
    // model is cut into short pieces and each piece goes to the least-loaded
    // CTA, so a model's rows are spread over many SMs.  When most models
    // have converged, the iterations left for the slow ones then run on the
    // whole GPU instead of on the few CTAs that would hold them.
    G = std::max(1, std::min(gmax, (R + 31) / 32));
    const double row_cost = 400.0, blk_cost = 9.0 * (eng.precision == B200FEM_PREC_MIXED ? 4 : 8) + 4 + 24;
    for (int P = eng.opt_piece_rows > 0 ? eng.opt_piece_rows : 64;; P *= 2) {
      piece_row.clear();
      piece_model.clear();
      for (int m = 0; m < M; m++) {
        const int a = eng.row_off[m], n = eng.row_off[m + 1] - a;
        if (n <= 0) continue;
        const int k = (n + P - 1) / P;
        for (int t = 0; t < k; t++) {
          piece_row.push_back(a + (int)((long long)n * t / k));
          piece_model.push_back(m);
        }
      }
      piece_row.push_back(R);
      const int np = (int)piece_model.size();
      std::vector<int> owner(np), count(G, 0);
      std::vector<std::pair<double, int>> heap;
      for (int c = 0; c < G; c++) heap.push_back({0.0, c});
      auto later = [](const std::pair<double, int>& x, const std::pair<double, int>& y) {
        return x.first != y.first ? x.first > y.first : x.second > y.second;
      };
      std::make_heap(heap.begin(), heap.end(), later);
      int maxp = 0;
      for (int k = 0; k < np; k++) {
        std::pop_heap(heap.begin(), heap.end(), later);
        auto& top = heap.back();
        const int ra = piece_row[k], rb = piece_row[k + 1];
        owner[k] = top.second;
        top.first += row_cost * (rb - ra) + blk_cost * (double)(wrow[rb] - wrow[ra]);
        maxp = std::max(maxp, ++count[top.second]);
        std::push_heap(heap.begin(), heap.end(), later);
      }
      if (maxp > pcg_max_cta_pieces()) {
        if (P >= R) return fail(&eng, B200FEM_ERR_UNSUPPORTED, "too many models for one PCG launch");
        continue;
      }
      cta_piece.assign(G + 1, 0);
      for (int k = 0; k < np; k++) cta_piece[owner[k] + 1]++;
      for (int c = 0; c < G; c++) cta_piece[c + 1] += cta_piece[c];
      cta_plist.assign(np, 0);
      std::vector<int> fill(cta_piece.begin(), cta_piece.end() - 1);
      for (int k = 0; k < np; k++) cta_plist[fill[owner[k]]++] = k;
      eng.pcg_nloc_max = 0;
      for (int c = 0; c < G; c++) {
        int rows = 0;
        for (int q = cta_piece[c]; q < cta_piece[c + 1]; q++)
          rows += piece_row[cta_plist[q] + 1] - piece_row[cta_plist[q]];
        eng.pcg_nloc_max = std::max(eng.pcg_nloc_max, rows);
      }
      eng.pcg_nb_max = 0;
      eng.pcg_resident = eng.pcg_cached = 0;
      eng.pcg_strided = 1;
      break;
    }
  }
  for (size_t k = 0; k < piece_model.size(); k++) model_piece[piece_model[k] + 1] = (int)k + 1;
  for (int m = 0; m < M; m++) model_piece[m + 1] = std::max(model_piece[m + 1], model_piece[m]);
  eng.pcg_grid = G;
  d.n_pieces = (int)piece_model.size();
  eng.pcg_every_cta_rows = 1;
  for (int c = 0; c < G; c++)
    if (cta_piece[c + 1] <= cta_piece[c]) eng.pcg_every_cta_rows = 0;
  // default SpMV row width (the autotuner may change it later)
  if (eng.opt_row_lanes > 0) {
    eng.pcg_row_lanes = eng.opt_row_lanes;
  } else {
    // (factored NODAL: the direct blocks and as many dilational entries)
    const double bpr = R > 0 ? (double)(eng.factored ? prow[R] + dil_rptr[R] : NB) / R : 1.0;
    // many rows in flight per warp do best up to hexes' ~27 blocks per row
    // (measured: 40x10x10 hex beam 6.8 us per iteration at 4 lanes, 7.1
    // at 16); NODAL 2-ring rows (~69 blocks) -> 16 (the 60x30x30
    // MooneyRivlin block: 60.4 us per iteration mixed at 16 lanes, 62.9 at
    // 32, 62.3 at 8); the same block factored (~24 entries per row) -> 4
    // (FP64 41.8 us at 4 lanes, 43.6 at 8, 47.3 at 16)
    eng.pcg_row_lanes = bpr <= 40 ? 4 : 16;
  }

  // ---- device upload
  CK(upload(eng, &d.x, x));
  CK(dalloc(eng, &d.v, 3 * (size_t)N));
  CK(cudaMemset(d.v, 0, 3 * sizeof(double) * (size_t)N));
  CK(dalloc(eng, &d.vprev, 3 * (size_t)N));
  CK(cudaMemset(d.vprev, 0, 3 * sizeof(double) * (size_t)N));
  CK(dalloc(eng, &d.vprev2, 3 * (size_t)N));
  CK(cudaMemset(d.vprev2, 0, 3 * sizeof(double) * (size_t)N));
  CK(dalloc(eng, &d.vprev3, 3 * (size_t)N));
  CK(cudaMemset(d.vprev3, 0, 3 * sizeof(double) * (size_t)N));
  CK(dalloc(eng, &d.vprev4, 3 * (size_t)N));
  CK(cudaMemset(d.vprev4, 0, 3 * sizeof(double) * (size_t)N));
  CK(dalloc(eng, &d.fext, 3 * (size_t)N));
  CK(cudaMemset(d.fext, 0, 3 * sizeof(double) * (size_t)N));
  CK(upload(eng, &d.mass, mass));
  CK(upload(eng, &d.node_model, node_model));
  CK(upload(eng, &d.sidx, sidx));
  CK(upload(eng, &d.act_node, act_node));
  CK(upload(eng, &d.row_model, row_model));
  CK(upload(eng, &d.conn, conn));
  CK(upload(eng, &d.elem_model, elem_model));
  if (own_mats) CK(upload(eng, &d.elem_mat, elem_mat));
  else d.elem_mat = d.elem_model;
  CK(upload(eng, &d.invJ0, invJ0));
  CK(upload(eng, &d.winvJ0, winvJ0));
  if (any_linear) {
    CK(upload(eng, &d.K0, K0));
    CK(upload(eng, &d.f0, f0));
  }
  CK(upload(eng, &d.blk_rowptr, rowptr));
  CK(upload(eng, &d.blk_col, col));
  CK(upload(eng, &d.blk_diag, blk_diag));
  CK(upload(eng, &d.blk_row, blk_row));
  CK(upload(eng, &d.contrib_ptr, cptr));
  CK(upload(eng, &d.contrib_idx, cidx));
  {
    std::vector<int> mirror(NB);
    for (int r = 0; r < R; r++)
      for (int p = rowptr[r]; p < rowptr[r + 1]; p++) mirror[p] = block_of(col[p], r);
    CK(upload(eng, &d.blk_mirror, mirror));
    std::vector<int> up;
    up.reserve(NB / 2 + R);
    for (long long p = 0; p < NB; p++)
      if (!(mirror[p] >= 0 && mirror[p] < p)) up.push_back((int)p);
    d.n_up = (long long)up.size();
    CK(upload(eng, &d.up_blocks, up));
    if (eng.factored) {
      // the step's gather: the upper direct blocks, written to S1
      std::vector<int> u1, u1d, u1m;
      for (int p : up)
        if (s1_of[p] >= 0) {
          u1.push_back(p);
          u1d.push_back(s1_of[p]);
          u1m.push_back(s1_of[mirror[p]]);
        }
      d.n_up1 = (long long)u1.size();
      CK(upload(eng, &d.up1, u1));
      CK(upload(eng, &d.up1_dst, u1d));
      CK(upload(eng, &d.up1_mdst, u1m));
    }
  }
  CK(upload(eng, &d.inc_ptr, iptr));
  CK(upload(eng, &d.inc_idx, iidx));
  if (eng.tet_rows) {
    CK(upload(eng, &d.task_row, task_row));
    CK(upload(eng, &d.row_incptr, row_incptr));
    CK(upload(eng, &d.row_inc, row_inc));
    CK(upload(eng, &d.contrib_byte, cbyte));
  }
  if (eng.fused) {
    CK(upload(eng, &d.chunk_row, chunk_row));
    CK(upload(eng, &d.chunk_eptr, chunk_eptr));
    CK(upload(eng, &d.chunk_elem, chunk_elem));
    CK(upload(eng, &d.contrib_loc, contrib_loc));
  }
  CK(dalloc(eng, &d.K, (size_t)NB * 9));
  if (eng.precision == B200FEM_PREC_MIXED) {
    // mixed form: FP32 rest data, tangent blocks and solve matrix; the
    // nodal forces (the force residual) stay FP64
    std::vector<float> invJ0_f(invJ0.begin(), invJ0.end());
    CK(upload(eng, &d.invJ0_f, invJ0_f));
    CK(dalloc(eng, &d.elemK_f, (size_t)proff[E] * 9));
    if (eng.factored) CK(dalloc(eng, &d.S1_f, std::max<size_t>(s1_col.size(), 1) * 9));
    else CK(dalloc(eng, &d.S_f, (size_t)NB * 9));
  } else {
    CK(dalloc(eng, &d.elemK, (size_t)proff[E] * 9));
    if (eng.factored) CK(dalloc(eng, &d.S1, std::max<size_t>(s1_col.size(), 1) * 9));
    else CK(dalloc(eng, &d.S, (size_t)NB * 9));
  }
  if (eng.factored) {
    d.s1_nnzb = (long long)s1_col.size();
    CK(upload(eng, &d.s1_rowptr, s1_rowptr));
    CK(upload(eng, &d.s1_col, s1_col));
    CK(upload(eng, &d.s1_diag, s1_diag));
    CK(upload(eng, &d.dil_rptr, dil_rptr));
    CK(upload(eng, &d.dil_node, dil_node));
    CK(upload(eng, &d.dil_slot, dil_slot));
    CK(upload(eng, &d.nbr_row, nbr_row));
    CK(upload(eng, &d.dil_nodes, dil_nodes));
    d.n_dil_nodes = (int)dil_nodes.size();
    CK(dalloc(eng, &d.dil_t, (size_t)N));
    CK(cudaMemset(d.dil_t, 0, sizeof(double) * (size_t)N));
  }
  CK(dalloc(eng, &d.elemF, (size_t)coff[E] * 3));
  CK(dalloc(eng, &d.Dinv, (size_t)R * 9));
  CK(dalloc(eng, &d.fint, 3 * (size_t)N));
  for (double** v : {&d.b, &d.sol, &d.r, &d.z, &d.p, &d.q, &d.w, &d.u, &d.s, &d.m0, &d.m1}) {
    CK(dalloc(eng, v, 3 * (size_t)R));
    CK(cudaMemset(*v, 0, 3 * sizeof(double) * (size_t)R));
  }
  CK(upload(eng, &d.mat, mat));
  CK(upload(eng, &d.step, step));
  {
    // ELEMENT soft incompressibility: rest volume per element of the pack
    bool any_elem = false;
    for (auto& h : eng.hosts) any_elem |= (h.incomp == B200FEM_INCOMP_ELEMENT);
    if (any_elem) {
      std::vector<double> erv((size_t)E, 1.0);
      for (int m = 0; m < M; m++)
        std::copy(eng.hosts[m].rest_vol.begin(), eng.hosts[m].rest_vol.end(), erv.begin() + eng.elem_off[m]);
      CK(upload(eng, &d.elem_rest_vol, erv));
      // one pressure value per element, or npv values and an npv x npv Rinv
      CK(dalloc(eng, &d.elem_p, (size_t)pvoff[E]));
      CK(dalloc(eng, &d.elem_r, (size_t)pv2off[E]));
      CK(cudaMemset(d.elem_p, 0, sizeof(double) * (size_t)pvoff[E]));
      CK(cudaMemset(d.elem_r, 0, sizeof(double) * (size_t)pv2off[E]));
      if (pvoff[E] > E) {
        std::vector<double> dj0((size_t)ipoff[E], 1.0);
        for (int m = 0; m < M; m++)
          std::copy(eng.hosts[m].detJ0.begin(), eng.hosts[m].detJ0.end(),
                    dj0.begin() + (size_t)ipoff[eng.elem_off[m]]);
        CK(upload(eng, &d.detJ0, dj0));
      }
    }
  }
  if (any_nodal) {
    d.has_nodal = 1;
    CK(upload(eng, &d.node_rest_vol, node_rest_vol));
    CK(dalloc(eng, &d.node_vol, (size_t)N));
    CK(dalloc(eng, &d.node_p, (size_t)N));
    CK(dalloc(eng, &d.node_kp, (size_t)N));
    CK(upload(eng, &d.mat_node, mat_node));
    CK(upload(eng, &d.nbr_ptr, nbr_ptr));
    CK(upload(eng, &d.inc_slot, inc_slot));
    if (mixed) CK(upload(eng, &d.inc_tl, itl));
    CK(dalloc(eng, &d.divblk, 3 * (size_t)nbr_ptr[N]));
    CK(upload(eng, &d.dil_ptr, dptr));
    CK(upload(eng, &d.dil_idx, didx));
  }
  CK(dalloc(eng, &d.partials, (size_t)d.n_pieces * 8));
  CK(upload(eng, &d.piece_row, piece_row));
  CK(upload(eng, &d.piece_model, piece_model));
  CK(upload(eng, &d.model_piece, model_piece));
  CK(upload(eng, &d.cta_piece, cta_piece));
  CK(upload(eng, &d.cta_plist, cta_plist));
  CK(upload(eng, &d.model_active, std::vector<int>(M, 1)));
  {
    // cluster split: model rows, the queue order (most blocks first) and the
    // queue counter
    std::vector<int> model_row(eng.row_off.begin(), eng.row_off.end()), order(M);
    for (int m = 0; m < M; m++) order[m] = m;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      return eng.blk_off[x + 1] - eng.blk_off[x] > eng.blk_off[y + 1] - eng.blk_off[y];
    });
    CK(upload(eng, &d.model_row, model_row));
    CK(upload(eng, &d.cl_order, order));
    CK(dalloc(eng, &d.cl_queue, 1));
  }
  eng.any_inactive = false;
  d.unconv_cap = 200000;
  CK(dalloc(eng, &d.unconv, (size_t)d.unconv_cap + 2));
  {
    // models without active rows never run PCG: report them converged
    std::vector<double> ms((size_t)M * 4, 0.0);
    for (int m = 0; m < M; m++) ms[(size_t)m * 4 + 2] = 1.0;
    CK(upload(eng, &d.model_scal, ms));
    CK(cudaHostAlloc((void**)&d.status_host, sizeof(double) * (5 + ms.size()), cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void**)&d.status_dev, d.status_host, 0));
    // refinement sweeps (mixed form): FP64 residual, correction, and the
    // correction solves' own per-model results
    eng.refine_ok = eng.precision == B200FEM_PREC_MIXED && eng.groups.size() == 1 && !eng.groups[0].nodal &&
                    !eng.groups[0].elem_inc &&
                    (eng.elem_type == B200FEM_ELEM_TET || eng.elem_type == B200FEM_ELEM_HEX) &&
                    (eng.groups[0].mat_kind == B200FEM_MAT_NEOHOOKEAN ||
                     eng.groups[0].mat_kind == B200FEM_MAT_MOONEYRIVLIN);
    if (eng.refine_ok) {
      CK(dalloc(eng, &d.rref, 3 * (size_t)R));
      CK(dalloc(eng, &d.dsol, 3 * (size_t)R));
      CK(upload(eng, &d.model_scal2, ms));
    }
  }
  CK(dalloc(eng, &d.barrier, 2));
  CK(cudaMemset(d.barrier, 0, 2 * sizeof(unsigned)));
  CK(dalloc(eng, &d.flags, 4));
  CK(cudaMemset(d.flags, 0, 4 * sizeof(int)));
  CK(dalloc(eng, &d.dmin, 1));
  // host copies for queries
  eng.h_rowptr = rowptr;
  eng.h_col = col;
  eng.h_sidx = sidx;
  eng.h_mass = mass;
  if (eng.att.active()) {
    std::string err;
    const int st = build_attachment_reduction(eng, err);
    if (st != B200FEM_OK) return fail(&eng, st, err);
  }
  CK(prepare_kernels(eng));
  CK(prepare_pcg(eng));
  eng.built = true;
  return B200FEM_OK;
}

}  // namespace b200fem

using namespace b200fem;

namespace {
// true when every value is finite: a NaN or an infinity in a caller's array
// is refused with B200FEM_ERR_INVALID_ARG before it reaches the device
// A double is finite iff its exponent field is not all ones: adding one to
// the masked exponent carries into bit 63 exactly for all-ones fields.  The
// OR-reduction vectorises (the host-state step checks 2 x 3N values per
// call: 9 us for the 40x10x10 hex beam's x or v with a per-element fabs
// compare, 3 us this way).
__attribute__((optimize("O3"))) bool all_finite(const double* a, size_t n) {
  const uint64_t kExp = 0x7ff0000000000000ull, kOne = 0x0010000000000000ull;
  uint64_t acc = 0;
  for (size_t i = 0; i < n; i++) {
    uint64_t b;
    std::memcpy(&b, a + i, sizeof b);
    acc |= (b & kExp) + kOne;
  }
  return (acc >> 63) == 0;
}
}  // namespace

struct b200fem_engine {
  Engine eng;
};

#define ENG(h)                                                    \
  if (!(h)) return fail(nullptr, B200FEM_ERR_INVALID_ARG, "null handle"); \
  Engine& eng = (h)->eng;                                         \
  {                                                               \
    cudaError_t _se = cudaSetDevice(eng.device);                  \
    if (_se != cudaSuccess) return cuda_fail(&eng, _se, "cudaSetDevice"); \
  }

#define NEED_BUILT()                                                       \
  if (!eng.built) return fail(&eng, B200FEM_ERR_STATE, "b200fem_build has not been called")

extern "C" {

int b200fem_version(void) { return 10000; }

b200fem_handle b200fem_create(const b200fem_config* cfg) {
  int dev = cfg ? cfg->device : 0;
  int prec = cfg ? cfg->precision : B200FEM_PREC_FP64;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    set_global_error(std::string("no CUDA device available: ") + cudaGetErrorString(e));
    return nullptr;
  }
  if (dev < 0 || dev >= count) {
    set_global_error("invalid device ordinal");
    return nullptr;
  }
  if (prec != B200FEM_PREC_FP64 && prec != B200FEM_PREC_MIXED) {
    set_global_error("invalid precision");
    return nullptr;
  }
  if ((e = cudaSetDevice(dev)) != cudaSuccess) {
    set_global_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return nullptr;
  }
  cudaDeviceProp prop;
  if ((e = cudaGetDeviceProperties(&prop, dev)) != cudaSuccess) {
    set_global_error(std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e));
    return nullptr;
  }
  if (prop.major < 10) {
    set_global_error("libb200fem requires an sm_100 (Blackwell) device");
    return nullptr;
  }
  b200fem_engine* h = new b200fem_engine();
  h->eng.device = dev;
  h->eng.precision = prec;
  h->eng.num_sms = prop.multiProcessorCount;
  if ((e = cudaStreamCreateWithFlags(&h->eng.stream, cudaStreamNonBlocking)) != cudaSuccess) {
    set_global_error(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    delete h;
    return nullptr;
  }
  for (auto& ev : h->eng.ev) cudaEventCreate(&ev);
  h->eng.models.assign(1, ModelDesc());
  return h;
}

int b200fem_destroy(b200fem_handle h) {
  if (!h) return B200FEM_OK;
  cudaSetDevice(h->eng.device);
  if (h->eng.stream) cudaStreamSynchronize(h->eng.stream);
  free_pack(h->eng);
  for (auto& ev : h->eng.ev)
    if (ev) cudaEventDestroy(ev);

  for (auto& ev : h->eng.ev_pool) cudaEventDestroy(ev);
  if (h->eng.stream) cudaStreamDestroy(h->eng.stream);
  delete h;
  return B200FEM_OK;
}

const char* b200fem_last_error(b200fem_handle h) {
  if (!h) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    static thread_local std::string copy;
    copy = g_global_err;
    return copy.c_str();
  }
  return h->eng.last_error.c_str();
}

int b200fem_grid_dims(int elem_type, int nx, int ny, int nz, int* n_nodes, int* n_elems) {
  if (!n_nodes || !n_elems) return fail(nullptr, B200FEM_ERR_INVALID_ARG, "null output");
  int st = grid_dims(elem_type, nx, ny, nz, n_nodes, n_elems);
  if (st != B200FEM_OK) return fail(nullptr, st, "invalid grid arguments");
  return B200FEM_OK;
}

int b200fem_create_grid(int elem_type, double wx, double wy, double wz, int nx, int ny, int nz, double* xyz,
                        int* conn) {
  int nn, ne;
  if (grid_dims(elem_type, nx, ny, nz, &nn, &ne) != B200FEM_OK || !xyz || !conn)
    return fail(nullptr, B200FEM_ERR_INVALID_ARG, "invalid grid arguments");
  create_grid(elem_type, wx, wy, wz, nx, ny, nz, xyz, conn);
  return B200FEM_OK;
}

int b200fem_quadratic_tet_mesh(int n_nodes, const double* xyz, int n_tets, const int* conn, int* n_nodes_out,
                               double* xyz_out, int* conn_out) {
  if (n_nodes <= 0 || n_tets <= 0 || !xyz || !conn || !n_nodes_out)
    return fail(nullptr, B200FEM_ERR_INVALID_ARG, "invalid mesh arguments");
  for (size_t q = 0; q < 4 * (size_t)n_tets; q++)
    if (conn[q] < 0 || conn[q] >= n_nodes) return fail(nullptr, B200FEM_ERR_INVALID_ARG, "connectivity index out of range");
  std::vector<double> qx;
  std::vector<int> qc;
  quadratic_mesh(B200FEM_ELEM_TET, n_nodes, xyz, n_tets, conn, qx, qc);
  *n_nodes_out = (int)(qx.size() / 3);
  if (xyz_out) std::copy(qx.begin(), qx.end(), xyz_out);
  if (conn_out) std::copy(qc.begin(), qc.end(), conn_out);
  return B200FEM_OK;
}

int b200fem_jitter_grid(int nx, int ny, int nz, double wx, double wy, double wz, double frac,
                        unsigned long long seed, double* xyz) {
  if (nx < 1 || ny < 1 || nz < 1 || !xyz) return fail(nullptr, B200FEM_ERR_INVALID_ARG, "invalid grid arguments");
  jitter_grid(nx, ny, nz, wx, wy, wz, frac, seed, xyz);
  return B200FEM_OK;
}

int b200fem_set_mesh(b200fem_handle h, int elem_type, int n_nodes, const double* rest_xyz, int n_elems,
                     const int* conn, const int* fixed) {
  ENG(h);
  if (elem_nen(elem_type) == 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown element type");
  if (n_nodes <= 0 || n_elems <= 0 || !rest_xyz || !conn)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "empty mesh");
  int nen = elem_nen(elem_type);
  if (!all_finite(rest_xyz, 3 * (size_t)n_nodes))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite rest position");
  ModelDesc& m = eng.models[0];
  m.elem_type = elem_type;
  m.n_nodes = n_nodes;
  m.n_elems = n_elems;
  m.rest.assign(rest_xyz, rest_xyz + 3 * (size_t)n_nodes);
  m.conn.assign(conn, conn + (size_t)nen * n_elems);
  m.etypes.clear();
  m.emat.clear();  // element materials name elements of the previous mesh
  m.emat_kind.clear();
  m.emat_params.clear();
  m.fixed.assign(n_nodes, 0);
  if (fixed) std::copy(fixed, fixed + n_nodes, m.fixed.begin());
  eng.att = FrameAttach();  // attachments name nodes of the previous mesh
  free_pack(eng);
  return B200FEM_OK;
}

int b200fem_set_mesh_mixed(b200fem_handle h, int n_nodes, const double* rest_xyz, int n_elems,
                           const int* elem_types, const int* conn, const int* fixed) {
  ENG(h);
  if (n_nodes <= 0 || n_elems <= 0 || !rest_xyz || !conn || !elem_types)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "empty mesh");
  size_t total = 0;
  for (int e = 0; e < n_elems; e++) {
    const int k = elem_nen(elem_types[e]);
    if (k == 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "element " + std::to_string(e) + ": unknown type");
    total += (size_t)k;
  }
  if (!all_finite(rest_xyz, 3 * (size_t)n_nodes))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite rest position");
  ModelDesc& m = eng.models[0];
  m.elem_type = kElemMixed;
  m.n_nodes = n_nodes;
  m.n_elems = n_elems;
  m.rest.assign(rest_xyz, rest_xyz + 3 * (size_t)n_nodes);
  m.conn.assign(conn, conn + total);
  m.etypes.assign(elem_types, elem_types + n_elems);
  m.emat.clear();
  m.emat_kind.clear();
  m.emat_params.clear();
  m.fixed.assign(n_nodes, 0);
  if (fixed) std::copy(fixed, fixed + n_nodes, m.fixed.begin());
  eng.att = FrameAttach();
  free_pack(eng);
  return B200FEM_OK;
}

int b200fem_set_element_materials(b200fem_handle h, int model, int n_elems, const int* mat_kinds,
                                  const double* params) {
  ENG(h);
  if (model < 0 || model >= (int)eng.models.size()) return fail(&eng, B200FEM_ERR_INVALID_ARG, "no such model");
  ModelDesc& m = eng.models[model];
  if (!mat_kinds) {
    m.emat.clear();
    m.emat_kind.clear();
    m.emat_params.clear();
    free_pack(eng);
    return B200FEM_OK;
  }
  if (n_elems != m.n_elems || n_elems <= 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "element count mismatch");
  // distinct materials, each once (equal kind and parameter values)
  std::vector<int> emat(n_elems, -1), kinds;
  std::vector<double> prm;
  std::map<std::pair<int, std::vector<double>>, int> seen;
  bool any = false;
  for (int e = 0; e < n_elems; e++) {
    const int k = mat_kinds[e];
    if (k == B200FEM_MAT_MODEL) continue;
    if (k < B200FEM_MAT_LINEAR || k > B200FEM_MAT_STVK || !params)
      return fail(&eng, B200FEM_ERR_INVALID_ARG, "element " + std::to_string(e) + ": unknown material");
    const int np = k == B200FEM_MAT_LINEAR ? 3 : k == B200FEM_MAT_MOONEYRIVLIN ? 8 : 2;
    const double* p = params + (size_t)e * kMatParams;
    if (!all_finite(p, np))
      return fail(&eng, B200FEM_ERR_INVALID_ARG, "element " + std::to_string(e) + ": non-finite material parameter");
    std::vector<double> key(p, p + np);
    key.resize(kMatParams, 0.0);
    auto it = seen.find({k, key});
    if (it == seen.end()) {
      it = seen.emplace(std::make_pair(k, key), (int)kinds.size()).first;
      kinds.push_back(k);
      prm.insert(prm.end(), key.begin(), key.end());
    }
    emat[e] = it->second;
    any = true;
  }
  if (any) {
    m.emat.swap(emat);
    m.emat_kind.swap(kinds);
    m.emat_params.swap(prm);
  } else {
    m.emat.clear();
    m.emat_kind.clear();
    m.emat_params.clear();
  }
  free_pack(eng);
  return B200FEM_OK;
}

int b200fem_set_material(b200fem_handle h, int mat_kind, const double* params, double density, int incomp) {
  ENG(h);
  if (mat_kind < B200FEM_MAT_LINEAR || mat_kind > B200FEM_MAT_STVK || !params)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown material");
  if (!(density > 0) || !(density <= DBL_MAX)) return fail(&eng, B200FEM_ERR_INVALID_ARG, "density must be positive");
  ModelDesc& m = eng.models[0];
  int np = mat_kind == B200FEM_MAT_LINEAR ? 3 : mat_kind == B200FEM_MAT_MOONEYRIVLIN ? 8 : 2;
  if (!all_finite(params, np)) return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite material parameter");
  m.mat_kind = mat_kind;
  std::fill(m.mat_params, m.mat_params + kMatParams, 0.0);
  std::copy(params, params + np, m.mat_params);
  m.density = density;
  m.incomp_request = incomp;
  m.has_material = true;
  free_pack(eng);
  return B200FEM_OK;
}

int b200fem_add_model(b200fem_handle h, int elem_type, int n_nodes, const double* rest_xyz, int n_elems,
                      const int* conn, const int* fixed, int mat_kind, const double* params, double density,
                      int incomp, int* model_index) {
  ENG(h);
  if (elem_nen(elem_type) == 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown element type");
  if (n_nodes <= 0 || n_elems <= 0 || !rest_xyz || !conn) return fail(&eng, B200FEM_ERR_INVALID_ARG, "empty mesh");
  if (mat_kind < B200FEM_MAT_LINEAR || mat_kind > B200FEM_MAT_STVK || !params)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown material");
  if (!(density > 0) || !(density <= DBL_MAX)) return fail(&eng, B200FEM_ERR_INVALID_ARG, "density must be positive");
  if (!all_finite(rest_xyz, 3 * (size_t)n_nodes))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite rest position");
  if (!all_finite(params, mat_kind == B200FEM_MAT_LINEAR ? 3 : mat_kind == B200FEM_MAT_MOONEYRIVLIN ? 8 : 2))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite material parameter");
  ModelDesc m;
  const int nen = elem_nen(elem_type);
  m.elem_type = elem_type;
  m.n_nodes = n_nodes;
  m.n_elems = n_elems;
  m.rest.assign(rest_xyz, rest_xyz + 3 * (size_t)n_nodes);
  m.conn.assign(conn, conn + (size_t)nen * n_elems);
  m.fixed.assign(n_nodes, 0);
  if (fixed) std::copy(fixed, fixed + n_nodes, m.fixed.begin());
  m.mat_kind = mat_kind;
  const int np = mat_kind == B200FEM_MAT_LINEAR ? 3 : mat_kind == B200FEM_MAT_MOONEYRIVLIN ? 8 : 2;
  std::copy(params, params + np, m.mat_params);
  m.density = density;
  m.incomp_request = incomp;
  m.has_material = true;
  if (eng.models.size() == 1 && eng.models[0].n_nodes == 0) eng.models[0] = std::move(m);
  else eng.models.push_back(std::move(m));
  if (model_index) *model_index = (int)eng.models.size() - 1;
  free_pack(eng);
  return B200FEM_OK;
}

int b200fem_clear_models(b200fem_handle h) {
  ENG(h);
  free_pack(eng);
  eng.models.assign(1, ModelDesc());
  return B200FEM_OK;
}

int b200fem_num_models(b200fem_handle h, int* n_models) {
  ENG(h);
  *n_models = (eng.models.size() == 1 && eng.models[0].n_nodes == 0) ? 0 : (int)eng.models.size();
  return B200FEM_OK;
}

int b200fem_model_range(b200fem_handle h, int model, int* node_offset, int* n_nodes, int* n_active) {
  ENG(h);
  NEED_BUILT();
  if (model < 0 || model >= (int)eng.models.size()) return fail(&eng, B200FEM_ERR_INVALID_ARG, "no such model");
  if (node_offset) *node_offset = eng.node_off[model];
  if (n_nodes) *n_nodes = eng.models[model].n_nodes;
  if (n_active) *n_active = eng.hosts[model].n_active;
  return B200FEM_OK;
}

int b200fem_get_model_stats(b200fem_handle h, int* iterations, double* rel_residual) {
  ENG(h);
  NEED_BUILT();
  std::vector<double> ms((size_t)eng.d.n_models * 4);
  CK(cudaMemcpy(ms.data(), eng.d.model_scal, ms.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int m = 0; m < eng.d.n_models; m++) {
    if (iterations) iterations[m] = (int)ms[(size_t)m * 4];
    if (rel_residual) rel_residual[m] = ms[(size_t)m * 4 + 1];
  }
  return B200FEM_OK;
}

int b200fem_build(b200fem_handle h) {
  ENG(h);
  return build_pack(eng);
}

int b200fem_memory_usage(b200fem_handle h, unsigned long long* bytes) {
  ENG(h);
  if (!bytes) return fail(&eng, B200FEM_ERR_INVALID_ARG, "null bytes");
  *bytes = eng.device_bytes;
  return B200FEM_OK;
}

int b200fem_set_active_models(b200fem_handle h, const int* active) {
  ENG(h);
  NEED_BUILT();
  const int M = eng.d.n_models;
  std::vector<int> a(M, 1);
  bool any_off = false;
  if (active)
    for (int m = 0; m < M; m++) {
      a[m] = active[m] != 0;
      any_off |= a[m] == 0;
    }
  CK(cudaMemcpyAsync(eng.d.model_active, a.data(), sizeof(int) * M, cudaMemcpyHostToDevice, eng.stream));
  CK(cudaStreamSynchronize(eng.stream));
  if (any_off != eng.any_inactive) {
    eng.any_inactive = any_off;
    eng.step_exec_max_iter = -1;  // recapture: the mask pointer is a kernel argument
  }
  return B200FEM_OK;
}

int b200fem_set_option(b200fem_handle h, int key, int value) {
  ENG(h);
  switch (key) {
    case B200FEM_OPT_PCG_SPLIT:
      if (value < 0 || value > 3) return fail(&eng, B200FEM_ERR_INVALID_ARG, "PCG_SPLIT must be 0, 1, 2 or 3");
      if (eng.built) return fail(&eng, B200FEM_ERR_STATE, "PCG_SPLIT is set before b200fem_build");
      eng.opt_split = value;
      return B200FEM_OK;
    case B200FEM_OPT_PCG_CTAS:
      if (value < 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "PCG_CTAS must be >= 0");
      if (eng.built) return fail(&eng, B200FEM_ERR_STATE, "PCG_CTAS is set before b200fem_build");
      eng.opt_ctas = value;
      return B200FEM_OK;
    case B200FEM_OPT_PIECE_ROWS:
      if (value < 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "PIECE_ROWS must be >= 0");
      if (eng.built) return fail(&eng, B200FEM_ERR_STATE, "PIECE_ROWS is set before b200fem_build");
      eng.opt_piece_rows = value;
      return B200FEM_OK;
    case B200FEM_OPT_REFINE:
      if (value < 0 || value > 4) return fail(&eng, B200FEM_ERR_INVALID_ARG, "REFINE must be 0..4");
      if (value != eng.opt_refine) {
        eng.opt_refine = value;
        eng.step_exec_max_iter = -1;  // recapture the solve phase
      }
      return B200FEM_OK;
    case B200FEM_OPT_FUSED_ASSEMBLY:
      if (value < 0 || value > 1) return fail(&eng, B200FEM_ERR_INVALID_ARG, "FUSED_ASSEMBLY must be 0 or 1");
      if (eng.built) return fail(&eng, B200FEM_ERR_STATE, "FUSED_ASSEMBLY is set before b200fem_build");
      eng.opt_fused = value;
      return B200FEM_OK;
    case B200FEM_OPT_ELEM_TILE:
      if (value < 0 || value > 2) return fail(&eng, B200FEM_ERR_INVALID_ARG, "ELEM_TILE must be 0, 1 or 2");
      if ((value == 2) != eng.elem_tile_small || (value >= 1) != eng.elem_staged) {
        eng.elem_tile_small = value == 2;
        eng.elem_staged = value >= 1 && value <= 2;
        eng.step_exec_max_iter = -1;  // recapture: another kernel instance
      }
      return B200FEM_OK;
    case B200FEM_OPT_WARM_START:
      if (value < 0 || value > 4) return fail(&eng, B200FEM_ERR_INVALID_ARG, "WARM_START must be 0 to 4");
      if (value != eng.opt_warm_start) {
        eng.opt_warm_start = value;
        eng.step_exec_max_iter = -1;  // recapture: the RHS kernel's arguments change
      }
      return B200FEM_OK;
    case B200FEM_OPT_ROW_LANES:
      if (value != 0 && value != 4 && value != 8 && value != 16 && value != 32)
        return fail(&eng, B200FEM_ERR_INVALID_ARG, "ROW_LANES must be 0, 4, 8, 16 or 32");
      eng.opt_row_lanes = value;
      if (eng.built && value != 0 && value != eng.pcg_row_lanes) {
        eng.pcg_row_lanes = value;
        eng.step_exec_max_iter = -1;  // recapture: the width is a kernel argument
      }
      return B200FEM_OK;
    case B200FEM_OPT_PCG_RESIDENT:
      if (value < 0 || value > 2) return fail(&eng, B200FEM_ERR_INVALID_ARG, "PCG_RESIDENT must be 0, 1 or 2");
      if (eng.built) return fail(&eng, B200FEM_ERR_STATE, "PCG_RESIDENT is set before b200fem_build");
      eng.opt_resident = value;
      return B200FEM_OK;
    case B200FEM_OPT_NODAL_FACTORED:
      if (value < 0 || value > 2) return fail(&eng, B200FEM_ERR_INVALID_ARG, "NODAL_FACTORED must be 0, 1 or 2");
      if (eng.built) return fail(&eng, B200FEM_ERR_STATE, "NODAL_FACTORED is set before b200fem_build");
      eng.opt_nodal_factored = value;
      return B200FEM_OK;
    case B200FEM_OPT_TET_ASSEMBLY:
      if (value < 0 || value > 1) return fail(&eng, B200FEM_ERR_INVALID_ARG, "TET_ASSEMBLY must be 0 or 1");
      if (eng.built) return fail(&eng, B200FEM_ERR_STATE, "TET_ASSEMBLY is set before b200fem_build");
      eng.opt_tet_assembly = value;
      return B200FEM_OK;
    case B200FEM_OPT_BARRIER_TIMEOUT_MS:
      if (value < 1 || value > 60000) return fail(&eng, B200FEM_ERR_INVALID_ARG, "BARRIER_TIMEOUT_MS must be 1..60000");
      if (value != eng.barrier_timeout_ms) {
        eng.barrier_timeout_ms = value;
        eng.step_exec_max_iter = -1;  // recapture: the bound is a kernel argument
      }
      return B200FEM_OK;
    case B200FEM_OPT_TEST_SKIP_ARRIVAL:
      if (value < 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "TEST_SKIP_ARRIVAL must be >= 0");
      if (value != eng.test_skip_arrival) {
        eng.test_skip_arrival = value;
        eng.step_exec_max_iter = -1;  // recapture: the knob is a kernel argument
      }
      return B200FEM_OK;
    default:
      return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown option");
  }
}

int b200fem_get_option(b200fem_handle h, int key, int* value) {
  ENG(h);
  if (!value) return fail(&eng, B200FEM_ERR_INVALID_ARG, "null value");
  switch (key) {
    case B200FEM_OPT_PCG_SPLIT:
      *value = eng.built ? (eng.pcg_cluster ? 3 : eng.pcg_strided ? 2 : 1) : eng.opt_split;
      break;
    case B200FEM_OPT_ROW_LANES: *value = eng.built ? eng.pcg_row_lanes : eng.opt_row_lanes; break;
    case B200FEM_OPT_PCG_CTAS: *value = eng.built ? eng.pcg_grid : eng.opt_ctas; break;
    case B200FEM_OPT_PIECE_ROWS: *value = eng.opt_piece_rows; break;
    case B200FEM_OPT_WARM_START: *value = eng.opt_warm_start; break;
    case B200FEM_OPT_ELEM_TILE: *value = eng.elem_staged ? (eng.elem_tile_small ? 2 : 1) : 0; break;
    case B200FEM_OPT_FUSED_ASSEMBLY: *value = eng.built ? (eng.fused ? 1 : 0) : eng.opt_fused; break;
    case B200FEM_OPT_REFINE: *value = (eng.built && !eng.refine_ok) ? 0 : eng.opt_refine; break;
    case B200FEM_OPT_BARRIER_TIMEOUT_MS: *value = eng.barrier_timeout_ms; break;
    case B200FEM_OPT_TET_ASSEMBLY: *value = eng.built ? (eng.tet_rows ? 0 : 1) : eng.opt_tet_assembly; break;
    case B200FEM_OPT_PCG_RESIDENT: *value = eng.built ? (eng.pcg_resident ? 2 : 1) : eng.opt_resident; break;
    case B200FEM_OPT_NODAL_FACTORED:
      *value = eng.built ? (eng.factored ? 2 : 1) : eng.opt_nodal_factored;
      break;
    case B200FEM_OPT_TEST_SKIP_ARRIVAL: *value = eng.test_skip_arrival; break;
    default: return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown option");
  }
  return B200FEM_OK;
}

// The block pattern the queries report: the solve pattern, or with frame
// attachments the reduced one (free nodes, then two block rows per frame)
struct QueryPattern {
  int rows;
  const std::vector<int>& rowptr;
  const std::vector<int>& col;
};
static QueryPattern query_pattern(const Engine& eng) {
  if (eng.att.active()) return {eng.att.n_red, eng.att.rowptr, eng.att.col};
  return {eng.d.n_rows, eng.h_rowptr, eng.h_col};
}

int b200fem_get_sizes(b200fem_handle h, int* n_active, int* nnzb, int* crs_full, int* crs_upper) {
  ENG(h);
  NEED_BUILT();
  const QueryPattern qp = query_pattern(eng);
  if (n_active) *n_active = qp.rows;
  if (nnzb) *nnzb = (int)qp.col.size();
  if (crs_full) *crs_full = (int)(9 * qp.col.size());
  if (crs_upper) {
    long long up = 0;
    for (int r = 0; r < qp.rows; r++)
      for (int p = qp.rowptr[r]; p < qp.rowptr[r + 1]; p++) {
        if (qp.col[p] > r) up += 9;
        else if (qp.col[p] == r) up += 6;
      }
    *crs_upper = (int)up;
  }
  return B200FEM_OK;
}

int b200fem_get_solve_index(b200fem_handle h, int* sidx) {
  ENG(h);
  NEED_BUILT();
  const std::vector<int>& v = eng.att.active() ? eng.att.sidx : eng.h_sidx;
  std::copy(v.begin(), v.end(), sidx);
  return B200FEM_OK;
}

int b200fem_get_pattern(b200fem_handle h, int* rowptr, int* col) {
  ENG(h);
  NEED_BUILT();
  const QueryPattern qp = query_pattern(eng);
  if (rowptr) std::copy(qp.rowptr.begin(), qp.rowptr.end(), rowptr);
  if (col) std::copy(qp.col.begin(), qp.col.end(), col);
  return B200FEM_OK;
}

// SparseBlockMatrix.getCRSIndices (SparseBlockMatrix.java:1511-1532) and
// SparseNumberedBlockMatrix.createCrsBlockSlotMap (:389-498), 0-based
static int crs_walk(Engine& eng, int partition, int* row_offs, int* col_idx, int* slots) {
  const QueryPattern qp = query_pattern(eng);
  int nnz = 0;
  for (int r = 0; r < qp.rows; r++) {
    for (int i = 0; i < 3; i++) {
      int row = 3 * r + i;
      if (row_offs) row_offs[row] = nnz;
      for (int p = qp.rowptr[r]; p < qp.rowptr[r + 1]; p++) {
        int bj = qp.col[p];
        for (int c = 0; c < 3; c++) {
          int colg = 3 * bj + c;
          if (partition == B200FEM_PART_UPPER && colg < row) {
            if (slots) slots[(size_t)p * 9 + 3 * i + c] = -1;
            continue;
          }
          if (col_idx) col_idx[nnz] = colg;
          if (slots) slots[(size_t)p * 9 + 3 * i + c] = nnz;
          nnz++;
        }
      }
    }
  }
  if (row_offs) row_offs[3 * qp.rows] = nnz;
  return nnz;
}

int b200fem_get_crs_indices(b200fem_handle h, int partition, int* row_offs, int* col_idx) {
  ENG(h);
  NEED_BUILT();
  if (partition != B200FEM_PART_FULL && partition != B200FEM_PART_UPPER)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown partition");
  crs_walk(eng, partition, row_offs, col_idx, nullptr);
  return B200FEM_OK;
}

int b200fem_get_slot_map(b200fem_handle h, int partition, int* slots) {
  ENG(h);
  NEED_BUILT();
  if (partition != B200FEM_PART_FULL && partition != B200FEM_PART_UPPER)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown partition");
  crs_walk(eng, partition, nullptr, nullptr, slots);
  return B200FEM_OK;
}

int b200fem_get_scatter_map(b200fem_handle h, int* map) {
  ENG(h);
  NEED_BUILT();
  if (eng.att.active())
    return fail(&eng, B200FEM_ERR_UNSUPPORTED, "an attached node's blocks go to several reduced blocks");
  std::copy(eng.h_scatter.begin(), eng.h_scatter.end(), map);
  return B200FEM_OK;
}

int b200fem_get_masses(b200fem_handle h, double* mass) {
  ENG(h);
  NEED_BUILT();
  std::copy(eng.h_mass.begin(), eng.h_mass.end(), mass);
  return B200FEM_OK;
}

int b200fem_get_incomp_method(b200fem_handle h, int* method) {
  ENG(h);
  NEED_BUILT();
  *method = eng.hosts[0].incomp;
  return B200FEM_OK;
}

int b200fem_set_state(b200fem_handle h, const double* x, const double* v) {
  ENG(h);
  NEED_BUILT();
  size_t n = 3 * (size_t)eng.d.n_nodes * sizeof(double);
  if ((x && !all_finite(x, 3 * (size_t)eng.d.n_nodes)) || (v && !all_finite(v, 3 * (size_t)eng.d.n_nodes)))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite position or velocity");
  if (x) CK(cudaMemcpyAsync(eng.d.x, x, n, cudaMemcpyHostToDevice, eng.stream));
  if (v) CK(cudaMemcpyAsync(eng.d.v, v, n, cudaMemcpyHostToDevice, eng.stream));
  // a state set from outside has no history: extrapolation starts at zero
  // acceleration
  if (v) CK(cudaMemcpyAsync(eng.d.vprev, v, n, cudaMemcpyHostToDevice, eng.stream));
  if (v) CK(cudaMemcpyAsync(eng.d.vprev2, v, n, cudaMemcpyHostToDevice, eng.stream));
  if (v) CK(cudaMemcpyAsync(eng.d.vprev3, v, n, cudaMemcpyHostToDevice, eng.stream));
  if (v) CK(cudaMemcpyAsync(eng.d.vprev4, v, n, cudaMemcpyHostToDevice, eng.stream));
  CK(cudaStreamSynchronize(eng.stream));
  return B200FEM_OK;
}

int b200fem_get_state(b200fem_handle h, double* x, double* v) {
  ENG(h);
  NEED_BUILT();
  size_t n = 3 * (size_t)eng.d.n_nodes * sizeof(double);
  if (x) CK(cudaMemcpyAsync(x, eng.d.x, n, cudaMemcpyDeviceToHost, eng.stream));
  if (v) CK(cudaMemcpyAsync(v, eng.d.v, n, cudaMemcpyDeviceToHost, eng.stream));
  CK(cudaStreamSynchronize(eng.stream));
  return B200FEM_OK;
}

int b200fem_set_external_forces(b200fem_handle h, const double* fext) {
  ENG(h);
  NEED_BUILT();
  size_t n = 3 * (size_t)eng.d.n_nodes * sizeof(double);
  if (fext && !all_finite(fext, 3 * (size_t)eng.d.n_nodes))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite external force");
  if (fext) CK(cudaMemcpyAsync(eng.d.fext, fext, n, cudaMemcpyHostToDevice, eng.stream));
  else CK(cudaMemsetAsync(eng.d.fext, 0, n, eng.stream));
  CK(cudaStreamSynchronize(eng.stream));
  return B200FEM_OK;
}

int b200fem_update_stress_stiffness(b200fem_handle h, const double* x, double* f_int, double* k_blocks,
                                    double* crs_vals) {
  ENG(h);
  NEED_BUILT();
  DevPack& d = eng.d;
  if (x && !all_finite(x, 3 * (size_t)d.n_nodes)) return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite position");
  if (x) CK(cudaMemcpyAsync(d.x, x, 3 * sizeof(double) * (size_t)d.n_nodes, cudaMemcpyHostToDevice, eng.stream));
  CK(launch_reset_status(eng));
  CK(cudaEventRecord(eng.ev[0], eng.stream));
  CK(launch_assemble(eng, 1.0, 0.0, true));
  // the factored solve matrix of the last step reads divBlk and kp, which
  // this assembly has just replaced
  if (eng.factored) eng.have_matrix = false;
  CK(launch_forces_only(eng));
  if (eng.att.active()) CK(launch_attach_reduce(eng));
  CK(cudaEventRecord(eng.ev[1], eng.stream));
  if (f_int)
    CK(cudaMemcpyAsync(f_int, d.fint, 3 * sizeof(double) * (size_t)d.n_nodes, cudaMemcpyDeviceToHost, eng.stream));
  std::vector<double> kbsr;
  if (eng.att.active()) {
    // the reduced stiffness and its scalar CRS export (reduced pattern)
    const long long nbr = eng.att.nnzb;
    if (k_blocks)
      CK(cudaMemcpyAsync(k_blocks, d.K_red, 9 * sizeof(double) * (size_t)nbr, cudaMemcpyDeviceToHost, eng.stream));
    if (crs_vals) {
      if (nbr > 0) {
        crs_export_kernel_launch(eng, nbr, d.red_row, d.red_rowptr, d.K_red, d.crs_red);
        CK(cudaGetLastError());
      }
      CK(cudaMemcpyAsync(crs_vals, d.crs_red, 9 * sizeof(double) * (size_t)nbr, cudaMemcpyDeviceToHost, eng.stream));
    }
  } else if (k_blocks)
    CK(cudaMemcpyAsync(k_blocks, d.K, 9 * sizeof(double) * (size_t)d.nnzb, cudaMemcpyDeviceToHost, eng.stream));
  if (eng.att.active()) {
    // nothing more to export
  } else if (crs_vals && d.S) {
    CK(launch_crs_export(eng, d.K, d.S));
    CK(cudaMemcpyAsync(crs_vals, d.S, 9 * sizeof(double) * (size_t)d.nnzb, cudaMemcpyDeviceToHost, eng.stream));
    eng.have_matrix = false;  // S was used as scratch
  } else if (crs_vals) {
    // mixed form (no FP64 S buffer): permute to the CRS slot order on the host
    kbsr.resize(9 * (size_t)d.nnzb);
    CK(cudaMemcpyAsync(kbsr.data(), d.K, kbsr.size() * sizeof(double), cudaMemcpyDeviceToHost, eng.stream));
  }
  int flags[4];
  long long dmin;
  CK(cudaMemcpyAsync(flags, d.flags, sizeof(flags), cudaMemcpyDeviceToHost, eng.stream));
  CK(cudaMemcpyAsync(&dmin, d.dmin, sizeof(dmin), cudaMemcpyDeviceToHost, eng.stream));
  CK(cudaStreamSynchronize(eng.stream));
  if (!kbsr.empty()) {
    for (int r = 0; r < d.n_rows; r++) {
      const long long p0 = eng.h_rowptr[r], nb = eng.h_rowptr[r + 1] - p0;
      for (long long p = p0; p < p0 + nb; p++)
        for (int q = 0; q < 9; q++)
          crs_vals[9 * p0 + (q / 3) * 3 * nb + 3 * (p - p0) + (q % 3)] = kbsr[9 * (size_t)p + q];
    }
  }
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, eng.ev[0], eng.ev[1]));
  eng.last_asm_ms = ms;
  eng.last_solve_ms = 0;
  eng.last_stats.num_inverted = flags[1];
  long long bits = dmin >= 0 ? dmin : (dmin ^ 0x7fffffffffffffffll);
  double md;
  std::memcpy(&md, &bits, sizeof(md));
  eng.last_stats.min_detJ = md;
  return B200FEM_OK;
}

// packed: the status record was already written on the stream (the host
// step's single graph ends with it)
static int read_step_status(Engine& eng, b200fem_stats* stats, int max_iter, bool packed = false) {
  DevPack& d = eng.d;
  if (!packed) CK(launch_status_pack(eng));
  CK(cudaStreamSynchronize(eng.stream));
  const double* rec = d.status_host;
  const double* ms = rec + 5;
  int flags[4];
  for (int i = 0; i < 4; i++) flags[i] = (int)rec[i];
  long long dmin;
  std::memcpy(&dmin, &rec[4], sizeof(dmin));
  b200fem_stats st{};
  bool all_conv = true;
  for (int m = 0; m < d.n_models; m++) {
    st.iterations = std::max(st.iterations, (int)ms[(size_t)m * 4]);
    st.rel_residual = std::max(st.rel_residual, ms[(size_t)m * 4 + 1]);
    all_conv &= ms[(size_t)m * 4 + 2] != 0.0;
  }
  st.num_inverted = flags[1];
  st.refinements = eng.refine_ok ? eng.opt_refine : 0;
  long long bits = dmin >= 0 ? dmin : (dmin ^ 0x7fffffffffffffffll);
  std::memcpy(&st.min_detJ, &bits, sizeof(double));
  eng.last_stats = st;
  if (stats) *stats = st;
  if (flags[0] == B200FEM_ERR_TIMEOUT) return fail(&eng, B200FEM_ERR_TIMEOUT, "PCG grid barrier timed out");
  if (flags[0] != 0) return fail(&eng, flags[0], "singular diagonal block in the solve matrix");
  if (flags[2] != 0 || !all_conv) {
    char buf[160];
    snprintf(buf, sizeof(buf), "PCG did not reach the tolerance (worst true relative residual %.3e after %d iterations, cap %d)",
             st.rel_residual, st.iterations, max_iter);
    return fail(&eng, B200FEM_ERR_NO_CONVERGE, buf);
  }
  return B200FEM_OK;
}

namespace {
// nsteps BackwardEuler steps.  With host buffers, the state is copied in
// before the first step (after any graph capture, outside the timed events)
// and back after the last, on the engine's stream, so the one
// synchronisation that reads the step status also covers the copies.
int backward_euler_steps(Engine& eng, const b200fem_step_params* p, int nsteps, b200fem_stats* stats,
                         double* x_host, double* v_host) {
  if (!p || nsteps < 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "invalid step parameters");
  if (eng.att.active())
    return fail(&eng, B200FEM_ERR_UNSUPPORTED,
                "BackwardEuler with frame attachments: the frames' rigid-body dynamics are not part of the engine");
  if (!(p->h > 0) || !(p->tol > 0) || p->max_iter <= 0)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "step size, tolerance and max_iter must be positive");
  {
    const double sp[7] = {p->h, p->alpha_m, p->beta_k, p->gravity[0], p->gravity[1], p->gravity[2], p->tol};
    if (!all_finite(sp, 7)) return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite step parameter");
  }
  DevPack& d = eng.d;
  int max_iter = std::min(p->max_iter, d.unconv_cap);
  if (p->pcg_variant < 0 || p->pcg_variant > 2) return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown pcg_variant");
  if (p->pcg_variant != eng.pcg_variant) {
    eng.pcg_variant = p->pcg_variant;
    eng.step_exec_max_iter = -1;  // recapture: the variant is a kernel argument
  }
  if (p->integrator < B200FEM_INTEGRATOR_BACKWARD_EULER || p->integrator > B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER)
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "unknown integrator");
  if (p->integrator == B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER && !eng.cons_node.empty() && eng.refine_ok &&
      eng.opt_refine > 0)
    return fail(&eng, B200FEM_ERR_UNSUPPORTED, "refinement sweeps with plane constraints");
  if (p->integrator == B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER && eng.pcons.active()) {
    if (!eng.cons_node.empty())
      return fail(&eng, B200FEM_ERR_UNSUPPORTED, "plane and point constraints in the same step");
    if (eng.refine_ok && eng.opt_refine > 0)
      return fail(&eng, B200FEM_ERR_UNSUPPORTED, "refinement sweeps with point constraints");
  }
  if (p->integrator != eng.integrator) {
    eng.integrator = p->integrator;
    eng.step_exec_max_iter = -1;  // recapture: the constraint arrays are kernel arguments
  }
  std::vector<double> step((size_t)d.n_models * 8);
  for (int m = 0; m < d.n_models; m++) {
    double* s = &step[(size_t)m * 8];
    s[0] = p->h;
    s[1] = p->alpha_m;
    s[2] = p->beta_k;
    s[3] = p->gravity[0];
    s[4] = p->gravity[1];
    s[5] = p->gravity[2];
    s[6] = p->tol;
    s[7] = 0;
  }
  if (step != eng.last_step_params) {
    CK(cudaMemcpyAsync(d.step, step.data(), step.size() * sizeof(double), cudaMemcpyHostToDevice, eng.stream));
    eng.last_step_params = step;
  }
  const bool graphs = eng.use_graphs && !p->abort_on_inverted;
  // One step from page-locked host state: the copies in and out, the step and
  // the status record run as one graph launch, with no gap between them
  // (the per-step call of a host that keeps the state)
  bool host_graph = graphs && nsteps == 1 && x_host && v_host;
  if (host_graph) {
    for (double* hp : {x_host, v_host}) {
      cudaPointerAttributes at{};
      if (cudaPointerGetAttributes(&at, hp) != cudaSuccess || at.type != cudaMemoryTypeHost) {
        cudaGetLastError();  // pageable memory: the copies are issued one by one
        host_graph = false;
      }
    }
  }
  if (!host_graph) CK(launch_reset_status(eng));
  while ((int)eng.ev_pool.size() < 3) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    eng.ev_pool.push_back(e);
  }
  if (graphs && (eng.step_exec == nullptr || eng.step_exec_max_iter != max_iter)) {
    // one captured graph per step: assembly (element kernels, block gather,
    // RHS), an event record node between the phases (times each phase), and
    // the solve (PCG); one launch per step leaves no gap between the phases
    for (cudaGraphExec_t* ex : {&eng.asm_exec, &eng.step_exec, &eng.host_exec})
      if (*ex) {
        cudaGraphExecDestroy(*ex);
        *ex = nullptr;
      }
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(eng.stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = launch_assemble(eng, 0, 0, false);
    if (ce == cudaSuccess) ce = launch_rhs(eng);
    // (an external record node: a plain record inside a capture only orders work)
    if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(eng.ev_pool[1], eng.stream, cudaEventRecordExternal);
    if (ce == cudaSuccess) ce = launch_solve(eng, max_iter);
    cudaError_t ee = cudaStreamEndCapture(eng.stream, &graph);
    if (ce != cudaSuccess) return cuda_fail(&eng, ce, "capture of the BackwardEuler step");
    if (ee != cudaSuccess) return cuda_fail(&eng, ee, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&eng.step_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_fail(&eng, ce, "cudaGraphInstantiate");
    eng.step_exec_max_iter = max_iter;
  }
  const size_t state_bytes = 3 * sizeof(double) * (size_t)d.n_nodes;
  if (host_graph) {
    if (eng.host_exec == nullptr || eng.host_x != x_host || eng.host_v != v_host) {
      // the same operations as the path below, captured with the caller's
      // buffers (a call with other buffers captures again)
      if (eng.host_exec) {
        cudaGraphExecDestroy(eng.host_exec);
        eng.host_exec = nullptr;
      }
      cudaGraph_t graph = nullptr;
      CK(cudaStreamBeginCapture(eng.stream, cudaStreamCaptureModeThreadLocal));
      const unsigned ext = cudaEventRecordExternal;
      cudaError_t ce = cudaMemcpyAsync(d.x, x_host, state_bytes, cudaMemcpyHostToDevice, eng.stream);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(d.v, v_host, state_bytes, cudaMemcpyHostToDevice, eng.stream);
      if (ce == cudaSuccess) ce = launch_reset_status(eng);
      if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(eng.ev[0], eng.stream, ext);
      if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(eng.ev_pool[0], eng.stream, ext);
      if (ce == cudaSuccess) ce = launch_assemble(eng, 0, 0, false);
      if (ce == cudaSuccess) ce = launch_rhs(eng);
      if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(eng.ev_pool[1], eng.stream, ext);
      if (ce == cudaSuccess) ce = launch_solve(eng, max_iter);
      if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(eng.ev_pool[2], eng.stream, ext);
      if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(eng.ev[1], eng.stream, ext);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(x_host, d.x, state_bytes, cudaMemcpyDeviceToHost, eng.stream);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(v_host, d.v, state_bytes, cudaMemcpyDeviceToHost, eng.stream);
      if (ce == cudaSuccess) ce = launch_status_pack(eng);
      cudaError_t ee = cudaStreamEndCapture(eng.stream, &graph);
      if (ce != cudaSuccess) return cuda_fail(&eng, ce, "capture of the host-state step");
      if (ee != cudaSuccess) return cuda_fail(&eng, ee, "cudaStreamEndCapture");
      ce = cudaGraphInstantiate(&eng.host_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return cuda_fail(&eng, ce, "cudaGraphInstantiate");
      eng.host_x = x_host;
      eng.host_v = v_host;
    }
    CK(cudaGraphLaunch(eng.host_exec, eng.stream));
    eng.have_matrix = true;
    int st = read_step_status(eng, stats, max_iter, true);
    float a = 0, b = 0, t = 0;
    CK(cudaEventElapsedTime(&a, eng.ev_pool[0], eng.ev_pool[1]));
    CK(cudaEventElapsedTime(&b, eng.ev_pool[1], eng.ev_pool[2]));
    CK(cudaEventElapsedTime(&t, eng.ev[0], eng.ev[1]));
    eng.last_asm_ms = a;
    eng.last_solve_ms = b;
    eng.last_call_ms = t;
    return st;
  }
  if (x_host) CK(cudaMemcpyAsync(d.x, x_host, state_bytes, cudaMemcpyHostToDevice, eng.stream));
  if (v_host) CK(cudaMemcpyAsync(d.v, v_host, state_bytes, cudaMemcpyHostToDevice, eng.stream));
  CK(cudaEventRecord(eng.ev[0], eng.stream));
  for (int s = 0; s < nsteps; s++) {
    CK(cudaEventRecord(eng.ev_pool[0], eng.stream));
    if (graphs) {
      CK(cudaGraphLaunch(eng.step_exec, eng.stream));
    } else {
      CK(launch_assemble(eng, 0, 0, false));
      CK(launch_rhs(eng));
      CK(cudaEventRecord(eng.ev_pool[1], eng.stream));
      if (p->abort_on_inverted) {
        int flags[4];
        CK(cudaMemcpyAsync(flags, d.flags, sizeof(flags), cudaMemcpyDeviceToHost, eng.stream));
        CK(cudaStreamSynchronize(eng.stream));
        if (flags[1] > 0)
          return fail(&eng, B200FEM_ERR_INVERTED, std::to_string(flags[1]) + " inverted elements");
      }
      CK(launch_solve(eng, max_iter));
    }
    CK(cudaEventRecord(eng.ev_pool[2], eng.stream));
  }
  CK(cudaEventRecord(eng.ev[1], eng.stream));
  if (x_host) CK(cudaMemcpyAsync(x_host, d.x, state_bytes, cudaMemcpyDeviceToHost, eng.stream));
  if (v_host) CK(cudaMemcpyAsync(v_host, d.v, state_bytes, cudaMemcpyDeviceToHost, eng.stream));
  eng.have_matrix = true;
  int st = read_step_status(eng, stats, max_iter);
  // device time of the last step's assembly (element, gather, RHS kernels)
  // and PCG phases, and of the whole call
  float a = 0, b = 0, t = 0;
  if (nsteps > 0) {
    CK(cudaEventElapsedTime(&a, eng.ev_pool[0], eng.ev_pool[1]));
    CK(cudaEventElapsedTime(&b, eng.ev_pool[1], eng.ev_pool[2]));
  }
  CK(cudaEventElapsedTime(&t, eng.ev[0], eng.ev[1]));
  eng.last_asm_ms = a;
  eng.last_solve_ms = b;
  eng.last_call_ms = t;
  return st;
}
}  // namespace

int b200fem_set_plane_constraints(b200fem_handle h, int n, const int* nodes, const double* normals,
                                  const double* offsets) {
  ENG(h);
  NEED_BUILT();
  DevPack& d = eng.d;
  if (n < 0 || (n > 0 && (!nodes || !normals || !offsets)))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "invalid plane constraints");
  const int R = d.n_rows;
  std::vector<double> nrm(3 * (size_t)R, 0.0), off((size_t)R, 0.0);
  std::vector<int> seen((size_t)R, 0);
  std::vector<int> cn;
  std::vector<double> cq, co;
  for (int k = 0; k < n; k++) {
    const int node = nodes[k];
    if (node < 0 || node >= (int)eng.h_sidx.size() || eng.h_sidx[node] < 0)
      return fail(&eng, B200FEM_ERR_INVALID_ARG, "plane constraint on a missing or fixed node");
    const int r = eng.h_sidx[node];
    if (seen[r]) return fail(&eng, B200FEM_ERR_UNSUPPORTED, "more than one plane constraint on a node");
    seen[r] = 1;
    const double* q = normals + 3 * (size_t)k;
    const double len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    if (!(len > 0)) return fail(&eng, B200FEM_ERR_INVALID_ARG, "plane constraint with a zero normal");
    for (int c = 0; c < 3; c++) nrm[3 * (size_t)r + c] = q[c] / len;
    off[r] = offsets[k] / len;
    cn.push_back(node);
    for (int c = 0; c < 3; c++) cq.push_back(q[c] / len);
    co.push_back(offsets[k] / len);
  }
  if (!d.row_nrm) {
    CK(dalloc(eng, &d.row_nrm, 3 * (size_t)R));
    CK(dalloc(eng, &d.row_off, (size_t)R));
    eng.step_exec_max_iter = -1;  // recapture with the new arrays
  }
  CK(cudaMemcpyAsync(d.row_nrm, nrm.data(), sizeof(double) * nrm.size(), cudaMemcpyHostToDevice, eng.stream));
  CK(cudaMemcpyAsync(d.row_off, off.data(), sizeof(double) * off.size(), cudaMemcpyHostToDevice, eng.stream));
  CK(cudaStreamSynchronize(eng.stream));
  eng.cons_node = cn;
  eng.cons_nrm = cq;
  eng.cons_off = co;
  return B200FEM_OK;
}

int b200fem_set_point_constraints(b200fem_handle h, int n, const int* ptr, const int* nodes, const double* weights,
                                  const double* targets) {
  ENG(h);
  NEED_BUILT();
  constexpr int kMaxPointConstraints = 32;
  if (n < 0 || n > kMaxPointConstraints || (n > 0 && (!ptr || !nodes || !weights || !targets)))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "invalid point constraints (at most 32)");
  DevPack& d = eng.d;
  PointCons pc;
  pc.n = n;
  if (n > 0) {
    if (ptr[0] != 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "constraint offsets must start at 0");
    for (int c = 0; c < n; c++)
      if (ptr[c + 1] <= ptr[c]) return fail(&eng, B200FEM_ERR_INVALID_ARG, "a constraint without points");
    const int ne = ptr[n];
    pc.ptr.assign(ptr, ptr + n + 1);
    pc.node.assign(nodes, nodes + ne);
    pc.w.assign(weights, weights + ne);
    pc.target.assign(targets, targets + 3 * (size_t)n);
    for (int q = 0; q < ne; q++)
      if (nodes[q] < 0 || nodes[q] >= d.n_nodes)
        return fail(&eng, B200FEM_ERR_INVALID_ARG, "constraint point out of range");
    if (!all_finite(weights, ne) || !all_finite(targets, 3 * (size_t)n))
      return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite constraint weight or target");
    std::vector<int> row(ne);
    for (int q = 0; q < ne; q++) row[q] = eng.h_sidx[nodes[q]];
    if (!d.pc_Y || d.pc_cap < n) {
      // the largest set so far: room for it once
      const int m = 3 * n;
      CK(dalloc(eng, &d.pc_Y, (size_t)m * 3 * d.n_rows));
      CK(dalloc(eng, &d.pc_rhs, 3 * (size_t)d.n_rows));
      CK(dalloc(eng, &d.pc_A, (size_t)m * m));
      CK(dalloc(eng, &d.pc_lam, (size_t)m));
      d.pc_cap = n;
    }
    // small per-set arrays: replaced with the set
    CK(dalloc(eng, &d.pc_ptr, (size_t)n + 1));
    CK(dalloc(eng, &d.pc_node, (size_t)ne));
    CK(dalloc(eng, &d.pc_row, (size_t)ne));
    CK(dalloc(eng, &d.pc_w, (size_t)ne));
    CK(dalloc(eng, &d.pc_target, 3 * (size_t)n));
    CK(cudaMemcpy(d.pc_ptr, ptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.pc_node, nodes, sizeof(int) * ne, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.pc_row, row.data(), sizeof(int) * ne, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.pc_w, weights, sizeof(double) * ne, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.pc_target, targets, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
  }
  eng.pcons = pc;
  eng.step_exec_max_iter = -1;  // recapture: the solve path and its arrays change
  return B200FEM_OK;
}

int b200fem_set_frame_attachments(b200fem_handle h, int n_frames, int n_att, const int* nodes, const int* frames,
                                  const double* H) {
  ENG(h);
  if (n_frames < 0 || n_att < 0 || (n_att > 0 && (!nodes || !frames || !H)) || (n_frames > 0) != (n_att > 0))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "invalid frame attachments");
  const int N = eng.models[0].n_nodes;
  std::vector<char> seen(N > 0 ? N : 0, 0);
  for (int k = 0; k < n_att; k++) {
    if (nodes[k] < 0 || nodes[k] >= N || frames[k] < 0 || frames[k] >= n_frames)
      return fail(&eng, B200FEM_ERR_INVALID_ARG, "attachment node or frame out of range");
    if (seen[nodes[k]]) return fail(&eng, B200FEM_ERR_INVALID_ARG, "a node attached twice");
    seen[nodes[k]] = 1;
  }
  if (n_att > 0 && !all_finite(H, 18 * (size_t)n_att))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite attachment block");
  FrameAttach& A = eng.att;
  A = FrameAttach();
  A.n_frames = n_frames;
  A.node.assign(nodes, nodes + n_att);
  A.frame.assign(frames, frames + n_att);
  A.H.assign(H, H + 18 * (size_t)n_att);
  free_pack(eng);  // the reduced pattern is built with the pack
  return B200FEM_OK;
}

int b200fem_backward_euler_step(b200fem_handle h, const b200fem_step_params* p, int nsteps, b200fem_stats* stats) {
  ENG(h);
  NEED_BUILT();
  return backward_euler_steps(eng, p, nsteps, stats, nullptr, nullptr);
}

int b200fem_backward_euler_step_host(b200fem_handle h, const b200fem_step_params* p, int nsteps, double* x,
                                     double* v, b200fem_stats* stats) {
  ENG(h);
  NEED_BUILT();
  if (!x || !v) return fail(&eng, B200FEM_ERR_INVALID_ARG, "x and v are required");
  if (!all_finite(x, 3 * (size_t)eng.d.n_nodes) || !all_finite(v, 3 * (size_t)eng.d.n_nodes))
    return fail(&eng, B200FEM_ERR_INVALID_ARG, "non-finite position or velocity");
  return backward_euler_steps(eng, p, nsteps, stats, x, v);
}

int b200fem_spmv(b200fem_handle h, const double* x, double* y) {
  ENG(h);
  NEED_BUILT();
  if (!eng.have_matrix) return fail(&eng, B200FEM_ERR_STATE, "no solve matrix assembled yet");
  DevPack& d = eng.d;
  size_t n = 3 * sizeof(double) * (size_t)d.n_rows;
  CK(cudaMemcpyAsync(d.w, x, n, cudaMemcpyHostToDevice, eng.stream));
  CK(launch_spmv(eng, d.w, d.q));
  CK(cudaMemcpyAsync(y, d.q, n, cudaMemcpyDeviceToHost, eng.stream));
  CK(cudaStreamSynchronize(eng.stream));
  return B200FEM_OK;
}

int b200fem_pcg_solve(b200fem_handle h, const double* b, double* x, double tol, int max_iter, b200fem_stats* stats) {
  ENG(h);
  NEED_BUILT();
  if (!eng.have_matrix) return fail(&eng, B200FEM_ERR_STATE, "no solve matrix assembled yet");
  if (!(tol > 0) || max_iter <= 0) return fail(&eng, B200FEM_ERR_INVALID_ARG, "invalid tolerance");
  DevPack& d = eng.d;
  max_iter = std::min(max_iter, d.unconv_cap);
  size_t n = 3 * sizeof(double) * (size_t)d.n_rows;
  std::vector<double> step((size_t)d.n_models * 8);
  CK(cudaMemcpy(step.data(), d.step, step.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int m = 0; m < d.n_models; m++) step[(size_t)m * 8 + 6] = tol;
  CK(cudaMemcpyAsync(d.step, step.data(), step.size() * sizeof(double), cudaMemcpyHostToDevice, eng.stream));
  CK(cudaMemcpyAsync(d.b, b, n, cudaMemcpyHostToDevice, eng.stream));
  CK(cudaMemcpyAsync(d.sol, x, n, cudaMemcpyHostToDevice, eng.stream));
  CK(launch_reset_status(eng));
  CK(launch_pcg(eng, max_iter, false, 0));
  CK(cudaMemcpyAsync(x, d.sol, n, cudaMemcpyDeviceToHost, eng.stream));
  return read_step_status(eng, stats, max_iter);
}

int b200fem_pcg_solve_noalloc(int n_rows, const int* rowptr, const int* col, const double* vals, const double* b,
                              double* x, double tol, int max_iter, void* stream, int* iterations,
                              double* rel_residual) {
  const char* err = "";
  int st = pcg_solve_noalloc(n_rows, rowptr, col, vals, b, x, tol, max_iter, stream, iterations, rel_residual, &err);
  if (st != B200FEM_OK) set_global_error(std::string("b200fem_pcg_solve_noalloc: ") + err);
  return st;
}

int b200fem_last_timing(b200fem_handle h, double* assemble_ms, double* solve_ms) {
  ENG(h);
  if (assemble_ms) *assemble_ms = eng.last_asm_ms;
  if (solve_ms) *solve_ms = eng.last_solve_ms;
  return B200FEM_OK;
}

}  // extern "C"
