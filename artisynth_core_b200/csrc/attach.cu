// attach.cu -- master-slave reduction of the stiffness for FEM nodes
// attached to frames (PointFrameAttachment with an active master frame).
//
// An attached node is not dynamic: its velocity follows its frame,
// v_s = H_s^T [v_F; w_F] with H_s the attachment's 6x3 master block (H =
// -PointFrameAttachment.getGT(0), FemModel3d.getGpuNodeReduction,
// FemModel3d.java:4356-4387).  The solve matrix is then P^T K P: every 3x3
// element block K_ij goes to the reduced block T_i K_ij T_j^T with T = I for
// a free node and T = H for an attached one (scatterReduced3Block,
// cudssBridgeKernels.cu:325-365).  The reference applies the reduction to
// each element block with FP64 atomics; here the stiffness of the extended
// system (free and attached nodes as rows) is assembled by the usual
// deterministic path and a second kernel forms every reduced block as a
// fixed-order sum over the extended blocks that map to it.
//
// Layout of the reduced system: the free active nodes first, in node order,
// then every frame as two 3x3 block rows (translation, rotation), so a
// frame's 6x6 and 6x3 blocks are 2x2 and 2x1 groups of 3x3 blocks and the
// scalar CRS indices are those of the reference's 6-wide frame blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "engine.h"

namespace b200fem {

// Reduced blocks and their contribution lists from the extended pattern
// (free and attached nodes as rows).  Returns B200FEM_OK or an error code
// with a message.
int build_attachment_reduction(Engine& eng, std::string& err) {
  FrameAttach& A = eng.att;
  const int R = eng.d.n_rows;  // extended rows
  if (eng.models.size() != 1) {
    err = "frame attachments need a single-model handle";
    return B200FEM_ERR_UNSUPPORTED;
  }
  const ModelHost& h = eng.hosts[0];
  const int N = eng.models[0].n_nodes;
  // attachment of every extended row (-1: a free node)
  std::vector<int> att_of_node(N, -1), att_row(R, -1);
  for (size_t k = 0; k < A.node.size(); k++) {
    const int n = A.node[k];
    if (h.sidx[n] < 0) {
      err = "an attached node is fixed";
      return B200FEM_ERR_INVALID_ARG;
    }
    att_of_node[n] = (int)k;
  }
  std::vector<int> frame_count(A.n_frames, 0);
  for (int f : A.frame) frame_count[f]++;
  for (int f = 0; f < A.n_frames; f++)
    if (frame_count[f] == 0) {
      err = "a frame without attached nodes";
      return B200FEM_ERR_INVALID_ARG;
    }
  std::vector<int> red_of_row(R, -1);
  A.n_free = 0;
  for (int r = 0; r < R; r++) {
    const int n = h.act_node[r];
    att_row[r] = att_of_node[n];
    if (att_row[r] < 0) red_of_row[r] = A.n_free++;
  }
  A.n_red = A.n_free + 2 * A.n_frames;
  A.sidx.assign(N, -1);
  for (int r = 0; r < R; r++)
    if (red_of_row[r] >= 0) A.sidx[h.act_node[r]] = red_of_row[r];
  // targets of an extended row: (reduced row, part of T): 0 identity,
  // 1 rows 0-2 of H (the frame's translation row), 2 rows 3-5 (rotation)
  auto targets = [&](int r, int* rows, int* parts) -> int {
    const int k = att_row[r];
    if (k < 0) {
      rows[0] = red_of_row[r];
      parts[0] = 0;
      return 1;
    }
    const int f = A.frame[k];
    rows[0] = A.n_free + 2 * f;
    rows[1] = rows[0] + 1;
    parts[0] = 1;
    parts[1] = 2;
    return 2;
  };
  // contributions per reduced block, in extended-block order
  std::vector<std::map<int, std::vector<std::pair<int, int>>>> rowmap(A.n_red);
  for (int ri = 0; ri < R; ri++)
    for (int p = eng.h_rowptr[ri]; p < eng.h_rowptr[ri + 1]; p++) {
      const int rj = eng.h_col[p];
      int I[2], J[2], li[2], lj[2];
      const int ni = targets(ri, I, li), nj = targets(rj, J, lj);
      for (int a = 0; a < ni; a++)
        for (int b = 0; b < nj; b++) rowmap[I[a]][J[b]].push_back({p, li[a] + 3 * lj[b]});
    }
  A.rowptr.assign(A.n_red + 1, 0);
  A.col.clear();
  std::vector<int> red_row, eptr(1, 0), ep;
  std::vector<unsigned char> esel;
  for (int I = 0; I < A.n_red; I++) {
    for (const auto& kv : rowmap[I]) {
      A.col.push_back(kv.first);
      red_row.push_back(I);
      for (const auto& c : kv.second) {
        ep.push_back(c.first);
        esel.push_back((unsigned char)c.second);
      }
      eptr.push_back((int)ep.size());
    }
    A.rowptr[I + 1] = (int)A.col.size();
  }
  A.nnzb = (long long)A.col.size();
  DevPack& d = eng.d;
  cudaError_t e = cudaSuccess;
  auto up_i = [&](int** ptr, const std::vector<int>& v) {
    if (e != cudaSuccess) return;
    e = cudaMalloc(ptr, sizeof(int) * std::max<size_t>(v.size(), 1));
    if (e == cudaSuccess) {
      eng.allocations.push_back(*ptr);
      eng.device_bytes += sizeof(int) * v.size();
      if (!v.empty()) e = cudaMemcpy(*ptr, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice);
    }
  };
  up_i(&d.att_row, att_row);
  up_i(&d.red_row, red_row);
  up_i(&d.red_rowptr, A.rowptr);
  up_i(&d.red_eptr, eptr);
  up_i(&d.red_ep, ep);
  auto up_raw = [&](void** ptr, const void* src, size_t bytes) {
    if (e != cudaSuccess) return;
    e = cudaMalloc(ptr, std::max<size_t>(bytes, 1));
    if (e == cudaSuccess) {
      eng.allocations.push_back(*ptr);
      eng.device_bytes += bytes;
      if (src && bytes) e = cudaMemcpy(*ptr, src, bytes, cudaMemcpyHostToDevice);
    }
  };
  up_raw((void**)&d.red_esel, esel.data(), esel.size());
  up_raw((void**)&d.att_H, A.H.data(), sizeof(double) * A.H.size());
  up_raw((void**)&d.K_red, nullptr, sizeof(double) * 9 * (size_t)A.nnzb);
  up_raw((void**)&d.crs_red, nullptr, sizeof(double) * 9 * (size_t)A.nnzb);
  if (e != cudaSuccess) {
    err = std::string("attachment reduction upload: ") + cudaGetErrorString(e);
    return B200FEM_ERR_CUDA;
  }
  return B200FEM_OK;
}

// One thread per reduced block q: K_red[q] = sum over its contributions c of
// L_c K_ext[p_c] R_c^T, with L (R) the identity or the 3x3 row block of the
// row (column) node's H; tmp = L K, then tmp R^T, as scatterReduced3Block
// orders the sums (cudssBridgeKernels.cu:338-364).
__global__ void attach_reduce_kernel(long long nnzb_red, const int* __restrict__ eptr, const int* __restrict__ ep,
                                     const unsigned char* __restrict__ esel, const int* __restrict__ blk_row,
                                     const int* __restrict__ blk_col, const int* __restrict__ att_row,
                                     const double* __restrict__ H, const double* __restrict__ Kext,
                                     double* __restrict__ Kred) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nnzb_red) return;
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int c1 = eptr[q + 1];
  for (int c = eptr[q]; c < c1; c++) {
    const int p = ep[c];
    const int sel = esel[c], ls = sel % 3, rs = sel / 3;
    double K[9];
#pragma unroll
    for (int k = 0; k < 9; k++) K[k] = Kext[(size_t)p * 9 + k];
    double T[9];
    if (ls == 0) {
#pragma unroll
      for (int k = 0; k < 9; k++) T[k] = K[k];
    } else {
      const double* L = H + 18 * (size_t)att_row[blk_row[p]] + (ls == 1 ? 0 : 9);
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
          double t = 0.0;
#pragma unroll
          for (int k = 0; k < 3; k++) t += L[r * 3 + k] * K[k * 3 + cc];
          T[r * 3 + cc] = t;
        }
    }
    if (rs == 0) {
#pragma unroll
      for (int k = 0; k < 9; k++) s[k] += T[k];
    } else {
      const double* Rb = H + 18 * (size_t)att_row[blk_col[p]] + (rs == 1 ? 0 : 9);
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
          double t = 0.0;
#pragma unroll
          for (int k = 0; k < 3; k++) t += T[r * 3 + k] * Rb[cc * 3 + k];
          s[r * 3 + cc] += t;
        }
    }
  }
#pragma unroll
  for (int k = 0; k < 9; k++) Kred[(size_t)q * 9 + k] = s[k];
}

cudaError_t launch_attach_reduce(Engine& eng) {
  DevPack& d = eng.d;
  const long long nb = eng.att.nnzb;
  if (nb <= 0) return cudaSuccess;
  attach_reduce_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, eng.stream>>>(
      nb, d.red_eptr, d.red_ep, d.red_esel, d.blk_row, d.blk_col, d.att_row, d.att_H, d.K, d.K_red);
  return cudaGetLastError();
}

}  // namespace b200fem
